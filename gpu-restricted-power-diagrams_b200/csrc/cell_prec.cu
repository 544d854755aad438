// Restricted cells with the FP32 clipping loop (mixed, or plain FP32): the
// k_cell instantiations of precisions 1 and 2 (device code in
// cell_kernels.cuh; the FP64 ones are in cell.cu).
#include "cell_kernels.cuh"

namespace rpd {

namespace {

// (the weighted security-radius guard is decided per launch record here)
template <int PREC>
cudaError_t launch_prec(const CellLaunch &a, const Layout &L, int vs, cudaStream_t st, int sm_count, int *launches) {
  if (vs <= 2) return launch_vs<2, PREC, 1>(a, L, st, sm_count, launches);
  if (vs <= 3) return launch_vs<3, PREC, 1>(a, L, st, sm_count, launches);
  if (vs <= 4) return launch_vs<4, PREC, 1>(a, L, st, sm_count, launches);
  if (vs <= 6) return launch_vs<6, PREC, 1>(a, L, st, sm_count, launches);
  return launch_vs<8, PREC, 1>(a, L, st, sm_count, launches);
}

}  // namespace

cudaError_t cell_launch_prec(const CellLaunch &a, cudaStream_t st, int sm_count, int *launches) {
  if (a.num <= 0) return cudaSuccess;
  if (a.precision < 1 || a.precision > 2) return cudaErrorInvalidValue;
  if (a.P > kMaxP || a.V > kMaxV || a.T > kMaxT || a.P < 7 || a.V < 8) return cudaErrorInvalidValue;
  if (a.hess && (a.defer.slots || a.H < 1 || (a.HC != 1 && a.HC != 4))) return cudaErrorInvalidValue;
  if (a.T_ahead > kMaxT || (a.T_ahead > a.T && (!a.defer.slots || a.hess))) return cudaErrorInvalidValue;
  const Layout L = make_layout(a.P, a.V, a.T, a.grid.size > 0, a.hess ? a.HC : 0, a.T_ahead, a.precision,
                               a.grid.lists_disjoint != 0);
  if (a.defer.slots && (a.defer.slot_bytes < slot_bytes_for(L, L.T) || a.defer.max_chunks * a.defer.chunk < L.T))
    return cudaErrorInvalidValue;
  const int vs = L.Vc / 32;
  if (a.precision == 1) return launch_prec<1>(a, L, vs, st, sm_count, launches);
  return launch_prec<2>(a, L, vs, st, sm_count, launches);
}

}  // namespace rpd
