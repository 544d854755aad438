// Restricted cells with the weighted security-radius guard compiled in
// (RPD_FLAG_SAFE_RADIUS, FP64 clipping): the k_cell and k_cell_batch
// instantiations that read the guard from their launch records (device code
// in cell_kernels.cuh; the default ones, without it, are in cell.cu).
#include "cell_kernels.cuh"

namespace rpd {

cudaError_t cell_launch_safe(const CellLaunch &a, cudaStream_t st, int sm_count, int *launches) {
  if (a.num <= 0) return cudaSuccess;
  if (a.P > kMaxP || a.V > kMaxV || a.T > kMaxT || a.P < 7 || a.V < 8) return cudaErrorInvalidValue;
  if (a.hess && (a.defer.slots || a.H < 1 || (a.HC != 1 && a.HC != 4))) return cudaErrorInvalidValue;
  if (a.T_ahead > kMaxT || (a.T_ahead > a.T && (!a.defer.slots || a.hess))) return cudaErrorInvalidValue;
  const Layout L = make_layout(a.P, a.V, a.T, a.grid.size > 0, a.hess ? a.HC : 0, a.T_ahead, 0,
                               a.grid.lists_disjoint != 0);
  if (a.defer.slots && (a.defer.slot_bytes < slot_bytes_for(L, L.T) || a.defer.max_chunks * a.defer.chunk < L.T))
    return cudaErrorInvalidValue;
  const int vs = L.Vc / 32;
  if (vs <= 2) return launch_vs<2, 0, 1>(a, L, st, sm_count, launches);
  if (vs <= 3) return launch_vs<3, 0, 1>(a, L, st, sm_count, launches);
  if (vs <= 4) return launch_vs<4, 0, 1>(a, L, st, sm_count, launches);
  if (vs <= 6) return launch_vs<6, 0, 1>(a, L, st, sm_count, launches);
  return launch_vs<8, 0, 1>(a, L, st, sm_count, launches);
}

cudaError_t cell_batch_launch_safe(const CellBatch &b, cudaStream_t st, int sm_count, int *launches) {
  if (b.ndiag <= 0) return cudaSuccess;
  if (b.P > kMaxP || b.V > kMaxV || b.T > kMaxT || b.P < 7 || b.V < 8) return cudaErrorInvalidValue;
  if (b.HC && b.defer.slots) return cudaErrorInvalidValue;  // Hessian rows are summed inline
  const Layout Lg = make_layout(b.P, b.V, b.T, true, b.HC, b.T_slot, 0, b.disjoint),
               Lp = make_layout(b.P, b.V, b.T, false, b.HC);
  if (b.defer.slots && (b.defer.slot_bytes < slot_bytes_for(Lg, Lg.T) || b.defer.max_chunks * b.defer.chunk < Lg.T))
    return cudaErrorInvalidValue;
  const int vs = Lg.Vc / 32;
  if (vs <= 2) return launch_batch_vs<2, 1>(b, Lg, Lp, st, sm_count, launches);
  if (vs <= 3) return launch_batch_vs<3, 1>(b, Lg, Lp, st, sm_count, launches);
  if (vs <= 4) return launch_batch_vs<4, 1>(b, Lg, Lp, st, sm_count, launches);
  if (vs <= 6) return launch_batch_vs<6, 1>(b, Lg, Lp, st, sm_count, launches);
  return launch_batch_vs<8, 1>(b, Lg, Lp, st, sm_count, launches);
}

}  // namespace rpd
