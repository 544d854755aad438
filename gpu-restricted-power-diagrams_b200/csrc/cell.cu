// Restricted power cell of every seed: host entry points of the cell, probe
// and batched launches (device code in cell_kernels.cuh).
#include "cell_kernels.cuh"

namespace rpd {

size_t cell_warp_smem(int P, int V, int T, bool grid) { return make_layout(P, V, T, grid).total; }

bool cell_caps_fit(int P, int V, int T, bool grid, int hc) {
  return warps_per_block_for(make_layout(P, V, T, grid, hc)) > 0;
}

cudaError_t cell_batch_launch(const CellBatch &b, cudaStream_t st, int sm_count, int *launches) {
  if (b.ndiag <= 0) return cudaSuccess;
  if (b.safe) return cell_batch_launch_safe(b, st, sm_count, launches);
  if (b.P > kMaxP || b.V > kMaxV || b.T > kMaxT || b.P < 7 || b.V < 8) return cudaErrorInvalidValue;
  if (b.HC && b.defer.slots) return cudaErrorInvalidValue;  // Hessian rows are summed inline
  const Layout Lg = make_layout(b.P, b.V, b.T, true, b.HC, b.T_slot, 0, b.disjoint),
               Lp = make_layout(b.P, b.V, b.T, false, b.HC);
  if (b.defer.slots && (b.defer.slot_bytes < slot_bytes_for(Lg, Lg.T) || b.defer.max_chunks * b.defer.chunk < Lg.T))
    return cudaErrorInvalidValue;
  const int vs = Lg.Vc / 32;
  if (vs <= 2) return launch_batch_vs<2>(b, Lg, Lp, st, sm_count, launches);
  if (vs <= 3) return launch_batch_vs<3>(b, Lg, Lp, st, sm_count, launches);
  if (vs <= 4) return launch_batch_vs<4>(b, Lg, Lp, st, sm_count, launches);
  if (vs <= 6) return launch_batch_vs<6>(b, Lg, Lp, st, sm_count, launches);
  return launch_batch_vs<8>(b, Lg, Lp, st, sm_count, launches);
}

size_t defer_slot_bytes(int P, int V, int T) { return slot_bytes_for(make_layout(P, V, T, true), T); }

cudaError_t cell_launch(const CellLaunch &a, cudaStream_t st, int sm_count, int *launches) {
  if (a.num <= 0) return cudaSuccess;
  if (a.precision != 0) return cell_launch_prec(a, st, sm_count, launches);
  if (a.safe_radius) return cell_launch_safe(a, st, sm_count, launches);
  if (a.P > kMaxP || a.V > kMaxV || a.T > kMaxT || a.P < 7 || a.V < 8) return cudaErrorInvalidValue;
  if (a.hess && (a.defer.slots || a.H < 1 || (a.HC != 1 && a.HC != 4))) return cudaErrorInvalidValue;
  if (a.T_ahead > kMaxT || (a.T_ahead > a.T && (!a.defer.slots || a.hess))) return cudaErrorInvalidValue;
  const Layout L = make_layout(a.P, a.V, a.T, a.grid.size > 0, a.hess ? a.HC : 0, a.T_ahead, 0,
                               a.grid.lists_disjoint != 0);
  if (a.defer.slots && (a.defer.slot_bytes < slot_bytes_for(L, L.T) || a.defer.max_chunks * a.defer.chunk < L.T))
    return cudaErrorInvalidValue;
  const int vs = L.Vc / 32;
  if (vs <= 2) return launch_vs<2>(a, L, st, sm_count, launches);
  if (vs <= 3) return launch_vs<3>(a, L, st, sm_count, launches);
  if (vs <= 4) return launch_vs<4>(a, L, st, sm_count, launches);
  if (vs <= 6) return launch_vs<6>(a, L, st, sm_count, launches);
  return launch_vs<8>(a, L, st, sm_count, launches);
}

cudaError_t probe_batch_launch(const ProbeLaunch *probes, const int *start, int ndiag, long rows, int P, int V,
                               cudaStream_t st) {
  if (rows <= 0) return cudaSuccess;
  if (P > kMaxP || V > kMaxV || P < 7 || V < 8) return cudaErrorInvalidValue;
  const Layout L = make_layout(P, V, 0, false);
  const int wpb = warps_per_block_for(L);
  if (wpb == 0) return cudaErrorInvalidValue;
  const size_t smem = size_t(L.total) * wpb;
  const int blocks = int((rows + wpb - 1) / wpb);
  const int vs = L.Vc / 32;
  cudaError_t e;
#define RPD_PROBE_BATCH(VSN)                                                        \
  e = allow_smem(reinterpret_cast<const void *>(k_probe_batch<VSN>), smem);         \
  if (e != cudaSuccess) return e;                                                   \
  k_probe_batch<VSN><<<blocks, wpb * 32, smem, st>>>(probes, start, ndiag, L);
  if (vs <= 2) {
    RPD_PROBE_BATCH(2)
  } else if (vs <= 3) {
    RPD_PROBE_BATCH(3)
  } else if (vs <= 4) {
    RPD_PROBE_BATCH(4)
  } else if (vs <= 6) {
    RPD_PROBE_BATCH(6)
  } else {
    RPD_PROBE_BATCH(8)
  }
#undef RPD_PROBE_BATCH
  return cudaGetLastError();
}

cudaError_t probe_launch(const ProbeLaunch &p, cudaStream_t st) {
  if (p.n <= 0) return cudaSuccess;
  if (p.P > kMaxP || p.V > kMaxV || p.P < 7 || p.V < 8 || !p.grid.sat || !p.wmin) return cudaErrorInvalidValue;
  const Layout L = make_layout(p.P, p.V, 0, false);
  const int wpb = warps_per_block_for(L);
  if (wpb == 0) return cudaErrorInvalidValue;
  const size_t smem = size_t(L.total) * wpb;
  const int blocks = (p.n + wpb - 1) / wpb;
  const int vs = L.Vc / 32;
  cudaError_t e;
#define RPD_PROBE(VSN)                                                              \
  e = allow_smem(reinterpret_cast<const void *>(k_probe<VSN>), smem);               \
  if (e != cudaSuccess) return e;                                                   \
  k_probe<VSN><<<blocks, wpb * 32, smem, st>>>(p, L);
  if (vs <= 2) {
    RPD_PROBE(2)
  } else if (vs <= 3) {
    RPD_PROBE(3)
  } else if (vs <= 4) {
    RPD_PROBE(4)
  } else if (vs <= 6) {
    RPD_PROBE(6)
  } else {
    RPD_PROBE(8)
  }
#undef RPD_PROBE
  return cudaGetLastError();
}

}  // namespace rpd
