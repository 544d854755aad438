// Batched solves: many independent diagrams (solvers of one context) solved
// together, every pass of every diagram in shared persistent launches, the
// whole solve one CUDA graph.
//
// Each diagram follows the pass schedule of rpd_solver_launch, which is the
// reference's (VoroAlgo::launch, voronoi.cpp:1275-1376): a first pass with
// the given caps, then up to max_extra_passes retries of the failing cells,
// each cap growing x1.5 when a failing cell reported its overflow.  Here the
// schedule runs on the device: after every pass a plan kernel reads each
// diagram's failing-cell counts and status histogram, grows its caps, and
// writes the next pass's launch records and row prefixes; the neighbour and
// cell kernels are persistent and read their rows from those prefixes.  The
// launch shapes are fixed at capture: pass j's shared-memory layout holds
// the first-pass maxima of K and T grown j times and of P and V grown at most
// kLayoutGrowths times (P and V grow only in diagrams with plane or vertex
// overflows, T in every pass of the heavy boundary cells), so a pass never
// needs the host.
//
// A diagram whose schedule does not fit the capture (its caps outgrow the
// pass's layout, its retry neighbour rows overflow the shared table, or it
// would run more passes than were captured) is marked unfinished and solved
// again on its own afterwards; results are deterministic, so they are the
// same either way.
#include <algorithm>
#include <cstring>
#include <vector>

#include "engine.cuh"

namespace rpd {
namespace batch_detail {

constexpr int kPassRecord = 8;

// Fixed description of one diagram.
struct DiagStatic {
  const float4 *stored;
  int n;
  const int *bins;  // dim^3+1 bin prefixes
  int dim;
  const float *ring_bound;
  unsigned *knn_full;  // n*K0: the first pass's neighbour table
  int K0, P0, V0, T0;
  int max_extra;   // retry passes allowed (0: first pass only)
  int out_domain;  // start-corner fallback of the retry passes
  int early_out, inner_apex;
  const int *wmin;  // the smallest weight of the seeds that are not walls (float_to_ordered)
  int T_ahead;      // first pass: triangle overflows up to this count parked at once (0: off)
  int probe;        // 1: the outside probe settles the seeds it can before the first pass
  // --hessian rows (H > 0): per seed H facets of HC values and their
  // neighbours, as rpd_solver_launch writes them (the inline kernels only)
  double *hess;
  int *hessid;
  int H, HC;
  int *tri_count;  // n: the triangle overflows' counts (CellLaunch::tri_count; null: none)
  int safe_radius;  // the weighted security-radius guard (RPD_FLAG_SAFE_RADIUS)
  float cube_eps;
  DevGrid grid;
  int *status;
  double4 *out;
  int *ids_a, *ids_b, *ids_c;  // n each: failing-cell lists
};

// Schedule state of one diagram (device; copied to the host at the end).
struct DiagState {
  int K, P, V, T;  // caps of the current pass
  int n0, n1;      // failing cells after the last pass: all of them, those to re-solve
  int step;        // retry passes run
  int active;      // runs the current pass
  int unfinished;  // has passes left that the capture could not run
  int npasses;
  int num, rc_num;  // rows of the current pass and of its recompute
  int *A, *B, *C;   // all failing, scratch, to re-solve (A and B swap after a retry)
  const int *rc_ids;  // rows of the recompute (null: every cell)
  int rc_cond;        // 1: empty cells are not re-solved
  int hist[16];       // status histogram of the failing cells of the last recompute
  int ahead_max;      // the largest triangle count the first pass parked ahead
  int probe_outside;  // seeds the outside probe proved empty
  int final_hist[16]; // status histogram of every cell at the end
  int pass_cells[kPassRecord], pass_K[kPassRecord], pass_P[kPassRecord], pass_V[kPassRecord], pass_T[kPassRecord];
};

// Device arrays the plan kernel writes.
struct Plan {
  CellLaunch *descs;
  CellLaunch *descs_inline;
  KnnDiag *knn;
  int *kstart;       // kKnnClasses x (ndiag+1)
  int *start_grid;   // ndiag+1
  int *start_plain;  // ndiag+1
  int *rc_start;     // ndiag+1
  const int *s0, *s1;  // exclusive scans of the last recompute's flags (before the first
                       // pass: of the probe's misses, over every cell)
  const int *all_start;  // ndiag+1: every cell's row prefix
};

struct PassArgs {
  int pass;     // index of the pass being planned
  int final_;   // 1: after the last captured pass (no pass to plan)
  unsigned *retry_knn;
  long long retry_cap;  // entries of retry_knn
  DeferQueue defer;
  int Pb, Vb, Tb, Kb;  // caps the pass's launches hold
};

// Index of K's slot class in kKnnClassSlots (1, 2, 3, 4, 6, 8 slots).
__device__ __forceinline__ int slot_class(int K) {
  const int s = (K + 31) / 32;
  return s <= 4 ? s - 1 : (s <= 6 ? 4 : (s <= 8 ? 5 : -1));
}

__global__ void __launch_bounds__(1024) k_plan(const DiagStatic *__restrict__ ds, DiagState *__restrict__ st,
                                               int ndiag, Plan pl, PassArgs pa) {
  const int tid = threadIdx.x, nt = blockDim.x;
  // 1. counts of the previous pass's recompute; a retry's still-failing
  //    cells went to B, which becomes A (voronoi.cpp:1364-1370)
  if (pa.pass > 0 || pa.final_) {
    for (int d = tid; d < ndiag; d += nt) {
      DiagState &s = st[d];
      if (!s.active) continue;
      const int a = pl.rc_start[d], b = pl.rc_start[d + 1];
      s.n0 = pl.s0[b] - pl.s0[a];
      s.n1 = pl.s1[b] - pl.s1[a];
      if (s.rc_ids) {
        int *t = s.A;
        s.A = s.B;
        s.B = t;
      }
    }
  }
  __syncthreads();
  // 2. the loop head of the retries (voronoi.cpp:1311-1330)
  for (int d = tid; d < ndiag; d += nt) {
    DiagState &s = st[d];
    const DiagStatic &g = ds[d];
    s.num = 0;
    s.rc_num = 0;
    if (pa.pass == 0 && !pa.final_) {
      s.K = g.K0;
      s.P = g.P0;
      s.V = g.V0;
      s.T = g.T0;
      s.n0 = s.n1 = 0;
      s.step = 0;
      s.active = 1;
      s.unfinished = 0;
      s.npasses = 0;
      s.A = g.ids_a;
      s.B = g.ids_b;
      s.C = g.ids_c;
      // with the probe, the first pass runs the seeds it left (their stored
      // ids in C, scattered before this kernel)
      s.num = g.probe ? pl.s0[pl.all_start[d + 1]] - pl.s0[pl.all_start[d]] : g.n;
      s.probe_outside = g.n - s.num;
      s.rc_ids = nullptr;
      s.rc_cond = 0;
      s.rc_num = g.n;
      s.ahead_max = 0;
      continue;
    }
    if (!s.active) continue;
    bool go = s.step < g.max_extra && s.n0 > 0;
    if (go) {
      int K = s.K, P = s.P, V = s.V, T = s.T;
      bool relaunch = false;
      if (s.hist[kVertexOverflow]) { relaunch = true; V = int(V * 1.5); }
      if (s.hist[kPlaneOverflow]) { relaunch = true; P = int(P * 1.5); }
      if (s.hist[kSecurityRadiusNotReached]) { relaunch = true; K = int(K * 1.5); }
      // cells parked ahead still fail in the reference's passes while T is
      // below their count, and keep T growing
      if (s.hist[kTriangleOverflow] || T < s.ahead_max) { relaunch = true; T = int(T * 1.5); }
      if (!relaunch || P > kMaxP || K > kMaxK) {
        go = false;  // the reference stops at P >= 256 (voronoi.cpp:867)
      } else {
        V = min(V, kMaxV);
        T = min(T, kMaxT);
        if (pa.final_ || P > pa.Pb || V > pa.Vb || T > pa.Tb || K > pa.Kb) {
          s.unfinished = 1;
          go = false;
        } else {
          s.K = K;
          s.P = P;
          s.V = V;
          s.T = T;
        }
      }
    }
    if (!go) {
      s.active = 0;
      continue;
    }
    s.step++;
    s.num = s.n1;
    s.rc_ids = s.A;
    s.rc_cond = 1;
    s.rc_num = s.n0;
  }
  __syncthreads();
  if (pa.final_) {
    for (int d = tid; d < ndiag; d += nt)
      for (int k = 0; k < 16; ++k) st[d].final_hist[k] = 0;
    return;
  }
  // 3. prefixes (one thread: a few passes over the diagrams)
  if (tid == 0) {
    const int stride = ndiag + 1;
    long long koff = 0;
    int g0 = 0, p0 = 0, r0 = 0;
    int kc[kKnnClasses] = {};
    for (int d = 0; d < ndiag; ++d) {
      DiagState &s = st[d];
      const DiagStatic &g = ds[d];
      if (s.active && pa.pass > 0) {
        // retry rows of the neighbour table: a shared buffer
        const long long need = (long long)s.num * s.K;
        if (koff + need > pa.retry_cap) {
          s.unfinished = 1;
          s.active = 0;
          s.num = 0;
          s.rc_num = 0;
        } else {
          pl.knn[d].out = pa.retry_knn + koff;
          koff += need;
        }
      }
      const int c = s.active ? slot_class(s.K) : -1;
      for (int q = 0; q < kKnnClasses; ++q) {
        pl.kstart[q * stride + d] = kc[q];
        if (q == c) kc[q] += s.num;
      }
      pl.start_grid[d] = g0;
      pl.start_plain[d] = p0;
      pl.rc_start[d] = r0;
      if (s.active) {
        if (g.grid.size > 0) g0 += s.num;
        else p0 += s.num;
        r0 += s.rc_num;
      }
    }
    for (int q = 0; q < kKnnClasses; ++q) pl.kstart[q * stride + ndiag] = kc[q];
    pl.start_grid[ndiag] = g0;
    pl.start_plain[ndiag] = p0;
    pl.rc_start[ndiag] = r0;
  }
  __syncthreads();
  // 4. launch records of the pass
  for (int d = tid; d < ndiag; d += nt) {
    DiagState &s = st[d];
    const DiagStatic &g = ds[d];
    if (!s.active) continue;
    const int pi = s.npasses;
    if (pi < kPassRecord) {
      s.pass_cells[pi] = pa.pass == 0 ? g.n : s.num;  // the reference's first pass: every seed
      s.pass_K[pi] = s.K;
      s.pass_P[pi] = s.P;
      s.pass_V[pi] = s.V;
      s.pass_T[pi] = s.T;
    }
    s.npasses++;
    for (int k = 0; k < 16; ++k) s.hist[k] = 0;
    const int *ids = pa.pass == 0 && !g.probe ? nullptr : s.C;
    unsigned *kout = pa.pass == 0 ? g.knn_full : pl.knn[d].out;
    KnnDiag &kd = pl.knn[d];
    kd.stored = g.stored;
    kd.counters = g.bins;
    kd.dim = g.dim;
    kd.K = s.K;
    kd.ids = ids;
    kd.ring_bound = g.ring_bound;
    kd.out = kout;
    CellLaunch a;
    a.stored = g.stored;
    a.n = g.n;
    a.knn = kout;
    a.K = s.K;
    a.ids = ids;
    a.num = s.num;
    a.P = s.P;
    a.V = s.V;
    a.T = s.T;
    a.cube_eps = g.cube_eps;
    a.out_domain = pa.pass == 0 ? 0 : g.out_domain;
    if (pa.pass == 0 && pa.defer.slots) {
      a.T_ahead = g.T_ahead;
      a.out_domain_ahead = g.out_domain;
      a.ahead_max = &s.ahead_max;
    }
    a.early_out = g.early_out;
    a.wmin = g.wmin;
    a.inner_apex = g.inner_apex;
    a.safe_radius = g.safe_radius;
    a.grid = g.grid;
    a.status = g.status;
    a.out = g.out;
    a.diag = d;
    a.hess = g.hess;
    a.hessid = g.hessid;
    a.H = g.H;
    a.HC = g.HC;
    a.tri_count = g.tri_count;
    a.tri_first = pa.pass == 0 ? 1 : 0;
    a.defer = pa.defer;
    pl.descs[d] = a;
    a.defer = DeferQueue();
    a.T_ahead = 0;
    pl.descs_inline[d] = a;
  }
}

// Failing cells among each diagram's recompute rows (recomputeIds,
// voronoi.cpp:793-826): flags f0 (failing) and f1 (failing and, in a
// retry, not empty), and the diagram's histogram of failing statuses.
__global__ void k_fail_flags_batch(const DiagStatic *__restrict__ ds, DiagState *__restrict__ st,
                                   const int *__restrict__ rc_start, int ndiag, int *__restrict__ f0,
                                   int *__restrict__ f1) {
  const int total = rc_start[ndiag];
  const int lane = threadIdx.x & 31;
  const int step = gridDim.x * blockDim.x;
  // warp-uniform trip count: the histogram match below needs the whole warp
  for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < total; base += step) {
    const int i = base + lane;
    int key = -1 - lane;  // unique per lane unless failing
    if (i < total) {
      const int d = owner_of_row(rc_start, ndiag, i);
      const DiagState &s = st[d];
      const int loc = i - rc_start[d];
      const int sid = s.rc_ids ? s.rc_ids[loc] : loc;
      const int stt = ds[d].status[sid];
      const bool fail = stt != kSuccess;
      f0[i] = fail;
      f1[i] = fail && (s.rc_cond == 0 || stt != kEmptyCell);
      if (fail && stt >= 0 && stt < 16) key = d * 16 + stt;
    }
    const unsigned grp = __match_any_sync(kFull, key);
    if (key >= 0 && lane == __ffs(grp) - 1) atomicAdd(&st[key >> 4].hist[key & 15], __popc(grp));
  }
}

__global__ void k_fail_scatter_batch(DiagState *__restrict__ st, const int *__restrict__ rc_start, int ndiag,
                                     const int *__restrict__ f0, const int *__restrict__ s0,
                                     const int *__restrict__ f1, const int *__restrict__ s1) {
  const int total = rc_start[ndiag];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    if (!f0[i] && !f1[i]) continue;
    const int d = owner_of_row(rc_start, ndiag, i);
    const DiagState &s = st[d];
    const int r = rc_start[d];
    const int loc = i - r;
    const int sid = s.rc_ids ? s.rc_ids[loc] : loc;
    if (f0[i]) (s.rc_ids ? s.B : s.A)[s0[i] - s0[r]] = sid;
    if (f1[i]) s.C[s1[i] - s1[r]] = sid;
  }
}

// The seeds the outside probe left (status kProbeMiss) in the probed
// diagrams: flags over every cell (f[total] = 0), then their stored ids into
// each diagram's C list in stored order.
__global__ void k_probe_flags_batch(const DiagStatic *__restrict__ ds, const int *__restrict__ all_start, int ndiag,
                                    int *__restrict__ f) {
  const int total = all_start[ndiag];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= total; i += gridDim.x * blockDim.x) {
    if (i == total) {
      f[i] = 0;
      continue;
    }
    const int d = owner_of_row(all_start, ndiag, i);
    f[i] = ds[d].probe && ds[d].status[i - all_start[d]] == kProbeMiss;
  }
}

__global__ void k_probe_scatter_batch(const DiagStatic *__restrict__ ds, const int *__restrict__ all_start, int ndiag,
                                      const int *__restrict__ f, const int *__restrict__ pos) {
  const int total = all_start[ndiag];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    if (!f[i]) continue;
    const int d = owner_of_row(all_start, ndiag, i);
    const int r = all_start[d];
    ds[d].ids_c[pos[i] - pos[r]] = i - r;
  }
}

// Final status histogram of every diagram.
__global__ void k_final_hist(const DiagStatic *__restrict__ ds, DiagState *__restrict__ st,
                             const int *__restrict__ all_start, int ndiag) {
  const int total = all_start[ndiag];
  const int lane = threadIdx.x & 31;
  const int step = gridDim.x * blockDim.x;
  for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < total; base += step) {
    const int i = base + lane;
    int key = -1 - lane;
    if (i < total) {
      const int d = owner_of_row(all_start, ndiag, i);
      const int stt = ds[d].status[i - all_start[d]];
      if (stt >= 0 && stt < 16) key = d * 16 + stt;
    }
    const unsigned grp = __match_any_sync(kFull, key);
    if (key >= 0 && lane == __ffs(grp) - 1) atomicAdd(&st[key >> 4].final_hist[key & 15], __popc(grp));
  }
}

int grow(int x, int times) {
  for (int i = 0; i < times; ++i) x = int(x * 1.5);
  return x;
}

// Growths of P and V the retry passes' layouts hold.  Layouts sized for
// every possible growth (V x7.6 by the sixth pass) ran the late passes at a
// quarter of the warps; on the uneven 256-diagram batch no diagram grows P
// or V more than twice.
constexpr int kLayoutGrowths = 2;

}  // namespace batch_detail
}  // namespace rpd

using namespace rpd;
using namespace rpd::batch_detail;

struct rpd_batch {
  rpd_context *ctx = nullptr;
  std::vector<rpd_solver *> solvers;
  std::vector<rpd_params> params;
  std::vector<DiagStatic> statics;  // of the capture
  int ndiag = 0;
  long long cells = 0;
  DevBuf d_statics, d_states, d_descs, d_descs_inline, d_knn, d_kstart, d_start_grid, d_start_plain, d_rc_start,
      d_all_start;
  DevBuf f0, f1, s0, s1, scan_tiles;
  DevBuf d_probes, d_probe_start;  // outside probe records of the probed diagrams, row prefixes
  bool probed = false;             // the capture runs the outside probe
  int stats_variant[kKnnClasses] = {};       // first pass's neighbour variant per slot class (-1: unused)
  float stats_trial_ms[kKnnClasses][2] = {};  // the capture's trial: warp, thread (0: no trial)
  cudaEvent_t ev_probe = nullptr;  // after the probe and its compaction
  DevBuf retry_knn, defer_slots, defer_part, defer_fail, defer_ctr, defer_chunk_slot, work;
  DiagState *host_states = nullptr;  // pinned
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev[3] = {};  // first pass: before the neighbours, before and after the cell kernel
  cudaEvent_t ev_pass[kPassRecord + 1] = {};  // pass boundaries
  int passes = 0;     // captured passes
  int launches = 0;   // kernels per replay
  int captures = 0;
  rpd_batch_stats stats{};

  ~rpd_batch() {
    drop_graph();
    if (host_states) cudaFreeHost(host_states);
    for (auto &e : ev)
      if (e) cudaEventDestroy(e);
    for (auto &e : ev_pass)
      if (e) cudaEventDestroy(e);
    if (ev_probe) cudaEventDestroy(ev_probe);
  }
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
};

namespace {

int check_params(rpd_context *ctx, const rpd_params &p) {
  if (p.K < 1 || knn_slots(p.K) < 0 || p.P < 7 || p.P > kMaxP || p.V < 8 || p.V > kMaxV || p.T < 0 ||
      p.T > kMaxT) {
    set_error(ctx, "caps out of range (1<=K<=256, 7<=P<=255, 8<=V<=256, 0<=T<=4096)");
    return RPD_ERR_CAPACITY;
  }
  if (p.flags & RPD_FLAG_COUNTERS) {
    set_error(ctx, "batched solves collect no work counters (RPD_FLAG_COUNTERS)");
    return RPD_ERR_INVALID;
  }
  if (p.hessian_h < 0 || (p.hessian_h > 0 && p.hessian_hc != 1 && p.hessian_hc != 4)) {
    set_error(ctx, "hessian_h must be >= 0 and hessian_hc 1 or 4");
    return RPD_ERR_INVALID;
  }
  if (p.precision != RPD_PRECISION_FP64) {
    set_error(ctx, "batched solves clip in FP64 only (precision): use rpd_solver_launch");
    return RPD_ERR_INVALID;
  }
  return RPD_OK;
}

// The solver buffers and the description the capture depends on.
int describe(rpd_batch *b, std::vector<DiagStatic> &out) {
  rpd_context *ctx = b->ctx;
  cudaError_t e;
  out.assign(b->ndiag, DiagStatic{});
  for (int d = 0; d < b->ndiag; ++d) {
    rpd_solver *s = b->solvers[d];
    const rpd_params &p = b->params[d];
    const int n = s->n;
    if (n <= 0) {
      set_error(ctx, "batch: a solver has no points");
      return RPD_ERR_INVALID;
    }
    const bool grid = s->grid.size > 0;
    if (grid && p.keep_distance >= 0) {
      set_error(ctx, "batch: used cells (keep_distance >= 0) are solved with rpd_solver_launch");
      return RPD_ERR_INVALID;
    }
    if ((e = s->out.ensure(sizeof(double4) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc out");
    if ((e = s->status.ensure(sizeof(int) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc status");
    if ((e = s->ids_a.ensure(sizeof(int) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc ids");
    if ((e = s->ids_b.ensure(sizeof(int) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc ids");
    if ((e = s->ids_c.ensure(sizeof(int) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc ids");
    if ((e = s->knn.ensure(sizeof(unsigned) * size_t(n) * p.K)) != cudaSuccess) return map_cuda(ctx, e, "alloc knn");
    DiagStatic &g = out[d];
    g.stored = s->stored.as<float4>();
    g.n = n;
    g.bins = s->counters.as<int>();
    g.dim = s->dim;
    g.ring_bound = s->ring_bound.as<float>();
    g.knn_full = s->knn.as<unsigned>();
    g.K0 = p.K;
    g.P0 = p.P;
    g.V0 = p.V;
    g.T0 = p.T;
    g.max_extra = (p.flags & RPD_FLAG_FIRST_PASS_ONLY) ? 0 : std::max(0, p.max_extra_passes);
    g.out_domain = p.out_domain >= 0 ? p.out_domain : (grid && s->grid.has_border_corners ? 1 : 0);
    g.early_out = (p.flags & RPD_FLAG_NO_EARLY_OUT) ? 0 : 1;
    g.wmin = s->wmin.as<int>();
    // triangle overflows parked ahead, as rpd_solver_launch does
    g.T_ahead = grid && s->grid.tsat && !(p.flags & (RPD_FLAG_NO_DEFER | RPD_FLAG_REFERENCE_APEX |
                                                     RPD_FLAG_FIRST_PASS_ONLY | RPD_FLAG_NO_T_AHEAD))
                    ? t_ahead_cap(p.P, p.K, p.T, std::max(0, p.max_extra_passes))
                    : 0;
    if (g.T_ahead <= p.T) g.T_ahead = 0;
    g.inner_apex = (p.flags & RPD_FLAG_REFERENCE_APEX) ? 0 : 1;
    g.safe_radius = (p.flags & RPD_FLAG_SAFE_RADIUS) ? 1 : 0;
    g.cube_eps = p.cube_eps >= 0 ? p.cube_eps : (grid ? 0.1f : 0.f);
    // the outside probe (RPD_FLAG_OUTSIDE_PROBE), as rpd_solver_launch runs
    // it on a launch with fresh neighbours (every replay computes its
    // neighbours afresh): with a domain that leaves plainly-outside voxels to
    // prove
    g.probe = 0;
    if (grid && g.early_out && s->grid.sat && (p.flags & RPD_FLAG_OUTSIDE_PROBE) && !(p.flags & RPD_FLAG_NO_PROBE)) {
      const long long S = s->grid.size, S1 = S + 1;
      if (s->grid_nonplain < 0) {
        int v = 0;
        if ((e = cudaMemcpyAsync(&v, s->grid.sat + (S1 * S1 * S1 - 1), sizeof(int), cudaMemcpyDeviceToHost,
                                 ctx->stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
          return map_cuda(ctx, e, "read grid table");
        s->grid_nonplain = v;
      }
      g.probe = s->grid_nonplain < 0.95 * double(S * S * S) ? 1 : 0;
    }
    g.hess = nullptr;
    g.hessid = nullptr;
    g.H = g.HC = 0;
    g.tri_count = nullptr;
    if (grid && s->grid.tsat) {
      if ((e = s->tri_count.ensure(sizeof(int) * size_t(n))) != cudaSuccess) return map_cuda(ctx, e, "alloc");
      g.tri_count = s->tri_count.as<int>();
    }
    if (p.hessian_h > 0) {
      // rows are summed in the cell's own warp: no cells parked ahead, no
      // probe (as rpd_solver_launch)
      if ((e = s->hess.ensure(sizeof(double) * size_t(n) * p.hessian_h * p.hessian_hc)) != cudaSuccess)
        return map_cuda(ctx, e, "alloc hessian");
      if ((e = s->hessid.ensure(sizeof(int) * size_t(n) * p.hessian_h)) != cudaSuccess)
        return map_cuda(ctx, e, "alloc hessian");
      g.hess = s->hess.as<double>();
      g.hessid = s->hessid.as<int>();
      g.H = p.hessian_h;
      g.HC = p.hessian_hc;
      g.T_ahead = 0;
      g.probe = 0;
    }
    g.grid = s->grid;
    g.status = s->status.as<int>();
    g.out = s->out.as<double4>();
    g.ids_a = s->ids_a.as<int>();
    g.ids_b = s->ids_b.as<int>();
    g.ids_c = s->ids_c.as<int>();
  }
  return RPD_OK;
}

bool same_statics(const std::vector<DiagStatic> &a, const std::vector<DiagStatic> &b) {
  return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), sizeof(DiagStatic) * a.size()) == 0);
}

// Buffers, then the graph of the whole solve.
int capture(rpd_batch *b) {
  rpd_context *ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  b->drop_graph();
  const int nd = b->ndiag;
  const std::vector<DiagStatic> &G = b->statics;
  long long cells = 0, table = 0;
  int Kmin = kMaxK, Kmax = 0, Pmax = 0, Vmax = 0, Tmax = 0, J = 0;
  bool any_grid = false, any_plain = false, defer = true, any_safe = false, all_disjoint = true;
  int hess_hc = 0;  // the Hessian rows' HC of the diagrams that ask for rows (one for the batch)
  bool class_used[kKnnClasses] = {};
  long class_rows[kKnnClasses] = {};
  long rows_grid0 = 0, rows_plain0 = 0;  // the first pass's rows
  std::vector<int> all_start(nd + 1, 0);
  for (int d = 0; d < nd; ++d) {
    const DiagStatic &g = G[d];
    all_start[d] = int(cells);
    cells += g.n;
    table += (long long)g.n * g.K0;
    Kmin = std::min(Kmin, g.K0);
    Kmax = std::max(Kmax, g.K0);
    Pmax = std::max(Pmax, g.P0);
    Vmax = std::max(Vmax, g.V0);
    Tmax = std::max(Tmax, g.T0);
    J = std::max(J, g.max_extra);
    (g.grid.size > 0 ? any_grid : any_plain) = true;
    if (g.grid.size > 0 && !g.grid.lists_disjoint) all_disjoint = false;
    if (g.safe_radius) any_safe = true;
    if (b->params[d].flags & RPD_FLAG_NO_DEFER) defer = false;
    if (g.H > 0) {
      if (hess_hc && hess_hc != g.HC) {
        set_error(ctx, "batch: Hessian rows with one hessian_hc for every diagram that asks for them");
        return RPD_ERR_INVALID;
      }
      hess_hc = g.HC;
      defer = false;  // rows are summed in the cell's own warp
    }
    for (int c = 0; c < kKnnClasses; ++c)
      if (knn_slots(g.K0) == kKnnClassSlots[c]) {
        class_used[c] = true;
        class_rows[c] += g.n;
      }
    (g.grid.size > 0 ? rows_grid0 : rows_plain0) += g.n;
  }
  if (cells >= (1ll << 31) - 2) {
    set_error(ctx, "batch: more than 2^31 cells");
    return RPD_ERR_INVALID;
  }
  // outside probe records of the probed diagrams (the single solve's, run_probe)
  std::vector<ProbeLaunch> probes;
  std::vector<int> probe_start(1, 0);
  for (int d = 0; d < nd; ++d) {
    const DiagStatic &g = G[d];
    if (!g.probe) continue;
    ProbeLaunch pr;
    pr.stored = g.stored;
    pr.n = g.n;
    pr.bins = g.bins;
    pr.dim = g.dim;
    pr.grid = g.grid;
    pr.P = g.P0;
    pr.V = g.V0;
    pr.cube_eps = g.cube_eps;
    const double spacing = 1000.0 / std::cbrt(double(g.n));
    pr.min_plain_cage = 1.0 * spacing;
    pr.min_plain = 1.5 * spacing;
    pr.wmin = g.wmin;
    pr.status = g.status;
    pr.out = g.out;
    probes.push_back(pr);
    probe_start.push_back(probe_start.back() + g.n);
  }
  const int nprobe = int(probes.size());
  const long probe_rows = probe_start.back();
  all_start[nd] = int(cells);
  b->cells = cells;
  // caps the launches of pass j hold: the first-pass maxima grown j times,
  // P and V at most kLayoutGrowths times
  std::vector<int> Pb, Vb, Tb, Kb;
  for (int j = 0; j <= J; ++j) {
    const int jl = std::min(j, kLayoutGrowths);
    const int P = std::min(grow(Pmax, jl), kMaxP), V = std::min(grow(Vmax, jl), kMaxV),
              T = std::min(grow(Tmax, j), kMaxT), K = std::min(grow(Kmax, j), kMaxK);
    if ((any_grid && !cell_caps_fit(P, V, T, true, hess_hc)) || (any_plain && !cell_caps_fit(P, V, T, false, hess_hc)))
      break;
    Pb.push_back(P);
    Vb.push_back(V);
    Tb.push_back(T);
    Kb.push_back(K);
  }
  const int passes = int(Pb.size());
  if (passes == 0) {
    set_error(ctx, "batch: the first pass's caps exceed the shared memory of a block");
    return RPD_ERR_CAPACITY;
  }
  // device arrays
  const size_t stride = size_t(nd) + 1;
  if ((e = b->d_statics.ensure(sizeof(DiagStatic) * nd)) != cudaSuccess ||
      (e = b->d_states.ensure(sizeof(DiagState) * nd)) != cudaSuccess ||
      (e = b->d_descs.ensure(sizeof(CellLaunch) * nd)) != cudaSuccess ||
      (e = b->d_descs_inline.ensure(sizeof(CellLaunch) * nd)) != cudaSuccess ||
      (e = b->d_knn.ensure(sizeof(KnnDiag) * nd)) != cudaSuccess ||
      (e = b->d_kstart.ensure(sizeof(int) * stride * kKnnClasses)) != cudaSuccess ||
      (e = b->d_start_grid.ensure(sizeof(int) * stride)) != cudaSuccess ||
      (e = b->d_start_plain.ensure(sizeof(int) * stride)) != cudaSuccess ||
      (e = b->d_rc_start.ensure(sizeof(int) * stride)) != cudaSuccess ||
      (e = b->d_all_start.ensure(sizeof(int) * stride)) != cudaSuccess ||
      (e = b->d_probes.ensure(sizeof(ProbeLaunch) * std::max(1, nprobe))) != cudaSuccess ||
      (e = b->d_probe_start.ensure(sizeof(int) * (size_t(nprobe) + 1))) != cudaSuccess)
    return map_cuda(ctx, e, "alloc batch");
  const int nscan = int(cells) + 1;
  if ((e = b->f0.ensure(sizeof(int) * nscan)) != cudaSuccess || (e = b->f1.ensure(sizeof(int) * nscan)) != cudaSuccess ||
      (e = b->s0.ensure(sizeof(int) * nscan)) != cudaSuccess || (e = b->s1.ensure(sizeof(int) * nscan)) != cudaSuccess ||
      (e = b->scan_tiles.ensure(sizeof(int) * scan_workspace_ints(nscan))) != cudaSuccess)
    return map_cuda(ctx, e, "alloc batch scans");
  // retry neighbour rows: as many entries as the first pass's tables
  const long long retry_cap = std::max<long long>(table, 1ll << 20);
  if ((e = b->retry_knn.ensure(sizeof(unsigned) * size_t(retry_cap))) != cudaSuccess)
    return map_cuda(ctx, e, "alloc batch knn");
  // parked boundary cells: one queue for the batch, its bytes fixed by the
  // first pass; later passes (larger slots) hold fewer cells
  const int chunk = 32;  // the cone kernels' chunk (a warp's lanes take one triangle each)
  const int cap0 = int(std::min<long long>(cells, std::max<long long>(32768, cells / 8)));
  // the first pass's slots hold the triangle overflows parked ahead
  int Tslot0 = Tb[0];
  for (int d = 0; d < nd; ++d) Tslot0 = std::max(Tslot0, G[d].T_ahead);
  const size_t slot0 = defer_slot_bytes(Pb[0], Vb[0], Tslot0);
  const size_t items0 = size_t(cap0) * std::max(1, (Tslot0 + chunk - 1) / chunk);
  if (any_grid && defer) {
    if ((e = b->defer_slots.ensure(slot0 * cap0)) != cudaSuccess ||
        (e = b->defer_part.ensure(sizeof(double) * 4 * items0)) != cudaSuccess ||
        (e = b->defer_fail.ensure(sizeof(int) * items0)) != cudaSuccess ||
        (e = b->defer_chunk_slot.ensure(sizeof(int) * items0)) != cudaSuccess ||
        (e = b->defer_ctr.ensure(sizeof(int) * kDeferCounters)) != cudaSuccess)
      return map_cuda(ctx, e, "alloc batch defer");
  }
  if ((e = b->work.ensure(sizeof(int))) != cudaSuccess) return map_cuda(ctx, e, "alloc batch");
  if (!b->host_states && (e = cudaMallocHost(&b->host_states, sizeof(DiagState) * nd)) != cudaSuccess)
    return map_cuda(ctx, e, "alloc batch host");
  for (auto &x : b->ev)
    if (!x && (e = cudaEventCreate(&x)) != cudaSuccess) return map_cuda(ctx, e, "batch events");
  for (auto &x : b->ev_pass)
    if (!x && (e = cudaEventCreate(&x)) != cudaSuccess) return map_cuda(ctx, e, "batch events");
  if (!b->ev_probe && (e = cudaEventCreate(&b->ev_probe)) != cudaSuccess) return map_cuda(ctx, e, "batch events");
  if ((e = cudaMemcpyAsync(b->d_statics.ptr, G.data(), sizeof(DiagStatic) * nd, cudaMemcpyHostToDevice, st)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(b->d_all_start.ptr, all_start.data(), sizeof(int) * stride, cudaMemcpyHostToDevice, st)) !=
          cudaSuccess ||
      (nprobe && (e = cudaMemcpyAsync(b->d_probes.ptr, probes.data(), sizeof(ProbeLaunch) * nprobe,
                                      cudaMemcpyHostToDevice, st)) != cudaSuccess) ||
      (e = cudaMemcpyAsync(b->d_probe_start.ptr, probe_start.data(), sizeof(int) * (nprobe + 1),
                           cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (e = cudaMemsetAsync(b->d_states.ptr, 0, sizeof(DiagState) * nd, st)) != cudaSuccess ||
      (e = cudaMemsetAsync(b->f0.ptr, 0, sizeof(int) * nscan, st)) != cudaSuccess ||
      (e = cudaMemsetAsync(b->f1.ptr, 0, sizeof(int) * nscan, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return map_cuda(ctx, e, "batch setup");

  const DiagStatic *ds = b->d_statics.as<DiagStatic>();
  DiagState *sts = b->d_states.as<DiagState>();
  Plan pl;
  pl.descs = b->d_descs.as<CellLaunch>();
  pl.descs_inline = b->d_descs_inline.as<CellLaunch>();
  pl.knn = b->d_knn.as<KnnDiag>();
  pl.kstart = b->d_kstart.as<int>();
  pl.start_grid = b->d_start_grid.as<int>();
  pl.start_plain = b->d_start_plain.as<int>();
  pl.rc_start = b->d_rc_start.as<int>();
  pl.s0 = b->s0.as<int>();
  pl.s1 = b->s1.as<int>();
  pl.all_start = b->d_all_start.as<int>();
  // persistent neighbour launches: a full SM of 256-thread blocks each
  const int knn_blocks = ctx->sm_count * (2048 / kKnnThreads);
  const int flat_blocks = ctx->sm_count * 8;
  int launches = 0;
  // The first pass's neighbour-search variant per slot class (the
  // autotuner): the probe and the first pass's plan run once outside the
  // graph, so the records and rows exist, then each class large enough to
  // tell (16K rows) is searched both ways on its own rows, timed with events
  // (one untimed round first); the graph takes the faster.  Retry passes
  // (few rows) take a warp per seed.
  int variant[kKnnClasses];
  for (int c = 0; c < kKnnClasses; ++c) {
    variant[c] = kKnnWarp;
    b->stats_trial_ms[c][0] = b->stats_trial_ms[c][1] = 0.f;
  }
  {
    bool trial = false;
    for (int c = 0; c < kKnnClasses; ++c)
      trial |= class_used[c] && 32 * kKnnClassSlots[c] <= kKnnThreadMaxK && class_rows[c] >= 16384;
    if (trial) {
      if (nprobe) {
        if ((e = probe_batch_launch(b->d_probes.as<ProbeLaunch>(), b->d_probe_start.as<int>(), nprobe, probe_rows,
                                    Pb[0], Vb[0], st)) != cudaSuccess)
          return map_cuda(ctx, e, "batch probe");
        k_probe_flags_batch<<<flat_blocks, 256, 0, st>>>(ds, b->d_all_start.as<int>(), nd, b->f0.as<int>());
        if ((e = exclusive_scan(b->f0.as<int>(), b->s0.as<int>(), nscan, b->scan_tiles.as<int>(), st)) != cudaSuccess)
          return map_cuda(ctx, e, "batch scan");
        k_probe_scatter_batch<<<flat_blocks, 256, 0, st>>>(ds, b->d_all_start.as<int>(), nd, b->f0.as<int>(),
                                                           b->s0.as<int>());
      }
      PassArgs pa0;
      pa0.pass = 0;
      pa0.final_ = 0;
      pa0.retry_knn = b->retry_knn.as<unsigned>();
      pa0.retry_cap = retry_cap;
      pa0.Pb = Pb[0];
      pa0.Vb = Vb[0];
      pa0.Tb = Tb[0];
      pa0.Kb = Kb[0];
      pa0.defer = DeferQueue();
      k_plan<<<1, 1024, 0, st>>>(ds, sts, nd, pl, pa0);
      cudaEvent_t te[3];
      for (auto &x : te) cudaEventCreate(&x);
      for (int c = 0; c < kKnnClasses; ++c) {
        const int S = kKnnClassSlots[c];
        if (!class_used[c] || 32 * S > kKnnThreadMaxK || class_rows[c] < 16384) continue;
        for (int round = 0; round < 2 && e == cudaSuccess; ++round) {
          if (round) cudaEventRecord(te[0], st);
          e = knn_batch_launch(S, pl.knn, pl.kstart + c * stride, nd, knn_blocks, st, -1, kKnnWarp);
          if (round) cudaEventRecord(te[1], st);
          if (e == cudaSuccess) e = knn_batch_launch(S, pl.knn, pl.kstart + c * stride, nd, knn_blocks, st, -1, kKnnThread);
          if (round) cudaEventRecord(te[2], st);
        }
        if (e == cudaSuccess) e = cudaEventSynchronize(te[2]);
        if (e != cudaSuccess) break;
        cudaEventElapsedTime(&b->stats_trial_ms[c][0], te[0], te[1]);
        cudaEventElapsedTime(&b->stats_trial_ms[c][1], te[1], te[2]);
        variant[c] = b->stats_trial_ms[c][1] < b->stats_trial_ms[c][0] ? kKnnThread : kKnnWarp;
      }
      for (auto &x : te) cudaEventDestroy(x);
      if (e != cudaSuccess || (e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "batch trial");
    }
  }
  for (int c = 0; c < kKnnClasses; ++c) b->stats_variant[c] = class_used[c] ? variant[c] : -1;
  if ((e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return map_cuda(ctx, e, "begin capture");
  auto fail = [&](cudaError_t err, const char *what) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(st, &g);
    if (g) cudaGraphDestroy(g);
    return map_cuda(ctx, err, what);
  };
  auto mark = [&](cudaEvent_t ev) { return cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal); };
  for (int j = 0; j < passes; ++j) {
    PassArgs pa;
    pa.pass = j;
    pa.final_ = 0;
    pa.retry_knn = b->retry_knn.as<unsigned>();
    pa.retry_cap = retry_cap;
    pa.Pb = Pb[j];
    pa.Vb = Vb[j];
    pa.Tb = Tb[j];
    pa.Kb = Kb[j];
    DeferQueue dq;
    if (any_grid && defer) {
      const int Ts = j == 0 ? Tslot0 : Tb[j];
      dq.slot_bytes = defer_slot_bytes(Pb[j], Vb[j], Ts);
      dq.chunk = chunk;
      dq.inline_max = 16;
      dq.max_chunks = std::max(1, (Ts + chunk - 1) / chunk);
      const size_t by_slots = (slot0 * cap0) / dq.slot_bytes, by_items = items0 / dq.max_chunks;
      dq.capacity = int(std::min<size_t>({size_t(cap0), by_slots, by_items}));
      dq.slots = b->defer_slots.as<unsigned char>();
      dq.part = b->defer_part.as<double>();
      dq.fail = b->defer_fail.as<int>();
      dq.counters = b->defer_ctr.as<int>();
      dq.chunk_slot = b->defer_chunk_slot.as<int>();
      if (dq.capacity < 1) dq = DeferQueue();
    }
    pa.defer = dq;
    if (j < kPassRecord && (e = mark(b->ev_pass[j])) != cudaSuccess) return fail(e, "batch event");
    if (j == 0 && nprobe) {
      // the outside probe over every seed of the probed diagrams, then the
      // stored ids of the seeds it left (the first pass's rows)
      if ((e = probe_batch_launch(b->d_probes.as<ProbeLaunch>(), b->d_probe_start.as<int>(), nprobe, probe_rows,
                                  Pb[0], Vb[0], st)) != cudaSuccess)
        return fail(e, "batch probe");
      k_probe_flags_batch<<<flat_blocks, 256, 0, st>>>(ds, b->d_all_start.as<int>(), nd, b->f0.as<int>());
      if ((e = exclusive_scan(b->f0.as<int>(), b->s0.as<int>(), nscan, b->scan_tiles.as<int>(), st)) != cudaSuccess)
        return fail(e, "batch scan");
      k_probe_scatter_batch<<<flat_blocks, 256, 0, st>>>(ds, b->d_all_start.as<int>(), nd, b->f0.as<int>(),
                                                         b->s0.as<int>());
      launches += 6;  // probe, flags, scan (3), scatter
      if ((e = mark(b->ev_probe)) != cudaSuccess) return fail(e, "batch event");
    }
    k_plan<<<1, 1024, 0, st>>>(ds, sts, nd, pl, pa);
    ++launches;
    if (j == 0 && (e = mark(b->ev[0])) != cudaSuccess) return fail(e, "batch event");
    // neighbours, one launch per slot class the pass can hold
    for (int c = 0; c < kKnnClasses; ++c) {
      const int S = kKnnClassSlots[c];
      const bool want = j == 0 ? class_used[c] : (S >= knn_slots(Kmin) && S <= knn_slots(Kb[j]));
      if (!want) continue;
      if ((e = knn_batch_launch(S, pl.knn, pl.kstart + c * stride, nd, knn_blocks, st,
                                j == 0 && !nprobe ? class_rows[c] : -1, j == 0 ? variant[c] : kKnnWarp)) !=
          cudaSuccess)
        return fail(e, "batch knn");
      ++launches;
    }
    if (dq.slots && (e = cudaMemsetAsync(dq.counters, 0, sizeof(int) * kDeferCounters, st)) != cudaSuccess)
      return fail(e, "batch memset");
    if (j == 0 && (e = mark(b->ev[1])) != cudaSuccess) return fail(e, "batch event");
    CellBatch cb;
    cb.descs = pl.descs;
    cb.descs_inline = pl.descs_inline;
    cb.start_grid = any_grid ? pl.start_grid : nullptr;
    cb.start_plain = any_plain ? pl.start_plain : nullptr;
    cb.ndiag = nd;
    cb.defer = dq;
    cb.P = Pb[j];
    cb.V = Vb[j];
    cb.T = Tb[j];
    cb.T_slot = j == 0 && dq.slots ? Tslot0 : 0;
    cb.HC = hess_hc;
    cb.disjoint = all_disjoint;
    cb.after_cell = j == 0 ? b->ev[2] : nullptr;
    // the first pass's rows are every cell: one warp per row; the retries'
    // rows are known on the device only: persistent, rows from a counter
    cb.rows_grid = j == 0 && !nprobe ? rows_grid0 : -1;
    cb.rows_plain = j == 0 ? rows_plain0 : -1;
    cb.work = b->work.as<int>();
    cb.safe = any_safe;
    if ((e = cell_batch_launch(cb, st, ctx->sm_count, &launches)) != cudaSuccess) return fail(e, "batch cells");
    // failing cells of the pass's diagrams
    k_fail_flags_batch<<<flat_blocks, 256, 0, st>>>(ds, sts, pl.rc_start, nd, b->f0.as<int>(), b->f1.as<int>());
    if ((e = exclusive_scan(b->f0.as<int>(), b->s0.as<int>(), nscan, b->scan_tiles.as<int>(), st)) != cudaSuccess)
      return fail(e, "batch scan");
    if ((e = exclusive_scan(b->f1.as<int>(), b->s1.as<int>(), nscan, b->scan_tiles.as<int>(), st)) != cudaSuccess)
      return fail(e, "batch scan");
    k_fail_scatter_batch<<<flat_blocks, 256, 0, st>>>(sts, pl.rc_start, nd, b->f0.as<int>(), b->s0.as<int>(),
                                                      b->f1.as<int>(), b->s1.as<int>());
    launches += 8;  // flags, 2 scans of 3 kernels, scatter
  }
  if ((e = mark(b->ev_pass[std::min(passes, kPassRecord)])) != cudaSuccess) return fail(e, "batch event");
  PassArgs fin{};
  fin.pass = passes;
  fin.final_ = 1;
  fin.Pb = Pb.back();
  fin.Vb = Vb.back();
  fin.Tb = Tb.back();
  fin.Kb = Kb.back();
  k_plan<<<1, 1024, 0, st>>>(ds, sts, nd, pl, fin);
  k_final_hist<<<flat_blocks, 256, 0, st>>>(ds, sts, b->d_all_start.as<int>(), nd);
  launches += 2;
  if ((e = cudaMemcpyAsync(b->host_states, sts, sizeof(DiagState) * nd, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return fail(e, "batch copy");
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "batch capture");
  if ((e = cudaStreamEndCapture(st, &b->graph)) != cudaSuccess) return map_cuda(ctx, e, "end capture");
  if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess) {
    b->drop_graph();
    return map_cuda(ctx, e, "instantiate graph");
  }
  b->passes = passes;
  b->launches = launches;
  b->probed = nprobe > 0;
  b->captures++;
  return RPD_OK;
}

}  // namespace

extern "C" {

rpd_batch *rpd_batch_create(rpd_context *ctx, rpd_solver *const *solvers, const rpd_params *params, int count,
                            int *err) {
  auto fail = [&](int code) -> rpd_batch * {
    if (err) *err = code;
    return nullptr;
  };
  if (!ctx || !solvers || count <= 0) return fail(RPD_ERR_INVALID);
  auto *b = new rpd_batch;
  b->ctx = ctx;
  b->ndiag = count;
  b->solvers.assign(solvers, solvers + count);
  b->params.resize(count);
  for (int d = 0; d < count; ++d) {
    if (!solvers[d] || solvers[d]->ctx != ctx) {
      set_error(ctx, "batch: every solver must belong to the batch's context");
      delete b;
      return fail(RPD_ERR_INVALID);
    }
    if (params) b->params[d] = params[d];
    else rpd_params_default(&b->params[d]);
    const int rc = check_params(ctx, b->params[d]);
    if (rc != RPD_OK) {
      delete b;
      return fail(rc);
    }
  }
  if (err) *err = RPD_OK;
  return b;
}

void rpd_batch_destroy(rpd_batch *b) {
  if (!b) return;
  cudaSetDevice(b->ctx->device);
  delete b;
}

int rpd_batch_launch(rpd_batch *b) {
  if (!b) return RPD_ERR_INVALID;
  rpd_context *ctx = b->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  std::vector<DiagStatic> now;
  int rc = describe(b, now);
  if (rc != RPD_OK) return rc;
  if (!b->exec || !same_statics(now, b->statics)) {
    // first launch, or a solver's seeds, domain or buffers changed
    b->statics = now;
    if ((rc = capture(b)) != RPD_OK) return rc;
  }
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, st);
  if ((e = cudaGraphLaunch(b->exec, st)) != cudaSuccess) return map_cuda(ctx, e, "graph launch");
  cudaEventRecord(t1, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "batch");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  rpd_batch_stats &S = b->stats;
  S = rpd_batch_stats{};
  S.diagrams = b->ndiag;
  S.cells = b->cells;
  S.graph_ms = ms;
  S.passes_captured = b->passes;
  S.kernel_launches = b->launches;
  S.captures = b->captures;
  cudaEventElapsedTime(&S.pass0_knn_ms, b->ev[0], b->ev[1]);
  cudaEventElapsedTime(&S.pass0_cell_kernel_ms, b->ev[1], b->ev[2]);
  const int rec = std::min(b->passes, kPassRecord);
  for (int j = 0; j < rec; ++j) cudaEventElapsedTime(&S.pass_ms[j], b->ev_pass[j], b->ev_pass[j + 1]);
  if (b->probed) cudaEventElapsedTime(&S.probe_ms, b->ev_pass[0], b->ev_probe);
  for (int c = 0; c < kKnnClasses; ++c) {
    S.knn_variant[c] = b->stats_variant[c];
    S.knn_trial_warp_ms[c] = b->stats_trial_ms[c][0];
    S.knn_trial_thread_ms[c] = b->stats_trial_ms[c][1];
  }
  std::vector<int> again;
  for (int d = 0; d < b->ndiag; ++d) {
    const DiagState &h = b->host_states[d];
    rpd_solver *s = b->solvers[d];
    if (h.unfinished) {
      again.push_back(d);
      continue;
    }
    rpd_stats &T = s->stats;
    T = rpd_stats{};
    T.npasses = h.npasses;
    for (int i = 0; i < kPassRecord && i < h.npasses; ++i) {
      T.pass_cells[i] = h.pass_cells[i];
      T.pass_K[i] = h.pass_K[i];
      T.pass_P[i] = h.pass_P[i];
      T.pass_V[i] = h.pass_V[i];
      T.pass_T[i] = h.pass_T[i];
      S.pass_cells[i] += h.pass_cells[i];
    }
    for (int i = 0; i < kStatusNum; ++i) T.status_hist[i] = h.final_hist[i];
    T.total_ms = ms;
    T.kernel_launches = b->launches;
    T.probe_outside = h.probe_outside;
    S.probe_outside += h.probe_outside;
    S.max_passes = std::max(S.max_passes, h.npasses);
    // with the probe the table holds the first pass's rows only
    s->knn_full_K = b->statics[d].probe ? 0 : b->params[d].K;
    s->used_on = false;
    s->used_count = -1;
    s->hess_h = b->statics[d].H;
    s->hess_hc = b->statics[d].HC;
    s->have_results = true;
  }
  // diagrams whose schedule outgrew the capture: solved alone
  for (int d : again) {
    b->solvers[d]->knn_full_K = 0;
    if ((rc = rpd_solver_launch(b->solvers[d], &b->params[d])) != RPD_OK) return rc;
    S.max_passes = std::max(S.max_passes, b->solvers[d]->stats.npasses);
  }
  S.solved_alone = int(again.size());
  return RPD_OK;
}

int rpd_batch_get_stats(const rpd_batch *b, rpd_batch_stats *st) {
  if (!b || !st) return RPD_ERR_INVALID;
  *st = b->stats;
  return RPD_OK;
}

}  // extern "C"
