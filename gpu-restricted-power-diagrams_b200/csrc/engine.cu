// Host side of the engine: context, seed binning and neighbour queries
// behind the C ABI declared in include/rpd.h.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "engine.cuh"

namespace rpd {

namespace pool_detail {
constexpr int kMaxDev = 64;
std::mutex g_alloc_mu;
cudaStream_t g_alloc_stream[kMaxDev] = {};

cudaError_t alloc_stream(cudaStream_t *out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_alloc_mu);
  if (!g_alloc_stream[dev]) {
    // keep freed blocks in the pool instead of returning them at every
    // synchronization
    cudaMemPool_t pool;
    if ((e = cudaDeviceGetDefaultMemPool(&pool, dev)) != cudaSuccess) return e;
    unsigned long long keep = ~0ull;
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
    if ((e = cudaStreamCreateWithFlags(&g_alloc_stream[dev], cudaStreamNonBlocking)) != cudaSuccess) return e;
  }
  *out = g_alloc_stream[dev];
  return cudaSuccess;
}
}  // namespace pool_detail

cudaError_t pool_alloc(void **p, size_t bytes) {
  cudaStream_t st;
  cudaError_t e = pool_detail::alloc_stream(&st);
  if (e != cudaSuccess) return e;
  if ((e = cudaMallocAsync(p, bytes, st)) != cudaSuccess) return e;
  // usable from every stream once the allocation stream has reached it
  return cudaStreamSynchronize(st);
}

void pool_free(void *p) {
  cudaStream_t st;
  if (pool_detail::alloc_stream(&st) == cudaSuccess) cudaFreeAsync(p, st);
}


namespace {
thread_local std::string g_cuda_error;
}

int cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  g_cuda_error = buf;
  return e == cudaErrorMemoryAllocation ? RPD_ERR_OOM : RPD_ERR_CUDA;
}

void set_error(rpd_context *ctx, const std::string &msg) {
  if (ctx) ctx->error = msg;
}

int map_cuda(rpd_context *ctx, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return RPD_OK;
  set_error(ctx, std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? RPD_ERR_OOM : RPD_ERR_CUDA;
}

__global__ void k_knn_to_user(const unsigned *__restrict__ knn, const int *__restrict__ perm,
                              const int *__restrict__ user_to_stored, int n, int K, int *__restrict__ out) {
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= long(n) * K) return;
  const int u = int(i / K), k = int(i % K);
  const unsigned v = knn[size_t(user_to_stored[u]) * K + k];
  out[i] = v == 0xffffffffu ? -1 : perm[v];
}

// Failing cells among `ids` (all seeds when null): f0 = status != success,
// f1 = failing and (cond == 0 or status != empty_cell); status histogram of
// the failing ones (recomputeIds, voronoi.cpp:793-826).
__global__ void k_fail_flags(const int *__restrict__ ids, int num, const int *__restrict__ status, int cond,
                             int *__restrict__ f0, int *__restrict__ f1, int *__restrict__ hist) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > num) return;
  if (i == num) {
    f0[i] = 0;
    f1[i] = 0;
    return;
  }
  const int sid = ids ? ids[i] : i;
  const int st = status[sid];
  const bool fail = st != kSuccess;
  f0[i] = fail;
  f1[i] = fail && (cond == 0 || st != kEmptyCell);
  if (fail) atomicAdd(&hist[st], 1);
}

__global__ void k_fail_scatter(const int *__restrict__ ids, int num, const int *__restrict__ f0,
                               const int *__restrict__ s0, const int *__restrict__ f1, const int *__restrict__ s1,
                               int *__restrict__ out0, int *__restrict__ out1, int *__restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == num) {
    counts[0] = s0[num];
    counts[1] = s1[num];
  }
  if (i >= num) return;
  const int sid = ids ? ids[i] : i;
  if (f0[i]) out0[s0[i]] = sid;
  if (f1[i]) out1[s1[i]] = sid;
}

// CUDA events of one call, destroyed on every return (a recorded event is
// released once the device has passed it).
template <int N>
struct Events {
  cudaEvent_t ev[N];
  Events() {
    for (auto &x : ev) cudaEventCreate(&x);
  }
  ~Events() {
    for (auto &x : ev) cudaEventDestroy(x);
  }
  Events(const Events &) = delete;
  Events &operator=(const Events &) = delete;
  cudaEvent_t operator[](int i) const { return ev[i]; }
};

// Rows the outside probe left among stored seeds first .. first + n - 1:
// f[i] = 1 where status is kProbeMiss; f[n] = 0.
__global__ void k_probe_flags(const int *__restrict__ status, int first, int n, int *__restrict__ f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) f[i] = status[first + i] == kProbeMiss;
  else if (i == n) f[i] = 0;
}

__global__ void k_probe_scatter(int first, int n, const int *__restrict__ f, const int *__restrict__ pos,
                                int *__restrict__ ids) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && f[i]) ids[pos[i]] = first + i;
}

// ids[i] = first + i (a contiguous range of stored ids).
__global__ void k_iota(int first, int n, int *__restrict__ ids) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ids[i] = first + i;
}

template <class T>
__global__ void k_gather_user(const T *__restrict__ src, const int *__restrict__ user_to_stored, int n,
                              T *__restrict__ dst) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n) dst[u] = src[user_to_stored[u]];
}

__global__ void k_status_hist(const int *__restrict__ status, int n, int *__restrict__ hist) {
  __shared__ int h[kStatusNum];
  if (threadIdx.x < kStatusNum) h[threadIdx.x] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int st = status[i];
    if (st >= 0 && st < kStatusNum) atomicAdd(&h[st], 1);
  }
  __syncthreads();
  if (threadIdx.x < kStatusNum && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// Hessian rows in user order: values copied up to a row's terminator, the
// neighbours as user ids; the rest of a row is zeros and -1.
__global__ void k_hessian_user(const double *__restrict__ hess, const int *__restrict__ hessid,
                               const int *__restrict__ user_to_stored, const int *__restrict__ perm, int n, int H,
                               int HC, double *__restrict__ vals, int *__restrict__ ids) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  const size_t sid = size_t(user_to_stored[u]);
  bool live = true;
  for (int k = 0; k < H; ++k) {
    const int v = live ? hessid[sid * H + k] : -1;
    live = v >= 0;
    ids[size_t(u) * H + k] = live ? perm[v] : -1;
    for (int c = 0; c < HC; ++c)
      vals[(size_t(u) * H + k) * HC + c] = live ? hess[(sid * H + k) * HC + c] : 0.0;
  }
}

// Hessian rows of the used cells (compact_result, voronoi.cpp:594-629): the
// row of used user u goes to its compacted position pos[u]; a cell lighter
// than eps has an empty row; a neighbour is kept when it is used and not
// lighter than eps, as its compacted position.
__global__ void k_hessian_used(const int *__restrict__ f, const int *__restrict__ pos, int n,
                               const int *__restrict__ user_to_stored, const int *__restrict__ perm,
                               const double4 *__restrict__ out, double eps, const double *__restrict__ hess,
                               const int *__restrict__ hessid, int H, int HC, double *__restrict__ vals,
                               int *__restrict__ ids) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n || !f[u]) return;
  const size_t sid = size_t(user_to_stored[u]), row = size_t(pos[u]);
  int w = 0;
  if (out[sid].w >= eps) {
    for (int k = 0; k < H; ++k) {
      const int v = hessid[sid * H + k];
      if (v < 0) break;
      const int uv = perm[v];
      if (!f[uv] || out[v].w < eps) continue;
      ids[row * H + w] = pos[uv];
      for (int c = 0; c < HC; ++c) vals[(row * H + w) * HC + c] = hess[(sid * H + k) * HC + c];
      ++w;
    }
  }
  for (int k = w; k < H; ++k) {
    ids[row * H + k] = -1;
    for (int c = 0; c < HC; ++c) vals[(row * H + k) * HC + c] = 0.0;
  }
}

// Stored ids of the bordering cells of distance d: marked d-1, not used
// themselves (find_bordering, voronoi.cpp:711-719), ascending.
__global__ void k_border_flags(const unsigned char *__restrict__ used, const double4 *__restrict__ out, int n, int d,
                               double eps, int *__restrict__ f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n) return;
  f[i] = i < n && int(used[i]) + 1 == d && out[i].w < eps;
}
__global__ void k_scatter_flagged(const int *__restrict__ f, const int *__restrict__ pos, int n, int *__restrict__ out,
                                  int *__restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == n) *count = pos[n];
  if (i < n && f[i]) out[pos[i]] = i;
}
// User-order flags of the used cells.
__global__ void k_used_flags(const unsigned char *__restrict__ used, const int *__restrict__ user_to_stored, int n,
                             int *__restrict__ f) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u > n) return;
  f[u] = u < n && used[user_to_stored[u]] != 0;
}
// compact_result (voronoi.cpp:590-625): rows in ascending user order.
__global__ void k_used_compact(const int *__restrict__ f, const int *__restrict__ pos, int n,
                               const int *__restrict__ user_to_stored, const double4 *__restrict__ out,
                               const unsigned char *__restrict__ used, int keep_distance, double eps,
                               double4 *__restrict__ rows, int *__restrict__ user_ids) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n || !f[u]) return;
  const int sid = user_to_stored[u];
  double4 r = out[sid];
  if (r.w < eps && int(used[sid]) == keep_distance) r.w = double(kNoCellLimits);
  rows[pos[u]] = r;
  user_ids[pos[u]] = u;
}

}  // namespace rpd

using namespace rpd;

namespace {

// Failing ids of the cells in `ids_in` (null: all n) into out0 (all
// failing) and out1 (failing, filtered by cond), their counts and the status
// histogram; synchronous.
int recompute_ids(rpd_solver *s, const int *ids_in, int num, int cond, int *out0, int *out1, int &n0, int &n1,
                  int hist[kStatusNum]) {
  rpd_context *ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const size_t nsc = scan_workspace_ints(num + 1);
  if ((e = s->fail_ws.ensure(sizeof(int) * (4 * size_t(num + 1) + nsc))) != cudaSuccess)
    return map_cuda(ctx, e, "alloc fail ws");
  int *f0 = s->fail_ws.as<int>(), *f1 = f0 + (num + 1), *s0 = f1 + (num + 1), *s1 = s0 + (num + 1),
      *tiles = s1 + (num + 1);
  int *h = s->hist.as<int>();
  if ((e = cudaMemsetAsync(h, 0, sizeof(int) * 16, st)) != cudaSuccess) return map_cuda(ctx, e, "memset");
  const int tb = 256;
  k_fail_flags<<<(num + 1 + tb - 1) / tb, tb, 0, st>>>(ids_in, num, s->status.as<int>(), cond, f0, f1, h);
  if ((e = exclusive_scan(f0, s0, num + 1, tiles, st)) != cudaSuccess) return map_cuda(ctx, e, "scan");
  if ((e = exclusive_scan(f1, s1, num + 1, tiles, st)) != cudaSuccess) return map_cuda(ctx, e, "scan");
  k_fail_scatter<<<(num + 1 + tb - 1) / tb, tb, 0, st>>>(ids_in, num, f0, s0, f1, s1, out0, out1, h + 12);
  s->stats.kernel_launches += 8;  // flags, 2 scans of 3 kernels, scatter
  int hh[16];
  if ((e = cudaMemcpyAsync(hh, h, sizeof(hh), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return map_cuda(ctx, e, "copy hist");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "recompute ids");
  for (int i = 0; i < kStatusNum; ++i) hist[i] = hh[i];
  n0 = hh[12];
  n1 = hh[13];
  return RPD_OK;
}

int select_bordering(rpd_solver *s, int d, int &count) {
  rpd_context *ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const int n = s->n;
  const size_t nsc = scan_workspace_ints(n + 1);
  if ((e = s->fail_ws.ensure(sizeof(int) * (2 * size_t(n + 1) + nsc + 1))) != cudaSuccess)
    return map_cuda(ctx, e, "alloc bordering ws");
  int *f = s->fail_ws.as<int>(), *pos = f + (n + 1), *tiles = pos + (n + 1), *cnt = tiles + nsc;
  const int tb = 256;
  k_border_flags<<<(n + 1 + tb - 1) / tb, tb, 0, st>>>(s->used.as<unsigned char>(), s->out.as<double4>(), n, d,
                                                        s->keep_volume, f);
  if ((e = exclusive_scan(f, pos, n + 1, tiles, st)) != cudaSuccess) return map_cuda(ctx, e, "scan");
  k_scatter_flagged<<<(n + 1 + tb - 1) / tb, tb, 0, st>>>(f, pos, n, s->ids_c.as<int>(), cnt);
  s->stats.kernel_launches += 5;
  if ((e = cudaMemcpyAsync(&count, cnt, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return map_cuda(ctx, e, "copy count");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "bordering ids");
  return RPD_OK;
}

// User-order flags and positions of the used cells in fail_ws; their count.
int used_positions(rpd_solver *s, int **f_out, int **pos_out, int &count) {
  rpd_context *ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const int n = s->n;
  const size_t nsc = scan_workspace_ints(n + 1);
  if ((e = s->fail_ws.ensure(sizeof(int) * (2 * size_t(n + 1) + nsc))) != cudaSuccess)
    return map_cuda(ctx, e, "alloc used ws");
  int *f = s->fail_ws.as<int>(), *pos = f + (n + 1), *tiles = pos + (n + 1);
  const int tb = 256;
  k_used_flags<<<(n + 1 + tb - 1) / tb, tb, 0, st>>>(s->used.as<unsigned char>(), s->user_to_stored.as<int>(), n, f);
  if ((e = exclusive_scan(f, pos, n + 1, tiles, st)) != cudaSuccess) return map_cuda(ctx, e, "scan");
  if ((e = cudaMemcpyAsync(&count, pos + n, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return map_cuda(ctx, e, "copy count");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "used cells");
  *f_out = f;
  *pos_out = pos;
  return RPD_OK;
}

int count_used(rpd_solver *s) {
  int *f = nullptr, *pos = nullptr, c = 0;
  const int rc = used_positions(s, &f, &pos, c);
  if (rc == RPD_OK) s->used_count = c;
  s->stats.kernel_launches += 4;
  return rc;
}

// Outside probe (probe_launch) over every seed of a first pass, then the
// stored ids of the seeds it left into `ids`, ascending; synchronous.  The
// cage test runs where the plainly-outside ball is at least one mean seed
// spacing wide, clipping where it is at least 1.5.
int run_probe(rpd_solver *s, int P, int V, float eps, int *ids, int &nmiss, int first, int n) {
  rpd_context *ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const size_t nsc = scan_workspace_ints(n + 1);
  if ((e = s->fail_ws.ensure(sizeof(int) * (2 * size_t(n + 1) + nsc))) != cudaSuccess)
    return map_cuda(ctx, e, "alloc probe ws");
  int *f = s->fail_ws.as<int>(), *pos = f + (n + 1), *tiles = pos + (n + 1);
  Events<2> ev;
  cudaEventRecord(ev[0], st);
  ProbeLaunch pr;
  pr.stored = s->stored.as<float4>();
  pr.n = n;
  pr.first = first;
  pr.bins = s->counters.as<int>();
  pr.dim = s->dim;
  pr.grid = s->grid;
  pr.P = P;
  pr.V = V;
  pr.cube_eps = eps;
  const double spacing = 1000.0 / std::cbrt(double(s->n));
  pr.min_plain_cage = 1.0 * spacing;
  pr.min_plain = 1.5 * spacing;
  pr.wmin = s->wmin.as<int>();
  pr.status = s->status.as<int>();
  pr.out = s->out.as<double4>();
  if ((e = probe_launch(pr, st)) != cudaSuccess) return map_cuda(ctx, e, "probe");
  const int tb = 256;
  k_probe_flags<<<(n + 1 + tb - 1) / tb, tb, 0, st>>>(s->status.as<int>(), first, n, f);
  if ((e = exclusive_scan(f, pos, n + 1, tiles, st)) != cudaSuccess) return map_cuda(ctx, e, "scan");
  k_probe_scatter<<<(n + tb - 1) / tb, tb, 0, st>>>(first, n, f, pos, ids);
  cudaEventRecord(ev[1], st);
  int cnt = 0;
  cudaMemcpyAsync(&cnt, pos + n, sizeof(int), cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "probe");
  cudaEventElapsedTime(&s->stats.probe_ms, ev[0], ev[1]);
  s->stats.probe_outside = n - cnt;
  s->stats.kernel_launches += 6;  // probe, flags, scan (3), scatter
  nmiss = cnt;
  return RPD_OK;
}

// The neighbour-search variant for K rows of this solver (rpd::KnnVariant).
// RPD_FLAG_KNN_WARP / RPD_FLAG_KNN_THREAD force one.  Otherwise the
// context's choice for K, made the first time K comes up with enough rows to
// tell: both variants run on the first rows (one untimed round, one timed
// with events), into `out`, which the real launch then overwrites; both give
// the same lists, so only their speed differs.  Fewer rows than a trial
// takes (retry passes): a warp per seed -- a thread per seed leaves most of
// the GPU idle there and each row's search serial (0.45 ms for 144 rows).
int knn_variant_for(rpd_solver *s, const int *ids, int num, int K, unsigned *out, unsigned flags) {
  if (flags & RPD_FLAG_KNN_WARP) return kKnnWarp;
  if (flags & RPD_FLAG_KNN_THREAD) return K <= kKnnThreadMaxK ? kKnnThread : kKnnWarp;
  constexpr int kTrialRows = 16384;
  if (K > kKnnThreadMaxK || num < kTrialRows) return kKnnWarp;
  rpd_context *ctx = s->ctx;
  if (ctx->knn_variant[K] >= 0) return ctx->knn_variant[K];
  const int m = kTrialRows;
  cudaStream_t st = ctx->stream;
  Events<4> ev;
  float ms[2] = {0.f, 0.f};
  for (int round = 0; round < 2; ++round)
    for (int v = 0; v < 2; ++v) {
      if (round) cudaEventRecord(ev[2 * v], st);
      if (knn_launch(s->stored.as<float4>(), s->counters.as<int>(), s->dim, ids, m, K, s->ring_bound.as<float>(),
                     out, nullptr, st, v) != cudaSuccess)
        return kKnnWarp;
      if (round) cudaEventRecord(ev[2 * v + 1], st);
    }
  if (cudaEventSynchronize(ev[3]) != cudaSuccess) return kKnnWarp;
  for (int v = 0; v < 2; ++v) cudaEventElapsedTime(&ms[v], ev[2 * v], ev[2 * v + 1]);
  ctx->knn_variant[K] = ms[kKnnThread] < ms[kKnnWarp] ? kKnnThread : kKnnWarp;
  return ctx->knn_variant[K];
}

// One pass (VoroAlgoComputeData::launch, voronoi.cpp:861-1036): the K
// nearest of the listed seeds, then their cells with this pass's caps.
static_assert(int(RPD_CTR_NUM) == int(kCtrNum), "counter enums out of sync");

int run_pass(rpd_solver *s, const int *ids, int num, int K, int P, int V, int T, float eps, int out_domain,
             bool counters, bool early_out, int border_d = 0, int T_ahead = 0, int out_domain_ahead = 0) {
  rpd_context *ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  rpd_stats &S = s->stats;
  const int pi = S.npasses;
  // the neighbours of every cell depend on the positions only: a table for
  // all cells with this K is kept across weight-only re-solves
  const bool all_cells = ids == nullptr && num == s->n;
  rpd::DevBuf &kb = all_cells ? s->knn : s->knn_part;
  const bool reuse = all_cells && s->knn_full_K == K && !counters && !s->fresh_knn;
  if ((e = kb.ensure(sizeof(unsigned) * size_t(num) * K)) != cudaSuccess) return map_cuda(ctx, e, "alloc knn");
  Events<4> ev;
  unsigned long long *ctr = counters ? s->counter64.as<unsigned long long>() : nullptr;
  cudaEventRecord(ev[0], st);
  if (!reuse) {
    if (all_cells) s->knn_full_K = 0;
    const int variant = knn_variant_for(s, ids, num, K, kb.as<unsigned>(), s->launch_flags);
    if (pi < 8) S.pass_knn_variant[pi] = variant;
    e = knn_launch(s->stored.as<float4>(), s->counters.as<int>(), s->dim, ids, num, K, s->ring_bound.as<float>(),
                   kb.as<unsigned>(), ctr ? ctr + RPD_CTR_NUM : nullptr, st, variant);
    if (e != cudaSuccess) return map_cuda(ctx, e, "knn");
    if (all_cells) s->knn_full_K = K;
    S.kernel_launches += 1;
  }
  cudaEventRecord(ev[1], st);
  CellLaunch a;
  a.stored = s->stored.as<float4>();
  a.n = s->n;
  a.knn = kb.as<unsigned>();
  a.K = K;
  a.ids = ids;
  a.num = num;
  a.P = P;
  a.V = V;
  a.T = T;
  a.cube_eps = eps;
  a.out_domain = out_domain;
  // an empty cell is used when keep_volume <= 0, and a used cell marks the
  // plane neighbours of its whole clipped cell: no early exit then
  a.early_out = early_out && !(s->used_on && s->keep_volume <= 0.0) ? 1 : 0;
  a.wmin = s->wmin.as<int>();
  a.inner_apex = s->inner_apex ? 1 : 0;
  a.safe_radius = (s->launch_flags & RPD_FLAG_SAFE_RADIUS) ? 1 : 0;
  if (s->used_on) {
    a.used = s->used.as<unsigned char>();
    a.keep_volume = s->keep_volume;
    a.mark_dist = std::min(s->keep_distance, 1);
    a.border_d = border_d;
  }
  a.grid = s->grid;
  a.precision = s->precision;
  if (s->grid.tsat && border_d == 0) {
    if ((e = s->tri_count.ensure(sizeof(int) * size_t(s->n))) != cudaSuccess) return map_cuda(ctx, e, "alloc");
    a.tri_count = s->tri_count.as<int>();
    a.tri_first = pi == 0 ? 1 : 0;
  }
  a.status = s->status.as<int>();
  a.out = s->out.as<double4>();
  a.counters = ctr;
  a.after_cell = ev[3];
  if (s->hess_h > 0 && border_d == 0) {
    a.hess = s->hess.as<double>();
    a.hessid = s->hessid.as<int>();
    a.H = s->hess_h;
    a.HC = s->hess_hc;
  }
  // Hessian rows are summed in the cell's own warp (no defer queue)
  if (s->grid.size > 0 && s->use_defer && border_d == 0 && s->hess_h == 0) {
    // boundary cells with many triangles are parked and their triangles
    // spread over all warps; cells past the capacity stay inline
    DeferQueue &dq = a.defer;
    const int t_slot = std::max(T, T_ahead);
    dq.capacity = std::min(num, std::max(32768, s->n / 8));
    dq.slot_bytes = defer_slot_bytes(P, V, t_slot);
    dq.chunk = 32;  // a warp's lanes take one triangle each
    dq.inline_max = 16;
    dq.max_chunks = std::max(1, (t_slot + dq.chunk - 1) / dq.chunk);
    a.T_ahead = T_ahead > T ? T_ahead : 0;
    a.out_domain_ahead = out_domain_ahead;
    const size_t items = size_t(dq.capacity) * dq.max_chunks;
    if ((e = s->defer_slots.ensure(dq.slot_bytes * dq.capacity)) != cudaSuccess) return map_cuda(ctx, e, "alloc defer");
    if ((e = s->defer_part.ensure(sizeof(double) * 4 * items)) != cudaSuccess) return map_cuda(ctx, e, "alloc defer");
    if ((e = s->defer_fail.ensure(sizeof(int) * items)) != cudaSuccess) return map_cuda(ctx, e, "alloc defer");
    if ((e = s->defer_chunk_slot.ensure(sizeof(int) * items)) != cudaSuccess) return map_cuda(ctx, e, "alloc defer");
    if ((e = s->defer_ctr.ensure(sizeof(int) * kDeferCounters)) != cudaSuccess) return map_cuda(ctx, e, "alloc defer");
    cudaMemsetAsync(s->defer_ctr.ptr, 0, sizeof(int) * kDeferCounters, st);
    dq.chunk_slot = s->defer_chunk_slot.as<int>();
    dq.slots = s->defer_slots.as<unsigned char>();
    dq.part = s->defer_part.as<double>();
    dq.fail = s->defer_fail.as<int>();
    dq.counters = s->defer_ctr.as<int>();
  }
  int launches = 0;
  if ((e = cell_launch(a, st, ctx->sm_count, &launches)) != cudaSuccess) return map_cuda(ctx, e, "cell kernel");
  if (a.defer.slots) {
    // cells that found the queue full run again with their cones inline
    int ctrs[kDeferCounters] = {};
    cudaMemcpyAsync(ctrs, a.defer.counters, sizeof(ctrs), cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "cell kernel");
    const int parked = ctrs[0];
    if (a.T_ahead > 0) s->ahead_max = ctrs[3];
    if (parked > a.defer.capacity) {
      CellLaunch b = a;
      b.defer = DeferQueue();
      b.T_ahead = 0;
      b.only_status = kParkOverflow;
      b.after_cell = nullptr;
      if ((e = cell_launch(b, st, ctx->sm_count, &launches)) != cudaSuccess) return map_cuda(ctx, e, "cell kernel");
    }
  }
  S.kernel_launches += launches - 1;
  cudaEventRecord(ev[2], st);
  if ((e = cudaEventSynchronize(ev[2])) != cudaSuccess) return map_cuda(ctx, e, "pass");
  if (pi < 8) {
    S.pass_cells[pi] = num;
    S.pass_K[pi] = K;
    S.pass_P[pi] = P;
    S.pass_V[pi] = V;
    S.pass_T[pi] = T;
    cudaEventElapsedTime(&S.pass_knn_ms[pi], ev[0], ev[1]);
    cudaEventElapsedTime(&S.pass_cell_ms[pi], ev[1], ev[2]);
    if (num > 0) cudaEventElapsedTime(&S.pass_cell_kernel_ms[pi], ev[1], ev[3]);
  }
  S.npasses++;
  S.kernel_launches += num > 0 ? 1 : 0;  // the cell kernel (the neighbour kernel counted above)
  return RPD_OK;
}

}  // namespace

extern "C" {

const char *rpd_version(void) { return "rpd-b200 0.1 (sm_100a)"; }

rpd_context *rpd_context_create(int device, int *err) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) {
    cudaGetLastError();
    if (err) *err = RPD_ERR_NO_DEVICE;
    return nullptr;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) {
    if (err) *err = RPD_ERR_NO_DEVICE;
    return nullptr;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    if (err) *err = RPD_ERR_CUDA;
    return nullptr;
  }
  auto *ctx = new rpd_context();
  ctx->device = device;
  ctx->sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    if (err) *err = RPD_ERR_CUDA;
    return nullptr;
  }
  if (err) *err = RPD_OK;
  return ctx;
}

void rpd_context_destroy(rpd_context *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
}

const char *rpd_context_error(const rpd_context *ctx) { return ctx ? ctx->error.c_str() : ""; }

void *rpd_context_stream(rpd_context *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

rpd_solver *rpd_solver_create(rpd_context *ctx, int *err) {
  if (!ctx) {
    if (err) *err = RPD_ERR_INVALID;
    return nullptr;
  }
  auto *s = new rpd_solver();
  s->ctx = ctx;
  if (err) *err = RPD_OK;
  return s;
}

int rpd_context_knn_variant(rpd_context *ctx, int K, int variant) {
  if (!ctx || K < 1 || K > kMaxK || variant < -2 || variant > 1) return RPD_ERR_INVALID;
  if (variant == kKnnThread && K > kKnnThreadMaxK) return RPD_ERR_CAPACITY;
  if (variant != -2) ctx->knn_variant[K] = (signed char)variant;
  return ctx->knn_variant[K];
}

void rpd_solver_destroy(rpd_solver *s) {
  if (!s) return;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  delete s;
}

// The smallest weight of the stored seeds that are not walls
// (w > RPD_NO_CELL_LIMITS) into *wmin (float_to_ordered; set to INT_MAX
// first; stays INT_MAX when every seed is a wall).
__global__ void k_weight_min(const float4 *__restrict__ stored, int n, int *__restrict__ wmin) {
  int m = INT_MAX;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float w = stored[i].w;
    if (w > kNoCellLimits) m = min(m, float_to_ordered(w));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(kFull, m, o));
  if ((threadIdx.x & 31) == 0) atomicMin(wmin, m);
}

cudaError_t update_wmin(rpd_solver *s, cudaStream_t st) {
  cudaError_t e;
  // wmin[1]: a flag of rpd_solver_set_weights
  if ((e = s->wmin.ensure(2 * sizeof(int))) != cudaSuccess) return e;
  static const int highest = INT_MAX;
  if ((e = cudaMemcpyAsync(s->wmin.ptr, &highest, sizeof(int), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
  const int blocks = std::min((s->n + 255) / 256, 4 * s->ctx->sm_count);
  k_weight_min<<<std::max(blocks, 1), 256, 0, st>>>(s->stored.as<float4>(), s->n, s->wmin.as<int>());
  return cudaGetLastError();
}

int rpd_solver_set_points(rpd_solver *s, const float *xyzw, int n, rpd_mem where) {
  if (!s || !xyzw || n <= 0) return RPD_ERR_INVALID;
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const int dim = bins_per_axis(n);
  const size_t nb = size_t(dim) * dim * dim;
  cudaError_t e;
  if ((e = s->user.ensure(sizeof(float4) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc seeds");
  if ((e = s->stored.ensure(sizeof(float4) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc stored");
  if ((e = s->perm.ensure(sizeof(int) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc perm");
  if ((e = s->user_to_stored.ensure(sizeof(int) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc inverse");
  if ((e = s->counters.ensure(sizeof(int) * (nb + 1))) != cudaSuccess) return map_cuda(ctx, e, "alloc bins");
  if ((e = s->bin_ws.ensure(BinWorkspace::bytes(n, dim))) != cudaSuccess) return map_cuda(ctx, e, "alloc ws");
  if ((e = s->ring_bound.ensure(sizeof(float) * (dim + 2))) != cudaSuccess) return map_cuda(ctx, e, "alloc ring");
  e = cudaMemcpyAsync(s->user.ptr, xyzw, sizeof(float4) * n,
                      where == RPD_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return map_cuda(ctx, e, "copy seeds");
  std::vector<float> rb(dim + 2);
  ring_bounds(dim, rb.data());
  if ((e = cudaMemcpyAsync(s->ring_bound.ptr, rb.data(), sizeof(float) * (dim + 2), cudaMemcpyHostToDevice, st)) !=
      cudaSuccess)
    return map_cuda(ctx, e, "copy ring bounds");
  int *w = s->bin_ws.as<int>();
  BinWorkspace ws;
  ws.seed_bin = w;
  ws.counts = ws.seed_bin + n;
  ws.cursor = ws.counts + (nb + 1);
  ws.scan_tiles = ws.cursor + (nb + 1);
  ws.max_fill = ws.scan_tiles + scan_workspace_ints(int(nb + 1));
  BinOutputs out{s->stored.as<float4>(), s->perm.as<int>(), s->counters.as<int>(), s->user_to_stored.as<int>()};
  int fill[2] = {0, 0};  // the largest bin fill, a non-finite seed
  if ((e = bin_seeds(s->user.as<float4>(), n, dim, ws, out, st, fill)) != cudaSuccess)
    return map_cuda(ctx, e, "bin seeds");
  const int max_fill = fill[0];
  if (fill[1]) {
    set_error(ctx, "a seed has a NaN or infinite coordinate or weight");
    s->n = 0;
    return RPD_ERR_INVALID;
  }
  if (max_fill > kMaxBinFill) {
    set_error(ctx, "seeds too clustered: " + std::to_string(max_fill) + " in one bin (limit " +
                       std::to_string(kMaxBinFill) + ")");
    s->n = 0;
    return RPD_ERR_DEGENERATE;
  }
  s->n = n;
  if ((e = update_wmin(s, st)) != cudaSuccess) return map_cuda(ctx, e, "smallest weight");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "bin seeds");
  s->dim = dim;
  s->knn_full_K = 0;
  s->launches_since_points = 0;
  return RPD_OK;
}

// New weights for the seeds already set (user order): the bins and, while K
// stays the same, the neighbour table of the last launch are kept.
__global__ void k_set_weights(const float *w, const int *user_to_stored, int n, float4 *user, float4 *stored) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = w[i];
  user[i].w = x;
  stored[user_to_stored[i]].w = x;
}

// Sets *bad when a value is NaN or infinite.
__global__ void k_any_nonfinite(const float *__restrict__ v, int n, int *__restrict__ bad) {
  bool b = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b |= !isfinite(v[i]);
  if (b) *bad = 1;
}

int rpd_solver_set_weights(rpd_solver *s, const float *w, rpd_mem where) {
  if (!s || !w || s->n <= 0) return RPD_ERR_INVALID;
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const int n = s->n;
  cudaError_t e;
  const float *src = w;
  if (where != RPD_DEVICE) {
    if ((e = s->weights.ensure(sizeof(float) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc weights");
    if ((e = cudaMemcpyAsync(s->weights.ptr, w, sizeof(float) * n, cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return map_cuda(ctx, e, "copy weights");
    src = s->weights.as<float>();
  }
  // a NaN or infinite weight is rejected before any seed changes
  if ((e = s->wmin.ensure(2 * sizeof(int))) != cudaSuccess) return map_cuda(ctx, e, "alloc flag");
  int *bad_dev = s->wmin.as<int>() + 1;
  if ((e = cudaMemsetAsync(bad_dev, 0, sizeof(int), st)) != cudaSuccess) return map_cuda(ctx, e, "clear flag");
  k_any_nonfinite<<<std::max(1, std::min((n + 255) / 256, 4 * ctx->sm_count)), 256, 0, st>>>(src, n, bad_dev);
  int bad = 0;
  if ((e = cudaMemcpyAsync(&bad, bad_dev, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return map_cuda(ctx, e, "read flag");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "check weights");
  if (bad) {
    set_error(ctx, "a weight is NaN or infinite");
    return RPD_ERR_INVALID;
  }
  k_set_weights<<<(n + 255) / 256, 256, 0, st>>>(src, s->user_to_stored.as<int>(), n, s->user.as<float4>(),
                                                 s->stored.as<float4>());
  if ((e = cudaGetLastError()) != cudaSuccess) return map_cuda(ctx, e, "set weights");
  if ((e = update_wmin(s, st)) != cudaSuccess) return map_cuda(ctx, e, "smallest weight");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "set weights");
  s->have_results = false;
  return RPD_OK;
}

int rpd_solver_num_points(const rpd_solver *s) { return s ? s->n : 0; }
int rpd_solver_bin_dim(const rpd_solver *s) { return s ? s->dim : 0; }

int rpd_solver_get_permutation(rpd_solver *s, int *perm, rpd_mem where) {
  if (!s || !perm || s->n <= 0) return RPD_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  cudaError_t e = cudaMemcpyAsync(perm, s->perm.ptr, sizeof(int) * s->n,
                                  where == RPD_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                  s->ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->ctx->stream);
  return map_cuda(s->ctx, e, "copy permutation");
}

int rpd_solver_knn(rpd_solver *s, int K, int *knn_user, rpd_mem where, float *device_ms) {
  if (!s || !knn_user || s->n <= 0 || K <= 0) return RPD_ERR_INVALID;
  if (knn_slots(K) < 0) {
    set_error(s->ctx, "K=" + std::to_string(K) + " above the supported maximum " + std::to_string(kMaxK));
    return RPD_ERR_CAPACITY;
  }
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const size_t nk = size_t(s->n) * K;
  cudaError_t e;
  if ((e = s->knn.ensure(sizeof(unsigned) * nk)) != cudaSuccess) return map_cuda(ctx, e, "alloc knn");
  if ((e = s->knn_user.ensure(sizeof(int) * nk)) != cudaSuccess) return map_cuda(ctx, e, "alloc knn");
  Events<2> ev;
  cudaEventRecord(ev[0], st);
  s->knn_full_K = 0;
  e = knn_launch(s->stored.as<float4>(), s->counters.as<int>(), s->dim, nullptr, s->n, K, s->ring_bound.as<float>(),
                 s->knn.as<unsigned>(), nullptr, st, knn_variant_for(s, nullptr, s->n, K, s->knn.as<unsigned>(), 0));
  cudaEventRecord(ev[1], st);
  if (e != cudaSuccess) return map_cuda(ctx, e, "knn");
  s->knn_full_K = K;
  int *dst = where == RPD_DEVICE ? knn_user : s->knn_user.as<int>();
  const int tb = 256;
  k_knn_to_user<<<int((nk + tb - 1) / tb), tb, 0, st>>>(s->knn.as<unsigned>(), s->perm.as<int>(),
                                                       s->user_to_stored.as<int>(), s->n, K, dst);
  if ((e = cudaGetLastError()) != cudaSuccess) return map_cuda(ctx, e, "knn to user");
  if (where != RPD_DEVICE) {
    if ((e = cudaMemcpyAsync(knn_user, dst, sizeof(int) * nk, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return map_cuda(ctx, e, "copy knn");
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "knn");
  if (device_ms) cudaEventElapsedTime(device_ms, ev[0], ev[1]);
  return RPD_OK;
}

}  // extern "C"

extern "C" {

void rpd_params_default(rpd_params *p) {
  if (!p) return;
  p->K = 20;
  p->P = 25;
  p->V = 30;
  p->T = 100;
  p->max_extra_passes = 5;
  p->cube_eps = -1.f;
  p->out_domain = -1;
  p->flags = 0;
  p->keep_distance = -1;
  p->keep_volume = 0.001;
  p->hessian_h = 0;
  p->hessian_hc = 1;
  p->precision = RPD_PRECISION_FP64;
}

int rpd_solver_set_grid(rpd_solver *s, const rpd_grid *gh) {
  if (!s) return RPD_ERR_INVALID;
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  s->grid = DevGrid();
  s->grid_nonplain = -1;
  if (!gh) return RPD_OK;
  const HostGrid *g = host_grid(gh);
  const size_t nv = size_t(g->size) * g->size * g->size;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  if ((e = s->g_flags.ensure(nv)) != cudaSuccess) return map_cuda(ctx, e, "alloc grid");
  if ((e = s->g_points.ensure(sizeof(float) * g->points.size())) != cudaSuccess) return map_cuda(ctx, e, "alloc grid");
  if ((e = s->g_tris.ensure(sizeof(int) * g->triangles.size())) != cudaSuccess) return map_cuda(ctx, e, "alloc grid");
  if ((e = s->g_list.ensure(sizeof(int) * g->tri_list.size())) != cudaSuccess) return map_cuda(ctx, e, "alloc grid");
  if ((e = s->g_offsets.ensure(sizeof(int) * g->offsets.size())) != cudaSuccess) return map_cuda(ctx, e, "alloc grid");
  cudaMemcpyAsync(s->g_flags.ptr, g->in_domain.data(), nv, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->g_points.ptr, g->points.data(), sizeof(float) * g->points.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->g_tris.ptr, g->triangles.data(), sizeof(int) * g->triangles.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->g_list.ptr, g->tri_list.data(), sizeof(int) * g->tri_list.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->g_offsets.ptr, g->offsets.data(), sizeof(int) * g->offsets.size(), cudaMemcpyHostToDevice, st);
  // summed-volume table of the voxels that are not plainly outside (a
  // first-corner flag other than 0, or triangles): lets a cell prove early
  // that the restriction will give it nothing
  const int S = g->size, S1 = S + 1;
  std::vector<int> sat(size_t(S1) * S1 * S1, 0);
  for (int z = 0; z < S; ++z)
    for (int y = 0; y < S; ++y)
      for (int x = 0; x < S; ++x) {
        const size_t v = x + size_t(S) * (y + size_t(S) * z);
        const int f = (g->in_domain[v] != 0 || g->offsets[v + 1] > g->offsets[v]) ? 1 : 0;
        auto at = [&](int i, int j, int k) -> int & { return sat[i + size_t(S1) * (j + size_t(S1) * k)]; };
        at(x + 1, y + 1, z + 1) = f + at(x, y + 1, z + 1) + at(x + 1, y, z + 1) + at(x + 1, y + 1, z) -
                                  at(x, y, z + 1) - at(x, y + 1, z) - at(x + 1, y, z) + at(x, y, z);
      }
  if ((e = s->g_sat.ensure(sizeof(int) * sat.size())) != cudaSuccess) return map_cuda(ctx, e, "alloc grid");
  cudaMemcpyAsync(s->g_sat.ptr, sat.data(), sizeof(int) * sat.size(), cudaMemcpyHostToDevice, st);
  bool disjoint = true;
  {
    std::vector<unsigned char> seen(size_t(g->num_triangles()), 0);
    for (int t : g->tri_list) {
      if (seen[size_t(t)]) {
        disjoint = false;
        break;
      }
      seen[size_t(t)] = 1;
    }
  }
  // with disjoint lists, the summed triangle counts: a cell whose voxel
  // range holds more than T triangles fails without reading the lists (the
  // union the reference merges has exactly that many ids)
  std::vector<int> tsat;
  if (disjoint) {
    tsat.assign(size_t(S1) * S1 * S1, 0);
    auto at = [&](int i, int j, int k) -> int & { return tsat[i + size_t(S1) * (j + size_t(S1) * k)]; };
    for (int z = 0; z < S; ++z)
      for (int y = 0; y < S; ++y)
        for (int x = 0; x < S; ++x) {
          const size_t v = x + size_t(S) * (y + size_t(S) * z);
          const int f = g->offsets[v + 1] - g->offsets[v];
          at(x + 1, y + 1, z + 1) = f + at(x, y + 1, z + 1) + at(x + 1, y, z + 1) + at(x + 1, y + 1, z) -
                                    at(x, y, z + 1) - at(x, y + 1, z) - at(x + 1, y, z) + at(x, y, z);
        }
    if ((e = s->g_tsat.ensure(sizeof(int) * tsat.size())) != cudaSuccess) return map_cuda(ctx, e, "alloc grid");
    cudaMemcpyAsync(s->g_tsat.ptr, tsat.data(), sizeof(int) * tsat.size(), cudaMemcpyHostToDevice, st);
  } else {
    s->g_tsat.release();
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "upload grid");
  DevGrid d;
  d.size = g->size;
  d.voxel = g->voxel;
  d.flags = s->g_flags.as<const signed char>();
  d.points = s->g_points.as<const float4>();
  d.tris = s->g_tris.as<const int>();
  d.list = s->g_list.as<const int>();
  d.offsets = s->g_offsets.as<const int>();
  d.sat = s->g_sat.as<const int>();
  d.lists_disjoint = disjoint ? 1 : 0;
  d.tsat = disjoint ? s->g_tsat.as<const int>() : nullptr;
  s->grid_points = g->num_points();
  s->grid_triangles = g->num_triangles();
  d.has_border_corners = 0;
  for (char c : g->in_domain)
    if (c == 1) {
      d.has_border_corners = 1;
      break;
    }
  s->grid = d;
  s->grid_nonplain = -1;
  return RPD_OK;
}

}  // extern "C"

// One part of a diagram split over several solvers (rpd_solver_launch_part):
// the stored seeds first .. first + count - 1, and the reduction that makes
// every part's retry schedule the whole diagram's.
struct PartSpec {
  int first, count;
  rpd_part_reduce_fn reduce;
  void *user;
};

// The pass schedule's counts combined over the parts: sums (the failing
// statuses' histogram, the failing cells) and maxima (the largest triangle
// count parked ahead).  Without parts nothing changes.
static int reduce_schedule(rpd_solver *s, const PartSpec *part, int hist[kStatusNum], int &n0) {
  if (!part) return RPD_OK;
  long long sums[kStatusNum + 1], maxes[1];
  for (int i = 0; i < kStatusNum; ++i) sums[i] = hist[i];
  sums[kStatusNum] = n0;
  maxes[0] = s->ahead_max;
  if (part->reduce(sums, kStatusNum + 1, maxes, 1, part->user) != 0) {
    set_error(s->ctx, "part reduction failed");
    return RPD_ERR_INVALID;
  }
  for (int i = 0; i < kStatusNum; ++i) hist[i] = int(sums[i]);
  n0 = int(sums[kStatusNum]);
  s->ahead_max = int(maxes[0]);
  return RPD_OK;
}

static int launch_impl(rpd_solver *s, const rpd_params *pp, const PartSpec *part) {
  if (!s || s->n <= 0) return RPD_ERR_INVALID;
  rpd_params p;
  if (pp) p = *pp;
  else rpd_params_default(&p);
  rpd_context *ctx = s->ctx;
  if (p.K < 1 || knn_slots(p.K) < 0 || p.P < 7 || p.P > kMaxP || p.V < 8 || p.V > kMaxV || p.T < 0 ||
      p.T > kMaxT) {
    set_error(ctx, "caps out of range (1<=K<=256, 7<=P<=255, 8<=V<=256, 0<=T<=4096)");
    return RPD_ERR_CAPACITY;
  }
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const int n = s->n;
  cudaError_t e;
  if ((e = s->out.ensure(sizeof(double4) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc out");
  if ((e = s->status.ensure(sizeof(int) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc status");
  if ((e = s->ids_a.ensure(sizeof(int) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc ids");
  if ((e = s->ids_b.ensure(sizeof(int) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc ids");
  if ((e = s->ids_c.ensure(sizeof(int) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc ids");
  if ((e = s->hist.ensure(sizeof(int) * 16)) != cudaSuccess) return map_cuda(ctx, e, "alloc hist");
  if ((e = s->counter64.ensure(sizeof(unsigned long long) * (RPD_CTR_NUM + 1))) != cudaSuccess)
    return map_cuda(ctx, e, "alloc counters");
  const bool counters = (p.flags & RPD_FLAG_COUNTERS) != 0;
  if (counters) cudaMemsetAsync(s->counter64.ptr, 0, sizeof(unsigned long long) * (RPD_CTR_NUM + 1), st);
  s->stats = rpd_stats{};
  s->have_results = false;
  const bool grid = s->grid.size > 0;
  const float eps = p.cube_eps >= 0 ? p.cube_eps : (grid ? 0.1f : 0.f);
  Events<2> tt;
  const cudaEvent_t t0 = tt[0], t1 = tt[1];
  cudaEventRecord(t0, st);
  // pass "first" + "tr_overflow" in one: T = caps.T from the start gives
  // every cell the result the two reference passes give it
  // (voronoi.cpp:1275-1310)
  const int T0 = p.T;
  const bool early = !(p.flags & RPD_FLAG_NO_EARLY_OUT);
  s->use_defer = !(p.flags & RPD_FLAG_NO_DEFER);
  s->inner_apex = !(p.flags & RPD_FLAG_REFERENCE_APEX);
  s->fresh_knn = (p.flags & RPD_FLAG_FRESH_NEIGHBOURS) != 0;
  s->launch_flags = p.flags;
  // used cells only with a domain (voronoi.cpp:1291)
  s->used_on = grid && p.keep_distance >= 0;
  if (p.hessian_h < 0 || (p.hessian_h > 0 && p.hessian_hc != 1 && p.hessian_hc != 4)) {
    set_error(ctx, "hessian_h must be >= 0 and hessian_hc 1 or 4");
    return RPD_ERR_INVALID;
  }
  if (p.precision < RPD_PRECISION_FP64 || p.precision > RPD_PRECISION_FP32) {
    set_error(ctx, "precision must be RPD_PRECISION_FP64, _MIXED or _FP32");
    return RPD_ERR_INVALID;
  }
  s->precision = p.precision;
  s->hess_h = 0;
  if (p.hessian_h > 0) {
    if ((e = s->hess.ensure(sizeof(double) * size_t(n) * p.hessian_h * p.hessian_hc)) != cudaSuccess)
      return map_cuda(ctx, e, "alloc hessian");
    if ((e = s->hessid.ensure(sizeof(int) * size_t(n) * p.hessian_h)) != cudaSuccess)
      return map_cuda(ctx, e, "alloc hessian");
    s->hess_h = p.hessian_h;
    s->hess_hc = p.hessian_hc;
  }
  s->keep_distance = p.keep_distance;
  s->keep_volume = p.keep_volume;
  s->used_count = -1;
  if (s->used_on) {
    if ((e = s->used.ensure(size_t(n))) != cudaSuccess) return map_cuda(ctx, e, "alloc used");
    cudaMemsetAsync(s->used.ptr, 0, size_t(n), st);
  }
  // outside probe (RPD_FLAG_OUTSIDE_PROBE): with a domain, most seeds outside
  // it are proven empty from a few neighbours and the first pass searches the
  // full K nearest of the others only.  On the first launch after the seeds
  // were set (or with fresh neighbours); later launches build the whole
  // neighbour table once, which weight-only re-solves then keep.
  const bool table_kept = s->knn_full_K == p.K && !s->fresh_knn;
  bool probe = grid && early && s->grid.sat && !counters && s->hess_h == 0 &&
               !(s->used_on && s->keep_volume <= 0.0) && !table_kept &&
               (s->launches_since_points == 0 || s->fresh_knn) && (p.flags & RPD_FLAG_OUTSIDE_PROBE) &&
               !(p.flags & RPD_FLAG_NO_PROBE);
  if (probe) {
    // a domain that fills (nearly) the whole box leaves nothing to prove
    const long long S = s->grid.size, S1 = S + 1;
    if (s->grid_nonplain < 0) {
      int v = 0;
      if ((e = cudaMemcpyAsync(&v, s->grid.sat + (S1 * S1 * S1 - 1), sizeof(int), cudaMemcpyDeviceToHost, st)) !=
              cudaSuccess ||
          (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return map_cuda(ctx, e, "read grid table");
      s->grid_nonplain = v;
    }
    probe = s->grid_nonplain < 0.95 * double(S * S * S);
  }
  // triangle overflows settled ahead: a cell that clips in the first pass
  // and holds more than T triangles is clipped to the same cell by every
  // retry pass, which restricts it once T has grown past its count.  The
  // retries certainly run while this cell fails, up to max_extra_passes,
  // unless P or K outgrow their limits; assuming both grow in every pass,
  // the first pass parks such cells up to the T of the last retry that
  // surely runs, and restricts them as a retry would
  const int out_domain = p.out_domain >= 0 ? p.out_domain : (grid && s->grid.has_border_corners ? 1 : 0);
  int T_ahead = 0;
  s->ahead_max = 0;
  if (grid && s->grid.tsat && s->use_defer && s->inner_apex && s->hess_h == 0 && !counters &&
      !(p.flags & (RPD_FLAG_FIRST_PASS_ONLY | RPD_FLAG_NO_T_AHEAD)))
    T_ahead = t_ahead_cap(p.P, p.K, p.T, p.max_extra_passes);
  int rc;
  // the cells of this launch: every seed, or a part's stored range
  const int first = part ? part->first : 0, count = part ? part->count : n;
  const int *range = nullptr;  // the part's stored ids (null: every seed)
  if (part) {
    if ((e = s->ids_range.ensure(sizeof(int) * size_t(std::max(count, 1)))) != cudaSuccess)
      return map_cuda(ctx, e, "alloc range");
    if (count > 0) k_iota<<<(count + 255) / 256, 256, 0, st>>>(first, count, s->ids_range.as<int>());
    range = s->ids_range.as<int>();
  }
  if (probe) {
    int nmiss = 0;
    int *miss = s->ids_b.as<int>();
    if ((rc = run_probe(s, p.P, p.V, eps, miss, nmiss, first, count)) != RPD_OK) return rc;
    rc = run_pass(s, miss, nmiss, p.K, p.P, p.V, T0, eps, 0, counters, early, 0, T_ahead, out_domain);
    s->stats.pass_cells[0] = count;  // the reference's first pass: every seed (of the part)
  } else {
    rc = run_pass(s, range, count, p.K, p.P, p.V, T0, eps, 0, counters, early, 0, T_ahead, out_domain);
  }
  if (rc != RPD_OK) return rc;
  int K = p.K, P = p.P, V = p.V, T = p.T;
  if (!(p.flags & RPD_FLAG_FIRST_PASS_ONLY)) {
    int hist[kStatusNum];
    int n0 = 0, n1 = 0, n0_all = 0;  // n0: this part's failing cells; n0_all: every part's
    int *A = s->ids_a.as<int>(), *B = s->ids_b.as<int>(), *Cc = s->ids_c.as<int>();
    // extra passes (voronoi.cpp:1311-1376): caps grow x1.5 by failing status
    if ((rc = recompute_ids(s, range, count, 0, A, Cc, n0, n1, hist)) != RPD_OK) return rc;
    n0_all = n0;
    if ((rc = reduce_schedule(s, part, hist, n0_all)) != RPD_OK) return rc;
    for (int step = 0; step < p.max_extra_passes && n0_all > 0; ++step) {
      bool relaunch = false;
      if (hist[kVertexOverflow]) { relaunch = true; V = int(V * 1.5); }
      if (hist[kPlaneOverflow]) { relaunch = true; P = int(P * 1.5); }
      if (hist[kSecurityRadiusNotReached]) { relaunch = true; K = int(K * 1.5); }
      // cells parked ahead still fail in the reference's passes while T is
      // below their count, and keep T growing
      if (hist[kTriangleOverflow] || T < s->ahead_max) { relaunch = true; T = int(T * 1.5); }
      if (!relaunch) break;
      if (P > kMaxP || knn_slots(K) < 0) break;  // the reference stops at P >= 256 (voronoi.cpp:867)
      V = std::min(V, kMaxV);
      T = std::min(T, kMaxT);
      if ((rc = run_pass(s, Cc, n1, K, P, V, T, eps, out_domain, counters, early)) != RPD_OK) return rc;
      if ((rc = recompute_ids(s, A, n0, 1, B, Cc, n0, n1, hist)) != RPD_OK) return rc;
      std::swap(A, B);
      n0_all = n0;
      if ((rc = reduce_schedule(s, part, hist, n0_all)) != RPD_OK) return rc;
    }
  }
  if (s->used_on) {
    // bordering passes (voronoi.cpp:1381-1393) with the last caps: the cells
    // of ring d-1 that are not used themselves mark their neighbours d
    for (int d = 2; d <= p.keep_distance; ++d) {
      int nb = 0;
      if ((rc = select_bordering(s, d, nb)) != RPD_OK) return rc;
      if (nb == 0) break;
      if ((rc = run_pass(s, s->ids_c.as<int>(), nb, K, P, V, T, eps, 0, false, false, d)) != RPD_OK) return rc;
    }
    if ((rc = count_used(s)) != RPD_OK) return rc;
  }
  cudaEventRecord(t1, st);
  int *h = s->hist.as<int>();
  cudaMemsetAsync(h, 0, sizeof(int) * 16, st);
  k_status_hist<<<s->ctx->sm_count, 256, 0, st>>>(s->status.as<int>() + first, count, h);
  s->stats.kernel_launches += 1;
  int hh[16];
  cudaMemcpyAsync(hh, h, sizeof(hh), cudaMemcpyDeviceToHost, st);
  unsigned long long c64[RPD_CTR_NUM + 1] = {};
  if (counters) cudaMemcpyAsync(c64, s->counter64.ptr, sizeof(c64), cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "launch");
  cudaEventElapsedTime(&s->stats.total_ms, t0, t1);
  for (int i = 0; i < kStatusNum; ++i) s->stats.status_hist[i] = hh[i];
  for (int i = 0; i < RPD_CTR_NUM; ++i) s->stats.counters[i] = c64[i];
  s->stats.knn_candidates = c64[RPD_CTR_NUM];
  s->have_results = !part;  // a part's results are complete once gathered (rpd_solver_set_stored)
  s->launches_since_points++;
  return RPD_OK;
}

extern "C" {

int rpd_solver_launch(rpd_solver *s, const rpd_params *p) { return launch_impl(s, p, nullptr); }

int rpd_solver_part_range(int n, int part, int parts, int *first, int *count) {
  if (n < 0 || parts < 1 || part < 0 || part >= parts || !first || !count) return RPD_ERR_INVALID;
  const long long per = (static_cast<long long>(n) + parts - 1) / parts;
  const long long a = std::min<long long>(n, per * part), b = std::min<long long>(n, per * (part + 1));
  *first = int(a);
  *count = int(b - a);
  return RPD_OK;
}

int rpd_solver_launch_part(rpd_solver *s, const rpd_params *pp, int part, int parts, rpd_part_reduce_fn reduce,
                           void *user) {
  if (!s || s->n <= 0 || !reduce) return RPD_ERR_INVALID;
  rpd_params p;
  if (pp) p = *pp;
  else rpd_params_default(&p);
  if (p.hessian_h > 0 || (s->grid.size > 0 && p.keep_distance >= 0)) {
    set_error(s->ctx, "a diagram split over parts returns no Hessian rows or used cells");
    return RPD_ERR_INVALID;
  }
  PartSpec spec{0, 0, reduce, user};
  int rc = rpd_solver_part_range(s->n, part, parts, &spec.first, &spec.count);
  if (rc != RPD_OK) return rc;
  return launch_impl(s, &p, &spec);
}

int rpd_solver_get_stored(rpd_solver *s, double *out4, int *status, int first, int count, rpd_mem where) {
  if (!s || first < 0 || count < 0 || first + count > s->n || (!out4 && !status)) return RPD_ERR_INVALID;
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const cudaMemcpyKind kind = where == RPD_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  cudaError_t e = cudaSuccess;
  if (out4 && count)
    e = cudaMemcpyAsync(out4, s->out.as<double4>() + first, sizeof(double4) * count, kind, st);
  if (e == cudaSuccess && status && count)
    e = cudaMemcpyAsync(status, s->status.as<int>() + first, sizeof(int) * count, kind, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return map_cuda(ctx, e, "get stored results");
}

int rpd_solver_set_stored(rpd_solver *s, const double *out4, const int *status, rpd_mem where) {
  if (!s || s->n <= 0 || !out4 || !status) return RPD_ERR_INVALID;
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const int n = s->n;
  if ((e = s->out.ensure(sizeof(double4) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc out");
  if ((e = s->status.ensure(sizeof(int) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc status");
  const cudaMemcpyKind kind = where == RPD_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if ((e = cudaMemcpyAsync(s->out.ptr, out4, sizeof(double4) * n, kind, st)) == cudaSuccess &&
      (e = cudaMemcpyAsync(s->status.ptr, status, sizeof(int) * n, kind, st)) == cudaSuccess)
    e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return map_cuda(ctx, e, "set stored results");
  s->used_count = -1;
  s->hess_h = 0;
  s->have_results = true;
  return RPD_OK;
}

int rpd_solver_get_moments(rpd_solver *s, double *out4, rpd_mem where) {
  if (!s || !out4 || !s->have_results) return RPD_ERR_INVALID;
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  double4 *dst = reinterpret_cast<double4 *>(out4);
  if (where != RPD_DEVICE) {
    if ((e = s->gather.ensure(sizeof(double4) * s->n)) != cudaSuccess) return map_cuda(ctx, e, "alloc gather");
    dst = s->gather.as<double4>();
  }
  k_gather_user<double4><<<(s->n + 255) / 256, 256, 0, st>>>(s->out.as<double4>(), s->user_to_stored.as<int>(), s->n, dst);
  if (where != RPD_DEVICE)
    cudaMemcpyAsync(out4, dst, sizeof(double4) * s->n, cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  return map_cuda(ctx, e, "get moments");
}

int rpd_solver_get_status(rpd_solver *s, int *status, rpd_mem where) {
  if (!s || !status || !s->have_results) return RPD_ERR_INVALID;
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  int *dst = status;
  if (where != RPD_DEVICE) {
    if ((e = s->gather.ensure(sizeof(double4) * s->n)) != cudaSuccess) return map_cuda(ctx, e, "alloc gather");
    dst = s->gather.as<int>();
  }
  k_gather_user<int><<<(s->n + 255) / 256, 256, 0, st>>>(s->status.as<int>(), s->user_to_stored.as<int>(), s->n, dst);
  if (where != RPD_DEVICE) cudaMemcpyAsync(status, dst, sizeof(int) * s->n, cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  return map_cuda(ctx, e, "get status");
}

int rpd_solver_trace_cell(rpd_solver *s, int user_id, const rpd_params *pp, double *records, int cap) {
  if (!s || !records || cap <= 0 || user_id < 0 || user_id >= s->n) return RPD_ERR_INVALID;
  rpd_params p;
  if (pp) p = *pp;
  else rpd_params_default(&p);
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const int n = s->n;
  if ((e = s->out.ensure(sizeof(double4) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc out");
  if ((e = s->status.ensure(sizeof(int) * n)) != cudaSuccess) return map_cuda(ctx, e, "alloc status");
  if ((e = s->knn_part.ensure(sizeof(unsigned) * p.K)) != cudaSuccess) return map_cuda(ctx, e, "alloc knn");
  DevBuf tr, id;
  if ((e = tr.ensure(sizeof(double) * (1 + size_t(cap) * kTraceRecord))) != cudaSuccess)
    return map_cuda(ctx, e, "alloc trace");
  if ((e = id.ensure(sizeof(int))) != cudaSuccess) return map_cuda(ctx, e, "alloc id");
  int sid = 0;
  cudaMemcpyAsync(&sid, s->user_to_stored.as<int>() + user_id, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  cudaMemcpyAsync(id.ptr, &sid, sizeof(int), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(tr.ptr, 0, sizeof(double), st);
  e = knn_launch(s->stored.as<float4>(), s->counters.as<int>(), s->dim, id.as<int>(), 1, p.K,
                 s->ring_bound.as<float>(), s->knn_part.as<unsigned>(), nullptr, st);
  if (e != cudaSuccess) return map_cuda(ctx, e, "knn");
  CellLaunch a;
  a.stored = s->stored.as<float4>();
  a.n = n;
  a.knn = s->knn_part.as<unsigned>();
  a.K = p.K;
  a.ids = id.as<int>();
  a.num = 1;
  a.P = p.P;
  a.V = p.V;
  a.T = p.T;
  const bool grid = s->grid.size > 0;
  a.cube_eps = p.cube_eps >= 0 ? p.cube_eps : (grid ? 0.1f : 0.f);
  a.out_domain = p.out_domain > 0 ? 1 : 0;
  a.early_out = (p.flags & RPD_FLAG_NO_EARLY_OUT) ? 0 : 1;
  a.wmin = s->wmin.as<int>();
  a.inner_apex = (p.flags & RPD_FLAG_REFERENCE_APEX) ? 0 : 1;
  a.grid = s->grid;
  a.status = s->status.as<int>();
  a.out = s->out.as<double4>();
  a.trace_seed = sid;
  a.trace = tr.as<double>();
  a.trace_cap = cap;
  if ((e = cell_launch(a, st)) != cudaSuccess) return map_cuda(ctx, e, "cell kernel");
  double count = 0;
  cudaMemcpyAsync(&count, tr.ptr, sizeof(double), cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "trace");
  const int nrec = int(count);
  cudaMemcpy(records, tr.as<double>() + 1, sizeof(double) * size_t(nrec) * kTraceRecord, cudaMemcpyDeviceToHost);
  return nrec;
}

int rpd_solver_get_hessian(rpd_solver *s, double *values, int *ids, rpd_mem where) {
  if (!s || !values || !ids || !s->have_results || s->hess_h <= 0) return RPD_ERR_INVALID;
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const int n = s->n, H = s->hess_h, HC = s->hess_hc;
  // with used cells, the rows of the used cells only (compacted)
  int *f = nullptr, *pos = nullptr, rows = n, rc;
  if (s->used_count >= 0 && (rc = used_positions(s, &f, &pos, rows)) != RPD_OK) return rc;
  const size_t nv = size_t(rows) * H * HC, ni = size_t(rows) * H;
  double *dv = values;
  int *di = ids;
  if (where == RPD_HOST) {
    if ((e = s->gather.ensure(sizeof(double) * nv + sizeof(int) * ni + 16)) != cudaSuccess)
      return map_cuda(ctx, e, "alloc gather");
    dv = s->gather.as<double>();
    di = reinterpret_cast<int *>(dv + nv);
  }
  const int tb = 256;
  if (f)
    k_hessian_used<<<(n + tb - 1) / tb, tb, 0, st>>>(f, pos, n, s->user_to_stored.as<int>(), s->perm.as<int>(),
                                                     s->out.as<double4>(), s->keep_volume, s->hess.as<double>(),
                                                     s->hessid.as<int>(), H, HC, dv, di);
  else
    k_hessian_user<<<(n + tb - 1) / tb, tb, 0, st>>>(s->hess.as<double>(), s->hessid.as<int>(),
                                                     s->user_to_stored.as<int>(), s->perm.as<int>(), n, H, HC, dv, di);
  if (where == RPD_HOST) {
    if ((e = cudaMemcpyAsync(values, dv, sizeof(double) * nv, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return map_cuda(ctx, e, "copy hessian");
    if ((e = cudaMemcpyAsync(ids, di, sizeof(int) * ni, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return map_cuda(ctx, e, "copy hessian");
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "hessian");
  return RPD_OK;
}

int rpd_solver_get_stats(const rpd_solver *s, rpd_stats *st) {
  if (!s || !st) return RPD_ERR_INVALID;
  *st = s->stats;
  return RPD_OK;
}

int rpd_solver_used_count(const rpd_solver *s) {
  if (!s || !s->have_results || s->used_count < 0) return RPD_ERR_INVALID;
  return s->used_count;
}

int rpd_solver_get_used(rpd_solver *s, double *rows4, int *user_ids, rpd_mem where) {
  if (!s || !rows4 || !user_ids || !s->have_results || s->used_count < 0) return RPD_ERR_INVALID;
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  int *f = nullptr, *pos = nullptr, c = 0;
  int rc = used_positions(s, &f, &pos, c);
  if (rc != RPD_OK) return rc;
  double4 *rows = reinterpret_cast<double4 *>(rows4);
  int *ids = user_ids;
  if (where != RPD_DEVICE) {
    if ((e = s->gather.ensure((sizeof(double4) + sizeof(int)) * size_t(std::max(c, 1)))) != cudaSuccess)
      return map_cuda(ctx, e, "alloc gather");
    rows = s->gather.as<double4>();
    ids = reinterpret_cast<int *>(rows + std::max(c, 1));
  }
  const int n = s->n, tb = 256;
  k_used_compact<<<(n + tb - 1) / tb, tb, 0, st>>>(f, pos, n, s->user_to_stored.as<int>(), s->out.as<double4>(),
                                                   s->used.as<unsigned char>(), s->keep_distance, s->keep_volume,
                                                   rows, ids);
  if (where != RPD_DEVICE && c > 0) {
    cudaMemcpyAsync(rows4, rows, sizeof(double4) * size_t(c), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(user_ids, ids, sizeof(int) * size_t(c), cudaMemcpyDeviceToHost, st);
  }
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return map_cuda(ctx, e, "get used");
  return c;
}

}  // extern "C"

namespace rpd {

// Runs a solver on another context's stream (no work of the solver may be
// pending).
void solver_rebind(rpd_solver *s, rpd_context *ctx) { s->ctx = ctx; }

// Uses another solver's device grid without a copy (that solver must
// outlive this one).
void solver_share_grid(rpd_solver *dst, const rpd_solver *src) {
  dst->g_flags.release();
  dst->g_points.release();
  dst->g_tris.release();
  dst->g_list.release();
  dst->g_offsets.release();
  dst->g_sat.release();
  dst->g_tsat.release();
  dst->grid = src->grid;
  dst->grid_nonplain = src->grid_nonplain;
  dst->grid_points = src->grid_points;
  dst->grid_triangles = src->grid_triangles;
}

// Releases what only a call in progress needs (binning workspace,
// failing-id lists, parked cells, staging); the seeds, bins, neighbour
// table and results stay.
void solver_trim(rpd_solver *s) {
  s->bin_ws.release();
  s->knn_part.release();
  s->tri_count.release();
  s->knn_user.release();
  s->ids_a.release();
  s->ids_b.release();
  s->ids_c.release();
  s->fail_ws.release();
  s->gather.release();
  s->weights.release();
  s->defer_slots.release();
  s->defer_part.release();
  s->defer_fail.release();
  s->defer_ctr.release();
  s->defer_chunk_slot.release();
  s->hess.release();  // --hessian rows are read out before a trim
  s->hessid.release();
  s->hess_h = 0;
}

size_t solver_device_bytes(const rpd_solver *s) {
  const DevBuf *b[] = {&s->user, &s->stored, &s->perm, &s->user_to_stored, &s->weights, &s->counters, &s->bin_ws,
                       &s->ring_bound, &s->knn, &s->knn_part, &s->tri_count, &s->knn_user, &s->counter64, &s->g_flags, &s->g_points,
                       &s->g_tris, &s->g_list, &s->g_offsets, &s->g_sat, &s->g_tsat, &s->out, &s->status, &s->ids_a, &s->ids_b,
                       &s->ids_c, &s->fail_ws, &s->hist, &s->gather, &s->defer_slots, &s->defer_part, &s->defer_fail,
                       &s->defer_ctr, &s->defer_chunk_slot, &s->wmin, &s->used, &s->hess, &s->hessid};
  size_t t = 0;
  for (const DevBuf *x : b) t += x->bytes;
  return t;
}

int t_ahead_cap(int P, int K, int T, int max_extra) {
  int T_ahead = 0;
  for (int j = 0; j < max_extra; ++j) {
    const int Pn = int(P * 1.5), Kn = int(K * 1.5);
    if (Pn > kMaxP || knn_slots(Kn) < 0) break;
    P = Pn;
    K = Kn;
    T = std::min(int(T * 1.5), kMaxT);
    T_ahead = T;
  }
  return T_ahead;
}

}  // namespace rpd

