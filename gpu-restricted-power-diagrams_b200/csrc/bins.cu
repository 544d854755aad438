// Seed binning on the device: a stable counting sort of the seeds into a
// regular dim^3 grid over [0,1000]^3 (the reference KNearests constructor,
// knearests.cpp:48-222).  The stored order is (bin, user id): deterministic,
// unlike the reference's atomic scatter, so that neighbour lists and cell
// results do not depend on scheduling.
#include "bins.cuh"

namespace rpd {

// Also flags (nonfinite = 1) a seed with a NaN or infinite coordinate or
// weight: the caller rejects the input, whose bins would be meaningless.
__global__ void k_bin_count(const float4 *__restrict__ user, int n, int dim, int *__restrict__ seed_bin,
                            int *__restrict__ counts, int *__restrict__ nonfinite) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool bad = i < n && !(isfinite(user[i].x) && isfinite(user[i].y) && isfinite(user[i].z) && isfinite(user[i].w));
  if (bad) *nonfinite = 1;
  if (i >= n) return;
  const int b = bin_of(user[i], dim);
  seed_bin[i] = b;
  atomicAdd(&counts[b], 1);
}

// Exclusive scan, three phases: per-block totals, a single-block scan of the
// totals, then per-block scans offset by the scanned totals.
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 2;  // elements per thread
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_inclusive_scan(int v, int *smem_warp) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) smem_warp[wid] = v;
  __syncthreads();
  if (wid == 0) {
    int w = lane < (blockDim.x >> 5) ? smem_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += t;
    }
    smem_warp[lane] = w;
  }
  __syncthreads();
  const int r = v + (wid > 0 ? smem_warp[wid - 1] : 0);
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const int *__restrict__ in, int n,
                                                            int *__restrict__ tile_sums) {
  __shared__ int sw[32];
  const long base = long(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) s += in[base + k];
  const int incl = block_inclusive_scan(s, sw);
  if (threadIdx.x == blockDim.x - 1) tile_sums[blockIdx.x] = incl;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(int *__restrict__ sums, int ntiles) {
  __shared__ int sw[32];
  __shared__ int chunk_total;
  int carry = 0;
  for (int base = 0; base < ntiles; base += kScanThreads) {
    const int i = base + threadIdx.x;
    const int v = i < ntiles ? sums[i] : 0;
    const int incl = block_inclusive_scan(v, sw);
    if (i < ntiles) sums[i] = carry + incl - v;  // exclusive
    if (threadIdx.x == blockDim.x - 1) chunk_total = incl;
    __syncthreads();
    carry += chunk_total;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const int *__restrict__ in, int n,
                                                            const int *__restrict__ tile_offsets,
                                                            int *__restrict__ out) {
  __shared__ int sw[32];
  const long base = long(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : 0;
    s += v[k];
  }
  const int incl = block_inclusive_scan(s, sw);
  int run = tile_offsets[blockIdx.x] + incl - s;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

__global__ void k_bin_scatter(int n, const int *__restrict__ seed_bin, int *__restrict__ cursor,
                              int *__restrict__ perm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  perm[atomicAdd(&cursor[seed_bin[i]], 1)] = i;
}

// Restores user-id order inside every bin (insertion sort; bins hold a few
// seeds, and their fill is bounded by kMaxBinFill before this runs).
__global__ void k_bin_sort(const int *__restrict__ counters, int nbins, int *__restrict__ perm) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbins) return;
  const int lo = counters[b], hi = counters[b + 1];
  for (int i = lo + 1; i < hi; ++i) {
    const int key = perm[i];
    int j = i - 1;
    while (j >= lo && perm[j] > key) {
      perm[j + 1] = perm[j];
      --j;
    }
    perm[j + 1] = key;
  }
}

__global__ void k_bin_gather(const float4 *__restrict__ user, const int *__restrict__ perm, int n,
                             float4 *__restrict__ stored, int *__restrict__ user_to_stored) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int u = perm[s];
  stored[s] = user[u];
  if (user_to_stored) user_to_stored[u] = s;
}

__global__ void k_max_reduce(const int *__restrict__ v, int n, int *__restrict__ out) {
  int m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, v[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(kFull, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

size_t scan_workspace_ints(int n) { return size_t((n + kScanTile - 1) / kScanTile) + 1; }

cudaError_t exclusive_scan(const int *in, int *out, int n, int *tile_ws, cudaStream_t st) {
  const int ntiles = (n + kScanTile - 1) / kScanTile;
  k_scan_tiles<<<ntiles, kScanThreads, 0, st>>>(in, n, tile_ws);
  k_scan_sums<<<1, kScanThreads, 0, st>>>(tile_ws, ntiles);
  k_scan_apply<<<ntiles, kScanThreads, 0, st>>>(in, n, tile_ws, out);
  return cudaGetLastError();
}

int bins_per_axis(int n) {
  const double d = std::round(std::pow(double(float(n) / 3.1f), double(1.0f / 3)));
  return d < 1 ? 1 : int(d);
}

size_t BinWorkspace::bytes(int n, int dim) {
  const size_t nb = size_t(dim) * dim * dim;
  return sizeof(int) * (size_t(n) + 2 * (nb + 1) + scan_workspace_ints(int(nb + 1)) + 4);
}

cudaError_t bin_seeds(const float4 *user, int n, int dim, BinWorkspace ws, BinOutputs out, cudaStream_t st,
                      int *max_fill_host) {
  const int nb = dim * dim * dim;
  cudaError_t e;
  if ((e = cudaMemsetAsync(ws.counts, 0, sizeof(int) * size_t(nb + 1), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(ws.max_fill, 0, 2 * sizeof(int), st)) != cudaSuccess) return e;
  const int tb = 256;
  k_bin_count<<<(n + tb - 1) / tb, tb, 0, st>>>(user, n, dim, ws.seed_bin, ws.counts, ws.max_fill + 1);
  k_max_reduce<<<148 * 4, 256, 0, st>>>(ws.counts, nb, ws.max_fill);
  if ((e = exclusive_scan(ws.counts, out.counters, nb + 1, ws.scan_tiles, st)) != cudaSuccess) return e;
  if (max_fill_host) {
    if ((e = cudaMemcpyAsync(max_fill_host, ws.max_fill, 2 * sizeof(int), cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
      return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    if (max_fill_host[0] > kMaxBinFill || max_fill_host[1]) return cudaSuccess;  // caller rejects the input
  }
  if ((e = cudaMemcpyAsync(ws.cursor, out.counters, sizeof(int) * size_t(nb), cudaMemcpyDeviceToDevice, st)) !=
      cudaSuccess)
    return e;
  k_bin_scatter<<<(n + tb - 1) / tb, tb, 0, st>>>(n, ws.seed_bin, ws.cursor, out.perm);
  k_bin_sort<<<(nb + tb - 1) / tb, tb, 0, st>>>(out.counters, nb, out.perm);
  k_bin_gather<<<(n + tb - 1) / tb, tb, 0, st>>>(user, out.perm, n, out.stored, out.user_to_stored);
  return cudaGetLastError();
}

}  // namespace rpd
