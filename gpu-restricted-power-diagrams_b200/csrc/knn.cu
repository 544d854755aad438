// K-nearest neighbours on the binned seeds, one warp per seed (replaces the
// reference's one-work-item heap search, knearests.cl:36-78).
//
// The warp scans Chebyshev shells of bins around the seed's bin.  Bins are
// stored x-fastest, so every row of a shell is one contiguous range of the
// stored seeds: the lanes enumerate the rows, prefix-sum their point counts
// and then take 32 candidates per round with coalesced float4 loads.
// Candidates closer than the current K-th best are staged in a 32-entry
// shared-memory buffer per warp; a full stage is bitonic-sorted across the
// warp and merged into
// the K-best list (32*S keys, S per lane, sorted lane-major) by S bitonic
// merges.  Keys are (float distance bits << 32 | stored index): ties break
// by index.  A shell is skipped once the K-th best is closer than the
// shell's bound ((shell-1) * bin width)^2, checked at shell granularity
// after every pending candidate is merged -- the exact rule of the oracle's
// exact mode, so lists agree bit for bit.
#include <algorithm>

#include "knn.cuh"
#include "select.cuh"

namespace rpd {

namespace {

// Merges 32 staged keys into the sorted list best[0..S) (slot s holds ranks
// s*32 .. s*32+31).  Keeps the 32*S smallest.
template <int S>
__device__ __forceinline__ void merge_stage(unsigned long long (&best)[S], unsigned long long stage, int lane) {
  unsigned long long low = bitonic_sort32(stage, lane);
#pragma unroll
  for (int s = S - 1; s >= 0; --s) {
    const unsigned long long rev = __shfl_sync(kFull, low, 31 - lane);
    const unsigned long long lo = umin64(best[s], rev);
    const unsigned long long hi = umax64(best[s], rev);
    if (s + 1 < S) best[s + 1] = bitonic_merge32(hi, lane);
    low = bitonic_merge32(lo, lane);
  }
  best[0] = low;
}

template <int S>
__device__ __forceinline__ unsigned long long key_at(const unsigned long long (&best)[S], int pos) {
  const int slot = pos >> 5, src = pos & 31;
  unsigned long long v = kEmptyKey;
#pragma unroll
  for (int s = 0; s < S; ++s)
    if (s == slot) v = best[s];
  return __shfl_sync(kFull, v, src);
}

// Row ranges of shell `ring` (rings 0 and 1 are scanned together as the
// 3x3x3 block, "ring 0").  Row q of the shell covers bins (x, cy+j, cz+k):
// the whole x span on the shell's faces, else the two end bins.
struct ShellRows {
  int cx, cy, cz, dim, ring;
  __device__ __forceinline__ int rows() const {
    const int w = 2 * (ring == 0 ? 1 : ring) + 1;
    return w * w;
  }
  // Point ranges [a0, a0+l0) and [a1, a1+l1) of row q.
  __device__ __forceinline__ void ranges(int q, const int *__restrict__ counters, int &a0, int &l0, int &a1,
                                         int &l1) const {
    const int r = ring == 0 ? 1 : ring;
    const int w = 2 * r + 1;
    const int j = q % w - r, k = q / w - r;
    a0 = l0 = a1 = l1 = 0;
    const int y = cy + j, z = cz + k;
    if (y < 0 || y >= dim || z < 0 || z >= dim) return;
    const int rowbase = (y + z * dim) * dim;
    const bool face = ring == 0 || j == -r || j == r || k == -r || k == r;
    if (face) {
      const int x0 = max(cx - r, 0), x1 = min(cx + r, dim - 1);
      a0 = __ldg(&counters[rowbase + x0]);
      l0 = __ldg(&counters[rowbase + x1 + 1]) - a0;
    } else {
      if (cx - r >= 0) {
        a0 = __ldg(&counters[rowbase + cx - r]);
        l0 = __ldg(&counters[rowbase + cx - r + 1]) - a0;
      }
      if (cx + r < dim) {
        a1 = __ldg(&counters[rowbase + cx + r]);
        l1 = __ldg(&counters[rowbase + cx + r + 1]) - a1;
      }
    }
  }
};

// The K nearest of stored seed `pin` into row[0..K) (one warp).
template <int S>
__device__ __forceinline__ void knn_row(const float4 *__restrict__ stored, const int *__restrict__ counters, int dim,
                                        int pin, int K, const float *__restrict__ ring_bound, unsigned *__restrict__ row,
                                        unsigned long long *__restrict__ candidates, unsigned long long *stage,
                                        int lane) {
  const float4 p = stored[pin];
  const int cin = bin_of(p, dim);
  ShellRows sh;
  sh.cx = cin % dim;
  sh.cy = (cin / dim) % dim;
  sh.cz = cin / (dim * dim);
  sh.dim = dim;

  unsigned long long best[S];
#pragma unroll
  for (int s = 0; s < S; ++s) best[s] = kEmptyKey;
  int nstage = 0;
  unsigned long long kth = kEmptyKey;
  unsigned long long ncand = 0;

  for (int ring = 0; ring <= dim; ring = ring == 0 ? 2 : ring + 1) {
    if (ring >= 2) {
      // whole-shell exit: the K-th best beats the shell bound
      const float kd = __uint_as_float(unsigned(kth >> 32));
      if (kd < ring_bound[ring]) break;
      if (sh.cx - ring < 0 && sh.cy - ring < 0 && sh.cz - ring < 0 && sh.cx + ring >= dim &&
          sh.cy + ring >= dim && sh.cz + ring >= dim)
        break;  // the shell lies outside the grid
    }
    sh.ring = ring;
    const int nrows = sh.rows();
    for (int q0 = 0; q0 < nrows; q0 += 32) {
      int a0 = 0, l0 = 0, a1 = 0, l1 = 0;
      if (q0 + lane < nrows) sh.ranges(q0 + lane, counters, a0, l0, a1, l1);
      const int cnt = l0 + l1;
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
      }
      const int total = __shfl_sync(kFull, incl, 31);
      for (int base = 0; base < total; base += 32) {
        const int c = base + lane;
        // owner lane: the first lane whose inclusive count exceeds c
        int lo = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int v = __shfl_sync(kFull, incl, lo + step - 1);
          if (v <= c) lo += step;
        }
        const int owner = lo;
        const int o_incl = __shfl_sync(kFull, incl, owner);
        const int o_cnt = __shfl_sync(kFull, cnt, owner);
        const int o_a0 = __shfl_sync(kFull, a0, owner);
        const int o_l0 = __shfl_sync(kFull, l0, owner);
        const int o_a1 = __shfl_sync(kFull, a1, owner);
        unsigned long long key = kEmptyKey;
        if (c < total) {
          const int off = c - (o_incl - o_cnt);
          const int ptr = off < o_l0 ? o_a0 + off : o_a1 + (off - o_l0);
          if (ptr != pin) {
            const float4 qv = __ldg(&stored[ptr]);
            const float dx = __fsub_rn(qv.x, p.x), dy = __fsub_rn(qv.y, p.y), dz = __fsub_rn(qv.z, p.z);
            const float d = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
            key = (static_cast<unsigned long long>(__float_as_uint(d)) << 32) | unsigned(ptr);
            ++ncand;
          }
        }
        const bool accept = key < kth;
        const unsigned m = __ballot_sync(kFull, accept);
        const int nacc = __popc(m);
        if (nacc == 0) continue;
        if (nstage + nacc > 32) {
          __syncwarp();
          const unsigned long long v = lane < nstage ? stage[lane] : kEmptyKey;
          __syncwarp();
          merge_stage<S>(best, v, lane);
          nstage = 0;
          kth = key_at<S>(best, K - 1);
        }
        if (accept) stage[nstage + __popc(m & ((1u << lane) - 1u))] = key;
        nstage += nacc;
      }
    }
    if (nstage) {
      __syncwarp();
      const unsigned long long v = lane < nstage ? stage[lane] : kEmptyKey;
      __syncwarp();
      merge_stage<S>(best, v, lane);
      nstage = 0;
      kth = key_at<S>(best, K - 1);
    }
  }
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int pos = s * 32 + lane;
    if (pos < K) row[pos] = unsigned(best[s] & 0xffffffffull);
  }
  if (candidates) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ncand += __shfl_xor_sync(kFull, ncand, o);
    if (lane == 0) atomicAdd(candidates, ncand);
  }
}

template <int S>
__global__ void __launch_bounds__(256) k_knn(const float4 *__restrict__ stored, const int *__restrict__ counters,
                                             int dim, const int *__restrict__ ids, int num, int K,
                                             const float *__restrict__ ring_bound, unsigned *__restrict__ out,
                                             unsigned long long *__restrict__ candidates) {
  __shared__ unsigned long long stage_buf[kKnnThreads / 32][32];
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= num) return;  // warp-uniform
  const int pin = ids ? ids[w] : w;
  knn_row<S>(stored, counters, dim, pin, K, ring_bound, out + size_t(w) * K, candidates, stage_buf[threadIdx.x >> 5],
             lane);
}

// ---- one thread per seed ----
//
// The same search with one seed per thread: the thread walks its shells row
// by row and keeps its K best keys in a max-heap in shared memory (root = the
// K-th best so far; a closer candidate replaces the root and sifts down),
// then heap-sorts them.  Far fewer instructions per seed than the warp's
// merges for small K; the keys, the shells scanned and so the lists are the
// same bit for bit.  Threads of a warp take consecutive stored seeds, whose
// shells overlap, so their candidate loads hit L1.  The heap of thread t is
// heap[i * kHeapStride + t], i < K: every thread owns one bank pair, and the
// coalesced output pass (a warp per row, lanes over i) is conflict-free.
constexpr int kThreadRows = 128;                 // seeds (threads) per block
constexpr int kHeapStride = kThreadRows + 1;

struct Heap {
  unsigned long long *h;  // h[i * kHeapStride]
  __device__ __forceinline__ unsigned long long &at(int i) const { return h[i * kHeapStride]; }
  // key into a heap of n < K keys (grows by one)
  __device__ __forceinline__ void push(int n, unsigned long long key) const {
    int i = n;
    while (i > 0) {
      const int parent = (i - 1) >> 1;
      const unsigned long long kp = at(parent);
      if (kp >= key) break;
      at(i) = kp;
      i = parent;
    }
    at(i) = key;
  }
  // key into the root's place of a heap of n keys, sifted down
  __device__ __forceinline__ void replace_root(int n, unsigned long long key) const {
    int i = 0;
    for (;;) {
      const int l = 2 * i + 1;
      if (l >= n) break;
      int c = l;
      unsigned long long kc = at(l);
      if (l + 1 < n) {
        const unsigned long long kr = at(l + 1);
        if (kr > kc) {
          c = l + 1;
          kc = kr;
        }
      }
      if (kc <= key) break;
      at(i) = kc;
      i = c;
    }
    at(i) = key;
  }
};

// The K nearest of stored seed pin into the heap of this thread, sorted
// ascending and padded with kEmptyKey to K; returns the candidates read.
__device__ __forceinline__ unsigned long long knn_thread_row(const float4 *__restrict__ stored,
                                                             const int *__restrict__ counters, int dim, int pin,
                                                             int K, const float *__restrict__ ring_bound,
                                                             const Heap &H) {
  unsigned long long ncand = 0;
  {
    const float4 p = __ldg(&stored[pin]);
    const int cin = bin_of(p, dim);
    ShellRows sh;
    sh.cx = cin % dim;
    sh.cy = (cin / dim) % dim;
    sh.cz = cin / (dim * dim);
    sh.dim = dim;
    int n = 0;
    unsigned long long root = kEmptyKey;  // the K-th best once the heap is full
    for (int ring = 0; ring <= dim; ring = ring == 0 ? 2 : ring + 1) {
      if (ring >= 2) {
        // whole-shell exit: the K-th best beats the shell bound
        const float kd = __uint_as_float(unsigned(root >> 32));
        if (kd < __ldg(&ring_bound[ring])) break;
        if (sh.cx - ring < 0 && sh.cy - ring < 0 && sh.cz - ring < 0 && sh.cx + ring >= dim &&
            sh.cy + ring >= dim && sh.cz + ring >= dim)
          break;  // the shell lies outside the grid
      }
      sh.ring = ring;
      const int nrows = sh.rows();
      for (int q = 0; q < nrows; ++q) {
        int a[2], l[2];
        sh.ranges(q, counters, a[0], l[0], a[1], l[1]);
#pragma unroll
        for (int part = 0; part < 2; ++part) {
          for (int ptr = a[part], end = a[part] + l[part]; ptr < end; ++ptr) {
            if (ptr == pin) continue;
            const float4 qv = __ldg(&stored[ptr]);
            const float dx = __fsub_rn(qv.x, p.x), dy = __fsub_rn(qv.y, p.y), dz = __fsub_rn(qv.z, p.z);
            const float d = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
            const unsigned long long key = (static_cast<unsigned long long>(__float_as_uint(d)) << 32) | unsigned(ptr);
            ++ncand;
            if (n < K) {
              H.push(n, key);
              ++n;
              if (n == K) root = H.at(0);
            } else if (key < root) {
              H.replace_root(K, key);
              root = H.at(0);
            }
          }
        }
      }
    }
    // ascending order: the root (largest) to the back, one by one
    for (int end = n - 1; end > 0; --end) {
      const unsigned long long last = H.at(end);
      H.at(end) = H.at(0);
      H.replace_root(end, last);
    }
    for (int i = n; i < K; ++i) H.at(i) = kEmptyKey;
  }
  return ncand;
}

__global__ void __launch_bounds__(kThreadRows) k_knn_thread(const float4 *__restrict__ stored,
                                                           const int *__restrict__ counters, int dim,
                                                           const int *__restrict__ ids, int num, int K,
                                                           const float *__restrict__ ring_bound,
                                                           unsigned *__restrict__ out,
                                                           unsigned long long *__restrict__ candidates) {
  extern __shared__ unsigned long long heap_smem[];
  const int t = threadIdx.x;
  const int row0 = blockIdx.x * kThreadRows;
  const int row = row0 + t;
  const Heap H{heap_smem + t};
  unsigned long long ncand = 0;
  if (row < num) ncand = knn_thread_row(stored, counters, dim, ids ? __ldg(&ids[row]) : row, K, ring_bound, H);
  __syncthreads();
  // coalesced rows: a warp per row, lanes over the row's entries
  const int lane = t & 31, warp = t >> 5;
  const int rows_here = min(kThreadRows, num - row0);
  for (int r = warp; r < rows_here; r += kThreadRows / 32) {
    unsigned *o = out + size_t(row0 + r) * K;
    for (int i = lane; i < K; i += 32) o[i] = unsigned(heap_smem[i * kHeapStride + r] & 0xffffffffull);
  }
  if (candidates) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ncand += __shfl_xor_sync(kFull, ncand, o);
    if (lane == 0) atomicAdd(candidates, ncand);
  }
}

// Rows of many diagrams (batched solves) with a thread per seed: the
// diagrams of one slot class own rows start[d] .. start[d+1]; threads stride
// over them, each writing its own row (K of its diagram, at most kmax).
__global__ void __launch_bounds__(kThreadRows) k_knn_thread_batch(const KnnDiag *__restrict__ diags,
                                                                 const int *__restrict__ start, int ndiag) {
  extern __shared__ unsigned long long heap_smem[];
  const Heap H{heap_smem + threadIdx.x};
  const int total = start[ndiag];
  const int nthreads = gridDim.x * blockDim.x;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < total; r += nthreads) {
    const int d = owner_of_row(start, ndiag, r);
    const KnnDiag &g = diags[d];
    const int i = r - start[d];
    knn_thread_row(g.stored, g.counters, g.dim, g.ids ? g.ids[i] : i, g.K, g.ring_bound, H);
    unsigned *o = g.out + size_t(i) * g.K;
    for (int k = 0; k < g.K; ++k) o[k] = unsigned(H.at(k) & 0xffffffffull);
  }
}

// Rows of many diagrams (batched solves): the diagrams of slot class S own
// rows start[d] .. start[d+1] of this launch; warps stride over them.
template <int S>
__global__ void __launch_bounds__(256) k_knn_batch(const KnnDiag *__restrict__ diags, const int *__restrict__ start,
                                                   int ndiag) {
  __shared__ unsigned long long stage_buf[kKnnThreads / 32][32];
  const int lane = threadIdx.x & 31;
  const int total = start[ndiag];
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < total; r += nwarps) {
    const int d = owner_of_row(start, ndiag, r);
    const KnnDiag &g = diags[d];
    const int i = r - start[d];
    const int pin = g.ids ? g.ids[i] : i;
    knn_row<S>(g.stored, g.counters, g.dim, pin, g.K, g.ring_bound, g.out + size_t(i) * g.K, nullptr,
               stage_buf[threadIdx.x >> 5], lane);
  }
}

}  // namespace

int knn_slots(int K) {
  const int s = (K + 31) / 32;
  if (s <= 1) return 1;
  if (s <= 2) return 2;
  if (s <= 3) return 3;
  if (s <= 4) return 4;
  if (s <= 6) return 6;
  if (s <= 8) return 8;
  return -1;
}

void ring_bounds(int dim, float *bound) {
  // ((ring-1) * 1000/dim)^2 in float, ring 0 -> 0 (knearests.cpp:84-86).
  for (int ring = 0; ring <= dim + 1; ++ring) {
    if (ring == 0) {
      bound[ring] = 0.f;
      continue;
    }
    const float d = 1000.f * float(ring - 1) / float(dim);
    bound[ring] = d * d;
  }
}

cudaError_t knn_batch_launch(int S, const KnnDiag *diags, const int *start, int ndiag, int blocks, cudaStream_t st,
                             long rows, int variant) {
  if (variant == kKnnThread) {
    // a thread per row, the heap sized for the class's largest K (32 S)
    if (32 * S > kKnnThreadMaxK) return cudaErrorInvalidValue;
    const size_t smem = sizeof(unsigned long long) * size_t(32 * S) * kHeapStride;
    cudaError_t e = cudaFuncSetAttribute(k_knn_thread_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(sizeof(unsigned long long) * kKnnThreadMaxK * kHeapStride));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_knn_thread_batch, kThreadRows, smem) !=
            cudaSuccess || per_sm < 1)
      per_sm = 1;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int tb = per_sm * sms;
    if (rows >= 0) tb = int(std::min<long>(tb, (rows + kThreadRows - 1) / kThreadRows + 1));
    k_knn_thread_batch<<<tb, kThreadRows, smem, st>>>(diags, start, ndiag);
    return cudaGetLastError();
  }
  if (rows >= 0) blocks = int(rows * 32 / kKnnThreads + 1);
  switch (S) {
    case 1: k_knn_batch<1><<<blocks, kKnnThreads, 0, st>>>(diags, start, ndiag); break;
    case 2: k_knn_batch<2><<<blocks, kKnnThreads, 0, st>>>(diags, start, ndiag); break;
    case 3: k_knn_batch<3><<<blocks, kKnnThreads, 0, st>>>(diags, start, ndiag); break;
    case 4: k_knn_batch<4><<<blocks, kKnnThreads, 0, st>>>(diags, start, ndiag); break;
    case 6: k_knn_batch<6><<<blocks, kKnnThreads, 0, st>>>(diags, start, ndiag); break;
    case 8: k_knn_batch<8><<<blocks, kKnnThreads, 0, st>>>(diags, start, ndiag); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t knn_launch(const float4 *stored, const int *counters, int dim, const int *ids, int num, int K,
                       const float *ring_bound, unsigned *out, unsigned long long *candidates, cudaStream_t st,
                       int variant) {
  if (num <= 0) return cudaSuccess;
  if (variant == kKnnThread) {
    if (K < 1 || K > kKnnThreadMaxK) return cudaErrorInvalidValue;
    const size_t smem = sizeof(unsigned long long) * size_t(K) * kHeapStride;
    // the dynamic shared memory limit of the current device (a cheap host call)
    cudaError_t e = cudaFuncSetAttribute(k_knn_thread, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(sizeof(unsigned long long) * kKnnThreadMaxK * kHeapStride));
    if (e != cudaSuccess) return e;
    const int blocks = (num + kThreadRows - 1) / kThreadRows;
    k_knn_thread<<<blocks, kThreadRows, smem, st>>>(stored, counters, dim, ids, num, K, ring_bound, out, candidates);
    return cudaGetLastError();
  }
  const int threads = kKnnThreads;
  const long warps = num;
  const int blocks = int((warps * 32 + threads - 1) / threads);
  switch (knn_slots(K)) {
    case 1: k_knn<1><<<blocks, threads, 0, st>>>(stored, counters, dim, ids, num, K, ring_bound, out, candidates); break;
    case 2: k_knn<2><<<blocks, threads, 0, st>>>(stored, counters, dim, ids, num, K, ring_bound, out, candidates); break;
    case 3: k_knn<3><<<blocks, threads, 0, st>>>(stored, counters, dim, ids, num, K, ring_bound, out, candidates); break;
    case 4: k_knn<4><<<blocks, threads, 0, st>>>(stored, counters, dim, ids, num, K, ring_bound, out, candidates); break;
    case 6: k_knn<6><<<blocks, threads, 0, st>>>(stored, counters, dim, ids, num, K, ring_bound, out, candidates); break;
    case 8: k_knn<8><<<blocks, threads, 0, st>>>(stored, counters, dim, ids, num, K, ring_bound, out, candidates); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace rpd
