// Seed binning (counting sort into a dim^3 grid over [0,1000]^3).
#pragma once
#include <cmath>

#include "common.cuh"

namespace rpd {

// Largest bin fill accepted: denser inputs are rejected (RPD_ERR_DEGENERATE)
// instead of running the neighbour search in quadratic time.
constexpr int kMaxBinFill = 4096;

// Bin of a seed: clamp(floor(p * dim / 1000)) per axis, in IEEE float with
// the reference's operation order (knearests.cpp:35-46).
__host__ __device__ __forceinline__ int bin_of(float4 p, int dim) {
  const float fd = float(dim);
#ifdef __CUDA_ARCH__
  int i = int(floorf(__fdiv_rn(__fmul_rn(p.x, fd), 1000.f)));
  int j = int(floorf(__fdiv_rn(__fmul_rn(p.y, fd), 1000.f)));
  int k = int(floorf(__fdiv_rn(__fmul_rn(p.z, fd), 1000.f)));
#else
  int i = int(std::floor(p.x * fd / 1000.f));
  int j = int(std::floor(p.y * fd / 1000.f));
  int k = int(std::floor(p.z * fd / 1000.f));
#endif
  i = i < 0 ? 0 : (i > dim - 1 ? dim - 1 : i);
  j = j < 0 ? 0 : (j > dim - 1 ? dim - 1 : j);
  k = k < 0 ? 0 : (k > dim - 1 ? dim - 1 : k);
  return i + j * dim + k * dim * dim;
}

struct BinWorkspace {
  int *seed_bin;    // n
  int *counts;      // nb+1
  int *cursor;      // nb+1
  int *scan_tiles;  // scan_workspace_ints(nb+1)
  int *max_fill;    // 2: the largest bin fill, then a non-finite-seed flag
  static size_t bytes(int n, int dim);
};
struct BinOutputs {
  float4 *stored;       // n: seeds in stored order
  int *perm;            // n: stored -> user id
  int *counters;        // nb+1: exclusive prefix of bin counts
  int *user_to_stored;  // n (optional): user id -> stored
};

size_t scan_workspace_ints(int n);
cudaError_t exclusive_scan(const int *in, int *out, int n, int *tile_ws, cudaStream_t st);

// Bins `user` (device, n seeds).  When max_fill_host (2 ints) is given, the
// largest bin fill and a flag for a seed with a non-finite value are read
// back first and, above kMaxBinFill or with the flag set, nothing else runs.
cudaError_t bin_seeds(const float4 *user, int n, int dim, BinWorkspace ws, BinOutputs out, cudaStream_t st,
                      int *max_fill_host);

}  // namespace rpd
