// Warp-wide selection of 64-bit keys (one key per lane): bitonic sort and
// merge across the 32 lanes.  Keys (float distance bits << 32 | index)
// order candidates by distance with ties broken by index.
#pragma once
#include "common.cuh"

namespace rpd {

constexpr unsigned long long kEmptyKey = (0x7f800000ull << 32) | 0xffffffffull;

__device__ __forceinline__ unsigned long long umin64(unsigned long long a, unsigned long long b) {
  return a < b ? a : b;
}
__device__ __forceinline__ unsigned long long umax64(unsigned long long a, unsigned long long b) {
  return a < b ? b : a;
}

// Sorts a bitonic sequence held one key per lane into ascending lane order.
__device__ __forceinline__ unsigned long long bitonic_merge32(unsigned long long v, int lane) {
#pragma unroll
  for (int j = 16; j > 0; j >>= 1) {
    const unsigned long long o = __shfl_xor_sync(kFull, v, j);
    v = (lane & j) ? umax64(v, o) : umin64(v, o);
  }
  return v;
}

__device__ __forceinline__ unsigned long long bitonic_sort32(unsigned long long v, int lane) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const unsigned long long o = __shfl_xor_sync(kFull, v, j);
      const bool up = (lane & k) == 0;
      const bool lower = (lane & j) == 0;
      v = (lower == up) ? umin64(v, o) : umax64(v, o);
    }
  }
  return v;
}

}  // namespace rpd
