// Shared device/host definitions of the B200 restricted-power-diagram engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace rpd {

// Cell status codes, identical to the reference's Status enum (Status.h:4-16).
enum CellStatus : int {
  kVertexOverflow = 0,
  kPlaneOverflow = 1,
  kInconsistentBoundary = 2,
  kSecurityRadiusNotReached = 3,
  kSuccess = 4,
  kNeedsExactPredicates = 5,
  kEmptyCell = 6,
  kFindAnotherBeginningVertex = 7,
  kTriangleOverflow = 8,
  kSeedOnBorder = 9,
  kHessianOverflow = 10,
};
constexpr int kStatusNum = 11;
constexpr float kNoCellLimits = -100000.f;  // voronoi.h:53

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// Bins per axis of the seed grid: round((n / 3.1)^(1/3)) (knearests.cpp:63).
int bins_per_axis(int n);

// Floats as ints in the same order (atomicMax on float values): the sign
// bit flips the rest for negative values.
__host__ __device__ __forceinline__ int float_to_ordered(float f) {
  union { float f; int i; } u{f};
  return u.i >= 0 ? u.i : u.i ^ 0x7fffffff;
}
__host__ __device__ __forceinline__ float ordered_to_float(int i) {
  union { int i; float f; } u{i >= 0 ? i : i ^ 0x7fffffff};
  return u.f;
}

// Batched launches: diagram d owns rows start[d] .. start[d+1]; the owner of
// row r (0 <= r < start[ndiag]) is the last d with start[d] <= r, which
// skips diagrams without rows.
__device__ __forceinline__ int owner_of_row(const int *__restrict__ start, int ndiag, int r) {
  int lo = 0, hi = ndiag - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= r) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

}  // namespace rpd

#define RPD_CUDA_TRY(expr)                                   \
  do {                                                       \
    cudaError_t rpd_err_ = (expr);                           \
    if (rpd_err_ != cudaSuccess) return rpd::cuda_fail(rpd_err_, #expr, __FILE__, __LINE__); \
  } while (0)

namespace rpd {
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);
}
