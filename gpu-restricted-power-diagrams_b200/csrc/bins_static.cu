// Seed binning for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code that runs inside another
// framework's memory pool or arena, inside a plugin whose host forbids
// allocation after start-up, or on a path that must not synchronize the
// device the way cudaMalloc/cudaFree can.  For them, rpd_bin_seeds_noalloc
// bins seeds that are already on the device into buffers the caller owns,
// and keeps its own scratch (bin of every seed, bin counts, insertion
// cursors, scan partials) in one fixed-size array in the library's static
// device memory instead of allocating it.  The array holds enough for
// RPD_NOALLOC_MAX_SEEDS seeds; every GPU that loads the library keeps it
// (about 1.7 MB) until the process exits.
#include "../../include/rpd.h"
#include "bins.cuh"

namespace rpd {

namespace {

// Largest bin grid: dim = round((n / 3.1)^(1/3)) grows with n.
constexpr int kStaticDim = 44;  // bins_per_axis(RPD_NOALLOC_MAX_SEEDS)
constexpr int kStaticBins = kStaticDim * kStaticDim * kStaticDim;
constexpr int kStaticScanInts = (kStaticBins + 1 + 2047) / 2048 + 1;
constexpr int kStaticMaxFill = 8;  // room of the max-fill word (+ padding)
constexpr size_t kStaticScratchInts =
    size_t(RPD_NOALLOC_MAX_SEEDS) + 2 * size_t(kStaticBins + 1) + kStaticScanInts + kStaticMaxFill;

// The scratch of every call, on every device that loads the library.  In
// host code this name is only a host-side stand-in: kernels get the device
// address from cudaGetSymbolAddress.
static __device__ __align__(256) int g_bin_scratch[kStaticScratchInts];

// Device address of g_bin_scratch on the current device, looked up on every
// call (cheap once the module is loaded), so a device reset by the host
// application between calls never leaves a stale address behind.
cudaError_t scratch_address(int **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_bin_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<int *>(p);
  return cudaSuccess;
}

}  // namespace

}  // namespace rpd

extern "C" int rpd_bin_seeds_noalloc(const float *xyzw, int n, float *stored, int *perm, int *counters,
                                     int counters_cap, int *dim_out, void *stream) {
  using namespace rpd;
  if (!xyzw || !stored || !perm || !counters || n <= 0) return RPD_ERR_INVALID;
  if (n > RPD_NOALLOC_MAX_SEEDS) return RPD_ERR_CAPACITY;
  if ((reinterpret_cast<uintptr_t>(xyzw) | reinterpret_cast<uintptr_t>(stored)) & 15u) return RPD_ERR_INVALID;
  const int dim = bins_per_axis(n);
  const int nb = dim * dim * dim;
  if (dim_out) *dim_out = dim;
  if (dim > kStaticDim) return RPD_ERR_CAPACITY;
  if (counters_cap < nb + 1) return RPD_ERR_INVALID;
  int *scratch = nullptr;
  if (scratch_address(&scratch) != cudaSuccess) return RPD_ERR_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  BinWorkspace ws;
  ws.seed_bin = scratch;
  ws.counts = ws.seed_bin + RPD_NOALLOC_MAX_SEEDS;
  ws.cursor = ws.counts + (kStaticBins + 1);
  ws.scan_tiles = ws.cursor + (kStaticBins + 1);
  ws.max_fill = ws.scan_tiles + kStaticScanInts;
  BinOutputs out{reinterpret_cast<float4 *>(stored), perm, counters, nullptr};
  // bin_seeds clears the counts and the max-fill word it accumulates into;
  // the rest of the scratch is fully overwritten before it is read
  int fill[2] = {0, 0};  // the largest bin fill, a non-finite seed
  cudaError_t e = bin_seeds(reinterpret_cast<const float4 *>(xyzw), n, dim, ws, out, st, fill);
  if (e != cudaSuccess) return RPD_ERR_CUDA;
  if (fill[1]) return RPD_ERR_INVALID;
  if (fill[0] > kMaxBinFill) return RPD_ERR_DEGENERATE;
  if (cudaStreamSynchronize(st) != cudaSuccess) return RPD_ERR_CUDA;
  return RPD_OK;
}
