// Host side of the engine: context, seed binning and neighbour queries
// behind the C ABI declared in include/rpd.h.
#include <cstdio>
#include <cstring>
#include <string>

#include "engine.cuh"

namespace rpd {

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

}  // namespace rpd

using namespace rpd;

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

void rpd_solver_destroy(rpd_solver *s) {
  if (!s) return;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  delete s;
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
  int max_fill = 0;
  if ((e = bin_seeds(s->user.as<float4>(), n, dim, ws, out, st, &max_fill)) != cudaSuccess)
    return map_cuda(ctx, e, "bin seeds");
  if (max_fill > kMaxBinFill) {
    set_error(ctx, "seeds too clustered: " + std::to_string(max_fill) + " in one bin (limit " +
                       std::to_string(kMaxBinFill) + ")");
    s->n = 0;
    return RPD_ERR_DEGENERATE;
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "bin seeds");
  s->n = n;
  s->dim = dim;
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
  cudaEvent_t ev[2];
  cudaEventCreate(&ev[0]);
  cudaEventCreate(&ev[1]);
  cudaEventRecord(ev[0], st);
  e = knn_launch(s->stored.as<float4>(), s->counters.as<int>(), s->dim, nullptr, s->n, K, s->ring_bound.as<float>(),
                 s->knn.as<unsigned>(), nullptr, st);
  cudaEventRecord(ev[1], st);
  if (e != cudaSuccess) return map_cuda(ctx, e, "knn");
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
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  return RPD_OK;
}

}  // extern "C"
