// Engine state behind the C ABI: device context, resident seed sets.
#pragma once
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rpd.h"
#include "bins.cuh"
#include "cell.cuh"
#include "grid_host.h"
#include "knn.cuh"

namespace rpd {

// Owning device allocation that only grows.
// Device memory comes from the stream-ordered pool of the current device,
// through one allocation stream per device: allocating and freeing never
// synchronize the device, so solvers on other streams keep running (the
// serving loop depends on it).  A buffer is grown or released only when no
// work that uses it is pending: every entry point of the engine ends with a
// synchronization of its stream.
cudaError_t pool_alloc(void **p, size_t bytes);
void pool_free(void *p);

struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (ptr) pool_free(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  cudaError_t ensure(size_t want) {
    if (want <= bytes && ptr) return cudaSuccess;
    release();
    cudaError_t e = pool_alloc(&ptr, want ? want : 16);
    if (e == cudaSuccess) bytes = want ? want : 16;
    else ptr = nullptr;
    return e;
  }
  template <class T>
  T *as() const {
    return static_cast<T *>(ptr);
  }
};

void set_error(rpd_context *ctx, const std::string &msg);
int map_cuda(rpd_context *ctx, cudaError_t e, const char *what);
const HostGrid *host_grid(const rpd_grid *g);
rpd_grid *grid_handle(HostGrid &&g);

}  // namespace rpd

struct rpd_context {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  std::string error;
  // neighbour-search variant per K (rpd::KnnVariant), picked by a timed
  // trial on this device the first time K comes up; -1 not tried yet
  signed char knn_variant[257];
  rpd_context() { std::memset(knn_variant, -1, sizeof(knn_variant)); }
};

struct rpd_solver {
  rpd_context *ctx = nullptr;
  int n = 0;
  int dim = 0;
  rpd::DevBuf user;            // float4[n] as given
  rpd::DevBuf stored;          // float4[n] stored (binned) order
  rpd::DevBuf perm;            // int[n] stored -> user
  rpd::DevBuf user_to_stored;  // int[n]
  rpd::DevBuf weights;         // float[n]: staging for rpd_solver_set_weights
  rpd::DevBuf wmin;            // int[2]: the smallest weight of the seeds that are not walls
                               // (float_to_ordered); a flag of rpd_solver_set_weights
  rpd::DevBuf counters;        // int[dim^3+1]
  rpd::DevBuf bin_ws;
  rpd::DevBuf ring_bound;      // float[dim+2]
  rpd::DevBuf knn;             // unsigned[n*K]: every cell's neighbours (stored ids)
  int knn_full_K = 0;          // K of the table in knn for all n cells (0: none)
  int launches_since_points = 0;  // launches since the seeds were set (the outside probe runs on the first)
  long long grid_nonplain = -1;   // voxels of the grid that are not plainly outside (-1: not read yet)
  rpd::DevBuf knn_part;        // unsigned[num*K]: rows of a retry pass or a trace
  rpd::DevBuf knn_user;        // int[n*K]
  rpd::DevBuf counter64;       // unsigned long long[RPD_CTR_NUM + 1]
  // domain on the device
  rpd::DevBuf g_flags, g_points, g_tris, g_list, g_offsets, g_sat, g_tsat;
  rpd::DevGrid grid;           // grid.size == 0: no domain
  int grid_points = 0, grid_triangles = 0;  // of the domain's surface
  // results (stored order) and pass bookkeeping
  rpd::DevBuf out;             // double4[n]
  rpd::DevBuf status;          // int[n]
  rpd::DevBuf ids_a, ids_b, ids_c;  // int[n] failing-id lists
  rpd::DevBuf ids_range;       // int[count]: a part's stored ids (rpd_solver_launch_part)
  rpd::DevBuf tri_count;       // int[n]: triangle counts of the triangle overflows (CellLaunch::tri_count)
  rpd::DevBuf fail_ws;         // flags + scans
  rpd::DevBuf hist;            // int[16]: status histogram + counts
  rpd::DevBuf gather;          // user-order staging for outputs
  rpd::DevBuf defer_slots, defer_part, defer_fail, defer_ctr, defer_chunk_slot;  // parked boundary cells
  int ahead_max = 0;           // the largest triangle count the first pass parked ahead
  bool have_results = false;
  bool use_defer = true;       // park heavy boundary cells for the chunked kernel
  bool inner_apex = true;      // cone apex at a grid corner inside the cell
  bool fresh_knn = false;      // recompute the neighbour table at this launch
  int precision = 0;           // RPD_PRECISION_* of the clipping loop
  unsigned launch_flags = 0;   // RPD_FLAG_* of the current launch
  // used cells (keep_distance >= 0 with a domain)
  rpd::DevBuf used;            // unsigned char[n], stored order: 0 or the ring distance
  bool used_on = false;
  int keep_distance = -1;
  double keep_volume = 0.0;
  int used_count = -1;         // of the last launch, -1: none
  // --hessian rows (stored order) of the last launch with hessian_h > 0
  rpd::DevBuf hess;            // double[n*H*HC]
  rpd::DevBuf hessid;          // int[n*H]: stored ids, -1 after a row's last facet
  int hess_h = 0, hess_hc = 1; // of the last launch (0: no rows)
  rpd_stats stats{};
};

namespace rpd {
// Hooks of the serving loop (csrc/server.cu).
void solver_rebind(rpd_solver *s, rpd_context *ctx);
void solver_share_grid(rpd_solver *dst, const rpd_solver *src);
size_t solver_device_bytes(const rpd_solver *s);
void solver_trim(rpd_solver *s);
// The T of the last retry pass that surely runs after a cell's triangle
// overflow: passes grow T x1.5 while the cell fails, up to max_extra, and
// stop once P or K (assumed to grow in every pass) outgrow their limits
// (voronoi.cpp:867); 0 when no retry surely runs.
int t_ahead_cap(int P, int K, int T, int max_extra);

}  // namespace rpd
