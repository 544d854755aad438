// Domain grids built on the device: an implicit function sampled on the
// voxel-corner lattice becomes a solver's domain -- corner flags, the
// marching-Kuhn-tetrahedra surface, per-voxel triangle lists and the summed
// tables the cell kernel reads -- without host preprocessing (the serving
// loop's requests with new domains).  The surface is the one
// make_ellipsoid_blob builds on the host (csrc/grid_host.cpp): same corner
// values, the same triangles in the same order in every voxel, the same
// vertex coordinates.  Only the numbering of the surface vertices differs:
// here a crossed lattice edge's vertex is numbered by (lattice point, edge
// direction), where the host numbers vertices by first use.
//
// The arithmetic that decides the surface is written with explicitly
// rounded operations (no contraction into fused multiply-adds), in the host
// code's order, so the device and the host agree bit for bit.
#include <algorithm>
#include <vector>

#include "engine.cuh"

namespace rpd {
namespace grid_detail {

__device__ __forceinline__ size_t lat(int i, int j, int k, int S1) {
  return size_t(i) + size_t(j) * S1 + size_t(k) * S1 * S1;
}

// The ellipsoid union of make_ellipsoid_blob at lattice point idx: +1 on
// the lattice's outer layer, else min over ellipsoids of (|R (p - c) / a|^2
// - 1), never exactly 0.
__global__ void k_blob_field(const double *__restrict__ c, const double *__restrict__ ax,
                             const double *__restrict__ rot, int nell, int S, float *__restrict__ f) {
  const int S1 = S + 1;
  const long n = long(S1) * S1 * S1;
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
    const int i = int(idx % S1), j = int((idx / S1) % S1), k = int(idx / (long(S1) * S1));
    double v = 1.0;
    if (i > 0 && j > 0 && k > 0 && i < S && j < S && k < S) {
      const double p[3] = {__ddiv_rn(double(i), double(S)), __ddiv_rn(double(j), double(S)),
                           __ddiv_rn(double(k), double(S))};
      for (int e = 0; e < nell; ++e) {
        const double d[3] = {__dsub_rn(p[0], c[3 * e]), __dsub_rn(p[1], c[3 * e + 1]), __dsub_rn(p[2], c[3 * e + 2])};
        double q = 0.0;
        for (int r = 0; r < 3; ++r) {
          const double *R = rot + 9 * e + 3 * r;
          const double t =
              __dadd_rn(__dadd_rn(__dmul_rn(R[0], d[0]), __dmul_rn(R[1], d[1])), __dmul_rn(R[2], d[2]));
          const double u = __ddiv_rn(t, ax[3 * e + r]);
          q = __dadd_rn(q, __dmul_rn(u, u));
        }
        const double w = __dsub_rn(q, 1.0);
        v = w < v ? w : v;
      }
      if (v == 0.0) v = 1e-12;  // the surface never passes through a corner
    }
    f[idx] = __double2float_rn(v);
  }
}

// A user's field: the outer layer is set outside, so the surface closes
// inside the grid.
__global__ void k_field_outer_layer(int S, float *__restrict__ f) {
  const int S1 = S + 1;
  const long n = long(S1) * S1 * S1;
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
    const int i = int(idx % S1), j = int((idx / S1) % S1), k = int(idx / (long(S1) * S1));
    if (i == 0 || j == 0 || k == 0 || i == S || j == S || k == S) f[idx] = 1.0f;
  }
}

// Per lattice point: a bit for each crossed edge towards a + bits(code),
// code 1..7 (x = bit 0, y = bit 1, z = bit 2), and their count.
__global__ void k_edge_masks(const float *__restrict__ f, int S, unsigned char *__restrict__ mask,
                             int *__restrict__ cnt) {
  const int S1 = S + 1;
  const long n = long(S1) * S1 * S1;
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
    const int i = int(idx % S1), j = int((idx / S1) % S1), k = int(idx / (long(S1) * S1));
    const bool in = f[idx] < 0.f;
    unsigned m = 0;
    for (int code = 1; code < 8; ++code) {
      const int b0 = i + (code & 1), b1 = j + ((code >> 1) & 1), b2 = k + (code >> 2);
      if (b0 > S || b1 > S || b2 > S) continue;
      if ((f[lat(b0, b1, b2, S1)] < 0.f) != in) m |= 1u << code;
    }
    mask[idx] = (unsigned char)m;
    cnt[idx] = __popc(m);
  }
}

// Crossed-edge vertices (make_ellipsoid_blob's edge_vertex): t = fa / (fa -
// fb) clamped to [0.1, 0.9], position (a + t (b - a)) h.
__global__ void k_edge_points(const float *__restrict__ f, int S, float h, const unsigned char *__restrict__ mask,
                              const int *__restrict__ base, float4 *__restrict__ pts) {
  const int S1 = S + 1;
  const long n = long(S1) * S1 * S1;
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
    const unsigned m = mask[idx];
    if (!m) continue;
    const int a[3] = {int(idx % S1), int((idx / S1) % S1), int(idx / (long(S1) * S1))};
    int id = base[idx];
    for (int code = 1; code < 8; ++code) {
      if (!((m >> code) & 1u)) continue;
      const int b[3] = {a[0] + (code & 1), a[1] + ((code >> 1) & 1), a[2] + (code >> 2)};
      const double fa = f[idx], fb = f[lat(b[0], b[1], b[2], S1)];
      double t = __ddiv_rn(fa, __dsub_rn(fa, fb));
      t = fmin(0.9, fmax(0.1, t));
      float p[3];
      for (int d = 0; d < 3; ++d)
        p[d] = __double2float_rn(
            __dmul_rn(__dadd_rn(double(a[d]), __dmul_rn(t, double(b[d] - a[d]))), double(h)));
      pts[id++] = make_float4(p[0], p[1], p[2], 0.f);
    }
  }
}

__device__ __forceinline__ int edge_id(const unsigned char *mask, const int *base, int S1, const int *a,
                                       const int *b) {
  const size_t p = lat(a[0], a[1], a[2], S1);
  const int code = (b[0] - a[0]) | ((b[1] - a[1]) << 1) | ((b[2] - a[2]) << 2);
  return base[p] + __popc(unsigned(mask[p]) & ((1u << code) - 1u));
}

__constant__ int kPerm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

// One voxel: its corner flag, and its triangles (count only when tris is
// null), in make_ellipsoid_blob's order: the six Kuhn tetrahedra in
// permutation order, one triangle for a lone corner, two for a quad split
// along its shorter diagonal, each oriented from the inside corners'
// centroid towards the outside ones'.
__global__ void k_voxel_surface(const float *__restrict__ f, int S, signed char *__restrict__ flags,
                                int *__restrict__ count, const unsigned char *__restrict__ mask,
                                const int *__restrict__ base, const float4 *__restrict__ pts,
                                const int *__restrict__ offsets, int *__restrict__ tris, int *__restrict__ list) {
  const int S1 = S + 1;
  const long n = long(S) * S * S;
  for (long vid = blockIdx.x * long(blockDim.x) + threadIdx.x; vid < n; vid += long(gridDim.x) * blockDim.x) {
    const int i = int(vid % S), j = int((vid / S) % S), k = int(vid / (long(S) * S));
    bool any_in = false, any_out = false;
    for (int c = 0; c < 8; ++c) {
      const bool in = f[lat(i + (c & 1), j + ((c >> 1) & 1), k + (c >> 2), S1)] < 0.f;
      any_in |= in;
      any_out |= !in;
    }
    if (!tris) flags[vid] = f[lat(i, j, k, S1)] < 0.f ? 2 : 0;
    int nt = 0;
    int out = tris ? offsets[vid] : 0;
    if (any_in && any_out) {
      for (int pm = 0; pm < 6; ++pm) {
        int v[4][3];
        v[0][0] = i;
        v[0][1] = j;
        v[0][2] = k;
        for (int s = 1; s < 4; ++s) {
          for (int d = 0; d < 3; ++d) v[s][d] = v[s - 1][d];
          v[s][kPerm[pm][s - 1]] += 1;
        }
        bool in[4];
        int nin = 0;
        for (int s = 0; s < 4; ++s) {
          in[s] = f[lat(v[s][0], v[s][1], v[s][2], S1)] < 0.f;
          nin += in[s];
        }
        if (nin == 0 || nin == 4) continue;
        if (!tris) {
          nt += nin == 2 ? 2 : 1;
          continue;
        }
        double ci[3] = {0, 0, 0}, co[3] = {0, 0, 0};
        for (int s = 0; s < 4; ++s)
          for (int d = 0; d < 3; ++d) {
            double &acc = in[s] ? ci[d] : co[d];
            acc = __dadd_rn(acc, __ddiv_rn(double(v[s][d]), double(in[s] ? nin : 4 - nin)));
          }
        auto vert = [&](int s0, int s1) {
          return s0 < s1 ? edge_id(mask, base, S1, v[s0], v[s1]) : edge_id(mask, base, S1, v[s1], v[s0]);
        };
        auto emit = [&](int a, int b, int c) {
          const float4 pa = pts[a], pb = pts[b], pc = pts[c];
          const double u[3] = {double(__fsub_rn(pb.x, pa.x)), double(__fsub_rn(pb.y, pa.y)),
                               double(__fsub_rn(pb.z, pa.z))};
          const double w[3] = {double(__fsub_rn(pc.x, pa.x)), double(__fsub_rn(pc.y, pa.y)),
                               double(__fsub_rn(pc.z, pa.z))};
          const double nn[3] = {__dsub_rn(__dmul_rn(u[1], w[2]), __dmul_rn(u[2], w[1])),
                                __dsub_rn(__dmul_rn(u[2], w[0]), __dmul_rn(u[0], w[2])),
                                __dsub_rn(__dmul_rn(u[0], w[1]), __dmul_rn(u[1], w[0]))};
          const double dir = __dadd_rn(__dadd_rn(__dmul_rn(nn[0], __dsub_rn(co[0], ci[0])),
                                                 __dmul_rn(nn[1], __dsub_rn(co[1], ci[1]))),
                                       __dmul_rn(nn[2], __dsub_rn(co[2], ci[2])));
          tris[3 * size_t(out)] = a;
          tris[3 * size_t(out) + 1] = dir >= 0 ? b : c;
          tris[3 * size_t(out) + 2] = dir >= 0 ? c : b;
          list[out] = out;
          ++out;
        };
        if (nin == 1 || nin == 3) {
          int lone = 0;
          for (int s = 0; s < 4; ++s)
            if (in[s] == (nin == 1)) lone = s;
          int o[3], m = 0;
          for (int s = 0; s < 4; ++s)
            if (s != lone) o[m++] = s;
          emit(vert(lone, o[0]), vert(lone, o[1]), vert(lone, o[2]));
        } else {
          int a[2], b[2], na = 0, nb = 0;
          for (int s = 0; s < 4; ++s) {
            if (in[s]) a[na++] = s;
            else b[nb++] = s;
          }
          const int q0 = vert(a[0], b[0]), q1 = vert(a[0], b[1]), q2 = vert(a[1], b[1]), q3 = vert(a[1], b[0]);
          auto dist2 = [&](int x, int y) {
            const float4 px = pts[x], py = pts[y];
            const double t0 = double(__fsub_rn(px.x, py.x)), t1 = double(__fsub_rn(px.y, py.y)),
                         t2 = double(__fsub_rn(px.z, py.z));
            return __dadd_rn(__dadd_rn(__dmul_rn(t0, t0), __dmul_rn(t1, t1)), __dmul_rn(t2, t2));
          };
          if (dist2(q0, q2) <= dist2(q1, q3)) {
            emit(q0, q1, q2);
            emit(q0, q2, q3);
          } else {
            emit(q0, q1, q3);
            emit(q1, q2, q3);
          }
        }
      }
    }
    if (!tris) count[vid] = nt;
  }
}

// 6 x the signed volume of the closed surface, summed (the sign decides the
// orientation, Grid.cpp:270-275).
__global__ void k_surface_volume(const float4 *__restrict__ pts, const int *__restrict__ tris, int ntri,
                                 double *__restrict__ vol) {
  double acc = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntri; t += gridDim.x * blockDim.x) {
    const float4 a = pts[tris[3 * t]], b = pts[tris[3 * t + 1]], c = pts[tris[3 * t + 2]];
    acc -= double(a.x) * (double(b.y) * c.z - double(b.z) * c.y) - double(a.y) * (double(b.x) * c.z - double(b.z) * c.x) +
           double(a.z) * (double(b.x) * c.y - double(b.y) * c.x);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(vol, acc);
}

// Reversed orientation: corners 0 and 1 swap, as HostGrid::swap_orientation
// (Grid.cpp:53-56) does.
__global__ void k_swap_orientation(int *__restrict__ tris, int ntri) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntri; t += gridDim.x * blockDim.x) {
    const int x = tris[3 * t];
    tris[3 * t] = tris[3 * t + 1];
    tris[3 * t + 1] = x;
  }
}

// Summed tables over voxels, (S+1)^3: entry (x+1, y+1, z+1) first holds
// voxel (x, y, z)'s value -- 1 for a voxel that is not plainly outside
// (sat), its triangle count (tsat) -- then prefix sums run along x, y, z.
__global__ void k_sat_values(const signed char *__restrict__ flags, const int *__restrict__ offsets, int S,
                             int *__restrict__ sat, int *__restrict__ tsat) {
  const int S1 = S + 1;
  const long n = long(S1) * S1 * S1;
  for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
    const int i = int(idx % S1), j = int((idx / S1) % S1), k = int(idx / (long(S1) * S1));
    int s = 0, t = 0;
    if (i > 0 && j > 0 && k > 0) {
      const size_t v = size_t(i - 1) + size_t(j - 1) * S + size_t(k - 1) * S * S;
      t = offsets[v + 1] - offsets[v];
      s = (flags[v] != 0 || t > 0) ? 1 : 0;
    }
    sat[idx] = s;
    tsat[idx] = t;
  }
}

// Prefix sums along axis `axis` of both tables: one thread per line.
__global__ void k_sat_lines(int S, int axis, int *__restrict__ sat, int *__restrict__ tsat) {
  const int S1 = S + 1;
  const long lines = long(S1) * S1;
  const long step = axis == 0 ? 1 : (axis == 1 ? S1 : long(S1) * S1);
  for (long l = blockIdx.x * long(blockDim.x) + threadIdx.x; l < lines; l += long(gridDim.x) * blockDim.x) {
    const int u = int(l % S1), w = int(l / S1);
    long start;
    if (axis == 0) start = long(u) * S1 + long(w) * S1 * S1;
    else if (axis == 1) start = u + long(w) * S1 * S1;
    else start = u + long(w) * S1;
    int a = 0, b = 0;
    for (int x = 0; x < S1; ++x) {
      const long p = start + x * step;
      a += sat[p];
      b += tsat[p];
      sat[p] = a;
      tsat[p] = b;
    }
  }
}

// Waits for the stream when it goes out of scope: declared after the
// temporaries a build launches kernels on, so that no error path frees them
// while those kernels may still run.
struct SyncOnExit {
  cudaStream_t st;
  ~SyncOnExit() { cudaStreamSynchronize(st); }
};

int grid_blocks(long n, int sm_count) {
  const long b = (n + 255) / 256;
  return int(std::max<long>(1, std::min<long>(b, long(sm_count) * 16)));
}

// Builds the solver's grid from the field f ((S+1)^3 floats on the device).
int build_from_field(rpd_solver *s, int S, DevBuf &f) {
  rpd_context *ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const int S1 = S + 1;
  const long nl = long(S1) * S1 * S1, nv = long(S) * S * S;
  DevBuf mask, ecnt, ebase, vcnt, tiles, vol;
  SyncOnExit guard{st};
  const size_t tiles_n = std::max(scan_workspace_ints(int(nl + 1)), scan_workspace_ints(int(nv + 1)));
  if ((e = mask.ensure(size_t(nl))) != cudaSuccess || (e = ecnt.ensure(sizeof(int) * size_t(nl + 1))) != cudaSuccess ||
      (e = ebase.ensure(sizeof(int) * size_t(nl + 1))) != cudaSuccess ||
      (e = vcnt.ensure(sizeof(int) * size_t(nv + 1))) != cudaSuccess ||
      (e = tiles.ensure(sizeof(int) * tiles_n)) != cudaSuccess || (e = vol.ensure(sizeof(double))) != cudaSuccess ||
      (e = s->g_flags.ensure(size_t(nv))) != cudaSuccess ||
      (e = s->g_offsets.ensure(sizeof(int) * size_t(nv + 1))) != cudaSuccess ||
      (e = s->g_sat.ensure(sizeof(int) * size_t(nl))) != cudaSuccess ||
      (e = s->g_tsat.ensure(sizeof(int) * size_t(nl))) != cudaSuccess)
    return map_cuda(ctx, e, "alloc device grid");
  const int sm = ctx->sm_count;
  float *fp = f.as<float>();
  k_edge_masks<<<grid_blocks(nl, sm), 256, 0, st>>>(fp, S, mask.as<unsigned char>(), ecnt.as<int>());
  cudaMemsetAsync(ecnt.as<int>() + nl, 0, sizeof(int), st);
  if ((e = exclusive_scan(ecnt.as<int>(), ebase.as<int>(), int(nl + 1), tiles.as<int>(), st)) != cudaSuccess)
    return map_cuda(ctx, e, "scan edges");
  k_voxel_surface<<<grid_blocks(nv, sm), 256, 0, st>>>(fp, S, s->g_flags.as<signed char>(), vcnt.as<int>(), nullptr,
                                                       nullptr, nullptr, nullptr, nullptr, nullptr);
  cudaMemsetAsync(vcnt.as<int>() + nv, 0, sizeof(int), st);
  if ((e = exclusive_scan(vcnt.as<int>(), s->g_offsets.as<int>(), int(nv + 1), tiles.as<int>(), st)) != cudaSuccess)
    return map_cuda(ctx, e, "scan voxels");
  int totals[2] = {0, 0};
  cudaMemcpyAsync(&totals[0], ebase.as<int>() + nl, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&totals[1], s->g_offsets.as<int>() + nv, sizeof(int), cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "device grid counts");
  const int npts = totals[0], ntri = totals[1];
  if ((e = s->g_points.ensure(sizeof(float4) * size_t(std::max(npts, 1)))) != cudaSuccess ||
      (e = s->g_tris.ensure(sizeof(int) * 3 * size_t(std::max(ntri, 1)))) != cudaSuccess ||
      (e = s->g_list.ensure(sizeof(int) * size_t(std::max(ntri, 1)))) != cudaSuccess)
    return map_cuda(ctx, e, "alloc device grid");
  const float h = 1000 / float(S);
  k_edge_points<<<grid_blocks(nl, sm), 256, 0, st>>>(fp, S, h, mask.as<unsigned char>(), ebase.as<int>(),
                                                     s->g_points.as<float4>());
  k_voxel_surface<<<grid_blocks(nv, sm), 256, 0, st>>>(fp, S, nullptr, nullptr, mask.as<unsigned char>(),
                                                       ebase.as<int>(), s->g_points.as<float4>(),
                                                       s->g_offsets.as<int>(), s->g_tris.as<int>(),
                                                       s->g_list.as<int>());
  cudaMemsetAsync(vol.ptr, 0, sizeof(double), st);
  k_surface_volume<<<grid_blocks(ntri, sm), 256, 0, st>>>(s->g_points.as<float4>(), s->g_tris.as<int>(), ntri,
                                                          vol.as<double>());
  double v6 = 0.0;
  cudaMemcpyAsync(&v6, vol.ptr, sizeof(double), cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "device grid surface");
  if (v6 < 0.0) k_swap_orientation<<<grid_blocks(ntri, sm), 256, 0, st>>>(s->g_tris.as<int>(), ntri);
  k_sat_values<<<grid_blocks(nl, sm), 256, 0, st>>>(s->g_flags.as<signed char>(), s->g_offsets.as<int>(), S,
                                                    s->g_sat.as<int>(), s->g_tsat.as<int>());
  for (int axis = 0; axis < 3; ++axis)
    k_sat_lines<<<grid_blocks(long(S1) * S1, sm), 256, 0, st>>>(S, axis, s->g_sat.as<int>(), s->g_tsat.as<int>());
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return map_cuda(ctx, e, "device grid tables");
  DevGrid d;
  d.size = S;
  d.voxel = h;
  d.flags = s->g_flags.as<const signed char>();
  d.points = s->g_points.as<const float4>();
  d.tris = s->g_tris.as<const int>();
  d.list = s->g_list.as<const int>();
  d.offsets = s->g_offsets.as<const int>();
  d.sat = s->g_sat.as<const int>();
  d.tsat = s->g_tsat.as<const int>();
  d.lists_disjoint = 1;       // every triangle is listed in its own voxel
  d.has_border_corners = 0;   // corner flags are 0 or 2
  s->grid = d;
  s->grid_nonplain = -1;
  s->grid_points = npts;
  s->grid_triangles = ntri;
  return RPD_OK;
}

constexpr int kMaxGridSize = 1024;

}  // namespace grid_detail
}  // namespace rpd

using namespace rpd;
using namespace rpd::grid_detail;

extern "C" {

int rpd_solver_set_grid_field(rpd_solver *s, int size, const float *field, rpd_mem where) {
  if (!s || !field || size < 1 || size > kMaxGridSize) return RPD_ERR_INVALID;
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  s->grid = DevGrid();
  s->grid_nonplain = -1;
  const long nl = long(size + 1) * (size + 1) * (size + 1);
  DevBuf f;
  SyncOnExit guard{st};
  if ((e = f.ensure(sizeof(float) * size_t(nl))) != cudaSuccess) return map_cuda(ctx, e, "alloc field");
  if ((e = cudaMemcpyAsync(f.ptr, field, sizeof(float) * size_t(nl),
                           where == RPD_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
    return map_cuda(ctx, e, "copy field");
  k_field_outer_layer<<<grid_blocks(nl, ctx->sm_count), 256, 0, st>>>(size, f.as<float>());
  return build_from_field(s, size, f);
}

int rpd_solver_set_grid_blob(rpd_solver *s, int size, int nellipsoids, uint64_t seed) {
  if (!s || size < 1 || size > kMaxGridSize || nellipsoids < 1 || nellipsoids > 4096) return RPD_ERR_INVALID;
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  s->grid = DevGrid();
  s->grid_nonplain = -1;
  std::vector<double> c, a, R;
  random_blob_params(nellipsoids, seed, c, a, R);
  std::vector<double> params(c);
  params.insert(params.end(), a.begin(), a.end());
  params.insert(params.end(), R.begin(), R.end());
  const long nl = long(size + 1) * (size + 1) * (size + 1);
  DevBuf f, dp;
  SyncOnExit guard{st};
  if ((e = f.ensure(sizeof(float) * size_t(nl))) != cudaSuccess ||
      (e = dp.ensure(sizeof(double) * params.size())) != cudaSuccess)
    return map_cuda(ctx, e, "alloc field");
  if ((e = cudaMemcpyAsync(dp.ptr, params.data(), sizeof(double) * params.size(), cudaMemcpyHostToDevice, st)) !=
      cudaSuccess)
    return map_cuda(ctx, e, "copy blob");
  const double *pc = dp.as<double>(), *pa = pc + 3 * nellipsoids, *pr = pa + 3 * nellipsoids;
  k_blob_field<<<grid_blocks(nl, ctx->sm_count), 256, 0, st>>>(pc, pa, pr, nellipsoids, size, f.as<float>());
  return build_from_field(s, size, f);
}

rpd_grid *rpd_solver_export_grid(rpd_solver *s, int *err) {
  auto fail = [&](int code) -> rpd_grid * {
    if (err) *err = code;
    return nullptr;
  };
  if (!s || s->grid.size <= 0) return fail(RPD_ERR_INVALID);
  rpd_context *ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const DevGrid &d = s->grid;
  const int S = d.size;
  const size_t nv = size_t(S) * S * S;
  HostGrid g;
  g.size = S;
  g.voxel = d.voxel;
  std::vector<signed char> flags(nv);
  g.offsets.resize(nv + 1);
  cudaMemcpyAsync(flags.data(), d.flags, nv, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(g.offsets.data(), d.offsets, sizeof(int) * (nv + 1), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail(map_cuda(ctx, cudaGetLastError(), "export grid"));
  const int nlist = g.offsets[nv];
  const int npts = s->grid_points, ntri = s->grid_triangles;
  if (npts < 0 || ntri < 0) return fail(RPD_ERR_INVALID);
  g.points.resize(4 * size_t(npts));
  g.triangles.resize(3 * size_t(ntri));
  g.tri_list.resize(size_t(nlist));
  if (npts) cudaMemcpyAsync(g.points.data(), d.points, sizeof(float4) * npts, cudaMemcpyDeviceToHost, st);
  if (ntri) cudaMemcpyAsync(g.triangles.data(), d.tris, sizeof(int) * 3 * size_t(ntri), cudaMemcpyDeviceToHost, st);
  if (nlist) cudaMemcpyAsync(g.tri_list.data(), d.list, sizeof(int) * size_t(nlist), cudaMemcpyDeviceToHost, st);
  cudaError_t e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(map_cuda(ctx, e, "export grid"));
  g.in_domain.assign(flags.begin(), flags.end());
  if (err) *err = RPD_OK;
  return grid_handle(std::move(g));
}

}  // extern "C"
