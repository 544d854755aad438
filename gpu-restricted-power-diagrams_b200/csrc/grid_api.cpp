// C ABI of the host-side domain container (rpd_grid).
#include <cstring>
#include <string>

#include "../../include/rpd.h"
#include "grid_host.h"

struct rpd_grid {
  rpd::HostGrid g;
};

namespace rpd {
const HostGrid *host_grid(const rpd_grid *g) { return g ? &g->g : nullptr; }
rpd_grid *grid_handle(HostGrid &&g) {
  auto *r = new rpd_grid();
  r->g = std::move(g);
  return r;
}
}  // namespace rpd

extern "C" {

rpd_grid *rpd_grid_create(int size, const char *in_domain, const float *points_xyz, int npoints,
                          const int *triangles, int ntriangles, const int *tri_list, int nlist,
                          const int *offsets, int *err) {
  if (size <= 0 || !in_domain || npoints < 0 || ntriangles < 0 || nlist < 0 || !offsets ||
      (npoints && !points_xyz) || (ntriangles && !triangles) || (nlist && !tri_list)) {
    if (err) *err = RPD_ERR_INVALID;
    return nullptr;
  }
  auto *r = new rpd_grid();
  rpd::HostGrid &g = r->g;
  g.size = size;
  g.voxel = 1000 / float(size);
  const size_t nv = size_t(size) * size * size;
  g.in_domain.assign(in_domain, in_domain + nv);
  g.points.resize(4 * size_t(npoints));
  for (int i = 0; i < npoints; ++i) {
    for (int d = 0; d < 3; ++d) g.points[4 * size_t(i) + d] = points_xyz[3 * size_t(i) + d];
    g.points[4 * size_t(i) + 3] = 0.f;
  }
  g.triangles.assign(triangles, triangles + 3 * size_t(ntriangles));
  g.tri_list.assign(tri_list, tri_list + nlist);
  g.offsets.assign(offsets, offsets + nv + 1);
  for (int t : g.triangles)
    if (t < 0 || t >= npoints) {
      delete r;
      if (err) *err = RPD_ERR_FORMAT;
      return nullptr;
    }
  for (int t : g.tri_list)
    if (t < 0 || t >= ntriangles) {
      delete r;
      if (err) *err = RPD_ERR_FORMAT;
      return nullptr;
    }
  for (size_t v = 0; v <= nv; ++v)
    if (g.offsets[v] < 0 || g.offsets[v] > nlist || (v && g.offsets[v] < g.offsets[v - 1])) {
      delete r;
      if (err) *err = RPD_ERR_FORMAT;
      return nullptr;
    }
  if (g.volume() < 0) g.swap_orientation();
  if (err) *err = RPD_OK;
  return r;
}

rpd_grid *rpd_grid_load(const char *path, int *err) {
  if (!path) {
    if (err) *err = RPD_ERR_INVALID;
    return nullptr;
  }
  auto *r = new rpd_grid();
  std::string why;
  if (!r->g.load(path, &why)) {
    delete r;
    if (err) *err = why.rfind("can not open", 0) == 0 ? RPD_ERR_IO : RPD_ERR_FORMAT;
    return nullptr;
  }
  if (err) *err = RPD_OK;
  return r;
}

int rpd_grid_save(const rpd_grid *g, const char *path) {
  if (!g || !path) return RPD_ERR_INVALID;
  return g->g.save(path) ? RPD_OK : RPD_ERR_IO;
}

int rpd_grid_valid(const rpd_grid *g, char *why, int why_len) {
  if (!g) return 0;
  std::string w;
  const bool ok = g->g.valid(&w);
  if (why && why_len > 0) {
    std::strncpy(why, w.c_str(), size_t(why_len) - 1);
    why[why_len - 1] = 0;
  }
  return ok ? 1 : 0;
}

double rpd_grid_volume(const rpd_grid *g) { return g ? g->g.volume() : 0.0; }

int rpd_grid_invariants(const rpd_grid *g, double *out4) {
  if (!g || !out4) return RPD_ERR_INVALID;
  g->g.invariants(out4);
  return RPD_OK;
}

int rpd_grid_info(const rpd_grid *g, int *size, int *npoints, int *ntriangles, int *nlist) {
  if (!g) return RPD_ERR_INVALID;
  if (size) *size = g->g.size;
  if (npoints) *npoints = g->g.num_points();
  if (ntriangles) *ntriangles = g->g.num_triangles();
  if (nlist) *nlist = int(g->g.tri_list.size());
  return RPD_OK;
}

int rpd_grid_export(const rpd_grid *g, char *in_domain, float *points_xyz, int *triangles, int *tri_list,
                    int *offsets) {
  if (!g) return RPD_ERR_INVALID;
  const rpd::HostGrid &h = g->g;
  if (in_domain) std::memcpy(in_domain, h.in_domain.data(), h.in_domain.size());
  if (points_xyz)
    for (int i = 0; i < h.num_points(); ++i)
      for (int d = 0; d < 3; ++d) points_xyz[3 * size_t(i) + d] = h.points[4 * size_t(i) + d];
  if (triangles) std::memcpy(triangles, h.triangles.data(), sizeof(int) * h.triangles.size());
  if (tri_list) std::memcpy(tri_list, h.tri_list.data(), sizeof(int) * h.tri_list.size());
  if (offsets) std::memcpy(offsets, h.offsets.data(), sizeof(int) * h.offsets.size());
  return RPD_OK;
}

void rpd_grid_destroy(rpd_grid *g) { delete g; }

rpd_grid *rpd_grid_make_blob(int size, int nellipsoids, uint64_t seed, int *err) {
  if (size < 2 || size > 1024 || nellipsoids < 1 || nellipsoids > 64) {
    if (err) *err = RPD_ERR_INVALID;
    return nullptr;
  }
  auto *r = new rpd_grid();
  rpd::make_random_blob(size, nellipsoids, seed, r->g);
  if (err) *err = RPD_OK;
  return r;
}

int rpd_synth_poisson_disk(int n, uint64_t seed, double rfac, float *xyzw) {
  if (n <= 0 || !xyzw || !(rfac > 0)) return RPD_ERR_INVALID;
  std::vector<float> v;
  const int k = rpd::poisson_disk(n, seed, rfac, 200, v);
  std::memcpy(xyzw, v.data(), sizeof(float) * v.size());
  return k;
}

rpd_grid *rpd_grid_make_cube(int size, int *err) {
  if (size < 2 || size > 1024) {
    if (err) *err = RPD_ERR_INVALID;
    return nullptr;
  }
  auto *r = new rpd_grid();
  rpd::make_cube_domain(size, r->g);
  if (err) *err = RPD_OK;
  return r;
}

}  // extern "C"
