// Host container of a volume domain in the reference --grid layout
// (Grid.h:14-70): voxel-corner flags, a closed boundary triangle surface and
// per-voxel sorted triangle-id lists.  Coordinates in [0,1000]^3.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace rpd {

struct HostGrid {
  int size = 0;              // voxels per axis
  float voxel = 0.f;         // 1000 / size
  std::vector<char> in_domain;  // size^3: 0 outside, 1 on border, 2 inside
  std::vector<float> points;    // xyzw, w = 0
  std::vector<int> triangles;   // 3 ids per triangle
  std::vector<int> tri_list;    // per-voxel sorted triangle ids
  std::vector<int> offsets;     // size^3 + 1

  int num_points() const { return int(points.size() / 4); }
  int num_triangles() const { return int(triangles.size() / 3); }

  // Grid::getVolume (Grid.cpp:30-35): sum of -det(p0, p1, p2)/6.
  double volume() const;
  // Volume and first moments (Grid.cpp:37-51): {m*x, m*y, m*z, m}.
  void invariants(double out[4]) const;
  // Grid::swapTrianglesOrientation (Grid.cpp:53-56).
  void swap_orientation();
  // Grid::valid (Grid.cpp:60-184); `why` receives the first failure.
  bool valid(std::string *why) const;
  // Grid::load / Grid::save: the reference text format (Grid.cpp:186-344).
  bool load(const char *path, std::string *why);
  bool save(const char *path) const;
};

// Union of `nell` ellipsoids (centre c, semi-axes a, rotation R row-major),
// all in [0,1]^3, voxelized on a size^3 grid: the implicit function is
// sampled at the voxel corners, every voxel is split into the 6 Kuhn
// tetrahedra of its main diagonal and the zero set is extracted by marching
// tetrahedra (surface vertices strictly inside tet edges, so no corner lies
// on the surface).  Triangles are listed in the voxel of their tetrahedron.
void make_ellipsoid_blob(int size, int nell, const double *centres, const double *axes, const double *rot,
                         HostGrid &g);
// Seeded random blob: centres U[0.35,0.65]^3, semi-axes U[0.15,0.35], random
// rotations (the domain of the benchmark configurations).
void make_random_blob(int size, int nell, uint64_t seed, HostGrid &g);
// The ellipsoids of make_random_blob (centres, semi-axes, rotations).
void random_blob_params(int nell, uint64_t seed, std::vector<double> &c, std::vector<double> &a,
                        std::vector<double> &R);
// The cube [d, 1000-d]^3, d = half a voxel, as a domain: no voxel corner on
// its surface (flags 0 outside, 2 inside); faces cut by the voxel columns,
// 2 triangles per rectangle, listed in their voxel.
void make_cube_domain(int size, HostGrid &g);

// Seeded Poisson-disk sample of the unit cube (reference frame x1000).
int poisson_disk(int n, uint64_t seed, double rfac, int max_batches, std::vector<float> &xyzw);

}  // namespace rpd
