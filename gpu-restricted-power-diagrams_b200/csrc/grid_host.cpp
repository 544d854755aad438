// Host-side domain grids: the reference --grid text format (Grid.cpp) and the
// synthetic domains of the benchmark configurations.
#include "grid_host.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <fstream>
#include <set>
#include <sstream>
#include <unordered_map>
#include <utility>

namespace rpd {

namespace {

inline double det3(double a11, double a12, double a13, double a21, double a22, double a23, double a31, double a32,
                   double a33) {
  return a11 * (a22 * a33 - a23 * a32) - a21 * (a12 * a33 - a13 * a32) + a31 * (a12 * a23 - a13 * a22);
}

inline double tet_volume(const std::vector<float> &p, int i0, int i1, int i2) {
  return -det3(p[4 * i0], p[4 * i0 + 1], p[4 * i0 + 2], p[4 * i1], p[4 * i1 + 1], p[4 * i1 + 2], p[4 * i2],
               p[4 * i2 + 1], p[4 * i2 + 2]) /
         6;
}

// splitmix64: the seeded stream of the synthetic domains.
struct SplitMix {
  uint64_t s;
  explicit SplitMix(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  }
  double uniform() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }
  double normal() {
    const double u1 = std::max(uniform(), 1e-300), u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

}  // namespace

double HostGrid::volume() const {
  double v = 0;
  for (int t = 0; t < num_triangles(); ++t) v += tet_volume(points, triangles[3 * t], triangles[3 * t + 1], triangles[3 * t + 2]);
  return v;
}

void HostGrid::invariants(double out[4]) const {
  double acc[4] = {0, 0, 0, 0};
  for (int t = 0; t < num_triangles(); ++t) {
    const int i0 = triangles[3 * t], i1 = triangles[3 * t + 1], i2 = triangles[3 * t + 2];
    const double v4 = tet_volume(points, i0, i1, i2) / 4;
    for (int d = 0; d < 3; ++d)
      acc[d] += v4 * (double(points[4 * i0 + d]) + double(points[4 * i1 + d]) + double(points[4 * i2 + d]));
    acc[3] += 4 * v4;
  }
  for (int d = 0; d < 4; ++d) out[d] = acc[d];
}

void HostGrid::swap_orientation() {
  for (int t = 0; t < num_triangles(); ++t) std::swap(triangles[3 * t], triangles[3 * t + 1]);
}

bool HostGrid::valid(std::string *why) const {
  auto fail = [&](const std::string &m) {
    if (why) *why = m;
    return false;
  };
  const size_t nvox = size_t(size) * size * size;
  if (in_domain.size() != nvox) return fail("unexpected inDomain size");
  for (char c : in_domain)
    if (c & 0xfc) return fail("unexpected inDomain value");
  if (points.size() % 4) return fail("unexpected points size");
  const int np = num_points();
  if (triangles.size() % 3) return fail("unexpected triangles size");
  const int nt = num_triangles();
  for (int p : triangles)
    if (p < 0 || p >= np) return fail("invalid point id in triangles");
  for (int t : tri_list)
    if (t < 0 || t >= nt) return fail("invalid triangle id in triangle list");
  if (offsets.size() <= nvox) return fail("unexpected offsets size");
  for (int o : offsets)
    if (o < 0 || o > int(tri_list.size())) return fail("invalid offset");
  if (volume() <= 0) return fail("bad volume (orientation)");
  const float eps = 0.01f;
  for (int t = 0; t < nt; ++t) {
    const float *a = &points[4 * triangles[3 * t]], *b = &points[4 * triangles[3 * t + 1]],
                *c = &points[4 * triangles[3 * t + 2]];
    const double u[3] = {double(b[0] - a[0]), double(b[1] - a[1]), double(b[2] - a[2])};
    const double v[3] = {double(c[0] - a[0]), double(c[1] - a[1]), double(c[2] - a[2])};
    const double x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
    if (float((x * x + y * y + z * z) / 4) < eps * eps) return fail("degenerate triangle " + std::to_string(t));
  }
  // every directed edge once, and its opposite present (closed, oriented)
  std::set<std::pair<int, int>> edges;
  for (int t = 0; t < nt; ++t)
    for (int j = 0; j < 3; ++j) {
      const auto e = std::make_pair(triangles[3 * t + j], triangles[3 * t + (j + 1) % 3]);
      if (!edges.insert(e).second) return fail("duplicated edge");
    }
  for (const auto &e : edges)
    if (!edges.count(std::make_pair(e.second, e.first))) return fail("open edge");
  // no voxel whose 8 corners are all on the border (flag 1): the restriction
  // could not find a start corner in it (Grid.cpp:147-168; corners past the
  // last layer count as outside).  The reference's loop adds the offsets to
  // the grid origin instead of to the voxel, so it only ever inspects voxel
  // 0; the rule is applied here to every voxel, as its comment states.
  for (int z = 0; z + 1 < size; ++z)
    for (int y = 0; y + 1 < size; ++y)
      for (int x = 0; x + 1 < size; ++x) {
        int border = 0;
        for (int c = 0; c < 8; ++c)
          border += in_domain[size_t(x + (c & 1)) + size_t(y + ((c >> 1) & 1)) * size +
                              size_t(z + (c >> 2)) * size * size] == 1;
        if (border == 8)
          return fail("voxel (" + std::to_string(x) + "," + std::to_string(y) + "," + std::to_string(z) +
                      ") has only border corners");
      }
  for (size_t o = 0; o + 1 < offsets.size(); ++o) {
    if (offsets[o] > offsets[o + 1]) return fail("bad offset ordering");
    for (int t = offsets[o]; t + 1 < offsets[o + 1]; ++t)
      if (tri_list[t] >= tri_list[t + 1]) return fail("triangle list not sorted");
  }
  return true;
}

bool HostGrid::load(const char *path, std::string *why) {
  auto fail = [&](const std::string &m) {
    if (why) *why = m;
    return false;
  };
  std::ifstream f(path);
  if (!f.is_open()) return fail(std::string("can not open ") + path);
  f >> size;
  if (!f.good() || size <= 0 || size > 4096) return fail("bad grid size");
  voxel = 1000 / float(size);
  const size_t nvox = size_t(size) * size * size;
  in_domain.resize(nvox);
  // corner flags are raw bytes 0/1/2 separated by blanks (Grid.cpp:197-203)
  for (size_t i = 0; i < nvox; ++i) {
    f >> in_domain[i];
    if (in_domain[i] & 0xfc) return fail("unexpected value in domain");
  }
  if (!f.good()) return fail("can not read the in domain vector");
  int np = 0;
  f >> np;
  if (!f.good() || np < 0) return fail("can not read the points");
  points.assign(4 * size_t(np), 0.f);
  for (int i = 0; i < np; ++i)
    for (int j = 0; j < 3; ++j) f >> points[4 * size_t(i) + j];
  if (!f.good()) return fail("can not read the points");
  int n3 = 0;
  f >> n3;
  if (!f.good() || n3 < 0 || n3 % 3) return fail("can not read the triplets");
  triangles.resize(n3);
  for (auto &t : triangles) {
    f >> t;
    if (t < 0 || t >= np) return fail("bad triangle point");
  }
  if (!f.good()) return fail("can not read the triplets");
  int nl = 0;
  f >> nl;
  if (!f.good() || nl < 0) return fail("can not read the triangles indirections");
  tri_list.resize(nl);
  for (auto &t : tri_list) {
    f >> t;
    if (t < 0 || t >= n3 / 3) return fail("bad triangle id");
  }
  if (!f.good()) return fail("can not read the triangles indirections");
  int no = 0;
  f >> no;
  if (no <= int(nvox)) return fail("the number of offsets seems bad");
  offsets.resize(no);
  for (auto &o : offsets) {
    f >> o;
    if (o < 0 || o > nl) return fail("bad offset");
  }
  if (f.fail()) return fail("can not read the offsets");
  if (volume() < 0) swap_orientation();  // Grid.cpp:270-275
  return true;
}

bool HostGrid::save(const char *path) const {
  std::ofstream f(path, std::ofstream::trunc);
  if (!f.is_open()) return false;
  f << size << "\n";
  for (char c : in_domain) f << c << " ";
  f << "\n" << num_points() << "\n";
  f.precision(9);
  for (int i = 0; i < num_points(); ++i)
    f << points[4 * i] << " " << points[4 * i + 1] << " " << points[4 * i + 2] << " ";
  f << "\n" << triangles.size() << "\n";
  for (int t : triangles) f << t << " ";
  f << "\n" << tri_list.size() << "\n";
  for (int t : tri_list) f << t << " ";
  f << "\n" << offsets.size() << "\n";
  for (int o : offsets) f << o << " ";
  f << "\n";
  return f.good();
}

void make_ellipsoid_blob(int size, int nell, const double *centres, const double *axes, const double *rot,
                         HostGrid &g) {
  const int S = size, S1 = size + 1;
  g = HostGrid();
  g.size = S;
  g.voxel = 1000 / float(S);
  // implicit function on the (S+1)^3 lattice, in [0,1] units; +1 on the
  // lattice boundary so that the surface is closed inside the grid
  std::vector<float> f(size_t(S1) * S1 * S1);
  for (int k = 0; k < S1; ++k)
    for (int j = 0; j < S1; ++j)
      for (int i = 0; i < S1; ++i) {
        double v = 1.0;
        if (i > 0 && j > 0 && k > 0 && i < S && j < S && k < S) {
          const double p[3] = {double(i) / S, double(j) / S, double(k) / S};
          for (int e = 0; e < nell; ++e) {
            const double d[3] = {p[0] - centres[3 * e], p[1] - centres[3 * e + 1], p[2] - centres[3 * e + 2]};
            double q = 0;
            for (int r = 0; r < 3; ++r) {
              const double t = rot[9 * e + 3 * r] * d[0] + rot[9 * e + 3 * r + 1] * d[1] + rot[9 * e + 3 * r + 2] * d[2];
              q += (t / axes[3 * e + r]) * (t / axes[3 * e + r]);
            }
            v = std::min(v, q - 1.0);
          }
          if (v == 0.0) v = 1e-12;  // the surface never passes through a corner
        }
        f[size_t(i) + size_t(j) * S1 + size_t(k) * S1 * S1] = float(v);
      }
  auto lat = [S1](int i, int j, int k) { return size_t(i) + size_t(j) * S1 + size_t(k) * S1 * S1; };
  g.in_domain.assign(size_t(S) * S * S, 0);
  for (int k = 0; k < S; ++k)
    for (int j = 0; j < S; ++j)
      for (int i = 0; i < S; ++i) g.in_domain[i + j * S + size_t(k) * S * S] = f[lat(i, j, k)] < 0 ? 2 : 0;

  std::unordered_map<uint64_t, int> vmap;
  const float h = g.voxel;
  // surface vertex on the lattice edge from a to a + d (d in {0,1}^3)
  auto edge_vertex = [&](const int a[3], const int b[3]) {
    const int code = (b[0] - a[0]) | ((b[1] - a[1]) << 1) | ((b[2] - a[2]) << 2);
    const uint64_t key = uint64_t(lat(a[0], a[1], a[2])) * 8 + code;
    auto it = vmap.find(key);
    if (it != vmap.end()) return it->second;
    const double fa = f[lat(a[0], a[1], a[2])], fb = f[lat(b[0], b[1], b[2])];
    double t = fa / (fa - fb);
    t = std::min(0.9, std::max(0.1, t));
    const int id = g.num_points();
    for (int d = 0; d < 3; ++d) g.points.push_back(float((a[d] + t * (b[d] - a[d])) * double(h)));
    g.points.push_back(0.f);
    vmap.emplace(key, id);
    return id;
  };
  static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  g.offsets.assign(size_t(S) * S * S + 1, 0);
  for (int k = 0; k < S; ++k)
    for (int j = 0; j < S; ++j)
      for (int i = 0; i < S; ++i) {
        const size_t vid = i + j * size_t(S) + k * size_t(S) * S;
        g.offsets[vid] = int(g.tri_list.size());
        bool any_in = false, any_out = false;
        for (int c = 0; c < 8; ++c) {
          const bool in = f[lat(i + (c & 1), j + ((c >> 1) & 1), k + (c >> 2))] < 0;
          any_in |= in;
          any_out |= !in;
        }
        if (!(any_in && any_out)) continue;
        for (const auto &pm : perms) {
          int v[4][3];
          v[0][0] = i; v[0][1] = j; v[0][2] = k;
          for (int s = 1; s < 4; ++s) {
            for (int d = 0; d < 3; ++d) v[s][d] = v[s - 1][d];
            v[s][pm[s - 1]] += 1;
          }
          bool in[4];
          int nin = 0;
          for (int s = 0; s < 4; ++s) {
            in[s] = f[lat(v[s][0], v[s][1], v[s][2])] < 0;
            nin += in[s];
          }
          if (nin == 0 || nin == 4) continue;
          // centroids of the inside and outside tet vertices: the surface
          // normal must point from the first to the second
          double ci[3] = {0, 0, 0}, co[3] = {0, 0, 0};
          for (int s = 0; s < 4; ++s)
            for (int d = 0; d < 3; ++d) (in[s] ? ci[d] : co[d]) += v[s][d] / double(in[s] ? nin : 4 - nin);
          auto vert = [&](int s0, int s1) { return s0 < s1 ? edge_vertex(v[s0], v[s1]) : edge_vertex(v[s1], v[s0]); };
          auto emit = [&](int a, int b, int c) {
            const float *pa = &g.points[4 * size_t(a)], *pb = &g.points[4 * size_t(b)], *pc = &g.points[4 * size_t(c)];
            const double u[3] = {double(pb[0] - pa[0]), double(pb[1] - pa[1]), double(pb[2] - pa[2])};
            const double w[3] = {double(pc[0] - pa[0]), double(pc[1] - pa[1]), double(pc[2] - pa[2])};
            const double n[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
            const double dir = n[0] * (co[0] - ci[0]) + n[1] * (co[1] - ci[1]) + n[2] * (co[2] - ci[2]);
            const int t = g.num_triangles();
            if (dir >= 0) {
              g.triangles.insert(g.triangles.end(), {a, b, c});
            } else {
              g.triangles.insert(g.triangles.end(), {a, c, b});
            }
            g.tri_list.push_back(t);
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
            for (int s = 0; s < 4; ++s) (in[s] ? a[na++] : b[nb++]) = s;
            // quad a0b0, a0b1, a1b1, a1b0 split along its shorter diagonal
            const int q0 = vert(a[0], b[0]), q1 = vert(a[0], b[1]), q2 = vert(a[1], b[1]), q3 = vert(a[1], b[0]);
            auto dist2 = [&](int x, int y) {
              double s2 = 0;
              for (int d = 0; d < 3; ++d) {
                const double t = g.points[4 * size_t(x) + d] - g.points[4 * size_t(y) + d];
                s2 += t * t;
              }
              return s2;
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
  g.offsets[size_t(S) * S * S] = int(g.tri_list.size());
  if (g.volume() < 0) g.swap_orientation();
}

void random_blob_params(int nell, uint64_t seed, std::vector<double> &c, std::vector<double> &a,
                        std::vector<double> &R) {
  SplitMix rng(seed);
  c.assign(3 * size_t(nell), 0.0);
  a.assign(3 * size_t(nell), 0.0);
  R.assign(9 * size_t(nell), 0.0);
  for (int e = 0; e < nell; ++e) {
    for (int d = 0; d < 3; ++d) c[3 * e + d] = 0.35 + 0.3 * rng.uniform();
    for (int d = 0; d < 3; ++d) a[3 * e + d] = 0.15 + 0.2 * rng.uniform();
    // uniform rotation from a normalised Gaussian quaternion
    double q[4];
    double n = 0;
    for (double &x : q) {
      x = rng.normal();
      n += x * x;
    }
    n = std::sqrt(n);
    for (double &x : q) x /= n;
    const double w = q[0], x = q[1], y = q[2], z = q[3];
    const double m[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - z * w),     2 * (x * z + y * w),
                         2 * (x * y + z * w),     1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                         2 * (x * z - y * w),     2 * (y * z + x * w),     1 - 2 * (x * x + y * y)};
    for (int r = 0; r < 9; ++r) R[9 * e + r] = m[r];
  }
}

void make_random_blob(int size, int nell, uint64_t seed, HostGrid &g) {
  std::vector<double> c, a, R;
  random_blob_params(nell, seed, c, a, R);
  make_ellipsoid_blob(size, nell, c.data(), a.data(), R.data(), g);
}

void make_cube_domain(int size, HostGrid &g) {
  // The box [d, 1000-d]^3 with d = half a voxel: every corner is strictly
  // inside (flag 2) or outside (flag 0), so no start corner of the domain
  // restriction can lie on the surface.  Each face is cut by the voxel
  // columns into rectangles, 2 triangles each, listed in their voxel.
  const int S = size;
  g = HostGrid();
  g.size = S;
  g.voxel = 1000 / float(S);
  const double h = g.voxel, d = 0.5 * h, lo = d, hi = 1000.0 - d;
  g.in_domain.assign(size_t(S) * S * S, 0);
  for (int k = 1; k < S; ++k)
    for (int j = 1; j < S; ++j)
      for (int i = 1; i < S; ++i) g.in_domain[i + j * size_t(S) + k * size_t(S) * S] = 2;
  // face lattice coordinate t in [0, S]: 0 -> lo, S -> hi, else t * h
  auto coord = [&](int t) { return t == 0 ? lo : (t == S ? hi : t * h); };
  std::unordered_map<uint64_t, int> pid;
  auto point = [&](int axis, int side, int a, int b) {
    // a, b: lattice coordinates along the two other axes (0..S)
    int c[3];
    c[axis] = side ? S : 0;
    c[(axis + 1) % 3] = a;
    c[(axis + 2) % 3] = b;
    const uint64_t key = uint64_t(c[0]) + uint64_t(c[1]) * (S + 1) + uint64_t(c[2]) * (S + 1) * (S + 1);
    auto it = pid.find(key);
    if (it != pid.end()) return it->second;
    const int id = g.num_points();
    g.points.insert(g.points.end(), {float(coord(c[0])), float(coord(c[1])), float(coord(c[2])), 0.f});
    pid.emplace(key, id);
    return id;
  };
  std::vector<std::vector<int>> per_voxel(size_t(S) * S * S);
  for (int axis = 0; axis < 3; ++axis)
    for (int side = 0; side < 2; ++side)
      for (int b = 0; b < S; ++b)
        for (int a = 0; a < S; ++a) {
          const int p00 = point(axis, side, a, b), p10 = point(axis, side, a + 1, b),
                    p11 = point(axis, side, a + 1, b + 1), p01 = point(axis, side, a, b + 1);
          int v[3];
          v[axis] = side ? S - 1 : 0;
          v[(axis + 1) % 3] = a;
          v[(axis + 2) % 3] = b;
          const size_t vid = v[0] + v[1] * size_t(S) + v[2] * size_t(S) * S;
          const int t0 = g.num_triangles();
          // (axis+1, axis+2) is right-handed around +axis: outward on side 1
          if (side)
            g.triangles.insert(g.triangles.end(), {p00, p10, p11, p00, p11, p01});
          else
            g.triangles.insert(g.triangles.end(), {p00, p11, p10, p00, p01, p11});
          per_voxel[vid].push_back(t0);
          per_voxel[vid].push_back(t0 + 1);
        }
  g.offsets.assign(size_t(S) * S * S + 1, 0);
  for (size_t v = 0; v < per_voxel.size(); ++v) {
    std::sort(per_voxel[v].begin(), per_voxel[v].end());
    g.offsets[v] = int(g.tri_list.size());
    g.tri_list.insert(g.tri_list.end(), per_voxel[v].begin(), per_voxel[v].end());
  }
  g.offsets[per_voxel.size()] = int(g.tri_list.size());
  if (g.volume() < 0) g.swap_orientation();
}


// Seeded Poisson-disk sample of [0,1]^3 by dart throwing (random sequential
// adsorption): a uniform candidate is kept when no kept point lies closer
// than r = rfac * n^(-1/3).  Candidates come in seeded batches; a batch is
// tried in the order of its candidates' background cells (side r, at most 8
// points each) for locality, every candidate against every point kept
// before it.  Stops at n points or after max_batches batches.  Output in the
// reference frame: xyz * 1000, w = 0.  Returns the number of points.
int poisson_disk(int n, uint64_t seed, double rfac, int max_batches, std::vector<float> &xyzw) {
  xyzw.clear();
  if (n <= 0) return 0;
  const double r = rfac * std::pow(double(n), -1.0 / 3.0), r2 = r * r;
  const int G = std::max(1, int(1.0 / r));
  const double cell = 1.0 / G;  // >= r: neighbours lie in the 27 cells around
  constexpr int kSlots = 8;     // a cube of side r holds at most 8 points r apart
  std::vector<uint8_t> cnt(size_t(G) * G * G, 0);
  std::vector<int> slot(size_t(G) * G * G * kSlots, -1);
  std::vector<double> pts;
  pts.reserve(size_t(n) * 3);
  SplitMix rng(seed);
  const size_t batch = std::max<size_t>(1 << 16, size_t(n) / 4);
  std::vector<std::pair<uint64_t, std::array<double, 3>>> cand(batch);
  int kept = 0;
  for (int b = 0; b < max_batches && kept < n; ++b) {
    for (auto &c : cand) {
      c.second = {rng.uniform(), rng.uniform(), rng.uniform()};
      const int ix = std::min(G - 1, int(c.second[0] / cell)), iy = std::min(G - 1, int(c.second[1] / cell)),
                iz = std::min(G - 1, int(c.second[2] / cell));
      c.first = (uint64_t(iz) * G + iy) * G + ix;
    }
    std::stable_sort(cand.begin(), cand.end(),
                     [](const auto &a, const auto &c) { return a.first < c.first; });
    for (const auto &c : cand) {
      if (kept >= n) break;
      const double x = c.second[0], y = c.second[1], z = c.second[2];
      const int ix = int(c.first % G), iy = int((c.first / G) % G), iz = int(c.first / (uint64_t(G) * G));
      bool ok = cnt[c.first] < kSlots;
      for (int dz = -1; dz <= 1 && ok; ++dz) {
        const int zz = iz + dz;
        if (zz < 0 || zz >= G) continue;
        for (int dy = -1; dy <= 1 && ok; ++dy) {
          const int yy = iy + dy;
          if (yy < 0 || yy >= G) continue;
          for (int dx = -1; dx <= 1 && ok; ++dx) {
            const int xx = ix + dx;
            if (xx < 0 || xx >= G) continue;
            const size_t id = (size_t(zz) * G + yy) * G + xx;
            for (int k = 0; k < cnt[id]; ++k) {
              const double *q = &pts[3 * size_t(slot[id * kSlots + k])];
              const double ex = q[0] - x, ey = q[1] - y, ez = q[2] - z;
              if (ex * ex + ey * ey + ez * ez < r2) {
                ok = false;
                break;
              }
            }
          }
        }
      }
      if (!ok) continue;
      slot[c.first * kSlots + cnt[c.first]++] = kept;
      pts.insert(pts.end(), {x, y, z});
      ++kept;
    }
  }
  xyzw.resize(size_t(kept) * 4);
  for (int i = 0; i < kept; ++i) {
    for (int d = 0; d < 3; ++d) xyzw[4 * size_t(i) + d] = float(pts[3 * size_t(i) + d] * 1000.0);
    xyzw[4 * size_t(i) + 3] = 0.f;
  }
  return kept;
}

}  // namespace rpd
