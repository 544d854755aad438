// Test infrastructure only -- the oracle (see rpd_oracle.h).  Restates the
// reference algorithm step by step, in the same floating-point operation
// order, so that with the same inputs it reproduces the reference kernels
// compiled for the CPU bit for bit.  Citations are file:line in the
// reference project.
#include "rpd_oracle.h"

#include <dlfcn.h>
#include <omp.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cfloat>
#include <chrono>
#include <climits>
#include <limits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "shim/ref_abi.h"

namespace {

// Status.h:4-16
enum Status : int {
  vertex_overflow = 0,
  plane_overflow = 1,
  inconsistent_boundary = 2,
  security_radius_not_reached = 3,
  success = 4,
  needs_exact_predicates = 5,
  empty_cell = 6,
  find_another_beginning_vertex = 7,
  triangle_overflow = 8,
  seed_on_border = 9,
  hessian_overflow = 10,
};
constexpr int kStatusNum = 11;
constexpr int kNoCellLimits = -100000;  // voronoi.h:53
constexpr uint8_t kEndOfList = 255;     // ConvexCell.cl:132

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class R>
struct Vec4 {
  R x, y, z, w;
};
template <class R>
inline Vec4<R> mk(R x, R y, R z, R w) {
  return Vec4<R>{x, y, z, w};
}
template <class R>
inline Vec4<R> add4(Vec4<R> a, Vec4<R> b) {
  return mk<R>(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
template <class R>
inline Vec4<R> sub4(Vec4<R> a, Vec4<R> b) {
  return mk<R>(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
template <class R>
inline Vec4<R> scale4(R s, Vec4<R> a) {
  return mk<R>(s * a.x, s * a.y, s * a.z, s * a.w);
}
// 3-component dot (ConvexCell.cl:62-64).
template <class R>
inline R dot3(Vec4<R> a, Vec4<R> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
// 4-component dot, as OpenCL's dot() on a 4-vector.
template <class R>
inline R dot4(Vec4<R> a, Vec4<R> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}
// OpenCL cross() on a 4-vector: w ignored, result w = 0.
template <class R>
inline Vec4<R> cross4(Vec4<R> a, Vec4<R> b) {
  return mk<R>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, R(0));
}
template <class R>
inline R det2(R a11, R a12, R a21, R a22) {
  return a11 * a22 - a12 * a21;
}
// det3x3 expanded along the first column (ConvexCell.cl:72-77).
template <class R>
inline R det3(R a11, R a12, R a13, R a21, R a22, R a23, R a31, R a32, R a33) {
  return a11 * det2(a22, a23, a32, a33) - a21 * det2(a12, a13, a32, a33) + a31 * det2(a12, a13, a22, a23);
}
template <class R>
inline R det3v(Vec4<R> a, Vec4<R> b, Vec4<R> c) {
  return det3(a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z);
}
// 4x4 determinant by 2x2 minors of the first two columns (ConvexCell.cl:79-97);
// instantiated in R for VHSAlgo 0 and in double for VHSAlgo 2.
template <class D>
inline D det4(D a11, D a12, D a13, D a14, D a21, D a22, D a23, D a24, D a31, D a32, D a33, D a34, D a41, D a42,
              D a43, D a44) {
  const D m12 = a21 * a12 - a11 * a22;
  const D m13 = a31 * a12 - a11 * a32;
  const D m14 = a41 * a12 - a11 * a42;
  const D m23 = a31 * a22 - a21 * a32;
  const D m24 = a41 * a22 - a21 * a42;
  const D m34 = a41 * a32 - a31 * a42;
  const D m123 = m23 * a13 - m13 * a23 + m12 * a33;
  const D m124 = m24 * a13 - m14 * a23 + m12 * a43;
  const D m134 = m34 * a13 - m14 * a33 + m13 * a43;
  const D m234 = m34 * a23 - m24 * a33 + m23 * a43;
  return m234 * a14 - m134 * a24 + m124 * a34 - m123 * a44;
}
template <class R>
inline R rmax(R a, R b) {
  return std::fmax(a, b);
}

// Per-thread operation counters (algorithmic work of the reference path).
struct Counters {
  long long hs = 0, vc = 0, clips = 0, cones = 0, exportv = 0, knn = 0;
};

// ---------------------------------------------------------------------------
// Grid access: the domain restriction's view of Grid (voronoi.cpp:42-144).
template <class R>
struct GridView {
  int size = 0;
  R voxel = 0;
  const char *in_domain = nullptr;
  std::vector<Vec4<R>> points;
  const int *triangles = nullptr;
  const int *tri_list = nullptr;
  const int *offsets = nullptr;
  bool has_border_corners = false;
};

// ---------------------------------------------------------------------------
// One convex cell (the ConvexCell struct and its functions,
// ConvexCell.cl:134-619), restated over per-thread arrays.
template <class R>
struct Cell {
  // caps of the pass
  int capP = 0, capV = 0, capT = 0, vhs = 2;
  R cube_eps = 0;
  const Vec4<R> *pts = nullptr;
  Vec4<R> seed{};
  Status *status = nullptr;
  std::vector<std::array<uint8_t, 4>> vert;
  std::vector<Vec4<R>> plane;
  std::vector<int> pnb;  // neighbour seed of each plane, -1 for box and cone planes (ConvexCell.cl:284-330)
  std::vector<uint8_t> next;
  int nb_vertex = 0, nb_plane = 0;
  Counters *cnt = nullptr;
  // --hessian: facet integrals per plane, HC values each (neighb_intr,
  // ConvexCell.cl:1059-1066); hc == 0: off
  int hc = 0;
  mutable std::vector<R> intr;

  void resize() {
    if (hc > 0) intr.assign(size_t(hc) * (std::max(capP, 1) + 4), R(0));
    vert.assign(256, {0, 0, 0, 0});
    plane.assign(std::max(capP, 1) + 4, Vec4<R>{0, 0, 0, 0});
    pnb.assign(std::max(capP, 1) + 4, -1);
    next.assign(std::max(capP, 1) + 4, 0);
  }

  uint8_t ith(int t, int i) const { return vert[t][i]; }

  // CCInit (ConvexCell.cl:278-308): the domain box [-eps, 1000+eps]^3.
  void init(int id, Status *st) {
    status = st;
    seed = pts[id];
    const R eps = cube_eps;
    const R vmin = -eps;
    const R vmax = 1000 + eps;
    plane[0] = mk<R>(R(1.0), R(0.0), R(0.0), -vmin);
    plane[1] = mk<R>(R(-1.0), R(0.0), R(0.0), vmax);
    plane[2] = mk<R>(R(0.0), R(1.0), R(0.0), -vmin);
    plane[3] = mk<R>(R(0.0), R(-1.0), R(0.0), vmax);
    plane[4] = mk<R>(R(0.0), R(0.0), R(1.0), -vmin);
    plane[5] = mk<R>(R(0.0), R(0.0), R(-1.0), vmax);
    for (int i = 0; i < 6; ++i) pnb[i] = -1;
    nb_plane = 6;
    static const uint8_t cube[8][3] = {{2, 5, 0}, {5, 3, 0}, {1, 5, 2}, {5, 1, 3},
                                       {4, 2, 0}, {4, 0, 3}, {2, 4, 1}, {4, 3, 1}};
    for (int v = 0; v < 8; ++v) vert[v] = {cube[v][0], cube[v][1], cube[v][2], 0};
    nb_vertex = 8;
  }

  // CCNewPlane (ConvexCell.cl:314-333): normalised power bisector; a
  // neighbour with w <= NO_CELL_LIMITS is a wall through its own position.
  int new_plane(unsigned vid) {
    if (nb_plane >= capP) {
      *status = plane_overflow;
      return -1;
    }
    const Vec4<R> B = pts[vid];
    const Vec4<R> dir = sub4(seed, B);
    const Vec4<R> ave2 = add4(seed, B);
    R dot = dot3(ave2, dir) - (B.w - seed.w);
    if (B.w <= kNoCellLimits) dot = 2 * dot3(B, dir);
    const R dir_norm = std::sqrt(dot3(dir, dir));
    plane[nb_plane] = mk<R>(dir.x / dir_norm, dir.y / dir_norm, dir.z / dir_norm, -dot / 2 / dir_norm);
    pnb[nb_plane] = int(vid);
    return nb_plane++;
  }

  void new_vertex(int i, int j, int k) {
    if (nb_vertex >= capV) {
      *status = vertex_overflow;
      return;
    }
    vert[nb_vertex++] = {uint8_t(i), uint8_t(j), uint8_t(k), 0};
  }

  // CCComputeVertexCoordinates (ConvexCell.cl:344-362): cofactor vector of
  // the three planes, optionally divided by its w.
  Vec4<R> vertex_coords(int t, bool persp) const {
    ++cnt->vc;
    const Vec4<R> p1 = plane[vert[t][0]], p2 = plane[vert[t][1]], p3 = plane[vert[t][2]];
    const R m12 = p2.x * p3.y - p2.y * p3.x;
    const R m13 = p2.x * p3.z - p2.z * p3.x;
    const R m14 = p2.x * p3.w - p2.w * p3.x;
    const R m23 = p2.y * p3.z - p2.z * p3.y;
    const R m24 = p2.y * p3.w - p2.w * p3.y;
    const R m34 = p2.z * p3.w - p2.w * p3.z;
    Vec4<R> r;
    r.x = -p1.w * m23 - p1.y * m34 + p1.z * m24;
    r.y = p1.x * m34 + p1.w * m13 - p1.z * m14;
    r.z = -p1.x * m24 + p1.y * m14 - p1.w * m12;
    r.w = p1.x * m23 - p1.y * m13 + p1.z * m12;
    if (persp) return mk<R>(r.x / r.w, r.y / r.w, r.z / r.w, R(1));
    return r;
  }

  // CCIsSecurityRadiusReached (ConvexCell.cl:364-382): the neighbour is
  // farther than twice the farthest vertex.
  bool radius_reached(Vec4<R> last) const {
    R v_dist = 0;
    for (int i = 0; i < nb_vertex; ++i) {
      const Vec4<R> pc = vertex_coords(i, true);
      const Vec4<R> d = sub4(pc, seed);
      v_dist = rmax(dot3(d, d), v_dist);
    }
    const Vec4<R> d = sub4(last, seed);
    return dot3(d, d) > 4 * v_dist;
  }

  // CCVertexIsInHalfSpace (ConvexCell.cl:400-461): sign of
  // det(plane_a, plane_b, plane_c, eqn); true = the vertex is cut away.
  bool in_half_space(int t, Vec4<R> e) {
    ++cnt->hs;
    const Vec4<R> p1 = plane[vert[t][0]], p2 = plane[vert[t][1]], p3 = plane[vert[t][2]];
    if (vhs == 2) {
      const double d = det4<double>(p1.x, p2.x, p3.x, e.x, p1.y, p2.y, p3.y, e.y, p1.z, p2.z, p3.z, e.z, p1.w,
                                    p2.w, p3.w, e.w);
      return d > 0.0;
    }
    if (vhs == 1) {
      // FP32 evaluation with a running magnitude bound; near-zero results
      // flag the cell for exact predicates (ConvexCell.cl:415-448).
      const Vec4<R> pl[3] = {p1, p2, p3};
      auto fmax_abs = [](R a, R b) { return std::fmax(std::fabs(a), std::fabs(b)); };
      auto fmax3 = [](R a, R b, R c) { return std::fmax(std::fmax(a, b), c); };
      R tmp;
      R m12 = pl[1].x * pl[0].y; tmp = -pl[0].x * pl[1].y;
      R M12 = fmax_abs(m12, tmp); m12 += tmp;
      R m13 = pl[2].x * pl[0].y; tmp = -pl[0].x * pl[2].y;
      R M13 = fmax_abs(m13, tmp); m13 += tmp;
      R m14 = e.x * pl[0].y; tmp = -pl[0].x * e.y;
      R M14 = fmax_abs(m14, tmp); m14 += tmp;
      R m23 = pl[2].x * pl[1].y; tmp = -pl[1].x * pl[2].y;
      R M23 = fmax_abs(m23, tmp); m23 += tmp;
      R m24 = e.x * pl[1].y; tmp = -pl[1].x * e.y;
      R M24 = fmax_abs(m24, tmp); m24 += tmp;
      R m34 = e.x * pl[2].y; tmp = -pl[2].x * e.y;
      R M34 = fmax_abs(m34, tmp); m34 += tmp;
      const R m123 = m23 * pl[0].z - m13 * pl[1].z + m12 * pl[2].z;
      const R M123 = fmax3(std::fabs(M23 * pl[0].z), std::fabs(M13 * pl[1].z), std::fabs(M12 * pl[2].z));
      const R m124 = m24 * pl[0].z - m14 * pl[1].z + m12 * e.z;
      const R M124 = fmax3(std::fabs(M24 * pl[0].z), std::fabs(M14 * pl[1].z), std::fabs(M12 * e.z));
      const R m134 = m34 * pl[0].z - m14 * pl[2].z + m13 * e.z;
      const R M134 = fmax3(std::fabs(M34 * pl[0].z), std::fabs(M14 * pl[2].z), std::fabs(M13 * e.z));
      const R m234 = m34 * pl[1].z - m24 * pl[2].z + m23 * e.z;
      const R M234 = fmax3(std::fabs(M34 * pl[1].z), std::fabs(M24 * pl[2].z), std::fabs(M23 * e.z));
      const R res = m234 * pl[0].w - m134 * pl[1].w + m124 * pl[2].w - m123 * e.w;
      const R M1234 = std::fmax(std::fmax(std::fabs(M234 * pl[0].w), std::fabs(M134 * pl[1].w)),
                                std::fmax(std::fabs(M124 * pl[2].w), std::fabs(M123 * e.w)));
      if (std::fabs(res) < 3.e-6 * M1234) {
        *status = needs_exact_predicates;
        return res > -2.e-7 * M1234;
      }
      return res > 0.0f;
    }
    const R d = det4<R>(p1.x, p2.x, p3.x, e.x, p1.y, p2.y, p3.y, e.y, p1.z, p2.z, p3.z, e.z, p1.w, p2.w, p3.w, e.w);
    return d > 0;
  }

  // CCComputeBoundary (ConvexCell.cl:463-515): walks the removed triangles
  // (dual of the removed vertices, parked after nb_vertex) and links the
  // cavity boundary as a circular list over plane ids.
  uint8_t compute_boundary(int nb_removed) {
    for (int i = 0; i < capP; ++i) next[i] = kEndOfList;
    uint8_t first = kEndOfList;
    int iter = 0;
    uint8_t t = uint8_t(nb_vertex);
    while (nb_removed > 0) {
      if (iter++ > 1000) {
        *status = inconsistent_boundary;
        return first;
      }
      bool in_border[3], next_opp[3];
      for (int e = 0; e < 3; ++e) in_border[e] = next[ith(t, e)] != kEndOfList;
      for (int e = 0; e < 3; ++e) next_opp[e] = next[ith(t, (e + 1) % 3)] == ith(t, e);
      bool simple = true;
      for (int e = 0; e < 3; ++e)
        if (!next_opp[e] && !next_opp[(e + 1) % 3] && in_border[(e + 1) % 3]) simple = false;
      if (!next_opp[0] && !next_opp[1] && !next_opp[2]) {
        if (first == kEndOfList) {
          for (int e = 0; e < 3; ++e) next[ith(t, e)] = ith(t, (e + 1) % 3);
          first = vert[t][0];
        } else {
          simple = false;
        }
      }
      if (!simple) {
        t++;
        if (t == nb_vertex + nb_removed) t = uint8_t(nb_vertex);
        continue;
      }
      for (int e = 0; e < 3; ++e)
        if (!next_opp[e]) next[ith(t, e)] = ith(t, (e + 1) % 3);
      for (int e = 0; e < 3; ++e)
        if (next_opp[e] && next_opp[(e + 1) % 3]) {
          if (first == ith(t, (e + 1) % 3)) first = next[ith(t, (e + 1) % 3)];
          next[ith(t, (e + 1) % 3)] = kEndOfList;
        }
      std::swap(vert[t], vert[nb_vertex + nb_removed - 1]);
      t = uint8_t(nb_vertex);
      nb_removed--;
    }
    return first;
  }

  // CCClipByPlane (ConvexCell.cl:517-563).
  void clip(int vid) {
    if (*status == plane_overflow) return;
    ++cnt->clips;
    const Vec4<R> e = plane[vid];
    int nb_removed = 0;
    int i = 0;
    while (i < nb_vertex) {
      if (in_half_space(i, e)) {
        nb_vertex--;
        std::swap(vert[i], vert[nb_vertex]);
        nb_removed++;
      } else {
        i++;
      }
    }
    if (nb_vertex < 1) {
      *status = empty_cell;
      return;
    }
    if (*status == needs_exact_predicates) return;
    if (nb_removed == 0) {
      --nb_plane;
      return;
    }
    const uint8_t first = compute_boundary(nb_removed);
    if (*status != success) return;
    if (first == kEndOfList) return;
    uint8_t cir = first;
    do {
      const int nc = next[cir];
      new_vertex(vid, cir, nc);
      if (*status != success) return;
      cir = uint8_t(nc);
    } while (cir != first);
  }

  static Vec4<R> plane_from_points(Vec4<R> A, Vec4<R> B, Vec4<R> C) {
    Vec4<R> p = cross4(sub4(B, A), sub4(C, A));
    p.w = -dot3(p, A);
    return p;
  }

  // CCClipTetFromPointsInfinite (ConvexCell.cl:565-575): the cone beyond
  // triangle BCD seen from A.
  void clip_cone(Vec4<R> A, Vec4<R> B, Vec4<R> C, Vec4<R> D) {
    ++cnt->cones;
    const Vec4<R> faces[4][3] = {{A, B, C}, {A, D, B}, {A, C, D}, {C, D, B}};
    for (int f = 0; f < 4; ++f) {
      if (nb_plane >= capP) {
        *status = plane_overflow;
        return;
      }
      pnb[nb_plane] = -1;
      plane[nb_plane++] = plane_from_points(faces[f][0], faces[f][1], faces[f][2]);
      clip(nb_plane - 1);
      if (*status != success) return;
    }
  }

  // CCExportBaryVolume (ConvexCell.cl:577-619): per vertex A and each of its
  // planes i, two signed tets (A, C, proj of C on plane i, proj of C on the
  // edge line i/j), C = seed; accumulates (sum w*centroid, sum w)/6 * factor.
  void export_bary(Vec4<R> *out, R factor, double vol_eps2) const {
    Vec4<R> sum_b = mk<R>(0, 0, 0, 0);
    const Vec4<R> C = seed;
    for (int ve = 0; ve < nb_vertex; ++ve) {
      ++cnt->exportv;
      const Vec4<R> A = vertex_coords(ve, true);
      const Vec4<R> AC = sub4(C, A);
      Vec4<R> pl[3], a_plane[3], a_line[3];
      for (int i = 0; i < 3; ++i) pl[i] = plane[ith(ve, i)];
      for (int i = 0; i < 3; ++i) {
        const Vec4<R> ni = pl[i];
        a_plane[i] = sub4(AC, scale4(dot3(AC, ni) / dot3(ni, ni), ni));
      }
      for (int i = 0; i < 3; ++i) {
        const Vec4<R> ninj = cross4(pl[i], pl[(i + 1) % 3]);
        const R ninj2 = dot4(ninj, ninj);
        if (ninj2 < vol_eps2 * dot3(pl[i], pl[i]) * dot3(pl[(i + 1) % 3], pl[(i + 1) % 3]))
          a_line[i] = mk<R>(0, 0, 0, 0);
        else
          a_line[i] = scale4(dot4(AC, ninj) / ninj2, ninj);
      }
      for (int i = 0; i < 3; ++i) {
        for (int st = 0; st < 2; ++st) {
          const int j = (i + 3 - st) % 3;
          const R w = (2 * st - 1) * det3v(AC, a_plane[i], a_line[j]);
          sum_b.w += w;
          const Vec4<R> s = add4(add4(AC, a_plane[i]), a_line[j]);
          sum_b.x += w * (A.x + 0.25 * s.x);
          sum_b.y += w * (A.y + 0.25 * s.y);
          sum_b.z += w * (A.z + 0.25 * s.z);
          if (hc > 0) {
            // CCExportBaryVolumeAndArea (ConvexCell.cl:621-678): the same
            // triangle (A, C's foot on plane i, C's foot on the edge line)
            // in plane i, signed by the plane's normal
            const R tri_area = (2 * st - 1) * factor * det3v(a_plane[i], a_line[j], pl[i]) / 2;
            const int pid = ith(ve, i);
            if (hc == 1) {
              intr[pid] += tri_area;
            } else {
              const Vec4<R> m = add4(a_plane[i], a_line[j]);
              intr[4 * pid + 0] += tri_area * (A.x + m.x / 3);
              intr[4 * pid + 1] += tri_area * (A.y + m.y / 3);
              intr[4 * pid + 2] += tri_area * (A.z + m.z / 3);
              intr[4 * pid + 3] += tri_area;
            }
          }
        }
      }
    }
    *out = add4(*out, scale4(factor / 6, sum_b));
  }
};

// Sorted-union of triangle-id lists, failing past T entries
// (ConvexCell.cl:722-749).
inline bool merge_lists(const int *l1, int n1, const int *l2, int n2, int *res, int *n, int capT) {
  int remain[2] = {n1, n2};
  *n = 0;
  for (int i = 0; i < n1 + n2; ++i) {
    if (remain[0] && remain[1] && l1[0] == l2[0]) {
      --remain[0];
      ++l1;
      ++i;
    }
    if (*n >= capT) return false;
    if (remain[0] != 0 && (remain[1] == 0 || l1[0] < l2[0])) {
      *(res++) = *(l1++);
      --remain[0];
    } else {
      *(res++) = *(l2++);
      --remain[1];
    }
    ++*n;
  }
  return true;
}

// Used cells (ConvexCell.cl:1118-1126, 680-690): relaxed byte accesses, as
// the reference's concurrent work-items race on the same flags.
struct UsedCells {
  uint8_t *flags = nullptr;  // stored order, null: off
  double eps = 0;            // USED_CELL_EPSILON (keepVolume)
  int dist = 0;              // CUSED_CELL_DIST of the main passes (0 or 1)
};

// CCUpdateUsedCell: every plane neighbour of the cell's vertices gets d
// when it has no mark yet.
template <class R>
void mark_neighbours(const Cell<R> &cc, uint8_t *flags, int d) {
  for (int ve = 0; ve < cc.nb_vertex; ++ve)
    for (int i = 0; i < 3; ++i) {
      const int nb = cc.pnb[cc.ith(ve, i)];
      if (nb >= 0 && __atomic_load_n(&flags[nb], __ATOMIC_RELAXED) == 0)
        __atomic_store_n(&flags[nb], uint8_t(d), __ATOMIC_RELAXED);
    }
}

// compute_voro_cell (ConvexCell.cl:812-1116) for one stored seed.
// Hessian rows of one pass's cells (stored order).
template <class R>
struct HessRows {
  int H = 0, HC = 1;
  R *vals = nullptr;  // n*H*HC
  int *ids = nullptr; // n*H
};

template <class R>
void voro_cell(Cell<R> &cc, int seed_id, const unsigned *neigs, int K, const GridView<R> *grid, bool out_domain,
               Status *st_all, Vec4<R> *out_all, double vol_eps2, std::vector<int> &tr0, std::vector<int> &tr1,
               const UsedCells &used, const HessRows<R> &hr) {
  Status *st = st_all + seed_id;
  *st = success;
  if (hr.H > 0) hr.ids[size_t(seed_id) * hr.H] = -1;
  const Vec4<R> *pts = cc.pts;
  if (pts[seed_id].w <= kNoCellLimits) {
    out_all[seed_id] = pts[seed_id];
    return;
  }
  out_all[seed_id] = mk<R>(0, 0, 0, 0);
  cc.init(seed_id, st);
  for (int i = 0; i < K; ++i) {
    const unsigned z = neigs[i];
    const int cur = cc.new_plane(z);
    cc.clip(cur);
    if (*st != success) return;
    if (cc.radius_reached(pts[z])) break;
  }
  if (!cc.radius_reached(pts[neigs[K - 1]])) {
    *st = security_radius_not_reached;
    return;
  }
  if (*st != success) return;

  char in_domain = 1;
  Vec4<R> pt0 = mk<R>(0, 0, 0, 0);
  int tr_size = 0, tr_wh = 0;
  if (grid) {
    // bounding box of the cell -> voxel range (ConvexCell.cl:924-940)
    R bb_min[3], bb_max[3];
    for (int d = 0; d < 3; ++d) {
      bb_min[d] = 1000;
      bb_max[d] = 0;
    }
    for (int ve = 0; ve < cc.nb_vertex; ++ve) {
      const Vec4<R> p = cc.vertex_coords(ve, true);
      const R tp[3] = {p.x, p.y, p.z};
      for (int d = 0; d < 3; ++d)
        if (bb_min[d] > tp[d]) bb_min[d] = tp[d];
      for (int d = 0; d < 3; ++d)
        if (bb_max[d] < tp[d]) bb_max[d] = tp[d];
    }
    const int S = grid->size;
    const R VS = grid->voxel;
    int vmin[3], vmax[3];
    for (int d = 0; d < 3; ++d) vmin[d] = std::max(0, int(bb_min[d] / VS));
    for (int d = 0; d < 3; ++d) vmax[d] = std::min(S - 1, int(bb_max[d] / VS));
    auto gid3 = [S](int x, int y, int z) { return x + y * S + z * S * S; };
    std::vector<int> *lists[2] = {&tr0, &tr1};
    // first corner that is not on the border + merged triangle ids
    // (ConvexCell.cl:950-979)
    for (int z = vmin[2]; z <= vmax[2]; z++) {
      for (int y = vmin[1]; y <= vmax[1]; y++) {
        const int id = gid3(0, y, z);
        for (int x = vmin[0]; x <= vmax[0]; x++) {
          if (in_domain == 1 && grid->in_domain[id + x] != 1) {
            in_domain = grid->in_domain[id + x];
            pt0 = mk<R>(x * VS, y * VS, z * VS, R(1));
          }
          const int lo = grid->offsets[id + x], hi = grid->offsets[id + x + 1];
          if (lo == hi) continue;
          if (!merge_lists(lists[tr_wh]->data(), tr_size, &grid->tri_list[lo], hi - lo, lists[1 - tr_wh]->data(),
                           &tr_size, cc.capT)) {
            *st = triangle_overflow;
            return;
          }
          tr_wh = 1 - tr_wh;
        }
      }
    }
    if (in_domain == 1) {
      if (!out_domain) {
        *st = find_another_beginning_vertex;
        return;
      }
      // look one voxel layer further in +z, +y, +x (ConvexCell.cl:986-1051)
      if (vmax[2] + 1 < S) {
        const int z = vmax[2] + 1;
        for (int y = vmin[1]; y <= vmax[1] + 1; y++) {
          if (y >= S) break;
          const int id = gid3(0, y, z);
          for (int x = vmin[0]; x <= vmax[0] + 1; x++) {
            if (x >= S) break;
            if (grid->in_domain[id + x] != 1) {
              in_domain = grid->in_domain[id + x];
              pt0 = mk<R>(x * VS, y * VS, z * VS, R(1));
              break;
            }
          }
          if (in_domain != 1) break;
        }
      } else {
        in_domain = 0;
        pt0 = mk<R>(vmin[0] * VS, vmin[1] * VS, (vmax[2] + 1) * VS, R(1));
      }
      if (in_domain == 1 && vmax[1] + 1 < S) {
        const int y = vmax[1] + 1;
        for (int z = vmin[2]; z <= vmax[2]; z++) {
          const int id = gid3(0, y, z);
          for (int x = vmin[0]; x <= vmax[0] + 1; x++) {
            if (x >= S) break;
            if (grid->in_domain[id + x] != 1) {
              in_domain = grid->in_domain[id + x];
              pt0 = mk<R>(x * VS, y * VS, z * VS, R(1));
              break;
            }
          }
          if (in_domain != 1) break;
        }
      } else if (in_domain == 1) {
        in_domain = 0;
        pt0 = mk<R>(vmin[0] * VS, (vmax[1] + 1) * VS, vmin[2] * VS, R(1));
      }
      if (in_domain == 1 && vmax[0] + 1 < S) {
        const int x = vmax[0] + 1;
        for (int z = vmin[2]; z <= vmax[2]; z++) {
          for (int y = vmin[1]; y <= vmax[1]; y++) {
            const int id = gid3(0, y, z);
            if (grid->in_domain[id + x] != 1) {
              in_domain = grid->in_domain[id + x];
              pt0 = mk<R>(x * VS, y * VS, z * VS, R(1));
              break;
            }
          }
          if (in_domain != 1) break;
        }
      } else if (in_domain == 1) {
        in_domain = 0;
        pt0 = mk<R>((vmax[0] + 1) * VS, vmin[1] * VS, vmin[2] * VS, R(1));
      }
      if (in_domain == 1) {
        *st = find_another_beginning_vertex;
        return;
      }
    }
  }

  if (cc.hc > 0) std::fill(cc.intr.begin(), cc.intr.end(), R(0));
  const bool add_volume = grid ? in_domain == 2 : true;
  if (add_volume) cc.export_bary(out_all + seed_id, R(1), vol_eps2);

  if (grid && tr_size) {
    // signed cone decomposition over the boundary triangles
    // (ConvexCell.cl:1082-1115), each from a backed-up cell.
    const int bk_nv = cc.nb_vertex, bk_np = cc.nb_plane;
    const Status bk_st = *st;
    std::vector<std::array<uint8_t, 4>> bk_vert(cc.vert.begin(), cc.vert.begin() + bk_nv);
    const std::vector<int> &ids = tr_wh ? tr1 : tr0;
    for (int i = 0; i < tr_size; ++i) {
      const int tri = ids[i];
      const Vec4<R> p1 = grid->points[grid->triangles[3 * tri + 0]];
      Vec4<R> p2 = grid->points[grid->triangles[3 * tri + 1]];
      Vec4<R> p3 = grid->points[grid->triangles[3 * tri + 2]];
      const bool go_out = det3v(sub4(p1, pt0), sub4(p2, pt0), sub4(p3, pt0)) > 0;
      if (!go_out) std::swap(p2, p3);
      cc.clip_cone(pt0, p1, p2, p3);
      auto restore = [&]() {
        cc.nb_vertex = bk_nv;
        cc.nb_plane = bk_np;
        std::copy(bk_vert.begin(), bk_vert.end(), cc.vert.begin());
        *st = bk_st;
      };
      if (*st == empty_cell) {
        restore();
        *st = success;
        continue;
      }
      if (*st != success) {
        out_all[seed_id].w = 0;
        return;
      }
      cc.export_bary(out_all + seed_id, go_out ? R(1.f) : R(-1.f), vol_eps2);
      restore();
    }
  }
  if (used.flags && out_all[seed_id].w >= R(used.eps)) {
    __atomic_store_n(&used.flags[seed_id], uint8_t(1), __ATOMIC_RELAXED);
    if (used.dist >= 1) mark_neighbours(cc, used.flags, 1);
  }
  if (hr.H > 0) {
    // the row: facets with a neighbour and an area above 0.2, in plane
    // order; more than H is hessian_overflow (ConvexCell.cl:1133-1150)
    const int HC = hr.HC;
    int c = 0;
    for (int p = 0; p < cc.nb_plane; ++p) {
      if (cc.pnb[p] < 0 || cc.intr[size_t(HC) * p + HC - 1] <= R(0.2)) continue;
      if (c >= hr.H) {
        *st = hessian_overflow;
        return;
      }
      for (int k = 0; k < HC; ++k) hr.vals[(size_t(seed_id) * hr.H + c) * HC + k] = cc.intr[size_t(HC) * p + k];
      hr.ids[size_t(seed_id) * hr.H + c] = cc.pnb[p];
      ++c;
    }
    if (c < hr.H) hr.ids[size_t(seed_id) * hr.H + c] = -1;
  }
}

// compute_bordering (ConvexCell.cl:756-809): the clipped cell only, then its
// plane neighbours get the mark d.
template <class R>
void border_cell(Cell<R> &cc, int seed_id, const unsigned *neigs, int K, Status *st_all, uint8_t *flags, int d) {
  Status *st = st_all + seed_id;
  *st = success;
  const Vec4<R> *pts = cc.pts;
  if (pts[seed_id].w <= kNoCellLimits) return;
  cc.init(seed_id, st);
  for (int i = 0; i < K; ++i) {
    const unsigned z = neigs[i];
    const int cur = cc.new_plane(z);
    cc.clip(cur);
    if (*st != success) return;
    if (cc.radius_reached(pts[z])) break;
  }
  if (!cc.radius_reached(pts[neigs[K - 1]])) {
    *st = security_radius_not_reached;
    return;
  }
  mark_neighbours(cc, flags, d);
}

// ---------------------------------------------------------------------------
// Binning (knearests.cpp:48-222) with a deterministic stored order: seeds
// sorted by bin, ties by user id (the reference's atomic scatter leaves the
// in-bin order unspecified).
template <class R>
struct Bins {
  int dim = 0;
  std::vector<int> counters;  // dim^3+1
  std::vector<int> perm;      // stored -> user
  std::vector<Vec4<R>> stored;
  std::vector<int> offsets;   // ring table, plus a sentinel entry
  std::vector<R> offset_dists;
  int num_offsets = 0;
};

template <class R>
inline int bin_of(int dim, Vec4<R> p) {
  int i = (int)std::floor(p.x * (R)dim / 1000.f);
  int j = (int)std::floor(p.y * (R)dim / 1000.f);
  int k = (int)std::floor(p.z * (R)dim / 1000.f);
  i = std::max(0, std::min(i, dim - 1));
  j = std::max(0, std::min(j, dim - 1));
  k = std::max(0, std::min(k, dim - 1));
  return i + j * dim + k * dim * dim;
}

// dim = round((n / 3.1)^(1/3)) (knearests.cpp:63), evaluated in double as
// the device engine does.
inline int bins_per_axis(int n) {
  const double d = std::round(std::pow(double(float(n) / 3.1f), double(1.0f / 3)));
  return d < 1 ? 1 : int(d);
}

template <class R>
int make_bins(const std::vector<Vec4<R>> &user, Bins<R> &b, bool ring_table) {
  const int n = int(user.size());
  b.dim = bins_per_axis(n);
  const int dim = b.dim;
  const size_t nb = size_t(dim) * dim * dim;
  std::vector<int> cell(n);
  b.counters.assign(nb + 1, 0);
  for (int i = 0; i < n; ++i) {
    cell[i] = bin_of(dim, user[i]);
    b.counters[cell[i]]++;
  }
  int acc = 0;
  for (auto &c : b.counters) {
    const int v = c;
    c = acc;
    acc += v;
  }
  std::vector<int> pos(b.counters.begin(), b.counters.end() - 1);
  b.perm.assign(n, 0);
  b.stored.assign(n, Vec4<R>{0, 0, 0, 0});
  for (int i = 0; i < n; ++i) {
    const int s = pos[cell[i]]++;
    b.perm[s] = i;
    b.stored[s] = user[i];
  }
  if (!ring_table) return 0;
  // Ring table (knearests.cpp:70-112): linear bin offsets of the Chebyshev
  // shells 1..Nmax-1, each with its squared minimum distance.
  int nmax = 16;
  while (nmax >= 8 && dim < nmax) nmax /= 2;
  if (dim < nmax) return -1;  // the reference exits here (knearests.cpp:72-75)
  b.offsets.assign(1, 0);
  b.offset_dists.assign(1, R(0));
  for (int ring = 1; ring < nmax; ring++) {
    const R d = 1000.f * R(ring - 1) / dim;
    for (int k = -nmax; k <= nmax; k++)
      for (int j = -nmax; j <= nmax; j++)
        for (int i = -nmax; i <= nmax; i++) {
          if (std::max(std::abs(i), std::max(std::abs(j), std::abs(k))) != ring) continue;
          b.offsets.push_back(i + j * dim + k * dim * dim);
          b.offset_dists.push_back(d * d);
        }
  }
  b.num_offsets = int(b.offsets.size());
  // The reference kernel's do/while reads one entry past the table
  // (knearests.cl:57-73); a sentinel that always stops the scan makes that
  // read defined.
  b.offsets.push_back(0);
  b.offset_dists.push_back(std::numeric_limits<R>::infinity());
  return 0;
}

// build_knearests (knearests.cl:36-78): per-seed max-heap of the K best over
// the ring-ordered bins, early exit on the ring bound, heap-sorted.
template <class R>
void knn_reference_order(const Bins<R> &b, const int *ids, int num, int K, unsigned *out, Counters &cnt) {
  std::vector<R> hd(K);
  std::vector<unsigned> hk(K);
  auto heapify = [&](int node, int size) {
    int j = node;
    while (true) {
      const int l = 2 * j + 1, r = 2 * j + 2;
      int largest = j;
      if (l < size && hd[l] > hd[largest]) largest = l;
      if (r < size && hd[r] > hd[largest]) largest = r;
      if (largest == j) return;
      std::swap(hd[j], hd[largest]);
      std::swap(hk[j], hk[largest]);
      j = largest;
    }
  };
  const int maxc = b.dim * b.dim * b.dim;
  for (int g = 0; g < num; ++g) {
    const int pin = ids[g];
    const Vec4<R> p = b.stored[pin];
    const int cin = bin_of(b.dim, p);
    for (int i = 0; i < K; ++i) {
      hd[i] = FLT_MAX;
      hk[i] = UINT_MAX;
    }
    for (int o = 0; o <= b.num_offsets; ++o) {
      if (hd[0] < b.offset_dists[o]) break;
      const int c = cin + b.offsets[o];
      if (c < 0 || c >= maxc) continue;
      for (int ptr = b.counters[c]; ptr < b.counters[c + 1]; ptr++) {
        if (ptr == pin) continue;
        ++cnt.knn;
        const Vec4<R> q = b.stored[ptr];
        const R d = (q.x - p.x) * (q.x - p.x) + (q.y - p.y) * (q.y - p.y) + (q.z - p.z) * (q.z - p.z);
        if (d < hd[0]) {
          hd[0] = d;
          hk[0] = unsigned(ptr);
          heapify(0, K);
        }
      }
    }
    for (int size = K; size;) {
      std::swap(hd[0], hd[size - 1]);
      std::swap(hk[0], hk[size - 1]);
      heapify(0, --size);
    }
    for (int i = 0; i < K; ++i) out[size_t(g) * K + i] = hk[i];
  }
}

// Exact K nearest by (distance, stored index), scanning whole Chebyshev
// shells of bins (3-D bin coordinates, no wrap-around) until the K-th best
// is closer than the next shell's bound ((shell-1) * bin width)^2.  This is
// the tie-broken order the device kernel reproduces bit for bit.
template <class R>
void knn_exact(const Bins<R> &b, const int *ids, int num, int K, unsigned *out, Counters &cnt) {
  const int dim = b.dim;
  std::vector<std::pair<R, unsigned>> best;
  best.reserve(K + 1);
  for (int g = 0; g < num; ++g) {
    const int pin = ids[g];
    const Vec4<R> p = b.stored[pin];
    const int cin = bin_of(dim, p);
    const int cx = cin % dim, cy = (cin / dim) % dim, cz = cin / (dim * dim);
    best.clear();
    for (int ring = 0; ring <= dim; ++ring) {
      const R dr = 1000.f * R(ring - 1) / dim;
      const R bound = ring == 0 ? R(0) : dr * dr;
      if (int(best.size()) == K && best.back().first < bound) break;
      if (ring > 0 && cx - ring < 0 && cy - ring < 0 && cz - ring < 0 && cx + ring >= dim && cy + ring >= dim &&
          cz + ring >= dim)
        break;  // the shell lies entirely outside the grid
      for (int k = -ring; k <= ring; ++k) {
        const int z = cz + k;
        if (z < 0 || z >= dim) continue;
        for (int j = -ring; j <= ring; ++j) {
          const int y = cy + j;
          if (y < 0 || y >= dim) continue;
          const bool face = std::abs(k) == ring || std::abs(j) == ring;
          for (int i = -ring; i <= ring; i += (face ? 1 : 2 * std::max(ring, 1))) {
            const int x = cx + i;
            if (x < 0 || x >= dim) continue;
            const int c = x + y * dim + z * dim * dim;
            for (int ptr = b.counters[c]; ptr < b.counters[c + 1]; ptr++) {
              if (ptr == pin) continue;
              ++cnt.knn;
              const Vec4<R> q = b.stored[ptr];
              const R d = (q.x - p.x) * (q.x - p.x) + (q.y - p.y) * (q.y - p.y) + (q.z - p.z) * (q.z - p.z);
              const std::pair<R, unsigned> e(d, unsigned(ptr));
              if (int(best.size()) == K && !(e < best.back())) continue;
              best.insert(std::upper_bound(best.begin(), best.end(), e), e);
              if (int(best.size()) > K) best.pop_back();
            }
            if (ring == 0) break;
          }
        }
      }
    }
    for (int i = 0; i < K; ++i) out[size_t(g) * K + i] = i < int(best.size()) ? best[i].second : UINT_MAX;
  }
}

// ---------------------------------------------------------------------------
// Reference kernels compiled for the CPU (oracle/_ref), loaded on demand.
typedef void (*RefCellFn)(const RefCellArgs *);
typedef void (*RefKnnFn)(const RefKnnArgs *);
struct RefLib {
  void *h = nullptr;
  std::string path;
  bool tried = false;
};
RefLib g_ref;

void *ref_sym(const char *name) {
  if (!g_ref.tried) {
    g_ref.tried = true;
    Dl_info info;
    std::string dir = ".";
    if (dladdr((void *)&oracle_ref_library, &info) && info.dli_fname) {
      dir = info.dli_fname;
      const size_t s = dir.rfind('/');
      dir = s == std::string::npos ? "." : dir.substr(0, s);
    }
    const char *env = std::getenv("RPD_ORACLE_REF_LIB");
    g_ref.path = env ? env : dir + "/_ref/libref_kernels.so";
    g_ref.h = dlopen(g_ref.path.c_str(), RTLD_NOW | RTLD_LOCAL);
  }
  return g_ref.h ? dlsym(g_ref.h, name) : nullptr;
}

// ---------------------------------------------------------------------------
// The solver: VoroAlgo::launch (voronoi.cpp:1244-1403) over either kernel set.
template <class R>
struct Solver {
  const OracleParams &prm;
  const GridView<R> *grid;
  Bins<R> bins;
  std::vector<Status> status;
  std::vector<Vec4<R>> out;
  std::vector<uint8_t> used;  // used-cell marks (stored order) when keep_distance >= 0 with a grid
  UsedCells uc;
  std::vector<R> hess;        // Hessian rows (stored order) when prm.H > 0
  std::vector<int> hess_ids;
  OracleStats *stats;
  Counters total;
  // VOLUME_EPSILON2 is a double literal in both builds (voronoi.cpp:919,922).
  double vol_eps2;

  Solver(const OracleParams &p, const GridView<R> *g, OracleStats *s) : prm(p), grid(g), stats(s) {
    vol_eps2 = std::is_same<R, double>::value ? 1.e-12 : 1.e-6;
  }
  int nthreads() const { return prm.nthreads > 0 ? prm.nthreads : omp_get_max_threads(); }

  bool knn(const std::vector<int> &ids, int K, std::vector<unsigned> &nn) {
    const int num = int(ids.size());
    nn.assign(size_t(num) * K, UINT_MAX);
    if (!num) return true;
    const double t0 = now_s();
    if (prm.kernels == 1) {
      RefKnnFn fn = (RefKnnFn)ref_sym(std::is_same<R, double>::value ? "ref_knn_d" : "ref_knn_f");
      if (!fn) return false;
      RefKnnArgs a{};
      a.dim = bins.dim;
      a.counters = bins.counters.data();
      a.stored = bins.stored.data();
      a.num_offsets = bins.num_offsets;
      a.offsets = bins.offsets.data();
      a.offset_dists = bins.offset_dists.data();
      a.ids = ids.data();
      a.num = num;
      a.offset = 0;
      a.out = nn.data();
      a.k = K;
      a.nthreads = nthreads();
      fn(&a);
    } else {
      const int nth = nthreads();
      std::vector<Counters> cs(nth);
#pragma omp parallel num_threads(nth)
      {
        const int tid = omp_get_thread_num();
#pragma omp for schedule(dynamic, 1)
        for (int g0 = 0; g0 < num; g0 += 64) {
          const int cnt = std::min(64, num - g0);
          if (prm.knn_mode == 1)
            knn_exact(bins, ids.data() + g0, cnt, K, nn.data() + size_t(g0) * K, cs[tid]);
          else
            knn_reference_order(bins, ids.data() + g0, cnt, K, nn.data() + size_t(g0) * K, cs[tid]);
        }
      }
      for (auto &c : cs) total.knn += c.knn;
    }
    if (stats) stats->knn_seconds += now_s() - t0;
    return true;
  }

  // bordering_d > 0: the bordering kernel (mark d), on a scratch status
  bool cells(const std::vector<int> &ids, const std::vector<unsigned> &nn, int K, int P, int V, int T, int vhs,
             bool out_domain, int bordering_d = 0) {
    const int num = int(ids.size());
    if (!num) return true;
    const double t0 = now_s();
    std::vector<Status> scratch;
    Status *st_out = status.data();
    if (bordering_d > 0) {
      scratch.assign(status.size(), success);
      st_out = scratch.data();
    }
    if (prm.kernels == 1) {
      std::string name = "ref_cell_";
      name += std::is_same<R, double>::value ? std::string("d") : "f" + std::to_string(vhs);
      if (bordering_d > 0)
        name += "_border" + std::to_string(bordering_d);
      else
        name += grid ? (out_domain ? "_gridout" : "_grid") : "_nogrid";
      if (bordering_d == 0 && uc.flags) name += "_used" + std::to_string(uc.dist);
      if (bordering_d == 0 && prm.H > 0) name += "_h" + std::to_string(prm.HC);
      RefCellFn fn = (RefCellFn)ref_sym(name.c_str());
      if (!fn) return false;
      std::vector<unsigned> uids(ids.begin(), ids.end());
      RefCellArgs a{};
      a.num = num;
      a.ids = uids.data();
      a.ids_offset = 0;
      a.pts = bins.stored.data();
      a.neigs = nn.data();
      if (grid) {
        a.grid_in_domain = grid->in_domain;
        a.grid_points = grid->points.data();
        a.grid_triangles = grid->triangles;
        a.grid_tri_list = grid->tri_list;
        a.grid_offsets = grid->offsets;
        a.grid_size = grid->size;
        a.voxel_size = double(grid->voxel);
      }
      a.cube_eps = prm.cube_eps;  // the bordering program keeps CUBE_EPSILON (voronoi.cpp:929)
      a.status = (int *)st_out;
      a.out = out.data();
      a.k = K;
      a.p = P;
      a.v = V;
      a.t = T;
      a.nthreads = nthreads();
      a.used = uc.flags;
      a.used_eps = uc.eps;
      if (prm.H > 0) {
        a.hessian = hess.data();
        a.hessidx = hess_ids.data();
        a.h = prm.H;
      }
      fn(&a);
    } else {
      const int nth = nthreads();
      std::vector<Counters> cs(nth);
#pragma omp parallel num_threads(nth)
      {
        const int tid = omp_get_thread_num();
        Cell<R> cc;
        cc.capP = P;
        cc.capV = V;
        cc.capT = T;
        cc.vhs = std::is_same<R, double>::value ? 2 : vhs;
        cc.cube_eps = R(prm.cube_eps);
        cc.pts = bins.stored.data();
        cc.cnt = &cs[tid];
        cc.hc = prm.H > 0 ? prm.HC : 0;
        cc.resize();
        HessRows<R> hr;
        if (prm.H > 0) {
          hr.H = prm.H;
          hr.HC = prm.HC;
          hr.vals = hess.data();
          hr.ids = hess_ids.data();
        }
        std::vector<int> tr0(std::max(T, 1) + 1), tr1(std::max(T, 1) + 1);
#pragma omp for schedule(dynamic, 16)
        for (int g = 0; g < num; ++g) {
          if (bordering_d > 0)
            border_cell<R>(cc, ids[g], nn.data() + size_t(g) * K, K, st_out, uc.flags, bordering_d);
          else
            voro_cell<R>(cc, ids[g], nn.data() + size_t(g) * K, K, grid, out_domain, status.data(), out.data(),
                         vol_eps2, tr0, tr1, uc, hr);
        }
      }
      for (auto &c : cs) {
        total.hs += c.hs;
        total.vc += c.vc;
        total.clips += c.clips;
        total.cones += c.cones;
        total.exportv += c.exportv;
      }
    }
    if (stats) stats->cell_seconds += now_s() - t0;
    return true;
  }

  // VoroAlgoComputeData::launch (voronoi.cpp:861-1036): one pass = kNN of the
  // ids with this pass's K, then the cell kernel.
  bool pass(const std::vector<int> &ids, int K, int P, int V, int T, int vhs, bool out_domain, int bordering_d = 0) {
    if (stats && stats->npasses < 8) {
      stats->pass_cells[stats->npasses] = int(ids.size());
    }
    const double t0 = now_s();
    if (ids.empty()) return true;
    if (P >= 256) return false;  // voronoi.cpp:867-870
    std::vector<unsigned> nn;
    if (!knn(ids, K, nn)) return false;
    const bool ok = cells(ids, nn, K, P, V, T, vhs, out_domain, bordering_d);
    if (stats && stats->npasses < 8) stats->pass_seconds[stats->npasses] = now_s() - t0;
    return ok;
  }
  void count_pass() {
    if (stats) stats->npasses++;
  }

  // recomputeIds (voronoi.cpp:770-859): failing ids, those matching `cond`,
  // and the status histogram of the failing ones.
  template <class Cond>
  void recompute(std::vector<int> &ids0, std::vector<int> &ids1, std::array<int, kStatusNum> &hist, Cond cond) {
    std::vector<int> n0;
    ids1.clear();
    hist.fill(0);
    for (int s : ids0) {
      const Status st = status[s];
      if (st == success) continue;
      hist[st]++;
      n0.push_back(s);
      if (cond(st)) ids1.push_back(s);
    }
    ids0.swap(n0);
  }

  int run(const std::vector<Vec4<R>> &user) {
    const int n = int(user.size());
    if (make_bins(user, bins, prm.kernels == 1 || prm.knn_mode == 0) < 0) return -2;
    status.assign(n, success);
    out.assign(n, Vec4<R>{0, 0, 0, 0});
    if (prm.H > 0) {
      hess.assign(size_t(n) * prm.H * prm.HC, R(0));
      hess_ids.assign(size_t(n) * prm.H, -1);
    }
    const bool dbl = std::is_same<R, double>::value;
    // used cells only with a grid (voronoi.cpp:1291); the main passes mark at
    // distance 0 or 1 (voronoi.cpp:1286)
    if (grid && prm.used_cells && prm.keep_distance >= 0) {
      used.assign(n, 0);
      uc.flags = used.data();
      uc.eps = prm.keep_volume;
      uc.dist = std::min(prm.keep_distance, 1);
    }
    int K = prm.K, P = prm.P, V = prm.V, T = prm.T;
    const int rc = passes(K, P, V, T, dbl);
    if (rc < 0) return rc;
    // bordering passes (voronoi.cpp:1381-1393) with the last caps: the cells
    // marked d-1 that are not used themselves mark their neighbours d
    if (uc.flags) {
      for (int d = 2; d <= prm.keep_distance; ++d) {
        std::vector<int> bids;
        for (int i = 0; i < n; ++i)
          if (used[i] + 1 == d && out[i].w < R(prm.keep_volume)) bids.push_back(i);
        if (bids.empty()) break;
        if (!pass(bids, K, P, V, T, dbl ? 2 : prm.vhs1, false, d)) return -3;
        count_pass();
      }
    }
    return 0;
  }

  int passes(int &K, int &P, int &V, int &T, bool dbl) {
    const int n = int(status.size());
    std::vector<int> ids0, ids1;
    const int stride = prm.sample_stride > 1 ? prm.sample_stride : 1;
    for (int i = 0; i < n; i += stride) ids0.push_back(i);
    std::array<int, kStatusNum> hist{};
    // pass "first": T=0 defers every boundary cell (voronoi.cpp:1275-1297)
    const int T_first = prm.first_pass_only ? prm.T : 0;
    if (!pass(ids0, prm.K, prm.P, prm.V, T_first, prm.vhs0, false)) return -3;
    count_pass();
    if (prm.first_pass_only) return 0;
    recompute(ids0, ids1, hist, [](Status s) { return s == triangle_overflow; });
    // pass "tr_overflow" (voronoi.cpp:1304-1310)
    if (!ids1.empty()) {
      if (!pass(ids1, prm.K, prm.P, prm.V, prm.T, prm.vhs0, false)) return -3;
      count_pass();
    }
    if (!ids0.empty()) {
      // extra passes with growing caps (voronoi.cpp:1311-1376)
      const int vhs = dbl ? 2 : prm.vhs1;
      const bool out_domain = grid && grid->has_border_corners;
      recompute(ids0, ids1, hist, [](Status) { return true; });
      for (int step = 0; step < prm.max_extra_passes; ++step) {
        if (!dbl && step > 0 && vhs <= 1) break;
        bool relaunch = false;
        if (hist[vertex_overflow]) { relaunch = true; V = int(V * 1.5); }
        if (hist[plane_overflow]) { relaunch = true; P = int(P * 1.5); }
        if (hist[security_radius_not_reached]) { relaunch = true; K = int(K * 1.5); }
        if (hist[triangle_overflow]) { relaunch = true; T = int(T * 1.5); }
        if (!relaunch) break;
        if (!pass(ids1, K, P, V, T, vhs, out_domain)) break;
        count_pass();
        recompute(ids0, ids1, hist, [](Status s) { return s != empty_cell; });
      }
    }
    return 0;
  }
};

template <class R>
GridView<R> make_grid_view(const OracleGrid *g) {
  GridView<R> v;
  v.size = g->size;
  v.voxel = R(g->voxel_size);
  v.in_domain = g->in_domain;
  v.points.resize(g->npoints);
  for (int i = 0; i < g->npoints; ++i)
    v.points[i] = mk<R>(R(g->points[4 * i]), R(g->points[4 * i + 1]), R(g->points[4 * i + 2]), R(0));
  v.triangles = g->triangles;
  v.tri_list = g->tri_list;
  v.offsets = g->offsets;
  const size_t nv = size_t(g->size) * g->size * g->size;
  for (size_t i = 0; i < nv; ++i)
    if (g->in_domain[i] == 1) {
      v.has_border_corners = true;
      break;
    }
  return v;
}

template <class R>
int solve_t(const double *xyzw, int n, const OracleGrid *grid, const OracleParams *p, double *bary, int *status,
            OracleStats *stats, unsigned char *used_out = nullptr, double *hess_out = nullptr,
            int *hess_ids_out = nullptr) {
  std::vector<Vec4<R>> user(n);
  for (int i = 0; i < n; ++i)
    user[i] = mk<R>(R(xyzw[4 * i]), R(xyzw[4 * i + 1]), R(xyzw[4 * i + 2]), R(xyzw[4 * i + 3]));
  GridView<R> gv;
  if (grid) gv = make_grid_view<R>(grid);
  Solver<R> s(*p, grid ? &gv : nullptr, stats);
  const int rc = s.run(user);
  if (rc < 0) return rc;
  for (int st = 0; st < n; ++st) {
    const int u = s.bins.perm[st];
    const Vec4<R> o = s.out[st];
    bary[4 * u + 0] = double(o.x);
    bary[4 * u + 1] = double(o.y);
    bary[4 * u + 2] = double(o.z);
    bary[4 * u + 3] = double(o.w);
    if (status) status[u] = int(s.status[st]);
    if (used_out) used_out[u] = s.used.empty() ? 0 : s.used[st];
    if (hess_out && p->H > 0) {
      const size_t H = size_t(p->H), HC = size_t(p->HC);
      for (size_t k = 0; k < H * HC; ++k) hess_out[u * H * HC + k] = double(s.hess[st * H * HC + k]);
      for (size_t k = 0; k < H; ++k) {
        const int v = s.hess_ids[st * H + k];
        hess_ids_out[u * H + k] = v < 0 ? -1 : s.bins.perm[v];
      }
    }
    if (stats && s.status[st] >= 0 && s.status[st] < kStatusNum) stats->final_status[s.status[st]]++;
  }
  if (stats) {
    stats->hs_tests = s.total.hs;
    stats->vertex_evals = s.total.vc;
    stats->plane_clips = s.total.clips;
    stats->cone_clips = s.total.cones;
    stats->export_vertices = s.total.exportv;
    stats->knn_candidates = s.total.knn;
  }
  return 0;
}

template <class R>
int knn_t(const double *xyzw, int n, int K, int kernels, int mode, int *knn, int nthreads) {
  std::vector<Vec4<R>> user(n);
  for (int i = 0; i < n; ++i)
    user[i] = mk<R>(R(xyzw[4 * i]), R(xyzw[4 * i + 1]), R(xyzw[4 * i + 2]), R(xyzw[4 * i + 3]));
  OracleParams prm{};
  prm.kernels = kernels;
  prm.knn_mode = mode;
  prm.nthreads = nthreads;
  Solver<R> s(prm, nullptr, nullptr);
  if (make_bins(user, s.bins, kernels == 1 || mode == 0) < 0) return -2;
  std::vector<int> ids(n);
  for (int i = 0; i < n; ++i) ids[i] = i;
  std::vector<unsigned> nn;
  if (!s.knn(ids, K, nn)) return -4;
  for (int st = 0; st < n; ++st) {
    const int u = s.bins.perm[st];
    for (int k = 0; k < K; ++k) {
      const unsigned v = nn[size_t(st) * K + k];
      knn[size_t(u) * K + k] = v == UINT_MAX ? -1 : s.bins.perm[v];
    }
  }
  return 0;
}

}  // namespace

extern "C" {

int oracle_solve(const double *xyzw, int n, const OracleGrid *grid, const OracleParams *p, double *bary, int *status,
                 OracleStats *stats) {
  if (n <= 0 || !xyzw || !p || !bary) return -1;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (p->use_double) return solve_t<double>(xyzw, n, grid, p, bary, status, stats);
  return solve_t<float>(xyzw, n, grid, p, bary, status, stats);
}

int oracle_solve_used(const double *xyzw, int n, const OracleGrid *grid, const OracleParams *p, double *bary,
                      int *status, unsigned char *used, OracleStats *stats) {
  if (n <= 0 || !xyzw || !p || !bary || !used) return -1;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (p->use_double) return solve_t<double>(xyzw, n, grid, p, bary, status, stats, used);
  return solve_t<float>(xyzw, n, grid, p, bary, status, stats, used);
}

int oracle_solve_hessian(const double *xyzw, int n, const OracleGrid *grid, const OracleParams *p, double *bary,
                         int *status, double *hess, int *hess_ids, OracleStats *stats) {
  if (n <= 0 || !xyzw || !p || !bary || p->H <= 0 || (p->HC != 1 && p->HC != 4) || !hess || !hess_ids) return -1;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (p->use_double) return solve_t<double>(xyzw, n, grid, p, bary, status, stats, nullptr, hess, hess_ids);
  return solve_t<float>(xyzw, n, grid, p, bary, status, stats, nullptr, hess, hess_ids);
}

int oracle_knn(const double *xyzw, int n, int K, int use_double, int kernels, int knn_mode, int *knn, int nthreads) {
  if (n <= 0 || K <= 0 || !xyzw || !knn) return -1;
  if (use_double) return knn_t<double>(xyzw, n, K, kernels, knn_mode, knn, nthreads);
  return knn_t<float>(xyzw, n, K, kernels, knn_mode, knn, nthreads);
}

int oracle_bin(const double *xyzw, int n, int use_double, int *perm, int *counters) {
  if (n <= 0 || !xyzw) return -1;
  auto go = [&](auto tag) {
    using R = decltype(tag);
    std::vector<Vec4<R>> user(n);
    for (int i = 0; i < n; ++i)
      user[i] = mk<R>(R(xyzw[4 * i]), R(xyzw[4 * i + 1]), R(xyzw[4 * i + 2]), R(xyzw[4 * i + 3]));
    Bins<R> b;
    make_bins(user, b, false);
    if (perm) std::copy(b.perm.begin(), b.perm.end(), perm);
    if (counters) std::copy(b.counters.begin(), b.counters.end(), counters);
    return b.dim;
  };
  return use_double ? go(double(0)) : go(float(0));
}

const char *oracle_ref_library(void) {
  ref_sym("ref_knn_f");
  return g_ref.h ? g_ref.path.c_str() : nullptr;
}

void oracle_grid_invariants(const OracleGrid *g, double *out4) {
  // Grid::getVolume / getBarycenter (Grid.cpp:19-51): tets from the origin.
  double acc[4] = {0, 0, 0, 0};
  for (int t = 0; t < g->ntri; ++t) {
    const double *a = g->points + 4 * g->triangles[3 * t];
    const double *b = g->points + 4 * g->triangles[3 * t + 1];
    const double *c = g->points + 4 * g->triangles[3 * t + 2];
    const double v = -det3<double>(a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]) / 6;
    for (int d = 0; d < 3; ++d) acc[d] += v / 4 * (a[d] + b[d] + c[d]);
    acc[3] += v;
  }
  std::memcpy(out4, acc, sizeof(acc));
}

}  // extern "C"
