// Restricted power cell of every seed, one warp per cell.  Replaces the
// reference's one-work-item compute_voro_cell (ConvexCell.cl:812-1116).
//
// Geometry is in the seed's local frame (seed at the origin): planes are
// (n, d) in double with the kept side n.x + d >= 0, built from the exact
// seed-relative neighbour vector (float inputs, differences exact in
// double).  A vertex is the triple of its planes (a, b, c) plus the cofactor
// vector c of det(pi_a, pi_b, pi_c, e), so that the reference's FP64
// half-space predicate det(...) > 0 (ConvexCell.cl:402-414, VHSAlgo 2) is
// e . c > 0: four DFMA per test.  The vertex position is c.xyz / c.w.  In
// the seed's frame every coordinate is of the cell's size, so thin boundary
// slivers keep their relative accuracy.
//
// Per warp, shared memory holds the planes, the vertices (SoA), the cavity
// scratch and, with a domain, a backup of the Voronoi cell.  One clip:
//   1. every lane tests its vertices (v = lane + 32 s) -> ballot masks;
//   2. boundary edges of the removed dual triangles = directed edges (u, v)
//      whose twin (v, u) is not removed; they must form one cycle over the
//      planes (else inconsistent_boundary, ConvexCell.cl:463-515);
//   3. survivors are compacted by moving the ones past the new count into
//      holes; new vertices (new plane, u, v) fill the remaining holes.
// The cell's security radius (ConvexCell.cl:364-382) uses the cached |p|^2
// of every vertex.  Integration (ConvexCell.cl:577-619) runs per vertex in
// double and is reduced across the warp.
#include <algorithm>

#include "cell.cuh"

namespace rpd {

namespace {

constexpr unsigned kNone = 0xffffffffu;
constexpr double kVolEps2 = 1e-12;  // VOLUME_EPSILON2 of the FP64 build (voronoi.cpp:922)

struct Layout {
  int Pc, Vc, G;
  unsigned o_plane, o_cx, o_cy, o_cz, o_cw, o_d2, o_tri, o_next, o_rem, o_hole, o_edge;
  unsigned o_bcx, o_bcy, o_bcz, o_bcw, o_bd2, o_btri, o_tlist;
  unsigned total;
};

__host__ __device__ inline unsigned align16(unsigned x) { return (x + 15u) & ~15u; }

__host__ __device__ inline int pow2_at_least(int x) {
  int g = 32;
  while (g < x) g <<= 1;
  return g;
}

__host__ __device__ inline Layout make_layout(int P, int V, int T, bool grid) {
  Layout L;
  L.Pc = (P + 3) & ~3;
  L.Vc = (V + 31) & ~31;
  L.G = grid ? pow2_at_least(2 * T) : 0;
  unsigned o = 0;
  L.o_plane = o; o = align16(o + 32u * L.Pc);
  L.o_cx = o; o = align16(o + 8u * L.Vc);
  L.o_cy = o; o = align16(o + 8u * L.Vc);
  L.o_cz = o; o = align16(o + 8u * L.Vc);
  L.o_cw = o; o = align16(o + 8u * L.Vc);
  L.o_d2 = o; o = align16(o + 8u * L.Vc);
  L.o_tri = o; o = align16(o + 4u * L.Vc);
  L.o_next = o; o = align16(o + 4u * L.Pc);
  L.o_rem = o; o = align16(o + 4u * L.Vc);
  L.o_hole = o; o = align16(o + 4u * L.Vc);
  L.o_edge = o; o = align16(o + 4u * L.Vc);
  if (grid) {
    L.o_bcx = o; o = align16(o + 8u * L.Vc);
    L.o_bcy = o; o = align16(o + 8u * L.Vc);
    L.o_bcz = o; o = align16(o + 8u * L.Vc);
    L.o_bcw = o; o = align16(o + 8u * L.Vc);
    L.o_bd2 = o; o = align16(o + 8u * L.Vc);
    L.o_btri = o; o = align16(o + 4u * L.Vc);
    L.o_tlist = o; o = align16(o + 4u * L.G);
  } else {
    L.o_bcx = L.o_bcy = L.o_bcz = L.o_bcw = L.o_bd2 = L.o_btri = L.o_tlist = 0;
  }
  L.total = o;
  return L;
}

struct Plane {
  double x, y, z, w;
};

// Per-warp views into shared memory.
struct WarpCell {
  Plane *plane;
  double *cx, *cy, *cz, *cw, *d2;
  unsigned *tri, *next, *rem, *hole, *edge;
  double *bcx, *bcy, *bcz, *bcw, *bd2;
  unsigned *btri;
  int *tlist;
  int nv, np;  // vertex and plane counts (warp-uniform)
};

__device__ __forceinline__ WarpCell bind(unsigned char *base, const Layout &L) {
  WarpCell w;
  w.plane = reinterpret_cast<Plane *>(base + L.o_plane);
  w.cx = reinterpret_cast<double *>(base + L.o_cx);
  w.cy = reinterpret_cast<double *>(base + L.o_cy);
  w.cz = reinterpret_cast<double *>(base + L.o_cz);
  w.cw = reinterpret_cast<double *>(base + L.o_cw);
  w.d2 = reinterpret_cast<double *>(base + L.o_d2);
  w.tri = reinterpret_cast<unsigned *>(base + L.o_tri);
  w.next = reinterpret_cast<unsigned *>(base + L.o_next);
  w.rem = reinterpret_cast<unsigned *>(base + L.o_rem);
  w.hole = reinterpret_cast<unsigned *>(base + L.o_hole);
  w.edge = reinterpret_cast<unsigned *>(base + L.o_edge);
  w.bcx = reinterpret_cast<double *>(base + L.o_bcx);
  w.bcy = reinterpret_cast<double *>(base + L.o_bcy);
  w.bcz = reinterpret_cast<double *>(base + L.o_bcz);
  w.bcw = reinterpret_cast<double *>(base + L.o_bcw);
  w.bd2 = reinterpret_cast<double *>(base + L.o_bd2);
  w.btri = reinterpret_cast<unsigned *>(base + L.o_btri);
  w.tlist = reinterpret_cast<int *>(base + L.o_tlist);
  w.nv = w.np = 0;
  return w;
}

__device__ __forceinline__ unsigned lanemask_lt(int lane) { return (1u << lane) - 1u; }

// One trace record (lane 0 only): kind, 4 plane or point values, 7 extras.
__device__ __forceinline__ void trace_rec(double *tr, int cap, int lane, double kind, double a, double b, double c,
                                          double d, double e0 = 0, double e1 = 0, double e2 = 0, double e3 = 0,
                                          double e4 = 0, double e5 = 0, double e6 = 0) {
  if (!tr || lane != 0) return;
  const int i = int(tr[0]);
  if (i >= cap) return;
  double *r = tr + 1 + size_t(i) * kTraceRecord;
  r[0] = kind; r[1] = a; r[2] = b; r[3] = c; r[4] = d;
  r[5] = e0; r[6] = e1; r[7] = e2; r[8] = e3; r[9] = e4; r[10] = e5; r[11] = e6;
  tr[0] = i + 1;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ int warp_sumi(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ Plane shfl_plane(Plane v, int src) {
  v.x = __shfl_sync(kFull, v.x, src);
  v.y = __shfl_sync(kFull, v.y, src);
  v.z = __shfl_sync(kFull, v.z, src);
  v.w = __shfl_sync(kFull, v.w, src);
  return v;
}

// Cofactor vector c of det(p1, p2, p3, e) = e . c, with the 2x2-minor
// expansion of the reference's det4x4 (ConvexCell.cl:79-97), in double.
__device__ __forceinline__ void cofactor(const Plane &p1, const Plane &p2, const Plane &p3, double &cx, double &cy,
                                         double &cz, double &cw) {
  const double a11 = p1.x, a21 = p1.y, a31 = p1.z, a41 = p1.w;
  const double a12 = p2.x, a22 = p2.y, a32 = p2.z, a42 = p2.w;
  const double a13 = p3.x, a23 = p3.y, a33 = p3.z, a43 = p3.w;
  const double m12 = a21 * a12 - a11 * a22;
  const double m13 = a31 * a12 - a11 * a32;
  const double m14 = a41 * a12 - a11 * a42;
  const double m23 = a31 * a22 - a21 * a32;
  const double m24 = a41 * a22 - a21 * a42;
  const double m34 = a41 * a32 - a31 * a42;
  const double m123 = m23 * a13 - m13 * a23 + m12 * a33;
  const double m124 = m24 * a13 - m14 * a23 + m12 * a43;
  const double m134 = m34 * a13 - m14 * a33 + m13 * a43;
  const double m234 = m34 * a23 - m24 * a33 + m23 * a43;
  cx = m234;
  cy = -m134;
  cz = m124;
  cw = -m123;
}

__device__ __forceinline__ void make_vertex(WarpCell &w, int slot, unsigned a, unsigned b, unsigned c) {
  double cx, cy, cz, cw;
  cofactor(w.plane[a], w.plane[b], w.plane[c], cx, cy, cz, cw);
  w.cx[slot] = cx;
  w.cy[slot] = cy;
  w.cz[slot] = cz;
  w.cw[slot] = cw;
  const double inv = 1.0 / cw;
  const double px = cx * inv, py = cy * inv, pz = cz * inv;
  w.d2[slot] = px * px + py * py + pz * pz;
  w.tri[slot] = a | (b << 8) | (c << 16);
}

__device__ __forceinline__ void copy_vertex(WarpCell &w, int dst, int src) {
  w.cx[dst] = w.cx[src];
  w.cy[dst] = w.cy[src];
  w.cz[dst] = w.cz[src];
  w.cw[dst] = w.cw[src];
  w.d2[dst] = w.d2[src];
  w.tri[dst] = w.tri[src];
}

// The domain box [-eps, 1000+eps]^3 as 6 planes and 8 vertices, in the
// reference's plane order and vertex triples (ConvexCell.cl:278-308).
__device__ void init_box(WarpCell &w, float4 s, float eps, int lane) {
  if (lane < 6) {
    const double vmin = -double(eps), vmax = 1000.0 + double(eps);
    const double sc = lane < 2 ? s.x : (lane < 4 ? s.y : s.z);
    const double sign = (lane & 1) ? -1.0 : 1.0;
    // global plane: sign * x + off, off = -vmin (sign +) or vmax (sign -)
    const double off = (lane & 1) ? vmax - sc : sc - vmin;
    Plane p{0.0, 0.0, 0.0, off};
    if (lane < 2) p.x = sign;
    else if (lane < 4) p.y = sign;
    else p.z = sign;
    w.plane[lane] = p;
  }
  __syncwarp();
  if (lane < 8) {
    const unsigned cube[8] = {2u | 5u << 8 | 0u << 16, 5u | 3u << 8 | 0u << 16, 1u | 5u << 8 | 2u << 16,
                              5u | 1u << 8 | 3u << 16, 4u | 2u << 8 | 0u << 16, 4u | 0u << 8 | 3u << 16,
                              2u | 4u << 8 | 1u << 16, 4u | 3u << 8 | 1u << 16};
    const unsigned t = cube[lane];
    make_vertex(w, lane, t & 0xff, (t >> 8) & 0xff, (t >> 16) & 0xff);
  }
  __syncwarp();
  w.nv = 8;
  w.np = 6;
}

template <int VS>
__device__ __forceinline__ double cell_radius2(const WarpCell &w, int lane) {
  double r = 0.0;
#pragma unroll
  for (int s = 0; s < VS; ++s) {
    const int v = s * 32 + lane;
    if (v < w.nv) r = fmax(r, w.d2[v]);
  }
  return warp_max(r);
}

__device__ __forceinline__ bool has_twin(const unsigned *rem, int nrem, unsigned u, unsigned v) {
  for (int q = 0; q < nrem; ++q) {
    const unsigned t = rem[q];
    const unsigned x = t & 0xff, y = (t >> 8) & 0xff, z = (t >> 16) & 0xff;
    if ((x == v && y == u) || (y == v && z == u) || (z == v && x == u)) return true;
  }
  return false;
}

// Clips the cell by plane e (kept side e(x) >= 0).  Returns 0 when nothing
// is cut (the plane is not kept), 1 when the cell changed, -1 on failure
// with `status` set.  The caller has checked np < P.
template <int VS>
__device__ int clip(WarpCell &w, const Plane &e, int V, int &status, int lane, unsigned long long *ctr,
                    double *tr = nullptr, int trcap = 0) {
  const double ex = e.x, ey = e.y, ez = e.z, ew = e.w;
  unsigned rm[VS];
  int nrem = 0;
#pragma unroll
  for (int s = 0; s < VS; ++s) {
    const int v = s * 32 + lane;
    bool r = false;
    if (v < w.nv) r = w.cx[v] * ex + w.cy[v] * ey + w.cz[v] * ez + w.cw[v] * ew > 0.0;
    rm[s] = __ballot_sync(kFull, r);
    nrem += __popc(rm[s]);
  }
  if (ctr && lane == 0) ctr[kCtrVertexTests] += w.nv;
  trace_rec(tr, trcap, lane, 1, ex, ey, ez, ew, w.nv, nrem, w.np);
  if (nrem == 0) return 0;
  if (nrem == w.nv) {
    status = kEmptyCell;
    return -1;
  }
  const int pid = w.np;
  if (lane == 0) w.plane[pid] = e;
  // removed triples, in position order
  {
    int base = 0;
#pragma unroll
    for (int s = 0; s < VS; ++s) {
      const int v = s * 32 + lane;
      if ((rm[s] >> lane) & 1u) w.rem[base + __popc(rm[s] & lanemask_lt(lane))] = w.tri[v];
      base += __popc(rm[s]);
    }
  }
  __syncwarp();
  for (int r = lane; r < nrem; r += 32) {
    const unsigned t = w.rem[r];
    w.next[t & 0xff] = kNone;
    w.next[(t >> 8) & 0xff] = kNone;
    w.next[(t >> 16) & 0xff] = kNone;
  }
  __syncwarp();
  // boundary edges: link next[u] = v; a plane that starts two edges makes
  // the cavity non-manifold
  int nb = 0;
  bool bad = false;
  unsigned first_u = kNone;
  for (int r = lane; r < nrem; r += 32) {
    const unsigned t = w.rem[r];
    const unsigned tv[3] = {t & 0xff, (t >> 8) & 0xff, (t >> 16) & 0xff};
#pragma unroll
    for (int e3 = 0; e3 < 3; ++e3) {
      const unsigned u = tv[e3], v = tv[(e3 + 1) % 3];
      if (has_twin(w.rem, nrem, u, v)) continue;
      if (atomicCAS(&w.next[u], kNone, v) != kNone) bad = true;
      if (first_u == kNone) first_u = u;
      ++nb;
    }
  }
  nb = warp_sumi(nb);
  bad = __any_sync(kFull, bad);
  __syncwarp();
  if (!bad) {
    // the links must form a single cycle through all nb edges
    const unsigned has = __ballot_sync(kFull, first_u != kNone);
    const unsigned u0 = __shfl_sync(kFull, first_u, has ? __ffs(has) - 1 : 0);
    int steps = 0;
    bool ok = false;
    if (lane == 0 && u0 != kNone) {
      unsigned u = u0;
      do {
        u = w.next[u];
        ++steps;
      } while (u != kNone && u != u0 && steps <= nb);
      ok = u == u0 && steps == nb;
    }
    bad = !__shfl_sync(kFull, ok, 0);
  }
  trace_rec(tr, trcap, lane, 2, nb, bad, 0, 0);
  if (bad || nb < 3) {
    status = kInconsistentBoundary;
    return -1;
  }
  const int nkeep = w.nv - nrem;
  const int F = nkeep + nb;
  if (F > V) {
    status = kVertexOverflow;
    return -1;
  }
  // boundary edge list in deterministic order
  {
    int base = 0;
    for (int r0 = 0; r0 < nrem; r0 += 32) {
      const int r = r0 + lane;
      unsigned ue[3], ve[3];
      int cnt = 0;
      if (r < nrem) {
        const unsigned t = w.rem[r];
        const unsigned tv[3] = {t & 0xff, (t >> 8) & 0xff, (t >> 16) & 0xff};
#pragma unroll
        for (int e3 = 0; e3 < 3; ++e3) {
          const unsigned u = tv[e3], v = tv[(e3 + 1) % 3];
          if (!has_twin(w.rem, nrem, u, v)) {
            ue[cnt] = u;
            ve[cnt] = v;
            ++cnt;
          }
        }
      }
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t2 = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t2;
      }
      for (int k = 0; k < cnt; ++k) w.edge[base + incl - cnt + k] = ue[k] | (ve[k] << 8);
      base += __shfl_sync(kFull, incl, 31);
    }
  }
  // holes = removed positions below F; movers = survivors at or past F
  int nholes = 0, nmov = 0;
#pragma unroll
  for (int s = 0; s < VS; ++s) {
    const int v = s * 32 + lane;
    const bool hole = ((rm[s] >> lane) & 1u) && v < F;
    const unsigned hm = __ballot_sync(kFull, hole);
    if (hole) w.hole[nholes + __popc(hm & lanemask_lt(lane))] = v;
    nholes += __popc(hm);
  }
  __syncwarp();
#pragma unroll
  for (int s = 0; s < VS; ++s) {
    const int v = s * 32 + lane;
    const bool mover = !((rm[s] >> lane) & 1u) && v >= F && v < w.nv;
    const unsigned mm = __ballot_sync(kFull, mover);
    if (mover) copy_vertex(w, w.hole[nmov + __popc(mm & lanemask_lt(lane))], v);
    nmov += __popc(mm);
  }
  __syncwarp();
  const int in_holes = nholes - nmov;
  for (int q = lane; q < nb; q += 32) {
    const unsigned ed = w.edge[q];
    const int dst = q < in_holes ? int(w.hole[nmov + q]) : w.nv + (q - in_holes);
    make_vertex(w, dst, unsigned(pid), ed & 0xff, (ed >> 8) & 0xff);
  }
  __syncwarp();
  if (ctr && lane == 0) {
    ctr[kCtrClips] += 1;
    ctr[kCtrVerticesMade] += nb;
  }
  w.nv = F;
  w.np = pid + 1;
  if (tr) {
    // every vertex after the clip: triple and cofactor
    for (int v = 0; v < F; ++v) {
      const unsigned t = w.tri[v];
      trace_rec(tr, trcap, lane, 3, w.cx[v], w.cy[v], w.cz[v], w.cw[v], t & 0xff, (t >> 8) & 0xff, (t >> 16) & 0xff, v);
    }
  }
  return 1;
}

// Signed-tet integration of the cell (ConvexCell.cl:577-619) in the local
// frame: per vertex A and each of its planes i, the two tets (A, C, C
// projected on plane i, C projected on the edge line of planes i, j).
// Accumulates (sum w*centroid, sum w)/6 * factor into acc (warp-uniform).
template <int VS>
__device__ void integrate(const WarpCell &w, double factor, double acc[4], int lane,
                          unsigned long long *ctr, double *tr = nullptr, int trcap = 0) {
  double sx = 0, sy = 0, sz = 0, sw = 0;
#pragma unroll
  for (int s = 0; s < VS; ++s) {
    const int v = s * 32 + lane;
    if (v >= w.nv) continue;
    const double inv = 1.0 / w.cw[v];
    const double Ax = w.cx[v] * inv, Ay = w.cy[v] * inv, Az = w.cz[v] * inv;
    const double ACx = -Ax, ACy = -Ay, ACz = -Az;
    const unsigned t = w.tri[v];
    double nx[3], ny[3], nz[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const Plane &p = w.plane[(t >> (8 * i)) & 0xff];
      nx[i] = p.x;
      ny[i] = p.y;
      nz[i] = p.z;
    }
    double Px[3], Py[3], Pz[3], Lx[3], Ly[3], Lz[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double k = (ACx * nx[i] + ACy * ny[i] + ACz * nz[i]) / (nx[i] * nx[i] + ny[i] * ny[i] + nz[i] * nz[i]);
      Px[i] = ACx - k * nx[i];
      Py[i] = ACy - k * ny[i];
      Pz[i] = ACz - k * nz[i];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int j = (i + 1) % 3;
      const double cxv = ny[i] * nz[j] - nz[i] * ny[j];
      const double cyv = nz[i] * nx[j] - nx[i] * nz[j];
      const double czv = nx[i] * ny[j] - ny[i] * nx[j];
      const double c2 = cxv * cxv + cyv * cyv + czv * czv;
      const double ni2 = nx[i] * nx[i] + ny[i] * ny[i] + nz[i] * nz[i];
      const double nj2 = nx[j] * nx[j] + ny[j] * ny[j] + nz[j] * nz[j];
      if (c2 < kVolEps2 * ni2 * nj2) {
        Lx[i] = Ly[i] = Lz[i] = 0.0;
      } else {
        const double k = (ACx * cxv + ACy * cyv + ACz * czv) / c2;
        Lx[i] = k * cxv;
        Ly[i] = k * cyv;
        Lz[i] = k * czv;
      }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int st = 0; st < 2; ++st) {
        const int j = (i + 3 - st) % 3;
        // det3 of rows AC, P_i, L_j expanded along the first column
        const double det = ACx * (Py[i] * Lz[j] - Pz[i] * Ly[j]) - Px[i] * (ACy * Lz[j] - ACz * Ly[j]) +
                           Lx[j] * (ACy * Pz[i] - ACz * Py[i]);
        const double wt = (2 * st - 1) * det;
        sw += wt;
        sx += wt * (Ax + 0.25 * (ACx + Px[i] + Lx[j]));
        sy += wt * (Ay + 0.25 * (ACy + Py[i] + Ly[j]));
        sz += wt * (Az + 0.25 * (ACz + Pz[i] + Lz[j]));
      }
    }
  }
  sx = warp_sum(sx);
  sy = warp_sum(sy);
  sz = warp_sum(sz);
  sw = warp_sum(sw);
  const double f = factor / 6.0;
  trace_rec(tr, trcap, lane, 4, f * sx, f * sy, f * sz, f * sw, factor, w.nv, w.np);
  acc[0] += f * sx;
  acc[1] += f * sy;
  acc[2] += f * sz;
  acc[3] += f * sw;
  if (ctr && lane == 0) {
    ctr[kCtrExports] += 1;
    ctr[kCtrExportVertices] += w.nv;
  }
}

template <int VS>
__device__ void backup(WarpCell &w, int lane) {
#pragma unroll
  for (int s = 0; s < VS; ++s) {
    const int v = s * 32 + lane;
    if (v < w.nv) {
      w.bcx[v] = w.cx[v];
      w.bcy[v] = w.cy[v];
      w.bcz[v] = w.cz[v];
      w.bcw[v] = w.cw[v];
      w.bd2[v] = w.d2[v];
      w.btri[v] = w.tri[v];
    }
  }
  __syncwarp();
}
template <int VS>
__device__ void restore(WarpCell &w, int nv, int np, int lane) {
  __syncwarp();
#pragma unroll
  for (int s = 0; s < VS; ++s) {
    const int v = s * 32 + lane;
    if (v < nv) {
      w.cx[v] = w.bcx[v];
      w.cy[v] = w.bcy[v];
      w.cz[v] = w.bcz[v];
      w.cw[v] = w.bcw[v];
      w.d2[v] = w.bd2[v];
      w.tri[v] = w.btri[v];
    }
  }
  __syncwarp();
  w.nv = nv;
  w.np = np;
}

// Plane through three points, normal (B-A) x (C-A), kept side where the
// normal points (get_plane_from_points, ConvexCell.cl:125-129), in the local
// frame.
__device__ __forceinline__ Plane plane_from_points(const double A[3], const double B[3], const double C[3]) {
  const double ux = B[0] - A[0], uy = B[1] - A[1], uz = B[2] - A[2];
  const double vx = C[0] - A[0], vy = C[1] - A[1], vz = C[2] - A[2];
  const double nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
  return Plane{nx, ny, nz, -(nx * A[0] + ny * A[1] + nz * A[2])};
}

// Pt0 fallback one voxel layer past the range (GRID_OUT_DOMAIN,
// ConvexCell.cl:986-1051): lane 0 scans, others wait.
__device__ int out_domain_corner(const DevGrid &g, const int vmin[3], const int vmax[3], int &px, int &py,
                                 int &pz) {
  const int S = g.size;
  auto flag = [&](int x, int y, int z) { return int(g.flags[x + y * S + z * S * S]); };
  int in_domain = 1;
  if (vmax[2] + 1 < S) {
    const int z = vmax[2] + 1;
    for (int y = vmin[1]; y <= vmax[1] + 1 && in_domain == 1; y++) {
      if (y >= S) break;
      for (int x = vmin[0]; x <= vmax[0] + 1; x++) {
        if (x >= S) break;
        if (flag(x, y, z) != 1) {
          in_domain = flag(x, y, z);
          px = x; py = y; pz = z;
          break;
        }
      }
    }
  } else {
    in_domain = 0;
    px = vmin[0]; py = vmin[1]; pz = vmax[2] + 1;
  }
  if (in_domain == 1 && vmax[1] + 1 < S) {
    const int y = vmax[1] + 1;
    for (int z = vmin[2]; z <= vmax[2] && in_domain == 1; z++) {
      for (int x = vmin[0]; x <= vmax[0] + 1; x++) {
        if (x >= S) break;
        if (flag(x, y, z) != 1) {
          in_domain = flag(x, y, z);
          px = x; py = y; pz = z;
          break;
        }
      }
    }
  } else if (in_domain == 1) {
    in_domain = 0;
    px = vmin[0]; py = vmax[1] + 1; pz = vmin[2];
  }
  if (in_domain == 1 && vmax[0] + 1 < S) {
    const int x = vmax[0] + 1;
    for (int z = vmin[2]; z <= vmax[2] && in_domain == 1; z++) {
      for (int y = vmin[1]; y <= vmax[1]; y++) {
        if (flag(x, y, z) != 1) {
          in_domain = flag(x, y, z);
          px = x; py = y; pz = z;
          break;
        }
      }
    }
  } else if (in_domain == 1) {
    in_domain = 0;
    px = vmax[0] + 1; py = vmin[1]; pz = vmin[2];
  }
  return in_domain;
}

// Sorted union of the triangle lists of the voxel range in (z, y, x) order,
// built by one thread in buf (G ints, two halves used alternately); returns
// its length, or -1 once it would exceed T (ConvexCell.cl:722-749,950-979).
__device__ int serial_union(const DevGrid &g, const int vmin[3], const int vmax[3], int T, int *buf, int G) {
  const int S = g.size;
  int *cur = buf, *nxt = buf + G / 2;
  int n = 0;
  for (int z = vmin[2]; z <= vmax[2]; ++z)
    for (int y = vmin[1]; y <= vmax[1]; ++y)
      for (int x = vmin[0]; x <= vmax[0]; ++x) {
        const int vid = x + y * S + z * S * S;
        int i = g.offsets[vid];
        const int end = g.offsets[vid + 1];
        if (i == end) continue;
        int j = 0, m = 0;
        while (j < n || i < end) {
          int v;
          if (i >= end || (j < n && cur[j] < g.list[i])) v = cur[j++];
          else if (j >= n || g.list[i] < cur[j]) v = g.list[i++];
          else { v = cur[j++]; ++i; }
          if (m >= T) return -1;
          nxt[m++] = v;
        }
        int *t = cur; cur = nxt; nxt = t;
        n = m;
      }
  if (cur != buf)
    for (int k = 0; k < n; ++k) buf[k] = cur[k];
  return n;
}

// Bitonic sort of n (power of two, >= 32) ints in shared memory by one warp.
__device__ void warp_sort_ints(int *a, int n, int lane) {
  for (int k = 2; k <= n; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < n; i += 32) {
        const int l = i ^ j;
        if (l > i) {
          const int x = a[i], y = a[l];
          const bool up = (i & k) == 0;
          if ((x > y) == up) {
            a[i] = y;
            a[l] = x;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Whether every voxel that a ball of radius sqrt(r2) around the seed can
// touch is plainly outside (flag 0 and no triangles).  The final cell lies in
// that ball, so the reference's restriction would find the start corner
// outside and no triangle: mass 0.  Ranges as ConvexCell.cl:937-940.
__device__ __forceinline__ bool ball_outside(const DevGrid &g, float4 s, double r2, int lane) {
  const double r = sqrt(r2);
  int lo[3], hi[3];
  const double c[3] = {s.x, s.y, s.z};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo[d] = max(0, int((c[d] - r) / double(g.voxel)));
    hi[d] = min(g.size - 1, int((c[d] + r) / double(g.voxel)));
    if (c[d] - r < 0.0) lo[d] = 0;
  }
  const int S1 = g.size + 1;
  int v = 0;
  if (lane < 8) {
    const int x = (lane & 1) ? hi[0] + 1 : lo[0];
    const int y = (lane & 2) ? hi[1] + 1 : lo[1];
    const int z = (lane & 4) ? hi[2] + 1 : lo[2];
    const int sign = ((lane & 1) ^ ((lane >> 1) & 1) ^ ((lane >> 2) & 1)) ? 1 : -1;
    v = sign * __ldg(&g.sat[x + S1 * (y + S1 * z)]);
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return __shfl_sync(kFull, v, 0) == 0;
}

template <int VS, bool GRID>
__global__ void __launch_bounds__(128) k_cell(CellLaunch a, Layout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= a.num) return;
  WarpCell w = bind(smem + size_t(wib) * L.total, L);
  unsigned long long *ctr = a.counters;
  // per-warp counters are accumulated in lane 0's registers, flushed once
  unsigned long long lc[kCtrNum];
#pragma unroll
  for (int i = 0; i < kCtrNum; ++i) lc[i] = 0;
  unsigned long long *lcp = ctr ? lc : nullptr;

  const int sid = a.ids ? a.ids[row] : row;
  const float4 s = a.stored[sid];
  double *tr = (a.trace && sid == a.trace_seed) ? a.trace : nullptr;
  const int trcap = a.trace_cap;
  trace_rec(tr, trcap, lane, 0, s.x, s.y, s.z, s.w, sid);
  int status = kSuccess;
  double acc[4] = {0, 0, 0, 0};
  if (s.w <= kNoCellLimits) {
    if (lane == 0) {
      a.status[sid] = kSuccess;
      a.out[sid] = make_double4(s.x, s.y, s.z, s.w);
    }
    return;
  }
  init_box(w, s, a.cube_eps, lane);
  double R2 = cell_radius2<VS>(w, lane);

  // ---- Voronoi / power clipping by the K nearest, in order ----
  const unsigned *nrow = a.knn + size_t(row) * a.K;
  bool reached = false, exhausted = false, outside = false;
  const bool early = GRID && a.early_out && a.grid.sat != nullptr;
  for (int i0 = 0; i0 < a.K && status == kSuccess && !reached && !exhausted && !outside; i0 += 32) {
    // every lane builds the bisector of one neighbour, in double
    const int i = i0 + lane;
    Plane pl{0.0, 0.0, 0.0, 0.0};
    double nd2 = 0.0;
    bool valid = false;
    if (i < a.K) {
      const unsigned z = __ldg(&nrow[i]);
      if (z != kNone) {
        const float4 b = __ldg(&a.stored[z]);
        const double bx = double(b.x) - double(s.x), by = double(b.y) - double(s.y), bz = double(b.z) - double(s.z);
        nd2 = bx * bx + by * by + bz * bz;
        const double len = sqrt(nd2);
        // kept side contains the seed: n = -(b - s)/|b - s|, offset from the
        // power bisector (ConvexCell.cl:321-328) or, for a wall neighbour,
        // through the neighbour itself
        const double off = b.w <= kNoCellLimits ? len : (nd2 + (double(b.w) - double(s.w))) / (2.0 * len);
        pl = Plane{-bx / len, -by / len, -bz / len, off};
        valid = true;
      }
    }
    const unsigned vmask = __ballot_sync(kFull, valid);
    const int cnt = min(32, a.K - i0);
    for (int j = 0; j < cnt; ++j) {
      if (!((vmask >> j) & 1u)) {
        exhausted = true;  // fewer than K other seeds: all have been clipped
        break;
      }
      const Plane e = shfl_plane(pl, j);
      const double d2j = __shfl_sync(kFull, nd2, j);
      if (lcp && lane == 0) ++lcp[kCtrPlanesTested];
      if (w.np >= a.P) {
        status = kPlaneOverflow;
        break;
      }
      const int r = clip<VS>(w, e, a.V, status, lane, lcp, tr, trcap);
      if (r < 0) break;
      if (r > 0) {
        R2 = cell_radius2<VS>(w, lane);
        if (early && ball_outside(a.grid, s, R2, lane)) {
          outside = true;
          break;
        }
      }
      if (d2j > 4.0 * R2) {
        reached = true;
        break;
      }
    }
  }
  if (status == kSuccess && !reached && !exhausted && !outside) status = kSecurityRadiusNotReached;
  if (outside && lcp && lane == 0) lcp[kCtrOutside] += 1;

  if (status == kSuccess && !outside) {
    bool add_volume = true;
    if (GRID) {
      const DevGrid &g = a.grid;
      // bounding box -> voxel range (ConvexCell.cl:924-940)
      double lo[3] = {1000.0, 1000.0, 1000.0}, hi[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int sl = 0; sl < VS; ++sl) {
        const int v = sl * 32 + lane;
        if (v < w.nv) {
          const double inv = 1.0 / w.cw[v];
          const double p[3] = {w.cx[v] * inv + s.x, w.cy[v] * inv + s.y, w.cz[v] * inv + s.z};
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            lo[d] = fmin(lo[d], p[d]);
            hi[d] = fmax(hi[d], p[d]);
          }
        }
      }
      int vmin[3], vmax[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          lo[d] = fmin(lo[d], __shfl_xor_sync(kFull, lo[d], o));
          hi[d] = fmax(hi[d], __shfl_xor_sync(kFull, hi[d], o));
        }
        vmin[d] = max(0, int(lo[d] / double(g.voxel)));
        vmax[d] = min(g.size - 1, int(hi[d] / double(g.voxel)));
      }
      const int S = g.size;
      const int ex = vmax[0] - vmin[0] + 1, ey = vmax[1] - vmin[1] + 1, ez = vmax[2] - vmin[2] + 1;
      const int nvox = (ex > 0 && ey > 0 && ez > 0) ? ex * ey * ez : 0;
      // first corner with flag != 1 in (z, y, x) scan order, and the gathered
      // triangle ids of every voxel in the range
      int in_domain = 1, c0 = -1;
      int ntr = 0;
      bool spill = false;
      for (int b0 = 0; b0 < nvox; b0 += 32) {
        const int q = b0 + lane;
        int vid = -1, lo_off = 0, cntv = 0;
        int f = 1;
        if (q < nvox) {
          const int x = vmin[0] + q % ex, y = vmin[1] + (q / ex) % ey, z = vmin[2] + q / (ex * ey);
          vid = x + y * S + z * S * S;
          f = g.flags[vid];
          lo_off = __ldg(&g.offsets[vid]);
          cntv = __ldg(&g.offsets[vid + 1]) - lo_off;
        }
        if (in_domain == 1) {
          const unsigned fm = __ballot_sync(kFull, f != 1);
          if (fm) {
            const int src = __ffs(fm) - 1;
            in_domain = __shfl_sync(kFull, f, src);
            c0 = __shfl_sync(kFull, vid, src);
          }
        }
        int incl = cntv;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t2 = __shfl_up_sync(kFull, incl, o);
          if (lane >= o) incl += t2;
        }
        const int tot = __shfl_sync(kFull, incl, 31);
        if (ntr + tot > L.G) {
          spill = true;
        } else {
          for (int k = 0; k < cntv; ++k) w.tlist[ntr + incl - cntv + k] = __ldg(&g.list[lo_off + k]);
        }
        ntr += tot;
      }
      __syncwarp();
      int nuniq = 0;
      if (spill) {
        // more ids (with repeats) than the sort buffer holds: lane 0 builds
        // the sorted union voxel by voxel, failing past T like the
        // reference's merge (ConvexCell.cl:722-749)
        int cntu = 0;
        if (lane == 0) cntu = serial_union(g, vmin, vmax, a.T, w.tlist, L.G);
        cntu = __shfl_sync(kFull, cntu, 0);
        __syncwarp();
        if (cntu < 0) status = kTriangleOverflow;
        else nuniq = cntu;
      } else if (ntr > 0) {
        const int n2 = pow2_at_least(ntr);
        for (int i = ntr + lane; i < n2; i += 32) w.tlist[i] = 0x7fffffff;
        __syncwarp();
        warp_sort_ints(w.tlist, n2, lane);
        // unique in place
        for (int i0 = 0; i0 < ntr; i0 += 32) {
          const int i = i0 + lane;
          const int v = i < ntr ? w.tlist[i] : 0x7fffffff;
          const bool keep = i < ntr && (i == 0 || w.tlist[i - 1] != v);
          const unsigned km = __ballot_sync(kFull, keep);
          __syncwarp();
          if (keep) w.tlist[nuniq + __popc(km & lanemask_lt(lane))] = v;
          __syncwarp();
          nuniq += __popc(km);
        }
        if (nuniq > a.T) status = kTriangleOverflow;
      }
      double pt0[3] = {0, 0, 0};
      if (status == kSuccess) {
        if (in_domain == 1) {
          int px = 0, py = 0, pz = 0, f = 1;
          if (a.out_domain && lane == 0) f = out_domain_corner(g, vmin, vmax, px, py, pz);
          f = __shfl_sync(kFull, f, 0);
          if (f == 1) {
            status = kFindAnotherBeginningVertex;
          } else {
            in_domain = f;
            pt0[0] = __shfl_sync(kFull, px, 0) * double(g.voxel) - s.x;
            pt0[1] = __shfl_sync(kFull, py, 0) * double(g.voxel) - s.y;
            pt0[2] = __shfl_sync(kFull, pz, 0) * double(g.voxel) - s.z;
          }
        } else {
          const int x = c0 % S, y = (c0 / S) % S, z = c0 / (S * S);
          pt0[0] = x * double(g.voxel) - s.x;
          pt0[1] = y * double(g.voxel) - s.y;
          pt0[2] = z * double(g.voxel) - s.z;
        }
      }
      if (status == kSuccess) {
        add_volume = in_domain == 2;
        trace_rec(tr, trcap, lane, 5, pt0[0], pt0[1], pt0[2], in_domain, nuniq, status);
        if (add_volume) integrate<VS>(w, 1.0, acc, lane, lcp, tr, trcap);
        if (nuniq > 0) {
          if (lcp && lane == 0) {
            lcp[kCtrBoundaryCells] += 1;
            lcp[kCtrTriangles] += nuniq;
          }
          const int bk_nv = w.nv, bk_np = w.np;
          backup<VS>(w, lane);
          // signed cone decomposition over the boundary triangles
          // (ConvexCell.cl:1082-1115)
          for (int ti = 0; ti < nuniq && status == kSuccess; ++ti) {
            const int tri = w.tlist[ti];
            double P1[3], P2[3], P3[3];
            const int i1 = __ldg(&g.tris[3 * tri]), i2 = __ldg(&g.tris[3 * tri + 1]), i3 = __ldg(&g.tris[3 * tri + 2]);
            const float4 q1 = __ldg(&g.points[i1]), q2 = __ldg(&g.points[i2]), q3 = __ldg(&g.points[i3]);
            P1[0] = double(q1.x) - s.x; P1[1] = double(q1.y) - s.y; P1[2] = double(q1.z) - s.z;
            P2[0] = double(q2.x) - s.x; P2[1] = double(q2.y) - s.y; P2[2] = double(q2.z) - s.z;
            P3[0] = double(q3.x) - s.x; P3[1] = double(q3.y) - s.y; P3[2] = double(q3.z) - s.z;
            const double ax = P1[0] - pt0[0], ay = P1[1] - pt0[1], az = P1[2] - pt0[2];
            const double bx = P2[0] - pt0[0], by = P2[1] - pt0[1], bz = P2[2] - pt0[2];
            const double cx = P3[0] - pt0[0], cy = P3[1] - pt0[1], cz = P3[2] - pt0[2];
            const double det = ax * (by * cz - bz * cy) - bx * (ay * cz - az * cy) + cx * (ay * bz - az * by);
            const bool go_out = det > 0;
            trace_rec(tr, trcap, lane, 6, tri, det, go_out, 0);
            if (!go_out) {
#pragma unroll
              for (int d = 0; d < 3; ++d) {
                const double tmp = P2[d];
                P2[d] = P3[d];
                P3[d] = tmp;
              }
            }
            // cone beyond triangle (P1, P2, P3) seen from pt0
            // (CCClipTetFromPointsInfinite, ConvexCell.cl:565-575)
            const double *faces[4][3] = {{pt0, P1, P2}, {pt0, P3, P1}, {pt0, P2, P3}, {P2, P3, P1}};
            int cstat = kSuccess;
            for (int f4 = 0; f4 < 4 && cstat == kSuccess; ++f4) {
              if (w.np >= a.P) {
                cstat = kPlaneOverflow;
                break;
              }
              const Plane e = plane_from_points(faces[f4][0], faces[f4][1], faces[f4][2]);
              clip<VS>(w, e, a.V, cstat, lane, lcp, tr, trcap);
            }
            if (cstat == kEmptyCell) {
              restore<VS>(w, bk_nv, bk_np, lane);
              continue;
            }
            if (cstat != kSuccess) {
              status = cstat;
              acc[3] = 0.0;
              break;
            }
            integrate<VS>(w, go_out ? 1.0 : -1.0, acc, lane, lcp, tr, trcap);
            restore<VS>(w, bk_nv, bk_np, lane);
          }
        }
      }
    }
    if (!GRID && status == kSuccess) integrate<VS>(w, 1.0, acc, lane, lcp, tr, trcap);
    (void)add_volume;
  }
  if (lane == 0) {
    a.status[sid] = status;
    // local moments -> global: sum w*(x_local + s) = m_local + m * s
    const double m = acc[3];
    if (status == kSuccess)
      a.out[sid] = make_double4(acc[0] + m * double(s.x), acc[1] + m * double(s.y), acc[2] + m * double(s.z), m);
    else
      a.out[sid] = make_double4(0.0, 0.0, 0.0, 0.0);
    if (ctr) {
#pragma unroll
      for (int i = 0; i < kCtrNum; ++i)
        if (lc[i]) atomicAdd(&ctr[i], lc[i]);
    }
  }
}

template <int VS>
cudaError_t launch_vs(const CellLaunch &a, const Layout &L, cudaStream_t st) {
  const int warps_per_block = 4;
  const size_t smem = size_t(L.total) * warps_per_block;
  const int blocks = (a.num + warps_per_block - 1) / warps_per_block;
  cudaError_t e;
  if (a.grid.size > 0) {
    e = cudaFuncSetAttribute(k_cell<VS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    k_cell<VS, true><<<blocks, warps_per_block * 32, smem, st>>>(a, L);
  } else {
    e = cudaFuncSetAttribute(k_cell<VS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    k_cell<VS, false><<<blocks, warps_per_block * 32, smem, st>>>(a, L);
  }
  return cudaGetLastError();
}

}  // namespace

size_t cell_warp_smem(int P, int V, int T, bool grid) { return make_layout(P, V, T, grid).total; }

cudaError_t cell_launch(const CellLaunch &a, cudaStream_t st) {
  if (a.num <= 0) return cudaSuccess;
  if (a.P > kMaxP || a.V > kMaxV || a.T > kMaxT || a.P < 7 || a.V < 8) return cudaErrorInvalidValue;
  const Layout L = make_layout(a.P, a.V, a.T, a.grid.size > 0);
  const int vs = L.Vc / 32;
  if (vs <= 2) return launch_vs<2>(a, L, st);
  if (vs <= 3) return launch_vs<3>(a, L, st);
  if (vs <= 4) return launch_vs<4>(a, L, st);
  if (vs <= 6) return launch_vs<6>(a, L, st);
  return launch_vs<8>(a, L, st);
}

}  // namespace rpd
