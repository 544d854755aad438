// Device code of the restricted cell kernels, included by the translation
// units that instantiate them: cell.cu (FP64 clipping, batched solves, the
// outside probe, the cone kernels) and cell_prec.cu (the FP32 clipping
// variants), so the two compile in parallel.
#pragma once
// Restricted power cell of every seed, one warp per cell.  Replaces the
// reference's one-work-item compute_voro_cell (ConvexCell.cl:812-1116).
//
// Geometry is in the seed's local frame (seed at the origin), in double:
// planes (n, d) have unit normals and keep the side n.x + d >= 0.  Bisectors
// come from the exact double difference of the float seed coordinates, so
// thin boundary slivers keep their relative accuracy.  A vertex is the
// triple of its planes (a, b, c) plus the cofactor vector c of
// det(pi_a, pi_b, pi_c, e): the reference's FP64 half-space predicate
// det(...) > 0 (ConvexCell.cl:402-414, VHSAlgo 2) is e . c > 0, four DFMA
// per test.  The vertex position is p = c.xyz / c.w (c.w < 0 for the
// orientation of the reference's initial box, ConvexCell.cl:299-306).
//
// Ties: a vertex is cut only when it lies beyond the plane by more than
// kTieEps (e . c > kTieEps |c.w|).  That is a cut by a slightly shifted
// plane, consistent for coincident vertices, so the cavity in the dual is
// always a disk even where the domain's planes pass exactly through cell
// vertices (lattice-aligned surfaces).
//
// Per warp, shared memory holds the planes, the vertices (SoA), the cavity
// scratch and, with a domain, a backup of the Voronoi cell.  One clip:
//   1. every lane tests its vertices (v = lane + 32 s) -> ballot masks;
//   2. the directed edges of the removed dual triangles are marked in a
//      per-plane bit mask; boundary edges (u, v) are those whose twin (v, u)
//      is unmarked; they must form one cycle over the planes (else
//      inconsistent_boundary, ConvexCell.cl:463-515);
//   3. survivors past the new count move into holes; new vertices
//      (new plane, u, v) fill the remaining holes (the reference's triangle
//      orientation (vid, cir, next[cir]), ConvexCell.cl:556-562).
// The security radius (ConvexCell.cl:364-382) uses the cached |p|^2 of every
// vertex.  Integration (ConvexCell.cl:577-619) runs per vertex in double and
// is reduced across the warp.
#include <algorithm>

#include <mutex>
#include <set>
#include <utility>

#include "cell.cuh"
#include "bins.cuh"
#include "select.cuh"

namespace rpd {

namespace {

constexpr unsigned kNone = 0xffffffffu;
constexpr double kVolEps2 = 1e-12;  // VOLUME_EPSILON2 of the FP64 build (voronoi.cpp:922)
constexpr double kTieEps = 1e-10;   // cut tolerance, reference-frame units
constexpr int kDeferred = 100;      // internal status: cell parked for k_cone

struct Layout {
  int Pc, Vc, G, Mw;  // Mw: 32-bit words of one plane's edge mask
  int T;              // triangle cap the layout holds (parked slots)
  int HC;             // Hessian components per facet (0: no Hessian)
  // FP32 clipping state (precision > 0): planes as float4, and per vertex the
  // float4 cofactor, its error majorants (float2) and squared-radius bounds;
  // with a domain the vertex arrays share the backup's space (unused while
  // clipping)
  int prec;
  unsigned o_fpl, o_fc, o_ft, o_fhi, o_flo;
  unsigned o_harea, o_hbuf, o_hstage;  // Hessian: per-plane sums, per-vertex terms, per-lane staging
  unsigned o_plane, o_cx, o_cy, o_cz, o_cw, o_d2, o_tri, o_next, o_emask, o_rem, o_hole, o_edge;
  unsigned o_bcx, o_bcy, o_bcz, o_bcw, o_bd2, o_btri, o_tlist, o_pts, o_fstart, o_fv, o_pnb;
  unsigned total;
};

__host__ __device__ inline unsigned align16(unsigned x) { return (x + 15u) & ~15u; }

__host__ __device__ inline int pow2_at_least(int x) {
  int g = 32;
  while (g < x) g <<= 1;
  return g;
}

// T: the pass's triangle cap (the warp's id buffer); t_slot: the ids a
// parked cell's slot holds, when more than T (triangle overflows parked
// ahead, CellLaunch::T_ahead).  disjoint: every grid of the launch lists
// each triangle in one voxel only (DevGrid::lists_disjoint), so a cell's ids
// are gathered without repeats and the buffer needs T of them; otherwise 2T,
// the gathered ids being sorted and their repeats dropped in place.
__host__ __device__ inline Layout make_layout(int P, int V, int T, bool grid, int hc = 0, int t_slot = 0,
                                              int prec = 0, bool disjoint = false) {
  Layout L;
  L.HC = hc;
  L.prec = prec;
  L.Pc = (P + 3) & ~3;
  L.Vc = (V + 31) & ~31;
  L.G = grid ? (disjoint ? (T + 31) & ~31 : pow2_at_least(2 * T)) : 0;
  L.Mw = (L.Pc + 31) / 32;
  L.T = T > t_slot ? T : t_slot;
  unsigned o = 0;
  L.o_plane = o; o = align16(o + 32u * L.Pc);
  L.o_cx = o; o = align16(o + 8u * L.Vc);
  L.o_cy = o; o = align16(o + 8u * L.Vc);
  L.o_cz = o; o = align16(o + 8u * L.Vc);
  L.o_cw = o; o = align16(o + 8u * L.Vc);
  L.o_d2 = o; o = align16(o + 8u * L.Vc);
  L.o_tri = o; o = align16(o + 4u * L.Vc);
  L.o_next = o; o = align16(o + 4u * L.Pc);
  L.o_emask = o; o = align16(o + 4u * L.Pc * L.Mw);
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
    L.o_pts = o; o = align16(o + 8u * 12);
    L.o_fstart = o; o = align16(o + 4u * (L.Pc + 1));
    L.o_fv = o; o = align16(o + 3u * L.Vc);
    L.o_pnb = o; o = align16(o + 4u * L.Pc);
  } else {
    L.o_bcx = L.o_bcy = L.o_bcz = L.o_bcw = L.o_bd2 = L.o_btri = L.o_tlist = L.o_pts = L.o_fstart = L.o_fv = 0;
    L.o_pnb = 0;
    if (hc > 0) {
      L.o_pnb = o;
      o = align16(o + 4u * L.Pc);
    }
  }
  L.o_fpl = L.o_fc = L.o_ft = L.o_fhi = L.o_flo = 0;
  if (prec > 0) {
    L.o_fpl = o; o = align16(o + 16u * L.Pc);
    unsigned f = o;
    if (grid) f = L.o_bcx;  // 28 Vc bytes inside the backup's 40 Vc
    L.o_fc = f;
    L.o_ft = f + 16u * L.Vc;
    L.o_fhi = f + 24u * L.Vc;
    L.o_flo = f + 28u * L.Vc;
    if (!grid) o = align16(f + 32u * L.Vc);
  }
  L.o_harea = L.o_hbuf = L.o_hstage = 0;
  if (hc > 0) {
    L.o_harea = o; o = align16(o + 8u * hc * (L.Pc + 4));
    L.o_hbuf = o; o = align16(o + 8u * hc * 3 * L.Vc);
    L.o_hstage = o; o = align16(o + (8u * hc + 4u) * 32);
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
  unsigned *tri, *next, *emask, *rem, *hole, *edge;
  double *bcx, *bcy, *bcz, *bcw, *bd2;
  unsigned *btri;
  int *tlist;
  double *pts;  // start corner and the current boundary triangle, local frame
  int *fstart;         // per plane: first entry of its face in fv (np + 1 entries)
  unsigned char *fv;   // vertex ids of every face, in cyclic order
  int *pnb;            // per plane: its neighbour seed (stored id), -1 for box planes (used cells, Hessian)
  // Hessian (null when off): per plane the facet sums (area, or moments and
  // area), per vertex slot the terms of one integration, per lane a staged piece
  double *harea, *hbuf, *hstage;
  int *hstage_f;
  int hc;
  int nv, np;  // vertex and plane counts (warp-uniform)
  int vc, mw;  // capacity of the vertex arrays, words per edge mask
  // FP32 clipping state (null in FP64 launches)
  float4 *fpl;  // per plane: the plane rounded to float
  float4 *fc;   // per vertex: the cofactor vector in float
  float2 *ft;   // per vertex: error majorants (offset terms, normal terms)
  float *fhi, *flo;  // per vertex: bounds of the FP64 squared radius
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
  w.emask = reinterpret_cast<unsigned *>(base + L.o_emask);
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
  w.pts = reinterpret_cast<double *>(base + L.o_pts);
  w.fstart = reinterpret_cast<int *>(base + L.o_fstart);
  w.fv = base + L.o_fv;
  w.pnb = reinterpret_cast<int *>(base + L.o_pnb);
  w.hc = L.HC;
  w.harea = L.HC ? reinterpret_cast<double *>(base + L.o_harea) : nullptr;
  w.hbuf = L.HC ? reinterpret_cast<double *>(base + L.o_hbuf) : nullptr;
  w.hstage = L.HC ? reinterpret_cast<double *>(base + L.o_hstage) : nullptr;
  w.hstage_f = L.HC ? reinterpret_cast<int *>(base + L.o_hstage + 8u * L.HC * 32) : nullptr;
  w.nv = w.np = 0;
  w.vc = L.Vc;
  w.mw = L.Mw;
  w.fpl = L.prec ? reinterpret_cast<float4 *>(base + L.o_fpl) : nullptr;
  w.fc = L.prec ? reinterpret_cast<float4 *>(base + L.o_fc) : nullptr;
  w.ft = L.prec ? reinterpret_cast<float2 *>(base + L.o_ft) : nullptr;
  w.fhi = L.prec ? reinterpret_cast<float *>(base + L.o_fhi) : nullptr;
  w.flo = L.prec ? reinterpret_cast<float *>(base + L.o_flo) : nullptr;
  return w;
}

__device__ __forceinline__ unsigned lanemask_lt(int lane) { return (1u << lane) - 1u; }

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += t;
  }
  return v;
}
__device__ __forceinline__ Plane shfl_plane(Plane v, int src) {
  v.x = __shfl_sync(kFull, v.x, src);
  v.y = __shfl_sync(kFull, v.y, src);
  v.z = __shfl_sync(kFull, v.z, src);
  v.w = __shfl_sync(kFull, v.w, src);
  return v;
}

__device__ __forceinline__ void count(unsigned long long *ctr, int k, unsigned long long v, int lane) {
  if (ctr && lane == 0) atomicAdd(&ctr[k], v);
}

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
  cx = m34 * a23 - m24 * a33 + m23 * a43;
  cy = -(m34 * a13 - m14 * a33 + m13 * a43);
  cz = m24 * a13 - m14 * a23 + m12 * a43;
  cw = -(m23 * a13 - m13 * a23 + m12 * a33);
}

// Squared distance of the vertex with cofactor c from the seed (the FP64
// clipping's cached |p|^2; the FP32 clipping reproduces it bit for bit when
// it needs the exact value).
__device__ __forceinline__ double vertex_d2(double cx, double cy, double cz, double cw) {
  const double inv = 1.0 / cw;
  const double px = cx * inv, py = cy * inv, pz = cz * inv;
  return px * px + py * py + pz * pz;
}

// e . c: the side of plane e the vertex with cofactor c lies on, scaled by
// the cofactor (ConvexCell.cl:402-414 as e . c > 0).
__device__ __forceinline__ double plane_side(double cx, double cy, double cz, double cw, const Plane &e) {
  return cx * e.x + cy * e.y + cz * e.z + cw * e.w;
}

// Makes vertex `slot` from planes (a, b, c); false when it is degenerate.
__device__ __forceinline__ bool make_vertex(WarpCell &w, int slot, unsigned a, unsigned b, unsigned c) {
  double cx, cy, cz, cw;
  cofactor(w.plane[a], w.plane[b], w.plane[c], cx, cy, cz, cw);
  w.cx[slot] = cx;
  w.cy[slot] = cy;
  w.cz[slot] = cz;
  w.cw[slot] = cw;
  const double d2 = vertex_d2(cx, cy, cz, cw);
  w.d2[slot] = d2;
  w.tri[slot] = a | (b << 8) | (c << 16);
  return d2 < 1e300;  // false for inf / NaN
}

__device__ __forceinline__ void copy_vertex(WarpCell &w, int dst, int src) {
  w.cx[dst] = w.cx[src];
  w.cy[dst] = w.cy[src];
  w.cz[dst] = w.cz[src];
  w.cw[dst] = w.cw[src];
  w.d2[dst] = w.d2[src];
  w.tri[dst] = w.tri[src];
}

// ---- FP32 clipping (precision 1: mixed, 2: plain FP32) ----
//
// The clipping loop can keep the cell in float: the planes rounded to float4
// and, per vertex, the float cofactor vector c32 of its three planes with two
// error majorants.  With N = |n.x| + |n.y| + |n.z| and D = |d| for a plane
// (n, d) of the FP64 clipping, every term of the cofactor components x, y, z
// is the product of two normal components and one offset of three distinct
// planes, and every term of w the product of three normal components, so
// their absolute sums are at most Td = Na Nb Dc + Na Db Nc + Da Nb Nc and
// Tn = Na Nb Nc.  Rounding the planes to float (u = 2^-24 per entry) and
// evaluating in float moves the components by at most about 8u Td (x, y, z)
// and 8u Tn (w) from the FP64 clipping's, and the sign test e . c (four
// terms, e rounded too) by at most 13u (Ne Td + De Tn); the FP64 values' own
// rounding is 2^-29 times smaller.  kCutErr and kCofErr keep a factor of
// 2.5 and 2 above those bounds.
//   mixed (1): the float test decides when its value is farther than the
//   bound from the FP64 test's threshold; otherwise the test is escalated:
//   the vertex's FP64 cofactor is recomputed from the FP64 planes exactly as
//   the FP64 clipping made it, and the FP64 test decides.  Every decision is
//   the FP64 clipping's, so the clipped cells are the same; once clipping
//   ends, the FP64 vertices are rebuilt from the FP64 planes (promote) and
//   the restriction and integration run in FP64 as before.  The squared
//   radius of a vertex is kept as bounds [flo, fhi]; the security-radius and
//   outside tests escalate to the exact FP64 radius when their threshold falls
//   between the bounds, and a vertex whose cofactor w is within its error
//   bound of 0 is made in FP64 (the FP64 clipping's degeneracy test).
//   plain FP32 (2): the planes themselves are rounded to float, the float
//   tests and radius decide everything (no bound, no escalation), and the
//   restriction and integration run on vertices rebuilt from the rounded
//   planes: the accuracy of float planes, for comparison.
constexpr float kU32 = 5.9604645e-8f;    // 2^-24
constexpr float kCutErr = 32.0f * kU32;  // sign test bound / (Ne Td + De Tn)
constexpr float kCofErr = 16.0f * kU32;  // cofactor bound / Td (x, y, z) or Tn (w)
constexpr float kTieEpsF = float(kTieEps);
enum { kEscTests = 0, kEscVertices = 1, kEscRadii = 2, kEscNum = 3 };  // per-lane escalation counts

// The cofactor vector of cofactor() in float.
__device__ __forceinline__ float4 cofactor_f(const float4 &p1, const float4 &p2, const float4 &p3) {
  const float a11 = p1.x, a21 = p1.y, a31 = p1.z, a41 = p1.w;
  const float a12 = p2.x, a22 = p2.y, a32 = p2.z, a42 = p2.w;
  const float a13 = p3.x, a23 = p3.y, a33 = p3.z, a43 = p3.w;
  const float m12 = a21 * a12 - a11 * a22;
  const float m13 = a31 * a12 - a11 * a32;
  const float m14 = a41 * a12 - a11 * a42;
  const float m23 = a31 * a22 - a21 * a32;
  const float m24 = a41 * a22 - a21 * a42;
  const float m34 = a41 * a32 - a31 * a42;
  return make_float4(m34 * a23 - m24 * a33 + m23 * a43, -(m34 * a13 - m14 * a33 + m13 * a43),
                     m24 * a13 - m14 * a23 + m12 * a43, -(m23 * a13 - m13 * a23 + m12 * a33));
}

__device__ __forceinline__ float normal_l1(const float4 &p) { return fabsf(p.x) + fabsf(p.y) + fabsf(p.z); }

// The FP64 clipping's cofactor of vertex v, rebuilt from the FP64 planes.
__device__ __forceinline__ void vertex_cofactor64(const WarpCell &w, int v, double &cx, double &cy, double &cz,
                                                  double &cw) {
  const unsigned t = w.tri[v];
  cofactor(w.plane[t & 0xff], w.plane[(t >> 8) & 0xff], w.plane[(t >> 16) & 0xff], cx, cy, cz, cw);
}

// Makes vertex `slot` from planes (a, b, c) in float; false when the FP64
// clipping would find it degenerate (mixed) or its float radius is not
// finite (plain).
template <int PREC>
__device__ __forceinline__ bool make_vertex_f(WarpCell &w, int slot, unsigned a, unsigned b, unsigned c,
                                              int *esc) {
  const float4 p1 = w.fpl[a], p2 = w.fpl[b], p3 = w.fpl[c];
  const float4 cf = cofactor_f(p1, p2, p3);
  const float n1 = normal_l1(p1), n2 = normal_l1(p2), n3 = normal_l1(p3);
  const float tn = n1 * n2 * n3;
  const float td = n1 * n2 * fabsf(p3.w) + n1 * fabsf(p2.w) * n3 + fabsf(p1.w) * n2 * n3;
  w.fc[slot] = cf;
  w.ft[slot] = make_float2(td, tn);
  w.tri[slot] = a | (b << 8) | (c << 16);
  float hi, lo;
  bool ok = true;
  if constexpr (PREC == 2) {
    const float inv = __frcp_rn(cf.w);
    const float px = cf.x * inv, py = cf.y * inv, pz = cf.z * inv;
    hi = lo = px * px + py * py + pz * pz;
    ok = hi < 3e38f;  // false for inf / NaN
  } else {
    const float ew = kCofErr * tn, ex = kCofErr * td, aw = fabsf(cf.w);
    if (aw > 2.0f * ew) {
      // |p_i| = |c_i| / |c_w| within these bounds for any cofactor within the
      // error bound of c32
      // reciprocals rounded outward, so the bounds need no further margin
      const float ihi = __frcp_ru(__fsub_rd(aw, ew)), ilo = __frcp_rd(__fadd_ru(aw, ew));
      const float qx = fabsf(cf.x), qy = fabsf(cf.y), qz = fabsf(cf.z);
      const float hx = (qx + ex) * ihi, hy = (qy + ex) * ihi, hz = (qz + ex) * ihi;
      const float lx = fmaxf(qx - ex, 0.0f) * ilo, ly = fmaxf(qy - ex, 0.0f) * ilo, lz = fmaxf(qz - ex, 0.0f) * ilo;
      hi = (hx * hx + hy * hy + hz * hz) * (1.0f + 16.0f * kU32);
      lo = (lx * lx + ly * ly + lz * lz) * (1.0f - 16.0f * kU32);
    } else {
      // near-degenerate: the FP64 vertex decides, as in the FP64 clipping
      double cx, cy, cz, cw;
      vertex_cofactor64(w, slot, cx, cy, cz, cw);
      const double d2 = vertex_d2(cx, cy, cz, cw);
      ++esc[kEscVertices];
      ok = d2 < 1e300;
      hi = ok ? __double2float_ru(d2) : 0.0f;
      lo = ok ? __double2float_rd(d2) : 0.0f;
    }
  }
  w.fhi[slot] = hi;
  w.flo[slot] = lo;
  return ok;
}

__device__ __forceinline__ void copy_vertex_f(WarpCell &w, int dst, int src) {
  w.fc[dst] = w.fc[src];
  w.ft[dst] = w.ft[src];
  w.fhi[dst] = w.fhi[src];
  w.flo[dst] = w.flo[src];
  w.tri[dst] = w.tri[src];
}

// Vertices cut by plane e (e32: e rounded to float), from the float state.
template <int VS, int PREC>
__device__ __forceinline__ int cut_masks_f(const WarpCell &w, const Plane &e, const float4 &e32, unsigned (&rm)[VS],
                                           int lane, int *esc) {
  const float eN = normal_l1(e32), eD = fabsf(e32.w);
  int nrem = 0;
#pragma unroll
  for (int s = 0; s < VS; ++s) {
    rm[s] = 0u;
    if (s * 32 >= w.nv) continue;
    const int v = s * 32 + lane;
    bool r = false;
    if (v < w.nv) {
      const float4 c = w.fc[v];
      const float x = c.x * e32.x + c.y * e32.y + c.z * e32.z + c.w * e32.w - kTieEpsF * fabsf(c.w);
      if constexpr (PREC == 2) {
        r = x > 0.0f;
      } else {
        const float2 t = w.ft[v];
        const float bound = kCutErr * (eN * t.x + eD * t.y) + 1e-30f;
        if (x > bound) {
          r = true;
        } else if (x >= -bound) {
          // too close to call in float: the FP64 clipping's own test
          double cx, cy, cz, cw;
          vertex_cofactor64(w, v, cx, cy, cz, cw);
          r = plane_side(cx, cy, cz, cw, e) > kTieEps * fabs(cw);
          ++esc[kEscTests];
        }
      }
    }
    rm[s] = __ballot_sync(kFull, r);
    nrem += __popc(rm[s]);
  }
  return nrem;
}

// Bounds of the cell's squared radius (the largest vertex |p|^2) from the
// float state.
template <int VS>
__device__ __forceinline__ void radius2_bounds(const WarpCell &w, int lane, float &hi, float &lo) {
  float h = 0.0f, l = 0.0f;
#pragma unroll
  for (int s = 0; s < VS; ++s) {
    if (s * 32 >= w.nv) break;
    const int v = s * 32 + lane;
    if (v < w.nv) {
      h = fmaxf(h, w.fhi[v]);
      l = fmaxf(l, w.flo[v]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    h = fmaxf(h, __shfl_xor_sync(kFull, h, o));
    l = fmaxf(l, __shfl_xor_sync(kFull, l, o));
  }
  hi = h;
  lo = l;
}

// The FP64 clipping's squared radius of the cell, bit for bit (its cached
// |p|^2 rebuilt from the FP64 planes).
template <int VS>
__device__ __noinline__ double radius2_exact(const WarpCell &w, int lane) {
  double r = 0.0;
  for (int v = lane; v < w.nv; v += 32) {
    double cx, cy, cz, cw;
    vertex_cofactor64(w, v, cx, cy, cz, cw);
    r = fmax(r, vertex_d2(cx, cy, cz, cw));
  }
  return warp_max(r);
}

// The FP64 vertex arrays from the FP64 planes and the vertex triples: the
// state the FP64 clipping ends with, for the restriction and integration.
__device__ __noinline__ void promote(WarpCell &w, int lane) {
  for (int v = lane; v < w.nv; v += 32) {
    double cx, cy, cz, cw;
    vertex_cofactor64(w, v, cx, cy, cz, cw);
    w.cx[v] = cx;
    w.cy[v] = cy;
    w.cz[v] = cz;
    w.cw[v] = cw;
    w.d2[v] = vertex_d2(cx, cy, cz, cw);
  }
  __syncwarp();
}

// A plane rounded to float.
__device__ __forceinline__ float4 plane_f(const Plane &p) {
  return make_float4(float(p.x), float(p.y), float(p.z), float(p.w));
}

// The domain box [-eps, 1000+eps]^3 as 6 planes and 8 vertices, in the
// reference's plane order and vertex triples (ConvexCell.cl:278-308).
template <int PREC = 0>
__device__ void init_box(WarpCell &w, float4 s, float eps, int lane) {
  if (lane < 6) {
    const double vmin = -double(eps), vmax = 1000.0 + double(eps);
    const double sc = lane < 2 ? s.x : (lane < 4 ? s.y : s.z);
    const double sign = (lane & 1) ? -1.0 : 1.0;
    // global plane sign * x + off, off = -vmin (sign +) or vmax (sign -)
    const double off = (lane & 1) ? vmax - sc : sc - vmin;
    Plane p{0.0, 0.0, 0.0, PREC == 2 ? double(float(off)) : off};
    if (lane < 2) p.x = sign;
    else if (lane < 4) p.y = sign;
    else p.z = sign;
    w.plane[lane] = p;
    if constexpr (PREC > 0) w.fpl[lane] = plane_f(p);
  }
  __syncwarp();
  if (lane < 8) {
    const unsigned cube[8] = {2u | 5u << 8 | 0u << 16, 5u | 3u << 8 | 0u << 16, 1u | 5u << 8 | 2u << 16,
                              5u | 1u << 8 | 3u << 16, 4u | 2u << 8 | 0u << 16, 4u | 0u << 8 | 3u << 16,
                              2u | 4u << 8 | 1u << 16, 4u | 3u << 8 | 1u << 16};
    const unsigned t = cube[lane];
    if constexpr (PREC > 0) {
      int esc[kEscNum] = {0, 0, 0};
      make_vertex_f<PREC>(w, lane, t & 0xff, (t >> 8) & 0xff, (t >> 16) & 0xff, esc);
    } else {
      make_vertex(w, lane, t & 0xff, (t >> 8) & 0xff, (t >> 16) & 0xff);
    }
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
    if (s * 32 >= w.nv) break;
    const int v = s * 32 + lane;
    if (v < w.nv) r = fmax(r, w.d2[v]);
  }
  return warp_max(r);
}

// Vertices cut by plane e, as ballot masks per slot; returns their count.
template <int VS>
__device__ __forceinline__ int cut_masks(const WarpCell &w, const Plane &e, unsigned (&rm)[VS], int lane) {
  int nrem = 0;
#pragma unroll
  for (int s = 0; s < VS; ++s) {
    rm[s] = 0u;
    if (s * 32 >= w.nv) continue;
    const int v = s * 32 + lane;
    bool r = false;
    if (v < w.nv) {
      const double cw = w.cw[v];
      r = plane_side(w.cx[v], w.cy[v], w.cz[v], cw, e) > kTieEps * fabs(cw);
    }
    rm[s] = __ballot_sync(kFull, r);
    nrem += __popc(rm[s]);
  }
  return nrem;
}

// Clips the cell by plane e.  Returns 0 when nothing is cut (the plane is
// not kept), 1 when the cell changed, -1 on failure with `status` set.  The
// caller has checked np < P.
// PREC > 0: the FP32 clipping of the cell's float state (e32: e rounded to
// float; esc: the lane's escalation counts).
template <int VS, int PREC = 0>
__device__ int clip(WarpCell &w, const Plane &e, int V, int &status, int lane, unsigned long long *ctr,
                    double *tr, int trcap, const float4 *e32 = nullptr, int *esc = nullptr) {
  unsigned rm[VS];
  int nrem;
  if constexpr (PREC > 0) nrem = cut_masks_f<VS, PREC>(w, e, *e32, rm, lane, esc);
  else nrem = cut_masks<VS>(w, e, rm, lane);
  count(ctr, kCtrVertexTests, w.nv, lane);
  trace_rec(tr, trcap, lane, 1, e.x, e.y, e.z, e.w, w.nv, nrem, w.np);
  if (nrem == 0) return 0;
  if (nrem == w.nv) {
    status = kEmptyCell;
    return -1;
  }
  const int pid = w.np;
  const int mw = w.mw;
  if (lane == 0) {
    w.plane[pid] = e;
    if constexpr (PREC > 0) w.fpl[pid] = *e32;
  }
  const int nkeep = w.nv - nrem;
  // The cavity boundary is the set of directed edges of removed triangles
  // whose twin belongs to a kept triangle: the edges that occur once among
  // the removed (or, reversed, among the kept) triangles.  When the smaller
  // side has at most 10 triangles, its edges fit one per lane and a match on
  // the undirected plane pair finds them; otherwise edge bitmasks do.
  const bool fast = min(nrem, nkeep) <= 10;
  const bool from_kept = fast && nkeep < nrem;
  const int nside = from_kept ? nkeep : nrem;
  // the side's triples, in position order
  {
    int base = 0;
#pragma unroll
    for (int s = 0; s < VS; ++s) {
      const int v = s * 32 + lane;
      const unsigned valid = s * 32 >= w.nv ? 0u : (w.nv - s * 32 >= 32 ? kFull : (1u << (w.nv - s * 32)) - 1u);
      const unsigned side = from_kept ? (~rm[s] & valid) : rm[s];
      if ((side >> lane) & 1u) w.rem[base + __popc(side & lanemask_lt(lane))] = w.tri[v];
      base += __popc(side);
    }
  }
  __syncwarp();
  int nb = 0;
  bool bad = false;
  bool bnd = false;          // fast path: this lane holds boundary edge (bu -> bv)
  unsigned bu = 0, bv = 0;
  int bpos = 0;
  if (fast) {
    const bool act = lane < 3 * nside;
    unsigned key = 0x10000u + lane;  // unique for idle lanes
    if (act) {
      const unsigned t = w.rem[lane / 3];
      const int e3 = lane % 3;
      bu = (t >> (8 * e3)) & 0xff;
      bv = (t >> (8 * ((e3 + 1) % 3))) & 0xff;
      if (from_kept) {
        const unsigned x = bu;
        bu = bv;
        bv = x;
      }
      key = bu < bv ? (bu << 8 | bv) : (bv << 8 | bu);
    }
    const int cnt = __popc(__match_any_sync(kFull, key));
    bnd = act && cnt == 1;
    bad = act && cnt > 2;
    const unsigned bmask = __ballot_sync(kFull, bnd);
    nb = __popc(bmask);
    bpos = __popc(bmask & lanemask_lt(lane));
    // every plane starts and ends at most one boundary edge (every lane
    // takes part in both matches)
    const unsigned mu = __match_any_sync(kFull, bnd ? bu : 0x10000u + lane);
    const unsigned mv = __match_any_sync(kFull, bnd ? bv : 0x10000u + lane);
    bad |= bnd && (__popc(mu) != 1 || __popc(mv) != 1);
    if (bnd) w.next[bu] = lane;
    __syncwarp();
    int succ = bnd ? int(w.next[bv] & 31u) : lane;
    const unsigned su = __shfl_sync(kFull, bu, succ);
    bad |= bnd && (!((bmask >> succ) & 1u) || su != bv);
    bad = __any_sync(kFull, bad);
    if (!bad) {
      // one cycle: the lowest lane of every orbit, by pointer jumping
      int mn = lane;
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const int om = __shfl_sync(kFull, mn, succ);
        succ = __shfl_sync(kFull, succ, succ);
        mn = min(mn, om);
      }
      bad = __popc(__ballot_sync(kFull, bnd && mn == lane)) != 1;
    }
  } else {
    // clear the links and edge masks of the planes of the removed triangles
    for (int r = lane; r < nrem; r += 32) {
      const unsigned t = w.rem[r];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const unsigned p = (t >> (8 * i)) & 0xff;
        w.next[p] = kNone;
        for (int k = 0; k < mw; ++k) w.emask[p * mw + k] = 0u;
      }
    }
    __syncwarp();
    // mark every directed edge a->b of a removed triangle: bit b of mask a
    for (int r = lane; r < nrem; r += 32) {
      const unsigned t = w.rem[r];
      const unsigned a = t & 0xff, b = (t >> 8) & 0xff, c = (t >> 16) & 0xff;
      atomicOr(&w.emask[a * mw + (b >> 5)], 1u << (b & 31));
      atomicOr(&w.emask[b * mw + (c >> 5)], 1u << (c & 31));
      atomicOr(&w.emask[c * mw + (a >> 5)], 1u << (a & 31));
    }
    __syncwarp();
    // boundary edges: directed edges whose twin is unmarked, in removed
    // order; link next[u] = v (a plane starting two edges makes the cavity
    // non-manifold)
    unsigned first_u = kNone;
    for (int r0 = 0; r0 < nrem; r0 += 32) {
      const int r = r0 + lane;
      unsigned t = 0, bmask = 0;  // bit e3: edge (tv[e3], tv[e3+1]) is on the boundary
      if (r < nrem) {
        t = w.rem[r];
#pragma unroll
        for (int e3 = 0; e3 < 3; ++e3) {
          const unsigned u = (t >> (8 * e3)) & 0xff, v = (t >> (8 * ((e3 + 1) % 3))) & 0xff;
          if (!((w.emask[v * mw + (u >> 5)] >> (u & 31)) & 1u)) bmask |= 1u << e3;
        }
      }
      const int cnt = __popc(bmask);
      const int incl = warp_incl_scan(cnt, lane);
      int pos = nb + incl - cnt;
#pragma unroll
      for (int e3 = 0; e3 < 3; ++e3) {
        if (!((bmask >> e3) & 1u)) continue;
        const unsigned u = (t >> (8 * e3)) & 0xff, v = (t >> (8 * ((e3 + 1) % 3))) & 0xff;
        if (pos < w.vc) w.edge[pos] = u | (v << 8);
        ++pos;
        if (atomicCAS(&w.next[u], kNone, v) != kNone) bad = true;
        if (first_u == kNone) first_u = u;
      }
      nb += __shfl_sync(kFull, incl, 31);
    }
    bad = __any_sync(kFull, bad);
    __syncwarp();
    if (!bad) {
      // the links must form a single cycle through all nb edges
      const unsigned has = __ballot_sync(kFull, first_u != kNone);
      const unsigned u0 = __shfl_sync(kFull, first_u, has ? __ffs(has) - 1 : 0);
      bool ok = false;
      if (lane == 0 && u0 != kNone) {
        unsigned u = u0;
        int steps = 0;
        do {
          u = w.next[u];
          ++steps;
        } while (u != kNone && u != u0 && steps <= nb);
        ok = u == u0 && steps == nb;
      }
      bad = !__shfl_sync(kFull, ok, 0);
    }
  }
  trace_rec(tr, trcap, lane, 2, nb, bad, 0, 0);
  if (bad || nb < 3) {
    status = kInconsistentBoundary;
    return -1;
  }
  const int F = nkeep + nb;
  if (F > V) {
    status = kVertexOverflow;
    return -1;
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
    if (mover) {
      if constexpr (PREC > 0) copy_vertex_f(w, w.hole[nmov + __popc(mm & lanemask_lt(lane))], v);
      else copy_vertex(w, w.hole[nmov + __popc(mm & lanemask_lt(lane))], v);
    }
    nmov += __popc(mm);
  }
  __syncwarp();
  const int in_holes = nholes - nmov;
  bool degenerate = false;
  if (fast) {
    if (bnd) {
      const int dst = bpos < in_holes ? int(w.hole[nmov + bpos]) : w.nv + (bpos - in_holes);
      if constexpr (PREC > 0) degenerate = !make_vertex_f<PREC>(w, dst, unsigned(pid), bu, bv, esc);
      else degenerate = !make_vertex(w, dst, unsigned(pid), bu, bv);
    }
  } else {
    for (int q = lane; q < nb; q += 32) {
      const unsigned ed = w.edge[q];
      const int dst = q < in_holes ? int(w.hole[nmov + q]) : w.nv + (q - in_holes);
      if constexpr (PREC > 0) degenerate |= !make_vertex_f<PREC>(w, dst, unsigned(pid), ed & 0xff, (ed >> 8) & 0xff, esc);
      else degenerate |= !make_vertex(w, dst, unsigned(pid), ed & 0xff, (ed >> 8) & 0xff);
    }
  }
  __syncwarp();
  if (__any_sync(kFull, degenerate)) {
    status = kInconsistentBoundary;
    return -1;
  }
  count(ctr, kCtrClips, 1, lane);
  count(ctr, kCtrVerticesMade, nb, lane);
  w.nv = F;
  w.np = pid + 1;
  if (tr) {
    for (int v = 0; v < F; ++v) {
      const unsigned t = w.tri[v];
      if constexpr (PREC > 0)
        trace_rec(tr, trcap, lane, 3, w.fc[v].x, w.fc[v].y, w.fc[v].z, w.fc[v].w, t & 0xff, (t >> 8) & 0xff,
                  (t >> 16) & 0xff, v);
      else
        trace_rec(tr, trcap, lane, 3, w.cx[v], w.cy[v], w.cz[v], w.cw[v], t & 0xff, (t >> 8) & 0xff, (t >> 16) & 0xff, v);
    }
  }
  return 1;
}

// Facet integrals of one integration (CCExportBaryVolumeAndArea,
// ConvexCell.cl:621-678) into w.harea: per vertex A and each pair (plane
// p, edge line l) of the volume decomposition, the triangle (A, the seed's
// foot on p, the seed's foot on l) in plane p, signed by p's normal, times
// factor; with 4 components also its area times its centroid (local frame).
// Each vertex slot's terms go to w.hbuf first, then one lane per plane adds
// them in vertex order: the sums do not depend on the warp schedule.
__device__ __noinline__ void hess_integrate(const WarpCell &w, double factor, int lane) {
  const int hc = w.hc;
  for (int v = lane; v < w.nv; v += 32) {
    const double inv = 1.0 / w.cw[v];
    const double Ax = w.cx[v] * inv, Ay = w.cy[v] * inv, Az = w.cz[v] * inv;
    const unsigned t = w.tri[v];
    double term[3][4] = {};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const Plane &pi = w.plane[(t >> (8 * i)) & 0xff];
      const Plane &pj = w.plane[(t >> (8 * ((i + 1) % 3))) & 0xff];
      const double cxv = pi.y * pj.z - pi.z * pj.y;
      const double cyv = pi.z * pj.x - pi.x * pj.z;
      const double czv = pi.x * pj.y - pi.y * pj.x;
      const double c2 = cxv * cxv + cyv * cyv + czv * czv;
      double Lx = 0, Ly = 0, Lz = 0;
      if (c2 >= kVolEps2) {
        const double k = -(Ax * cxv + Ay * cyv + Az * czv) / c2;
        Lx = k * cxv;
        Ly = k * cyv;
        Lz = k * czv;
      }
      // line i pairs with plane i (sign -) and plane i+1 (sign +)
#pragma unroll
      for (int st = 0; st < 2; ++st) {
        const Plane &pp = st ? pj : pi;
        const double k = -(Ax * pp.x + Ay * pp.y + Az * pp.z);
        const double Px = -Ax - k * pp.x, Py = -Ay - k * pp.y, Pz = -Az - k * pp.z;
        // det(P, L, n) / 2 with the foot vectors taken from A
        const double det = Px * (Ly * pp.z - Lz * pp.y) - Py * (Lx * pp.z - Lz * pp.x) + Pz * (Lx * pp.y - Ly * pp.x);
        const double ar = (st ? 0.5 : -0.5) * det;
        const int slot = st ? (i + 1) % 3 : i;
        if (hc == 1) {
          term[slot][0] += ar;
        } else {
          term[slot][0] += ar * (Ax + (Px + Lx) * (1.0 / 3.0));
          term[slot][1] += ar * (Ay + (Py + Ly) * (1.0 / 3.0));
          term[slot][2] += ar * (Az + (Pz + Lz) * (1.0 / 3.0));
          term[slot][3] += ar;
        }
      }
    }
    for (int i = 0; i < 3; ++i)
      for (int c = 0; c < hc; ++c) w.hbuf[(3 * v + i) * hc + c] = term[i][c];
  }
  __syncwarp();
  for (int p = lane; p < w.np; p += 32) {
    double sum[4] = {0, 0, 0, 0};
    for (int v = 0; v < w.nv; ++v) {
      const unsigned t = w.tri[v];
#pragma unroll
      for (int i = 0; i < 3; ++i)
        if (int((t >> (8 * i)) & 0xff) == p)
          for (int c = 0; c < hc; ++c) sum[c] += w.hbuf[(3 * v + i) * hc + c];
    }
    for (int c = 0; c < hc; ++c) w.harea[p * hc + c] += factor * sum[c];
  }
  __syncwarp();
}

// Signed-tet integration of the cell (ConvexCell.cl:577-619) in the local
// frame: per vertex A and each of its planes i, the two tets (A, C, C
// projected on plane i, C projected on the edge line of planes i, j), C the
// seed at the origin.  Unit normals make the plane projection division-free.
// Accumulates (sum w*centroid, sum w)/6 * factor into acc (warp-uniform).
template <int VS, bool HESS = false>
__device__ void integrate(const WarpCell &w, double factor, double acc[4], int lane, unsigned long long *ctr,
                          double *tr, int trcap) {
  double sx = 0, sy = 0, sz = 0, sw = 0;
#pragma unroll 1
  for (int s = 0; s < VS; ++s) {
    if (s * 32 >= w.nv) break;
    const int v = s * 32 + lane;
    if (v >= w.nv) continue;
    const double inv = 1.0 / w.cw[v];
    const double Ax = w.cx[v] * inv, Ay = w.cy[v] * inv, Az = w.cz[v] * inv;
    const unsigned t = w.tri[v];
    // AC = -A; projections of C on plane i: P_i = AC - (AC . n_i) n_i
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const Plane &pi = w.plane[(t >> (8 * i)) & 0xff];
      const Plane &pj = w.plane[(t >> (8 * ((i + 1) % 3))) & 0xff];
      const double cxv = pi.y * pj.z - pi.z * pj.y;
      const double cyv = pi.z * pj.x - pi.x * pj.z;
      const double czv = pi.x * pj.y - pi.y * pj.x;
      const double c2 = cxv * cxv + cyv * cyv + czv * czv;
      double Lx = 0, Ly = 0, Lz = 0;
      if (c2 >= kVolEps2) {
        const double k = -(Ax * cxv + Ay * cyv + Az * czv) / c2;
        Lx = k * cxv;
        Ly = k * cyv;
        Lz = k * czv;
      }
      // line i (planes i, i+1) pairs with plane i (sign -) and plane i+1
      // (sign +): the reference's j = (i + 3 - st) % 3, w = (2 st - 1) det
#pragma unroll
      for (int st = 0; st < 2; ++st) {
        const Plane &pp = st ? pj : pi;
        const double k = -(Ax * pp.x + Ay * pp.y + Az * pp.z);
        const double Px = -Ax - k * pp.x, Py = -Ay - k * pp.y, Pz = -Az - k * pp.z;
        const double det = -Ax * (Py * Lz - Pz * Ly) - Px * (-Ay * Lz + Az * Ly) + Lx * (-Ay * Pz + Az * Py);
        const double wt = st ? det : -det;
        sw += wt;
        sx += wt * (Ax + 0.25 * (Px + Lx - Ax));
        sy += wt * (Ay + 0.25 * (Py + Ly - Ay));
        sz += wt * (Az + 0.25 * (Pz + Lz - Az));
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(kFull, sx, o);
    sy += __shfl_xor_sync(kFull, sy, o);
    sz += __shfl_xor_sync(kFull, sz, o);
    sw += __shfl_xor_sync(kFull, sw, o);
  }
  const double f = factor / 6.0;
  trace_rec(tr, trcap, lane, 4, f * sx, f * sy, f * sz, f * sw, factor, w.nv, w.np);
  acc[0] += f * sx;
  acc[1] += f * sy;
  acc[2] += f * sz;
  acc[3] += f * sw;
  if constexpr (HESS) {
    if (w.harea) hess_integrate(w, factor, lane);
  }
  count(ctr, kCtrExports, 1, lane);
  count(ctr, kCtrExportVertices, w.nv, lane);
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

// Plane through three points with normal (B-A) x (C-A), normalised, kept side
// where the normal points (get_plane_from_points, ConvexCell.cl:125-129), in
// the local frame; all zero when the points are collinear.
__device__ __forceinline__ Plane plane_from_points(const double A[3], const double B[3], const double C[3]) {
  const double ux = B[0] - A[0], uy = B[1] - A[1], uz = B[2] - A[2];
  const double vx = C[0] - A[0], vy = C[1] - A[1], vz = C[2] - A[2];
  double nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
  const double l2 = nx * nx + ny * ny + nz * nz;
  if (!(l2 > 0.0)) return Plane{0.0, 0.0, 0.0, 0.0};
  const double il = rsqrt(l2);
  nx *= il;
  ny *= il;
  nz *= il;
  return Plane{nx, ny, nz, -(nx * A[0] + ny * A[1] + nz * A[2])};
}

// Pt0 fallback one voxel layer past the range (GRID_OUT_DOMAIN,
// ConvexCell.cl:986-1051): run by one lane.
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

// Squared radius of a ball around the seed whose voxels are all plainly
// outside (flag 0 and no triangles), or -1.  The final cell lies in any ball
// around the seed that holds its current vertices, so once that ball fits,
// the reference's restriction would find the start corner outside and no
// triangle in the cell's voxel range (ConvexCell.cl:924-940): mass 0.  Lane k
// counts the non-plain voxels of the cube of half-size k voxels around the
// seed's voxel from the summed-volume table; below the first non-empty cube,
// the ball may reach the cube's faces that are not on the grid's border.
__device__ double plain_radius2(const DevGrid &g, float4 s, int lane) {
  const int S = g.size, S1 = S + 1;
  const double h = double(g.voxel);
  const double c[3] = {s.x, s.y, s.z};
  int v[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) v[d] = min(S - 1, max(0, int(c[d] / h)));
  int lo[3], hi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo[d] = max(0, v[d] - lane);
    hi[d] = min(S - 1, v[d] + lane) + 1;
  }
  int cnt = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int x = (q & 1) ? hi[0] : lo[0], y = (q & 2) ? hi[1] : lo[1], z = (q & 4) ? hi[2] : lo[2];
    const int sign = ((q & 1) ^ ((q >> 1) & 1) ^ ((q >> 2) & 1)) ? 1 : -1;
    cnt -= sign * __ldg(&g.sat[x + S1 * (y + S1 * z)]);
  }
  const unsigned hit = __ballot_sync(kFull, cnt != 0);
  const int k = hit ? __ffs(hit) - 1 : 32;  // cubes below k are plain
  if (k == 0) return -1.0;
  double r = 1e300;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (v[d] - (k - 1) > 0) r = fmin(r, c[d] - (v[d] - (k - 1)) * h);
    if (v[d] + (k - 1) < S - 1) r = fmin(r, (v[d] + k) * h - c[d]);
  }
  r -= 1e-6 * h;
  return r > 0.0 ? (r >= 1e150 ? 1e300 : r * r) : -1.0;
}

// Signed cone decomposition over boundary triangles tids[t0, t1)
// (ConvexCell.cl:1082-1115): for each, the cone beyond the triangle seen
// from the start corner (w.pts[0..2]) clips the backed-up cell, the piece is
// integrated with the triangle's sign, and the cell is restored.  Returns
// the status; on failure fail_at is the failing triangle's position.
// With the apex inside the cell (inner), a cone rarely misses the cell: the
// quick classification is skipped and the triangle's plane clips first.
// HESS: the Hessian facet sums as well (when w.harea is set).
template <int VS, bool HESS = false>
__device__ int cone_triangles(WarpCell &w, const CellLaunch &a, float4 s, const int *tids, int t0, int t1,
                              int bk_nv, int bk_np, bool inner, double acc[4], int &fail_at, int lane,
                              unsigned long long *ctr, double *tr, int trcap) {
  const DevGrid &g = a.grid;
  for (int ti = t0; ti < t1; ++ti) {
    const int tri = tids[ti];
    bool go_out = false;
    if (lane == 0) {
      // triangle in the local frame, oriented to go out from pt0
      const double p0x = w.pts[0], p0y = w.pts[1], p0z = w.pts[2];
      const int i1 = __ldg(&g.tris[3 * tri]), i2 = __ldg(&g.tris[3 * tri + 1]), i3 = __ldg(&g.tris[3 * tri + 2]);
      const float4 q1 = __ldg(&g.points[i1]), q2 = __ldg(&g.points[i2]), q3 = __ldg(&g.points[i3]);
      const double P1[3] = {double(q1.x) - s.x, double(q1.y) - s.y, double(q1.z) - s.z};
      const double P2[3] = {double(q2.x) - s.x, double(q2.y) - s.y, double(q2.z) - s.z};
      const double P3[3] = {double(q3.x) - s.x, double(q3.y) - s.y, double(q3.z) - s.z};
      const double ax = P1[0] - p0x, ay = P1[1] - p0y, az = P1[2] - p0z;
      const double bx = P2[0] - p0x, by = P2[1] - p0y, bz = P2[2] - p0z;
      const double cx = P3[0] - p0x, cy = P3[1] - p0y, cz = P3[2] - p0z;
      const double det = ax * (by * cz - bz * cy) - bx * (ay * cz - az * cy) + cx * (ay * bz - az * by);
      go_out = det > 0;
      trace_rec(tr, trcap, lane, 6, tri, det, go_out, 0);
      for (int d = 0; d < 3; ++d) {
        w.pts[3 + d] = P1[d];
        w.pts[6 + d] = go_out ? P2[d] : P3[d];
        w.pts[9 + d] = go_out ? P3[d] : P2[d];
      }
    }
    go_out = __shfl_sync(kFull, go_out, 0);
    __syncwarp();
    // the cone beyond triangle (P1, P2, P3) seen from pt0
    // (CCClipTetFromPointsInfinite, ConvexCell.cl:565-575): faces
    // (pt0, P1, P2), (pt0, P3, P1), (pt0, P2, P3), (P2, P3, P1)
    if (w.np >= a.P) {
      fail_at = ti;
      return kPlaneOverflow;
    }
    const double *q0 = w.pts, *q1 = w.pts + 3, *q2 = w.pts + 6, *q3 = w.pts + 9;
    auto cone = [&](int f4) {
      return f4 == 0 ? plane_from_points(q0, q1, q2)
                     : f4 == 1 ? plane_from_points(q0, q3, q1)
                               : f4 == 2 ? plane_from_points(q0, q2, q3) : plane_from_points(q2, q3, q1);
    };
    // quick classification: a plane that cuts every vertex empties the
    // piece; no plane cutting any vertex means the cell lies in the cone
    bool empty = false, any_cut = inner;
#pragma unroll 1
    for (int f4 = 0; f4 < 4 && !empty && !inner; ++f4) {
      unsigned rm[VS];
      const int nr = cut_masks<VS>(w, cone(f4), rm, lane);
      empty |= nr == w.nv;
      any_cut |= nr > 0;
    }
    if (empty) {
      count(ctr, kCtrConeEmpty, 1, lane);
      continue;
    }
    if (any_cut) {
      int cstat = kSuccess;
#pragma unroll 1
      for (int k = 0; k < 4 && cstat == kSuccess; ++k) {
        if (w.np >= a.P) {
          cstat = kPlaneOverflow;
          break;
        }
        clip<VS>(w, cone(inner ? (k + 3) & 3 : k), a.V, cstat, lane, ctr, tr, trcap);
      }
      if (cstat == kEmptyCell) {
        if (inner) count(ctr, kCtrConeEmpty, 1, lane);
        restore<VS>(w, bk_nv, bk_np, lane);
        continue;
      }
      if (cstat != kSuccess) {
        fail_at = ti;
        return cstat;
      }
    }
    integrate<VS, HESS>(w, go_out ? 1.0 : -1.0, acc, lane, ctr, tr, trcap);
    if (any_cut) restore<VS>(w, bk_nv, bk_np, lane);
  }
  return kSuccess;
}

// Whether the cone clipping from the start corner p0 (cone_triangles, the
// reference's) surely overflows no cap on this cell, so that an apex inside
// the cell, which clips nothing, gives the reference's status.  Per triangle
// of the union: a cone plane with every vertex beyond it (margin included)
// empties the piece and the triangle clips nothing; otherwise the planes
// that may cut a vertex number c, and no part of the cell that one of them
// misses can it cut later, so np + c < P keeps every plane check before a
// clip below P and nv + 2c <= V every clip within V (a clip adds at most
// one face; f faces make 2f - 4 vertices).  The margin, 1e-9 of the plane
// offset plus the cell radius R, covers the rounding of the planes (built
// here as cone_triangles builds them) and of later vertices; a triangle
// nearly flat from p0 counts as a failure.  One triangle per lane.
__device__ bool ref_cones_fit(const WarpCell &w, const DevGrid &g, float4 s, const int *tids, int ntri,
                              const double p0[3], int P, int V, double R, int lane) {
  if (w.np >= P) return false;  // the check before each triangle's cone
  bool bad = false;
  for (int b0 = 0; b0 < ntri; b0 += 32) {
    const int ti = b0 + lane;
    if (ti < ntri && !bad) {
      const int tri = tids[ti];
      const int i1 = __ldg(&g.tris[3 * tri]), i2 = __ldg(&g.tris[3 * tri + 1]), i3 = __ldg(&g.tris[3 * tri + 2]);
      const float4 r1 = __ldg(&g.points[i1]), r2 = __ldg(&g.points[i2]), r3 = __ldg(&g.points[i3]);
      const double P1[3] = {double(r1.x) - s.x, double(r1.y) - s.y, double(r1.z) - s.z};
      const double P2[3] = {double(r2.x) - s.x, double(r2.y) - s.y, double(r2.z) - s.z};
      const double P3[3] = {double(r3.x) - s.x, double(r3.y) - s.y, double(r3.z) - s.z};
      const double ax = P1[0] - p0[0], ay = P1[1] - p0[1], az = P1[2] - p0[2];
      const double bx = P2[0] - p0[0], by = P2[1] - p0[1], bz = P2[2] - p0[2];
      const double cx = P3[0] - p0[0], cy = P3[1] - p0[1], cz = P3[2] - p0[2];
      const double det = ax * (by * cz - bz * cy) - bx * (ay * cz - az * cy) + cx * (ay * bz - az * by);
      const double scale = sqrt((ax * ax + ay * ay + az * az) * (bx * bx + by * by + bz * bz) *
                                (cx * cx + cy * cy + cz * cz));
      if (!(fabs(det) > 1e-9 * scale)) {
        bad = true;
      } else {
        const bool go_out = det > 0;
        const double *q1 = P1, *q2 = go_out ? P2 : P3, *q3 = go_out ? P3 : P2;
        const Plane f[4] = {plane_from_points(p0, q1, q2), plane_from_points(p0, q3, q1),
                            plane_from_points(p0, q2, q3), plane_from_points(q2, q3, q1)};
        int c = 0;
        bool empty = false;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const double m = 1e-9 * (fabs(f[k].w) + R);
          bool any = false, all = true;
          for (int v = 0; v < w.nv; ++v) {
            const double cw = w.cw[v], ps = plane_side(w.cx[v], w.cy[v], w.cz[v], cw, f[k]);
            any |= ps > (kTieEps - m) * fabs(cw);
            all &= ps > (kTieEps + m) * fabs(cw);
          }
          empty |= all;
          c += any ? 1 : 0;
        }
        bad = !empty && c > 0 && !(w.np + c < P && w.nv + 2 * c <= V);
      }
    }
    if (__any_sync(kFull, bad)) return false;
  }
  return true;
}

// Apex inside the cell.  The signed cone decomposition holds for any apex on
// a known side of the surface.  From a point inside the convex cell, the
// segment to any point of the cell stays in the cell, so a triangle that
// misses the cell crosses none of them and its cone holds no part of the
// cell.  The apex is the grid corner with flag 0 or 2 of the voxel range
// deepest in the cell (at least kApexDepth voxels; ties to the lowest corner
// id), moved by kApexShift voxels along kApexDir: grid triangles have
// vertices on lattice lines and planes through the corners, so cone planes
// through the corner itself can contain face edges of the cell exactly, and
// a facet's boundary then depends on rounding.  No triangle comes within
// 4 kApexShift of the corner (else -1: the caller keeps the reference's
// start corner), so the moved apex keeps the corner's side.  Returns the
// flag, or -1.
constexpr double kApexDepth = 4e-3;    // voxels
constexpr double kApexShift = 1e-3;    // voxels
constexpr double kSeparation = 1e-9;   // reference-frame units
__device__ __constant__ double kApexDir[3] = {0.5317 / 1.0001074492, 0.3229 / 1.0001074492, 0.7831 / 1.0001074492};

__device__ int inner_apex(const WarpCell &w, const DevGrid &g, float4 s, const int vmin[3], const int vmax[3],
                          const int *tids, int ntri, double apex[3], int lane) {
  const int S = g.size;
  int lo[3], n[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo[d] = vmin[d];
    n[d] = min(vmax[d] + 1, S - 1) - vmin[d] + 1;
  }
  const int ncorner = (n[0] > 0 && n[1] > 0 && n[2] > 0) ? n[0] * n[1] * n[2] : 0;
  const double h = double(g.voxel);
  double best = kApexDepth * h;
  int best_id = 0x7fffffff;
  for (int q = lane; q < ncorner; q += 32) {
    const int x = lo[0] + q % n[0], y = lo[1] + (q / n[0]) % n[1], z = lo[2] + q / (n[0] * n[1]);
    const int vid = x + y * S + z * S * S;
    if (g.flags[vid] == 1) continue;
    const double cx = x * h - s.x, cy = y * h - s.y, cz = z * h - s.z;
    double depth = 1e300;
    for (int i = 0; i < w.np && depth > best; ++i) {
      const Plane p = w.plane[i];
      depth = fmin(depth, fma(p.x, cx, fma(p.y, cy, fma(p.z, cz, p.w))));
    }
    if (depth > best || (depth == best && vid < best_id)) {
      best = depth;
      best_id = vid;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(kFull, best, o);
    const int oi = __shfl_xor_sync(kFull, best_id, o);
    if (ob > best || (ob == best && oi < best_id)) {
      best = ob;
      best_id = oi;
    }
  }
  if (best_id == 0x7fffffff) return -1;
  const int x = best_id % S, y = (best_id / S) % S, z = best_id / (S * S);
  const double c[3] = {x * h - s.x, y * h - s.y, z * h - s.z};
  // no triangle near the corner: the shifted apex is on the corner's side
  const double near = 4.0 * kApexShift * h;
  bool close = false;
  for (int i = lane; i < ntri && !close; i += 32) {
    const int tri = tids[i];
    double P[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float4 q = __ldg(&g.points[__ldg(&g.tris[3 * tri + k])]);
      P[k][0] = double(q.x) - s.x;
      P[k][1] = double(q.y) - s.y;
      P[k][2] = double(q.z) - s.z;
    }
    double lo3[3], hi3[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      lo3[d] = fmin(P[0][d], fmin(P[1][d], P[2][d])) - near;
      hi3[d] = fmax(P[0][d], fmax(P[1][d], P[2][d])) + near;
    }
    if (c[0] < lo3[0] || c[0] > hi3[0] || c[1] < lo3[1] || c[1] > hi3[1] || c[2] < lo3[2] || c[2] > hi3[2])
      continue;
    const double e1[3] = {P[1][0] - P[0][0], P[1][1] - P[0][1], P[1][2] - P[0][2]};
    const double e2[3] = {P[2][0] - P[0][0], P[2][1] - P[0][1], P[2][2] - P[0][2]};
    const double nn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    const double len = sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
    const double dist = fabs(nn[0] * (c[0] - P[0][0]) + nn[1] * (c[1] - P[0][1]) + nn[2] * (c[2] - P[0][2]));
    close = !(dist > near * len);
  }
  if (__any_sync(kFull, close)) return -1;
#pragma unroll
  for (int d = 0; d < 3; ++d) apex[d] = c[d] + kApexShift * h * kApexDir[d];
  return g.flags[best_id];
}

// Drops from tids[0, n) the triangles that a plane of the cell separates
// from it (all three corners more than kSeparation outside), keeping the
// order; returns the number kept.
__device__ int drop_separated(const WarpCell &w, const DevGrid &g, float4 s, int *tids, int n, int lane) {
  int kept = 0;
  for (int i0 = 0; i0 < n; i0 += 32) {
    const int i = i0 + lane;
    int tri = 0;
    bool keep = false;
    if (i < n) {
      tri = tids[i];
      const float4 q1 = __ldg(&g.points[__ldg(&g.tris[3 * tri])]);
      const float4 q2 = __ldg(&g.points[__ldg(&g.tris[3 * tri + 1])]);
      const float4 q3 = __ldg(&g.points[__ldg(&g.tris[3 * tri + 2])]);
      const double x1 = double(q1.x) - s.x, y1 = double(q1.y) - s.y, z1 = double(q1.z) - s.z;
      const double x2 = double(q2.x) - s.x, y2 = double(q2.y) - s.y, z2 = double(q2.z) - s.z;
      const double x3 = double(q3.x) - s.x, y3 = double(q3.y) - s.y, z3 = double(q3.z) - s.z;
      keep = true;
      for (int k = 0; k < w.np && keep; ++k) {
        const Plane p = w.plane[k];
        const double d1 = fma(p.x, x1, fma(p.y, y1, fma(p.z, z1, p.w)));
        const double d2 = fma(p.x, x2, fma(p.y, y2, fma(p.z, z2, p.w)));
        const double d3 = fma(p.x, x3, fma(p.y, y3, fma(p.z, z3, p.w)));
        keep = fmax(d1, fmax(d2, d3)) >= -kSeparation;
      }
    }
    const unsigned km = __ballot_sync(kFull, keep);
    __syncwarp();
    if (keep) tids[kept + __popc(km & lanemask_lt(lane))] = tri;
    __syncwarp();
    kept += __popc(km);
  }
  return kept;
}

// ---- Cone pieces from their facets, for an apex inside the cell ----
//
// With the apex a inside the convex cell C, the piece C ∩ cone(a, t) beyond
// triangle t is bounded by t ∩ C, by the parts of the cell's faces inside the
// cone beyond t, and by the cone's three sides.  Its volume and first moment
// are sums over the facets of the cones from a, and the cone over a facet G
// is a sum over G's boundary edges (u, v), counter-clockwise around the
// outward normal, of the signed tetrahedra (a, c, u, v), c any point of G's
// plane.  The sides pass through a and give nothing.  Every edge is a
// segment clipped by a few planes, so a piece needs neither 3D clipping nor
// polygon buffers: one triangle per lane, registers only.  Equal to the
// reference's clipped-cone integral (ConvexCell.cl:1082-1115) in exact
// arithmetic.
constexpr int kFaceCap = 64;  // faces of one cell culled per batch of a 64-bit mask

// Face lists of the cell, each counter-clockwise around the face's outward
// normal (-n of its plane), and vertex positions (local frame) in px/py/pz.
// Angular bounds of the faces seen from the apex: per face, the unit axis
// and the half-angle (with cos, sin) of a cone from a that holds the face,
// as floats in the backup arrays (unused on this path); kAngFaces faces fit.
__device__ __forceinline__ float *face_angles(const WarpCell &w) { return reinterpret_cast<float *>(w.bcw); }
__device__ __forceinline__ int face_angle_cap(const WarpCell &w) { return (20 * w.vc) / 24; }
__device__ __forceinline__ unsigned char *face_nb(const WarpCell &w) { return reinterpret_cast<unsigned char *>(w.edge); }

__device__ void build_faces(const WarpCell &w, double *px, double *py, double *pz, const double a[3], int lane) {
  const int np = w.np, nv = w.nv;
  int *fstart = w.fstart;
  unsigned char *fv = w.fv;
  for (int p = lane; p <= np; p += 32) fstart[p] = 0;
  __syncwarp();
  for (int v = lane; v < nv; v += 32) {
    const double inv = 1.0 / w.cw[v];
    px[v] = w.cx[v] * inv;
    py[v] = w.cy[v] * inv;
    pz[v] = w.cz[v] * inv;
    const unsigned t = w.tri[v];
    atomicAdd(&fstart[(t & 0xff) + 1], 1);
    atomicAdd(&fstart[((t >> 8) & 0xff) + 1], 1);
    atomicAdd(&fstart[((t >> 16) & 0xff) + 1], 1);
  }
  __syncwarp();
  int carry = 0;
  for (int b0 = 1; b0 <= np; b0 += 32) {
    const int p = b0 + lane;
    const int c = p <= np ? fstart[p] : 0;
    const int incl = warp_incl_scan(c, lane);
    __syncwarp();
    if (p <= np) fstart[p] = carry + incl;
    carry += __shfl_sync(kFull, incl, 31);
  }
  __syncwarp();
  // lane per face: its vertices, chained (vertex (p, y, z) is followed by
  // the vertex (p, z, .)), then turned counter-clockwise around -n_p
  for (int p = lane; p < np; p += 32) {
    const int f0 = fstart[p], k = fstart[p + 1] - f0;
    int m = 0;
    for (int v = 0; v < nv && m < k; ++v) {
      const unsigned t = w.tri[v];
      if ((t & 0xff) == unsigned(p) || ((t >> 8) & 0xff) == unsigned(p) || ((t >> 16) & 0xff) == unsigned(p))
        fv[f0 + m++] = (unsigned char)v;
    }
    auto rot = [&](int v, bool to) {
      const unsigned t = w.tri[v];
      const unsigned a = t & 0xff, b = (t >> 8) & 0xff, c = (t >> 16) & 0xff;
      if (to) return a == unsigned(p) ? c : (b == unsigned(p) ? a : b);
      return a == unsigned(p) ? b : (b == unsigned(p) ? c : a);
    };
    for (int i = 1; i < k; ++i) {
      const unsigned want = rot(fv[f0 + i - 1], true);
      for (int j = i; j < k; ++j) {
        if (rot(fv[f0 + j], false) == want) {
          const unsigned char x = fv[f0 + i];
          fv[f0 + i] = fv[f0 + j];
          fv[f0 + j] = x;
          break;
        }
      }
    }
    if (k >= 3) {
      const Plane pl = w.plane[p];
      double sx = 0, sy = 0, sz = 0;
      for (int i = 0; i < k; ++i) {
        const int u = fv[f0 + i], v = fv[f0 + (i + 1 == k ? 0 : i + 1)];
        sx += py[u] * pz[v] - pz[u] * py[v];
        sy += pz[u] * px[v] - px[u] * pz[v];
        sz += px[u] * py[v] - py[u] * px[v];
      }
      if (sx * pl.x + sy * pl.y + sz * pl.z > 0.0) {
        for (int i = 0, j = k - 1; i < j; ++i, --j) {
          const unsigned char x = fv[f0 + i];
          fv[f0 + i] = fv[f0 + j];
          fv[f0 + j] = x;
        }
      }
    }
    // plane of edge (i, i+1): shared by the two vertices, other than p
    unsigned char *nb = face_nb(w);
    for (int i = 0; i < k; ++i) {
      const unsigned t1 = w.tri[fv[f0 + i]], t2 = w.tri[fv[f0 + (i + 1 == k ? 0 : i + 1)]];
      unsigned e = 0xffu;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const unsigned x = (t1 >> (8 * b)) & 0xff;
        if (x != unsigned(p) && (x == (t2 & 0xff) || x == ((t2 >> 8) & 0xff) || x == ((t2 >> 16) & 0xff))) e = x;
      }
      nb[f0 + i] = (unsigned char)e;
    }
    if (p < face_angle_cap(w)) {
      float *ang = face_angles(w) + 6 * p;
      float ux = 0.f, uy = 0.f, uz = 0.f;
      for (int i = 0; i < k; ++i) {
        const int v = fv[f0 + i];
        const float dx = float(px[v] - a[0]), dy = float(py[v] - a[1]), dz = float(pz[v] - a[2]);
        const float il = rsqrtf(fmaxf(dx * dx + dy * dy + dz * dz, 1e-30f));
        ux += dx * il;
        uy += dy * il;
        uz += dz * il;
      }
      const float ul = rsqrtf(fmaxf(ux * ux + uy * uy + uz * uz, 1e-30f));
      ux *= ul;
      uy *= ul;
      uz *= ul;
      float cmin = 1.f;
      for (int i = 0; i < k; ++i) {
        const int v = fv[f0 + i];
        const float dx = float(px[v] - a[0]), dy = float(py[v] - a[1]), dz = float(pz[v] - a[2]);
        const float il = rsqrtf(fmaxf(dx * dx + dy * dy + dz * dz, 1e-30f));
        cmin = fminf(cmin, (dx * ux + dy * uy + dz * uz) * il);
      }
      const float th = acosf(fmaxf(-1.f, fminf(1.f, cmin)));
      ang[0] = ux;
      ang[1] = uy;
      ang[2] = uz;
      ang[3] = th;
      ang[4] = cosf(th);
      ang[5] = sinf(th);
    }
  }
  __syncwarp();
}

struct ConePiece {
  double a[3];      // apex
  double c[4][4];   // side planes (through a) and the triangle's plane, inside >= 0
  double t[3][3];   // triangle corners, counter-clockwise around c[3]
  double acc[4];    // sum of w*x, w*y, w*z, w (unscaled: 6x the volume)
};

__device__ __forceinline__ double pval(const double *n, double x, double y, double z) {
  return fma(n[0], x, fma(n[1], y, fma(n[2], z, n[3])));
}

// Signed tetrahedron (a, c, u, v) into acc: 6 * volume and 6 * volume * 4 * centroid.
__device__ __forceinline__ void edge_tet(ConePiece &q, const double c[3], const double u[3], const double v[3]) {
  const double cx = c[0] - q.a[0], cy = c[1] - q.a[1], cz = c[2] - q.a[2];
  const double ux = u[0] - q.a[0], uy = u[1] - q.a[1], uz = u[2] - q.a[2];
  const double vx = v[0] - q.a[0], vy = v[1] - q.a[1], vz = v[2] - q.a[2];
  const double det = cx * (uy * vz - uz * vy) - cy * (ux * vz - uz * vx) + cz * (ux * vy - uy * vx);
  q.acc[0] += det * (q.a[0] + c[0] + u[0] + v[0]);
  q.acc[1] += det * (q.a[1] + c[1] + u[1] + v[1]);
  q.acc[2] += det * (q.a[2] + c[2] + u[2] + v[2]);
  q.acc[3] += det * 4.0;
}

// Clips segment u + s (v - u), s in [lo, hi], by plane n (inside >= 0).
__device__ __forceinline__ void clip_seg(double eu, double ev, double &lo, double &hi) {
  if (eu >= 0.0 && ev >= 0.0) return;
  if (eu < 0.0 && ev < 0.0) {
    hi = -1.0;
    return;
  }
  const double s = eu / (eu - ev);
  if (eu < 0.0) lo = fmax(lo, s);
  else hi = fmin(hi, s);
}

// Line of planes n1 and n2 (inside >= 0 each) as x0 + s d with d = n1 x n2;
// false when they are parallel.
__device__ __forceinline__ bool plane_line(const double *n1, const double *n2, double x0[3], double d[3]) {
  d[0] = n1[1] * n2[2] - n1[2] * n2[1];
  d[1] = n1[2] * n2[0] - n1[0] * n2[2];
  d[2] = n1[0] * n2[1] - n1[1] * n2[0];
  const double dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  const double nn = (n1[0] * n1[0] + n1[1] * n1[1] + n1[2] * n1[2]) * (n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2]);
  if (!(dd > 1e-24 * nn)) return false;
  // x0 = (-w1 (n2 x d) - w2 (d x n1)) / |d|^2
  const double a0 = n2[1] * d[2] - n2[2] * d[1], a1 = n2[2] * d[0] - n2[0] * d[2], a2 = n2[0] * d[1] - n2[1] * d[0];
  const double b0 = d[1] * n1[2] - d[2] * n1[1], b1 = d[2] * n1[0] - d[0] * n1[2], b2 = d[0] * n1[1] - d[1] * n1[0];
  const double inv = 1.0 / dd;
  x0[0] = (-n1[3] * a0 - n2[3] * b0) * inv;
  x0[1] = (-n1[3] * a1 - n2[3] * b1) * inv;
  x0[2] = (-n1[3] * a2 - n2[3] * b2) * inv;
  return true;
}

// Parameter range of the line x0 + s d inside plane n.
__device__ __forceinline__ void clip_line(const double *n, const double x0[3], const double d[3], double &lo, double &hi) {
  const double v0 = pval(n, x0[0], x0[1], x0[2]);
  const double sl = n[0] * d[0] + n[1] * d[1] + n[2] * d[2];
  if (sl > 0.0) lo = fmax(lo, -v0 / sl);
  else if (sl < 0.0) hi = fmin(hi, -v0 / sl);
  else if (v0 < 0.0) hi = -1e300;
}

// Face f's facet: its edges inside the cone, and the cone planes' lines
// inside the face (bounded by the face's edge planes and the other cone
// planes), as boundary segments (U, V) of the facet; emit(c, U, V) for each,
// c the face's first vertex.
template <class Emit>
__device__ __forceinline__ void face_segments(const ConePiece &q, const WarpCell &w, const double *px,
                                              const double *py, const double *pz, int f, Emit emit) {
  const int f0 = w.fstart[f], k = w.fstart[f + 1] - f0;
  const int v0 = w.fv[f0];
  const double c[3] = {px[v0], py[v0], pz[v0]};
  for (int i = 0; i < k; ++i) {
    const int iu = w.fv[f0 + i], iv = w.fv[f0 + (i + 1 == k ? 0 : i + 1)];
    const double u[3] = {px[iu], py[iu], pz[iu]}, v[3] = {px[iv], py[iv], pz[iv]};
    double lo = 0.0, hi = 1.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) clip_seg(pval(q.c[j], u[0], u[1], u[2]), pval(q.c[j], v[0], v[1], v[2]), lo, hi);
    if (lo < hi) {
      const double U[3] = {fma(lo, v[0] - u[0], u[0]), fma(lo, v[1] - u[1], u[1]), fma(lo, v[2] - u[2], u[2])};
      const double V[3] = {fma(hi, v[0] - u[0], u[0]), fma(hi, v[1] - u[1], u[1]), fma(hi, v[2] - u[2], u[2])};
      emit(c, U, V);
    }
  }
  const Plane pf = w.plane[f];
  const double nf[4] = {pf.x, pf.y, pf.z, pf.w};
#pragma unroll 1
  for (int j = 0; j < 4; ++j) {
    double x0[3], d[3];
    if (!plane_line(nf, q.c[j], x0, d)) continue;
    double lo = -1e300, hi = 1e300;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
      if (jj != j) clip_line(q.c[jj], x0, d, lo, hi);
    const unsigned char *nb = face_nb(w);
    for (int i = 0; i < k && lo < hi; ++i) {
      // the plane of the face's edge (i, i+1)
      const unsigned e = nb[f0 + i];
      if (e == 0xffu) continue;
      const Plane pe = w.plane[e];
      const double ne[4] = {pe.x, pe.y, pe.z, pe.w};
      clip_line(ne, x0, d, lo, hi);
    }
    if (lo < hi) {
      const double U[3] = {fma(lo, d[0], x0[0]), fma(lo, d[1], x0[1]), fma(lo, d[2], x0[2])};
      const double V[3] = {fma(hi, d[0], x0[0]), fma(hi, d[1], x0[1]), fma(hi, d[2], x0[2])};
      emit(c, U, V);
    }
  }
}

__device__ void face_facet(ConePiece &q, const WarpCell &w, const double *px, const double *py, const double *pz,
                           int f) {
  face_segments(q, w, px, py, pz, f,
                [&](const double *c, const double *U, const double *V) { edge_tet(q, c, U, V); });
}

// The facet of face f inside the cone as Hessian terms: its area (the
// boundary segments fanned from c, against the face's outward normal -n),
// and with 4 components its area times its centroid (local frame).
__device__ __noinline__ void face_piece(const ConePiece &q, const WarpCell &w, const double *px, const double *py,
                                        const double *pz, int f, double out[4]) {
  const Plane pf = w.plane[f];
  double a = 0, mx = 0, my = 0, mz = 0;
  face_segments(q, w, px, py, pz, f, [&](const double *c, const double *U, const double *V) {
    const double ux = U[0] - c[0], uy = U[1] - c[1], uz = U[2] - c[2];
    const double vx = V[0] - c[0], vy = V[1] - c[1], vz = V[2] - c[2];
    const double t = -0.5 * ((uy * vz - uz * vy) * pf.x + (uz * vx - ux * vz) * pf.y + (ux * vy - uy * vx) * pf.z);
    a += t;
    mx += t * (c[0] + U[0] + V[0]) * (1.0 / 3.0);
    my += t * (c[1] + U[1] + V[1]) * (1.0 / 3.0);
    mz += t * (c[2] + U[2] + V[2]) * (1.0 / 3.0);
  });
  if (w.hc == 1) {
    out[0] = a;
  } else {
    out[0] = mx;
    out[1] = my;
    out[2] = mz;
    out[3] = a;
  }
}

// One round of facet pieces (lane: face f >= 0 or none) into w.harea,
// signed: each lane stages its piece, then lane c adds component c of
// every staged piece in lane order.
__device__ __noinline__ void hess_pieces(const ConePiece &q, const WarpCell &w, const double *px, const double *py,
                                         const double *pz, int f, double sgn, int lane) {
  const int hc = w.hc;
  double out[4] = {0, 0, 0, 0};
  if (f >= 0) face_piece(q, w, px, py, pz, f, out);
  for (int c = 0; c < hc; ++c) w.hstage[lane * hc + c] = sgn * out[c];
  w.hstage_f[lane] = f;
  __syncwarp();
  if (lane < hc)
    for (int l = 0; l < 32; ++l) {
      const int g = w.hstage_f[l];
      if (g >= 0) w.harea[g * hc + lane] += w.hstage[l * hc + lane];
    }
  __syncwarp();
}

// Sets up the cone of triangle tri from apex a; false for a flat cone.
__device__ bool cone_setup(ConePiece &q, const DevGrid &g, float4 s, int tri, const double a[3], double &sgn) {
  const float4 q1 = __ldg(&g.points[__ldg(&g.tris[3 * tri])]);
  const float4 q2 = __ldg(&g.points[__ldg(&g.tris[3 * tri + 1])]);
  const float4 q3 = __ldg(&g.points[__ldg(&g.tris[3 * tri + 2])]);
  const float4 qs[3] = {q1, q2, q3};
  double d[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    q.t[i][0] = double(qs[i].x) - s.x;
    q.t[i][1] = double(qs[i].y) - s.y;
    q.t[i][2] = double(qs[i].z) - s.z;
#pragma unroll
    for (int k = 0; k < 3; ++k) d[i][k] = q.t[i][k] - a[k];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) q.a[k] = a[k];
  const double det = d[0][0] * (d[1][1] * d[2][2] - d[1][2] * d[2][1]) -
                     d[0][1] * (d[1][0] * d[2][2] - d[1][2] * d[2][0]) +
                     d[0][2] * (d[1][0] * d[2][1] - d[1][1] * d[2][0]);
  if (!(fabs(det) > 0.0)) return false;
  // the reference's sign: + when the triangle is seen positively from a
  sgn = det > 0.0 ? 1.0 : -1.0;
  if (det < 0.0) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double x = q.t[1][k];
      q.t[1][k] = q.t[2][k];
      q.t[2][k] = x;
      x = d[1][k];
      d[1][k] = d[2][k];
      d[2][k] = x;
    }
  }
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double *u = d[j], *v = d[(j + 1) % 3];
    q.c[j][0] = u[1] * v[2] - u[2] * v[1];
    q.c[j][1] = u[2] * v[0] - u[0] * v[2];
    q.c[j][2] = u[0] * v[1] - u[1] * v[0];
    q.c[j][3] = -(q.c[j][0] * a[0] + q.c[j][1] * a[1] + q.c[j][2] * a[2]);
  }
  const double e1[3] = {q.t[1][0] - q.t[0][0], q.t[1][1] - q.t[0][1], q.t[1][2] - q.t[0][2]};
  const double e2[3] = {q.t[2][0] - q.t[0][0], q.t[2][1] - q.t[0][1], q.t[2][2] - q.t[0][2]};
  q.c[3][0] = e1[1] * e2[2] - e1[2] * e2[1];
  q.c[3][1] = e1[2] * e2[0] - e1[0] * e2[2];
  q.c[3][2] = e1[0] * e2[1] - e1[1] * e2[0];
  q.c[3][3] = -(q.c[3][0] * q.t[0][0] + q.c[3][1] * q.t[0][1] + q.c[3][2] * q.t[0][2]);
  q.acc[0] = q.acc[1] = q.acc[2] = q.acc[3] = 0.0;
  return true;
}

// Cone pieces of triangles tids[t0, t1) (at most 32), one per lane, summed
// over the warp into acc.  Needs build_faces.
template <bool HESS = false>
__device__ void facet_triangles(const WarpCell &w, const double *px, const double *py, const double *pz,
                                const DevGrid &g, float4 s, const int *tids, int t0, int t1, const double a[3],
                                double acc[4], int lane, unsigned long long *ctr) {
  ConePiece q;
  double sgn = 0.0;
  const bool act = t0 + lane < t1 && cone_setup(q, g, s, tids[t0 + lane], a, sgn);
  if (!act) q.acc[0] = q.acc[1] = q.acc[2] = q.acc[3] = 0.0;
  const int np = w.np;
  // t ∩ C, seen from a (outer side): edges t0 -> t2 -> t1 -> t0 clipped by
  // the cell planes, and the lines of the cell planes that cut t
  // cone axis and half-angle seen from a (floats, for culling the faces)
  float tux = 0.f, tuy = 0.f, tuz = 0.f, tth = 4.f, tc = -1.f, ts = 0.f;
  if (act) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const float dx = float(q.t[i][0] - a[0]), dy = float(q.t[i][1] - a[1]), dz = float(q.t[i][2] - a[2]);
      const float il = rsqrtf(fmaxf(dx * dx + dy * dy + dz * dz, 1e-30f));
      tux += dx * il;
      tuy += dy * il;
      tuz += dz * il;
    }
    const float ul = rsqrtf(fmaxf(tux * tux + tuy * tuy + tuz * tuz, 1e-30f));
    tux *= ul;
    tuy *= ul;
    tuz *= ul;
    float cmin = 1.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const float dx = float(q.t[i][0] - a[0]), dy = float(q.t[i][1] - a[1]), dz = float(q.t[i][2] - a[2]);
      const float il = rsqrtf(fmaxf(dx * dx + dy * dy + dz * dz, 1e-30f));
      cmin = fminf(cmin, (dx * tux + dy * tuy + dz * tuz) * il);
    }
    tth = acosf(fmaxf(-1.f, fminf(1.f, cmin)));
    tc = cosf(tth);
    ts = sinf(tth);
  }
  if (act) {
    // bounding sphere of t: a plane farther than its radius does not cut t
    const double gx = (q.t[0][0] + q.t[1][0] + q.t[2][0]) * (1.0 / 3.0);
    const double gy = (q.t[0][1] + q.t[1][1] + q.t[2][1]) * (1.0 / 3.0);
    const double gz = (q.t[0][2] + q.t[1][2] + q.t[2][2]) * (1.0 / 3.0);
    double r2 = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double dx = q.t[i][0] - gx, dy = q.t[i][1] - gy, dz = q.t[i][2] - gz;
      r2 = fmax(r2, dx * dx + dy * dy + dz * dz);
    }
    const double rad = sqrt(r2) * (1.0 + 1e-9) + 1e-9;
    double lo[3] = {0.0, 0.0, 0.0}, hi[3] = {1.0, 1.0, 1.0};
    for (int kb = 0; kb < np; kb += 64) {
      unsigned long long cutm = 0;
      const int ke = min(np, kb + 64);
      for (int kp = kb; kp < ke; ++kp) {
        const Plane pl = w.plane[kp];
        const double n[4] = {pl.x, pl.y, pl.z, pl.w};
        if (pval(n, gx, gy, gz) > rad) continue;
        const double e0 = pval(n, q.t[0][0], q.t[0][1], q.t[0][2]);
        const double e1 = pval(n, q.t[1][0], q.t[1][1], q.t[1][2]);
        const double e2 = pval(n, q.t[2][0], q.t[2][1], q.t[2][2]);
        if (e0 >= 0.0 && e1 >= 0.0 && e2 >= 0.0) continue;
        cutm |= 1ull << (kp - kb);
        clip_seg(e0, e2, lo[0], hi[0]);
        clip_seg(e2, e1, lo[1], hi[1]);
        clip_seg(e1, e0, lo[2], hi[2]);
      }
      // lines of the cutting planes in the triangle's plane (direction
      // n_3 x n_k keeps t ∩ C on the left seen from a), bounded by t's edges
      // and the other cutting planes: every other plane holds all of t
      const unsigned long long all = cutm;
      while (cutm) {
        const int kp = kb + __ffsll(cutm) - 1;
        cutm &= cutm - 1;
        const Plane pl = w.plane[kp];
        const double n[4] = {pl.x, pl.y, pl.z, pl.w};
        double x0[3], d[3];
        if (!plane_line(q.c[3], n, x0, d)) continue;
        double l = -1e300, h = 1e300;
#pragma unroll
        for (int j = 0; j < 3; ++j) clip_line(q.c[j], x0, d, l, h);
        unsigned long long others = all & ~(1ull << (kp - kb));
        while (others && l < h) {
          const int k2 = kb + __ffsll(others) - 1;
          others &= others - 1;
          const Plane p2 = w.plane[k2];
          const double n2[4] = {p2.x, p2.y, p2.z, p2.w};
          clip_line(n2, x0, d, l, h);
        }
        // cutting planes of the other batches
        for (int k2 = 0; k2 < np && l < h && np > 64; ++k2) {
          if (k2 >= kb && k2 < ke) continue;
          const Plane p2 = w.plane[k2];
          const double n2[4] = {p2.x, p2.y, p2.z, p2.w};
          clip_line(n2, x0, d, l, h);
        }
        if (l < h) {
          const double U[3] = {fma(l, d[0], x0[0]), fma(l, d[1], x0[1]), fma(l, d[2], x0[2])};
          const double V[3] = {fma(h, d[0], x0[0]), fma(h, d[1], x0[1]), fma(h, d[2], x0[2])};
          edge_tet(q, q.t[0], U, V);
        }
      }
    }
    const int ord[4] = {0, 2, 1, 0};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (!(lo[i] < hi[i])) continue;
      const double *u = q.t[ord[i]], *v = q.t[ord[i + 1]];
      const double U[3] = {fma(lo[i], v[0] - u[0], u[0]), fma(lo[i], v[1] - u[1], u[1]), fma(lo[i], v[2] - u[2], u[2])};
      const double V[3] = {fma(hi[i], v[0] - u[0], u[0]), fma(hi[i], v[1] - u[1], u[1]), fma(hi[i], v[2] - u[2], u[2])};
      edge_tet(q, q.t[0], U, V);
    }
  }
  // faces of the cell that the cone meets beyond t, 64 at a time
  for (int fb = 0; fb < np; fb += kFaceCap) {
    unsigned long long hit = 0;
    if (act) {
      const int fe = min(np, fb + kFaceCap);
      const float *ang = face_angles(w);
      const int acap = face_angle_cap(w);
      for (int f = fb; f < fe; ++f) {
        const int f0 = w.fstart[f], k = w.fstart[f + 1] - f0;
        if (k < 3) continue;
        if (f < acap) {
          // the cones from a around the face and around t must meet (both
          // narrower than a half-space, so each holds its convex hull)
          const float *g4 = ang + 6 * f;
          if (g4[3] < 1.5f && tth < 1.5f) {
            const float cosang = g4[0] * tux + g4[1] * tuy + g4[2] * tuz;
            if (cosang < g4[4] * tc - g4[5] * ts - 1e-3f) continue;
          }
        }
        unsigned any_in = 0;
        for (int i = 0; i < k && any_in != 15u; ++i) {
          const int v = w.fv[f0 + i];
          const double x = px[v], y = py[v], z = pz[v];
#pragma unroll
          for (int j = 0; j < 4; ++j) any_in |= (pval(q.c[j], x, y, z) >= 0.0 ? 1u : 0u) << j;
        }
        if (any_in == 15u) hit |= 1ull << (f - fb);
      }
    }
    while (__any_sync(kFull, hit != 0)) {
      int f = -1;
      if (hit) {
        f = fb + __ffsll(hit) - 1;
        hit &= hit - 1;
        face_facet(q, w, px, py, pz, f);
      }
      if constexpr (HESS) {
        if (w.harea) hess_pieces(q, w, px, py, pz, f, sgn, lane);
      }
    }
  }
  count(ctr, kCtrExports, t1 - t0, lane);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double v = act ? sgn * q.acc[k] * (1.0 / 24.0) : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    acc[k] += v;
  }
}

// Parked boundary cell: header, planes, vertices, triangle ids.
struct DeferHeader {
  int sid, nuniq, nv, np;
  double pt0[3];
  double acc[4];
  int inner, diag;  // diag: index of the cell's diagram in a batched launch
  int chunk_base;   // its first work item
  int fixed;        // >= 0: the cell's status, without any work (a cell parked ahead that failed)
  double pad[7];
};
static_assert(sizeof(DeferHeader) == 144, "defer header size");

__host__ __device__ inline size_t slot_bytes_for(const Layout &L, int T) {
  return size_t(align16(unsigned(sizeof(DeferHeader) + 32u * L.Pc + 44u * L.Vc + 4u * ((T + 3) & ~3) + 4u * L.Pc)));
}

// The slot's triangle-id list (nuniq ids, room for L.T).
__device__ __forceinline__ int *slot_list(const DeferQueue &dq, int slot, const Layout &L) {
  unsigned char *base = dq.slots + size_t(slot) * dq.slot_bytes;
  return reinterpret_cast<int *>(base + sizeof(DeferHeader) + 32u * L.Pc + 44u * L.Vc);
}

// list_in_place: the ids were gathered into the slot already.
__device__ void park_cell(const WarpCell &w, const DeferQueue &dq, int slot, const Layout &L, int diag, int sid,
                          int nuniq, bool inner, const double acc[4], int lane, bool list_in_place = false) {
  const int T = L.T;
  unsigned char *base = dq.slots + size_t(slot) * dq.slot_bytes;
  DeferHeader *h = reinterpret_cast<DeferHeader *>(base);
  Plane *pl = reinterpret_cast<Plane *>(base + sizeof(DeferHeader));
  double *vx = reinterpret_cast<double *>(pl + L.Pc);
  double *vy = vx + L.Vc, *vz = vy + L.Vc, *vw = vz + L.Vc, *vd = vw + L.Vc;
  unsigned *vt = reinterpret_cast<unsigned *>(vd + L.Vc);
  int *tl = reinterpret_cast<int *>(vt + L.Vc);
  const int nch = (nuniq + dq.chunk - 1) / dq.chunk;
  int cb = 0;
  if (lane == 0) {
    cb = atomicAdd(&dq.counters[2], nch);
    h->sid = sid;
    h->nuniq = nuniq;
    h->nv = w.nv;
    h->np = w.np;
    h->inner = inner ? 1 : 0;
    h->diag = diag;
    h->chunk_base = cb;
    h->fixed = -1;
    for (int d = 0; d < 3; ++d) h->pt0[d] = w.pts[d];
    for (int d = 0; d < 4; ++d) h->acc[d] = acc[d];
  }
  cb = __shfl_sync(kFull, cb, 0);
  for (int c = lane; c < nch; c += 32) dq.chunk_slot[cb + c] = slot;
  for (int i = lane; i < w.np; i += 32) pl[i] = w.plane[i];
  for (int v = lane; v < w.nv; v += 32) {
    vx[v] = w.cx[v];
    vy[v] = w.cy[v];
    vz[v] = w.cz[v];
    vw[v] = w.cw[v];
    vd[v] = w.d2[v];
    vt[v] = w.tri[v];
  }
  if (!list_in_place)
    for (int i = lane; i < nuniq; i += 32) tl[i] = w.tlist[i];
  if (w.pnb) {
    int *nb = tl + ((T + 3) & ~3);
    for (int i = lane; i < w.np; i += 32) nb[i] = w.pnb[i];
  }
}

// A slot taken for a cell parked ahead whose restriction ended early: its
// status, no work items (k_cone_finish writes every taken slot's cell).
__device__ void park_fixed(const DeferQueue &dq, int slot, int diag, int sid, int status, int lane) {
  if (lane == 0) {
    DeferHeader *h = reinterpret_cast<DeferHeader *>(dq.slots + size_t(slot) * dq.slot_bytes);
    h->sid = sid;
    h->nuniq = 0;
    h->nv = h->np = 0;
    h->inner = 0;
    h->diag = diag;
    h->chunk_base = 0;
    h->fixed = status;
    for (int d = 0; d < 4; ++d) h->acc[d] = 0.0;
  }
}

// Domain restriction of the clipped cell (ConvexCell.cl:918-1116): start
// corner, boundary triangles, signed cone decomposition.  Adds the cell's
// moments to acc; returns the status.
template <int VS, bool INL>
__device__ int restrict_to_domain(WarpCell &w, const CellLaunch &a, const Layout &L, float4 s, int sid_of_cell,
                                  double acc[4], int lane, unsigned long long *ctr, double *tr, int trcap) {
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
  bool ahead = false;
  if (g.tsat && nvox > 0) {
    // disjoint lists: the range's triangle count from the summed counts
    // (lane q < 8 reads corner q); more than T fails as the merge would,
    // before any list is read
    int part = 0;
    if (lane < 8) {
      const int S1 = S + 1;
      const int x = (lane & 1) ? vmax[0] + 1 : vmin[0], y = (lane & 2) ? vmax[1] + 1 : vmin[1],
                z = (lane & 4) ? vmax[2] + 1 : vmin[2];
      const int sign = ((lane & 1) ^ ((lane >> 1) & 1) ^ ((lane >> 2) & 1)) ? 1 : -1;
      part = sign * __ldg(&g.tsat[x + S1 * (y + S1 * z)]);  // + for an odd number of upper corners
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
    const int count = __shfl_sync(kFull, part, 0);
    if (count > a.T) {
      // more than T: the retry passes would clip this cell again to the
      // same cell and restrict it with a larger T; within T_ahead it is
      // parked now, its ids gathered straight into its slot
      if (INL || count > a.T_ahead || !a.defer.slots) {
        if (a.tri_count && lane == 0) a.tri_count[sid_of_cell] = count;
        return kTriangleOverflow;
      }
      ahead = true;
    }
  }
  const DeferQueue &dq = a.defer;
  int *tl = w.tlist, tcap = L.G, slot = 0;
  if (ahead) {
    if (lane == 0) slot = atomicAdd(&dq.counters[0], 1);
    slot = __shfl_sync(kFull, slot, 0);
    if (slot >= dq.capacity) return kTriangleOverflow;  // the retry passes take it (count unknown to them)
    tl = slot_list(dq, slot, L);
    tcap = L.T;
  }
  // first corner with flag != 1 in (z, y, x) scan order, and the triangle ids
  // of every voxel in the range
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
    const int incl = warp_incl_scan(cntv, lane);
    const int tot = __shfl_sync(kFull, incl, 31);
    if (ntr + tot > tcap) {
      spill = true;
    } else if (!spill) {
      for (int k = 0; k < cntv; ++k) tl[ntr + incl - cntv + k] = __ldg(&g.list[lo_off + k]);
    }
    ntr += tot;
  }
  __syncwarp();
  int nuniq = 0;
  if (g.lists_disjoint) {
    // no triangle is listed twice: the union is the concatenation
    if (ntr > (ahead ? a.T_ahead : a.T)) {
      if (ahead) park_fixed(dq, slot, a.diag, sid_of_cell, kTriangleOverflow, lane);
      return ahead ? kDeferred : kTriangleOverflow;
    }
    nuniq = ntr;
  } else if (spill) {
    // more ids (with repeats) than the sort buffer holds: one lane builds the
    // sorted union voxel by voxel, failing past T like the reference's merge
    int cntu = 0;
    if (lane == 0) cntu = serial_union(g, vmin, vmax, a.T, w.tlist, L.G);
    cntu = __shfl_sync(kFull, cntu, 0);
    __syncwarp();
    if (cntu < 0) return kTriangleOverflow;
    nuniq = cntu;
  } else if (ntr > 0) {
    const int n2 = pow2_at_least(ntr);
    for (int i = ntr + lane; i < n2; i += 32) w.tlist[i] = 0x7fffffff;
    __syncwarp();
    warp_sort_ints(w.tlist, n2, lane);
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
    if (nuniq > a.T) return kTriangleOverflow;
  }
  double pt0[3] = {0, 0, 0};
  if (in_domain == 1) {
    int px = 0, py = 0, pz = 0, f = 1;
    // a cell parked ahead is restricted as a retry pass would restrict it
    if ((ahead ? a.out_domain_ahead : a.out_domain) && lane == 0) f = out_domain_corner(g, vmin, vmax, px, py, pz);
    f = __shfl_sync(kFull, f, 0);
    if (f == 1) {
      if (ahead) park_fixed(dq, slot, a.diag, sid_of_cell, kFindAnotherBeginningVertex, lane);
      return ahead ? kDeferred : kFindAnotherBeginningVertex;
    }
    in_domain = f;
    pt0[0] = __shfl_sync(kFull, px, 0) * double(g.voxel) - s.x;
    pt0[1] = __shfl_sync(kFull, py, 0) * double(g.voxel) - s.y;
    pt0[2] = __shfl_sync(kFull, pz, 0) * double(g.voxel) - s.z;
  } else {
    const int x = c0 % S, y = (c0 / S) % S, z = c0 / (S * S);
    pt0[0] = x * double(g.voxel) - s.x;
    pt0[1] = y * double(g.voxel) - s.y;
    pt0[2] = z * double(g.voxel) - s.z;
  }
  if (nuniq > 0) {
    count(ctr, kCtrBoundaryCells, 1, lane);
    count(ctr, kCtrTriangles, nuniq, lane);
  }
  bool inner = false;
  // The facet pieces of an inner apex clip nothing, so they cannot overflow
  // a cap; the reference's cones clip the cell by up to 4 planes each (its
  // status is plane_overflow when a plane check before one finds P planes,
  // vertex_overflow past V vertices).  A clip adds at most one face, and a
  // closed cell of f faces has 2f - 4 vertices, so with P >= planes + 4 and
  // V >= vertices + 8 no cone can overflow and the inner apex gives the
  // reference's status; else a count of the cuts per cone (ref_cones_fit)
  // may still show it.  Otherwise the cones run from the start corner and
  // fail where the reference's fail.
  if (nuniq > 0 && a.inner_apex &&
      ((w.np + 4 <= a.P && w.nv + 8 <= a.V) ||
       ref_cones_fit(w, g, s, tl, nuniq, pt0, a.P, a.V, sqrt(cell_radius2<VS>(w, lane)), lane))) {
    double ap[3];
    const int f = inner_apex(w, g, s, vmin, vmax, tl, nuniq, ap, lane);
    if (f >= 0) {
      inner = true;
      in_domain = f;
      for (int d = 0; d < 3; ++d) pt0[d] = ap[d];
      const int kept = drop_separated(w, g, s, tl, nuniq, lane);
      count(ctr, kCtrConesSkipped, nuniq - kept, lane);
      nuniq = kept;
    }
  }
  if (nuniq > 0 && !inner) count(ctr, kCtrStartCorner, 1, lane);
  trace_rec(tr, trcap, lane, 5, pt0[0], pt0[1], pt0[2], in_domain, nuniq);
  if (in_domain == 2) integrate<VS, INL>(w, 1.0, acc, lane, ctr, tr, trcap);
  if (nuniq == 0 && !ahead) return kSuccess;
  if (lane < 3) w.pts[lane] = pt0[lane];
  __syncwarp();
  if (ahead) {
    // its slot is taken: parked even without triangles.  Without an inner
    // apex the cones clip the cell, which depends on the retry pass's P and
    // V: the retries take it, as a triangle overflow now
    if (!inner) {
      park_fixed(dq, slot, a.diag, sid_of_cell, kTriangleOverflow, lane);
    } else {
      park_cell(w, dq, slot, L, a.diag, sid_of_cell, nuniq, inner, acc, lane, true);
      // the retry passes' T schedule follows the counts settled ahead
      if (lane == 0) atomicMax(a.ahead_max ? a.ahead_max : &dq.counters[3], ntr);
    }
    return kDeferred;
  }
  if (dq.slots && (!INL || nuniq > dq.inline_max)) {
    // park the cell: its triangles become work items of k_cone
    int slot = 0;
    if (lane == 0) slot = atomicAdd(&dq.counters[0], 1);
    slot = __shfl_sync(kFull, slot, 0);
    if (slot < dq.capacity) {
      park_cell(w, dq, slot, L, a.diag, sid_of_cell, nuniq, inner, acc, lane);
      return kDeferred;
    }
  }
  if constexpr (!INL) {
    return kParkOverflow;  // re-run by the inline variant
  } else {
    if (inner) {
      build_faces(w, w.bcx, w.bcy, w.bcz, pt0, lane);
      for (int b0 = 0; b0 < nuniq; b0 += 32)
        facet_triangles<INL>(w, w.bcx, w.bcy, w.bcz, g, s, w.tlist, b0, min(nuniq, b0 + 32), pt0, acc, lane, ctr);
      return kSuccess;
    }
    const int bk_nv = w.nv, bk_np = w.np;
    backup<VS>(w, lane);
    // the triangles in chunks of 32, each summed on its own and then added,
    // as k_cone sums a parked cell: a cell's result does not depend on
    // whether it was parked
    for (int c0 = 0; c0 < nuniq; c0 += 32) {
      double part[4] = {0, 0, 0, 0};
      int fail_at = 0;
      const int st = cone_triangles<VS, INL>(w, a, s, w.tlist, c0, min(nuniq, c0 + 32), bk_nv, bk_np, inner, part,
                                        fail_at, lane, ctr, tr, trcap);
      if (st != kSuccess) return st;
      for (int d = 0; d < 4; ++d) acc[d] += part[d];
    }
    return kSuccess;
  }
}

// CCUpdateUsedCell (ConvexCell.cl:680-690): the plane neighbours of the
// cell's vertices get mark d where they have none.  Concurrent cells write
// the same flags: relaxed byte accesses, as in the reference.
__device__ __forceinline__ void mark_neighbours(unsigned char *used, const unsigned *tri, int nv, const int *pnb, int d,
                                                int lane, int nlanes) {
  for (int v = lane; v < nv; v += nlanes) {
    const unsigned t = tri[v];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int nb = pnb[(t >> (8 * i)) & 0xff];
      if (nb >= 0 && *(volatile unsigned char *)&used[nb] == 0) *(volatile unsigned char *)&used[nb] = (unsigned char)d;
    }
  }
}

// Whether the seed lies strictly inside its own power cell, which is then
// not empty.  The bisector with b keeps the seed when |s - b|^2 + w_b - w_s
// > 0 (a wall's plane always does), which holds for every b when
// w_s - min w < d^2, d^2 a lower bound of the nearest other seed's squared
// distance (vmask bit 0: there is one) and min w over the seeds that are not
// walls.  The early exits outside the domain need it: an empty cell's status
// is empty_cell, not success.  The factor covers the float rounding of
// neighbour orders and bins.
__device__ __forceinline__ bool nonempty_cell(float4 s, unsigned vmask, double d2_nearest, const int *wmin) {
  return (vmask & 1u) && double(s.w) - double(ordered_to_float(__ldg(wmin))) < 0.999 * d2_nearest;
}

// The security-radius test: no neighbour past the j-th (at squared distance
// d2j, the neighbours sorted by distance) can cut the cell of squared radius
// R2.  The reference's test is the Voronoi one, d2j > 4 R2
// (ConvexCell.cl:364-382).  With safe_dw >= 0 (CellLaunch::safe_radius; it
// is w_s - min w, the weights added to the squared distances as the
// reference adds them) the weighted guard instead: a neighbour at distance
// d' >= d_j with weight >= min w has its bisector at offset
// (d'^2 + w' - w_s) / (2 d') >= R -- so it cannot cut the ball of radius R
// around the seed, which holds the cell -- once d_j > R and
// d_j^2 - 2 R d_j > w_s - min w (the left side grows with d' past R).
// Squared, without roots: d_j > R and 2 R d_j < d_j^2 - c hold together when
// d2j > R2, d2j > c and 4 R2 d2j < (d2j - c)^2 (c = safe_dw >= 0).
__device__ __forceinline__ bool radius_reached(double d2j, double R2, double safe_dw) {
  if (!(safe_dw >= 0.0)) return d2j > 4.0 * R2;
  const double e = d2j - safe_dw;
  return d2j > R2 && e > 0.0 && 4.0 * R2 * d2j < e * e;
}

// Squared distance between two seeds, as the clipping loop computes it.
__device__ __forceinline__ double seed_dist2(float4 b, float4 s) {
  const double bx = double(b.x) - double(s.x), by = double(b.y) - double(s.y), bz = double(b.z) - double(s.z);
  return bx * bx + by * by + bz * bz;
}

// A cell proven outside the domain (its squared radius at most r_plain^2)
// has the reference's result mass 0 and status success only if the
// reference's clipping of it, which goes on through the neighbours, ends in
// success.  How far it goes at most: the cell's radius only shrinks, so past
// neighbour j (clipped, squared radius R2) the first neighbour z >= j that
// reaches the security radius at R2 ends it (the last neighbour clipped: z),
// as does the end of the list at z (z - 1: every other seed clipped).
// Returns that index, or -1 when neither comes within K.  R2 carries a
// relative margin of 1e-9 for the rounding of the later cells' vertices.
__device__ int last_clip(const CellLaunch &a, const unsigned *nrow, float4 s, int j, double R2, double dw, int lane) {
  const double R2m = R2 * (1.0 + 1e-9);
  for (int c0 = j & ~31; c0 < a.K; c0 += 32) {
    const int i = c0 + lane;
    bool stop = false, none = false;
    if (i >= j && i < a.K) {
      const unsigned z = __ldg(&nrow[i]);
      none = z == kNone;
      stop = none || radius_reached(seed_dist2(__ldg(&a.stored[z]), s), R2m, dw);
    }
    const unsigned m = __ballot_sync(kFull, stop);
    if (m) {
      const int src = __ffs(m) - 1;
      return c0 + src - (__shfl_sync(kFull, none, src) ? 1 : 0);
    }
  }
  return -1;
}

// Whether the reference's clipping of a cell proven outside the domain,
// continued past neighbour j (clipped; the cell has w.np planes, w.nv
// vertices and squared radius R2), surely ends in success.  It goes on to
// the last neighbour e (last_clip; the lanes' bisectors pl / squared
// distances nd2 / valid flags of neighbours i0 + lane serve the current
// chunk), and of the neighbours j+1 .. e only those whose bisector has a
// vertex of the current cell on its far side can cut a later cell: every
// later cell lies in this one, whose farthest point beyond a plane is a
// vertex (a margin of 1e-9 of the plane offset plus the radius covers the
// rounding of the later cells' vertices).  With c of them, np + c < P keeps
// every plane check before a clip below P and nv + 2c <= V every clip within
// V (a cut adds at most one face to the closed cell, whose f faces make
// 2f - 4 vertices); counting stops once c passes that.  The cell cannot
// become empty (nonempty_cell gates the exits).  A later clip that meets a
// degenerate cavity (inconsistent_boundary) is the one failure this cannot
// foresee.  The FP32 clipping keeps no FP64 vertices: there every later
// neighbour counts as a cut.  One neighbour per lane, every vertex in turn.
template <int VS, int PREC>
__device__ bool outside_certain(const WarpCell &w, const CellLaunch &a, const unsigned *nrow, float4 s, int i0, int j,
                                const Plane &pl, double nd2, bool valid, double R2, double dw, int lane) {
  const int cmax = min(a.P - w.np - 1, (a.V - w.nv) >> 1);  // the most cuts the caps allow
  // the last neighbour clipped: in the current chunk from the lanes' data,
  // past it from the table
  int e;
  {
    const int i = i0 + lane;
    const bool stop = i >= j && i < a.K && (!valid || radius_reached(nd2, R2 * (1.0 + 1e-9), dw));
    const unsigned m = __ballot_sync(kFull, stop);
    if (m) {
      const int src = __ffs(m) - 1;
      e = i0 + src - (__shfl_sync(kFull, valid, src) ? 0 : 1);
    } else {
      e = i0 + 32 < a.K ? last_clip(a, nrow, s, i0 + 32, R2, dw, lane) : -1;
    }
  }
  if (e < 0) return false;
  if (e - j <= max(cmax, 0)) return e - j == 0 || cmax >= e - j;
  if (cmax < 0) return false;
  if constexpr (PREC > 0) {
    return false;
  } else {
    const double R = sqrt(R2);
    int c = 0;
    for (int c0 = i0; c0 <= e; c0 += 32) {
      const int i = c0 + lane;
      Plane pc = pl;
      if (c0 > i0 && i <= e) {
        // a later chunk: the lanes build its bisectors as the clipping loop does
        const float4 b = __ldg(&a.stored[__ldg(&nrow[i])]);
        const double bx = double(b.x) - double(s.x), by = double(b.y) - double(s.y), bz = double(b.z) - double(s.z);
        const double d2 = bx * bx + by * by + bz * bz;
        const double len = sqrt(d2), inv = 1.0 / len;
        const double off = b.w <= kNoCellLimits ? len : (d2 + (double(b.w) - double(s.w))) * (0.5 * inv);
        pc = Plane{-bx * inv, -by * inv, -bz * inv, off};
      }
      bool cut = false;
      if (i > j && i <= e) {
        const double tol = kTieEps - 1e-9 * (fabs(pc.w) + R);
        for (int v = 0; v < w.nv && !cut; ++v) {
          const double cw = w.cw[v];
          cut = plane_side(w.cx[v], w.cy[v], w.cz[v], cw, pc) > tol * fabs(cw);
        }
      }
      c += __popc(__ballot_sync(kFull, cut));
      if (c > cmax) return false;
    }
    return true;
  }
}

// The vertex capacity a cell of this launch works with.  A batched launch's
// layout may hold more vertices than a diagram's cap (it is sized for every
// diagram); capacity-dependent choices follow the diagram's own cap, so a
// cell's result does not depend on the other diagrams of its batch.
__device__ __forceinline__ int vertex_capacity(const CellLaunch &a, const Layout &L) {
  return min(L.Vc, (a.V + 31) & ~31);
}

// One row of a cell launch (one warp): clip, restrict, integrate, write.
// `only_status` >= 0: skip the row unless its cell has that status; vc:
// the vertex capacity (vertex_capacity).
// SAFE: 1 -- the launch record's safe_radius selects the weighted
// security-radius guard (radius_reached); 0 -- the reference's test, compiled
// without the guard (its code costs the default clipping loop ~5%).
template <int VS, bool GRID, bool INL, int PREC = 0, int SAFE = 0>
__device__ __forceinline__ void cell_row(const CellLaunch &a, const Layout &L, unsigned char *wsmem, int row,
                                         int only_status, int vc, int lane) {
  WarpCell w = bind(wsmem, L);
  w.vc = vc;
  unsigned long long *ctr = a.counters;
  const int sid = a.ids ? a.ids[row] : row;
  if (only_status >= 0 && a.status[sid] != only_status) return;
  // Hessian rows run inline only (no defer queue)
  if constexpr (INL) {
    if (a.hess && lane == 0) a.hessid[size_t(sid) * a.H] = -1;  // an empty row until the cell succeeds
  }
  if constexpr (GRID) {
    if (a.tri_count && a.border_d == 0) {
      if (a.tri_first) {
        if (lane == 0) a.tri_count[sid] = 0;
      } else if (a.tri_count[sid] > a.T) {
        // clipped again it would be the same cell, past T again
        if (lane == 0) {
          a.status[sid] = kTriangleOverflow;
          a.out[sid] = make_double4(0.0, 0.0, 0.0, 0.0);
        }
        return;
      }
    }
  }
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
  init_box<PREC>(w, s, a.cube_eps, lane);
  if constexpr (INL) {
    if (w.harea) {
      for (int i = lane; i < w.hc * (L.Pc + 4); i += 32) w.harea[i] = 0.0;
      __syncwarp();
    }
  }
  // FP64: the squared radius.  FP32 clipping: its bounds, and the exact value
  // once escalated (R2 < 0: not known for the current cell)
  double R2 = PREC ? -1.0 : cell_radius2<VS>(w, lane);
  float R2hi = 0.0f, R2lo = 0.0f;
  int esc[kEscNum] = {0, 0, 0};
  if constexpr (PREC > 0) radius2_bounds<VS>(w, lane, R2hi, R2lo);
  // plane neighbours for the used cells and the Hessian
  const bool used_on = GRID && a.used != nullptr;
  const bool track_nb = used_on || (INL && a.hess != nullptr);
  if (track_nb && lane < 6) w.pnb[lane] = -1;

  // ---- power clipping by the K nearest, in order ----
  const unsigned *nrow = a.knn + size_t(row) * a.K;
  bool reached = false, exhausted = false, outside = false;
  const bool early = GRID && a.early_out && a.grid.sat != nullptr && a.wmin != nullptr && a.border_d == 0;
  double plain2 = early ? plain_radius2(a.grid, s, lane) : -1.0;
  // once the cell is proven outside (out_known), clipping stops where the
  // rest of the reference's clipping surely succeeds (outside_certain), else
  // goes on, and the cell, once it succeeds, skips the restriction
  bool out_known = false;
  // the weighted security-radius guard (radius_reached): w_s - min w when
  // on (computed where used, so the default loop carries nothing), else -1
  auto safe_dw = [&]() -> double {
    if constexpr (SAFE) {
      return a.safe_radius && a.wmin ? fmax(0.0, double(s.w) - double(ordered_to_float(__ldg(a.wmin)))) : -1.0;
    } else {
      return -1.0;
    }
  };
  for (int i0 = 0; i0 < a.K && status == kSuccess && !reached && !exhausted && !outside; i0 += 32) {
    // every lane builds the bisector of one neighbour, in double
    const int i = i0 + lane;
    Plane pl{0.0, 0.0, 0.0, 0.0};
    double nd2 = 0.0;
    bool valid = false;
    unsigned zl = kNone;
    if (i < a.K) {
      const unsigned z = __ldg(&nrow[i]);
      zl = z;
      if (z != kNone) {
        const float4 b = __ldg(&a.stored[z]);
        const double bx = double(b.x) - double(s.x), by = double(b.y) - double(s.y), bz = double(b.z) - double(s.z);
        nd2 = bx * bx + by * by + bz * bz;
        const double len = sqrt(nd2), inv = 1.0 / len;
        // kept side contains the seed: n = -(b - s)/|b - s|, offset of the
        // power bisector (ConvexCell.cl:321-328) or, for a wall neighbour,
        // through the neighbour itself
        const double off = b.w <= kNoCellLimits ? len : (nd2 + (double(b.w) - double(s.w))) * (0.5 * inv);
        pl = Plane{-bx * inv, -by * inv, -bz * inv, off};
        if constexpr (PREC == 2) pl = Plane{double(float(pl.x)), double(float(pl.y)), double(float(pl.z)), double(float(pl.w))};
        valid = true;
      }
    }
    const float4 pl32 = PREC ? plane_f(pl) : make_float4(0.f, 0.f, 0.f, 0.f);
    const unsigned vmask = __ballot_sync(kFull, valid);
    if (i0 == 0 && plain2 >= 0.0 && !nonempty_cell(s, vmask, __shfl_sync(kFull, nd2, 0), a.wmin)) plain2 = -1.0;
    const int cnt = min(32, a.K - i0);
    for (int j = 0; j < cnt; ++j) {
      if (!((vmask >> j) & 1u)) {
        exhausted = true;  // fewer than K other seeds: all have been clipped
        break;
      }
      const Plane e = shfl_plane(pl, j);
      const double d2j = __shfl_sync(kFull, nd2, j);
      count(ctr, kCtrPlanesTested, 1, lane);
      if (w.np >= a.P) {
        status = kPlaneOverflow;
        break;
      }
      int r;
      if constexpr (PREC > 0) {
        const float4 e32 = make_float4(__shfl_sync(kFull, pl32.x, j), __shfl_sync(kFull, pl32.y, j),
                                       __shfl_sync(kFull, pl32.z, j), __shfl_sync(kFull, pl32.w, j));
        r = clip<VS, PREC>(w, e, a.V, status, lane, ctr, tr, trcap, &e32, esc);
      } else {
        r = clip<VS>(w, e, a.V, status, lane, ctr, tr, trcap);
      }
      if (track_nb) {
        const unsigned zj = __shfl_sync(kFull, zl, j);
        if (r > 0 && lane == 0) w.pnb[w.np - 1] = int(zj);
      }
      if (r < 0) break;
      if constexpr (PREC == 0) {
        if (r > 0) {
          R2 = cell_radius2<VS>(w, lane);
          if (R2 <= plain2) {
            out_known = true;
            if (outside_certain<VS, PREC>(w, a, nrow, s, i0, i0 + j, pl, nd2, valid, R2, safe_dw(), lane)) {
              outside = true;
              break;
            }
          }
        }
        if (radius_reached(d2j, R2, safe_dw())) {
          reached = true;
          break;
        }
      } else {
        if (r > 0) {
          radius2_bounds<VS>(w, lane, R2hi, R2lo);
          R2 = -1.0;
          if (plain2 >= 0.0) {
            bool out;
            if (PREC == 2 || double(R2hi) <= plain2) {
              out = double(R2hi) <= plain2;
            } else if (double(R2lo) > plain2) {
              out = false;
            } else {
              R2 = radius2_exact<VS>(w, lane);
              ++esc[kEscRadii];
              out = R2 <= plain2;
            }
            if (out) {
              out_known = true;
              if (outside_certain<VS, PREC>(w, a, nrow, s, i0, i0 + j, pl, nd2, valid,
                                            R2 >= 0.0 ? R2 : double(R2hi), safe_dw(), lane)) {
                outside = true;
                break;
              }
            }
          }
        }
        // the test is monotone in R2: reached at the upper bound means
        // reached, not reached at the lower bound means not
        bool done;
        if (PREC == 2 || radius_reached(d2j, double(R2hi), safe_dw())) {
          done = radius_reached(d2j, double(R2hi), safe_dw());
        } else if (!radius_reached(d2j, double(R2lo), safe_dw())) {
          done = false;
        } else {
          if (R2 < 0.0) {
            R2 = radius2_exact<VS>(w, lane);
            ++esc[kEscRadii];
          }
          done = radius_reached(d2j, R2, safe_dw());
        }
        if (done) {
          reached = true;
          break;
        }
      }
    }
  }
  if constexpr (PREC > 0) {
    if (ctr) {
      // escalations of the FP32 clipping (counted by the lanes that ran them;
      // the radius ones by every lane)
#pragma unroll
      for (int k = 0; k < kEscNum; ++k) {
        int v = k == kEscRadii ? (lane == 0 ? esc[k] : 0) : esc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
        count(ctr, kCtrEscTests + k, (unsigned long long)v, lane);
      }
    }
    // the FP64 state for the restriction and integration
    if (status == kSuccess && !outside && a.border_d == 0) promote(w, lane);
  }
  if (status == kSuccess && !reached && !exhausted && !outside) status = kSecurityRadiusNotReached;
  if (status == kSuccess && out_known) outside = true;
  const int np_cell = w.np;  // the clipped cell's planes (cone planes come after)
  if (a.border_d > 0) {
    // bordering pass (ConvexCell.cl:756-809): the clipped cell marks its
    // neighbours; statuses and moments stay those of the main passes
    __syncwarp();
    if (status == kSuccess) mark_neighbours(a.used, w.tri, w.nv, w.pnb, a.border_d, lane, 32);
    return;
  }
  if (outside) count(ctr, kCtrOutside, 1, lane);
  if (status == kSuccess && !outside) {
    if (GRID)
      status = restrict_to_domain<VS, INL>(w, a, L, s, sid, acc, lane, ctr, tr, trcap);
    else
      integrate<VS, INL>(w, 1.0, acc, lane, ctr, tr, trcap);
  }
  if (status == kDeferred) return;  // k_cone_finish writes it
  if (status == kParkOverflow) {
    if (lane == 0) a.status[sid] = kParkOverflow;
    return;
  }
  if (INL && a.hess && status == kSuccess) {
    // the row (ConvexCell.cl:1133-1150): facets with a neighbour and an area
    // above 0.2, in plane order; more than H is hessian_overflow, which
    // keeps the moments
    __syncwarp();
    if (lane == 0) {
      const int hc = a.HC, H = a.H;
      double *hrow = a.hess + size_t(sid) * H * hc;
      int *hids = a.hessid + size_t(sid) * H;
      int cnt = 0;
      for (int p = 0; p < np_cell; ++p) {
        const double ar = w.harea[p * hc + hc - 1];
        if (w.pnb[p] < 0 || ar <= 0.2) continue;
        if (cnt >= H) {
          status = kHessianOverflow;
          break;
        }
        if (hc == 1) {
          hrow[cnt] = ar;
        } else {
          hrow[4 * cnt + 0] = w.harea[4 * p + 0] + ar * double(s.x);
          hrow[4 * cnt + 1] = w.harea[4 * p + 1] + ar * double(s.y);
          hrow[4 * cnt + 2] = w.harea[4 * p + 2] + ar * double(s.z);
          hrow[4 * cnt + 3] = ar;
        }
        hids[cnt] = w.pnb[p];
        ++cnt;
      }
      if (status == kSuccess && cnt < H) hids[cnt] = -1;
    }
    status = __shfl_sync(kFull, status, 0);
  }
  if (lane == 0) {
    a.status[sid] = status;
    // local moments -> global: sum w*(x_local + s) = m_local + m * s
    const double m = acc[3];
    if (status == kSuccess || status == kHessianOverflow)
      a.out[sid] = make_double4(acc[0] + m * double(s.x), acc[1] + m * double(s.y), acc[2] + m * double(s.z), m);
    else
      a.out[sid] = make_double4(0.0, 0.0, 0.0, 0.0);
  }
  if (used_on && status == kSuccess && acc[3] >= a.keep_volume) {
    // a used cell (ConvexCell.cl:1118-1126)
    if (lane == 0) *(volatile unsigned char *)&a.used[sid] = 1;
    __syncwarp();
    if (a.mark_dist >= 1) mark_neighbours(a.used, w.tri, w.nv, w.pnb, 1, lane, 32);
  }
}

template <int VS, bool GRID, bool INL, int PREC = 0, int SAFE = 0>
__global__ void __launch_bounds__(128, 5) k_cell(const __grid_constant__ CellLaunch a, const __grid_constant__ Layout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= a.num) return;
  cell_row<VS, GRID, INL, PREC, SAFE>(a, L, smem + size_t(threadIdx.x >> 5) * L.total, row, a.only_status, L.Vc,
                                      lane);
}

// Cage test of the outside probe: bit i of the result is set when the
// candidate's bisector bounds every direction u within kCageCover of the
// stencil direction d_i (the 26 unit vectors (x, y, z)/|(x, y, z)|, x, y, z
// in {-1, 0, 1}) to at most r from the seed.  Those directions cover the
// sphere: every unit vector lies within 27.57 degrees of one of them
// (kCageCover = 28 keeps a margin).  The bisector keeps x . n <= off (n the
// unit vector towards the candidate, off its offset, positive for a cell
// that cannot be empty); along u at angle at most c + t from n (t = the
// angle of n to d_i) that bounds the cell by off / cos(c + t), which is at
// most r when cos(c) cos(t) - off/r >= sin(c) sin(t) -- squared, no root.
// Float, with margins far above its rounding: off/r raised by 0.1%, cos(t)
// lowered by 1e-3.
constexpr float kCageCos = 0.882947592858927f;   // cos(28 deg)
constexpr float kCageSin2 = 0.2204035482646266f;  // sin(28 deg)^2
constexpr unsigned kCageAll = (1u << 26) - 1u;

__device__ __forceinline__ unsigned cage_bits(float nx, float ny, float nz, float q) {
  unsigned bits = 0;
  int i = 0;
#pragma unroll
  for (int z = -1; z <= 1; ++z)
#pragma unroll
    for (int y = -1; y <= 1; ++y)
#pragma unroll
      for (int x = -1; x <= 1; ++x) {
        if (x == 0 && y == 0 && z == 0) continue;
        const int nnz = (x != 0) + (y != 0) + (z != 0);
        const float inv_norm = nnz == 1 ? 1.0f : (nnz == 2 ? 0.70710678f : 0.57735027f);
        const float ct = (float(x) * nx + float(y) * ny + float(z) * nz) * inv_norm - 1e-3f;
        const float lhs = kCageCos * ct - q;
        if (lhs >= 0.0f && lhs * lhs >= kCageSin2 * (1.0f - ct * ct)) bits |= 1u << i;
        ++i;
      }
  return bits;
}

// Outside probe (ProbeLaunch), one warp per stored seed, over the seeds of
// the 3x3x3 bins around the seed's bin (up to 8 rounds of 32).  First the
// cage test (cage_bits) with every candidate: all 26 directions bounded to
// the plainly-outside ball proves the cell outside without clipping.  Else,
// with a ball of at least min_plain, the 32 nearest candidates (warp
// bitonic merges) clip the box in distance order until the cell fits the
// ball.
// vc: the vertex capacity the warp works with (the layout's, or a batched
// diagram's own, vertex_capacity).
template <int VS>
__device__ __forceinline__ void probe_row(const ProbeLaunch &p, const Layout &L, unsigned char *wsmem, int r,
                                          int vc, int lane) {
  WarpCell w = bind(wsmem, L);
  w.vc = vc;
  const int row = p.first + r;  // the seed's stored index
  const float4 s = p.stored[row];
  const double plain2 = s.w <= kNoCellLimits ? -1.0 : plain_radius2(p.grid, s, lane);
  bool proven = false;
  if (plain2 >= p.min_plain_cage * p.min_plain_cage) {
    // candidate rows of the 3x3x3 block: lane q < 9 holds row (y, z) offsets
    const int dim = p.dim, cin = bin_of(s, dim);
    const int cx = cin % dim, cy = (cin / dim) % dim, cz = cin / (dim * dim);
    int a0 = 0, cnt = 0;
    if (lane < 9) {
      const int y = cy + lane % 3 - 1, z = cz + lane / 3 - 1;
      if (y >= 0 && y < dim && z >= 0 && z < dim) {
        const int rb = (y + z * dim) * dim;
        a0 = __ldg(&p.bins[rb + max(cx - 1, 0)]);
        cnt = __ldg(&p.bins[rb + min(cx + 1, dim - 1) + 1]) - a0;
      }
    }
    const int incl = warp_incl_scan(cnt, lane);
    const int all = __shfl_sync(kFull, incl, 31);
    const int total = min(all, 8 * 32);
    // stored index of candidate c (c < total): its row's first seed plus
    // its rank in the row (owner: the first lane whose inclusive count
    // exceeds c)
    auto candidate = [&](int c) {
      int owner = 0;
#pragma unroll
      for (int step = 8; step > 0; step >>= 1) {
        const int v = __shfl_sync(kFull, incl, owner + step - 1);
        if (v <= c) owner += step;
      }
      return __shfl_sync(kFull, a0, owner) - (__shfl_sync(kFull, incl, owner) - __shfl_sync(kFull, cnt, owner)) + c;
    };
    // cage test over the candidates within 2 r of the seed.  The reference's
    // clipping stops at a neighbour z past twice the cell's radius R_z;
    // either it has clipped every cage candidate (its cell lies in the cage)
    // or one at distance d_c >= d_z > 2 R_z is left, and R_z < d_c / 2 <= r:
    // with weights, where its cell can be larger than the power cell, it
    // still lies in the ball
    const float inv_r = float(1.0 / sqrt(plain2)) * 1.001f;
    const float max_d2 = float(4.0 * plain2) * 0.999f;
    unsigned mask = 0;
    float mind2 = INFINITY;
    for (int base = 0; base < total; base += 32) {
      const int c = base + lane;
      const int ptr = candidate(c);
      if (c < total && ptr != row) {
        const float4 q = __ldg(&p.stored[ptr]);
        const float dx = q.x - s.x, dy = q.y - s.y, dz = q.z - s.z;
        const float d2 = dx * dx + dy * dy + dz * dz;
        const float len = sqrtf(d2), inv = 1.0f / len;
        const float off = q.w <= kNoCellLimits ? len : (d2 + (q.w - s.w)) * (0.5f * inv);
        mind2 = fminf(mind2, d2);
        if (d2 <= max_d2) mask |= cage_bits(dx * inv, dy * inv, dz * inv, off * inv_r);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mask |= __shfl_xor_sync(kFull, mask, o);
      mind2 = fminf(mind2, __shfl_xor_sync(kFull, mind2, o));
    }
    // every seed within a bin width of this one lies in the block, so the
    // nearest candidate (when all were read) or that width bounds the
    // nearest seed's distance
    const double bw = 0.999 * 1000.0 / dim;
    const double d2n = fmin(double(mind2) * (1.0 - 1e-5), bw * bw);
    const bool nonempty = all == total && nonempty_cell(s, mind2 < INFINITY ? 1u : 0u, d2n, p.wmin);
    proven = nonempty && mask == kCageAll;
    if (nonempty && !proven && plain2 >= p.min_plain * p.min_plain) {
      // the 32 nearest candidates, sorted
      unsigned long long best = kEmptyKey;
      for (int base = 0; base < total; base += 32) {
        const int c = base + lane;
        const int ptr = candidate(c);
        unsigned long long key = kEmptyKey;
        if (c < total && ptr != row) {
          const float4 q = __ldg(&p.stored[ptr]);
          const float dx = q.x - s.x, dy = q.y - s.y, dz = q.z - s.z;
          const float d = dx * dx + dy * dy + dz * dz;
          key = (static_cast<unsigned long long>(__float_as_uint(d)) << 32) | unsigned(ptr);
        }
        const unsigned long long sorted = bitonic_sort32(key, lane);
        best = bitonic_merge32(umin64(best, __shfl_sync(kFull, sorted, 31 - lane)), lane);
      }
      // lane j: the bisector with the j-th nearest candidate (as cell_row
      // builds it); those past 2 r are left out, as in the cage test
      Plane pl{0.0, 0.0, 0.0, 0.0};
      const bool valid = best != kEmptyKey && __uint_as_float(unsigned(best >> 32)) <= max_d2;
      if (valid) {
        const float4 b = __ldg(&p.stored[unsigned(best & 0xffffffffull)]);
        const double bx = double(b.x) - double(s.x), by = double(b.y) - double(s.y), bz = double(b.z) - double(s.z);
        const double nd2 = bx * bx + by * by + bz * bz;
        const double len = sqrt(nd2), inv = 1.0 / len;
        const double off = b.w <= kNoCellLimits ? len : (nd2 + (double(b.w) - double(s.w))) * (0.5 * inv);
        pl = Plane{-bx * inv, -by * inv, -bz * inv, off};
      }
      const int nb = __popc(__ballot_sync(kFull, valid));
      init_box(w, s, p.cube_eps, lane);
      int status = kSuccess;
      for (int j = 0; j < nb && w.np < p.P; ++j) {
        const int r = clip<VS>(w, shfl_plane(pl, j), p.V, status, lane, nullptr, nullptr, 0);
        if (r < 0) break;
        if (r > 0 && cell_radius2<VS>(w, lane) <= plain2) {
          proven = true;
          break;
        }
      }
    }
  }
  if (lane == 0) {
    p.status[row] = proven ? kSuccess : kProbeMiss;
    if (proven) p.out[row] = make_double4(0.0, 0.0, 0.0, 0.0);
  }
}

template <int VS>
__global__ void __launch_bounds__(128, 6) k_probe(const __grid_constant__ ProbeLaunch p,
                                                  const __grid_constant__ Layout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= p.n) return;
  probe_row<VS>(p, L, smem + size_t(threadIdx.x >> 5) * L.total, row, L.Vc, lane);
}

// The outside probe over the rows of many diagrams (batched solves):
// diagram d owns rows start[d] .. start[d+1] (all its seeds) and its own
// record probes[d]; one warp per row.  The layout holds every diagram's
// caps; each works with its own vertex capacity.
template <int VS>
__global__ void __launch_bounds__(128, 6) k_probe_batch(const ProbeLaunch *__restrict__ probes,
                                                        const int *__restrict__ start, int ndiag,
                                                        const __grid_constant__ Layout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (r >= start[ndiag]) return;
  const int d = owner_of_row(start, ndiag, r);
  const ProbeLaunch &p = probes[d];
  probe_row<VS>(p, L, smem + size_t(threadIdx.x >> 5) * L.total, r - start[d], min(L.Vc, (p.V + 31) & ~31), lane);
}

// Rows of many diagrams in one persistent launch (batched solves): diagram
// d owns rows start[d] .. start[d+1] and its own launch record descs[d];
// warps stride over the rows.  park_counter (optional): the re-run of the
// cells that found the defer queue full, which exits unless the queue
// overflowed.
// work (optional, zeroed before the launch): warps take their rows one at a
// time from this counter (persistent launches of unknown row counts, so a
// warp that drew heavy rows does not hold the launch back); null: warp w
// takes rows w, w + warps, ... (a grid of one warp per row takes one each).
template <int VS, bool GRID, bool INL, int SAFE = 0>
__global__ void __launch_bounds__(128, 5)
    k_cell_batch(const CellLaunch *__restrict__ descs, const int *__restrict__ start, int ndiag,
                 const __grid_constant__ Layout L, int only_status, const int *__restrict__ park_counter,
                 int park_capacity, int *__restrict__ work) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (park_counter && *park_counter <= park_capacity) return;
  const int lane = threadIdx.x & 31;
  unsigned char *wsmem = smem + size_t(threadIdx.x >> 5) * L.total;
  const int total = start[ndiag];
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (work) {
    r = lane == 0 ? atomicAdd(work, 1) : 0;
    r = __shfl_sync(kFull, r, 0);
  }
  while (r < total) {
    const int d = owner_of_row(start, ndiag, r);
    const CellLaunch &a = descs[d];
    cell_row<VS, GRID, INL, 0, SAFE>(a, L, wsmem, r - start[d], only_status, vertex_capacity(a, L), lane);
    __syncwarp();  // the warp's shared memory is reused by its next row
    if (work) {
      r = lane == 0 ? atomicAdd(work, 1) : 0;
      r = __shfl_sync(kFull, r, 0);
    } else {
      r += nwarps;
    }
  }
}

// Triangles of the parked boundary cells, CH at a time: every warp takes
// work items (cell, chunk) from a counter, loads the cell into its shared
// memory and runs the chunk's cones.  Partial moments and the first failure
// go to per-item slots; k_cone_finish reduces them in order.
// Launch-record accessors: desc(d) is the record of diagram d.
struct SingleDesc {
  static constexpr bool kBatch = false;
  const CellLaunch *a;  // the one record of a single launch
  __device__ __forceinline__ const CellLaunch &operator()(int) const { return *a; }
};
struct BatchDesc {
  static constexpr bool kBatch = true;
  const CellLaunch *descs;
  __device__ __forceinline__ const CellLaunch &operator()(int d) const { return descs[d]; }
};

// MODE: kConeAll every work item; kConeInner the items of cells with an
// apex inside (facet pieces), kConeCorner those with the reference's start
// corner (cone clipping), each from its own counter.  Two launches, one per
// kind, keep each kernel's code small: a warp running one kind beside warps
// running the other stalls on instruction fetch.
constexpr int kConeAll = 0, kConeInner = 1, kConeCorner = 2;

template <int VS, class Desc, int MODE = kConeAll>
__device__ __forceinline__ void cone_items(const DeferQueue &dq, const Layout &L, Desc desc, unsigned char *wsmem,
                                           int lane) {
  WarpCell w = bind(wsmem, L);
  const int items = min(*(volatile int *)&dq.counters[2], dq.capacity * dq.max_chunks);
  int *next = &dq.counters[MODE == kConeCorner ? 4 : 1];
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(next, 1);
    item = __shfl_sync(kFull, item, 0);
    if (item >= items) break;
    const int slot = dq.chunk_slot[item];
    const unsigned char *base = dq.slots + size_t(slot) * dq.slot_bytes;
    const DeferHeader *h = reinterpret_cast<const DeferHeader *>(base);
    const int nuniq = h->nuniq, chunk = item - h->chunk_base;
    const int t0 = chunk * dq.chunk;
    if (t0 >= nuniq) continue;
    if (MODE == kConeInner && h->inner == 0) continue;
    if (MODE == kConeCorner && h->inner != 0) continue;
    const int t1 = min(t0 + dq.chunk, nuniq);
    const int nv = h->nv, np = h->np, sid = h->sid;
    const Plane *pl = reinterpret_cast<const Plane *>(base + sizeof(DeferHeader));
    const double *vx = reinterpret_cast<const double *>(pl + L.Pc);
    const double *vy = vx + L.Vc, *vz = vy + L.Vc, *vw = vz + L.Vc, *vd = vw + L.Vc;
    const unsigned *vt = reinterpret_cast<const unsigned *>(vd + L.Vc);
    const int *tl = reinterpret_cast<const int *>(vt + L.Vc);
    const bool inner = MODE == kConeAll ? h->inner != 0 : MODE == kConeInner;
    const CellLaunch &a = desc(h->diag);
    if constexpr (Desc::kBatch) w.vc = vertex_capacity(a, L);
    for (int i = lane; i < np; i += 32) w.plane[i] = pl[i];
    for (int v = lane; v < nv; v += 32) {
      w.cx[v] = vx[v];
      w.cy[v] = vy[v];
      w.cz[v] = vz[v];
      w.cw[v] = vw[v];
      w.d2[v] = vd[v];
      w.tri[v] = vt[v];
      if (!inner) {
        w.bcx[v] = vx[v];
        w.bcy[v] = vy[v];
        w.bcz[v] = vz[v];
        w.bcw[v] = vw[v];
        w.bd2[v] = vd[v];
        w.btri[v] = vt[v];
      }
    }
    if (lane < 3) w.pts[lane] = h->pt0[lane];
    __syncwarp();
    w.nv = nv;
    w.np = np;
    const float4 s = a.stored[sid];
    double acc[4] = {0, 0, 0, 0};
    int fail_at = 0;
    int st;
    if (inner) {
      const double ap[3] = {h->pt0[0], h->pt0[1], h->pt0[2]};
      build_faces(w, w.bcx, w.bcy, w.bcz, ap, lane);
      for (int b0 = t0; b0 < t1; b0 += 32)
        facet_triangles(w, w.bcx, w.bcy, w.bcz, a.grid, s, tl, b0, min(t1, b0 + 32), ap, acc, lane, a.counters);
      st = kSuccess;
    } else {
      st = cone_triangles<VS>(w, a, s, tl, t0, t1, nv, np, false, acc, fail_at, lane, a.counters, nullptr, 0);
    }
    if (lane == 0) {
      double *part = dq.part + size_t(item) * 4;
      for (int d = 0; d < 4; ++d) part[d] = acc[d];
      dq.fail[item] = st == kSuccess ? 0x7fffffff : ((fail_at << 4) | st);
    }
    __syncwarp();
  }
}

template <int VS, int MODE>
__global__ void __launch_bounds__(128, 4) k_cone(const __grid_constant__ CellLaunch a, const __grid_constant__ Layout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  cone_items<VS, SingleDesc, MODE>(a.defer, L, SingleDesc{&a}, smem + size_t(threadIdx.x >> 5) * L.total,
                                   threadIdx.x & 31);
}

template <int VS, int MODE>
__global__ void __launch_bounds__(128, 4)
    k_cone_batch(const CellLaunch *__restrict__ descs, const __grid_constant__ DeferQueue dq,
                 const __grid_constant__ Layout L) {
  extern __shared__ __align__(16) unsigned char smem[];
  cone_items<VS, BatchDesc, MODE>(dq, L, BatchDesc{descs}, smem + size_t(threadIdx.x >> 5) * L.total,
                                  threadIdx.x & 31);
}

// Per parked cell: its in-domain part plus the chunk partials in order; the
// first failing chunk decides the status (the reference stops at the first
// failing triangle, ConvexCell.cl:1104-1107).
template <class Desc>
__device__ __forceinline__ void finish_slot(const DeferQueue &dq, const Layout &L, Desc desc, int slot) {
  const DeferHeader *h = reinterpret_cast<const DeferHeader *>(dq.slots + size_t(slot) * dq.slot_bytes);
  const CellLaunch &a = desc(h->diag);
  const int sid = h->sid, nch = (h->nuniq + dq.chunk - 1) / dq.chunk;
  double acc[4] = {h->acc[0], h->acc[1], h->acc[2], h->acc[3]};
  int status = h->fixed >= 0 ? h->fixed : kSuccess;
  for (int c = 0; c < nch; ++c) {
    const int item = h->chunk_base + c;
    const int f = dq.fail[item];
    if (f != 0x7fffffff) {
      status = f & 15;
      break;
    }
    const double *part = dq.part + size_t(item) * 4;
    for (int d = 0; d < 4; ++d) acc[d] += part[d];
  }
  const float4 s = a.stored[sid];
  a.status[sid] = status;
  const double m = acc[3];
  a.out[sid] = status == kSuccess
                   ? make_double4(acc[0] + m * double(s.x), acc[1] + m * double(s.y), acc[2] + m * double(s.z), m)
                   : make_double4(0.0, 0.0, 0.0, 0.0);
  if (a.used && status == kSuccess && m >= a.keep_volume) {
    // a used cell (ConvexCell.cl:1118-1126), marked from the parked copy
    *(volatile unsigned char *)&a.used[sid] = 1;
    if (a.mark_dist >= 1) {
      const unsigned char *base = dq.slots + size_t(slot) * dq.slot_bytes;
      const double *vx = reinterpret_cast<const double *>(base + sizeof(DeferHeader) + 32u * L.Pc);
      const unsigned *vt = reinterpret_cast<const unsigned *>(vx + 5 * size_t(L.Vc));
      const int *tl = reinterpret_cast<const int *>(vt + L.Vc);
      const int *nb = tl + ((L.T + 3) & ~3);
      mark_neighbours(a.used, vt, h->nv, nb, 1, 0, 1);
    }
  }
}

__global__ void k_cone_finish(const __grid_constant__ CellLaunch a, const __grid_constant__ Layout L) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= min(a.defer.counters[0], a.defer.capacity)) return;
  finish_slot(a.defer, L, SingleDesc{&a}, slot);
}

__global__ void k_cone_finish_batch(const CellLaunch *__restrict__ descs, const __grid_constant__ DeferQueue dq,
                                    const __grid_constant__ Layout L) {
  const int parked = min(dq.counters[0], dq.capacity);
  for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < parked; slot += gridDim.x * blockDim.x)
    finish_slot(dq, L, BatchDesc{descs}, slot);
}

// Raises a kernel's dynamic shared memory limit to the device's opt-in
// maximum, once per kernel and device.  The limit is process-wide: set per
// launch to the launch's own size, a launch on another thread could lower it
// between this thread's setting and its launch (the serving loop runs
// launches from several threads).
cudaError_t allow_smem(const void *fn, size_t smem) {
  static std::mutex mu;
  static std::set<std::pair<const void *, int>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int optin = 0;
  if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
  cudaFuncAttributes fa;
  if ((e = cudaFuncGetAttributes(&fa, fn)) != cudaSuccess) return e;
  // the dynamic limit leaves room for the kernel's static shared memory
  const int room = optin - int(fa.sharedSizeBytes);
  if (smem > size_t(room)) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({fn, dev})) return cudaSuccess;
  if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, room)) != cudaSuccess) return e;
  done.insert({fn, dev});
  return cudaSuccess;
}

// Warps per block for a per-warp layout: 4 where they fit the shared memory
// of one block, else fewer (large caps); 0 when one warp does not fit.
int warps_per_block_for(const Layout &L) {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  // a little room for the kernels' static shared memory
  const size_t room = size_t(optin) - 256;
  int w = 4;
  while (w > 0 && size_t(L.total) * w > room) w >>= 1;
  return w;
}

template <int VS, int PREC = 0, int SAFE = 0>
cudaError_t launch_vs(const CellLaunch &a, const Layout &L, cudaStream_t st, int sm_count, int *launches) {
  const int warps_per_block = warps_per_block_for(L);
  if (warps_per_block == 0) return cudaErrorInvalidValue;
  const size_t smem = size_t(L.total) * warps_per_block;
  const int blocks = (a.num + warps_per_block - 1) / warps_per_block;
  cudaError_t e;
  if (a.grid.size > 0 && a.defer.slots) {
    // every boundary cell parks; the chunked kernel does the triangles
    e = allow_smem(reinterpret_cast<const void *>(k_cell<VS, true, false, PREC, SAFE>), smem);
    if (e != cudaSuccess) return e;
    k_cell<VS, true, false, PREC, SAFE><<<blocks, warps_per_block * 32, smem, st>>>(a, L);
    if (a.after_cell) cudaEventRecord(a.after_cell, st);
    if ((e = allow_smem(reinterpret_cast<const void *>(k_cone<VS, kConeInner>), smem)) != cudaSuccess ||
        (e = allow_smem(reinterpret_cast<const void *>(k_cone<VS, kConeCorner>), smem)) != cudaSuccess)
      return e;
    k_cone<VS, kConeInner><<<sm_count * 4, warps_per_block * 32, smem, st>>>(a, L);
    k_cone<VS, kConeCorner><<<sm_count * 4, warps_per_block * 32, smem, st>>>(a, L);
    k_cone_finish<<<(a.defer.capacity + 127) / 128, 128, 0, st>>>(a, L);
    if (launches) *launches += 4;
  } else if (a.grid.size > 0) {
    e = allow_smem(reinterpret_cast<const void *>(k_cell<VS, true, true, PREC, SAFE>), smem);
    if (e != cudaSuccess) return e;
    k_cell<VS, true, true, PREC, SAFE><<<blocks, warps_per_block * 32, smem, st>>>(a, L);
    if (a.after_cell) cudaEventRecord(a.after_cell, st);
    if (launches) ++*launches;
  } else {
    e = allow_smem(reinterpret_cast<const void *>(k_cell<VS, false, true, PREC, SAFE>), smem);
    if (e != cudaSuccess) return e;
    k_cell<VS, false, true, PREC, SAFE><<<blocks, warps_per_block * 32, smem, st>>>(a, L);
    if (a.after_cell) cudaEventRecord(a.after_cell, st);
    if (launches) ++*launches;
  }
  return cudaGetLastError();
}

// Blocks of a persistent launch: as many as stay resident on every SM.
template <class Kernel>
int resident_blocks(Kernel k, int threads, size_t smem, int sm_count) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return per_sm * sm_count;
}

// rows >= 0: the launch's row count is known: one warp per row.  Else a
// persistent launch; with `work`, rows are taken from that counter (zeroed
// here, on the stream).
template <int VS, bool GRID, bool INL, int SAFE = 0>
cudaError_t batch_cells(const CellLaunch *descs, const int *start, int ndiag, const Layout &L, int only_status,
                        const int *park_counter, int park_capacity, long rows, int *work, cudaStream_t st,
                        int sm_count) {
  const int wpb = warps_per_block_for(L);
  if (wpb == 0) return cudaErrorInvalidValue;
  const size_t smem = size_t(L.total) * wpb;
  auto k = k_cell_batch<VS, GRID, INL, SAFE>;
  cudaError_t e = allow_smem(reinterpret_cast<const void *>(k), smem);
  if (e != cudaSuccess) return e;
  int blocks;
  if (rows >= 0) {
    blocks = int(std::max<long>(1, (rows + wpb - 1) / wpb));
    work = nullptr;
  } else {
    blocks = resident_blocks(k, wpb * 32, smem, sm_count);
    if (work && (e = cudaMemsetAsync(work, 0, sizeof(int), st)) != cudaSuccess) return e;
  }
  k<<<blocks, wpb * 32, smem, st>>>(descs, start, ndiag, L, only_status, park_counter, park_capacity, work);
  return cudaGetLastError();
}

cudaError_t record_after_cell(const CellBatch &b, cudaStream_t st) {
  // an event node when the stream is being captured
  return b.after_cell ? cudaEventRecordWithFlags(b.after_cell, st, cudaEventRecordExternal) : cudaSuccess;
}

template <int VS, int SAFE = 0>
cudaError_t launch_batch_vs(const CellBatch &b, const Layout &Lg, const Layout &Lp, cudaStream_t st, int sm_count,
                            int *launches) {
  cudaError_t e;
  if (b.start_plain) {
    if ((e = batch_cells<VS, false, true, SAFE>(b.descs_inline, b.start_plain, b.ndiag, Lp, -1, nullptr, 0, b.rows_plain,
                                          b.work, st, sm_count)) != cudaSuccess)
      return e;
    if (launches) ++*launches;
  }
  if (!b.start_grid) return record_after_cell(b, st);
  if (!b.defer.slots) {
    if ((e = batch_cells<VS, true, true, SAFE>(b.descs_inline, b.start_grid, b.ndiag, Lg, -1, nullptr, 0, b.rows_grid,
                                         b.work, st, sm_count)) != cudaSuccess)
      return e;
    if (launches) ++*launches;
    return record_after_cell(b, st);
  }
  // every boundary cell parks; the chunked kernel does the triangles, then
  // the cells that found the queue full run again inline
  if ((e = batch_cells<VS, true, false, SAFE>(b.descs, b.start_grid, b.ndiag, Lg, -1, nullptr, 0, b.rows_grid, b.work, st,
                                        sm_count)) != cudaSuccess)
    return e;
  if ((e = record_after_cell(b, st)) != cudaSuccess) return e;
  const int wpb = warps_per_block_for(Lg);
  const size_t smem = size_t(Lg.total) * wpb;
  auto ki = k_cone_batch<VS, kConeInner>;
  auto kr = k_cone_batch<VS, kConeCorner>;
  if ((e = allow_smem(reinterpret_cast<const void *>(ki), smem)) != cudaSuccess ||
      (e = allow_smem(reinterpret_cast<const void *>(kr), smem)) != cudaSuccess)
    return e;
  ki<<<resident_blocks(ki, wpb * 32, smem, sm_count), wpb * 32, smem, st>>>(b.descs, b.defer, Lg);
  kr<<<resident_blocks(kr, wpb * 32, smem, sm_count), wpb * 32, smem, st>>>(b.descs, b.defer, Lg);
  k_cone_finish_batch<<<sm_count * 4, 128, 0, st>>>(b.descs, b.defer, Lg);
  if ((e = batch_cells<VS, true, true, SAFE>(b.descs_inline, b.start_grid, b.ndiag, Lg, kParkOverflow, b.defer.counters,
                                       b.defer.capacity, -1, b.work, st, sm_count)) != cudaSuccess)
    return e;
  if (launches) *launches += 5;
  return cudaGetLastError();
}

}  // namespace

}  // namespace rpd
