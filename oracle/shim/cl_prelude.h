// Test infrastructure only: never linked into the product library.
//
// OpenCL-C -> C++ shim used to compile the reference's own kernels
// (ConvexCell.cl, knearests.cl) for the host CPU, so that the reference
// algorithm itself can be run here as a checker and as the timed CPU
// baseline.  One work-item = one call on one host thread; work-group size 1,
// so every `__local` array is a private per-call buffer.
//
// Compile-time knobs that the reference bakes into its OpenCL program
// (voronoi.cpp:915-947, knearests.cpp:269-275) become thread-local runtime
// values here, so one build covers every K/P/V/T and grid size:
//   * K, P, GRID_SIZE, GRID_VOXEL_SIZE, CUBE_EPSILON ... plain runtime ints.
//   * V is an array bound in ConvexCellBackUp (ConvexCell.cl:696) and a
//     runtime bound in CCNewVertex (ConvexCell.cl:337): a tag object whose
//     constexpr conversion gives the array bound (255, the uchar maximum)
//     and whose operator>= compares against the runtime value.
//   * T is tested by `#if T>0` (ConvexCell.cl:721,945,980,1081) and used as a
//     VLA bound: the macro below reads as 1 in #if (identifiers are 0 there)
//     and as the runtime value in code.  T=0 then reproduces the first-pass
//     behaviour (triangle_overflow at the first voxel with triangles).
#pragma once
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <vector>
#include <omp.h>
#include "ref_abi.h"

using std::sqrt;
using std::fabs;
using std::fmax;
using std::floor;

#ifndef REF_REAL
#error "REF_REAL must be float or double"
#endif

typedef unsigned char uchar;

struct ref_real4 {
  REF_REAL x, y, z, w;
};
struct ref_uchar4 {
  uchar x, y, z, w;
};
typedef ref_uchar4 ref_uchar3;  // OpenCL uchar3 occupies 4 bytes

static inline ref_real4 real4_make(REF_REAL x, REF_REAL y, REF_REAL z, REF_REAL w) {
  ref_real4 r;
  r.x = x; r.y = y; r.z = z; r.w = w;
  return r;
}
static inline ref_uchar3 uchar3_make(int x, int y, int z) {
  ref_uchar3 r;
  r.x = (uchar)x; r.y = (uchar)y; r.z = (uchar)z; r.w = 0;
  return r;
}
static inline ref_real4 operator+(ref_real4 a, ref_real4 b) { return real4_make(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
static inline ref_real4 operator-(ref_real4 a, ref_real4 b) { return real4_make(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
static inline ref_real4 operator*(REF_REAL s, ref_real4 a) { return real4_make(s * a.x, s * a.y, s * a.z, s * a.w); }
static inline ref_real4 operator*(ref_real4 a, REF_REAL s) { return real4_make(a.x * s, a.y * s, a.z * s, a.w * s); }
// OpenCL dot() on a 4-vector uses all four lanes.
static inline REF_REAL dot(ref_real4 a, ref_real4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
// OpenCL cross() on a 4-vector ignores w and returns w=0.
static inline ref_real4 cross(ref_real4 a, ref_real4 b) {
  return real4_make(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, 0);
}
static inline int max(int a, int b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }
static inline float max(float a, float b) { return std::fmax(a, b); }
static inline double max(double a, double b) { return std::fmax(a, b); }

// OpenCL work-item builtins: one work-item per call, group size 1.
static thread_local int ref_global_id;
static inline int get_global_id(int) { return ref_global_id; }
static inline int get_local_id(int) { return 0; }
static inline int get_local_size(int) { return 1; }

static inline int atomic_add(volatile int *p, int v) { return __atomic_fetch_add((int *)p, v, __ATOMIC_RELAXED); }
static inline int atomic_max(volatile int *p, int v) {
  int old = __atomic_load_n((int *)p, __ATOMIC_RELAXED);
  while (old < v && !__atomic_compare_exchange_n((int *)p, &old, v, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
  }
  return old;
}

// Runtime values of the reference's compile-time knobs (set per call).
// Internal linkage: every build variant is its own translation unit.
static thread_local int ref_K, ref_P, ref_T, ref_V;
static thread_local int ref_grid_size;
static thread_local REF_REAL ref_grid_voxel_size;
static thread_local REF_REAL ref_cube_epsilon;
static thread_local REF_REAL ref_used_eps;
static thread_local int ref_H;  // CHESSIAN builds: the Hessian row length
static const int ref_one = 1;

struct RefVTag {
  constexpr operator int() const { return 255; }
};
static inline bool operator>=(int a, RefVTag) { return a >= ref_V; }
static constexpr RefVTag ref_V_tag{};

#define __kernel
#define __global
#define __local
#define __constant
#define real REF_REAL
#define real4 ref_real4
#define uchar3 ref_uchar3
#define uchar4 ref_uchar4
#define make_uchar3(x, y, z) uchar3_make(x, y, z)
#define K ref_K
#define P ref_P
#define V ref_V_tag
#define T (ref_T + 1 - ref_one)
#define P1 0
#define GRID_SIZE ref_grid_size
#define GRID_VOXEL_SIZE ref_grid_voxel_size
#define CUBE_EPSILON ref_cube_epsilon
#define USED_CELL_EPSILON ref_used_eps
#define H ref_H
#define NO_CELL_LIMITS -100000
#if REF_IS_DOUBLE
#define VOLUME_EPSILON2 1.e-12
#else
#define VOLUME_EPSILON2 1.e-6
#endif
// The reference prints a '.' per triangle-list overflow (ConvexCell.cl:735)
// and a warning on unexpected states; silence them on the host.
#define printf(...) ((void)0)

// knearests.cl expects cellFromPoint from the host-side source string
// (knearests.cpp:35-46): bin = clamp(floor(p * dim / 1000)).
static inline int cellFromPoint(int dim, ref_real4 p) {
  int i = (int)std::floor(p.x * (REF_REAL)dim / 1000.f);
  int j = (int)std::floor(p.y * (REF_REAL)dim / 1000.f);
  int k = (int)std::floor(p.z * (REF_REAL)dim / 1000.f);
  i = max((int)0, min(i, dim - 1));
  j = max((int)0, min(j, dim - 1));
  k = max((int)0, min(k, dim - 1));
  return i + j * dim + k * dim * dim;
}
