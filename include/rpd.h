/* rpd.h -- C ABI of the B200 restricted power diagram engine (librpd.so).
 *
 * Drop-in boundary for the reference's hot path: the KNearests / Grid /
 * VoroAlgo entry points of basselin7u/GPU-Restricted-Power-Diagrams
 * (knearests.h:9-50, Grid.h:14-70, voronoi.h:105-256).  Plain pointers and
 * sizes only; coordinates are in the reference frame [0,1000]^3 and weights
 * in that frame's squared units (a [0,1]^3 input scales x1000, weights x1e6).
 *
 * Every function returns an rpd_error (0 = RPD_OK) unless stated otherwise.
 * The text of the last failure of a context is rpd_context_error().  Nothing
 * here aborts the process; the reference's exit() paths (knearests.cpp:72-75)
 * become error codes.
 */
#ifndef RPD_H
#define RPD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rpd_error {
  RPD_OK = 0,
  RPD_ERR_INVALID = -1,     /* bad argument or call order */
  RPD_ERR_CUDA = -2,        /* a CUDA call failed (text in rpd_context_error) */
  RPD_ERR_NO_DEVICE = -3,   /* no usable sm_100 device */
  RPD_ERR_OOM = -4,         /* device memory exhausted */
  RPD_ERR_IO = -5,          /* file could not be read or written */
  RPD_ERR_FORMAT = -6,      /* malformed grid or seed file */
  RPD_ERR_DEGENERATE = -7,  /* seeds too clustered for the bin grid */
  RPD_ERR_CAPACITY = -8     /* a cap (K, P, V, T) beyond what this build supports */
} rpd_error;

/* Per-cell status, the values of the reference's Status enum (Status.h:4-16). */
typedef enum rpd_cell_status {
  RPD_VERTEX_OVERFLOW = 0,
  RPD_PLANE_OVERFLOW = 1,
  RPD_INCONSISTENT_BOUNDARY = 2,
  RPD_SECURITY_RADIUS_NOT_REACHED = 3,
  RPD_SUCCESS = 4,
  RPD_NEEDS_EXACT_PREDICATES = 5,
  RPD_EMPTY_CELL = 6,
  RPD_FIND_ANOTHER_BEGINNING_VERTEX = 7,
  RPD_TRIANGLE_OVERFLOW = 8,
  RPD_SEED_ON_BORDER = 9,
  RPD_HESSIAN_OVERFLOW = 10
} rpd_cell_status;
#define RPD_STATUS_NUM 11

/* A seed with w <= RPD_NO_CELL_LIMITS has no cell and acts as a wall
 * through its own position for its neighbours (voronoi.h:53). */
#define RPD_NO_CELL_LIMITS (-100000.0f)

typedef enum rpd_mem { RPD_HOST = 0, RPD_DEVICE = 1 } rpd_mem;

typedef struct rpd_context rpd_context;
typedef struct rpd_solver rpd_solver;

/* ---------------------------------------------------------------- context */

/* Binds CUDA device `device` and creates the engine's stream.  Replaces
 * OpenCLContext::createContext (openCL.h:59-169). */
rpd_context *rpd_context_create(int device, int *err);
void rpd_context_destroy(rpd_context *ctx);
const char *rpd_context_error(const rpd_context *ctx);
/* The engine's cudaStream_t (as void *); all device work of a context is
 * ordered on it. */
void *rpd_context_stream(rpd_context *ctx);
/* Library version string. */
const char *rpd_version(void);

/* ------------------------------------------------------ seeds + neighbours */

rpd_solver *rpd_solver_create(rpd_context *ctx, int *err);
void rpd_solver_destroy(rpd_solver *s);

/* VoroAlgo::setInputPoints (voronoi.cpp:1088-1107) and the KNearests
 * constructor (knearests.cpp:48-222): copies n seeds (4 floats x y z w each,
 * from host or device memory) and bins them on the device.  The caller may
 * free `xyzw` when this returns. */
int rpd_solver_set_points(rpd_solver *s, const float *xyzw, int n, rpd_mem where);
/* KNearests::getNumPoints. */
int rpd_solver_num_points(const rpd_solver *s);
/* Bins per axis of the seed grid (KNearests::dim). */
int rpd_solver_bin_dim(const rpd_solver *s);
/* KNearests::getPermutation: perm[stored index] = user index, n ints. */
int rpd_solver_get_permutation(rpd_solver *s, int *perm, rpd_mem where);
/* KNearests::buildKnearests for every seed (knearests.cpp:238-315): the K
 * nearest other seeds, ascending distance, ties by stored index, written as
 * USER indices (-1 where fewer than K exist), n*K ints in user order. */
int rpd_solver_knn(rpd_solver *s, int K, int *knn_user, rpd_mem where, float *device_ms);

#ifdef __cplusplus
}
#endif
#endif /* RPD_H */
