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
  RPD_ERR_CAPACITY = -8     /* a cap (K, P, V, T) beyond what the library supports */
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
/* The neighbour-search variant the context uses for K (0: a warp per seed,
 * 1: a thread per seed, K <= 128): variant 0 or 1 pins it, -1 forgets it
 * (the next search with K times both again), -2 only reads it.  Returns the
 * variant for K afterwards, -1 when not chosen yet, or an rpd_error.  No
 * counterpart in the reference (one kernel, knearests.cl:36-78). */
int rpd_context_knn_variant(rpd_context *ctx, int K, int variant);

/* ------------------------------------------------------ seeds + neighbours */

rpd_solver *rpd_solver_create(rpd_context *ctx, int *err);
void rpd_solver_destroy(rpd_solver *s);

/* VoroAlgo::setInputPoints (voronoi.cpp:1088-1107) and the KNearests
 * constructor (knearests.cpp:48-222): copies n seeds (4 floats x y z w each,
 * from host or device memory) and bins them on the device.  The caller may
 * free `xyzw` when this returns.  A NaN or infinite coordinate or weight is
 * RPD_ERR_INVALID (the solver then holds no seeds). */
int rpd_solver_set_points(rpd_solver *s, const float *xyzw, int n, rpd_mem where);
/* KNearests::getNumPoints. */
int rpd_solver_num_points(const rpd_solver *s);
/* Bins per axis of the seed grid (KNearests::dim). */
int rpd_solver_bin_dim(const rpd_solver *s);
/* KNearests::getPermutation: perm[stored index] = user index, n ints. */
int rpd_solver_get_permutation(rpd_solver *s, int *perm, rpd_mem where);
/* New weights (n floats, user order) for the seeds already set, without
   re-binning: a weight-only re-solve (Lloyd / optimal-transport iterations).
   The neighbour table of the last launch with the same K is reused, since
   the reference's neighbours ignore weights (knearests.cl:36-78).  No
   counterpart in the reference, which re-uploads all seeds
   (voronoi.cpp:1088-1107).  A NaN or infinite weight is RPD_ERR_INVALID,
   with the seeds left unchanged. */
int rpd_solver_set_weights(rpd_solver *s, const float *w, rpd_mem where);
/* KNearests::buildKnearests for every seed (knearests.cpp:238-315): the K
 * nearest other seeds, ascending distance, ties by stored index, written as
 * USER indices (-1 where fewer than K exist), n*K ints in user order. */
int rpd_solver_knn(rpd_solver *s, int K, int *knn_user, rpd_mem where, float *device_ms);

/* -------------------------------------------------------------- seed files */

/* Utils::loadSeedsFile (Utils.cpp:36-79): a count line, then "x y z" per
 * line ("x y z w" with four_d, --points4D; w = 0 otherwise), not normalised
 * (test_voronoi.cpp:88).  With binary (--loadBinaryPoints,
 * readBinarySeedsFile, Utils.cpp:81-97): a 64-bit count N, then 4N floats.
 * On success *xyzw (4 * *n floats, malloc'ed; free with rpd_seeds_free) and
 * *n are set.  RPD_ERR_IO when the file cannot be opened, RPD_ERR_FORMAT
 * when a line does not parse, the count does not match or a value is NaN or
 * infinite. */
int rpd_seeds_load(const char *path, int four_d, int binary, float **xyzw, int *n);
void rpd_seeds_free(float *xyzw);
/* saveBinarySeedsFile (Utils.cpp:99-113, --saveBinaryPoints). */
int rpd_seeds_save_binary(const char *path, const float *xyzw, int n);

/* ------------------------------------------------------------------ domain */

/* A volume domain in the reference --grid layout (Grid.h:14-70): size^3
 * voxel-corner flags (0 outside, 1 on the border, 2 inside), a closed
 * triangle surface, and per voxel the sorted ids of its triangles.  Host
 * container; solvers copy it to the device in rpd_solver_set_grid. */
typedef struct rpd_grid rpd_grid;

/* From arrays (copied).  points: 3 floats per vertex; offsets: size^3+1.
 * The orientation is flipped when the volume is negative, as Grid::load
 * does (Grid.cpp:270-275). */
rpd_grid *rpd_grid_create(int size, const char *in_domain, const float *points_xyz, int npoints,
                          const int *triangles, int ntriangles, const int *tri_list, int nlist,
                          const int *offsets, int *err);
/* Grid::load / Grid::save: the reference text format (Grid.cpp:186-344). */
rpd_grid *rpd_grid_load(const char *path, int *err);
int rpd_grid_save(const rpd_grid *g, const char *path);
/* Grid::valid (Grid.cpp:60-184): 1 valid, 0 invalid (reason copied to why). */
int rpd_grid_valid(const rpd_grid *g, char *why, int why_len);
/* Grid::getVolume (Grid.cpp:30-35). */
double rpd_grid_volume(const rpd_grid *g);
/* Volume and first moments of the domain (Grid::printInvariants,
 * Grid.cpp:281-288): out = (m*x, m*y, m*z, m). */
int rpd_grid_invariants(const rpd_grid *g, double *out4);
int rpd_grid_info(const rpd_grid *g, int *size, int *npoints, int *ntriangles, int *nlist);
/* Copies the arrays out (sizes from rpd_grid_info; points 3 floats each). */
int rpd_grid_export(const rpd_grid *g, char *in_domain, float *points_xyz, int *triangles, int *tri_list,
                    int *offsets);
void rpd_grid_destroy(rpd_grid *g);
/* Synthetic domains.  Blob: union of `nellipsoids` seeded random ellipsoids
 * (centres U[0.35,0.65]^3, semi-axes U[0.15,0.35] of the unit cube, random
 * rotations) voxelized on size^3, each voxel split into the 6 Kuhn tetrahedra
 * of its main diagonal, surface by marching tetrahedra.  Cube: the box
 * [d, 1000-d]^3 with d half a voxel (no voxel corner on its surface), faces
 * triangulated along the voxel columns. */
rpd_grid *rpd_grid_make_blob(int size, int nellipsoids, uint64_t seed, int *err);
rpd_grid *rpd_grid_make_cube(int size, int *err);
/* Synthetic seeds of the blue-noise configuration (no counterpart in the
 * reference): up to n points of [0,1000]^3 by seeded dart throwing with
 * minimum distance rfac * n^(-1/3) * 1000, weights 0, into xyzw (4n floats).
 * Returns the number of points (n unless the darts saturate). */
int rpd_synth_poisson_disk(int n, uint64_t seed, double rfac, float *xyzw);

/* Domains built on the device (no counterpart in the reference, whose
 * domains come from its host tool utils/createGrid): no host preprocessing
 * and no host copy, e.g. for served requests with new domains.
 *
 * rpd_solver_set_grid_field: the domain {field < 0} of an implicit function
 * sampled on the (size+1)^3 voxel-corner lattice (x fastest, the lattice
 * spans [0,1000]^3; host or device memory; the lattice's outer layer is taken
 * as outside so the surface closes inside the grid).  Corner flags, the
 * surface by marching the 6 Kuhn tetrahedra of every voxel, per-voxel
 * triangle lists and the solver's lookup tables are built on the device.
 * rpd_solver_set_grid_blob: the seeded blob of rpd_grid_make_blob, evaluated
 * and built on the device: the same corner flags and, voxel by voxel, the
 * same triangles (vertex coordinates bit for bit) in the same order, so
 * solves give the same results; only the numbering of the surface vertices
 * differs.  size <= 1024.  rpd_solver_export_grid copies a solver's domain
 * (however it was set) into a new host grid, e.g. to save it in the --grid
 * format. */
int rpd_solver_set_grid_field(rpd_solver *s, int size, const float *field, rpd_mem where);
int rpd_solver_set_grid_blob(rpd_solver *s, int size, int nellipsoids, uint64_t seed);
rpd_grid *rpd_solver_export_grid(rpd_solver *s, int *err);

/* --------------------------------------------------------------- solve */

/* Launch flags. */
#define RPD_FLAG_FIRST_PASS_ONLY 1u /* no retry passes */
#define RPD_FLAG_COUNTERS 2u        /* collect work counters (rpd_stats.counters) */
#define RPD_FLAG_NO_EARLY_OUT 4u    /* clip every cell to the end even when it is
                                       provably outside the domain (same results) */
#define RPD_FLAG_NO_DEFER 8u        /* run every boundary cell's triangles in the
                                       cell's own warp (same results, slower) */
#define RPD_FLAG_REFERENCE_APEX 16u /* cone apex at the reference's start corner for
                                       every cell, with all triangles of its voxels
                                       (same results up to rounding, slower) */
#define RPD_FLAG_FRESH_NEIGHBOURS 32u /* recompute the neighbour table even when the
                                         seeds' positions and K are unchanged since
                                         the last launch (same results) */
#define RPD_FLAG_NO_PROBE 64u       /* no outside probe (the default; overrides
                                       RPD_FLAG_OUTSIDE_PROBE) */
#define RPD_FLAG_NO_T_AHEAD 128u    /* leave every triangle overflow of the first pass
                                       to the retry passes instead of restricting at
                                       once the cells the retries would settle (same
                                       results) */
#define RPD_FLAG_OUTSIDE_PROBE 2048u /* before the first pass, settle the cells that a probe of
                                       their 3x3x3 bins proves outside the domain (mass 0,
                                       status success) without their K-nearest search and
                                       clipping.  Moments equal the reference's; a status can
                                       differ: where the reference's clipping of such a cell
                                       fails in every pass (security radius not reached or a
                                       cap overflow) it reports that failure, this success,
                                       and a failure the reference counts can grow its retry
                                       caps where these do not */
#define RPD_FLAG_SAFE_RADIUS 1024u  /* --safeRadius: stop clipping on the weighted security-radius
                                       guard instead of the reference's Voronoi test d^2 > 4 R^2
                                       (ConvexCell.cl:364-382): with the neighbours sorted by
                                       distance d and the weights added to squared distances, no
                                       later neighbour cuts the cell once d_j > R and
                                       d_j^2 - 2 R d_j > w_s - min w.  A cell the reference's test
                                       stops early on comes out exact (different from the
                                       reference's); equal weights give the reference's test */
#define RPD_FLAG_KNN_WARP 256u      /* neighbour search with a warp per seed (bitonic
                                       merges) for every K (same results) */
#define RPD_FLAG_KNN_THREAD 512u    /* neighbour search with a thread per seed (a
                                       shared-memory heap) for K <= 128 (same results).
                                       Without either flag, searches of at least 16K
                                       rows use the variant each context picks for K by
                                       a timed trial the first time K comes up, smaller
                                       ones a warp per seed (rpd_stats.pass_knn_variant) */

/* VoroAlgo's knobs (voronoi.h:199-246; defaults of Options.cpp:22-28). */
typedef struct rpd_params {
  int K;                /* neighbours of the first pass (--K, 20) */
  int P;                /* planes per cell (--P, 25; < 256) */
  int V;                /* vertices per cell (--V, 30; <= 256) */
  int T;                /* boundary triangles per cell (--T, 100) */
  int max_extra_passes; /* retry passes with caps x1.5 (voronoi.cpp:1321: 5) */
  float cube_eps;       /* box [-eps, 1000+eps]^3; < 0: 0.1 with a domain, else 0 */
  int out_domain;       /* start-corner fallback one voxel layer out in the
                           retry passes: -1 auto (when the grid has border
                           corners, voronoi.cpp:1320), 0 never, 1 always */
  unsigned flags;       /* RPD_FLAG_* */
  int keep_distance;    /* used cells, with a domain only (--keepDist2; voronoi.cpp:1286-1393):
                           -1 off (the default), 0 the cells of mass >= keep_volume,
                           d >= 1 also the cells up to d face rings around them */
  double keep_volume;   /* --keepVolume: the mass that makes a cell used (default 0.001,
                           the FP64 build's, Options.cpp:40) */
  int hessian_h;        /* --hessian with --H: facets per Hessian row, 0 off (the default;
                           Options.cpp:22,269) */
  int hessian_hc;       /* --HC: 1 (facet area) or 4 (area-weighted facet centroid and area) */
  int precision;        /* RPD_PRECISION_*: arithmetic of the clipping loop */
} rpd_params;

/* Arithmetic of the clipping loop (the reference's VHSAlgo / USE_DOUBLE
 * choice, ConvexCell.cl:400-461, voronoi.cpp:917-923).  Restriction to the
 * domain and integration are FP64 in every mode.
 *   FP64:  planes, vertices (cofactors), half-space tests and radius in FP64
 *          (the reference's FP64 predicate, VHSAlgo 2, everywhere).
 *   MIXED: the clipping state in float -- planes, vertex cofactors with error
 *          majorants -- and every half-space test in float; a test whose value
 *          lies within its rigorous error bound of the threshold (and a vertex
 *          or radius test as close) is escalated to FP64, recomputed from the
 *          FP64 planes, so every decision is the FP64 mode's: the same cells,
 *          statuses and moments.  The reference's filtered FP32 predicate
 *          (VHSAlgo 1, ConvexCell.cl:415-448) per test instead of per cell.
 *          Escalations are counted (RPD_CTR_ESCALATED_*).
 *   FP32:  plain float: planes rounded to float and every test in float with
 *          no escalation (the reference's float build, VHSAlgo 0); the cells
 *          are integrated from the float planes.  For comparison. */
#define RPD_PRECISION_FP64 0
#define RPD_PRECISION_MIXED 1
#define RPD_PRECISION_FP32 2

void rpd_params_default(rpd_params *p);

/* Work counters (RPD_FLAG_COUNTERS), summed over passes. */
enum {
  RPD_CTR_PLANES_TESTED = 0,
  RPD_CTR_CLIPS,
  RPD_CTR_VERTEX_TESTS,
  RPD_CTR_VERTICES_MADE,
  RPD_CTR_BOUNDARY_CELLS,
  RPD_CTR_TRIANGLES,
  RPD_CTR_EXPORTS,
  RPD_CTR_EXPORT_VERTICES,
  RPD_CTR_OUTSIDE, /* cells proven outside the domain before the end of clipping */
  RPD_CTR_CONE_EMPTY,   /* boundary triangles whose cone misses the cell */
  RPD_CTR_CONES_SKIPPED, /* boundary triangles dropped because they miss the cell
                            (cone apex at a grid corner inside the cell) */
  RPD_CTR_ESCALATED_TESTS,    /* RPD_PRECISION_MIXED: vertex half-space tests decided
                                 in FP64 (of RPD_CTR_VERTEX_TESTS) */
  RPD_CTR_ESCALATED_VERTICES, /* RPD_PRECISION_MIXED: vertices made in FP64 */
  RPD_CTR_ESCALATED_RADII,    /* RPD_PRECISION_MIXED: security-radius / outside tests
                                 decided on the exact FP64 radius */
  RPD_CTR_START_CORNER,       /* boundary cells whose cones run from the reference's
                                 start corner: no grid corner inside the cell, or caps
                                 too tight to rule out an overflow of the reference's
                                 cone clipping (P < planes + 4 or V < vertices + 8) */
  RPD_CTR_NUM
};

typedef struct rpd_stats {
  int npasses;
  int pass_cells[8];
  int pass_K[8], pass_P[8], pass_V[8], pass_T[8];
  float pass_knn_ms[8];
  float pass_cell_ms[8];
  int status_hist[RPD_STATUS_NUM]; /* final status of every seed */
  unsigned long long counters[RPD_CTR_NUM];
  unsigned long long knn_candidates;
  float total_ms;                  /* device time of the whole launch */
  int kernel_launches;             /* device kernels this launch ran */
  float pass_cell_kernel_ms[8];    /* of pass_cell_ms: the cell kernel alone (no cone kernels) */
  /* Outside probe of the first pass (with a domain, on the first launch
   * after rpd_solver_set_points or with RPD_FLAG_FRESH_NEIGHBOURS; not with
   * counters, Hessian rows or used cells at keep_volume <= 0): the cells it
   * proved empty outside the domain without a full neighbour search, and its
   * device time.  The first pass's neighbour search and cell kernel then
   * cover the other seeds; pass_cells[0] still counts every seed.  A later
   * launch builds the whole neighbour table, which weight-only re-solves
   * keep. */
  int probe_outside;
  float probe_ms;
  int pass_knn_variant[8];         /* neighbour search of each pass: 0 a warp per seed,
                                      1 a thread per seed */
} rpd_stats;

/* VoroAlgo::setGrid (voronoi.cpp:1079-1082): uploads the domain; null
 * removes it (the cell is then restricted to the box only). */
int rpd_solver_set_grid(rpd_solver *s, const rpd_grid *g);

/* VoroAlgo::launch (voronoi.cpp:1244-1403): every seed's power cell clipped
 * to the box and the domain, integrated; failing cells are retried with
 * caps x1.5 as the reference does.  Results stay on the device until the
 * next launch or set_points. */
int rpd_solver_launch(rpd_solver *s, const rpd_params *p);

/* ---------------------------------------------------- one diagram, several GPUs */

/* A diagram split over several solvers, e.g. one per GPU (no counterpart in
 * the reference, which solves one id batch after another on one device,
 * voronoi.cpp:960-973; this cuts the diagram at those batches).  Every part
 * holds all seeds and the domain (rpd_solver_set_points / _set_grid with the
 * same inputs) and solves the cells of its range of stored (binned) seeds,
 * part p of `parts`: rpd_solver_part_range gives first and count.  The retry
 * schedule is the whole diagram's: after every pass the launch calls
 * `reduce` with this part's counts -- sums[0 .. RPD_STATUS_NUM) the failing
 * cells' status histogram, sums[RPD_STATUS_NUM] their number, maxes[0] the
 * largest triangle count settled ahead -- and the callback must replace each
 * with its sum (maximum) over all parts (an all-reduce over the parts'
 * processes, e.g. NCCL; every part calls it the same number of times) and
 * return 0.  Then every part holds its range's results in stored order:
 * gather the ranges (rpd_solver_get_stored, then e.g. an all-gather) and
 * install them on a solver with rpd_solver_set_stored, whose getters then
 * give the whole diagram -- the results rpd_solver_launch gives, bit for bit.
 * Not with Hessian rows or used cells. */
typedef int (*rpd_part_reduce_fn)(long long *sums, int nsum, long long *maxes, int nmax, void *user);
int rpd_solver_part_range(int n, int part, int parts, int *first, int *count);
int rpd_solver_launch_part(rpd_solver *s, const rpd_params *p, int part, int parts, rpd_part_reduce_fn reduce,
                           void *user);
/* Results of stored seeds first .. first + count - 1 (4 doubles and a status
 * each; either pointer may be null); stored order = the binned order of
 * rpd_solver_get_permutation. */
int rpd_solver_get_stored(rpd_solver *s, double *out4, int *status, int first, int count, rpd_mem where);
/* Installs every stored seed's results (n of each), e.g. gathered from the
 * parts, as this solver's last results. */
int rpd_solver_set_stored(rpd_solver *s, const double *out4, const int *status, rpd_mem where);

/* Per seed in USER order: (m*x, m*y, m*z, m) in the reference frame, as
 * getBarycenters + getPermutationToUser give them (voronoi.cpp:1165-1209);
 * zeros for failed cells; the seed itself for w <= RPD_NO_CELL_LIMITS. */
int rpd_solver_get_moments(rpd_solver *s, double *out4, rpd_mem where);
/* Per seed in user order: rpd_cell_status. */
int rpd_solver_get_status(rpd_solver *s, int *status, rpd_mem where);
int rpd_solver_get_stats(const rpd_solver *s, rpd_stats *st);
/* Used cells of the last launch with keep_distance >= 0 and a domain
 * (VoroAlgoComputeData::compressResult, voronoi.cpp:513-691): how many, and
 * their rows in ascending user order -- (m*x, m*y, m*z, m), with m =
 * RPD_NO_CELL_LIMITS for the outermost ring's cells below keep_volume (the
 * reference's border seeds, voronoi.cpp:604-611) -- with each row's user id
 * (getPermutationToUser).  The reference's order is that of an atomic
 * counter; here it is deterministic.  Returns the count or an error < 0. */
int rpd_solver_used_count(const rpd_solver *s);
int rpd_solver_get_used(rpd_solver *s, double *rows4, int *user_ids, rpd_mem where);

/* --------------------------------------------------------------- serving */

/* A request loop on one GPU (no counterpart in the reference, which solves
 * one diagram per process).  A session is one diagram kept on the device:
 * seeds, bins, neighbour table, results, and a device copy of its grid shared
 * by every session on the same rpd_grid (which must outlive the server).
 * Requests -- a new session's solve, or a weight-only re-solve of a session --
 * are admitted in arrival order as one of `slots` concurrent streams and
 * device memory free up: resident sessions plus the requests in flight stay
 * within mem_budget bytes (0: 90% of the free memory).  A session runs one
 * request at a time; requests of different sessions overlap on the device.
 * A request's result depends only on its own inputs. */
typedef struct rpd_server rpd_server;
typedef struct rpd_request_info {
  int status;         /* RPD_OK or the request's error */
  int session;
  int n;              /* seeds */
  int slot;           /* slot that ran it */
  double queue_ms;    /* submitted -> admitted */
  double latency_ms;  /* submitted -> done (moments written) */
  double device_ms;   /* the solve on the device (rpd_stats.total_ms) */
  int npasses;
  double admitted_at_ms;  /* since the server was created */
  double done_at_ms;      /* since the server was created */
  int failed_cells;   /* cells whose final status is neither success nor empty */
  char error[160];    /* the context's error text when status != RPD_OK */
  int status_hist[RPD_STATUS_NUM]; /* final status of every cell of the request */
  int last_caps[4];   /* K, P, V, T of the request's last pass */
} rpd_request_info;

rpd_server *rpd_server_create(int device, int slots, size_t mem_budget, int *err);
/* Waits for every submitted request, then frees everything. */
void rpd_server_destroy(rpd_server *sv);
/* A new session: the seeds (xyzw, host memory) are copied; when the request
 * is done its moments (4n doubles, user order) are in `moments`, which the
 * caller keeps valid until then (may be NULL).  Returns a ticket >= 0 or an
 * error < 0, and the session id in *session. */
int rpd_server_submit_solve(rpd_server *sv, const float *xyzw, int n, const rpd_grid *grid, const rpd_params *p,
                            double *moments, int *session);
/* A weight-only re-solve of a session: n weights (host memory, user order),
 * copied; runs after the session's earlier requests. */
int rpd_server_submit_reweight(rpd_server *sv, int session, const float *w, const rpd_params *p, double *moments);
/* The same requests with --hessian output: with p->hessian_h > 0 the
 * request also writes the Hessian rows of its solve into `hessian` (n *
 * hessian_h * hessian_hc doubles) and `hessian_ids` (n * hessian_h ints), user
 * order, as rpd_solver_get_hessian gives them (both kept valid by the caller
 * until the request is done; required then).  The plain submits reject
 * hessian_h > 0. */
int rpd_server_submit_solve_hessian(rpd_server *sv, const float *xyzw, int n, const rpd_grid *grid,
                                    const rpd_params *p, double *moments, double *hessian, int *hessian_ids,
                                    int *session);
int rpd_server_submit_reweight_hessian(rpd_server *sv, int session, const float *w, const rpd_params *p,
                                       double *moments, double *hessian, int *hessian_ids);
/* A new session whose domain is built on the device by its own solver, as
 * rpd_solver_set_grid_blob / rpd_solver_set_grid_field build it: no host grid
 * and no host preprocessing, e.g. for served requests with new domains (no
 * counterpart in the reference, whose domains come from its host tool).
 * The session keeps the domain for its re-solves; it is not shared with other
 * sessions.  field: (grid_size+1)^3 floats (host memory, copied; the domain
 * is {field < 0}).  grid_size <= 1024.  hessian / hessian_ids as in the
 * _hessian forms (required when p->hessian_h > 0, else may be NULL).  The
 * build's workspace counts in the request's memory, the domain in the
 * session's. */
int rpd_server_submit_solve_blob(rpd_server *sv, const float *xyzw, int n, int grid_size, int nellipsoids,
                                 uint64_t grid_seed, const rpd_params *p, double *moments, double *hessian,
                                 int *hessian_ids, int *session);
int rpd_server_submit_solve_field(rpd_server *sv, const float *xyzw, int n, int grid_size, const float *field,
                                  const rpd_params *p, double *moments, double *hessian, int *hessian_ids,
                                  int *session);
/* Blocks until the ticket's request is done and returns its status; each
 * ticket is waited for once. */
int rpd_server_wait(rpd_server *sv, int ticket, rpd_request_info *info);
/* Frees a session once its requests are done. */
int rpd_server_release(rpd_server *sv, int session);
/* Device bytes held by resident sessions, grids and admitted requests. */
size_t rpd_server_bytes_in_use(rpd_server *sv);

/* --hessian output of the last launch with hessian_h > 0 (VoroAlgo::
 * getHessians / getHessianIds, voronoi.h:161-180; CCExportBaryVolumeAndArea,
 * ConvexCell.cl:621-678): per seed (user order) a row of hessian_h facets of
 * its restricted cell -- one per neighbour whose shared facet inside the
 * domain has an area above 0.2 (squared reference-frame units), in the order
 * the neighbours' planes entered the cell -- with hessian_hc values each
 * (the area; or the area-weighted centroid x, y, z and the area, reference
 * frame).  values: n*hessian_h*hessian_hc doubles; ids: n*hessian_h ints,
 * the neighbours' user ids, -1 after a row's last facet (rows of cells that
 * did not succeed are empty).  A cell with more facets than hessian_h gets
 * the status RPD_HESSIAN_OVERFLOW and its first hessian_h facets.  With used
 * cells (keep_distance >= 0 and a domain) the rows are those of the used
 * cells, in the order of rpd_solver_get_used, and a facet's id is its
 * neighbour's position in that order (compact_result, voronoi.cpp:594-629):
 * rows of cells lighter than keep_volume are empty, and neighbours that are
 * not used or lighter than keep_volume are left out. */
int rpd_solver_get_hessian(rpd_solver *s, double *values, int *ids, rpd_mem where);

/* ------------------------------------------------------- result comparison */

/* The figures of the reference's result-diff tool (utils/diffResult/
 * main.cpp:62-121) for two moment sets a and b of n cells each (m*x, m*y,
 * m*z, m per cell, e.g. two rpd_solver_get_moments outputs or two .xyzw
 * result files): the summed moments of each, the largest mass difference
 * over all cells, and over the cells where both masses are positive the
 * largest and mean differences of mass, barycentre and first moments.  Host
 * memory; no device work. */
typedef struct rpd_moment_diff {
  long long cells;         /* n */
  long long cells_both;    /* cells with both masses > 0 */
  double sum_a[4], sum_b[4];
  double max_mass;         /* over all cells */
  double max_bary[3], max_moment[3];
  double avg_mass, avg_bary[3], avg_moment[3];  /* over cells_both */
} rpd_moment_diff;
int rpd_compare_moments(const double *a, const double *b, size_t n, rpd_moment_diff *out);

/* -------------------------------------------------------- batched solves */

/* Many independent diagrams solved together (no counterpart in the
 * reference, which solves one diagram per VoroAlgo::launch).  The solvers
 * belong to one context; each keeps its own seeds, domain and caps (params[i]
 * for solvers[i]; NULL: defaults for all).  Every pass of every diagram runs
 * in shared persistent launches -- one neighbour launch per K class, one cell
 * launch, the cone kernels, the failing-cell compaction -- and the retry
 * schedule (cap growth, failing-cell lists) is decided on the device, so the
 * whole solve is one CUDA graph, captured at the first rpd_batch_launch and
 * replayed after.  Each solver then holds exactly the results
 * rpd_solver_launch would give it (statuses, moments, stats' passes and
 * histogram), read with the solver's own getters.  Changing a solver's seeds
 * or domain is allowed between launches (the graph is captured again);
 * changing weights (rpd_solver_set_weights) is not a change.  --hessian rows
 * (hessian_h > 0, one hessian_hc for every diagram that asks for them) are
 * read with rpd_solver_get_hessian; their cells are summed in the cell's own
 * warp, so a batch with rows parks no boundary cell for the chunked kernel
 * and settles no triangle overflow ahead for any of its diagrams: per-pass
 * counts then equal those of rpd_solver_launch with RPD_FLAG_NO_DEFER (the
 * results, every solve's alike).  Not supported: RPD_FLAG_COUNTERS, used
 * cells (keep_distance >= 0 with a domain), precision other than FP64. */
typedef struct rpd_batch rpd_batch;
typedef struct rpd_batch_stats {
  int diagrams;
  long long cells;      /* seeds of all diagrams */
  float graph_ms;       /* device time of the last replay */
  int passes_captured;  /* passes in the graph */
  int max_passes;       /* most passes a diagram ran */
  int kernel_launches;  /* kernels per replay */
  int captures;         /* graph captures so far */
  int solved_alone;     /* diagrams whose retries outgrew the graph, solved after it on their own */
  float pass0_knn_ms;   /* of graph_ms: the first pass's neighbour launches */
  float pass0_cell_kernel_ms; /* of graph_ms: the first pass's cell kernel (no cone kernels) */
  float pass_ms[8];     /* of graph_ms: each captured pass (plan, neighbours, cells, compaction) */
  long long pass_cells[8]; /* cells of each pass, all diagrams */
  float probe_ms;       /* of pass_ms[0]: the outside probe and its compaction (0: no diagram probed) */
  long long probe_outside; /* seeds the probe proved empty outside their domains, all diagrams */
  /* The first pass's neighbour search per K class (K <= 32, 64, 96, 128, 192,
   * 256): 0 a warp per seed, 1 a thread per seed, -1 no diagram in the
   * class; chosen at capture by timing both on the class's own rows (0 ms:
   * no trial, too few rows or K too large for a thread per seed). */
  int knn_variant[6];
  float knn_trial_warp_ms[6], knn_trial_thread_ms[6];
} rpd_batch_stats;

rpd_batch *rpd_batch_create(rpd_context *ctx, rpd_solver *const *solvers, const rpd_params *params, int count,
                            int *err);
/* Solves every diagram; synchronous. */
int rpd_batch_launch(rpd_batch *b);
int rpd_batch_get_stats(const rpd_batch *b, rpd_batch_stats *st);
void rpd_batch_destroy(rpd_batch *b);

/* Debugging: re-runs one seed's cell (user id) with the caps of `p` and
 * records every clip and integration into `records` (cap records of 12
 * doubles: kind 0 seed, 1 plane test, 2 cavity, 3 vertex, 4 integration,
 * 5 start corner, 6 boundary triangle).  Returns the record count (>= 0) or
 * an rpd_error. */
int rpd_solver_trace_cell(rpd_solver *s, int user_id, const rpd_params *p, double *records, int cap);

/* --------------------------------------------------- allocation-free binning */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory (code running inside another framework's memory pool, plugins whose
 * host forbids allocation after start-up, paths that must not synchronize
 * the device the way cudaMalloc/cudaFree do): bins n seeds that are already
 * on the device into caller-owned device buffers, exactly as
 * rpd_solver_set_points does (stable counting sort, same permutation and bin
 * prefix sums), without allocating.  Its scratch lives in a fixed array of
 * the library's static device memory (about 1.7 MB, held by every GPU that
 * loads the library until the process exits).
 *
 *   xyzw      device, 4n floats, 16-byte aligned
 *   stored    device, 4n floats, 16-byte aligned: seeds in stored order
 *   perm      device, n ints: stored index -> user index
 *   counters  device, counters_cap ints (>= dim^3 + 1): bin prefix sums
 *   dim_out   receives dim = round((n / 3.1)^(1/3))
 *   stream    cudaStream_t (null: the default stream)
 *
 * n > RPD_NOALLOC_MAX_SEEDS returns RPD_ERR_CAPACITY; counters_cap below
 * dim^3 + 1 or a misaligned seed pointer returns RPD_ERR_INVALID (dim_out is
 * set first when n is in range); more than 4096 seeds in one bin returns
 * RPD_ERR_DEGENERATE and a NaN or infinite value RPD_ERR_INVALID.  After any
 * error the contents of stored, perm and counters are unspecified.
 *
 * The call is synchronous: it reads two words back from the device and waits
 * for its stream before returning, so it must never be called on a stream
 * that is being captured into a CUDA graph.  Every call looks up the array's
 * device address on the current device (so a device reset between calls is
 * harmless); the first call on a device also loads the library's device code
 * there.  Every call shares the one array, so calls that overlap on the GPU
 * (other streams, other host threads) race: serialize them. */
#define RPD_NOALLOC_MAX_SEEDS 262144
int rpd_bin_seeds_noalloc(const float *xyzw, int n, float *stored, int *perm, int *counters, int counters_cap,
                          int *dim_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* RPD_H */
