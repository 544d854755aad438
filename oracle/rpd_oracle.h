// Test infrastructure only -- the oracle.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg may load liboracle_rpd.so; the product
// library never links or calls it.
//
// A CPU restatement of the reference restricted-power-diagram path:
//   * seed binning + ring table        knearests.cpp:35-112,127-198
//   * K-nearest search                 knearests.cl:12-78
//   * convex-cell clipping             ConvexCell.cl:278-575
//   * domain restriction               ConvexCell.cl:918-1116
//   * signed-tet integration           ConvexCell.cl:577-619
//   * pass scheduler with retries      voronoi.cpp:770-859,861-1036,1244-1403
// in float (the reference default build, predicates VHSAlgo 0/1/2) or double
// (the reference USE_DOUBLE build, the FP64 truth).  The same host flow can
// drive either its own restated kernels or the reference's kernels compiled
// for the CPU (oracle/_ref/libref_kernels.so, see oracle/build_ref.sh), which
// is how the restatement is pinned.
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleGrid {
  int size;                 // voxels per axis (Grid::m_size, Grid.h:56)
  double voxel_size;        // Grid::m_voxelSize (1000/size)
  const char *in_domain;    // size^3 corner flags 0 out / 1 border / 2 in
  const double *points;     // 4*npoints, xyzw with w=0
  int npoints;
  const int *triangles;     // 3*ntri vertex ids
  int ntri;
  const int *tri_list;      // per-voxel sorted triangle ids
  int nlist;
  const int *offsets;       // size^3+1
} OracleGrid;

typedef struct OracleParams {
  int K, P, V, T;           // VoroAlgo::m_K/m_P/m_V/m_T (voronoi.h:199-206)
  int vhs0, vhs1;           // VoroAlgo::m_vhsAlgo[0..1] (float build only)
  int use_double;           // 1: the USE_DOUBLE build
  int kernels;              // 0: restated kernels, 1: reference kernels
  int knn_mode;             // 0: reference heap order, 1: exact (dist, stored index)
  int max_extra_passes;     // reference: 5 (voronoi.cpp:1321)
  int first_pass_only;      // 1: only pass "first" with T=caps.T (no retries)
  double cube_eps;          // CUBE_EPSILON: 0.1 with a grid, 0 without
  int nthreads;             // 0: all host threads
  int sample_stride;        // >1: only every stride-th stored seed is solved (timing samples)
  int used_cells;           // 1: mark used cells (needs a grid; voronoi.cpp:1291)
  int keep_distance;        // VoroAlgo::m_keepDistance (>= 0)
  double keep_volume;       // VoroAlgo::m_keepVolume
  int H;                    // VoroAlgo::m_H: facets per Hessian row, 0 = off (voronoi.h:207)
  int HC;                   // VoroAlgo::m_HC: 1 (area) or 4 (area-weighted centroid, area)
} OracleParams;

typedef struct OracleStats {
  int npasses;
  int pass_cells[8];
  double pass_seconds[8];
  int final_status[11];     // histogram over all seeds (Status.h)
  long long hs_tests;       // CCVertexIsInHalfSpace calls     (restated kernels)
  long long vertex_evals;   // CCComputeVertexCoordinates calls
  long long plane_clips;    // CCClipByPlane calls
  long long cone_clips;     // CCClipTetFromPointsInfinite calls
  long long export_vertices;// vertices visited by CCExportBaryVolume
  long long knn_candidates; // distance evaluations in the kNN scan
  double knn_seconds, cell_seconds;
} OracleStats;

// Full solve.  xyzw: 4*n seeds in the reference [0,1000]^3 frame.  Outputs in
// user order: bary 4*n (m*x, m*y, m*z, m, or the seed itself for w <=
// NO_CELL_LIMITS seeds), status n.  Returns 0 on success, <0 on error.
int oracle_solve(const double *xyzw, int n, const OracleGrid *grid, const OracleParams *p,
                 double *bary, int *status, OracleStats *stats);

// As oracle_solve, with the used-cell marks (user order, one byte per seed:
// 0 unused, else the ring distance, 1 for used cells) when p->used_cells.
int oracle_solve_used(const double *xyzw, int n, const OracleGrid *grid, const OracleParams *p, double *bary,
                      int *status, unsigned char *used, OracleStats *stats);

// As oracle_solve, with the Hessian rows of --hessian (p->H > 0;
// ConvexCell.cl:621-678,1133-1150) in user order: hess n*H*HC (per facet the
// area, or with HC = 4 the area-weighted centroid and the area), ids n*H
// (the facet's neighbour as a user id, -1 after the last facet of a row).
int oracle_solve_hessian(const double *xyzw, int n, const OracleGrid *grid, const OracleParams *p, double *bary,
                         int *status, double *hess, int *hess_ids, OracleStats *stats);

// K nearest neighbours of every seed, in user ids, ascending distance, -1 when
// fewer exist.  knn_mode as in OracleParams.
int oracle_knn(const double *xyzw, int n, int K, int use_double, int kernels, int knn_mode,
               int *knn, int nthreads);

// Counting-sort binning: stored order -> user id (perm), bins per axis, bin
// prefix sums (dim^3+1 entries, may be null).  Returns dim or <0.
int oracle_bin(const double *xyzw, int n, int use_double, int *perm, int *counters);

// Path of the loaded reference kernel library, or null when absent.
const char *oracle_ref_library(void);

// Domain volume and first moments of a grid's closed surface (Grid.cpp:30-51):
// out = (sum vol*x, sum vol*y, sum vol*z, vol).
void oracle_grid_invariants(const OracleGrid *grid, double *out4);

#ifdef __cplusplus
}
#endif
