// Test infrastructure only: argument blocks passed from the oracle host flow
// to the reference kernels compiled for the CPU (oracle/_ref/libref_kernels.so).
// Real-typed buffers are `void *`: they hold float or double depending on
// the build variant (the reference's USE_DOUBLE, cvoro_config.h.in:6-12).
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

typedef struct RefCellArgs {
  int num;                    // work-items in this batch
  const unsigned *ids;        // stored-order seed ids
  int ids_offset;             // first id of the batch in `ids`
  const void *pts;            // real4[n] stored (binned) seeds
  const unsigned *neigs;      // num*k neighbour ids (stored order)
  const char *grid_in_domain; // size^3 corner flags (null without a grid)
  const void *grid_points;    // real4[] triangle vertices
  const int *grid_triangles;  // 3 ids per triangle
  const int *grid_tri_list;   // per-voxel sorted triangle ids
  const int *grid_offsets;    // size^3+1 offsets into grid_tri_list
  int grid_size;
  double voxel_size;          // GRID_VOXEL_SIZE
  double cube_eps;            // CUBE_EPSILON
  int *status;                // Status[n]
  void *out;                  // real4[n]: (m*x, m*y, m*z, m)
  int k, p, v, t;             // caps of this pass
  int nthreads;               // 0 = all
  unsigned char *used;        // CUSED_CELL builds: usedCells[n] (stored order)
  double used_eps;            // USED_CELL_EPSILON
  void *hessian;              // CHESSIAN builds: real[n*H*HC] (stored order)
  int *hessidx;               // CHESSIAN builds: int[n*H]
  int h;                      // H
} RefCellArgs;

typedef struct RefKnnArgs {
  int dim;
  const int *counters;        // dim^3+1 exclusive prefix of bin counts
  const void *stored;         // real4[n] stored seeds
  int num_offsets;            // ring table entries (a sentinel follows)
  const int *offsets;
  const void *offset_dists;   // real[num_offsets+1]
  const int *ids;             // stored ids to process
  int num;
  int offset;
  unsigned *out;              // num*k
  int k;
  int nthreads;
} RefKnnArgs;

#ifdef __cplusplus
}
#endif
