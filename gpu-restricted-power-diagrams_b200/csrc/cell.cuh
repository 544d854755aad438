// Per-seed restricted power cell: clipping, domain restriction, integration.
#pragma once
#include "common.cuh"

namespace rpd {

// Domain grid on the device (the reference Grid, Grid.h:14-70).
struct DevGrid {
  int size = 0;                       // voxels per axis
  float voxel = 0.f;                  // 1000 / size
  const signed char *flags = nullptr; // size^3 corner flags: 0 out, 1 border, 2 in
  const float4 *points = nullptr;     // triangle vertices (w unused)
  const int *tris = nullptr;          // 3 ids per triangle
  const int *list = nullptr;          // per-voxel sorted triangle ids
  const int *offsets = nullptr;       // size^3 + 1
  int has_border_corners = 0;         // any flag == 1
  // Summed-volume table, (size+1)^3, of voxels that are not plainly outside
  // (first-corner flag != 0 or a non-empty triangle list); null: unused.
  const int *sat = nullptr;
  // No triangle id appears in two voxel lists: the union of the lists of a
  // voxel range is their concatenation (no sort needed).
  int lists_disjoint = 0;
  // With disjoint lists: summed triangle counts, (size+1)^3, so a voxel
  // range's triangle count is 8 reads; null: unused.
  const int *tsat = nullptr;
};

// Counters of one launch (optional): cells by outcome and work done.
enum CellCounter {
  kCtrPlanesTested = 0,   // neighbour planes tested against the cell
  kCtrClips,              // clips that removed vertices
  kCtrVertexTests,        // vertex half-space tests
  kCtrVerticesMade,       // vertices created
  kCtrBoundaryCells,      // cells with at least one boundary triangle
  kCtrTriangles,          // boundary triangles processed
  kCtrExports,            // integrations (cell or cone pieces)
  kCtrExportVertices,     // vertices integrated
  kCtrOutside,            // cells proven outside the domain before the end of clipping
  kCtrConeEmpty,          // boundary triangles whose cone misses the cell
  kCtrConesSkipped,       // boundary triangles dropped: they miss the cell (apex inside it)
  kCtrEscTests,           // FP32 clipping: sign tests escalated to FP64
  kCtrEscVertices,        // FP32 clipping: vertices made in FP64 (near-degenerate)
  kCtrEscRadii,           // FP32 clipping: radius tests escalated to the exact FP64 radius
  kCtrStartCorner,        // boundary cells with cones from the reference's start corner
  kCtrNum
};

// Boundary cells with many triangles park their clipped cell here; a second
// kernel spreads their triangles over all warps in chunks.
struct DeferQueue {
  unsigned char *slots = nullptr;  // capacity slots of slot_bytes
  int capacity = 0;
  size_t slot_bytes = 0;
  // [0] cells parked, [1] next work item (cells with an inner apex), [2]
  // chunks taken, [3] the largest triangle count parked ahead
  // (CellLaunch::T_ahead), [4] next work item (cells with the reference's
  // start corner); zeroed before a pass
  int *counters = nullptr;
  // Work items are chunks, numbered compactly: a parked cell takes its
  // chunks' range from counters[2] and writes its slot for each of them
  int *chunk_slot = nullptr;       // capacity * max_chunks
  double *part = nullptr;          // capacity * max_chunks * 4 partial moments, by work item
  int *fail = nullptr;             // capacity * max_chunks: (triangle << 4) | status, or INT_MAX
  int max_chunks = 0;              // ceil(T / chunk)
  int chunk = 32;                  // triangles per work item
  int inline_max = 16;             // cells with at most this many triangles stay inline
};

struct CellLaunch {
  const float4 *stored = nullptr;  // n seeds in stored order (reference frame)
  int n = 0;
  const unsigned *knn = nullptr;   // num rows of K stored neighbour ids
  int K = 0;
  const int *ids = nullptr;        // stored ids of the rows (null: row i = seed i)
  int num = 0;
  int P = 0, V = 0, T = 0;         // caps of this pass
  // clipping precision: 0 FP64; 1 mixed (FP32 with FP64 escalation, the FP64
  // clipping's decisions); 2 plain FP32 (float planes, no escalation)
  int precision = 0;
  // first pass: a cell whose clip succeeded and whose range holds more than T
  // but at most T_ahead triangles (with disjoint lists, counted by grid.tsat)
  // is parked now with all of them -- the result the retry passes would give
  // it -- its start corner found as they would (out_domain_ahead); 0: off
  int T_ahead = 0;
  int out_domain_ahead = 0;
  int *ahead_max = nullptr;  // the largest count parked ahead (atomicMax; null: defer.counters[3])
  float cube_eps = 0.f;            // box [-eps, 1000+eps]^3
  int out_domain = 0;              // GRID_OUT_DOMAIN fallback for the start corner
  int early_out = 1;               // stop clipping cells proven outside the domain (needs grid.sat)
  // Triangle counts of the cells that failed with triangle_overflow (n ints,
  // stored order; optional, with disjoint lists): the first pass of a launch
  // (tri_first) writes every row's (0: none); a later pass settles a row whose
  // count is above its T at once -- the clip would give the same cell and
  // the same overflow
  int *tri_count = nullptr;
  int tri_first = 0;
  const int *wmin = nullptr;       // the smallest weight of the seeds that are not walls
                                   // (float_to_ordered); null: no early exit
  int inner_apex = 1;              // cone apex at a grid corner inside the cell when there is one
  int safe_radius = 0;             // the weighted security-radius guard instead of the reference's test
  DevGrid grid;                    // grid.size == 0: no domain
  int *status = nullptr;           // n, stored order
  double4 *out = nullptr;          // n, stored order: (m*x, m*y, m*z, m)
  unsigned long long *counters = nullptr;  // kCtrNum, optional
  // Trace of one cell (debugging): every clip and integration of stored seed
  // `trace_seed` appended to `trace` as records of kTraceRecord doubles;
  // trace[0] counts the records.
  int trace_seed = -1;
  double *trace = nullptr;
  int trace_cap = 0;  // records
  DeferQueue defer;   // slots == null: every boundary cell inline
  int only_status = -1;  // >= 0: process only the rows whose status equals it
  cudaEvent_t after_cell = nullptr;  // recorded after the cell kernel, before the cone kernels
  // used cells (a domain only): a successful cell with mass >= keep_volume
  // sets used[sid] = 1 and, with mark_dist >= 1, marks its face neighbours;
  // border_d > 0: bordering pass, clip only and mark the neighbours border_d
  unsigned char *used = nullptr;
  double keep_volume = 0.0;
  int mark_dist = 0;
  int border_d = 0;
  int diag = 0;  // index of this diagram in a batched launch (parked cells record it)
  // --hessian (no defer queue): per cell a row of H facets, HC values each,
  // and their neighbours (stored ids, -1 after the last), stored order
  double *hess = nullptr;
  int *hessid = nullptr;
  int H = 0, HC = 1;
};
constexpr int kParkOverflow = 101;  // internal status: the queue was full
constexpr int kProbeMiss = 102;     // internal status: the outside probe proved nothing
constexpr int kDeferCounters = 5;   // ints of DeferQueue::counters
constexpr int kTraceRecord = 12;

// Largest caps of one build: P <= 255 (uchar plane ids in the reference,
// voronoi.cpp:867), V <= 256, T <= kMaxT.
constexpr int kMaxP = 255;
constexpr int kMaxV = 256;
constexpr int kMaxT = 4096;

// Shared memory bytes one warp needs for these caps.
size_t cell_warp_smem(int P, int V, int T, bool grid);
// Bytes of one parked boundary cell for these caps.
size_t defer_slot_bytes(int P, int V, int T);
// k_cell over the rows; with a domain and a defer queue, also the chunked
// boundary-triangle kernel and the per-cell reduction (3 launches).
cudaError_t cell_launch(const CellLaunch &a, cudaStream_t st, int sm_count = 148, int *launches = nullptr);
// The same for a.precision > 0 (cell_prec.cu), and for FP64 clipping with
// the weighted security-radius guard (a.safe_radius; cell_safe.cu).
cudaError_t cell_launch_prec(const CellLaunch &a, cudaStream_t st, int sm_count, int *launches);
cudaError_t cell_launch_safe(const CellLaunch &a, cudaStream_t st, int sm_count, int *launches);

// Outside probe of a first pass with a domain.  The seeds of the 3x3x3 bins
// around a seed's own are a subset of all seeds, so their bisectors bound a
// region that contains the seed's power cell.  When that region fits the
// ball of plainly-outside voxels (flag 0, no triangle) around the seed, the
// cell is the domain's empty cell: status success and mass 0, as the full
// solve gives it.  Shown by a closed-form bound over 26 directions (balls of
// at least min_plain_cage) or by clipping with the 32 nearest of them
// (balls of at least min_plain).  Every other row gets kProbeMiss and is
// solved by the full pass.
struct ProbeLaunch {
  const float4 *stored = nullptr;  // n seeds in stored (bin) order
  int n = 0;                       // rows: the stored seeds first .. first + n - 1
  int first = 0;
  const int *bins = nullptr;       // dim^3 + 1 bin starts of the stored order
  int dim = 0;
  DevGrid grid;                    // with its summed-volume table (grid.sat)
  int P = 0, V = 0;                // caps of the first pass
  float cube_eps = 0.f;
  double min_plain_cage = 0.0;     // the cage test for balls at least this wide (reference frame)
  double min_plain = 0.0;          // clipping for balls at least this wide
  const int *wmin = nullptr;       // the smallest weight of the seeds that are not walls (float_to_ordered)
  int *status = nullptr;           // n, stored order
  double4 *out = nullptr;          // n, stored order
};
cudaError_t probe_launch(const ProbeLaunch &p, cudaStream_t st);
// The probe over every seed of many diagrams (batched solves): diagram d's
// record probes[d] (device) and rows start[d] .. start[d+1] (device; `rows`
// of them in all, known when the launch is made); P and V at least every
// diagram's first-pass caps.
cudaError_t probe_batch_launch(const ProbeLaunch *probes, const int *start, int ndiag, long rows, int P, int V,
                               cudaStream_t st);

// Whether one warp's layout for these caps fits a block's shared memory.
bool cell_caps_fit(int P, int V, int T, bool grid, int hc = 0);

// The cells of many diagrams in shared persistent launches (batched
// solves).  Row prefixes and launch records live on the device, written by
// earlier kernels of the same stream, so the launches can be captured in a
// graph before their row counts are known.
struct CellBatch {
  const CellLaunch *descs = nullptr;         // ndiag records; defer = the shared queue
  const CellLaunch *descs_inline = nullptr;  // the same records without the queue
  const int *start_grid = nullptr;   // ndiag+1 row prefixes of the diagrams with a domain (null: none)
  const int *start_plain = nullptr;  // ndiag+1 row prefixes of the diagrams without one (null: none)
  int ndiag = 0;
  DeferQueue defer;                  // slots == null: every boundary cell inline
  int P = 0, V = 0, T = 0;           // layout caps: at least every diagram's caps of this pass
  int T_slot = 0;                    // ids a parked cell's slot holds, when more than T (T_ahead)
  cudaEvent_t after_cell = nullptr;  // recorded (as a graph node when capturing) after the cell kernel
  // rows of the diagrams with / without a domain when known when the launch
  // is made (one warp per row), else -1 (persistent launches)
  long rows_grid = -1, rows_plain = -1;
  int *work = nullptr;  // one device int: the row counter of persistent launches (optional)
  bool safe = false;    // a diagram uses the weighted security-radius guard (its launch record decides)
  int HC = 0;           // Hessian rows' components (a diagram with rows; then no defer queue), else 0
  bool disjoint = false;  // every diagram's grid lists each triangle in one voxel (a smaller id buffer)
};
cudaError_t cell_batch_launch(const CellBatch &b, cudaStream_t st, int sm_count, int *launches = nullptr);
// The same with the guard compiled in (cell_safe.cu).
cudaError_t cell_batch_launch_safe(const CellBatch &b, cudaStream_t st, int sm_count, int *launches);

}  // namespace rpd
