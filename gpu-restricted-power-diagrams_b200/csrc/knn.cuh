// K-nearest-neighbour search over binned seeds (one warp per seed).
#pragma once
#include "bins.cuh"

namespace rpd {

constexpr int kKnnThreads = 256;
constexpr int kMaxK = 256;

// Register slots per lane for a K-best list of K keys (32 keys per slot);
// -1 when K exceeds kMaxK.
int knn_slots(int K);

// Squared shell bounds ((ring-1) * 1000/dim)^2, ring 0..dim+1 (dim+2 floats).
void ring_bounds(int dim, float *bound);

// For every stored id in `ids` (or 0..num-1 when ids is null): the K nearest
// other seeds as stored indices, ascending (distance, index); 0xffffffff
// pads when fewer exist.  `candidates` (optional) accumulates the number of
// distance evaluations.
// variant: kKnnWarp (a warp per seed, bitonic merges) or kKnnThread (a
// thread per seed, a shared-memory heap; K <= kKnnThreadMaxK); the lists
// are the same bit for bit.
enum KnnVariant { kKnnWarp = 0, kKnnThread = 1 };
constexpr int kKnnThreadMaxK = 128;
cudaError_t knn_launch(const float4 *stored, const int *counters, int dim, const int *ids, int num, int K,
                       const float *ring_bound, unsigned *out, unsigned long long *candidates, cudaStream_t st,
                       int variant = kKnnWarp);

// One diagram of a batched neighbour launch: rows are ids[0..) (null: the
// seeds 0..), row i written to out + i*K.
struct KnnDiag {
  const float4 *stored;
  const int *counters;
  int dim;
  int K;
  const int *ids;
  const float *ring_bound;
  unsigned *out;
};
// Slot classes of knn_slots, in order.
constexpr int kKnnClasses = 6;
constexpr int kKnnClassSlots[kKnnClasses] = {1, 2, 3, 4, 6, 8};
// Persistent launch over the rows of every diagram of slot class S:
// start[0..ndiag] (device) are the row prefixes of the diagrams in this
// class (empty for the others); `blocks` fixed, the rows read on the device.
// rows >= 0: the class's row count, known when the launch is made: one warp
// per row; else `blocks` persistent blocks.
cudaError_t knn_batch_launch(int S, const KnnDiag *diags, const int *start, int ndiag, int blocks, cudaStream_t st,
                             long rows = -1, int variant = 0);

}  // namespace rpd
