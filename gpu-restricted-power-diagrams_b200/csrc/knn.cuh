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
cudaError_t knn_launch(const float4 *stored, const int *counters, int dim, const int *ids, int num, int K,
                       const float *ring_bound, unsigned *out, unsigned long long *candidates, cudaStream_t st);

}  // namespace rpd
