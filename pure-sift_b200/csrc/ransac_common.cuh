// Sampling shared by the RANSAC kernels (homography / similarity in ransac.cu,
// fundamental matrix in fundamental.cu).
//
// Reference: splitmix64_next (src/pipeline.rs:1862-1868), sample_weighted_index
// (:2029-2036).  splitmix64's state advances by a constant per draw, so draw t
// of a seed is a pure function of (seed, t): draws can be resolved in parallel
// ahead of the sequential loop that consumes them.
#pragma once
#include <stdint.h>

#include "psift_gpu.h"

namespace psift {

// One match set of the homography / similarity kernel (ransac.cu), filled by the
// host entry points (ransac_api.cu).
struct RansacJob {
  const psift_match* m;
  int n;
  float thr;
  uint64_t sim_seed, hom_seed;
  int homography;           // 0: similarity only, 1: homography (similarity seed first)
  const float* weights;     // optional sampling weights replacing 1/clamp(ratio) (guided sampling)
  // scratch (n entries each)
  double* cdf;
  double* err;
  int* list;
  float4* xy;               // (query x, query y, target x, target y) per match
  double* pts;              // 4 per match: the current inlier list's coordinates, gathered
  // outputs
  uint8_t* mask;
  float* model;             // similarity: a, b, tx, ty, scale, rotation_deg; homography: 9 (row-major)
  int* has_model;
  int* count;
  int* iters;               // [0] similarity iterations, [1] homography iterations
};

__device__ __forceinline__ uint64_t sm64_draw(uint64_t seed, uint64_t t) {
  uint64_t z = seed + (t + 1ull) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// sample_weighted_index: first index with cdf >= u, clamped to n-1.
__device__ __forceinline__ int sample_at(const double* __restrict__ cdf, int n, uint64_t seed, uint64_t t) {
  const double u = (double)(sm64_draw(seed, t) >> 11) * (1.0 / 9007199254740992.0);
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (cdf[mid] < u) lo = mid + 1;
    else hi = mid;
  }
  return lo < n - 1 ? lo : n - 1;
}

}  // namespace psift
