// Shared definitions of the descriptor matcher (Matcher::match_).
#pragma once

#include <stdint.h>

#include "psift_gpu.h"

namespace psift {

// One matching problem (query set vs target set), device pointers.
struct MatchPair {
  const float* q;      // nq x 128 descriptors
  const float* t;      // nt x 128
  const float* qxy;    // nq x 2 keypoint coordinates
  const float* txy;    // nt x 2
  int nq, nt;
  // per-query exact top-2 (filled by the FP32 kernels or the re-rank)
  float* best;         // nq
  float* second;       // nq
  int* best_idx;       // nq
  // reverse nearest query per target (mutual check)
  float* col_best;     // nt
  int* col_idx;        // nt
  // outputs
  psift_match* out;    // capacity >= nq
  uint32_t* out_count;
  // BF16 path: row offsets of this pair in the concatenated bf16 operands
  int q_row0, t_row0;  // rows in the concatenated (padded) bf16 buffers
  const float* qn;     // nq exact f32 squared norms
  const float* tn;     // nt
  float* tn_max;       // scalar: max target squared norm
  float* qn_max;       // scalar: max query squared norm
};

// Tensor-core matcher tiles: 128-row A tiles x 256-row B tiles.  A pass's tiles
// are ordered (problem, A tile, B tile) and cut into equal ranges, one per CTA;
// the pieces of one A tile (at most kTcSplits: ranges are at least
// (B tiles - 1) / (kTcSplits - 1) long) write their partial results into their
// own slots, merged by window_kernel (pass 1) and rerank_kernel (pass 2).
constexpr int kTcBM = 128;
constexpr int kTcBN1 = 256;  // B tile rows (MMA N) of both passes
constexpr int kTcSplits = 4;
constexpr int kTcColl = 32;  // window indices kept per (slot, row)

// Tensor-core matcher problem (A rows matched against B rows).
struct TcPair {
  int na, nb;
  const float* an;   // f32 squared norms of A rows
  const float* bn;   // f32 squared norms of B rows
  float* top2;       // pass 1 output: [kTcSplits][na][2] two smallest approximate distances (+inf: no piece)
  const float* thr;  // pass 2 input: [na] candidate window (-inf: nothing to collect)
  int* coll_idx;     // pass 2 output: [kTcSplits][na][kTcColl] window indices
  int* coll_cnt;     // [kTcSplits][na] window sizes (may exceed kTcColl = overflow)
  // Pass 2 runs over the compacted A operand: the number of rows window_kernel
  // kept and, per compacted row, its row in the problem.
  const int* ccount;
  const int* rowmap;
  int a_row0, b_row0;  // first rows of the problem in the concatenated A / B operands
  int bt[2];           // B tiles in pass 1 / pass 2
  int at[2];           // A tiles in pass 1 / pass 2 (pass 2: written by tc_plan_kernel)
  long long g0[2];     // the problem's first tile in pass 1 / pass 2 order
};

// Tiles of one pass and the length of each CTA's range.
struct TcPlan {
  long long total;
  int per_cta;
  int pad;
};

// Copies the kept rows' bf16 descriptors into the compacted operand (one per
// problem and direction).
struct GatherJob {
  const uint16_t* src;  // the pair's A rows (bf16, 128 per row)
  uint16_t* dst;        // its compacted rows
  const int* rowmap;
  const int* count;
};

// Certified re-rank job (one per problem and direction).
struct RerankJob {
  const float* a;       // A descriptors (f32)
  const float* b;       // B descriptors (f32)
  int na, nb;
  const float* an;
  const float* bn_max;  // scalar
  const float* top2;    // [splits][na][2]
  float* thr;           // [na]
  const int* coll_idx;  // [splits][na][kTcColl]
  int* coll_cnt;        // [splits][na] (window_kernel clears the slots of the rows it keeps)
  int splits;           // kTcSplits
  float* best;          // outputs; `second` is null for the reverse (best-only) pass
  float* second;
  int* best_idx;
  uint32_t* fallbacks;  // rows that needed the exact scan
  float ratio;          // Lowe ratio (forward pass: rows certified to fail it are skipped)
  int* flags;           // forward: set flags[best] = 1 for accepted matches (mutual);
                        // reverse: only rows with flags[row] != 0 are ranked (null = all)
  int* ccount;          // window_kernel: rows kept for pass 2 (null: no compaction)
  int* rowmap;          // [na] their rows, in the order they were kept
  int* scan_count;      // rows handed to rerank_scan_kernel (all jobs of a direction share it)
  int2* scan_rows;      // their (job, row)
};

// Merge of two (best, idx, second) triples over disjoint target sets where ties
// on the best value keep the lower index and `second` is the second smallest
// value of the union multiset.  Commutative and associative, so any reduction
// order gives the sequential loop's result (src/pipeline.rs:1768-1786).
__device__ __forceinline__ void top2_merge(float& b, int& bi, float& s, float b2, int bi2, float s2) {
  if (b2 < b || (b2 == b && bi2 < bi)) {
    s = fminf(b, s2);
    b = b2;
    bi = bi2;
  } else {
    s = fminf(s, b2);
  }
}

__device__ __forceinline__ void top2_push(float& b, int& bi, float& s, float d, int idx) {
  if (d < b || (d == b && idx < bi)) {
    s = b;
    b = d;
    bi = idx;
  } else if (d < s) {
    s = d;
  }
}

}  // namespace psift
