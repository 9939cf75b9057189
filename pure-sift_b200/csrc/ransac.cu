// K10: similarity RANSAC and homography LO-RANSAC on the GPU, one CTA per match set.
//
// Reference (src/pipeline.rs): splitmix64_next (:1862-1868),
// evaluate_similarity_hypothesis (:1873-1897), fit_procrustes_similarity
// (:1900-1975), adaptive_ransac_iters (:1979-2002), build_ratio_weighted_cdf /
// sample_weighted_index (:2006-2036), filter_matches_ransac_with_seed
// (:2055-2191), smallest_eigenvector_9x9 (:2276-2353), has_degenerate_triangle /
// is_degenerate_quad (:2357-2404), fit_homography_dlt_f64 (:2408-2528),
// evaluate_homography_hypothesis_f64 / collect (:2550-2601),
// local_optimize_homography (:2605-2631), estimate_homography_ransac_with_seeds
// (:2663-2755).
//
// Identical results for the same seed.  The random stream does not depend on
// the data except through the CDF, so samples are drawn ahead: splitmix64's
// state advances by a constant, draw t is a pure function of (seed, t).
// Hypotheses are generated and fitted 32 at a time: a quad of lanes per
// homography fit (f64 DLT; the cyclic Jacobi's rotations shared by the quad in
// shared memory, each lane updating rows ql, ql + 4, ql + 8, so every value is
// the sequential solver's), then counted by warps (two hypotheses per pass over
// the packed match coordinates, no block barrier), and the reference's loop is
// replayed in order by every thread on identical shared values: every decision
// (count, tie on the sequential error sum, adaptive iteration budget, LO
// refinement) is taken exactly as the reference takes it.  Error sums are needed
// only to break a tie on the count, so they are computed when a tie occurs (for
// the incumbent too, if its sum is not known yet): an error sum is a function of
// the model alone, so the deferred value is the one the reference computed.
// Error sums are the reference's sequential sums over the matches in input order
// (terms computed in parallel, summed serially); LO refits accumulate A^T A per
// entry sequentially over the inliers in order (45 threads) and solve it with one
// quad.
#include <stdint.h>

#include "psift_internal.cuh"
#include "ransac_common.cuh"

namespace psift {

// 128 threads and 32 hypotheses per batch: the serial parts (replay, sequential
// sums, the Jacobi of a refit) leave most of a CTA idle, so four CTAs per SM
// (128 registers, ~51 KB of shared memory each) overlap more match sets.
constexpr int kRThreads = 128;
constexpr int kRWarps = kRThreads / 32;
constexpr int kBatch = 32;
constexpr int kRCtasPerSm = 4;
static_assert(kBatch * 4 == kRThreads, "a quad of lanes per hypothesis fit");
constexpr int kDrawChunk = kBatch * 16;
// Jacobi matrix and eigenvectors (81 doubles each) of every hypothesis of a batch
constexpr size_t kJacSmem = sizeof(double) * 162 * kBatch;
// LO refits stage row values (10 doubles per point) in the same buffer
constexpr int kRowChunk = (int)(kJacSmem / (sizeof(double) * 10));
// sequential sums over an inlier list stage its points (float4) there
constexpr int kPtChunk = (int)(kJacSmem / sizeof(float4));

struct RShared {
  int n;
  float tsq_f;
  double tsq_d;
  int top32[32];
  // batch of hypotheses
  float ha[kBatch], hb[kBatch], htx[kBatch], hty[kBatch];
  double H[kBatch][9];
  int hvalid[kBatch];
  int hcnt[kBatch];
  int quad[kBatch][4];
  // scratch scalars
  unsigned long long key_min;
  int flag;
  float fres[8];
  double dres[16];
  double ata[9][9];
  int draw_ptr, draws_ready;
  int draws_s[2 * kDrawChunk];  // draw t lives at [t % (2 * kDrawChunk)]
  int sim_count;
  float sim_model[6];
  int has_sim;
  uint32_t red_u[32];
  double red_d[32];
};

// build_ratio_weighted_cdf: weights in parallel, the running sum sequentially.
__device__ void build_cdf(const RansacJob& J, RShared& S) {
  const int n = S.n;
  for (int i = threadIdx.x; i < n; i += kRThreads) {
    double w;
    if (J.weights) {
      w = (double)J.weights[i];
    } else {
      const float r = J.m[i].ratio;
      double rd = 1.0;
      if (isfinite(r)) {
        rd = (double)r;
        rd = rd < 0.05 ? 0.05 : (rd > 1.0 ? 1.0 : rd);
      }
      w = 1.0 / rd;
    }
    J.cdf[i] = w;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // running sum in order; 16 weights are loaded ahead of the dependent additions
    double acc = 0.0;
    int i = 0;
    for (; i + 16 <= n; i += 16) {
      double w[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) w[u] = J.cdf[i + u];
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        acc += w[u];
        J.cdf[i + u] = acc;
      }
    }
    for (; i < n; ++i) {
      acc += J.cdf[i];
      J.cdf[i] = acc;
    }
    S.dres[0] = acc;
  }
  __syncthreads();
  const double acc = S.dres[0];
  if (acc > 0.0) {
    const double inv = 1.0 / acc;
    for (int i = threadIdx.x; i < n; i += kRThreads) J.cdf[i] *= inv;
  }
  __syncthreads();
  if (threadIdx.x == 0 && n > 0) J.cdf[n - 1] = 1.0;
  __syncthreads();
}

// adaptive_ransac_iters (src/pipeline.rs:1979-2002).
__device__ int adaptive_iters(int inl, int total, int ss, int min_it, int cap) {
  if (total == 0 || inl == 0) return cap;
  double w = (double)inl / (double)total;
  w = w < 1e-3 ? 1e-3 : (w > 1.0 - 1e-6 ? 1.0 - 1e-6 : w);
  double p = w * w;  // powi(w, 2) / powi(w, 4) as the compiler runtime evaluates them
  if (ss == 4) p = p * p;
  p = p < 1e-12 ? 1e-12 : (p > 1.0 - 1e-9 ? 1.0 - 1e-9 : p);
  const double num = log(1.0 - 0.999);
  const double den = log(1.0 - p);
  if (fabs(den) < 1e-12) return min_it;
  const double est = ceil(num / den);
  if (!isfinite(est)) return cap;
  double c = est;
  if (c < (double)min_it) c = (double)min_it;
  if (c > (double)cap) c = (double)cap;
  return (int)c;
}

// ---------------------------------------------------------- block reductions
__device__ __forceinline__ int block_sum_int(int v, RShared& S) {
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) S.red_u[threadIdx.x >> 5] = (uint32_t)v;
  __syncthreads();
  int t = 0;
  for (int w = 0; w < kRWarps; ++w) t += (int)S.red_u[w];
  __syncthreads();
  return t;
}

__device__ __forceinline__ double block_sum_double(double v, RShared& S) {
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) S.red_d[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < kRWarps; ++w) t += S.red_d[w];
  __syncthreads();
  return t;
}

// Guided sampling stops on the sampled inlier mass: the probability that one
// draw hits an inlier of the current model is w = sum over its inliers of the
// sampling weight / total weight (the reference's count / n when the weights are
// uniform).  Same formula as adaptive_ransac_iters otherwise.
__device__ int adaptive_iters_w(double w, int ss, int min_it, int cap) {
  if (!(w > 0.0)) return cap;
  w = w < 1e-3 ? 1e-3 : (w > 1.0 - 1e-6 ? 1.0 - 1e-6 : w);
  double p = w * w;
  if (ss == 4) p = p * p;
  p = p < 1e-12 ? 1e-12 : (p > 1.0 - 1e-9 ? 1.0 - 1e-9 : p);
  const double num = log(1.0 - 0.999);
  const double den = log(1.0 - p);
  if (fabs(den) < 1e-12) return min_it;
  const double est = ceil(num / den);
  if (!isfinite(est)) return cap;
  double c = est;
  if (c < (double)min_it) c = (double)min_it;
  if (c > (double)cap) c = (double)cap;
  return (int)c;
}

// Sequential sum, in match order, of term(i) for i < n: the CTA computes the
// terms of a chunk into shared memory (the batch's Jacobi space, free whenever a
// sum is taken), thread 0 adds them in order with its loads issued ahead of the
// dependent additions; the result is returned to every thread.  Terms of matches
// that are not inliers are zero, which leaves the running sum unchanged (x + 0 ==
// x for the finite, non-negative partial sums), so this equals the reference's
// sum over the inliers alone.
template <typename T, typename Term>
__device__ T ordered_sum(RShared& S, int n, Term term) {
  extern __shared__ double jac[];
  T* buf = reinterpret_cast<T*>(jac);
  constexpr int cap = (int)(kJacSmem / sizeof(T));
  T s = T(0);
  for (int c0 = 0; c0 < n; c0 += cap) {
    const int cn = min(cap, n - c0);
    for (int j = threadIdx.x; j < cn; j += kRThreads) buf[j] = term(c0 + j);
    __syncthreads();
    if (threadIdx.x == 0) {
      int j = 0;
      for (; j + 16 <= cn; j += 16) {
        T e[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) e[u] = buf[j + u];
#pragma unroll
        for (int u = 0; u < 16; ++u) s += e[u];
      }
      for (; j < cn; ++j) s += buf[j];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) S.dres[15] = (double)s;  // exact for float too
  __syncthreads();
  const T r = (T)S.dres[15];
  __syncthreads();
  return r;
}

// ------------------------------------------------------------- similarity
// evaluate_similarity_hypothesis's per-match test (src/pipeline.rs:1884-1893).
__device__ __forceinline__ bool sim_inlier(const float4 p, float a, float b, float tx, float ty, float tsq, float& e) {
  const float px = a * p.x - b * p.y + tx;
  const float py = b * p.x + a * p.y + ty;
  const float dx = px - p.z;
  const float dy = py - p.w;
  e = dx * dx + dy * dy;
  return e <= tsq;
}

// Inlier counts of the similarity hypotheses h < nh of the batch (S.ha.. /
// S.hvalid -> S.hcnt): warp w takes h = w, w + 8, ..., two per pass over the
// matches.  Ends with a block barrier.
__device__ void sim_count_batch(const RansacJob& J, RShared& S, int nh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float tsq = S.tsq_f;
  for (int h = warp; h < nh; h += 2 * kRWarps) {
    const int h2 = h + kRWarps;
    const bool v1 = S.hvalid[h] != 0, v2 = h2 < nh && S.hvalid[h2] != 0;
    int c1 = 0, c2 = 0;
    if (v1 || v2) {
      const float a1 = S.ha[h], b1 = S.hb[h], x1 = S.htx[h], y1 = S.hty[h];
      const float a2 = v2 ? S.ha[h2] : 0.f, b2 = v2 ? S.hb[h2] : 0.f, x2 = v2 ? S.htx[h2] : 0.f,
                  y2 = v2 ? S.hty[h2] : 0.f;
      for (int i = lane; i < S.n; i += 32) {
        const float4 p = J.xy[i];
        float e;
        c1 += (v1 && sim_inlier(p, a1, b1, x1, y1, tsq, e)) ? 1 : 0;
        c2 += (v2 && sim_inlier(p, a2, b2, x2, y2, tsq, e)) ? 1 : 0;
      }
    }
    for (int o = 16; o >= 1; o >>= 1) {
      c1 += __shfl_xor_sync(0xffffffffu, c1, o);
      c2 += __shfl_xor_sync(0xffffffffu, c2, o);
    }
    if (lane == 0) {
      S.hcnt[h] = c1;
      if (h2 < nh) S.hcnt[h2] = c2;
    }
  }
  __syncthreads();
}

__device__ double weight_total(const RansacJob& J, RShared& S) {
  double t = 0.0;
  for (int i = threadIdx.x; i < S.n; i += kRThreads) t += (double)J.weights[i];
  return block_sum_double(t, S);
}

__device__ double sim_mass(const RansacJob& J, RShared& S, float a, float b, float tx, float ty) {
  double t = 0.0;
  for (int i = threadIdx.x; i < S.n; i += kRThreads) {
    float e;
    if (sim_inlier(J.xy[i], a, b, tx, ty, S.tsq_f, e)) t += (double)J.weights[i];
  }
  return block_sum_double(t, S);
}

// Sequential f32 error sum over inliers in input order (whole CTA; result broadcast).
__device__ float sim_err(const RansacJob& J, RShared& S, float a, float b, float tx, float ty) {
  const float tsq = S.tsq_f;
  return ordered_sum<float>(S, S.n, [&](int i) {
    float e;
    return sim_inlier(J.xy[i], a, b, tx, ty, tsq, e) ? e : 0.0f;
  });
}

// Ordered inlier list of a similarity model into J.list; returns its length.
__device__ int sim_collect(const RansacJob& J, RShared& S, float a, float b, float tx, float ty) {
  int base = 0;
  for (int c0 = 0; c0 < S.n; c0 += kRThreads) {
    const int i = c0 + threadIdx.x;
    bool in = false;
    if (i < S.n) {
      const float4 p = J.xy[i];
      // the collection expression of src/pipeline.rs:2161-2166 / :2172-2178
      const float dx = (a * p.x - b * p.y + tx) - p.z;
      const float dy = (b * p.x + a * p.y + ty) - p.w;
      in = dx * dx + dy * dy <= S.tsq_f;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, in);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) S.red_u[threadIdx.x >> 5] = __popc(bal);
    __syncthreads();
    int pre = 0, tot = 0;
    for (int w = 0; w < kRWarps; ++w) {
      if (w < (int)(threadIdx.x >> 5)) pre += (int)S.red_u[w];
      tot += (int)S.red_u[w];
    }
    if (in) J.list[base + pre + __popc(bal & ((1u << (threadIdx.x & 31)) - 1u))] = i;
    base += tot;
    __syncthreads();
  }
  return base;
}

// fit_procrustes_similarity over J.list[0..k) (sequential sums; threads 0..6).
__device__ bool procrustes(const RansacJob& J, RShared& S, float* jac, int k, float* out6) {
  if (k == 0) return false;
  if (k == 1) {
    if (threadIdx.x == 0) {
      const psift_match& m = J.m[J.list[0]];
      S.fres[0] = 1.0f;
      S.fres[1] = 0.0f;
      S.fres[2] = m.displacement_x;
      S.fres[3] = m.displacement_y;
      S.fres[4] = 1.0f;
      S.fres[5] = 0.0f;
    }
    __syncthreads();
    for (int i = 0; i < 6; ++i) out6[i] = S.fres[i];
    __syncthreads();
    return true;
  }
  const float inv_n = 1.0f / (float)k;
  // The inliers' points (list order) staged in shared memory a chunk at a time;
  // the sums stay sequential in list order (threads 0..3, then 0..2), their
  // terms read at shared-memory latency.  One chunk is staged once for both.
  float4* st = reinterpret_cast<float4*>(jac);
  auto stage = [&](int c0, int cn) {
    for (int j = threadIdx.x; j < cn; j += kRThreads) st[j] = J.xy[J.list[c0 + j]];
  };
  float s = 0.0f;
  for (int c0 = 0; c0 < k; c0 += kPtChunk) {
    const int cn = min(kPtChunk, k - c0);
    stage(c0, cn);
    __syncthreads();
    if (threadIdx.x < 4) {
      const float* col = reinterpret_cast<const float*>(st) + threadIdx.x;
#pragma unroll 8
      for (int j = 0; j < cn; ++j) s += col[4 * j];
    }
    __syncthreads();
  }
  if (threadIdx.x < 4) S.fres[threadIdx.x] = s * inv_n;
  __syncthreads();
  const float mqx = S.fres[0], mqy = S.fres[1], mtx = S.fres[2], mty = S.fres[3];
  s = 0.0f;
  for (int c0 = 0; c0 < k; c0 += kPtChunk) {
    const int cn = min(kPtChunk, k - c0);
    if (k > kPtChunk) {
      stage(c0, cn);
      __syncthreads();
    }
    if (threadIdx.x < 3) {
#pragma unroll 8
      for (int j = 0; j < cn; ++j) {
        const float4 p = st[j];
        const float qx = p.x - mqx, qy = p.y - mqy, tx = p.z - mtx, ty = p.w - mty;
        const float v = threadIdx.x == 0 ? qx * qx + qy * qy : threadIdx.x == 1 ? qx * tx + qy * ty : qx * ty - qy * tx;
        s += v;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x < 3) S.fres[4 + threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    const float sqq = S.fres[4], na = S.fres[5], nb = S.fres[6];
    float a = 1.0f, b = 0.0f;
    if (sqq > 1e-5f) {
      const float af = na / sqq, bf = nb / sqq;
      const float s2 = af * af + bf * bf;
      if (s2 >= 0.04f && s2 <= 25.0f) {
        a = af;
        b = bf;
      }
    }
    S.dres[0] = a;  // staging through doubles is exact for f32 values
    S.dres[1] = b;
    S.dres[2] = mtx - (a * mqx - b * mqy);
    S.dres[3] = mty - (b * mqx + a * mqy);
    S.dres[4] = sqrtf(a * a + b * b);
    S.dres[5] = atan2f(b, a) * 57.2957795130823208767981548141051703f;
  }
  __syncthreads();
  for (int i = 0; i < 6; ++i) out6[i] = (float)S.dres[i];
  __syncthreads();
  return true;
}

// The incumbent of a replay: every thread holds the same copy (the replay reads
// only shared values that stay fixed while it runs, so every thread takes the
// same decisions); err is valid when err_known.
struct SimBest {
  float a, b, tx, ty;
  int count;
  float err;
  bool err_known;
};

// Replays hypothesis h of the batch against the incumbent (count first, the
// sequential error sum on a tie): true if it replaces the incumbent.
__device__ bool sim_consider(const RansacJob& J, RShared& S, SimBest& B, int h) {
  const int c = S.hcnt[h];
  if (c < B.count) return false;
  const float a = S.ha[h], b = S.hb[h], tx = S.htx[h], ty = S.hty[h];
  if (c > B.count) {
    B.count = c;
    B.err_known = false;
  } else {
    // the same parameters as the incumbent give the same error sum: not below it
    if (__float_as_uint(a) == __float_as_uint(B.a) && __float_as_uint(b) == __float_as_uint(B.b) &&
        __float_as_uint(tx) == __float_as_uint(B.tx) && __float_as_uint(ty) == __float_as_uint(B.ty))
      return false;
    if (!B.err_known) {
      B.err = sim_err(J, S, B.a, B.b, B.tx, B.ty);
      B.err_known = true;
    }
    const float e = sim_err(J, S, a, b, tx, ty);
    if (!(e < B.err)) return false;
    B.err = e;
  }
  B.a = a;
  B.b = b;
  B.tx = tx;
  B.ty = ty;
  return true;
}

// filter_matches_ransac_with_seed (src/pipeline.rs:2055-2191).  Writes the
// inlier list (J.list, length S.sim_count) and S.sim_model / S.has_sim.
__device__ void similarity_ransac(const RansacJob& J, RShared& S, double* jac, uint64_t seed, float thr) {
  const int n = S.n;
  if (threadIdx.x == 0) {
    S.has_sim = 0;
    S.sim_count = 0;
  }
  __syncthreads();
  if (n == 0) return;
  if (n == 1) {
    if (threadIdx.x == 0) J.list[0] = 0;
    __syncthreads();
    float m6[6];
    procrustes(J, S, reinterpret_cast<float*>(jac), 1, m6);
    if (threadIdx.x == 0) {
      for (int i = 0; i < 6; ++i) S.sim_model[i] = m6[i];
      S.has_sim = 1;
      S.sim_count = 1;
    }
    __syncthreads();
    return;
  }
  const float thresh = fmaxf(thr, 0.5f);
  if (threadIdx.x == 0) {
    S.tsq_f = thresh * thresh;
    S.key_min = 0;
  }
  __syncthreads();
  // the 32 lowest-ratio matches in stable order: keys (ratio bits, index) ascending
  const int ntop = n < 32 ? n : 32;
  for (int r = 0; r < ntop; ++r) {
    unsigned long long best = ~0ull;
    const unsigned long long floor_key = r == 0 ? 0ull : S.key_min;
    for (int i = threadIdx.x; i < n; i += kRThreads) {
      const float ratio = J.m[i].ratio;
      const uint32_t rb = __float_as_uint(ratio) ^ ((__float_as_uint(ratio) >> 31) ? 0xFFFFFFFFu : 0x80000000u);
      const unsigned long long key = ((unsigned long long)rb << 32) | (uint32_t)i;
      if ((r == 0 || key > floor_key) && key < best) best = key;
    }
    for (int o = 16; o >= 1; o >>= 1) {
      const unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
      best = t < best ? t : best;
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) S.dres[threadIdx.x >> 5] = __longlong_as_double((long long)best);
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long b = ~0ull;
      for (int w = 0; w < kRWarps; ++w) {
        const unsigned long long v = (unsigned long long)__double_as_longlong(S.dres[w]);
        b = v < b ? v : b;
      }
      S.key_min = b;
      S.top32[r] = (int)(b & 0xFFFFFFFFu);
    }
    __syncthreads();
  }
  // Phase A: the initial model (translation of the lowest-ratio match) and the 32
  // one-point translations, counted together, replayed in order.  The initial
  // model is translation 0: its evaluation is hypothesis 0's.
  if (threadIdx.x < ntop) {
    const psift_match& mr = J.m[S.top32[threadIdx.x]];
    S.ha[threadIdx.x] = 1.0f;
    S.hb[threadIdx.x] = 0.0f;
    S.htx[threadIdx.x] = mr.displacement_x;
    S.hty[threadIdx.x] = mr.displacement_y;
    S.hvalid[threadIdx.x] = 1;
  }
  __syncthreads();
  sim_count_batch(J, S, ntop);
  SimBest B{1.0f, 0.0f, S.htx[0], S.hty[0], S.hcnt[0], 0.0f, false};
  for (int r = 0; r < ntop; ++r) sim_consider(J, S, B, r);
  __syncthreads();  // the batch slots are rewritten below
  // Phase B: adaptive 2-point hypotheses
  build_cdf(J, S);
  const bool guided = J.weights != nullptr;
  const double wtot = guided ? weight_total(J, S) : 1.0;
  int max_iters = guided ? adaptive_iters_w(sim_mass(J, S, B.a, B.b, B.tx, B.ty) / wtot, 2, 64, 1000)
                         : adaptive_iters(B.count, n, 2, 64, 1000);
  int iters_done = 0;
  bool stop = false;
  for (int base = 0; !stop && base < 1000; base += kBatch) {
    if (base >= max_iters) break;
    const int t = threadIdx.x;
    if (t < kBatch) {
      const int it = base + t;  // 0-based iteration; draws 2it, 2it+1
      int i1 = sample_at(J.cdf, n, seed, 2ull * it);
      int i2 = sample_at(J.cdf, n, seed, 2ull * it + 1ull);
      if (i2 == i1) i2 = (i1 + 1) % n;
      const float4 m1 = J.xy[i1];
      const float4 m2 = J.xy[i2];
      const float dxq = m2.x - m1.x, dyq = m2.y - m1.y;
      const float dq = dxq * dxq + dyq * dyq;
      int valid = 0;
      float a = 0.f, b = 0.f, tx = 0.f, ty = 0.f;
      if (!(dq < 16.0f)) {
        const float dxt = m2.z - m1.z, dyt = m2.w - m1.w;
        a = (dxq * dxt + dyq * dyt) / dq;
        b = (dxq * dyt - dyq * dxt) / dq;
        const float s2 = a * a + b * b;
        if (s2 >= 0.04f && s2 <= 25.0f) {
          tx = m1.z - (a * m1.x - b * m1.y);
          ty = m1.w - (b * m1.x + a * m1.y);
          valid = 1;
        }
      }
      S.ha[t] = a;
      S.hb[t] = b;
      S.htx[t] = tx;
      S.hty[t] = ty;
      S.hvalid[t] = valid;
    }
    __syncthreads();
    sim_count_batch(J, S, kBatch);
    // replay in order
    for (int h = 0; h < kBatch; ++h) {
      const int it = base + h;
      if (it >= max_iters) {
        stop = true;
        break;
      }
      iters_done = it + 1;
      if (!S.hvalid[h]) continue;
      if (sim_consider(J, S, B, h))
        max_iters = guided ? adaptive_iters_w(sim_mass(J, S, B.a, B.b, B.tx, B.ty) / wtot, 2, 64, 1000)
                           : adaptive_iters(B.count, n, 2, 64, 1000);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && J.iters) J.iters[0] = iters_done;
  // consensus, Procrustes refit, re-collection
  int k = sim_collect(J, S, B.a, B.b, B.tx, B.ty);
  float refined[6];
  const bool has_ref = procrustes(J, S, reinterpret_cast<float*>(jac), k, refined);
  if (has_ref) {
    // count of the refined model's consensus (same expression as the collection)
    int c = 0;
    for (int i = threadIdx.x; i < n; i += kRThreads) {
      const float4 p = J.xy[i];
      const float dx = (refined[0] * p.x - refined[1] * p.y + refined[2]) - p.z;
      const float dy = (refined[1] * p.x + refined[0] * p.y + refined[3]) - p.w;
      c += dx * dx + dy * dy <= S.tsq_f ? 1 : 0;
    }
    c = block_sum_int(c, S);
    if (c >= k) k = sim_collect(J, S, refined[0], refined[1], refined[2], refined[3]);
  }
  float fin[6];
  const bool has_fin = procrustes(J, S, reinterpret_cast<float*>(jac), k, fin);
  if (threadIdx.x == 0) {
    S.sim_count = k;
    if (has_fin) {
      for (int i = 0; i < 6; ++i) S.sim_model[i] = fin[i];
      S.has_sim = 1;
    } else if (has_ref) {
      for (int i = 0; i < 6; ++i) S.sim_model[i] = refined[i];
      S.has_sim = 1;
    }
  }
  __syncthreads();
}

// ------------------------------------------------------------- homography
// evaluate_homography_hypothesis_f64's per-match test (src/pipeline.rs:2557-2573).
__device__ __forceinline__ bool h_inlier(const float4 p, const double* H, double tsq, double& e) {
  const double qx = p.x, qy = p.y;
  const double w = H[6] * qx + H[7] * qy + H[8];
  if (fabs(w) < 1e-9) return false;
  const double iw = 1.0 / w;
  const double px = (H[0] * qx + H[1] * qy + H[2]) * iw;
  const double py = (H[3] * qx + H[4] * qy + H[5]) * iw;
  const double dx = px - (double)p.z, dy = py - (double)p.w;
  e = dx * dx + dy * dy;
  return e <= tsq;
}

// Inlier counts of the homographies h < nh of the batch (S.H / S.hvalid ->
// S.hcnt): warp w takes h = w, w + 8, ..., two per pass.  Ends with a barrier.
__device__ void h_count_batch(const RansacJob& J, RShared& S, int nh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double tsq = S.tsq_d;
  for (int h = warp; h < nh; h += 2 * kRWarps) {
    const int h2 = h + kRWarps;
    const bool v1 = S.hvalid[h] != 0, v2 = h2 < nh && S.hvalid[h2] != 0;
    int c1 = 0, c2 = 0;
    if (v1 || v2) {
      double H1[9], H2[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) {
        H1[i] = S.H[h][i];
        H2[i] = v2 ? S.H[h2][i] : 0.0;
      }
      for (int i = lane; i < S.n; i += 32) {
        const float4 p = J.xy[i];
        double e;
        c1 += (v1 && h_inlier(p, H1, tsq, e)) ? 1 : 0;
        c2 += (v2 && h_inlier(p, H2, tsq, e)) ? 1 : 0;
      }
    }
    for (int o = 16; o >= 1; o >>= 1) {
      c1 += __shfl_xor_sync(0xffffffffu, c1, o);
      c2 += __shfl_xor_sync(0xffffffffu, c2, o);
    }
    if (lane == 0) {
      S.hcnt[h] = c1;
      if (h2 < nh) S.hcnt[h2] = c2;
    }
  }
  __syncthreads();
}

__device__ int h_count(const RansacJob& J, RShared& S, const double* H) {
  int c = 0;
  for (int i = threadIdx.x; i < S.n; i += kRThreads) {
    double e;
    c += h_inlier(J.xy[i], H, S.tsq_d, e) ? 1 : 0;
  }
  return block_sum_int(c, S);
}

__device__ double h_mass(const RansacJob& J, RShared& S, const double* H) {
  double t = 0.0;
  for (int i = threadIdx.x; i < S.n; i += kRThreads) {
    double e;
    if (h_inlier(J.xy[i], H, S.tsq_d, e)) t += (double)J.weights[i];
  }
  return block_sum_double(t, S);
}

// Sequential f64 error sum over the inliers in input order (whole CTA).
__device__ double h_err(const RansacJob& J, RShared& S, const double* H) {
  const double tsq = S.tsq_d;
  double Hl[9];
  for (int i = 0; i < 9; ++i) Hl[i] = H[i];
  return ordered_sum<double>(S, S.n, [&](int i) {
    double e;
    return h_inlier(J.xy[i], Hl, tsq, e) ? e : 0.0;
  });
}

__device__ int h_collect(const RansacJob& J, RShared& S, const double* H) {
  int base = 0;
  for (int c0 = 0; c0 < S.n; c0 += kRThreads) {
    const int i = c0 + threadIdx.x;
    bool in = false;
    if (i < S.n) {
      double e;
      in = h_inlier(J.xy[i], H, S.tsq_d, e);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, in);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) S.red_u[threadIdx.x >> 5] = __popc(bal);
    __syncthreads();
    int pre = 0, tot = 0;
    for (int w = 0; w < kRWarps; ++w) {
      if (w < (int)(threadIdx.x >> 5)) pre += (int)S.red_u[w];
      tot += (int)S.red_u[w];
    }
    if (in) J.list[base + pre + __popc(bal & ((1u << (threadIdx.x & 31)) - 1u))] = i;
    base += tot;
    __syncthreads();
  }
  return base;
}

// Offset i * 9 + j of strict upper-triangle entry k (row-major, 36 entries).
__device__ __forceinline__ int strict_upper_offset(int k) {
  int i = 0;
  while (k >= 8 - i) {
    k -= 8 - i;
    ++i;
  }
  return i * 9 + i + 1 + k;
}

// (a, b), a <= b, of upper-triangle entry e (row-major, 45 entries).
__device__ __forceinline__ void upper_entry(int e, int& a, int& b) {
  a = 0;
  while (e >= 9 - a) {
    e -= 9 - a;
    ++a;
  }
  b = a + e;
}

// smallest_eigenvector_9x9 (src/pipeline.rs:2276-2353), the cyclic Jacobi shared
// by a quad of lanes (ql = 0..3, converged, qmask their lane mask).  A (81
// doubles, shared memory, symmetric and complete) is diagonalised in place; V
// (81 doubles) accumulates the eigenvectors.  Every lane computes each
// rotation's parameters from the same values; lane ql updates rows ql, ql + 4,
// ql + 8 (a rotation's row updates touch disjoint entries), so every value and
// decision is the sequential solver's.  Returns the column of the smallest
// diagonal entry (the first on ties), or -1 if that eigenvector is not finite.
// A and V are complete and visible to the quad on return.
__device__ int quad_cyclic_jacobi(double* A, double* V, int ql, unsigned qmask) {
  for (int r = ql; r < 9; r += 4)
#pragma unroll
    for (int c = 0; c < 9; ++c) V[r * 9 + c] = r == c ? 1.0 : 0.0;
  // this lane's 9 of the 36 upper-triangle entries (row-major entries ql, ql + 4, ...)
  int off[9];
#pragma unroll
  for (int s = 0; s < 9; ++s) off[s] = strict_upper_offset(ql + 4 * s);
  __syncwarp(qmask);
  for (int sweep = 0; sweep < 20; ++sweep) {
    double mx = 0.0;
#pragma unroll
    for (int s = 0; s < 9; ++s) {
      const double v = fabs(A[off[s]]);
      if (v > mx) mx = v;
    }
    mx = fmax(mx, __shfl_xor_sync(qmask, mx, 1));
    mx = fmax(mx, __shfl_xor_sync(qmask, mx, 2));
    if (mx < 1e-13) break;
    for (int p = 0; p < 8; ++p)
      for (int q = p + 1; q < 9; ++q) {
        const double apq = A[p * 9 + q];
        if (fabs(apq) < 1e-15) continue;
        const double app = A[p * 9 + p], aqq = A[q * 9 + q];
        const double tau = (aqq - app) / (2.0 * apq);
        // __drcp_rn(x) is 1.0 / x: both are IEEE round-to-nearest, the reciprocal is the cheaper sequence
        const double t = tau >= 0.0 ? __drcp_rn(tau + sqrt(1.0 + tau * tau)) : -__drcp_rn(-tau + sqrt(1.0 + tau * tau));
        const double c = __drcp_rn(sqrt(1.0 + t * t));
        const double s = t * c;
        __syncwarp(qmask);  // every pivot read precedes the writes
        if (ql == 0) {
          A[p * 9 + p] = app - t * apq;
          A[q * 9 + q] = aqq + t * apq;
          A[p * 9 + q] = 0.0;
          A[q * 9 + p] = 0.0;
        }
        for (int r = ql; r < 9; r += 4) {
          if (r != p && r != q) {
            const double arp = A[r * 9 + p], arq = A[r * 9 + q];
            const double nrp = c * arp - s * arq, nrq = s * arp + c * arq;
            A[r * 9 + p] = nrp;
            A[p * 9 + r] = nrp;
            A[r * 9 + q] = nrq;
            A[q * 9 + r] = nrq;
          }
          const double vrp = V[r * 9 + p], vrq = V[r * 9 + q];
          V[r * 9 + p] = c * vrp - s * vrq;
          V[r * 9 + q] = s * vrp + c * vrq;
        }
        __syncwarp(qmask);
      }
  }
  int mi = 0;
  double me = A[0];
  for (int i = 1; i < 9; ++i)
    if (A[i * 10] < me) {
      me = A[i * 10];
      mi = i;
    }
  for (int r = 0; r < 9; ++r)
    if (!isfinite(V[r * 9 + mi])) return -1;
  return mi;
}

// De-normalisation of the null vector hv (src/pipeline.rs:2500-2528).
__device__ void denormalise(const double* hv, double sq, double st, double cxq, double cyq, double cxt, double cyt,
                            double* H) {
  const double hn[3][3] = {{hv[0], hv[1], hv[2]}, {hv[3], hv[4], hv[5]}, {hv[6], hv[7], hv[8]}};
  const double tq[3][3] = {{sq, 0.0, -sq * cxq}, {0.0, sq, -sq * cyq}, {0.0, 0.0, 1.0}};
  const double ist = 1.0 / st;
  const double tti[3][3] = {{ist, 0.0, cxt}, {0.0, ist, cyt}, {0.0, 0.0, 1.0}};
  double tmp[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) tmp[r][c] = hn[r][0] * tq[0][c] + hn[r][1] * tq[1][c] + hn[r][2] * tq[2][c];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) H[3 * r + c] = tti[r][0] * tmp[0][c] + tti[r][1] * tmp[1][c] + tti[r][2] * tmp[2][c];
  if (fabs(H[8]) > 1e-12) {
    const double inv = 1.0 / H[8];
    for (int i = 0; i < 9; ++i) H[i] *= inv;
  }
}

// The two A^T A rows of one normalised correspondence (x, y) -> (x', y')
// (src/pipeline.rs:2466-2479) take 10 distinct values, kept as one row:
//   [-x, -y, -1, 0, x x', y x', x', x y', y y', y']
// Row 1's entry a is row[(kSlot1 >> 4a) & 15], row 2's row[(kSlot2 >> 4a) & 15];
// every value is the reference's (negation is exact, the products are the same
// rounded products), so a sum of r1[a] r1[b] + r2[a] r2[b] terms is unchanged.
constexpr int kRowVals = 10;
constexpr unsigned long long kSlot1 = 0x654333210ull;  // -x -y -1 0 0 0 xx' yx' x'
constexpr unsigned long long kSlot2 = 0x987210333ull;  // 0 0 0 -x -y -1 xy' yy' y'

__device__ __forceinline__ void dlt_row_values(double x, double y, double xp, double yp, double* r) {
  r[0] = -x, r[1] = -y, r[2] = -1.0, r[3] = 0.0, r[4] = x * xp, r[5] = y * xp, r[6] = xp, r[7] = x * yp,
  r[8] = y * yp, r[9] = yp;
}

// fit_homography_dlt_f64 on 4 correspondences by a quad of lanes: every lane
// normalises; lane i writes point i's row values (in V, free until the Jacobi
// starts); the 45 A^T A entries are split over the lanes, each summed over the 4
// points in order; the quad runs the Jacobi.  The result (H, return value) is
// the leader's (ql == 0).
__device__ bool quad_fit4(const float4* __restrict__ xy, const int* idx, double* A, double* V, int ql,
                          unsigned qmask, double* H) {
  double qx[4], qy[4], tx[4], ty[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float4 p = xy[idx[i]];
    qx[i] = p.x, qy[i] = p.y, tx[i] = p.z, ty[i] = p.w;
  }
  const double inv_n = 1.0 / 4.0;
  double cxq = 0, cyq = 0, cxt = 0, cyt = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (!isfinite(qx[i]) || !isfinite(qy[i]) || !isfinite(tx[i]) || !isfinite(ty[i])) return false;
    cxq += qx[i];
    cyq += qy[i];
    cxt += tx[i];
    cyt += ty[i];
  }
  cxq *= inv_n;
  cyq *= inv_n;
  cxt *= inv_n;
  cyt *= inv_n;
  double mdq = 0, mdt = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double dxq = qx[i] - cxq, dyq = qy[i] - cyq;
    const double dxt = tx[i] - cxt, dyt = ty[i] - cyt;
    mdq += sqrt(dxq * dxq + dyq * dyq);
    mdt += sqrt(dxt * dxt + dyt * dyt);
  }
  mdq *= inv_n;
  mdt *= inv_n;
  if (!isfinite(mdq) || !isfinite(mdt) || mdq < 1e-6 || mdt < 1e-6) return false;
  const double sq = 1.41421356237309504880 / mdq, st = 1.41421356237309504880 / mdt;
  {
    const float4 p = xy[idx[ql]];
    dlt_row_values(((double)p.x - cxq) * sq, ((double)p.y - cyq) * sq, ((double)p.z - cxt) * st,
                   ((double)p.w - cyt) * st, V + ql * kRowVals);
  }
  __syncwarp(qmask);
  for (int e = ql; e < 45; e += 4) {
    int a, b;
    upper_entry(e, a, b);
    const int s1a = (int)(kSlot1 >> (4 * a)) & 15, s1b = (int)(kSlot1 >> (4 * b)) & 15;
    const int s2a = (int)(kSlot2 >> (4 * a)) & 15, s2b = (int)(kSlot2 >> (4 * b)) & 15;
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double* r = V + i * kRowVals;
      s += r[s1a] * r[s1b] + r[s2a] * r[s2b];
    }
    A[a * 9 + b] = s;
    A[b * 9 + a] = s;
  }
  __syncwarp(qmask);  // rows read, A complete
  const int mi = quad_cyclic_jacobi(A, V, ql, qmask);
  if (mi < 0 || ql != 0) return mi >= 0;
  double hv[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) hv[r] = V[r * 9 + mi];
  denormalise(hv, sq, st, cxq, cyq, cxt, cyt, H);
  return true;
}

// fit_homography_dlt_f64 over J.list[0..k) (k >= 4), whole CTA; jac holds one
// free A / V pair.  Result in H (every thread); false if the fit fails.
__device__ bool fit_dlt_list(const RansacJob& J, RShared& S, double* jac, int k, double* H) {
  const double inv_n = 1.0 / (double)k;
  // The inliers' points (list order) staged in shared memory a chunk at a time;
  // every sum below stays sequential in list order, its terms read at
  // shared-memory latency (the centroids by threads 0..3, the mean distances'
  // terms computed by the CTA and added by threads 0, 1).
  constexpr int kChunk = (int)(kJacSmem / (sizeof(float4) + 2 * sizeof(double)));
  float4* st = reinterpret_cast<float4*>(jac);
  double* dq = reinterpret_cast<double*>(st + kChunk);
  double* dt = dq + kChunk;
  auto stage = [&](int c0, int cn) {
    for (int j = threadIdx.x; j < cn; j += kRThreads) st[j] = J.xy[J.list[c0 + j]];
  };
  if (threadIdx.x == 0) S.flag = 1;
  double s = 0.0;
  for (int c0 = 0; c0 < k; c0 += kChunk) {
    const int cn = min(kChunk, k - c0);
    stage(c0, cn);
    __syncthreads();
    for (int j = threadIdx.x; j < cn; j += kRThreads) {
      const float4 p = st[j];
      if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z) || !isfinite(p.w)) S.flag = 0;
    }
    if (threadIdx.x < 4) {
      const float* col = reinterpret_cast<const float*>(st) + threadIdx.x;
#pragma unroll 8
      for (int j = 0; j < cn; ++j) s += (double)col[4 * j];
    }
    __syncthreads();
  }
  if (threadIdx.x < 4) S.dres[threadIdx.x] = s * inv_n;
  __syncthreads();
  const bool finite = S.flag != 0;
  const double cxq = S.dres[0], cyq = S.dres[1], cxt = S.dres[2], cyt = S.dres[3];
  __syncthreads();
  if (!finite) return false;
  s = 0.0;
  for (int c0 = 0; c0 < k; c0 += kChunk) {
    const int cn = min(kChunk, k - c0);
    if (k > kChunk) {
      stage(c0, cn);
      __syncthreads();
    }
    for (int j = threadIdx.x; j < cn; j += kRThreads) {
      const float4 p = st[j];
      const double ax = (double)p.x - cxq, ay = (double)p.y - cyq;
      const double bx = (double)p.z - cxt, by = (double)p.w - cyt;
      dq[j] = sqrt(ax * ax + ay * ay);
      dt[j] = sqrt(bx * bx + by * by);
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      const double* d = threadIdx.x == 0 ? dq : dt;
      int j = 0;
      for (; j + 16 <= cn; j += 16) {
        double e[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) e[u] = d[j + u];
#pragma unroll
        for (int u = 0; u < 16; ++u) s += e[u];
      }
      for (; j < cn; ++j) s += d[j];
    }
    __syncthreads();
  }
  if (threadIdx.x < 2) S.dres[4 + threadIdx.x] = s * inv_n;
  __syncthreads();
  const double mdq = S.dres[4], mdt = S.dres[5];
  __syncthreads();
  if (!isfinite(mdq) || !isfinite(mdt) || mdq < 1e-6 || mdt < 1e-6) return false;
  const double sq = 1.41421356237309504880 / mdq, st_ = 1.41421356237309504880 / mdt;
  // upper triangle of A^T A: entry (a, b), a <= b, one thread each, sequential
  // over the list; the points' normalised row values staged through jac a chunk
  // at a time
  {
    int a = 0, b = 0;
    if (threadIdx.x < 45) upper_entry(threadIdx.x, a, b);
    const int s1a = (int)(kSlot1 >> (4 * a)) & 15, s1b = (int)(kSlot1 >> (4 * b)) & 15;
    const int s2a = (int)(kSlot2 >> (4 * a)) & 15, s2b = (int)(kSlot2 >> (4 * b)) & 15;
    double sum = 0.0;
    for (int c0 = 0; c0 < k; c0 += kRowChunk) {
      const int cn = min(kRowChunk, k - c0);
      for (int j = threadIdx.x; j < cn; j += kRThreads) {
        const float4 p = J.xy[J.list[c0 + j]];
        dlt_row_values(((double)p.x - cxq) * sq, ((double)p.y - cyq) * sq, ((double)p.z - cxt) * st_,
                       ((double)p.w - cyt) * st_, jac + j * kRowVals);
      }
      __syncthreads();
      if (threadIdx.x < 45) {
#pragma unroll 8
        for (int j = 0; j < cn; ++j) {
          const double* r = jac + j * kRowVals;
          sum += r[s1a] * r[s1b] + r[s2a] * r[s2b];
        }
      }
      __syncthreads();
    }
    if (threadIdx.x < 45) {
      S.ata[a][b] = sum;
      S.ata[b][a] = sum;
    }
  }
  __syncthreads();
  if (threadIdx.x < 4) {  // the eigen-decomposition by the first quad
    const int ql = threadIdx.x;
    double* A = jac;
    double* V = jac + 81;
    for (int e = ql; e < 81; e += 4) A[e] = S.ata[e / 9][e % 9];
    __syncwarp(0xFu);
    const int mi = quad_cyclic_jacobi(A, V, ql, 0xFu);
    if (ql == 0) {
      S.flag = mi >= 0 ? 1 : 0;
      if (mi >= 0) {
        double hv[9], Hl[9];
        for (int r = 0; r < 9; ++r) hv[r] = V[r * 9 + mi];
        denormalise(hv, sq, st_, cxq, cyq, cxt, cyt, Hl);
        for (int i = 0; i < 9; ++i) S.dres[i] = Hl[i];
      }
    }
  }
  __syncthreads();
  const bool ok = S.flag != 0;
  for (int i = 0; i < 9; ++i) H[i] = S.dres[i];
  __syncthreads();
  return ok;
}

// has_degenerate_triangle (src/pipeline.rs:2357-2388)
__device__ bool degenerate4(const double (&p)[4][2]) {
  const int T[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
  for (int t = 0; t < 4; ++t) {
    const double xi = p[T[t][0]][0], yi = p[T[t][0]][1], xj = p[T[t][1]][0], yj = p[T[t][1]][1];
    const double xk = p[T[t][2]][0], yk = p[T[t][2]][1];
    if (!isfinite(xi) || !isfinite(yi) || !isfinite(xj) || !isfinite(yj) || !isfinite(xk) || !isfinite(yk)) return true;
    const double dx1 = xj - xi, dy1 = yj - yi, dx2 = xk - xi, dy2 = yk - yi, dx3 = xk - xj, dy3 = yk - yj;
    const double cross = fabs(dx1 * dy2 - dy1 * dx2);
    const double me = fmax(fmax(dx1 * dx1 + dy1 * dy1, dx2 * dx2 + dy2 * dy2), dx3 * dx3 + dy3 * dy3);
    if (cross < 4.0 || cross < 1e-3 * me) return true;
  }
  return false;
}

// local_optimize_homography (src/pipeline.rs:2605-2631); updates H / count /
// err in place (err valid when err_known; computed only for a tie).
__device__ void local_optimize(const RansacJob& J, RShared& S, double* jac, double* H, int& count, double& err,
                               bool& err_known) {
  for (int round = 0; round < 2; ++round) {
    const int k = h_collect(J, S, H);
    if (k < 4) break;
    double R[9];
    if (!fit_dlt_list(J, S, jac, k, R)) break;
    const int rc = h_count(J, S, R);
    if (rc < count) break;
    if (rc == count) {
      if (!err_known) {
        err = h_err(J, S, H);
        err_known = true;
      }
      const double re = h_err(J, S, R);
      if (!(re < err)) break;
      err = re;
    } else {
      err_known = false;
    }
    for (int i = 0; i < 9; ++i) H[i] = R[i];
    count = rc;
  }
}

__global__ void __launch_bounds__(kRThreads, kRCtasPerSm) ransac_kernel(const RansacJob* __restrict__ jobs) {
  __shared__ RShared S;
  extern __shared__ double jac[];
  const RansacJob& J = jobs[blockIdx.x];
  const int n = J.n;
  if (threadIdx.x == 0) S.n = n;
  for (int i = threadIdx.x; i < n; i += kRThreads) {
    J.mask[i] = 0;
    const psift_match& m = J.m[i];
    J.xy[i] = make_float4(m.query_x, m.query_y, m.target_x, m.target_y);
  }
  __syncthreads();
  similarity_ransac(J, S, jac, J.sim_seed, J.thr);
  if (!J.homography) {
    const int k = S.sim_count;
    for (int j = threadIdx.x; j < k; j += kRThreads) J.mask[J.list[j]] = 1;
    if (threadIdx.x == 0) {
      *J.count = k;
      *J.has_model = S.has_sim;
      for (int i = 0; i < 6; ++i) J.model[i] = S.has_sim ? S.sim_model[i] : 0.0f;
    }
    return;
  }
  // ---- homography (src/pipeline.rs:2663-2755)
  const double thresh = (double)fmaxf(J.thr, 0.5f);
  if (threadIdx.x == 0) S.tsq_d = thresh * thresh;
  __syncthreads();
  // The incumbent, held identically by every thread.
  bool has_bh = S.has_sim != 0;
  double BH[9];
  {
    const double a = S.sim_model[0], b = S.sim_model[1];
    BH[0] = a, BH[1] = -b, BH[2] = S.sim_model[2];
    BH[3] = b, BH[4] = a, BH[5] = S.sim_model[3];
    BH[6] = 0.0, BH[7] = 0.0, BH[8] = 1.0;
  }
  int best_count = 0;
  double best_err = __longlong_as_double(0x7ff0000000000000ll);
  bool err_known = true;
  if (has_bh) {
    best_count = h_count(J, S, BH);
    err_known = false;
  }
  auto finish_sim = [&]() {
    const int k = S.sim_count;
    for (int j = threadIdx.x; j < k; j += kRThreads) J.mask[J.list[j]] = 1;
    if (threadIdx.x == 0) {
      *J.count = k;
      *J.has_model = has_bh ? 1 : 0;
      for (int i = 0; i < 9; ++i) J.model[i] = has_bh ? (float)BH[i] : 0.0f;
    }
  };
  if (n < 4) {
    finish_sim();
    return;
  }
  build_cdf(J, S);
  const bool guided = J.weights != nullptr;
  const double wtot = guided ? weight_total(J, S) : 1.0;
  int max_iters = guided ? adaptive_iters_w((has_bh ? h_mass(J, S, BH) : 0.0) / wtot, 4, 64, 2000)
                         : adaptive_iters(best_count, n, 4, 64, 2000);
  if (threadIdx.x == 0) {
    S.draw_ptr = 0;
    S.draws_ready = 0;
  }
  __syncthreads();
  const uint64_t seed = J.hom_seed;
  const int draw_cap = 2000 * 16;  // at most 16 draws per iteration
  int iters_done = 0;
  bool stop = false;
  for (int base = 0; !stop && base < 2000; base += kBatch) {
    if (base >= max_iters) break;
    // draws for this batch: at most 16 per iteration
    {
      const int need = S.draw_ptr + kDrawChunk;
      for (int t0 = S.draws_ready; t0 < need && t0 < draw_cap; t0 += kRThreads) {
        const int t = t0 + threadIdx.x;
        if (t < need && t < draw_cap) S.draws_s[t % (2 * kDrawChunk)] = sample_at(J.cdf, n, seed, (uint64_t)t);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        S.draws_ready = need < draw_cap ? need : draw_cap;
        int p = S.draw_ptr;
        for (int h = 0; h < kBatch; ++h) {
          // distinct draws in order, held in registers (q0 first)
          int chosen = 0, attempts = 0;
          int q0 = 0, q1 = 0, q2 = 0, q3 = 0;
          while (chosen < 4 && attempts < 16) {
            ++attempts;
            const int c = S.draws_s[(p++) % (2 * kDrawChunk)];
            const bool dup = (chosen > 0 && q0 == c) || (chosen > 1 && q1 == c) || (chosen > 2 && q2 == c);
            if (!dup) {
              if (chosen == 0) q0 = c;
              else if (chosen == 1) q1 = c;
              else if (chosen == 2) q2 = c;
              else q3 = c;
              ++chosen;
            }
          }
          S.quad[h][0] = q0;
          S.quad[h][1] = q1;
          S.quad[h][2] = q2;
          S.quad[h][3] = q3;
          S.hvalid[h] = chosen == 4 ? 1 : 0;
        }
        S.draw_ptr = p;
      }
      __syncthreads();
    }
    // fits: a quad of lanes per hypothesis
    {
      const int h = threadIdx.x >> 2, ql = threadIdx.x & 3;
      const unsigned qmask = 0xFu << (threadIdx.x & 28);
      bool valid = S.hvalid[h] != 0;
      if (valid) {
        double qp[4][2], tp[4][2];
        for (int i = 0; i < 4; ++i) {
          const float4 p = J.xy[S.quad[h][i]];
          qp[i][0] = p.x;
          qp[i][1] = p.y;
          tp[i][0] = p.z;
          tp[i][1] = p.w;
        }
        if (degenerate4(qp) || degenerate4(tp)) {
          valid = false;
        } else {
          double Hh[9];
          valid = quad_fit4(J.xy, S.quad[h], jac + h * 162, jac + h * 162 + 81, ql, qmask, Hh);
          if (valid && ql == 0)
            for (int i = 0; i < 9; ++i) S.H[h][i] = Hh[i];
        }
      }
      __syncwarp();  // every lane of the quad has read S.hvalid[h]
      if (ql == 0) S.hvalid[h] = valid ? 1 : 0;
    }
    __syncthreads();
    h_count_batch(J, S, kBatch);
    // replay in order
    for (int h = 0; h < kBatch; ++h) {
      const int it = base + h;
      if (it >= max_iters) {
        stop = true;
        break;
      }
      iters_done = it + 1;
      if (!S.hvalid[h]) continue;
      int c = S.hcnt[h];
      if (c < best_count) continue;
      double e = 0.0;
      bool e_known = false;
      if (c == best_count) {
        if (!err_known) {
          best_err = h_err(J, S, BH);
          err_known = true;
        }
        e = h_err(J, S, S.H[h]);
        e_known = true;
        if (!(e < best_err)) continue;
      }
      double Hc[9];
      for (int i = 0; i < 9; ++i) Hc[i] = S.H[h][i];
      local_optimize(J, S, jac, Hc, c, e, e_known);
      best_count = c;
      best_err = e;
      err_known = e_known;
      for (int i = 0; i < 9; ++i) BH[i] = Hc[i];
      has_bh = true;
      max_iters = guided ? adaptive_iters_w(h_mass(J, S, BH) / wtot, 4, 64, 2000)
                         : adaptive_iters(best_count, n, 4, 64, 2000);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && J.iters) J.iters[1] = iters_done;
  if (!has_bh) {
    // no model at all: no hypothesis was accepted, so no LO ran and J.list still
    // holds the similarity inliers
    finish_sim();
    return;
  }
  local_optimize(J, S, jac, BH, best_count, best_err, err_known);
  const int k = h_collect(J, S, BH);
  for (int j = threadIdx.x; j < k; j += kRThreads) J.mask[J.list[j]] = 1;
  if (threadIdx.x == 0) {
    *J.count = k;
    *J.has_model = 1;
    for (int i = 0; i < 9; ++i) J.model[i] = (float)BH[i];
  }
}

cudaError_t launch_ransac(const RansacJob* jobs, int n_jobs, cudaStream_t st) {
  if (n_jobs <= 0) return cudaSuccess;
  cudaError_t e = ensure_smem_attr((const void*)ransac_kernel, kJacSmem);
  if (e != cudaSuccess) return e;
  ransac_kernel<<<n_jobs, kRThreads, kJacSmem, st>>>(jobs);
  return cudaGetLastError();
}

}  // namespace psift
