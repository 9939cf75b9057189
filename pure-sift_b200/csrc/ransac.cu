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
// Hypotheses are generated and fitted 64 at a time (one thread each; f64 DLT with
// the reference's cyclic Jacobi, same operation order), their inlier counts are
// computed by the whole CTA, and thread 0 replays the reference's loop in order:
// every decision (count, tie on the sequential error sum, adaptive iteration
// budget, LO refinement) is taken exactly as the reference takes it.  Error sums
// that decide something are the reference's sequential sums over the matches in
// input order (computed in parallel per match, summed serially); LO refits
// accumulate A^T A per entry sequentially over the inliers in order (45 threads).
#include <stdint.h>

#include "psift_internal.cuh"
#include "ransac_common.cuh"

namespace psift {

constexpr int kRThreads = 256;
constexpr int kBatch = 64;
constexpr int kDrawChunk = kBatch * 16;

struct RansacJob {
  const psift_match* m;
  int n;
  float thr;
  uint64_t sim_seed, hom_seed;
  int homography;           // 0: similarity only, 1: homography (similarity seed first)
  const float* weights;     // optional sampling weights replacing 1/clamp(ratio) (guided sampling)
  // scratch (n entries each, draws: draw_cap)
  double* cdf;
  double* err;
  int* list;
  int* draws;
  int draw_cap;
  // outputs
  uint8_t* mask;
  float* model;             // similarity: a, b, tx, ty, scale, rotation_deg; homography: 9 (row-major)
  int* has_model;
  int* count;
  int* iters;               // [0] similarity iterations, [1] homography iterations
  double* pts;              // 4 per match: the current inlier list's coordinates, gathered
};

struct RShared {
  int n;
  float tsq_f;
  double tsq_d;
  // similarity state
  float ba, bb, btx, bty;
  int best_count;
  float best_err_f;
  double best_err_d;
  int max_iters;
  int stop;
  int top32[32];
  int ntop;
  // batch of hypotheses
  float ha[kBatch], hb[kBatch], htx[kBatch], hty[kBatch];
  double H[kBatch][9];
  int hvalid[kBatch];
  int hcnt[kBatch];
  int quad[kBatch][4];
  // homography state
  double BH[9];
  int has_bh;
  // scratch scalars
  unsigned long long key_min;
  int flag;
  int ires[4];
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
  for (int w = 0; w < kRThreads / 32; ++w) t += (int)S.red_u[w];
  __syncthreads();
  return t;
}

__device__ __forceinline__ double block_sum_double(double v, RShared& S) {
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) S.red_d[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < kRThreads / 32; ++w) t += S.red_d[w];
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

// ------------------------------------------------------------- similarity
__device__ __forceinline__ bool sim_inlier(const psift_match& m, float a, float b, float tx, float ty, float tsq,
                                           float& e) {
  const float px = a * m.query_x - b * m.query_y + tx;
  const float py = b * m.query_x + a * m.query_y + ty;
  const float dx = px - m.target_x;
  const float dy = py - m.target_y;
  e = dx * dx + dy * dy;
  return e <= tsq;
}

// Count of a similarity hypothesis (whole CTA).
__device__ int sim_count(const RansacJob& J, RShared& S, float a, float b, float tx, float ty) {
  int c = 0;
  for (int i = threadIdx.x; i < S.n; i += kRThreads) {
    float e;
    c += sim_inlier(J.m[i], a, b, tx, ty, S.tsq_f, e) ? 1 : 0;
  }
  return block_sum_int(c, S);
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
    if (sim_inlier(J.m[i], a, b, tx, ty, S.tsq_f, e)) t += (double)J.weights[i];
  }
  return block_sum_double(t, S);
}

// Sequential f32 error sum over inliers in input order (whole CTA; result broadcast).
__device__ float sim_err(const RansacJob& J, RShared& S, float a, float b, float tx, float ty) {
  float* buf = reinterpret_cast<float*>(J.err);
  for (int i = threadIdx.x; i < S.n; i += kRThreads) {
    float e;
    buf[i] = sim_inlier(J.m[i], a, b, tx, ty, S.tsq_f, e) ? e : -1.0f;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // in order; 16 loads are issued ahead of the dependent additions
    float s = 0.0f;
    const int n = S.n;
    int i = 0;
    for (; i + 16 <= n; i += 16) {
      float e[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) e[u] = buf[i + u];
#pragma unroll
      for (int u = 0; u < 16; ++u)
        if (e[u] >= 0.0f) s += e[u];
    }
    for (; i < n; ++i) {
      const float e = buf[i];
      if (e >= 0.0f) s += e;
    }
    S.fres[0] = s;
  }
  __syncthreads();
  const float r = S.fres[0];
  __syncthreads();
  return r;
}

// Ordered inlier list of a similarity model into J.list; returns its length.
__device__ int sim_collect(const RansacJob& J, RShared& S, float a, float b, float tx, float ty) {
  int base = 0;
  for (int c0 = 0; c0 < S.n; c0 += kRThreads) {
    const int i = c0 + threadIdx.x;
    bool in = false;
    if (i < S.n) {
      const psift_match& m = J.m[i];
      // the collection expression of src/pipeline.rs:2161-2166 / :2172-2178
      const float dx = (a * m.query_x - b * m.query_y + tx) - m.target_x;
      const float dy = (b * m.query_x + a * m.query_y + ty) - m.target_y;
      in = dx * dx + dy * dy <= S.tsq_f;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, in);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) S.red_u[threadIdx.x >> 5] = __popc(bal);
    __syncthreads();
    int pre = 0, tot = 0;
    for (int w = 0; w < kRThreads / 32; ++w) {
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
__device__ bool procrustes(const RansacJob& J, RShared& S, int k, float* out6) {
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
  // Gather the inliers (list order): P[j] = (q.x, q.y, t.x, t.y); the sums stay
  // sequential in list order, their loads contiguous and issued ahead.
  float4* P = reinterpret_cast<float4*>(J.pts);
  for (int j = threadIdx.x; j < k; j += kRThreads) {
    const psift_match& m = J.m[J.list[j]];
    P[j] = make_float4(m.query_x, m.query_y, m.target_x, m.target_y);
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    float s = 0.0f;
    const int c = threadIdx.x;
#pragma unroll 8
    for (int j = 0; j < k; ++j) {
      const float4 p = P[j];
      s += c == 0 ? p.x : c == 1 ? p.y : c == 2 ? p.z : p.w;
    }
    S.fres[threadIdx.x] = s * inv_n;
  }
  __syncthreads();
  const float mqx = S.fres[0], mqy = S.fres[1], mtx = S.fres[2], mty = S.fres[3];
  if (threadIdx.x < 3) {
    float s = 0.0f;
#pragma unroll 8
    for (int j = 0; j < k; ++j) {
      const float4 p = P[j];
      const float qx = p.x - mqx, qy = p.y - mqy, tx = p.z - mtx, ty = p.w - mty;
      const float v = threadIdx.x == 0 ? qx * qx + qy * qy : threadIdx.x == 1 ? qx * tx + qy * ty : qx * ty - qy * tx;
      s += v;
    }
    S.fres[4 + threadIdx.x] = s;
  }
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

// filter_matches_ransac_with_seed (src/pipeline.rs:2055-2191).  Writes the
// inlier list (J.list, length S.sim_count) and S.sim_model / S.has_sim.
__device__ void similarity_ransac(const RansacJob& J, RShared& S, uint64_t seed, float thr) {
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
    procrustes(J, S, 1, m6);
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
      for (int w = 0; w < kRThreads / 32; ++w) {
        const unsigned long long v = (unsigned long long)__double_as_longlong(S.dres[w]);
        b = v < b ? v : b;
      }
      S.key_min = b;
      S.top32[r] = (int)(b & 0xFFFFFFFFu);
    }
    __syncthreads();
  }
  // initial model: translation of the lowest-ratio match
  {
    const psift_match& m0 = J.m[S.top32[0]];
    const float a = 1.0f, b = 0.0f, tx = m0.displacement_x, ty = m0.displacement_y;
    const int c = sim_count(J, S, a, b, tx, ty);
    const float e = sim_err(J, S, a, b, tx, ty);
    if (threadIdx.x == 0) {
      S.ba = a;
      S.bb = b;
      S.btx = tx;
      S.bty = ty;
      S.best_count = c;
      S.best_err_f = e;
    }
    __syncthreads();
  }
  // Phase A: the 32 one-point translations, in order
  for (int r = 0; r < ntop; ++r) {
    const psift_match& mr = J.m[S.top32[r]];
    const float tx = mr.displacement_x, ty = mr.displacement_y;
    const int c = sim_count(J, S, 1.0f, 0.0f, tx, ty);
    if (c >= S.best_count) {
      const float e = sim_err(J, S, 1.0f, 0.0f, tx, ty);
      if (threadIdx.x == 0 && (c > S.best_count || e < S.best_err_f)) {
        S.best_count = c;
        S.best_err_f = e;
        S.ba = 1.0f;
        S.bb = 0.0f;
        S.btx = tx;
        S.bty = ty;
      }
    }
    __syncthreads();
  }
  // Phase B: adaptive 2-point hypotheses
  build_cdf(J, S);
  const bool guided = J.weights != nullptr;
  const double wtot = guided ? weight_total(J, S) : 1.0;
  {
    const double mass = guided ? sim_mass(J, S, S.ba, S.bb, S.btx, S.bty) : 0.0;
    if (threadIdx.x == 0) {
      S.max_iters = guided ? adaptive_iters_w(mass / wtot, 2, 64, 1000) : adaptive_iters(S.best_count, n, 2, 64, 1000);
      S.stop = 0;
    }
  }
  __syncthreads();
  int iters_done = 0;
  for (int base = 0; !S.stop && base < 1000; base += kBatch) {
    if (base >= S.max_iters) break;
    const int t = threadIdx.x;
    if (t < kBatch) {
      const int it = base + t;  // 0-based iteration; draws 2it, 2it+1
      int i1 = sample_at(J.cdf, n, seed, 2ull * it);
      int i2 = sample_at(J.cdf, n, seed, 2ull * it + 1ull);
      if (i2 == i1) i2 = (i1 + 1) % n;
      const psift_match& m1 = J.m[i1];
      const psift_match& m2 = J.m[i2];
      const float dxq = m2.query_x - m1.query_x, dyq = m2.query_y - m1.query_y;
      const float dq = dxq * dxq + dyq * dyq;
      int valid = 0;
      float a = 0.f, b = 0.f, tx = 0.f, ty = 0.f;
      if (!(dq < 16.0f)) {
        const float dxt = m2.target_x - m1.target_x, dyt = m2.target_y - m1.target_y;
        a = (dxq * dxt + dyq * dyt) / dq;
        b = (dxq * dyt - dyq * dxt) / dq;
        const float s2 = a * a + b * b;
        if (s2 >= 0.04f && s2 <= 25.0f) {
          tx = m1.target_x - (a * m1.query_x - b * m1.query_y);
          ty = m1.target_y - (b * m1.query_x + a * m1.query_y);
          valid = 1;
        }
      }
      S.ha[t] = a;
      S.hb[t] = b;
      S.htx[t] = tx;
      S.hty[t] = ty;
      S.hvalid[t] = valid;
      S.hcnt[t] = 0;
    }
    __syncthreads();
    for (int h = 0; h < kBatch; ++h) {
      if (!S.hvalid[h]) continue;
      const int c = sim_count(J, S, S.ha[h], S.hb[h], S.htx[h], S.hty[h]);
      if (threadIdx.x == 0) S.hcnt[h] = c;
    }
    __syncthreads();
    // replay in order
    for (int h = 0; h < kBatch; ++h) {
      const int it = base + h;
      if (it >= S.max_iters) {
        if (threadIdx.x == 0) S.stop = 1;
        __syncthreads();
        break;
      }
      iters_done = it + 1;
      if (!S.hvalid[h]) continue;
      const int c = S.hcnt[h];
      if (c < S.best_count) continue;
      const float e = sim_err(J, S, S.ha[h], S.hb[h], S.htx[h], S.hty[h]);
      const bool improved = c > S.best_count || e < S.best_err_f;
      __syncthreads();
      if (improved) {
        const double mass = guided ? sim_mass(J, S, S.ha[h], S.hb[h], S.htx[h], S.hty[h]) : 0.0;
        if (threadIdx.x == 0) {
          S.best_count = c;
          S.best_err_f = e;
          S.ba = S.ha[h];
          S.bb = S.hb[h];
          S.btx = S.htx[h];
          S.bty = S.hty[h];
          S.max_iters = guided ? adaptive_iters_w(mass / wtot, 2, 64, 1000) : adaptive_iters(c, n, 2, 64, 1000);
        }
      }
      __syncthreads();
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && J.iters) J.iters[0] = iters_done;
  // consensus, Procrustes refit, re-collection
  const float a0 = S.ba, b0 = S.bb, tx0 = S.btx, ty0 = S.bty;
  int k = sim_collect(J, S, a0, b0, tx0, ty0);
  float refined[6];
  const bool has_ref = procrustes(J, S, k, refined);
  if (has_ref) {
    // count of the refined model's consensus (same expression as the collection)
    int c = 0;
    for (int i = threadIdx.x; i < n; i += kRThreads) {
      const psift_match& m = J.m[i];
      const float dx = (refined[0] * m.query_x - refined[1] * m.query_y + refined[2]) - m.target_x;
      const float dy = (refined[1] * m.query_x + refined[0] * m.query_y + refined[3]) - m.target_y;
      c += dx * dx + dy * dy <= S.tsq_f ? 1 : 0;
    }
    c = block_sum_int(c, S);
    if (c >= k) k = sim_collect(J, S, refined[0], refined[1], refined[2], refined[3]);
  }
  float fin[6];
  const bool has_fin = procrustes(J, S, k, fin);
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
__device__ __forceinline__ bool h_inlier(const psift_match& m, const double* H, double tsq, double& e) {
  const double qx = m.query_x, qy = m.query_y;
  const double w = H[6] * qx + H[7] * qy + H[8];
  if (fabs(w) < 1e-9) return false;
  const double iw = 1.0 / w;
  const double px = (H[0] * qx + H[1] * qy + H[2]) * iw;
  const double py = (H[3] * qx + H[4] * qy + H[5]) * iw;
  const double dx = px - (double)m.target_x, dy = py - (double)m.target_y;
  e = dx * dx + dy * dy;
  return e <= tsq;
}

__device__ int h_count(const RansacJob& J, RShared& S, const double* H) {
  int c = 0;
  for (int i = threadIdx.x; i < S.n; i += kRThreads) {
    double e;
    c += h_inlier(J.m[i], H, S.tsq_d, e) ? 1 : 0;
  }
  return block_sum_int(c, S);
}

__device__ double h_mass(const RansacJob& J, RShared& S, const double* H) {
  double t = 0.0;
  for (int i = threadIdx.x; i < S.n; i += kRThreads) {
    double e;
    if (h_inlier(J.m[i], H, S.tsq_d, e)) t += (double)J.weights[i];
  }
  return block_sum_double(t, S);
}

__device__ double h_err(const RansacJob& J, RShared& S, const double* H) {
  for (int i = threadIdx.x; i < S.n; i += kRThreads) {
    double e;
    J.err[i] = h_inlier(J.m[i], H, S.tsq_d, e) ? e : -1.0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // in order; 16 loads are issued ahead of the dependent additions
    double s = 0.0;
    const int n = S.n;
    int i = 0;
    for (; i + 16 <= n; i += 16) {
      double e[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) e[u] = J.err[i + u];
#pragma unroll
      for (int u = 0; u < 16; ++u)
        if (e[u] >= 0.0) s += e[u];
    }
    for (; i < n; ++i) {
      const double e = J.err[i];
      if (e >= 0.0) s += e;
    }
    S.dres[15] = s;
  }
  __syncthreads();
  const double r = S.dres[15];
  __syncthreads();
  return r;
}

__device__ int h_collect(const RansacJob& J, RShared& S, const double* H) {
  int base = 0;
  for (int c0 = 0; c0 < S.n; c0 += kRThreads) {
    const int i = c0 + threadIdx.x;
    bool in = false;
    if (i < S.n) {
      double e;
      in = h_inlier(J.m[i], H, S.tsq_d, e);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, in);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) S.red_u[threadIdx.x >> 5] = __popc(bal);
    __syncthreads();
    int pre = 0, tot = 0;
    for (int w = 0; w < kRThreads / 32; ++w) {
      if (w < (int)(threadIdx.x >> 5)) pre += (int)S.red_u[w];
      tot += (int)S.red_u[w];
    }
    if (in) J.list[base + pre + __popc(bal & ((1u << (threadIdx.x & 31)) - 1u))] = i;
    base += tot;
    __syncthreads();
  }
  return base;
}

// smallest_eigenvector_9x9 (src/pipeline.rs:2276-2353), one thread.
__device__ bool smallest_eigvec9(double (&a)[9][9], double* h) {
  double v[9][9];
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < 9; ++j) v[i][j] = i == j ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 20; ++sweep) {
    double max_off = 0.0;
    for (int p = 0; p < 9; ++p)
      for (int q = p + 1; q < 9; ++q) {
        const double av = fabs(a[p][q]);
        if (av > max_off) max_off = av;
      }
    if (max_off < 1e-13) break;
    for (int p = 0; p < 8; ++p)
      for (int q = p + 1; q < 9; ++q) {
        const double apq = a[p][q];
        if (fabs(apq) < 1e-15) continue;
        const double app = a[p][p], aqq = a[q][q];
        const double tau = (aqq - app) / (2.0 * apq);
        const double t = tau >= 0.0 ? 1.0 / (tau + sqrt(1.0 + tau * tau)) : -1.0 / (-tau + sqrt(1.0 + tau * tau));
        const double c = 1.0 / sqrt(1.0 + t * t);
        const double s = t * c;
        a[p][p] = app - t * apq;
        a[q][q] = aqq + t * apq;
        a[p][q] = 0.0;
        a[q][p] = 0.0;
        for (int r = 0; r < 9; ++r) {
          if (r != p && r != q) {
            const double arp = a[r][p], arq = a[r][q];
            a[r][p] = c * arp - s * arq;
            a[p][r] = a[r][p];
            a[r][q] = s * arp + c * arq;
            a[q][r] = a[r][q];
          }
          const double vrp = v[r][p], vrq = v[r][q];
          v[r][p] = c * vrp - s * vrq;
          v[r][q] = s * vrp + c * vrq;
        }
      }
  }
  int mi = 0;
  double me = a[0][0];
  for (int i = 1; i < 9; ++i)
    if (a[i][i] < me) {
      me = a[i][i];
      mi = i;
    }
  for (int r = 0; r < 9; ++r) {
    h[r] = v[r][mi];
    if (!isfinite(h[r])) return false;
  }
  return true;
}

// Normalisation + eigenvector -> de-normalised H (src/pipeline.rs:2482-2528).
__device__ bool finish_dlt(double (&ata)[9][9], double sq, double st, double cxq, double cyq, double cxt, double cyt,
                           double* H) {
  double hv[9];
  if (!smallest_eigvec9(ata, hv)) return false;
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
  return true;
}

// fit_homography_dlt_f64 on 4 matches, one thread.
__device__ bool fit_dlt4(const psift_match* const* s, double* H) {
  const double inv_n = 1.0 / 4.0;
  double cxq = 0, cyq = 0, cxt = 0, cyt = 0;
  for (int i = 0; i < 4; ++i) {
    const double qx = s[i]->query_x, qy = s[i]->query_y, tx = s[i]->target_x, ty = s[i]->target_y;
    if (!isfinite(qx) || !isfinite(qy) || !isfinite(tx) || !isfinite(ty)) return false;
    cxq += qx;
    cyq += qy;
    cxt += tx;
    cyt += ty;
  }
  cxq *= inv_n;
  cyq *= inv_n;
  cxt *= inv_n;
  cyt *= inv_n;
  double mdq = 0, mdt = 0;
  for (int i = 0; i < 4; ++i) {
    const double dxq = (double)s[i]->query_x - cxq, dyq = (double)s[i]->query_y - cyq;
    const double dxt = (double)s[i]->target_x - cxt, dyt = (double)s[i]->target_y - cyt;
    mdq += sqrt(dxq * dxq + dyq * dyq);
    mdt += sqrt(dxt * dxt + dyt * dyt);
  }
  mdq *= inv_n;
  mdt *= inv_n;
  if (!isfinite(mdq) || !isfinite(mdt) || mdq < 1e-6 || mdt < 1e-6) return false;
  const double sq = 1.41421356237309504880 / mdq, st = 1.41421356237309504880 / mdt;
  double ata[9][9];
  for (int a = 0; a < 9; ++a)
    for (int b = 0; b < 9; ++b) ata[a][b] = 0.0;
  for (int i = 0; i < 4; ++i) {
    const double x = ((double)s[i]->query_x - cxq) * sq, y = ((double)s[i]->query_y - cyq) * sq;
    const double xp = ((double)s[i]->target_x - cxt) * st, yp = ((double)s[i]->target_y - cyt) * st;
    const double r1[9] = {-x, -y, -1.0, 0.0, 0.0, 0.0, x * xp, y * xp, xp};
    const double r2[9] = {0.0, 0.0, 0.0, -x, -y, -1.0, x * yp, y * yp, yp};
    for (int a = 0; a < 9; ++a)
      for (int b = a; b < 9; ++b) ata[a][b] += r1[a] * r1[b] + r2[a] * r2[b];
  }
  for (int a = 0; a < 9; ++a)
    for (int b = 0; b < a; ++b) ata[a][b] = ata[b][a];
  return finish_dlt(ata, sq, st, cxq, cyq, cxt, cyt, H);
}

// fit_homography_dlt_f64 over J.list[0..k) (k >= 4), whole CTA; result in S.dres[0..8], flag in S.flag.
__device__ bool fit_dlt_list(const RansacJob& J, RShared& S, int k, double* H) {
  const double inv_n = 1.0 / (double)k;
  // Gather the inliers (list order) as doubles: P[j] = (q.x, q.y, t.x, t.y).  The
  // sums below stay sequential in list order (the reference's order); only the
  // loads change: contiguous, issued ahead of the dependent additions.
  double4* P = reinterpret_cast<double4*>(J.pts);
  for (int j = threadIdx.x; j < k; j += kRThreads) {
    const psift_match& m = J.m[J.list[j]];
    P[j] = make_double4((double)m.query_x, (double)m.query_y, (double)m.target_x, (double)m.target_y);
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = 0.0;
    bool finite = true;
    const int c = threadIdx.x;
#pragma unroll 8
    for (int j = 0; j < k; ++j) {
      const double4 p = P[j];
      const double v = c == 0 ? p.x : c == 1 ? p.y : c == 2 ? p.z : p.w;
      if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z) || !isfinite(p.w)) finite = false;
      s += v;
    }
    S.dres[threadIdx.x] = s * inv_n;
    if (threadIdx.x == 0) S.flag = finite ? 1 : 0;
  }
  __syncthreads();
  const bool finite = S.flag != 0;
  const double cxq = S.dres[0], cyq = S.dres[1], cxt = S.dres[2], cyt = S.dres[3];
  __syncthreads();
  if (!finite) return false;
  if (threadIdx.x < 2) {
    double s = 0.0;
    const double cx = threadIdx.x == 0 ? cxq : cxt, cy = threadIdx.x == 0 ? cyq : cyt;
#pragma unroll 8
    for (int j = 0; j < k; ++j) {
      const double4 p = P[j];
      const double dx = (threadIdx.x == 0 ? p.x : p.z) - cx;
      const double dy = (threadIdx.x == 0 ? p.y : p.w) - cy;
      s += sqrt(dx * dx + dy * dy);
    }
    S.dres[4 + threadIdx.x] = s * inv_n;
  }
  __syncthreads();
  const double mdq = S.dres[4], mdt = S.dres[5];
  __syncthreads();
  if (!isfinite(mdq) || !isfinite(mdt) || mdq < 1e-6 || mdt < 1e-6) return false;
  const double sq = 1.41421356237309504880 / mdq, st = 1.41421356237309504880 / mdt;
  // normalised coordinates in place: (x, y, x', y')
  for (int j = threadIdx.x; j < k; j += kRThreads) {
    const double4 p = P[j];
    P[j] = make_double4((p.x - cxq) * sq, (p.y - cyq) * sq, (p.z - cxt) * st, (p.w - cyt) * st);
  }
  __syncthreads();
  // upper triangle of A^T A: entry (a, b), a <= b, one thread each, sequential over the list
  if (threadIdx.x < 45) {
    int a = 0, rem = threadIdx.x;
    while (rem >= 9 - a) {
      rem -= 9 - a;
      ++a;
    }
    const int b = a + rem;
    double s = 0.0;
#pragma unroll 8
    for (int j = 0; j < k; ++j) {
      const double4 p = P[j];
      const double x = p.x, y = p.y, xp = p.z, yp = p.w;
      const double r1[9] = {-x, -y, -1.0, 0.0, 0.0, 0.0, x * xp, y * xp, xp};
      const double r2[9] = {0.0, 0.0, 0.0, -x, -y, -1.0, x * yp, y * yp, yp};
      s += r1[a] * r1[b] + r2[a] * r2[b];
    }
    S.ata[a][b] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ata[9][9];
    for (int a = 0; a < 9; ++a)
      for (int b = 0; b < 9; ++b) ata[a][b] = a <= b ? S.ata[a][b] : S.ata[b][a];
    double Hl[9];
    const bool ok = finish_dlt(ata, sq, st, cxq, cyq, cxt, cyt, Hl);
    S.flag = ok ? 1 : 0;
    for (int i = 0; i < 9; ++i) S.dres[i] = Hl[i];
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

// local_optimize_homography (src/pipeline.rs:2605-2631); updates H/count/err in place.
__device__ void local_optimize(const RansacJob& J, RShared& S, double* H, int& count, double& err) {
  for (int round = 0; round < 2; ++round) {
    const int k = h_collect(J, S, H);
    if (k < 4) break;
    double R[9];
    if (!fit_dlt_list(J, S, k, R)) break;
    const int rc = h_count(J, S, R);
    const double re = h_err(J, S, R);
    if (rc > count || (rc == count && re < err)) {
      for (int i = 0; i < 9; ++i) H[i] = R[i];
      count = rc;
      err = re;
    } else {
      break;
    }
  }
}

__global__ void __launch_bounds__(kRThreads) ransac_kernel(const RansacJob* __restrict__ jobs) {
  __shared__ RShared S;
  const RansacJob& J = jobs[blockIdx.x];
  const int n = J.n;
  if (threadIdx.x == 0) S.n = n;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += kRThreads) J.mask[i] = 0;
  similarity_ransac(J, S, J.sim_seed, J.thr);
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
  if (threadIdx.x == 0) {
    S.tsq_d = thresh * thresh;
    S.has_bh = S.has_sim;
    if (S.has_sim) {
      const double a = S.sim_model[0], b = S.sim_model[1];
      S.BH[0] = a;
      S.BH[1] = -b;
      S.BH[2] = S.sim_model[2];
      S.BH[3] = b;
      S.BH[4] = a;
      S.BH[5] = S.sim_model[3];
      S.BH[6] = 0.0;
      S.BH[7] = 0.0;
      S.BH[8] = 1.0;
    }
  }
  __syncthreads();
  int best_count = 0;
  double best_err = __longlong_as_double(0x7ff0000000000000ll);
  double BH[9];
  for (int i = 0; i < 9; ++i) BH[i] = S.BH[i];
  if (S.has_bh) {
    best_count = h_count(J, S, BH);
    best_err = h_err(J, S, BH);
  }
  auto finish_sim = [&]() {
    const int k = S.sim_count;
    for (int j = threadIdx.x; j < k; j += kRThreads) J.mask[J.list[j]] = 1;
    if (threadIdx.x == 0) {
      *J.count = k;
      *J.has_model = S.has_bh;
      for (int i = 0; i < 9; ++i) J.model[i] = S.has_bh ? (float)BH[i] : 0.0f;
    }
  };
  if (n < 4) {
    finish_sim();
    return;
  }
  // keep the similarity inliers for the no-model exit: they are in J.list only until
  // the first collection below, so record the flag now
  build_cdf(J, S);
  const bool guided = J.weights != nullptr;
  const double wtot = guided ? weight_total(J, S) : 1.0;
  {
    const double mass = (guided && S.has_bh) ? h_mass(J, S, BH) : 0.0;
    if (threadIdx.x == 0) {
      S.max_iters = guided ? adaptive_iters_w(mass / wtot, 4, 64, 2000) : adaptive_iters(best_count, n, 4, 64, 2000);
      S.stop = 0;
      S.draw_ptr = 0;
      S.draws_ready = 0;
    }
  }
  __syncthreads();
  const uint64_t seed = J.hom_seed;
  int iters_done = 0;
  bool list_is_sim = true;
  for (int base = 0; !S.stop && base < 2000; base += kBatch) {
    if (base >= S.max_iters) break;
    // draws for this batch: at most 16 per iteration
    {
      const int need = S.draw_ptr + kDrawChunk;
      for (int t0 = S.draws_ready; t0 < need && t0 < J.draw_cap; t0 += kRThreads) {
        const int t = t0 + threadIdx.x;
        if (t < need && t < J.draw_cap) S.draws_s[t % (2 * kDrawChunk)] = sample_at(J.cdf, n, seed, (uint64_t)t);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        S.draws_ready = need < J.draw_cap ? need : J.draw_cap;
        int p = S.draw_ptr;
        for (int h = 0; h < kBatch; ++h) {
          int chosen = 0, attempts = 0;
          int q[4] = {0, 0, 0, 0};
          while (chosen < 4 && attempts < 16) {
            ++attempts;
            const int c = S.draws_s[(p++) % (2 * kDrawChunk)];
            bool dup = false;
            for (int j = 0; j < chosen; ++j) dup |= q[j] == c;
            if (!dup) q[chosen++] = c;
          }
          S.quad[h][0] = q[0];
          S.quad[h][1] = q[1];
          S.quad[h][2] = q[2];
          S.quad[h][3] = q[3];
          S.hvalid[h] = chosen == 4 ? 1 : 0;
        }
        S.draw_ptr = p;
      }
      __syncthreads();
    }
    if (threadIdx.x < kBatch) {
      const int h = threadIdx.x;
      int valid = S.hvalid[h];
      if (valid) {
        const psift_match* quad[4] = {&J.m[S.quad[h][0]], &J.m[S.quad[h][1]], &J.m[S.quad[h][2]], &J.m[S.quad[h][3]]};
        double qp[4][2], tp[4][2];
        for (int i = 0; i < 4; ++i) {
          qp[i][0] = quad[i]->query_x;
          qp[i][1] = quad[i]->query_y;
          tp[i][0] = quad[i]->target_x;
          tp[i][1] = quad[i]->target_y;
        }
        if (degenerate4(qp) || degenerate4(tp)) {
          valid = 0;
        } else {
          double Hh[9];
          if (fit_dlt4(quad, Hh)) {
            for (int i = 0; i < 9; ++i) S.H[h][i] = Hh[i];
          } else {
            valid = 0;
          }
        }
      }
      S.hvalid[h] = valid;
      S.hcnt[h] = 0;
    }
    __syncthreads();
    for (int h = 0; h < kBatch; ++h) {
      if (!S.hvalid[h]) continue;
      const int c = h_count(J, S, S.H[h]);
      if (threadIdx.x == 0) S.hcnt[h] = c;
    }
    __syncthreads();
    for (int h = 0; h < kBatch; ++h) {
      const int it = base + h;
      if (it >= S.max_iters) {
        if (threadIdx.x == 0) S.stop = 1;
        __syncthreads();
        break;
      }
      iters_done = it + 1;
      if (!S.hvalid[h]) continue;
      int c = S.hcnt[h];
      if (c < best_count) continue;
      double e = h_err(J, S, S.H[h]);
      if (c > best_count || e < best_err) {
        double Hc[9];
        for (int i = 0; i < 9; ++i) Hc[i] = S.H[h][i];
        local_optimize(J, S, Hc, c, e);
        list_is_sim = false;
        best_count = c;
        best_err = e;
        for (int i = 0; i < 9; ++i) BH[i] = Hc[i];
        const double mass = guided ? h_mass(J, S, BH) : 0.0;
        if (threadIdx.x == 0) {
          S.has_bh = 1;
          S.max_iters = guided ? adaptive_iters_w(mass / wtot, 4, 64, 2000) : adaptive_iters(best_count, n, 4, 64, 2000);
        }
      }
      __syncthreads();
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && J.iters) J.iters[1] = iters_done;
  if (!S.has_bh) {
    // no model at all: the similarity inliers (still in J.list when no LO ran)
    if (list_is_sim) finish_sim();
    return;
  }
  local_optimize(J, S, BH, best_count, best_err);
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
  ransac_kernel<<<n_jobs, kRThreads, 0, st>>>(jobs);
  return cudaGetLastError();
}

size_t ransac_job_bytes() { return sizeof(RansacJob); }

}  // namespace psift
