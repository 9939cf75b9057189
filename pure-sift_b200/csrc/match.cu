// K7: exact FP32 brute-force Lowe-ratio matcher, and the stages shared with the
// BF16 tensor-core path (K8): partial merge, certified exact re-rank, emission.
//
// Reference: descriptor_dist_sq_early_exit (src/pipeline.rs:1700-1717),
// match_descriptors_with_options (:1744-1841), FeatureMatch (:1076-1091).
//
// Exactness: every distance is the reference's f32 value -- 128 squared
// differences accumulated sequentially from 0 in element order (rounded
// subtract, rounded multiply, rounded add; -fmad=false).  The early exit of the
// reference never changes best/second (a partial sum >= second cannot win), so
// full sums give the same top-2.  best/second are reduced with an index-aware
// merge (match_common.cuh) that equals the sequential loop for any order.
#include "match_common.cuh"
#include "psift_internal.cuh"

namespace psift {

constexpr int kMT = 128;  // query / target tile

// Grid (t_splits, q_tiles, pairs), 256 threads, 128 KB dynamic smem.
template <bool MUTUAL>
__global__ void __launch_bounds__(256) match_fp32_kernel(const MatchPair* __restrict__ pairs, int t_splits,
                                                         float* __restrict__ part, int* __restrict__ part_idx,
                                                         float* __restrict__ cpart, int* __restrict__ cpart_idx,
                                                         const long long* __restrict__ part_off,
                                                         const long long* __restrict__ cpart_off) {
  const MatchPair& P = pairs[blockIdx.z];
  const int q0 = blockIdx.y * kMT;
  if (q0 >= P.nq) return;
  const int n_ttiles = (P.nt + kMT - 1) / kMT;
  const int split = blockIdx.x;
  const int tt_begin = (int)((long long)n_ttiles * split / t_splits);
  const int tt_end = (int)((long long)n_ttiles * (split + 1) / t_splits);
  extern __shared__ float4 smem4[];
  float* sq = reinterpret_cast<float*>(smem4);  // [128 k][128 q]
  float* st = sq + 128 * kMT;                   // [128 k][128 t]
  const int tid = threadIdx.x;
  const int tq = tid >> 4, tt = tid & 15;

  // stage the query tile, transposed
  for (int i = tid; i < kMT * 32; i += 256) {
    const int q = i % kMT, c4 = i / kMT;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (q0 + q < P.nq) v = reinterpret_cast<const float4*>(P.q + (size_t)(q0 + q) * 128)[c4];
    sq[(4 * c4 + 0) * kMT + q] = v.x;
    sq[(4 * c4 + 1) * kMT + q] = v.y;
    sq[(4 * c4 + 2) * kMT + q] = v.z;
    sq[(4 * c4 + 3) * kMT + q] = v.w;
  }

  float best[8], second[8];
  int bidx[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    best[i] = __int_as_float(0x7f800000);
    second[i] = best[i];
    bidx[i] = 0x7fffffff;
  }
  int qrow[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) qrow[i] = q0 + (i < 4 ? 4 * tq + i : 64 + 4 * tq + (i - 4));

  for (int ti = tt_begin; ti < tt_end; ++ti) {
    const int t0 = ti * kMT;
    __syncthreads();
    for (int i = tid; i < kMT * 32; i += 256) {
      const int t = i % kMT, c4 = i / kMT;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (t0 + t < P.nt) v = reinterpret_cast<const float4*>(P.t + (size_t)(t0 + t) * 128)[c4];
      st[(4 * c4 + 0) * kMT + t] = v.x;
      st[(4 * c4 + 1) * kMT + t] = v.y;
      st[(4 * c4 + 2) * kMT + t] = v.z;
      st[(4 * c4 + 3) * kMT + t] = v.w;
    }
    __syncthreads();
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
#pragma unroll 2
    for (int k = 0; k < 128; ++k) {
      const float4 qa = *reinterpret_cast<const float4*>(sq + k * kMT + 4 * tq);
      const float4 qb = *reinterpret_cast<const float4*>(sq + k * kMT + 64 + 4 * tq);
      const float4 ta = *reinterpret_cast<const float4*>(st + k * kMT + 4 * tt);
      const float4 tb = *reinterpret_cast<const float4*>(st + k * kMT + 64 + 4 * tt);
      const float qv[8] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z, qb.w};
      const float tv[8] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const float d = __fsub_rn(qv[i], tv[j]);
          acc[i][j] = __fadd_rn(acc[i][j], __fmul_rn(d, d));
        }
    }
    int tcol[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) tcol[j] = t0 + (j < 4 ? 4 * tt + j : 64 + 4 * tt + (j - 4));
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (tcol[j] < P.nt) top2_push(best[i], bidx[i], second[i], acc[i][j], tcol[j]);
    if constexpr (MUTUAL) {
      // column (reverse) best over this tile's 128 queries, lowest query index on ties
      float cb[8];
      int ci[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        cb[j] = __int_as_float(0x7f800000);
        ci[j] = 0x7fffffff;
#pragma unroll
        for (int i = 0; i < 8; ++i)
          if (qrow[i] < P.nq && (acc[i][j] < cb[j] || (acc[i][j] == cb[j] && qrow[i] < ci[j]))) {
            cb[j] = acc[i][j];
            ci[j] = qrow[i];
          }
      }
      __syncthreads();
      float* sb = st;                                  // reuse: [16 tq][128 t]
      int* si = reinterpret_cast<int*>(st + 16 * kMT);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int c = j < 4 ? 4 * tt + j : 64 + 4 * tt + (j - 4);
        sb[tq * kMT + c] = cb[j];
        si[tq * kMT + c] = ci[j];
      }
      __syncthreads();
      if (tid < kMT && t0 + tid < P.nt) {
        float b = sb[tid];
        int bi = si[tid];
        for (int g = 1; g < 16; ++g) {
          const float v = sb[g * kMT + tid];
          const int vi = si[g * kMT + tid];
          if (v < b || (v == b && vi < bi)) {
            b = v;
            bi = vi;
          }
        }
        const long long o = cpart_off[blockIdx.z] + (long long)blockIdx.y * P.nt + t0 + tid;
        cpart[o] = b;
        cpart_idx[o] = bi;
      }
    }
  }
  // reduce the 16 threads (tt) that share each query row: lanes differ in bits 0..3
#pragma unroll
  for (int i = 0; i < 8; ++i) {
#pragma unroll
    for (int off = 8; off >= 1; off >>= 1) {
      const float b2 = __shfl_xor_sync(0xffffffffu, best[i], off);
      const int i2 = __shfl_xor_sync(0xffffffffu, bidx[i], off);
      const float s2 = __shfl_xor_sync(0xffffffffu, second[i], off);
      top2_merge(best[i], bidx[i], second[i], b2, i2, s2);
    }
  }
  if (tt == 0) {
    const long long base = part_off[blockIdx.z] + (long long)split * P.nq;
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (qrow[i] < P.nq) {
        part[2 * (base + qrow[i]) + 0] = best[i];
        part[2 * (base + qrow[i]) + 1] = second[i];
        part_idx[base + qrow[i]] = bidx[i];
      }
  }
}

// Per query: merge the split partials.  Per target (mutual): merge column partials.
__global__ void match_merge_kernel(const MatchPair* __restrict__ pairs, int t_splits, const float* __restrict__ part,
                                   const int* __restrict__ part_idx, const float* __restrict__ cpart,
                                   const int* __restrict__ cpart_idx, const long long* __restrict__ part_off,
                                   const long long* __restrict__ cpart_off, int mutual) {
  const MatchPair& P = pairs[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < P.nq) {
    float b = __int_as_float(0x7f800000), s = b;
    int bi = 0x7fffffff;
    for (int sp = 0; sp < t_splits; ++sp) {
      const long long o = part_off[blockIdx.y] + (long long)sp * P.nq + i;
      top2_merge(b, bi, s, part[2 * o], part_idx[o], part[2 * o + 1]);
    }
    P.best[i] = b;
    P.second[i] = s;
    P.best_idx[i] = bi;
  }
  if (mutual && i < P.nt) {
    const int n_qtiles = (P.nq + kMT - 1) / kMT;
    float b = __int_as_float(0x7f800000);
    int bi = 0x7fffffff;
    for (int qt = 0; qt < n_qtiles; ++qt) {
      const long long o = cpart_off[blockIdx.y] + (long long)qt * P.nt + i;
      const float v = cpart[o];
      const int vi = cpart_idx[o];
      if (v < b || (v == b && vi < bi)) {
        b = v;
        bi = vi;
      }
    }
    P.col_best[i] = b;
    P.col_idx[i] = bi;
  }
}

// Ratio test + ordered compaction (one block of 1024 threads per pair).
__global__ void __launch_bounds__(1024) match_emit_kernel(const MatchPair* __restrict__ pairs, float ratio,
                                                          int mutual) {
  const MatchPair& P = pairs[blockIdx.x];
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_total;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t carry = 0;
  for (int base = 0; base < P.nq; base += 1024) {
    const int q = base + threadIdx.x;
    bool keep = false;
    psift_match m;
    if (q < P.nq) {
      const float b = P.best[q], s = P.second[q];
      const int bi = P.best_idx[q];
      if (s > 1e-12f && b < __int_as_float(0x7f800000) && bi >= 0 && bi < P.nt) {
        const float d1 = sqrtf(b), d2 = sqrtf(s);
        const float r = d1 / d2;
        if (r < ratio) {
          keep = !mutual || P.col_idx[bi] == q;
          m.query_index = (uint32_t)q;
          m.target_index = (uint32_t)bi;
          m.query_x = P.qxy[2 * q];
          m.query_y = P.qxy[2 * q + 1];
          m.target_x = P.txy[2 * bi];
          m.target_y = P.txy[2 * bi + 1];
          m.distance = d1;
          m.ratio = r;
          m.displacement_x = m.target_x - m.query_x;
          m.displacement_y = m.target_y - m.query_y;
        }
      }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) s_warp[wid] = __popc(bal);
    __syncthreads();
    if (wid == 0) {
      const uint32_t v = s_warp[lane];
      uint32_t x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
      }
      s_warp[lane] = x - v;  // exclusive offset of each warp
      if (lane == 31) s_total = x;
    }
    __syncthreads();
    if (keep) P.out[carry + s_warp[wid] + __popc(bal & ((1u << lane) - 1u))] = m;
    carry += s_total;
    __syncthreads();
  }
  if (threadIdx.x == 0) *P.out_count = carry;
}

cudaError_t launch_match_fp32(const MatchPair* d_pairs, int n_pairs, int max_q_tiles, int t_splits, float* part,
                              int* part_idx, float* cpart, int* cpart_idx, const long long* part_off,
                              const long long* cpart_off, bool mutual, cudaStream_t st) {
  const size_t smem = 2 * 128 * kMT * sizeof(float);
  const void* fn = mutual ? (const void*)match_fp32_kernel<true> : (const void*)match_fp32_kernel<false>;
  cudaError_t e = ensure_smem_attr(fn, smem);
  if (e != cudaSuccess) return e;
  dim3 grid(t_splits, max_q_tiles, n_pairs);
  if (mutual)
    match_fp32_kernel<true><<<grid, 256, smem, st>>>(d_pairs, t_splits, part, part_idx, cpart, cpart_idx, part_off,
                                                     cpart_off);
  else
    match_fp32_kernel<false><<<grid, 256, smem, st>>>(d_pairs, t_splits, part, part_idx, cpart, cpart_idx, part_off,
                                                      cpart_off);
  return cudaGetLastError();
}

cudaError_t launch_match_merge(const MatchPair* d_pairs, int n_pairs, int max_n, int t_splits, const float* part,
                               const int* part_idx, const float* cpart, const int* cpart_idx,
                               const long long* part_off, const long long* cpart_off, bool mutual, cudaStream_t st) {
  dim3 grid((max_n + 255) / 256, n_pairs);
  match_merge_kernel<<<grid, 256, 0, st>>>(d_pairs, t_splits, part, part_idx, cpart, cpart_idx, part_off, cpart_off,
                                           mutual ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_match_emit(const MatchPair* d_pairs, int n_pairs, float ratio, bool mutual, cudaStream_t st) {
  match_emit_kernel<<<n_pairs, 1024, 0, st>>>(d_pairs, ratio, mutual ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace psift
