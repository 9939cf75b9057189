// K4: 26-neighbour DoG extrema + Hessian edge test + 3D Taylor refinement, with
// ordered compaction, and the 4096-feature cap (stable top-K by |response|).
//
// Reference: passes_hessian_edge_test (src/pipeline.rs:664-687),
// refine_extremum_3d (:697-770), is_greater/less_than_patch3x3 (:775-808),
// extract_extrema_in_octave_slices (:810-916), Pyramid::extract_extrema
// (:535-547), the cap in extract_sift_features_with_kind (:1643-1651).
//
// Order: the reference emits keypoints octave by octave, slice by slice, row by
// row, column by column.  extrema_mark writes one bit per pixel plus a count per
// (octave, slice, row); row_scan turns the counts into exclusive offsets; and
// extrema_emit (one warp per row) writes each keypoint at its rank, so the list
// is identical in content and order to the reference's.
//
// Every arithmetic step repeats the reference's f32 expression in order
// (no FMA: the library is built with -fmad=false).  The single transcendental,
// k^ds, is evaluated in double and rounded once to f32.
#include "detect_plan.cuh"
#include "psift_internal.cuh"

namespace psift {

// refine_extremum_3d (src/pipeline.rs:697-770).
__device__ __forceinline__ void refine3d(const float* __restrict__ p, const float* __restrict__ c,
                                         const float* __restrict__ n, long long pitch, int x, float& ox_o,
                                         float& oy_o, float& os_o, float& interp_o) {
  const float* c_prev = c - pitch;
  const float* c_next = c + pitch;
  const float* p_prev = p - pitch;
  const float* p_next = p + pitch;
  const float* n_prev = n - pitch;
  const float* n_next = n + pitch;
  const float center = c[x];
  const float gx = 0.5f * (c[x + 1] - c[x - 1]);
  const float gy = 0.5f * (c_next[x] - c_prev[x]);
  const float gs = 0.5f * (n[x] - p[x]);
  const float dxx = c[x + 1] - 2.0f * center + c[x - 1];
  const float dyy = c_next[x] - 2.0f * center + c_prev[x];
  const float dss = n[x] - 2.0f * center + p[x];
  const float dxy = 0.25f * ((c_next[x + 1] - c_next[x - 1]) - (c_prev[x + 1] - c_prev[x - 1]));
  const float dxs = 0.25f * ((n[x + 1] - n[x - 1]) - (p[x + 1] - p[x - 1]));
  const float dys = 0.25f * ((n_next[x] - n_prev[x]) - (p_next[x] - p_prev[x]));
  const float c00 = dyy * dss - dys * dys;
  const float c01 = dys * dxs - dxy * dss;
  const float c02 = dxy * dys - dyy * dxs;
  const float c11 = dxx * dss - dxs * dxs;
  const float c12 = dxy * dxs - dxx * dys;
  const float c22 = dxx * dyy - dxy * dxy;
  const float det3 = dxx * c00 + dxy * c01 + dxs * c02;
  if (fabsf(det3) > 1e-9f) {
    const float inv_det = -1.0f / det3;
    const float ox = (c00 * gx + c01 * gy + c02 * gs) * inv_det;
    const float oy = (c01 * gx + c11 * gy + c12 * gs) * inv_det;
    const float os = (c02 * gx + c12 * gy + c22 * gs) * inv_det;
    if (fabsf(ox) <= 0.5f && fabsf(oy) <= 0.5f && fabsf(os) <= 0.5f) {
      ox_o = ox;
      oy_o = oy;
      os_o = os;
      interp_o = center + 0.5f * (gx * ox + gy * oy + gs * os);
      return;
    }
  }
  if (fabsf(c22) > 1e-9f) {
    const float inv_det2 = -1.0f / c22;
    float ox = (dyy * gx - dxy * gy) * inv_det2;
    float oy = (-dxy * gx + dxx * gy) * inv_det2;
    ox = ox < -0.5f ? -0.5f : (ox > 0.5f ? 0.5f : ox);
    oy = oy < -0.5f ? -0.5f : (oy > 0.5f ? 0.5f : oy);
    float os = 0.0f;
    if (fabsf(dss) > 1e-6f) {
      os = -gs / dss;
      os = os < -0.5f ? -0.5f : (os > 0.5f ? 0.5f : os);
    }
    ox_o = ox;
    oy_o = oy;
    os_o = os;
    interp_o = center + 0.5f * (gx * ox + gy * oy + gs * os);
    return;
  }
  ox_o = oy_o = os_o = 0.0f;
  interp_o = center;
}

// Full acceptance test for pixel (x, y) of slice `c` (rows already offset to y).
// The reference's comparison chain (is_greater/less_than_patch3x3 over the
// current, previous and next slices) is evaluated on loads issued together: the
// 8 same-slice neighbours first, then, only if they pass, the 18 of the other
// two slices.  Short-circuiting does not change the outcome (all must hold).
__device__ __forceinline__ bool accept_pixel(const float* __restrict__ p, const float* __restrict__ c,
                                             const float* __restrict__ n, long long pitch, int x, float thr) {
  const float v = c[x];
  if (fabsf(v) <= thr) return false;
  // All 26 neighbours are loaded before the first test: a warp's candidates are
  // tested together, so one of them passing the same-slice test would otherwise
  // make the whole warp wait for a second round of loads.
  const float* ca = c - pitch;
  const float* cb = c + pitch;
  float nb[9];
  nb[0] = ca[x - 1]; nb[1] = ca[x]; nb[2] = ca[x + 1];
  nb[3] = c[x - 1];  nb[4] = c[x + 1];
  nb[5] = cb[x - 1]; nb[6] = cb[x]; nb[7] = cb[x + 1];
  float pn[18];
  {
    const float* pa = p - pitch;
    const float* pb = p + pitch;
    const float* na = n - pitch;
    const float* nbp = n + pitch;
    pn[0] = pa[x - 1];  pn[1] = pa[x];  pn[2] = pa[x + 1];
    pn[3] = p[x - 1];   pn[4] = p[x];   pn[5] = p[x + 1];
    pn[6] = pb[x - 1];  pn[7] = pb[x];  pn[8] = pb[x + 1];
    pn[9] = na[x - 1];  pn[10] = na[x]; pn[11] = na[x + 1];
    pn[12] = n[x - 1];  pn[13] = n[x];  pn[14] = n[x + 1];
    pn[15] = nbp[x - 1]; pn[16] = nbp[x]; pn[17] = nbp[x + 1];
  }
  const bool pos = v > 0.0f;
  bool ext = true;
#pragma unroll
  for (int k = 0; k < 8; ++k) ext = ext && (pos ? v > nb[k] : v < nb[k]);
  if (!ext) return false;
#pragma unroll
  for (int k = 0; k < 18; ++k) ext = ext && (pos ? v > pn[k] : v < pn[k]);
  if (!ext) return false;
  // passes_hessian_edge_test (src/pipeline.rs:664-687)
  {
    const float dxx = nb[4] - 2.0f * v + nb[3];
    const float dyy = nb[6] - 2.0f * v + nb[1];
    const float dxy = 0.25f * ((nb[7] - nb[5]) - (nb[2] - nb[0]));
    const float trace = dxx + dyy;
    const float det = dxx * dyy - dxy * dxy;
    const float ratio = (11.0f * 11.0f) / 10.0f;
    if (!(det > 1e-9f && (trace * trace) < ratio * det)) return false;
  }
  float ox, oy, os, interp;
  refine3d(p, c, n, pitch, x, ox, oy, os, interp);
  return fabsf(interp) > thr;
}

// Grid (ceil(max_h / 4), scales, images), 128 threads: one warp per (row,
// slice, image), no block-wide barriers.  The warp walks its row in 256-pixel
// spans (a lane reads 8 pixels as two 128-bit loads, 128 pixels apart; the
// next span's loads are issued before the current span is processed); a span is
// exactly 8 mask words.
//   A. streaming: pixels with |v| > threshold (the reference's first test, a
//      small fraction of the row) become candidates; a span without any writes
//      zero words;
//   B. otherwise the candidates are compacted into the warp's shared-memory
//      queue and the warp runs the full 26-neighbour / Hessian / refinement
//      test on them only, setting bits of the span's 8 mask words.
constexpr int kMarkWarps = 4;
constexpr int kMarkSpan = 256;  // pixels per warp step

__device__ __forceinline__ void mark_load_span(const float* __restrict__ Dc, int xb, int lane, int w, float4 (&v)[2]) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int x0 = xb + h * 128 + 4 * lane;
    if (x0 + 3 < w) {
      v[h] = *reinterpret_cast<const float4*>(Dc + x0);
    } else {
      v[h] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (x0 + 0 < w) v[h].x = Dc[x0 + 0];
      if (x0 + 1 < w) v[h].y = Dc[x0 + 1];
      if (x0 + 2 < w) v[h].z = Dc[x0 + 2];
    }
  }
}

__global__ void __launch_bounds__(kMarkWarps * 32) extrema_mark_kernel(const ImagePlan* __restrict__ plans,
                                                                       int octave, ExtremaParams prm) {
  const ImagePlan& P = plans[blockIdx.z];
  if (octave >= P.n_oct) return;
  const OctaveDev& O = P.oct[octave];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int y = blockIdx.y * kMarkWarps + warp;
  if (y >= O.h) return;
  const int s = blockIdx.x + 1;  // slices fastest: the three slices of a row band share D rows in L2
  const long long ps = O.plane_stride;
  const float* Dp = O.d + (long long)(s - 1) * ps + (long long)y * O.pitch;
  const float* Dc = O.d + (long long)s * ps + (long long)y * O.pitch;
  const float* Dn = O.d + (long long)(s + 1) * ps + (long long)y * O.pitch;
  uint32_t* mrow = O.masks + ((long long)(s - 1) * O.h + y) * O.words;
  const float thr = prm.threshold;
  const bool row_ok = y >= 1 && y < O.h - 1;
  const int w = O.w;
  const int span_end = O.words * 32;

  __shared__ uint16_t s_q[kMarkWarps][kMarkSpan];
  __shared__ uint32_t s_mask[kMarkWarps][kMarkSpan / 32];
  uint16_t* q = s_q[warp];
  uint32_t* wm = s_mask[warp];
  uint32_t cnt = 0;

  float4 cur[2], nxt[2];
  if (row_ok) mark_load_span(Dc, 0, lane, w, cur);
  for (int xb = 0; xb < span_end; xb += kMarkSpan) {
    if (row_ok && xb + kMarkSpan < span_end) mark_load_span(Dc, xb + kMarkSpan, lane, w, nxt);
    uint32_t m = 0;  // bit 4h + i: pixel xb + 128 h + 4 lane + i
    if (row_ok) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const float e[4] = {cur[h].x, cur[h].y, cur[h].z, cur[h].w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int x = xb + h * 128 + 4 * lane + i;
          // the reference's first rejection is |v| <= threshold (NaN continues)
          if (x >= 1 && x < w - 1 && !(fabsf(e[i]) <= thr)) m |= 1u << (4 * h + i);
        }
      }
    }
    uint32_t word_bits = 0;  // lane < 8: mask word (xb >> 5) + lane
    if (__any_sync(0xffffffffu, m != 0)) {
      const uint32_t c = __popc(m);
      uint32_t incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      const int total = (int)__shfl_sync(0xffffffffu, incl, 31);
      uint32_t pos = incl - c;
#pragma unroll
      for (int b = 0; b < 8; ++b)
        if (m & (1u << b)) q[pos++] = (uint16_t)((b >> 2) * 128 + 4 * lane + (b & 3));
      if (lane < 8) wm[lane] = 0;
      __syncwarp();
      for (int i = lane; i < total; i += 32) {
        const int off = q[i];
        if (accept_pixel(Dp, Dc, Dn, O.pitch, xb + off, thr)) atomicOr(&wm[off >> 5], 1u << (off & 31));
      }
      __syncwarp();
      if (lane < 8) word_bits = wm[lane];
      __syncwarp();
    }
    if (lane < 8) {
      const int word = (xb >> 5) + lane;
      if (word < O.words) {
        mrow[word] = word_bits;
        cnt += __popc(word_bits);
      }
    }
    cur[0] = nxt[0];
    cur[1] = nxt[1];
  }
  cnt = __reduce_add_sync(0xffffffffu, cnt);
  if (lane == 0) P.row_counts[O.row_base + (s - 1) * O.h + y] = cnt;
}

// Block-wide exclusive scan helper for 1024 threads; returns the block total.
__device__ __forceinline__ uint32_t block_exclusive_scan_1024(uint32_t v, uint32_t& excl, uint32_t* s_warp) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) s_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t w = s_warp[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    s_warp[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  const uint32_t warp_prefix = wid > 0 ? s_warp[wid - 1] : 0u;
  excl = warp_prefix + x - v;
  const uint32_t total = s_warp[31];
  __syncthreads();
  return total;
}

// One block (1024 threads) per image: exclusive offsets over all (octave, slice, row).
__global__ void __launch_bounds__(1024) row_scan_kernel(const ImagePlan* __restrict__ plans, uint32_t kp_cap,
                                                        uint32_t* err) {
  const ImagePlan& P = plans[blockIdx.x];
  __shared__ uint32_t s_warp[32];
  uint32_t carry = 0;
  for (int base = 0; base < P.total_rows; base += 1024) {
    const int i = base + threadIdx.x;
    const uint32_t v = i < P.total_rows ? P.row_counts[i] : 0u;
    uint32_t excl;
    const uint32_t tot = block_exclusive_scan_1024(v, excl, s_warp);
    if (i < P.total_rows) P.row_offsets[i] = carry + excl;
    carry += tot;
  }
  if (threadIdx.x == 0) {
    *P.kp_count = carry;
    if (carry > kp_cap) atomicOr(err, kErrKeypointCapacity);
  }
}

// Grid (ceil(scales*max_h / 8), images), 256 threads: one warp per (slice, row).
__global__ void __launch_bounds__(256) extrema_emit_kernel(const ImagePlan* __restrict__ plans, int octave,
                                                           ExtremaParams prm, uint32_t kp_cap) {
  const ImagePlan& P = plans[blockIdx.y];
  if (octave >= P.n_oct) return;
  const OctaveDev& O = P.oct[octave];
  const int lane = threadIdx.x & 31;
  const int row_local = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (row_local >= prm.scales * O.h) return;
  const int r = O.row_base + row_local;
  if (P.row_counts[r] == 0) return;
  const int s = 1 + row_local / O.h;
  const int y = row_local - (s - 1) * O.h;
  uint32_t pos_base = P.row_offsets[r];
  const long long ps = O.plane_stride;
  const float* Dp = O.d + (long long)(s - 1) * ps + (long long)y * O.pitch;
  const float* Dc = O.d + (long long)s * ps + (long long)y * O.pitch;
  const float* Dn = O.d + (long long)(s + 1) * ps + (long long)y * O.pitch;
  const uint32_t* mrow = O.masks + ((long long)(s - 1) * O.h + y) * O.words;
  const float mult = O.scale_factor;
  const float eff = prm.eff_scale[octave][s];
  for (int wb = 0; wb < O.words; wb += 32) {
    uint32_t word = (wb + lane < O.words) ? mrow[wb + lane] : 0u;
    const uint32_t c = __popc(word);
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    uint32_t pos = pos_base + incl - c;
    while (word) {
      const int b = __ffs(word) - 1;
      word &= word - 1;
      const int x = (wb + lane) * 32 + b;
      float dx, dy, ds, interp;
      refine3d(Dp, Dc, Dn, O.pitch, x, dx, dy, ds, interp);
      if (pos < kp_cap) {
        psift_keypoint kp;
        const float kds = (float)pow((double)prm.k, (double)ds);
        const float refined_scale = eff * kds;
        float lf = roundf((float)s + ds);
        lf = lf < 1.0f ? 1.0f : (lf > (float)prm.scales ? (float)prm.scales : lf);
        kp.x = ((float)x + dx) * mult;
        kp.y = ((float)y + dy) * mult;
        kp.scale = fmaxf(refined_scale, 0.25f * kBaseSigma);
        kp.response = interp;
        kp.octave = (uint32_t)octave;
        kp.layer = (uint32_t)lf;
        P.kps[pos] = kp;
      }
      ++pos;
    }
    pos_base += __shfl_sync(0xffffffffu, incl, 31);
  }
}

// Stable top-K by |response| (descending; ties keep keypoint order), then
// sorted -- exactly `sort_by(|b| b.response.abs() ...)` + `truncate(K)`.
// One block (1024 threads) per image.  The K selected sort keys live in
// dynamic shared memory (next_pow2(K) x 8 bytes).
__global__ void __launch_bounds__(1024) select_topk_kernel(const ImagePlan* __restrict__ plans, uint32_t kp_cap,
                                                           uint32_t max_features, uint32_t* err) {
  const ImagePlan& P = plans[blockIdx.x];
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_hist[256];
  __shared__ uint32_t s_sel[4];
  extern __shared__ unsigned long long s_keys[];
  const uint32_t found = *P.kp_count;
  const uint32_t N = found < kp_cap ? found : kp_cap;
  const uint32_t K = max_features;
  if (K == 0 || N <= K) {
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) P.sel[i] = P.kps[i];
    if (threadIdx.x == 0) *P.sel_count = N;
    return;
  }
  // Radix select of the K-th largest key, most significant byte first.
  uint32_t prefix = 0, mask = 0, need = K;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
      const uint32_t key = __float_as_uint(fabsf(P.kps[i].response));
      if ((key & mask) == prefix) atomicAdd(&s_hist[(key >> shift) & 0xFF], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t above = 0;
      int b = 255;
      for (; b > 0; --b) {
        if (above + s_hist[b] >= need) break;
        above += s_hist[b];
      }
      s_sel[0] = (uint32_t)b;
      s_sel[1] = need - above;
    }
    __syncthreads();
    prefix |= s_sel[0] << shift;
    mask |= 0xFFu << shift;
    need = s_sel[1];
    __syncthreads();
  }
  const uint32_t T = prefix;  // K-th largest key; take all keys > T and the first `need` keys == T
  uint32_t n_sel = 0, n_eq = 0;
  for (uint32_t base = 0; base < N; base += 1024) {
    const uint32_t i = base + threadIdx.x;
    uint32_t key = 0;
    if (i < N) key = __float_as_uint(fabsf(P.kps[i].response));
    const uint32_t is_eq = (i < N && key == T) ? 1u : 0u;
    uint32_t eq_excl;
    const uint32_t eq_tot = block_exclusive_scan_1024(is_eq, eq_excl, s_warp);
    const uint32_t take = (i < N) && (key > T || (is_eq && n_eq + eq_excl < need)) ? 1u : 0u;
    uint32_t sel_excl;
    const uint32_t sel_tot = block_exclusive_scan_1024(take, sel_excl, s_warp);
    if (take) {
      const uint32_t slot = n_sel + sel_excl;
      if (slot < K) s_keys[slot] = ((unsigned long long)(~key) << 32) | (unsigned long long)i;
    }
    n_eq += eq_tot;
    n_sel += sel_tot;
  }
  uint32_t n2 = 1;
  while (n2 < K) n2 <<= 1;
  for (uint32_t i = K + threadIdx.x; i < n2; i += blockDim.x) s_keys[i] = ~0ull;
  if (threadIdx.x == 0 && n_sel != K) atomicOr(err, kErrSortCapacity);
  __syncthreads();
  // Bitonic sort ascending on (~|response|, index).
  for (uint32_t k = 2; k <= n2; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) {
        const uint32_t ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long a = s_keys[i], b = s_keys[ixj];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            s_keys[i] = b;
            s_keys[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  for (uint32_t i = threadIdx.x; i < K; i += blockDim.x) P.sel[i] = P.kps[(uint32_t)(s_keys[i] & 0xFFFFFFFFu)];
  if (threadIdx.x == 0) *P.sel_count = K;
}

cudaError_t launch_extrema_mark(const ImagePlan* plans, int n, int octave, int max_h, const ExtremaParams& prm,
                                cudaStream_t st) {
  dim3 grid(prm.scales, (max_h + kMarkWarps - 1) / kMarkWarps, n);
  extrema_mark_kernel<<<grid, kMarkWarps * 32, 0, st>>>(plans, octave, prm);
  return cudaGetLastError();
}

cudaError_t launch_row_scan(const ImagePlan* plans, int n, uint32_t kp_cap, uint32_t* err, cudaStream_t st) {
  row_scan_kernel<<<n, 1024, 0, st>>>(plans, kp_cap, err);
  return cudaGetLastError();
}

cudaError_t launch_extrema_emit(const ImagePlan* plans, int n, int octave, int max_h, const ExtremaParams& prm,
                                uint32_t kp_cap, cudaStream_t st) {
  dim3 grid((prm.scales * max_h + 7) / 8, n);
  extrema_emit_kernel<<<grid, 256, 0, st>>>(plans, octave, prm, kp_cap);
  return cudaGetLastError();
}

cudaError_t launch_select_topk(const ImagePlan* plans, int n, uint32_t kp_cap, uint32_t max_features, uint32_t* err,
                               cudaStream_t st) {
  uint32_t n2 = 1;
  while (n2 < max_features) n2 <<= 1;
  const size_t smem = max_features ? n2 * sizeof(unsigned long long) : 0;
  cudaError_t e = ensure_smem_attr((const void*)select_topk_kernel, 128 * 1024);
  if (e != cudaSuccess) return e;
  select_topk_kernel<<<n, 1024, smem, st>>>(plans, kp_cap, max_features, err);
  return cudaGetLastError();
}

}  // namespace psift
