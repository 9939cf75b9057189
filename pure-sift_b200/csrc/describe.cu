// K5/K6: canonical orientations (36-bin histogram, circular smoothing, >=80%
// secondary peaks) and 128-D SIFT / RootSIFT descriptors.
//
// Reference: OctaveGradientPlanes::from_gaussian (src/pipeline.rs:1158-1203),
// resolve_octave_and_layer (:1206-1227), compute_keypoint_orientations
// (:1233-1347), compute_128d_descriptor (:1352-1480), to_rootsift_descriptor
// (:1012-1019), compute_sift_descriptors_from_pyramid_with_kind (:1482-1577),
// and the feature truncation of extract_sift_features_with_kind (:1653-1656).
//
// Gradients are computed on the fly from the keypoint's Gaussian level (the
// reference materialises magnitude/angle planes for every used level; the values
// per pixel are the same expression).  One warp handles one keypoint (orientation)
// or one keypoint's orientations in turn (descriptor).  Histogram accumulation is
// deterministic: each lane owns a private column of a bin-major shared-memory
// histogram ([bin][lane], conflict-free), and columns are summed in lane order.
// Per-bin sums therefore differ from the reference's raster-order sums only by
// f32 rounding; all selection logic (peak tests, sort, truncation) and the final
// normalisation repeat the reference's sequence exactly.
#include <algorithm>

#include "detect_plan.cuh"
#include "psift_internal.cuh"

namespace psift {

constexpr int kOriBins = 36;
constexpr uint32_t kKpPerLaunchRow = 4096;  // keypoints per image covered by one grid row
constexpr int kOriWarps = 8;
constexpr int kDescWarps = 4;

// rem_euclid(v, 2pi) for |v| <= 2pi (fmod is exact: identity below 2pi).
__device__ __forceinline__ float rem_2pi(float v, float two_pi) {
  float r = fabsf(v) < two_pi ? v : fmodf(v, two_pi);
  return r < 0.0f ? r + two_pi : r;
}

struct OctKp {
  float x, y, scale;
  int o, l;
};

// resolve_octave_and_layer (src/pipeline.rs:1206-1227) + the octave-local keypoint (:1516-1526).
__device__ __forceinline__ OctKp to_octave(const ImagePlan& P, const psift_keypoint& kp) {
  OctKp r;
  const int n_oct = P.n_oct;
  if (kp.layer > 0) {
    r.o = min((int)kp.octave, n_oct - 1);
  } else {
    const float ratio = fmaxf(kp.scale / kBaseSigma, 1.0f);
    const float f = floorf(log2f(ratio));
    r.o = f <= 0.0f ? 0 : min((int)f, n_oct - 1);
  }
  r.l = 0;  // resolved by resolve_layer
  const float sf = P.oct[r.o].scale_factor;
  const float inv = 1.0f / sf;
  r.x = kp.x * inv;
  r.y = kp.y * inv;
  r.scale = fmaxf(kp.scale * inv, 0.5f * kBaseSigma);
  return r;
}

__device__ __forceinline__ int resolve_layer(const psift_keypoint& kp, int o, int scales) {
  const int g_len = scales + 3;
  if (kp.layer > 0) return min((int)kp.layer, g_len - 1);
  const int searchable = max(g_len - 3, 1);
  const float oct_mult = (float)(1u << o);
  const float local_sigma = fmaxf(kp.scale / (kBaseSigma * oct_mult), 1.0f);
  const float v = roundf(log2f(local_sigma) * (float)searchable);
  const int l = v <= 0.0f ? 0 : (int)v;
  const int hi = max(g_len - 2, 1);
  return l < 1 ? 1 : (l > hi ? hi : l);
}

// Gradient magnitude and angle at interior pixel (x, y) of plane g.
__device__ __forceinline__ void grad_at(const float* __restrict__ g, long long pitch, int x, int y, float& mag,
                                        float& ang, float two_pi) {
  const float* rc = g + (long long)y * pitch;
  const float dx = rc[x + 1] - rc[x - 1];
  const float dy = rc[pitch + x] - rc[x - pitch];
  mag = sqrtf(dx * dx + dy * dy);
  float a = atan2f(dy, dx);
  ang = a < 0.0f ? a + two_pi : a;  // rem_euclid(2pi) of a value in [-pi, pi]
}

// The descriptor's per-pixel gradient, with cheaper functions than grad_at's:
// every value it feeds enters the histogram through weights that move
// continuously with it (trilinear bins, Gaussian weight, magnitude), so a few
// ulps of difference change a descriptor by about 1e-6 relative, against the
// 1e-4 tolerance of the descriptor rows.  The orientations keep grad_at (their
// peak selection decides how many features a keypoint gets).
//  - magnitude: q * rsqrt(q) (q = dx^2 + dy^2 > 0), about 3 ulp;
//  - angle: atan2 by octant reduction to t = min / max in [0, 1] (approximate
//    quotient) and atan(t) = t * P(t^2), P of degree 7 fitted for this library
//    (iteratively reweighted least squares toward minimax on Chebyshev nodes of
//    [0, 1]; largest error 1.3e-7 rad when evaluated in f32 with fused steps).
__device__ __forceinline__ float atan2_fast(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
  const float t = mx > 0.0f ? __fdividef(mn, mx) : 0.0f;
  const float s = __fmul_rn(t, t);
  float p = -0.004054563120007515f;
  p = __fmaf_rn(p, s, 0.021862944588065147f);
  p = __fmaf_rn(p, s, -0.0559123158454895f);
  p = __fmaf_rn(p, s, 0.0964219719171524f);
  p = __fmaf_rn(p, s, -0.1390862911939621f);
  p = __fmaf_rn(p, s, 0.19946566224098206f);
  p = __fmaf_rn(p, s, -0.33329859375953674f);
  p = __fmaf_rn(p, s, 0.9999993443489075f);
  float a = __fmul_rn(p, t);
  if (ay > ax) a = __fsub_rn(0.5f * kPiF, a);
  if (x < 0.0f) a = __fsub_rn(kPiF, a);
  return y < 0.0f ? -a : a;
}

__device__ __forceinline__ void grad_at_desc(const float* __restrict__ g, long long pitch, int x, int y, float& mag,
                                             float& ang, float two_pi) {
  const float* rc = g + (long long)y * pitch;
  const float dx = rc[x + 1] - rc[x - 1];
  const float dy = rc[pitch + x] - rc[x - pitch];
  const float q = dx * dx + dy * dy;
  mag = q > 0.0f ? q * rsqrtf(q) : 0.0f;
  const float a = atan2_fast(dy, dx);
  ang = a < 0.0f ? a + two_pi : a;
}

// Orientations of selected keypoint i of image P, one warp (hist, bins: the
// warp's shared-memory histograms).
__device__ void orient_one(const ImagePlan& P, const DescribeParams& prm, uint32_t i, float (*hist)[32],
                           float* bins_w) {
  const int lane = threadIdx.x & 31;
  const psift_keypoint kp = P.sel[i];
  OctKp ok = to_octave(P, kp);
  ok.l = resolve_layer(kp, ok.o, prm.scales);
  const OctaveDev& O = P.oct[ok.o];
  const float* g = O.g + (long long)ok.l * O.plane_stride;
  const float two_pi = 2.0f * kPiF;

  for (int b = 0; b < kOriBins; ++b) hist[b][lane] = 0.0f;

  const float sigma_ori = fmaxf(1.5f * ok.scale, 1.0f);
  const float two_sigma_sq = 2.0f * sigma_ori * sigma_ori;
  int radius = (int)ceilf(3.0f * sigma_ori);
  radius = radius < 2 ? 2 : radius;
  const int cx = (int)roundf(ok.x), cy = (int)roundf(ok.y);
  const float bin_scale = (float)kOriBins / two_pi;
  const int y_min = max(cy - radius, 1);
  const int y_max = max(min(cy + radius, O.h - 2), 1);
  const int x_min = max(cx - radius, 1);
  const int x_max = max(min(cx + radius, O.w - 2), 1);
  const float r_sq_max = (float)(radius * radius);
  const int wx = x_max - x_min + 1;
  const int n = (y_max >= y_min && x_max >= x_min) ? (y_max - y_min + 1) * wx : 0;
  const bool planes_ok = O.h >= 3 && O.w >= 3;
  // lane's pixel t = lane, lane + 32, ...: its (row, column) stepped by 32 pixels
  // (q32 whole rows plus r32 columns, at most one wrap) instead of a division each
  const int q32 = wx > 0 ? 32 / wx : 0, r32 = wx > 0 ? 32 - q32 * wx : 0;
  int yy = wx > 0 ? y_min + lane / wx : 0, xx = wx > 0 ? x_min + lane % wx : 0;
  for (int t = lane; planes_ok && t < n; t += 32, xx += r32, yy += q32) {
    if (xx > x_max) {
      xx -= wx;
      ++yy;
    }
    const float dy = (float)(yy - cy), dx = (float)(xx - cx);
    const float r_sq = dx * dx + dy * dy;
    if (r_sq > r_sq_max) continue;
    float m, ang;
    grad_at(g, O.pitch, xx, yy, m, ang, two_pi);
    if (m <= 1e-7f) continue;
    const float weight = expf(-r_sq / two_sigma_sq);
    const int bin = ((int)floorf(ang * bin_scale)) % kOriBins;
    hist[bin][lane] += m * weight;
  }
  __syncwarp();
  for (int b = lane; b < kOriBins; b += 32) {
    float s = 0.0f;
    for (int j = 0; j < 32; ++j) s += hist[b][j];
    bins_w[b] = s;
  }
  __syncwarp();
  if (lane != 0) return;
  const float* hb = bins_w;
  float sm[kOriBins];
  for (int b = 0; b < kOriBins; ++b) {
    const float prev = hb[(b + kOriBins - 1) % kOriBins];
    const float cur = hb[b];
    const float next = hb[(b + 1) % kOriBins];
    sm[b] = (prev + cur + next) * (1.0f / 3.0f);
  }
  int best_bin = 0;
  float best_val = sm[0];
  for (int b = 1; b < kOriBins; ++b)
    if (sm[b] > best_val) {
      best_val = sm[b];
      best_bin = b;
    }
  float* out = P.oris + (size_t)i * 4;
  if (best_val <= 1e-7f) {
    out[0] = 0.0f;
    P.ori_count[i] = 1;
    return;
  }
  const float split = 0.80f * best_val;
  // Peaks sorted by (value desc, bin asc), at most 4: insertion into a 4-slot list.
  int pk_bin[4];
  float pk_val[4];
  int np = 0;
  for (int b = 0; b < kOriBins; ++b) {
    const float v = sm[b];
    if (v < split) continue;
    const float l = sm[(b + kOriBins - 1) % kOriBins];
    const float r = sm[(b + 1) % kOriBins];
    if (v > l && v >= r) {
      // bins arrive ascending: a new peak goes after every peak with value >= v
      int pos = np;
      while (pos > 0 && pk_val[pos - 1] < v) --pos;
      if (pos < 4) {
        const int last = np < 4 ? np : 3;
        for (int q = last; q > pos; --q) {
          pk_bin[q] = pk_bin[q - 1];
          pk_val[q] = pk_val[q - 1];
        }
        pk_bin[pos] = b;
        pk_val[pos] = v;
        if (np < 4) ++np;
      }
    }
  }
  if (np == 0) {
    pk_bin[0] = best_bin;
    pk_val[0] = best_val;
    np = 1;
  }
  for (int q = 0; q < np; ++q) {
    const int bin = pk_bin[q];
    const float val = pk_val[q];
    const float l = sm[(bin + kOriBins - 1) % kOriBins];
    const float r = sm[(bin + 1) % kOriBins];
    const float denom = l - 2.0f * val + r;
    float off = fabsf(denom) > 1e-6f ? 0.5f * (l - r) / denom : 0.0f;
    off = off < -0.5f ? -0.5f : (off > 0.5f ? 0.5f : off);
    const float th = (((float)bin + 0.5f) + off) * (two_pi / (float)kOriBins);
    out[q] = rem_2pi(th, two_pi);
  }
  P.ori_count[i] = (uint32_t)np;
}

// Grid (min(keypoint capacity, kKpPerLaunchRow) / 8, images): warp w of CTA b
// takes selected keypoints 8b + w, then a grid-width further on, of image
// blockIdx.y.  Capacity-sized rows keep one warp per keypoint when the cap is
// small; an uncapped batch (capacity 2^18) gets bounded rows instead of
// millions of empty CTAs.
__global__ void __launch_bounds__(kOriWarps * 32) orientation_kernel(const ImagePlan* __restrict__ plans,
                                                                     DescribeParams prm) {
  __shared__ float s_hist[kOriWarps][kOriBins][32];
  __shared__ float s_bins[kOriWarps][kOriBins];
  const int warp = threadIdx.x >> 5;
  const ImagePlan& P = plans[blockIdx.y];
  const uint32_t cnt = *P.sel_count, stride = gridDim.x * kOriWarps;
  for (uint32_t i = blockIdx.x * kOriWarps + warp; i < cnt; i += stride) {
    orient_one(P, prm, i, s_hist[warp], s_bins[warp]);
    __syncwarp();
  }
}

// Exclusive offsets of orientations per keypoint; feature count = min(total, cap).
__global__ void __launch_bounds__(1024) feature_scan_kernel(const ImagePlan* __restrict__ plans, uint32_t max_features) {
  const ImagePlan& P = plans[blockIdx.x];
  __shared__ uint32_t s_warp[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t n = *P.sel_count;
  uint32_t carry = 0;
  for (uint32_t base = 0; base < n; base += 1024) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < n ? P.ori_count[i] : 0u;
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
      s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t pre = wid > 0 ? s_warp[wid - 1] : 0u;
    if (i < n) P.feat_offsets[i] = carry + pre + x - v;
    carry += s_warp[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    uint32_t f = carry;
    if (max_features > 0 && f > max_features) f = max_features;
    if (f > P.feat_cap) f = P.feat_cap;
    *P.feat_count = f;
    *P.feat_total = carry;
    if (P.out_count) *P.out_count = f;
  }
}

// Grid (sel_cap, images), 128 threads: one CTA (4 warps) per keypoint, one
// descriptor per orientation.
//
// The window is cut into chunks of 256 pixels dealt round-robin to the 4 warps.
// Per chunk, phase 1: each lane tests 8 pixels against the rotated 4x4-cell
// square (the reference's r_bin/c_bin test; about half of the window passes) and
// the passing ones are compacted into the warp's queue; phase 2: full lanes take
// queued pixels for the gradient, weight and trilinear binning.  Histograms: 16
// private columns per warp ([bin][16], 8 KB); the pixels of lanes l and l + 16 both
// go to column l, in two fixed rounds in which the two lanes split each pixel's
// cells (see the binning loop).  Bin b's value is the sum over (warp, column) in a
// fixed order, so the result does not depend on scheduling (deterministic).
constexpr int kDescChunk = 256;
constexpr int kHistCols = 16;
constexpr int kDescWarpSmem = kDescLen * kHistCols * 4 + kDescChunk * 4;
constexpr int kDescSmem = kDescWarps * kDescWarpSmem + 64;

// Block-wide sum of one value per thread (128 threads), same result on every thread.
__device__ __forceinline__ float block_sum128(float v, float* s_red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
  __syncthreads();
  return (s_red[0] + s_red[1]) + (s_red[2] + s_red[3]);
}

// Descriptors of selected keypoint i of image P, the whole CTA (base_smem: the
// CTA's dynamic shared memory); returns with the CTA converged.
__device__ void describe_one(const ImagePlan& P, const DescribeParams& prm, uint32_t i, char* base_smem) {
  static_assert(kDescWarps == 4, "one thread per bin in the final sums");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t fcount = *P.feat_count;
  const uint32_t f0 = P.feat_offsets[i];
  if (f0 >= fcount) return;
  char* wbase = base_smem + warp * kDescWarpSmem;
  float (*hist)[kHistCols] = reinterpret_cast<float (*)[kHistCols]>(wbase);
  uint32_t* queue = reinterpret_cast<uint32_t*>(wbase + kDescLen * kHistCols * 4);
  float* s_red = reinterpret_cast<float*>(base_smem + kDescWarps * kDescWarpSmem);

  const psift_keypoint kp = P.sel[i];
  OctKp ok = to_octave(P, kp);
  ok.l = resolve_layer(kp, ok.o, prm.scales);
  const OctaveDev& O = P.oct[ok.o];
  const float* g = O.g + (long long)ok.l * O.plane_stride;
  const float two_pi = 2.0f * kPiF;
  const uint32_t nori = P.ori_count[i];

  const float hist_width = fmaxf(3.0f * ok.scale, 1.5f);
  const float inv_hw = 1.0f / hist_width;
  const float exp_scale = -1.0f / (2.0f * 2.0f * 2.0f);
  const float sqrt2 = 1.41421356237309504880f;
  int max_radius = (int)ceilf(hist_width * sqrt2 * (4.0f + 1.0f) * 0.5f);
  max_radius = max_radius < 4 ? 4 : max_radius;
  const int cx = (int)roundf(ok.x), cy = (int)roundf(ok.y);
  const int y_min = max(cy - max_radius, 1);
  const int y_max = max(min(cy + max_radius, O.h - 2), 1);
  const int x_min = max(cx - max_radius, 1);
  const int x_max = max(min(cx + max_radius, O.w - 2), 1);
  const int wx = x_max - x_min + 1;
  const int n = (y_max >= y_min && x_max >= x_min && O.h >= 3 && O.w >= 3) ? (y_max - y_min + 1) * wx : 0;
  const float bin_per_rad = 8.0f / two_pi;
  const int col = lane & (kHistCols - 1), half = lane >> 4;
  const int q32 = wx > 0 ? 32 / wx : 0, r32 = wx > 0 ? 32 - q32 * wx : 0;

  for (uint32_t q = 0; q < nori; ++q) {
    const uint32_t f = f0 + q;
    if (f >= fcount) break;
    const float theta = P.oris[(size_t)i * 4 + q];
#pragma unroll 4
    for (int b = lane; b < kDescLen * kHistCols / 4; b += 32)
      reinterpret_cast<float4*>(&hist[0][0])[b] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float cos_t = cosf(theta), sin_t = sinf(theta);
    // phase 1's square test only: the rotated bins by two fused steps each (a pixel
    // that this moves across the square's edge has a weight of about 0 there: its
    // trilinear share in the edge cell is the distance past the edge)
    const float ci = cos_t * inv_hw, si = sin_t * inv_hw;
    for (int base = warp * kDescChunk; base < n; base += kDescWarps * kDescChunk) {
      // Phase 1: rotated-square test for 8 pixels per lane.
      const int t0 = base + lane;
      int yy = y_min + t0 / wx, xx = x_min + t0 % wx;
      uint32_t m = 0, packed[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int t = t0 + 32 * k;
        const int py = yy, px = xx;
        packed[k] = ((uint32_t)py << 16) | (uint32_t)px;
        // advance 32 pixels: q32 whole rows plus r32 columns, at most one wrap
        xx += r32;
        yy += q32;
        if (xx > x_max) {
          xx -= wx;
          ++yy;
        }
        if (t < n) {
          const float dy = (float)py - ok.y;
          const float dx = (float)px - ok.x;
          const float r_bin = __fmaf_rn(dx, ci, __fmaf_rn(dy, si, 1.5f));
          const float c_bin = __fmaf_rn(-dx, si, __fmaf_rn(dy, ci, 1.5f));
          if (!(r_bin <= -1.0f || r_bin >= 4.0f || c_bin <= -1.0f || c_bin >= 4.0f)) m |= 1u << k;
        }
      }
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
      for (int k = 0; k < 8; ++k)
        if (m & (1u << k)) queue[pos++] = packed[k];
      __syncwarp();
      // Phase 2: queued pixels, all lanes busy.
      for (int e0 = 0; e0 < total; e0 += 32) {
        const int e = e0 + lane;
        bool live = false;
        int r0 = 0, c0 = 0, o0 = 0;
        float dr = 0.0f, dc = 0.0f, dof = 0.0f, wm = 0.0f;
        if (e < total) {
          const uint32_t pk = queue[e];
          const int py = (int)(pk >> 16), px = (int)(pk & 0xFFFFu);
          const float dy = (float)py - ok.y;
          const float dx = (float)px - ok.x;
          const float r_rot = (dx * cos_t + dy * sin_t) * inv_hw;
          const float c_rot = (-dx * sin_t + dy * cos_t) * inv_hw;
          const float r_bin = r_rot + 4.0f * 0.5f - 0.5f;
          const float c_bin = c_rot + 4.0f * 0.5f - 0.5f;
          float mg, ang;
          grad_at_desc(g, O.pitch, px, py, mg, ang, two_pi);
          if (mg > 1e-7f) {
            live = true;
            const float w_gauss = __expf((r_rot * r_rot + c_rot * c_rot) * exp_scale);  // about 3 ulp here
            wm = mg * w_gauss;
            const float rel = rem_2pi(ang - theta, two_pi);
            const float o_bin = rel * bin_per_rad;
            r0 = (int)floorf(r_bin);
            c0 = (int)floorf(c_bin);
            o0 = (int)floorf(o_bin);
            dr = r_bin - (float)r0;
            dc = c_bin - (float)c0;
            dof = o_bin - (float)o0;
          }
        }
        // Branch-free trilinear update: a cell outside the 4x4 grid (or a lane
        // without a pixel) adds +0 to a valid bin.  Every contribution is >= +0
        // and every bin starts at +0, so adding +0 leaves the bin unchanged and
        // the real contributions keep their order.
        if (!live) wm = 0.0f;
        // Two rounds, all lanes busy: round 0 bins the pixels of lanes 0-15, round 1
        // those of lanes 16-31.  In each, the pixel's own lane adds its row-bin r0
        // cells and the partner lane (lane ^ 16) its row-bin r0 + 1 cells, both into
        // the pixel's column (lane & 15).  The two lanes' cells are never the same
        // address in one instruction: their row bins differ, and a row bin outside
        // the grid (+0 added) is sent to row 3 (own lane) or row 0 (partner), which
        // the other lane's valid row cannot be.
        const int pr0 = __shfl_xor_sync(0xffffffffu, r0, 16), pc0 = __shfl_xor_sync(0xffffffffu, c0, 16);
        const int po0 = __shfl_xor_sync(0xffffffffu, o0, 16);
        const float pdr = __shfl_xor_sync(0xffffffffu, dr, 16), pdc = __shfl_xor_sync(0xffffffffu, dc, 16);
        const float pdof = __shfl_xor_sync(0xffffffffu, dof, 16), pwm = __shfl_xor_sync(0xffffffffu, wm, 16);
#pragma unroll
        for (int rnd = 0; rnd < 2; ++rnd) {
          const bool own = half == rnd;
          const int R0 = own ? r0 : pr0, C0 = own ? c0 : pc0, O0 = own ? o0 : po0;
          const float DR = own ? dr : pdr, DC = own ? dc : pdc, DOF = own ? dof : pdof, WM = own ? wm : pwm;
          const int ir = own ? 0 : 1;
          const int rb = R0 + ir;
          const bool vr = (unsigned)rb < 4u;
          const float wr = vr ? (ir == 0 ? 1.0f - DR : DR) : 0.0f;
          const int row = vr ? rb : (own ? 3 : 0);
#pragma unroll
          for (int ic = 0; ic <= 1; ++ic) {
            const int cb = C0 + ic;
            const bool vc = (unsigned)cb < 4u;
            const float wc = vc ? (ic == 0 ? 1.0f - DC : DC) : 0.0f;
            float* cell = &hist[(row * 4 + (vc ? cb : 0)) * 8][col];
            const float wrc = WM * wr * wc;
            cell[(O0 & 7) * kHistCols] += wrc * (1.0f - DOF);
            cell[((O0 + 1) & 7) * kHistCols] += wrc * DOF;
          }
          __syncwarp();
        }
      }
    }
    __syncthreads();
    // Bin b = threadIdx.x: sum over warps 0..3, each over its 16 columns read
    // rotated by b >> 1 (the 32 lanes of a warp hit 32 distinct banks).
    const int b = threadIdx.x;
    float d = 0.0f;
#pragma unroll
    for (int w4 = 0; w4 < kDescWarps; ++w4) {
      const float* row = reinterpret_cast<const float*>(base_smem + w4 * kDescWarpSmem) + b * kHistCols;
      float acc = 0.0f;
#pragma unroll
      for (int j = 0; j < kHistCols; ++j) acc += row[(j + (b >> 1)) & (kHistCols - 1)];
      d += acc;
    }
    // L2 -> clamp 0.2 -> L2 (src/pipeline.rs:1462-1477); block sums in a fixed order.
    float n1 = sqrtf(block_sum128(d * d, s_red));
    if (n1 > 1e-7f) {
      d = fminf(d * (1.0f / n1), 0.2f);
      const float n2 = sqrtf(block_sum128(d * d, s_red));
      if (n2 > 1e-7f) d *= 1.0f / n2;
    }
    if (prm.descriptor_kind == 1) {
      // to_rootsift_descriptor (src/pipeline.rs:1012-1019)
      const float l1 = block_sum128(fmaxf(d, 0.0f), s_red);
      if (l1 > 1e-7f) d = sqrtf(fmaxf(d, 0.0f) * (1.0f / l1));
    }
    P.fdesc[(size_t)f * kDescLen + b] = d;
    if (threadIdx.x == 0) {
      P.fx[f] = kp.x;
      P.fy[f] = kp.y;
      P.fscale[f] = kp.scale;
      P.fresp[f] = kp.response;
      P.fori[f] = theta;
    }
    __syncthreads();  // histograms are cleared for the next orientation
  }
}

// Grid (min(keypoint capacity, kKpPerLaunchRow), images): CTA b takes selected
// keypoint b, then a grid-width further on, of image blockIdx.y (see
// orientation_kernel); every output slot is fixed by the keypoint's feature
// offset, so the result does not depend on which CTA computes it.
__global__ void __launch_bounds__(kDescWarps * 32) descriptor_kernel(const ImagePlan* __restrict__ plans,
                                                                     DescribeParams prm) {
  extern __shared__ float4 s_dyn4[];
  char* base_smem = reinterpret_cast<char*>(s_dyn4);
  const ImagePlan& P = plans[blockIdx.y];
  const uint32_t cnt = *P.sel_count;
  for (uint32_t i = blockIdx.x; i < cnt; i += gridDim.x) describe_one(P, prm, i, base_smem);
}

cudaError_t launch_orientation(const ImagePlan* plans, int n, uint32_t sel_cap, const DescribeParams& prm,
                               cudaStream_t st) {
  const uint32_t row = std::min<uint32_t>(std::max<uint32_t>(sel_cap, 1), kKpPerLaunchRow);
  dim3 grid((row + kOriWarps - 1) / kOriWarps, n);
  orientation_kernel<<<grid, kOriWarps * 32, 0, st>>>(plans, prm);
  return cudaGetLastError();
}

cudaError_t launch_feature_scan(const ImagePlan* plans, int n, uint32_t max_features, cudaStream_t st) {
  feature_scan_kernel<<<n, 1024, 0, st>>>(plans, max_features);
  return cudaGetLastError();
}

cudaError_t launch_descriptor(const ImagePlan* plans, int n, uint32_t sel_cap, const DescribeParams& prm,
                              cudaStream_t st) {
  const size_t smem = kDescSmem;
  cudaError_t e = ensure_smem_attr((const void*)descriptor_kernel, smem);
  if (e != cudaSuccess) return e;
  dim3 grid(std::min<uint32_t>(std::max<uint32_t>(sel_cap, 1), kKpPerLaunchRow), n);
  descriptor_kernel<<<grid, kDescWarps * 32, smem, st>>>(plans, prm);
  return cudaGetLastError();
}

}  // namespace psift
