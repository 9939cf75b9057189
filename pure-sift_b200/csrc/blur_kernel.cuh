// K1-K3: octave base (luma->f32, 2x bilinear upsample, initial blur), separable
// Gaussian blur chain + DoG, and the 2x decimation that seeds the next octave.
//
// Reference: gaussian_blur (src/pipeline.rs:314-425), upsample_2x_bilinear
// (:455-483), downsample_2x (:429-449), build_scale_space_pyramid_with_options
// (:550-638), luma_to_array2 (:957-966).
//
// Bit-exactness: every output equals the reference's f32 result.  Each tap is a
// rounded multiply followed by a rounded add (the library is built with
// -fmad=false, and the reference never contracts), taps are accumulated from 0
// in the reference's order (k = 0..2r), borders clamp the source index exactly
// like `(x + k).saturating_sub(r).min(w - 1)`, and the kernel weights are
// computed on the host with the reference's f32 formula.  The single-rounding
// mode (template flag FUSED, selected per context) issues each tap as one fused
// multiply-add instead: same order and borders, one rounding per tap.
//
// Tiling: one CTA of 256 threads produces a 64x64 output tile.
//   1. Staging: the (64+2R) x (64+2R') input tile (R' = R rounded up to 4, so
//      every interior chunk is one aligned 128-bit load) goes to shared memory
//      with rows interleaved in pairs: element (2p+i, c) sits at s_in[p][c].i.
//   2. Horizontal pass: each thread makes 4 (or 8) adjacent outputs of a row
//      pair.  A 128-bit shared load yields two {row 2p, row 2p+1} pairs, so each
//      tap is one packed multiply and one packed rounded add (see mul_add2_rn) for
//      two outputs, with the scalar operations' rounding per component.
//   3. Vertical pass: each thread makes a column pair x rows of outputs from the
//      row-major intermediate, again with packed f32x2 operations.
//   Taps are consumed in input order; for every output that is k = 0..2R, the
//   reference's order.  The row-pair stride is 2 (mod 16) float2 and lanes are
//   assigned so that the 8 lanes of a quarter-warp hit 8 distinct 16-byte bank
//   groups.  Outputs: G_s and D_{s-1} = G_s - G_{s-1} as 64-bit stores; level
//   `scales` also writes the even/even samples that form the next octave's base
//   (fused downsample_2x).  Images alternate direction between consecutive
//   levels (blockIdx.z reversed on odd levels) so the planes written last by
//   one launch, still in L2, are read first by the next.
#pragma once
#include "detect_plan.cuh"
#include "psift_internal.cuh"

namespace psift {

constexpr int kBlurThreads = 256;
constexpr int kTmpStride = kTileW + 8;  // floats per intermediate row
constexpr int kStageBatch = 4;          // staging units per thread with loads in flight
// Level-blur variants (outputs per thread: columns x rows), chosen per radius by
// the context's tuning table (psift_ctx_autotune): 0 = 4 x 8, 1 = 8 x 8, 2 = 4 x 4.
constexpr int kPrefetchWaves = 1;       // level blur: L2 prefetch distance in resident-CTA waves

// Per-launch parameters (passed by value).  The tile work list of a launch over
// images of different sizes is a separate parameter of the tiled kernels only,
// so the equal-size launches keep the small parameter block and a kernel body
// without the work-list lookup (measured: 2 % of the 8-image 1080p step).
struct Taps2 {
  float2 w[kMaxTaps];  // {w_k, w_k}
  float2 one;          // {1, 1}: the multiplier of the packed add (see mul_add2_rn)
};

// Linear tile `lin` of a work list (reversed when zrev) -> image and tile; false
// past the end.
__device__ __forceinline__ bool tile_of(const TileMap& tm, long long lin, int zrev, int& z, int& bx, int& by) {
  const int total = tm.prefix[tm.n];
  if (lin >= total) return false;
  const int l = zrev ? total - 1 - (int)lin : (int)lin;
  int lo = 0, hi = tm.n - 1;  // the last z with prefix[z] <= l
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tm.prefix[mid] <= l) lo = mid;
    else hi = mid - 1;
  }
  z = lo;
  const int local = l - tm.prefix[z];
  by = local / tm.tiles_x[z];
  bx = local - by * tm.tiles_x[z];
  return true;
}

enum BlurMode : int { MODE_LEVEL = 0, MODE_INIT_F32 = 1, MODE_INIT_U8 = 2, MODE_INIT_F32_UP = 3, MODE_INIT_U8_UP = 4 };

template <int R, int TH = kTileH>
struct BlurGeom {
  static constexpr int RP = (R + 3) / 4 * 4;                          // column halo, whole float4 chunks
  static constexpr int IN_W = kTileW + 2 * RP;                        // staged columns
  static constexpr int IN_H = TH + 2 * R;                             // staged rows (even)
  static constexpr int IN_PAIRS = IN_H / 2;
  static constexpr int IN_S = IN_W + (((2 - IN_W) % 16) + 16) % 16;   // float2 per row pair, = 2 (mod 16)
  static constexpr int C4 = IN_W / 4;
  static constexpr int SMEM_BYTES = IN_PAIRS * IN_S * 8 + IN_H * kTmpStride * 4;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// acc + v * w per component with two roundings, never fused into one.
// The packed multiply and add are each exact IEEE operations, but ptxas
// contracts a single-use mul.rn.f32x2 feeding add.rn.f32x2 into a packed FMA
// (even with explicit .rn and --fmad false), which changes about 6% of the
// results by an ulp.  The add is therefore issued as fma.rn(p, one, acc) with
// `one` = {1, 1} taken from the kernel parameters: p * 1 is exact, so this is
// round(p + acc), and the compiler cannot fold a multiplier it does not know.
// The bit-exact blur and pyramid tests guard this.
__device__ __forceinline__ float2 mul_add2_rn(float2 acc, float2 v, float2 w, float2 one) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pv, pw, po, pp;\n\t"
      "mov.b64 pa, {%2, %3};\n\t"
      "mov.b64 pv, {%4, %5};\n\t"
      "mov.b64 pw, {%6, %7};\n\t"
      "mov.b64 po, {%8, %9};\n\t"
      "mul.rn.f32x2 pp, pv, pw;\n\t"
      "fma.rn.f32x2 pa, pp, po, pa;\n\t"
      "mov.b64 {%0, %1}, pa;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(acc.x), "f"(acc.y), "f"(v.x), "f"(v.y), "f"(w.x), "f"(w.y), "f"(one.x), "f"(one.y));
  return r;
}

// One tap, acc + v * w per component: two roundings (the reference's), or one
// (FUSED: fma.rn.f32x2, the single-rounding blur mode).
template <bool FUSED>
__device__ __forceinline__ float2 tap2(float2 acc, float2 v, float2 w, float2 one) {
  if constexpr (FUSED) {
    float2 r;
    asm("{\n\t.reg .b64 pa, pv, pw;\n\t"
        "mov.b64 pa, {%2, %3};\n\t"
        "mov.b64 pv, {%4, %5};\n\t"
        "mov.b64 pw, {%6, %7};\n\t"
        "fma.rn.f32x2 pa, pv, pw, pa;\n\t"
        "mov.b64 {%0, %1}, pa;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(acc.x), "f"(acc.y), "f"(v.x), "f"(v.y), "f"(w.x), "f"(w.y));
    return r;
  } else {
    return mul_add2_rn(acc, v, w, one);
  }
}

// Source sample at octave-0 coordinates (gy, gx), already clamped to the plane.
template <int MODE>
__device__ __forceinline__ float fetch_src(const ImagePlan& P, const OctaveDev& O, int level_src, int gy, int gx) {
  if constexpr (MODE == MODE_LEVEL) {
    return O.g[(long long)level_src * O.plane_stride + (long long)gy * O.pitch + gx];
  } else if constexpr (MODE == MODE_INIT_F32) {
    return ((const float*)P.src)[(long long)gy * P.src_stride + gx];
  } else if constexpr (MODE == MODE_INIT_U8) {
    const float inv255 = 1.0f / 255.0f;
    return (float)((const uint8_t*)P.src)[(long long)gy * P.src_stride + gx] * inv255;
  } else {
    // upsample_2x_bilinear: 0.25 * (r0[x0] + r0[x1] + r1[x0] + r1[x1]) with x1/y1 = +parity, clamped.
    const int y0 = gy >> 1, x0 = gx >> 1;
    const int y1 = min(y0 + (gy & 1), P.src_h - 1);
    const int x1 = min(x0 + (gx & 1), P.src_w - 1);
    float a, b, c, d;
    if constexpr (MODE == MODE_INIT_F32_UP) {
      const float* s = (const float*)P.src;
      a = s[(long long)y0 * P.src_stride + x0];
      b = s[(long long)y0 * P.src_stride + x1];
      c = s[(long long)y1 * P.src_stride + x0];
      d = s[(long long)y1 * P.src_stride + x1];
    } else {
      const uint8_t* s = (const uint8_t*)P.src;
      const float inv255 = 1.0f / 255.0f;
      a = (float)s[(long long)y0 * P.src_stride + x0] * inv255;
      b = (float)s[(long long)y0 * P.src_stride + x1] * inv255;
      c = (float)s[(long long)y1 * P.src_stride + x0] * inv255;
      d = (float)s[(long long)y1 * P.src_stride + x1] * inv255;
    }
    return 0.25f * (((a + b) + c) + d);
  }
}

// L2 prefetch of the input rows of the tile `ahead` CTAs further in launch order
// (one thread per staged row).  With `ahead` = the CTAs resident at once, that
// tile is staged about one tile-time later and its loads hit L2, so the HBM
// reads of the next wave overlap the arithmetic of this one.
template <int R, bool TILED, int TH>
__device__ __forceinline__ void prefetch_ahead_rows(const ImagePlan* __restrict__ plans, int octave, int level,
                                                    int zrev, int ahead, const TileMap* tm) {
  using Gm = BlurGeom<R, TH>;
  int z, bx, by;
  if constexpr (TILED) {
    if (!tile_of(*tm, (long long)blockIdx.x + ahead, zrev, z, bx, by)) return;
  } else {
    const long long nxy = (long long)gridDim.x * gridDim.y;
    const long long lin = blockIdx.x + (long long)gridDim.x * blockIdx.y + nxy * blockIdx.z + ahead;
    if (lin >= nxy * gridDim.z) return;
    const int bz = (int)(lin / nxy);
    const int rem = (int)(lin - (long long)bz * nxy);
    by = rem / (int)gridDim.x;
    bx = rem - by * (int)gridDim.x;
    z = zrev ? (int)gridDim.z - 1 - bz : bz;
  }
  const ImagePlan& P = plans[z];
  if (octave >= P.n_oct) return;
  const OctaveDev& O = P.oct[octave];
  const int tx0 = bx * kTileW, ty0 = by * TH;
  if (tx0 >= O.w || ty0 >= O.h) return;
  // rows clamped like the staging; columns [c0, c1) are 16-byte aligned and end
  // inside the row pitch (a multiple of 32 floats)
  const int gy = clampi(ty0 - R + (int)threadIdx.x, 0, O.h - 1);
  const int c0 = max(tx0 - Gm::RP, 0);
  const int c1 = min(tx0 + kTileW + Gm::RP, (O.w + 3) & ~3);
  const float* row = O.g + (long long)(level - 1) * O.plane_stride + (long long)gy * O.pitch + c0;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(row), "r"((c1 - c0) * 4) : "memory");
}

// One blur level for every image of the batch (blockIdx.z = image, reversed when
// zrev; or, over images of different sizes, one CTA per existing tile of the
// launch's tile work list, the list reversed when zrev).
//   MODE_LEVEL: G[s] = blur(G[s-1]); D[s-1] = G[s] - G[s-1]; level `down_level` also
//               writes the next octave's G[0] (even rows/columns).
//   MODE_INIT_*: G[0] of octave 0 from the input image.
// TH x 64 tiles (TH = 64, or 128 for the tall variant), NT threads.
template <int R, int HC, int RV, int MODE, bool FUSED, bool TILED, int TH = kTileH, int NT = kBlurThreads>
__device__ __forceinline__ void blur_level_body(const ImagePlan* __restrict__ plans, int octave, int level,
                                                int down_level, int zrev, int pf_ahead, const Taps2& taps,
                                                const TileMap* tm) {
  using Gm = BlurGeom<R, TH>;
  static_assert(!TILED || TH == kTileH, "tile work lists are in 64 x 64 tiles");
  if constexpr (MODE == MODE_LEVEL) {
    if (pf_ahead > 0 && threadIdx.x < Gm::IN_H)
      prefetch_ahead_rows<R, TILED, TH>(plans, octave, level, zrev, pf_ahead, tm);
  }
  static_assert(HC == 4 || HC == 8, "horizontal outputs per thread");
  // The Gaussian taps are bit-symmetric (gaussian_kernel_1d evaluates the same
  // x^2 for +-x and normalises both by one sum), so w[k] = w[2R - k] exactly and
  // R + 1 register pairs hold them all for the whole kernel.
  float2 wv[R + 1];
#pragma unroll
  for (int k = 0; k <= R; ++k) wv[k] = taps.w[k];
  const float2 one = taps.one;
  static_assert(RV % 2 == 0 && TH % (RV * (NT / 32)) == 0, "vertical rows per thread");
  int z, bx, by;
  if constexpr (TILED) {
    if (!tile_of(*tm, blockIdx.x, zrev, z, bx, by)) return;
  } else {
    z = zrev ? (int)gridDim.z - 1 - (int)blockIdx.z : (int)blockIdx.z;
    bx = blockIdx.x;
    by = blockIdx.y;
  }
  const ImagePlan& P = plans[z];
  if (octave >= P.n_oct) return;
  const OctaveDev& O = P.oct[octave];
  const int h = O.h, w = O.w;
  const int tx0 = bx * kTileW, ty0 = by * TH;
  if (tx0 >= w || ty0 >= h) return;

  extern __shared__ float4 smem4[];
  float2* s_in = reinterpret_cast<float2*>(smem4);                               // [IN_PAIRS][IN_S]
  float* s_tmp = reinterpret_cast<float*>(s_in + Gm::IN_PAIRS * Gm::IN_S);       // [IN_H][kTmpStride]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  // 0. Upsampling base modes: the half-resolution source tile the staged tile
  //    needs (at most 32 + R + 2 rows, 32 + R' + 2 columns) goes to shared memory
  //    once, already in f32 (u8 * (1/255), luma_to_array2), in the intermediate
  //    buffer that the horizontal pass only fills later.
  constexpr bool kUp = MODE == MODE_INIT_F32_UP || MODE == MODE_INIT_U8_UP;
  constexpr int SRC_H = (Gm::IN_H + 1) / 2 + 2, SRC_W = (Gm::IN_W + 1) / 2 + 2;
  static_assert(!kUp || SRC_H * SRC_W <= Gm::IN_H * kTmpStride, "source tile fits the intermediate buffer");
  int sy_lo = 0, sx_lo = 0;
  if constexpr (kUp) {
    sy_lo = clampi(ty0 - R, 0, h - 1) >> 1;
    sx_lo = clampi(tx0 - Gm::RP, 0, w - 1) >> 1;
    const int sh = min(SRC_H, P.src_h - sy_lo), sw = min(SRC_W, P.src_w - sx_lo);
    // every load of the thread is issued before the first store
    constexpr int kSrcIter = (SRC_H * SRC_W + NT - 1) / NT;
    float v[kSrcIter];
#pragma unroll
    for (int q = 0; q < kSrcIter; ++q) {
      const int i = threadIdx.x + q * NT;
      const int r = i / SRC_W, c = i - r * SRC_W;
      v[q] = 0.0f;
      if (i < SRC_H * SRC_W && r < sh && c < sw) {
        const long long off = (long long)(sy_lo + r) * P.src_stride + (sx_lo + c);
        if constexpr (MODE == MODE_INIT_U8_UP) {
          const float inv255 = 1.0f / 255.0f;
          v[q] = (float)__ldg((const uint8_t*)P.src + off) * inv255;
        } else {
          v[q] = __ldg((const float*)P.src + off);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kSrcIter; ++q) {
      const int i = threadIdx.x + q * NT;
      if (i < SRC_H * SRC_W) s_tmp[i] = v[q];
    }
    __syncthreads();
  }
  // upsample_2x_bilinear sample at octave-0 (gy, gx), both already clamped
  auto up_sample = [&](int gy, int gx) -> float {
    const int y0 = gy >> 1, x0 = gx >> 1;
    const int y1 = min(y0 + (gy & 1), P.src_h - 1);
    const int x1 = min(x0 + (gx & 1), P.src_w - 1);
    const float* r0 = s_tmp + (y0 - sy_lo) * SRC_W - sx_lo;
    const float* r1 = s_tmp + (y1 - sy_lo) * SRC_W - sx_lo;
    const float a = r0[x0], b = r0[x1], c = r1[x0], d = r1[x1];
    return 0.25f * (((a + b) + c) + d);
  };

  // 1. Stage the clamped input tile, rows interleaved in pairs.  A thread's units
  //    are taken kStageBatch at a time with all their loads issued before any
  //    shared-memory store, so several loads are in flight per thread.
  const float* src_plane = O.g + (long long)(level - 1) * O.plane_stride;  // MODE_LEVEL only
  auto load_unit = [&](int u, float4& a, float4& b) {
    const int rp = u / Gm::C4, c4 = u - rp * Gm::C4;
    const int gy0 = clampi(ty0 - R + 2 * rp, 0, h - 1);
    const int gy1 = clampi(ty0 - R + 2 * rp + 1, 0, h - 1);
    const int gx = tx0 - Gm::RP + 4 * c4;
    if constexpr (kUp && R % 2 == 0) {
      // Interior unit of an even-radius base: rows (gy0, gy0 + 1) = (2 y0, 2 y0 + 1)
      // and columns 2 xs .. 2 xs + 3 need source rows y0, y1 and columns xs ..
      // xs + 2 only; each output is the same four-term sum as up_sample.
      if (gy0 == ty0 - R + 2 * rp && gy0 + 1 < h && gx >= 0 && gx + 3 < w) {
        const int y0 = gy0 >> 1, y1 = min(y0 + 1, P.src_h - 1), xs = gx >> 1;
        const int x2 = min(xs + 2, P.src_w - 1);
        const float* r0 = s_tmp + (y0 - sy_lo) * SRC_W - sx_lo;
        const float* r1 = s_tmp + (y1 - sy_lo) * SRC_W - sx_lo;
        const float p0 = r0[xs], p1 = r0[xs + 1], p2 = r0[x2];
        const float q0 = r1[xs], q1 = r1[xs + 1], q2 = r1[x2];
        a = make_float4(0.25f * (((p0 + p0) + p0) + p0), 0.25f * (((p0 + p1) + p0) + p1),
                        0.25f * (((p1 + p1) + p1) + p1), 0.25f * (((p1 + p2) + p1) + p2));
        b = make_float4(0.25f * (((p0 + p0) + q0) + q0), 0.25f * (((p0 + p1) + q0) + q1),
                        0.25f * (((p1 + p1) + q1) + q1), 0.25f * (((p1 + p2) + q1) + q2));
        return;
      }
    }
    if (MODE == MODE_LEVEL && gx >= 0 && gx + 3 < w) {
      a = __ldg(reinterpret_cast<const float4*>(src_plane + (long long)gy0 * O.pitch + gx));
      b = __ldg(reinterpret_cast<const float4*>(src_plane + (long long)gy1 * O.pitch + gx));
    } else {
      float av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int cx = clampi(gx + i, 0, w - 1);
        if constexpr (kUp) {
          av[i] = up_sample(gy0, cx);
          bv[i] = up_sample(gy1, cx);
        } else {
          av[i] = fetch_src<MODE>(P, O, level - 1, gy0, cx);
          bv[i] = fetch_src<MODE>(P, O, level - 1, gy1, cx);
        }
      }
      a = make_float4(av[0], av[1], av[2], av[3]);
      b = make_float4(bv[0], bv[1], bv[2], bv[3]);
    }
  };
  constexpr int kUnits = Gm::IN_PAIRS * Gm::C4;
  for (int u0 = threadIdx.x; u0 < kUnits; u0 += kStageBatch * NT) {
    float4 a[kStageBatch], b[kStageBatch];
#pragma unroll
    for (int q = 0; q < kStageBatch; ++q)
      if (u0 + q * NT < kUnits) load_unit(u0 + q * NT, a[q], b[q]);
#pragma unroll
    for (int q = 0; q < kStageBatch; ++q) {
      const int u = u0 + q * NT;
      if (u < kUnits) {
        const int rp = u / Gm::C4, c4 = u - rp * Gm::C4;
        float4* d = reinterpret_cast<float4*>(s_in + rp * Gm::IN_S + 4 * c4);
        d[0] = make_float4(a[q].x, b[q].x, a[q].y, b[q].y);
        d[1] = make_float4(a[q].z, b[q].z, a[q].w, b[q].w);
      }
    }
  }
  __syncthreads();

  // 2. Horizontal pass over row pairs.
  {
    constexpr int QX = 16 / HC, QR = 8 / QX;  // a quarter-warp covers QR row pairs x QX column groups
    constexpr int OFF = Gm::RP - R, SH = OFF & 1;
    constexpr int NP = (HC + 2 * R + SH + 1) / 2;  // 128-bit loads per row pair
    const int qi = lane & 7;
    const int rsub = qi / QX;
    const int xg = (lane >> 3) * QX + (qi % QX);
    for (int rp = warp * QR + rsub; rp < Gm::IN_PAIRS; rp += (NT / 32) * QR) {
      const float4* src = reinterpret_cast<const float4*>(s_in + rp * Gm::IN_S + HC * xg + OFF - SH);
      float2 acc[HC];
#pragma unroll
      for (int j = 0; j < HC; ++j) acc[j] = make_float2(0.0f, 0.0f);
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        const float4 t = src[q];
        const float2 p0 = make_float2(t.x, t.y), p1 = make_float2(t.z, t.w);
#pragma unroll
        for (int j = 0; j < HC; ++j) {
          const int k0 = 2 * q - SH - j;
          if (k0 >= 0 && k0 <= 2 * R) acc[j] = tap2<FUSED>(acc[j], p0, wv[(k0) <= R ? (k0) : 2 * R - (k0)], one);
          if (k0 + 1 >= 0 && k0 + 1 <= 2 * R) acc[j] = tap2<FUSED>(acc[j], p1, wv[(k0 + 1) <= R ? (k0 + 1) : 2 * R - (k0 + 1)], one);
        }
      }
      float* t0 = s_tmp + (2 * rp) * kTmpStride + HC * xg;
#pragma unroll
      for (int jj = 0; jj < HC / 4; ++jj) {
        *reinterpret_cast<float4*>(t0 + 4 * jj) =
            make_float4(acc[4 * jj].x, acc[4 * jj + 1].x, acc[4 * jj + 2].x, acc[4 * jj + 3].x);
        *reinterpret_cast<float4*>(t0 + kTmpStride + 4 * jj) =
            make_float4(acc[4 * jj].y, acc[4 * jj + 1].y, acc[4 * jj + 2].y, acc[4 * jj + 3].y);
      }
    }
  }
  __syncthreads();

  // 3. Vertical pass: a column pair x RV rows per thread.
  const long long gbase = (long long)level * O.plane_stride;
  float* gout = O.g + gbase;
  float* dout = (MODE == MODE_LEVEL) ? O.d + (long long)(level - 1) * O.plane_stride : nullptr;
  const bool do_down = (MODE == MODE_LEVEL) && level == down_level && octave + 1 < P.n_oct;
  const int x = 2 * lane;
  const int gx = tx0 + x;
  for (int yb = warp * RV; yb < TH; yb += RV * (NT / 32)) {
    if (ty0 + yb >= h) break;
    float2 acc[RV];
#pragma unroll
    for (int j = 0; j < RV; ++j) acc[j] = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int i = 0; i < RV + 2 * R; ++i) {
      const float2 v = *reinterpret_cast<const float2*>(s_tmp + (yb + i) * kTmpStride + x);
#pragma unroll
      for (int j = 0; j < RV; ++j) {
        const int k = i - j;
        if (k >= 0 && k <= 2 * R) acc[j] = tap2<FUSED>(acc[j], v, wv[(k) <= R ? (k) : 2 * R - (k)], one);
      }
    }
    if (gx >= w) continue;
    const bool pair_ok = gx + 1 < w;
    constexpr int NPR = ((R & 1) + RV + 1) / 2;
    float4 prevp[MODE == MODE_LEVEL ? NPR : 1];
    if constexpr (MODE == MODE_LEVEL) {
      const float4* pp = reinterpret_cast<const float4*>(s_in + ((R >> 1) + (yb >> 1)) * Gm::IN_S + Gm::RP + x);
#pragma unroll
      for (int p = 0; p < NPR; ++p) prevp[p] = pp[p * (Gm::IN_S / 2)];
    }
#pragma unroll
    for (int j = 0; j < RV; ++j) {
      const int gy = ty0 + yb + j;
      if (gy >= h) break;
      float* grow = gout + (long long)gy * O.pitch + gx;
      if (pair_ok) {
        *reinterpret_cast<float2*>(grow) = acc[j];
      } else {
        grow[0] = acc[j].x;
      }
      if constexpr (MODE == MODE_LEVEL) {
        const int idx = (R & 1) + j;
        const float4 pv = prevp[idx >> 1];
        const float px = (idx & 1) ? pv.y : pv.x;
        const float py = (idx & 1) ? pv.w : pv.z;
        float* drow = dout + (long long)gy * O.pitch + gx;
        const float dx0 = __fsub_rn(acc[j].x, px);
        if (pair_ok) {
          __stcs(reinterpret_cast<float2*>(drow), make_float2(dx0, __fsub_rn(acc[j].y, py)));
        } else {
          __stcs(drow, dx0);
        }
        if (do_down && !(gy & 1)) {
          const OctaveDev& N = P.oct[octave + 1];
          const int dy = gy >> 1, dxn = gx >> 1;
          if (dy < N.h && dxn < N.w) N.g[(long long)dy * N.pitch + dxn] = acc[j].x;
        }
      }
    }
  }
}

template <int R, int HC, int RV, int MODE, bool FUSED, int TH = kTileH, int NT = kBlurThreads>
__global__ void __launch_bounds__(NT, NT == kBlurThreads ? 4 : 2)
    blur_level_kernel(const ImagePlan* __restrict__ plans, int octave, int level, int down_level, int zrev,
                      int pf_ahead, const __grid_constant__ Taps2 taps) {
  blur_level_body<R, HC, RV, MODE, FUSED, false, TH, NT>(plans, octave, level, down_level, zrev, pf_ahead, taps,
                                                         nullptr);
}

// The same over a tile work list (one CTA per listed tile).
template <int R, int HC, int RV, int MODE, bool FUSED>
__global__ void __launch_bounds__(kBlurThreads, 4)
    blur_level_tiled_kernel(const ImagePlan* __restrict__ plans, int octave, int level, int down_level, int zrev,
                            int pf_ahead, const __grid_constant__ Taps2 taps, const __grid_constant__ TileMap tiles) {
  blur_level_body<R, HC, RV, MODE, FUSED, true>(plans, octave, level, down_level, zrev, pf_ahead, taps, &tiles);
}

template <int R, int HC, int RV, int MODE, bool FUSED, bool TILED, int TH = kTileH, int NT = kBlurThreads>
static cudaError_t launch_blur_r(const ImagePlan* plans, int n_images, int octave, int level, int down_level,
                                 int zrev, const Taps2& taps, const TileMap* tiles, int max_h, int max_w,
                                 cudaStream_t st) {
  using Gm = BlurGeom<R, TH>;
  const size_t smem = Gm::SMEM_BYTES;
  const void* fn = TILED ? (const void*)blur_level_tiled_kernel<R, HC, RV, MODE, FUSED>
                         : (const void*)blur_level_kernel<R, HC, RV, MODE, FUSED, TH, NT>;
  cudaError_t e = ensure_smem_attr(fn, smem);
  if (e != cudaSuccess) return e;
  int pf_ahead = 0;
  if (MODE == MODE_LEVEL) {
    e = resident_ctas(fn, NT, smem, &pf_ahead);
    if (e != cudaSuccess) return e;
    pf_ahead *= kPrefetchWaves;
  }
  if constexpr (TILED) {
    const dim3 grid((unsigned)tiles->prefix[tiles->n], 1, 1);
    blur_level_tiled_kernel<R, HC, RV, MODE, FUSED><<<grid, kBlurThreads, smem, st>>>(plans, octave, level,
                                                                                down_level, zrev, pf_ahead, taps,
                                                                                *tiles);
  } else {
    const dim3 grid((max_w + kTileW - 1) / kTileW, (max_h + TH - 1) / TH, n_images);
    blur_level_kernel<R, HC, RV, MODE, FUSED, TH, NT><<<grid, NT, smem, st>>>(plans, octave, level, down_level,
                                                                            zrev, pf_ahead, taps);
  }
  return cudaGetLastError();
}

template <int MODE, int HC, int RV, bool FUSED, bool TILED = false, int TH = kTileH, int NT = kBlurThreads>
static cudaError_t launch_blur_mode(int radius, const ImagePlan* plans, int n, int octave, int level, int down_level,
                                    int zrev, const Taps2& taps, const TileMap* tiles, int max_h, int max_w,
                                    cudaStream_t st) {
  switch (radius) {
#define PSIFT_R(RR)                                                                                              \
  case RR:                                                                                                       \
    return launch_blur_r<RR, HC, RV, MODE, FUSED, TILED, TH, NT>(plans, n, octave, level, down_level, zrev, taps, \
                                                                 tiles, max_h, max_w, st);
    PSIFT_R(1) PSIFT_R(2) PSIFT_R(3) PSIFT_R(4) PSIFT_R(5) PSIFT_R(6) PSIFT_R(7) PSIFT_R(8)
    PSIFT_R(9) PSIFT_R(10) PSIFT_R(11) PSIFT_R(12) PSIFT_R(13) PSIFT_R(14) PSIFT_R(15)
#undef PSIFT_R
    default:
      return cudaErrorInvalidValue;
  }
}

// The single-rounding level and base blurs (pyramid_fused.cu): level blur with
// 4 x 8 outputs per thread, and the four octave-base modes.
cudaError_t launch_blur_fused(int mode, int radius, const ImagePlan* plans, int n, int octave, int level,
                              int down_level, int zrev, const Taps2& taps, int max_h, int max_w, cudaStream_t st);
// Launches over a tile work list (images of different sizes; pyramid_tiled.cu):
// the level blur with 4 x 8 outputs per thread and the four octave-base modes,
// either rounding.
cudaError_t launch_blur_tiled(int mode, bool fused, int radius, const ImagePlan* plans, int n, int octave, int level,
                              int down_level, int zrev, const Taps2& taps, const TileMap& tiles, cudaStream_t st);

}  // namespace psift
