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
// computed on the host with the reference's f32 formula.
//
// Tiling: one CTA produces a 64x64 output tile.  The (64+2r)^2 input tile is
// staged in shared memory, the horizontal pass writes (64+2r)x64 partial rows to
// shared memory (4 outputs per thread from 128-bit loads), the vertical pass
// produces 4 rows per thread and writes G_s and D_{s-1} = G_s - G_{s-1} with
// coalesced 128-byte row segments.  Level `scales` also writes the even/even
// samples that form the next octave's base (fused downsample_2x).
#include "detect_plan.cuh"
#include "psift_internal.cuh"

namespace psift {

constexpr int kTileW = 64;
constexpr int kTileH = 64;
constexpr int kBlurThreads = 256;

struct Taps {
  float w[kMaxTaps];
};

enum BlurMode : int { MODE_LEVEL = 0, MODE_INIT_F32 = 1, MODE_INIT_U8 = 2, MODE_INIT_F32_UP = 3, MODE_INIT_U8_UP = 4 };

template <int R>
struct BlurGeom {
  static constexpr int NV = ((2 * R + 4) + 3) / 4 * 4;           // floats per thread in the H pass
  static constexpr int IN_H = kTileH + 2 * R;
  static constexpr int IN_WL = kTileW + 2 * R;                    // columns actually needed
  static constexpr int IN_P0 = (IN_WL + 3) / 4 * 4;
  static constexpr int IN_P = IN_P0 > (kTileW - 4 + NV) ? IN_P0 : (kTileW - 4 + NV);
  static constexpr int SMEM_FLOATS = IN_H * IN_P + IN_H * kTileW;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

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

// One blur level for every image of the batch (blockIdx.z = image).
//   MODE_LEVEL: G[s] = blur(G[s-1]); D[s-1] = G[s] - G[s-1]; level `down_level` also
//               writes the next octave's G[0] (even rows/columns).
//   MODE_INIT_*: G[0] of octave 0 from the input image.
template <int R, int MODE>
__global__ void __launch_bounds__(kBlurThreads) blur_level_kernel(const ImagePlan* __restrict__ plans, int octave,
                                                                   int level, int down_level, Taps taps) {
  using Gm = BlurGeom<R>;
  const ImagePlan& P = plans[blockIdx.z];
  if (octave >= P.n_oct) return;
  const OctaveDev& O = P.oct[octave];
  const int h = O.h, w = O.w;
  const int tx0 = blockIdx.x * kTileW, ty0 = blockIdx.y * kTileH;
  if (tx0 >= w || ty0 >= h) return;

  extern __shared__ float4 smem4[];
  float* s_in = reinterpret_cast<float*>(smem4);
  float* s_tmp = s_in + Gm::IN_H * Gm::IN_P;

  // Stage the clamped input tile.
  for (int i = threadIdx.x; i < Gm::IN_H * Gm::IN_P; i += kBlurThreads) {
    const int r = i / Gm::IN_P, c = i - r * Gm::IN_P;
    float v = 0.0f;
    if (c < Gm::IN_WL) {
      const int gy = clampi(ty0 - R + r, 0, h - 1);
      const int gx = clampi(tx0 - R + c, 0, w - 1);
      v = fetch_src<MODE>(P, O, level - 1, gy, gx);
    }
    s_in[i] = v;
  }
  __syncthreads();

  // Horizontal pass: 16 threads per row, 4 consecutive outputs each.
  {
    const int x0 = (threadIdx.x & 15) * 4;
    for (int row = threadIdx.x >> 4; row < Gm::IN_H; row += kBlurThreads / 16) {
      float v[Gm::NV];
      const float4* src4 = reinterpret_cast<const float4*>(s_in + row * Gm::IN_P + x0);
#pragma unroll
      for (int q = 0; q < Gm::NV / 4; ++q) {
        const float4 t = src4[q];
        v[4 * q + 0] = t.x;
        v[4 * q + 1] = t.y;
        v[4 * q + 2] = t.z;
        v[4 * q + 3] = t.w;
      }
      float o[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        float acc = 0.0f;
#pragma unroll
        for (int k = 0; k <= 2 * R; ++k) acc = __fadd_rn(acc, __fmul_rn(v[j + k], taps.w[k]));
        o[j] = acc;
      }
      *reinterpret_cast<float4*>(s_tmp + row * kTileW + x0) = make_float4(o[0], o[1], o[2], o[3]);
    }
  }
  __syncthreads();

  // Vertical pass (row AXPY order of the reference): 4 consecutive rows per thread.
  const long long gbase = (long long)level * O.plane_stride;
  float* gout = O.g + gbase;
  float* dout = (MODE == MODE_LEVEL) ? O.d + (long long)(level - 1) * O.plane_stride : nullptr;
  const bool do_down = (MODE == MODE_LEVEL) && level == down_level && octave + 1 < P.n_oct;
  for (int item = threadIdx.x; item < kTileW * (kTileH / 4); item += kBlurThreads) {
    const int x = item % kTileW;
    const int y0 = (item / kTileW) * 4;
    const int gx = tx0 + x;
    float v[4 + 2 * R];
#pragma unroll
    for (int i = 0; i < 4 + 2 * R; ++i) v[i] = s_tmp[(y0 + i) * kTileW + x];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float acc = 0.0f;
#pragma unroll
      for (int k = 0; k <= 2 * R; ++k) acc = __fadd_rn(acc, __fmul_rn(v[j + k], taps.w[k]));
      const int gy = ty0 + y0 + j;
      if (gy < h && gx < w) {
        gout[(long long)gy * O.pitch + gx] = acc;
        if constexpr (MODE == MODE_LEVEL) {
          const float prev = s_in[(R + y0 + j) * Gm::IN_P + (R + x)];
          dout[(long long)gy * O.pitch + gx] = __fsub_rn(acc, prev);
          if (do_down && !(gy & 1) && !(gx & 1)) {
            const OctaveDev& N = P.oct[octave + 1];
            const int dy = gy >> 1, dx = gx >> 1;
            if (dy < N.h && dx < N.w) N.g[(long long)dy * N.pitch + dx] = acc;
          }
        }
      }
    }
  }
}

template <int R, int MODE>
static cudaError_t launch_blur_r(const ImagePlan* plans, int n_images, int octave, int level, int down_level,
                                 const Taps& taps, int max_h, int max_w, cudaStream_t st) {
  using Gm = BlurGeom<R>;
  const size_t smem = sizeof(float) * Gm::SMEM_FLOATS;
  cudaError_t e = ensure_smem_attr((const void*)blur_level_kernel<R, MODE>, smem);
  if (e != cudaSuccess) return e;
  dim3 grid((max_w + kTileW - 1) / kTileW, (max_h + kTileH - 1) / kTileH, n_images);
  blur_level_kernel<R, MODE><<<grid, kBlurThreads, smem, st>>>(plans, octave, level, down_level, taps);
  return cudaGetLastError();
}

template <int MODE>
static cudaError_t launch_blur_mode(int radius, const ImagePlan* plans, int n, int octave, int level, int down_level,
                                    const Taps& taps, int max_h, int max_w, cudaStream_t st) {
  switch (radius) {
#define PSIFT_R(RR) \
  case RR: return launch_blur_r<RR, MODE>(plans, n, octave, level, down_level, taps, max_h, max_w, st);
    PSIFT_R(1) PSIFT_R(2) PSIFT_R(3) PSIFT_R(4) PSIFT_R(5) PSIFT_R(6) PSIFT_R(7) PSIFT_R(8)
    PSIFT_R(9) PSIFT_R(10) PSIFT_R(11) PSIFT_R(12) PSIFT_R(13) PSIFT_R(14) PSIFT_R(15)
#undef PSIFT_R
    default:
      return cudaErrorInvalidValue;
  }
}

// Host entry: mode 0 = level blur (octave, level >= 1); modes 1..4 = octave-0 base.
cudaError_t launch_blur(int mode, const float* taps_host, int radius, const ImagePlan* plans, int n, int octave,
                        int level, int down_level, int max_h, int max_w, cudaStream_t st) {
  Taps t;
  for (int i = 0; i < kMaxTaps; ++i) t.w[i] = i <= 2 * radius ? taps_host[i] : 0.0f;
  switch (mode) {
    case MODE_LEVEL: return launch_blur_mode<MODE_LEVEL>(radius, plans, n, octave, level, down_level, t, max_h, max_w, st);
    case MODE_INIT_F32: return launch_blur_mode<MODE_INIT_F32>(radius, plans, n, octave, level, down_level, t, max_h, max_w, st);
    case MODE_INIT_U8: return launch_blur_mode<MODE_INIT_U8>(radius, plans, n, octave, level, down_level, t, max_h, max_w, st);
    case MODE_INIT_F32_UP: return launch_blur_mode<MODE_INIT_F32_UP>(radius, plans, n, octave, level, down_level, t, max_h, max_w, st);
    case MODE_INIT_U8_UP: return launch_blur_mode<MODE_INIT_U8_UP>(radius, plans, n, octave, level, down_level, t, max_h, max_w, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace psift
