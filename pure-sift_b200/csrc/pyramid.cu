// K1-K3 host dispatch: octave base and level blurs (the kernel template lives in
// blur_kernel.cuh; this file instantiates the reference-rounding blur over a
// (tiles x, tiles y, images) grid, pyramid_fused.cu the single-rounding one, and
// pyramid_tiled*.cu both over a tile work list).
#include "blur_kernel.cuh"

namespace psift {

// Host entry: mode 0 = level blur (octave, level >= 1); modes 1..4 = octave-0 base.
// variant (level blur only) picks the outputs per thread (0-2, see
// blur_kernel.cuh), the TMA-tile kernel (3, blur_tma.cuh; needs the host copy
// of the plans for its tensor maps) or 128 x 64 tiles of 512 threads (4: half
// the horizontal pass's halo rows per output); every variant computes the same
// values.  fused: the single-rounding blur
// (one fused multiply-add per tap; not the reference's rounding).
cudaError_t launch_blur_tma(int radius, bool fused, const ImagePlan* d_plans, const ImagePlan* h_plans, int n,
                            int octave, int level, int down_level, int zrev, const Taps2& taps, uint32_t* err,
                            cudaStream_t st);

cudaError_t launch_blur(int mode, const float* taps_host, int radius, const ImagePlan* plans, int n, int octave,
                        int level, int down_level, int max_h, int max_w, cudaStream_t st, int variant, bool fused,
                        const TileMap* tiles, const ImagePlan* h_plans, uint32_t* err) {
  Taps2 t;
  for (int i = 0; i < kMaxTaps; ++i) {
    const float v = i <= 2 * radius ? taps_host[i] : 0.0f;
    t.w[i] = make_float2(v, v);
  }
  t.one = make_float2(1.0f, 1.0f);
  const int zrev = (octave * 8 + level) & 1;
  // variant 3: TMA tiles, persistent CTAs (blur_tma.cuh), either rounding
  if (mode == MODE_LEVEL && variant == 3)
    return launch_blur_tma(radius, fused, plans, h_plans, n, octave, level, down_level, zrev, t, err, st);
  // images of different sizes: one CTA per listed tile (4 x 8 outputs per thread)
  if (tiles && tiles->n > 0)
    return launch_blur_tiled(mode, fused, radius, plans, n, octave, level, down_level, zrev, t, *tiles, st);
  if (fused) return launch_blur_fused(mode, radius, plans, n, octave, level, down_level, zrev, t, max_h, max_w, st);
  switch (mode) {
    case MODE_LEVEL:
      switch (variant) {
        case 0: return launch_blur_mode<MODE_LEVEL, 4, 8, false>(radius, plans, n, octave, level, down_level, zrev, t, nullptr, max_h, max_w, st);
        case 1: return launch_blur_mode<MODE_LEVEL, 8, 8, false>(radius, plans, n, octave, level, down_level, zrev, t, nullptr, max_h, max_w, st);
        case 2: return launch_blur_mode<MODE_LEVEL, 4, 4, false>(radius, plans, n, octave, level, down_level, zrev, t, nullptr, max_h, max_w, st);
        case 4:  // 128-row tiles, 512 threads
          return launch_blur_mode<MODE_LEVEL, 4, 8, false, false, 128, 512>(radius, plans, n, octave, level, down_level,
                                                                            zrev, t, nullptr, max_h, max_w, st);
        default: return cudaErrorInvalidValue;
      }
    case MODE_INIT_F32: return launch_blur_mode<MODE_INIT_F32, 4, 8, false>(radius, plans, n, octave, level, down_level, zrev, t, nullptr, max_h, max_w, st);
    case MODE_INIT_U8: return launch_blur_mode<MODE_INIT_U8, 4, 8, false>(radius, plans, n, octave, level, down_level, zrev, t, nullptr, max_h, max_w, st);
    case MODE_INIT_F32_UP: return launch_blur_mode<MODE_INIT_F32_UP, 4, 8, false>(radius, plans, n, octave, level, down_level, zrev, t, nullptr, max_h, max_w, st);
    case MODE_INIT_U8_UP: return launch_blur_mode<MODE_INIT_U8_UP, 4, 8, false>(radius, plans, n, octave, level, down_level, zrev, t, nullptr, max_h, max_w, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace psift
