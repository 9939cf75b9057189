// Blur launches over a tile work list with the single-rounding taps (one fused
// multiply-add per tap; see pyramid_fused.cu): level blur with 4 x 8 outputs per
// thread and the four octave-base modes.
#include "blur_kernel.cuh"

namespace psift {

cudaError_t launch_blur_tiled_fused(int mode, int radius, const ImagePlan* plans, int n, int octave, int level,
                                    int down_level, int zrev, const Taps2& taps, const TileMap& tiles,
                                    cudaStream_t st) {
  const TileMap* tm = &tiles;
  switch (mode) {
    case MODE_LEVEL:
      return launch_blur_mode<MODE_LEVEL, 4, 8, true, true>(radius, plans, n, octave, level, down_level, zrev, taps,
                                                            tm, 0, 0, st);
    case MODE_INIT_F32:
      return launch_blur_mode<MODE_INIT_F32, 4, 8, true, true>(radius, plans, n, octave, level, down_level, zrev, taps,
                                                               tm, 0, 0, st);
    case MODE_INIT_U8:
      return launch_blur_mode<MODE_INIT_U8, 4, 8, true, true>(radius, plans, n, octave, level, down_level, zrev, taps,
                                                              tm, 0, 0, st);
    case MODE_INIT_F32_UP:
      return launch_blur_mode<MODE_INIT_F32_UP, 4, 8, true, true>(radius, plans, n, octave, level, down_level, zrev,
                                                                  taps, tm, 0, 0, st);
    case MODE_INIT_U8_UP:
      return launch_blur_mode<MODE_INIT_U8_UP, 4, 8, true, true>(radius, plans, n, octave, level, down_level, zrev,
                                                                 taps, tm, 0, 0, st);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace psift
