// The single-rounding blur mode's kernels: every tap one fused multiply-add
// (fma.rn.f32x2) instead of the reference's rounded multiply and rounded add.
// Not bit-equal to the reference; its error against an f64 run of the pipeline is
// held to the same bar as the f32 path's (keypoints within 0.01 px / 0.01 scale,
// descriptors within 1e-4 relative L2).  Level blur with 4 x 8 outputs per thread
// and the four octave-base modes.
#include "blur_kernel.cuh"

namespace psift {

cudaError_t launch_blur_fused(int mode, int radius, const ImagePlan* plans, int n, int octave, int level,
                              int down_level, int zrev, const Taps2& taps, int max_h, int max_w, cudaStream_t st) {
  switch (mode) {
    case MODE_LEVEL:
      return launch_blur_mode<MODE_LEVEL, 4, 8, true>(radius, plans, n, octave, level, down_level, zrev, taps, nullptr,
                                                      max_h, max_w, st);
    case MODE_INIT_F32:
      return launch_blur_mode<MODE_INIT_F32, 4, 8, true>(radius, plans, n, octave, level, down_level, zrev, taps, nullptr,
                                                      max_h, max_w, st);
    case MODE_INIT_U8:
      return launch_blur_mode<MODE_INIT_U8, 4, 8, true>(radius, plans, n, octave, level, down_level, zrev, taps, nullptr,
                                                      max_h, max_w, st);
    case MODE_INIT_F32_UP:
      return launch_blur_mode<MODE_INIT_F32_UP, 4, 8, true>(radius, plans, n, octave, level, down_level, zrev, taps, nullptr,
                                                      max_h, max_w, st);
    case MODE_INIT_U8_UP:
      return launch_blur_mode<MODE_INIT_U8_UP, 4, 8, true>(radius, plans, n, octave, level, down_level, zrev, taps, nullptr,
                                                      max_h, max_w, st);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace psift
