// Host side of the TMA level blur (blur_tma.cuh): one tensor map per image over
// its G[s-1] plane, the launch's tile list, persistent CTAs (the resident ones).
#include <cstring>
#include <vector>

#include "blur_tma.cuh"

namespace psift {
namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

template <int R, bool FUSED>
cudaError_t launch_tma_r(const ImagePlan* d_plans, const ImagePlan* h_plans, int n, int octave, int level,
                         int down_level, int zrev, const Taps2& taps, uint32_t* err, cudaStream_t st) {
  using G = TmaGeom<R>;
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return cudaErrorNotSupported;
  TileMap tm;
  tm.n = n;
  tm.prefix[0] = 0;
  TmaPlanes maps;
  for (int i = 0; i < n; ++i) {
    const bool has = octave < h_plans[i].n_oct;
    const OctaveDev& O = h_plans[i].oct[has ? octave : 0];
    const int tx = has ? (O.w + kTileW - 1) / kTileW : 0, ty = has ? (O.h + kTileH - 1) / kTileH : 0;
    tm.tiles_x[i] = tx > 0 ? tx : 1;
    tm.prefix[i + 1] = tm.prefix[i] + tx * ty;
    if (!has) {
      std::memset(&maps.m[i], 0, sizeof(CUtensorMap));
      continue;
    }
    const float* plane = O.g + (long long)(level - 1) * O.plane_stride;
    cuuint64_t dims[2] = {(cuuint64_t)O.w, (cuuint64_t)O.h};
    cuuint64_t strides[1] = {(cuuint64_t)O.pitch * 4};
    cuuint32_t box[2] = {(cuuint32_t)G::IN_W, (cuuint32_t)G::IN_H};
    cuuint32_t estr[2] = {1, 1};
    if (enc(&maps.m[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(plane), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return cudaErrorInvalidValue;
  }
  const int total = tm.prefix[n];
  if (total == 0) return cudaSuccess;
  const void* fn = (const void*)blur_tma_kernel<R, FUSED>;
  cudaError_t e = ensure_smem_attr(fn, G::SMEM_BYTES);
  if (e != cudaSuccess) return e;
  int resident = 0;
  e = resident_ctas(fn, kBlurThreads, G::SMEM_BYTES, &resident);
  if (e != cudaSuccess) return e;
  const int grid = resident < total ? resident : total;
  blur_tma_kernel<R, FUSED><<<grid, kBlurThreads, G::SMEM_BYTES, st>>>(d_plans, octave, level, down_level, zrev, taps,
                                                                    tm, maps, err);
  return cudaGetLastError();
}

}  // namespace

// The level blur of images [0, n) with TMA tiles (variant 3 of the level blur).
cudaError_t launch_blur_tma(int radius, bool fused, const ImagePlan* d_plans, const ImagePlan* h_plans, int n,
                            int octave, int level, int down_level, int zrev, const Taps2& taps, uint32_t* err,
                            cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (n > kTmaMaxImages || !h_plans || !err) return cudaErrorInvalidValue;
  switch (radius) {
#define PSIFT_TR(RR)                                                                                               \
  case RR:                                                                                                         \
    return fused ? launch_tma_r<RR, true>(d_plans, h_plans, n, octave, level, down_level, zrev, taps, err, st)    \
                 : launch_tma_r<RR, false>(d_plans, h_plans, n, octave, level, down_level, zrev, taps, err, st);
    PSIFT_TR(1) PSIFT_TR(2) PSIFT_TR(3) PSIFT_TR(4) PSIFT_TR(5) PSIFT_TR(6) PSIFT_TR(7) PSIFT_TR(8)
    PSIFT_TR(9) PSIFT_TR(10) PSIFT_TR(11) PSIFT_TR(12) PSIFT_TR(13) PSIFT_TR(14) PSIFT_TR(15)
#undef PSIFT_TR
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace psift
