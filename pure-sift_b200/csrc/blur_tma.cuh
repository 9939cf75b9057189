// Level blur with 2-D TMA tiles: the input tile of G[s-1] (tile + halo) arrives
// in shared memory by one cp.async.bulk.tensor.2d (no multicast) on an mbarrier,
// issued for the CTA's next tile while the current one's vertical pass runs.
//
// Reference: gaussian_blur (src/pipeline.rs:314-425), build_scale_space_pyramid
// (:550-638); the same values as blur_level_kernel<R, HC, RV, MODE_LEVEL, FUSED>
// (same taps, order and roundings), so both kernels' planes are identical.
//
// Structure: persistent CTAs (resident ones only) walk the launch's tile list
// (every existing 64x64 tile of every image; reversed on odd levels), 256
// threads each.  Interior tiles (tile + halo inside the plane) load by TMA into
// a row-major stage; border tiles, whose halo clamps to the plane like
// `(x + k).saturating_sub(r).min(w - 1)`, are staged by the threads.  The
// horizontal pass takes two rows at a time: a thread's four outputs of rows 2p
// and 2p + 1 as packed f32x2 pairs, each pair's operand {x[2p][c], x[2p+1][c]}
// built from the two rows' 128-bit loads.  Once the horizontal pass has read
// the stage, thread 0 issues the next tile's TMA into it and the vertical pass
// runs from the intermediate; D = G[s] - G[s-1] takes G[s-1] from memory (the
// tile just loaded, still in L2).  The wait on the copy is bounded: on timeout
// the CTA records kErrTimeout and leaves.
#pragma once
#include <cuda.h>

#include "blur_kernel.cuh"

namespace psift {

constexpr int kTmaMaxImages = kTileMapMax;
constexpr uint32_t kTmaSpin = 1u << 26;

// One tensor map per image of the launch: G[s-1] of the launch's octave (f32,
// w x h, row pitch; box = the tile with its halo, IN_W x IN_H).
struct TmaPlanes {
  CUtensorMap m[kTmaMaxImages];
};

template <int R>
struct TmaGeom {
  static constexpr int RP = BlurGeom<R>::RP;  // column halo in whole float4 (16-byte TMA x alignment)
  static constexpr int IN_W = kTileW + 2 * RP;
  static constexpr int IN_H = kTileH + 2 * R;
  static constexpr int OFF = RP - R;          // staged column of output 0's first tap
  static constexpr int NQ = (OFF + 2 * R + 4 + 3) / 4;  // float4 loads per row for four outputs
  static constexpr uint32_t STAGE_BYTES = (uint32_t)IN_W * IN_H * 4;
  static constexpr uint32_t SMEM_STAGE = (STAGE_BYTES + 127) / 128 * 128;
  static constexpr uint32_t SMEM_BYTES = SMEM_STAGE + IN_H * kTmpStride * 4 + 128;
  static_assert(IN_W <= 256 && IN_H <= 256, "TMA box");
  static_assert((IN_W * 4) % 16 == 0, "TMA box rows are whole 16-byte units");
};

__device__ __forceinline__ bool tma_mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  for (uint32_t i = 0; i < kTmaSpin; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

template <int R, bool FUSED>
__global__ void __launch_bounds__(kBlurThreads, 3)
    blur_tma_kernel(const ImagePlan* __restrict__ plans, int octave, int level, int down_level, int zrev,
                    const __grid_constant__ Taps2 taps, const __grid_constant__ TmaPlanes maps, uint32_t* err) {
  using G = TmaGeom<R>;
  constexpr int RV = 8;
  extern __shared__ __align__(128) uint8_t tsm[];
  float* s_in = reinterpret_cast<float*>(tsm);                               // [IN_H][IN_W]
  float* s_tmp = reinterpret_cast<float*>(tsm + G::SMEM_STAGE);              // [IN_H][kTmpStride]
  uint64_t* bar = reinterpret_cast<uint64_t*>(tsm + G::SMEM_BYTES - 128);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float2 wv[R + 1];
#pragma unroll
  for (int k = 0; k <= R; ++k) wv[k] = taps.w[k];
  const float2 one = taps.one;
  const TileMap& tm = taps.tiles;
  const int total = tm.prefix[tm.n];

  // tile lin -> image, tile origin, interior?
  auto tile_info = [&](int lin, int& z, int& tx0, int& ty0, bool& interior) {
    int bx, by;
    tile_of(tm, lin, zrev, z, bx, by);
    const OctaveDev& O = plans[z].oct[octave];
    tx0 = bx * kTileW;
    ty0 = by * kTileH;
    interior = tx0 - G::RP >= 0 && tx0 + kTileW + G::RP <= O.w && ty0 - R >= 0 && ty0 + kTileH + R <= O.h;
  };
  auto issue = [&](int z, int tx0, int ty0) {  // thread 0
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(bar)),
                 "r"(G::STAGE_BYTES)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::
            "r"((uint32_t)__cvta_generic_to_shared(s_in)),
        "l"(reinterpret_cast<uint64_t>(&maps.m[z])), "r"((uint32_t)__cvta_generic_to_shared(bar)), "r"(tx0 - G::RP),
        "r"(ty0 - R)
        : "memory");
  };

  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  int lin = blockIdx.x;
  if (lin >= total) return;
  uint32_t phase = 0;
  {
    int z, tx0, ty0;
    bool in;
    tile_info(lin, z, tx0, ty0, in);
    if (in && threadIdx.x == 0) issue(z, tx0, ty0);
  }
  while (lin < total) {
    int z, tx0, ty0;
    bool interior;
    tile_info(lin, z, tx0, ty0, interior);
    const ImagePlan& P = plans[z];
    const OctaveDev& O = P.oct[octave];
    const int h = O.h, w = O.w;
    const float* src_plane = O.g + (long long)(level - 1) * O.plane_stride;
    if (interior) {
      const bool ok = tma_mbar_wait(bar, phase);
      phase ^= 1u;
      if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(err, kErrTimeout);
        return;
      }
    } else {
      // border tile: clamped staging by the threads (row-major, like the TMA box)
      for (int i = threadIdx.x; i < G::IN_H * G::IN_W; i += kBlurThreads) {
        const int r = i / G::IN_W, c = i - r * G::IN_W;
        const int gy = clampi(ty0 - R + r, 0, h - 1), gx = clampi(tx0 - G::RP + c, 0, w - 1);
        s_in[i] = src_plane[(long long)gy * O.pitch + gx];
      }
      __syncthreads();
    }

    // Horizontal pass: rows 2p, 2p + 1 x four outputs per thread.
    {
      constexpr int PAIRS = G::IN_H / 2;
      for (int item = threadIdx.x; item < PAIRS * (kTileW / 4); item += kBlurThreads) {
        const int xg = item & 15, rp = item >> 4;
        const float4* r0 = reinterpret_cast<const float4*>(s_in + (2 * rp) * G::IN_W + 4 * xg);
        const float4* r1 = reinterpret_cast<const float4*>(s_in + (2 * rp + 1) * G::IN_W + 4 * xg);
        float2 acc[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[j] = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int q = 0; q < G::NQ; ++q) {
          const float4 a = r0[q], b = r1[q];
          const float2 p[4] = {make_float2(a.x, b.x), make_float2(a.y, b.y), make_float2(a.z, b.z),
                               make_float2(a.w, b.w)};
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int m = 4 * q + e;  // window column
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int k = m - G::OFF - j;
              if (k >= 0 && k <= 2 * R) acc[j] = tap2<FUSED>(acc[j], p[e], wv[k <= R ? k : 2 * R - k], one);
            }
          }
        }
        float* t0 = s_tmp + (2 * rp) * kTmpStride + 4 * xg;
        *reinterpret_cast<float4*>(t0) = make_float4(acc[0].x, acc[1].x, acc[2].x, acc[3].x);
        *reinterpret_cast<float4*>(t0 + kTmpStride) = make_float4(acc[0].y, acc[1].y, acc[2].y, acc[3].y);
      }
    }
    __syncthreads();
    // the stage is free: the next tile's TMA runs under the vertical pass
    const int next = lin + (int)gridDim.x;
    if (next < total) {
      int nz, nx0, ny0;
      bool nin;
      tile_info(next, nz, nx0, ny0, nin);
      if (nin && threadIdx.x == 0) issue(nz, nx0, ny0);
    }

    // Vertical pass: a column pair x RV rows per thread (as blur_level_kernel).
    {
      const long long gbase = (long long)level * O.plane_stride;
      float* gout = O.g + gbase;
      float* dout = O.d + (long long)(level - 1) * O.plane_stride;
      const bool do_down = level == down_level && octave + 1 < P.n_oct;
      const int x = 2 * lane;
      const int gx = tx0 + x;
      for (int yb = warp * RV; yb < kTileH; yb += RV * (kBlurThreads / 32)) {
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
            if (k >= 0 && k <= 2 * R) acc[j] = tap2<FUSED>(acc[j], v, wv[k <= R ? k : 2 * R - k], one);
          }
        }
        if (gx >= w) continue;
        const bool pair_ok = gx + 1 < w;
#pragma unroll
        for (int j = 0; j < RV; ++j) {
          const int gy = ty0 + yb + j;
          if (gy >= h) break;
          float* grow = gout + (long long)gy * O.pitch + gx;
          const float* prow = src_plane + (long long)gy * O.pitch + gx;
          float* drow = dout + (long long)gy * O.pitch + gx;
          if (pair_ok) {
            const float2 pv = __ldg(reinterpret_cast<const float2*>(prow));
            *reinterpret_cast<float2*>(grow) = acc[j];
            __stcs(reinterpret_cast<float2*>(drow), make_float2(__fsub_rn(acc[j].x, pv.x), __fsub_rn(acc[j].y, pv.y)));
          } else {
            grow[0] = acc[j].x;
            __stcs(drow, __fsub_rn(acc[j].x, __ldg(prow)));
          }
          if (do_down && !(gy & 1)) {
            const OctaveDev& N = P.oct[octave + 1];
            const int dy = gy >> 1, dxn = gx >> 1;
            if (dy < N.h && dxn < N.w) N.g[(long long)dy * N.pitch + dxn] = acc[j].x;
          }
        }
      }
    }
    __syncthreads();  // the intermediate is free for the next tile
    lin = next;
  }
}

}  // namespace psift
