// Level blur with 2-D TMA tiles: the input tile of G[s-1] (tile + halo) arrives
// in shared memory by one cp.async.bulk.tensor.2d on an mbarrier,
// into a double-buffered stage: the CTA's next tile is copied during the whole of
// the current tile's horizontal and vertical passes.
//
// Reference: gaussian_blur (src/pipeline.rs:314-425), build_scale_space_pyramid
// (:550-638); the same values as blur_level_kernel<R, HC, RV, MODE_LEVEL, FUSED>
// (same taps, order and roundings), so both kernels' planes are identical.
//
// Structure: persistent CTAs (the resident ones) walk the launch's tile list
// (every existing 64x64 tile of every image; reversed on odd levels), 256
// threads each.  Every tile's box (IN_W x IN_H from (tx0 - RP, ty0 - R)) is one
// TMA copy; where the box leaves the plane the copy fills zeros, and the threads
// then replace each such element by the in-plane element that the reference's
// clamp `(x + k).saturating_sub(r).min(w - 1)` selects (it lies inside the box,
// and only out-of-plane elements are written, so the fix-up has no read/write
// overlap).  The horizontal pass takes two rows at a time: a thread's four
// outputs of rows 2p and 2p + 1 as packed f32x2 pairs, each pair's operand
// {x[2p][c], x[2p+1][c]} built from the two rows' 128-bit loads.  The vertical
// pass runs from the intermediate and forms D = G[s] - G[s-1] with G[s-1] from
// the stage.  Waits on the copies are bounded: on timeout the CTA records
// kErrTimeout, waits (bounded) for its copies in flight and leaves.
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
  static constexpr uint32_t SMEM_BYTES = 2 * SMEM_STAGE + IN_H * kTmpStride * 4 + 128;
  // CTAs per SM that the shared memory allows (228 KB per SM, 1 KB reserved per CTA)
  static constexpr int MIN_CTAS = 3 * (SMEM_BYTES + 1024) <= 228 * 1024 ? 3 : 2;
  static_assert(IN_W <= 256 && IN_H <= 256, "TMA box");
  static_assert((IN_W * 4) % 16 == 0, "TMA box rows are whole 16-byte units");
  static_assert(IN_W % 2 == 0 && RP % 2 == 0, "float2 reads of G[s-1] from the stage");
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
__global__ void __launch_bounds__(kBlurThreads, TmaGeom<R>::MIN_CTAS)
    blur_tma_kernel(const ImagePlan* __restrict__ plans, int octave, int level, int down_level, int zrev,
                    const __grid_constant__ Taps2 taps, const __grid_constant__ TileMap tm,
                    const __grid_constant__ TmaPlanes maps, uint32_t* err) {
  using G = TmaGeom<R>;
  constexpr int RV = 8;
  extern __shared__ __align__(128) uint8_t tsm[];
  float* s_tmp = reinterpret_cast<float*>(tsm + 2 * G::SMEM_STAGE);  // [IN_H][kTmpStride]
  uint64_t* bars = reinterpret_cast<uint64_t*>(tsm + G::SMEM_BYTES - 128);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float2 wv[R + 1];
#pragma unroll
  for (int k = 0; k <= R; ++k) wv[k] = taps.w[k];
  const float2 one = taps.one;
  const int total = tm.prefix[tm.n];

  // tile lin -> image and tile origin
  auto tile_info = [&](int lin, int& z, int& tx0, int& ty0) {
    int bx, by;
    tile_of(tm, lin, zrev, z, bx, by);
    tx0 = bx * kTileW;
    ty0 = by * kTileH;
  };
  auto issue = [&](int b, int z, int tx0, int ty0) {  // thread 0
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(bars + b);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(G::STAGE_BYTES)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::
            "r"((uint32_t)__cvta_generic_to_shared(tsm + b * G::SMEM_STAGE)),
        "l"(reinterpret_cast<uint64_t>(&maps.m[z])), "r"(bar), "r"(tx0 - G::RP), "r"(ty0 - R)
        : "memory");
  };

  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(bars)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(bars + 1))
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if ((int)blockIdx.x >= total) return;
  if (threadIdx.x == 0) {
    int z, tx0, ty0;
    tile_info(blockIdx.x, z, tx0, ty0);
    issue(0, z, tx0, ty0);
  }
  int it = 0;
  for (int lin = blockIdx.x; lin < total; lin += (int)gridDim.x, ++it) {
    const int b = it & 1;
    // stage b ^ 1 was last read by the previous tile, finished at the loop's end barrier
    const int next = lin + (int)gridDim.x;
    if (next < total && threadIdx.x == 0) {
      int nz, nx0, ny0;
      tile_info(next, nz, nx0, ny0);
      issue(b ^ 1, nz, nx0, ny0);
    }
    int z, tx0, ty0;
    tile_info(lin, z, tx0, ty0);
    const ImagePlan& P = plans[z];
    const OctaveDev& O = P.oct[octave];
    const int h = O.h, w = O.w;
    const bool ok = tma_mbar_wait(bars + b, (uint32_t)(it >> 1) & 1u);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicOr(err, kErrTimeout);
        // the copies in flight land in this CTA's shared memory: wait (bounded) for them
        tma_mbar_wait(bars + b, (uint32_t)(it >> 1) & 1u);
        if (next < total) tma_mbar_wait(bars + (b ^ 1), (uint32_t)((it + 1) >> 1) & 1u);
      }
      return;
    }
    float* s_in = reinterpret_cast<float*>(tsm + b * G::SMEM_STAGE);  // [IN_H][IN_W]
    const int x_lo = tx0 - G::RP, y_lo = ty0 - R;
    if (x_lo < 0 || y_lo < 0 || x_lo + G::IN_W > w || y_lo + G::IN_H > h) {
      // border tile: the zero-filled out-of-plane elements take their clamped values
      for (int i = threadIdx.x; i < G::IN_H * G::IN_W; i += kBlurThreads) {
        const int r = i / G::IN_W, c = i - r * G::IN_W;
        const int gy = y_lo + r, gx = x_lo + c;
        const int cy = clampi(gy, 0, h - 1), cx = clampi(gx, 0, w - 1);
        if (cy != gy || cx != gx) s_in[i] = s_in[(cy - y_lo) * G::IN_W + (cx - x_lo)];
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
          const float4 a = r0[q], c = r1[q];
          const float2 p[4] = {make_float2(a.x, c.x), make_float2(a.y, c.y), make_float2(a.z, c.z),
                               make_float2(a.w, c.w)};
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

    // Vertical pass: a column pair x RV rows per thread (as blur_level_kernel).
    {
      float* gout = O.g + (long long)level * O.plane_stride;
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
        // G[s-1] at (ty0 + yb + j, gx): stage row yb + j + R, column x + RP
        const float* prev = s_in + (yb + R) * G::IN_W + x + G::RP;
#pragma unroll
        for (int j = 0; j < RV; ++j) {
          const int gy = ty0 + yb + j;
          if (gy >= h) break;
          const float2 pv = *reinterpret_cast<const float2*>(prev + j * G::IN_W);
          float* grow = gout + (long long)gy * O.pitch + gx;
          float* drow = dout + (long long)gy * O.pitch + gx;
          if (pair_ok) {
            *reinterpret_cast<float2*>(grow) = acc[j];
            __stcs(reinterpret_cast<float2*>(drow), make_float2(__fsub_rn(acc[j].x, pv.x), __fsub_rn(acc[j].y, pv.y)));
          } else {
            grow[0] = acc[j].x;
            __stcs(drow, __fsub_rn(acc[j].x, pv.x));
          }
          if (do_down && !(gy & 1)) {
            const OctaveDev& N = P.oct[octave + 1];
            const int dy = gy >> 1, dxn = gx >> 1;
            if (dy < N.h && dxn < N.w) N.g[(long long)dy * N.pitch + dxn] = acc[j].x;
          }
        }
      }
    }
    __syncthreads();  // the intermediate and stage b are free for the next tiles
  }
}

}  // namespace psift
