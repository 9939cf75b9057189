// K12: warp_and_stitch -- the query image warped into the target's frame by
// bilinear inverse mapping and feather-blended with the target on the union
// canvas, one thread per canvas pixel.
//
// Reference: warp_and_stitch (src/visualize.rs:379-483), invert_matrix_3x3
// (:202-233), project_f64 (:236-247), sample_bilinear_rgba (:250-287),
// Homography2D::project (src/pipeline.rs:1122-1132), MAX_WARP_DIM /
// MAX_WARP_PIXELS (src/visualize.rs:10-12).
//
// Arithmetic: the reference's f64 expressions in its order (the library is
// built with -fmad=false, so no product is fused into an add); floor / round
// are exact; `as u8` saturates as Rust's cast does.  The canvas geometry
// (inverse, projected corners in f32, bounds) is computed on the host with the
// same expressions.  Each thread reads one target texel and four query texels
// (32-bit loads, neighbouring threads share rows through L1/L2) and writes one
// 32-bit canvas pixel.  The f64 arithmetic (the query's projection and bilinear
// weights, three IEEE divisions), not HBM, bounds the kernel.
#include <cmath>
#include <cstring>
#include <string>

#include "psift_internal.cuh"

namespace psift {
namespace {

constexpr double kMaxWarpDim = 8192.0;        // MAX_WARP_DIM
constexpr double kMaxWarpPixels = 25000000.0;  // MAX_WARP_PIXELS

struct WarpGeom {
  double hinv[9];
  double ox0, oy0;
  int width, height;
};

struct WarpImages {
  const uint8_t* q;
  const uint8_t* t;
  long long q_stride, t_stride;  // bytes, multiples of 4
  int qh, qw, th, tw;
};

// sample_bilinear_rgba: false outside [0, w-1] x [0, h-1].
__device__ __forceinline__ bool sample_rgba(const uint8_t* __restrict__ img, int h, int w, long long stride, double x,
                                            double y, double rgba[4], double& feather) {
  const double wf = (double)w, hf = (double)h;
  if (x < 0.0 || y < 0.0 || x > (wf - 1.0) || y > (hf - 1.0)) return false;
  const unsigned x0 = (unsigned)floor(x), y0 = (unsigned)floor(y);
  const unsigned x1 = min(x0 + 1u, (unsigned)w - 1u), y1 = min(y0 + 1u, (unsigned)h - 1u);
  const double fx = x - (double)x0, fy = y - (double)y0;
  const double w00 = (1.0 - fx) * (1.0 - fy), w10 = fx * (1.0 - fy), w01 = (1.0 - fx) * fy, w11 = fx * fy;
  const uint8_t* r0 = img + (long long)y0 * stride;
  const uint8_t* r1 = img + (long long)y1 * stride;
  const uint32_t p00 = __ldg(reinterpret_cast<const uint32_t*>(r0) + x0);
  const uint32_t p10 = __ldg(reinterpret_cast<const uint32_t*>(r0) + x1);
  const uint32_t p01 = __ldg(reinterpret_cast<const uint32_t*>(r1) + x0);
  const uint32_t p11 = __ldg(reinterpret_cast<const uint32_t*>(r1) + x1);
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int sh = 8 * c;
    rgba[c] = (double)((p00 >> sh) & 255u) * w00 + (double)((p10 >> sh) & 255u) * w10 +
              (double)((p01 >> sh) & 255u) * w01 + (double)((p11 >> sh) & 255u) * w11;
  }
  // x.min(w-1-x).min(y).min(h-1-y): all finite here
  const double dist_edge = fmin(fmin(fmin(x, (wf - 1.0) - x), y), (hf - 1.0) - y);
  const double f = (dist_edge + 1.0) / 32.0;
  feather = f < 0.02 ? 0.02 : (f > 1.0 ? 1.0 : f);
  return true;
}

__device__ __forceinline__ uint32_t sat_u8(double v) {  // Rust `as u8`
  if (!(v == v)) return 0u;
  return v <= 0.0 ? 0u : (v >= 255.0 ? 255u : (uint32_t)v);
}

__global__ void __launch_bounds__(256) warp_stitch_kernel(WarpImages im, WarpGeom g, uint32_t* __restrict__ canvas) {
  const int ox = blockIdx.x * 32 + (threadIdx.x & 31);
  const int oy = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (ox >= g.width || oy >= g.height) return;
  const double tx = (double)ox + g.ox0, ty = (double)oy + g.oy0;
  double tc[4], qc[4], tw = 0.0, qw = 0.0;
  // The canvas origin is integral, so the target is sampled at whole pixels:
  // sample_bilinear_rgba's weights are (1, 0, 0, 0) there and its sum is the
  // texel itself (the zero-weight terms add +0), its feather weight
  // ((min edge distance) + 1) / 32 clamped.
  const bool has_t = tx >= 0.0 && ty >= 0.0 && tx <= (double)im.tw - 1.0 && ty <= (double)im.th - 1.0;
  if (has_t) {
    const int ix = (int)tx, iy = (int)ty;
    const uint32_t p = __ldg(reinterpret_cast<const uint32_t*>(im.t + (long long)iy * im.t_stride) + ix);
#pragma unroll
    for (int c = 0; c < 4; ++c) tc[c] = (double)((p >> (8 * c)) & 255u);
    const double dist_edge = fmin(fmin(fmin(tx, ((double)im.tw - 1.0) - tx), ty), ((double)im.th - 1.0) - ty);
    const double f = (dist_edge + 1.0) / 32.0;
    tw = f < 0.02 ? 0.02 : (f > 1.0 ? 1.0 : f);
  }
  bool has_q = false;
  const double w = g.hinv[6] * tx + g.hinv[7] * ty + g.hinv[8];
  if (!(fabs(w) < 1e-7)) {
    const double iw = 1.0 / w;
    const double qx = (g.hinv[0] * tx + g.hinv[1] * ty + g.hinv[2]) * iw;
    const double qy = (g.hinv[3] * tx + g.hinv[4] * ty + g.hinv[5]) * iw;
    has_q = sample_rgba(im.q, im.qh, im.qw, im.q_stride, qx, qy, qc, qw);
  }
  uint32_t out = 0u;
  if (has_t && has_q) {
    const double den = tw + qw, wt = tw / den, wq = qw / den;
    double al = round(tc[3] * wt + qc[3] * wq);
    al = al < 0.0 ? 0.0 : (al > 255.0 ? 255.0 : al);
    out = sat_u8(round(tc[0] * wt + qc[0] * wq)) | (sat_u8(round(tc[1] * wt + qc[1] * wq)) << 8) |
          (sat_u8(round(tc[2] * wt + qc[2] * wq)) << 16) | (sat_u8(al) << 24);
  } else if (has_t) {
    out = sat_u8(round(tc[0])) | (sat_u8(round(tc[1])) << 8) | (sat_u8(round(tc[2])) << 16) |
          (sat_u8(round(tc[3])) << 24);
  } else if (has_q) {
    out = sat_u8(round(qc[0])) | (sat_u8(round(qc[1])) << 8) | (sat_u8(round(qc[2])) << 16) |
          (sat_u8(round(qc[3])) << 24);
  }
  __stcs(canvas + (long long)oy * g.width + ox, out);
}

// Canvas geometry of warp_and_stitch (src/visualize.rs:384-434), with its errors.
psift_status warp_geometry(psift_ctx* ctx, uint32_t qh, uint32_t qw, uint32_t th, uint32_t tw, const float* h9,
                           WarpGeom* g) {
  double a[3][3];
  for (int i = 0; i < 9; ++i) a[i / 3][i % 3] = (double)h9[i];
  const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
  const double c01 = -(a[1][0] * a[2][2] - a[1][2] * a[2][0]);
  const double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
  const double c10 = -(a[0][1] * a[2][2] - a[0][2] * a[2][1]);
  const double c11 = a[0][0] * a[2][2] - a[0][2] * a[2][0];
  const double c12 = -(a[0][0] * a[2][1] - a[0][1] * a[2][0]);
  const double c20 = a[0][1] * a[1][2] - a[0][2] * a[1][1];
  const double c21 = -(a[0][0] * a[1][2] - a[0][2] * a[1][0]);
  const double c22 = a[0][0] * a[1][1] - a[0][1] * a[1][0];
  const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
  if (std::fabs(det) < 1e-12 || !std::isfinite(det))
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "Homography matrix is singular and cannot be inverted");
  const double id = 1.0 / det;
  const double hi[9] = {c00 * id, c10 * id, c20 * id, c01 * id, c11 * id, c21 * id, c02 * id, c12 * id, c22 * id};
  std::memcpy(g->hinv, hi, sizeof hi);
  const double qwf = qw, qhf = qh, twf = tw, thf = th;
  double min_x = 0.0, min_y = 0.0, max_x = std::fmax(twf - 1.0, 0.0), max_y = std::fmax(thf - 1.0, 0.0);
  const double corners[4][2] = {{0.0, 0.0}, {qwf - 1.0, 0.0}, {0.0, qhf - 1.0}, {qwf - 1.0, qhf - 1.0}};
  for (const auto& c : corners) {
    const float x = (float)c[0], y = (float)c[1];
    const float w = h9[6] * x + h9[7] * y + h9[8];
    if (std::fabs(w) < 1e-6f)
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "Projected query corner hit infinity under homography");
    const float iw = 1.0f / w;
    const double px = (double)((h9[0] * x + h9[1] * y + h9[2]) * iw);
    const double py = (double)((h9[3] * x + h9[4] * y + h9[5]) * iw);
    if (!std::isfinite(px) || !std::isfinite(py))
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "Projected query corner produced non-finite coordinate");
    min_x = std::fmin(min_x, px);
    min_y = std::fmin(min_y, py);
    max_x = std::fmax(max_x, px);
    max_y = std::fmax(max_y, py);
  }
  const double ox0 = std::floor(min_x), oy0 = std::floor(min_y);
  const double wf = std::fmax(std::ceil(max_x) - ox0 + 1.0, 1.0), hf = std::fmax(std::ceil(max_y) - oy0 + 1.0, 1.0);
  if (wf > kMaxWarpDim || hf > kMaxWarpDim || wf * hf > kMaxWarpPixels) {
    char buf[200];
    snprintf(buf, sizeof buf, "Stitched canvas dimensions %zux%zu exceed safety limits (8192x8192, 25000000 px)",
             (size_t)wf, (size_t)hf);
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, buf);
  }
  g->ox0 = ox0;
  g->oy0 = oy0;
  g->width = (int)wf;
  g->height = (int)hf;
  return PSIFT_OK;
}

cudaError_t launch_warp(const WarpImages& im, const WarpGeom& g, uint32_t* canvas, cudaStream_t st) {
  dim3 grid((g.width + 31) / 32, (g.height + 7) / 8);
  warp_stitch_kernel<<<grid, 256, 0, st>>>(im, g, canvas);
  return cudaGetLastError();
}

}  // namespace
}  // namespace psift

using namespace psift;

extern "C" {

psift_status psift_warp_and_stitch(psift_ctx* ctx, const uint8_t* query, uint32_t qh, uint32_t qw, size_t q_stride,
                                   const uint8_t* target, uint32_t th, uint32_t tw, size_t t_stride, const float* h9,
                                   uint8_t* canvas, size_t canvas_capacity, uint32_t* width, uint32_t* height,
                                   double* origin) {
  if (!ctx || !h9 || !width || !height) return PSIFT_ERR_INVALID_ARGUMENT;
  if ((qh && qw && (!query || q_stride < 4ull * qw)) || (th && tw && (!target || t_stride < 4ull * tw)))
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null image or row stride below 4 x width");
  WarpGeom g;
  psift_status st = warp_geometry(ctx, qh, qw, th, tw, h9, &g);
  if (st != PSIFT_OK) return st;
  *width = (uint32_t)g.width;
  *height = (uint32_t)g.height;
  if (origin) {
    origin[0] = g.ox0;
    origin[1] = g.oy0;
  }
  if (!canvas) return PSIFT_OK;
  const size_t cbytes = (size_t)g.width * g.height * 4;
  if (canvas_capacity < cbytes) return set_error(ctx, PSIFT_ERR_CAPACITY, "canvas capacity below width x height x 4");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(ctx, e, "cudaSetDevice");
  const size_t qb = align_up((size_t)qh * qw * 4, 256), tb = align_up((size_t)th * tw * 4, 256);
  if ((st = io_reserve(ctx, qb + tb + cbytes + 1024)) != PSIFT_OK) return st;
  uint8_t* d_q = (uint8_t*)ctx->io.base;
  uint8_t* d_t = d_q + qb;
  uint32_t* d_c = (uint32_t*)(d_t + tb);
  cudaStream_t s = ctx->stream;
  if (qh && qw) PSIFT_CUDA_TRY(ctx, cudaMemcpy2DAsync(d_q, 4 * (size_t)qw, query, q_stride, 4 * (size_t)qw, qh,
                                                      cudaMemcpyHostToDevice, s));
  if (th && tw) PSIFT_CUDA_TRY(ctx, cudaMemcpy2DAsync(d_t, 4 * (size_t)tw, target, t_stride, 4 * (size_t)tw, th,
                                                      cudaMemcpyHostToDevice, s));
  WarpImages im{d_q, d_t, 4ll * qw, 4ll * tw, (int)qh, (int)qw, (int)th, (int)tw};
  e = launch_warp(im, g, d_c, s);
  ctx->launches++;
  if (e != cudaSuccess) return cuda_error(ctx, e, "warp_and_stitch");
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(canvas, d_c, cbytes, cudaMemcpyDeviceToHost, s));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return PSIFT_OK;
}

psift_status psift_warp_and_stitch_dev(psift_ctx* ctx, const uint8_t* query, uint32_t qh, uint32_t qw,
                                       size_t q_stride, const uint8_t* target, uint32_t th, uint32_t tw,
                                       size_t t_stride, const float* h9, uint8_t* canvas, size_t canvas_capacity,
                                       uint32_t* width, uint32_t* height) {
  if (!ctx || !h9 || !width || !height || !canvas) return PSIFT_ERR_INVALID_ARGUMENT;
  if ((qh && qw && (!query || q_stride < 4ull * qw || q_stride % 4)) ||
      (th && tw && (!target || t_stride < 4ull * tw || t_stride % 4)))
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null image or row stride not a multiple of 4 >= 4 x width");
  if ((reinterpret_cast<uintptr_t>(query) | reinterpret_cast<uintptr_t>(target) | reinterpret_cast<uintptr_t>(canvas)) & 3)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "device images must be 4-byte aligned");
  WarpGeom g;
  psift_status st = warp_geometry(ctx, qh, qw, th, tw, h9, &g);
  if (st != PSIFT_OK) return st;
  *width = (uint32_t)g.width;
  *height = (uint32_t)g.height;
  if (canvas_capacity < (size_t)g.width * g.height * 4)
    return set_error(ctx, PSIFT_ERR_CAPACITY, "canvas capacity below width x height x 4");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(ctx, e, "cudaSetDevice");
  WarpImages im{query, target, (long long)q_stride, (long long)t_stride, (int)qh, (int)qw, (int)th, (int)tw};
  e = launch_warp(im, g, reinterpret_cast<uint32_t*>(canvas), ctx->stream);
  ctx->launches++;
  if (e != cudaSuccess) return cuda_error(ctx, e, "warp_and_stitch");
  return PSIFT_OK;
}

}  // extern "C"
