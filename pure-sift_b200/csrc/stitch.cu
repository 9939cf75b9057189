// K13: stitch_panorama -- multi-image registration and compositing.
//
// Reference: src/stitch.rs (warp_image_cylindrical :166-201,
// sample_patch_intensity :203-229, solve_exposure_gains :232-316,
// downsample_half_rgba_weighted :318-393, upsample_to_size_rgb :395-434,
// downsample_half_scalar :436-470, stitch_panorama :472-948) with
// src/visualize.rs (invert_matrix_3x3 :202-233, project_f64 :236-247,
// sample_bilinear_rgba :250-287, is_sane_homography_for_dims :303-357,
// resolve_safe_alignment_homography :361-375).
//
// Registration: the prepared images (cylindrical warp on the GPU when asked)
// are converted to luma on the GPU and go through the batch detection entry in
// one call; every pair (i < j) is matched in one batched matcher call and its
// similarity and homography RANSAC run as two batched launches (the reference's
// default seeds).  The graph steps on the results -- edge construction,
// connected components, reference choice, maximum spanning tree, exposure
// gains, canvas bounds -- are O(n^2) host arithmetic in the reference's f64 /
// f32 order.
//
// Compositing, one thread per canvas pixel (per level pixel in the pyramids),
// each kernel the reference's per-pixel expression in its order (the library
// is built with -fmad=false; the images' contributions are accumulated one
// launch per image, in the reference's image order, so every sum has the
// reference's order):
//   feather: every registered image projected (f64) and sampled, weighted sum;
//   multi-band: Voronoi owner by the largest f32 feather weight, then per image
//     its warped level 0, Gaussian pyramid (5-tap weighted separable
//     decimation of colour + validity, plain decimation of the seam mask),
//     Laplacian bands accumulated into the blend pyramid, then normalisation and
//     the collapse from the top level down.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <vector>

#include "psift_internal.cuh"

namespace psift {
namespace {

constexpr double kPanoMaxDim = 8192.0;         // MAX_WARP_DIM (src/visualize.rs:10)
constexpr uint64_t kPanoMaxPixels = 25000000;  // MAX_WARP_PIXELS (src/visualize.rs:12)

// One registered image as the compositing kernels see it.
struct PanoImg {
  const uint8_t* px;  // device RGBA8
  long long stride;   // bytes, multiple of 4
  int h, w;
  double inv[9];      // reference -> image
  float gain;
};

// sample_bilinear_rgba: false outside [0, w-1] x [0, h-1].
__device__ __forceinline__ bool pano_sample(const uint8_t* __restrict__ img, int h, int w, long long stride, double x,
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
  const double dist_edge = fmin(fmin(fmin(x, (wf - 1.0) - x), y), (hf - 1.0) - y);
  const double f = (dist_edge + 1.0) / 32.0;
  feather = f < 0.02 ? 0.02 : (f > 1.0 ? 1.0 : f);
  return true;
}

// project_f64 through the image's inverse, then sample.
__device__ __forceinline__ bool pano_fetch(const PanoImg& I, double rx, double ry, double rgba[4], double& fw) {
  const double w = I.inv[6] * rx + I.inv[7] * ry + I.inv[8];
  if (fabs(w) < 1e-7) return false;
  const double iw = 1.0 / w;
  const double sx = (I.inv[0] * rx + I.inv[1] * ry + I.inv[2]) * iw;
  const double sy = (I.inv[3] * rx + I.inv[4] * ry + I.inv[5]) * iw;
  return pano_sample(I.px, I.h, I.w, I.stride, sx, sy, rgba, fw);
}

__device__ __forceinline__ uint32_t sat_u8(double v) {  // Rust `as u8`
  if (!(v == v)) return 0u;
  return v <= 0.0 ? 0u : (v >= 255.0 ? 255u : (uint32_t)v);
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------- kernels
__global__ void cyl_warp_kernel(const uint8_t* __restrict__ src, long long stride, int h, int w, double f, double cx,
                                double cy, uint32_t* __restrict__ dst) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= w) return;
  uint32_t out = 0u;
  const double theta = ((double)x - cx) / f;
  if (!(fabs(theta) >= 1.45)) {
    const double cos_t = cos(theta);
    const double sx = f * tan(theta) + cx;
    const double sy = ((double)y - cy) / cos_t + cy;
    double px[4], fw;
    if (pano_sample(src, h, w, stride, sx, sy, px, fw))
      out = sat_u8(round(px[0])) | (sat_u8(round(px[1])) << 8) | (sat_u8(round(px[2])) << 16) | (255u << 24);
  }
  dst[(long long)y * w + x] = out;
}

// DynamicImage::to_luma8 of an RGBA8 image: the image crate's Rec. 709 u32 formula.
__global__ void rgba_luma_kernel(const uint8_t* __restrict__ src, long long stride, int h, int w,
                                 uint8_t* __restrict__ luma) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= w) return;
  const uint32_t p = __ldg(reinterpret_cast<const uint32_t*>(src + (long long)y * stride) + x);
  luma[(long long)y * w + x] = (uint8_t)((2126u * (p & 255u) + 7152u * ((p >> 8) & 255u) + 722u * ((p >> 16) & 255u)) /
                                         10000u);
}

__global__ void pano_feather_kernel(const PanoImg* __restrict__ imgs, int n, double ox, double oy, int W, int H,
                                    uint32_t* __restrict__ canvas) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const double rx = ox + (double)x, ry = oy + (double)y;
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, aw = 0.0;
  for (int k = 0; k < n; ++k) {
    double px[4], fw;
    if (!pano_fetch(imgs[k], rx, ry, px, fw)) continue;
    const double g = (double)imgs[k].gain, wt = fmax(fw, 1e-4);
    double v0 = px[0] * g, v1 = px[1] * g, v2 = px[2] * g;
    v0 = v0 < 0.0 ? 0.0 : (v0 > 255.0 ? 255.0 : v0);
    v1 = v1 < 0.0 ? 0.0 : (v1 > 255.0 ? 255.0 : v1);
    v2 = v2 < 0.0 ? 0.0 : (v2 > 255.0 ? 255.0 : v2);
    acc0 += wt * v0;
    acc1 += wt * v1;
    acc2 += wt * v2;
    aw += wt;
  }
  uint32_t out = 0u;
  if (aw > 0.0) {
    const double iw = 1.0 / aw;
    out = sat_u8(round(acc0 * iw)) | (sat_u8(round(acc1 * iw)) << 8) | (sat_u8(round(acc2 * iw)) << 16) |
          (255u << 24);
  }
  canvas[(long long)y * W + x] = out;
}

// Voronoi seam owner: the image with the largest f32 feather weight (the first on ties).
__global__ void pano_owner_kernel(const PanoImg* __restrict__ imgs, int n, double ox, double oy, int W, int H,
                                  int* __restrict__ owner) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const double rx = ox + (double)x, ry = oy + (double)y;
  float best = -1.0f;
  int own = -1;
  for (int k = 0; k < n; ++k) {
    double px[4], fw;
    if (!pano_fetch(imgs[k], rx, ry, px, fw)) continue;
    const float f32 = (float)fw;
    if (f32 > best) {
      best = f32;
      own = k;
    }
  }
  owner[(long long)y * W + x] = own;
}

// Image `pos` warped onto the canvas: level 0 of its pyramid (colour, validity)
// and of its seam mask.
__global__ void pano_warp_kernel(const PanoImg* __restrict__ imgs, int pos, const int* __restrict__ owner, double ox,
                                 double oy, int W, int H, float4* __restrict__ g0, float* __restrict__ m0) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const long long i = (long long)y * W + x;
  const double rx = ox + (double)x, ry = oy + (double)y;
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  double px[4], fw;
  if (pano_fetch(imgs[pos], rx, ry, px, fw)) {
    const float gain = imgs[pos].gain;
    v = make_float4(clampf((float)px[0] * gain, 0.0f, 255.0f), clampf((float)px[1] * gain, 0.0f, 255.0f),
                    clampf((float)px[2] * gain, 0.0f, 255.0f), 1.0f);
  }
  g0[i] = v;
  m0[i] = owner[i] == pos ? 1.0f : 0.0f;
}

__constant__ float kPyrK[5] = {1.0f / 16.0f, 4.0f / 16.0f, 6.0f / 16.0f, 4.0f / 16.0f, 1.0f / 16.0f};

// downsample_half_rgba_weighted / downsample_half_scalar, horizontal pass: row y
// of the (w x h) level into the (nw x h) intermediate.
__global__ void pano_down_h_kernel(const float4* __restrict__ src, const float* __restrict__ ms, int w, int h, int nw,
                                   float4* __restrict__ tmp, float* __restrict__ tms) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= nw) return;
  float r = 0.f, g = 0.f, b = 0.f, m = 0.f, vw = 0.f, s = 0.f;
  const long long row = (long long)y * w;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const int sx = min(max(2 * x + k - 2, 0), w - 1);
    const float4 p = src[row + sx];
    const float kw = kPyrK[k];
    m += kw * p.w;
    if (p.w > 0.0f) {
      const float v = kw * p.w;
      vw += v;
      r += v * p.x;
      g += v * p.y;
      b += v * p.z;
    }
    s += kw * ms[row + sx];
  }
  float4 o = make_float4(0.f, 0.f, 0.f, m);
  if (vw > 1e-6f) {
    const float inv = 1.0f / vw;
    o.x = r * inv;
    o.y = g * inv;
    o.z = b * inv;
  }
  tmp[(long long)y * nw + x] = o;
  tms[(long long)y * nw + x] = s;
}

// Vertical pass: the (nw x h) intermediate into the (nw x nh) next level.
__global__ void pano_down_v_kernel(const float4* __restrict__ tmp, const float* __restrict__ tms, int h, int nw,
                                   float4* __restrict__ dst, float* __restrict__ dms) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= nw) return;
  float r = 0.f, g = 0.f, b = 0.f, m = 0.f, vw = 0.f, s = 0.f;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const int sy = min(max(2 * y + k - 2, 0), h - 1);
    const long long i = (long long)sy * nw + x;
    const float4 p = tmp[i];
    const float kw = kPyrK[k];
    m += kw * p.w;
    if (p.w > 0.0f) {
      const float v = kw * p.w;
      vw += v;
      r += v * p.x;
      g += v * p.y;
      b += v * p.z;
    }
    s += kw * tms[i];
  }
  float4 o = make_float4(0.f, 0.f, 0.f, m);
  if (vw > 1e-6f) {
    const float inv = 1.0f / vw;
    o.x = r * inv;
    o.y = g * inv;
    o.z = b * inv;
  }
  dst[(long long)y * nw + x] = o;
  dms[(long long)y * nw + x] = s;
}

// upsample_to_size_rgb at (x, y) of the destination from the (sw x sh) source.
__device__ __forceinline__ float3 pano_up(const float4* __restrict__ src, int sw, int sh, int x, int y) {
  const float fy = clampf((float)y * 0.5f, 0.0f, (float)(sh - 1));
  const int y0 = min((int)floorf(fy), sh - 1), y1 = min(y0 + 1, sh - 1);
  const float wy1 = fy - (float)y0, wy0 = 1.0f - wy1;
  const float fx = clampf((float)x * 0.5f, 0.0f, (float)(sw - 1));
  const int x0 = min((int)floorf(fx), sw - 1), x1 = min(x0 + 1, sw - 1);
  const float wx1 = fx - (float)x0, wx0 = 1.0f - wx1;
  const float4 p00 = src[(long long)y0 * sw + x0], p10 = src[(long long)y0 * sw + x1];
  const float4 p01 = src[(long long)y1 * sw + x0], p11 = src[(long long)y1 * sw + x1];
  const float w00 = wx0 * wy0, w10 = wx1 * wy0, w01 = wx0 * wy1, w11 = wx1 * wy1;
  return make_float3(p00.x * w00 + p10.x * w10 + p01.x * w01 + p11.x * w11,
                     p00.y * w00 + p10.y * w10 + p01.y * w01 + p11.y * w11,
                     p00.z * w00 + p10.z * w10 + p01.z * w01 + p11.z * w11);
}

// One image's band at one level into the blend pyramid: the Laplacian
// (level - expanded next level) or, at the top level, the level itself.
__global__ void pano_accum_kernel(const float4* __restrict__ g, const float* __restrict__ m,
                                  const float4* __restrict__ g_next, int lw, int lh, int nw, int nh,
                                  float4* __restrict__ bl) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= lw) return;
  const long long i = (long long)y * lw + x;
  const float w = m[i];
  const float4 v = g[i];
  if (!(w > 0.0f && v.w > 1e-3f)) return;
  float3 lap = make_float3(v.x, v.y, v.z);
  if (g_next) {
    const float3 e = pano_up(g_next, nw, nh, x, y);
    lap = make_float3(v.x - e.x, v.y - e.y, v.z - e.z);
  }
  float4 o = bl[i];
  o.x += w * lap.x;
  o.y += w * lap.y;
  o.z += w * lap.z;
  o.w += w;
  bl[i] = o;
}

__global__ void pano_norm_kernel(float4* __restrict__ bl, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 o = bl[i];
  if (o.w > 1e-6f && fabsf(o.w - 1.0f) > 1e-5f) {
    const float inv = 1.0f / o.w;
    o.x *= inv;
    o.y *= inv;
    o.z *= inv;
    bl[i] = o;
  }
}

// recon_l = upsample(recon_{l+1}) + band_l, in place over band_l.
__global__ void pano_collapse_kernel(const float4* __restrict__ next, int nw, int nh, float4* __restrict__ bl, int lw,
                                     int lh) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= lw) return;
  const long long i = (long long)y * lw + x;
  const float3 u = pano_up(next, nw, nh, x, y);
  float4 o = bl[i];
  o.x = u.x + o.x;
  o.y = u.y + o.y;
  o.z = u.z + o.z;
  bl[i] = o;
}

__global__ void pano_final_kernel(const float4* __restrict__ rec, const int* __restrict__ owner, long long n,
                                  uint32_t* __restrict__ canvas) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t out = 0u;
  if (owner[i] >= 0) {
    const float4 v = rec[i];
    out = sat_u8((double)roundf(v.x)) | (sat_u8((double)roundf(v.y)) << 8) | (sat_u8((double)roundf(v.z)) << 16) |
          (255u << 24);
  }
  canvas[i] = out;
}

// ---------------------------------------------------------------- host helpers
inline dim3 row_grid(int w, int h) { return dim3((unsigned)((w + 255) / 256), (unsigned)h); }

bool invert_f32(const float* m, double out[9]) {  // invert_matrix_3x3
  double a[3][3];
  for (int i = 0; i < 9; ++i) a[i / 3][i % 3] = (double)m[i];
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
  if (std::fabs(det) < 1e-12 || !std::isfinite(det)) return false;
  const double id = 1.0 / det;
  const double r[9] = {c00 * id, c10 * id, c20 * id, c01 * id, c11 * id, c21 * id, c02 * id, c12 * id, c22 * id};
  std::memcpy(out, r, sizeof r);
  return true;
}

bool project_h(const double* m, double x, double y, double& px, double& py) {  // project_f64
  const double w = m[6] * x + m[7] * y + m[8];
  if (std::fabs(w) < 1e-7) return false;
  const double iw = 1.0 / w;
  px = (m[0] * x + m[1] * y + m[2]) * iw;
  py = (m[3] * x + m[4] * y + m[5]) * iw;
  return true;
}

bool sane_h(const float* m, int src_w, int src_h) {  // is_sane_homography_for_dims
  if (src_w < 2 || src_h < 2) return false;
  const double w = (double)(src_w - 1), ht = (double)(src_h - 1);
  const double corners[4][2] = {{0.0, 0.0}, {w, 0.0}, {w, ht}, {0.0, ht}};
  const double wc = (double)m[6] * (w * 0.5) + (double)m[7] * (ht * 0.5) + (double)m[8];
  if (!std::isfinite(wc) || std::fabs(wc) < 1e-6) return false;
  double P[4][2];
  for (int i = 0; i < 4; ++i) {
    const double cx = corners[i][0], cy = corners[i][1];
    const double wi = (double)m[6] * cx + (double)m[7] * cy + (double)m[8];
    if (!std::isfinite(wi) || wi * wc <= 0.0 || std::fabs(wi) < 0.1 * std::fabs(wc)) return false;
    const double px = ((double)m[0] * cx + (double)m[1] * cy + (double)m[2]) / wi;
    const double py = ((double)m[3] * cx + (double)m[4] * cy + (double)m[5]) / wi;
    if (!std::isfinite(px) || !std::isfinite(py)) return false;
    P[i][0] = px;
    P[i][1] = py;
  }
  int pos = 0, neg = 0;
  double shoelace = 0.0;
  for (int i = 0; i < 4; ++i) {
    const double* a = P[i];
    const double* b = P[(i + 1) % 4];
    const double* c = P[(i + 2) % 4];
    shoelace += a[0] * b[1] - b[0] * a[1];
    const double cross = (b[0] - a[0]) * (c[1] - b[1]) - (b[1] - a[1]) * (c[0] - b[0]);
    if (cross > 1e-3) ++pos;
    else if (cross < -1e-3) ++neg;
    else return false;
  }
  if (!(pos == 4 || neg == 4)) return false;
  const double area = 0.5 * std::fabs(shoelace), src_area = w * ht;
  return area >= 0.04 * src_area && area <= 25.0 * src_area;
}

// sample_patch_intensity on the luma plane (luma_to_array2's f32 values).
double patch_intensity(const uint8_t* luma, int h, int w, float x, float y) {
  if (h == 0 || w == 0 || !std::isfinite(x) || !std::isfinite(y)) return 0.0;
  auto to_i = [](float v) -> long long {  // Rust `as isize` of a finite value
    if (v >= 9.2e18f) return (long long)9.2e18;
    if (v <= -9.2e18f) return -(long long)9.2e18;
    return (long long)v;
  };
  auto clampll = [](long long v, long long lo, long long hi) { return v < lo ? lo : (v > hi ? hi : v); };
  const long long cx = clampll(to_i(std::round(x)), 0, w - 1), cy = clampll(to_i(std::round(y)), 0, h - 1);
  const long long y0 = cy > 0 ? cy - 1 : 0, y1 = std::min(cy + 1, (long long)h - 1);
  const long long x0 = cx > 0 ? cx - 1 : 0, x1 = std::min(cx + 1, (long long)w - 1);
  const float inv255 = 1.0f / 255.0f;
  double sum = 0.0;
  long long cnt = 0;
  for (long long yy = y0; yy <= y1; ++yy)
    for (long long xx = x0; xx <= x1; ++xx) {
      sum += (double)((float)luma[yy * w + xx] * inv255);
      ++cnt;
    }
  return cnt == 0 ? 0.0 : (sum / (double)cnt) * 255.0;
}

void compose_h(const double* a, const double* b, double* out) {  // compose_mat3
  double o[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) o[3 * r + c] = a[3 * r] * b[c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c];
  if (std::fabs(o[8]) > 1e-12) {
    const double inv = 1.0 / o[8];
    for (int i = 0; i < 9; ++i) o[i] *= inv;
  }
  std::memcpy(out, o, sizeof o);
}

// solve_exposure_gains: pairs (i, j, n_ij, mean_i, mean_j).
std::vector<float> solve_gains(const std::vector<std::array<double, 5>>& pairs, int n, int ref_idx, double sigma_n,
                               double sigma_g) {
  std::vector<float> out(n, 1.0f);
  if (n == 0) return out;
  std::vector<std::vector<double>> a(n, std::vector<double>(n, 0.0));
  std::vector<double> b(n, 0.0);
  const double sn = std::fmax(sigma_n, 1e-3), sg = std::fmax(sigma_g, 1e-3);
  const double inv_sn2 = 1.0 / (sn * sn), prior_w = 1.0 / (sg * sg);
  for (int i = 0; i < n; ++i) {
    a[i][i] += prior_w;
    b[i] += prior_w;
  }
  for (const auto& e : pairs) {
    const long long i = (long long)e[0], j = (long long)e[1];
    const double nij = e[2], mi = e[3], mj = e[4];
    if (i >= n || j >= n || i == j || nij <= 0.0) continue;
    const double w = nij * inv_sn2;
    a[i][i] += w * mi * mi;
    a[j][j] += w * mj * mj;
    const double cross = -w * mi * mj;
    a[i][j] += cross;
    a[j][i] += cross;
  }
  std::vector<double> g(n, 1.0);
  for (int col = 0; col < n; ++col) {
    int piv = col;
    double mx = std::fabs(a[col][col]);
    for (int r = col + 1; r < n; ++r)
      if (std::fabs(a[r][col]) > mx) {
        mx = std::fabs(a[r][col]);
        piv = r;
      }
    if (mx < 1e-12) return std::vector<float>(n, 1.0f);
    std::swap(a[col], a[piv]);
    std::swap(b[col], b[piv]);
    const double diag = a[col][col];
    for (int r = col + 1; r < n; ++r) {
      const double factor = a[r][col] / diag;
      a[r][col] = 0.0;
      for (int c = col + 1; c < n; ++c) a[r][c] -= factor * a[col][c];
      b[r] -= factor * b[col];
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int c = i + 1; c < n; ++c) s -= a[i][c] * g[c];
    g[i] = s / a[i][i];
  }
  const double rg = ref_idx < n ? g[ref_idx] : 1.0;
  const double norm = (std::isfinite(rg) && rg > 0.1) ? 1.0 / rg : 1.0;
  for (int i = 0; i < n; ++i) {
    const double sc = std::isfinite(g[i]) ? g[i] * norm : 1.0;
    const float f = (float)sc;
    out[i] = f < 0.4f ? 0.4f : (f > 2.5f ? 2.5f : f);
  }
  return out;
}

// The compositing stage on device-resident registered images.  The canvas
// (W x H RGBA8, *d_canvas) and every buffer come from the context's io arena.
psift_status composite(psift_ctx* ctx, const std::vector<PanoImg>& imgs, double ox, double oy, int W, int H, int blend,
                       int levels, uint32_t** d_canvas_out) {
  cudaStream_t st = ctx->stream;
  const int n = (int)imgs.size();
  const long long np = (long long)W * H;
  // level dimensions (multi-band)
  std::vector<std::pair<int, int>> dims;
  int nl = 1;
  if (blend == PSIFT_BLEND_MULTIBAND) {
    const int maxl = std::max((int)std::floor(std::log2((double)std::min(W, H))), 1);
    nl = std::min(std::min(std::max(levels, 1), 6), maxl);
  }
  int cw = W, ch = H;
  size_t bytes = align_up(sizeof(PanoImg) * std::max(n, 1), 256) + align_up((size_t)np * 4, 256) + 4096;
  if (blend == PSIFT_BLEND_MULTIBAND) bytes += align_up((size_t)np * 4, 256);  // owner
  for (int l = 0; l < nl; ++l) {
    dims.push_back({cw, ch});
    cw = std::max((cw + 1) / 2, 1);
    ch = std::max((ch + 1) / 2, 1);
  }
  // per level: colour + validity (g), blend accumulator (bl), seam mask (m); the
  // horizontal decimation's intermediate into level l is w_l x h_{l-1} (tmp, tm)
  auto tmp_px = [&](int l) { return l == 0 ? (size_t)1 : (size_t)dims[l].first * dims[l - 1].second; };
  if (blend == PSIFT_BLEND_MULTIBAND)
    for (int l = 0; l < nl; ++l) {
      const size_t c = (size_t)dims[l].first * dims[l].second;
      bytes += 2 * align_up(c * 16, 256) + align_up(c * 4, 256) + align_up(tmp_px(l) * 16, 256) +
               align_up(tmp_px(l) * 4, 256);
    }
  psift_status s = io_reserve(ctx, bytes);
  if (s != PSIFT_OK) return s;
  auto take = [&](size_t b) {
    const size_t off = align_up(ctx->io.offset, 256);
    ctx->io.offset = off + b;
    return (void*)(ctx->io.base + off);
  };
  PanoImg* d_imgs = (PanoImg*)take(sizeof(PanoImg) * std::max(n, 1));
  uint32_t* d_canvas = (uint32_t*)take((size_t)np * 4);
  *d_canvas_out = d_canvas;
  if (n) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_imgs, imgs.data(), sizeof(PanoImg) * n, cudaMemcpyHostToDevice, st));
  if (blend != PSIFT_BLEND_MULTIBAND) {
    pano_feather_kernel<<<row_grid(W, H), 256, 0, st>>>(d_imgs, n, ox, oy, W, H, d_canvas);
    ctx->launches++;
    PSIFT_CUDA_TRY(ctx, cudaGetLastError());
    return PSIFT_OK;
  }
  int* owner = (int*)take((size_t)np * 4);
  std::vector<float4*> g(nl), bl(nl), tmp(nl);
  std::vector<float*> m(nl), tm(nl);
  for (int l = 0; l < nl; ++l) {
    const size_t c = (size_t)dims[l].first * dims[l].second;
    g[l] = (float4*)take(c * 16);
    bl[l] = (float4*)take(c * 16);
    m[l] = (float*)take(c * 4);
    tmp[l] = (float4*)take(tmp_px(l) * 16);
    tm[l] = (float*)take(tmp_px(l) * 4);
  }
  if (ctx->io.offset > ctx->io.capacity) return set_error(ctx, PSIFT_ERR_INTERNAL, "panorama workspace overflow");
  pano_owner_kernel<<<row_grid(W, H), 256, 0, st>>>(d_imgs, n, ox, oy, W, H, owner);
  ctx->launches++;
  for (int l = 0; l < nl; ++l)
    PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(bl[l], 0, (size_t)dims[l].first * dims[l].second * 16, st));
  for (int pos = 0; pos < n; ++pos) {
    pano_warp_kernel<<<row_grid(W, H), 256, 0, st>>>(d_imgs, pos, owner, ox, oy, W, H, g[0], m[0]);
    ctx->launches++;
    for (int l = 1; l < nl; ++l) {
      const int pw = dims[l - 1].first, ph = dims[l - 1].second, nw = dims[l].first;
      pano_down_h_kernel<<<row_grid(nw, ph), 256, 0, st>>>(g[l - 1], m[l - 1], pw, ph, nw, tmp[l], tm[l]);
      pano_down_v_kernel<<<row_grid(nw, dims[l].second), 256, 0, st>>>(tmp[l], tm[l], ph, nw, g[l], m[l]);
      ctx->launches += 2;
    }
    for (int l = nl - 1; l >= 0; --l) {
      const bool top = l == nl - 1;
      pano_accum_kernel<<<row_grid(dims[l].first, dims[l].second), 256, 0, st>>>(
          g[l], m[l], top ? nullptr : g[l + 1], dims[l].first, dims[l].second, top ? 0 : dims[l + 1].first,
          top ? 0 : dims[l + 1].second, bl[l]);
      ctx->launches++;
    }
    PSIFT_CUDA_TRY(ctx, cudaGetLastError());
  }
  for (int l = 0; l < nl; ++l) {
    const long long c = (long long)dims[l].first * dims[l].second;
    pano_norm_kernel<<<(unsigned)((c + 255) / 256), 256, 0, st>>>(bl[l], c);
    ctx->launches++;
  }
  for (int l = nl - 2; l >= 0; --l) {
    pano_collapse_kernel<<<row_grid(dims[l].first, dims[l].second), 256, 0, st>>>(
        bl[l + 1], dims[l + 1].first, dims[l + 1].second, bl[l], dims[l].first, dims[l].second);
    ctx->launches++;
  }
  pano_final_kernel<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(bl[0], owner, np, d_canvas);
  ctx->launches++;
  PSIFT_CUDA_TRY(ctx, cudaGetLastError());
  return PSIFT_OK;
}

// Uploads n host RGBA8 images into the stitch arena (tight rows); returns their device pointers.
psift_status upload_images(psift_ctx* ctx, const psift_rgba_image* images, uint32_t n, std::vector<uint8_t*>& dev,
                           size_t extra_bytes) {
  size_t bytes = extra_bytes + 4096;
  for (uint32_t i = 0; i < n; ++i) bytes += align_up((size_t)images[i].height * images[i].width * 4, 256);
  psift_status s = stitch_reserve(ctx, bytes);
  if (s != PSIFT_OK) return s;
  dev.assign(n, nullptr);
  for (uint32_t i = 0; i < n; ++i) {
    const psift_rgba_image& I = images[i];
    const size_t off = align_up(ctx->stitch.offset, 256);
    ctx->stitch.offset = off + (size_t)I.height * I.width * 4;
    dev[i] = (uint8_t*)ctx->stitch.base + off;
    if (I.height && I.width)
      PSIFT_CUDA_TRY(ctx, cudaMemcpy2DAsync(dev[i], (size_t)I.width * 4, I.data, I.row_stride, (size_t)I.width * 4,
                                            I.height, cudaMemcpyHostToDevice, ctx->stream));
  }
  return PSIFT_OK;
}

void* stitch_take(psift_ctx* ctx, size_t bytes) {
  const size_t off = align_up(ctx->stitch.offset, 256);
  if (off + bytes > ctx->stitch.capacity) return nullptr;
  ctx->stitch.offset = off + bytes;
  return ctx->stitch.base + off;
}

psift_status check_images(psift_ctx* ctx, const psift_rgba_image* images, uint32_t n) {
  for (uint32_t i = 0; i < n; ++i) {
    const psift_rgba_image& I = images[i];
    if ((I.height && I.width && !I.data) || I.row_stride < (size_t)I.width * 4)
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null image or row stride below 4 x width");
    if ((uint64_t)I.height * I.width > (1ull << 31))
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "image larger than 2^31 pixels");
  }
  return PSIFT_OK;
}

struct Edge {
  int from, to;
  double h[9];
  int inliers;
  double mean_from, mean_to;
};

}  // namespace
}  // namespace psift

using namespace psift;

extern "C" {

void psift_panorama_options_default(psift_panorama_options* o) {
  if (!o) return;
  o->octaves = 3;
  o->scales = 3;
  o->threshold = 0.015f;         // DEFAULT_CONTRAST_THRESHOLD
  o->ratio = 0.75f;              // DEFAULT_MATCH_RATIO
  o->ransac_threshold = 3.0f;    // DEFAULT_RANSAC_REPROJ_THRESHOLD
  o->projection = PSIFT_PROJECTION_PLANAR;
  o->focal_px = 0.0f;
  o->blend = PSIFT_BLEND_MULTIBAND;
  o->levels = 4;
  o->exposure_compensation = 1;
  o->max_canvas_dim = (uint32_t)kPanoMaxDim;
  o->max_canvas_pixels = kPanoMaxPixels;
  o->tile_size = 512;
}

psift_status psift_warp_cylindrical(psift_ctx* ctx, const psift_rgba_image* image, float focal_px, uint8_t* out) {
  if (!ctx || !image || !out) return PSIFT_ERR_INVALID_ARGUMENT;
  psift_status s = check_images(ctx, image, 1);
  if (s != PSIFT_OK) return s;
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaSetDevice");
  const int h = (int)image->height, w = (int)image->width;
  if (!h || !w) return PSIFT_OK;
  std::vector<uint8_t*> dev;
  if ((s = upload_images(ctx, image, 1, dev, (size_t)h * w * 4 + 256)) != PSIFT_OK) return s;
  uint32_t* d_out = (uint32_t*)stitch_take(ctx, (size_t)h * w * 4);
  if (!d_out) return set_error(ctx, PSIFT_ERR_INTERNAL, "panorama workspace overflow");
  const double f = std::fmax(std::fmax((double)focal_px, (double)std::max(w, h) * 0.25), 16.0);
  cyl_warp_kernel<<<row_grid(w, h), 256, 0, ctx->stream>>>(dev[0], (long long)w * 4, h, w, f, ((double)w - 1.0) * 0.5,
                                                            ((double)h - 1.0) * 0.5, d_out);
  ctx->launches++;
  PSIFT_CUDA_TRY(ctx, cudaGetLastError());
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(out, d_out, (size_t)h * w * 4, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PSIFT_OK;
}

psift_status psift_panorama_composite(psift_ctx* ctx, const psift_rgba_image* images, uint32_t n,
                                      const uint8_t* registered, const float* gains, const double* inverses,
                                      double origin_x, double origin_y, uint32_t width, uint32_t height,
                                      int32_t blend, uint32_t levels, uint8_t* canvas) {
  if (!ctx || (n && (!images || !registered || !gains || !inverses)) || (width && height && !canvas))
    return PSIFT_ERR_INVALID_ARGUMENT;
  if (blend != PSIFT_BLEND_FEATHER && blend != PSIFT_BLEND_MULTIBAND)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "blend must be PSIFT_BLEND_FEATHER or PSIFT_BLEND_MULTIBAND");
  psift_status s = check_images(ctx, images, n);
  if (s != PSIFT_OK) return s;
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaSetDevice");
  const size_t cbytes = (size_t)width * height * 4;
  if (!cbytes) return PSIFT_OK;
  std::vector<uint8_t*> dev;
  if ((s = upload_images(ctx, images, n, dev, 0)) != PSIFT_OK) return s;
  uint32_t* d_canvas = nullptr;
  std::vector<PanoImg> imgs;
  for (uint32_t i = 0; i < n; ++i)
    if (registered[i]) {
      PanoImg P{dev[i], (long long)images[i].width * 4, (int)images[i].height, (int)images[i].width, {}, gains[i]};
      std::memcpy(P.inv, inverses + 9 * (size_t)i, sizeof P.inv);
      imgs.push_back(P);
    }
  if ((s = composite(ctx, imgs, origin_x, origin_y, (int)width, (int)height, blend, (int)levels, &d_canvas)) !=
      PSIFT_OK)
    return s;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(canvas, d_canvas, cbytes, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PSIFT_OK;
}

psift_status psift_stitch_panorama(psift_ctx* ctx, const psift_rgba_image* images, uint32_t n,
                                   const psift_panorama_options* opt, uint8_t* canvas, size_t canvas_capacity,
                                   psift_panorama_info* info, uint8_t* registered_out, float* gains_out,
                                   float* homographies_out) {
  if (!ctx || !opt || !info || (n && !images)) return PSIFT_ERR_INVALID_ARGUMENT;
  std::memset(info, 0, sizeof *info);
  info->reference_index = -1;
  if (n < 2) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "Panorama stitching requires at least 2 input images");
  if (opt->blend != PSIFT_BLEND_FEATHER && opt->blend != PSIFT_BLEND_MULTIBAND)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "blend must be PSIFT_BLEND_FEATHER or PSIFT_BLEND_MULTIBAND");
  if (opt->projection != PSIFT_PROJECTION_PLANAR && opt->projection != PSIFT_PROJECTION_CYLINDRICAL)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "projection must be planar or cylindrical");
  psift_status s = check_images(ctx, images, n);
  if (s != PSIFT_OK) return s;
  psift_sift_config cfg;
  psift_sift_config_default(&cfg);
  cfg.octaves = opt->octaves;
  cfg.scales = opt->scales;
  cfg.contrast_threshold = opt->threshold;
  cfg.upsample_first_octave = 1;  // extract_sift_features: DEFAULT_UPSAMPLE_FIRST_OCTAVE
  cfg.max_features = PSIFT_MAX_FEATURES_PER_IMAGE;
  char msg[256];
  if ((s = psift_sift_config_validate(&cfg, msg, sizeof msg)) != PSIFT_OK) return set_error(ctx, s, msg);
  psift_match_options mopt;
  psift_match_options_default(&mopt);
  mopt.ratio = opt->ratio;
  if ((s = psift_match_options_validate(&mopt, msg, sizeof msg)) != PSIFT_OK) return set_error(ctx, s, msg);
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaSetDevice");
  cudaStream_t st = ctx->stream;
  const int N = (int)n;
  const int cap = (int)PSIFT_MAX_FEATURES_PER_IMAGE;
  const int n_pairs = N * (N - 1) / 2;
  // ---- stitch arena: prepared images, luma, features, matches, RANSAC outputs
  // (upload_images adds the uploaded images themselves)
  size_t extra = 0;
  for (int i = 0; i < N; ++i) {
    const size_t px = (size_t)images[i].height * images[i].width;
    extra += align_up(px * 4, 256) + align_up(px + 1, 256);  // cylindrical output, luma
  }
  extra += (size_t)N * (align_up((size_t)cap * 4, 256) * 5 + align_up((size_t)cap * 512, 256) +
                        align_up((size_t)cap * 8, 256)) + align_up((size_t)N * 4, 256);
  extra += align_up((size_t)std::max(n_pairs, 1) * 4, 256);
  extra += (size_t)n_pairs * (align_up((size_t)cap * sizeof(psift_match), 256) + 2 * align_up((size_t)cap, 256) +
                              3 * 256);
  extra += 8192;
  std::vector<uint8_t*> raw;
  if ((s = upload_images(ctx, images, n, raw, extra)) != PSIFT_OK) return s;
  std::vector<uint8_t*> prep(N), luma(N);
  std::vector<int> hs(N), ws(N);
  for (int i = 0; i < N; ++i) {
    hs[i] = (int)images[i].height;
    ws[i] = (int)images[i].width;
    prep[i] = raw[i];
    if (opt->projection == PSIFT_PROJECTION_CYLINDRICAL && hs[i] && ws[i]) {
      prep[i] = (uint8_t*)stitch_take(ctx, (size_t)hs[i] * ws[i] * 4);
      if (!prep[i]) return set_error(ctx, PSIFT_ERR_INTERNAL, "panorama workspace overflow");
      const double f = std::fmax(std::fmax((double)opt->focal_px, (double)std::max(ws[i], hs[i]) * 0.25), 16.0);
      cyl_warp_kernel<<<row_grid(ws[i], hs[i]), 256, 0, st>>>(raw[i], (long long)ws[i] * 4, hs[i], ws[i], f,
                                                               ((double)ws[i] - 1.0) * 0.5,
                                                               ((double)hs[i] - 1.0) * 0.5, (uint32_t*)prep[i]);
      ctx->launches++;
    }
    luma[i] = (uint8_t*)stitch_take(ctx, (size_t)hs[i] * ws[i] + 1);
    if (!luma[i]) return set_error(ctx, PSIFT_ERR_INTERNAL, "panorama workspace overflow");
    if (hs[i] && ws[i]) {
      rgba_luma_kernel<<<row_grid(ws[i], hs[i]), 256, 0, st>>>(prep[i], (long long)ws[i] * 4, hs[i], ws[i], luma[i]);
      ctx->launches++;
    }
  }
  PSIFT_CUDA_TRY(ctx, cudaGetLastError());
  // ---- features: one batch call over every image's luma
  std::vector<psift_image_u8> lims(N);
  std::vector<psift_features> feats(N);
  std::vector<float*> fxy(N);
  for (int i = 0; i < N; ++i) {
    lims[i] = psift_image_u8{luma[i], (uint32_t)hs[i], (uint32_t)ws[i], (size_t)ws[i]};
    psift_features& F = feats[i];
    F.capacity = (uint32_t)cap;
    F.count = 0;
    F.x = (float*)stitch_take(ctx, (size_t)cap * 4);
    F.y = (float*)stitch_take(ctx, (size_t)cap * 4);
    F.scale = (float*)stitch_take(ctx, (size_t)cap * 4);
    F.response = (float*)stitch_take(ctx, (size_t)cap * 4);
    F.orientation = (float*)stitch_take(ctx, (size_t)cap * 4);
    F.descriptors = (float*)stitch_take(ctx, (size_t)cap * 512);
    fxy[i] = (float*)stitch_take(ctx, (size_t)cap * 8);
  }
  uint32_t* d_counts = (uint32_t*)stitch_take(ctx, (size_t)N * 4);
  if (!d_counts) return set_error(ctx, PSIFT_ERR_INTERNAL, "panorama workspace overflow");
  if ((s = psift_detect_and_compute_batch_dev(ctx, lims.data(), n, &cfg, feats.data(), d_counts)) != PSIFT_OK)
    return s;
  std::vector<uint32_t> nf(N);
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(nf.data(), d_counts, 4 * (size_t)N, cudaMemcpyDeviceToHost, st));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  // interleaved (x, y) for the matcher
  for (int i = 0; i < N; ++i)
    if (nf[i]) {
      PSIFT_CUDA_TRY(ctx, cudaMemcpy2DAsync(fxy[i], 8, feats[i].x, 4, 4, nf[i], cudaMemcpyDeviceToDevice, st));
      PSIFT_CUDA_TRY(ctx, cudaMemcpy2DAsync(fxy[i] + 1, 8, feats[i].y, 4, 4, nf[i], cudaMemcpyDeviceToDevice, st));
    }
  // ---- every pair (i < j): matching in one batch
  std::vector<std::pair<int, int>> pairs;
  std::vector<psift_match_job> mjobs;
  std::vector<psift_match*> mout;
  uint32_t* d_mcount = (uint32_t*)stitch_take(ctx, (size_t)std::max(n_pairs, 1) * 4);
  for (int i = 0; i < N; ++i)
    for (int j = i + 1; j < N; ++j) {
      psift_match* o = (psift_match*)stitch_take(ctx, (size_t)cap * sizeof(psift_match));
      if (!o || !d_mcount) return set_error(ctx, PSIFT_ERR_INTERNAL, "panorama workspace overflow");
      const int k = (int)pairs.size();
      pairs.push_back({i, j});
      mout.push_back(o);
      mjobs.push_back(psift_match_job{feats[i].descriptors, feats[j].descriptors, fxy[i], fxy[j], nf[i], nf[j], o,
                                      (uint32_t)cap, d_mcount + k});
    }
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(d_mcount, 0, (size_t)n_pairs * 4, st));
  if ((s = psift_match_batch_dev(ctx, mjobs.data(), (uint32_t)n_pairs, &mopt)) != PSIFT_OK) return s;
  std::vector<uint32_t> mc(n_pairs);
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(mc.data(), d_mcount, 4 * (size_t)n_pairs, cudaMemcpyDeviceToHost, st));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  // ---- similarity and homography RANSAC of every pair with >= 6 matches
  struct PairOut {
    uint8_t *smask, *hmask;
    float* model;  // 6 similarity + 9 homography
    int32_t* has;  // [0] similarity [1] homography
    uint32_t* cnt; // [0] [1]
  };
  std::vector<PairOut> po(n_pairs);
  std::vector<psift_ransac_job> sj, hj;
  std::vector<int> rp;
  for (int k = 0; k < n_pairs; ++k) {
    if (mc[k] < 6) continue;
    PairOut& P = po[k];
    P.smask = (uint8_t*)stitch_take(ctx, cap);
    P.hmask = (uint8_t*)stitch_take(ctx, cap);
    P.model = (float*)stitch_take(ctx, 64);
    P.has = (int32_t*)stitch_take(ctx, 8);
    P.cnt = (uint32_t*)stitch_take(ctx, 8);
    if (!P.cnt) return set_error(ctx, PSIFT_ERR_INTERNAL, "panorama workspace overflow");
    sj.push_back(psift_ransac_job{mout[k], mc[k], P.smask, P.model, P.has, P.cnt, nullptr, nullptr});
    hj.push_back(psift_ransac_job{mout[k], mc[k], P.hmask, P.model + 6, P.has + 1, P.cnt + 1, nullptr, nullptr});
    rp.push_back(k);
  }
  psift_ransac_options ropt;
  psift_ransac_options_default(&ropt);
  ropt.reproj_threshold = opt->ransac_threshold;
  if (!sj.empty()) {
    if ((s = psift_ransac_batch_dev(ctx, sj.data(), (uint32_t)sj.size(), &ropt, 0)) != PSIFT_OK) return s;
    if ((s = psift_ransac_batch_dev(ctx, hj.data(), (uint32_t)hj.size(), &ropt, 1)) != PSIFT_OK) return s;
  }
  // ---- results to the host
  std::vector<std::vector<uint8_t>> hluma(N);
  for (int i = 0; i < N; ++i) {
    hluma[i].resize((size_t)hs[i] * ws[i] + 1);
    if (hs[i] && ws[i])
      PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hluma[i].data(), luma[i], (size_t)hs[i] * ws[i], cudaMemcpyDeviceToHost, st));
  }
  struct HostPair {
    std::vector<psift_match> m;
    std::vector<uint8_t> smask, hmask;
    float model[16];
    int32_t has[2];
    uint32_t cnt[2];
  };
  std::vector<HostPair> hp(n_pairs);
  for (int k : rp) {
    HostPair& H = hp[k];
    H.m.resize(mc[k]);
    H.smask.resize(mc[k]);
    H.hmask.resize(mc[k]);
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(H.m.data(), mout[k], sizeof(psift_match) * mc[k], cudaMemcpyDeviceToHost, st));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(H.smask.data(), po[k].smask, mc[k], cudaMemcpyDeviceToHost, st));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(H.hmask.data(), po[k].hmask, mc[k], cudaMemcpyDeviceToHost, st));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(H.model, po[k].model, 60, cudaMemcpyDeviceToHost, st));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(H.has, po[k].has, 8, cudaMemcpyDeviceToHost, st));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(H.cnt, po[k].cnt, 8, cudaMemcpyDeviceToHost, st));
  }
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  // ---- pair edges (src/stitch.rs:530-600)
  std::vector<Edge> edges;
  for (int k : rp) {
    const HostPair& H = hp[k];
    const int i = pairs[k].first, j = pairs[k].second;
    const int ns = (int)H.cnt[0], nh = (int)H.cnt[1];
    const std::vector<uint8_t>& best = nh >= ns ? H.hmask : H.smask;
    const int nb = nh >= ns ? nh : ns;
    if (nb < 6) continue;
    float hij[9];
    const float* h9 = H.model + 6;
    if (H.has[1] && nh >= 6 && sane_h(h9, ws[i], hs[i])) {
      std::memcpy(hij, h9, sizeof hij);
    } else if (H.has[0]) {
      const float* sm = H.model;
      const float r[9] = {sm[0], -sm[1], sm[2], sm[1], sm[0], sm[3], 0.0f, 0.0f, 1.0f};
      std::memcpy(hij, r, sizeof hij);
    } else {
      continue;
    }
    double hji[9];
    if (!invert_f32(hij, hji)) continue;
    double si = 0.0, sj2 = 0.0;
    for (size_t q = 0; q < H.m.size(); ++q)
      if (best[q]) {
        si += patch_intensity(hluma[i].data(), hs[i], ws[i], H.m[q].query_x, H.m[q].query_y);
        sj2 += patch_intensity(hluma[j].data(), hs[j], ws[j], H.m[q].target_x, H.m[q].target_y);
      }
    const double ic = 1.0 / (double)nb;
    const double mi = std::fmax(si * ic, 1.0), mj = std::fmax(sj2 * ic, 1.0);
    Edge e1{i, j, {}, nb, mi, mj}, e2{j, i, {}, nb, mj, mi};
    for (int q = 0; q < 9; ++q) e1.h[q] = (double)hij[q], e2.h[q] = hji[q];
    edges.push_back(e1);
    edges.push_back(e2);
  }
  if (edges.empty()) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "No valid overlapping image pairs could be matched");
  std::vector<std::vector<Edge>> adj(N);
  for (const Edge& e : edges) adj[e.from].push_back(e);
  // largest connected component (the first of the largest), BFS order
  std::vector<char> visited(N, 0);
  std::vector<int> comp_best;
  for (int s0 = 0; s0 < N; ++s0) {
    if (visited[s0] || adj[s0].empty()) continue;
    std::vector<int> comp;
    std::deque<int> q;
    visited[s0] = 1;
    q.push_back(s0);
    while (!q.empty()) {
      const int u = q.front();
      q.pop_front();
      comp.push_back(u);
      for (const Edge& e : adj[u])
        if (!visited[e.to]) {
          visited[e.to] = 1;
          q.push_back(e.to);
        }
    }
    if (comp.size() > comp_best.size()) comp_best = comp;
  }
  if (comp_best.size() < 2)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "Could not form a connected panorama graph of >= 2 images");
  // reference image: the largest (total inliers, index)
  int ref = -1;
  long long best_w = -1;
  for (int u : comp_best) {
    long long wsum = 0;
    for (const Edge& e : adj[u]) wsum += e.inliers;
    if (wsum > best_w || (wsum == best_w && u > ref)) {
      best_w = wsum;
      ref = u;
    }
  }
  // Prim's maximum spanning tree rooted at the reference
  std::vector<char> has(N, 0);
  std::vector<double> Hr(9 * (size_t)N, 0.0);
  has[ref] = 1;
  const double I3[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  std::memcpy(&Hr[9 * (size_t)ref], I3, sizeof I3);
  for (size_t it = 1; it < comp_best.size(); ++it) {
    const Edge* be = nullptr;
    for (int u : comp_best) {
      if (!has[u]) continue;
      for (const Edge& e : adj[u])
        if (!has[e.to] && (!be || e.inliers > be->inliers)) be = &e;
    }
    if (!be) break;
    const int parent = be->from, child = be->to;
    const Edge* rev = nullptr;
    for (const Edge& e : adj[child])
      if (e.to == parent) {
        rev = &e;
        break;
      }
    compose_h(&Hr[9 * (size_t)parent], rev->h, &Hr[9 * (size_t)child]);
    has[child] = 1;
  }
  std::vector<int> reg;
  for (int i = 0; i < N; ++i)
    if (has[i]) reg.push_back(i);
  // exposure gains over the registered component's edges
  std::vector<float> gains(N, 1.0f);
  if (opt->exposure_compensation) {
    std::map<std::pair<int, int>, std::array<double, 3>> seen;
    for (int u : reg)
      for (const Edge& e : adj[u])
        if (has[e.to]) {
          const bool lt = e.from < e.to;
          seen[lt ? std::make_pair(e.from, e.to) : std::make_pair(e.to, e.from)] = {
              (double)e.inliers, lt ? e.mean_from : e.mean_to, lt ? e.mean_to : e.mean_from};
        }
    std::vector<std::array<double, 5>> pr;
    for (const auto& kv : seen)
      pr.push_back({(double)kv.first.first, (double)kv.first.second, kv.second[0], kv.second[1], kv.second[2]});
    gains = solve_gains(pr, N, ref, 10.0, 0.25);
  }
  // union bounding box in reference coordinates
  double min_x = INFINITY, min_y = INFINITY, max_x = -INFINITY, max_y = -INFINITY;
  std::vector<double> inv(9 * (size_t)N, 0.0);
  std::vector<float> h32(9 * (size_t)N, 0.0f);
  for (int idx : reg) {
    const double* hm = &Hr[9 * (size_t)idx];
    for (int q = 0; q < 9; ++q) h32[9 * (size_t)idx + q] = (float)hm[q];
    char buf[160];
    if (!invert_f32(&h32[9 * (size_t)idx], &inv[9 * (size_t)idx])) {
      snprintf(buf, sizeof buf, "Registered image %d has singular homography", idx);
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, buf);
    }
    const double w = std::fmax((double)ws[idx] - 1.0, 0.0), hh = std::fmax((double)hs[idx] - 1.0, 0.0);
    const double cs[4][2] = {{0.0, 0.0}, {w, 0.0}, {0.0, hh}, {w, hh}};
    for (const auto& c : cs) {
      double px, py;
      if (!project_h(hm, c[0], c[1], px, py)) {
        snprintf(buf, sizeof buf, "Projected corner hit infinity for image %d", idx);
        return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, buf);
      }
      if (!std::isfinite(px) || !std::isfinite(py)) {
        snprintf(buf, sizeof buf, "Non-finite projected corner for image %d", idx);
        return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, buf);
      }
      min_x = std::fmin(min_x, px);
      min_y = std::fmin(min_y, py);
      max_x = std::fmax(max_x, px);
      max_y = std::fmax(max_y, py);
    }
  }
  const double ox = std::floor(min_x), oy = std::floor(min_y);
  const double wf = std::fmax(std::ceil(max_x) - ox + 1.0, 1.0), hf = std::fmax(std::ceil(max_y) - oy + 1.0, 1.0);
  if (wf > (double)opt->max_canvas_dim || hf > (double)opt->max_canvas_dim || wf * hf > (double)opt->max_canvas_pixels) {
    char buf[200];
    snprintf(buf, sizeof buf, "Panorama canvas size %llux%llu exceeds safety limits (%u dim, %llu px)",
             (unsigned long long)wf, (unsigned long long)hf, opt->max_canvas_dim,
             (unsigned long long)opt->max_canvas_pixels);
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, buf);
  }
  info->width = (uint32_t)wf;
  info->height = (uint32_t)hf;
  info->reference_index = ref;
  info->registered_count = (int32_t)reg.size();
  info->origin_x = ox;
  info->origin_y = oy;
  for (int i = 0; i < N; ++i) {
    if (registered_out) registered_out[i] = has[i];
    if (gains_out) gains_out[i] = gains[i];
    if (homographies_out) std::memcpy(homographies_out + 9 * (size_t)i, &h32[9 * (size_t)i], 36);
  }
  const size_t cbytes = (size_t)info->width * info->height * 4;
  if (!canvas) return PSIFT_OK;
  if (canvas_capacity < cbytes) return set_error(ctx, PSIFT_ERR_CAPACITY, "canvas capacity below width x height x 4");
  // ---- compositing
  uint32_t* d_canvas = nullptr;
  std::vector<PanoImg> imgs;
  for (int i : reg) {
    PanoImg P{prep[i], (long long)ws[i] * 4, hs[i], ws[i], {}, gains[i]};
    std::memcpy(P.inv, &inv[9 * (size_t)i], sizeof P.inv);
    imgs.push_back(P);
  }
  if ((s = composite(ctx, imgs, ox, oy, (int)info->width, (int)info->height, opt->blend, (int)opt->levels,
                     &d_canvas)) != PSIFT_OK)
    return s;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(canvas, d_canvas, cbytes, cudaMemcpyDeviceToHost, st));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PSIFT_OK;
}

}  // extern "C"
