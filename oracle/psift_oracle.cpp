// psift_oracle.cpp -- CPU restatement of pure-sift 0.2.0's feature hot path.
//
// TEST INFRASTRUCTURE ONLY (the checker, never the product).  Pinning and the
// arithmetic rules are described in psift_oracle.h.  Every function names the
// reference lines it restates (paths are relative to the pure-sift project).
//
// Parallelism: OpenMP over exactly the loops the reference hands to rayon
// (blur rows, DoG slices, gradient levels, keypoints, queries, catalog entries).
// Every parallel loop writes disjoint, pre-sized outputs, so results are
// identical for any thread count (reference property: tests/invariance_sweeps.rs:219-244).
#include "psift_oracle.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <array>
#include <deque>
#include <map>
#include <limits>
#include <vector>

namespace {

constexpr float BASE_SIGMA = 1.6f;            // src/pipeline.rs:10
constexpr float PI_F = 3.14159265358979323846f;
constexpr size_t DESC_LEN = 128;              // src/pipeline.rs:1000
constexpr float RAD_TO_DEG_F = 57.2957795130823208767981548141051703f;
constexpr int PAR_MIN_PIXELS = 16384;         // src/pipeline.rs:381,:410,:901

// The detection path (pyramid, extrema, orientations, descriptors) is written
// once over the arithmetic type T.  T = float is the restatement of the
// reference's f32 arithmetic; T = double runs the same algorithm with every
// value, constant and libm call in f64, the yardstick that the f32 results
// (the reference's and the GPU's) state their error against.  lit<T>(f, d)
// picks the f32 literal as written in the reference for float and the same
// decimal constant in f64 for double.
template <typename T> constexpr T lit(float f, double d);
template <> constexpr float lit<float>(float f, double) { return f; }
template <> constexpr double lit<double>(float, double d) { return d; }
#define K(x) lit<T>(x##f, x)

template <typename T> constexpr T base_sigma() { return K(1.6); }           // src/pipeline.rs:10
template <typename T> constexpr T assumed_input_sigma() { return K(0.5); }  // src/pipeline.rs:13
template <typename T> constexpr T pi_t() { return K(3.14159265358979323846); }
template <typename T> constexpr T sqrt_2_t() { return K(1.41421356237309504880); }
template <typename T> constexpr T secondary_ori_peak_ratio() { return K(0.80); }  // src/pipeline.rs:1155

template <typename T>
struct PlaneT {
  int h = 0, w = 0;
  std::vector<T> d;
  PlaneT() = default;
  PlaneT(int hh, int ww) : h(hh), w(ww), d((size_t)hh * ww, T(0)) {}
  T* row(int y) { return d.data() + (size_t)y * w; }
  const T* row(int y) const { return d.data() + (size_t)y * w; }
};
using Plane = PlaneT<float>;

template <typename T>
struct OctaveT {
  std::vector<PlaneT<T>> g, dog;
  T scale_factor = T(1);
};
using Octave = OctaveT<float>;

// Keypoint record: the C struct for f32, the same fields in f64 otherwise.
struct keypoint_f64 {
  double x, y, scale, response;
  uint32_t octave, layer;
};
template <typename T> struct KpOf { using type = oracle_keypoint; };
template <> struct KpOf<double> { using type = keypoint_f64; };
template <typename T> using KpT = typename KpOf<T>::type;

// Rust `f32::rem_euclid` / `f64::rem_euclid`: r = a % b; if r < 0 { r + |b| } else { r }.
template <typename T> inline T rem_euclid(T a, T b) {
  T r = std::fmod(a, b);
  return r < T(0) ? r + std::fabs(b) : r;
}
inline float rem_euclid_f(float a, float b) { return rem_euclid<float>(a, b); }

// Rust `clamp(lo, hi)`.
template <typename T> inline T clampt(T x, T lo, T hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
inline float clampf(float x, float lo, float hi) { return clampt<float>(x, lo, hi); }

// Rust `as isize` / `as usize` from a float: saturating, NaN -> 0.
template <typename T> inline long long to_i_sat(T v) {
  if (std::isnan(v)) return 0;
  if (v >= T(9.2233720368547758e18)) return std::numeric_limits<long long>::max();
  if (v <= T(-9.2233720368547758e18)) return std::numeric_limits<long long>::min();
  return (long long)v;
}
template <typename T> inline unsigned long long to_u_sat(T v) {
  if (std::isnan(v) || v <= T(0)) return 0;
  if (v >= T(1.8446744073709552e19)) return std::numeric_limits<unsigned long long>::max();
  return (unsigned long long)v;
}
inline long long f2i_sat(float v) { return to_i_sat<float>(v); }
inline unsigned long long f2u_sat(float v) { return to_u_sat<float>(v); }
inline unsigned long long d2u_sat(double v) { return to_u_sat<double>(v); }

// `f32::powi(i32)` / `f64::powi` lower to the compiler runtime's binary
// exponentiation (square-and-multiply, low bit first); restated here.
template <typename T> inline T powi_t(T a, int b) {
  const bool recip = b < 0;
  T r = T(1);
  for (;;) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? T(1) / r : r;
}
inline float powi_f(float a, int b) { return powi_t<float>(a, b); }
inline double powi_d(double a, int b) { return powi_t<double>(a, b); }

// src/pipeline.rs:275-296
template <typename T>
std::vector<T> gaussian_kernel_1d(T sigma) {
  const T cs = std::fmax(sigma, K(1e-3));
  long long radius = to_i_sat<T>(std::ceil(K(3.0) * cs));
  if (radius < 1) radius = 1;
  const T two_sigma_sq = K(2.0) * cs * cs;
  const T norm_factor = K(1.0) / (std::sqrt(K(2.0) * pi_t<T>()) * cs);
  std::vector<T> k;
  k.reserve((size_t)(2 * radius + 1));
  for (long long x = -radius; x <= radius; ++x) {
    const T xf = (T)x;
    k.push_back(norm_factor * std::exp(-((xf * xf) / two_sigma_sq)));
  }
  T sum = T(0);
  for (T v : k) sum += v;
  if (sum > T(0)) {
    const T inv = K(1.0) / sum;
    for (T& v : k) v *= inv;
  }
  return k;
}

// src/pipeline.rs:314-425 (horizontal pass :329-377, vertical AXPY pass :395-406).
template <typename T>
PlaneT<T> gaussian_blur(const PlaneT<T>& img, T sigma) {
  const int h = img.h, w = img.w;
  if (h == 0 || w == 0) return PlaneT<T>(h, w);
  const std::vector<T> kernel = gaussian_kernel_1d<T>(sigma);
  const int klen = (int)kernel.size();
  const int radius = klen / 2;
  const bool par = (long long)h * w >= PAR_MIN_PIXELS;

  PlaneT<T> temp(h, w);
#pragma omp parallel for schedule(static) if (par)
  for (int y = 0; y < h; ++y) {
    const T* in_row = img.row(y);
    T* out_row = temp.row(y);
    for (int x = 0; x < w; ++x) {
      T acc = T(0);
      for (int k = 0; k < klen; ++k) {
        int sx = x + k - radius;            // (x + k).saturating_sub(r).min(w-1)
        if (sx < 0) sx = 0;
        if (sx > w - 1) sx = w - 1;
        acc += in_row[sx] * kernel[k];
      }
      out_row[x] = acc;
    }
  }

  PlaneT<T> dst(h, w);
#pragma omp parallel for schedule(static) if (par)
  for (int y = 0; y < h; ++y) {
    T* out_row = dst.row(y);
    for (int k = 0; k < klen; ++k) {
      int sy = y + k - radius;
      if (sy < 0) sy = 0;
      if (sy > h - 1) sy = h - 1;
      const T* in_row = temp.row(sy);
      const T wgt = kernel[k];
      for (int x = 0; x < w; ++x) out_row[x] += in_row[x] * wgt;
    }
  }
  return dst;
}

// src/pipeline.rs:429-449
template <typename T>
PlaneT<T> downsample_2x(const PlaneT<T>& img) {
  const int nh = img.h / 2, nw = img.w / 2;
  if (nh == 0 || nw == 0) return PlaneT<T>(0, 0);
  PlaneT<T> out(nh, nw);
  for (int y = 0; y < nh; ++y)
    for (int x = 0; x < nw; ++x) out.row(y)[x] = img.row(2 * y)[2 * x];
  return out;
}

// src/pipeline.rs:455-483
template <typename T>
PlaneT<T> upsample_2x_bilinear(const PlaneT<T>& img) {
  const int h = img.h, w = img.w;
  const int nh = h * 2, nw = w * 2;
  if (nh == 0 || nw == 0) return PlaneT<T>(0, 0);
  PlaneT<T> out(nh, nw);
  for (int uy = 0; uy < nh; ++uy) {
    const int y0 = uy / 2;
    const int y1 = std::min(y0 + (uy & 1), h - 1);
    const T* r0 = img.row(y0);
    const T* r1 = img.row(y1);
    T* o = out.row(uy);
    for (int ux = 0; ux < nw; ++ux) {
      const int x0 = ux / 2;
      const int x1 = std::min(x0 + (ux & 1), w - 1);
      o[ux] = K(0.25) * (r0[x0] + r0[x1] + r1[x0] + r1[x1]);
    }
  }
  return out;
}

// src/pipeline.rs:550-638
template <typename T>
std::vector<OctaveT<T>> build_pyramid(const PlaneT<T>& img, int octaves, int scales, bool upsample) {
  std::vector<OctaveT<T>> pyr;
  if (img.h == 0 || img.w == 0 || octaves == 0 || scales == 0) return pyr;
  const int dog_slices = scales + 2;
  const T k = std::pow(K(2.0), K(1.0) / (T)scales);
  const T bs = base_sigma<T>();

  PlaneT<T> base;
  T base_mult;
  if (upsample) {
    PlaneT<T> up = upsample_2x_bilinear(img);
    const T sigma_in = K(2.0) * assumed_input_sigma<T>();
    const T init_sigma = std::sqrt(std::fmax(bs * bs - sigma_in * sigma_in, K(1e-4)));
    base = gaussian_blur(up, init_sigma);
    base_mult = K(0.5);
  } else {
    const T sigma_in = assumed_input_sigma<T>();
    const T init_sigma = std::sqrt(std::fmax(bs * bs - sigma_in * sigma_in, K(1e-4)));
    base = gaussian_blur(img, init_sigma);
    base_mult = K(1.0);
  }

  for (int o = 0; o < octaves; ++o) {
    const int h = base.h, w = base.w;
    if (h < 3 || w < 3) break;
    OctaveT<T> oct;
    oct.g.push_back(base);
    T prev_sigma = bs;
    for (int s = 1; s <= dog_slices; ++s) {
      const T target = bs * powi_t<T>(k, s);
      const T delta = std::sqrt(std::fmax(target * target - prev_sigma * prev_sigma, K(1e-4)));
      PlaneT<T> next = gaussian_blur(oct.g.back(), delta);
      PlaneT<T> dog(h, w);
      const PlaneT<T>& prev = oct.g.back();
      for (size_t i = 0; i < dog.d.size(); ++i) dog.d[i] = next.d[i] - prev.d[i];
      oct.dog.push_back(std::move(dog));
      oct.g.push_back(std::move(next));
      prev_sigma = target;
    }
    if (o + 1 < octaves) base = downsample_2x(oct.g[scales]);
    else base = oct.g.back();
    oct.scale_factor = base_mult * (T)(1ull << o);
    pyr.push_back(std::move(oct));
  }
  return pyr;
}

// src/pipeline.rs:664-687
template <typename T>
bool passes_hessian_edge_test(const PlaneT<T>& c, int x, int y, T center) {
  const T* rp = c.row(y - 1);
  const T* rc = c.row(y);
  const T* rn = c.row(y + 1);
  const T dxx = rc[x + 1] - K(2.0) * center + rc[x - 1];
  const T dyy = rn[x] - K(2.0) * center + rp[x];
  const T dxy = K(0.25) * ((rn[x + 1] - rn[x - 1]) - (rp[x + 1] - rp[x - 1]));
  const T trace = dxx + dyy;
  const T det = dxx * dyy - dxy * dxy;
  const T threshold_ratio = (K(11.0) * K(11.0)) / K(10.0);
  return det > K(1e-9) && (trace * trace) < threshold_ratio * det;
}

// src/pipeline.rs:697-770
template <typename T>
void refine_extremum_3d(const PlaneT<T>& p, const PlaneT<T>& c, const PlaneT<T>& n, int x, int y, T& ox_out,
                        T& oy_out, T& os_out, T& interp_out) {
  const T* c_prev = c.row(y - 1);
  const T* c_curr = c.row(y);
  const T* c_next = c.row(y + 1);
  const T* p_prev = p.row(y - 1);
  const T* p_curr = p.row(y);
  const T* p_next = p.row(y + 1);
  const T* n_prev = n.row(y - 1);
  const T* n_curr = n.row(y);
  const T* n_next = n.row(y + 1);
  const T center = c_curr[x];

  const T gx = K(0.5) * (c_curr[x + 1] - c_curr[x - 1]);
  const T gy = K(0.5) * (c_next[x] - c_prev[x]);
  const T gs = K(0.5) * (n_curr[x] - p_curr[x]);

  const T dxx = c_curr[x + 1] - K(2.0) * center + c_curr[x - 1];
  const T dyy = c_next[x] - K(2.0) * center + c_prev[x];
  const T dss = n_curr[x] - K(2.0) * center + p_curr[x];

  const T dxy = K(0.25) * ((c_next[x + 1] - c_next[x - 1]) - (c_prev[x + 1] - c_prev[x - 1]));
  const T dxs = K(0.25) * ((n_curr[x + 1] - n_curr[x - 1]) - (p_curr[x + 1] - p_curr[x - 1]));
  const T dys = K(0.25) * ((n_next[x] - n_prev[x]) - (p_next[x] - p_prev[x]));

  const T c00 = dyy * dss - dys * dys;
  const T c01 = dys * dxs - dxy * dss;
  const T c02 = dxy * dys - dyy * dxs;
  const T c11 = dxx * dss - dxs * dxs;
  const T c12 = dxy * dxs - dxx * dys;
  const T c22 = dxx * dyy - dxy * dxy;

  const T det3 = dxx * c00 + dxy * c01 + dxs * c02;
  if (std::fabs(det3) > K(1e-9)) {
    const T inv_det = K(-1.0) / det3;
    const T ox = (c00 * gx + c01 * gy + c02 * gs) * inv_det;
    const T oy = (c01 * gx + c11 * gy + c12 * gs) * inv_det;
    const T os = (c02 * gx + c12 * gy + c22 * gs) * inv_det;
    if (std::fabs(ox) <= K(0.5) && std::fabs(oy) <= K(0.5) && std::fabs(os) <= K(0.5)) {
      ox_out = ox;
      oy_out = oy;
      os_out = os;
      interp_out = center + K(0.5) * (gx * ox + gy * oy + gs * os);
      return;
    }
  }
  if (std::fabs(c22) > K(1e-9)) {
    const T inv_det2 = K(-1.0) / c22;
    const T ox = clampt<T>((dyy * gx - dxy * gy) * inv_det2, K(-0.5), K(0.5));
    const T oy = clampt<T>((-dxy * gx + dxx * gy) * inv_det2, K(-0.5), K(0.5));
    const T os = std::fabs(dss) > K(1e-6) ? clampt<T>(-gs / dss, K(-0.5), K(0.5)) : T(0);
    ox_out = ox;
    oy_out = oy;
    os_out = os;
    interp_out = center + K(0.5) * (gx * ox + gy * oy + gs * os);
    return;
  }
  ox_out = oy_out = os_out = T(0);
  interp_out = center;
}

template <typename T>
inline bool gt_patch(const PlaneT<T>& pl, int x, int y, T v) {
  const T* r0 = pl.row(y - 1);
  const T* r1 = pl.row(y);
  const T* r2 = pl.row(y + 1);
  return v > r0[x - 1] && v > r0[x] && v > r0[x + 1] && v > r1[x - 1] && v > r1[x] &&
         v > r1[x + 1] && v > r2[x - 1] && v > r2[x] && v > r2[x + 1];
}
template <typename T>
inline bool lt_patch(const PlaneT<T>& pl, int x, int y, T v) {
  const T* r0 = pl.row(y - 1);
  const T* r1 = pl.row(y);
  const T* r2 = pl.row(y + 1);
  return v < r0[x - 1] && v < r0[x] && v < r0[x + 1] && v < r1[x - 1] && v < r1[x] &&
         v < r1[x + 1] && v < r2[x - 1] && v < r2[x] && v < r2[x + 1];
}

// src/pipeline.rs:810-916
template <typename T>
void extract_extrema_in_octave(int octave_idx, const std::vector<PlaneT<T>>& dogs, T mult,
                               T threshold, std::vector<KpT<T>>& out) {
  if (dogs.size() < 3) return;
  const int h = dogs[0].h, w = dogs[0].w;
  if (h < 3 || w < 3) return;
  const int searchable = std::max((int)dogs.size() - 2, 1);
  const T k = std::pow(K(2.0), K(1.0) / (T)searchable);
  const int nslices = (int)dogs.size() - 2;
  std::vector<std::vector<KpT<T>>> per_slice(nslices);
  const bool par = (long long)h * w >= PAR_MIN_PIXELS;

#pragma omp parallel for schedule(dynamic, 1) if (par)
  for (int si = 0; si < nslices; ++si) {
    const int s = si + 1;
    const PlaneT<T>& prev = dogs[s - 1];
    const PlaneT<T>& curr = dogs[s];
    const PlaneT<T>& next = dogs[s + 1];
    const T eff_scale = base_sigma<T>() * mult * powi_t<T>(k, s);
    auto& kps = per_slice[si];
    for (int y = 1; y < h - 1; ++y) {
      const T* ra = curr.row(y - 1);
      const T* rc = curr.row(y);
      const T* rb = curr.row(y + 1);
      for (int x = 1; x < w - 1; ++x) {
        const T v = rc[x];
        if (std::fabs(v) <= threshold) continue;
        bool ext;
        if (v > T(0)) {
          ext = v > rc[x - 1] && v > rc[x + 1] && v > ra[x - 1] && v > ra[x] && v > ra[x + 1] &&
                v > rb[x - 1] && v > rb[x] && v > rb[x + 1] && gt_patch(prev, x, y, v) &&
                gt_patch(next, x, y, v);
        } else {
          ext = v < rc[x - 1] && v < rc[x + 1] && v < ra[x - 1] && v < ra[x] && v < ra[x + 1] &&
                v < rb[x - 1] && v < rb[x] && v < rb[x + 1] && lt_patch(prev, x, y, v) &&
                lt_patch(next, x, y, v);
        }
        if (ext && passes_hessian_edge_test(curr, x, y, v)) {
          T dx, dy, ds, interp;
          refine_extremum_3d(prev, curr, next, x, y, dx, dy, ds, interp);
          if (std::fabs(interp) > threshold) {
            const T refined_scale = eff_scale * std::pow(k, ds);
            const T lf = clampt<T>(std::round((T)s + ds), K(1.0), (T)searchable);
            KpT<T> kp;
            kp.x = ((T)x + dx) * mult;
            kp.y = ((T)y + dy) * mult;
            kp.scale = std::fmax(refined_scale, K(0.25) * base_sigma<T>());
            kp.response = interp;
            kp.octave = (uint32_t)octave_idx;
            kp.layer = (uint32_t)to_u_sat<T>(lf);
            kps.push_back(kp);
          }
        }
      }
    }
  }
  for (auto& v : per_slice) out.insert(out.end(), v.begin(), v.end());
}

// src/pipeline.rs:535-547
template <typename T>
std::vector<KpT<T>> pyramid_extract(const std::vector<OctaveT<T>>& pyr, T thr) {
  std::vector<KpT<T>> kps;
  for (size_t o = 0; o < pyr.size(); ++o)
    extract_extrema_in_octave<T>((int)o, pyr[o].dog, pyr[o].scale_factor, thr, kps);
  return kps;
}

// src/pipeline.rs:1158-1203
template <typename T>
struct GradPlanesT {
  int octave, layer, w, h;
  std::vector<T> mag, ang;
};
template <typename T>
GradPlanesT<T> gradient_planes(int octave, int layer, const PlaneT<T>& g) {
  GradPlanesT<T> gp;
  gp.octave = octave;
  gp.layer = layer;
  gp.w = g.w;
  gp.h = g.h;
  gp.mag.assign((size_t)g.h * g.w, T(0));
  gp.ang.assign((size_t)g.h * g.w, T(0));
  const T two_pi = K(2.0) * pi_t<T>();
  if (g.h >= 3 && g.w >= 3) {
    for (int y = 1; y < g.h - 1; ++y) {
      const T* ra = g.row(y - 1);
      const T* rc = g.row(y);
      const T* rb = g.row(y + 1);
      for (int x = 1; x < g.w - 1; ++x) {
        const T dx = rc[x + 1] - rc[x - 1];
        const T dy = rb[x] - ra[x];
        gp.mag[(size_t)y * g.w + x] = std::sqrt(dx * dx + dy * dy);
        gp.ang[(size_t)y * g.w + x] = rem_euclid<T>(std::atan2(dy, dx), two_pi);
      }
    }
  }
  return gp;
}

// src/pipeline.rs:1206-1227
template <typename T>
void resolve_octave_and_layer(const KpT<T>& kp, const std::vector<OctaveT<T>>& pyr, int& oct, int& layer) {
  if (pyr.empty()) {
    oct = layer = 0;
    return;
  }
  const int nocts = (int)pyr.size();
  if (kp.layer > 0) {
    oct = std::min((int)kp.octave, nocts - 1);
  } else {
    const T ratio = std::fmax(kp.scale / base_sigma<T>(), K(1.0));
    oct = (int)std::min<unsigned long long>(to_u_sat<T>(std::floor(std::log2(ratio))),
                                            (unsigned long long)(nocts - 1));
  }
  const int g_len = (int)pyr[oct].g.size();
  const int searchable = std::max(g_len - 3, 1);
  if (kp.layer > 0) {
    layer = std::min((int)kp.layer, g_len - 1);
  } else {
    const T oct_mult = (T)(1ull << oct);
    const T local_sigma = std::fmax(kp.scale / (base_sigma<T>() * oct_mult), K(1.0));
    const unsigned long long l = to_u_sat<T>(std::round(std::log2(local_sigma) * (T)searchable));
    const int hi = std::max(g_len - 2, 1);
    layer = (int)std::min<unsigned long long>(std::max<unsigned long long>(l, 1ull), (unsigned long long)hi);
  }
}

// src/pipeline.rs:1233-1347
template <typename T>
std::vector<T> keypoint_orientations(const GradPlanesT<T>& gp, const KpT<T>& kp) {
  const int NB = 36;
  const T two_pi = K(2.0) * pi_t<T>();
  const T sigma_ori = std::fmax(K(1.5) * kp.scale, K(1.0));
  const T two_sigma_sq = K(2.0) * sigma_ori * sigma_ori;
  long long radius = to_i_sat<T>(std::ceil(K(3.0) * sigma_ori));
  if (radius < 2) radius = 2;
  const long long cx = to_i_sat<T>(std::round(kp.x));
  const long long cy = to_i_sat<T>(std::round(kp.y));
  T hist[NB] = {0};
  const T bin_scale = (T)NB / two_pi;
  const long long H = gp.h, W = gp.w;
  const long long y_min = std::max(cy - radius, 1ll);
  const long long y_max = std::max(std::min(cy + radius, H - 2), 1ll);
  const long long x_min = std::max(cx - radius, 1ll);
  const long long x_max = std::max(std::min(cx + radius, W - 2), 1ll);
  const T r_sq_max = (T)(radius * radius);
  for (long long y = y_min; y <= y_max; ++y) {
    const T dy = (T)(y - cy);
    for (long long x = x_min; x <= x_max; ++x) {
      const T dx = (T)(x - cx);
      const T r_sq = dx * dx + dy * dy;
      if (r_sq > r_sq_max) continue;
      const T m = gp.mag[(size_t)(y * W + x)];
      if (m <= K(1e-7)) continue;
      const T weight = std::exp(-r_sq / two_sigma_sq);
      const T ang = gp.ang[(size_t)(y * W + x)];
      const int bin = (int)(to_u_sat<T>(std::floor(ang * bin_scale)) % NB);
      hist[bin] += m * weight;
    }
  }
  T sm[NB];
  for (int b = 0; b < NB; ++b) {
    const T prev = hist[(b + NB - 1) % NB];
    const T curr = hist[b];
    const T next = hist[(b + 1) % NB];
    sm[b] = (prev + curr + next) * (K(1.0) / K(3.0));
  }
  int best_bin = 0;
  T best_val = sm[0];
  for (int b = 1; b < NB; ++b)
    if (sm[b] > best_val) {
      best_val = sm[b];
      best_bin = b;
    }
  if (best_val <= K(1e-7)) return {T(0)};
  const T split = secondary_ori_peak_ratio<T>() * best_val;
  std::vector<std::pair<int, T>> peaks;
  for (int b = 0; b < NB; ++b) {
    const T v = sm[b];
    if (v < split) continue;
    const T l = sm[(b + NB - 1) % NB];
    const T r = sm[(b + 1) % NB];
    if (v > l && v >= r) peaks.push_back({b, v});
  }
  if (peaks.empty()) {
    peaks.push_back({best_bin, best_val});
  } else {
    std::stable_sort(peaks.begin(), peaks.end(), [](const auto& a, const auto& b) {
      if (b.second > a.second) return false;  // b.1.partial_cmp(a.1): a before b iff b.1 < a.1
      if (b.second < a.second) return true;
      return a.first < b.first;
    });
    if (peaks.size() > 4) peaks.resize(4);
  }
  std::vector<T> oris;
  for (const auto& pk : peaks) {
    const int bin = pk.first;
    const T val = pk.second;
    const T l = sm[(bin + NB - 1) % NB];
    const T r = sm[(bin + 1) % NB];
    const T denom = l - K(2.0) * val + r;
    T off = std::fabs(denom) > K(1e-6) ? K(0.5) * (l - r) / denom : T(0);
    off = clampt<T>(off, K(-0.5), K(0.5));
    oris.push_back(rem_euclid<T>((((T)bin + K(0.5)) + off) * (two_pi / (T)NB), two_pi));
  }
  return oris;
}

// src/pipeline.rs:1352-1480
template <typename T>
void descriptor_128(const GradPlanesT<T>& gp, const KpT<T>& kp, T orientation, T* desc) {
  const int GW = 4;
  const T two_pi = K(2.0) * pi_t<T>();
  std::fill(desc, desc + DESC_LEN, T(0));
  if (gp.w < 3 || gp.h < 3) return;
  const T cos_t = std::cos(orientation);
  const T sin_t = std::sin(orientation);
  const T hist_width = std::fmax(K(3.0) * kp.scale, K(1.5));
  const T inv_hw = K(1.0) / hist_width;
  const T exp_scale = K(-1.0) / (K(2.0) * K(2.0) * K(2.0));
  long long max_radius = to_i_sat<T>(std::ceil(hist_width * sqrt_2_t<T>() * ((T)GW + K(1.0)) * K(0.5)));
  if (max_radius < 4) max_radius = 4;
  const long long cx = to_i_sat<T>(std::round(kp.x));
  const long long cy = to_i_sat<T>(std::round(kp.y));
  const long long H = gp.h, W = gp.w;
  const long long y_min = std::max(cy - max_radius, 1ll);
  const long long y_max = std::max(std::min(cy + max_radius, H - 2), 1ll);
  const long long x_min = std::max(cx - max_radius, 1ll);
  const long long x_max = std::max(std::min(cx + max_radius, W - 2), 1ll);
  const T bin_per_rad = K(8.0) / two_pi;
  for (long long y = y_min; y <= y_max; ++y) {
    const T dy = (T)y - kp.y;
    for (long long x = x_min; x <= x_max; ++x) {
      const T dx = (T)x - kp.x;
      const T r_rot = (dx * cos_t + dy * sin_t) * inv_hw;
      const T c_rot = (-dx * sin_t + dy * cos_t) * inv_hw;
      const T r_bin = r_rot + (T)GW * K(0.5) - K(0.5);
      const T c_bin = c_rot + (T)GW * K(0.5) - K(0.5);
      if (r_bin <= K(-1.0) || r_bin >= (T)GW || c_bin <= K(-1.0) || c_bin >= (T)GW) continue;
      const T m = gp.mag[(size_t)(y * W + x)];
      if (m <= K(1e-7)) continue;
      const T w_gauss = std::exp((r_rot * r_rot + c_rot * c_rot) * exp_scale);
      const T wm = m * w_gauss;
      const T rel = rem_euclid<T>(gp.ang[(size_t)(y * W + x)] - orientation, two_pi);
      const T o_bin = rel * bin_per_rad;
      const long long r0 = to_i_sat<T>(std::floor(r_bin));
      const long long c0 = to_i_sat<T>(std::floor(c_bin));
      const long long o0 = to_i_sat<T>(std::floor(o_bin));
      const T dr = r_bin - (T)r0;
      const T dc = c_bin - (T)c0;
      const T dof = o_bin - (T)o0;
      for (int ir = 0; ir <= 1; ++ir) {
        const long long rb = r0 + ir;
        if (rb < 0 || rb >= GW) continue;
        const T wr = ir == 0 ? K(1.0) - dr : dr;
        for (int ic = 0; ic <= 1; ++ic) {
          const long long cb = c0 + ic;
          if (cb < 0 || cb >= GW) continue;
          const T wc = ic == 0 ? K(1.0) - dc : dc;
          for (int io = 0; io <= 1; ++io) {
            long long ob = (o0 + io) % 8;
            if (ob < 0) ob += 8;
            const T wo = io == 0 ? K(1.0) - dof : dof;
            const size_t idx = (size_t)((rb * GW + cb) * 8 + ob);
            desc[idx] += wm * wr * wc * wo;
          }
        }
      }
    }
  }
  T n1 = T(0);
  for (size_t i = 0; i < DESC_LEN; ++i) n1 += desc[i] * desc[i];
  n1 = std::sqrt(n1);
  if (n1 > K(1e-7)) {
    const T inv1 = K(1.0) / n1;
    for (size_t i = 0; i < DESC_LEN; ++i) desc[i] = std::fmin(desc[i] * inv1, K(0.2));
    T n2 = T(0);
    for (size_t i = 0; i < DESC_LEN; ++i) n2 += desc[i] * desc[i];
    n2 = std::sqrt(n2);
    if (n2 > K(1e-7)) {
      const T inv2 = K(1.0) / n2;
      for (size_t i = 0; i < DESC_LEN; ++i) desc[i] *= inv2;
    }
  }
}

// src/pipeline.rs:1012-1019
template <typename T>
void rootsift(const T* d, T* out) {
  T l1 = T(0);
  for (size_t i = 0; i < DESC_LEN; ++i) l1 += std::fmax(d[i], T(0));
  if (l1 <= K(1e-7)) {
    std::memmove(out, d, DESC_LEN * sizeof(T));
    return;
  }
  const T inv = K(1.0) / l1;
  for (size_t i = 0; i < DESC_LEN; ++i) out[i] = std::sqrt(std::fmax(d[i], T(0)) * inv);
}

template <typename T>
struct FeatureT {
  T x, y, scale, response, orientation;
  T desc[DESC_LEN];
};

// src/pipeline.rs:1482-1577
template <typename T>
std::vector<FeatureT<T>> describe_from_pyramid(const std::vector<OctaveT<T>>& pyr,
                                               const std::vector<KpT<T>>& kps, int kind) {
  std::vector<FeatureT<T>> feats;
  if (pyr.empty() || kps.empty()) return feats;
  std::vector<std::pair<int, int>> levels;
  for (const auto& kp : kps) {
    int o, l;
    resolve_octave_and_layer<T>(kp, pyr, o, l);
    if (std::find(levels.begin(), levels.end(), std::make_pair(o, l)) == levels.end())
      levels.push_back({o, l});
  }
  std::vector<GradPlanesT<T>> cache(levels.size());
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < (int)levels.size(); ++i)
    cache[i] = gradient_planes<T>(levels[i].first, levels[i].second, pyr[levels[i].first].g[levels[i].second]);

  std::vector<std::vector<FeatureT<T>>> per_kp(kps.size());
#pragma omp parallel for schedule(dynamic, 16)
  for (long long i = 0; i < (long long)kps.size(); ++i) {
    const KpT<T>& kp = kps[i];
    int o, l;
    resolve_octave_and_layer<T>(kp, pyr, o, l);
    const GradPlanesT<T>* gp = nullptr;
    for (const auto& c : cache)
      if (c.octave == o && c.layer == l) {
        gp = &c;
        break;
      }
    const T oct_mult = pyr[o].scale_factor;
    const T inv = K(1.0) / oct_mult;
    KpT<T> okp;
    okp.x = kp.x * inv;
    okp.y = kp.y * inv;
    okp.scale = std::fmax(kp.scale * inv, K(0.5) * base_sigma<T>());
    okp.response = kp.response;
    okp.octave = (uint32_t)o;
    okp.layer = (uint32_t)l;
    const std::vector<T> oris = keypoint_orientations<T>(*gp, okp);
    for (T ori : oris) {
      FeatureT<T> f;
      f.x = kp.x;
      f.y = kp.y;
      f.scale = kp.scale;
      f.response = kp.response;
      f.orientation = ori;
      T raw[DESC_LEN];
      descriptor_128<T>(*gp, okp, ori, raw);
      if (kind == 1) rootsift<T>(raw, f.desc);
      else std::memcpy(f.desc, raw, sizeof(raw));
      per_kp[i].push_back(f);
    }
  }
  for (auto& v : per_kp) feats.insert(feats.end(), v.begin(), v.end());
  return feats;
}

template <typename T>
PlaneT<T> make_plane(const T* img, int h, int w) {
  PlaneT<T> p(h, w);
  std::memcpy(p.d.data(), img, sizeof(T) * (size_t)h * w);
  return p;
}

template <typename T>
int write_features(const std::vector<FeatureT<T>>& f, T* meta, T* desc, int cap) {
  const int n = (int)f.size();
  for (int i = 0; i < n && i < cap; ++i) {
    if (meta) {
      meta[5 * i + 0] = f[i].x;
      meta[5 * i + 1] = f[i].y;
      meta[5 * i + 2] = f[i].scale;
      meta[5 * i + 3] = f[i].response;
      meta[5 * i + 4] = f[i].orientation;
    }
    if (desc) std::memcpy(desc + (size_t)i * DESC_LEN, f[i].desc, sizeof(T) * DESC_LEN);
  }
  return n;
}

// src/pipeline.rs:1633-1658.  max_features = 0 disables the cap (the reference
// always caps at MAX_FEATURES_PER_IMAGE = 4096, src/pipeline.rs:1054).
template <typename T>
int detect_and_compute_t(const PlaneT<T>& img, int octaves, int scales, T thr, int upsample, int kind,
                         int max_features, T* meta, T* desc, int cap) {
  const auto pyr = build_pyramid<T>(img, octaves, scales, upsample != 0);
  auto kps = pyramid_extract<T>(pyr, thr);
  if (max_features > 0 && (int)kps.size() > max_features) {
    std::stable_sort(kps.begin(), kps.end(), [](const KpT<T>& a, const KpT<T>& b) {
      return std::fabs(b.response) < std::fabs(a.response);
    });
    kps.resize(max_features);
  }
  auto feats = describe_from_pyramid<T>(pyr, kps, kind);
  if (max_features > 0 && (int)feats.size() > max_features) feats.resize(max_features);
  return write_features<T>(feats, meta, desc, cap);
}

#undef K

// ---------------------------------------------------------------- matching
// src/pipeline.rs:1700-1717
inline float dist_sq_early_exit(const float* a, const float* b, float cutoff) {
  float sum = 0.0f;
  for (int c = 0; c < 4; ++c) {
    for (int i = 0; i < 32; ++i) {
      const float d = a[c * 32 + i] - b[c * 32 + i];
      sum += d * d;
    }
    if (sum >= cutoff) return sum;
  }
  return sum;
}

// ---------------------------------------------------------------- RANSAC
uint64_t splitmix64(uint64_t& s) {  // src/pipeline.rs:1862-1868
  s += 0x9E3779B97F4A7C15ull;
  uint64_t z = s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// src/pipeline.rs:1873-1897
void eval_similarity(const oracle_match* m, int n, float a, float b, float tx, float ty,
                     float thresh_sq, size_t& count, float& err_sum) {
  count = 0;
  err_sum = 0.0f;
  for (int i = 0; i < n; ++i) {
    const float px = a * m[i].qx - b * m[i].qy + tx;
    const float py = b * m[i].qx + a * m[i].qy + ty;
    const float dx = px - m[i].tx;
    const float dy = py - m[i].ty;
    const float e = dx * dx + dy * dy;
    if (e <= thresh_sq) {
      ++count;
      err_sum += e;
    }
  }
}

struct Sim {
  float a, b, tx, ty, scale, rot;
};

// src/pipeline.rs:1900-1975
bool procrustes(const std::vector<oracle_match>& in, Sim& out) {
  if (in.empty()) return false;
  if (in.size() == 1) {
    out = {1.0f, 0.0f, in[0].dx, in[0].dy, 1.0f, 0.0f};
    return true;
  }
  const float inv_n = 1.0f / (float)in.size();
  float mqx = 0, mqy = 0, mtx = 0, mty = 0;
  for (const auto& m : in) {
    mqx += m.qx;
    mqy += m.qy;
    mtx += m.tx;
    mty += m.ty;
  }
  mqx *= inv_n;
  mqy *= inv_n;
  mtx *= inv_n;
  mty *= inv_n;
  float sqq = 0, na = 0, nb = 0;
  for (const auto& m : in) {
    const float qx = m.qx - mqx, qy = m.qy - mqy, tx = m.tx - mtx, ty = m.ty - mty;
    sqq += qx * qx + qy * qy;
    na += qx * tx + qy * ty;
    nb += qx * ty - qy * tx;
  }
  float a = 1.0f, b = 0.0f;
  if (sqq > 1e-5f) {
    const float af = na / sqq, bf = nb / sqq;
    const float s2 = af * af + bf * bf;
    if (s2 >= 0.04f && s2 <= 25.0f) {
      a = af;
      b = bf;
    }
  }
  out.a = a;
  out.b = b;
  out.tx = mtx - (a * mqx - b * mqy);
  out.ty = mty - (b * mqx + a * mqy);
  out.scale = std::sqrt(a * a + b * b);
  out.rot = std::atan2(b, a) * RAD_TO_DEG_F;
  return true;
}

// src/pipeline.rs:1979-2002
size_t adaptive_iters(size_t inl, size_t total, int ss, double conf, size_t min_it, size_t cap) {
  if (total == 0 || inl == 0) return cap;
  double w = (double)inl / (double)total;
  if (w < 1e-3) w = 1e-3;
  if (w > 1.0 - 1e-6) w = 1.0 - 1e-6;
  double p = powi_d(w, ss);
  if (p < 1e-12) p = 1e-12;
  if (p > 1.0 - 1e-9) p = 1.0 - 1e-9;
  const double num = std::log(1.0 - conf);
  const double den = std::log(1.0 - p);
  if (std::fabs(den) < 1e-12) return min_it;
  const double est = std::ceil(num / den);
  if (!std::isfinite(est)) return cap;
  size_t e = (size_t)d2u_sat(est);
  if (e < min_it) e = min_it;
  if (e > cap) e = cap;
  return e;
}

// src/pipeline.rs:2006-2026
std::vector<double> ratio_cdf(const oracle_match* m, int n) {
  std::vector<double> cdf;
  cdf.reserve(n);
  double acc = 0.0;
  for (int i = 0; i < n; ++i) {
    double r = 1.0;
    if (std::isfinite(m[i].ratio)) {
      r = (double)m[i].ratio;
      if (r < 0.05) r = 0.05;
      if (r > 1.0) r = 1.0;
    }
    acc += 1.0 / r;
    cdf.push_back(acc);
  }
  if (acc > 0.0) {
    const double inv = 1.0 / acc;
    for (double& v : cdf) v *= inv;
  }
  if (!cdf.empty()) cdf.back() = 1.0;
  return cdf;
}

// src/pipeline.rs:2029-2036
size_t sample_weighted(const std::vector<double>& cdf, uint64_t& st) {
  const double u = (double)(splitmix64(st) >> 11) * (1.0 / (double)(1ull << 53));
  size_t lo = (size_t)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
  const size_t hi = cdf.empty() ? 0 : cdf.size() - 1;
  return std::min(lo, hi);
}

// src/pipeline.rs:2055-2191
int similarity_ransac(const oracle_match* m, int n, float thr, uint64_t seed, std::vector<uint8_t>& mask,
                      Sim& model, bool& has_model) {
  mask.assign(n, 0);
  has_model = false;
  if (n == 0) return 0;
  if (n == 1) {
    std::vector<oracle_match> v(m, m + 1);
    has_model = procrustes(v, model);
    mask[0] = 1;
    return 1;
  }
  const float thresh = std::fmax(thr, 0.5f);
  const float tsq = thresh * thresh;
  std::vector<int> sorted(n);
  for (int i = 0; i < n; ++i) sorted[i] = i;
  std::stable_sort(sorted.begin(), sorted.end(), [&](int i, int j) { return m[i].ratio < m[j].ratio; });

  float ba = 1.0f, bb = 0.0f, btx = m[sorted[0]].dx, bty = m[sorted[0]].dy;
  size_t best_count;
  float best_err;
  eval_similarity(m, n, ba, bb, btx, bty, tsq, best_count, best_err);
  for (int i = 0; i < n && i < 32; ++i) {
    const int idx = sorted[i];
    size_t c;
    float e;
    eval_similarity(m, n, 1.0f, 0.0f, m[idx].dx, m[idx].dy, tsq, c, e);
    if (c > best_count || (c == best_count && e < best_err)) {
      best_count = c;
      best_err = e;
      ba = 1.0f;
      bb = 0.0f;
      btx = m[idx].dx;
      bty = m[idx].dy;
    }
  }
  const std::vector<double> cdf = ratio_cdf(m, n);
  uint64_t rng = seed;
  const size_t hard_cap = 1000, min_iters = 64;
  size_t max_iters = adaptive_iters(best_count, n, 2, 0.999, min_iters, hard_cap);
  size_t iter = 0;
  while (iter < max_iters) {
    ++iter;
    const size_t i1 = sample_weighted(cdf, rng);
    size_t i2 = sample_weighted(cdf, rng);
    if (i2 == i1) i2 = (i1 + 1) % n;
    const oracle_match& m1 = m[i1];
    const oracle_match& m2 = m[i2];
    const float dxq = m2.qx - m1.qx, dyq = m2.qy - m1.qy;
    const float dq = dxq * dxq + dyq * dyq;
    if (dq < 16.0f) continue;
    const float dxt = m2.tx - m1.tx, dyt = m2.ty - m1.ty;
    const float a = (dxq * dxt + dyq * dyt) / dq;
    const float b = (dxq * dyt - dyq * dxt) / dq;
    const float s2 = a * a + b * b;
    if (!(s2 >= 0.04f && s2 <= 25.0f)) continue;
    const float tx = m1.tx - (a * m1.qx - b * m1.qy);
    const float ty = m1.ty - (b * m1.qx + a * m1.qy);
    size_t c;
    float e;
    eval_similarity(m, n, a, b, tx, ty, tsq, c, e);
    if (c > best_count || (c == best_count && e < best_err)) {
      best_count = c;
      best_err = e;
      ba = a;
      bb = b;
      btx = tx;
      bty = ty;
      max_iters = adaptive_iters(best_count, n, 2, 0.999, min_iters, hard_cap);
    }
  }
  std::vector<oracle_match> inl;
  std::vector<uint8_t> inl_mask(n, 0);
  for (int i = 0; i < n; ++i) {
    const float dx = (ba * m[i].qx - bb * m[i].qy + btx) - m[i].tx;
    const float dy = (bb * m[i].qx + ba * m[i].qy + bty) - m[i].ty;
    if (dx * dx + dy * dy <= tsq) {
      inl.push_back(m[i]);
      inl_mask[i] = 1;
    }
  }
  Sim refined;
  const bool has_refined = procrustes(inl, refined);
  if (has_refined) {
    std::vector<oracle_match> rin;
    std::vector<uint8_t> rmask(n, 0);
    for (int i = 0; i < n; ++i) {
      const float dx = (refined.a * m[i].qx - refined.b * m[i].qy + refined.tx) - m[i].tx;
      const float dy = (refined.b * m[i].qx + refined.a * m[i].qy + refined.ty) - m[i].ty;
      if (dx * dx + dy * dy <= tsq) {
        rin.push_back(m[i]);
        rmask[i] = 1;
      }
    }
    if (rin.size() >= inl.size()) {
      inl = std::move(rin);
      inl_mask = std::move(rmask);
    }
  }
  Sim fin;
  if (procrustes(inl, fin)) {
    model = fin;
    has_model = true;
  } else if (has_refined) {
    model = refined;
    has_model = true;
  }
  mask = inl_mask;
  return (int)inl.size();
}

using H3 = double[3][3];

// src/pipeline.rs:2276-2353
bool smallest_eigvec9(double a[9][9], double h[9]) {
  double v[9][9] = {{0}};
  for (int i = 0; i < 9; ++i) v[i][i] = 1.0;
  for (int sweep = 0; sweep < 20; ++sweep) {
    double max_off = 0.0;
    for (int p = 0; p < 9; ++p)
      for (int q = p + 1; q < 9; ++q)
        if (std::fabs(a[p][q]) > max_off) max_off = std::fabs(a[p][q]);
    if (max_off < 1e-13) break;
    for (int p = 0; p < 8; ++p)
      for (int q = p + 1; q < 9; ++q) {
        const double apq = a[p][q];
        if (std::fabs(apq) < 1e-15) continue;
        const double app = a[p][p], aqq = a[q][q];
        const double tau = (aqq - app) / (2.0 * apq);
        const double t = tau >= 0.0 ? 1.0 / (tau + std::sqrt(1.0 + tau * tau))
                                    : -1.0 / (-tau + std::sqrt(1.0 + tau * tau));
        const double c = 1.0 / std::sqrt(1.0 + t * t);
        const double s = t * c;
        a[p][p] = app - t * apq;
        a[q][q] = aqq + t * apq;
        a[p][q] = 0.0;
        a[q][p] = 0.0;
        for (int r = 0; r < 9; ++r) {
          if (r != p && r != q) {
            const double arp = a[r][p], arq = a[r][q];
            a[r][p] = c * arp - s * arq;
            a[p][r] = a[r][p];
            a[r][q] = s * arp + c * arq;
            a[q][r] = a[r][q];
          }
          const double vrp = v[r][p], vrq = v[r][q];
          v[r][p] = c * vrp - s * vrq;
          v[r][q] = s * vrp + c * vrq;
        }
      }
  }
  int mi = 0;
  double me = a[0][0];
  for (int i = 1; i < 9; ++i)
    if (a[i][i] < me) {
      me = a[i][i];
      mi = i;
    }
  for (int r = 0; r < 9; ++r) {
    h[r] = v[r][mi];
    if (!std::isfinite(h[r])) return false;
  }
  return true;
}

// src/pipeline.rs:2357-2404
bool degenerate_triangle(const double p[4][2]) {
  static const int T[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
  for (const auto& t : T) {
    const double xi = p[t[0]][0], yi = p[t[0]][1], xj = p[t[1]][0], yj = p[t[1]][1];
    const double xk = p[t[2]][0], yk = p[t[2]][1];
    if (!std::isfinite(xi) || !std::isfinite(yi) || !std::isfinite(xj) || !std::isfinite(yj) ||
        !std::isfinite(xk) || !std::isfinite(yk))
      return true;
    const double dx1 = xj - xi, dy1 = yj - yi, dx2 = xk - xi, dy2 = yk - yi, dx3 = xk - xj, dy3 = yk - yj;
    const double cross = std::fabs(dx1 * dy2 - dy1 * dx2);
    const double me = std::fmax(std::fmax(dx1 * dx1 + dy1 * dy1, dx2 * dx2 + dy2 * dy2), dx3 * dx3 + dy3 * dy3);
    if (cross < 4.0 || cross < 1e-3 * me) return true;
  }
  return false;
}
bool degenerate_quad(const oracle_match* q[4]) {
  double qp[4][2], tp[4][2];
  for (int i = 0; i < 4; ++i) {
    qp[i][0] = q[i]->qx;
    qp[i][1] = q[i]->qy;
    tp[i][0] = q[i]->tx;
    tp[i][1] = q[i]->ty;
  }
  return degenerate_triangle(qp) || degenerate_triangle(tp);
}

// src/pipeline.rs:2408-2528
bool fit_dlt(const oracle_match* const* s, int n, double H[3][3]) {
  if (n < 4) return false;
  const double inv_n = 1.0 / (double)n;
  double cxq = 0, cyq = 0, cxt = 0, cyt = 0;
  for (int i = 0; i < n; ++i) {
    const double qx = s[i]->qx, qy = s[i]->qy, tx = s[i]->tx, ty = s[i]->ty;
    if (!std::isfinite(qx) || !std::isfinite(qy) || !std::isfinite(tx) || !std::isfinite(ty)) return false;
    cxq += qx;
    cyq += qy;
    cxt += tx;
    cyt += ty;
  }
  cxq *= inv_n;
  cyq *= inv_n;
  cxt *= inv_n;
  cyt *= inv_n;
  double mdq = 0, mdt = 0;
  for (int i = 0; i < n; ++i) {
    const double dxq = (double)s[i]->qx - cxq, dyq = (double)s[i]->qy - cyq;
    const double dxt = (double)s[i]->tx - cxt, dyt = (double)s[i]->ty - cyt;
    mdq += std::sqrt(dxq * dxq + dyq * dyq);
    mdt += std::sqrt(dxt * dxt + dyt * dyt);
  }
  mdq *= inv_n;
  mdt *= inv_n;
  if (!std::isfinite(mdq) || !std::isfinite(mdt) || mdq < 1e-6 || mdt < 1e-6) return false;
  const double sq = 1.41421356237309504880 / mdq;
  const double st = 1.41421356237309504880 / mdt;
  double ata[9][9] = {{0}};
  for (int i = 0; i < n; ++i) {
    const double x = ((double)s[i]->qx - cxq) * sq;
    const double y = ((double)s[i]->qy - cyq) * sq;
    const double xp = ((double)s[i]->tx - cxt) * st;
    const double yp = ((double)s[i]->ty - cyt) * st;
    const double r1[9] = {-x, -y, -1.0, 0.0, 0.0, 0.0, x * xp, y * xp, xp};
    const double r2[9] = {0.0, 0.0, 0.0, -x, -y, -1.0, x * yp, y * yp, yp};
    for (int a = 0; a < 9; ++a)
      for (int b = a; b < 9; ++b) ata[a][b] += r1[a] * r1[b] + r2[a] * r2[b];
  }
  for (int a = 0; a < 9; ++a)
    for (int b = 0; b < a; ++b) ata[a][b] = ata[b][a];
  double hv[9];
  if (!smallest_eigvec9(ata, hv)) return false;
  const double hn[3][3] = {{hv[0], hv[1], hv[2]}, {hv[3], hv[4], hv[5]}, {hv[6], hv[7], hv[8]}};
  const double tq[3][3] = {{sq, 0.0, -sq * cxq}, {0.0, sq, -sq * cyq}, {0.0, 0.0, 1.0}};
  const double ist = 1.0 / st;
  const double tti[3][3] = {{ist, 0.0, cxt}, {0.0, ist, cyt}, {0.0, 0.0, 1.0}};
  double tmp[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) tmp[r][c] = hn[r][0] * tq[0][c] + hn[r][1] * tq[1][c] + hn[r][2] * tq[2][c];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) H[r][c] = tti[r][0] * tmp[0][c] + tti[r][1] * tmp[1][c] + tti[r][2] * tmp[2][c];
  if (std::fabs(H[2][2]) > 1e-12) {
    const double inv = 1.0 / H[2][2];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) H[r][c] *= inv;
  }
  return true;
}

// src/pipeline.rs:2550-2576
void eval_h(const oracle_match* m, int n, const double H[3][3], double tsq, size_t& count, double& err) {
  count = 0;
  err = 0.0;
  for (int i = 0; i < n; ++i) {
    const double qx = m[i].qx, qy = m[i].qy;
    const double w = H[2][0] * qx + H[2][1] * qy + H[2][2];
    if (std::fabs(w) < 1e-9) continue;
    const double iw = 1.0 / w;
    const double px = (H[0][0] * qx + H[0][1] * qy + H[0][2]) * iw;
    const double py = (H[1][0] * qx + H[1][1] * qy + H[1][2]) * iw;
    const double dx = px - (double)m[i].tx, dy = py - (double)m[i].ty;
    const double e = dx * dx + dy * dy;
    if (e <= tsq) {
      ++count;
      err += e;
    }
  }
}

// src/pipeline.rs:2578-2601
std::vector<int> collect_h(const oracle_match* m, int n, const double H[3][3], double tsq) {
  std::vector<int> out;
  for (int i = 0; i < n; ++i) {
    const double qx = m[i].qx, qy = m[i].qy;
    const double w = H[2][0] * qx + H[2][1] * qy + H[2][2];
    if (std::fabs(w) < 1e-9) continue;
    const double iw = 1.0 / w;
    const double px = (H[0][0] * qx + H[0][1] * qy + H[0][2]) * iw;
    const double py = (H[1][0] * qx + H[1][1] * qy + H[1][2]) * iw;
    const double dx = px - (double)m[i].tx, dy = py - (double)m[i].ty;
    if (dx * dx + dy * dy <= tsq) out.push_back(i);
  }
  return out;
}

// src/pipeline.rs:2605-2631
void local_optimize(const oracle_match* m, int n, double H[3][3], size_t& count, double& err, double tsq) {
  for (int it = 0; it < 2; ++it) {
    const std::vector<int> in = collect_h(m, n, H, tsq);
    if (in.size() < 4) break;
    std::vector<const oracle_match*> ptr(in.size());
    for (size_t i = 0; i < in.size(); ++i) ptr[i] = &m[in[i]];
    double R[3][3];
    if (!fit_dlt(ptr.data(), (int)ptr.size(), R)) break;
    size_t rc;
    double re;
    eval_h(m, n, R, tsq, rc, re);
    if (rc > count || (rc == count && re < err)) {
      std::memcpy(H, R, sizeof(R));
      count = rc;
      err = re;
    } else {
      break;
    }
  }
}

// src/pipeline.rs:2663-2755
int homography_ransac(const oracle_match* m, int n, float thr, uint64_t sim_seed, uint64_t hom_seed,
                      std::vector<uint8_t>& mask, double H_out[3][3], bool& has_h) {
  mask.assign(n, 0);
  has_h = false;
  if (n == 0) return 0;
  const double thresh = (double)std::fmax(thr, 0.5f);
  const double tsq = thresh * thresh;
  std::vector<uint8_t> sim_mask;
  Sim sim;
  bool has_sim;
  const int sim_count = similarity_ransac(m, n, thr, sim_seed, sim_mask, sim, has_sim);
  double best[3][3] = {{0}};
  bool has_best = false;
  size_t best_count = 0;
  double best_err = std::numeric_limits<double>::infinity();
  if (has_sim) {
    const double hs[3][3] = {{(double)sim.a, -(double)sim.b, (double)sim.tx},
                             {(double)sim.b, (double)sim.a, (double)sim.ty},
                             {0.0, 0.0, 1.0}};
    std::memcpy(best, hs, sizeof(hs));
    has_best = true;
    eval_h(m, n, best, tsq, best_count, best_err);
  }
  if (n < 4) {
    mask = sim_mask;
    if (has_best) {
      std::memcpy(H_out, best, sizeof(best));
      has_h = true;
    }
    return sim_count;
  }
  const std::vector<double> cdf = ratio_cdf(m, n);
  uint64_t rng = hom_seed;
  const size_t hard_cap = 2000, min_iters = 64;
  size_t max_iters = adaptive_iters(best_count, n, 4, 0.999, min_iters, hard_cap);
  size_t iter = 0;
  while (iter < max_iters) {
    ++iter;
    size_t idx[4] = {0, 0, 0, 0};
    int chosen = 0, attempts = 0;
    while (chosen < 4 && attempts < 16) {
      ++attempts;
      const size_t c = sample_weighted(cdf, rng);
      bool dup = false;
      for (int j = 0; j < chosen; ++j)
        if (idx[j] == c) dup = true;
      if (!dup) idx[chosen++] = c;
    }
    if (chosen < 4) continue;
    const oracle_match* quad[4] = {&m[idx[0]], &m[idx[1]], &m[idx[2]], &m[idx[3]]};
    if (degenerate_quad(quad)) continue;
    double Hc[3][3];
    if (fit_dlt(quad, 4, Hc)) {
      size_t c;
      double e;
      eval_h(m, n, Hc, tsq, c, e);
      if (c > best_count || (c == best_count && e < best_err)) {
        local_optimize(m, n, Hc, c, e, tsq);
        best_count = c;
        best_err = e;
        std::memcpy(best, Hc, sizeof(Hc));
        has_best = true;
        max_iters = adaptive_iters(best_count, n, 4, 0.999, min_iters, hard_cap);
      }
    }
  }
  if (!has_best) {
    mask = sim_mask;
    return sim_count;
  }
  local_optimize(m, n, best, best_count, best_err, tsq);
  const std::vector<int> in = collect_h(m, n, best, tsq);
  for (int i : in) mask[i] = 1;
  std::memcpy(H_out, best, sizeof(best));
  has_h = true;
  return (int)in.size();
}

float median_f32(std::vector<float> v) {  // src/pipeline.rs:2195-2206
  if (v.empty()) return 0.0f;
  std::stable_sort(v.begin(), v.end(), [](float a, float b) { return a < b; });
  const size_t mid = v.size() / 2;
  return v.size() % 2 == 1 ? v[mid] : 0.5f * (v[mid - 1] + v[mid]);
}

inline int popc128(uint64_t a0, uint64_t a1, uint64_t b0, uint64_t b1) {
  return __builtin_popcountll(a0 ^ b0) + __builtin_popcountll(a1 ^ b1);
}
inline bool has_zero_byte128(uint64_t x0, uint64_t x1) {
  for (int i = 0; i < 8; ++i) {
    if (((x0 >> (8 * i)) & 0xFF) == 0) return true;
    if (((x1 >> (8 * i)) & 0xFF) == 0) return true;
  }
  return false;
}

}  // namespace

namespace {

// ------------------------------------------------- fundamental matrix (src/geometry.rs)
struct M3 {
  double v[3][3];
};
static M3 f_mul(const M3& a, const M3& b) {  // mul_mat3 (:145-154)
  M3 o;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) o.v[r][c] = a.v[r][0] * b.v[0][c] + a.v[r][1] * b.v[1][c] + a.v[r][2] * b.v[2][c];
  return o;
}
static M3 f_tr(const M3& m) {  // transpose_3x3 (:156-163)
  M3 o;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) o.v[r][c] = m.v[c][r];
  return o;
}
static double f_det(const M3& m) {  // det_3x3 (:165-170)
  return m.v[0][0] * (m.v[1][1] * m.v[2][2] - m.v[1][2] * m.v[2][1]) -
         m.v[0][1] * (m.v[1][0] * m.v[2][2] - m.v[1][2] * m.v[2][0]) +
         m.v[0][2] * (m.v[1][0] * m.v[2][1] - m.v[1][1] * m.v[2][0]);
}
static bool f_norm_frob(M3& m) {  // normalize_frobenius (:172-185)
  double s = 0.0;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) s += m.v[r][c] * m.v[r][c];
  if (!std::isfinite(s) || s < 1e-24) return false;
  const double inv = 1.0 / std::sqrt(s);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) m.v[r][c] *= inv;
  return true;
}
static double f_dot(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void f_cross(const double a[3], const double b[3], double o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
static bool f_normalize(const double v[3], double o[3]) {  // normalize_vec3 (:201-207)
  const double n = std::sqrt(f_dot(v, v));
  if (!std::isfinite(n) || n < 1e-12) return false;
  o[0] = v[0] / n;
  o[1] = v[1] / n;
  o[2] = v[2] / n;
  return true;
}

// One rotation step of the reference's classical Jacobi on an N x N symmetric
// matrix (largest off-diagonal pivot, first in row-major order on ties).
// Returns 1 to continue, 0 converged, -1 non-finite.
template <int N>
static int f_jacobi_step(double a[N][N], double v[N][N], double tol) {
  int p = 0, q = 1;
  double max_off = 0.0;
  for (int i = 0; i < N; ++i)
    for (int j = i + 1; j < N; ++j)
      if (std::fabs(a[i][j]) > max_off) {
        max_off = std::fabs(a[i][j]);
        p = i;
        q = j;
      }
  if (!std::isfinite(max_off)) return -1;
  if (max_off < tol) return 0;
  const double app = a[p][p], aqq = a[q][q], apq = a[p][q];
  const double tau = (aqq - app) / (2.0 * apq);
  const double t = tau >= 0.0 ? 1.0 / (tau + std::sqrt(1.0 + tau * tau)) : -1.0 / (-tau + std::sqrt(1.0 + tau * tau));
  const double c = 1.0 / std::sqrt(1.0 + t * t);
  const double s = t * c;
  a[p][p] = app - t * apq;
  a[q][q] = aqq + t * apq;
  a[p][q] = 0.0;
  a[q][p] = 0.0;
  for (int r = 0; r < N; ++r) {
    if (r != p && r != q) {
      const double arp = a[r][p], arq = a[r][q];
      const double nrp = c * arp - s * arq, nrq = s * arp + c * arq;
      a[r][p] = nrp;
      a[p][r] = nrp;
      a[r][q] = nrq;
      a[q][r] = nrq;
    }
  }
  for (int r = 0; r < N; ++r) {
    const double vrp = v[r][p], vrq = v[r][q];
    v[r][p] = c * vrp - s * vrq;
    v[r][q] = s * vrp + c * vrq;
  }
  return 1;
}

// jacobi_symmetric_eigen_9x9 (:209-295): eigenvectors as columns, ascending.
static bool f_eigen9(double a[9][9], double vecs[9][9]) {
  double v[9][9] = {};
  for (int i = 0; i < 9; ++i) v[i][i] = 1.0;
  for (int it = 0; it < 500; ++it) {
    const int r = f_jacobi_step<9>(a, v, 1e-13);
    if (r < 0) return false;
    if (r == 0) break;
  }
  int order[9] = {0, 1, 2, 3, 4, 5, 6, 7, 8};
  std::stable_sort(order, order + 9, [&](int i, int j) { return a[i][i] < a[j][j]; });
  for (int dc = 0; dc < 9; ++dc)
    for (int r = 0; r < 9; ++r) {
      const double val = v[r][order[dc]];
      if (!std::isfinite(val)) return false;
      vecs[r][dc] = val;
    }
  return true;
}

// jacobi_symmetric_eigen_3x3 (:297-372): descending.
static bool f_eigen3(double a[3][3], double vals[3], double vecs[3][3]) {
  double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int it = 0; it < 100; ++it) {
    const int r = f_jacobi_step<3>(a, v, 1e-14);
    if (r < 0) return false;
    if (r == 0) break;
  }
  int order[3] = {0, 1, 2};
  std::stable_sort(order, order + 3, [&](int i, int j) { return a[j][j] < a[i][i]; });
  for (int dc = 0; dc < 3; ++dc) {
    vals[dc] = a[order[dc]][order[dc]];
    for (int r = 0; r < 3; ++r) vecs[r][dc] = v[r][order[dc]];
  }
  return true;
}

// svd_3x3 (:463-531) + rank2_project_f (:533-545).
static bool f_rank2(M3& f) {
  const M3 m = f;
  M3 mtm = f_mul(f_tr(m), m);
  double vals[3], vm[3][3];
  if (!f_eigen3(mtm.v, vals, vm)) return false;
  double s[3];
  for (int i = 0; i < 3; ++i) s[i] = std::sqrt(std::fmax(vals[i], 0.0));
  auto mul_mv = [&](const double x[3], double o[3]) {
    for (int r = 0; r < 3; ++r) o[r] = m.v[r][0] * x[0] + m.v[r][1] * x[1] + m.v[r][2] * x[2];
  };
  const double v0[3] = {vm[0][0], vm[1][0], vm[2][0]}, v1[3] = {vm[0][1], vm[1][1], vm[2][1]},
               v2[3] = {vm[0][2], vm[1][2], vm[2][2]};
  double u0[3] = {1.0, 0.0, 0.0}, u1[3], u2[3], t[3];
  if (s[0] > 1e-12) {
    mul_mv(v0, t);
    if (!f_normalize(t, u0)) u0[0] = 1.0, u0[1] = 0.0, u0[2] = 0.0;
  }
  auto fallback = [&](double o[3]) {
    const double basis[3] = {std::fabs(u0[0]) < 0.9 ? 1.0 : 0.0, std::fabs(u0[0]) < 0.9 ? 0.0 : 1.0, 0.0};
    double c[3];
    f_cross(u0, basis, c);
    if (!f_normalize(c, o)) o[0] = 0.0, o[1] = 1.0, o[2] = 0.0;
  };
  if (s[1] > 1e-12) {
    double raw[3];
    mul_mv(v1, raw);
    const double proj = f_dot(raw, u0);
    const double orth[3] = {raw[0] - proj * u0[0], raw[1] - proj * u0[1], raw[2] - proj * u0[2]};
    if (!f_normalize(orth, u1)) fallback(u1);
  } else {
    fallback(u1);
  }
  f_cross(u0, u1, t);
  if (!f_normalize(t, u2)) return false;
  if (s[2] > 1e-12) {
    double mv2[3];
    mul_mv(v2, mv2);
    if (f_dot(u2, mv2) < 0.0) u2[0] = -u2[0], u2[1] = -u2[1], u2[2] = -u2[2];
  }
  M3 u, d = {}, vt;
  for (int r = 0; r < 3; ++r) u.v[r][0] = u0[r], u.v[r][1] = u1[r], u.v[r][2] = u2[r];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) vt.v[r][c] = vm[c][r];
  d.v[0][0] = s[0];
  d.v[1][1] = s[1];
  f = f_mul(u, f_mul(d, vt));
  return f_norm_frob(f);
}

// normalize_points_2d (:547-583).
static bool f_norm_pts(const std::vector<double>& x, const std::vector<double>& y, std::vector<double>& nx,
                       std::vector<double>& ny, M3& t) {
  const size_t n = x.size();
  if (n == 0) return false;
  const double inv_n = 1.0 / (double)n;
  double cx = 0.0, cy = 0.0;
  for (size_t i = 0; i < n; ++i) {
    if (!std::isfinite(x[i]) || !std::isfinite(y[i])) return false;
    cx += x[i];
    cy += y[i];
  }
  cx *= inv_n;
  cy *= inv_n;
  double md = 0.0;
  for (size_t i = 0; i < n; ++i) md += std::hypot(x[i] - cx, y[i] - cy);
  md *= inv_n;
  if (!std::isfinite(md) || md < 1e-9) return false;
  const double scale = 1.41421356237309504880 / md;
  nx.resize(n);
  ny.resize(n);
  for (size_t i = 0; i < n; ++i) {
    nx[i] = (x[i] - cx) * scale;
    ny[i] = (y[i] - cy) * scale;
  }
  t = M3{{{scale, 0.0, -scale * cx}, {0.0, scale, -scale * cy}, {0.0, 0.0, 1.0}}};
  return true;
}

// assemble_fundamental_ata (:586-604) -> jacobi -> the two smallest eigenvectors.
static bool f_null2(const std::vector<oracle_match>& s, M3& tq, M3& tt, M3& f1, M3& f2) {
  std::vector<double> qx, qy, tx, ty, nqx, nqy, ntx, nty;
  for (const auto& m : s) {
    qx.push_back((double)m.qx);
    qy.push_back((double)m.qy);
    tx.push_back((double)m.tx);
    ty.push_back((double)m.ty);
  }
  if (!f_norm_pts(qx, qy, nqx, nqy, tq) || !f_norm_pts(tx, ty, ntx, nty, tt)) return false;
  double ata[9][9] = {};
  for (size_t k = 0; k < s.size(); ++k) {
    const double x1 = nqx[k], y1 = nqy[k], x2 = ntx[k], y2 = nty[k];
    const double r[9] = {x2 * x1, x2 * y1, x2, y2 * x1, y2 * y1, y2, x1, y1, 1.0};
    for (int i = 0; i < 9; ++i)
      for (int j = i; j < 9; ++j) ata[i][j] += r[i] * r[j];
  }
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < i; ++j) ata[i][j] = ata[j][i];
  double vecs[9][9];
  if (!f_eigen9(ata, vecs)) return false;
  for (int k = 0; k < 9; ++k) {
    f1.v[k / 3][k % 3] = vecs[k][0];
    f2.v[k / 3][k % 3] = vecs[k][1];
  }
  return true;
}

// fit_fundamental_8point (:638-665).
static bool f_fit8(const std::vector<oracle_match>& s, M3& f) {
  if (s.size() < 8) return false;
  M3 tq, tt, f1, f2;
  if (!f_null2(s, tq, tt, f1, f2)) return false;
  if (!f_rank2(f1)) return false;
  f = f_mul(f_tr(tt), f_mul(f1, tq));
  return f_norm_frob(f);
}

// solve_cubic_real (:667-725).
static std::vector<double> f_cubic(double c3, double c2, double c1, double c0) {
  std::vector<double> roots;
  if (std::fabs(c3) < 1e-12) {
    if (std::fabs(c2) < 1e-12) {
      if (std::fabs(c1) < 1e-12) return roots;
      roots.push_back(-c0 / c1);
      return roots;
    }
    const double disc = c1 * c1 - 4.0 * c2 * c0;
    if (disc < 0.0) return roots;
    const double sq = std::sqrt(disc);
    roots.push_back((-c1 + sq) / (2.0 * c2));
    roots.push_back((-c1 - sq) / (2.0 * c2));
    return roots;
  }
  const double a = c2 / c3, b = c1 / c3, c = c0 / c3;
  const double a3 = a / 3.0;
  const double p = b - a * a3;
  const double q = (2.0 * a * a * a) / 27.0 - (a * b) / 3.0 + c;
  const double disc = (q * 0.5) * (q * 0.5) + powi_d(p / 3.0, 3);
  if (disc > 1e-14) {
    const double sq = std::sqrt(disc);
    roots.push_back(std::cbrt(-0.5 * q + sq) + std::cbrt(-0.5 * q - sq) - a3);
  } else if (disc >= -1e-14) {
    const double u = std::cbrt(-0.5 * q);
    roots.push_back(2.0 * u - a3);
    roots.push_back(-u - a3);
  } else {
    const double r = std::sqrt(-p / 3.0);
    double cp = (-0.5 * q) / (r * r * r);
    cp = cp < -1.0 ? -1.0 : (cp > 1.0 ? 1.0 : cp);
    const double phi = std::acos(cp);
    const double two_r = 2.0 * r;
    const double pi = 3.14159265358979323846;
    roots.push_back(two_r * std::cos(phi / 3.0) - a3);
    roots.push_back(two_r * std::cos((phi + 2.0 * pi) / 3.0) - a3);
    roots.push_back(two_r * std::cos((phi + 4.0 * pi) / 3.0) - a3);
  }
  for (double& t : roots)
    for (int k = 0; k < 3; ++k) {
      const double fv = ((c3 * t + c2) * t + c1) * t + c0;
      const double df = (3.0 * c3 * t + 2.0 * c2) * t + c1;
      if (std::fabs(df) > 1e-14) t -= fv / df;
    }
  return roots;
}

// fit_fundamental_7point (:727-806).
static std::vector<M3> f_fit7(const std::vector<oracle_match>& s) {
  std::vector<M3> out;
  M3 tq, tt, f1, f2;
  if (!f_null2(s, tq, tt, f1, f2)) return out;
  M3 b;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) b.v[r][c] = f1.v[r][c] - f2.v[r][c];
  auto eval = [&](double t) {
    M3 m;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) m.v[r][c] = f2.v[r][c] + t * b.v[r][c];
    return m;
  };
  const double p0 = f_det(f2), p1 = f_det(eval(1.0)), pm1 = f_det(eval(-1.0)), p2 = f_det(eval(2.0));
  const double c0 = p0;
  const double c2 = 0.5 * (p1 + pm1) - c0;
  const double s1 = 0.5 * (p1 - pm1);
  const double s2 = p2 - c0 - 4.0 * c2;
  const double c3 = (s2 - 2.0 * s1) / 6.0;
  const double c1 = s1 - c3;
  const M3 ttt = f_tr(tt);
  for (double t : f_cubic(c3, c2, c1, c0)) {
    if (!std::isfinite(t)) continue;
    M3 f = f_mul(ttt, f_mul(eval(t), tq));
    if (f_norm_frob(f)) out.push_back(f);
  }
  if (std::fabs(c3) < 1e-12 && std::fabs(f_det(b)) < 1e-10) {
    M3 f = f_mul(ttt, f_mul(b, tq));
    if (f_norm_frob(f)) out.push_back(f);
  }
  return out;
}

// sampson_distance_sq (:617-636).
static double f_sampson(const M3& f, double x1, double y1, double x2, double y2) {
  const auto& m = f.v;
  const double a0 = m[0][0] * x1 + m[0][1] * y1 + m[0][2];
  const double a1 = m[1][0] * x1 + m[1][1] * y1 + m[1][2];
  const double a2 = m[2][0] * x1 + m[2][1] * y1 + m[2][2];
  const double b0 = m[0][0] * x2 + m[1][0] * y2 + m[2][0];
  const double b1 = m[0][1] * x2 + m[1][1] * y2 + m[2][1];
  const double e = x2 * a0 + y2 * a1 + a2;
  const double den = a0 * a0 + a1 * a1 + b0 * b0 + b1 * b1;
  if (den < 1e-18 || !std::isfinite(den)) return std::numeric_limits<double>::infinity();
  return (e * e) / den;
}
static double f_sampson_m(const M3& f, const oracle_match& m) {
  return f_sampson(f, (double)m.qx, (double)m.qy, (double)m.tx, (double)m.ty);
}

// evaluate_fundamental_hypothesis (:808-829).
static void f_eval(const oracle_match* m, int n, const M3& f, double tsq, int& count, double& err) {
  count = 0;
  err = 0.0;
  for (int i = 0; i < n; ++i) {
    const double d2 = f_sampson_m(f, m[i]);
    if (d2 <= tsq) {
      ++count;
      err += d2;
    } else {
      err += tsq;
    }
  }
}

// adaptive_epipolar_iters (:831-855).
static int f_adaptive(int best, int total, int ss, double conf, int min_it, int max_it) {
  if (total <= ss || best == 0) return max_it;
  const double w = (double)best / (double)total;
  if (w >= 0.9999) return min_it;
  const double pg = powi_d(w, ss);
  if (pg <= 1e-12) return max_it;
  const double den = std::log(std::fmax(1.0 - pg, 1e-15));
  const double c = conf < 0.5 ? 0.5 : (conf > 0.999999 ? 0.999999 : conf);
  const double num = std::log(1.0 - c);
  const double est = std::ceil(num / den);
  const unsigned long long e = d2u_sat(est);
  return (int)std::min<unsigned long long>(std::max<unsigned long long>(e, (unsigned long long)min_it),
                                           (unsigned long long)max_it);
}

// estimate_fundamental_ransac_with_options (:868-1016).
static int f_ransac(const oracle_match* m, int n, double sampson_thr, int max_iters_opt, double conf, uint64_t seed,
                    uint8_t* mask, M3& out_f, bool& has_f, int* iters_out) {
  has_f = false;
  for (int i = 0; i < n; ++i) mask[i] = 0;
  if (iters_out) *iters_out = 0;
  if (n < 7) return 0;
  const double thr = std::fmax(sampson_thr, 0.25);
  const double tsq = thr * thr;
  M3 best_f{};
  bool have = false;
  int best_count = 0;
  double best_err = std::numeric_limits<double>::infinity();
  if (n == 7) {
    std::vector<oracle_match> s(m, m + 7);
    for (const M3& c : f_fit7(s)) {
      int cnt;
      double err;
      f_eval(m, n, c, tsq, cnt, err);
      if (cnt > best_count || (cnt == best_count && err < best_err)) {
        best_count = cnt;
        best_err = err;
        best_f = c;
        have = true;
      }
    }
  } else {
    const std::vector<double> cdf = ratio_cdf(m, n);
    uint64_t rng = seed;
    const int hard_cap = std::max(max_iters_opt, 64);
    const int min_iters = std::min(64, hard_cap);
    int max_iters = hard_cap;
    int iter = 0;
    while (iter < max_iters) {
      ++iter;
      size_t idx[8];
      int chosen = 0, attempts = 0;
      while (chosen < 8 && attempts < 32) {
        ++attempts;
        const size_t c = sample_weighted(cdf, rng);
        bool dup = false;
        for (int k = 0; k < chosen; ++k) dup = dup || idx[k] == c;
        if (!dup) idx[chosen++] = c;
      }
      if (chosen < 8) continue;
      std::vector<oracle_match> s;
      for (int k = 0; k < 8; ++k) s.push_back(m[idx[k]]);
      M3 f;
      if (f_fit8(s, f)) {
        int cnt;
        double err;
        f_eval(m, n, f, tsq, cnt, err);
        if (cnt > best_count || (cnt == best_count && err < best_err)) {
          best_count = cnt;
          best_err = err;
          best_f = f;
          have = true;
          max_iters = f_adaptive(best_count, n, 8, conf, min_iters, hard_cap);
        }
      }
    }
    if (iters_out) *iters_out = iter;
    if (have) {
      for (int r = 0; r < 2; ++r) {
        std::vector<oracle_match> inl;
        for (int i = 0; i < n; ++i)
          if (f_sampson_m(best_f, m[i]) <= tsq) inl.push_back(m[i]);
        if (inl.size() < 8) break;
        M3 rf;
        if (!f_fit8(inl, rf)) break;
        int cnt;
        double err;
        f_eval(m, n, rf, tsq, cnt, err);
        if (cnt > best_count || (cnt == best_count && err < best_err)) {
          best_count = cnt;
          best_err = err;
          best_f = rf;
        } else {
          break;
        }
      }
    }
  }
  if (!have) return 0;
  int k = 0;
  for (int i = 0; i < n; ++i) {
    mask[i] = f_sampson_m(best_f, m[i]) <= tsq ? 1 : 0;
    k += mask[i];
  }
  out_f = best_f;
  has_f = true;
  return k;
}

}  // namespace

extern "C" {

uint64_t oracle_splitmix64_next(uint64_t* state) { return splitmix64(*state); }

int oracle_gaussian_kernel_1d(float sigma, float* out, int cap) {
  const std::vector<float> k = gaussian_kernel_1d(sigma);
  for (int i = 0; i < (int)k.size() && i < cap; ++i) out[i] = k[i];
  return (int)k.size();
}

void oracle_gaussian_blur(const float* img, int h, int w, float sigma, float* out) {
  const Plane r = gaussian_blur(make_plane(img, h, w), sigma);
  std::memcpy(out, r.d.data(), sizeof(float) * (size_t)h * w);
}

void oracle_upsample_2x(const float* img, int h, int w, float* out) {
  const Plane r = upsample_2x_bilinear(make_plane(img, h, w));
  std::memcpy(out, r.d.data(), sizeof(float) * r.d.size());
}

// src/pipeline.rs:957-966
void oracle_luma_to_f32(const uint8_t* px, size_t n, float* out) {
  const float inv_255 = 1.0f / 255.0f;
  for (size_t i = 0; i < n; ++i) out[i] = (float)px[i] * inv_255;
}

void* oracle_pyramid_build(const float* img, int h, int w, int octaves, int scales, int upsample) {
  return new std::vector<Octave>(build_pyramid(make_plane(img, h, w), octaves, scales, upsample != 0));
}
int oracle_pyramid_num_octaves(const void* pyr) { return (int)((const std::vector<Octave>*)pyr)->size(); }
void oracle_pyramid_octave_info(const void* pyr, int o, int* h, int* w, float* sf) {
  const auto& oc = (*(const std::vector<Octave>*)pyr)[o];
  *h = oc.g[0].h;
  *w = oc.g[0].w;
  *sf = oc.scale_factor;
}
void oracle_pyramid_copy_plane(const void* pyr, int o, int kind, int idx, float* out) {
  const auto& oc = (*(const std::vector<Octave>*)pyr)[o];
  const Plane& p = kind == 0 ? oc.g[idx] : oc.dog[idx];
  std::memcpy(out, p.d.data(), sizeof(float) * p.d.size());
}
int oracle_pyramid_extract_extrema(const void* pyr, float thr, oracle_keypoint* out, int cap) {
  const auto kps = pyramid_extract(*(const std::vector<Octave>*)pyr, thr);
  for (int i = 0; i < (int)kps.size() && i < cap; ++i) out[i] = kps[i];
  return (int)kps.size();
}
void oracle_pyramid_free(void* pyr) { delete (std::vector<Octave>*)pyr; }

int oracle_detect_keypoints(const float* img, int h, int w, int octaves, int scales, float thr,
                            int upsample, oracle_keypoint* out, int cap) {
  const auto pyr = build_pyramid(make_plane(img, h, w), octaves, scales, upsample != 0);
  const auto kps = pyramid_extract(pyr, thr);
  for (int i = 0; i < (int)kps.size() && i < cap; ++i) out[i] = kps[i];
  return (int)kps.size();
}

// src/pipeline.rs:1633-1658 (see detect_and_compute_t).
int oracle_detect_and_compute(const float* img, int h, int w, int octaves, int scales, float thr,
                              int upsample, int kind, int max_features, float* meta, float* desc,
                              int cap) {
  return detect_and_compute_t<float>(make_plane(img, h, w), octaves, scales, thr, upsample, kind, max_features,
                                     meta, desc, cap);
}

// The same pipeline in f64 from the u8 luma (src/pipeline.rs:957-966 with
// `px as f64 * (1.0 / 255.0)`): the yardstick for the f32 results' error.
int oracle_detect_and_compute_f64(const uint8_t* luma, int h, int w, int octaves, int scales, double thr,
                                  int upsample, int kind, int max_features, double* meta, double* desc,
                                  int cap) {
  PlaneT<double> img(h, w);
  const double inv_255 = 1.0 / 255.0;
  for (size_t i = 0; i < img.d.size(); ++i) img.d[i] = (double)luma[i] * inv_255;
  return detect_and_compute_t<double>(img, octaves, scales, thr, upsample, kind, max_features, meta, desc, cap);
}

// Keypoints of the f64 pipeline: 6 doubles each (x, y, scale, response, octave, layer).
int oracle_detect_keypoints_f64(const uint8_t* luma, int h, int w, int octaves, int scales, double thr,
                                int upsample, double* out, int cap) {
  PlaneT<double> img(h, w);
  const double inv_255 = 1.0 / 255.0;
  for (size_t i = 0; i < img.d.size(); ++i) img.d[i] = (double)luma[i] * inv_255;
  const auto pyr = build_pyramid<double>(img, octaves, scales, upsample != 0);
  const auto kps = pyramid_extract<double>(pyr, thr);
  for (int i = 0; i < (int)kps.size() && i < cap; ++i) {
    const keypoint_f64& k = kps[i];
    double* o = out + 6 * (size_t)i;
    o[0] = k.x;
    o[1] = k.y;
    o[2] = k.scale;
    o[3] = k.response;
    o[4] = (double)k.octave;
    o[5] = (double)k.layer;
  }
  return (int)kps.size();
}

// src/pipeline.rs:1581-1629
int oracle_compute_descriptors(const float* img, int h, int w, const oracle_keypoint* kps_in, int n,
                               int kind, float* meta, float* desc, int cap) {
  if (h < 3 || w < 3 || n == 0) return 0;
  std::vector<oracle_keypoint> kps(kps_in, kps_in + n);
  unsigned max_layer = 0;
  for (const auto& kp : kps) max_layer = std::max(max_layer, kp.layer);
  const int scales = (int)std::max(max_layer, 3u);
  const float k = std::pow(2.0f, 1.0f / (float)scales);
  bool upsample = false;
  for (const auto& kp : kps)
    if (kp.layer > 0) {
      const float expected = BASE_SIGMA * (float)(1ull << kp.octave) * powi_f(k, (int)kp.layer);
      upsample = (kp.scale / expected) < 0.707f;
      break;
    }
  unsigned long long max_oct = 0;
  for (const auto& kp : kps) {
    unsigned long long o = kp.layer > 0 ? kp.octave
                                        : f2u_sat(std::floor(std::log2(std::fmax(kp.scale / BASE_SIGMA, 1.0f))));
    max_oct = std::max(max_oct, o);
  }
  const auto pyr = build_pyramid(make_plane(img, h, w), (int)(max_oct + 1), scales, upsample);
  return write_features(describe_from_pyramid(pyr, kps, kind), meta, desc, cap);
}

void oracle_rootsift(const float* d, float* out) { rootsift(d, out); }

// src/pipeline.rs:1024-1030
void oracle_quantize_u8(const float* d, int n, uint8_t* out) {
  for (int i = 0; i < n; ++i) {
    const float v = clampf(std::round(d[i] * 512.0f), 0.0f, 255.0f);
    out[i] = (uint8_t)f2u_sat(v);
  }
}

// src/pipeline.rs:1034-1044
void oracle_dequantize_u8(const uint8_t* q, int n, float* out) {
  for (int i = 0; i < n; ++i) out[i] = (float)q[i] * (1.0f / 512.0f);
  float s = 0.0f;
  for (int i = 0; i < n; ++i) s += out[i] * out[i];
  const float norm = std::sqrt(s);
  if (norm > 1e-7f) {
    const float inv = 1.0f / norm;
    for (int i = 0; i < n; ++i) out[i] *= inv;
  }
}

// src/catalog.rs:37-45 (u128 little endian: bits 0..63 in word 0)
void oracle_quantize_u128(const float* d, int n, uint64_t* out) {
  for (int f = 0; f < n; ++f) {
    uint64_t lo = 0, hi = 0;
    for (int i = 0; i < 128; ++i)
      if (d[(size_t)f * 128 + i] > 0.065f) {
        if (i < 64) lo |= 1ull << i;
        else hi |= 1ull << (i - 64);
      }
    out[2 * f] = lo;
    out[2 * f + 1] = hi;
  }
}

// src/pipeline.rs:1744-1841
int oracle_match_descriptors(const float* qd, int nq, const float* td, int nt, const float* qxy, const float* txy,
                 float ratio, int mutual, oracle_match* out, int cap) {
  if (nq == 0 || nt < 2) return 0;
  std::vector<int> ok(nq, 0);
  std::vector<oracle_match> fwd_all(nq);
#pragma omp parallel for schedule(dynamic, 16)
  for (int q = 0; q < nq; ++q) {
    float best = std::numeric_limits<float>::infinity();
    float second = best;
    int bi = 0;
    const float* a = qd + (size_t)q * 128;
    for (int t = 0; t < nt; ++t) {
      const float d = dist_sq_early_exit(a, td + (size_t)t * 128, second);
      if (d < best) {
        second = best;
        best = d;
        bi = t;
      } else if (d < second) {
        second = d;
      }
    }
    if (second > 1e-12f && std::isfinite(best)) {
      const float d1 = std::sqrt(best), d2 = std::sqrt(second);
      const float r = d1 / d2;
      if (r < ratio) {
        oracle_match m;
        m.query_index = (uint32_t)q;
        m.target_index = (uint32_t)bi;
        m.qx = qxy[2 * q];
        m.qy = qxy[2 * q + 1];
        m.tx = txy[2 * bi];
        m.ty = txy[2 * bi + 1];
        m.distance = d1;
        m.ratio = r;
        m.dx = m.tx - m.qx;
        m.dy = m.ty - m.qy;
        fwd_all[q] = m;
        ok[q] = 1;
      }
    }
  }
  std::vector<oracle_match> fwd;
  for (int q = 0; q < nq; ++q)
    if (ok[q]) fwd.push_back(fwd_all[q]);
  if (mutual && !fwd.empty()) {
    std::vector<int> keep(fwd.size(), 0);
#pragma omp parallel for schedule(dynamic, 16)
    for (long long i = 0; i < (long long)fwd.size(); ++i) {
      const float* t = td + (size_t)fwd[i].target_index * 128;
      float best = std::numeric_limits<float>::infinity();
      long long bq = -1;
      for (int q = 0; q < nq; ++q) {
        const float d = dist_sq_early_exit(t, qd + (size_t)q * 128, best);
        if (d < best) {
          best = d;
          bq = q;
        }
      }
      keep[i] = bq == (long long)fwd[i].query_index;
    }
    std::vector<oracle_match> kept;
    for (size_t i = 0; i < fwd.size(); ++i)
      if (keep[i]) kept.push_back(fwd[i]);
    fwd.swap(kept);
  }
  for (int i = 0; i < (int)fwd.size() && i < cap; ++i) out[i] = fwd[i];
  return (int)fwd.size();
}

int oracle_similarity_ransac(const oracle_match* m, int n, float thr, uint64_t seed, uint8_t* inlier_mask,
                             float* model, int* has_model) {
  std::vector<uint8_t> mask;
  Sim s{};
  bool hm = false;
  const int c = similarity_ransac(m, n, thr, seed, mask, s, hm);
  if (inlier_mask && n > 0) std::memcpy(inlier_mask, mask.data(), n);
  if (model) {
    model[0] = s.a;
    model[1] = s.b;
    model[2] = s.tx;
    model[3] = s.ty;
    model[4] = s.scale;
    model[5] = s.rot;
  }
  if (has_model) *has_model = hm ? 1 : 0;
  return c;
}

int oracle_homography_ransac(const oracle_match* m, int n, float thr, uint64_t sim_seed, uint64_t hom_seed,
                             uint8_t* inlier_mask, float* h9, int* has_h) {
  std::vector<uint8_t> mask;
  double H[3][3] = {{0}};
  bool hh = false;
  const int c = homography_ransac(m, n, thr, sim_seed, hom_seed, mask, H, hh);
  if (inlier_mask && n > 0) std::memcpy(inlier_mask, mask.data(), n);
  if (h9)
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc) h9[3 * r + cc] = (float)H[r][cc];
  if (has_h) *has_h = hh ? 1 : 0;
  return c;
}

// src/pipeline.rs:2210-2272
void oracle_summarize_tracking(const oracle_match* m, int n, const float* q_scale, const float* q_ori,
                               const float* t_scale, const float* t_ori, oracle_tracking* out) {
  if (n == 0) {
    *out = {0, 0, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f};
    return;
  }
  std::vector<uint8_t> mask;
  Sim s;
  bool hm;
  similarity_ransac(m, n, 3.0f, 0xD1B54A32D192ED03ull, mask, s, hm);
  std::vector<const oracle_match*> act;
  for (int i = 0; i < n; ++i)
    if (mask[i]) act.push_back(&m[i]);
  if (act.empty())
    for (int i = 0; i < n; ++i) act.push_back(&m[i]);
  const float inv_n = 1.0f / (float)act.size();
  float sdx = 0, sdy = 0, ssr = 0, ssin = 0, scos = 0;
  std::vector<float> dxs, dys;
  for (const oracle_match* a : act) {
    sdx += a->dx;
    sdy += a->dy;
    dxs.push_back(a->dx);
    dys.push_back(a->dy);
    const float qs = q_scale[a->query_index], ts = t_scale[a->target_index];
    if (qs > 1e-6f) ssr += ts / qs;
    const float dth = t_ori[a->target_index] - q_ori[a->query_index];
    ssin += std::sin(dth);
    scos += std::cos(dth);
  }
  const float mrot = std::atan2(ssin, scos);
  out->raw_match_count = (uint32_t)n;
  out->match_count = (uint32_t)act.size();
  out->inlier_ratio = (float)act.size() / (float)n;
  out->mean_dx = sdx * inv_n;
  out->mean_dy = sdy * inv_n;
  out->median_dx = median_f32(dxs);
  out->median_dy = median_f32(dys);
  out->mean_scale_ratio = ssr * inv_n;
  out->mean_rotation_deg = mrot * RAD_TO_DEG_F;
}

// src/catalog.rs:596-633 (MIH: entries > 32) and :707-728 (exhaustive)
void oracle_hamming_votes(const uint64_t* q, int nq, const uint64_t* cat, const int64_t* offsets, int ne,
                          int mih, uint32_t* votes) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int e = 0; e < ne; ++e) {
    uint32_t v = 0;
    for (int qi = 0; qi < nq; ++qi) {
      const uint64_t q0 = q[2 * qi], q1 = q[2 * qi + 1];
      bool hit = false;
      for (int64_t s = offsets[e]; s < offsets[e + 1] && !hit; ++s) {
        const uint64_t x0 = q0 ^ cat[2 * s], x1 = q1 ^ cat[2 * s + 1];
        const int d = __builtin_popcountll(x0) + __builtin_popcountll(x1);
        if (d <= 24 && (!mih || has_zero_byte128(x0, x1))) hit = true;
      }
      v += hit ? 1 : 0;
    }
    votes[e] = v;
  }
}

// The MIH branch as the reference runs it: the 16 x 256 inverted tables of
// (entry, signature) pairs (src/catalog.rs:291-306, filled in entry and
// signature order) and, per query, the walk over the 16 buckets its bytes
// select with seen_stamp deduplication (:596-615).  Sequential, for small
// cases: the pin of the zero-byte rule that oracle_hamming_votes evaluates.
void oracle_mih_votes_tables(const uint64_t* q, int nq, const uint64_t* cat, const int64_t* offsets, int ne,
                             uint32_t* votes) {
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> tables((size_t)16 * 256);
  for (int e = 0; e < ne; ++e)
    for (int64_t s = offsets[e]; s < offsets[e + 1]; ++s) {
      const uint64_t w[2] = {cat[2 * s], cat[2 * s + 1]};
      for (int band = 0; band < 16; ++band) {
        const unsigned key = (unsigned)((w[band / 8] >> (8 * (band % 8))) & 0xFF);
        tables[(size_t)band * 256 + key].emplace_back((uint32_t)e, (uint32_t)(s - offsets[e]));
      }
    }
  std::vector<size_t> seen(ne, 0);
  for (int e = 0; e < ne; ++e) votes[e] = 0;
  for (int qi = 0; qi < nq; ++qi) {
    const size_t stamp = (size_t)qi + 1;
    const uint64_t qw[2] = {q[2 * qi], q[2 * qi + 1]};
    for (int band = 0; band < 16; ++band) {
      const unsigned key = (unsigned)((qw[band / 8] >> (8 * (band % 8))) & 0xFF);
      for (const auto& es : tables[(size_t)band * 256 + key]) {
        if (seen[es.first] == stamp) continue;
        const int64_t s = offsets[es.first] + es.second;
        const int d = __builtin_popcountll(qw[0] ^ cat[2 * s]) + __builtin_popcountll(qw[1] ^ cat[2 * s + 1]);
        if (d <= 24) {
          seen[es.first] = stamp;
          votes[es.first] += 1;
        }
      }
    }
  }
}

void oracle_hamming_topk(const uint64_t* q, int nq, const uint64_t* cat, int64_t ncat, int k, uint32_t* idx,
                         uint32_t* dist) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int qi = 0; qi < nq; ++qi) {
    // bounded max-heap keyed by (dist, index)
    std::vector<std::pair<uint32_t, uint32_t>> heap;
    heap.reserve(k + 1);
    for (int64_t c = 0; c < ncat; ++c) {
      const uint32_t d = (uint32_t)popc128(q[2 * qi], q[2 * qi + 1], cat[2 * c], cat[2 * c + 1]);
      const std::pair<uint32_t, uint32_t> key{d, (uint32_t)c};
      if ((int)heap.size() < k) {
        heap.push_back(key);
        std::push_heap(heap.begin(), heap.end());
      } else if (key < heap.front()) {
        std::pop_heap(heap.begin(), heap.end());
        heap.back() = key;
        std::push_heap(heap.begin(), heap.end());
      }
    }
    std::sort(heap.begin(), heap.end());
    for (int j = 0; j < k; ++j) {
      idx[(size_t)qi * k + j] = j < (int)heap.size() ? heap[j].second : 0xFFFFFFFFu;
      dist[(size_t)qi * k + j] = j < (int)heap.size() ? heap[j].first : 0xFFFFFFFFu;
    }
  }
}

void oracle_l2_rerank(const float* qd, int nq, const float* cat_desc, const uint32_t* cand, int k,
                      uint32_t* out_idx, float* out_d2) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int qi = 0; qi < nq; ++qi) {
    std::vector<std::pair<float, uint32_t>> v;
    for (int j = 0; j < k; ++j) {
      const uint32_t c = cand[(size_t)qi * k + j];
      if (c == 0xFFFFFFFFu) continue;
      float s = 0.0f;
      for (int i = 0; i < 128; ++i) {
        const float d = qd[(size_t)qi * 128 + i] - cat_desc[(size_t)c * 128 + i];
        s += d * d;
      }
      v.push_back({s, c});
    }
    std::sort(v.begin(), v.end());
    for (int j = 0; j < k; ++j) {
      out_idx[(size_t)qi * k + j] = j < (int)v.size() ? v[j].second : 0xFFFFFFFFu;
      out_d2[(size_t)qi * k + j] = j < (int)v.size() ? v[j].first : INFINITY;
    }
  }
}

// warp_and_stitch (src/visualize.rs:379-483) with invert_matrix_3x3 (:202-233),
// project_f64 (:236-247), sample_bilinear_rgba (:250-287) and Homography2D::project
// (src/pipeline.rs:1122-1132).  Returns 0 and the canvas geometry (canvas = NULL:
// geometry only), or a negative code: -1 singular, -2 corner at infinity,
// -3 non-finite corner, -4 canvas over the safety limits.
static bool ow_sample(const uint8_t* img, int h, int w, size_t stride, double x, double y, double rgba[4],
                      double* feather) {
  const double wf = (double)w, hf = (double)h;
  if (x < 0.0 || y < 0.0 || x > (wf - 1.0) || y > (hf - 1.0)) return false;
  const uint32_t x0 = (uint32_t)std::floor(x), y0 = (uint32_t)std::floor(y);
  const uint32_t x1 = std::min<uint32_t>(x0 + 1, (uint32_t)w - 1), y1 = std::min<uint32_t>(y0 + 1, (uint32_t)h - 1);
  const double fx = x - (double)x0, fy = y - (double)y0;
  const double w00 = (1.0 - fx) * (1.0 - fy), w10 = fx * (1.0 - fy), w01 = (1.0 - fx) * fy, w11 = fx * fy;
  const uint8_t* p00 = img + y0 * stride + 4 * (size_t)x0;
  const uint8_t* p10 = img + y0 * stride + 4 * (size_t)x1;
  const uint8_t* p01 = img + y1 * stride + 4 * (size_t)x0;
  const uint8_t* p11 = img + y1 * stride + 4 * (size_t)x1;
  for (int c = 0; c < 4; ++c)
    rgba[c] = (double)p00[c] * w00 + (double)p10[c] * w10 + (double)p01[c] * w01 + (double)p11[c] * w11;
  auto fmin_ = [](double a, double b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a < b ? a : b)); };
  const double dist_edge = fmin_(fmin_(fmin_(x, (wf - 1.0) - x), y), (hf - 1.0) - y);
  double f = (dist_edge + 1.0) / 32.0;
  f = f < 0.02 ? 0.02 : (f > 1.0 ? 1.0 : f);
  *feather = f;
  return true;
}

static uint8_t ow_u8(double v) {  // Rust `as u8`: saturating, NaN -> 0
  if (!(v == v)) return 0;
  return v <= 0.0 ? 0 : (v >= 255.0 ? 255 : (uint8_t)v);
}

int oracle_warp_and_stitch(const uint8_t* q, int qh, int qw, size_t qs, const uint8_t* t, int th, int tw, size_t ts,
                           const float* h9, uint8_t* canvas, int* out_w, int* out_h, double* origin) {
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
  if (std::fabs(det) < 1e-12 || !std::isfinite(det)) return -1;
  const double id = 1.0 / det;
  const double hi[3][3] = {{c00 * id, c10 * id, c20 * id}, {c01 * id, c11 * id, c21 * id}, {c02 * id, c12 * id, c22 * id}};
  const double qwf = qw, qhf = qh, twf = tw, thf = th;
  double min_x = 0.0, min_y = 0.0, max_x = std::max(twf - 1.0, 0.0), max_y = std::max(thf - 1.0, 0.0);
  const double corners[4][2] = {{0.0, 0.0}, {qwf - 1.0, 0.0}, {0.0, qhf - 1.0}, {qwf - 1.0, qhf - 1.0}};
  for (const auto& c : corners) {
    const float x = (float)c[0], y = (float)c[1];
    const float w = h9[6] * x + h9[7] * y + h9[8];
    if (std::fabs(w) < 1e-6f) return -2;
    const float iw = 1.0f / w;
    const double px = (double)((h9[0] * x + h9[1] * y + h9[2]) * iw);
    const double py = (double)((h9[3] * x + h9[4] * y + h9[5]) * iw);
    if (!std::isfinite(px) || !std::isfinite(py)) return -3;
    min_x = std::min(min_x, px);
    min_y = std::min(min_y, py);
    max_x = std::max(max_x, px);
    max_y = std::max(max_y, py);
  }
  const double ox0 = std::floor(min_x), oy0 = std::floor(min_y);
  const double wf = std::max(std::ceil(max_x) - ox0 + 1.0, 1.0), hf = std::max(std::ceil(max_y) - oy0 + 1.0, 1.0);
  if (wf > 8192.0 || hf > 8192.0 || wf * hf > 25000000.0) return -4;
  *out_w = (int)wf;
  *out_h = (int)hf;
  origin[0] = ox0;
  origin[1] = oy0;
  if (!canvas) return 0;
  const int W = *out_w, H = *out_h;
#pragma omp parallel for schedule(static)
  for (int oy = 0; oy < H; ++oy) {
    const double ty = (double)oy + oy0;
    for (int ox = 0; ox < W; ++ox) {
      const double tx = (double)ox + ox0;
      double tc[4], qc[4], tw_ = 0, qw_ = 0;
      const bool has_t = ow_sample(t, th, tw, ts, tx, ty, tc, &tw_);
      bool has_q = false;
      const double w = hi[2][0] * tx + hi[2][1] * ty + hi[2][2];
      if (!(std::fabs(w) < 1e-7)) {
        const double iw = 1.0 / w;
        const double qx = (hi[0][0] * tx + hi[0][1] * ty + hi[0][2]) * iw;
        const double qy = (hi[1][0] * tx + hi[1][1] * ty + hi[1][2]) * iw;
        has_q = ow_sample(q, qh, qw, qs, qx, qy, qc, &qw_);
      }
      uint8_t* o = canvas + ((size_t)oy * W + ox) * 4;
      if (has_t && has_q) {
        const double den = tw_ + qw_, wt = tw_ / den, wq = qw_ / den;
        for (int c = 0; c < 3; ++c) o[c] = ow_u8(std::round(tc[c] * wt + qc[c] * wq));
        double al = std::round(tc[3] * wt + qc[3] * wq);
        al = al < 0.0 ? 0.0 : (al > 255.0 ? 255.0 : al);
        o[3] = ow_u8(al);
      } else if (has_t) {
        for (int c = 0; c < 4; ++c) o[c] = ow_u8(std::round(tc[c]));
      } else if (has_q) {
        for (int c = 0; c < 4; ++c) o[c] = ow_u8(std::round(qc[c]));
      } else {
        o[0] = o[1] = o[2] = o[3] = 0;
      }
    }
  }
  return 0;
}

int oracle_fundamental_ransac(const oracle_match* m, int n, double sampson_threshold, int max_iters,
                              double confidence, uint64_t seed, uint8_t* mask, double* f9, int* has_f, int* iters) {
  M3 f{};
  bool has = false;
  const int k = f_ransac(m, n, sampson_threshold, max_iters, confidence, seed, mask, f, has, iters);
  *has_f = has ? 1 : 0;
  for (int i = 0; i < 9; ++i) f9[i] = has ? f.v[i / 3][i % 3] : 0.0;
  return k;
}

int oracle_fit_fundamental_7point(const oracle_match* m, double* f9s) {
  std::vector<oracle_match> s(m, m + 7);
  const std::vector<M3> c = f_fit7(s);
  for (size_t k = 0; k < c.size(); ++k)
    for (int i = 0; i < 9; ++i) f9s[9 * k + i] = c[k].v[i / 3][i % 3];
  return (int)c.size();
}

int oracle_fit_fundamental_8point(const oracle_match* m, int n, double* f9) {
  std::vector<oracle_match> s(m, m + n);
  M3 f;
  if (!f_fit8(s, f)) return 0;
  for (int i = 0; i < 9; ++i) f9[i] = f.v[i / 3][i % 3];
  return 1;
}

double oracle_sampson_distance_sq(const double* f9, double x1, double y1, double x2, double y2) {
  M3 f;
  for (int i = 0; i < 9; ++i) f.v[i / 3][i % 3] = f9[i];
  return f_sampson(f, x1, y1, x2, y2);
}

// ---------------------------------------------------------------- stitch_panorama
// src/stitch.rs.  Helpers from src/visualize.rs: invert_matrix_3x3 (:202-233),
// project_f64 (:236-247), sample_bilinear_rgba (:250-287, ow_sample above),
// is_sane_homography_for_dims (:303-357), resolve_safe_alignment_homography
// (:361-375).
static bool pano_invert_f32(const float* m, double out[9]) {  // invert_matrix_3x3
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
  for (int i = 0; i < 9; ++i) out[i] = r[i];
  return true;
}

static bool pano_project(const double* m, double x, double y, double& px, double& py) {  // project_f64
  const double w = m[6] * x + m[7] * y + m[8];
  if (std::fabs(w) < 1e-7) return false;
  const double iw = 1.0 / w;
  px = (m[0] * x + m[1] * y + m[2]) * iw;
  py = (m[3] * x + m[4] * y + m[5]) * iw;
  return true;
}

static bool pano_sane(const float* m, int src_w, int src_h) {  // is_sane_homography_for_dims
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

// sample_patch_intensity (src/stitch.rs:203-229) on the f32 luma plane.
static double pano_patch(const std::vector<float>& g, int h, int w, float x, float y) {
  if (h == 0 || w == 0 || !std::isfinite(x) || !std::isfinite(y)) return 0.0;
  auto clampi = [](long long v, long long lo, long long hi) { return v < lo ? lo : (v > hi ? hi : v); };
  const long long cx = clampi(f2i_sat(std::round(x)), 0, w - 1), cy = clampi(f2i_sat(std::round(y)), 0, h - 1);
  const long long y0 = cy > 0 ? cy - 1 : 0, y1 = std::min(cy + 1, (long long)h - 1);
  const long long x0 = cx > 0 ? cx - 1 : 0, x1 = std::min(cx + 1, (long long)w - 1);
  double sum = 0.0;
  long long cnt = 0;
  for (long long yy = y0; yy <= y1; ++yy)
    for (long long xx = x0; xx <= x1; ++xx) {
      sum += (double)g[(size_t)yy * w + xx];
      ++cnt;
    }
  return cnt == 0 ? 0.0 : (sum / (double)cnt) * 255.0;
}

// compose_mat3 (src/stitch.rs:115-132)
static void pano_compose(const double* a, const double* b, double* out) {
  double o[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) o[3 * r + c] = a[3 * r] * b[c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c];
  if (std::fabs(o[8]) > 1e-12) {
    const double inv = 1.0 / o[8];
    for (int i = 0; i < 9; ++i) o[i] *= inv;
  }
  for (int i = 0; i < 9; ++i) out[i] = o[i];
}

void oracle_warp_cylindrical(const uint8_t* img, int h, int w, size_t stride, float focal_px, uint8_t* out) {
  const double f = std::fmax(std::fmax((double)focal_px, (double)std::max(w, h) * 0.25), 16.0);
  const double cx = ((double)w - 1.0) * 0.5, cy = ((double)h - 1.0) * 0.5;
  std::memset(out, 0, (size_t)w * h * 4);
  for (int y = 0; y < h; ++y) {
    const double dy = (double)y - cy;
    for (int x = 0; x < w; ++x) {
      const double theta = ((double)x - cx) / f;
      if (std::fabs(theta) >= 1.45) continue;
      const double cos_t = std::cos(theta);
      const double sx = f * std::tan(theta) + cx;
      const double sy = dy / cos_t + cy;
      double px[4], fw;
      if (ow_sample(img, h, w, stride, sx, sy, px, &fw)) {
        uint8_t* o = out + ((size_t)y * w + x) * 4;
        for (int c = 0; c < 3; ++c) o[c] = ow_u8(std::round(px[c]));
        o[3] = 255;
      }
    }
  }
}

void oracle_solve_exposure_gains(const double* pairs, int n_pairs, int n, int ref_idx, double sigma_n,
                                 double sigma_g, float* out) {
  if (n == 0) return;
  std::vector<std::vector<double>> a(n, std::vector<double>(n, 0.0));
  std::vector<double> b(n, 0.0);
  const double sn = std::fmax(sigma_n, 1e-3), sg = std::fmax(sigma_g, 1e-3);
  const double inv_sn2 = 1.0 / (sn * sn), prior_w = 1.0 / (sg * sg);
  for (int i = 0; i < n; ++i) {
    a[i][i] += prior_w;
    b[i] += prior_w;
  }
  for (int p = 0; p < n_pairs; ++p) {
    const double* e = pairs + 5 * p;
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
    if (mx < 1e-12) {
      for (int i = 0; i < n; ++i) out[i] = 1.0f;
      return;
    }
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
    out[i] = clampf((float)sc, 0.4f, 2.5f);
  }
}

namespace {
struct PanoEdge {
  int from, to;
  double h[9];
  int inliers;
  double mean_from, mean_to;
};
}  // namespace

int oracle_panorama_register(const uint8_t* const* imgs, const int* hs, const int* ws, int n,
                             const oracle_panorama_options* opt, int* ref_index, uint8_t* registered, float* gains,
                             double* h_to_ref, double* inv_out, double* origin, int* out_w, int* out_h) {
  if (n < 2) return -1;
  // gray planes and features (extract_sift_features: upsampling on, the 4096 cap)
  std::vector<std::vector<float>> gray(n);
  std::vector<std::vector<float>> meta(n), desc(n);
  std::vector<int> nf(n);
  for (int i = 0; i < n; ++i) {
    const size_t np = (size_t)hs[i] * ws[i];
    gray[i].resize(np);
    for (size_t p = 0; p < np; ++p) {
      const uint8_t* px = imgs[i] + 4 * p;
      const uint32_t l = (2126u * px[0] + 7152u * px[1] + 722u * px[2]) / 10000u;
      gray[i][p] = (float)l * (1.0f / 255.0f);
    }
    meta[i].resize(5 * 4096);
    desc[i].resize(128 * 4096);
    nf[i] = std::min(4096, oracle_detect_and_compute(gray[i].data(), hs[i], ws[i], opt->octaves, opt->scales,
                                                     opt->threshold, 1, 0, 4096, meta[i].data(), desc[i].data(),
                                                     4096));
  }
  std::vector<PanoEdge> edges;
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      std::vector<float> xi(2 * (size_t)nf[i]), xj(2 * (size_t)nf[j]);
      for (int k = 0; k < nf[i]; ++k) xi[2 * k] = meta[i][5 * k], xi[2 * k + 1] = meta[i][5 * k + 1];
      for (int k = 0; k < nf[j]; ++k) xj[2 * k] = meta[j][5 * k], xj[2 * k + 1] = meta[j][5 * k + 1];
      std::vector<oracle_match> raw(std::max(nf[i], 1));
      const int nr = oracle_match_descriptors(desc[i].data(), nf[i], desc[j].data(), nf[j], xi.data(), xj.data(),
                                              opt->ratio, 0, raw.data(), (int)raw.size());
      if (nr < 6) continue;
      std::vector<uint8_t> sm(nr), hm(nr);
      float sim[6], h9[9];
      int has_s = 0, has_h = 0;
      const int ns = oracle_similarity_ransac(raw.data(), nr, opt->ransac_threshold, 0xD1B54A32D192ED03ull,
                                              sm.data(), sim, &has_s);
      const int nh = oracle_homography_ransac(raw.data(), nr, opt->ransac_threshold, 0xD1B54A32D192ED03ull,
                                              0x517CC1B727220A95ull, hm.data(), h9, &has_h);
      const std::vector<uint8_t>& best = nh >= ns ? hm : sm;
      const int nb = nh >= ns ? nh : ns;
      if (nb < 6) continue;
      float hij[9];
      if (has_h && nh >= 6 && pano_sane(h9, ws[i], hs[i])) {
        std::memcpy(hij, h9, sizeof hij);
      } else if (has_s) {
        const float r[9] = {sim[0], -sim[1], sim[2], sim[1], sim[0], sim[3], 0.0f, 0.0f, 1.0f};
        std::memcpy(hij, r, sizeof hij);
      } else {
        continue;
      }
      double hji[9];
      if (!pano_invert_f32(hij, hji)) continue;
      double si = 0.0, sj = 0.0;
      for (int k = 0; k < nr; ++k)
        if (best[k]) {
          si += pano_patch(gray[i], hs[i], ws[i], raw[k].qx, raw[k].qy);
          sj += pano_patch(gray[j], hs[j], ws[j], raw[k].tx, raw[k].ty);
        }
      const double ic = 1.0 / (double)nb;
      const double mi = std::fmax(si * ic, 1.0), mj = std::fmax(sj * ic, 1.0);
      PanoEdge e1{i, j, {}, nb, mi, mj}, e2{j, i, {}, nb, mj, mi};
      for (int k = 0; k < 9; ++k) e1.h[k] = (double)hij[k], e2.h[k] = hji[k];
      edges.push_back(e1);
      edges.push_back(e2);
    }
  if (edges.empty()) return -2;
  std::vector<std::vector<PanoEdge>> adj(n);
  for (const PanoEdge& e : edges) adj[e.from].push_back(e);
  // largest connected component (first of the largest), BFS order
  std::vector<char> visited(n, 0);
  std::vector<int> best_comp;
  for (int s0 = 0; s0 < n; ++s0) {
    if (visited[s0] || adj[s0].empty()) continue;
    std::vector<int> comp;
    std::deque<int> q;
    visited[s0] = 1;
    q.push_back(s0);
    while (!q.empty()) {
      const int u = q.front();
      q.pop_front();
      comp.push_back(u);
      for (const PanoEdge& e : adj[u])
        if (!visited[e.to]) {
          visited[e.to] = 1;
          q.push_back(e.to);
        }
    }
    if (comp.size() > best_comp.size()) best_comp = comp;
  }
  if (best_comp.size() < 2) return -3;
  // reference: the largest (total inliers, index)
  int ref = -1;
  long long best_w = -1;
  for (int u : best_comp) {
    long long wsum = 0;
    for (const PanoEdge& e : adj[u]) wsum += e.inliers;
    if (wsum > best_w || (wsum == best_w && u > ref)) {
      best_w = wsum;
      ref = u;
    }
  }
  // Prim's maximum spanning tree from the reference
  std::vector<char> has(n, 0);
  std::vector<double> H(9 * (size_t)n, 0.0);
  has[ref] = 1;
  const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  std::memcpy(&H[9 * (size_t)ref], I, sizeof I);
  for (size_t it = 1; it < best_comp.size(); ++it) {
    const PanoEdge* be = nullptr;
    for (int u : best_comp) {
      if (!has[u]) continue;
      for (const PanoEdge& e : adj[u])
        if (!has[e.to] && (!be || e.inliers > be->inliers)) be = &e;
    }
    if (!be) break;
    const int parent = be->from, child = be->to;
    const PanoEdge* rev = nullptr;
    for (const PanoEdge& e : adj[child])
      if (e.to == parent) {
        rev = &e;
        break;
      }
    pano_compose(&H[9 * (size_t)parent], rev->h, &H[9 * (size_t)child]);
    has[child] = 1;
  }
  std::vector<int> reg;
  for (int i = 0; i < n; ++i)
    if (has[i]) reg.push_back(i);
  // exposure gains over the registered component's edges
  std::vector<float> g(n, 1.0f);
  if (opt->exposure_compensation) {
    std::map<std::pair<int, int>, std::array<double, 3>> seen;
    for (int u : reg)
      for (const PanoEdge& e : adj[u])
        if (has[e.to]) {
          const bool lt = e.from < e.to;
          const std::pair<int, int> key = lt ? std::make_pair(e.from, e.to) : std::make_pair(e.to, e.from);
          seen[key] = {(double)e.inliers, lt ? e.mean_from : e.mean_to, lt ? e.mean_to : e.mean_from};
        }
    std::vector<double> pairs;
    for (const auto& kv : seen) {
      pairs.push_back(kv.first.first);
      pairs.push_back(kv.first.second);
      pairs.push_back(kv.second[0]);
      pairs.push_back(kv.second[1]);
      pairs.push_back(kv.second[2]);
    }
    oracle_solve_exposure_gains(pairs.data(), (int)(pairs.size() / 5), n, ref, 10.0, 0.25, g.data());
  }
  // union bounding box in reference coordinates
  double min_x = INFINITY, min_y = INFINITY, max_x = -INFINITY, max_y = -INFINITY;
  std::vector<double> inv(9 * (size_t)n, 0.0);
  for (int idx : reg) {
    const double* hm = &H[9 * (size_t)idx];
    float h2[9];
    for (int k = 0; k < 9; ++k) h2[k] = (float)hm[k];
    if (!pano_invert_f32(h2, &inv[9 * (size_t)idx])) return -4;
    const double w = std::fmax((double)ws[idx] - 1.0, 0.0), hh = std::fmax((double)hs[idx] - 1.0, 0.0);
    const double cs[4][2] = {{0.0, 0.0}, {w, 0.0}, {0.0, hh}, {w, hh}};
    for (const auto& c : cs) {
      double px, py;
      if (!pano_project(hm, c[0], c[1], px, py)) return -5;
      if (!std::isfinite(px) || !std::isfinite(py)) return -6;
      min_x = std::fmin(min_x, px);
      min_y = std::fmin(min_y, py);
      max_x = std::fmax(max_x, px);
      max_y = std::fmax(max_y, py);
    }
  }
  const double ox = std::floor(min_x), oy = std::floor(min_y);
  const double wf = std::fmax(std::ceil(max_x) - ox + 1.0, 1.0), hf = std::fmax(std::ceil(max_y) - oy + 1.0, 1.0);
  if (wf > (double)opt->max_canvas_dim || hf > (double)opt->max_canvas_dim ||
      wf * hf > (double)opt->max_canvas_pixels)
    return -7;
  *ref_index = ref;
  for (int i = 0; i < n; ++i) {
    registered[i] = has[i];
    gains[i] = g[i];
  }
  std::memcpy(h_to_ref, H.data(), sizeof(double) * 9 * n);
  std::memcpy(inv_out, inv.data(), sizeof(double) * 9 * n);
  origin[0] = ox;
  origin[1] = oy;
  *out_w = (int)wf;
  *out_h = (int)hf;
  return 0;
}

namespace {
using Rgb = std::array<float, 3>;
const float kPyrK[5] = {1.0f / 16.0f, 4.0f / 16.0f, 6.0f / 16.0f, 4.0f / 16.0f, 1.0f / 16.0f};

// downsample_half_rgba_weighted (src/stitch.rs:318-393)
void pano_down_rgb(const std::vector<Rgb>& src, const std::vector<float>& mask, int w, int h, std::vector<Rgb>& dst,
                   std::vector<float>& dmask, int& nw, int& nh) {
  nw = std::max((w + 1) / 2, 1);
  nh = std::max((h + 1) / 2, 1);
  std::vector<Rgb> trgb((size_t)h * nw, Rgb{0, 0, 0});
  std::vector<float> tm((size_t)h * nw, 0.0f);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < nw; ++x) {
      Rgb acc{0, 0, 0};
      float m = 0.0f, vw = 0.0f;
      for (int k = 0; k < 5; ++k) {
        const int sx = std::min(std::max(2 * x + k - 2, 0), w - 1);
        const float mw = mask[(size_t)y * w + sx];
        m += kPyrK[k] * mw;
        if (mw > 0.0f) {
          const float v = kPyrK[k] * mw;
          vw += v;
          for (int c = 0; c < 3; ++c) acc[c] += v * src[(size_t)y * w + sx][c];
        }
      }
      tm[(size_t)y * nw + x] = m;
      if (vw > 1e-6f) {
        const float inv = 1.0f / vw;
        trgb[(size_t)y * nw + x] = Rgb{acc[0] * inv, acc[1] * inv, acc[2] * inv};
      }
    }
  dst.assign((size_t)nw * nh, Rgb{0, 0, 0});
  dmask.assign((size_t)nw * nh, 0.0f);
  for (int y = 0; y < nh; ++y)
    for (int x = 0; x < nw; ++x) {
      Rgb acc{0, 0, 0};
      float m = 0.0f, vw = 0.0f;
      for (int k = 0; k < 5; ++k) {
        const int sy = std::min(std::max(2 * y + k - 2, 0), h - 1);
        const size_t i = (size_t)sy * nw + x;
        const float mw = tm[i];
        m += kPyrK[k] * mw;
        if (mw > 0.0f) {
          const float v = kPyrK[k] * mw;
          vw += v;
          for (int c = 0; c < 3; ++c) acc[c] += v * trgb[i][c];
        }
      }
      dmask[(size_t)y * nw + x] = m;
      if (vw > 1e-6f) {
        const float inv = 1.0f / vw;
        dst[(size_t)y * nw + x] = Rgb{acc[0] * inv, acc[1] * inv, acc[2] * inv};
      }
    }
}

// downsample_half_scalar (src/stitch.rs:436-470)
void pano_down_scalar(const std::vector<float>& src, int w, int h, std::vector<float>& dst) {
  const int nw = std::max((w + 1) / 2, 1), nh = std::max((h + 1) / 2, 1);
  std::vector<float> t((size_t)h * nw, 0.0f);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < nw; ++x) {
      float acc = 0.0f;
      for (int k = 0; k < 5; ++k) acc += kPyrK[k] * src[(size_t)y * w + std::min(std::max(2 * x + k - 2, 0), w - 1)];
      t[(size_t)y * nw + x] = acc;
    }
  dst.assign((size_t)nw * nh, 0.0f);
  for (int y = 0; y < nh; ++y)
    for (int x = 0; x < nw; ++x) {
      float acc = 0.0f;
      for (int k = 0; k < 5; ++k) acc += kPyrK[k] * t[(size_t)std::min(std::max(2 * y + k - 2, 0), h - 1) * nw + x];
      dst[(size_t)y * nw + x] = acc;
    }
}

// upsample_to_size_rgb (src/stitch.rs:395-434)
void pano_up_rgb(const std::vector<Rgb>& src, int sw, int sh, int dw, int dh, std::vector<Rgb>& out) {
  out.assign((size_t)dw * dh, Rgb{0, 0, 0});
  for (int y = 0; y < dh; ++y) {
    const float fy = clampf((float)y * 0.5f, 0.0f, (float)(sh > 0 ? sh - 1 : 0));
    const int y0 = std::min((int)std::floor(fy), sh - 1), y1 = std::min(y0 + 1, sh - 1);
    const float wy1 = fy - (float)y0, wy0 = 1.0f - wy1;
    for (int x = 0; x < dw; ++x) {
      const float fx = clampf((float)x * 0.5f, 0.0f, (float)(sw > 0 ? sw - 1 : 0));
      const int x0 = std::min((int)std::floor(fx), sw - 1), x1 = std::min(x0 + 1, sw - 1);
      const float wx1 = fx - (float)x0, wx0 = 1.0f - wx1;
      const Rgb& p00 = src[(size_t)y0 * sw + x0];
      const Rgb& p10 = src[(size_t)y0 * sw + x1];
      const Rgb& p01 = src[(size_t)y1 * sw + x0];
      const Rgb& p11 = src[(size_t)y1 * sw + x1];
      const float w00 = wx0 * wy0, w10 = wx1 * wy0, w01 = wx0 * wy1, w11 = wx1 * wy1;
      for (int c = 0; c < 3; ++c) out[(size_t)y * dw + x][c] = p00[c] * w00 + p10[c] * w10 + p01[c] * w01 + p11[c] * w11;
    }
  }
}
}  // namespace

void oracle_panorama_composite(const uint8_t* const* imgs, const int* hs, const int* ws, int n,
                               const uint8_t* registered, const float* gains, const double* inv,
                               const double* origin, int W, int Hh, int blend, int levels, int tile_size,
                               uint8_t* canvas) {
  (void)tile_size;  // the tiling does not change a pixel's value
  std::memset(canvas, 0, (size_t)W * Hh * 4);
  std::vector<int> reg;
  for (int i = 0; i < n; ++i)
    if (registered[i]) reg.push_back(i);
  const double ox = origin[0], oy = origin[1];
  if (blend == 0) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < Hh; ++y) {
      const double ry = oy + (double)y;
      for (int x = 0; x < W; ++x) {
        const double rx = ox + (double)x;
        double acc[3] = {0, 0, 0}, aw = 0.0;
        for (int idx : reg) {
          double sx, sy, px[4], fw;
          if (!pano_project(inv + 9 * (size_t)idx, rx, ry, sx, sy)) continue;
          if (!ow_sample(imgs[idx], hs[idx], ws[idx], (size_t)ws[idx] * 4, sx, sy, px, &fw)) continue;
          const double g = (double)gains[idx], wt = std::fmax(fw, 1e-4);
          for (int c = 0; c < 3; ++c) acc[c] += wt * clampt<double>(px[c] * g, 0.0, 255.0);
          aw += wt;
        }
        if (aw > 0.0) {
          const double iw = 1.0 / aw;
          uint8_t* o = canvas + ((size_t)y * W + x) * 4;
          for (int c = 0; c < 3; ++c) o[c] = ow_u8(std::round(acc[c] * iw));
          o[3] = 255;
        }
      }
    }
    return;
  }
  const size_t np = (size_t)W * Hh;
  const int k_reg = (int)reg.size();
  std::vector<std::vector<Rgb>> warped(k_reg, std::vector<Rgb>(np, Rgb{0, 0, 0}));
  std::vector<std::vector<float>> valid(k_reg, std::vector<float>(np, 0.0f));
  std::vector<float> best_w(np, -1.0f);
  std::vector<int> owner(np, -1);
  for (int pos = 0; pos < k_reg; ++pos) {
    const int idx = reg[pos];
    const float gain = gains[idx];
    for (int y = 0; y < Hh; ++y) {
      const double ry = oy + (double)y;
      for (int x = 0; x < W; ++x) {
        const double rx = ox + (double)x;
        double sx, sy, px[4], fw;
        if (!pano_project(inv + 9 * (size_t)idx, rx, ry, sx, sy)) continue;
        if (!ow_sample(imgs[idx], hs[idx], ws[idx], (size_t)ws[idx] * 4, sx, sy, px, &fw)) continue;
        const size_t p = (size_t)y * W + x;
        for (int c = 0; c < 3; ++c) warped[pos][p][c] = clampf((float)px[c] * gain, 0.0f, 255.0f);
        valid[pos][p] = 1.0f;
        const float f32 = (float)fw;
        if (f32 > best_w[p]) {
          best_w[p] = f32;
          owner[p] = pos;
        }
      }
    }
  }
  const int maxl = std::max((int)std::floor(std::log2((double)std::min(W, Hh))), 1);
  const int nl = std::min(std::min(std::max(levels, 1), 6), maxl);
  std::vector<std::pair<int, int>> dims;
  std::vector<std::vector<Rgb>> bl;
  std::vector<std::vector<float>> ms;
  {
    int cw = W, ch = Hh;
    for (int l = 0; l < nl; ++l) {
      dims.push_back({cw, ch});
      bl.push_back(std::vector<Rgb>((size_t)cw * ch, Rgb{0, 0, 0}));
      ms.push_back(std::vector<float>((size_t)cw * ch, 0.0f));
      cw = std::max((cw + 1) / 2, 1);
      ch = std::max((ch + 1) / 2, 1);
    }
  }
  for (int pos = 0; pos < k_reg; ++pos) {
    std::vector<std::vector<Rgb>> gi(nl);
    std::vector<std::vector<float>> gv(nl), gm(nl);
    gi[0].swap(warped[pos]);
    gv[0].swap(valid[pos]);
    gm[0].assign(np, 0.0f);
    for (size_t p = 0; p < np; ++p) gm[0][p] = owner[p] == pos ? 1.0f : 0.0f;
    for (int l = 1; l < nl; ++l) {
      int nw, nh;
      pano_down_rgb(gi[l - 1], gv[l - 1], dims[l - 1].first, dims[l - 1].second, gi[l], gv[l], nw, nh);
      pano_down_scalar(gm[l - 1], dims[l - 1].first, dims[l - 1].second, gm[l]);
    }
    const int top = nl - 1;
    for (size_t i = 0; i < gm[top].size(); ++i) {
      const float w = gm[top][i];
      if (w > 0.0f && gv[top][i] > 1e-3f) {
        for (int c = 0; c < 3; ++c) bl[top][i][c] += w * gi[top][i][c];
        ms[top][i] += w;
      }
    }
    for (int l = 0; l < top; ++l) {
      std::vector<Rgb> ex;
      pano_up_rgb(gi[l + 1], dims[l + 1].first, dims[l + 1].second, dims[l].first, dims[l].second, ex);
      const size_t cnt = (size_t)dims[l].first * dims[l].second;
      for (size_t i = 0; i < cnt; ++i) {
        const float w = gm[l][i];
        if (w > 0.0f && gv[l][i] > 1e-3f) {
          for (int c = 0; c < 3; ++c) bl[l][i][c] += w * (gi[l][i][c] - ex[i][c]);
          ms[l][i] += w;
        }
      }
    }
  }
  for (int l = 0; l < nl; ++l)
    for (size_t i = 0; i < bl[l].size(); ++i) {
      const float m = ms[l][i];
      if (m > 1e-6f && std::fabs(m - 1.0f) > 1e-5f) {
        const float iv = 1.0f / m;
        for (int c = 0; c < 3; ++c) bl[l][i][c] *= iv;
      }
    }
  std::vector<Rgb> recon = bl[nl - 1];
  for (int l = nl - 2; l >= 0; --l) {
    std::vector<Rgb> up;
    pano_up_rgb(recon, dims[l + 1].first, dims[l + 1].second, dims[l].first, dims[l].second, up);
    for (size_t i = 0; i < up.size(); ++i)
      for (int c = 0; c < 3; ++c) up[i][c] = up[i][c] + bl[l][i][c];
    recon.swap(up);
  }
  for (size_t p = 0; p < np; ++p)
    if (owner[p] >= 0) {
      uint8_t* o = canvas + p * 4;
      for (int c = 0; c < 3; ++c) o[c] = ow_u8(std::round((double)recon[p][c]));
      o[3] = 255;
    }
}

}  // extern "C"
