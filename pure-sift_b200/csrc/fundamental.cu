// K13: fundamental-matrix LO-RANSAC (normalised 8-point, Sampson distance) on the
// GPU, one CTA per match set.
//
// Reference (src/geometry.rs): FundamentalRansacOptions (:107-143), mul_mat3 /
// transpose / det / normalize_frobenius / vector helpers (:145-207),
// jacobi_symmetric_eigen_9x9 (:209-295), jacobi_symmetric_eigen_3x3 (:297-372),
// svd_3x3 (:463-531), rank2_project_f (:533-545), normalize_points_2d
// (:547-583), assemble_fundamental_ata (:586-604), sampson_distance_sq
// (:617-636), fit_fundamental_8point (:638-665), solve_cubic_real (:667-725),
// fit_fundamental_7point (:727-806), evaluate_fundamental_hypothesis
// (:808-829), adaptive_epipolar_iters (:831-855),
// estimate_fundamental_ransac_with_options (:868-1016); the sampler of
// src/pipeline.rs:2006-2036.
//
// The reference's loop is replayed exactly: its draws are resolved in parallel
// (ransac_common.cuh), thread 0 walks them to form the same 8-index samples
// (distinct indices, at most 32 attempts), 64 samples are fitted at a time (one
// quad of lanes each, the reference's f64 operations in its order), each warp counts
// the inliers of 8 of them, and thread 0 takes every decision in order: count,
// the tie-break on the truncated error sum (the reference's sequential sum over
// the matches, evaluated only when a tie needs it), the adaptive iteration
// budget, then up to two LO refits over the ordered inlier list (the 45 entries
// of A^T A and the normalisation sums each accumulated in order by one thread).
// Results equal the reference's except where libm differs from CUDA's math
// functions: `hypot` in the point normalisation (glibc's is not correctly
// rounded), and `cbrt` / `acos` / `cos` in the 7-point solver.
#include <cmath>
#include <cstring>
#include <vector>

#include "psift_internal.cuh"
#include "ransac_common.cuh"

namespace psift {
namespace {

constexpr int kFThreads = 256;
constexpr int kFB = 64;      // hypotheses per batch
constexpr int kFWin = 2048;  // resolved draws per window (>= 32 per iteration)

struct FundJob {
  const psift_match* m;
  int n;
  double tsq, conf;
  int hard_cap, min_iters;
  uint64_t seed;
  double* cdf;    // n
  double* terms;  // n
  double* pts;    // 4 per match: the ordered inlier list's coordinates, gathered
  uint8_t* mask;
  double* f9;
  int* has_f;
  int* count;
  int* iters;
};

struct FShared {
  double F[kFB][9];
  int samp[kFB][8];
  int sok[kFB], fok[kFB], cnt[kFB], sdup[kFB];
  int draws[kFWin];
  double best[9], cand[9];
  double best_err;
  int best_err_known, best_count, have, max_iters, iter;
  int nb, refill;
  long long tpos, wb;
  // decision flags of the replay
  int act;
  double ev_err;
  int ev_cnt;
  // LO refit
  int list_n, fit_ok;
  double sums[6];  // qx qy tx ty (sums), then mean distances q, t
  double ata[9][9];
  uint32_t red_u[kFThreads / 32];
  int scan[kFThreads / 32];
};

// ------------------------------------------------------------ 3x3 / vector helpers
struct M3 {
  double v[3][3];
};

__device__ M3 m3_mul(const M3& a, const M3& b) {
  M3 o;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) o.v[r][c] = a.v[r][0] * b.v[0][c] + a.v[r][1] * b.v[1][c] + a.v[r][2] * b.v[2][c];
  return o;
}

__device__ M3 m3_tr(const M3& m) {
  M3 o;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) o.v[r][c] = m.v[c][r];
  return o;
}

__device__ double m3_det(const M3& m) {
  return m.v[0][0] * (m.v[1][1] * m.v[2][2] - m.v[1][2] * m.v[2][1]) -
         m.v[0][1] * (m.v[1][0] * m.v[2][2] - m.v[1][2] * m.v[2][0]) +
         m.v[0][2] * (m.v[1][0] * m.v[2][1] - m.v[1][1] * m.v[2][0]);
}

__device__ bool norm_frob(M3& m) {
  double s = 0.0;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) s += m.v[r][c] * m.v[r][c];
  if (!isfinite(s) || s < 1e-24) return false;
  const double inv = 1.0 / sqrt(s);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) m.v[r][c] *= inv;
  return true;
}

__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ bool normalize3(const double v[3], double o[3]) {
  const double n = sqrt(dot3(v, v));
  if (!isfinite(n) || n < 1e-12) return false;
  o[0] = v[0] / n;
  o[1] = v[1] / n;
  o[2] = v[2] / n;
  return true;
}

// One rotation of the reference's classical Jacobi (largest off-diagonal pivot,
// first in row-major order on ties): 1 continue, 0 converged, -1 non-finite.
template <int N>
__device__ int jacobi_step(double (&a)[N][N], double (&v)[N][N], double tol) {
  // the N(N-1)/2 magnitudes are loaded together, then scanned in row-major order
  constexpr int kOff = N * (N - 1) / 2;
  double mag[kOff];
  {
    int k = 0;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
      for (int j = i + 1; j < N; ++j) mag[k++] = fabs(a[i][j]);
  }
  int p = 0, q = 1;
  double max_off = 0.0;
  {
    int k = 0;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
      for (int j = i + 1; j < N; ++j, ++k)
        if (mag[k] > max_off) {
          max_off = mag[k];
          p = i;
          q = j;
        }
  }
  if (!isfinite(max_off)) return -1;
  if (max_off < tol) return 0;
  const double app = a[p][p], aqq = a[q][q], apq = a[p][q];
  const double tau = (aqq - app) / (2.0 * apq);
  // __drcp_rn(x) is 1.0 / x: both are IEEE round-to-nearest, the reciprocal is the cheaper sequence
  const double t = tau >= 0.0 ? __drcp_rn(tau + sqrt(1.0 + tau * tau)) : -__drcp_rn(-tau + sqrt(1.0 + tau * tau));
  const double c = __drcp_rn(sqrt(1.0 + t * t));
  const double s = t * c;
  a[p][p] = app - t * apq;
  a[q][q] = aqq + t * apq;
  a[p][q] = 0.0;
  a[q][p] = 0.0;
#pragma unroll
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
#pragma unroll
  for (int r = 0; r < N; ++r) {
    const double vrp = v[r][p], vrq = v[r][q];
    v[r][p] = c * vrp - s * vrq;
    v[r][q] = s * vrp + c * vrq;
  }
  return 1;
}

// jacobi_symmetric_eigen_9x9: the eigenvectors of the two smallest eigenvalues
// (ascending, stable order) as 3x3 matrices (one thread: the 7-point solver and
// the LO refits).
__device__ bool null2_of_ata(double (&a)[9][9], M3& f1, M3& f2) {
  double v[9][9];
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < 9; ++j) v[i][j] = i == j ? 1.0 : 0.0;
  for (int it = 0; it < 500; ++it) {
    const int r = jacobi_step<9>(a, v, 1e-13);
    if (r < 0) return false;
    if (r == 0) break;
  }
  int order[9];
  for (int i = 0; i < 9; ++i) order[i] = i;
  for (int i = 1; i < 9; ++i) {  // stable insertion sort by eigenvalue
    const int k = order[i];
    int j = i - 1;
    while (j >= 0 && a[k][k] < a[order[j]][order[j]]) {
      order[j + 1] = order[j];
      --j;
    }
    order[j + 1] = k;
  }
  for (int dc = 0; dc < 9; ++dc)
    for (int r = 0; r < 9; ++r)
      if (!isfinite(v[r][order[dc]])) return false;
  for (int k = 0; k < 9; ++k) {
    f1.v[k / 3][k % 3] = v[k][order[0]];
    f2.v[k / 3][k % 3] = v[k][order[1]];
  }
  return true;
}

// svd_3x3 + rank2_project_f.
__device__ bool rank2(M3& f) {
  const M3 m = f;
  M3 mtm = m3_mul(m3_tr(m), m);
  double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int it = 0; it < 100; ++it) {
    const int r = jacobi_step<3>(mtm.v, v, 1e-14);
    if (r < 0) return false;
    if (r == 0) break;
  }
  int order[3] = {0, 1, 2};
  for (int i = 1; i < 3; ++i) {  // stable, descending
    const int k = order[i];
    int j = i - 1;
    while (j >= 0 && mtm.v[order[j]][order[j]] < mtm.v[k][k]) {
      order[j + 1] = order[j];
      --j;
    }
    order[j + 1] = k;
  }
  double s[3], vm[3][3];
  for (int dc = 0; dc < 3; ++dc) {
    s[dc] = sqrt(fmax(mtm.v[order[dc]][order[dc]], 0.0));
    for (int r = 0; r < 3; ++r) vm[r][dc] = v[r][order[dc]];
  }
  auto mul_mv = [&](const double x[3], double o[3]) {
    for (int r = 0; r < 3; ++r) o[r] = m.v[r][0] * x[0] + m.v[r][1] * x[1] + m.v[r][2] * x[2];
  };
  const double v0[3] = {vm[0][0], vm[1][0], vm[2][0]}, v1[3] = {vm[0][1], vm[1][1], vm[2][1]},
               v2[3] = {vm[0][2], vm[1][2], vm[2][2]};
  double u0[3] = {1.0, 0.0, 0.0}, u1[3], u2[3], t[3];
  if (s[0] > 1e-12) {
    mul_mv(v0, t);
    if (!normalize3(t, u0)) u0[0] = 1.0, u0[1] = 0.0, u0[2] = 0.0;
  }
  auto fallback = [&](double o[3]) {
    const bool small = fabs(u0[0]) < 0.9;
    const double basis[3] = {small ? 1.0 : 0.0, small ? 0.0 : 1.0, 0.0};
    double c[3];
    cross3(u0, basis, c);
    if (!normalize3(c, o)) o[0] = 0.0, o[1] = 1.0, o[2] = 0.0;
  };
  if (s[1] > 1e-12) {
    double raw[3];
    mul_mv(v1, raw);
    const double proj = dot3(raw, u0);
    const double orth[3] = {raw[0] - proj * u0[0], raw[1] - proj * u0[1], raw[2] - proj * u0[2]};
    if (!normalize3(orth, u1)) fallback(u1);
  } else {
    fallback(u1);
  }
  cross3(u0, u1, t);
  if (!normalize3(t, u2)) return false;
  if (s[2] > 1e-12) {
    double mv2[3];
    mul_mv(v2, mv2);
    if (dot3(u2, mv2) < 0.0) u2[0] = -u2[0], u2[1] = -u2[1], u2[2] = -u2[2];
  }
  M3 u, d, vt;
  for (int r = 0; r < 3; ++r) {
    u.v[r][0] = u0[r];
    u.v[r][1] = u1[r];
    u.v[r][2] = u2[r];
    for (int c = 0; c < 3; ++c) {
      vt.v[r][c] = vm[c][r];
      d.v[r][c] = 0.0;
    }
  }
  d.v[0][0] = s[0];
  d.v[1][1] = s[1];
  f = m3_mul(u, m3_mul(d, vt));
  return norm_frob(f);
}

__device__ __forceinline__ M3 norm_T(double scale, double cx, double cy) {
  M3 t;
  t.v[0][0] = scale, t.v[0][1] = 0.0, t.v[0][2] = -scale * cx;
  t.v[1][0] = 0.0, t.v[1][1] = scale, t.v[1][2] = -scale * cy;
  t.v[2][0] = 0.0, t.v[2][1] = 0.0, t.v[2][2] = 1.0;
  return t;
}

// ata row of a normalised correspondence (assemble_fundamental_ata).
__device__ __forceinline__ void ata_row(double x1, double y1, double x2, double y2, double r[9]) {
  r[0] = x2 * x1, r[1] = x2 * y1, r[2] = x2, r[3] = y2 * x1, r[4] = y2 * y1, r[5] = y2, r[6] = x1, r[7] = y1,
  r[8] = 1.0;
}

// normalize_points_2d of k points (one thread): false when the reference returns None.
__device__ bool norm_pts(const double* x, const double* y, int k, double& cx, double& cy, double& scale) {
  const double inv_n = 1.0 / (double)k;
  cx = 0.0, cy = 0.0;
  for (int i = 0; i < k; ++i) {
    if (!isfinite(x[i]) || !isfinite(y[i])) return false;
    cx += x[i];
    cy += y[i];
  }
  cx *= inv_n;
  cy *= inv_n;
  double md = 0.0;
  for (int i = 0; i < k; ++i) md += hypot(x[i] - cx, y[i] - cy);
  md *= inv_n;
  if (!isfinite(md) || md < 1e-9) return false;
  scale = 1.41421356237309504880 / md;
  return true;
}

// Normalised points of k <= 8 matches -> T_q, T_t and A^T A (one thread).
__device__ bool small_ata(const psift_match* __restrict__ m, const int* idx, int k, M3& tq, M3& tt,
                          double (&ata)[9][9]) {
  double qx[8], qy[8], tx[8], ty[8];
  for (int i = 0; i < k; ++i) {
    const psift_match& a = m[idx[i]];
    qx[i] = (double)a.query_x, qy[i] = (double)a.query_y, tx[i] = (double)a.target_x, ty[i] = (double)a.target_y;
  }
  double qcx, qcy, qs, tcx, tcy, ts;
  if (!norm_pts(qx, qy, k, qcx, qcy, qs) || !norm_pts(tx, ty, k, tcx, tcy, ts)) return false;
  tq = norm_T(qs, qcx, qcy);
  tt = norm_T(ts, tcx, tcy);
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < 9; ++j) ata[i][j] = 0.0;
  for (int p = 0; p < k; ++p) {
    double r[9];
    ata_row((qx[p] - qcx) * qs, (qy[p] - qcy) * qs, (tx[p] - tcx) * ts, (ty[p] - tcy) * ts, r);
    for (int i = 0; i < 9; ++i)
      for (int j = i; j < 9; ++j) ata[i][j] += r[i] * r[j];
  }
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < i; ++j) ata[i][j] = ata[j][i];
  return true;
}

// jacobi_symmetric_eigen_9x9's rotations on A (eigenvectors accumulated in V),
// shared by a quad of lanes (see quad_fit8); false on a non-finite pivot.
// A and V are complete and visible to the quad on entry and on return.
__device__ bool quad_jacobi(double* A, double* V, int ql, unsigned qmask) {
  // this lane's 9 pivot candidates: upper-triangle entries 9 ql .. 9 ql + 8 in row-major order
  int ki[9], kj[9];
  {
    int i = 0, rem = 9 * ql;
    while (rem >= 8 - i) {
      rem -= 8 - i;
      ++i;
    }
    int j = i + 1 + rem;
#pragma unroll
    for (int s = 0; s < 9; ++s) {
      ki[s] = i;
      kj[s] = j;
      if (++j == 9) {
        ++i;
        j = i + 1;
      }
    }
  }
  bool finite = true;
  for (int it = 0; it < 500; ++it) {
    double mx = -1.0;
    int mk = 99;
#pragma unroll
    for (int s = 0; s < 9; ++s) {
      const double v = fabs(A[ki[s] * 9 + kj[s]]);
      if (v > mx) {
        mx = v;
        mk = 9 * ql + s;
      }
    }
#pragma unroll
    for (int o = 1; o <= 2; o <<= 1) {
      const double om = __shfl_xor_sync(qmask, mx, o);
      const int ok = __shfl_xor_sync(qmask, mk, o);
      if (om > mx || (om == mx && ok < mk)) {
        mx = om;
        mk = ok;
      }
    }
    if (!isfinite(mx)) {
      finite = false;
      break;
    }
    if (mx < 1e-13) break;
    int p = 0, rem = mk;
    while (rem >= 8 - p) {
      rem -= 8 - p;
      ++p;
    }
    const int q = p + 1 + rem;
    const double app = A[p * 9 + p], aqq = A[q * 9 + q], apq = A[p * 9 + q];
    const double tau = (aqq - app) / (2.0 * apq);
    const double t = tau >= 0.0 ? __drcp_rn(tau + sqrt(1.0 + tau * tau)) : -__drcp_rn(-tau + sqrt(1.0 + tau * tau));
    const double c = __drcp_rn(sqrt(1.0 + t * t));
    const double s = t * c;
    __syncwarp(qmask);  // every pivot read precedes the writes
    if (ql == 0) {
      A[p * 9 + p] = app - t * apq;
      A[q * 9 + q] = aqq + t * apq;
      A[p * 9 + q] = 0.0;
      A[q * 9 + p] = 0.0;
    }
    for (int r = ql; r < 9; r += 4) {
      if (r != p && r != q) {
        const double arp = A[r * 9 + p], arq = A[r * 9 + q];
        const double nrp = c * arp - s * arq, nrq = s * arp + c * arq;
        A[r * 9 + p] = nrp;
        A[p * 9 + r] = nrp;
        A[r * 9 + q] = nrq;
        A[q * 9 + r] = nrq;
      }
      const double vrp = V[r * 9 + p], vrq = V[r * 9 + q];
      V[r * 9 + p] = c * vrp - s * vrq;
      V[r * 9 + q] = s * vrp + c * vrq;
    }
    __syncwarp(qmask);
  }
  return finite;
}

// The leader's tail of jacobi_symmetric_eigen_9x9 (stable ascending order,
// finite eigenvectors) and of fit_fundamental_8point (rank 2, de-normalisation).
__device__ bool finish_from_eigen(const double* A, const double* V, const M3& tq, const M3& tt, double* out) {
  int order[9];
  for (int i = 0; i < 9; ++i) order[i] = i;
  for (int i = 1; i < 9; ++i) {
    const int k = order[i];
    int j = i - 1;
    while (j >= 0 && A[k * 9 + k] < A[order[j] * 9 + order[j]]) {
      order[j + 1] = order[j];
      --j;
    }
    order[j + 1] = k;
  }
  for (int dc = 0; dc < 9; ++dc)
    for (int r = 0; r < 9; ++r)
      if (!isfinite(V[r * 9 + order[dc]])) return false;
  M3 f1;
  for (int k = 0; k < 9; ++k) f1.v[k / 3][k % 3] = V[k * 9 + order[0]];
  if (!rank2(f1)) return false;
  M3 f = m3_mul(m3_tr(tt), m3_mul(f1, tq));
  if (!norm_frob(f)) return false;
  for (int i = 0; i < 9; ++i) out[i] = f.v[i / 3][i % 3];
  return true;
}

// fit_fundamental_8point of one sample by a quad of lanes (ql = 0..3, converged,
// qmask their lane mask); A and V (81 doubles each, shared memory) hold the
// Jacobi matrix and eigenvectors.  Every lane computes the normalisation; the 45
// A^T A entries and the rotations' row updates are split over the lanes; each
// lane scans 9 of the 36 pivot candidates in row-major order and the quad keeps
// the first largest, so every value and decision is the sequential solver's.
// The result (out, return value) is the leader's (ql == 0).
__device__ bool quad_fit8(const psift_match* __restrict__ m, const int* idx, double* A, double* V, int ql,
                          unsigned qmask, double* out) {
  double qx[8], qy[8], tx[8], ty[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const psift_match& a = m[idx[i]];
    qx[i] = (double)a.query_x, qy[i] = (double)a.query_y, tx[i] = (double)a.target_x, ty[i] = (double)a.target_y;
  }
  double qcx, qcy, qs, tcx, tcy, ts;
  if (!norm_pts(qx, qy, 8, qcx, qcy, qs) || !norm_pts(tx, ty, 8, tcx, tcy, ts)) return false;
  for (int e = ql; e < 45; e += 4) {
    int i = 0, rem = e;
    while (rem >= 9 - i) {
      rem -= 9 - i;
      ++i;
    }
    const int j = i + rem;
    double sum = 0.0;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      double r[9];
      ata_row((qx[p] - qcx) * qs, (qy[p] - qcy) * qs, (tx[p] - tcx) * ts, (ty[p] - tcy) * ts, r);
      sum += r[i] * r[j];
    }
    A[i * 9 + j] = sum;
    A[j * 9 + i] = sum;
  }
  for (int r = ql; r < 9; r += 4)
#pragma unroll
    for (int c = 0; c < 9; ++c) V[r * 9 + c] = r == c ? 1.0 : 0.0;
  __syncwarp(qmask);
  const bool finite = quad_jacobi(A, V, ql, qmask);
  if (ql != 0 || !finite) return false;
  return finish_from_eigen(A, V, norm_T(qs, qcx, qcy), norm_T(ts, tcx, tcy), out);
}

__device__ __forceinline__ double sampson(const double* f, const psift_match& a) {
  const double x1 = (double)a.query_x, y1 = (double)a.query_y, x2 = (double)a.target_x, y2 = (double)a.target_y;
  const double a0 = f[0] * x1 + f[1] * y1 + f[2];
  const double a1 = f[3] * x1 + f[4] * y1 + f[5];
  const double a2 = f[6] * x1 + f[7] * y1 + f[8];
  const double b0 = f[0] * x2 + f[3] * y2 + f[6];
  const double b1 = f[1] * x2 + f[4] * y2 + f[7];
  const double e = x2 * a0 + y2 * a1 + a2;
  const double den = a0 * a0 + a1 * a1 + b0 * b0 + b1 * b1;
  if (den < 1e-18 || !isfinite(den)) return __longlong_as_double(0x7ff0000000000000ll);
  return (e * e) / den;
}

// sampson(f, a) <= tsq without the division where the comparison is clear:
// with ee = e * e and p = tsq * den (both rounded), ee / den <= tsq when
// ee <= p (1 - 2^-50) and round(ee / den) > tsq when ee >= p (1 + 2^-50) (the
// margins cover the roundings of p, of the margin product and of the quotient);
// in between, and for NaN, the reference's quotient decides.
__device__ __forceinline__ bool sampson_in(const double* f, const psift_match& a, double tsq) {
  const double x1 = (double)a.query_x, y1 = (double)a.query_y, x2 = (double)a.target_x, y2 = (double)a.target_y;
  const double a0 = f[0] * x1 + f[1] * y1 + f[2];
  const double a1 = f[3] * x1 + f[4] * y1 + f[5];
  const double a2 = f[6] * x1 + f[7] * y1 + f[8];
  const double b0 = f[0] * x2 + f[3] * y2 + f[6];
  const double b1 = f[1] * x2 + f[4] * y2 + f[7];
  const double e = x2 * a0 + y2 * a1 + a2;
  const double den = a0 * a0 + a1 * a1 + b0 * b0 + b1 * b1;
  if (den < 1e-18 || !isfinite(den)) return false;  // infinite distance
  const double ee = e * e;
  const double p = tsq * den;
  if (ee <= p * (1.0 - 0x1p-50)) return true;
  if (ee >= p * (1.0 + 0x1p-50)) return false;
  return ee / den <= tsq;
}

// powi as the compiler runtime evaluates it (square-and-multiply, low bit first).
__device__ double powi_d(double a, int b) {
  double r = 1.0;
  for (;;) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return r;
}

// adaptive_epipolar_iters with sample size 8.
__device__ int adaptive_epipolar(int best, int total, double conf, int min_it, int max_it) {
  if (total <= 8 || best == 0) return max_it;
  const double w = (double)best / (double)total;
  if (w >= 0.9999) return min_it;
  const double pg = powi_d(w, 8);
  if (pg <= 1e-12) return max_it;
  const double den = log(fmax(1.0 - pg, 1e-15));
  const double c = conf < 0.5 ? 0.5 : (conf > 0.999999 ? 0.999999 : conf);
  const double num = log(1.0 - c);
  const double est = ceil(num / den);
  // `as usize` saturates (NaN -> 0), then clamp(min, max)
  double e = est == est ? est : 0.0;
  e = e < (double)min_it ? (double)min_it : (e > (double)max_it ? (double)max_it : e);
  return (int)e;
}

// solve_cubic_real.
__device__ int cubic_roots(double c3, double c2, double c1, double c0, double* roots) {
  int k = 0;
  if (fabs(c3) < 1e-12) {
    if (fabs(c2) < 1e-12) {
      if (fabs(c1) < 1e-12) return 0;
      roots[0] = -c0 / c1;
      return 1;
    }
    const double disc = c1 * c1 - 4.0 * c2 * c0;
    if (disc < 0.0) return 0;
    const double sq = sqrt(disc);
    roots[0] = (-c1 + sq) / (2.0 * c2);
    roots[1] = (-c1 - sq) / (2.0 * c2);
    return 2;
  }
  const double a = c2 / c3, b = c1 / c3, c = c0 / c3;
  const double a3 = a / 3.0;
  const double p = b - a * a3;
  const double q = (2.0 * a * a * a) / 27.0 - (a * b) / 3.0 + c;
  const double disc = (q * 0.5) * (q * 0.5) + powi_d(p / 3.0, 3);
  if (disc > 1e-14) {
    const double sq = sqrt(disc);
    roots[k++] = cbrt(-0.5 * q + sq) + cbrt(-0.5 * q - sq) - a3;
  } else if (disc >= -1e-14) {
    const double u = cbrt(-0.5 * q);
    roots[k++] = 2.0 * u - a3;
    roots[k++] = -u - a3;
  } else {
    const double r = sqrt(-p / 3.0);
    double cp = (-0.5 * q) / (r * r * r);
    cp = cp < -1.0 ? -1.0 : (cp > 1.0 ? 1.0 : cp);
    const double phi = acos(cp);
    const double two_r = 2.0 * r;
    const double pi = 3.14159265358979323846;
    roots[k++] = two_r * cos(phi / 3.0) - a3;
    roots[k++] = two_r * cos((phi + 2.0 * pi) / 3.0) - a3;
    roots[k++] = two_r * cos((phi + 4.0 * pi) / 3.0) - a3;
  }
  for (int i = 0; i < k; ++i)
    for (int it = 0; it < 3; ++it) {
      const double t = roots[i];
      const double fv = ((c3 * t + c2) * t + c1) * t + c0;
      const double df = (3.0 * c3 * t + 2.0 * c2) * t + c1;
      if (fabs(df) > 1e-14) roots[i] = t - fv / df;
    }
  return k;
}

// ------------------------------------------------------------ block helpers
__device__ int block_sum(int v, FShared& S) {
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) S.red_u[threadIdx.x >> 5] = (uint32_t)v;
  __syncthreads();
  int t = 0;
  for (int w = 0; w < kFThreads / 32; ++w) t += (int)S.red_u[w];
  __syncthreads();
  return t;
}

// Sequential sum of v[0..n) in order, the loads issued kSeqAhead at a time ahead
// of the dependent adds (one thread).
constexpr int kSeqAhead = 16;
__device__ double seq_sum(const double* __restrict__ v, int n) {
  double acc = 0.0;
  int i = 0;
  for (; i + kSeqAhead <= n; i += kSeqAhead) {
    double w[kSeqAhead];
#pragma unroll
    for (int k = 0; k < kSeqAhead; ++k) w[k] = v[i + k];
#pragma unroll
    for (int k = 0; k < kSeqAhead; ++k) acc += w[k];
  }
  for (; i < n; ++i) acc += v[i];
  return acc;
}

// evaluate_fundamental_hypothesis of f (shared): count (whole CTA) and the
// truncated error sum in match order (terms in parallel, summed by thread 0).
__device__ void evaluate(const FundJob& J, FShared& S, const double* f, int& count, double& err) {
  int c = 0;
  for (int i = threadIdx.x; i < J.n; i += kFThreads) {
    const double d2 = sampson(f, J.m[i]);
    const bool in = d2 <= J.tsq;
    c += in;
    J.terms[i] = in ? d2 : J.tsq;
  }
  count = block_sum(c, S);  // its barriers also order the term stores before the sum
  if (threadIdx.x == 0) S.ev_err = seq_sum(J.terms, J.n);
  __syncthreads();
  err = S.ev_err;
  __syncthreads();
}

// Ordered inlier list of S.best, its coordinates gathered into J.pts; returns its
// length (whole CTA).
__device__ int collect(const FundJob& J, FShared& S) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int base = 0;
  for (int b0 = 0; b0 < J.n; b0 += kFThreads) {
    const int i = b0 + threadIdx.x;
    const bool in = i < J.n && sampson(S.best, J.m[i]) <= J.tsq;
    const uint32_t bal = __ballot_sync(0xffffffffu, in);
    if (lane == 0) S.scan[warp] = __popc(bal);
    __syncthreads();
    int off = base;
    for (int w = 0; w < warp; ++w) off += S.scan[w];
    if (in) {
      const int pos = off + __popc(bal & ((1u << lane) - 1u));
      const psift_match& a = J.m[i];
      reinterpret_cast<double4*>(J.pts)[pos] =
          make_double4((double)a.query_x, (double)a.query_y, (double)a.target_x, (double)a.target_y);
    }
    int tot = 0;
    for (int w = 0; w < kFThreads / 32; ++w) tot += S.scan[w];
    base += tot;
    __syncthreads();
  }
  return base;
}

// fit_fundamental_8point over the gathered inliers J.pts[0..k) (k >= 8) into
// S.cand; S.fit_ok.  Every sum runs over the list in order, one thread each, with
// the coordinates of kSeqAhead points loaded ahead of the dependent adds.
__device__ void fit_list(const FundJob& J, FShared& S, double* jac, int k) {
  const int t = threadIdx.x;
  const double4* P = reinterpret_cast<const double4*>(J.pts);
  auto coord = [](const double4& p, int c) { return c == 0 ? p.x : c == 1 ? p.y : c == 2 ? p.z : p.w; };
  if (t < 4) {  // normalisation sums: qx, qy, tx, ty
    double s = 0.0;
    bool fin = true;
    int i = 0;
    for (; i + kSeqAhead <= k; i += kSeqAhead) {
      double w[kSeqAhead];
#pragma unroll
      for (int q = 0; q < kSeqAhead; ++q) w[q] = coord(P[i + q], t);
#pragma unroll
      for (int q = 0; q < kSeqAhead; ++q) {
        fin = fin && isfinite(w[q]);
        s += w[q];
      }
    }
    for (; i < k; ++i) {
      const double w = coord(P[i], t);
      fin = fin && isfinite(w);
      s += w;
    }
    S.sums[t] = fin ? s : __longlong_as_double(0x7ff8000000000000ll);
  }
  __syncthreads();
  const double inv_n = 1.0 / (double)k;
  const double qcx = S.sums[0] * inv_n, qcy = S.sums[1] * inv_n, tcx = S.sums[2] * inv_n, tcy = S.sums[3] * inv_n;
  if (t < 2) {  // mean distances to the centroid: query, target
    const double cx = t == 0 ? qcx : tcx, cy = t == 0 ? qcy : tcy;
    double md = 0.0;
    int i = 0;
    for (; i + kSeqAhead <= k; i += kSeqAhead) {
      double w[kSeqAhead];
#pragma unroll
      for (int q = 0; q < kSeqAhead; ++q) {
        const double4 p = P[i + q];
        w[q] = t == 0 ? hypot(p.x - cx, p.y - cy) : hypot(p.z - cx, p.w - cy);
      }
#pragma unroll
      for (int q = 0; q < kSeqAhead; ++q) md += w[q];
    }
    for (; i < k; ++i) {
      const double4 p = P[i];
      md += t == 0 ? hypot(p.x - cx, p.y - cy) : hypot(p.z - cx, p.w - cy);
    }
    S.sums[4 + t] = md * inv_n;
  }
  __syncthreads();
  const double qmd = S.sums[4], tmd = S.sums[5];
  const bool ok = isfinite(S.sums[0]) && isfinite(S.sums[1]) && isfinite(S.sums[2]) && isfinite(S.sums[3]) &&
                  isfinite(qmd) && qmd >= 1e-9 && isfinite(tmd) && tmd >= 1e-9;
  const double qs = 1.41421356237309504880 / qmd, ts = 1.41421356237309504880 / tmd;
  // A^T A: entry (i, j), j >= i, one thread each, summed over the list in order
  if (ok && t < 45) {
    int i = 0, rem = t;
    while (rem >= 9 - i) {
      rem -= 9 - i;
      ++i;
    }
    const int j = i + rem;
    // row entry k of assemble_fundamental_ata is U[k / 3] * W[k % 3] with
    // U = (x2, y2, 1), W = (x1, y1, 1) (the 1 factors are exact): r_i * r_j
    // without a per-point array
    const int ui = i / 3, wi = i % 3, uj = j / 3, wj = j % 3;
    auto term = [&](const double4& p) {
      const double x1 = (p.x - qcx) * qs, y1 = (p.y - qcy) * qs, x2 = (p.z - tcx) * ts, y2 = (p.w - tcy) * ts;
      const double u_i = ui == 0 ? x2 : (ui == 1 ? y2 : 1.0), w_i = wi == 0 ? x1 : (wi == 1 ? y1 : 1.0);
      const double u_j = uj == 0 ? x2 : (uj == 1 ? y2 : 1.0), w_j = wj == 0 ? x1 : (wj == 1 ? y1 : 1.0);
      return (u_i * w_i) * (u_j * w_j);
    };
    double s = 0.0;
    int p0 = 0;
    for (; p0 + kSeqAhead <= k; p0 += kSeqAhead) {
      double w[kSeqAhead];
#pragma unroll
      for (int q = 0; q < kSeqAhead; ++q) w[q] = term(P[p0 + q]);
#pragma unroll
      for (int q = 0; q < kSeqAhead; ++q) s += w[q];
    }
    for (; p0 < k; ++p0) s += term(P[p0]);
    S.ata[i][j] = s;
    S.ata[j][i] = s;
  }
  __syncthreads();
  if (t < 4) {  // the eigen-decomposition by the first quad, in the (now free) slot of sample 0
    const unsigned qmask = 0xFu;
    double* A = jac;
    double* V = jac + 81;
    bool good = ok;
    if (good) {
      for (int e = t; e < 81; e += 4) {
        A[e] = S.ata[e / 9][e % 9];
        V[e] = e / 9 == e % 9 ? 1.0 : 0.0;
      }
      __syncwarp(qmask);
      const bool fin = quad_jacobi(A, V, t, qmask);
      if (t == 0) good = fin && finish_from_eigen(A, V, norm_T(qs, qcx, qcy), norm_T(ts, tcx, tcy), S.cand);
    }
    if (t == 0) S.fit_ok = good ? 1 : 0;
  }
  __syncthreads();
}

// n == 7: fit_fundamental_7point and the best candidate (thread 0).
__device__ void seven_point(const FundJob& J, FShared& S) {
  const int idx[7] = {0, 1, 2, 3, 4, 5, 6};
  M3 tq, tt;
  double ata[9][9];
  S.have = 0;
  if (!small_ata(J.m, idx, 7, tq, tt, ata)) return;
  M3 f1, f2;
  if (!null2_of_ata(ata, f1, f2)) return;
  M3 b;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) b.v[r][c] = f1.v[r][c] - f2.v[r][c];
  auto eval_m = [&](double t) {
    M3 m;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) m.v[r][c] = f2.v[r][c] + t * b.v[r][c];
    return m;
  };
  const double p0 = m3_det(f2), p1 = m3_det(eval_m(1.0)), pm1 = m3_det(eval_m(-1.0)), p2 = m3_det(eval_m(2.0));
  const double c0 = p0;
  const double c2 = 0.5 * (p1 + pm1) - c0;
  const double s1 = 0.5 * (p1 - pm1);
  const double s2 = p2 - c0 - 4.0 * c2;
  const double c3 = (s2 - 2.0 * s1) / 6.0;
  const double c1 = s1 - c3;
  double roots[3];
  const int nr = cubic_roots(c3, c2, c1, c0, roots);
  const M3 ttt = m3_tr(tt);
  M3 cands[4];
  int nc = 0;
  for (int i = 0; i < nr; ++i) {
    if (!isfinite(roots[i])) continue;
    M3 f = m3_mul(ttt, m3_mul(eval_m(roots[i]), tq));
    if (norm_frob(f)) cands[nc++] = f;
  }
  if (fabs(c3) < 1e-12 && fabs(m3_det(b)) < 1e-10) {
    M3 f = m3_mul(ttt, m3_mul(b, tq));
    if (norm_frob(f)) cands[nc++] = f;
  }
  int best_count = 0;
  double best_err = __longlong_as_double(0x7ff0000000000000ll);
  for (int c = 0; c < nc; ++c) {
    double f9[9];
    for (int i = 0; i < 9; ++i) f9[i] = cands[c].v[i / 3][i % 3];
    int cnt = 0;
    double err = 0.0;
    for (int i = 0; i < 7; ++i) {
      const double d2 = sampson(f9, J.m[i]);
      if (d2 <= J.tsq) {
        ++cnt;
        err += d2;
      } else {
        err += J.tsq;
      }
    }
    if (cnt > best_count || (cnt == best_count && err < best_err)) {
      best_count = cnt;
      best_err = err;
      for (int i = 0; i < 9; ++i) S.best[i] = f9[i];
      S.have = 1;
    }
  }
}

constexpr size_t kJacSmem = sizeof(double) * 162 * kFB;  // A and V of every sample of a batch

__global__ void __launch_bounds__(kFThreads) fundamental_kernel(const FundJob* __restrict__ jobs) {
  __shared__ FShared S;
  extern __shared__ double jac[];
  const FundJob& J = jobs[blockIdx.x];
  const int n = J.n, t = threadIdx.x;
  if (t == 0) {
    *J.has_f = 0;
    *J.count = 0;
    if (J.iters) *J.iters = 0;
    S.have = 0;
  }
  for (int i = t; i < n; i += kFThreads) J.mask[i] = 0;
  if (n < 7) return;
  if (n == 7) {
    if (t == 0) seven_point(J, S);
    __syncthreads();
  } else {
    // build_ratio_weighted_cdf: weights in parallel, the running sum in order
    for (int i = t; i < n; i += kFThreads) {
      const float rf = J.m[i].ratio;
      double r = 1.0;
      if (isfinite(rf)) r = fmin(fmax((double)rf, 0.05), 1.0);
      J.cdf[i] = 1.0 / r;
    }
    __syncthreads();
    if (t == 0) {
      double acc = 0.0;
      int i = 0;
      for (; i + kSeqAhead <= n; i += kSeqAhead) {
        double w[kSeqAhead];
#pragma unroll
        for (int q = 0; q < kSeqAhead; ++q) w[q] = J.cdf[i + q];
#pragma unroll
        for (int q = 0; q < kSeqAhead; ++q) {
          acc += w[q];
          J.cdf[i + q] = acc;
        }
      }
      for (; i < n; ++i) {
        acc += J.cdf[i];
        J.cdf[i] = acc;
      }
      S.ev_err = acc;
      S.best_count = 0;
      S.best_err = __longlong_as_double(0x7ff0000000000000ll);
      S.best_err_known = 1;
      S.max_iters = J.hard_cap;
      S.iter = 0;
      S.tpos = 0;
      S.wb = 0;
    }
    __syncthreads();
    if (S.ev_err > 0.0) {
      const double inv = 1.0 / S.ev_err;
      for (int i = t; i < n; i += kFThreads) J.cdf[i] *= inv;
    }
    __syncthreads();
    if (t == 0) J.cdf[n - 1] = 1.0;
    for (int k = t; k < kFWin; k += kFThreads) S.draws[k] = sample_at(J.cdf, n, J.seed, (uint64_t)k);
    __syncthreads();

    while (S.iter < S.max_iters) {
      // 1. samples of the next iterations (thread 0 walks the resolved draws)
      const int want = min(kFB, S.max_iters - S.iter);
      if (t == 0) S.nb = 0;
      __syncthreads();
      while (true) {
        // Speculation: almost every iteration's first 8 draws are distinct, so
        // iteration nb0 + k uses draws tp0 + 8k .. tp0 + 8k + 7 until the first one
        // holding a repeat; thread 0 walks on from there as the reference does.
        {
          const int nb0 = S.nb;
          const long long tp0 = S.tpos;
          const long long room = S.wb + kFWin - 32 - tp0;  // iteration k needs tp0 + 8k + 32 <= wb + kFWin
          const int K = room < 0 ? 0 : (int)min((long long)(want - nb0), room / 8 + 1);
          if (t < K) {
            int d[8];
            const int base = (int)(tp0 - S.wb) + 8 * t;
#pragma unroll
            for (int q = 0; q < 8; ++q) d[q] = S.draws[base + q];
            bool dup = false;
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
              for (int b = a + 1; b < 8; ++b) dup = dup || d[a] == d[b];
            S.sdup[t] = dup ? 1 : 0;
            if (!dup)
#pragma unroll
              for (int q = 0; q < 8; ++q) S.samp[nb0 + t][q] = d[q];
          }
          __syncthreads();
          if (t == 0) {
            int k = 0;
            while (k < K && !S.sdup[k]) S.sok[nb0 + k++] = 1;
            S.nb = nb0 + k;
            S.tpos = tp0 + 8ll * k;
          }
          __syncthreads();
        }
        if (t == 0) {
          int nb = S.nb;
          long long tp = S.tpos;
          while (nb < want && tp + 32 <= S.wb + kFWin) {
            int idx[8], chosen = 0, attempts = 0;
            while (chosen < 8 && attempts < 32) {
              ++attempts;
              const int c = S.draws[(int)(tp - S.wb)];
              ++tp;
              bool dup = false;
              for (int k = 0; k < chosen; ++k) dup = dup || idx[k] == c;
              if (!dup) idx[chosen++] = c;
            }
            for (int k = 0; k < 8; ++k) S.samp[nb][k] = k < chosen ? idx[k] : 0;
            S.sok[nb] = chosen == 8;
            ++nb;
          }
          S.nb = nb;
          S.tpos = tp;
          S.refill = nb < want;
        }
        __syncthreads();
        if (!S.refill) break;
        const long long wb = S.tpos;
        for (int k = t; k < kFWin; k += kFThreads) S.draws[k] = sample_at(J.cdf, n, J.seed, (uint64_t)(wb + k));
        __syncthreads();
        if (t == 0) S.wb = wb;
        __syncthreads();
      }
      const int nb = S.nb;
      // 2. fits, a quad of lanes per sample
      {
        const int h = t >> 2, ql = t & 3;
        const unsigned qmask = 0xFu << (t & 28);
        if (h < nb) {
          bool ok = false;
          if (S.sok[h]) ok = quad_fit8(J.m, S.samp[h], jac + h * 162, jac + h * 162 + 81, ql, qmask, S.F[h]);
          if (ql == 0) S.fok[h] = ok ? 1 : 0;
        }
      }
      __syncthreads();
      // 3. inlier counts: warp w takes hypotheses w, w + 8, ...
      {
        const int lane = t & 31, warp = t >> 5;
        // two hypotheses per pass over the matches (one load, two independent evaluations)
        for (int h = warp; h < nb; h += 2 * (kFThreads / 32)) {
          const int h2 = h + kFThreads / 32;
          const bool v1 = S.fok[h] != 0, v2 = h2 < nb && S.fok[h2] != 0;
          int c1 = 0, c2 = 0;
          if (v1 || v2) {
            double f1[9], f2[9];
            for (int i = 0; i < 9; ++i) {
              f1[i] = S.F[h][i];
              f2[i] = h2 < nb ? S.F[h2][i] : 0.0;
            }
            for (int i = lane; i < n; i += 32) {
              const psift_match& a = J.m[i];
              c1 += v1 && sampson_in(f1, a, J.tsq);
              c2 += v2 && sampson_in(f2, a, J.tsq);
            }
          }
          for (int o = 16; o >= 1; o >>= 1) {
            c1 += __shfl_xor_sync(0xffffffffu, c1, o);
            c2 += __shfl_xor_sync(0xffffffffu, c2, o);
          }
          if (lane == 0) {
            S.cnt[h] = c1;
            if (h2 < nb) S.cnt[h2] = c2;
          }
        }
      }
      __syncthreads();
      // 4. the reference's decisions, in order
      for (int k = 0; k < nb; ++k) {
        if (t == 0) {
          S.act = 0;  // 0 nothing, 1 stop, 2 tie needs errors
          if (S.iter >= S.max_iters) {
            S.act = 1;
          } else {
            ++S.iter;
            if (S.sok[k] && S.fok[k]) {
              const int c = S.cnt[k];
              if (c > S.best_count) {
                S.best_count = c;
                for (int i = 0; i < 9; ++i) S.best[i] = S.F[k][i];
                S.best_err_known = 0;
                S.have = 1;
                S.max_iters = adaptive_epipolar(c, n, J.conf, J.min_iters, J.hard_cap);
              } else if (c == S.best_count) {
                S.act = 2;
              }
            }
          }
        }
        __syncthreads();
        if (S.act == 1) break;
        if (S.act == 2) {
          int c;
          double e;
          if (!S.best_err_known) {
            evaluate(J, S, S.best, c, e);
            if (t == 0) {
              S.best_err = e;
              S.best_err_known = 1;
            }
          }
          evaluate(J, S, S.F[k], c, e);
          if (t == 0 && e < S.best_err) {
            S.best_err = e;
            for (int i = 0; i < 9; ++i) S.best[i] = S.F[k][i];
            S.have = 1;
            S.max_iters = adaptive_epipolar(S.best_count, n, J.conf, J.min_iters, J.hard_cap);
          }
        }
        __syncthreads();  // every thread has read S.act before thread 0 rewrites it
      }
      __syncthreads();
    }
    if (t == 0 && J.iters) *J.iters = S.iter;
    // 5. LO refits over the ordered inlier list
    if (S.have) {
      for (int round = 0; round < 2; ++round) {
        const int k = collect(J, S);
        if (k < 8) break;
        fit_list(J, S, jac, k);
        if (!S.fit_ok) break;
        int c;
        double e;
        evaluate(J, S, S.cand, c, e);
        if (!S.best_err_known) {
          int c2;
          double e2;
          evaluate(J, S, S.best, c2, e2);
          if (t == 0) {
            S.best_err = e2;
            S.best_err_known = 1;
          }
          __syncthreads();
        }
        const bool better = c > S.best_count || (c == S.best_count && e < S.best_err);
        __syncthreads();
        if (!better) break;
        if (t == 0) {
          S.best_count = c;
          S.best_err = e;
          for (int i = 0; i < 9; ++i) S.best[i] = S.cand[i];
        }
        __syncthreads();
      }
    }
  }
  __syncthreads();
  if (!S.have) return;
  int c = 0;
  for (int i = t; i < n; i += kFThreads) {
    const bool in = sampson(S.best, J.m[i]) <= J.tsq;
    J.mask[i] = in ? 1 : 0;
    c += in;
  }
  c = block_sum(c, S);
  if (t == 0) {
    *J.count = c;
    *J.has_f = 1;
    for (int i = 0; i < 9; ++i) J.f9[i] = S.best[i];
  }
}

psift_status validate_fundamental_options(psift_ctx* ctx, const psift_fundamental_options* o) {
  if (!o) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null fundamental options");
  if (!(o->sampson_threshold == o->sampson_threshold) || !(o->confidence == o->confidence))
    return set_error(ctx, PSIFT_ERR_INVALID_CONFIG, "sampson_threshold and confidence must not be NaN");
  return PSIFT_OK;
}

psift_status run_fundamental(psift_ctx* ctx, const psift_fundamental_job* jobs, int n,
                             const psift_fundamental_options& o) {
  size_t bytes = sizeof(FundJob) * (size_t)n + 4096;
  for (int i = 0; i < n; ++i) bytes += 48 * (size_t)jobs[i].n + 3 * 256;
  psift_status st = arena_reserve(ctx, bytes);
  if (st != PSIFT_OK) return st;
  FundJob* d_jobs = (FundJob*)arena_alloc(ctx, sizeof(FundJob) * n);
  std::vector<FundJob> hj(n);
  const double thr = fmax(o.sampson_threshold, 0.25);
  const int hard_cap = (int)std::min<uint64_t>(std::max<uint64_t>(o.max_iters, 64), 0x7FFFFFFF);
  for (int i = 0; i < n; ++i) {
    const psift_fundamental_job& J = jobs[i];
    FundJob& F = hj[i];
    F.m = J.matches;
    F.n = (int)J.n;
    F.tsq = thr * thr;
    F.conf = o.confidence;
    F.hard_cap = hard_cap;
    F.min_iters = std::min(64, hard_cap);
    F.seed = o.seed;
    F.cdf = (double*)arena_alloc(ctx, 8 * (size_t)J.n + 8);
    F.terms = (double*)arena_alloc(ctx, 8 * (size_t)J.n + 8);
    F.pts = (double*)arena_alloc(ctx, 32 * (size_t)J.n + 32);
    F.mask = J.inlier_mask;
    F.f9 = J.f9;
    F.has_f = J.has_f;
    F.count = (int*)J.inlier_count;
    F.iters = (int*)J.iterations;
    if (!F.pts) return set_error(ctx, PSIFT_ERR_INTERNAL, "fundamental workspace carve overflow");
  }
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_jobs, hj.data(), sizeof(FundJob) * n, cudaMemcpyHostToDevice, ctx->stream));
  StageScope sc(ctx, STAGE_RANSAC);
  cudaError_t ea = ensure_smem_attr((const void*)fundamental_kernel, kJacSmem);
  if (ea != cudaSuccess) return cuda_error(ctx, ea, "cudaFuncSetAttribute(fundamental_kernel)");
  fundamental_kernel<<<n, kFThreads, kJacSmem, ctx->stream>>>(d_jobs);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(ctx, e, "fundamental_ransac");
  return PSIFT_OK;
}

}  // namespace
}  // namespace psift

using namespace psift;

extern "C" {

void psift_fundamental_options_default(psift_fundamental_options* o) {
  if (!o) return;
  o->sampson_threshold = 1.5;
  o->max_iters = 2000;
  o->confidence = 0.999;
  o->seed = 0xF00DCAFE12345678ull;
}

psift_status psift_fundamental_batch_dev(psift_ctx* ctx, const psift_fundamental_job* jobs, uint32_t n,
                                         const psift_fundamental_options* opt) {
  if (!ctx || (n && !jobs)) return PSIFT_ERR_INVALID_ARGUMENT;
  psift_status st = validate_fundamental_options(ctx, opt);
  if (st != PSIFT_OK) return st;
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaSetDevice");
  for (uint32_t i = 0; i < n; ++i) {
    const psift_fundamental_job& J = jobs[i];
    if (!J.f9 || !J.has_f || !J.inlier_count || (J.n && (!J.matches || !J.inlier_mask)))
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null pointer in fundamental job");
    if (J.n > 0x7FFFFFFFu) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "more than 2^31-1 matches");
  }
  if (n == 0) return PSIFT_OK;
  return run_fundamental(ctx, jobs, (int)n, *opt);
}

psift_status psift_fundamental_estimate(psift_ctx* ctx, const psift_match* matches, uint32_t n,
                                        const psift_fundamental_options* opt, uint8_t* inlier_mask, double* f9,
                                        int32_t* has_f, uint32_t* inlier_count, uint32_t* iterations) {
  if (!ctx || !f9 || !has_f || !inlier_count) return PSIFT_ERR_INVALID_ARGUMENT;
  if (n && (!matches || !inlier_mask)) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null matches/mask");
  psift_status st = validate_fundamental_options(ctx, opt);
  if (st != PSIFT_OK) return st;
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaSetDevice");
  const size_t mb = sizeof(psift_match) * (size_t)n;
  if ((st = io_reserve(ctx, mb + n + 4096)) != PSIFT_OK) return st;
  char* base = ctx->io.base;
  psift_match* d_m = (psift_match*)base;
  uint8_t* d_mask = (uint8_t*)(base + align_up(mb, 256));
  char* d_out = base + align_up(mb, 256) + align_up((size_t)n + 1, 256);  // 9 f64, then has, count, iters
  if (n) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_m, matches, mb, cudaMemcpyHostToDevice, ctx->stream));
  psift_fundamental_job job{d_m, n, d_mask, (double*)d_out, (int32_t*)(d_out + 72), (uint32_t*)(d_out + 76),
                            (uint32_t*)(d_out + 80)};
  if ((st = run_fundamental(ctx, &job, 1, *opt)) != PSIFT_OK) return st;
  if ((st = pinned_reserve(ctx, (size_t)n + 512)) != PSIFT_OK) return st;
  char* pin = ctx->pinned.base;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(pin, d_out, 84, cudaMemcpyDeviceToHost, ctx->stream));
  if (n) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(pin + 128, d_mask, n, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(f9, pin, 72);
  std::memcpy(has_f, pin + 72, 4);
  std::memcpy(inlier_count, pin + 76, 4);
  if (iterations) std::memcpy(iterations, pin + 80, 4);
  if (n) std::memcpy(inlier_mask, pin + 128, n);
  return PSIFT_OK;
}

}  // extern "C"
