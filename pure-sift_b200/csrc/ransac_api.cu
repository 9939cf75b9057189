// C-ABI entry points of the RANSAC estimators (Homography::estimate,
// Homography::estimate_similarity, RansacOptions::validate).
//
// Reference: src/pipeline.rs:177-247 (options, seeds), :2038-2049, :2635-2661.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "psift_internal.cuh"
#include "ransac_common.cuh"

namespace psift {

cudaError_t launch_ransac(const RansacJob* jobs, int n_jobs, cudaStream_t st);

namespace {
constexpr uint64_t kSimSeed = 0xD1B54A32D192ED03ull;   // DEFAULT_SIMILARITY_RANSAC_SEED, src/pipeline.rs:172
constexpr uint64_t kHomSeed = 0x517CC1B727220A95ull;   // DEFAULT_HOMOGRAPHY_RANSAC_SEED, src/pipeline.rs:174

void seeds_for(const psift_ransac_options& o, bool homography, uint64_t& s1, uint64_t& s2) {
  if (!o.has_seed) {
    s1 = kSimSeed;
    s2 = kHomSeed;
  } else {
    s1 = o.seed;
    s2 = homography ? (o.seed ^ 0x9E3779B97F4A7C15ull) : 0;
  }
}

psift_status run_batch(psift_ctx* ctx, const psift_ransac_job* jobs, int n, const psift_ransac_options& opt,
                       bool homography) {
  size_t bytes = sizeof(RansacJob) * n + 4096;
  for (int i = 0; i < n; ++i) {
    const size_t m = jobs[i].n;
    bytes += 8 * m + 8 * m + 4 * m + 16 * m + 32 * m + 6 * 256;
  }
  psift_status st = arena_reserve(ctx, bytes);
  if (st != PSIFT_OK) return st;
  RansacJob* d_jobs = (RansacJob*)arena_alloc(ctx, sizeof(RansacJob) * n);
  std::vector<RansacJob> hj(n);
  uint64_t s1, s2;
  seeds_for(opt, homography, s1, s2);
  for (int i = 0; i < n; ++i) {
    const psift_ransac_job& J = jobs[i];
    RansacJob& R = hj[i];
    std::memset(&R, 0, sizeof R);
    const size_t m = J.n;
    R.m = J.matches;
    R.n = (int)J.n;
    R.thr = opt.reproj_threshold;
    R.sim_seed = s1;
    R.hom_seed = s2;
    R.homography = homography ? 1 : 0;
    R.weights = J.sampling_weights;
    R.cdf = (double*)arena_alloc(ctx, 8 * m + 8);
    R.err = (double*)arena_alloc(ctx, 8 * m + 8);
    R.list = (int*)arena_alloc(ctx, 4 * m + 4);
    R.xy = (float4*)arena_alloc(ctx, 16 * m + 16);
    R.pts = (double*)arena_alloc(ctx, 32 * m + 32);
    R.mask = J.inlier_mask;
    R.model = J.model;
    R.has_model = J.has_model;
    R.count = (int*)J.inlier_count;
    R.iters = (int*)J.iterations;
    if (!R.pts) return set_error(ctx, PSIFT_ERR_INTERNAL, "ransac workspace carve overflow");
  }
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_jobs, hj.data(), sizeof(RansacJob) * n, cudaMemcpyHostToDevice, ctx->stream));
  StageScope sc(ctx, STAGE_RANSAC);
  cudaError_t e = launch_ransac(d_jobs, n, ctx->stream);
  ctx->launches++;
  if (e != cudaSuccess) return cuda_error(ctx, e, "ransac");
  return PSIFT_OK;
}

psift_status estimate_host(psift_ctx* ctx, const psift_match* m, uint32_t n, const psift_ransac_options* opt,
                           bool homography, uint8_t* mask, float* model, int32_t* has_model, uint32_t* count) {
  if (!ctx || !opt || !count || !has_model || !model) return PSIFT_ERR_INVALID_ARGUMENT;
  if (n && (!m || !mask)) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null matches/mask");
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaSetDevice");
  const size_t mb = sizeof(psift_match) * (size_t)n;
  psift_status st = io_reserve(ctx, mb + n + 256 + 1024);
  if (st != PSIFT_OK) return st;
  char* base = ctx->io.base;
  psift_match* d_m = (psift_match*)base;
  uint8_t* d_mask = (uint8_t*)(base + align_up(mb, 256));
  int* d_out = (int*)(base + align_up(mb, 256) + align_up(n + 1, 256));  // [0] count [1] has [2..3] iters [8..16] model
  if (n) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_m, m, mb, cudaMemcpyHostToDevice, ctx->stream));
  psift_ransac_job job{d_m, n, d_mask, (float*)(d_out + 8), d_out + 1, (uint32_t*)d_out, nullptr, (uint32_t*)(d_out + 2)};
  st = run_batch(ctx, &job, 1, *opt, homography);
  if (st != PSIFT_OK) return st;
  st = pinned_reserve(ctx, n + 256);
  if (st != PSIFT_OK) return st;
  char* pin = ctx->pinned.base;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(pin, d_out, 17 * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (n) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(pin + 128, d_mask, n, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  const int* o = (const int*)pin;
  *count = (uint32_t)o[0];
  *has_model = o[1];
  std::memcpy(model, o + 8, sizeof(float) * (homography ? 9 : 6));
  if (n) std::memcpy(mask, pin + 128, n);
  return PSIFT_OK;
}

}  // namespace
}  // namespace psift

using namespace psift;

extern "C" {

void psift_ransac_options_default(psift_ransac_options* o) {
  if (!o) return;
  o->reproj_threshold = 3.0f;  // DEFAULT_RANSAC_REPROJ_THRESHOLD, src/pipeline.rs:1050
  o->has_seed = 0;
  o->seed = 0;
}

// RansacOptions::validate (src/pipeline.rs:209-217).
psift_status psift_ransac_options_validate(const psift_ransac_options* o, char* msg, size_t cap) {
  char buf[160] = {0};
  psift_status st = PSIFT_OK;
  if (!o) {
    snprintf(buf, sizeof buf, "null options");
    st = PSIFT_ERR_INVALID_ARGUMENT;
  } else if (!(o->reproj_threshold == o->reproj_threshold) || o->reproj_threshold > 3.4e38f ||
             o->reproj_threshold < -3.4e38f || o->reproj_threshold < 0.5f || o->reproj_threshold > 100.0f) {
    snprintf(buf, sizeof buf, "Invalid `reproj_threshold`=%g: must be between 0.5 and 100.0",
             (double)o->reproj_threshold);
    st = PSIFT_ERR_INVALID_CONFIG;
  }
  if (msg && cap) {
    strncpy(msg, buf, cap - 1);
    msg[cap - 1] = 0;
  }
  return st;
}

psift_status psift_homography_estimate(psift_ctx* ctx, const psift_match* matches, uint32_t n,
                                       const psift_ransac_options* opt, uint8_t* inlier_mask, float* h9,
                                       int32_t* has_h, uint32_t* inlier_count) {
  return estimate_host(ctx, matches, n, opt, true, inlier_mask, h9, has_h, inlier_count);
}

psift_status psift_similarity_estimate(psift_ctx* ctx, const psift_match* matches, uint32_t n,
                                       const psift_ransac_options* opt, uint8_t* inlier_mask, float* model6,
                                       int32_t* has_model, uint32_t* inlier_count) {
  return estimate_host(ctx, matches, n, opt, false, inlier_mask, model6, has_model, inlier_count);
}

psift_status psift_ransac_batch_dev(psift_ctx* ctx, const psift_ransac_job* jobs, uint32_t n,
                                    const psift_ransac_options* opt, int32_t homography) {
  if (!ctx || !opt || (n && !jobs)) return PSIFT_ERR_INVALID_ARGUMENT;
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaSetDevice");
  for (uint32_t i = 0; i < n; ++i)
    if (!jobs[i].model || !jobs[i].has_model || !jobs[i].inlier_count || (jobs[i].n && (!jobs[i].matches || !jobs[i].inlier_mask)))
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null pointer in ransac job");
  if (n == 0) return PSIFT_OK;
  return run_batch(ctx, jobs, (int)n, *opt, homography != 0);
}

}  // extern "C"

namespace psift {
namespace {
// Reference median_f32 (src/pipeline.rs:2195-2206).
float median_f32(std::vector<float> v) {
  if (v.empty()) return 0.0f;
  std::stable_sort(v.begin(), v.end(), [](float a, float b) { return a < b; });
  const size_t mid = v.size() / 2;
  return v.size() % 2 == 1 ? v[mid] : 0.5f * (v[mid - 1] + v[mid]);
}
}  // namespace

// The statistics of summarize_tracking (src/pipeline.rs:2227-2271) over the
// matches that `mask` marks (all of them when it marks none), in the reference's
// f32 order.  n > 0.
void tracking_stats(const psift_match* m, uint32_t n, const uint8_t* mask, const float* q_scale,
                    const float* q_ori, const float* t_scale, const float* t_ori, psift_tracking_summary* out) {
  std::vector<const psift_match*> act;
  for (uint32_t i = 0; i < n; ++i)
    if (mask[i]) act.push_back(&m[i]);
  if (act.empty())
    for (uint32_t i = 0; i < n; ++i) act.push_back(&m[i]);
  const float inv_n = 1.0f / (float)act.size();
  float sdx = 0, sdy = 0, ssr = 0, ssin = 0, scos = 0;
  std::vector<float> dxs, dys;
  dxs.reserve(act.size());
  dys.reserve(act.size());
  for (const psift_match* a : act) {
    sdx += a->displacement_x;
    sdy += a->displacement_y;
    dxs.push_back(a->displacement_x);
    dys.push_back(a->displacement_y);
    const float qs = q_scale[a->query_index], ts = t_scale[a->target_index];
    if (qs > 1e-6f) ssr += ts / qs;
    const float dth = t_ori[a->target_index] - q_ori[a->query_index];
    ssin += std::sin(dth);
    scos += std::cos(dth);
  }
  const float mrot = std::atan2(ssin, scos);
  out->raw_match_count = n;
  out->match_count = (uint32_t)act.size();
  out->inlier_ratio = (float)act.size() / (float)n;
  out->mean_dx = sdx * inv_n;
  out->mean_dy = sdy * inv_n;
  out->median_dx = median_f32(dxs);
  out->median_dy = median_f32(dys);
  out->mean_scale_ratio = ssr * inv_n;
  out->mean_rotation_deg = mrot * 57.2957795130823208767981548141051703f;
}
}  // namespace psift

extern "C" psift_status psift_summarize_tracking(psift_ctx* ctx, const psift_match* m, uint32_t n,
                                                 const float* q_scale, const float* q_ori, uint32_t nq,
                                                 const float* t_scale, const float* t_ori, uint32_t nt,
                                                 psift_tracking_summary* out) {
  // summarize_tracking (src/pipeline.rs:2210-2272): the similarity RANSAC runs on the
  // device; the O(n) summary repeats the reference's f32 sums on the host.
  if (!ctx || !out) return PSIFT_ERR_INVALID_ARGUMENT;
  if (n == 0) {
    *out = psift_tracking_summary{0, 0, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f};
    return PSIFT_OK;
  }
  if (!m || !q_scale || !q_ori || !t_scale || !t_ori) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  for (uint32_t i = 0; i < n; ++i)
    if (m[i].query_index >= nq || m[i].target_index >= nt)
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "match index outside the feature arrays");
  std::vector<uint8_t> mask(n);
  float model[9];
  int32_t has = 0;
  uint32_t cnt = 0;
  psift_ransac_options opt;
  psift_ransac_options_default(&opt);
  psift_status st = psift_similarity_estimate(ctx, m, n, &opt, mask.data(), model, &has, &cnt);
  if (st != PSIFT_OK) return st;
  psift::tracking_stats(m, n, mask.data(), q_scale, q_ori, t_scale, t_ori, out);
  return PSIFT_OK;
}
