// Orchestration of the detect-and-describe path and its C-ABI entry points.
//
// Reference call stack (src/pipeline.rs): Sift::detect_and_compute (:136-145)
// -> extract_sift_features_with_kind (:1633-1658) -> Pyramid::build_with_params
// (:519-530) -> build_scale_space_pyramid_with_options (:550-638), then
// Pyramid::extract_extrema (:535-547), the 4096 cap, and
// compute_sift_descriptors_from_pyramid_with_kind (:1482-1577).
//
// One call processes a batch of images; every kernel covers the whole batch
// (blockIdx.z / blockIdx.y = image), so uneven image sizes share one launch per
// stage.  Host code only computes the octave geometry and the f32 blur weights
// (the reference's own formula, evaluated with the same libm) and carves the
// workspace; all data-dependent work stays on the device.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "detect_plan.cuh"
#include "psift_internal.cuh"

namespace psift {

// Declared in pyramid.cu / extrema.cu / describe.cu.
cudaError_t launch_blur(int mode, const float* taps_host, int radius, const ImagePlan* plans, int n, int octave,
                        int level, int down_level, int max_h, int max_w, cudaStream_t st, int variant = 0,
                        bool fused = false, const TileMap* tiles = nullptr, const ImagePlan* h_plans = nullptr,
                        uint32_t* err = nullptr);
cudaError_t launch_extrema_mark(const ImagePlan* plans, int n, int octave, int max_h, const ExtremaParams& prm,
                                cudaStream_t st);
cudaError_t launch_row_scan(const ImagePlan* plans, int n, uint32_t kp_cap, uint32_t* err, cudaStream_t st);
cudaError_t launch_extrema_emit(const ImagePlan* plans, int n, int octave, int max_h, const ExtremaParams& prm,
                                uint32_t kp_cap, cudaStream_t st);
cudaError_t launch_select_topk(const ImagePlan* plans, int n, uint32_t kp_cap, uint32_t max_features, uint32_t* err,
                               cudaStream_t st);
cudaError_t launch_orientation(const ImagePlan* plans, int n, uint32_t sel_cap, const DescribeParams& prm,
                               cudaStream_t st);
cudaError_t launch_feature_scan(const ImagePlan* plans, int n, uint32_t max_features, cudaStream_t st);
cudaError_t launch_descriptor(const ImagePlan* plans, int n, uint32_t sel_cap, const DescribeParams& prm,
                              cudaStream_t st);

namespace {

constexpr uint32_t kDefaultKeypointCapacity = 1u << 18;

// f32::powi lowers to square-and-multiply (low bit first); same sequence here.
float powi_f(float a, int b) {
  const bool recip = b < 0;
  float r = 1.0f;
  for (;;) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? 1.0f / r : r;
}

// gaussian_kernel_1d (src/pipeline.rs:275-296), evaluated on the host in f32.
std::vector<float> gaussian_taps(float sigma) {
  const float cs = std::fmax(sigma, 1e-3f);
  long long radius = (long long)std::ceil(3.0f * cs);
  if (radius < 1) radius = 1;
  const float two_sigma_sq = 2.0f * cs * cs;
  const float norm = 1.0f / (std::sqrt(2.0f * kPiF) * cs);
  std::vector<float> k;
  for (long long x = -radius; x <= radius; ++x) {
    const float xf = (float)x;
    k.push_back(norm * std::exp(-((xf * xf) / two_sigma_sq)));
  }
  float sum = 0.0f;
  for (float v : k) sum += v;
  if (sum > 0.0f) {
    const float inv = 1.0f / sum;
    for (float& v : k) v *= inv;
  }
  return k;
}

struct HostOctave {
  int h, w;
  long long pitch;
};

// Octave geometry of build_scale_space_pyramid_with_options: stop when the base
// is smaller than 3x3; downsample_2x floors and returns 0x0 when a side hits 0.
int plan_octaves(int h, int w, int octaves, bool upsample, HostOctave* out) {
  int ch = upsample ? 2 * h : h, cw = upsample ? 2 * w : w;
  int n = 0;
  if (h == 0 || w == 0) return 0;
  for (int o = 0; o < octaves && o < kMaxOctaves; ++o) {
    if (ch < 3 || cw < 3) break;
    out[n++] = {ch, cw, (long long)align_up((size_t)cw, 32)};
    int nh = ch / 2, nw = cw / 2;
    if (nh == 0 || nw == 0) nh = nw = 0;
    ch = nh;
    cw = nw;
  }
  return n;
}

struct SigmaSchedule {
  std::vector<float> init_taps;
  int init_radius;
  std::vector<std::vector<float>> level_taps;  // index s = 1..S+2
  std::vector<int> level_radius;
  float k;
};

SigmaSchedule make_schedule(int scales, bool upsample) {
  SigmaSchedule sc;
  sc.k = std::pow(2.0f, 1.0f / (float)scales);
  const float sigma_in = upsample ? 2.0f * kAssumedInputSigma : kAssumedInputSigma;
  const float init_sigma = std::sqrt(std::fmax(kBaseSigma * kBaseSigma - sigma_in * sigma_in, 1e-4f));
  sc.init_taps = gaussian_taps(init_sigma);
  sc.init_radius = (int)sc.init_taps.size() / 2;
  sc.level_taps.resize(scales + 3);
  sc.level_radius.assign(scales + 3, 0);
  float prev = kBaseSigma;
  for (int s = 1; s <= scales + 2; ++s) {
    const float target = kBaseSigma * powi_f(sc.k, s);
    const float delta = std::sqrt(std::fmax(target * target - prev * prev, 1e-4f));
    sc.level_taps[s] = gaussian_taps(delta);
    sc.level_radius[s] = (int)sc.level_taps[s].size() / 2;
    prev = target;
  }
  return sc;
}

struct DetectJob {
  int n = 0;
  std::vector<ImagePlan> plans;      // host copy
  std::vector<HostOctave> oct;       // n * kMaxOctaves
  std::vector<int> n_oct;
  ImagePlan* d_plans = nullptr;
  uint32_t kp_cap = 0, sel_cap = 0;
  int8_t blur_variant[16] = {0};     // level-blur variant per radius (the context's tuning)
  bool blur_fused = false;           // single-rounding blur mode (the context's setting)
};

struct ImageDesc {
  const void* src;      // device pointer
  long long stride;
  int h, w;
  int kind;             // SRC_F32 / SRC_U8
  // device outputs (nullptr: allocate in the workspace)
  float *fx, *fy, *fscale, *fresp, *fori, *fdesc;
  uint32_t feat_cap;
  uint32_t* out_count;
};

size_t plane_bytes(const HostOctave& o) { return sizeof(float) * (size_t)o.pitch * o.h; }

// Sizes and carves the workspace for n images; fills job.plans (host) with device pointers.
psift_status build_job(psift_ctx* ctx, const std::vector<ImageDesc>& imgs, const psift_sift_config& cfg,
                       DetectJob& job, size_t extra_bytes, void** extra_ptr) {
  const int n = (int)imgs.size();
  const int S = (int)cfg.scales;
  job.n = n;
  job.kp_cap = kDefaultKeypointCapacity;
  job.sel_cap = cfg.max_features ? cfg.max_features : job.kp_cap;
  std::memcpy(job.blur_variant, ctx->tune.blur, sizeof job.blur_variant);
  job.blur_fused = ctx->blur_fused;
  job.oct.assign((size_t)n * kMaxOctaves, HostOctave{0, 0, 0});
  job.n_oct.assign(n, 0);
  size_t total = align_up(sizeof(ImagePlan) * n, 256) + align_up(extra_bytes, 256);
  for (int i = 0; i < n; ++i) {
    job.n_oct[i] = plan_octaves(imgs[i].h, imgs[i].w, (int)cfg.octaves, cfg.upsample_first_octave != 0,
                                &job.oct[(size_t)i * kMaxOctaves]);
    if (job.n_oct[i] > 0 && (job.oct[(size_t)i * kMaxOctaves].h > 65535 || job.oct[(size_t)i * kMaxOctaves].w > 65535))
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "octave-0 side above 65535 pixels is not supported");
    int rows = 0;
    for (int o = 0; o < job.n_oct[i]; ++o) {
      const HostOctave& O = job.oct[(size_t)i * kMaxOctaves + o];
      total += align_up(plane_bytes(O) * (2 * S + 5), 256);
      total += align_up(sizeof(uint32_t) * (size_t)S * O.h * ((O.w + 31) / 32), 256);
      rows += S * O.h;
    }
    total += 2 * align_up(sizeof(uint32_t) * (size_t)rows + 4, 256);
    total += align_up(sizeof(psift_keypoint) * job.kp_cap, 256) + align_up(sizeof(psift_keypoint) * job.sel_cap, 256);
    total += align_up(sizeof(float) * 4 * job.sel_cap, 256) + 2 * align_up(sizeof(uint32_t) * job.sel_cap, 256);
    total += 256;  // counters
    if (!imgs[i].fx) total += align_up(sizeof(float) * imgs[i].feat_cap * (5 + kDescLen), 256) + 5 * 256;
  }
  psift_status st = arena_reserve(ctx, total);
  if (st != PSIFT_OK) return st;
  job.d_plans = (ImagePlan*)arena_alloc(ctx, sizeof(ImagePlan) * n);
  if (extra_ptr) *extra_ptr = extra_bytes ? arena_alloc(ctx, extra_bytes) : nullptr;
  job.plans.assign(n, ImagePlan{});
  for (int i = 0; i < n; ++i) {
    ImagePlan& P = job.plans[i];
    std::memset(&P, 0, sizeof(P));
    P.src = imgs[i].src;
    P.src_stride = imgs[i].stride;
    P.src_h = imgs[i].h;
    P.src_w = imgs[i].w;
    P.src_kind = imgs[i].kind;
    P.upsample = cfg.upsample_first_octave != 0;
    P.n_oct = job.n_oct[i];
    int row_base = 0;
    const float base_mult = cfg.upsample_first_octave ? 0.5f : 1.0f;
    for (int o = 0; o < P.n_oct; ++o) {
      const HostOctave& H = job.oct[(size_t)i * kMaxOctaves + o];
      OctaveDev& O = P.oct[o];
      O.h = H.h;
      O.w = H.w;
      O.pitch = H.pitch;
      O.plane_stride = H.pitch * H.h;
      float* planes = (float*)arena_alloc(ctx, plane_bytes(H) * (2 * S + 5));
      O.g = planes;
      O.d = planes + O.plane_stride * (S + 3);
      O.words = (H.w + 31) / 32;
      O.masks = (uint32_t*)arena_alloc(ctx, sizeof(uint32_t) * (size_t)S * H.h * O.words);
      O.row_base = row_base;
      O.scale_factor = base_mult * (float)(1ull << o);
      row_base += S * H.h;
    }
    P.total_rows = row_base;
    P.row_counts = (uint32_t*)arena_alloc(ctx, sizeof(uint32_t) * (size_t)row_base + 4);
    P.row_offsets = (uint32_t*)arena_alloc(ctx, sizeof(uint32_t) * (size_t)row_base + 4);
    P.kps = (psift_keypoint*)arena_alloc(ctx, sizeof(psift_keypoint) * job.kp_cap);
    P.sel = (psift_keypoint*)arena_alloc(ctx, sizeof(psift_keypoint) * job.sel_cap);
    P.oris = (float*)arena_alloc(ctx, sizeof(float) * 4 * job.sel_cap);
    P.ori_count = (uint32_t*)arena_alloc(ctx, sizeof(uint32_t) * job.sel_cap);
    P.feat_offsets = (uint32_t*)arena_alloc(ctx, sizeof(uint32_t) * job.sel_cap);
    uint32_t* counters = (uint32_t*)arena_alloc(ctx, 256);
    P.kp_count = counters + 0;
    P.sel_count = counters + 1;
    P.feat_count = counters + 2;
    P.feat_total = counters + 3;
    P.out_count = imgs[i].out_count;
    P.feat_cap = imgs[i].feat_cap;
    if (imgs[i].fx) {
      P.fx = imgs[i].fx;
      P.fy = imgs[i].fy;
      P.fscale = imgs[i].fscale;
      P.fresp = imgs[i].fresp;
      P.fori = imgs[i].fori;
      P.fdesc = imgs[i].fdesc;
    } else {
      const size_t fc = imgs[i].feat_cap;
      P.fx = (float*)arena_alloc(ctx, sizeof(float) * fc);
      P.fy = (float*)arena_alloc(ctx, sizeof(float) * fc);
      P.fscale = (float*)arena_alloc(ctx, sizeof(float) * fc);
      P.fresp = (float*)arena_alloc(ctx, sizeof(float) * fc);
      P.fori = (float*)arena_alloc(ctx, sizeof(float) * fc);
      P.fdesc = (float*)arena_alloc(ctx, sizeof(float) * fc * kDescLen);
    }
    if (!P.row_offsets || !P.kps || !P.fdesc || !counters) return set_error(ctx, PSIFT_ERR_INTERNAL, "workspace carve overflow");
  }
  return PSIFT_OK;
}

// Tile work list of octave o over the job's images, so that a blur launch over
// images of different sizes runs one CTA per existing tile; n = 0 (the (tiles x,
// tiles y, images) grid over the largest image) when every image has that size
// at octave o or the job has more than kTileMapMax images.
TileMap tile_map(const DetectJob& job, int o, int mh, int mw) {
  TileMap tm;
  tm.n = 0;
  tm.prefix[0] = 0;
  if (job.n > kTileMapMax) return tm;
  bool uneven = false;
  for (int i = 0; i < job.n; ++i) {
    const HostOctave& H = job.oct[(size_t)i * kMaxOctaves + o];
    uneven |= o >= job.n_oct[i] || H.h != mh || H.w != mw;
  }
  if (!uneven) return tm;
  for (int i = 0; i < job.n; ++i) {
    const HostOctave& H = job.oct[(size_t)i * kMaxOctaves + o];
    const bool has = o < job.n_oct[i];
    const int tx = has ? (H.w + kTileW - 1) / kTileW : 0, ty = has ? (H.h + kTileH - 1) / kTileH : 0;
    tm.tiles_x[i] = std::max(tx, 1);
    tm.prefix[i + 1] = tm.prefix[i] + tx * ty;
  }
  tm.n = tm.prefix[job.n] > 0 ? job.n : 0;
  return tm;
}

// One blur level (octave o, level s >= 1) of every image of the job.
cudaError_t launch_level(const DetectJob& job, const SigmaSchedule& sc, int o, int s, int S, int mh, int mw,
                         cudaStream_t st, uint32_t* err) {
  const int r = sc.level_radius[s];
  const TileMap tm = tile_map(job, o, mh, mw);
  int variant = r >= 0 && r < 16 ? job.blur_variant[r] : 0;
  if (variant == 3 && job.n > kTileMapMax) variant = 0;  // the TMA kernel's tile list holds kTileMapMax images
  return launch_blur(0, sc.level_taps[s].data(), r, job.d_plans, job.n, o, s, S, mh, mw, st, variant,
                     job.blur_fused, &tm, job.plans.data(), err);
}

// Queue every stage of the path for the batch (no host synchronisation).
// stop_after_keypoints: end after extrema_emit (Sift::detect_keypoints).
psift_status launch_detect(psift_ctx* ctx, DetectJob& job, const psift_sift_config& cfg, bool stop_after_keypoints,
                           cudaStream_t stream = nullptr, bool plans_uploaded = false) {
  cudaStream_t st = stream ? stream : ctx->stream;
  const int n = job.n;
  const int S = (int)cfg.scales;
  if (!plans_uploaded)
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(job.d_plans, job.plans.data(), sizeof(ImagePlan) * n, cudaMemcpyHostToDevice, st));
  const SigmaSchedule sc = make_schedule(S, cfg.upsample_first_octave != 0);
  int max_oct = 0;
  for (int i = 0; i < n; ++i) max_oct = std::max(max_oct, job.n_oct[i]);
  if (max_oct == 0) {
    // Every image is empty/too small: zero all counters.
    for (int i = 0; i < n; ++i) {
      PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(job.plans[i].kp_count, 0, 16, st));
      if (job.plans[i].out_count) PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(job.plans[i].out_count, 0, 4, st));
    }
    return PSIFT_OK;
  }
  auto max_dims = [&](int o, int& mh, int& mw) {
    mh = mw = 0;
    for (int i = 0; i < n; ++i)
      if (o < job.n_oct[i]) {
        mh = std::max(mh, job.oct[(size_t)i * kMaxOctaves + o].h);
        mw = std::max(mw, job.oct[(size_t)i * kMaxOctaves + o].w);
      }
  };
  // Octave-0 base: luma -> f32 (+ 2x bilinear upsample) + initial blur.
  {
    StageScope sc_pyr(ctx, STAGE_PYRAMID, st);
    int mh, mw;
    max_dims(0, mh, mw);
    const bool up = cfg.upsample_first_octave != 0;
    const int kind = job.plans[0].src_kind;
    const int mode = kind == SRC_U8 ? (up ? 4 : 2) : (up ? 3 : 1);
    const TileMap tm0 = tile_map(job, 0, mh, mw);
    cudaError_t e = launch_blur(mode, sc.init_taps.data(), sc.init_radius, job.d_plans, n, 0, 0, -1, mh, mw, st, 0,
                                job.blur_fused, &tm0);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "blur(init)");
  }
  ExtremaParams xp;
  std::memset(&xp, 0, sizeof xp);
  xp.threshold = cfg.contrast_threshold;
  xp.scales = S;
  xp.k = sc.k;
  const float base_mult = cfg.upsample_first_octave ? 0.5f : 1.0f;
  for (int o = 0; o < kMaxOctaves; ++o) {
    const float mult = base_mult * (float)(1ull << o);
    for (int s = 0; s <= S && s < 11; ++s) xp.eff_scale[o][s] = kBaseSigma * mult * powi_f(sc.k, s);
  }
  for (int o = 0; o < max_oct; ++o) {
    int mh, mw;
    max_dims(o, mh, mw);
    {
      StageScope sc_pyr(ctx, STAGE_PYRAMID, st);
      for (int s = 1; s <= S + 2; ++s) {
        cudaError_t e = launch_level(job, sc, o, s, S, mh, mw, st, ctx->d_error);
        ctx->launches++;
        if (e != cudaSuccess) return cuda_error(ctx, e, "blur(level)");
      }
    }
    StageScope sc_x(ctx, STAGE_EXTREMA, st);
    cudaError_t e = launch_extrema_mark(job.d_plans, n, o, mh, xp, st);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "extrema_mark");
  }
  cudaError_t e;
  {
  StageScope sc_x2(ctx, STAGE_EXTREMA, st);
  e = launch_row_scan(job.d_plans, n, job.kp_cap, ctx->d_error, st);
  ctx->launches++;
  if (e != cudaSuccess) return cuda_error(ctx, e, "row_scan");
  for (int o = 0; o < max_oct; ++o) {
    int mh, mw;
    max_dims(o, mh, mw);
    e = launch_extrema_emit(job.d_plans, n, o, mh, xp, job.kp_cap, st);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "extrema_emit");
  }
  }
  if (stop_after_keypoints) return PSIFT_OK;
  {
    StageScope sc_s(ctx, STAGE_SELECT, st);
    e = launch_select_topk(job.d_plans, n, job.kp_cap, cfg.max_features, ctx->d_error, st);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "select_topk");
  }
  DescribeParams dp{S, cfg.max_features, cfg.descriptor_kind};
  {
    StageScope sc_o(ctx, STAGE_ORIENTATION, st);
    e = launch_orientation(job.d_plans, n, job.sel_cap, dp, st);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "orientation");
  }
  {
    StageScope sc_d(ctx, STAGE_DESCRIPTOR, st);
    e = launch_feature_scan(job.d_plans, n, cfg.max_features, st);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "feature_scan");
    e = launch_descriptor(job.d_plans, n, job.sel_cap, dp, st);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "descriptor");
  }
  return PSIFT_OK;
}

// Octave base + blur/DoG levels only (used by the descriptor-only path).
psift_status launch_pyramid_only(psift_ctx* ctx, DetectJob& job, const psift_sift_config& cfg) {
  cudaStream_t st = ctx->stream;
  const int n = job.n;
  const int S = (int)cfg.scales;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(job.d_plans, job.plans.data(), sizeof(ImagePlan) * n, cudaMemcpyHostToDevice, st));
  const SigmaSchedule sc = make_schedule(S, cfg.upsample_first_octave != 0);
  int max_oct = 0;
  for (int i = 0; i < n; ++i) max_oct = std::max(max_oct, job.n_oct[i]);
  StageScope sc_pyr(ctx, STAGE_PYRAMID);
  for (int o = 0; o < max_oct; ++o) {
    int mh = 0, mw = 0;
    for (int i = 0; i < n; ++i)
      if (o < job.n_oct[i]) {
        mh = std::max(mh, job.oct[(size_t)i * kMaxOctaves + o].h);
        mw = std::max(mw, job.oct[(size_t)i * kMaxOctaves + o].w);
      }
    if (o == 0) {
      const bool up = cfg.upsample_first_octave != 0;
      const int mode = job.plans[0].src_kind == SRC_U8 ? (up ? 4 : 2) : (up ? 3 : 1);
      const TileMap tm0 = tile_map(job, 0, mh, mw);
      cudaError_t e = launch_blur(mode, sc.init_taps.data(), sc.init_radius, job.d_plans, n, 0, 0, -1, mh, mw, st, 0,
                                  job.blur_fused, &tm0);
      ctx->launches++;
      if (e != cudaSuccess) return cuda_error(ctx, e, "blur(init)");
    }
    for (int s = 1; s <= S + 2; ++s) {
      cudaError_t e = launch_level(job, sc, o, s, S, mh, mw, st, ctx->d_error);
      ctx->launches++;
      if (e != cudaSuccess) return cuda_error(ctx, e, "blur(level)");
    }
  }
  return PSIFT_OK;
}

uint32_t float_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

// Queues the job as two chunk views, chunk c on stream c (images [0, n/2) and
// [n/2, n)), forked from and joined back to the context's stream by events; the
// two chunks' kernels fill each other's idle SMs (small octaves, launch tails,
// serial stages).  The plan table must already be on the device.
psift_status launch_detect_split(psift_ctx* ctx, DetectJob& job, const psift_sift_config& cfg);

// True when p lies in page-locked host memory (cudaMallocHost / cudaHostRegister).
bool is_host_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

psift_status launch_detect_split(psift_ctx* ctx, DetectJob& job, const psift_sift_config& cfg) {
  const int n = job.n;
  if (n < 2) return launch_detect(ctx, job, cfg, false, nullptr, true);
  PSIFT_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream2, ctx->ev_fork, 0));
  const int split = (n + 1) / 2;
  cudaStream_t streams[2] = {ctx->stream, ctx->stream2};
  for (int c = 0; c < 2; ++c) {
    const int b = c == 0 ? 0 : split, e = c == 0 ? split : n;
    DetectJob v;
    v.n = e - b;
    v.plans.assign(job.plans.begin() + b, job.plans.begin() + e);
    v.oct.assign(job.oct.begin() + (size_t)b * kMaxOctaves, job.oct.begin() + (size_t)e * kMaxOctaves);
    v.n_oct.assign(job.n_oct.begin() + b, job.n_oct.begin() + e);
    v.d_plans = job.d_plans + b;
    v.kp_cap = job.kp_cap;
    v.sel_cap = job.sel_cap;
    std::memcpy(v.blur_variant, job.blur_variant, sizeof v.blur_variant);  // the context's tuning
    v.blur_fused = job.blur_fused;
    psift_status st = launch_detect(ctx, v, cfg, false, streams[c], true);
    if (st != PSIFT_OK) return st;
  }
  PSIFT_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_join, ctx->stream2));
  PSIFT_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
  return PSIFT_OK;
}

psift_status check_common(psift_ctx* ctx, const psift_sift_config* cfg) {
  if (!ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  char msg[256];
  psift_status st = psift_sift_config_validate(cfg, msg, sizeof msg);
  if (st != PSIFT_OK) return set_error(ctx, st, msg);
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(ctx, e, "cudaSetDevice");
  return PSIFT_OK;
}

psift_status read_error_word(psift_ctx* ctx, uint32_t* host_word) {
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(host_word, ctx->d_error, 4, cudaMemcpyDeviceToHost, ctx->stream));
  return PSIFT_OK;
}

psift_status error_from_word(psift_ctx* ctx, uint32_t w) {
  if (w & kErrKeypointCapacity)
    return set_error(ctx, PSIFT_ERR_CAPACITY, "more DoG extrema than the keypoint workspace holds (262144)");
  if (w & kErrSortCapacity) return set_error(ctx, PSIFT_ERR_INTERNAL, "top-K selection inconsistency");
  if (w & kErrTimeout) return set_error(ctx, PSIFT_ERR_TIMEOUT, "device wait timed out");
  return PSIFT_OK;
}

// Host-pointer detect_and_compute for one image (f32 or u8 source).
// Runs the detection work of a job whose plan table is already uploaded: the
// first call with a launch geometry runs eagerly, the second captures a CUDA graph
// (keyed by the geometry, the configuration and the workspace addresses the
// kernels take as arguments), later ones replay it.
psift_status run_detect_cached(psift_ctx* ctx, DetectJob& job, const psift_sift_config& cfg, const char* tag) {
  if (!ctx->graphs_enabled) return launch_detect_split(ctx, job, cfg);
  const int n = job.n;
  std::string key;
  {
    char buf[192];
    snprintf(buf, sizeof buf, "%s n%d o%u s%u t%08x u%d k%d m%u kc%u sc%u p%p e%p g%u|", tag, n, cfg.octaves,
             cfg.scales, float_bits(cfg.contrast_threshold), cfg.upsample_first_octave, cfg.descriptor_kind,
             cfg.max_features, job.kp_cap, job.sel_cap, (void*)job.d_plans, (void*)ctx->d_error, ctx->tune.gen);
    key = buf;
    for (int i = 0; i < n; ++i) {
      snprintf(buf, sizeof buf, "%dx%d:%d:%d,", job.plans[i].oct[0].h, job.plans[i].oct[0].w, job.n_oct[i],
               job.plans[i].src_kind);
      key += buf;
    }
  }
  auto it = ctx->graphs.find(key);
  if (it == ctx->graphs.end()) {
    if (ctx->graph_seen[key]++ == 0) return launch_detect_split(ctx, job, cfg);
    if (ctx->graphs.size() >= 32) {
      for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second.exec);
      ctx->graphs.clear();
    }
    const uint64_t l0 = ctx->launches;
    PSIFT_CUDA_TRY(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    psift_status st = launch_detect_split(ctx, job, cfg);
    cudaGraph_t graph = nullptr;
    cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
    if (st != PSIFT_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaStreamEndCapture");
    psift_ctx::GraphEntry ent;
    ce = cudaGraphInstantiate(&ent.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaGraphInstantiate");
    ent.launches = ctx->launches - l0;
    ctx->launches = l0;
    it = ctx->graphs.emplace(key, ent).first;
  }
  PSIFT_CUDA_TRY(ctx, cudaGraphLaunch(it->second.exec, ctx->stream));
  ctx->launches += it->second.launches;
  ctx->graph_replays++;
  return PSIFT_OK;
}

psift_status detect_host(psift_ctx* ctx, const void* image, int kind, uint32_t h, uint32_t w, size_t stride,
                         const psift_sift_config* cfg, psift_features* out) {
  psift_status st = check_common(ctx, cfg);
  if (st != PSIFT_OK) return st;
  if (!out || (h && w && !image) || stride < w) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "bad image/output argument");
  const size_t esz = kind == SRC_U8 ? 1 : 4;
  const size_t img_bytes = esz * (size_t)h * w;
  const uint32_t feat_cap = cfg->max_features ? cfg->max_features : std::min<uint32_t>(out->capacity ? out->capacity : 1, 4u * kDefaultKeypointCapacity);
  ImageDesc d{};
  d.stride = w;
  d.h = (int)h;
  d.w = (int)w;
  d.kind = kind;
  d.feat_cap = feat_cap;
  std::vector<ImageDesc> imgs{d};
  DetectJob job;
  void* d_img = nullptr;
  st = build_job(ctx, imgs, *cfg, job, img_bytes, &d_img);
  if (st != PSIFT_OK) return st;
  job.plans[0].src = d_img;
  // stage the image (tight rows) through pinned memory
  const size_t meta_bytes = 64;
  st = pinned_reserve(ctx, std::max(img_bytes, (size_t)feat_cap * sizeof(float) * (5 + kDescLen)) + meta_bytes);
  if (st != PSIFT_OK) return st;
  char* pin = ctx->pinned.base;
  // rows staged in bands: the upload of one band overlaps the host copy of the next
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_error, 0, 4, ctx->stream));
  if (img_bytes) {
    const uint32_t band = std::max<uint32_t>(1, (uint32_t)((256u << 10) / std::max<size_t>((size_t)w * esz, 1)));
    for (uint32_t y0 = 0; y0 < h; y0 += band) {
      const uint32_t y1 = std::min(h, y0 + band);
      for (uint32_t y = y0; y < y1; ++y)
        std::memcpy(pin + (size_t)y * w * esz, (const char*)image + (size_t)y * stride * esz, (size_t)w * esz);
      PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync((char*)d_img + (size_t)y0 * w * esz, pin + (size_t)y0 * w * esz,
                                          (size_t)(y1 - y0) * w * esz, cudaMemcpyHostToDevice, ctx->stream));
    }
  }
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(job.d_plans, job.plans.data(), sizeof(ImagePlan) * job.n,
                                      cudaMemcpyHostToDevice, ctx->stream));
  st = ctx->timer.enabled ? launch_detect(ctx, job, *cfg, false, nullptr, true)
                          : run_detect_cached(ctx, job, *cfg, "host");
  if (st != PSIFT_OK) return st;
  uint32_t* hmeta = (uint32_t*)(pin + ctx->pinned.capacity - meta_bytes);
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hmeta, job.plans[0].kp_count, 16, cudaMemcpyDeviceToHost, ctx->stream));
  st = read_error_word(ctx, hmeta + 4);
  if (st != PSIFT_OK) return st;
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  st = error_from_word(ctx, hmeta[4]);
  if (st != PSIFT_OK) return st;
  const uint32_t count = hmeta[2];
  const uint32_t total = cfg->max_features ? count : hmeta[3];
  if (total > out->capacity) {
    out->count = total;
    return set_error(ctx, PSIFT_ERR_CAPACITY, "feature output capacity too small");
  }
  if (count && (!out->x || !out->y || !out->scale || !out->response || !out->orientation || !out->descriptors))
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null feature output array");
  const ImagePlan& P = job.plans[0];
  float* hp = (float*)pin;
  const size_t c = count;
  if (c) {
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hp + 0 * c, P.fx, 4 * c, cudaMemcpyDeviceToHost, ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hp + 1 * c, P.fy, 4 * c, cudaMemcpyDeviceToHost, ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hp + 2 * c, P.fscale, 4 * c, cudaMemcpyDeviceToHost, ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hp + 3 * c, P.fresp, 4 * c, cudaMemcpyDeviceToHost, ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hp + 4 * c, P.fori, 4 * c, cudaMemcpyDeviceToHost, ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hp + 5 * c, P.fdesc, 4 * c * kDescLen, cudaMemcpyDeviceToHost, ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    std::memcpy(out->x, hp + 0 * c, 4 * c);
    std::memcpy(out->y, hp + 1 * c, 4 * c);
    std::memcpy(out->scale, hp + 2 * c, 4 * c);
    std::memcpy(out->response, hp + 3 * c, 4 * c);
    std::memcpy(out->orientation, hp + 4 * c, 4 * c);
    std::memcpy(out->descriptors, hp + 5 * c, 4 * c * kDescLen);
  }
  out->count = count;
  return PSIFT_OK;
}

// Autotuner, level blur: every variant of every level radius of cfg's schedule,
// timed alone on octave 0 of n synthetic u8 images of h x w (pseudo-random
// bytes, the pyramid built once first).  Another variant replaces variant 0 only
// when its time is under kBlurTuneMargin x variant 0's (3 % faster): the batch
// entries run two chunks' stages concurrently on two streams, where smaller
// gains measured alone did not carry over.  report: per distinct radius (radius, ms of each variant, chosen).
constexpr int kBlurVariantCount = 5;  // 0-2: outputs per thread; 3: TMA tiles; 4: 128-row tiles
constexpr double kBlurTuneMargin = 0.97;
psift_status autotune_blur(psift_ctx* ctx, uint32_t h, uint32_t w, uint32_t n, const psift_sift_config& cfg,
                           std::vector<double>& report) {
  if (h == 0 || w == 0 || n == 0) return PSIFT_OK;
  const size_t img = (size_t)h * w;
  ImageDesc d{};
  d.stride = w;
  d.h = (int)h;
  d.w = (int)w;
  d.kind = SRC_U8;
  d.feat_cap = 1;
  std::vector<ImageDesc> imgs(n, d);
  DetectJob job;
  void* d_img = nullptr;
  psift_status st = build_job(ctx, imgs, cfg, job, img * n, &d_img);
  if (st != PSIFT_OK) return st;
  if (job.n_oct[0] == 0) return PSIFT_OK;
  std::vector<uint8_t> bytes(img * n);
  uint64_t x = 0x9E3779B97F4A7C15ull;
  for (size_t i = 0; i < bytes.size(); ++i) {
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    bytes[i] = (uint8_t)(x >> 24);
  }
  for (uint32_t i = 0; i < n; ++i) job.plans[i].src = (uint8_t*)d_img + img * i;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_img, bytes.data(), bytes.size(), cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(job.d_plans, job.plans.data(), sizeof(ImagePlan) * n, cudaMemcpyHostToDevice,
                                      ctx->stream));
  if ((st = launch_detect(ctx, job, cfg, true, nullptr, true)) != PSIFT_OK) return st;
  const int S = (int)cfg.scales;
  const SigmaSchedule sc = make_schedule(S, cfg.upsample_first_octave != 0);
  const int mh = job.oct[0].h, mw = job.oct[0].w;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  PSIFT_CUDA_TRY(ctx, cudaEventCreate(&e0));
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    return cuda_error(ctx, ce, "cudaEventCreate");
  }
  bool seen[16] = {false};
  for (int s = 1; s <= S + 2 && st == PSIFT_OK; ++s) {
    const int r = sc.level_radius[s];
    if (r < 1 || r > 15 || seen[r]) continue;
    seen[r] = true;
    report.push_back(r);
    double best_ms = 1e30;
    int best = 0;
    for (int v = 0; v < kBlurVariantCount; ++v) {
      float ms = 1e30f;
      for (int rep = 0; rep < 4 && ce == cudaSuccess; ++rep) {  // rep 0 warms up
        if (rep > 0) ce = cudaEventRecord(e0, ctx->stream);
        if (ce == cudaSuccess) ce = launch_blur(0, sc.level_taps[s].data(), r, job.d_plans, (int)n, 0, s, -1, mh, mw,
                                                ctx->stream, v, false, nullptr, job.plans.data(), ctx->d_error);
        ctx->launches++;
        if (rep == 0 || ce != cudaSuccess) continue;
        ce = cudaEventRecord(e1, ctx->stream);
        if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
        float t = 0.0f;
        if (ce == cudaSuccess) ce = cudaEventElapsedTime(&t, e0, e1);
        ms = std::min(ms, t);
      }
      if (ce != cudaSuccess) {
        st = cuda_error(ctx, ce, "autotune blur");
        break;
      }
      report.push_back(ms);
      const double eff = v == 0 ? ms : ms / kBlurTuneMargin;  // variant 0 keeps ties within the margin
      if (eff < best_ms) {
        best_ms = eff;
        best = v;
      }
    }
    if (st != PSIFT_OK) break;
    ctx->tune.blur[r] = (int8_t)best;
    report.push_back(best);
  }
  ctx->tune.gen++;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

}  // namespace
}  // namespace psift

using namespace psift;

extern "C" {

psift_status psift_ctx_autotune(psift_ctx* ctx, uint32_t height, uint32_t width, uint32_t n_images,
                                const psift_sift_config* cfg, uint32_t n_desc, uint32_t n_pairs, double* report,
                                uint32_t report_capacity, uint32_t* report_count) {
  psift_status st = check_common(ctx, cfg);
  if (st != PSIFT_OK) return st;
  std::vector<double> rep;
  if ((st = autotune_blur(ctx, height, width, n_images, *cfg, rep)) != PSIFT_OK) return st;
  rep.push_back(-1.0);  // separator between the blur and the matcher entries
  if ((st = autotune_match(ctx, n_desc, n_pairs, rep)) != PSIFT_OK) return st;
  if (report_count) *report_count = (uint32_t)rep.size();
  if (report) std::memcpy(report, rep.data(), sizeof(double) * std::min<size_t>(rep.size(), report_capacity));
  if (report && rep.size() > report_capacity) return set_error(ctx, PSIFT_ERR_CAPACITY, "report capacity too small");
  return PSIFT_OK;
}

psift_status psift_ctx_tuning_get(const psift_ctx* ctx, int32_t what, int32_t index, int32_t* value) {
  if (!ctx || !value) return PSIFT_ERR_INVALID_ARGUMENT;
  if (what == PSIFT_TUNE_BLUR && index >= 1 && index <= 15) *value = ctx->tune.blur[index];
  else if (what == PSIFT_TUNE_MATCH_FP32 && index == 0) *value = ctx->tune.match_per_sm[0];
  else if (what == PSIFT_TUNE_MATCH_TC && index == 0) *value = ctx->tune.match_per_sm[1];
  else return PSIFT_ERR_INVALID_ARGUMENT;
  return PSIFT_OK;
}

psift_status psift_ctx_tuning_set(psift_ctx* ctx, int32_t what, int32_t index, int32_t value) {
  if (!ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  if (what == PSIFT_TUNE_BLUR && index >= 1 && index <= 15 && value >= 0 && value < kBlurVariantCount)
    ctx->tune.blur[index] = (int8_t)value;
  else if ((what == PSIFT_TUNE_MATCH_FP32 || what == PSIFT_TUNE_MATCH_TC) && index == 0 && value >= 1 && value <= 64)
    ctx->tune.match_per_sm[what == PSIFT_TUNE_MATCH_TC ? 1 : 0] = (int8_t)value;
  else
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "tuning entry or value out of range");
  ctx->tune.gen++;
  return PSIFT_OK;
}

psift_status psift_ctx_set_blur_rounding(psift_ctx* ctx, int32_t mode) {
  if (!ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  if (mode != PSIFT_BLUR_REFERENCE && mode != PSIFT_BLUR_FUSED)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "blur rounding must be PSIFT_BLUR_REFERENCE or PSIFT_BLUR_FUSED");
  ctx->blur_fused = mode == PSIFT_BLUR_FUSED;
  ctx->tune.gen++;  // captured graphs hold the other mode's kernels
  return PSIFT_OK;
}

psift_status psift_detect_and_compute(psift_ctx* ctx, const float* image, uint32_t height, uint32_t width,
                                      size_t row_stride, const psift_sift_config* cfg, psift_features* out) {
  return detect_host(ctx, image, SRC_F32, height, width, row_stride, cfg, out);
}

psift_status psift_detect_and_compute_u8(psift_ctx* ctx, const uint8_t* luma, uint32_t height, uint32_t width,
                                         size_t row_stride, const psift_sift_config* cfg, psift_features* out) {
  return detect_host(ctx, luma, SRC_U8, height, width, row_stride, cfg, out);
}

psift_status psift_detect_keypoints(psift_ctx* ctx, const float* image, uint32_t h, uint32_t w, size_t stride,
                                    const psift_sift_config* cfg, psift_keypoint* out, uint32_t capacity,
                                    uint32_t* count) {
  psift_status st = check_common(ctx, cfg);
  if (st != PSIFT_OK) return st;
  if (!count || (h && w && !image) || stride < w) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "bad argument");
  const size_t img_bytes = sizeof(float) * (size_t)h * w;
  ImageDesc d{};
  d.stride = w;
  d.h = (int)h;
  d.w = (int)w;
  d.kind = SRC_F32;
  d.feat_cap = 1;
  std::vector<ImageDesc> imgs{d};
  DetectJob job;
  void* d_img = nullptr;
  st = build_job(ctx, imgs, *cfg, job, img_bytes, &d_img);
  if (st != PSIFT_OK) return st;
  job.plans[0].src = d_img;
  st = pinned_reserve(ctx, std::max(img_bytes, sizeof(psift_keypoint) * (size_t)job.kp_cap) + 64);
  if (st != PSIFT_OK) return st;
  char* pin = ctx->pinned.base;
  for (uint32_t y = 0; y < h; ++y) std::memcpy(pin + (size_t)y * w * 4, image + (size_t)y * stride, (size_t)w * 4);
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_error, 0, 4, ctx->stream));
  if (img_bytes) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_img, pin, img_bytes, cudaMemcpyHostToDevice, ctx->stream));
  st = launch_detect(ctx, job, *cfg, true);
  if (st != PSIFT_OK) return st;
  uint32_t* hmeta = (uint32_t*)(pin + ctx->pinned.capacity - 64);
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hmeta, job.plans[0].kp_count, 4, cudaMemcpyDeviceToHost, ctx->stream));
  st = read_error_word(ctx, hmeta + 4);
  if (st != PSIFT_OK) return st;
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  st = error_from_word(ctx, hmeta[4]);
  if (st != PSIFT_OK) return st;
  const uint32_t n = job.n_oct[0] ? hmeta[0] : 0;
  *count = n;
  if (n > capacity) return set_error(ctx, PSIFT_ERR_CAPACITY, "keypoint output capacity too small");
  if (n) {
    if (!out) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null keypoint output");
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(pin, job.plans[0].kps, sizeof(psift_keypoint) * n, cudaMemcpyDeviceToHost, ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    std::memcpy(out, pin, sizeof(psift_keypoint) * n);
  }
  return PSIFT_OK;
}

psift_status psift_host_alloc(psift_ctx* ctx, size_t bytes, void** out) {
  if (!ctx || !out) return PSIFT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = cudaMallocHost(out, bytes ? bytes : 1);
  if (e != cudaSuccess) {
    *out = nullptr;
    return cuda_error(ctx, e, "cudaMallocHost");
  }
  return PSIFT_OK;
}

psift_status psift_host_free(psift_ctx* ctx, void* p) {
  if (!ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  if (p) PSIFT_CUDA_TRY(ctx, cudaFreeHost(p));
  return PSIFT_OK;
}

// Host-pointer batch.  Layout of the work:
//   one workspace for all images (build_job) and one device copy of each image;
//   the batch is split into two chunks on two streams: chunk c's uploads and
//   kernels run on stream c, so chunk 1's upload overlaps chunk 0's kernels and
//   chunk 0's feature download overlaps chunk 1's kernels;
//   counts come back first (one small copy per image), then exactly the feature
//   bytes, straight into the caller's arrays when they are page-locked, else
//   through the context's pinned staging.
psift_status psift_detect_and_compute_u8_batch(psift_ctx* ctx, const psift_image_u8* images, uint32_t n,
                                               const psift_sift_config* cfg, psift_features* outs) {
  return psift::detect_batch_host_out(ctx, images, n, cfg, outs, nullptr);
}

}  // extern "C"

namespace psift {

// The host-output batch: features of n u8 images into host arrays, one launch
// per stage, two chunks on two streams.  Inputs come from host memory
// (images[i].data, copied per chunk), or, with `fill`, are written into their
// device slots by fill, per chunk on the chunk's stream just before its stages
// (images[i].data is then unused and the slots are dense rows of width bytes).
psift_status detect_batch_host_out(psift_ctx* ctx, const psift_image_u8* images, uint32_t n,
                                   const psift_sift_config* cfg, psift_features* outs, const DeviceFill* fill) {
  psift_status st = check_common(ctx, cfg);
  if (st != PSIFT_OK) return st;
  if (!images || !outs || n == 0) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "bad batch argument");
  std::vector<ImageDesc> imgs(n);
  std::vector<size_t> dev_off(n), in_off(n), out_off(n);
  std::vector<char> in_pin(n), out_pin(n);
  size_t dev_total = 0, stage_in = 0, stage_out = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const psift_image_u8& im = images[i];
    const psift_features& o = outs[i];
    if (!fill && ((im.height && im.width && !im.data) || im.row_stride < im.width))
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "bad batch image descriptor");
    if (o.capacity && (!o.x || !o.y || !o.scale || !o.response || !o.orientation || !o.descriptors))
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null feature output array");
    ImageDesc& d = imgs[i];
    d.stride = im.width;
    d.h = (int)im.height;
    d.w = (int)im.width;
    d.kind = SRC_U8;
    d.feat_cap = cfg->max_features ? cfg->max_features
                                   : std::min<uint32_t>(o.capacity ? o.capacity : 1, 4u * kDefaultKeypointCapacity);
    const size_t px = (size_t)im.height * im.width;
    dev_off[i] = dev_total;
    dev_total += align_up(px, 256);
    in_pin[i] = (fill || !px) ? 1 : (char)is_host_pinned(im.data);
    in_off[i] = stage_in;
    if (!in_pin[i]) stage_in += align_up(px, 64);
    out_pin[i] = (char)(o.capacity && is_host_pinned(o.x) && is_host_pinned(o.y) && is_host_pinned(o.scale) &&
                        is_host_pinned(o.response) && is_host_pinned(o.orientation) && is_host_pinned(o.descriptors));
    out_off[i] = stage_out;
    if (!out_pin[i]) stage_out += align_up((size_t)std::min(d.feat_cap, o.capacity) * sizeof(float) * (5 + kDescLen), 64);
  }
  DetectJob job;
  void* extra = nullptr;
  st = build_job(ctx, imgs, *cfg, job, dev_total, &extra);
  if (st != PSIFT_OK) return st;
  for (uint32_t i = 0; i < n; ++i) job.plans[i].src = (char*)extra + dev_off[i];
  const size_t meta_bytes = align_up(16 * (size_t)n + 64, 64);
  st = pinned_reserve(ctx, meta_bytes + stage_in + stage_out);
  if (st != PSIFT_OK) return st;
  uint32_t* meta = (uint32_t*)ctx->pinned.base;
  char* pin_in = ctx->pinned.base + meta_bytes;
  char* pin_out = pin_in + stage_in;

  const uint32_t n_chunks = n >= 2 ? 2 : 1;
  const uint32_t split = (n + 1) / 2;
  cudaStream_t streams[2] = {ctx->stream, ctx->stream2};
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_error, 0, 4, ctx->stream));
  // the device plan table is uploaded once for the whole batch; chunk views index into it
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(job.d_plans, job.plans.data(), sizeof(ImagePlan) * n, cudaMemcpyHostToDevice,
                                      ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream2, ctx->ev_fork, 0));
  for (uint32_t c = 0; c < n_chunks; ++c) {
    const uint32_t b = c == 0 ? 0 : split, e = c == 0 ? (n_chunks == 1 ? n : split) : n;
    cudaStream_t sc = streams[c];
    for (uint32_t i = b; i < e && !fill; ++i) {
      const psift_image_u8& im = images[i];
      const size_t px = (size_t)im.height * im.width;
      if (!px) continue;
      char* dst = (char*)extra + dev_off[i];
      if (in_pin[i]) {
        PSIFT_CUDA_TRY(ctx, cudaMemcpy2DAsync(dst, im.width, im.data, im.row_stride, im.width, im.height,
                                              cudaMemcpyHostToDevice, sc));
      } else {
        char* stg = pin_in + in_off[i];
        for (uint32_t y = 0; y < im.height; ++y)
          std::memcpy(stg + (size_t)y * im.width, im.data + (size_t)y * im.row_stride, im.width);
        PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dst, stg, px, cudaMemcpyHostToDevice, sc));
      }
    }
    // device-filled inputs: this chunk's, on its stream (the host part of the fill
    // for chunk 1 overlaps chunk 0's kernels)
    if (fill && (st = (*fill)((char*)extra, dev_off, b, e, sc)) != PSIFT_OK) return st;
    DetectJob v;
    v.n = (int)(e - b);
    v.plans.assign(job.plans.begin() + b, job.plans.begin() + e);
    v.oct.assign(job.oct.begin() + (size_t)b * kMaxOctaves, job.oct.begin() + (size_t)e * kMaxOctaves);
    v.n_oct.assign(job.n_oct.begin() + b, job.n_oct.begin() + e);
    v.d_plans = job.d_plans + b;
    v.kp_cap = job.kp_cap;
    v.sel_cap = job.sel_cap;
    std::memcpy(v.blur_variant, job.blur_variant, sizeof v.blur_variant);  // the context's tuning
    v.blur_fused = job.blur_fused;
    st = launch_detect(ctx, v, *cfg, false, sc, /*plans_uploaded=*/true);
    if (st != PSIFT_OK) return st;
    for (uint32_t i = b; i < e; ++i)
      PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(meta + 4 * i, job.plans[i].kp_count, 16, cudaMemcpyDeviceToHost, sc));
  }
  // Per chunk: wait for its counts, then queue its feature download on its stream.
  bool capacity_short = false;
  for (uint32_t c = 0; c < n_chunks; ++c) {
    const uint32_t b = c == 0 ? 0 : split, e = c == 0 ? (n_chunks == 1 ? n : split) : n;
    cudaStream_t sc = streams[c];
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(sc));
    for (uint32_t i = b; i < e; ++i) {
      psift_features& o = outs[i];
      const uint32_t count = meta[4 * i + 2];
      const uint32_t total = cfg->max_features ? count : meta[4 * i + 3];
      if (total > o.capacity) {
        o.count = total;
        capacity_short = true;
        continue;
      }
      o.count = count;
      if (!count) continue;
      const ImagePlan& P = job.plans[i];
      const size_t cb = 4 * (size_t)count;
      float* dsts[6];
      if (out_pin[i]) {
        dsts[0] = o.x; dsts[1] = o.y; dsts[2] = o.scale; dsts[3] = o.response; dsts[4] = o.orientation;
        dsts[5] = o.descriptors;
      } else {
        float* hp = (float*)(pin_out + out_off[i]);
        for (int k = 0; k < 6; ++k) dsts[k] = hp + (size_t)k * count;
      }
      const float* srcs[6] = {P.fx, P.fy, P.fscale, P.fresp, P.fori, P.fdesc};
      for (int k = 0; k < 6; ++k)
        PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dsts[k], srcs[k], k == 5 ? cb * kDescLen : cb, cudaMemcpyDeviceToHost, sc));
    }
  }
  PSIFT_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_join, ctx->stream2));
  PSIFT_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(meta + 4 * n, ctx->d_error, 4, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  st = error_from_word(ctx, meta[4 * n]);
  if (st != PSIFT_OK) return st;
  for (uint32_t i = 0; i < n; ++i) {
    psift_features& o = outs[i];
    if (out_pin[i] || o.count > o.capacity || !o.count) continue;
    const float* hp = (const float*)(pin_out + out_off[i]);
    const size_t c = o.count;
    std::memcpy(o.x, hp + 0 * c, 4 * c);
    std::memcpy(o.y, hp + 1 * c, 4 * c);
    std::memcpy(o.scale, hp + 2 * c, 4 * c);
    std::memcpy(o.response, hp + 3 * c, 4 * c);
    std::memcpy(o.orientation, hp + 4 * c, 4 * c);
    std::memcpy(o.descriptors, hp + 5 * c, 4 * c * kDescLen);
  }
  if (capacity_short) return set_error(ctx, PSIFT_ERR_CAPACITY, "feature output capacity too small");
  return PSIFT_OK;
}

}  // namespace psift

extern "C" {

psift_status psift_detect_and_compute_batch_dev(psift_ctx* ctx, const psift_image_u8* images, uint32_t n,
                                                const psift_sift_config* cfg, psift_features* outs,
                                                uint32_t* d_counts) {
  psift_status st = check_common(ctx, cfg);
  if (st != PSIFT_OK) return st;
  if (!images || !outs || n == 0) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "bad batch argument");
  std::vector<ImageDesc> imgs(n);
  for (uint32_t i = 0; i < n; ++i) {
    const psift_image_u8& im = images[i];
    const psift_features& o = outs[i];
    if ((im.height && im.width && !im.data) || im.row_stride < im.width || !o.x || !o.y || !o.scale || !o.response ||
        !o.orientation || !o.descriptors || o.capacity == 0)
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "bad batch image/output descriptor");
    ImageDesc& d = imgs[i];
    d.src = im.data;
    d.stride = (long long)im.row_stride;
    d.h = (int)im.height;
    d.w = (int)im.width;
    d.kind = SRC_U8;
    d.fx = o.x;
    d.fy = o.y;
    d.fscale = o.scale;
    d.fresp = o.response;
    d.fori = o.orientation;
    d.fdesc = o.descriptors;
    d.feat_cap = o.capacity;
    d.out_count = d_counts ? d_counts + i : nullptr;
  }
  DetectJob job;
  st = build_job(ctx, imgs, *cfg, job, 0, nullptr);
  if (st != PSIFT_OK) return st;
  // The plan table (image, output and workspace pointers) is data: it is uploaded
  // before every run, so one graph serves every call with the same geometry.
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(job.d_plans, job.plans.data(), sizeof(ImagePlan) * n, cudaMemcpyHostToDevice,
                                      ctx->stream));
  if (ctx->timer.enabled) return launch_detect(ctx, job, *cfg, false, nullptr, true);
  return run_detect_cached(ctx, job, *cfg, "dev");
}


// compute_sift_descriptors_with_kind (src/pipeline.rs:1585-1620): orientations and
// descriptors for caller-given keypoints.  Like the reference, the pyramid is
// rebuilt with scales = max(max layer, 3), the first-octave upsampling inferred
// from the first layered keypoint's scale, octaves = max octave + 1, and no
// feature cap.
psift_status psift_gaussian_blur(psift_ctx* ctx, const float* image, uint32_t h, uint32_t w, size_t stride,
                                 float sigma, float* out) {
  if (!ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaSetDevice");
  if (h == 0 || w == 0) return PSIFT_OK;
  if (!image || !out || stride < w) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "bad image/output argument");
  if (!(sigma == sigma)) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "sigma is NaN");
  const std::vector<float> taps = gaussian_taps(sigma);
  const int radius = (int)taps.size() / 2;
  if (radius > kMaxTaps / 2 - 1)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "sigma gives a radius above 15 (sigma > 5)");
  HostOctave H{(int)h, (int)w, (long long)align_up((size_t)w, 32)};
  const size_t img_bytes = sizeof(float) * (size_t)h * w;
  psift_status st = arena_reserve(ctx, align_up(sizeof(ImagePlan), 256) + align_up(img_bytes, 256) +
                                           align_up(plane_bytes(H), 256) + 256);
  if (st != PSIFT_OK) return st;
  ImagePlan* d_plan = (ImagePlan*)arena_alloc(ctx, sizeof(ImagePlan));
  float* d_src = (float*)arena_alloc(ctx, img_bytes);
  float* d_out = (float*)arena_alloc(ctx, plane_bytes(H));
  ImagePlan P;
  std::memset(&P, 0, sizeof P);
  P.src = d_src;
  P.src_stride = w;
  P.src_h = (int)h;
  P.src_w = (int)w;
  P.src_kind = SRC_F32;
  P.n_oct = 1;
  P.oct[0].h = (int)h;
  P.oct[0].w = (int)w;
  P.oct[0].pitch = H.pitch;
  P.oct[0].plane_stride = H.pitch * h;
  P.oct[0].g = d_out;
  PSIFT_CUDA_TRY(ctx, cudaMemcpy2DAsync(d_src, sizeof(float) * w, image, sizeof(float) * stride, sizeof(float) * w, h,
                                        cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_plan, &P, sizeof P, cudaMemcpyHostToDevice, ctx->stream));
  cudaError_t e = launch_blur(1, taps.data(), radius, d_plan, 1, 0, 0, -1, (int)h, (int)w, ctx->stream);
  ctx->launches++;
  if (e != cudaSuccess) return cuda_error(ctx, e, "gaussian_blur");
  PSIFT_CUDA_TRY(ctx, cudaMemcpy2DAsync(out, sizeof(float) * w, d_out, sizeof(float) * H.pitch, sizeof(float) * w, h,
                                        cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PSIFT_OK;
}

psift_status psift_build_pyramid(psift_ctx* ctx, const float* image, uint32_t h, uint32_t w, size_t stride,
                                 const psift_sift_config* cfg, float* planes, size_t capacity, uint32_t* dims,
                                 uint32_t* n_octaves) {
  psift_status st = check_common(ctx, cfg);
  if (st != PSIFT_OK) return st;
  if (!n_octaves || !dims || (h && w && !image) || stride < w)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "bad image/output argument");
  const int S = (int)cfg->scales;
  HostOctave oct[kMaxOctaves];
  const int no = plan_octaves((int)h, (int)w, (int)cfg->octaves, cfg->upsample_first_octave != 0, oct);
  *n_octaves = (uint32_t)no;
  size_t need = 0;
  for (int o = 0; o < no; ++o) {
    dims[2 * o] = (uint32_t)oct[o].h;
    dims[2 * o + 1] = (uint32_t)oct[o].w;
    need += (size_t)(2 * S + 5) * oct[o].h * oct[o].w;
  }
  if (!planes || no == 0) return PSIFT_OK;  // geometry query
  if (capacity < need) return set_error(ctx, PSIFT_ERR_CAPACITY, "plane buffer smaller than the pyramid");
  ImageDesc d{};
  d.stride = w;
  d.h = (int)h;
  d.w = (int)w;
  d.kind = SRC_F32;
  d.feat_cap = 1;
  std::vector<ImageDesc> imgs{d};
  DetectJob job;
  const size_t img_bytes = sizeof(float) * (size_t)h * w;
  void* extra = nullptr;
  psift_sift_config c = *cfg;
  c.max_features = 0;
  st = build_job(ctx, imgs, c, job, img_bytes, &extra);
  if (st != PSIFT_OK) return st;
  job.plans[0].src = extra;
  PSIFT_CUDA_TRY(ctx, cudaMemcpy2DAsync(extra, sizeof(float) * w, image, sizeof(float) * stride, sizeof(float) * w, h,
                                        cudaMemcpyHostToDevice, ctx->stream));
  st = launch_pyramid_only(ctx, job, c);
  if (st != PSIFT_OK) return st;
  float* dst = planes;
  for (int o = 0; o < no; ++o) {
    const OctaveDev& O = job.plans[0].oct[o];
    const size_t hw = (size_t)O.h * O.w;
    for (int i = 0; i < 2 * S + 5; ++i) {
      const float* src = i < S + 3 ? O.g + (size_t)i * O.plane_stride : O.d + (size_t)(i - S - 3) * O.plane_stride;
      PSIFT_CUDA_TRY(ctx, cudaMemcpy2DAsync(dst, sizeof(float) * O.w, src, sizeof(float) * O.pitch,
                                            sizeof(float) * O.w, O.h, cudaMemcpyDeviceToHost, ctx->stream));
      dst += hw;
    }
  }
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PSIFT_OK;
}

psift_status psift_compute_descriptors(psift_ctx* ctx, const float* image, uint32_t h, uint32_t w, size_t stride,
                                       const psift_keypoint* kps, uint32_t n, int32_t kind, psift_features* out) {
  if (!ctx || !out) return PSIFT_ERR_INVALID_ARGUMENT;
  if (kind != 0 && kind != 1) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "descriptor kind must be 0 or 1");
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaSetDevice");
  out->count = 0;
  if (h < 3 || w < 3 || n == 0) return PSIFT_OK;
  if (!image || !kps || stride < w) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "bad image/keypoint argument");
  uint32_t max_layer = 0;
  for (uint32_t i = 0; i < n; ++i) max_layer = std::max(max_layer, kps[i].layer);
  const uint32_t scales = std::max(max_layer, 3u);
  if (scales > 10) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "keypoint layer beyond 10 scales");
  const float k = std::pow(2.0f, 1.0f / (float)scales);
  bool upsample = false;
  for (uint32_t i = 0; i < n; ++i)
    if (kps[i].layer > 0) {
      const float expected = kBaseSigma * (float)(1ull << std::min(kps[i].octave, 62u)) * powi_f(k, (int)kps[i].layer);
      upsample = (kps[i].scale / expected) < 0.707f;
      break;
    }
  uint64_t max_oct = 0;
  for (uint32_t i = 0; i < n; ++i) {
    uint64_t o;
    if (kps[i].layer > 0) {
      o = kps[i].octave;
    } else {
      const float f = std::floor(std::log2(std::fmax(kps[i].scale / kBaseSigma, 1.0f)));
      o = f <= 0.0f ? 0 : (uint64_t)f;
    }
    max_oct = std::max(max_oct, o);
  }
  psift_sift_config cfg;
  psift_sift_config_default(&cfg);
  cfg.octaves = (uint32_t)std::min<uint64_t>(max_oct + 1, (uint64_t)kMaxOctaves);
  cfg.scales = scales;
  cfg.upsample_first_octave = upsample ? 1 : 0;
  cfg.descriptor_kind = kind;
  cfg.max_features = 0;
  const uint32_t feat_cap = std::min<uint64_t>(4ull * n, 0xFFFFFFFFull);
  ImageDesc d{};
  d.stride = w;
  d.h = (int)h;
  d.w = (int)w;
  d.kind = SRC_F32;
  d.feat_cap = feat_cap;
  std::vector<ImageDesc> imgs{d};
  DetectJob job;
  const size_t img_bytes = sizeof(float) * (size_t)h * w;
  void* extra = nullptr;
  psift_status st = build_job(ctx, imgs, cfg, job, img_bytes + sizeof(psift_keypoint) * (size_t)n + 512, &extra);
  if (st != PSIFT_OK) return st;
  if (n > job.sel_cap) return set_error(ctx, PSIFT_ERR_CAPACITY, "more keypoints than the workspace holds (262144)");
  job.plans[0].src = extra;
  st = pinned_reserve(ctx, std::max(img_bytes + sizeof(psift_keypoint) * (size_t)n,
                                    (size_t)feat_cap * sizeof(float) * (5 + kDescLen)) + 64);
  if (st != PSIFT_OK) return st;
  char* pin = ctx->pinned.base;
  for (uint32_t y = 0; y < h; ++y) std::memcpy(pin + (size_t)y * w * 4, image + (size_t)y * stride, (size_t)w * 4);
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(extra, pin, img_bytes, cudaMemcpyHostToDevice, ctx->stream));
  // the keypoints replace the detector's output (sel list) unchanged
  std::memcpy(pin + img_bytes, kps, sizeof(psift_keypoint) * n);
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(job.plans[0].sel, pin + img_bytes, sizeof(psift_keypoint) * n,
                                      cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(job.plans[0].sel_count, &n, 4, cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));  // staging reuse below
  // pyramid only (the extrema stages are skipped), then orientation + descriptors
  st = launch_pyramid_only(ctx, job, cfg);
  if (st != PSIFT_OK) return st;
  DescribeParams dp{(int)scales, 0u, kind};
  cudaError_t e = launch_orientation(job.d_plans, 1, n, dp, ctx->stream);
  if (e == cudaSuccess) e = launch_feature_scan(job.d_plans, 1, 0, ctx->stream);
  if (e == cudaSuccess) e = launch_descriptor(job.d_plans, 1, n, dp, ctx->stream);
  ctx->launches += 3;
  if (e != cudaSuccess) return cuda_error(ctx, e, "compute_descriptors");
  uint32_t hc[2] = {0, 0};
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(pin, job.plans[0].feat_count, 8, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(hc, pin, 8);
  const uint32_t c = hc[0];
  if (c > out->capacity) {
    out->count = c;
    return set_error(ctx, PSIFT_ERR_CAPACITY, "feature output capacity too small");
  }
  const ImagePlan& P = job.plans[0];
  float* hp = (float*)pin;
  if (c) {
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hp + 0 * (size_t)c, P.fx, 4 * (size_t)c, cudaMemcpyDeviceToHost, ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hp + 1 * (size_t)c, P.fy, 4 * (size_t)c, cudaMemcpyDeviceToHost, ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hp + 2 * (size_t)c, P.fscale, 4 * (size_t)c, cudaMemcpyDeviceToHost, ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hp + 3 * (size_t)c, P.fresp, 4 * (size_t)c, cudaMemcpyDeviceToHost, ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hp + 4 * (size_t)c, P.fori, 4 * (size_t)c, cudaMemcpyDeviceToHost, ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hp + 5 * (size_t)c, P.fdesc, 4 * (size_t)c * kDescLen, cudaMemcpyDeviceToHost,
                                        ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (!out->x || !out->y || !out->scale || !out->response || !out->orientation || !out->descriptors)
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null feature output array");
    std::memcpy(out->x, hp + 0 * (size_t)c, 4 * (size_t)c);
    std::memcpy(out->y, hp + 1 * (size_t)c, 4 * (size_t)c);
    std::memcpy(out->scale, hp + 2 * (size_t)c, 4 * (size_t)c);
    std::memcpy(out->response, hp + 3 * (size_t)c, 4 * (size_t)c);
    std::memcpy(out->orientation, hp + 4 * (size_t)c, 4 * (size_t)c);
    std::memcpy(out->descriptors, hp + 5 * (size_t)c, 4 * (size_t)c * kDescLen);
  }
  out->count = c;
  return PSIFT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free detect+describe.
//
// For callers that must not allocate device memory: code running inside a
// memory-pool-less plugin host, a real-time loop where cudaMalloc's implicit
// device synchronisation is not allowed, or an embedding that hands this library
// only a stream.  Their scratch lives in one file-scope device array that every
// GPU loading this library holds until the process exits.  Inputs and outputs
// stay caller-owned device memory.
//
// Size limit: kNoAllocScratchBytes (32 MiB).  That holds the scale space of a
// 320x240 image with the reference's defaults (octaves <= 4, scales 3, first-octave
// upsampling) plus 65536 keypoint slots; requests needing more are rejected.
// ---------------------------------------------------------------------------
namespace psift {
namespace {

constexpr size_t kNoAllocScratchBytes = 32u << 20;
constexpr uint32_t kNoAllocKeypointCapacity = 1u << 16;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device (host code may not use the
// symbol itself: on the host it names a stand-in, not device memory).
std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {nullptr};

psift_status noalloc_scratch_address(psift_ctx* ctx, void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_error(ctx, e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(ctx, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return PSIFT_OK;
}

// Bump carve inside the fixed scratch; returns nullptr when it would overflow.
struct FixedCarver {
  char* base;
  size_t cap, off = 0, need = 0;
  void* take(size_t bytes) {
    const size_t o = align_up(off, 256);
    off = o + bytes;
    need = off;
    return off <= cap ? base + o : nullptr;
  }
};

// Lays out one image's buffers (same layout as build_job) inside the scratch.
bool carve_noalloc_job(FixedCarver& cv, const ImageDesc& img, const psift_sift_config& cfg, DetectJob& job) {
  const int S = (int)cfg.scales;
  job.n = 1;
  job.kp_cap = kNoAllocKeypointCapacity;
  job.sel_cap = cfg.max_features ? cfg.max_features : job.kp_cap;
  job.oct.assign(kMaxOctaves, HostOctave{0, 0, 0});
  job.n_oct.assign(1, plan_octaves(img.h, img.w, (int)cfg.octaves, cfg.upsample_first_octave != 0, job.oct.data()));
  job.plans.assign(1, ImagePlan{});
  ImagePlan& P = job.plans[0];
  std::memset(&P, 0, sizeof(P));
  job.d_plans = (ImagePlan*)cv.take(sizeof(ImagePlan));
  P.src = img.src;
  P.src_stride = img.stride;
  P.src_h = img.h;
  P.src_w = img.w;
  P.src_kind = img.kind;
  P.upsample = cfg.upsample_first_octave != 0;
  P.n_oct = job.n_oct[0];
  int row_base = 0;
  const float base_mult = cfg.upsample_first_octave ? 0.5f : 1.0f;
  for (int o = 0; o < P.n_oct; ++o) {
    const HostOctave& H = job.oct[o];
    OctaveDev& O = P.oct[o];
    O.h = H.h;
    O.w = H.w;
    O.pitch = H.pitch;
    O.plane_stride = H.pitch * H.h;
    float* planes = (float*)cv.take(plane_bytes(H) * (2 * S + 5));
    O.g = planes;
    O.d = planes ? planes + O.plane_stride * (S + 3) : nullptr;
    O.words = (H.w + 31) / 32;
    O.masks = (uint32_t*)cv.take(sizeof(uint32_t) * (size_t)S * H.h * O.words);
    O.row_base = row_base;
    O.scale_factor = base_mult * (float)(1ull << o);
    row_base += S * H.h;
  }
  P.total_rows = row_base;
  P.row_counts = (uint32_t*)cv.take(sizeof(uint32_t) * (size_t)row_base + 4);
  P.row_offsets = (uint32_t*)cv.take(sizeof(uint32_t) * (size_t)row_base + 4);
  P.kps = (psift_keypoint*)cv.take(sizeof(psift_keypoint) * job.kp_cap);
  P.sel = (psift_keypoint*)cv.take(sizeof(psift_keypoint) * job.sel_cap);
  P.oris = (float*)cv.take(sizeof(float) * 4 * job.sel_cap);
  P.ori_count = (uint32_t*)cv.take(sizeof(uint32_t) * job.sel_cap);
  P.feat_offsets = (uint32_t*)cv.take(sizeof(uint32_t) * job.sel_cap);
  uint32_t* counters = (uint32_t*)cv.take(256);
  if (counters) {
    P.kp_count = counters + 0;
    P.sel_count = counters + 1;
    P.feat_count = counters + 2;
    P.feat_total = counters + 3;
  }
  P.out_count = img.out_count;
  P.feat_cap = img.feat_cap;
  P.fx = img.fx;
  P.fy = img.fy;
  P.fscale = img.fscale;
  P.fresp = img.fresp;
  P.fori = img.fori;
  P.fdesc = img.fdesc;
  return cv.need <= cv.cap;
}

}  // namespace
}  // namespace psift

extern "C" psift_status psift_detect_and_compute_u8_noalloc_dev(const uint8_t* luma, uint32_t height, uint32_t width,
                                                                size_t row_stride, const psift_sift_config* cfg,
                                                                psift_features* out, uint32_t* d_count,
                                                                void* cuda_stream) {
  // A stack context carries the caller's stream and the error message; it owns
  // no device memory and is never passed to an allocating helper.
  psift_ctx local;
  local.stream = (cudaStream_t)cuda_stream;
  char msg[256];
  psift_status st = psift_sift_config_validate(cfg, msg, sizeof msg);
  if (st != PSIFT_OK) return st;
  if (!out || !d_count || (height && width && !luma) || row_stride < width || !out->x || !out->y || !out->scale ||
      !out->response || !out->orientation || !out->descriptors || out->capacity == 0)
    return PSIFT_ERR_INVALID_ARGUMENT;
  if (local.stream) {
    // the stream must belong to the current device, whose scratch address is used
    int cur = 0, sdev = 0;
    if (cudaGetDevice(&cur) != cudaSuccess || cudaStreamGetDevice(local.stream, &sdev) != cudaSuccess)
      return PSIFT_ERR_CUDA;
    if (sdev != cur) return PSIFT_ERR_INVALID_ARGUMENT;
  }
  void* scratch = nullptr;
  st = noalloc_scratch_address(&local, &scratch);
  if (st != PSIFT_OK) return st;
  // First 256 bytes: the device error word; the job is carved after it.
  uint32_t* d_err = (uint32_t*)scratch;
  FixedCarver cv{(char*)scratch + 256, kNoAllocScratchBytes - 256};
  ImageDesc img{};
  img.src = luma;
  img.stride = (long long)row_stride;
  img.h = (int)height;
  img.w = (int)width;
  img.kind = SRC_U8;
  img.fx = out->x;
  img.fy = out->y;
  img.fscale = out->scale;
  img.fresp = out->response;
  img.fori = out->orientation;
  img.fdesc = out->descriptors;
  img.feat_cap = out->capacity;
  img.out_count = d_count;
  DetectJob job;
  if (!carve_noalloc_job(cv, img, *cfg, job)) return PSIFT_ERR_CAPACITY;
  local.d_error = d_err;
  cudaError_t e = cudaMemsetAsync(d_err, 0, sizeof(uint32_t), local.stream);
  if (e != cudaSuccess) return PSIFT_ERR_CUDA;
  st = launch_detect(&local, job, *cfg, false);
  if (st != PSIFT_OK) return st;
  // the error word and the number of features found (before the output cut)
  uint32_t h_err = 0, h_total = 0;
  e = cudaMemcpyAsync(&h_err, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, local.stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&h_total, job.plans[0].feat_total, sizeof(uint32_t), cudaMemcpyDeviceToHost, local.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(local.stream);
  if (e != cudaSuccess) return PSIFT_ERR_CUDA;
  // same mapping as the regular entries: capacity, timeout, internal
  if (h_err & kErrKeypointCapacity) return PSIFT_ERR_CAPACITY;
  if (h_err & kErrSortCapacity) return PSIFT_ERR_INTERNAL;
  if (h_err & kErrTimeout) return PSIFT_ERR_TIMEOUT;
  if (h_err) return PSIFT_ERR_INTERNAL;
  const uint32_t needed = cfg->max_features && h_total > cfg->max_features ? cfg->max_features : h_total;
  if (needed > out->capacity) {
    // the kernels cut the list at the capacity; report the size that was needed
    e = cudaMemcpyAsync(d_count, &needed, sizeof(uint32_t), cudaMemcpyHostToDevice, local.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(local.stream);
    if (e != cudaSuccess) return PSIFT_ERR_CUDA;
    return PSIFT_ERR_CAPACITY;
  }
  return PSIFT_OK;
}
