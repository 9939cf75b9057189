/*
 * psift_gpu.h -- C ABI of libpsift_gpu.so, the sm_100a (B200) implementation of
 * pure-sift's feature hot path.
 *
 * The reference exposes this path as a Rust API (src/lib.rs:26-52) with no FFI
 * of its own.  Each entry point below names the reference function it replaces;
 * a Rust binding crate maps the reference's structs onto
 * these plain-pointer signatures so `Sift::detect_and_compute`, `Matcher::match_`,
 * `Homography::estimate` and the catalog search keep their signatures.
 *
 * Conventions
 *  - Every call returns psift_status; nothing aborts.  A failing call leaves a
 *    message retrievable with psift_last_error(ctx).
 *  - Pointers are HOST memory unless the function name ends in `_dev`, in which
 *    case every array argument is device memory on the context's GPU.
 *  - Outputs are caller-owned.  When an output would exceed the capacity the
 *    caller gave, the call returns PSIFT_ERR_CAPACITY and stores the required
 *    size in the `count` field / out-parameter.
 *  - A context owns one CUDA stream and its workspaces; it is not thread-safe.
 *    Use one context per host thread.
 *  - There is no CPU fallback: without a usable CUDA device psift_ctx_create
 *    returns PSIFT_ERR_NO_DEVICE.
 */
#ifndef PSIFT_GPU_H
#define PSIFT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSIFT_DESCRIPTOR_LEN 128u          /* SIFT_DESCRIPTOR_LEN, src/pipeline.rs:1000 */
#define PSIFT_MAX_FEATURES_PER_IMAGE 4096u /* MAX_FEATURES_PER_IMAGE, src/pipeline.rs:1054 */

typedef enum psift_status {
  PSIFT_OK = 0,
  PSIFT_ERR_INVALID_ARGUMENT = 1, /* null pointer, zero size, bad enum */
  PSIFT_ERR_INVALID_CONFIG = 2,   /* SiftConfig::validate / Matcher::new / RansacOptions::validate failed */
  PSIFT_ERR_CAPACITY = 3,         /* output larger than the caller's capacity (required size reported) */
  PSIFT_ERR_CUDA = 4,             /* a CUDA runtime call failed */
  PSIFT_ERR_OUT_OF_MEMORY = 5,    /* device or pinned allocation failed */
  PSIFT_ERR_TIMEOUT = 6,          /* a bounded device-side wait gave up */
  PSIFT_ERR_NO_DEVICE = 7,        /* no usable sm_100 device */
  PSIFT_ERR_INTERNAL = 8,
  PSIFT_ERR_IO = 9,               /* a catalog file could not be opened, read, written or renamed */
  PSIFT_ERR_FORMAT = 10           /* a PSIFTCAT file is malformed (magic, version, kind, truncation, UTF-8) */
} psift_status;

typedef struct psift_ctx psift_ctx;

/* SiftConfig (src/pipeline.rs:22-104) plus the feature cap that
 * extract_sift_features_with_kind applies (src/pipeline.rs:1643-1656). */
typedef struct psift_sift_config {
  uint32_t octaves;            /* 1..=8, default 3 */
  uint32_t scales;             /* 3..=10, default 3 */
  float contrast_threshold;    /* (0, 1], default 0.015 */
  int32_t upsample_first_octave; /* default 1 */
  int32_t descriptor_kind;     /* 0 = Sift (default), 1 = RootSift */
  uint32_t max_features;       /* default 4096 (the reference's cap); 0 = uncapped */
} psift_sift_config;

/* Keypoint (src/pipeline.rs:252-267). */
typedef struct psift_keypoint {
  float x, y, scale, response;
  uint32_t octave, layer;
} psift_keypoint;

/* Structure-of-arrays SiftFeature list (src/pipeline.rs:1059-1072). */
typedef struct psift_features {
  uint32_t capacity;   /* in: number of features the arrays can hold */
  uint32_t count;      /* out: features produced (or required, on PSIFT_ERR_CAPACITY) */
  float* x;
  float* y;
  float* scale;
  float* response;
  float* orientation;
  float* descriptors;  /* capacity * 128, row-major */
} psift_features;

/* FeatureMatch (src/pipeline.rs:1076-1091); 40 bytes. */
typedef struct psift_match {
  uint32_t query_index, target_index;
  float query_x, query_y;
  float target_x, target_y;
  float distance;   /* sqrt of the best squared distance */
  float ratio;      /* d1 / d2 */
  float displacement_x, displacement_y;
} psift_match;

/* ---------------------------------------------------------------- context */
psift_status psift_ctx_create(int device, psift_ctx** out);
psift_status psift_ctx_destroy(psift_ctx* ctx);
const char* psift_last_error(const psift_ctx* ctx);
/* Number of this library's kernel launches issued on the context so far. */
uint64_t psift_ctx_launch_count(const psift_ctx* ctx);
/* The context's CUDA stream (cudaStream_t) for event timing / interop. */
void* psift_ctx_stream(const psift_ctx* ctx);
psift_status psift_ctx_synchronize(psift_ctx* ctx);
/* Optional per-stage device timing (CUDA events on the context stream).
 * Stages: 0 pyramid (octave base + blur/DoG levels), 1 extrema (mark, scan,
 * emit), 2 top-K cap, 3 orientation, 4 descriptors, 5 matching, 6 Hamming,
 * 7 RANSAC, 8 MLP.  psift_ctx_stage_times synchronises the stream and returns
 * the accumulated milliseconds and the number of timed intervals per stage. */
/* CUDA graphs for psift_detect_and_compute_batch_dev and the one-image host
 * entries psift_detect_and_compute[_u8] (on by default): the first call with a
 * given launch geometry (image count and sizes, input type, config) runs
 * eagerly, the second is captured into a graph, later ones replay it.  The
 * plan table of each call (image and output pointers) is uploaded before the
 * replay, so pointers may change between calls.  Off while stage timing is on. */
psift_status psift_ctx_enable_graphs(psift_ctx* ctx, int enable);
uint64_t psift_ctx_graph_replays(const psift_ctx* ctx);
psift_status psift_ctx_enable_stage_timing(psift_ctx* ctx, int enable);

/* Tile shapes, chosen by the library's autotuner.  No counterpart in the
 * reference.  Every choice computes identical results; only time differs.
 *  - PSIFT_TUNE_BLUR, index = radius 1..15: the level blur's kernel: outputs per
 *    thread 0: 4 columns x 8 rows (the default), 1: 8 x 8, 2: 4 x 4; 3: TMA
 *    tiles with persistent CTAs (batches of at most 64 images; larger ones use 0);
 *    4: 128-row tiles of 512 threads (4 x 8 outputs per thread).
 *    A batch of images of different sizes runs variant 0's shape (or 3) over a
 *    list of every image's tiles.  Every variant computes the same values.
 *  - PSIFT_TUNE_MATCH_FP32 / PSIFT_TUNE_MATCH_TC, index 0: the matchers' work items
 *    per SM (default 2); a query tile's target tiles are split into that many
 *    ranges overall, which sets each CTA's target extent.
 * psift_ctx_autotune times every candidate on synthetic inputs of the caller's
 * geometry (n_images u8 images of height x width with cfg's blur schedule;
 * n_pairs matching problems of n_desc x n_desc descriptors, both matcher paths)
 * and keeps the fastest in the context (for the blur, another variant replaces
 * variant 0 only when it is at least 3 % faster).  report (optional, report_capacity
 * doubles; report_count = the doubles written): per blur radius (radius, ms of
 * variants 0..4, chosen), then -1, then per matcher path (path 0 FP32 / 1 tensor
 * core, ms for 1, 2, 4, 8 work items per SM, chosen). */
#define PSIFT_TUNE_BLUR 0
#define PSIFT_TUNE_MATCH_FP32 1
#define PSIFT_TUNE_MATCH_TC 2
psift_status psift_ctx_autotune(psift_ctx* ctx, uint32_t height, uint32_t width, uint32_t n_images,
                                const psift_sift_config* cfg, uint32_t n_desc, uint32_t n_pairs, double* report,
                                uint32_t report_capacity, uint32_t* report_count);
psift_status psift_ctx_tuning_get(const psift_ctx* ctx, int32_t what, int32_t index, int32_t* value);
/* Blur rounding of the detection entries on this context.  No counterpart in
 * the reference.  PSIFT_BLUR_REFERENCE (default): every tap a rounded multiply
 * and a rounded add, bit-equal to gaussian_blur (src/pipeline.rs:314-425).
 * PSIFT_BLUR_FUSED: every tap one fused multiply-add (one rounding), which halves
 * the blur's arithmetic; results are no longer bit-equal to the reference's, and
 * their error against an f64 run of the pipeline is held to the f32 path's
 * tolerances (keypoints within 0.01 px and 0.01 scale, descriptors within 1e-4
 * relative L2).  psift_gaussian_blur always uses the reference's rounding. */
#define PSIFT_BLUR_REFERENCE 0
#define PSIFT_BLUR_FUSED 1
psift_status psift_ctx_set_blur_rounding(psift_ctx* ctx, int32_t mode);
psift_status psift_ctx_tuning_set(psift_ctx* ctx, int32_t what, int32_t index, int32_t value);
psift_status psift_ctx_stage_times(psift_ctx* ctx, double* ms, uint64_t* counts, uint32_t n, int reset);

/* ---------------------------------------------------------------- config */
/* SiftConfig::default() (src/pipeline.rs:36-46) with max_features = 4096. */
void psift_sift_config_default(psift_sift_config* cfg);
/* SiftConfig::validate (src/pipeline.rs:80-103); message copied into msg. */
psift_status psift_sift_config_validate(const psift_sift_config* cfg, char* msg, size_t msg_capacity);

/* ---------------------------------------------------------------- SIFT */
/* Sift::detect_and_compute (src/pipeline.rs:136-145) on a row-major f32 image
 * (luma in [0, 1], `Array2<f32>`); row_stride in elements (>= width). */
psift_status psift_detect_and_compute(psift_ctx* ctx, const float* image, uint32_t height,
                                      uint32_t width, size_t row_stride,
                                      const psift_sift_config* cfg, psift_features* out);
/* Same, from u8 luma; fuses luma_to_array2 (src/pipeline.rs:957-966). */
psift_status psift_detect_and_compute_u8(psift_ctx* ctx, const uint8_t* luma, uint32_t height,
                                         uint32_t width, size_t row_stride,
                                         const psift_sift_config* cfg, psift_features* out);
/* Sift::detect_keypoints (src/pipeline.rs:125-133). */
psift_status psift_detect_keypoints(psift_ctx* ctx, const float* image, uint32_t height,
                                    uint32_t width, size_t row_stride,
                                    const psift_sift_config* cfg, psift_keypoint* out,
                                    uint32_t capacity, uint32_t* count);

/* gaussian_blur (src/pipeline.rs:314-425): separable blur with the f32 weights of
 * gaussian_kernel_1d (:275-311) and clamp-to-edge borders; `out` is a dense
 * height x width host array.  Bit-identical to the reference.  Radii above 15
 * (sigma > 5) are rejected; the pyramid never needs them. */
psift_status psift_gaussian_blur(psift_ctx* ctx, const float* image, uint32_t height, uint32_t width,
                                 size_t row_stride, float sigma, float* out);
/* build_scale_space_pyramid_with_options (src/pipeline.rs:550-638): for each
 * octave o < *n_octaves, its scales+3 Gaussian planes then its scales+2 DoG
 * planes, each dims[2o] x dims[2o+1] dense row-major, octave after octave in
 * `planes` (capacity in floats).  dims holds 2 * cfg->octaves entries.  With
 * planes == NULL only the geometry is returned.  Bit-identical to the reference. */
psift_status psift_build_pyramid(psift_ctx* ctx, const float* image, uint32_t height, uint32_t width,
                                 size_t row_stride, const psift_sift_config* cfg, float* planes,
                                 size_t capacity, uint32_t* dims, uint32_t* n_octaves);

/* compute_sift_descriptors_with_kind (src/pipeline.rs:1585-1629): orientations
 * and descriptors for caller-given keypoints (the CLI extract path).  The pyramid
 * is rebuilt with scales / octaves / upsampling inferred from the keypoints as
 * the reference does; no feature cap.  kind: 0 = Sift, 1 = RootSift. */
psift_status psift_compute_descriptors(psift_ctx* ctx, const float* image, uint32_t height,
                                       uint32_t width, size_t row_stride, const psift_keypoint* kps,
                                       uint32_t n, int32_t kind, psift_features* out);

/* Device-resident batch: `n` u8 images already in device memory, results left
 * in device memory (feature SoA pointers in outs[i] are device pointers) and the
 * per-image feature counts written to the device array d_counts.  No host
 * synchronisation; work is queued on the context's stream. */
typedef struct psift_image_u8 {
  const uint8_t* data;   /* device pointer (host pointer for the host batch entry) */
  uint32_t height, width;
  size_t row_stride;     /* elements */
} psift_image_u8;
psift_status psift_detect_and_compute_batch_dev(psift_ctx* ctx, const psift_image_u8* images,
                                                uint32_t n, const psift_sift_config* cfg,
                                                psift_features* outs, uint32_t* d_counts);

/* Host-pointer batch of u8 images (psift_image_u8.data are host pointers,
 * row_stride in bytes); features into the host arrays of outs[i] (capacity per
 * image, count written back).  One launch per stage for the whole batch, two
 * chunks on two streams so transfers overlap kernels, one final synchronisation.
 * Page-locked inputs/outputs (psift_host_alloc, cudaMallocHost, cudaHostRegister)
 * are transferred directly.  No counterpart in the reference (which handles one
 * image per Sift::detect_and_compute call); per image, results equal
 * psift_detect_and_compute_u8.  If any image's features exceed its capacity the
 * call returns PSIFT_ERR_CAPACITY with that image's count set to the size needed. */
psift_status psift_detect_and_compute_u8_batch(psift_ctx* ctx, const psift_image_u8* images, uint32_t n,
                                               const psift_sift_config* cfg, psift_features* outs);
/* ---------------------------------------------------------------- JPEG input */
/* decode_validated_dynamic_image / decode_validated_luma8 (src/cli.rs:129-170)
 * for JPEG bytes, decoded on the GPU by nvJPEG (hardware JPEG engines when
 * available, else its GPU-assisted backend; loaded on first use) and converted
 * with the image crate's rgb_to_luma ((2126 R + 7152 G + 722 B) / 10000, u32,
 * truncating).  Header checks as the reference: width and height >= 8
 * (MIN_IMAGE_DIM), and with enforce_pixel_cap <= 8192 each and <= 25,000,000
 * pixels (MAX_IMAGE_DIM, MAX_IMAGE_PIXELS); violations return
 * PSIFT_ERR_INVALID_ARGUMENT with the reference's message, undecodable bytes
 * PSIFT_ERR_FORMAT, a missing nvJPEG PSIFT_ERR_INTERNAL.  Decoded pixels follow
 * nvJPEG's IDCT and chroma upsampling (not the image crate's decoder). */
psift_status psift_jpeg_info(psift_ctx* ctx, const uint8_t* data, size_t length, int32_t enforce_pixel_cap,
                             uint32_t* width, uint32_t* height, uint32_t* components);
/* One JPEG to host u8 luma (width x height, dense rows; capacity in bytes). */
psift_status psift_decode_jpeg_luma(psift_ctx* ctx, const uint8_t* data, size_t length, int32_t enforce_pixel_cap,
                                    uint8_t* luma, size_t capacity, uint32_t* width, uint32_t* height);
/* The extract path from bytes (run_extract_from_bytes, src/cli.rs:173-185, with
 * Sift::detect_and_compute's features): n JPEG buffers (host) decoded on the GPU
 * straight into the batch's device inputs, then as psift_detect_and_compute_u8_batch
 * (features into the host arrays of outs[i]).  Per image, the features equal
 * psift_detect_and_compute_u8 of the luma psift_decode_jpeg_luma returns. */
psift_status psift_detect_and_compute_jpeg_batch(psift_ctx* ctx, const uint8_t* const* data, const size_t* lengths,
                                                 uint32_t n, int32_t enforce_pixel_cap,
                                                 const psift_sift_config* cfg, psift_features* outs);
/* PNG input (decode_validated_luma8 with the image crate's PNG decoder,
 * src/cli.rs:129-170): the header checks and messages as for JPEG; every
 * chunk's CRC is checked; colour types 0, 2, 3, 4, 6 at all their bit depths,
 * Adam7 interlacing.  The zlib stream is inflated on host threads; the row
 * filters are undone and the samples converted to luma on the GPU (into_luma8:
 * rgb_to_luma on 8- or 16-bit samples, 16-bit results to u8 by rounding,
 * alpha dropped, palettes and low bit depths expanded).  Lossless: the luma
 * equals the reference's.  components = channels (1, 2, 3 or 4). */
psift_status psift_png_info(psift_ctx* ctx, const uint8_t* data, size_t length, int32_t enforce_pixel_cap,
                            uint32_t* width, uint32_t* height, uint32_t* components);
/* One PNG to host u8 luma (width x height, dense rows; capacity in bytes). */
psift_status psift_decode_png_luma(psift_ctx* ctx, const uint8_t* data, size_t length, int32_t enforce_pixel_cap,
                                   uint8_t* luma, size_t capacity, uint32_t* width, uint32_t* height);
/* The extract path from n PNG buffers (host), as psift_detect_and_compute_jpeg_batch. */
psift_status psift_detect_and_compute_png_batch(psift_ctx* ctx, const uint8_t* const* data, const size_t* lengths,
                                                uint32_t n, int32_t enforce_pixel_cap,
                                                const psift_sift_config* cfg, psift_features* outs);
/* The extract path from n image buffers of either format, told apart by their
 * leading bytes (the PNG signature, else JPEG): each format's batch entry over
 * its images, features into outs[i] in the callers' order. */
psift_status psift_detect_and_compute_image_batch(psift_ctx* ctx, const uint8_t* const* data, const size_t* lengths,
                                                  uint32_t n, int32_t enforce_pixel_cap,
                                                  const psift_sift_config* cfg, psift_features* outs);
/* How a context decodes a JPEG batch.  threads = 0 (default): the batch is split
 * into contiguous shares of at most 50 images over up to 16 host threads (the
 * hardware concurrency), each share decoded by nvJPEG's hybrid backend (Huffman
 * stage on its thread, the rest on its own stream; the context's stream waits
 * for all); threads = k > 1: k threads; threads = 1: one batched call on the
 * calling thread (the hardware backend when available, else the GPU-assisted
 * one, which moves the Huffman stage to the GPU for batches above 50 images). */
psift_status psift_ctx_set_jpeg_threads(psift_ctx* ctx, int32_t threads);
/* nvJPEG backend of the context's last decoded batch: 3 = hardware, 2 = GPU-assisted,
 * 1 = hybrid on host threads, -1 = none yet. */
psift_status psift_ctx_jpeg_backend(psift_ctx* ctx, int32_t* backend);

/* Page-locked host memory for the batch entry's inputs and outputs. */
psift_status psift_host_alloc(psift_ctx* ctx, size_t bytes, void** out);
psift_status psift_host_free(psift_ctx* ctx, void* p);

/* ---------------------------------------------------------------- matching */
#define PSIFT_PRECISION_FP32 0        /* exact f32 distances, the reference's summation order */
#define PSIFT_PRECISION_BF16_RERANK 1 /* bf16 tcgen05 distances + certified exact f32 re-rank:
                                         the same match list as PSIFT_PRECISION_FP32 */
/* MatchOptions (src/pipeline.rs:1721-1736) plus the arithmetic path. */
typedef struct psift_match_options {
  float ratio;        /* (0, 1], default 0.75 (DEFAULT_MATCH_RATIO) */
  int32_t mutual;     /* mutual nearest-neighbour cross-check, default 0 */
  int32_t precision;  /* PSIFT_PRECISION_*, default BF16_RERANK */
} psift_match_options;
void psift_match_options_default(psift_match_options* opt);
/* Matcher::new (src/pipeline.rs:156-164). */
psift_status psift_match_options_validate(const psift_match_options* opt, char* msg, size_t msg_capacity);
/* Matcher::match_ (src/pipeline.rs:167-169 -> :1744-1841).  Descriptors are
 * n x 128 f32 row-major, coordinates n x 2 (x, y).  Matches come out in query
 * order; at most nq of them. */
psift_status psift_match_descriptors(psift_ctx* ctx, const float* query_descriptors, uint32_t nq,
                                     const float* target_descriptors, uint32_t nt, const float* query_xy,
                         const float* target_xy, const psift_match_options* opt,
                         psift_match* out, uint32_t capacity, uint32_t* count);
/* Device-resident batch of independent matching problems (one launch per stage
 * for all of them); every pointer is device memory; capacity must be >= nq.
 * The match count of each problem is written to its d_count.  Asynchronous. */
typedef struct psift_match_job {
  const float* query_descriptors;
  const float* target_descriptors;
  const float* query_xy;
  const float* target_xy;
  uint32_t nq, nt;
  psift_match* out;
  uint32_t capacity;
  uint32_t* d_count;
} psift_match_job;
psift_status psift_match_batch_dev(psift_ctx* ctx, const psift_match_job* jobs, uint32_t n,
                                   const psift_match_options* opt);
/* Rows (queries, or targets in the mutual pass) whose bf16 candidate list could
 * not be certified and were matched by an exact scan, since context creation. */
psift_status psift_ctx_rerank_fallbacks(psift_ctx* ctx, uint64_t* rows);

/* ---------------------------------------------------------------- RANSAC */
/* RansacOptions (src/pipeline.rs:177-218). */
typedef struct psift_ransac_options {
  float reproj_threshold;  /* default 3.0 (DEFAULT_RANSAC_REPROJ_THRESHOLD) */
  int32_t has_seed;        /* 0: the built-in default seeds */
  uint64_t seed;
} psift_ransac_options;
void psift_ransac_options_default(psift_ransac_options* opt);
/* RansacOptions::validate (src/pipeline.rs:209-217). */
psift_status psift_ransac_options_validate(const psift_ransac_options* opt, char* msg, size_t msg_capacity);
/* Homography::estimate (src/pipeline.rs:225-235 -> :2663-2755): inlier_mask[i] = 1
 * for the returned inliers (in input order), h9 row-major, has_h = 0 for None.
 * Same result as the reference for the same seed. */
psift_status psift_homography_estimate(psift_ctx* ctx, const psift_match* matches, uint32_t n,
                                       const psift_ransac_options* opt, uint8_t* inlier_mask,
                                       float* h9, int32_t* has_h, uint32_t* inlier_count);
/* Homography::estimate_similarity (src/pipeline.rs:238-246 -> :2055-2191):
 * model6 = a, b, tx, ty, scale, rotation_deg. */
psift_status psift_similarity_estimate(psift_ctx* ctx, const psift_match* matches, uint32_t n,
                                       const psift_ransac_options* opt, uint8_t* inlier_mask,
                                       float* model6, int32_t* has_model, uint32_t* inlier_count);
/* TrackingSummary (src/pipeline.rs:1137-1152) of summarize_tracking
 * (src/pipeline.rs:2210-2272): similarity RANSAC (default threshold and seed) on
 * the device, the summary statistics on the host.  Scales / orientations are
 * indexed by the matches' query / target indices. */
typedef struct psift_tracking_summary {
  uint32_t raw_match_count, match_count;
  float inlier_ratio;
  float mean_dx, mean_dy, median_dx, median_dy;
  float mean_scale_ratio, mean_rotation_deg;
} psift_tracking_summary;
psift_status psift_summarize_tracking(psift_ctx* ctx, const psift_match* matches, uint32_t n,
                                      const float* query_scale, const float* query_orientation,
                                      uint32_t nq, const float* target_scale,
                                      const float* target_orientation, uint32_t nt,
                                      psift_tracking_summary* out);
/* Device-resident batch of independent estimations, one CTA each.  model holds 9
 * (homography) or 6 (similarity) floats.  sampling_weights (optional) replaces the
 * reference's 1/clamp(ratio, 0.05, 1) CDF weights (learned guided sampling);
 * iterations (optional, 2 ints) receives the similarity and homography iteration
 * counts.  Asynchronous. */
typedef struct psift_ransac_job {
  const psift_match* matches;
  uint32_t n;
  uint8_t* inlier_mask;
  float* model;
  int32_t* has_model;
  uint32_t* inlier_count;
  const float* sampling_weights;
  uint32_t* iterations;
} psift_ransac_job;
psift_status psift_ransac_batch_dev(psift_ctx* ctx, const psift_ransac_job* jobs, uint32_t n,
                                    const psift_ransac_options* opt, int32_t homography);

/* Fundamental matrix.  FundamentalRansacOptions (src/geometry.rs:107-143). */
typedef struct psift_fundamental_options {
  double sampson_threshold; /* default 1.5 (px, Sampson distance; at least 0.25 is used) */
  uint32_t max_iters;       /* default 2000 (at least 64 are allowed) */
  double confidence;        /* default 0.999 */
  uint64_t seed;            /* default 0xF00DCAFE12345678 */
} psift_fundamental_options;
void psift_fundamental_options_default(psift_fundamental_options* opt);
/* estimate_fundamental_ransac_with_options (src/geometry.rs:868-1016): normalised
 * 8-point LO-RANSAC with Sampson scoring (the 7-point solver for exactly 7 matches).
 * f9 row-major f64 (x2^T F x1 = 0 with x1 the query point), has_f = 0 for None;
 * inlier_mask[i] = 1 for the returned inliers; iterations (optional) the loop count. */
psift_status psift_fundamental_estimate(psift_ctx* ctx, const psift_match* matches, uint32_t n,
                                        const psift_fundamental_options* opt, uint8_t* inlier_mask,
                                        double* f9, int32_t* has_f, uint32_t* inlier_count,
                                        uint32_t* iterations);
/* Device-resident batch, one CTA per match set.  Asynchronous. */
typedef struct psift_fundamental_job {
  const psift_match* matches;
  uint32_t n;
  uint8_t* inlier_mask;
  double* f9;
  int32_t* has_f;
  uint32_t* inlier_count;
  uint32_t* iterations; /* optional */
} psift_fundamental_job;
psift_status psift_fundamental_batch_dev(psift_ctx* ctx, const psift_fundamental_job* jobs, uint32_t n,
                                         const psift_fundamental_options* opt);

/* ---------------------------------------------------------------- learned sampler */
/* A small MLP (8 -> 64 -> 64 -> 1, ReLU, ReLU, sigmoid; bf16 operands, f32
 * accumulation, f32 master weights) scoring each putative match's inlier
 * probability.  No counterpart in the reference.  Its output, passed as
 * psift_ransac_job.sampling_weights, drives guided RANSAC sampling.
 * Parameter layout: W1[64][8], b1[64], W2[64][64], b2[64], W3[64], b3.
 * Features (8 per match): ratio, log scale ratio, orientation difference,
 * best distance, query x / width, query y / height, target x / width,
 * target y / height. */
#define PSIFT_MLP_NUM_PARAMS 4801u
#define PSIFT_MLP_NUM_FEATURES 8u
void psift_mlp_init(uint64_t seed, float* params);
psift_status psift_mlp_infer(psift_ctx* ctx, const float* params, const float* features, uint32_t n,
                             float* prob);
psift_status psift_mlp_infer_dev(psift_ctx* ctx, const float* params, const float* features, uint32_t n,
                                 float* prob);
/* Gradients of the mean binary cross-entropy over n samples (labels 0/1). */
psift_status psift_mlp_gradients(psift_ctx* ctx, const float* params, const float* features,
                                 const float* labels, uint32_t n, float* grad, float* loss);
psift_status psift_mlp_gradients_dev(psift_ctx* ctx, const float* params, const float* features,
                                     const float* labels, uint32_t n, float* grad, float* loss);
/* Adam (beta 0.9/0.999, eps 1e-8) over seeded-shuffled minibatches; params in/out;
 * losses (optional, `steps` floats) receives each step's minibatch loss. */
psift_status psift_mlp_train(psift_ctx* ctx, float* params, const float* features, const float* labels,
                             uint32_t n, uint32_t steps, uint32_t batch, float lr, uint64_t seed,
                             float* losses);
psift_status psift_mlp_train_dev(psift_ctx* ctx, float* params, const float* features,
                                 const float* labels, uint32_t n, uint32_t steps, uint32_t batch,
                                 float lr, uint64_t seed, float* losses);

/* ---------------------------------------------------------------- catalog */
/* quantize_descriptor_u128 (src/catalog.rs:37-45): bit i set iff desc[i] > 0.065.
 * codes: 2 x u64 per descriptor, little endian (word 0 = bits 0..63). */
psift_status psift_quantize_u128(psift_ctx* ctx, const float* desc, uint32_t n, uint64_t* codes);
psift_status psift_quantize_u128_dev(psift_ctx* ctx, const float* desc, uint32_t n, uint64_t* codes);
/* Diagnostic: measured 32-bit popcount throughput of this GPU (independent
 * register chains, no memory traffic), the INT roofline of the Hamming kernels. */
psift_status psift_popc_throughput(psift_ctx* ctx, double* popc_per_s);
/* quantize_descriptor_u8 (src/pipeline.rs:1024-1030): round(v * 512) clamped to [0, 255]. */
psift_status psift_quantize_u8(psift_ctx* ctx, const float* desc, uint32_t n, uint8_t* out);
/* dequantize_descriptor_u8 (src/pipeline.rs:1034-1044): v / 512, then L2 renormalised. */
psift_status psift_dequantize_u8(psift_ctx* ctx, const uint8_t* q, uint32_t n, float* out);
/* Coarse Hamming votes of FeatureCatalog::search_features (src/catalog.rs:588-633,
 * :707-728).  Entry e owns catalog codes [entry_offsets[e], entry_offsets[e+1]).
 * votes[e] = number of queries with a signature of the entry within 24 bits; with
 * mih != 0 the signature must also share one exact byte band with the query
 * (the multi-index-hashing path the reference takes for catalogs of > 32 entries). */
psift_status psift_hamming_votes(psift_ctx* ctx, const uint64_t* query_codes, uint32_t nq,
                                 const uint64_t* catalog_codes, const int64_t* entry_offsets,
                                 uint32_t n_entries, int32_t mih, uint32_t* votes);
/* Per query, the k (<= 64) catalog codes nearest in Hamming distance, ordered by
 * (distance, catalog index); missing entries are 0xFFFFFFFF.  No counterpart in
 * the reference (its shortlist is per entry); used to shortlist catalogs of
 * millions of descriptors before an exact re-rank. */
psift_status psift_hamming_topk(psift_ctx* ctx, const uint64_t* query_codes, uint32_t nq,
                                const uint64_t* catalog_codes, uint64_t ncat, uint32_t k,
                                uint32_t* idx, uint32_t* dist);
psift_status psift_hamming_topk_dev(psift_ctx* ctx, const uint64_t* query_codes, uint32_t nq,
                                    const uint64_t* catalog_codes, uint64_t ncat, uint32_t k,
                                    uint32_t* idx, uint32_t* dist);
/* Exact f32 squared L2 distances (the reference's summation order) between each
 * query and its k candidates, re-sorted by (d2, index). */
psift_status psift_l2_rerank(psift_ctx* ctx, const float* query_desc, uint32_t nq,
                             const float* catalog_desc, uint64_t ncat, const uint32_t* candidates,
                             uint32_t k, uint32_t* out_idx, float* out_d2);
psift_status psift_l2_rerank_dev(psift_ctx* ctx, const float* query_desc, uint32_t nq,
                                 const float* catalog_desc, const uint32_t* candidates, uint32_t k,
                                 uint32_t* out_idx, float* out_d2);

/* ---------------------------------------------------------------- device-resident catalog */
/* FeatureCatalog (src/catalog.rs:182-702) with every entry's features, 128-bit
 * codes and the entry table held in device memory, so that a search runs its
 * votes, shortlist verification (Lowe matching, similarity and homography
 * RANSAC) and tracking summaries as a few batched launches.  Entry order,
 * upsert (replace in place or append), remove (swap_remove) and the PSIFTCAT v1
 * file format follow the reference.  A catalog belongs to the context it was
 * created with (its device and stream) and, like the context, is not
 * thread-safe. */
typedef struct psift_catalog psift_catalog;
/* FeatureCatalog::new (src/catalog.rs:279-289) fields plus descriptor_kind. */
typedef struct psift_catalog_params {
  uint32_t octaves, scales;
  float threshold;
  int32_t descriptor_kind; /* 0 = Sift, 1 = RootSift */
} psift_catalog_params;
psift_status psift_catalog_create(psift_ctx* ctx, const psift_catalog_params* params, psift_catalog** out);
psift_status psift_catalog_destroy(psift_catalog* cat);
psift_status psift_catalog_params_get(const psift_catalog* cat, psift_catalog_params* out);
uint32_t psift_catalog_size(const psift_catalog* cat);
/* list_summaries (src/catalog.rs:355-366) for entry i: id copied NUL-terminated
 * into id (truncated to id_capacity - 1 bytes; id_len receives the full length). */
psift_status psift_catalog_entry(const psift_catalog* cat, uint32_t i, char* id, size_t id_capacity,
                                 uint32_t* id_len, uint32_t* width, uint32_t* height, uint64_t* feature_count);
/* Index of the entry with this id (the reference's id_index), or PSIFT_ERR_INVALID_ARGUMENT. */
psift_status psift_catalog_find(const psift_catalog* cat, const char* id, uint32_t* index);
/* upsert_entry (src/catalog.rs:324-342): host SoA features (count = features->count);
 * the entry's codes are quantize_descriptor_u128 of its descriptors. */
psift_status psift_catalog_upsert(psift_catalog* cat, const char* id, uint32_t width, uint32_t height,
                                  const psift_features* features);
/* remove (src/catalog.rs:345-353): swap_remove; removed = 0 when the id is absent. */
psift_status psift_catalog_remove(psift_catalog* cat, const char* id, int32_t* removed);
/* Entry i's features back to the host (out->capacity >= the entry's count) and,
 * when codes is not NULL, its 2 x u64 codes. */
psift_status psift_catalog_features(psift_catalog* cat, uint32_t i, psift_features* out, uint64_t* codes);
/* load_binary (src/catalog.rs:447-540): the file's records go to device memory
 * through pinned staging and are split into the feature arrays there; the u8
 * descriptors are expanded by dequantize_descriptor_u8 and the stored codes are
 * kept as they are.  save_binary (:401-445): written to "<name>.tmp.<pid>" in
 * the same directory, then renamed over the target. */
psift_status psift_catalog_load_binary(psift_ctx* ctx, const char* path, psift_catalog** out);
psift_status psift_catalog_save_binary(psift_catalog* cat, const char* path);
/* One ranked hit of search_features (src/catalog.rs:576-702).  tracking.match_count
 * and tracking.inlier_ratio already hold the better of the two estimates, as in
 * the reference. */
typedef struct psift_catalog_hit {
  uint32_t entry;         /* catalog index */
  uint32_t coarse_votes;
  psift_tracking_summary tracking;
  float similarity[6];    /* a, b, tx, ty, scale, rotation_deg */
  int32_t has_similarity;
  float homography[9];
  int32_t has_homography;
} psift_catalog_hit;
/* search_features: query features are host SoA (count = query->count).  At most
 * top_k hits; *count receives their number (PSIFT_ERR_CAPACITY if > capacity). */
psift_status psift_catalog_search(psift_catalog* cat, const psift_features* query, uint32_t top_k,
                                  uint32_t shortlist_k, float ratio, float ransac_threshold,
                                  psift_catalog_hit* hits, uint32_t capacity, uint32_t* count);
/* How the coarse votes of search_features (src/catalog.rs:588-633) are computed.
 * AUTO is the reference's choice: for at most 32 entries the exhaustive rule
 * (count_coarse_hamming_votes, :707-728: some signature within 24 bits); beyond,
 * the multi-index-hashing rule (:596-621: some signature within 24 bits that
 * shares one of the query's 16 bytes), answered through the device MIH tables
 * (FeatureCatalog's 16 x 256 inverted tables, :291-321) when the query's
 * (query, entry) bitmap fits in 128 MB, else by scanning every code.  The other
 * values force one computation; all give the votes of their rule exactly. */
#define PSIFT_VOTES_AUTO 0
#define PSIFT_VOTES_MIH_SCAN 1  /* MIH rule, every code scanned */
#define PSIFT_VOTES_MIH_INDEX 2 /* MIH rule through the tables (PSIFT_ERR_CAPACITY when they cannot serve the query) */
#define PSIFT_VOTES_EXHAUSTIVE 3
/* Votes for host query codes (2 x u64 each, quantize_descriptor_u128) against the
 * resident codes; votes: host, psift_catalog_size(cat) words.  The MIH tables
 * are built on the device by the first index use after the catalog changed. */
psift_status psift_catalog_votes(psift_catalog* cat, const uint64_t* query_codes, uint32_t nq, int32_t path,
                                 uint32_t* votes);
/* The votes computation psift_catalog_search uses: PSIFT_VOTES_AUTO (default) or
 * PSIFT_VOTES_MIH_SCAN (for comparison; the same votes, the same hits). */
psift_status psift_catalog_set_search_votes(psift_catalog* cat, int32_t path);

/* ---------------------------------------------------------------- warp and stitch */
/* warp_and_stitch (src/visualize.rs:379-483): the query warped into the target's
 * frame through the inverse of h9 (row-major, f32; bilinear inverse mapping in
 * f64) and feather-blended with the target on the union canvas.  Images are RGBA8
 * with row strides in bytes.  Call with canvas = NULL for the canvas size (and
 * origin, 2 doubles, optional: the canvas corner in target coordinates), then
 * with canvas_capacity >= width * height * 4 bytes.  Errors carry the reference's
 * messages: singular homography, a corner projected to infinity or to a
 * non-finite coordinate, a canvas over 8192 x 8192 or 25,000,000 px. */
psift_status psift_warp_and_stitch(psift_ctx* ctx, const uint8_t* query, uint32_t qh, uint32_t qw,
                                   size_t q_stride, const uint8_t* target, uint32_t th, uint32_t tw,
                                   size_t t_stride, const float* h9, uint8_t* canvas, size_t canvas_capacity,
                                   uint32_t* width, uint32_t* height, double* origin);
/* Device-resident variant: query, target and canvas are device pointers (4-byte
 * aligned, strides multiples of 4); queued on the context's stream. */
psift_status psift_warp_and_stitch_dev(psift_ctx* ctx, const uint8_t* query, uint32_t qh, uint32_t qw,
                                       size_t q_stride, const uint8_t* target, uint32_t th, uint32_t tw,
                                       size_t t_stride, const float* h9, uint8_t* canvas,
                                       size_t canvas_capacity, uint32_t* width, uint32_t* height);

/* ---------------------------------------------------------------- panorama */
/* stitch_panorama (src/stitch.rs:472-948): two or more overlapping RGBA8 images
 * registered by SIFT features (the batch detection entry), pairwise Lowe
 * matching and similarity + homography RANSAC (default seeds), chained to the
 * best-connected image through a maximum spanning tree of inlier counts,
 * exposure-compensated (Brown & Lowe gains) and composited on the union canvas
 * by feather or multi-band (Laplacian pyramid over Voronoi seams) blending.
 * Images are host RGBA8 with row strides in bytes.  The canvas is host RGBA8,
 * width x height x 4 bytes, tight rows; call with canvas = NULL (or too small a
 * capacity: PSIFT_ERR_CAPACITY) to learn the size from info.  registered (n
 * bytes), gains (n floats) and homographies (n x 9 floats, row-major, image ->
 * reference; zero when not registered) are optional.  The reference's errors
 * come back as PSIFT_ERR_INVALID_ARGUMENT with its message (fewer than 2
 * images, no pair matched, no connected pair, singular homography, corner at
 * infinity or non-finite, canvas over the limits). */
typedef struct psift_rgba_image {
  const uint8_t* data;
  uint32_t height, width;
  size_t row_stride;  /* bytes, >= 4 x width */
} psift_rgba_image;
#define PSIFT_PROJECTION_PLANAR 0
#define PSIFT_PROJECTION_CYLINDRICAL 1
#define PSIFT_BLEND_FEATHER 0
#define PSIFT_BLEND_MULTIBAND 1
/* PanoramaOptions (src/stitch.rs:45-89). */
typedef struct psift_panorama_options {
  uint32_t octaves, scales;   /* default 3, 3 */
  float threshold;            /* default 0.015 */
  float ratio;                /* default 0.75 */
  float ransac_threshold;     /* default 3.0 */
  int32_t projection;         /* default planar */
  float focal_px;             /* cylindrical projection's focal length */
  int32_t blend;              /* default multi-band */
  uint32_t levels;            /* multi-band levels, default 4 (clamped to 1..=6) */
  int32_t exposure_compensation;  /* default 1 */
  uint32_t max_canvas_dim;    /* default 8192 */
  uint64_t max_canvas_pixels; /* default 25,000,000 */
  uint32_t tile_size;         /* feather tiles, default 512 (does not change results) */
} psift_panorama_options;
void psift_panorama_options_default(psift_panorama_options* opt);
/* PanoramaResult's geometry (src/stitch.rs:91-103) and the canvas origin in
 * reference coordinates. */
typedef struct psift_panorama_info {
  uint32_t width, height;
  int32_t reference_index;
  int32_t registered_count;
  double origin_x, origin_y;
} psift_panorama_info;
psift_status psift_stitch_panorama(psift_ctx* ctx, const psift_rgba_image* images, uint32_t n,
                                   const psift_panorama_options* opt, uint8_t* canvas, size_t canvas_capacity,
                                   psift_panorama_info* info, uint8_t* registered, float* gains,
                                   float* homographies);
/* warp_image_cylindrical (src/stitch.rs:166-201): out is height x width x 4 bytes. */
psift_status psift_warp_cylindrical(psift_ctx* ctx, const psift_rgba_image* image, float focal_px, uint8_t* out);
/* The compositing half of stitch_panorama (src/stitch.rs:790-940) on given
 * registration results: for each registered image its inverse homography
 * (reference -> image, 9 doubles, row-major) and gain; the canvas origin and
 * size; blend and levels as in the options.  canvas: width x height x 4 bytes. */
psift_status psift_panorama_composite(psift_ctx* ctx, const psift_rgba_image* images, uint32_t n,
                                      const uint8_t* registered, const float* gains, const double* inverses,
                                      double origin_x, double origin_y, uint32_t width, uint32_t height,
                                      int32_t blend, uint32_t levels, uint8_t* canvas);

/* Allocation-free variant of psift_detect_and_compute_batch_dev for one u8 image.
 * No counterpart in the reference: it exists for callers that cannot allocate
 * device memory -- plugin hosts that hand out only a stream, real-time loops in
 * which cudaMalloc's implicit device synchronisation is not acceptable.  All
 * scratch lives in a 32 MiB file-scope device array inside this library (held by
 * every GPU that loads it until exit); the call makes no cudaMalloc/cudaFree or
 * other allocating call.  Enough for a 320x240 image at the reference defaults
 * (octaves <= 4, scales 3, first-octave upsampling) with at most 65536 DoG
 * extrema (the regular entries hold 262144); a request needing more scratch
 * returns PSIFT_ERR_CAPACITY without touching the GPU, and more extrema than
 * 65536 returns PSIFT_ERR_CAPACITY after the run.
 *  - luma, out->x..descriptors (capacity out->capacity) and d_count are device
 *    pointers; cuda_stream is a cudaStream_t (NULL = legacy default stream)
 *    that must belong to the current device (else PSIFT_ERR_INVALID_ARGUMENT).
 *  - More features than out->capacity: the first out->capacity are written,
 *    *d_count is set to the number needed and the call returns
 *    PSIFT_ERR_CAPACITY, as the regular entries do.
 *  - The first call on a device looks up the scratch array's device address
 *    (cudaGetSymbolAddress) and keeps it for the life of the process; make that
 *    first call before any stream capture.  After cudaDeviceReset the kept
 *    address is stale: the entry does not support a device reset.
 *  - The call queues the work on cuda_stream and waits for it to finish.
 *  - Every call shares the one scratch array: calls that overlap on the GPU
 *    (other streams, other host threads) race and corrupt each other. */
psift_status psift_detect_and_compute_u8_noalloc_dev(const uint8_t* luma, uint32_t height,
                                                     uint32_t width, size_t row_stride,
                                                     const psift_sift_config* cfg,
                                                     psift_features* out, uint32_t* d_count,
                                                     void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* PSIFT_GPU_H */
