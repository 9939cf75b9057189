/*
 * psift_oracle.h -- CPU restatement of the pure-sift 0.2.0 feature hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA build:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * leg may load it.  The product library (libpsift_gpu.so) never links or calls it.
 *
 * Pinning: the reference is Rust and cannot be compiled in this environment
 * (no cargo/rustc, crates.io dependencies not vendored), and the reference
 * ships no numeric golden vectors.  The restatement is pinned against every
 * known-answer and property test the reference holds for this path
 * (tests/pipeline_tests.rs, tests/homography_properties.rs), ported to
 * tests/test_oracle_pins.py.  Bit-level numeric parity with a Rust build of the
 * reference is therefore "pinned by the reference's known-answer tests, not by
 * reference-produced vectors".
 *
 * Each function cites the reference file:line it restates.  Arithmetic follows
 * the Rust source operation by operation: f32 everywhere the reference uses f32,
 * no FMA contraction (built with -ffp-contract=off), glibc libm for
 * exp/atan2/sin/cos/pow/log2 (what Rust's f32 methods call on Linux), sequential
 * summation in the reference's order.
 */
#ifndef PSIFT_ORACLE_H
#define PSIFT_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  float x, y, scale, response;
  uint32_t octave, layer;
} oracle_keypoint;

typedef struct {
  uint32_t query_index, target_index;
  float qx, qy, tx, ty;
  float distance, ratio;
  float dx, dy;
} oracle_match;

typedef struct {
  uint32_t raw_match_count, match_count;
  float inlier_ratio;
  float mean_dx, mean_dy, median_dx, median_dy;
  float mean_scale_ratio, mean_rotation_deg;
} oracle_tracking;

int oracle_gaussian_kernel_1d(float sigma, float* out, int cap);
void oracle_gaussian_blur(const float* img, int h, int w, float sigma, float* out);
void oracle_upsample_2x(const float* img, int h, int w, float* out);
void oracle_luma_to_f32(const uint8_t* px, size_t n, float* out);

void* oracle_pyramid_build(const float* img, int h, int w, int octaves, int scales, int upsample);
int oracle_pyramid_num_octaves(const void* pyr);
void oracle_pyramid_octave_info(const void* pyr, int octave, int* h, int* w, float* scale_factor);
/* kind 0 = Gaussian level idx (0..scales+2), kind 1 = DoG slice idx (0..scales+1) */
void oracle_pyramid_copy_plane(const void* pyr, int octave, int kind, int idx, float* out);
int oracle_pyramid_extract_extrema(const void* pyr, float threshold, oracle_keypoint* out, int cap);
void oracle_pyramid_free(void* pyr);

/* Returns the total feature count (may exceed cap; only cap are written).
 * meta: 5 floats per feature (x, y, scale, response, orientation). */
int oracle_detect_and_compute(const float* img, int h, int w, int octaves, int scales,
                              float threshold, int upsample, int kind, int max_features,
                              float* meta, float* desc, int cap);
/* The same pipeline run in f64 (values, constants and libm calls), from the u8
 * luma: the yardstick that f32 results state their error against.
 * meta: 5 doubles per feature; keypoints: 6 doubles (x, y, scale, response,
 * octave, layer). */
int oracle_detect_and_compute_f64(const uint8_t* luma, int h, int w, int octaves, int scales,
                                  double threshold, int upsample, int kind, int max_features,
                                  double* meta, double* desc, int cap);
int oracle_detect_keypoints_f64(const uint8_t* luma, int h, int w, int octaves, int scales,
                                double threshold, int upsample, double* out, int cap);
int oracle_detect_keypoints(const float* img, int h, int w, int octaves, int scales,
                            float threshold, int upsample, oracle_keypoint* out, int cap);
int oracle_compute_descriptors(const float* img, int h, int w, const oracle_keypoint* kps, int n,
                               int kind, float* meta, float* desc, int cap);

void oracle_rootsift(const float* desc, float* out);
void oracle_quantize_u8(const float* desc, int n, uint8_t* out);
void oracle_dequantize_u8(const uint8_t* q, int n, float* out);
void oracle_quantize_u128(const float* desc, int n, uint64_t* out);

int oracle_match_descriptors(const float* qd, int nq, const float* td, int nt, const float* qxy,
                 const float* txy, float ratio, int mutual, oracle_match* out, int cap);

/* model: a, b, tx, ty, scale, rotation_deg.  Returns inlier count; mask[i] = 1 for inliers. */
int oracle_similarity_ransac(const oracle_match* m, int n, float thr, uint64_t seed,
                             uint8_t* inlier_mask, float* model, int* has_model);
int oracle_homography_ransac(const oracle_match* m, int n, float thr, uint64_t sim_seed,
                             uint64_t hom_seed, uint8_t* inlier_mask, float* h9, int* has_h);
/* scales/orientations indexed by the matches' query/target indices. */
void oracle_summarize_tracking(const oracle_match* m, int n, const float* q_scale,
                               const float* q_ori, const float* t_scale, const float* t_ori,
                               oracle_tracking* out);

/* Catalog coarse votes.  codes are 2 x u64 (lo, hi) per signature; entry e owns
 * codes [offsets[e], offsets[e+1]).  mih != 0 selects the multi-index-hashing
 * semantics, else the exhaustive scan. */
void oracle_hamming_votes(const uint64_t* q, int nq, const uint64_t* cat, const int64_t* offsets,
                          int n_entries, int mih, uint32_t* votes);
/* The MIH votes through the reference's inverted tables and seen_stamp walk (src/catalog.rs:291-306, :596-615). */
void oracle_mih_votes_tables(const uint64_t* q, int nq, const uint64_t* cat, const int64_t* offsets, int ne,
                             uint32_t* votes);
/* Per-query top-k nearest codes by (Hamming distance, global index). */
void oracle_hamming_topk(const uint64_t* q, int nq, const uint64_t* cat, int64_t ncat, int k,
                         uint32_t* idx, uint32_t* dist);
/* Exact FP32 L2^2 re-rank of k candidates per query, sorted by (d2, index). */
void oracle_l2_rerank(const float* qd, int nq, const float* cat_desc, const uint32_t* cand, int k,
                      uint32_t* out_idx, float* out_d2);

uint64_t oracle_splitmix64_next(uint64_t* state);

/* estimate_fundamental_ransac_with_options (src/geometry.rs:868-1016): returns the
 * inlier count; mask[i] = 1 for inliers; f9 row-major; iters (optional) the
 * iterations run.  fit_fundamental_8point (:638-665) and sampson_distance_sq
 * (:617-636) for direct checks. */
int oracle_fundamental_ransac(const oracle_match* m, int n, double sampson_threshold, int max_iters,
                              double confidence, uint64_t seed, uint8_t* mask, double* f9, int* has_f,
                              int* iters);
int oracle_fit_fundamental_8point(const oracle_match* m, int n, double* f9);
/* fit_fundamental_7point (:727-806): up to 4 candidates (9 doubles each); returns their number. */
int oracle_fit_fundamental_7point(const oracle_match* m, double* f9s);
double oracle_sampson_distance_sq(const double* f9, double x1, double y1, double x2, double y2);

/* warp_and_stitch (src/visualize.rs:379-483) on RGBA8 images (row strides in
 * bytes): the canvas geometry (out_w, out_h, origin[2]) and, when canvas is not
 * NULL, the out_w x out_h x 4 composite.  0 or a negative error code (-1 singular
 * homography, -2 corner at infinity, -3 non-finite corner, -4 canvas too large). */
int oracle_warp_and_stitch(const uint8_t* q, int qh, int qw, size_t qs, const uint8_t* t, int th, int tw,
                           size_t ts, const float* h9, uint8_t* canvas, int* out_w, int* out_h,
                           double* origin);

/* stitch_panorama (src/stitch.rs:472-948) and its parts. */
typedef struct {
  int octaves, scales;
  float threshold, ratio, ransac_threshold;
  int projection;   /* 0 planar, 1 cylindrical */
  float focal_px;
  int blend;        /* 0 feather, 1 multi-band */
  int levels;
  int exposure_compensation;
  int max_canvas_dim;
  long long max_canvas_pixels;
  int tile_size;
} oracle_panorama_options;

/* warp_image_cylindrical (:166-201): RGBA8 in (row stride in bytes), RGBA8 out (w*4 per row). */
void oracle_warp_cylindrical(const uint8_t* img, int h, int w, size_t stride, float focal_px, uint8_t* out);
/* The registration half of stitch_panorama (:472-788) on n prepared RGBA8 images
 * (tight rows): features, pairwise matching + RANSAC, the largest component, the
 * reference, the maximum spanning tree, exposure gains, the canvas.  Outputs:
 * ref_index, registered[n] (0/1), gains[n], h_to_ref[n*9] (f64, row-major, zero
 * when unregistered), inv[n*9] (f64 inverse of the f32-cast matrix), origin[2],
 * out_w, out_h.  Returns 0 or a negative error: -1 fewer than 2 images, -2 no
 * pair matched, -3 no connected pair, -4 singular registered homography, -5
 * projected corner at infinity, -6 non-finite corner, -7 canvas over the limits. */
int oracle_panorama_register(const uint8_t* const* imgs, const int* hs, const int* ws, int n,
                             const oracle_panorama_options* opt, int* ref_index, uint8_t* registered,
                             float* gains, double* h_to_ref, double* inv, double* origin, int* out_w, int* out_h);
/* The blending half (:790-940): the out_w x out_h RGBA8 canvas of the registered
 * images (tight rows) through their inverse matrices, with their gains. */
void oracle_panorama_composite(const uint8_t* const* imgs, const int* hs, const int* ws, int n,
                               const uint8_t* registered, const float* gains, const double* inv,
                               const double* origin, int out_w, int out_h, int blend, int levels, int tile_size,
                               uint8_t* canvas);
/* solve_exposure_gains (:232-316): pairs are (i, j, n_ij, mean_i, mean_j) as 5 doubles. */
void oracle_solve_exposure_gains(const double* pairs, int n_pairs, int n_images, int ref_idx, double sigma_n,
                                 double sigma_g, float* gains);

#ifdef __cplusplus
}
#endif
#endif
