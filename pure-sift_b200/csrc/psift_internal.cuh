// Internal declarations shared by the libpsift_gpu translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <map>
#include <string>
#include <vector>

#include "psift_gpu.h"

namespace psift {

constexpr float kBaseSigma = 1.6f;          // BASE_SIGMA, src/pipeline.rs:10
constexpr float kAssumedInputSigma = 0.5f;  // ASSUMED_INPUT_SIGMA, src/pipeline.rs:13
constexpr float kPiF = 3.14159265358979323846f;
constexpr int kDescLen = 128;
constexpr int kMaxOctaves = 8;
constexpr int kMaxTaps = 32;                // radius <= 15 (largest used: 10)

// Grows-only device arena: one cudaMalloc, bump sub-allocation per call.
struct DeviceArena {
  char* base = nullptr;
  size_t capacity = 0;
  size_t offset = 0;
};

// Pinned host staging used for host<->device transfers of the host-pointer API.
struct PinnedBuffer {
  char* base = nullptr;
  size_t capacity = 0;
};

}  // namespace psift

namespace psift {
// Stages timed by the optional per-stage CUDA-event timer.
enum Stage : int {
  STAGE_PYRAMID = 0,     // octave base + blur/DoG levels
  STAGE_EXTREMA = 1,     // mark + scan + emit
  STAGE_SELECT = 2,      // top-K cap
  STAGE_ORIENTATION = 3,
  STAGE_DESCRIPTOR = 4,  // feature scan + descriptors
  STAGE_MATCH = 5,
  STAGE_HAMMING = 6,
  STAGE_RANSAC = 7,
  STAGE_MLP = 8,
  STAGE_COUNT = 16
};
struct StageTimer {
  bool enabled = false;
  std::vector<cudaEvent_t> pool;                    // free events
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  double ms[STAGE_COUNT] = {0};
  uint64_t count[STAGE_COUNT] = {0};
};
}  // namespace psift

struct psift_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // Second stream for the host-pointer batch entry (chunks of a batch overlap
  // their uploads and downloads with the other chunk's kernels), and the events
  // that fork it from and join it back to `stream`.
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::string last_error;
  uint64_t launches = 0;
  psift::DeviceArena arena;   // per-call workspace
  psift::DeviceArena io;      // device copies of host-pointer inputs/outputs
  psift::DeviceArena stitch;  // panorama: images, features, matches (held across the entries it calls)
  psift::PinnedBuffer pinned;
  int num_sms = 148;
  // Device status words: [0] error bits (kErr* below), [1] re-rank fallback rows.
  uint32_t* d_error = nullptr;
  psift::StageTimer timer;
  // CUDA graphs of the device batch path, keyed by launch geometry: a key seen
  // once runs eagerly, the second time it is captured, afterwards replayed.
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    uint64_t launches = 0;
  };
  // Tile shapes chosen by the autotuner (psift_ctx_autotune, tune.cu): the
  // level-blur variant per radius and the matchers' work items per SM (FP32,
  // tensor-core path).  gen changes with them (part of the graph cache key).
  struct Tuning {
    int8_t blur[16] = {0};
    int8_t match_per_sm[2] = {2, 1};
    uint32_t gen = 0;
  } tune;
  // Single-rounding blur mode (psift_ctx_set_blur_rounding); part of the graph
  // cache key through tune.gen.
  bool blur_fused = false;
  bool graphs_enabled = true;
  std::map<std::string, GraphEntry> graphs;
  std::map<std::string, int> graph_seen;
  uint64_t graph_replays = 0;
  // nvJPEG decoder of the JPEG entries (decode.cu), created on first use.
  void* jpeg = nullptr;
  // PNG decoder state (png.cu): staging buffers, created on first use.
  void* png = nullptr;
};

namespace psift {

// Device error-word bits.
constexpr uint32_t kErrKeypointCapacity = 1u;
constexpr uint32_t kErrSortCapacity = 2u;
constexpr uint32_t kErrTimeout = 4u;

psift_status set_error(psift_ctx* ctx, psift_status st, const std::string& msg);
psift_status cuda_error(psift_ctx* ctx, cudaError_t e, const char* what);
// Ensure the arena can hold `bytes`; resets the bump pointer.  Synchronises the
// stream before reallocating.
psift_status arena_reserve(psift_ctx* ctx, size_t bytes);
// Bump-allocate (256-byte aligned).  Caller must have reserved enough.
void* arena_alloc(psift_ctx* ctx, size_t bytes);
psift_status pinned_reserve(psift_ctx* ctx, size_t bytes);
// Grow-only device buffer for the host-pointer entry points' inputs/outputs.
psift_status io_reserve(psift_ctx* ctx, size_t bytes);
// Grow-only device buffer of the panorama entries (not used by the entries they call).
psift_status stitch_reserve(psift_ctx* ctx, size_t bytes);
inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }
// Raise a kernel's dynamic shared-memory limit once per (kernel, device).
cudaError_t ensure_smem_attr(const void* func, size_t bytes);
// Autotuner of the matchers' work decomposition (match_api.cu); appends
// (path, ms per candidate, chosen) per path to report.
psift_status autotune_match(psift_ctx* ctx, uint32_t n_desc, uint32_t n_pairs, std::vector<double>& report);
// Statistics of summarize_tracking over the masked matches (ransac_api.cu).
void tracking_stats(const psift_match* m, uint32_t n, const uint8_t* mask, const float* q_scale,
                    const float* q_ori, const float* t_scale, const float* t_ori, psift_tracking_summary* out);
// CTAs of `func` resident on the whole device at once (occupancy x SMs), cached.
cudaError_t resident_ctas(const void* func, int threads, size_t smem, int* out);
// Writes the u8 inputs of images [b, e) of the batch into their device slots
// (extra + dev_off[i], dense rows of the image's width) on stream st, the stream
// that then runs those images' stages; called once per chunk, just before it.
using DeviceFill = std::function<psift_status(char* extra, const std::vector<size_t>& dev_off, uint32_t b,
                                              uint32_t e, cudaStream_t st)>;
psift_status detect_batch_host_out(psift_ctx* ctx, const psift_image_u8* images, uint32_t n,
                                   const psift_sift_config* cfg, psift_features* outs, const DeviceFill* fill);
void jpeg_release(psift_ctx* ctx);
void png_release(psift_ctx* ctx);
// The reference's size checks of a decoded image's header (decode.cu).
psift_status check_image_dims(psift_ctx* ctx, uint32_t w, uint32_t h, bool enforce_cap);

// Stage timing: `StageScope sc(ctx, STAGE_X);` records events around the launches
// issued while it is alive (no-op unless timing is enabled).
struct StageScope {
  psift_ctx* ctx;
  int stage;
  cudaStream_t st;
  cudaEvent_t start = nullptr;
  StageScope(psift_ctx* c, int s);
  StageScope(psift_ctx* c, int s, cudaStream_t stream);
  ~StageScope();
};

#define PSIFT_CUDA_TRY(ctx, expr)                                   \
  do {                                                              \
    cudaError_t _e = (expr);                                        \
    if (_e != cudaSuccess) return ::psift::cuda_error(ctx, _e, #expr); \
  } while (0)

#define PSIFT_LAUNCH_CHECK(ctx)                                            \
  do {                                                                     \
    (ctx)->launches++;                                                     \
    cudaError_t _e = cudaGetLastError();                                   \
    if (_e != cudaSuccess) return ::psift::cuda_error(ctx, _e, "kernel launch"); \
  } while (0)

}  // namespace psift
