// Context, error reporting and workspace management for the C ABI.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <map>
#include <tuple>

#include "psift_internal.cuh"

namespace psift {

psift_status set_error(psift_ctx* ctx, psift_status st, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return st;
}

psift_status cuda_error(psift_ctx* ctx, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return set_error(ctx, e == cudaErrorMemoryAllocation ? PSIFT_ERR_OUT_OF_MEMORY : PSIFT_ERR_CUDA, m);
}

psift_status arena_reserve(psift_ctx* ctx, size_t bytes) {
  bytes = align_up(bytes + 4096, 1 << 20);
  if (bytes > ctx->arena.capacity) {
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->arena.base) cudaFree(ctx->arena.base);
    ctx->arena.base = nullptr;
    ctx->arena.capacity = 0;
    cudaError_t e = cudaMalloc(&ctx->arena.base, bytes);
    if (e != cudaSuccess) {
      ctx->arena.base = nullptr;
      return cuda_error(ctx, e, "cudaMalloc(workspace)");
    }
    ctx->arena.capacity = bytes;
  }
  ctx->arena.offset = 0;
  return PSIFT_OK;
}

void* arena_alloc(psift_ctx* ctx, size_t bytes) {
  size_t off = align_up(ctx->arena.offset, 256);
  if (off + bytes > ctx->arena.capacity) return nullptr;
  ctx->arena.offset = off + bytes;
  return ctx->arena.base + off;
}

cudaError_t resident_ctas(const void* func, int threads, size_t smem, int* out) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, int, size_t>, int> cache;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_tuple(func, dev, threads, smem);
  auto it = cache.find(key);
  if (it != cache.end()) {
    *out = it->second;
    return cudaSuccess;
  }
  int per_sm = 0, sms = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, threads, smem);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  *out = cache[key] = per_sm * sms;
  return cudaSuccess;
}

cudaError_t ensure_smem_attr(const void* func, size_t bytes) {
  // The attribute is an upper bound: only ever raise it (a lower value set for a
  // small launch would make a later, larger launch fail).
  // Static plus dynamic shared memory above 48 KB needs the opt-in.
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> limit;
  if (bytes == 0) return cudaSuccess;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  auto it = limit.find({func, dev});
  if (it != limit.end() && it->second >= bytes) return cudaSuccess;
  cudaFuncAttributes fa;
  e = cudaFuncGetAttributes(&fa, func);
  if (e != cudaSuccess) return e;
  if (fa.sharedSizeBytes + bytes <= 48 * 1024) {
    limit[{func, dev}] = bytes;
    return cudaSuccess;
  }
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) limit[{func, dev}] = bytes;
  return e;
}

static cudaEvent_t take_event(psift_ctx* ctx) {
  if (!ctx->timer.pool.empty()) {
    cudaEvent_t e = ctx->timer.pool.back();
    ctx->timer.pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

StageScope::StageScope(psift_ctx* c, int s) : StageScope(c, s, c ? c->stream : nullptr) {}

StageScope::StageScope(psift_ctx* c, int s, cudaStream_t stream) : ctx(c), stage(s), st(stream) {
  if (ctx && ctx->timer.enabled) {
    start = take_event(ctx);
    cudaEventRecord(start, st);
  }
}

StageScope::~StageScope() {
  if (start) {
    cudaEvent_t end = take_event(ctx);
    cudaEventRecord(end, st);
    ctx->timer.pending.push_back({stage, {start, end}});
  }
}

static void drain_timer(psift_ctx* ctx) {
  if (ctx->timer.pending.empty()) return;
  cudaStreamSynchronize(ctx->stream);
  cudaStreamSynchronize(ctx->stream2);
  for (auto& p : ctx->timer.pending) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, p.second.first, p.second.second) == cudaSuccess) {
      ctx->timer.ms[p.first] += ms;
      ctx->timer.count[p.first] += 1;
    }
    ctx->timer.pool.push_back(p.second.first);
    ctx->timer.pool.push_back(p.second.second);
  }
  ctx->timer.pending.clear();
}

psift_status io_reserve(psift_ctx* ctx, size_t bytes) {
  bytes = align_up(bytes + 4096, 1 << 20);
  if (bytes > ctx->io.capacity) {
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->io.base) cudaFree(ctx->io.base);
    ctx->io.base = nullptr;
    ctx->io.capacity = 0;
    cudaError_t e = cudaMalloc(&ctx->io.base, bytes);
    if (e != cudaSuccess) {
      ctx->io.base = nullptr;
      return cuda_error(ctx, e, "cudaMalloc(io)");
    }
    ctx->io.capacity = bytes;
  }
  ctx->io.offset = 0;
  return PSIFT_OK;
}

psift_status stitch_reserve(psift_ctx* ctx, size_t bytes) {
  bytes = align_up(bytes + 4096, 1 << 20);
  if (bytes > ctx->stitch.capacity) {
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->stitch.base) cudaFree(ctx->stitch.base);
    ctx->stitch.base = nullptr;
    ctx->stitch.capacity = 0;
    cudaError_t e = cudaMalloc(&ctx->stitch.base, bytes);
    if (e != cudaSuccess) {
      ctx->stitch.base = nullptr;
      return cuda_error(ctx, e, "cudaMalloc(panorama)");
    }
    ctx->stitch.capacity = bytes;
  }
  ctx->stitch.offset = 0;
  return PSIFT_OK;
}

psift_status pinned_reserve(psift_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->pinned.capacity) return PSIFT_OK;
  bytes = align_up(bytes, 1 << 20);
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->pinned.base) cudaFreeHost(ctx->pinned.base);
  ctx->pinned.base = nullptr;
  ctx->pinned.capacity = 0;
  cudaError_t e = cudaMallocHost(&ctx->pinned.base, bytes);
  if (e != cudaSuccess) {
    ctx->pinned.base = nullptr;
    return cuda_error(ctx, e, "cudaMallocHost(staging)");
  }
  ctx->pinned.capacity = bytes;
  return PSIFT_OK;
}

}  // namespace psift

extern "C" {

psift_status psift_ctx_create(int device, psift_ctx** out) {
  if (!out) return PSIFT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return PSIFT_ERR_NO_DEVICE;
  if (device < 0 || device >= n) return PSIFT_ERR_INVALID_ARGUMENT;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return PSIFT_ERR_NO_DEVICE;
  if (prop.major < 10) return PSIFT_ERR_NO_DEVICE;  // built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return PSIFT_ERR_NO_DEVICE;
  psift_ctx* ctx = new psift_ctx();
  ctx->device = device;
  ctx->num_sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return PSIFT_ERR_CUDA;
  }
  if (cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return PSIFT_ERR_CUDA;
  }
  if (cudaMalloc(&ctx->d_error, 64) != cudaSuccess || cudaMemset(ctx->d_error, 0, 64) != cudaSuccess) {
    cudaStreamDestroy(ctx->stream2);
    cudaEventDestroy(ctx->ev_fork);
    cudaEventDestroy(ctx->ev_join);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return PSIFT_ERR_OUT_OF_MEMORY;
  }
  *out = ctx;
  return PSIFT_OK;
}

psift_status psift_ctx_destroy(psift_ctx* ctx) {
  if (!ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaStreamSynchronize(ctx->stream2);
  if (ctx->arena.base) cudaFree(ctx->arena.base);
  if (ctx->io.base) cudaFree(ctx->io.base);
  if (ctx->stitch.base) cudaFree(ctx->stitch.base);
  if (ctx->pinned.base) cudaFreeHost(ctx->pinned.base);
  if (ctx->d_error) cudaFree(ctx->d_error);
  psift::jpeg_release(ctx);
  psift::png_release(ctx);
  for (auto& p : ctx->timer.pending) {
    cudaEventDestroy(p.second.first);
    cudaEventDestroy(p.second.second);
  }
  for (cudaEvent_t e : ctx->timer.pool) cudaEventDestroy(e);
  for (auto& g : ctx->graphs)
    if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
  cudaEventDestroy(ctx->ev_fork);
  cudaEventDestroy(ctx->ev_join);
  cudaStreamDestroy(ctx->stream2);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return PSIFT_OK;
}

const char* psift_last_error(const psift_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : "null context";
}

uint64_t psift_ctx_launch_count(const psift_ctx* ctx) { return ctx ? ctx->launches : 0; }

void* psift_ctx_stream(const psift_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

psift_status psift_ctx_synchronize(psift_ctx* ctx) {
  if (!ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PSIFT_OK;
}

psift_status psift_ctx_enable_graphs(psift_ctx* ctx, int enable) {
  if (!ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  ctx->graphs_enabled = enable != 0;
  return PSIFT_OK;
}

uint64_t psift_ctx_graph_replays(const psift_ctx* ctx) { return ctx ? ctx->graph_replays : 0; }


psift_status psift_ctx_enable_stage_timing(psift_ctx* ctx, int enable) {
  if (!ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  ctx->timer.enabled = enable != 0;
  return PSIFT_OK;
}

psift_status psift_ctx_stage_times(psift_ctx* ctx, double* ms, uint64_t* counts, uint32_t n, int reset) {
  if (!ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  psift::drain_timer(ctx);
  for (uint32_t i = 0; i < n && i < psift::STAGE_COUNT; ++i) {
    if (ms) ms[i] = ctx->timer.ms[i];
    if (counts) counts[i] = ctx->timer.count[i];
  }
  if (reset) {
    for (int i = 0; i < psift::STAGE_COUNT; ++i) {
      ctx->timer.ms[i] = 0.0;
      ctx->timer.count[i] = 0;
    }
  }
  return PSIFT_OK;
}

void psift_sift_config_default(psift_sift_config* cfg) {
  if (!cfg) return;
  cfg->octaves = 3;
  cfg->scales = 3;
  cfg->contrast_threshold = 0.015f;
  cfg->upsample_first_octave = 1;
  cfg->descriptor_kind = 0;
  cfg->max_features = PSIFT_MAX_FEATURES_PER_IMAGE;
}

// SiftConfig::validate, src/pipeline.rs:80-103 (same messages).
psift_status psift_sift_config_validate(const psift_sift_config* cfg, char* msg, size_t cap) {
  char buf[256] = {0};
  psift_status st = PSIFT_OK;
  if (!cfg) {
    snprintf(buf, sizeof buf, "null config");
    st = PSIFT_ERR_INVALID_ARGUMENT;
  } else if (cfg->octaves < 1 || cfg->octaves > 8) {
    snprintf(buf, sizeof buf, "Invalid `octaves`=%u: must be between 1 and 8", cfg->octaves);
    st = PSIFT_ERR_INVALID_CONFIG;
  } else if (cfg->scales < 3 || cfg->scales > 10) {
    snprintf(buf, sizeof buf,
             "Invalid `scales`=%u: must be between 3 and 10 for 3D extrema extraction", cfg->scales);
    st = PSIFT_ERR_INVALID_CONFIG;
  } else if (!(cfg->contrast_threshold == cfg->contrast_threshold) ||
             cfg->contrast_threshold > 3.4e38f || cfg->contrast_threshold <= 0.0f ||
             cfg->contrast_threshold > 1.0f) {
    snprintf(buf, sizeof buf, "Invalid `contrast_threshold`=%g: must be finite and in (0.0, 1.0]",
             (double)cfg->contrast_threshold);
    st = PSIFT_ERR_INVALID_CONFIG;
  } else if (cfg->descriptor_kind != 0 && cfg->descriptor_kind != 1) {
    snprintf(buf, sizeof buf, "Invalid `descriptor_kind`=%d: must be 0 (Sift) or 1 (RootSift)",
             cfg->descriptor_kind);
    st = PSIFT_ERR_INVALID_CONFIG;
  } else if (cfg->max_features > 16384) {
    snprintf(buf, sizeof buf, "Invalid `max_features`=%u: must be 0 (uncapped) or at most 16384",
             cfg->max_features);
    st = PSIFT_ERR_INVALID_CONFIG;
  }
  if (msg && cap) {
    strncpy(msg, buf, cap - 1);
    msg[cap - 1] = 0;
  }
  return st;
}

}  // extern "C"
