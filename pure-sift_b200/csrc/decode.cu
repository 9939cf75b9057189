// Input step of the extract path: JPEG bytes -> u8 luma in device memory -> features.
//
// Reference: decode_validated_dynamic_image / decode_validated_luma8
// (src/cli.rs:129-170): the header's size is checked (MIN_IMAGE_DIM, and
// MAX_IMAGE_DIM / MAX_IMAGE_PIXELS when the pixel cap is enforced, :46-48), the
// bytes are decoded by the image crate (0.25.10) and converted by
// DynamicImage::into_luma8.  For RGB the crate's rgb_to_luma computes, in u32,
// (2126 R + 7152 G + 722 B) / 10000 with truncation (Rec. 709 weights); a
// grayscale JPEG's plane is its luma, and (w R + w G + w B) / 10000 of a gray
// pixel returns it unchanged, so one conversion serves both.
//
// Here the JPEG is decoded on the GPU by nvJPEG into interleaved RGB — with the
// hardware backend (the B200's JPEG engines) when it is present and accepts the
// batch, else with its GPU-assisted backend — and rgb_to_luma_kernel writes the
// luma straight into the detection batch's input slots.  nvJPEG is loaded with
// dlopen on first use: the library loads without it, and these entries then
// report PSIFT_ERR_INTERNAL.  The decoded pixels come from nvJPEG's IDCT and
// chroma upsampling, not the image crate's decoder, so they can differ from the
// reference's by a few levels; the luma conversion itself is exact.  PNG stays
// on the host (inflate and the row filters are sequential).
#include <dlfcn.h>
#include <nvjpeg.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "psift_internal.cuh"

namespace psift {
namespace {


struct NvjpegApi {
  bool tried = false, ok = false;
  void* lib = nullptr;
  decltype(&nvjpegCreateEx) create_ex = nullptr;
  decltype(&nvjpegDestroy) destroy = nullptr;
  decltype(&nvjpegJpegStateCreate) state_create = nullptr;
  decltype(&nvjpegJpegStateDestroy) state_destroy = nullptr;
  decltype(&nvjpegGetImageInfo) image_info = nullptr;
  decltype(&nvjpegDecodeBatchedInitialize) batched_init = nullptr;
  decltype(&nvjpegDecodeBatched) batched = nullptr;
};

NvjpegApi& nvjpeg() {
  static NvjpegApi a;
  static std::mutex m;
  std::lock_guard<std::mutex> lock(m);
  if (a.tried) return a;
  a.tried = true;
  for (const char* name : {"libnvjpeg.so.12", "libnvjpeg.so"}) {
    a.lib = dlopen(name, RTLD_NOW | RTLD_LOCAL);
    if (a.lib) break;
  }
  if (!a.lib) return a;
  bool ok = true;
  auto sym = [&](auto& fp, const char* name) {
    fp = reinterpret_cast<std::remove_reference_t<decltype(fp)>>(dlsym(a.lib, name));
    ok = ok && fp != nullptr;
  };
  sym(a.create_ex, "nvjpegCreateEx");
  sym(a.destroy, "nvjpegDestroy");
  sym(a.state_create, "nvjpegJpegStateCreate");
  sym(a.state_destroy, "nvjpegJpegStateDestroy");
  sym(a.image_info, "nvjpegGetImageInfo");
  sym(a.batched_init, "nvjpegDecodeBatchedInitialize");
  sym(a.batched, "nvjpegDecodeBatched");
  a.ok = ok;
  return a;
}

struct Backend {
  nvjpegBackend_t kind;
  nvjpegHandle_t h = nullptr;
  nvjpegJpegState_t st = nullptr;
  int batch = 0;        // batch size the state is initialised for
  bool unusable = false;
  explicit Backend(nvjpegBackend_t k) : kind(k) {}
};

// Per context: the hardware backend, the GPU-assisted one (created when the
// hardware one is missing or refuses a batch), the RGB staging buffer.
// A host thread's share of a batch: its own handle and state (only the header
// query is documented thread-safe), CUDA stream and completion event.
struct Worker {
  Backend b{NVJPEG_BACKEND_HYBRID};
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  nvjpegStatus_t status = NVJPEG_STATUS_SUCCESS;
};

struct Decoder {
  Backend hw{NVJPEG_BACKEND_HARDWARE};
  Backend gpu{NVJPEG_BACKEND_GPU_HYBRID};
  std::vector<Worker> workers;
  cudaEvent_t start = nullptr;
  cudaEvent_t all_done = nullptr;  // the whole batch decoded with chunk 0
  int threads = 0;  // 0: automatic; 1: one batched call on the calling thread
  uint8_t* rgb = nullptr;
  size_t rgb_cap = 0;
  int last = -1;  // backend of the last successful batch
};

Decoder* decoder(psift_ctx* ctx) {
  if (!ctx->jpeg) ctx->jpeg = new Decoder;
  return static_cast<Decoder*>(ctx->jpeg);
}

bool backend_ready(Backend& b) {
  if (b.unusable) return false;
  if (b.h) return true;
  NvjpegApi& A = nvjpeg();
  if (A.create_ex(b.kind, nullptr, nullptr, 0, &b.h) != NVJPEG_STATUS_SUCCESS) {
    b.h = nullptr;
    b.unusable = true;
    return false;
  }
  if (A.state_create(b.h, &b.st) != NVJPEG_STATUS_SUCCESS) {
    A.destroy(b.h);
    b.h = nullptr;
    b.unusable = true;
    return false;
  }
  return true;
}

void backend_release(Backend& b) {
  NvjpegApi& A = nvjpeg();
  if (b.st) A.state_destroy(b.st);
  if (b.h) A.destroy(b.h);
  b.st = nullptr;
  b.h = nullptr;
}

constexpr int kMaxJpegThreads = 16;
constexpr uint32_t kWorkerBatchMax = 50;  // the hybrid stage stays on the host up to 50 images

bool worker_ready(psift_ctx* ctx, Worker& w) {
  if (!backend_ready(w.b)) return false;
  if (!w.stream && cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking) != cudaSuccess) {
    w.stream = nullptr;
    return false;
  }
  if (!w.done && cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming) != cudaSuccess) {
    w.done = nullptr;
    return false;
  }
  (void)ctx;
  return true;
}

// Decodes images [b, e) of the batch with worker w: the Huffman stage on this
// host thread, the rest on w.stream; w.done is recorded after it.
void worker_decode(const psift_ctx* ctx, Worker& w, const uint8_t* const* data, const size_t* lengths,
                   nvjpegImage_t* dst, uint32_t b, uint32_t e) {
  NvjpegApi& A = nvjpeg();
  w.status = NVJPEG_STATUS_SUCCESS;
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    w.status = NVJPEG_STATUS_EXECUTION_FAILED;
    return;
  }
  const int n = (int)(e - b);
  if (w.b.batch != n) {
    w.status = A.batched_init(w.b.h, w.b.st, n, 1, NVJPEG_OUTPUT_RGBI);
    if (w.status != NVJPEG_STATUS_SUCCESS) return;
    w.b.batch = n;
  }
  w.status = A.batched(w.b.h, w.b.st, data + b, lengths + b, dst + b, w.stream);
  if (w.status == NVJPEG_STATUS_SUCCESS && cudaEventRecord(w.done, w.stream) != cudaSuccess)
    w.status = NVJPEG_STATUS_EXECUTION_FAILED;
}

// The batch over T host threads (the calling one included), contiguous shares.
// Returns false when the workers cannot be set up or one of them failed.
bool decode_threaded(psift_ctx* ctx, Decoder* dec, const uint8_t* const* data, const size_t* lengths, uint32_t n,
                     nvjpegImage_t* dst, cudaStream_t st) {
  const unsigned hc = std::max(1u, std::thread::hardware_concurrency());
  int T = dec->threads > 1 ? dec->threads : (int)std::min<unsigned>(hc, kMaxJpegThreads);
  T = std::max(1, std::min<int>(T, (int)n));
  while ((n + T - 1) / T > kWorkerBatchMax && T < (int)n) ++T;
  if ((int)dec->workers.size() < T) dec->workers.resize(T);
  for (int t = 0; t < T; ++t)
    if (!worker_ready(ctx, dec->workers[t])) return false;
  if (!dec->start && cudaEventCreateWithFlags(&dec->start, cudaEventDisableTiming) != cudaSuccess) return false;
  // The RGB staging buffer is free once the work queued before on st is done.
  if (cudaEventRecord(dec->start, st) != cudaSuccess) return false;
  for (int t = 0; t < T; ++t)
    if (cudaStreamWaitEvent(dec->workers[t].stream, dec->start, 0) != cudaSuccess) return false;
  std::vector<std::thread> pool;
  const uint32_t per = n / T, extra = n % T;
  uint32_t b = 0;
  std::vector<std::pair<uint32_t, uint32_t>> range(T);
  for (int t = 0; t < T; ++t) {
    const uint32_t e = b + per + ((uint32_t)t < extra ? 1 : 0);
    range[t] = {b, e};
    b = e;
  }
  for (int t = 1; t < T; ++t) {
    try {
      pool.emplace_back(worker_decode, ctx, std::ref(dec->workers[t]), data, lengths, dst, range[t].first,
                        range[t].second);
    } catch (...) {  // no thread available: this share runs on the calling thread
      worker_decode(ctx, dec->workers[t], data, lengths, dst, range[t].first, range[t].second);
    }
  }
  worker_decode(ctx, dec->workers[0], data, lengths, dst, range[0].first, range[0].second);
  for (auto& th : pool) th.join();
  bool ok = true;
  for (int t = 0; t < T; ++t) {
    Worker& w = dec->workers[t];
    if (w.status == NVJPEG_STATUS_SUCCESS) {
      ok = ok && cudaStreamWaitEvent(st, w.done, 0) == cudaSuccess;
    } else {
      ok = false;
      cudaStreamSynchronize(w.stream);  // nothing of a failed share may still write the staging buffer
    }
  }
  return ok;
}


// rgb_to_luma of the image crate for u8 (see the file comment), one pixel per thread.
__global__ void rgb_to_luma_kernel(const uint8_t* __restrict__ rgb, uint8_t* __restrict__ luma, uint32_t n_px) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_px) return;
  const uint32_t r = rgb[3 * (size_t)i], g = rgb[3 * (size_t)i + 1], b = rgb[3 * (size_t)i + 2];
  luma[i] = (uint8_t)((2126u * r + 7152u * g + 722u * b) / 10000u);
}

struct JpegDims {
  uint32_t w = 0, h = 0, comps = 0;
};

// Header read and the reference's size checks (src/cli.rs:137-158).
psift_status read_header(psift_ctx* ctx, const uint8_t* data, size_t len, bool enforce_cap, JpegDims* d) {
  NvjpegApi& A = nvjpeg();
  if (!A.ok) return set_error(ctx, PSIFT_ERR_INTERNAL, "nvJPEG (libnvjpeg.so.12) could not be loaded");
  Decoder* dec = decoder(ctx);
  Backend& b = backend_ready(dec->hw) ? dec->hw : dec->gpu;
  if (!backend_ready(b)) return set_error(ctx, PSIFT_ERR_INTERNAL, "no nvJPEG backend could be created");
  if (!data || len == 0) return set_error(ctx, PSIFT_ERR_FORMAT, "Invalid or unsupported image header: empty buffer");
  int nc = 0, ws[NVJPEG_MAX_COMPONENT] = {0}, hs[NVJPEG_MAX_COMPONENT] = {0};
  nvjpegChromaSubsampling_t sub;
  const nvjpegStatus_t s = A.image_info(b.h, data, len, &nc, &sub, ws, hs);
  if (s != NVJPEG_STATUS_SUCCESS)
    return set_error(ctx, PSIFT_ERR_FORMAT,
                     "Invalid or unsupported image header (nvJPEG status " + std::to_string((int)s) + ")");
  d->w = (uint32_t)ws[0];
  d->h = (uint32_t)hs[0];
  d->comps = (uint32_t)nc;
  return check_image_dims(ctx, d->w, d->h, enforce_cap);
}

// Decodes n JPEGs (host bytes) and writes their luma to luma[i] (dense rows) on st.
// RGB staging offsets of every image of a batch (each image its own region, so
// chunks decoded on different streams never share one); grows the buffer.
psift_status reserve_rgb(psift_ctx* ctx, const std::vector<JpegDims>& dims, std::vector<size_t>& off) {
  Decoder* dec = decoder(ctx);
  off.assign(dims.size(), 0);
  size_t total = 0;
  for (size_t i = 0; i < dims.size(); ++i) {
    off[i] = total;
    total += align_up(3 * (size_t)dims[i].w * dims[i].h, 256);
  }
  if (total > dec->rgb_cap) {
    cudaFree(dec->rgb);  // synchronises the device: no earlier decode still writes it
    dec->rgb = nullptr;
    dec->rgb_cap = 0;
    const size_t cap = align_up(total, 1 << 20);
    cudaError_t e = cudaMalloc(&dec->rgb, cap);
    if (e != cudaSuccess) return cuda_error(ctx, e, "cudaMalloc(jpeg rgb)");
    dec->rgb_cap = cap;
  }
  return PSIFT_OK;
}

// Decodes images [b, e) of the batch (host bytes) and writes their luma to
// luma[i - b] (dense rows) on st.
psift_status decode_range(psift_ctx* ctx, const uint8_t* const* data, const size_t* lengths,
                          const std::vector<JpegDims>& dims, const std::vector<size_t>& off, uint32_t b, uint32_t e,
                          uint8_t* const* luma, cudaStream_t st) {
  NvjpegApi& A = nvjpeg();
  Decoder* dec = decoder(ctx);
  const uint32_t n = e - b;
  std::vector<nvjpegImage_t> dst(n);
  for (uint32_t i = 0; i < n; ++i) {
    std::memset(&dst[i], 0, sizeof(nvjpegImage_t));
    dst[i].channel[0] = dec->rgb + off[b + i];
    dst[i].pitch[0] = 3 * (size_t)dims[b + i].w;
  }
  nvjpegStatus_t s = NVJPEG_STATUS_NOT_INITIALIZED;
  int used = -1;
  if (dec->threads != 1 && decode_threaded(ctx, dec, data + b, lengths + b, n, dst.data(), st)) {
    used = (int)NVJPEG_BACKEND_HYBRID;
    s = NVJPEG_STATUS_SUCCESS;
  }
  for (Backend* bk : {&dec->hw, &dec->gpu}) {
    if (used >= 0) break;
    if (!backend_ready(*bk)) continue;
    if (bk->batch != (int)n) {
      s = A.batched_init(bk->h, bk->st, (int)n, 1, NVJPEG_OUTPUT_RGBI);
      if (s != NVJPEG_STATUS_SUCCESS) continue;
      bk->batch = (int)n;
    }
    s = A.batched(bk->h, bk->st, data + b, lengths + b, dst.data(), st);
    if (s == NVJPEG_STATUS_SUCCESS) {
      used = (int)bk->kind;
      break;
    }
  }
  if (used < 0)
    return set_error(ctx, PSIFT_ERR_FORMAT,
                     "Failed to decode image payload (nvJPEG status " + std::to_string((int)s) + ")");
  dec->last = used;
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t px = dims[b + i].w * dims[b + i].h;
    rgb_to_luma_kernel<<<(px + 255) / 256, 256, 0, st>>>(dec->rgb + off[b + i], luma[i], px);
    ctx->launches++;
  }
  PSIFT_CUDA_TRY(ctx, cudaGetLastError());
  return PSIFT_OK;
}

}  // namespace

// The reference's size checks of a decoded image's header (src/cli.rs:137-158):
// MIN_IMAGE_DIM, and MAX_IMAGE_DIM / MAX_IMAGE_PIXELS when the cap is enforced.
psift_status check_image_dims(psift_ctx* ctx, uint32_t w, uint32_t h, bool enforce_cap) {
  constexpr uint32_t kMinImageDim = 8;            // MIN_IMAGE_DIM, src/cli.rs:46
  constexpr uint32_t kMaxImageDim = 8192;         // MAX_IMAGE_DIM, src/cli.rs:47
  constexpr uint64_t kMaxImagePixels = 25000000;  // MAX_IMAGE_PIXELS, src/cli.rs:48
  if (w < kMinImageDim || h < kMinImageDim)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT,
                     "Image dimensions " + std::to_string(w) + "x" + std::to_string(h) +
                         " are too small (minimum 8x8)");
  const uint64_t total = (uint64_t)w * h;
  if (total > (1ull << 31))
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT,
                     "Image dimensions " + std::to_string(w) + "x" + std::to_string(h) + " exceed 2^31 pixels");
  if (enforce_cap && (w > kMaxImageDim || h > kMaxImageDim || total > kMaxImagePixels))
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT,
                     "Image dimensions " + std::to_string(w) + "x" + std::to_string(h) + " (" +
                         std::to_string(total) + " px) exceed maximum allowed (8192x8192, 25000000 px)");
  return PSIFT_OK;
}

void jpeg_release(psift_ctx* ctx) {
  if (!ctx->jpeg) return;
  Decoder* dec = static_cast<Decoder*>(ctx->jpeg);
  if (nvjpeg().ok) {
    backend_release(dec->hw);
    backend_release(dec->gpu);
    for (Worker& w : dec->workers) backend_release(w.b);
  }
  for (Worker& w : dec->workers) {
    if (w.done) cudaEventDestroy(w.done);
    if (w.stream) cudaStreamDestroy(w.stream);
  }
  if (dec->start) cudaEventDestroy(dec->start);
  if (dec->all_done) cudaEventDestroy(dec->all_done);
  cudaFree(dec->rgb);
  delete dec;
  ctx->jpeg = nullptr;
}

}  // namespace psift

using namespace psift;

extern "C" {

psift_status psift_jpeg_info(psift_ctx* ctx, const uint8_t* data, size_t length, int32_t enforce_pixel_cap,
                             uint32_t* width, uint32_t* height, uint32_t* components) {
  if (!ctx || !width || !height) return PSIFT_ERR_INVALID_ARGUMENT;
  PSIFT_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  JpegDims d;
  psift_status st = read_header(ctx, data, length, enforce_pixel_cap != 0, &d);
  *width = d.w;
  *height = d.h;
  if (components) *components = d.comps;
  return st;
}

psift_status psift_decode_jpeg_luma(psift_ctx* ctx, const uint8_t* data, size_t length, int32_t enforce_pixel_cap,
                                    uint8_t* luma, size_t capacity, uint32_t* width, uint32_t* height) {
  if (!ctx || !width || !height) return PSIFT_ERR_INVALID_ARGUMENT;
  PSIFT_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  std::vector<JpegDims> dims(1);
  psift_status st = read_header(ctx, data, length, enforce_pixel_cap != 0, &dims[0]);
  *width = dims[0].w;
  *height = dims[0].h;
  if (st != PSIFT_OK) return st;
  const size_t px = (size_t)dims[0].w * dims[0].h;
  if (px > capacity) return set_error(ctx, PSIFT_ERR_CAPACITY, "luma output capacity too small");
  if (!luma) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null luma output");
  if ((st = io_reserve(ctx, px)) != PSIFT_OK) return st;
  uint8_t* d_luma = (uint8_t*)ctx->io.base;
  const uint8_t* const bufs[1] = {data};
  const size_t lens[1] = {length};
  uint8_t* const outs[1] = {d_luma};
  std::vector<size_t> off;
  if ((st = reserve_rgb(ctx, dims, off)) != PSIFT_OK) return st;
  if ((st = decode_range(ctx, bufs, lens, dims, off, 0, 1, outs, ctx->stream)) != PSIFT_OK) return st;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(luma, d_luma, px, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PSIFT_OK;
}

psift_status psift_detect_and_compute_jpeg_batch(psift_ctx* ctx, const uint8_t* const* data, const size_t* lengths,
                                                 uint32_t n, int32_t enforce_pixel_cap,
                                                 const psift_sift_config* cfg, psift_features* outs) {
  if (!ctx || !data || !lengths || !outs || n == 0) return PSIFT_ERR_INVALID_ARGUMENT;
  PSIFT_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  std::vector<JpegDims> dims(n);
  std::vector<psift_image_u8> imgs(n);
  for (uint32_t i = 0; i < n; ++i) {
    const psift_status st = read_header(ctx, data[i], lengths[i], enforce_pixel_cap != 0, &dims[i]);
    if (st != PSIFT_OK) return st;
    imgs[i] = psift_image_u8{nullptr, dims[i].h, dims[i].w, dims[i].w};
  }
  std::vector<size_t> rgb_off;
  psift_status rs = reserve_rgb(ctx, dims, rgb_off);
  if (rs != PSIFT_OK) return rs;
  Decoder* dec = decoder(ctx);
  if (!dec->all_done && cudaEventCreateWithFlags(&dec->all_done, cudaEventDisableTiming) != cudaSuccess)
    return set_error(ctx, PSIFT_ERR_CUDA, "cudaEventCreate(jpeg)");
  // Per chunk: its images decoded on its stream, so that the host part of chunk
  // 1's decode overlaps chunk 0's kernels -- when a chunk has at least as many
  // images as there are decode threads (fewer would leave threads idle for longer
  // than the overlap gains).  Otherwise, and for one batched call (threads = 1;
  // above 50 images its Huffman stage then runs on the GPU), chunk 0 decodes the
  // whole batch and chunk 1's stream waits for it.
  const unsigned hc = std::max(1u, std::thread::hardware_concurrency());
  const uint32_t decode_threads = dec->threads > 1 ? (uint32_t)dec->threads : std::min<unsigned>(hc, kMaxJpegThreads);
  const bool whole = dec->threads == 1 || (n + 1) / 2 < decode_threads;
  const DeviceFill fill = [&](char* extra, const std::vector<size_t>& dev_off, uint32_t b, uint32_t e,
                              cudaStream_t st) -> psift_status {
    if (whole) {
      if (b > 0) return cudaStreamWaitEvent(st, dec->all_done, 0) == cudaSuccess
                            ? PSIFT_OK
                            : set_error(ctx, PSIFT_ERR_CUDA, "cudaStreamWaitEvent(jpeg)");
      b = 0;
      e = n;
    }
    std::vector<uint8_t*> luma(e - b);
    for (uint32_t i = b; i < e; ++i) luma[i - b] = (uint8_t*)extra + dev_off[i];
    psift_status r = decode_range(ctx, data, lengths, dims, rgb_off, b, e, luma.data(), st);
    if (r == PSIFT_OK && whole && cudaEventRecord(dec->all_done, st) != cudaSuccess)
      r = set_error(ctx, PSIFT_ERR_CUDA, "cudaEventRecord(jpeg)");
    return r;
  };
  return detect_batch_host_out(ctx, imgs.data(), n, cfg, outs, &fill);
}

psift_status psift_ctx_set_jpeg_threads(psift_ctx* ctx, int32_t threads) {
  if (!ctx || threads < 0 || threads > 256) return PSIFT_ERR_INVALID_ARGUMENT;
  decoder(ctx)->threads = threads;
  return PSIFT_OK;
}

psift_status psift_ctx_jpeg_backend(psift_ctx* ctx, int32_t* backend) {
  if (!ctx || !backend) return PSIFT_ERR_INVALID_ARGUMENT;
  *backend = ctx->jpeg ? static_cast<Decoder*>(ctx->jpeg)->last : -1;
  return PSIFT_OK;
}

}  // extern "C"
