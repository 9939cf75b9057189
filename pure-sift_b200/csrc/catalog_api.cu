// C-ABI entry points of the descriptor quantisers and the catalog Hamming stages.
//
// Reference: quantize_descriptor_u128 (src/catalog.rs:37-45), coarse voting of
// FeatureCatalog::search_features (src/catalog.rs:588-641, :707-728),
// quantize_descriptor_u8 / dequantize_descriptor_u8 (src/pipeline.rs:1024-1044).
#include <algorithm>
#include <cstring>

#include "psift_internal.cuh"

namespace psift {

cudaError_t launch_quantize(const float* desc, int n, uint64_t* codes, uint8_t* u8, cudaStream_t st);
cudaError_t launch_popc_probe(int blocks, int iters, uint32_t* out, cudaStream_t st);
cudaError_t launch_dequantize(const uint8_t* q, int n, float* out, cudaStream_t st);
cudaError_t launch_votes(const uint64_t* q, int nq, const uint64_t* cat, const long long* offsets, int n_entries,
                         int mih, uint32_t* votes, cudaStream_t st);
int topk_chunks(long long ncat, int nq, int num_sms);
cudaError_t launch_topk(const uint64_t* q, int nq, const uint64_t* cat, long long ncat, int k, int n_chunks,
                        unsigned long long* part, uint32_t* out_idx, uint32_t* out_dist, cudaStream_t st);
cudaError_t launch_l2_rerank(const float* qd, int nq, const float* cd, const uint32_t* cand, int k,
                             uint32_t* out_idx, float* out_d2, cudaStream_t st);

namespace {

psift_status begin(psift_ctx* ctx) {
  if (!ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(ctx, e, "cudaSetDevice");
  return PSIFT_OK;
}

// Bump-carve in the io arena (already reserved).
void* io_take(psift_ctx* ctx, size_t bytes) {
  const size_t off = align_up(ctx->io.offset, 256);
  if (off + bytes > ctx->io.capacity) return nullptr;
  ctx->io.offset = off + bytes;
  return ctx->io.base + off;
}

psift_status h2d(psift_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (bytes) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return PSIFT_OK;
}

psift_status d2h_sync(psift_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (bytes) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PSIFT_OK;
}

}  // namespace
}  // namespace psift

using namespace psift;

extern "C" {

psift_status psift_quantize_u128(psift_ctx* ctx, const float* desc, uint32_t n, uint64_t* codes) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (n == 0) return PSIFT_OK;
  if (!desc || !codes) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  st = io_reserve(ctx, (size_t)n * (512 + 16) + 1024);
  if (st != PSIFT_OK) return st;
  float* d_desc = (float*)io_take(ctx, (size_t)n * 512);
  uint64_t* d_codes = (uint64_t*)io_take(ctx, (size_t)n * 16);
  if ((st = h2d(ctx, d_desc, desc, (size_t)n * 512)) != PSIFT_OK) return st;
  cudaError_t e = launch_quantize(d_desc, (int)n, d_codes, nullptr, ctx->stream);
  ctx->launches++;
  if (e != cudaSuccess) return cuda_error(ctx, e, "quantize");
  return d2h_sync(ctx, codes, d_codes, (size_t)n * 16);
}

psift_status psift_quantize_u128_dev(psift_ctx* ctx, const float* desc, uint32_t n, uint64_t* codes) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (n == 0) return PSIFT_OK;
  if (!desc || !codes) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  StageScope sc(ctx, STAGE_HAMMING);
  cudaError_t e = launch_quantize(desc, (int)n, codes, nullptr, ctx->stream);
  ctx->launches++;
  if (e != cudaSuccess) return cuda_error(ctx, e, "quantize");
  return PSIFT_OK;
}

psift_status psift_popc_throughput(psift_ctx* ctx, double* popc_per_s) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (!popc_per_s) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  const int blocks = ctx->num_sms * 8, iters = 4096;
  st = io_reserve(ctx, (size_t)blocks * 256 * 4 + 1024);
  if (st != PSIFT_OK) return st;
  uint32_t* d_out = (uint32_t*)io_take(ctx, (size_t)blocks * 256 * 4);
  cudaEvent_t a = nullptr, b = nullptr;
  PSIFT_CUDA_TRY(ctx, cudaEventCreate(&a));
  PSIFT_CUDA_TRY(ctx, cudaEventCreate(&b));
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(a, ctx->stream);
    cudaError_t e = launch_popc_probe(blocks, iters, d_out, ctx->stream);
    cudaEventRecord(b, ctx->stream);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "popc probe");
    PSIFT_CUDA_TRY(ctx, cudaEventSynchronize(b));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    if (rep > 0) best = std::min(best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *popc_per_s = (double)blocks * 256.0 * iters * 8.0 / (best * 1e-3);
  return PSIFT_OK;
}

psift_status psift_quantize_u8(psift_ctx* ctx, const float* desc, uint32_t n, uint8_t* out) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (n == 0) return PSIFT_OK;
  if (!desc || !out) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  st = io_reserve(ctx, (size_t)n * (512 + 128) + 1024);
  if (st != PSIFT_OK) return st;
  float* d_desc = (float*)io_take(ctx, (size_t)n * 512);
  uint8_t* d_u8 = (uint8_t*)io_take(ctx, (size_t)n * 128);
  if ((st = h2d(ctx, d_desc, desc, (size_t)n * 512)) != PSIFT_OK) return st;
  cudaError_t e = launch_quantize(d_desc, (int)n, nullptr, d_u8, ctx->stream);
  ctx->launches++;
  if (e != cudaSuccess) return cuda_error(ctx, e, "quantize_u8");
  return d2h_sync(ctx, out, d_u8, (size_t)n * 128);
}

psift_status psift_dequantize_u8(psift_ctx* ctx, const uint8_t* q, uint32_t n, float* out) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (n == 0) return PSIFT_OK;
  if (!q || !out) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  st = io_reserve(ctx, (size_t)n * (512 + 128) + 1024);
  if (st != PSIFT_OK) return st;
  uint8_t* d_q = (uint8_t*)io_take(ctx, (size_t)n * 128);
  float* d_out = (float*)io_take(ctx, (size_t)n * 512);
  if ((st = h2d(ctx, d_q, q, (size_t)n * 128)) != PSIFT_OK) return st;
  cudaError_t e = launch_dequantize(d_q, (int)n, d_out, ctx->stream);
  ctx->launches++;
  if (e != cudaSuccess) return cuda_error(ctx, e, "dequantize_u8");
  return d2h_sync(ctx, out, d_out, (size_t)n * 512);
}

psift_status psift_hamming_votes(psift_ctx* ctx, const uint64_t* q_codes, uint32_t nq, const uint64_t* cat_codes,
                                 const int64_t* entry_offsets, uint32_t n_entries, int32_t mih, uint32_t* votes) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (n_entries == 0) return PSIFT_OK;
  if (!entry_offsets || !votes || (nq && !q_codes)) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  const int64_t ncat = entry_offsets[n_entries];
  for (uint32_t e = 0; e < n_entries; ++e)
    if (entry_offsets[e] < 0 || entry_offsets[e] > entry_offsets[e + 1])
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "entry offsets must be non-decreasing from 0");
  if (ncat && !cat_codes) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null catalog codes");
  st = io_reserve(ctx, (size_t)nq * 16 + (size_t)ncat * 16 + (size_t)(n_entries + 1) * 8 + (size_t)n_entries * 4 + 4096);
  if (st != PSIFT_OK) return st;
  uint64_t* d_q = (uint64_t*)io_take(ctx, (size_t)nq * 16 + 16);
  uint64_t* d_cat = (uint64_t*)io_take(ctx, (size_t)ncat * 16 + 16);
  long long* d_off = (long long*)io_take(ctx, (size_t)(n_entries + 1) * 8);
  uint32_t* d_votes = (uint32_t*)io_take(ctx, (size_t)n_entries * 4);
  if ((st = h2d(ctx, d_q, q_codes, (size_t)nq * 16)) != PSIFT_OK) return st;
  if ((st = h2d(ctx, d_cat, cat_codes, (size_t)ncat * 16)) != PSIFT_OK) return st;
  if ((st = h2d(ctx, d_off, entry_offsets, (size_t)(n_entries + 1) * 8)) != PSIFT_OK) return st;
  cudaError_t e;
  {
    StageScope sc(ctx, STAGE_HAMMING);
    e = launch_votes(d_q, (int)nq, d_cat, d_off, (int)n_entries, mih ? 1 : 0, d_votes, ctx->stream);
    ctx->launches++;
  }
  if (e != cudaSuccess) return cuda_error(ctx, e, "hamming_votes");
  return d2h_sync(ctx, votes, d_votes, (size_t)n_entries * 4);
}

psift_status psift_hamming_topk_dev(psift_ctx* ctx, const uint64_t* q_codes, uint32_t nq, const uint64_t* cat_codes,
                                    uint64_t ncat, uint32_t k, uint32_t* idx, uint32_t* dist) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (k == 0 || k > 64) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "k must be in 1..=64");
  if (nq == 0) return PSIFT_OK;
  if (!q_codes || !idx || !dist || (ncat && !cat_codes)) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  if (ncat >= 0xFFFFFFFFull) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "catalog larger than 2^32-1 codes");
  const int chunks = topk_chunks((long long)ncat, (int)nq, ctx->num_sms);
  st = arena_reserve(ctx, (size_t)nq * chunks * k * 8 + 4096);
  if (st != PSIFT_OK) return st;
  unsigned long long* part = (unsigned long long*)arena_alloc(ctx, (size_t)nq * chunks * k * 8);
  StageScope sc(ctx, STAGE_HAMMING);
  cudaError_t e = launch_topk(q_codes, (int)nq, cat_codes, (long long)ncat, (int)k, chunks, part, idx, dist, ctx->stream);
  ctx->launches += 2;
  if (e != cudaSuccess) return cuda_error(ctx, e, "hamming_topk");
  return PSIFT_OK;
}

psift_status psift_hamming_topk(psift_ctx* ctx, const uint64_t* q_codes, uint32_t nq, const uint64_t* cat_codes,
                                uint64_t ncat, uint32_t k, uint32_t* idx, uint32_t* dist) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (nq == 0) return PSIFT_OK;
  if (!q_codes || !idx || !dist || (ncat && !cat_codes)) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  st = io_reserve(ctx, (size_t)nq * 16 + (size_t)ncat * 16 + (size_t)nq * k * 8 + 4096);
  if (st != PSIFT_OK) return st;
  uint64_t* d_q = (uint64_t*)io_take(ctx, (size_t)nq * 16);
  uint64_t* d_cat = (uint64_t*)io_take(ctx, (size_t)ncat * 16 + 16);
  uint32_t* d_idx = (uint32_t*)io_take(ctx, (size_t)nq * k * 4);
  uint32_t* d_dist = (uint32_t*)io_take(ctx, (size_t)nq * k * 4);
  if ((st = h2d(ctx, d_q, q_codes, (size_t)nq * 16)) != PSIFT_OK) return st;
  if ((st = h2d(ctx, d_cat, cat_codes, (size_t)ncat * 16)) != PSIFT_OK) return st;
  st = psift_hamming_topk_dev(ctx, d_q, nq, d_cat, ncat, k, d_idx, d_dist);
  if (st != PSIFT_OK) return st;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(idx, d_idx, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, ctx->stream));
  return d2h_sync(ctx, dist, d_dist, (size_t)nq * k * 4);
}

psift_status psift_l2_rerank_dev(psift_ctx* ctx, const float* q_desc, uint32_t nq, const float* cat_desc,
                                 const uint32_t* cand, uint32_t k, uint32_t* out_idx, float* out_d2) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (k == 0 || k > 64) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "k must be in 1..=64");
  if (nq == 0) return PSIFT_OK;
  if (!q_desc || !cat_desc || !cand || !out_idx || !out_d2) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  StageScope sc(ctx, STAGE_HAMMING);
  cudaError_t e = launch_l2_rerank(q_desc, (int)nq, cat_desc, cand, (int)k, out_idx, out_d2, ctx->stream);
  ctx->launches++;
  if (e != cudaSuccess) return cuda_error(ctx, e, "l2_rerank");
  return PSIFT_OK;
}

psift_status psift_l2_rerank(psift_ctx* ctx, const float* q_desc, uint32_t nq, const float* cat_desc, uint64_t ncat,
                             const uint32_t* cand, uint32_t k, uint32_t* out_idx, float* out_d2) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (nq == 0) return PSIFT_OK;
  if (!q_desc || !cat_desc || !cand || !out_idx || !out_d2) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  for (size_t i = 0; i < (size_t)nq * k; ++i)
    if (cand[i] != 0xFFFFFFFFu && cand[i] >= ncat)
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "candidate index out of range");
  st = io_reserve(ctx, (size_t)nq * 512 + (size_t)ncat * 512 + (size_t)nq * k * 12 + 4096);
  if (st != PSIFT_OK) return st;
  float* d_q = (float*)io_take(ctx, (size_t)nq * 512);
  float* d_cat = (float*)io_take(ctx, (size_t)ncat * 512 + 16);
  uint32_t* d_cand = (uint32_t*)io_take(ctx, (size_t)nq * k * 4);
  uint32_t* d_idx = (uint32_t*)io_take(ctx, (size_t)nq * k * 4);
  float* d_d2 = (float*)io_take(ctx, (size_t)nq * k * 4);
  if ((st = h2d(ctx, d_q, q_desc, (size_t)nq * 512)) != PSIFT_OK) return st;
  if ((st = h2d(ctx, d_cat, cat_desc, (size_t)ncat * 512)) != PSIFT_OK) return st;
  if ((st = h2d(ctx, d_cand, cand, (size_t)nq * k * 4)) != PSIFT_OK) return st;
  st = psift_l2_rerank_dev(ctx, d_q, nq, d_cat, d_cand, k, d_idx, d_d2);
  if (st != PSIFT_OK) return st;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(out_idx, d_idx, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, ctx->stream));
  return d2h_sync(ctx, out_d2, d_d2, (size_t)nq * k * 4);
}

}  // extern "C"
