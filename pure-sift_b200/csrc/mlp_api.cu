// C-ABI entry points of the learned correspondence scorer (no reference counterpart).
#include <cmath>
#include <cstring>
#include <vector>

#include "psift_internal.cuh"

namespace psift {

cudaError_t launch_mlp_infer(const float* params, const float* X, int n, float* prob, int num_sms, uint32_t* err,
                             cudaStream_t st);
size_t mlp_batch_floats(int B);
cudaError_t launch_mlp_step(float* params, const float* X, const float* Y, const int* idx, int B, float* work,
                            float* grad, float* m, float* v, float lr, int t, float* loss_out, bool update,
                            cudaStream_t st);

namespace {
constexpr int kNumParams = PSIFT_MLP_NUM_PARAMS;
constexpr int kFeat = PSIFT_MLP_NUM_FEATURES;

uint64_t sm64(uint64_t& s) {
  s += 0x9E3779B97F4A7C15ull;
  uint64_t z = s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

psift_status begin(psift_ctx* ctx) {
  if (!ctx) return PSIFT_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(ctx, e, "cudaSetDevice");
  return PSIFT_OK;
}

// Seeded Fisher-Yates permutation of [0, n), followed by its first `tail` entries.
std::vector<int> permutation(uint32_t n, uint32_t tail, uint64_t seed) {
  std::vector<int> p(n + tail);
  for (uint32_t i = 0; i < n; ++i) p[i] = (int)i;
  uint64_t s = seed;
  for (uint32_t i = n; i > 1; --i) {
    const uint32_t j = (uint32_t)(sm64(s) % i);
    std::swap(p[i - 1], p[j]);
  }
  for (uint32_t i = 0; i < tail; ++i) p[n + i] = p[i % n];
  return p;
}
}  // namespace
}  // namespace psift

using namespace psift;

extern "C" {

// Kaiming-uniform weights from a splitmix64 stream, zero biases.
void psift_mlp_init(uint64_t seed, float* params) {
  if (!params) return;
  uint64_t s = seed;
  auto uni = [&](double bound) {
    const double u = (double)(sm64(s) >> 11) * (1.0 / 9007199254740992.0);
    return (float)((2.0 * u - 1.0) * bound);
  };
  int o = 0;
  for (int i = 0; i < 64 * 8; ++i) params[o++] = uni(std::sqrt(6.0 / 8.0));
  for (int i = 0; i < 64; ++i) params[o++] = 0.0f;
  for (int i = 0; i < 64 * 64; ++i) params[o++] = uni(std::sqrt(6.0 / 64.0));
  for (int i = 0; i < 64; ++i) params[o++] = 0.0f;
  for (int i = 0; i < 64; ++i) params[o++] = uni(std::sqrt(6.0 / 64.0));
  params[o++] = 0.0f;
}

psift_status psift_mlp_infer_dev(psift_ctx* ctx, const float* params, const float* x, uint32_t n, float* prob) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (n == 0) return PSIFT_OK;
  if (!params || !x || !prob) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  StageScope sc(ctx, STAGE_MLP);
  cudaError_t e = launch_mlp_infer(params, x, (int)n, prob, ctx->num_sms, ctx->d_error, ctx->stream);
  ctx->launches++;
  if (e != cudaSuccess) return cuda_error(ctx, e, "mlp_infer");
  return PSIFT_OK;
}

psift_status psift_mlp_train_dev(psift_ctx* ctx, float* params, const float* x, const float* y, uint32_t n,
                                 uint32_t steps, uint32_t batch, float lr, uint64_t seed, float* losses) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (!params || !x || !y || n == 0 || batch == 0 || batch > 65536)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "bad training arguments (batch must be 1..=65536)");
  const std::vector<int> perm = permutation(n, batch, seed);
  const size_t bytes = sizeof(float) * (mlp_batch_floats((int)batch) + 3 * (size_t)kNumParams) +
                       sizeof(int) * perm.size() + 8192;
  st = arena_reserve(ctx, bytes);
  if (st != PSIFT_OK) return st;
  float* work = (float*)arena_alloc(ctx, sizeof(float) * mlp_batch_floats((int)batch));
  float* grad = (float*)arena_alloc(ctx, sizeof(float) * kNumParams);
  float* m = (float*)arena_alloc(ctx, sizeof(float) * kNumParams);
  float* v = (float*)arena_alloc(ctx, sizeof(float) * kNumParams);
  int* d_perm = (int*)arena_alloc(ctx, sizeof(int) * perm.size());
  if (!d_perm) return set_error(ctx, PSIFT_ERR_INTERNAL, "mlp workspace carve overflow");
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(m, 0, sizeof(float) * kNumParams, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(v, 0, sizeof(float) * kNumParams, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_perm, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice, ctx->stream));
  StageScope sc(ctx, STAGE_MLP);
  for (uint32_t t = 0; t < steps; ++t) {
    const uint32_t start = (uint32_t)(((uint64_t)t * batch) % n);
    cudaError_t e = launch_mlp_step(params, x, y, d_perm + start, (int)batch, work, grad, m, v, lr, (int)t + 1,
                                    losses ? losses + t : nullptr, true, ctx->stream);
    ctx->launches += losses ? 5 : 4;
    if (e != cudaSuccess) return cuda_error(ctx, e, "mlp_train_step");
  }
  return PSIFT_OK;
}

psift_status psift_mlp_gradients_dev(psift_ctx* ctx, const float* params, const float* x, const float* y, uint32_t n,
                                     float* grad, float* loss) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (!params || !x || !y || !grad || n == 0 || n > 65536)
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "bad gradient arguments (n must be 1..=65536)");
  st = arena_reserve(ctx, sizeof(float) * mlp_batch_floats((int)n) + 4096);
  if (st != PSIFT_OK) return st;
  float* work = (float*)arena_alloc(ctx, sizeof(float) * mlp_batch_floats((int)n));
  cudaError_t e = launch_mlp_step(const_cast<float*>(params), x, y, nullptr, (int)n, work, grad, nullptr, nullptr,
                                  0.0f, 1, loss, false, ctx->stream);
  ctx->launches += loss ? 4 : 3;
  if (e != cudaSuccess) return cuda_error(ctx, e, "mlp_gradients");
  return PSIFT_OK;
}

// Host-pointer wrappers.
psift_status psift_mlp_infer(psift_ctx* ctx, const float* params, const float* x, uint32_t n, float* prob) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (n == 0) return PSIFT_OK;
  if (!params || !x || !prob) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  st = io_reserve(ctx, sizeof(float) * ((size_t)kNumParams + (size_t)n * (kFeat + 1)) + 4096);
  if (st != PSIFT_OK) return st;
  float* dp = (float*)ctx->io.base;
  float* dx = dp + align_up(kNumParams, 64);
  float* dprob = dx + (size_t)n * kFeat;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dp, params, sizeof(float) * kNumParams, cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dx, x, sizeof(float) * n * kFeat, cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_error, 0, 4, ctx->stream));
  st = psift_mlp_infer_dev(ctx, dp, dx, n, dprob);
  if (st != PSIFT_OK) return st;
  if ((st = pinned_reserve(ctx, 64)) != PSIFT_OK) return st;
  uint32_t* hword = (uint32_t*)ctx->pinned.base;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(prob, dprob, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hword, ctx->d_error, 4, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (*hword & kErrTimeout) return set_error(ctx, PSIFT_ERR_TIMEOUT, "mlp_infer: device wait timed out");
  return PSIFT_OK;
}

psift_status psift_mlp_gradients(psift_ctx* ctx, const float* params, const float* x, const float* y, uint32_t n,
                                 float* grad, float* loss) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (!params || !x || !y || !grad || n == 0) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  st = io_reserve(ctx, sizeof(float) * (2 * (size_t)kNumParams + (size_t)n * (kFeat + 1) + 64) + 4096);
  if (st != PSIFT_OK) return st;
  float* dp = (float*)ctx->io.base;
  float* dg = dp + align_up(kNumParams, 64);
  float* dx = dg + align_up(kNumParams, 64);
  float* dy = dx + (size_t)n * kFeat;
  float* dl = dy + align_up(n, 64);
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dp, params, sizeof(float) * kNumParams, cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dx, x, sizeof(float) * n * kFeat, cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dy, y, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
  st = psift_mlp_gradients_dev(ctx, dp, dx, dy, n, dg, dl);
  if (st != PSIFT_OK) return st;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(grad, dg, sizeof(float) * kNumParams, cudaMemcpyDeviceToHost, ctx->stream));
  if (loss) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(loss, dl, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PSIFT_OK;
}

psift_status psift_mlp_train(psift_ctx* ctx, float* params, const float* x, const float* y, uint32_t n,
                             uint32_t steps, uint32_t batch, float lr, uint64_t seed, float* losses) {
  psift_status st = begin(ctx);
  if (st != PSIFT_OK) return st;
  if (!params || !x || !y || n == 0) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null argument");
  st = io_reserve(ctx, sizeof(float) * ((size_t)kNumParams + (size_t)n * (kFeat + 1) + steps + 128) + 4096);
  if (st != PSIFT_OK) return st;
  float* dp = (float*)ctx->io.base;
  float* dx = dp + align_up(kNumParams, 64);
  float* dy = dx + (size_t)n * kFeat;
  float* dl = dy + align_up(n, 64);
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dp, params, sizeof(float) * kNumParams, cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dx, x, sizeof(float) * n * kFeat, cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(dy, y, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
  st = psift_mlp_train_dev(ctx, dp, dx, dy, n, steps, batch, lr, seed, losses ? dl : nullptr);
  if (st != PSIFT_OK) return st;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(params, dp, sizeof(float) * kNumParams, cudaMemcpyDeviceToHost, ctx->stream));
  if (losses) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(losses, dl, sizeof(float) * steps, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return PSIFT_OK;
}

}  // extern "C"
