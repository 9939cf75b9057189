// K11: the learned correspondence scorer that drives guided RANSAC sampling.
// No counterpart in the reference (its sampler weights matches by 1/ratio,
// src/pipeline.rs:2006-2036).
//
// Network 8 -> 64 -> 64 -> 1, ReLU, ReLU, sigmoid.  Parameters are f32 masters;
// the forward pass rounds weights and activations to bf16 (round to nearest even)
// and accumulates in f32.  The backward pass is f32 on the same bf16-rounded
// operands (straight-through rounding).  Training is deterministic:
//   mlp_fwd_bwd_kernel   one thread per sample: forward, dL/dz for every layer;
//   mlp_grad_partial_kernel / mlp_grad_reduce_kernel: per-parameter sums over
//                        chunks of samples in order, then over the chunks in order;
//   mlp_adam_kernel      Adam update of the f32 masters.
// Loss: mean binary cross-entropy over the minibatch.
#include <algorithm>

#include "psift_internal.cuh"

namespace psift {

constexpr int kF = 8, kH = 64;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kF, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH,
              kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH, kNP = kOffB3 + 1;  // 4801

__device__ __forceinline__ float bf16r(float x) {
  const uint32_t u = __float_as_uint(x);
  if ((u & 0x7f800000u) == 0x7f800000u) return x;  // inf / nan unchanged
  const uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
  return __uint_as_float(r & 0xFFFF0000u);
}

struct MlpSmem {
  float w1[kH][kF];
  float b1[kH];
  float w2[kH][kH];
  float b2[kH];
  float w3[kH];
  float b3;
};

__device__ void load_params(const float* __restrict__ p, MlpSmem& s) {
  for (int i = threadIdx.x; i < kH * kF; i += blockDim.x) (&s.w1[0][0])[i] = bf16r(p[kOffW1 + i]);
  for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) (&s.w2[0][0])[i] = bf16r(p[kOffW2 + i]);
  for (int i = threadIdx.x; i < kH; i += blockDim.x) {
    s.b1[i] = p[kOffB1 + i];
    s.b2[i] = p[kOffB2 + i];
    s.w3[i] = bf16r(p[kOffW3 + i]);
  }
  if (threadIdx.x == 0) s.b3 = p[kOffB3];
  __syncthreads();
}

// Forward of one sample; returns z3 and fills xb, h1b (and z1 signs) on request.
__device__ __forceinline__ float forward1(const MlpSmem& s, const float* __restrict__ x, float (&xb)[kF],
                                          float (&h1b)[kH], float* h2b_out, uint64_t* z1pos, uint64_t* z2pos) {
#pragma unroll
  for (int k = 0; k < kF; ++k) xb[k] = bf16r(x[k]);
  uint64_t p1 = 0;
#pragma unroll
  for (int j = 0; j < kH; ++j) {
    float z = s.b1[j];
#pragma unroll
    for (int k = 0; k < kF; ++k) z = __fmaf_rn(s.w1[j][k], xb[k], z);
    p1 |= (z > 0.0f ? 1ull : 0ull) << j;
    h1b[j] = bf16r(z > 0.0f ? z : 0.0f);
  }
  float z3 = s.b3;
  uint64_t p2 = 0;
#pragma unroll 4
  for (int j = 0; j < kH; ++j) {
    float z = s.b2[j];
#pragma unroll
    for (int k = 0; k < kH; ++k) z = __fmaf_rn(s.w2[j][k], h1b[k], z);
    p2 |= (z > 0.0f ? 1ull : 0ull) << j;
    const float h2 = bf16r(z > 0.0f ? z : 0.0f);
    if (h2b_out) h2b_out[j] = h2;
    z3 = __fmaf_rn(s.w3[j], h2, z3);
  }
  if (z1pos) *z1pos = p1;
  if (z2pos) *z2pos = p2;
  return z3;
}

__device__ __forceinline__ float sigmoidf_(float z) { return 1.0f / (1.0f + expf(-z)); }

__global__ void __launch_bounds__(256) mlp_infer_kernel(const float* __restrict__ params, const float* __restrict__ X,
                                                        int n, float* __restrict__ prob) {
  __shared__ MlpSmem s;
  load_params(params, s);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float xb[kF], h1b[kH];
    const float z3 = forward1(s, X + (size_t)i * kF, xb, h1b, nullptr, nullptr, nullptr);
    prob[i] = sigmoidf_(z3);
  }
}

// One thread per minibatch sample b (sample index idx[b]).  Stores the operands
// and deltas the per-parameter gradient sums need.
__global__ void __launch_bounds__(128) mlp_fwd_bwd_kernel(const float* __restrict__ params,
                                                          const float* __restrict__ X, const float* __restrict__ Y,
                                                          const int* __restrict__ idx, int B, float* __restrict__ xb_o,
                                                          float* __restrict__ h1b_o, float* __restrict__ h2b_o,
                                                          float* __restrict__ dz1_o, float* __restrict__ dz2_o,
                                                          float* __restrict__ dz3_o, float* __restrict__ loss_o) {
  __shared__ MlpSmem s;
  load_params(params, s);
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const int i = idx ? idx[b] : b;
  float xb[kF], h1b[kH], h2b[kH];
  uint64_t p1, p2;
  const float z3 = forward1(s, X + (size_t)i * kF, xb, h1b, h2b, &p1, &p2);
  const float p = sigmoidf_(z3);
  const float y = Y[i];
  // BCE with logits: softplus(z) - y z, numerically stable form
  const float l = fmaxf(z3, 0.0f) - z3 * y + log1pf(expf(-fabsf(z3)));
  const float invB = 1.0f / (float)B;
  const float dz3 = (p - y) * invB;
  float dz2[kH];
#pragma unroll
  for (int j = 0; j < kH; ++j) dz2[j] = ((p2 >> j) & 1ull) ? dz3 * s.w3[j] : 0.0f;
#pragma unroll 4
  for (int k = 0; k < kH; ++k) {
    float dh = 0.0f;
#pragma unroll
    for (int j = 0; j < kH; ++j) dh = __fmaf_rn(s.w2[j][k], dz2[j], dh);
    dz1_o[(size_t)b * kH + k] = ((p1 >> k) & 1ull) ? dh : 0.0f;
  }
#pragma unroll
  for (int j = 0; j < kH; ++j) {
    h1b_o[(size_t)b * kH + j] = h1b[j];
    h2b_o[(size_t)b * kH + j] = h2b[j];
    dz2_o[(size_t)b * kH + j] = dz2[j];
  }
#pragma unroll
  for (int k = 0; k < kF; ++k) xb_o[(size_t)b * kF + k] = xb[k];
  dz3_o[b] = dz3;
  loss_o[b] = l;
}

// Gradient sums, deterministic: the batch is cut into chunks of kGradChunk
// samples; mlp_grad_partial_kernel (one thread per (parameter, chunk)) sums a
// chunk in sample order, mlp_grad_reduce_kernel adds the chunks' sums in chunk
// order.  Fixed order, so every run gives the same bits.
constexpr int kGradChunk = 128;

__global__ void mlp_grad_partial_kernel(int B, const float* __restrict__ xb, const float* __restrict__ h1b,
                                        const float* __restrict__ h2b, const float* __restrict__ dz1,
                                        const float* __restrict__ dz2, const float* __restrict__ dz3,
                                        float* __restrict__ partial) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNP) return;
  const int b0 = blockIdx.y * kGradChunk;
  const int b1 = min(B, b0 + kGradChunk);
  float g = 0.0f;
  if (p < kOffB1) {
    const int j = (p - kOffW1) / kF, k = (p - kOffW1) % kF;
    for (int b = b0; b < b1; ++b) g = __fmaf_rn(dz1[(size_t)b * kH + j], xb[(size_t)b * kF + k], g);
  } else if (p < kOffW2) {
    const int j = p - kOffB1;
    for (int b = b0; b < b1; ++b) g += dz1[(size_t)b * kH + j];
  } else if (p < kOffB2) {
    const int j = (p - kOffW2) / kH, k = (p - kOffW2) % kH;
    for (int b = b0; b < b1; ++b) g = __fmaf_rn(dz2[(size_t)b * kH + j], h1b[(size_t)b * kH + k], g);
  } else if (p < kOffW3) {
    const int j = p - kOffB2;
    for (int b = b0; b < b1; ++b) g += dz2[(size_t)b * kH + j];
  } else if (p < kOffB3) {
    const int j = p - kOffW3;
    for (int b = b0; b < b1; ++b) g = __fmaf_rn(dz3[b], h2b[(size_t)b * kH + j], g);
  } else {
    for (int b = b0; b < b1; ++b) g += dz3[b];
  }
  partial[(size_t)blockIdx.y * kNP + p] = g;
}

__global__ void mlp_grad_reduce_kernel(int chunks, const float* __restrict__ partial, float* __restrict__ grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNP) return;
  float g = 0.0f;
  for (int c = 0; c < chunks; ++c) g += partial[(size_t)c * kNP + p];
  grad[p] = g;
}

__global__ void mlp_adam_kernel(float* __restrict__ params, const float* __restrict__ grad, float* __restrict__ m,
                                float* __restrict__ v, float lr, float beta1, float beta2, float eps, float bc1,
                                float bc2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNP) return;
  const float g = grad[p];
  const float mm = beta1 * m[p] + (1.0f - beta1) * g;
  const float vv = beta2 * v[p] + (1.0f - beta2) * g * g;
  m[p] = mm;
  v[p] = vv;
  params[p] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
}

// Mean of the per-sample losses into loss[step], in a fixed order (deterministic):
// thread t sums samples t, t + 256, t + 512, ... in that order (coalesced loads
// across a warp), then a fixed pairwise tree over the 256 partial sums.  One CTA.
constexpr int kLossThreads = 256;
__global__ void __launch_bounds__(kLossThreads) mlp_loss_kernel(const float* __restrict__ l, int B,
                                                                float* __restrict__ out) {
  __shared__ float part[kLossThreads];
  const int t = threadIdx.x;
  float s = 0.0f;
  for (int b = t; b < B; b += kLossThreads) s += l[b];
  part[t] = s;
  __syncthreads();
  for (int h = kLossThreads / 2; h > 0; h >>= 1) {
    if (t < h) part[t] += part[t + h];
    __syncthreads();
  }
  if (t == 0) *out = part[0] / (float)B;
}

// ------------------------------------------------------------ tensor-core inference
// mlp_infer_tc_kernel: the same network on bf16 tensor-core tiles
// (mma.sync m16n8k16, f32 accumulation).  A warp evaluates 16 samples per tile:
// layer 1 (K = 8 features, padded to 16) and layer 2 (K = 64) are MMAs whose f32
// accumulators start at the biases; the layer-1 accumulator fragment, ReLU'd and
// rounded to bf16, is exactly the layer-2 A fragment (rows g / g + 8, columns
// 2t, 2t + 1 of consecutive 8-column tiles), so activations never leave the
// registers; layer 3 is a per-row dot product reduced over the 4 lanes of a
// quad.  The bf16-rounded weights live in registers for the whole kernel.
// Operand rounding is the scalar kernel's (bf16, round to nearest even); only
// the f32 summation order inside a product differs.
//
// Input staging: persistent CTAs (one per SM) take chunks of kMlpChunk samples
// (32 KB) round-robin; thread 0 streams them into a kMlpStages-deep shared-memory
// ring with 1-D bulk async copies (cp.async.bulk, mbarrier completion), so the
// HBM reads run ahead of the tensor work.  Every wait is bounded: on timeout the
// CTA records kErrTimeout in err and returns once its issued copies have landed.
constexpr int kMlpThreads = 256;
constexpr int kMlpWarps = kMlpThreads / 32;
constexpr int kMlpChunk = 1024;  // samples per ring stage
constexpr int kMlpStages = 4;
constexpr uint32_t kMlpSpin = 1u << 24;
constexpr size_t kMlpSmem = (size_t)kMlpStages * kMlpChunk * kF * sizeof(float) + 128;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// {lo, hi} -> bf16x2 (round to nearest even), lo in the low half.
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ bool mlp_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < kMlpSpin; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__global__ void __launch_bounds__(kMlpThreads, 1) mlp_infer_tc_kernel(const float* __restrict__ params,
                                                                      const float* __restrict__ X, int n,
                                                                      float* __restrict__ prob, uint32_t* err) {
  extern __shared__ __align__(128) uint8_t mlp_smem[];
  float* xs = reinterpret_cast<float*>(mlp_smem);
  uint64_t* full = reinterpret_cast<uint64_t*>(mlp_smem + (size_t)kMlpStages * kMlpChunk * kF * sizeof(float));
  uint64_t* empty = full + kMlpStages;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int n_chunks = (n + kMlpChunk - 1) / kMlpChunk;
  if ((int)blockIdx.x >= n_chunks) return;
  const int my_chunks = (n_chunks - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  auto chunk_samples = [&](int i) {
    const int base = ((int)blockIdx.x + i * (int)gridDim.x) * kMlpChunk;
    return min(kMlpChunk, n - base);
  };
  auto issue = [&](int i) {  // thread 0: chunk i of this CTA into stage i % kMlpStages
    const int s = i % kMlpStages;
    const long long base = ((long long)blockIdx.x + (long long)i * gridDim.x) * kMlpChunk;
    const uint32_t bytes = (uint32_t)chunk_samples(i) * kF * sizeof(float);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&full[s])), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(xs + (size_t)s * kMlpChunk * kF)),
        "l"(X + base * kF), "r"(bytes), "r"(smem_addr(&full[s]))
        : "memory");
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < kMlpStages; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&full[s])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&empty[s])), "r"(kMlpWarps) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    for (int i = 0; i < kMlpStages && i < my_chunks; ++i) issue(i);
  }
  // bf16 weight fragments (B operands: column n = output g of the 8-column tile,
  // rows k = 2t, 2t + 1 and 2t + 8, 2t + 9 of the 16-deep K step) and biases for
  // the accumulator columns 2t, 2t + 1 of each 8-column tile
  uint32_t w1r[8], w2r[4][8][2];
  float b1v[8][2], b2v[8][2], w3v[8][2];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int j = nt * 8 + g;
    w1r[nt] = pack_bf16(params[kOffW1 + j * kF + 2 * t], params[kOffW1 + j * kF + 2 * t + 1]);
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const float* w = params + kOffW2 + j * kH + kk * 16 + 2 * t;
      w2r[kk][nt][0] = pack_bf16(w[0], w[1]);
      w2r[kk][nt][1] = pack_bf16(w[8], w[9]);
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      b1v[nt][c] = params[kOffB1 + nt * 8 + 2 * t + c];
      b2v[nt][c] = params[kOffB2 + nt * 8 + 2 * t + c];
      w3v[nt][c] = bf16r(params[kOffW3 + nt * 8 + 2 * t + c]);
    }
  }
  const float b3 = params[kOffB3];
  __syncthreads();  // barriers initialised
  bool ok = true;
  for (int i = 0; i < my_chunks; ++i) {
    const int s = i % kMlpStages;
    const uint32_t par = (uint32_t)(i / kMlpStages) & 1u;
    if (!mlp_wait(&full[s], par)) {
      ok = false;
      break;
    }
    const float* xc = xs + (size_t)s * kMlpChunk * kF;
    const int cnt = chunk_samples(i);
    const long long base = ((long long)blockIdx.x + (long long)i * gridDim.x) * kMlpChunk;
    for (int tile = warp; tile * 16 < cnt; tile += kMlpWarps) {
      // layer 1: A = the tile's 16 x 8 features (K padded with zeros)
      const float2 xa = *reinterpret_cast<const float2*>(xc + (tile * 16 + g) * kF + 2 * t);
      const float2 xb = *reinterpret_cast<const float2*>(xc + (tile * 16 + g + 8) * kF + 2 * t);
      const uint32_t a1[4] = {pack_bf16(xa.x, xa.y), pack_bf16(xb.x, xb.y), 0u, 0u};
      uint32_t a2[4][4];
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        float c[4] = {b1v[nt][0], b1v[nt][1], b1v[nt][0], b1v[nt][1]};
        mma_bf16_16816(c, a1, w1r[nt], 0u);
        // ReLU, bf16: this tile is K columns 8 (nt & 1) .. of layer 2's K step nt / 2
        a2[nt >> 1][(nt & 1) * 2 + 0] = pack_bf16(fmaxf(c[0], 0.0f), fmaxf(c[1], 0.0f));
        a2[nt >> 1][(nt & 1) * 2 + 1] = pack_bf16(fmaxf(c[2], 0.0f), fmaxf(c[3], 0.0f));
      }
      // layer 2 and the layer-3 dot products of rows g and g + 8
      float z_lo = 0.0f, z_hi = 0.0f;
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        float c[4] = {b2v[nt][0], b2v[nt][1], b2v[nt][0], b2v[nt][1]};
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) mma_bf16_16816(c, a2[kk], w2r[kk][nt][0], w2r[kk][nt][1]);
        z_lo = __fmaf_rn(w3v[nt][0], bf16r(fmaxf(c[0], 0.0f)), z_lo);
        z_lo = __fmaf_rn(w3v[nt][1], bf16r(fmaxf(c[1], 0.0f)), z_lo);
        z_hi = __fmaf_rn(w3v[nt][0], bf16r(fmaxf(c[2], 0.0f)), z_hi);
        z_hi = __fmaf_rn(w3v[nt][1], bf16r(fmaxf(c[3], 0.0f)), z_hi);
      }
      z_lo += __shfl_xor_sync(0xffffffffu, z_lo, 1);
      z_hi += __shfl_xor_sync(0xffffffffu, z_hi, 1);
      z_lo += __shfl_xor_sync(0xffffffffu, z_lo, 2);
      z_hi += __shfl_xor_sync(0xffffffffu, z_hi, 2);
      if (t == 0) {
        const int r0 = tile * 16 + g, r1 = r0 + 8;
        if (r0 < cnt) prob[base + r0] = sigmoidf_(b3 + z_lo);
        if (r1 < cnt) prob[base + r1] = sigmoidf_(b3 + z_hi);
      }
    }
    __syncwarp();
    if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&empty[s])) : "memory");
    if (threadIdx.x == 0 && i + kMlpStages < my_chunks) {
      // refill this stage once every warp is done with it
      if (!mlp_wait(&empty[s], par)) {
        ok = false;
        break;
      }
      issue(i + kMlpStages);
    }
  }
  if (!ok) {
    atomicOr(err, kErrTimeout);
    // wait (bounded) for this CTA's copies still in flight before the CTA exits
    if (threadIdx.x == 0) {
      const int issued = min(my_chunks, kMlpStages);
      for (int i = 0; i < issued; ++i) mlp_wait(&full[i % kMlpStages], (uint32_t)(i / kMlpStages) & 1u);
    }
  }
}

cudaError_t launch_mlp_infer(const float* params, const float* X, int n, float* prob, int num_sms, uint32_t* err,
                             cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if ((reinterpret_cast<uintptr_t>(X) & 15u) == 0) {
    // tensor-core path: the bulk copies need 16-byte aligned rows (32 B per sample)
    cudaError_t e = ensure_smem_attr((const void*)mlp_infer_tc_kernel, kMlpSmem);
    if (e != cudaSuccess) return e;
    const int chunks = (n + kMlpChunk - 1) / kMlpChunk;
    mlp_infer_tc_kernel<<<std::min(chunks, num_sms), kMlpThreads, kMlpSmem, st>>>(params, X, n, prob, err);
    return cudaGetLastError();
  }
  const int blocks = std::min((n + 255) / 256, num_sms * 8);
  mlp_infer_kernel<<<blocks, 256, 0, st>>>(params, X, n, prob);
  return cudaGetLastError();
}

// Workspace for a minibatch of B: (8 + 64*4 + 2) * B floats of per-sample
// operands, then one row of kNP partial gradient sums per kGradChunk samples.
size_t mlp_batch_floats(int B) {
  return (size_t)B * (kF + 4 * kH + 2) + (size_t)((B + kGradChunk - 1) / kGradChunk) * kNP;
}

cudaError_t launch_mlp_step(float* params, const float* X, const float* Y, const int* idx, int B, float* work,
                            float* grad, float* m, float* v, float lr, int t, float* loss_out, bool update,
                            cudaStream_t st) {
  float* xb = work;
  float* h1b = xb + (size_t)B * kF;
  float* h2b = h1b + (size_t)B * kH;
  float* dz1 = h2b + (size_t)B * kH;
  float* dz2 = dz1 + (size_t)B * kH;
  float* dz3 = dz2 + (size_t)B * kH;
  float* lb = dz3 + B;
  float* partial = lb + B;
  const int chunks = (B + kGradChunk - 1) / kGradChunk;
  mlp_fwd_bwd_kernel<<<(B + 127) / 128, 128, 0, st>>>(params, X, Y, idx, B, xb, h1b, h2b, dz1, dz2, dz3, lb);
  mlp_grad_partial_kernel<<<dim3((kNP + 127) / 128, chunks), 128, 0, st>>>(B, xb, h1b, h2b, dz1, dz2, dz3, partial);
  mlp_grad_reduce_kernel<<<(kNP + 127) / 128, 128, 0, st>>>(chunks, partial, grad);
  if (loss_out) mlp_loss_kernel<<<1, kLossThreads, 0, st>>>(lb, B, loss_out);
  if (update) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.0f - powf(b1, (float)t), bc2 = 1.0f - powf(b2, (float)t);
    mlp_adam_kernel<<<(kNP + 255) / 256, 256, 0, st>>>(params, grad, m, v, lr, b1, b2, 1e-8f, bc1, bc2);
  }
  return cudaGetLastError();
}

}  // namespace psift
