// Multi-index hashing on the device: the catalog's 16 x 256 inverted tables
// (src/catalog.rs:291-321) and the MIH branch of search_features' coarse votes
// (:596-621).
//
// Tables.  Bucket (b, k) lists the features whose signature byte b equals k;
// all 4096 buckets are one bucket-major array of u32 feature indices (16 per
// feature) with u64 starts.  Built by a blocked counting sort: every build block
// takes a contiguous run of features and histograms its 16 keys per feature in
// shared memory; a column scan over the blocks gives each block its start inside
// every bucket; the scatter pass re-reads the run and places each feature with
// shared-memory cursors.  The order inside a bucket is not fixed (the cursors are
// atomics); the votes do not depend on it.
//
// Votes.  The reference walks, per query, the 16 buckets its own bytes select,
// tests popcount(q ^ s) <= 24 for every listed signature and counts an entry
// once per query.  Here the walk is bucket-major: the queries are grouped by
// (band, key) (one CTA, counting sort), and each CTA of the votes kernel takes a
// chunk of <= 1024 listed features of one bucket (4 per thread, codes gathered
// from the catalog's L2-resident code array) and tests them against every query
// of that bucket staged in shared memory.  A pair within 24 bits sets bit
// (query, entry) of a bitmap; the atomicOr that sets it first adds the vote, so
// each (query, entry) counts once, as with seen_stamp.  Work: sum over buckets
// of queries x listed features, 1/16 of an exhaustive scan's pairs for
// uniformly distributed bytes.  All integer: the votes are exact.
#include <algorithm>

#include "mih.cuh"

namespace psift {

namespace {

constexpr int kBuildBlocksMax = 512;
constexpr int kBuildRun = 2048;  // features per build block at least
constexpr uint64_t kMihMaxFeatures = 1ull << 28;

__device__ __forceinline__ int mih_popc4(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3) {
  // x0 + x1 + x2 = s + 2c bit by bit (carry-save), so three popcounts give the sum.
  const uint32_t s = x0 ^ x1 ^ x2;
  const uint32_t c = (x0 & x1) | (x2 & (x0 ^ x1));
  return __popc(s) + 2 * __popc(c) + __popc(x3);
}

// Band b of a signature held as 4 little-endian u32 words: byte b % 4 of word b / 4.
__device__ __forceinline__ uint32_t band_key(const uint4& c, int b) {
  const uint32_t w = b < 4 ? c.x : (b < 8 ? c.y : (b < 12 ? c.z : c.w));
  return (w >> (8 * (b & 3))) & 0xFFu;
}

__global__ void __launch_bounds__(256) mih_hist_kernel(const uint4* __restrict__ codes, uint64_t n, uint64_t run,
                                                       uint32_t* __restrict__ block_hist) {
  __shared__ uint32_t h[kMihBuckets];
  for (int j = threadIdx.x; j < kMihBuckets; j += blockDim.x) h[j] = 0;
  __syncthreads();
  const uint64_t i0 = (uint64_t)blockIdx.x * run, i1 = min(n, i0 + run);
  for (uint64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const uint4 c = codes[i];
#pragma unroll
    for (int b = 0; b < kMihBands; ++b) atomicAdd(&h[b * kMihKeys + band_key(c, b)], 1u);
  }
  __syncthreads();
  uint32_t* out = block_hist + (size_t)blockIdx.x * kMihBuckets;
  for (int j = threadIdx.x; j < kMihBuckets; j += blockDim.x) out[j] = h[j];
}

// Per bucket, the exclusive prefix over build blocks (in place) and the total.
__global__ void __launch_bounds__(256) mih_colscan_kernel(uint32_t* __restrict__ block_hist, int n_blocks,
                                                          uint32_t* __restrict__ totals) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kMihBuckets) return;
  uint32_t run = 0;
  for (int b = 0; b < n_blocks; ++b) {
    const uint32_t v = block_hist[(size_t)b * kMihBuckets + t];
    block_hist[(size_t)b * kMihBuckets + t] = run;
    run += v;
  }
  totals[t] = run;
}

// Exclusive scan of 4096 u32 counts into u64 starts (one block of 1024 threads,
// 4 consecutive buckets each).  off[4096] = the sum.
template <typename Out>
__device__ void scan4096(const uint32_t* cnt, Out* off, uint32_t* cursor) {
  __shared__ unsigned long long warp_tot[32];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const uint32_t a0 = cnt[4 * t], a1 = cnt[4 * t + 1], a2 = cnt[4 * t + 2], a3 = cnt[4 * t + 3];
  unsigned long long s = (unsigned long long)a0 + a1 + a2 + a3, incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    unsigned long long w = warp_tot[lane], wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long v = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += v;
    }
    warp_tot[lane] = wi - w;  // exclusive warp offsets
  }
  __syncthreads();
  const unsigned long long base = warp_tot[wid] + incl - s;
  const unsigned long long e0 = base, e1 = e0 + a0, e2 = e1 + a1, e3 = e2 + a2;
  off[4 * t] = (Out)e0;
  off[4 * t + 1] = (Out)e1;
  off[4 * t + 2] = (Out)e2;
  off[4 * t + 3] = (Out)e3;
  if (cursor) {
    cursor[4 * t] = (uint32_t)e0;
    cursor[4 * t + 1] = (uint32_t)e1;
    cursor[4 * t + 2] = (uint32_t)e2;
    cursor[4 * t + 3] = (uint32_t)e3;
  }
  if (t == 1023) off[kMihBuckets] = (Out)(e3 + a3);
}

__global__ void __launch_bounds__(1024) mih_offsets_kernel(const uint32_t* __restrict__ totals,
                                                           unsigned long long* __restrict__ off) {
  scan4096<unsigned long long>(totals, off, nullptr);
}

__global__ void __launch_bounds__(256) mih_scatter_kernel(const uint4* __restrict__ codes, uint64_t n, uint64_t run,
                                                          const uint32_t* __restrict__ block_hist,
                                                          const unsigned long long* __restrict__ off,
                                                          uint32_t* __restrict__ items) {
  __shared__ uint32_t cur[kMihBuckets];
  const uint32_t* pre = block_hist + (size_t)blockIdx.x * kMihBuckets;
  for (int j = threadIdx.x; j < kMihBuckets; j += blockDim.x) cur[j] = pre[j];
  __syncthreads();
  const uint64_t i0 = (uint64_t)blockIdx.x * run, i1 = min(n, i0 + run);
  for (uint64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const uint4 c = codes[i];
#pragma unroll
    for (int b = 0; b < kMihBands; ++b) {
      const int bk = b * kMihKeys + band_key(c, b);
      const uint32_t pos = atomicAdd(&cur[bk], 1u);
      items[off[bk] + pos] = (uint32_t)i;
    }
  }
}

// Queries grouped by (band, key): q_off[4097] and q_items[16 nq] (query indices).
__global__ void __launch_bounds__(1024) mih_group_kernel(const uint4* __restrict__ q, uint32_t nq,
                                                         uint32_t* __restrict__ q_off,
                                                         uint32_t* __restrict__ q_items) {
  __shared__ uint32_t h[kMihBuckets];
  for (int j = threadIdx.x; j < kMihBuckets; j += blockDim.x) h[j] = 0;
  __syncthreads();
  const uint64_t pairs = (uint64_t)nq * kMihBands;
  for (uint64_t p = threadIdx.x; p < pairs; p += blockDim.x) {
    const int b = (int)(p & 15);
    atomicAdd(&h[b * kMihKeys + band_key(q[p >> 4], b)], 1u);
  }
  __syncthreads();
  __shared__ uint32_t cnt[kMihBuckets];
  for (int j = threadIdx.x; j < kMihBuckets; j += blockDim.x) cnt[j] = h[j];
  __syncthreads();
  scan4096<uint32_t>(cnt, q_off, h);  // h becomes the cursors
  __syncthreads();
  for (uint64_t p = threadIdx.x; p < pairs; p += blockDim.x) {
    const int b = (int)(p & 15);
    const uint32_t qi = (uint32_t)(p >> 4);
    const uint32_t pos = atomicAdd(&h[b * kMihKeys + band_key(q[qi], b)], 1u);
    q_items[pos] = qi;
  }
}

__device__ __forceinline__ void mih_hit(uint32_t qi, uint32_t e, uint32_t n_entries, uint32_t* __restrict__ bitmap,
                                        uint32_t* __restrict__ votes) {
  const unsigned long long bit = (unsigned long long)qi * n_entries + e;
  const uint32_t mask = 1u << (uint32_t)(bit & 31);
  const uint32_t old = atomicOr(&bitmap[bit >> 5], mask);
  if (!(old & mask)) atomicAdd(&votes[e], 1u);
}

constexpr int kPerThread = kMihChunk / 256;

__global__ void __launch_bounds__(256) mih_votes_kernel(const MihChunk* __restrict__ chunks,
                                                        const uint32_t* __restrict__ items,
                                                        const uint32_t* __restrict__ entry_of,
                                                        const uint4* __restrict__ cat, const uint4* __restrict__ q,
                                                        const uint32_t* __restrict__ q_off,
                                                        const uint32_t* __restrict__ q_items, uint32_t n_entries,
                                                        uint32_t* __restrict__ bitmap, uint32_t* __restrict__ votes) {
  const MihChunk ch = chunks[blockIdx.x];
  const uint32_t q0 = q_off[ch.bucket], qn = q_off[ch.bucket + 1] - q0;
  if (qn == 0) return;  // the whole CTA leaves: no query selects this bucket
  uint4 code[kPerThread];
  uint32_t ent[kPerThread];
  bool ok[kPerThread];
#pragma unroll
  for (int k = 0; k < kPerThread; ++k) {
    const uint32_t idx = threadIdx.x + 256u * k;
    ok[k] = idx < ch.count;
    if (ok[k]) {
      const uint32_t f = items[ch.start + idx];
      code[k] = cat[f];
      ent[k] = entry_of[f];
    } else {
      code[k] = make_uint4(0, 0, 0, 0);
      ent[k] = 0;
    }
  }
  __shared__ uint4 sq[256];
  __shared__ uint32_t sqi[256];
  for (uint32_t t0 = 0; t0 < qn; t0 += 256) {
    const uint32_t m = min(256u, qn - t0);
    __syncthreads();
    if (threadIdx.x < m) {
      const uint32_t qi = q_items[q0 + t0 + threadIdx.x];
      sqi[threadIdx.x] = qi;
      sq[threadIdx.x] = q[qi];
    }
    __syncthreads();
    for (uint32_t j = 0; j < m; ++j) {
      const uint4 qq = sq[j];
#pragma unroll
      for (int k = 0; k < kPerThread; ++k) {
        const int d = mih_popc4(qq.x ^ code[k].x, qq.y ^ code[k].y, qq.z ^ code[k].z, qq.w ^ code[k].w);
        if (ok[k] && d <= 24) mih_hit(sqi[j], ent[k], n_entries, bitmap, votes);
      }
    }
  }
}

}  // namespace

void mih_free(MihIndex& m) {
  cudaFree(m.items);
  cudaFree(m.off);
  cudaFree(m.entry_of);
  cudaFree(m.block_hist);
  cudaFree(m.chunks);
  m = MihIndex{};
}

psift_status mih_build(psift_ctx* ctx, MihIndex& m, const uint64_t* codes, uint64_t n,
                       const std::vector<long long>& offsets) {
  m.valid = false;
  if (n > kMihMaxFeatures) return set_error(ctx, PSIFT_ERR_CAPACITY, "MIH tables: more than 2^28 features");
  cudaStream_t st = ctx->stream;
  const uint64_t n_entries = offsets.empty() ? 0 : offsets.size() - 1;
  if (n > m.cap_n || !m.items) {
    const uint64_t cap = std::max<uint64_t>(std::max<uint64_t>(n, 2 * m.cap_n), 1024);
    cudaFree(m.items);
    cudaFree(m.entry_of);
    m.items = nullptr;
    m.entry_of = nullptr;
    m.cap_n = 0;
    cudaError_t e = cudaMalloc(&m.items, cap * kMihBands * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m.entry_of, cap * 4);
    if (e != cudaSuccess) return cuda_error(ctx, e, "cudaMalloc(MIH tables)");
    m.cap_n = cap;
  }
  if (!m.off) {
    cudaError_t e = cudaMalloc(&m.off, (kMihBuckets + 1) * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&m.block_hist, (size_t)(kBuildBlocksMax + 1) * kMihBuckets * 4);
    if (e != cudaSuccess) return cuda_error(ctx, e, "cudaMalloc(MIH tables)");
  }
  // entry of every feature (host fill, one upload)
  std::vector<uint32_t> ent(n);
  for (uint64_t e = 0; e < n_entries; ++e)
    for (long long i = offsets[e]; i < offsets[e + 1]; ++i) ent[(size_t)i] = (uint32_t)e;
  if (n) PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(m.entry_of, ent.data(), n * 4, cudaMemcpyHostToDevice, st));

  const int nb = (int)std::max<uint64_t>(1, std::min<uint64_t>(kBuildBlocksMax, (n + kBuildRun - 1) / kBuildRun));
  const uint64_t run = (n + nb - 1) / nb;
  uint32_t* totals = m.block_hist + (size_t)kBuildBlocksMax * kMihBuckets;
  mih_hist_kernel<<<nb, 256, 0, st>>>((const uint4*)codes, n, run, m.block_hist);
  mih_colscan_kernel<<<kMihBuckets / 256, 256, 0, st>>>(m.block_hist, nb, totals);
  mih_offsets_kernel<<<1, 1024, 0, st>>>(totals, m.off);
  mih_scatter_kernel<<<nb, 256, 0, st>>>((const uint4*)codes, n, run, m.block_hist, m.off, m.items);
  ctx->launches += 4;
  PSIFT_CUDA_TRY(ctx, cudaGetLastError());

  // Chunk list (host): every bucket cut into runs of <= kMihChunk items.
  std::vector<unsigned long long> off(kMihBuckets + 1);
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(off.data(), m.off, off.size() * 8, cudaMemcpyDeviceToHost, st));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  std::vector<MihChunk> chunks;
  m.max_bucket = 0;
  for (int b = 0; b < kMihBuckets; ++b) {
    const unsigned long long len = off[b + 1] - off[b];
    m.max_bucket = std::max<uint64_t>(m.max_bucket, len);
    for (unsigned long long s = 0; s < len; s += kMihChunk)
      chunks.push_back(MihChunk{(uint32_t)b, (uint32_t)std::min<unsigned long long>(kMihChunk, len - s), off[b] + s});
  }
  if (chunks.size() > m.cap_chunks) {
    const size_t cap = std::max<size_t>(chunks.size(), 2 * (size_t)m.cap_chunks);
    cudaFree(m.chunks);
    m.chunks = nullptr;
    m.cap_chunks = 0;
    cudaError_t e = cudaMalloc(&m.chunks, cap * sizeof(MihChunk));
    if (e != cudaSuccess) return cuda_error(ctx, e, "cudaMalloc(MIH chunks)");
    m.cap_chunks = cap;
  }
  if (!chunks.empty())
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(m.chunks, chunks.data(), chunks.size() * sizeof(MihChunk),
                                        cudaMemcpyHostToDevice, st));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  m.n_chunks = (uint32_t)chunks.size();
  m.n = n;
  m.n_entries = (uint32_t)n_entries;
  m.valid = true;
  return PSIFT_OK;
}

size_t mih_votes_scratch_bytes(uint32_t nq, uint32_t n_entries) {
  const uint64_t bits = (uint64_t)nq * n_entries;
  return align_up((kMihBuckets + 1) * 4, 256) + align_up((size_t)nq * kMihBands * 4, 256) +
         align_up((size_t)((bits + 31) / 32) * 4, 256);
}

cudaError_t mih_votes(const MihIndex& m, const uint64_t* catalog_codes, const uint64_t* qcodes, uint32_t nq,
                      uint32_t* votes, void* scratch, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(votes, 0, (size_t)m.n_entries * 4, st);
  if (e != cudaSuccess || nq == 0 || m.n_entries == 0 || m.n_chunks == 0) return e;
  char* w = (char*)scratch;
  uint32_t* q_off = (uint32_t*)w;
  uint32_t* q_items = (uint32_t*)(w + align_up((kMihBuckets + 1) * 4, 256));
  uint32_t* bitmap = (uint32_t*)(w + align_up((kMihBuckets + 1) * 4, 256) + align_up((size_t)nq * kMihBands * 4, 256));
  const uint64_t bits = (uint64_t)nq * m.n_entries;
  e = cudaMemsetAsync(bitmap, 0, (size_t)((bits + 31) / 32) * 4, st);
  if (e != cudaSuccess) return e;
  mih_group_kernel<<<1, 1024, 0, st>>>((const uint4*)qcodes, nq, q_off, q_items);
  mih_votes_kernel<<<m.n_chunks, 256, 0, st>>>(m.chunks, m.items, m.entry_of, (const uint4*)catalog_codes,
                                               (const uint4*)qcodes, q_off, q_items, m.n_entries, bitmap, votes);
  return cudaGetLastError();
}

}  // namespace psift
