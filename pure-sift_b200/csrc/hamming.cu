// K9: 128-bit binary signatures and the catalog's Hamming stages.
//
// Reference: quantize_descriptor_u128 (src/catalog.rs:37-45),
// FeatureCatalog::search_features coarse voting (src/catalog.rs:588-641) with the
// multi-index-hashing tables (:291-321) and count_coarse_hamming_votes
// (:707-728); quantize_descriptor_u8 / dequantize_descriptor_u8
// (src/pipeline.rs:1024-1044).
//
// Signatures are two little-endian u64 words (bit i of the u128 = bit i%64 of
// word i/64).  All comparisons are integer: results are bit-exact.
//
// Votes.  The exhaustive path counts the queries whose nearest signature in the
// entry is within 24 bits.  The MIH path (more than 32 entries) only reaches a
// signature through one of its 16 byte bands, i.e. when some byte of q ^ s is
// zero; a (query, entry) pair votes iff some signature of the entry has
// popcount(q ^ s) <= 24 AND a zero byte in q ^ s.  Both are evaluated directly,
// without the inverted tables.
//
// Top-k shortlist (no reference counterpart; the catalog search at scale): the k
// codes nearest to each query by (Hamming distance, catalog index).  One warp
// serves 16 queries over one chunk of codes: lane i scores code base+i against the
// 16 queries (4 XOR + 4 POPC each); a ballot finds codes beating a query's current
// k-th entry, and the warp replaces that entry cooperatively (rare after the list
// fills).  Chunk lists are merged per query by a second kernel.
#include <algorithm>

#include "psift_internal.cuh"

namespace psift {

constexpr int kQG = 16;       // queries per warp
constexpr int kTopKMax = 64;  // shortlist length upper bound
constexpr int kHamWarps = 4;

// popc(x0) + popc(x1) + popc(x2) + popc(x3) with three popcounts: a carry-save
// step gives, bit by bit, x0 + x1 + x2 = s + 2c (s = x0 ^ x1 ^ x2, c = majority),
// so the sum is popc(s) + 2 popc(c) + popc(x3), the same integer.  The popcount
// pipe bounds the Hamming scans; s and c are one LOP3 each on the ALU pipe.
__device__ __forceinline__ int popc4(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3) {
  const uint32_t s = x0 ^ x1 ^ x2;
  const uint32_t c = (x0 & x1) | (x2 & (x0 ^ x1));
  return __popc(s) + 2 * __popc(c) + __popc(x3);
}

__device__ __forceinline__ int ham128(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint4 c) {
  return popc4(a0 ^ c.x, a1 ^ c.y, a2 ^ c.z, a3 ^ c.w);
}

__device__ __forceinline__ bool has_zero_byte(uint32_t x) { return ((x - 0x01010101u) & ~x & 0x80808080u) != 0; }

// quantize_descriptor_u128 (src/catalog.rs:37-45): bit d = desc[d] > 0.065.
// A warp handles kQDesc descriptors; lane l reads dims l, l + 32, l + 64, l + 96
// of each (coalesced 128-byte rows, all loads issued first) and the ballot of
// "dim 32 w + l > 0.065" over the lanes is code word w, bit l.
constexpr int kQDesc = 4;
__global__ void __launch_bounds__(256) quantize_codes_kernel(const float* __restrict__ desc, int n,
                                                             uint64_t* __restrict__ codes) {
  const int lane = threadIdx.x & 31;
  const int row0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * kQDesc;
  float v[kQDesc][4];
#pragma unroll
  for (int d = 0; d < kQDesc; ++d)
#pragma unroll
    for (int w = 0; w < 4; ++w) v[d][w] = row0 + d < n ? __ldcs(desc + (size_t)(row0 + d) * 128 + 32 * w + lane) : 0.0f;
#pragma unroll
  for (int d = 0; d < kQDesc; ++d) {
    uint32_t word[4];
#pragma unroll
    for (int w = 0; w < 4; ++w) word[w] = __ballot_sync(0xffffffffu, v[d][w] > 0.065f);
    const uint32_t lo = lane ? word[2] : word[0], hi = lane ? word[3] : word[1];  // no indexed local array
    if (lane < 2 && row0 + d < n) codes[2 * (size_t)(row0 + d) + lane] = (uint64_t)lo | ((uint64_t)hi << 32);
  }
}

// quantize_descriptor_u128 + quantize_descriptor_u8: one warp per descriptor.
__global__ void quantize_kernel(const float* __restrict__ desc, int n, uint64_t* __restrict__ codes,
                                uint8_t* __restrict__ u8) {
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const float4 v = reinterpret_cast<const float4*>(desc + (size_t)row * 128)[lane];
  const float e[4] = {v.x, v.y, v.z, v.w};
  if (codes) {
    // element 4*lane + j -> bit (4*lane + j)
    uint32_t nib = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) nib |= (e[j] > 0.065f ? 1u : 0u) << j;
    uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
    for (int l = 0; l < 32; ++l) {
      const uint32_t x = __shfl_sync(0xffffffffu, nib, l);
      w[l >> 3] |= x << (4 * (l & 7));
    }
    if (lane == 0) {
      codes[2 * (size_t)row] = (uint64_t)w[0] | ((uint64_t)w[1] << 32);
      codes[2 * (size_t)row + 1] = (uint64_t)w[2] | ((uint64_t)w[3] << 32);
    }
  }
  if (u8) {
    uint32_t packed = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float q = roundf(e[j] * 512.0f);
      q = q < 0.0f ? 0.0f : (q > 255.0f ? 255.0f : q);
      packed |= (uint32_t)q << (8 * j);
    }
    reinterpret_cast<uint32_t*>(u8 + (size_t)row * 128)[lane] = packed;
  }
}

// dequantize_descriptor_u8: v/512 then L2 renormalisation (sequential sum).  A
// warp per 32 rows: the u8 rows are copied into shared memory (16-byte
// asynchronous copies, all in flight together), lane j adds up row j's squared
// norm sequentially from there, and the scaled rows are written back coalesced
// (a float4 per lane and row).
constexpr int kDqWarps = 4;
constexpr int kDqStride = 144;  // bytes per staged row: lanes reading 16 B of different rows hit distinct banks

__device__ __forceinline__ float4 dq4(uint32_t p) {
  return make_float4((float)(p & 0xFF) * (1.0f / 512.0f), (float)((p >> 8) & 0xFF) * (1.0f / 512.0f),
                     (float)((p >> 16) & 0xFF) * (1.0f / 512.0f), (float)(p >> 24) * (1.0f / 512.0f));
}

__global__ void __launch_bounds__(32 * kDqWarps) dequantize_kernel(const uint8_t* __restrict__ q, int n,
                                                                   float* __restrict__ out) {
  __shared__ __align__(16) uint8_t stage[kDqWarps][32 * kDqStride];
  __shared__ float inv_s[kDqWarps][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = (blockIdx.x * kDqWarps + warp) * 32;
  if (row0 >= n) return;
  const int nr = min(32, n - row0);
  uint8_t* st = stage[warp];
  // the warp's rows as 16-byte pieces: piece t of the block is row t / 8, bytes 16 (t % 8)
  for (int t = lane; t < nr * 8; t += 32) {
    const int r = t >> 3, c = (t & 7) * 16;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(st + r * kDqStride + c)),
                 "l"(q + (size_t)(row0 + r) * 128 + c)
                 : "memory");
  }
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
  __syncwarp();
  if (lane < nr) {
    const uint8_t* rr = st + lane * kDqStride;
    float s = 0.0f;
#pragma unroll 2
    for (int c = 0; c < 8; ++c) {
      const uint4 w = *reinterpret_cast<const uint4*>(rr + 16 * c);
      const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float4 v = dq4(ws[k]);
        s += v.x * v.x;
        s += v.y * v.y;
        s += v.z * v.z;
        s += v.w * v.w;
      }
    }
    const float norm = sqrtf(s);
    inv_s[warp][lane] = norm > 1e-7f ? 1.0f / norm : 1.0f;  // 1: the row is kept as it is
  }
  __syncwarp();
  for (int r = 0; r < nr; ++r) {
    float4 v = dq4(*reinterpret_cast<const uint32_t*>(st + r * kDqStride + 4 * lane));
    const float inv = inv_s[warp][r];
    if (inv != 1.0f) {
      v.x *= inv;
      v.y *= inv;
      v.z *= inv;
      v.w *= inv;
    }
    reinterpret_cast<float4*>(out + (size_t)(row0 + r) * 128)[lane] = v;
  }
}

// Votes: one block per entry, each thread owns queries tid, tid+blockDim, ...
// The entry's signatures are read in the same order by every lane (broadcast
// loads from L1); a query stops at its first qualifying signature.
__global__ void __launch_bounds__(256) votes_kernel(const uint4* __restrict__ q, int nq, const uint4* __restrict__ cat,
                                                     const long long* __restrict__ offsets, int mih,
                                                     uint32_t* __restrict__ votes) {
  const int e = blockIdx.x;
  const long long s0 = offsets[e], s1 = offsets[e + 1];
  uint32_t hits = 0;
  for (int qi = threadIdx.x; qi < nq; qi += blockDim.x) {
    const uint4 qq = q[qi];
    for (long long s = s0; s < s1; ++s) {
      const uint4 c = cat[s];
      const uint32_t x0 = qq.x ^ c.x, x1 = qq.y ^ c.y, x2 = qq.z ^ c.z, x3 = qq.w ^ c.w;
      const int d = popc4(x0, x1, x2, x3);
      if (d <= 24 && (!mih || has_zero_byte(x0) || has_zero_byte(x1) || has_zero_byte(x2) || has_zero_byte(x3))) {
        ++hits;
        break;
      }
    }
  }
  __shared__ uint32_t s_sum[8];
  for (int o = 16; o >= 1; o >>= 1) hits += __shfl_xor_sync(0xffffffffu, hits, o);
  if ((threadIdx.x & 31) == 0) s_sum[threadIdx.x >> 5] = hits;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_sum[w];
    votes[e] = t;
  }
}

// Per (16-query group, code chunk): the k smallest (distance, index) keys.
// Grid (n_chunks, ceil(n_groups / kHamWarps)), kHamWarps warps per block.
//
// Each query keeps its list sorted, entries [k, 64) at ~0, and maxd = the
// distance of its k-th key.  Within a chunk the codes come in increasing index,
// so every listed entry has a smaller index than the current code: a code can
// only enter when its distance is below maxd.  Such codes are appended to the
// query's buffer (up to kTopKBuf keys); a full buffer (and the buffer at the end
// of the chunk) is merged into the list: the buffer sorted across the warp's
// lanes, each key's place in the merged order found by binary search in the
// other sorted sequence (ties: the list's key first; only the empty ~0 keys tie),
// the first k kept.  A candidate that passed against an older maxd and no longer
// belongs falls out at its merge.
constexpr int kTopKBuf = 32;
constexpr size_t kTopKWarpSmem = (size_t)kQG * (kTopKMax + kTopKBuf) * 8 + kTopKMax * 8 + kQG * 4;

__device__ __forceinline__ unsigned long long shfl_xor_u64(unsigned long long v, int o) {
  return __shfl_xor_sync(0xffffffffu, v, o);
}

// Merges buf[0..n) into the sorted list (k entries kept); returns the new k-th distance.
__device__ __forceinline__ uint32_t topk_merge_buffer(unsigned long long* list, unsigned long long* buf, int n,
                                                      int k, unsigned long long* scratch, int lane) {
  __syncwarp();
  // sort the buffer across the lanes (ascending; missing entries ~0)
  unsigned long long v = lane < n ? buf[lane] : ~0ull;
#pragma unroll
  for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
    for (int j = kk >> 1; j > 0; j >>= 1) {
      const unsigned long long o = shfl_xor_u64(v, j);
      const bool up = (lane & kk) == 0, low = (lane & j) == 0;
      v = (low == up) ? (o < v ? o : v) : (o > v ? o : v);
    }
  }
  buf[lane] = v;
  __syncwarp();
  // buffer key at lane: rank = lane + (list keys <= it)
  {
    int lo = 0, hi = kTopKMax;  // first list index with key > v
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (list[mid] <= v) lo = mid + 1;
      else hi = mid;
    }
    const int r = lane + lo;
    if (r < k) scratch[r] = v;
  }
  // list keys at lane and lane + 32: rank = i + (buffer keys < it)
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int i = lane + 32 * h;
    const unsigned long long x = list[i];
    int lo = 0, hi = 32;  // first buffer index with key >= x
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (buf[mid] < x) lo = mid + 1;
      else hi = mid;
    }
    const int r = i + lo;
    if (r < k) scratch[r] = x;
  }
  __syncwarp();
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int i = lane + 32 * h;
    if (i < k) list[i] = scratch[i];
  }
  __syncwarp();
  return (uint32_t)(list[k - 1] >> 32);
}

__global__ void __launch_bounds__(kHamWarps * 32, 4) topk_chunk_kernel(const uint4* __restrict__ q, int nq,
                                                                        const uint4* __restrict__ cat, long long ncat,
                                                                        int k, int n_chunks,
                                                                        unsigned long long* __restrict__ part) {
  extern __shared__ __align__(16) unsigned long long s_topk[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int group = blockIdx.y * kHamWarps + warp;
  const int q0 = group * kQG;
  if (q0 >= nq) return;
  const int chunk = blockIdx.x;
  const long long c_begin = ncat * chunk / n_chunks, c_end = ncat * (chunk + 1) / n_chunks;
  unsigned long long* wbase = s_topk + (size_t)warp * (kTopKWarpSmem / 8);
  unsigned long long(*list)[kTopKMax] = reinterpret_cast<unsigned long long(*)[kTopKMax]>(wbase);
  unsigned long long(*buf)[kTopKBuf] = reinterpret_cast<unsigned long long(*)[kTopKBuf]>(wbase + kQG * kTopKMax);
  unsigned long long* scratch = wbase + kQG * (kTopKMax + kTopKBuf);
  uint32_t* cnt = reinterpret_cast<uint32_t*>(scratch + kTopKMax);
  uint32_t qw[kQG][4];
#pragma unroll
  for (int j = 0; j < kQG; ++j) {
    const uint4 v = (q0 + j < nq) ? q[q0 + j] : make_uint4(0, 0, 0, 0);
    qw[j][0] = v.x;
    qw[j][1] = v.y;
    qw[j][2] = v.z;
    qw[j][3] = v.w;
  }
  uint32_t maxd[kQG];
#pragma unroll
  for (int j = 0; j < kQG; ++j) {
    list[j][lane] = ~0ull;
    list[j][lane + 32] = ~0ull;
    maxd[j] = 0xFFFFFFFFu;
  }
  if (lane < kQG) cnt[lane] = 0;
  __syncwarp();
  const unsigned lt = (1u << lane) - 1u;
  // the next 32 codes are loaded while the current ones are compared
  uint4 c_next = c_begin + lane < c_end ? cat[c_begin + lane] : make_uint4(0, 0, 0, 0);
  for (long long base = c_begin; base < c_end; base += 32) {
    const long long idx = base + lane;
    const bool valid = idx < c_end;
    const uint4 c = c_next;
    c_next = idx + 32 < c_end ? cat[idx + 32] : make_uint4(0, 0, 0, 0);
#pragma unroll
    for (int j = 0; j < kQG; ++j) {
      const uint32_t d = (uint32_t)ham128(qw[j][0], qw[j][1], qw[j][2], qw[j][3], c);
      const unsigned m = __ballot_sync(0xffffffffu, valid && d < maxd[j]);
      if (m) {
        const int nc = __popc(m);
        int n = (int)cnt[j];
        if (n + nc > kTopKBuf) {
          maxd[j] = topk_merge_buffer(list[j], buf[j], n, k, scratch, lane);
          n = 0;
        }
        if (m & (1u << lane))
          buf[j][n + __popc(m & lt)] = ((unsigned long long)d << 32) | (unsigned long long)(uint32_t)idx;
        __syncwarp();
        if (lane == 0) cnt[j] = (uint32_t)(n + nc);
        __syncwarp();
      }
    }
  }
  // the buffers' last keys, then this chunk's lists: part[(query * n_chunks + chunk) * k + t]
#pragma unroll
  for (int j = 0; j < kQG; ++j) {
    if (cnt[j] > 0) topk_merge_buffer(list[j], buf[j], (int)cnt[j], k, scratch, lane);
    if (q0 + j >= nq) continue;
    unsigned long long* dst = part + ((long long)(q0 + j) * n_chunks + chunk) * k;
    for (int t = lane; t < k; t += 32) dst[t] = list[j][t];
  }
}

// Ascending bitonic sort of a[0..m) (m a power of two) by one warp.
__device__ __forceinline__ void warp_bitonic_u64(unsigned long long* a, int m, int lane) {
  for (int kk = 2; kk <= m; kk <<= 1) {
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < m; i += 32) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long x = a[i], y = a[ixj];
          const bool up = (i & kk) == 0;
          if ((x > y) == up) {
            a[i] = y;
            a[ixj] = x;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Per query (one warp): the k smallest of the chunks' n_chunks * k keys
// (distance << 32 | index; empty slots ~0), ascending.  Keys are unique apart
// from the empty slots (the chunks partition the catalog).  A histogram of the
// distances (0..128, bin 129 for empty slots) gives the distance D of the k-th
// smallest key and the count `below` of keys under D (< k).  Those keys are
// compacted into `low`, the keys at D into the front of `keys` (in place: a
// round writes only at or below the positions it has read), each group is
// sorted, and the result is low[0..below) followed by the first k - below keys
// at D, i.e. by index.  Shared memory per warp: keys[n2], low[64], hist[132].
constexpr int kMergeBins = 130;
constexpr int kMergeHist = 132;
__global__ void topk_merge_kernel(const unsigned long long* __restrict__ part, int nq, int k, int n_chunks, int n2,
                                  uint32_t* __restrict__ out_idx, uint32_t* __restrict__ out_dist) {
  extern __shared__ unsigned long long s_keys[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int qi = blockIdx.x * (blockDim.x >> 5) + warp;
  unsigned long long* keys = s_keys + (size_t)warp * (n2 + kTopKMax + kMergeHist / 2);
  unsigned long long* low = keys + n2;
  uint32_t* hist = reinterpret_cast<uint32_t*>(low + kTopKMax);
  if (qi >= nq) return;
  const int total = n_chunks * k;
  const unsigned long long* src = part + (long long)qi * total;
  for (int t = lane; t < kMergeHist; t += 32) hist[t] = 0;
  for (int t = lane; t < total; t += 32) keys[t] = src[t];
  __syncwarp();
  auto bin_of = [](unsigned long long key) {
    const uint32_t d = (uint32_t)(key >> 32);
    return d <= 128u ? (int)d : kMergeBins - 1;
  };
  for (int t = lane; t < total; t += 32) atomicAdd(&hist[bin_of(keys[t])], 1u);
  __syncwarp();
  // D: the bin where the running count reaches k (lane l scans bins 5l .. 5l + 4)
  int local = 0;
#pragma unroll
  for (int b = 0; b < 5; ++b) local += 5 * lane + b < kMergeBins ? (int)hist[5 * lane + b] : 0;
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const int excl = incl - local;
  int my_d = -1, my_below = 0;
  if (excl < k && incl >= k) {
    int run = excl;
    for (int b = 5 * lane; b < 5 * lane + 5; ++b) {
      const int c = (int)hist[b];
      if (run + c >= k) {
        my_d = b;
        my_below = run;
        break;
      }
      run += c;
    }
  }
  const int owner = __ffs(__ballot_sync(0xffffffffu, my_d >= 0)) - 1;
  const int D = __shfl_sync(0xffffffffu, my_d, owner);
  const int below = __shfl_sync(0xffffffffu, my_below, owner);
  const int n_tie = (int)hist[D];
  // compaction, in key order of the chunks
  int n_low = 0, n_at = 0;
  const unsigned lt = (1u << lane) - 1u;
  for (int base = 0; base < total; base += 32) {
    const int t = base + lane;
    const unsigned long long key = t < total ? keys[t] : ~0ull;
    const int b = t < total ? bin_of(key) : kMergeBins;
    const unsigned ml = __ballot_sync(0xffffffffu, b < D);
    const unsigned mt = __ballot_sync(0xffffffffu, b == D);
    __syncwarp();
    if (b < D) low[n_low + __popc(ml & lt)] = key;
    if (b == D) keys[n_at + __popc(mt & lt)] = key;
    n_low += __popc(ml);
    n_at += __popc(mt);
    __syncwarp();
  }
  // sort the group under D (padded to a power of two) and, unless they are all
  // empty slots, the keys at D
  int m = 1;
  while (m < below) m <<= 1;
  for (int t = below + lane; t < m; t += 32) low[t] = ~0ull;
  int m2 = 1;
  while (m2 < n_tie) m2 <<= 1;
  const bool sort_tie = D < kMergeBins - 1 && n_tie > 1;
  if (sort_tie)
    for (int t = n_tie + lane; t < m2; t += 32) keys[t] = ~0ull;
  __syncwarp();
  if (below > 1) warp_bitonic_u64(low, m, lane);
  if (sort_tie) warp_bitonic_u64(keys, m2, lane);
  for (int t = lane; t < k; t += 32) {
    const unsigned long long key = t < below ? low[t] : keys[t - below];
    const bool ok = key != ~0ull;
    out_idx[(long long)qi * k + t] = ok ? (uint32_t)(key & 0xFFFFFFFFu) : 0xFFFFFFFFu;
    out_dist[(long long)qi * k + t] = ok ? (uint32_t)(key >> 32) : 0xFFFFFFFFu;
  }
}

// Exact FP32 L2^2 re-rank of each query's k candidates (reference summation
// order), sorted by (d2, index).  One warp per query.
__global__ void l2_rerank_kernel(const float* __restrict__ qd, int nq, const float* __restrict__ cd,
                                 const uint32_t* __restrict__ cand, int k, uint32_t* __restrict__ out_idx,
                                 float* __restrict__ out_d2) {
  __shared__ unsigned long long s_keys[8][kTopKMax];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int qi = blockIdx.x * 8 + warp;
  if (qi >= nq) return;
  unsigned long long* keys = s_keys[warp];
  const float* a = qd + (size_t)qi * 128;
  for (int t = lane; t < kTopKMax; t += 32) {
    unsigned long long key = ~0ull;
    if (t < k) {
      const uint32_t c = cand[(long long)qi * k + t];
      if (c != 0xFFFFFFFFu) {
        const float* b = cd + (size_t)c * 128;
        float s = 0.0f;
        for (int i = 0; i < 128; i += 4) {
          const float4 x = *reinterpret_cast<const float4*>(a + i);
          const float4 y = *reinterpret_cast<const float4*>(b + i);
          float d = x.x - y.x;
          s += d * d;
          d = x.y - y.y;
          s += d * d;
          d = x.z - y.z;
          s += d * d;
          d = x.w - y.w;
          s += d * d;
        }
        // non-negative floats order like their bit patterns
        key = ((unsigned long long)__float_as_uint(s) << 32) | c;
      }
    }
    keys[t] = key;
  }
  __syncwarp();
  for (int kk = 2; kk <= kTopKMax; kk <<= 1) {
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < kTopKMax; i += 32) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long x = keys[i], y = keys[ixj];
          const bool up = (i & kk) == 0;
          if ((x > y) == up) {
            keys[i] = y;
            keys[ixj] = x;
          }
        }
      }
      __syncwarp();
    }
  }
  for (int t = lane; t < k; t += 32) {
    const unsigned long long key = keys[t];
    const bool ok = key != ~0ull;
    out_idx[(long long)qi * k + t] = ok ? (uint32_t)(key & 0xFFFFFFFFu) : 0xFFFFFFFFu;
    out_d2[(long long)qi * k + t] = ok ? __uint_as_float((uint32_t)(key >> 32)) : __int_as_float(0x7f800000);
  }
}

cudaError_t launch_quantize(const float* desc, int n, uint64_t* codes, uint8_t* u8, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (codes) quantize_codes_kernel<<<(n + 8 * kQDesc - 1) / (8 * kQDesc), 256, 0, st>>>(desc, n, codes);
  if (u8) quantize_kernel<<<(n + 7) / 8, 256, 0, st>>>(desc, n, nullptr, u8);
  return cudaGetLastError();
}

cudaError_t launch_dequantize(const uint8_t* q, int n, float* out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  dequantize_kernel<<<(n + 32 * kDqWarps - 1) / (32 * kDqWarps), 32 * kDqWarps, 0, st>>>(q, n, out);
  return cudaGetLastError();
}

cudaError_t launch_votes(const uint64_t* q, int nq, const uint64_t* cat, const long long* offsets, int n_entries,
                         int mih, uint32_t* votes, cudaStream_t st) {
  if (n_entries <= 0) return cudaSuccess;
  votes_kernel<<<n_entries, 256, 0, st>>>((const uint4*)q, nq, (const uint4*)cat, offsets, mih, votes);
  return cudaGetLastError();
}

int topk_chunks(long long ncat, int nq, int num_sms) {
  const int groups = (nq + kQG - 1) / kQG;
  long long want = (long long)num_sms * 16 * 2 / std::max(groups, 1);  // ~2 waves of 16 warps per SM
  want = std::max<long long>(1, std::min<long long>(want, 64));
  want = std::min<long long>(want, std::max<long long>(1, ncat / 1024));
  return (int)want;
}

cudaError_t launch_topk(const uint64_t* q, int nq, const uint64_t* cat, long long ncat, int k, int n_chunks,
                        unsigned long long* part, uint32_t* out_idx, uint32_t* out_dist, cudaStream_t st) {
  if (nq <= 0) return cudaSuccess;
  const int groups = (nq + kQG - 1) / kQG;
  dim3 g1(n_chunks, (groups + kHamWarps - 1) / kHamWarps);
  const size_t smem1 = kHamWarps * kTopKWarpSmem;
  cudaError_t e = ensure_smem_attr((const void*)topk_chunk_kernel, smem1);
  if (e != cudaSuccess) return e;
  topk_chunk_kernel<<<g1, kHamWarps * 32, smem1, st>>>((const uint4*)q, nq, (const uint4*)cat, ncat, k, n_chunks,
                                                      part);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  int n2 = 1;
  while (n2 < n_chunks * k) n2 <<= 1;
  const size_t per_warp = ((size_t)n2 + kTopKMax + kMergeHist / 2) * 8;
  const int warps = std::max(1, std::min(8, (int)(96 * 1024 / per_warp)));
  const size_t smem = (size_t)warps * per_warp;
  e = ensure_smem_attr((const void*)topk_merge_kernel, smem);
  if (e != cudaSuccess) return e;
  topk_merge_kernel<<<(nq + warps - 1) / warps, warps * 32, smem, st>>>(part, nq, k, n_chunks, n2, out_idx, out_dist);
  return cudaGetLastError();
}

// Throughput probe for the INT roofline of the Hamming kernels: every thread
// keeps 8 independent 32-bit popcount chains in registers (no memory traffic in
// the loop); the sum is stored so nothing is dead code.
__global__ void __launch_bounds__(256) popc_probe_kernel(uint32_t seed, int iters, uint32_t* out) {
  uint32_t v[8], acc[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    v[j] = seed * (threadIdx.x + 1u) + 0x9E3779B9u * (uint32_t)(j + 1) + blockIdx.x;
    acc[j] = 0;
  }
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      acc[j] += __popc(v[j]);
      v[j] ^= acc[j];
    }
  }
  uint32_t t = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) t += acc[j];
  out[blockIdx.x * blockDim.x + threadIdx.x] = t;
}

cudaError_t launch_popc_probe(int blocks, int iters, uint32_t* out, cudaStream_t st) {
  popc_probe_kernel<<<blocks, 256, 0, st>>>(12345u, iters, out);
  return cudaGetLastError();
}

cudaError_t launch_l2_rerank(const float* qd, int nq, const float* cd, const uint32_t* cand, int k,
                             uint32_t* out_idx, float* out_d2, cudaStream_t st) {
  if (nq <= 0) return cudaSuccess;
  l2_rerank_kernel<<<(nq + 7) / 8, 256, 0, st>>>(qd, nq, cd, cand, k, out_idx, out_d2);
  return cudaGetLastError();
}

}  // namespace psift
