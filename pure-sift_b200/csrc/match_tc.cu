// K8: BF16 tcgen05 distance GEMM with a fused top-8 epilogue, and the certified
// exact FP32 re-rank that makes its match list identical to the FP32 path.
//
// Reference: match_descriptors_with_options (src/pipeline.rs:1744-1841).
//
// Scheme.  The GEMM carries the target norms in one extra K step: the A
// operand's extension is [1, 1, 0, ...] and the B operand's [h_j, l_j, 0, ...]
// with h_j + l_j the bf16 hi/lo split of -|t_j|^2 / 2, so the accumulator is
//   D_ij = <bf16(q_i), bf16(t_j)> + h_j + l_j  (f32 accumulation in TMEM)
// and a_ij = |q_i|^2 - 2 D_ij (one f32 rounding) approximates the reference's
// f32 squared distance d_ij with
//   |a_ij - d_ij| <= eps_i = 0.008 |q_i| max_j|t_j| + 7e-5 (|q_i|^2 + max_j|t_j|^2) + 1e-6
// (bf16 rounding of both operands <= 2^-8 relative per product, the hi/lo split
// of the norm <= 2^-18 relative, tensor-core f32 accumulation, the f32 norms and
// the reference's own sequential f32 rounding, all bounded with margin).  a_ij
// is a non-increasing function of D_ij, so a row's two smallest a are the
// images of its two largest D, and the epilogue works on D alone.  Every target
// that can be the exact best or second has a_ij <= a_(2) + 2 eps_i.  Pass 1 of
// the GEMM keeps each row's two largest D; window_kernel either certifies that
// the row fails the ratio test (then no exact work is needed) or sets the row's
// window thr = a_(2) + 2 eps_i; pass 2 (same GEMM, deterministic) collects every
// index whose D is at least (|q_i|^2 - thr) / 2 less a margin that covers the
// rounding of a (a superset of {a_ij <= thr}), and the exact reference distances
// of those candidates give best/second/index equal to the FP32 path bit for bit.
// A row whose window holds more than kColl indices in one split (or more than
// kXColl in one column part) is matched by an exact scan of all targets.
//
// Kernel structure (one CTA = one 128-row A tile x a range of 256-row B tiles,
// 576 threads): warp 0 issues TMA loads (SWIZZLE_128B, two 64-column boxes per
// operand tile plus the 16-column norm extension with SWIZZLE_32B,
// double-buffered B), warp 1 owns TMEM (512 columns = two 128x256 f32
// accumulators) and issues tcgen05.mma (M=128, N=256, K=16; nine per tile) from
// one thread, warps 2-17 read the accumulators with tcgen05.ld (four warps per
// TMEM lane quarter, one per 64-column part of the tile; the parts are merged per
// row at the end).  All waits are bounded: on timeout the CTA records
// kErrTimeout, stops issuing, drains what it issued and frees its TMEM.
#include <cuda.h>

#include "match_common.cuh"
#include "psift_internal.cuh"

namespace psift {

constexpr int kEpiParts = 4;                    // epilogue warps per TMEM lane quarter (column parts)
constexpr int kEpiWarps = 4 * kEpiParts;        // warps 2 .. 2 + kEpiWarps - 1
constexpr int kTcThreads = 32 * (2 + kEpiWarps);  // warp 0 TMA, warp 1 MMA, then the epilogue
static_assert(256 / kEpiParts == 64, "the epilogue folds four 16-column TMEM loads per part");
constexpr int kBM = 128;
constexpr int kBN = 256;
constexpr uint32_t kSpinLimit = 1u << 25;
constexpr int kColl = 32;   // window indices kept per (split, row)
constexpr int kXColl = 16;  // window indices a column part 1..3 hands to part 0 (more: exact scan)

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait; false on timeout or when the CTA is aborting.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255u) == 255u && *abort_flag) return false;
  }
  return false;
}
__device__ __forceinline__ void tma_load_2d(const CUtensorMap* tm, uint64_t* bar, void* dst, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major, 128-byte-swizzled operand tile: rows of 128 B, 8-row atoms 1024 B apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);  // start address
  d |= (uint64_t)1 << 16;                    // leading byte offset (unused when swizzled)
  d |= (uint64_t)(1024u >> 4) << 32;         // stride byte offset: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                    // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                    // SWIZZLE_128B
  return d;
}

// K-major, 32-byte-swizzled 16-column extension tile: rows of 32 B, 8-row atoms 256 B apart.
__device__ __forceinline__ uint64_t sw32_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);  // start address
  d |= (uint64_t)1 << 16;                    // leading byte offset (unused: one swizzle atom wide)
  d |= (uint64_t)(256u >> 4) << 32;          // stride byte offset: 8 rows x 32 B
  d |= (uint64_t)1 << 46;                    // descriptor version (sm_100)
  d |= (uint64_t)6 << 61;                    // SWIZZLE_32B
  return d;
}

// kind::f16 instruction descriptor: D f32, A/B bf16, both K-major, M=128, N=256.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                            ((uint32_t)(kBM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 16 columns of a TMEM lane quarter, without waiting: the registers are valid
// only after tmem_wait16 on them.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr));
}
// Waits for this thread's outstanding TMEM loads; r is tied so that no read of
// it moves above the wait.
__device__ __forceinline__ void tmem_wait16(uint32_t (&r)[16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
}

// Smem map (offsets from a 1024-aligned base).
constexpr uint32_t kSmA = 0;                      // 2 halves x 128 rows x 128 B = 32 KB
constexpr uint32_t kSmAx = 32768;                 // A norm extension: 128 rows x 32 B
constexpr uint32_t kSmB = 36864;                  // 2 stages of: 2 halves x 256 rows x 128 B, then 256 x 32 B
constexpr uint32_t kSmBStage = 65536 + 8192;
constexpr uint32_t kSmBar = kSmB + 2 * kSmBStage;  // barriers
// epilogue exchange, per row and column part 1..kEpiParts-1: pass 1 the part's two
// largest values, pass 2 its count and up to kXColl indices
constexpr uint32_t kSmX = kSmBar + 256;
constexpr uint32_t kSmTotal = kSmX + (kEpiParts - 1) * kBM * (kXColl + 2) * 4 + 1024;  // + alignment slack
static_assert(kSmTotal <= 227 * 1024, "shared memory per CTA");

__global__ void __launch_bounds__(kTcThreads, 1)
    match_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    const __grid_constant__ CUtensorMap tmAx, const __grid_constant__ CUtensorMap tmBx,
                    const TcItem* __restrict__ items, const TcPair* __restrict__ pairs, uint32_t* err, int mode) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kSmBar);  // [2]
  uint64_t* empty = full + 2;                                    // [2]
  uint64_t* afull = full + 4;                                    // [1]
  uint64_t* accf = full + 5;                                     // [2]
  uint64_t* acce = full + 7;                                     // [2]
  volatile uint32_t* taddr_slot = reinterpret_cast<volatile uint32_t*>(full + 9);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(full + 10);

  const TcItem it = items[blockIdx.x];
  const TcPair& PR = pairs[it.pair];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // pass 2 over the compacted rows: a tile past the kept rows has nothing to do
  const bool compact = mode == 1 && PR.ccount != nullptr;
  const int n_rows = compact ? *PR.ccount : PR.na;
  if (it.a_local >= n_rows) return;

  if (threadIdx.x == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    mbar_init(&empty[0], 1);
    mbar_init(&empty[1], 1);
    mbar_init(afull, 1);
    mbar_init(&accf[0], 1);
    mbar_init(&accf[1], 1);
    mbar_init(&acce[0], kEpiWarps);
    mbar_init(&acce[1], kEpiWarps);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32((const void*)taddr_slot)),
                 "r"(512u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *taddr_slot;
  const int nt = it.n_tiles;
  // epilogue row state (warps 2..9)
  const int quarter = warp & 3;
  const int part = warp >= 2 ? (warp - 2) >> 2 : 0;  // column part of the tile
  const int row = quarter * 32 + lane;
  // the row's index in the pair (through the row map when the operand is compacted)
  const bool row_ok = it.a_local + row < n_rows;
  const int a_local = compact ? (row_ok ? PR.rowmap[it.a_local + row] : 0) : it.a_local + row;
  const float inf = __int_as_float(0x7f800000);
  float u0 = -inf, u1 = -inf;  // mode 0: the two largest D of the row
  int cnt = 0;                 // mode 1: indices with D >= the row's window bound
  // exchange slot of (part, row) for parts >= 1
  int* xrow = reinterpret_cast<int*>(smem + kSmX) + ((part > 0 ? part - 1 : 0) * kBM + row) * (kXColl + 2);

  if (warp == 0) {
    if (lane == 0) {
      // A tile: two 64-column boxes of 128 rows and the constant norm extension
      mbar_expect_tx(afull, 2u * kBM * 128u + kBM * 32u);
      tma_load_2d(&tmA, afull, smem + kSmA, 0, it.a_row);
      tma_load_2d(&tmA, afull, smem + kSmA + kBM * 128, 64, it.a_row);
      tma_load_2d(&tmAx, afull, smem + kSmAx, 0, 0);
      for (int j = 0; j < nt; ++j) {
        const int s = j & 1;
        const uint32_t use = (uint32_t)(j >> 1);
        if (!mbar_wait(&empty[s], (use & 1u) ^ 1u, abort_flag)) {
          atomicOr(err, kErrTimeout);
          *abort_flag = 1;
          break;
        }
        uint8_t* bst = smem + kSmB + s * kSmBStage;
        mbar_expect_tx(&full[s], 2u * kBN * 128u + kBN * 32u);
        tma_load_2d(&tmB, &full[s], bst, 0, it.b_row + j * kBN);
        tma_load_2d(&tmB, &full[s], bst + kBN * 128, 64, it.b_row + j * kBN);
        tma_load_2d(&tmBx, &full[s], bst + 2 * kBN * 128, 0, it.b_row + j * kBN);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int issued = 0;
      bool ok = mbar_wait(afull, 0, abort_flag);
      for (int j = 0; ok && j < nt; ++j) {
        const int s = j & 1;
        const uint32_t use = (uint32_t)(j >> 1);
        if (!mbar_wait(&full[s], use & 1u, abort_flag) || !mbar_wait(&acce[s], (use & 1u) ^ 1u, abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t a_base = smem_u32(smem + kSmA);
        const uint32_t b_base = smem_u32(smem + kSmB + s * kSmBStage);
        const uint32_t d = tmem + (uint32_t)(s * kBN);
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
          const uint32_t half = (uint32_t)(kk >> 2), koff = (uint32_t)(kk & 3) * 32u;
          umma_bf16(d, sw128_desc(a_base + half * (kBM * 128) + koff), sw128_desc(b_base + half * (kBN * 128) + koff),
                    kk > 0 ? 1u : 0u);
        }
        // the norm extension: D += h_j + l_j
        umma_bf16(d, sw32_desc(smem_u32(smem + kSmAx)), sw32_desc(b_base + 2 * kBN * 128), 1u);
        umma_commit(&empty[s]);
        umma_commit(&accf[s]);
        ++issued;
      }
      if (!ok) {
        atomicOr(err, kErrTimeout);
        *abort_flag = 1;
        // drain: wait (bounded, ignoring the abort flag) for the last issued MMA group
        if (issued > 0) {
          const int j = issued - 1;
          const int s = j & 1;
          const uint32_t use = (uint32_t)(j >> 1);
          for (uint32_t i = 0; i < kSpinLimit && !mbar_try_wait(&accf[s], use & 1u); ++i) {
          }
        }
      }
    }
  } else {
    // epilogue: TMEM lane quarter warp % 4, column part (warp - 2) / 4
    const float an = row_ok ? PR.an[a_local] : 0.0f;
    const float thr = (mode == 1 && row_ok) ? PR.thr[a_local] : -inf;
    // pass 2 window in D: every D with |q|^2 - 2 D <= thr (one f32 rounding) has
    // D >= (|q|^2 - thr) / 2 - 2^-24 (|q|^2 + |thr|); the margin below is larger
    const float dthr = thr == -inf ? inf : 0.5f * (an - thr) - 1e-6f * (fabsf(an) + fabsf(thr));
    // part 0 collects into the row's list, the other parts into their exchange slots
    int* coll = part == 0 ? PR.coll_idx + ((long long)it.split * PR.na + (row_ok ? a_local : 0)) * kColl
                          : xrow + 2;
    const int ccap = part == 0 ? kColl : kXColl;
    for (int j = 0; j < nt; ++j) {
      const int s = j & 1;
      const uint32_t use = (uint32_t)(j >> 1);
      if (!mbar_wait(&accf[s], use & 1u, abort_flag)) {
        atomicOr(err, kErrTimeout);
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(s * kBN);
      const int col0 = it.b_local + j * kBN;
      // This warp's 64 columns as four 16-column TMEM loads, double-buffered: the
      // next load is in flight while the current 16 values are folded in.
      const int cbase = col0 + part * (kBN / kEpiParts);
      const uint32_t tbase = taddr + (uint32_t)(part * (kBN / kEpiParts));
      auto fold16 = [&](const uint32_t(&rr)[16], int cstart) {
        if (mode == 0) {
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const float d = __uint_as_float(rr[q]);
            const float lo = fminf(u0, d);
            u0 = fmaxf(u0, d);
            u1 = fmaxf(u1, lo);
          }
        } else {
          // the tests branch-free into a mask, then the (rare) hits in column order
          uint32_t hits = 0;
#pragma unroll
          for (int q = 0; q < 16; ++q) hits |= (__uint_as_float(rr[q]) >= dthr ? 1u : 0u) << q;
          // a row past the kept ones reads stale operand rows: it collects nothing
          if (!row_ok) hits = 0;
          while (hits) {
            const int q = __ffs(hits) - 1;
            hits &= hits - 1;
            if (cnt < ccap) coll[cnt] = cstart + q;
            ++cnt;
          }
        }
      };
      uint32_t ra[16], rb[16];
      __syncwarp();
      tmem_ld16(tbase, ra);
      tmem_wait16(ra);
      tmem_ld16(tbase + 16, rb);
      fold16(ra, cbase);
      tmem_wait16(rb);
      tmem_ld16(tbase + 32, ra);
      fold16(rb, cbase + 16);
      tmem_wait16(ra);
      tmem_ld16(tbase + 48, rb);
      fold16(ra, cbase + 32);
      tmem_wait16(rb);
      fold16(rb, cbase + 48);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[s]);
    }
    if (part > 0) {
      if (mode == 0) {
        xrow[0] = __float_as_int(u0);
        xrow[1] = __float_as_int(u1);
      } else {
        xrow[0] = cnt;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  // Part 0 merges the other parts into its row, in part order: the two largest D
  // of all, mapped to the two smallest a = |q|^2 - 2 D (pass 1), or the
  // concatenated index lists with the summed count (pass 2; a count above kColl,
  // or a part that overflowed its kXColl slots, sends the row to the exact scan).
  if (warp >= 2 && part == 0 && row_ok) {
    const long long o = (long long)it.split * PR.na + a_local;
    int* coll0 = PR.coll_idx + o * kColl;
    bool part_overflow = false;
    for (int p = 1; p < kEpiParts; ++p) {
      const int* x = reinterpret_cast<const int*>(smem + kSmX) + ((p - 1) * kBM + row) * (kXColl + 2);
      if (mode == 0) {
        const float w0 = __int_as_float(x[0]), w1 = __int_as_float(x[1]);
        const float m1 = fmaxf(fminf(u0, w0), fmaxf(u1, w1));
        u0 = fmaxf(u0, w0);
        u1 = m1;
      } else {
        const int c1 = x[0];
        part_overflow |= c1 > kXColl;
        for (int k = 0; k < c1 && k < kXColl && cnt + k < kColl; ++k) coll0[cnt + k] = x[2 + k];
        cnt += c1;
      }
    }
    if (mode == 0) {
      const float an = PR.an[a_local];
      PR.top2[2 * o] = __fmaf_rn(-2.0f, u0, an);
      PR.top2[2 * o + 1] = __fmaf_rn(-2.0f, u1, an);
    } else {
      PR.coll_cnt[o] = part_overflow ? max(cnt, kColl + 1) : cnt;
    }
  }
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
  }
}

// ------------------------------------------------------------ bf16 operands
// One warp per row: bf16 copy (zero rows for padding are pre-cleared), exact f32
// squared norm (sequential), running max of the norms, and the row's GEMM norm
// extension [h, l, 0, ...] with h = bf16(-|x|^2 / 2), l = bf16(-|x|^2 / 2 - h);
// padding rows up to n_pad get [-inf, 0, ...], which no window or top-2 takes.
// A job with x = null writes n_pad rows of the A operand's extension [1, 1, 0, ...].
struct Bf16Job {
  const float* x;
  int n;
  uint16_t* out;
  float* norms;
  float* norm_max;
  uint16_t* ext;  // n_pad rows x 16
  int n_pad;
};

__device__ __forceinline__ uint16_t bf16_rne(float f) {
  const uint32_t u = __float_as_uint(f);
  return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}

__global__ void to_bf16_kernel(const Bf16Job* __restrict__ jobs) {
  const Bf16Job& J = jobs[blockIdx.y];
  const float* __restrict__ x = J.x;
  uint16_t* __restrict__ out = J.out;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (!x) {
    // the A operand's constant extension rows [1, 1, 0, ...]
    if (row < J.n_pad && lane < 4)
      reinterpret_cast<uint2*>(J.ext + (size_t)row * 16)[lane] = make_uint2(lane == 0 ? 0x3F803F80u : 0u, 0u);
    return;
  }
  if (row >= J.n) {
    if (row < J.n_pad && lane < 4)
      reinterpret_cast<uint2*>(J.ext + (size_t)row * 16)[lane] = make_uint2(lane == 0 ? 0xFF80u : 0u, 0u);
    return;
  }
  const float4 v = reinterpret_cast<const float4*>(x + (size_t)row * 128)[lane];
  const float e[4] = {v.x, v.y, v.z, v.w};
  unsigned short b[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) b[i] = bf16_rne(e[i]);  // round to nearest even
  uint2 packed;
  packed.x = (uint32_t)b[0] | ((uint32_t)b[1] << 16);
  packed.y = (uint32_t)b[2] | ((uint32_t)b[3] << 16);
  reinterpret_cast<uint2*>(out + (size_t)row * 128)[lane] = packed;
  // exact sequential norm: lane 0 gathers the 128 values in order
  float s = 0.0f;
  for (int i = 0; i < 128; ++i) {
    const float xi = __shfl_sync(0xffffffffu, e[i & 3], i >> 2);
    s += xi * xi;
  }
  if (lane == 0) {
    J.norms[row] = s;
    atomicMax(reinterpret_cast<unsigned int*>(J.norm_max), __float_as_uint(s));
  }
  if (lane < 4) {
    uint2 w = make_uint2(0u, 0u);
    if (lane == 0) {
      const float half = -0.5f * s;  // exact
      const uint16_t hi = bf16_rne(half);
      const uint16_t lo = bf16_rne(half - __uint_as_float((uint32_t)hi << 16));
      w.x = (uint32_t)hi | ((uint32_t)lo << 16);
    }
    reinterpret_cast<uint2*>(J.ext + (size_t)row * 16)[lane] = w;
  }
}

// Exact reference distance between two descriptors (sequential order).
__device__ __forceinline__ float exact_d2(const float* __restrict__ a, const float* __restrict__ b) {
  float s = 0.0f;
#pragma unroll 4
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
  return s;
}

// Per A row (thread): merge the splits' two smallest values, certify rejection
// or set the candidate window thr = a_(2) + 2 eps (forward) / a_(1) + 2 eps (reverse).
__global__ void window_kernel(const RerankJob* __restrict__ jobs) {
  const RerankJob& J = jobs[blockIdx.y];
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= J.na) return;
  const bool forward = J.second != nullptr;
  const float inf = __int_as_float(0x7f800000);
  float v0 = inf, v1 = inf;
  for (int s = 0; s < J.splits; ++s) {
    const long long o = (long long)s * J.na + row;
    const float a = J.top2[2 * o], b = J.top2[2 * o + 1];
    // union multiset of {v0, v1} and {a, b}: two smallest
    const float lo = fminf(v0, a), hi = fmaxf(v0, a);
    v1 = fminf(fminf(v1, b), hi);
    v0 = lo;
  }
  const float an = J.an[row];
  const float bmax = *J.bn_max;
  const float eps = 0.008f * sqrtf(an) * sqrtf(bmax) + 7e-5f * (an + bmax) + 1e-6f;
  float thr = (forward ? v1 : v0) + 2.0f * eps;
  if (!forward && J.flags && J.flags[row] == 0) thr = -inf;
  if (forward && v1 < inf) {
    // Certified rejection: exact d1 >= a_(1) - eps and exact d2 <= a_(2) + eps, so
    // if (a_(1) - eps) >= R^2 (a_(2) + eps)(1 + 1e-5) the reference's
    // sqrt(d1)/sqrt(d2) (three f32 roundings) is >= R and the query has no match.
    const double lo1 = (double)v0 - (double)eps;
    const double hi2 = (double)v1 + (double)eps;
    const double r = (double)J.ratio;
    if (lo1 > 0.0 && lo1 >= r * r * hi2 * (1.0 + 1e-5)) thr = -inf;
  }
  J.thr[row] = thr;
  // rows with a window go to pass 2 (compacted; the order does not matter: every
  // row's collection depends on that row alone and lands in its own slot)
  if (J.ccount && thr != -inf) J.rowmap[atomicAdd(J.ccount, 1)] = row;
}

// One warp per compacted row: its 256 bytes of bf16 descriptor, coalesced.
__global__ void gather_rows_kernel(const GatherJob* __restrict__ jobs) {
  const GatherJob& G = jobs[blockIdx.y];
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= *G.count) return;
  const int r = G.rowmap[c];
  reinterpret_cast<uint2*>(G.dst + (size_t)c * 128)[lane] = reinterpret_cast<const uint2*>(G.src + (size_t)r * 128)[lane];
}

// One warp per A row: exact reference distances over the window candidates
// (every index with a <= thr, collected by the second GEMM pass), or over all
// B rows when a split's window overflowed kColl.
__global__ void rerank_kernel(const RerankJob* __restrict__ jobs) {
  const RerankJob& J = jobs[blockIdx.y];
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= J.na) return;
  const bool forward = J.second != nullptr;
  const float inf = __int_as_float(0x7f800000);
  float b = inf, sec = inf;
  int bi = 0x7fffffff;
  if (J.thr[row] != -inf) {
    bool overflow = false;
    for (int s = 0; s < J.splits; ++s) overflow |= J.coll_cnt[(long long)s * J.na + row] > kColl;
    const float* arow = J.a + (size_t)row * 128;
    if (!overflow) {
      for (int s = 0; s < J.splits; ++s) {
        const long long o = (long long)s * J.na + row;
        const int c = J.coll_cnt[o];
        for (int k = lane; k < c; k += 32) {
          const int t = J.coll_idx[o * kColl + k];
          top2_push(b, bi, sec, exact_d2(arow, J.b + (size_t)t * 128), t);
        }
      }
    } else {
      if (lane == 0) atomicAdd(J.fallbacks, 1u);
      for (int t = lane; t < J.nb; t += 32) top2_push(b, bi, sec, exact_d2(arow, J.b + (size_t)t * 128), t);
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
      const float b2 = __shfl_xor_sync(0xffffffffu, b, off);
      const int i2 = __shfl_xor_sync(0xffffffffu, bi, off);
      const float s2 = __shfl_xor_sync(0xffffffffu, sec, off);
      top2_merge(b, bi, sec, b2, i2, s2);
    }
    if (forward && J.flags && lane == 0 && sec > 1e-12f && b < inf && bi < J.nb) {
      // the reference's ratio test (src/pipeline.rs:1789-1794): mark the target for the reverse pass
      if (sqrtf(b) / sqrtf(sec) < J.ratio) J.flags[bi] = 1;
    }
  }
  if (lane == 0) {
    J.best[row] = b;
    J.best_idx[row] = bi;
    if (forward) J.second[row] = sec;
  }
}

// ------------------------------------------------------------------- host
namespace {
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}
}  // namespace

// 2D bf16 tensor map over `rows` x 128, box = 64 columns x box_rows, 128B swizzle.
bool make_operand_map(CUtensorMap* tm, const void* base, long long rows, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {128, (cuuint64_t)rows};
  cuuint64_t strides[1] = {256};
  cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 2D bf16 tensor map over `rows` x 16 (the norm extension), box = 16 columns x
// box_rows, 32B swizzle.
bool make_ext_map(CUtensorMap* tm, const void* base, long long rows, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {16, (cuuint64_t)rows};
  cuuint64_t strides[1] = {32};
  cuuint32_t box[2] = {16, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_to_bf16(const void* jobs, int n_jobs, int max_rows, cudaStream_t st) {
  if (n_jobs <= 0 || max_rows <= 0) return cudaSuccess;
  dim3 grid((max_rows + 7) / 8, n_jobs);
  to_bf16_kernel<<<grid, 256, 0, st>>>((const Bf16Job*)jobs);
  return cudaGetLastError();
}

cudaError_t launch_match_tc(const CUtensorMap& tmA, const CUtensorMap& tmB, const CUtensorMap& tmAx,
                            const CUtensorMap& tmBx, const TcItem* items, int n_items, const TcPair* pairs,
                            uint32_t* err, int mode, cudaStream_t st) {
  cudaError_t e = ensure_smem_attr((const void*)match_tc_kernel, kSmTotal);
  if (e != cudaSuccess) return e;
  match_tc_kernel<<<n_items, kTcThreads, kSmTotal, st>>>(tmA, tmB, tmAx, tmBx, items, pairs, err, mode);
  return cudaGetLastError();
}

cudaError_t launch_window(const RerankJob* jobs, int n_jobs, int max_rows, cudaStream_t st) {
  dim3 grid((max_rows + 255) / 256, n_jobs);
  window_kernel<<<grid, 256, 0, st>>>(jobs);
  return cudaGetLastError();
}

cudaError_t launch_gather_rows(const GatherJob* jobs, int n_jobs, int max_rows, cudaStream_t st) {
  if (n_jobs <= 0 || max_rows <= 0) return cudaSuccess;
  dim3 grid((max_rows + 7) / 8, n_jobs);
  gather_rows_kernel<<<grid, 256, 0, st>>>(jobs);
  return cudaGetLastError();
}

cudaError_t launch_rerank(const RerankJob* jobs, int n_jobs, int max_rows, cudaStream_t st) {
  dim3 grid((max_rows + 7) / 8, n_jobs);
  rerank_kernel<<<grid, 256, 0, st>>>(jobs);
  return cudaGetLastError();
}

}  // namespace psift
