// K8: BF16 tcgen05 distance GEMM with a fused top-2 epilogue, and the certified
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
// is a non-increasing function of D_ij, so a row's smallest a are the images of
// its largest D, and the epilogue works on D alone.  Every target that can be
// the exact best or second has a_ij <= a_(2) + 2 eps_i.  Pass 1 of the GEMM keeps
// each row's largest D and a lower bound on its second largest (the second
// largest of 8 column-class maxima); window_kernel either certifies that the
// row fails the ratio test (then no exact work is needed) or sets the row's
// window thr = a'_(2) + 2 eps_i >= a_(2) + 2 eps_i; pass 2 (same GEMM,
// deterministic) collects every index whose D is at least (|q_i|^2 - thr) / 2
// less a margin that covers the rounding of a (a superset of {a_ij <= thr}), and
// the exact reference distances of those candidates give best/second/index
// equal to the FP32 path bit for bit.  A row whose window holds more than kColl
// indices in one slot (or more than kXColl in one column part) is matched by an
// exact scan of all targets.
//
// Kernel structure: persistent, one CTA per SM, 576 threads.  A pass's tiles
// (128-row A tile x 128-row B tile, ordered problem, A tile, B tile) are cut into
// equal ranges, one per CTA; each range is walked as pieces (one A tile's run of
// B tiles).  Warp 0 issues TMA loads (SWIZZLE_128B, two 64-column boxes per
// operand tile plus the 16-column norm extension with SWIZZLE_32B; A tiles
// double-buffered, B tiles in a ring of three), warp 1 owns TMEM (512 columns =
// four 128x128 f32 accumulators) and issues tcgen05.mma (M=128, N=128, K=16;
// nine per tile) from one thread, warps 2-17 read the accumulators with
// tcgen05.ld (four warps per TMEM lane quarter, one per 32-column part; the next
// tile's load in flight while the current one is folded, each accumulator
// released as soon as it is in registers; the parts are merged per row at the
// end of a piece).  All waits are bounded: on timeout the CTA records
// kErrTimeout, stops issuing, drains what it issued and frees its TMEM.
#include <cuda.h>

#include "match_common.cuh"
#include "psift_internal.cuh"

namespace psift {

constexpr int kEpiParts = 4;                      // epilogue warps per TMEM lane quarter (32-column parts)
constexpr int kEpiWarps = 4 * kEpiParts;          // warps 2 .. 2 + kEpiWarps - 1
constexpr int kTcThreads = 32 * (2 + kEpiWarps);  // warp 0 TMA, warp 1 MMA, then the epilogue
constexpr int kBM = kTcBM;
// B tile rows = MMA N = columns of one accumulator stage: N = 256 (two 128 x 256
// accumulators in TMEM); an M = 128, N = 128 MMA keeps the tensor pipe only about
// half busy.
template <int MODE>
struct TcShape {
  static constexpr int BN = kTcBN1;
  static constexpr int AccStages = 512 / BN;  // TMEM: 512 columns
  static constexpr int Cols = BN / kEpiParts;  // columns per epilogue warp and tile
  static constexpr uint32_t BStage = 2u * BN * 128u + BN * 32u;  // two halves, then the norm extension
  // kind::f16 instruction descriptor: D f32, A/B bf16, both K-major, M = 128, N = BN
  static constexpr uint32_t Idesc =
      (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
};
static_assert(TcShape<0>::Cols == 64 && TcShape<1>::Cols == 64, "two 32-column TMEM loads per warp and tile");
constexpr uint32_t kSpinLimit = 1u << 25;
constexpr int kColl = 32;   // window indices kept per (split, row)
constexpr int kXColl = 16;  // window indices a column part 1..3 hands to part 0 (more: exact scan)
static_assert(kColl == kTcColl, "window list length");

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

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 32 columns of a TMEM lane quarter, without waiting: the registers are valid
// only after tmem_wait32 on them.
__device__ __forceinline__ void tmem_ld32_nowait(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
// Waits for this thread's outstanding TMEM loads; r is tied so that no read of
// it moves above the wait.
__device__ __forceinline__ void tmem_wait32(uint32_t (&r)[32]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                 "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                 "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
}

// Smem map (offsets from a 1024-aligned base).
constexpr uint32_t kAStage = 2u * kBM * 128u;                     // two 64-column halves of 128 rows
constexpr uint32_t kSmA = 0;                                      // the A stages
static_assert(TcShape<0>::BStage % 1024 == 0 && TcShape<1>::BStage % 1024 == 0 && kAStage % 1024 == 0,
              "128B-swizzle atoms");
// Per pass: A tiles (double-buffered in pass 1), B tiles in flight, then barriers, then the epilogue exchange per row and column part
// 1..kEpiParts-1 (pass 1: the part's two largest values; pass 2: its count and up
// to kXColl indices).
template <int MODE>
struct TcLayout {
  static constexpr int kAStages = MODE == 0 ? 2 : 1;  // pass 2's larger exchange leaves room for one A tile
  static constexpr int kBStages = 2;
  static constexpr int kXStride = MODE == 0 ? 2 : kXColl + 2;  // ints per (part, row)
  static constexpr uint32_t kSmAx = kAStages * kAStage;     // A norm extension: 128 rows x 32 B
  static constexpr uint32_t kSmB = kSmAx + kBM * 32u;       // the B stages
  static_assert(kSmB % 1024 == 0, "128B-swizzle atoms");
  static constexpr uint32_t kSmBar = kSmB + kBStages * TcShape<MODE>::BStage;
  static constexpr uint32_t kSmX = kSmBar + 256;
  static constexpr uint32_t kSmTotal = kSmX + (kEpiParts - 1) * kBM * kXStride * 4 + 1024;  // + alignment slack
  static_assert(kSmTotal <= 227 * 1024, "shared memory per CTA");
};

// The CTA's range of the pass's tiles is cut into pieces, one per A tile it
// touches: problem k, A tile a, B tiles [b, b + len), and the piece's slot among
// the A tile's pieces (ranges are R tiles long, R >= (bt - 1) / (kTcSplits - 1),
// so an A tile meets at most kTcSplits ranges).
struct Piece {
  int k, a, b, len, split;
};
// The last problem whose first tile is <= g (problems without tiles share their
// successor's first tile, so the one found has tiles at g).
__device__ __forceinline__ int find_problem(const TcPair* P, int n, int mode, long long g) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (P[mid].g0[mode] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
__device__ __forceinline__ Piece make_piece(const TcPair* P, int mode, int R, int k, long long g,
                                            long long g_end) {
  Piece p;
  const int bt = P[k].bt[mode];
  const long long off = g - P[k].g0[mode];
  p.k = k;
  p.a = (int)(off / bt);
  p.b = (int)(off - (long long)p.a * bt);
  p.len = (int)min((long long)(bt - p.b), g_end - g);
  p.split = (int)(g / R - (g - p.b) / R);
  return p;
}
__device__ __forceinline__ int advance_problem(const TcPair* P, int n, int mode, int k, long long g) {
  while (k + 1 < n && P[k + 1].g0[mode] <= g) ++k;
  return k;
}

// Top-2 of a multiset kept as u0 >= u1: merge the pair {d0, d1}.
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
__device__ __forceinline__ void top2_pair(float& u0, float& u1, float d0, float d1) {
  const float hi = fmaxf(d0, d1), lo = fminf(d0, d1);
  u1 = max3f(u1, lo, fminf(u0, hi));
  u0 = fmaxf(u0, hi);
}

// MODE 0: pass 1 (top-2 per row); MODE 1: pass 2 (window collection over the
// compacted rows).
template <int MODE>
__global__ void __launch_bounds__(kTcThreads, 1)
    match_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    const __grid_constant__ CUtensorMap tmAx, const __grid_constant__ CUtensorMap tmBx,
                    const TcPair* __restrict__ P, int n_problems, const TcPlan* __restrict__ plan, uint32_t* err) {
  constexpr int mode = MODE;
  using L = TcLayout<MODE>;
  using Sh = TcShape<MODE>;
  constexpr int kBStages = L::kBStages;
  constexpr int kBN = Sh::BN;
  constexpr int kAccStages = Sh::AccStages;
  constexpr uint32_t kBStage = Sh::BStage;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L::kSmBar);  // [kBStages] B tile landed
  uint64_t* empty = full + kBStages;                             // [kBStages] B tile consumed by its MMAs
  uint64_t* afull = empty + kBStages;                            // [2] A tile landed
  uint64_t* aempty = afull + 2;                                  // [2] A tile's last MMA done
  uint64_t* accf = aempty + 2;                                   // [kAccStages] accumulator ready
  uint64_t* acce = accf + kAccStages;                            // [kAccStages] accumulator read out
  uint64_t* xfull = acce + kAccStages;                           // [1] A norm extension landed
  volatile uint32_t* taddr_slot = reinterpret_cast<volatile uint32_t*>(xfull + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(xfull + 2);

  // this CTA's tiles [g_begin, g_end) of the pass (pass 2's plan is written on the device)
  const long long total = plan[mode].total;
  const int R = plan[mode].per_cta;
  const long long g_begin = (long long)blockIdx.x * R;
  if (g_begin >= total) return;
  const long long g_end = min(total, g_begin + R);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool compact = mode == 1;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kBStages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&afull[i], 1);
      mbar_init(&aempty[i], 1);
    }
    for (int i = 0; i < kAccStages; ++i) {
      mbar_init(&accf[i], 1);
      mbar_init(&acce[i], kEpiWarps);
    }
    mbar_init(xfull, 1);
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

  if (warp == 0) {
    if (lane == 0) {
      // the constant A norm extension once, then per piece its A tile and B tiles
      mbar_expect_tx(xfull, kBM * 32u);
      tma_load_2d(&tmAx, xfull, smem + L::kSmAx, 0, 0);
      uint64_t* last_bar = xfull;  // the last load issued, for the drain on abort
      uint32_t last_par = 0;
      bool ok = true;
      int bs = 0;
      uint32_t bph = 0;  // B ring slot and its phase
      long long g = g_begin;
      int k = find_problem(P, n_problems, mode, g);
      for (int pi = 0; ok && g < g_end; ++pi) {
        const Piece pc = make_piece(P, mode, R, k, g, g_end);
        const int as = pi % L::kAStages;
        const uint32_t apar = ((uint32_t)(pi / L::kAStages)) & 1u;
        if (!mbar_wait(&aempty[as], apar ^ 1u, abort_flag)) {
          ok = false;
          break;
        }
        const int a_row = P[k].a_row0 + pc.a * kBM;
        uint8_t* ast = smem + kSmA + as * kAStage;
        mbar_expect_tx(&afull[as], kAStage);
        tma_load_2d(&tmA, &afull[as], ast, 0, a_row);
        tma_load_2d(&tmA, &afull[as], ast + kBM * 128, 64, a_row);
        last_bar = &afull[as];
        last_par = apar;
        for (int j = 0; j < pc.len; ++j) {
          if (!mbar_wait(&empty[bs], bph ^ 1u, abort_flag)) {
            ok = false;
            break;
          }
          const int b_row = P[k].b_row0 + (pc.b + j) * kBN;
          uint8_t* bst = smem + L::kSmB + bs * kBStage;
          mbar_expect_tx(&full[bs], kBStage);
          tma_load_2d(&tmB, &full[bs], bst, 0, b_row);
          tma_load_2d(&tmB, &full[bs], bst + kBN * 128, 64, b_row);
          tma_load_2d(&tmBx, &full[bs], bst + 2 * kBN * 128, 0, b_row);
          last_bar = &full[bs];
          last_par = bph;
          if (++bs == kBStages) {
            bs = 0;
            bph ^= 1u;
          }
        }
        g += pc.len;
        if (g < g_end) k = advance_problem(P, n_problems, mode, k, g);
      }
      if (!ok) {
        atomicOr(err, kErrTimeout);
        *abort_flag = 1;
        // drain: the copies already issued land before the CTA leaves (bounded)
        for (uint32_t i = 0; i < kSpinLimit && !mbar_try_wait(last_bar, last_par); ++i) {
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      bool ok = mbar_wait(xfull, 0, abort_flag);
      int issued = 0;
      uint64_t* last_bar = nullptr;
      uint32_t last_par = 0;
      int bs = 0, s = 0;
      uint32_t bph = 0, sph = 0;
      long long g = g_begin;
      int k = find_problem(P, n_problems, mode, g);
      const uint32_t ax = smem_u32(smem + L::kSmAx);
      for (int pi = 0; ok && g < g_end; ++pi) {
        const Piece pc = make_piece(P, mode, R, k, g, g_end);
        const int as = pi % L::kAStages;
        if (!mbar_wait(&afull[as], ((uint32_t)(pi / L::kAStages)) & 1u, abort_flag)) {
          ok = false;
          break;
        }
        const uint32_t a_base = smem_u32(smem + kSmA + as * kAStage);
        for (int j = 0; j < pc.len; ++j) {
          if (!mbar_wait(&full[bs], bph, abort_flag) || !mbar_wait(&acce[s], sph ^ 1u, abort_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t b_base = smem_u32(smem + L::kSmB + bs * kBStage);
          const uint32_t d = tmem + (uint32_t)(s * kBN);
#pragma unroll
          for (int kk = 0; kk < 8; ++kk) {
            const uint32_t half = (uint32_t)(kk >> 2), koff = (uint32_t)(kk & 3) * 32u;
            umma_bf16(d, sw128_desc(a_base + half * (kBM * 128) + koff),
                      sw128_desc(b_base + half * (kBN * 128) + koff), Sh::Idesc, kk > 0 ? 1u : 0u);
          }
          // the norm extension: D += h_j + l_j
          umma_bf16(d, sw32_desc(ax), sw32_desc(b_base + 2 * kBN * 128), Sh::Idesc, 1u);
          umma_commit(&empty[bs]);
          umma_commit(&accf[s]);
          last_bar = &accf[s];
          last_par = sph;
          ++issued;
          if (++bs == kBStages) {
            bs = 0;
            bph ^= 1u;
          }
          if (++s == kAccStages) {
            s = 0;
            sph ^= 1u;
          }
        }
        if (!ok) break;
        umma_commit(&aempty[as]);  // the A stage is free once this piece's MMAs are done
        g += pc.len;
        if (g < g_end) k = advance_problem(P, n_problems, mode, k, g);
      }
      if (!ok) {
        atomicOr(err, kErrTimeout);
        *abort_flag = 1;
        // drain: wait (bounded, ignoring the abort flag) for the last issued MMA group
        if (issued > 0)
          for (uint32_t i = 0; i < kSpinLimit && !mbar_try_wait(last_bar, last_par); ++i) {
          }
      }
    }
  } else {
    // epilogue: TMEM lane quarter warp % 4, 32-column part (warp - 2) / 4 of each tile
    const int quarter = warp & 3;
    const int part = (warp - 2) >> 2;
    const int row_in_tile = quarter * 32 + lane;
    int* xrow = reinterpret_cast<int*>(smem + L::kSmX) + ((part > 0 ? part - 1 : 0) * kBM + row_in_tile) * L::kXStride;
    const float inf = __int_as_float(0x7f800000);
    bool live = true;
    int s = 0;
    uint32_t sph = 0;
    long long g = g_begin;
    int k = find_problem(P, n_problems, mode, g);
    while (g < g_end) {
      const Piece pc = make_piece(P, mode, R, k, g, g_end);
      const TcPair& PR = P[k];
      // the previous piece's exchange slots have been merged
      asm volatile("bar.sync 1, %0;" ::"n"(32 * kEpiWarps) : "memory");
      const int n_rows = compact ? *PR.ccount : PR.na;
      const int r = pc.a * kBM + row_in_tile;
      const bool row_ok = r < n_rows;
      const int a_local = compact ? (row_ok ? PR.rowmap[r] : 0) : r;
      const long long o = (long long)pc.split * PR.na + a_local;
      // pass 1: the largest D of each of 8 column classes (column mod 8), one
      // three-input max per two values
      float cm[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) cm[q] = -inf;
      int cnt = 0;  // pass 2: indices with D >= the row's window bound
      float dthr = inf;
      int* coll = xrow + 2;
      int ccap = kXColl;
      if constexpr (mode == 1) {
        const float an = row_ok ? PR.an[a_local] : 0.0f;
        const float thr = row_ok ? PR.thr[a_local] : -inf;
        // every D with |q|^2 - 2 D <= thr (one f32 rounding) has
        // D >= (|q|^2 - thr) / 2 - 2^-24 (|q|^2 + |thr|); the margin below is larger
        dthr = thr == -inf ? inf : 0.5f * (an - thr) - 1e-6f * (fabsf(an) + fabsf(thr));
        if (part == 0) {
          coll = PR.coll_idx + o * kColl;
          ccap = kColl;
        }
      }
      auto fold = [&](const uint32_t(&v)[32], int cstart) {
        if constexpr (mode == 0) {
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            cm[q] = max3f(cm[q], __uint_as_float(v[q]), __uint_as_float(v[q + 8]));
            cm[q] = max3f(cm[q], __uint_as_float(v[q + 16]), __uint_as_float(v[q + 24]));
          }
        } else {
          // the 8 column-class maxima (column mod 8) against the window bound; only
          // a class that reaches it (rare) has its four values tested and collected
          uint32_t cls = 0;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const float m = fmaxf(max3f(__uint_as_float(v[q]), __uint_as_float(v[q + 8]), __uint_as_float(v[q + 16])),
                                  __uint_as_float(v[q + 24]));
            cls |= (m >= dthr ? 1u : 0u) << q;
          }
          if (!row_ok) cls = 0;
          if (cls) {
            // the hit classes' values in column order (static indices: v stays in registers)
#pragma unroll
            for (int c = 0; c < 32; ++c) {
              if (((cls >> (c & 7)) & 1u) && __uint_as_float(v[c]) >= dthr) {
                if (cnt < ccap) coll[cnt] = cstart + c;
                ++cnt;
              }
            }
          }
        }
      };
      // Each wait covers the warp's 64 columns of a tile as two 32-column TMEM
      // loads in flight together; the accumulator is released as soon as its
      // values are in registers, then the values are folded.
      const uint32_t tq = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(part * Sh::Cols);
      const int col0 = pc.b * kBN + part * Sh::Cols;
      uint32_t ra[32], rb[32];
      // waits for accumulator st; false (nothing to load) on timeout
      auto ready = [&](int st, uint32_t ph) -> bool {
        if (live && !__all_sync(0xffffffffu, mbar_wait(&accf[st], ph, abort_flag))) {
          live = false;
          atomicOr(err, kErrTimeout);
          *abort_flag = 1;
        }
        if (!live) return false;
        tc_fence_after();
        __syncwarp();
        return true;
      };
      auto advance = [&](int n) {
        s += n;
        if (s >= kAccStages) {
          s -= kAccStages;
          sph ^= 1u;
        }
      };
      for (int j = 0; j < pc.len; ++j) {
        const bool la = ready(s, sph);
        if (la) {
          tmem_ld32_nowait(tq + (uint32_t)(s * kBN), ra);
          tmem_ld32_nowait(tq + (uint32_t)(s * kBN) + 32u, rb);
          // every issued load completes before the registers are read (or the CTA leaves)
          tmem_wait32(ra);
          tmem_wait32(rb);
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acce[s]);
          fold(ra, col0 + j * kBN);
          fold(rb, col0 + j * kBN + 32);
        }
        advance(1);
      }
      // The row's largest D, and the second largest of the class maxima: a lower
      // bound on the row's second largest D (equal to it unless the two largest
      // share a class), which can only widen the candidate window.
      float u0 = -inf, u1 = -inf;
      if constexpr (mode == 0) {
#pragma unroll
        for (int q = 0; q < 8; q += 2) top2_pair(u0, u1, cm[q], cm[q + 1]);
      }
      if (part > 0) {
        if constexpr (mode == 0) {
          xrow[0] = __float_as_int(u0);
          xrow[1] = __float_as_int(u1);
        } else {
          xrow[0] = cnt;
        }
      }
      asm volatile("bar.sync 1, %0;" ::"n"(32 * kEpiWarps) : "memory");
      // Part 0 merges the other parts into its row, in part order: the two largest
      // D of all, mapped to the two smallest a = |q|^2 - 2 D (pass 1), or the
      // concatenated index lists with the summed count (pass 2; a count above
      // kColl, or a part that overflowed its kXColl slots, sends the row to the
      // exact scan).
      if (part == 0 && row_ok && live) {
        bool part_overflow = false;
        for (int p = 1; p < kEpiParts; ++p) {
          const int* x = reinterpret_cast<const int*>(smem + L::kSmX) + ((p - 1) * kBM + row_in_tile) * L::kXStride;
          if constexpr (mode == 0) {
            const float x0 = __int_as_float(x[0]), x1 = __int_as_float(x[1]);
            u1 = max3f(u1, x1, fminf(u0, x0));
            u0 = fmaxf(u0, x0);
          } else {
            const int c1 = x[0];
            part_overflow |= c1 > kXColl;
            for (int q = 0; q < c1 && q < kXColl && cnt + q < kColl; ++q) coll[cnt + q] = x[2 + q];
            cnt += c1;
          }
        }
        if constexpr (mode == 0) {
          const float an = PR.an[a_local];
          PR.top2[2 * o] = __fmaf_rn(-2.0f, u0, an);
          PR.top2[2 * o + 1] = __fmaf_rn(-2.0f, u1, an);
        } else {
          PR.coll_cnt[o] = part_overflow ? max(cnt, kColl + 1) : cnt;
        }
      }
      g += pc.len;
      if (g < g_end) k = advance_problem(P, n_problems, mode, k, g);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
  }
}

// ------------------------------------------------------------ bf16 operands
// Per row: bf16 copy (zero rows for padding are pre-cleared), exact f32 squared
// norm (sequential), running max of the norms, the row's GEMM norm extension
// [h, l, 0, ...] with h = bf16(-|x|^2 / 2), l = bf16(-|x|^2 / 2 - h), and its
// pass-1 result slots set to +inf; padding rows up to n_pad get [-inf, 0, ...],
// which no window or top-2 takes.  A job with x = null writes n_pad rows of the
// A operand's extension [1, 1, 0, ...].
struct Bf16Job {
  const float* x;
  int n;
  uint16_t* out;
  float* norms;
  float* norm_max;
  uint16_t* ext;  // n_pad rows x 16
  int n_pad;
  float* top2;    // null, or the pass-1 slots [kTcSplits][n][2] of the problem with these A rows: set to +inf
};

__device__ __forceinline__ uint16_t bf16_rne(float f) {
  const uint32_t u = __float_as_uint(f);
  return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}

// A warp per 32 rows: the rows are copied coalesced into shared memory (a 16-byte
// asynchronous copy per lane and row, all in flight together), written out as
// bf16, and lane j adds up row j's squared norm sequentially from there (the
// rows' sums run side by side instead of one row's 128 terms being passed lane
// to lane).
constexpr int kBf16Warps = 2;  // 33.8 KB of static shared memory per block
constexpr int kBf16Stride = 132;  // floats per staged row: lanes reading 16 B of different rows hit distinct banks

__global__ void __launch_bounds__(32 * kBf16Warps) to_bf16_kernel(const Bf16Job* __restrict__ jobs) {
  __shared__ __align__(16) float stage[kBf16Warps][32 * kBf16Stride];
  const Bf16Job& J = jobs[blockIdx.y];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = (blockIdx.x * kBf16Warps + warp) * 32;
  if (row0 >= J.n_pad) return;
  const int row = row0 + lane;  // this lane's row for the norm and the extension
  if (!J.x) {
    // the A operand's constant extension rows [1, 1, 0, ...]
    if (row < J.n_pad) {
      uint4* e = reinterpret_cast<uint4*>(J.ext + (size_t)row * 16);
      e[0] = make_uint4(0x3F803F80u, 0u, 0u, 0u);
      e[1] = make_uint4(0u, 0u, 0u, 0u);
    }
    return;
  }
  const float* __restrict__ x = J.x;
  float* st = stage[warp];
  const int nr = min(32, J.n - row0);  // rows with data
  // all of the warp's row loads in flight at once: asynchronous copies into the stage
  for (int r = 0; r < nr; ++r)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(st + r * kBf16Stride + 4 * lane)),
                 "l"(x + (size_t)(row0 + r) * 128 + 4 * lane)
                 : "memory");
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
  __syncwarp();
  for (int r = 0; r < nr; ++r) {
    const float4 v = *reinterpret_cast<const float4*>(st + r * kBf16Stride + 4 * lane);
    uint2 packed;
    packed.x = (uint32_t)bf16_rne(v.x) | ((uint32_t)bf16_rne(v.y) << 16);  // round to nearest even
    packed.y = (uint32_t)bf16_rne(v.z) | ((uint32_t)bf16_rne(v.w) << 16);
    reinterpret_cast<uint2*>(J.out + (size_t)(row0 + r) * 128)[lane] = packed;
  }
  if (row < J.n) {
    // exact sequential norm of row `row`
    const float* rr = st + lane * kBf16Stride;
    float s = 0.0f;
#pragma unroll 8
    for (int c = 0; c < 32; ++c) {
      const float4 v = *reinterpret_cast<const float4*>(rr + 4 * c);
      s += v.x * v.x;
      s += v.y * v.y;
      s += v.z * v.z;
      s += v.w * v.w;
    }
    J.norms[row] = s;
    atomicMax(reinterpret_cast<unsigned int*>(J.norm_max), __float_as_uint(s));
    const float half = -0.5f * s;  // exact
    const uint16_t hi = bf16_rne(half);
    const uint16_t lo = bf16_rne(half - __uint_as_float((uint32_t)hi << 16));
    uint4* e = reinterpret_cast<uint4*>(J.ext + (size_t)row * 16);
    e[0] = make_uint4((uint32_t)hi | ((uint32_t)lo << 16), 0u, 0u, 0u);
    e[1] = make_uint4(0u, 0u, 0u, 0u);
    if (J.top2)
      for (int q = 0; q < 2 * kTcSplits; ++q)
        J.top2[((size_t)(q >> 1) * J.n + row) * 2 + (q & 1)] = __int_as_float(0x7f800000);
  } else if (row < J.n_pad) {
    // padding rows: [-inf, 0, ...], which no window or top-2 takes
    uint4* e = reinterpret_cast<uint4*>(J.ext + (size_t)row * 16);
    e[0] = make_uint4(0xFF80u, 0u, 0u, 0u);
    e[1] = make_uint4(0u, 0u, 0u, 0u);
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

// A row's result: best / index / second, and for the forward pass of a mutual
// match the target's mark when the reference's ratio test (src/pipeline.rs:1789-1794)
// accepts the row.
__device__ __forceinline__ void rerank_row_out(const RerankJob& J, int row, float b, int bi, float sec) {
  const bool forward = J.second != nullptr;
  if (forward && J.flags && sec > 1e-12f && b < __int_as_float(0x7f800000) && bi < J.nb) {
    if (sqrtf(b) / sqrtf(sec) < J.ratio) J.flags[bi] = 1;
  }
  J.best[row] = b;
  J.best_idx[row] = bi;
  if (forward) J.second[row] = sec;
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
  if (thr == -inf) {
    // nothing to rank: the row's result is final here (no match / not a candidate)
    rerank_row_out(J, row, inf, 0x7fffffff, inf);
    return;
  }
  for (int s = 0; s < J.splits; ++s) J.coll_cnt[(long long)s * J.na + row] = 0;  // slots without a piece stay empty
  // rows with a window go to pass 2 and the re-rank (compacted; the order does not
  // matter: every row's collection depends on that row alone and lands in its own slot)
  J.rowmap[atomicAdd(J.ccount, 1)] = row;
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

// One warp per kept A row (window_kernel's compacted list): exact reference
// distances over the window candidates (every index with a <= thr, collected by
// the second GEMM pass).  Candidates go
// four at a time: every lane loads its 16 bytes of each candidate's B row (all
// four loads in flight) and writes the squared differences to shared memory,
// then lane c adds up candidate c's 128 terms in the reference's order.  A row
// whose window overflowed kColl in some slot is left to rerank_scan_kernel.
constexpr int kRrBatch = 4;
constexpr int kRrStride = 132;  // floats per staged candidate (conflict-free reads across candidates)

__global__ void __launch_bounds__(256, 4) rerank_kernel(const RerankJob* __restrict__ jobs) {
  __shared__ __align__(16) float terms[8][kRrBatch * kRrStride];
  const RerankJob& J = jobs[blockIdx.y];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // the rows window_kernel kept (the others' results are final already)
  const int c_row = blockIdx.x * 8 + warp;
  if (c_row >= *J.ccount) return;
  const int row = J.rowmap[c_row];
  const float inf = __int_as_float(0x7f800000);
  float b = inf, sec = inf;
  int bi = 0x7fffffff;
  // the slots' counts and their running offsets (same in every lane)
  int cnt[kTcSplits], total = 0;
  bool overflow = false;
#pragma unroll
  for (int sl = 0; sl < kTcSplits; ++sl) {
    cnt[sl] = J.coll_cnt[(long long)sl * J.na + row];
    overflow |= cnt[sl] > kColl;
    total += cnt[sl];
  }
  if (overflow) {
    // the exact scan over all B rows is left to rerank_scan_kernel (a CTA per row)
    if (lane == 0) {
      atomicAdd(J.fallbacks, 1u);
      J.scan_rows[atomicAdd(J.scan_count, 1)] = make_int2((int)blockIdx.y, row);
    }
    return;
  }
  const float4 a4 = reinterpret_cast<const float4*>(J.a + (size_t)row * 128)[lane];
  float* tw = terms[warp];
  for (int c0 = 0; c0 < total; c0 += kRrBatch) {
    const int nb = min(kRrBatch, total - c0);
    int idx[kRrBatch];
    float4 bv[kRrBatch];
#pragma unroll
    for (int c = 0; c < kRrBatch; ++c) {
      // candidate c0 + c: its slot and position there
      int m = c0 + c, sl = 0;
#pragma unroll
      for (int q = 0; q < kTcSplits - 1; ++q)
        if (sl == q && m >= cnt[q]) {
          m -= cnt[q];
          sl = q + 1;
        }
      idx[c] = c < nb ? J.coll_idx[((long long)sl * J.na + row) * kColl + m] : 0;
    }
#pragma unroll
    for (int c = 0; c < kRrBatch; ++c)
      if (c < nb) bv[c] = reinterpret_cast<const float4*>(J.b + (size_t)idx[c] * 128)[lane];
#pragma unroll
    for (int c = 0; c < kRrBatch; ++c) {
      if (c < nb) {
        float4 d;
        d.x = a4.x - bv[c].x;
        d.y = a4.y - bv[c].y;
        d.z = a4.z - bv[c].z;
        d.w = a4.w - bv[c].w;
        *reinterpret_cast<float4*>(tw + c * kRrStride + 4 * lane) =
            make_float4(d.x * d.x, d.y * d.y, d.z * d.z, d.w * d.w);
      }
    }
    __syncwarp();
    if (lane < nb) {
      const float* t = tw + lane * kRrStride;
      float sum = 0.0f;
#pragma unroll 8
      for (int i = 0; i < 128; i += 4) {
        const float4 v = *reinterpret_cast<const float4*>(t + i);
        sum += v.x;
        sum += v.y;
        sum += v.z;
        sum += v.w;
      }
      int my = idx[0];
#pragma unroll
      for (int c = 1; c < kRrBatch; ++c)
        if (lane == c) my = idx[c];
      top2_push(b, bi, sec, sum, my);
    }
    __syncwarp();
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    const float b2 = __shfl_xor_sync(0xffffffffu, b, off);
    const int i2 = __shfl_xor_sync(0xffffffffu, bi, off);
    const float s2 = __shfl_xor_sync(0xffffffffu, sec, off);
    top2_merge(b, bi, sec, b2, i2, s2);
  }
  if (lane == 0) rerank_row_out(J, row, b, bi, sec);
}

// A row whose window overflowed: one CTA computes the exact reference distances
// to all B rows (a thread per B row, two at a time), merged order-independently.
// The CTAs walk the list of such rows that rerank_kernel left.
__device__ __forceinline__ void exact_d2_x2(const float* __restrict__ a, const float* __restrict__ b0,
                                            const float* __restrict__ b1, float& s0, float& s1) {
  s0 = 0.0f;
  s1 = 0.0f;
#pragma unroll 4
  for (int i = 0; i < 128; i += 4) {
    const float4 x = *reinterpret_cast<const float4*>(a + i);
    const float4 y = *reinterpret_cast<const float4*>(b0 + i);
    const float4 z = *reinterpret_cast<const float4*>(b1 + i);
    float d = x.x - y.x, e = x.x - z.x;
    s0 += d * d;
    s1 += e * e;
    d = x.y - y.y, e = x.y - z.y;
    s0 += d * d;
    s1 += e * e;
    d = x.z - y.z, e = x.z - z.z;
    s0 += d * d;
    s1 += e * e;
    d = x.w - y.w, e = x.w - z.w;
    s0 += d * d;
    s1 += e * e;
  }
}

__global__ void __launch_bounds__(256) rerank_scan_kernel(const RerankJob* __restrict__ jobs,
                                                          const int2* __restrict__ rows, const int* __restrict__ count) {
  __shared__ float sb[8], ss[8];
  __shared__ int si[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float inf = __int_as_float(0x7f800000);
  const int n = *count;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int2 e = rows[it];
    const RerankJob& J = jobs[e.x];
    const int row = e.y;
    const float* arow = J.a + (size_t)row * 128;
    float b = inf, sec = inf;
    int bi = 0x7fffffff;
    int t = threadIdx.x;
    for (; t + 256 < J.nb; t += 512) {
      float d0, d1;
      exact_d2_x2(arow, J.b + (size_t)t * 128, J.b + (size_t)(t + 256) * 128, d0, d1);
      top2_push(b, bi, sec, d0, t);
      top2_push(b, bi, sec, d1, t + 256);
    }
    if (t < J.nb) top2_push(b, bi, sec, exact_d2(arow, J.b + (size_t)t * 128), t);
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
      const float b2 = __shfl_xor_sync(0xffffffffu, b, off);
      const int i2 = __shfl_xor_sync(0xffffffffu, bi, off);
      const float s2 = __shfl_xor_sync(0xffffffffu, sec, off);
      top2_merge(b, bi, sec, b2, i2, s2);
    }
    if (lane == 0) {
      sb[warp] = b;
      si[warp] = bi;
      ss[warp] = sec;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < 8; ++w) top2_merge(b, bi, sec, sb[w], si[w], ss[w]);
      rerank_row_out(J, row, b, bi, sec);
    }
    __syncthreads();
  }
}

// Pass 2's tile order, on the device (the kept row counts are known there): per
// problem its A tiles (kept rows / 128) and first tile, and the range length of
// each of `ctas` CTAs, at least (B tiles - 1) / (kTcSplits - 1) so that an A tile
// meets at most kTcSplits ranges.  One block.
__global__ void __launch_bounds__(1024) tc_plan_kernel(TcPair* __restrict__ P, int n, TcPlan* __restrict__ plan, int ctas) {
  __shared__ long long warp_sums[32];
  __shared__ long long carry;
  __shared__ int bt_max;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) {
    carry = 0;
    bt_max = 1;
  }
  __syncthreads();
  for (int base = 0; base < n; base += blockDim.x) {
    const int k = base + tid;
    long long tiles = 0;
    if (k < n) {
      const int at = (*P[k].ccount + kTcBM - 1) / kTcBM;
      P[k].at[1] = at;
      tiles = (long long)at * P[k].bt[1];
      if (at > 0) atomicMax(&bt_max, P[k].bt[1]);
    }
    // block-wide exclusive scan of the tile counts
    long long v = tiles;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const long long u = __shfl_up_sync(0xffffffffu, v, off);
      if (lane >= off) v += u;
    }
    if (lane == 31) warp_sums[wid] = v;
    __syncthreads();
    if (wid == 0) {
      long long w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const long long u = __shfl_up_sync(0xffffffffu, w, off);
        if (lane >= off) w += u;
      }
      warp_sums[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const long long before = carry + (wid > 0 ? warp_sums[wid - 1] : 0) + v - tiles;
    if (k < n) P[k].g0[1] = before;
    __syncthreads();
    if (tid == 0) carry += warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
  }
  if (tid == 0) {
    const long long total = carry;
    long long r = (total + ctas - 1) / ctas;
    r = max(r, (long long)((bt_max - 1 + kTcSplits - 2) / (kTcSplits - 1)));
    plan[1].total = total;
    plan[1].per_cta = (int)max(r, 1LL);
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
  dim3 grid((max_rows + 32 * kBf16Warps - 1) / (32 * kBf16Warps), n_jobs);
  to_bf16_kernel<<<grid, 32 * kBf16Warps, 0, st>>>((const Bf16Job*)jobs);
  return cudaGetLastError();
}

cudaError_t launch_match_tc(const CUtensorMap& tmA, const CUtensorMap& tmB, const CUtensorMap& tmAx,
                            const CUtensorMap& tmBx, const TcPair* problems, int n_problems, const TcPlan* plan,
                            int ctas, uint32_t* err, int mode, cudaStream_t st) {
  if (ctas <= 0 || n_problems <= 0) return cudaSuccess;
  const void* fn = mode == 0 ? (const void*)match_tc_kernel<0> : (const void*)match_tc_kernel<1>;
  const uint32_t smem = mode == 0 ? TcLayout<0>::kSmTotal : TcLayout<1>::kSmTotal;
  cudaError_t e = ensure_smem_attr(fn, smem);
  if (e != cudaSuccess) return e;
  if (mode == 0)
    match_tc_kernel<0><<<ctas, kTcThreads, smem, st>>>(tmA, tmB, tmAx, tmBx, problems, n_problems, plan, err);
  else
    match_tc_kernel<1><<<ctas, kTcThreads, smem, st>>>(tmA, tmB, tmAx, tmBx, problems, n_problems, plan, err);
  return cudaGetLastError();
}

cudaError_t launch_tc_plan(TcPair* problems, int n_problems, TcPlan* plan, int ctas, cudaStream_t st) {
  if (n_problems <= 0) return cudaSuccess;
  tc_plan_kernel<<<1, 1024, 0, st>>>(problems, n_problems, plan, ctas);
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

cudaError_t launch_rerank(const RerankJob* jobs, int n_jobs, int max_rows, const int2* scan_rows,
                          const int* scan_count, int scan_ctas, cudaStream_t st) {
  dim3 grid((max_rows + 7) / 8, n_jobs);  // a warp per row
  rerank_kernel<<<grid, 256, 0, st>>>(jobs);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  rerank_scan_kernel<<<scan_ctas, 256, 0, st>>>(jobs, scan_rows, scan_count);
  return cudaGetLastError();
}

}  // namespace psift
