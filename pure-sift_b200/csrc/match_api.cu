// Orchestration and C-ABI entry points of the matcher (Matcher::new / match_).
//
// Reference: Matcher::new (src/pipeline.rs:156-164), Matcher::match_ (:167-169),
// match_descriptors_with_options (:1744-1841).
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "match_common.cuh"
#include "psift_internal.cuh"

namespace psift {

cudaError_t launch_match_fp32(const MatchPair* d_pairs, int n_pairs, int max_q_tiles, int t_splits, float* part,
                              int* part_idx, float* cpart, int* cpart_idx, const long long* part_off,
                              const long long* cpart_off, bool mutual, cudaStream_t st);
cudaError_t launch_match_merge(const MatchPair* d_pairs, int n_pairs, int max_n, int t_splits, const float* part,
                               const int* part_idx, const float* cpart, const int* cpart_idx,
                               const long long* part_off, const long long* cpart_off, bool mutual, cudaStream_t st);
cudaError_t launch_match_emit(const MatchPair* d_pairs, int n_pairs, float ratio, bool mutual, cudaStream_t st);
bool make_operand_map(CUtensorMap* tm, const void* base, long long rows, int box_rows);
bool make_ext_map(CUtensorMap* tm, const void* base, long long rows, int box_rows);
struct Bf16Job {
  const float* x;
  int n;
  uint16_t* out;
  float* norms;
  float* norm_max;
  uint16_t* ext;
  int n_pad;
  float* top2;
};
cudaError_t launch_to_bf16(const void* jobs, int n_jobs, int max_rows, cudaStream_t st);
cudaError_t launch_match_tc(const CUtensorMap& tmA, const CUtensorMap& tmB, const CUtensorMap& tmAx,
                            const CUtensorMap& tmBx, const TcPair* problems, int n_problems, const TcPlan* plan,
                            int ctas, uint32_t* err, int mode, cudaStream_t st);
cudaError_t launch_tc_plan(TcPair* problems, int n_problems, TcPlan* plan, int ctas, cudaStream_t st);
cudaError_t launch_window(const RerankJob* jobs, int n_jobs, int max_rows, cudaStream_t st);
cudaError_t launch_rerank(const RerankJob* jobs, int n_jobs, int max_rows, const int2* scan_rows,
                          const int* scan_count, int scan_ctas, cudaStream_t st);
cudaError_t launch_gather_rows(const GatherJob* jobs, int n_jobs, int max_rows, cudaStream_t st);

namespace {

constexpr int kTile = 128;

// Matcher::new (src/pipeline.rs:156-164): same message.
psift_status validate_match_options(psift_ctx* ctx, const psift_match_options* o) {
  if (!o) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null match options");
  if (!(o->ratio == o->ratio) || o->ratio > 3.4e38f || o->ratio <= 0.0f || o->ratio > 1.0f) {
    char buf[128];
    snprintf(buf, sizeof buf, "Invalid `ratio`=%g: must be finite and in (0.0, 1.0]", (double)o->ratio);
    return set_error(ctx, PSIFT_ERR_INVALID_CONFIG, buf);
  }
  if (o->precision != PSIFT_PRECISION_FP32 && o->precision != PSIFT_PRECISION_BF16_RERANK)
    return set_error(ctx, PSIFT_ERR_INVALID_CONFIG, "Invalid `precision`: must be FP32 (0) or BF16_RERANK (1)");
  return PSIFT_OK;
}

long long pad_rows(int n) { return ((long long)n + kTcBN1 - 1) / kTcBN1 * kTcBN1; }

// Device-side batch: every pointer in jobs is device memory.  Queues all work.
psift_status match_batch(psift_ctx* ctx, const psift_match_job* jobs, int n, const psift_match_options& opt) {
  cudaStream_t st = ctx->stream;
  const bool mutual = opt.mutual != 0;
  const bool tc = opt.precision == PSIFT_PRECISION_BF16_RERANK;
  // Active problems: the reference returns nothing for an empty query set or < 2 targets.
  std::vector<int> active;
  for (int i = 0; i < n; ++i) {
    const psift_match_job& J = jobs[i];
    if (J.nq > 0 && J.nt >= 2) active.push_back(i);
  }
  // zero the counts of inactive problems
  for (int i = 0; i < n; ++i)
    if (std::find(active.begin(), active.end(), i) == active.end())
      PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(jobs[i].d_count, 0, sizeof(uint32_t), st));
  const int na = (int)active.size();
  if (na == 0) return PSIFT_OK;

  // ---- sizes
  size_t bytes = sizeof(MatchPair) * na + 4096;
  int max_q_tiles = 0, max_n = 0;
  std::vector<int> t_splits_v(na), q_tiles(na);
  long long part_total = 0, cpart_total = 0;
  long long q_rows = 0, t_rows = 0;
  long long cand_f = 0, cand_r = 0;
  const int target_ctas = ctx->tune.match_per_sm[tc ? 1 : 0] * ctx->num_sms;
  for (int k = 0; k < na; ++k) {
    const psift_match_job& J = jobs[active[k]];
    const int qt = (int)((J.nq + kTile - 1) / kTile);
    q_tiles[k] = qt;
    max_q_tiles = std::max(max_q_tiles, qt);
    max_n = std::max(max_n, (int)std::max(J.nq, J.nt));
    bytes += 3 * sizeof(float) * (size_t)J.nq + 2 * sizeof(float) * (size_t)J.nt + 1024;
    if (!tc) {
      const int tt = (int)((J.nt + kTile - 1) / kTile);
      int sp = (target_ctas + na * qt - 1) / (na * qt);
      sp = std::max(1, std::min(sp, tt));
      t_splits_v[k] = sp;
      part_total += (long long)sp * J.nq;
      if (mutual) cpart_total += (long long)qt * J.nt;
    } else {
      q_rows += pad_rows((int)J.nq);
      t_rows += pad_rows((int)J.nt);
      cand_f += (long long)kTcSplits * J.nq;
      if (mutual) cand_r += (long long)kTcSplits * J.nt;
    }
  }
  int t_splits = 1;
  for (int k = 0; k < na; ++k) t_splits = std::max(t_splits, t_splits_v[k]);
  if (!tc) {
    // one uniform split count (grid x); per-pair offsets cover it
    part_total = 0;
    cpart_total = 0;
    for (int k = 0; k < na; ++k) {
      const psift_match_job& J = jobs[active[k]];
      part_total += (long long)t_splits * J.nq;
      if (mutual) cpart_total += (long long)q_tiles[k] * J.nt;
    }
    bytes += (size_t)part_total * 12 + (size_t)cpart_total * 8 + 2 * sizeof(long long) * na + 1024;
  } else {
    bytes += (size_t)(q_rows + t_rows) * 256 + (size_t)(q_rows + t_rows) * 4 + 4096;
    bytes += (size_t)(q_rows + t_rows) * 32 + (size_t)kTcBM * 32 + 3 * 256;  // GEMM norm extensions
    bytes += (size_t)(cand_f + cand_r) * (8 + 4 * kTcColl + 4) + (size_t)(q_rows + t_rows) * 4 +
             sizeof(TcPlan) * 4 + 256 +
             sizeof(TcPair) * 2 * na + sizeof(RerankJob) * 2 * na + 8192 + (size_t)t_rows * 4 +
             sizeof(Bf16Job) * 2 * na + 512;
    // pass 2's compacted operands, row maps, counts and gather jobs
    bytes += (size_t)(q_rows + t_rows) * 256 + (size_t)(q_rows + t_rows) * 4 + sizeof(int) * 2 * na +
             sizeof(GatherJob) * 2 * na + 5 * 256;
    bytes += sizeof(int2) * (size_t)(q_rows + t_rows) + 2 * 256;  // exact-scan row lists
  }
  psift_status s = arena_reserve(ctx, bytes);
  if (s != PSIFT_OK) return s;

  // ---- pairs
  std::vector<MatchPair> pairs(na);
  MatchPair* d_pairs = (MatchPair*)arena_alloc(ctx, sizeof(MatchPair) * na);
  for (int k = 0; k < na; ++k) {
    const psift_match_job& J = jobs[active[k]];
    MatchPair& P = pairs[k];
    std::memset(&P, 0, sizeof P);
    P.q = J.query_descriptors;
    P.t = J.target_descriptors;
    P.qxy = J.query_xy;
    P.txy = J.target_xy;
    P.nq = (int)J.nq;
    P.nt = (int)J.nt;
    P.best = (float*)arena_alloc(ctx, sizeof(float) * J.nq);
    P.second = (float*)arena_alloc(ctx, sizeof(float) * J.nq);
    P.best_idx = (int*)arena_alloc(ctx, sizeof(int) * J.nq);
    P.col_best = (float*)arena_alloc(ctx, sizeof(float) * J.nt);
    P.col_idx = (int*)arena_alloc(ctx, sizeof(int) * J.nt);
    P.out = J.out;
    P.out_count = J.d_count;
  }

  if (!tc) {
    std::vector<long long> poff(na), cpoff(na);
    long long a = 0, b = 0;
    for (int k = 0; k < na; ++k) {
      poff[k] = a;
      cpoff[k] = b;
      a += (long long)t_splits * pairs[k].nq;
      b += (long long)q_tiles[k] * pairs[k].nt;
    }
    float* part = (float*)arena_alloc(ctx, sizeof(float) * 2 * std::max<long long>(part_total, 1));
    int* part_idx = (int*)arena_alloc(ctx, sizeof(int) * std::max<long long>(part_total, 1));
    float* cpart = (float*)arena_alloc(ctx, sizeof(float) * std::max<long long>(cpart_total, 1));
    int* cpart_idx = (int*)arena_alloc(ctx, sizeof(int) * std::max<long long>(cpart_total, 1));
    long long* d_poff = (long long*)arena_alloc(ctx, sizeof(long long) * na);
    long long* d_cpoff = (long long*)arena_alloc(ctx, sizeof(long long) * na);
    if (!part || !d_cpoff) return set_error(ctx, PSIFT_ERR_INTERNAL, "match workspace carve overflow");
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_pairs, pairs.data(), sizeof(MatchPair) * na, cudaMemcpyHostToDevice, st));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_poff, poff.data(), sizeof(long long) * na, cudaMemcpyHostToDevice, st));
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_cpoff, cpoff.data(), sizeof(long long) * na, cudaMemcpyHostToDevice, st));
    StageScope sc(ctx, STAGE_MATCH);
    cudaError_t e = launch_match_fp32(d_pairs, na, max_q_tiles, t_splits, part, part_idx, cpart, cpart_idx, d_poff,
                                      d_cpoff, mutual, st);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "match_fp32");
    e = launch_match_merge(d_pairs, na, max_n, t_splits, part, part_idx, cpart, cpart_idx, d_poff, d_cpoff, mutual, st);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "match_merge");
    e = launch_match_emit(d_pairs, na, opt.ratio, mutual, st);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "match_emit");
    return PSIFT_OK;
  }

  // ---- BF16 tensor-core path
  uint16_t* qb = (uint16_t*)arena_alloc(ctx, (size_t)q_rows * 256);
  uint16_t* tb = (uint16_t*)arena_alloc(ctx, (size_t)t_rows * 256);
  float* qn = (float*)arena_alloc(ctx, sizeof(float) * q_rows);
  float* tn = (float*)arena_alloc(ctx, sizeof(float) * t_rows);
  float* maxes = (float*)arena_alloc(ctx, sizeof(float) * 2 * na);  // [k]: t max, [na + k]: q max
  const long long cand = std::max<long long>(cand_f + cand_r, 1);
  float* top2 = (float*)arena_alloc(ctx, sizeof(float) * 2 * cand);
  int* coll_idx = (int*)arena_alloc(ctx, sizeof(int) * kTcColl * cand);
  int* coll_cnt = (int*)arena_alloc(ctx, sizeof(int) * cand);
  float* thr = (float*)arena_alloc(ctx, sizeof(float) * (q_rows + t_rows));
  TcPlan* d_plan = (TcPlan*)arena_alloc(ctx, sizeof(TcPlan) * 4);  // [direction][pass]
  TcPair* d_tcp = (TcPair*)arena_alloc(ctx, sizeof(TcPair) * 2 * na);
  RerankJob* d_rj = (RerankJob*)arena_alloc(ctx, sizeof(RerankJob) * 2 * na);
  int* flags = mutual ? (int*)arena_alloc(ctx, sizeof(int) * t_rows) : nullptr;  // matched-target marks
  Bf16Job* d_bj = (Bf16Job*)arena_alloc(ctx, sizeof(Bf16Job) * (2 * na + 1));
  std::vector<Bf16Job> bj(2 * na + 1);
  // GEMM norm extensions (16 bf16 per row): the rows' own [h, l, 0, ...] when
  // they are the B operand, the constant [1, 1, 0, ...] tile for the A operand
  uint16_t* qx = (uint16_t*)arena_alloc(ctx, (size_t)q_rows * 32);
  uint16_t* tx = (uint16_t*)arena_alloc(ctx, (size_t)t_rows * 32);
  uint16_t* ones = (uint16_t*)arena_alloc(ctx, (size_t)kTcBM * 32);
  // pass 2 runs over the rows window_kernel keeps, gathered into these operands
  uint16_t* qbc = (uint16_t*)arena_alloc(ctx, (size_t)q_rows * 256);
  uint16_t* tbc = (uint16_t*)arena_alloc(ctx, (size_t)t_rows * 256);
  int* rowmap = (int*)arena_alloc(ctx, sizeof(int) * (q_rows + t_rows));
  int* ccount = (int*)arena_alloc(ctx, sizeof(int) * 2 * na);
  int* scan_count = (int*)arena_alloc(ctx, sizeof(int) * 2);  // per direction
  int2* scan_rows = (int2*)arena_alloc(ctx, sizeof(int2) * (q_rows + t_rows));
  GatherJob* d_gj = (GatherJob*)arena_alloc(ctx, sizeof(GatherJob) * 2 * na);
  std::vector<GatherJob> gj(2 * na);
  if (!qb || !tb || !thr || !coll_cnt || !d_rj || !d_bj || (mutual && !flags) || !qbc || !tbc || !rowmap ||
      !ccount || !d_gj || !qx || !tx || !ones || !d_plan || !scan_count || !scan_rows)
    return set_error(ctx, PSIFT_ERR_INTERNAL, "match workspace carve overflow");
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(ccount, 0, sizeof(int) * 2 * na, st));
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(scan_count, 0, sizeof(int) * 2, st));
  if (mutual) PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(flags, 0, sizeof(int) * t_rows, st));
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(qb, 0, (size_t)q_rows * 256, st));
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(tb, 0, (size_t)t_rows * 256, st));
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(maxes, 0, sizeof(float) * 2 * na, st));
  std::vector<long long> q0(na), t0(na);
  {
    long long a = 0, b = 0;
    for (int k = 0; k < na; ++k) {
      q0[k] = a;
      t0[k] = b;
      a += pad_rows(pairs[k].nq);
      b += pad_rows(pairs[k].nt);
    }
  }
  // B operands per pass: boxes of the B tile rows
  CUtensorMap tmQA, tmTA, tmQAc, tmTAc, tmOnes, tmTB[2], tmTBx[2], tmQB[2], tmQBx[2];
  bool maps_ok = make_operand_map(&tmQA, qb, q_rows, kTcBM) && make_operand_map(&tmQAc, qbc, q_rows, kTcBM) &&
                 make_ext_map(&tmOnes, ones, kTcBM, kTcBM);
  for (int ps = 0; ps < 2 && maps_ok; ++ps) {
    const int box = kTcBN1;
    maps_ok = make_operand_map(&tmTB[ps], tb, t_rows, box) && make_ext_map(&tmTBx[ps], tx, t_rows, box);
    if (maps_ok && mutual)
      maps_ok = make_operand_map(&tmQB[ps], qb, q_rows, box) && make_ext_map(&tmQBx[ps], qx, q_rows, box);
  }
  if (maps_ok && mutual)
    maps_ok = make_operand_map(&tmTA, tb, t_rows, kTcBM) && make_operand_map(&tmTAc, tbc, t_rows, kTcBM);
  if (!maps_ok) return set_error(ctx, PSIFT_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  std::vector<TcPair> tcp(2 * na);
  std::vector<RerankJob> rj(2 * na);
  TcPlan plan[4] = {};
  int ctas1[2] = {0, 0};
  const int tc_ctas = target_ctas;  // tile ranges per pass (one CTA each; one resident per SM)
  long long cf = 0;
  // one direction: A rows matched against B rows
  auto add_problem = [&](int slot, int nA, int nB, const float* an, const float* bn, long long a_row0,
                         long long b_row0, float* thr_rows, int* rowmap_rows) {
    TcPair& T = tcp[slot];
    std::memset(&T, 0, sizeof T);
    T.ccount = ccount + slot;
    T.rowmap = rowmap_rows;
    T.na = nA;
    T.nb = nB;
    T.an = an;
    T.bn = bn;
    T.top2 = top2 + 2 * cf;
    T.thr = thr_rows;
    T.coll_idx = coll_idx + (long long)kTcColl * cf;
    T.coll_cnt = coll_cnt + cf;
    cf += (long long)kTcSplits * nA;
    T.a_row0 = (int)a_row0;
    T.b_row0 = (int)b_row0;
    T.bt[0] = T.bt[1] = (nB + kTcBN1 - 1) / kTcBN1;
    T.at[0] = (nA + kTcBM - 1) / kTcBM;
  };
  // pass 1's tile order of one direction: problems in order, equal ranges over the CTAs
  auto plan_pass1 = [&](int dir) {
    long long total = 0;
    int bt_max = 1;
    for (int k = 0; k < na; ++k) {
      TcPair& T = tcp[dir * na + k];
      T.g0[0] = total;
      total += (long long)T.at[0] * T.bt[0];
      bt_max = std::max(bt_max, T.bt[0]);
    }
    long long r = std::max<long long>((total + tc_ctas - 1) / tc_ctas,
                                      (bt_max - 1 + kTcSplits - 2) / (kTcSplits - 1));
    r = std::max<long long>(r, 1);
    plan[2 * dir] = TcPlan{total, (int)r, 0};
    ctas1[dir] = (int)((total + r - 1) / r);
  };
  for (int k = 0; k < na; ++k) {
    MatchPair& P = pairs[k];
    P.q_row0 = (int)q0[k];
    P.t_row0 = (int)t0[k];
    P.qn = qn + q0[k];
    P.tn = tn + t0[k];
    P.tn_max = maxes + k;
    P.qn_max = maxes + na + k;
    add_problem(k, P.nq, P.nt, P.qn, P.tn, q0[k], t0[k], thr + q0[k], rowmap + q0[k]);
    const TcPair& T = tcp[k];
    rj[k] = RerankJob{P.q, P.t, P.nq, P.nt, P.qn, P.tn_max, T.top2, thr + q0[k], T.coll_idx, T.coll_cnt,
                      kTcSplits, P.best, P.second, P.best_idx, ctx->d_error + 1, opt.ratio,
                      mutual ? flags + t0[k] : nullptr};
    rj[k].ccount = ccount + k;
    rj[k].scan_count = scan_count;
    rj[k].scan_rows = scan_rows;
    rj[k].rowmap = rowmap + q0[k];
    gj[k] = GatherJob{qb + (size_t)q0[k] * 128, qbc + (size_t)q0[k] * 128, rowmap + q0[k], ccount + k};
  }
  plan_pass1(0);
  if (mutual) {
    for (int k = 0; k < na; ++k) {
      MatchPair& P = pairs[k];
      add_problem(na + k, P.nt, P.nq, P.tn, P.qn, t0[k], q0[k], thr + q_rows + t0[k], rowmap + q_rows + t0[k]);
      const TcPair& T = tcp[na + k];
      rj[na + k] = RerankJob{P.t, P.q, P.nt, P.nq, P.tn, P.qn_max, T.top2, thr + q_rows + t0[k], T.coll_idx,
                             T.coll_cnt, kTcSplits, P.col_best, nullptr, P.col_idx, ctx->d_error + 1, opt.ratio,
                             flags + t0[k]};
      rj[na + k].ccount = ccount + na + k;
      rj[na + k].scan_count = scan_count + 1;
      rj[na + k].scan_rows = scan_rows + q_rows;
      rj[na + k].rowmap = rowmap + q_rows + t0[k];
      gj[na + k] = GatherJob{tb + (size_t)t0[k] * 128, tbc + (size_t)t0[k] * 128, rowmap + q_rows + t0[k],
                             ccount + na + k};
    }
    plan_pass1(1);
  }
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_pairs, pairs.data(), sizeof(MatchPair) * na, cudaMemcpyHostToDevice, st));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_plan, plan, sizeof plan, cudaMemcpyHostToDevice, st));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_tcp, tcp.data(), sizeof(TcPair) * tcp.size(), cudaMemcpyHostToDevice, st));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_rj, rj.data(), sizeof(RerankJob) * rj.size(), cudaMemcpyHostToDevice, st));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_gj, gj.data(), sizeof(GatherJob) * gj.size(), cudaMemcpyHostToDevice, st));
  StageScope sc(ctx, STAGE_MATCH);
  int max_a = 0, max_b = 0;
  {
    for (int k = 0; k < na; ++k) {
      bj[2 * k] = Bf16Job{pairs[k].q, pairs[k].nq, qb + (size_t)q0[k] * 128, qn + q0[k], maxes + na + k,
                          qx + (size_t)q0[k] * 16, (int)pad_rows(pairs[k].nq), tcp[k].top2};
      bj[2 * k + 1] = Bf16Job{pairs[k].t, pairs[k].nt, tb + (size_t)t0[k] * 128, tn + t0[k], maxes + k,
                              tx + (size_t)t0[k] * 16, (int)pad_rows(pairs[k].nt),
                              mutual ? tcp[na + k].top2 : nullptr};
      max_a = std::max(max_a, pairs[k].nq);
      max_b = std::max(max_b, pairs[k].nt);
    }
    bj[2 * na] = Bf16Job{nullptr, 0, nullptr, nullptr, nullptr, ones, kTcBM, nullptr};
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_bj, bj.data(), sizeof(Bf16Job) * bj.size(), cudaMemcpyHostToDevice, st));
    const int ext_rows = (int)std::max(pad_rows(std::max(max_a, max_b)), (long long)kTcBM);
    cudaError_t e = launch_to_bf16(d_bj, 2 * na + 1, ext_rows, st);
    ctx->launches++;
    if (e != cudaSuccess) return cuda_error(ctx, e, "to_bf16");
  }
  // forward: queries vs targets; reverse (mutual): matched targets vs queries
  for (int dir = 0; dir < (mutual ? 2 : 1); ++dir) {
    const CUtensorMap& A = dir == 0 ? tmQA : tmTA;
    const CUtensorMap& Ac = dir == 0 ? tmQAc : tmTAc;
    const CUtensorMap* B = dir == 0 ? tmTB : tmQB;    // [pass]
    const CUtensorMap* Bx = dir == 0 ? tmTBx : tmQBx;
    TcPair* probs = d_tcp + dir * na;
    TcPlan* pl = d_plan + 2 * dir;
    const RerankJob* jobs_dir = d_rj + dir * na;
    const int rows = dir == 0 ? max_a : max_b;
    const char* what = "match_tc pass 1";
    cudaError_t e = launch_match_tc(A, B[0], tmOnes, Bx[0], probs, na, pl, ctas1[dir], ctx->d_error, 0, st);
    if (e == cudaSuccess && (what = "window", true)) e = launch_window(jobs_dir, na, rows, st);
    if (e == cudaSuccess && (what = "tc_plan", true)) e = launch_tc_plan(probs, na, pl, tc_ctas, st);
    if (e == cudaSuccess && (what = "gather_rows", true)) e = launch_gather_rows(d_gj + dir * na, na, rows, st);
    if (e == cudaSuccess && (what = "match_tc pass 2", true))
      e = launch_match_tc(Ac, B[1], tmOnes, Bx[1], probs, na, pl, tc_ctas, ctx->d_error, 1, st);
    if (e == cudaSuccess && (what = "rerank", true))
      e = launch_rerank(jobs_dir, na, rows, scan_rows + (dir == 0 ? 0 : q_rows), scan_count + dir, 2 * ctx->num_sms, st);
    ctx->launches += 6;
    if (e != cudaSuccess) return cuda_error(ctx, e, what);
  }
  cudaError_t e = launch_match_emit(d_pairs, na, opt.ratio, mutual, st);
  ctx->launches++;
  if (e != cudaSuccess) return cuda_error(ctx, e, "match_emit");
  return PSIFT_OK;
}

}  // namespace

// Autotuner, matchers: work items per SM in {1, 2, 4, 8} for the FP32 path (how
// many ranges of target tiles each query tile is split into follows) and the
// tensor-core path (how many equal tile ranges, one CTA each, a pass is cut into), timed on n_pairs problems of n_desc x n_desc SIFT-like
// descriptors (|N(0,1)|, L2-normalised, clipped at 0.2, renormalised; seeded);
// the fastest is kept.  report: per path (path, ms for 1, 2, 4, 8, chosen).
psift_status autotune_match(psift_ctx* ctx, uint32_t n_desc, uint32_t n_pairs, std::vector<double>& report) {
  if (n_desc < 2 || n_pairs == 0) return PSIFT_OK;
  const size_t nd = n_desc;
  std::vector<float> host(2 * nd * 130);
  uint64_t sm = 0x5EED1234ABCDull;
  auto next = [&]() {
    uint64_t z = (sm += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return (double)((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
  };
  for (size_t r = 0; r < 2 * nd; ++r) {
    float* d = host.data() + r * 128;
    double ss = 0.0;
    for (int k = 0; k < 128; ++k) {
      const double u1 = next() + 1e-12, u2 = next();
      d[k] = (float)std::fabs(std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
      ss += (double)d[k] * d[k];
    }
    double s2 = 0.0;
    for (int k = 0; k < 128; ++k) {
      d[k] = std::min((float)(d[k] / std::sqrt(ss)), 0.2f);
      s2 += (double)d[k] * d[k];
    }
    for (int k = 0; k < 128; ++k) d[k] = (float)(d[k] / std::sqrt(s2));
  }
  float* xy = host.data() + 2 * nd * 128;
  for (size_t i = 0; i < 4 * nd; ++i) xy[i] = (float)(1000.0 * next());
  float* d_in = nullptr;
  psift_match* d_out = nullptr;
  uint32_t* d_cnt = nullptr;
  cudaError_t e = cudaMalloc(&d_in, host.size() * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(psift_match) * nd * n_pairs);
  if (e == cudaSuccess) e = cudaMalloc(&d_cnt, 4 * (size_t)n_pairs);
  auto release = [&]() {
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFree(d_cnt);
  };
  if (e != cudaSuccess) {
    release();
    return cuda_error(ctx, e, "cudaMalloc(autotune match)");
  }
  e = cudaMemcpyAsync(d_in, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
  std::vector<psift_match_job> jobs(n_pairs);
  for (uint32_t k = 0; k < n_pairs; ++k)
    jobs[k] = psift_match_job{d_in, d_in + nd * 128, d_in + 2 * nd * 128, d_in + 2 * nd * 128 + 2 * nd,
                              (uint32_t)nd, (uint32_t)nd, d_out + nd * k, (uint32_t)nd, d_cnt + k};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  psift_status st = e == cudaSuccess ? PSIFT_OK : cuda_error(ctx, e, "autotune match setup");
  const int cands[4] = {1, 2, 4, 8};
  for (int path = 0; path < 2 && st == PSIFT_OK; ++path) {
    psift_match_options opt{0.8f, 0, path ? PSIFT_PRECISION_BF16_RERANK : PSIFT_PRECISION_FP32};
    double best_ms = 1e30;
    int best = ctx->tune.match_per_sm[path];
    report.push_back(path);
    for (int c = 0; c < 4 && st == PSIFT_OK; ++c) {
      ctx->tune.match_per_sm[path] = (int8_t)cands[c];
      float ms = 1e30f;
      for (int rep = 0; rep < 3 && st == PSIFT_OK; ++rep) {
        if ((st = match_batch(ctx, jobs.data(), (int)n_pairs, opt)) != PSIFT_OK) break;  // warm-up on rep 0
        if (rep == 0) continue;
        cudaEventRecord(e0, ctx->stream);
        if ((st = match_batch(ctx, jobs.data(), (int)n_pairs, opt)) != PSIFT_OK) break;
        cudaEventRecord(e1, ctx->stream);
        cudaEventSynchronize(e1);
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        ms = std::min(ms, t);
      }
      report.push_back(ms);
      if (ms < best_ms) {
        best_ms = ms;
        best = cands[c];
      }
    }
    ctx->tune.match_per_sm[path] = (int8_t)best;
    report.push_back(best);
  }
  ctx->tune.gen++;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaStreamSynchronize(ctx->stream);
  release();
  return st;
}

}  // namespace psift

using namespace psift;

extern "C" {

void psift_match_options_default(psift_match_options* o) {
  if (!o) return;
  o->ratio = 0.75f;  // DEFAULT_MATCH_RATIO, src/pipeline.rs:1047
  o->mutual = 0;
  o->precision = PSIFT_PRECISION_BF16_RERANK;
}

psift_status psift_match_options_validate(const psift_match_options* o, char* msg, size_t cap) {
  psift_ctx tmp;
  psift_status st = validate_match_options(&tmp, o);
  if (msg && cap) {
    strncpy(msg, tmp.last_error.c_str(), cap - 1);
    msg[cap - 1] = 0;
  }
  return st;
}

psift_status psift_match_batch_dev(psift_ctx* ctx, const psift_match_job* jobs, uint32_t n,
                                   const psift_match_options* opt) {
  if (!ctx || !jobs) return PSIFT_ERR_INVALID_ARGUMENT;
  psift_status st = validate_match_options(ctx, opt);
  if (st != PSIFT_OK) return st;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(ctx, e, "cudaSetDevice");
  for (uint32_t i = 0; i < n; ++i) {
    const psift_match_job& J = jobs[i];
    if (!J.d_count || (J.nq && (!J.query_descriptors || !J.query_xy || !J.out)) ||
        (J.nt && (!J.target_descriptors || !J.target_xy)))
      return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null pointer in match job");
    if (J.nq > 0 && J.nt >= 2 && J.capacity < J.nq)
      return set_error(ctx, PSIFT_ERR_CAPACITY, "match output capacity must be >= number of queries");
  }
  if (n == 0) return PSIFT_OK;
  return match_batch(ctx, jobs, (int)n, *opt);
}

psift_status psift_match_descriptors(psift_ctx* ctx, const float* q_desc, uint32_t nq, const float* t_desc, uint32_t nt,
                         const float* q_xy, const float* t_xy, const psift_match_options* opt, psift_match* out,
                         uint32_t capacity, uint32_t* count) {
  if (!ctx || !count) return PSIFT_ERR_INVALID_ARGUMENT;
  psift_status st = validate_match_options(ctx, opt);
  if (st != PSIFT_OK) return st;
  if ((nq && (!q_desc || !q_xy)) || (nt && (!t_desc || !t_xy)))
    return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null descriptor/coordinate array");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(ctx, e, "cudaSetDevice");
  *count = 0;
  if (nq == 0 || nt < 2) return PSIFT_OK;
  // Stage inputs in a separate device buffer (the batch path owns the arena).
  const size_t in_bytes = sizeof(float) * ((size_t)nq * 130 + (size_t)nt * 130) + sizeof(psift_match) * nq + 1024;
  st = io_reserve(ctx, in_bytes);
  if (st != PSIFT_OK) return st;
  char* base = ctx->io.base;
  float* d_q = (float*)base;
  float* d_t = d_q + (size_t)nq * 128;
  float* d_qxy = d_t + (size_t)nt * 128;
  float* d_txy = d_qxy + (size_t)nq * 2;
  psift_match* d_out = (psift_match*)align_up((size_t)(d_txy + (size_t)nt * 2), 16);
  uint32_t* d_count = (uint32_t*)(d_out + nq);
  st = pinned_reserve(ctx, std::max(sizeof(psift_match) * nq, (size_t)64) + 64);
  if (st != PSIFT_OK) return st;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_q, q_desc, sizeof(float) * nq * 128, cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_t, t_desc, sizeof(float) * nt * 128, cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_qxy, q_xy, sizeof(float) * nq * 2, cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(d_txy, t_xy, sizeof(float) * nt * 2, cudaMemcpyHostToDevice, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_error, 0, sizeof(uint32_t), ctx->stream));
  psift_match_job job{d_q, d_t, d_qxy, d_txy, nq, nt, d_out, nq, d_count};
  st = match_batch(ctx, &job, 1, *opt);
  if (st != PSIFT_OK) return st;
  uint32_t* hm = (uint32_t*)(ctx->pinned.base + ctx->pinned.capacity - 64);
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hm, d_count, 4, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(hm + 1, ctx->d_error, 4, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (hm[1] & kErrTimeout) return set_error(ctx, PSIFT_ERR_TIMEOUT, "tensor-core matcher wait timed out");
  const uint32_t c = hm[0];
  *count = c;
  if (c > capacity) return set_error(ctx, PSIFT_ERR_CAPACITY, "match output capacity too small");
  if (c) {
    if (!out) return set_error(ctx, PSIFT_ERR_INVALID_ARGUMENT, "null match output");
    PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->pinned.base, d_out, sizeof(psift_match) * c, cudaMemcpyDeviceToHost,
                                        ctx->stream));
    PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    std::memcpy(out, ctx->pinned.base, sizeof(psift_match) * c);
  }
  return PSIFT_OK;
}

psift_status psift_ctx_rerank_fallbacks(psift_ctx* ctx, uint64_t* rows) {
  if (!ctx || !rows) return PSIFT_ERR_INVALID_ARGUMENT;
  uint32_t h = 0;
  PSIFT_CUDA_TRY(ctx, cudaMemcpyAsync(&h, ctx->d_error + 1, 4, cudaMemcpyDeviceToHost, ctx->stream));
  PSIFT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  *rows = h;
  return PSIFT_OK;
}

}  // extern "C"
