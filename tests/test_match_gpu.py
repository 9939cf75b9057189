"""Matcher::match_ on the GPU: the exact FP32 kernel equals the CPU restatement
field for field, and the BF16 tensor-core path with certified exact re-rank
returns the identical match list (src/pipeline.rs:1744-1841)."""
import numpy as np
import pytest

import oracle as O
import psift
import synth

pytestmark = pytest.mark.gpu

FP32 = psift.PRECISION_FP32
BF16 = psift.PRECISION_BF16_RERANK


def _rand_xy(n, seed):
    return (synth.SplitMix64(seed).uniform(2 * n).reshape(n, 2) * 1000).astype(np.float32)


def _assert_same(got, ref):
    assert len(got) == len(ref), (len(got), len(ref))
    for f_got, f_ref in zip(got.dtype.names, ref.dtype.names):
        np.testing.assert_array_equal(got[f_got], ref[f_ref], err_msg=f_got)


def _case(nq, nt, seed, dup=0):
    q = synth.sift_like_descriptors(nq, seed)
    t = synth.sift_like_descriptors(nt, seed + 1)
    if dup and nt > 2 and nq > 2:
        # exact ties: duplicated targets and queries equal to targets
        t[1] = t[0]
        q[0] = t[0]
        t[nt - 1] = t[nt // 2]
    # plant near matches so the ratio test accepts some
    k = min(nq, nt) // 3
    q[:k] = t[:k] + 0.01 * synth.sift_like_descriptors(k, seed + 2)
    return q, t, _rand_xy(nq, seed + 3), _rand_xy(nt, seed + 4)


@pytest.mark.parametrize("nq,nt", [(1, 2), (5, 3), (129, 257), (300, 700), (1000, 1500)])
@pytest.mark.parametrize("mutual", [False, True])
def test_fp32_and_bf16_equal_oracle(nq, nt, mutual):
    q, t, qxy, txy = _case(nq, nt, seed=nq * 7 + nt)
    ref = O.match(q, t, qxy, txy, 0.8, mutual)
    for prec in (FP32, BF16):
        got = psift.match_arrays(q, t, qxy, txy, psift.MatchOptions(0.8, mutual, prec))
        _assert_same(got, ref)


def test_ties_and_duplicates():
    q, t, qxy, txy = _case(200, 300, seed=9, dup=1)
    for mutual in (False, True):
        ref = O.match(q, t, qxy, txy, 1.0, mutual)
        for prec in (FP32, BF16):
            _assert_same(psift.match_arrays(q, t, qxy, txy, psift.MatchOptions(1.0, mutual, prec)), ref)


def test_real_features_640x480_pair():
    a, b, _ = synth.pair_640x480()
    sift = psift.Sift.new(psift.SiftConfig().with_octaves(4))
    fa, fb = sift.detect_and_compute_u8(a), sift.detect_and_compute_u8(b)
    ref = O.match(fa.descriptors, fb.descriptors, fa.xy, fb.xy, 0.75, False)
    assert len(ref) > 50
    for prec in (FP32, BF16):
        _assert_same(psift.Matcher.new(psift.MatchOptions(0.75, False, prec)).match_(fa, fb), ref)


def test_large_4096_bf16_equals_fp32_and_rarely_falls_back():
    q, t, qxy, txy = _case(4096, 4096, seed=77)
    ctx = psift.default_context()
    import ctypes as C
    before = C.c_uint64()
    ctx.check(ctx.lib.psift_ctx_rerank_fallbacks(ctx.handle, C.byref(before)))
    f32 = psift.match_arrays(q, t, qxy, txy, psift.MatchOptions(0.8, False, FP32))
    bf = psift.match_arrays(q, t, qxy, txy, psift.MatchOptions(0.8, False, BF16))
    _assert_same(bf, f32)
    after = C.c_uint64()
    ctx.check(ctx.lib.psift_ctx_rerank_fallbacks(ctx.handle, C.byref(after)))
    assert after.value - before.value < 0.05 * 4096


def test_empty_and_degenerate():
    q, t, qxy, txy = _case(10, 10, seed=3)
    assert len(psift.match_arrays(q[:0], t, qxy[:0], txy)) == 0
    assert len(psift.match_arrays(q, t[:1], qxy, txy[:1])) == 0
    # identical descriptors everywhere: second distance 0 -> no match (second > 1e-12 fails)
    same = np.tile(q[:1], (6, 1))
    assert len(psift.match_arrays(same, same, qxy[:6], txy[:6])) == 0
