"""Catalog codes and Hamming stages on the GPU, bit-exact with the CPU
restatement (src/catalog.rs:37-45, :588-641, :707-728; src/pipeline.rs:1024-1044)."""
import numpy as np
import pytest

import oracle as O
import psift
import synth

pytestmark = pytest.mark.gpu


def _catalog(n_entries, per_entry, seed):
    d = synth.sift_like_descriptors(n_entries * per_entry, seed)
    off = np.arange(0, n_entries * per_entry + 1, per_entry, dtype=np.int64)
    return d, off


def test_quantizers_bit_exact():
    d = synth.sift_like_descriptors(1000, 5)
    d[0] = 0.065  # boundary: strictly greater
    d[1, :64] = np.nextafter(np.float32(0.065), np.float32(1))
    np.testing.assert_array_equal(psift.quantize_descriptor_u128(d), O.quantize_u128(d))
    np.testing.assert_array_equal(psift.quantize_descriptor_u8(d), O.quantize_u8(d))
    q = O.quantize_u8(d)
    np.testing.assert_array_equal(psift.dequantize_descriptor_u8(q), O.dequantize_u8(q))


@pytest.mark.parametrize("mih", [False, True])
def test_votes_equal_oracle(mih):
    cat, off = _catalog(60, 50, seed=11)
    q, src = synth.perturbed_queries(cat, 300, seed=12, noise=0.01)
    qc, cc = O.quantize_u128(q), O.quantize_u128(cat)
    ref = O.hamming_votes(qc, cc, off, mih)
    got = psift.hamming_votes(qc, cc, off, mih)
    np.testing.assert_array_equal(got, ref)
    assert ref.sum() > 0


def test_votes_uneven_entries_and_empty():
    rng = np.random.default_rng(3)
    sizes = rng.integers(0, 40, size=37)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    cat = synth.sift_like_descriptors(int(off[-1]), 21)
    q, _ = synth.perturbed_queries(cat, 100, seed=22, noise=0.02)
    qc, cc = O.quantize_u128(q), O.quantize_u128(cat)
    for mih in (False, True):
        np.testing.assert_array_equal(psift.hamming_votes(qc, cc, off, mih), O.hamming_votes(qc, cc, off, mih))


@pytest.mark.parametrize("ncat,k", [(50, 64), (5000, 64), (70000, 16), (3, 5)])
def test_topk_equal_oracle(ncat, k):
    cat = synth.sift_like_descriptors(ncat, 31 + ncat)
    q, _ = synth.perturbed_queries(cat, 77, seed=32, noise=0.02)
    qc, cc = O.quantize_u128(q), O.quantize_u128(cat)
    ridx, rdist = O.hamming_topk(qc, cc, k)
    gidx, gdist = psift.hamming_topk(qc, cc, k)
    np.testing.assert_array_equal(gdist, rdist)
    np.testing.assert_array_equal(gidx, ridx)


def test_topk_ties_keep_lower_index():
    cat = synth.sift_like_descriptors(40, 41)
    cat = np.concatenate([cat, cat, cat])  # every code three times
    q, _ = synth.perturbed_queries(cat, 20, seed=42, noise=0.0)
    qc, cc = O.quantize_u128(q), O.quantize_u128(cat)
    ridx, rdist = O.hamming_topk(qc, cc, 10)
    gidx, gdist = psift.hamming_topk(qc, cc, 10)
    np.testing.assert_array_equal(gidx, ridx)
    np.testing.assert_array_equal(gdist, rdist)


def test_l2_rerank_equal_oracle():
    cat = synth.sift_like_descriptors(3000, 51)
    q, _ = synth.perturbed_queries(cat, 64, seed=52, noise=0.02)
    qc, cc = O.quantize_u128(q), O.quantize_u128(cat)
    cand, _ = O.hamming_topk(qc, cc, 64)
    ridx, rd2 = O.l2_rerank(q, cat, cand)
    gidx, gd2 = psift.l2_rerank(q, cat, cand)
    np.testing.assert_array_equal(gidx, ridx)
    np.testing.assert_array_equal(gd2, rd2)
