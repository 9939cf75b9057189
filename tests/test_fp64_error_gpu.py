"""The GPU's f32 detect/describe results stated against the same pipeline run in
f64 (the oracle's f64 instantiation, from the same u8 luma).

Tolerances (the f32 path's contract): keypoint position within 0.01 px and scale
within 0.01, descriptor relative L2 difference within 1e-4.  The reference's own
f32 arithmetic misses them on a few keypoints (tests/test_fp64_error_cpu.py), so
each is a fraction of the paired keypoints / features: >= 99.5 % of keypoints and
>= 99 % of features, with >= 99 % of either list paired.  Each case also checks
that the GPU is no further from f64 than the f32 restatement is (its fractions
within the tolerances are at most 0.2 percentage points lower), and prints the
statement.
"""
import numpy as np
import pytest

import fp64_error as E
import oracle as O
import psift
import synth

pytestmark = pytest.mark.gpu


def _sift(cap=4096):
    return psift.Sift.new(psift.SiftConfig().with_octaves(4).with_contrast_threshold(0.015).max_features(cap))


def _gpu_keypoint_error(u8, k64):
    kg = _sift().detect_keypoints(O.luma_to_f32(u8))
    return E.keypoint_error(kg["x"], kg["y"], kg["scale"], kg["octave"], kg["layer"], k64)


def _feature_error_of(feats: psift.Features, m64, d64):
    mg = np.stack([feats.x, feats.y, feats.scale, feats.response, feats.orientation], axis=1)
    return E.feature_error(mg, feats.descriptors, m64, d64)


def _check(label, kp, ft, u8=None, k64=None, m64=None, d64=None):
    print(E.statement(label, kp, ft))
    assert kp["paired"] >= 0.99 * max(kp["n_f32"], kp["n_f64"])
    assert kp["frac_within"] >= 0.995, kp
    assert ft["paired"] >= 0.99 * max(ft["n_f32"], ft["n_f64"])
    assert ft["frac_within"] >= 0.99, ft
    if u8 is not None:
        # The f32 restatement on the same image: the GPU may not be worse than it.
        f = O.luma_to_f32(u8)
        k32 = O.detect_keypoints(f, 4, 3, 0.015, True)
        kr = E.keypoint_error(k32["x"], k32["y"], k32["scale"], k32["octave"], k32["layer"], k64)
        m32, dd32 = O.detect_and_compute(f, 4, 3, 0.015, True, 0, 4096)
        fr = E.feature_error(m32, dd32, m64, d64)
        assert kp["frac_within"] >= kr["frac_within"] - 0.002, (kp, kr)
        assert ft["frac_within"] >= fr["frac_within"] - 0.002, (ft, fr)


@pytest.mark.parametrize("which", [0, 1])
def test_gpu_vs_f64_640x480(which):
    u8 = synth.pair_640x480(1)[which]
    k64 = O.detect_keypoints_f64(u8, 4, 3, 0.015, True)
    m64, d64 = O.detect_and_compute_f64(u8, 4, 3, 0.015, True, 0, 4096)
    kp = _gpu_keypoint_error(u8, k64)
    ft = _feature_error_of(_sift().detect_and_compute_u8(u8), m64, d64)
    _check(f"GPU 640x480 {'AB'[which]}", kp, ft, u8, k64, m64, d64)


@pytest.mark.parametrize("which", [0, 1])
def test_gpu_vs_f64_1080p(which):
    u8 = synth.pair_1080p(2)[which]
    k64 = O.detect_keypoints_f64(u8, 4, 3, 0.015, True)
    m64, d64 = O.detect_and_compute_f64(u8, 4, 3, 0.015, True, 0, 4096)
    kp = _gpu_keypoint_error(u8, k64)
    ft = _feature_error_of(_sift().detect_and_compute_u8(u8), m64, d64)
    _check(f"GPU 1920x1080 {'AB'[which]}", kp, ft, u8, k64, m64, d64)


def test_gpu_batch_vs_f64_uneven():
    # Three images of the uneven batch (the smallest of its first 44 shapes) in one
    # host batch call, uncapped as in the batched workload.
    imgs = [synth.uneven_pair(k)[0] for k in (0, 3, 43)]
    outs = _sift(0).detect_and_compute_batch_u8(imgs)
    for k, u8, feats in zip((0, 3, 43), imgs, outs):
        m64, d64 = O.detect_and_compute_f64(u8, 4, 3, 0.015, True, 0, 0)
        ft = _feature_error_of(feats, m64, d64)
        k64 = O.detect_keypoints_f64(u8, 4, 3, 0.015, True)
        kp = _gpu_keypoint_error(u8, k64)
        _check(f"GPU batch image {k} ({u8.shape[1]}x{u8.shape[0]})", kp, ft)


def test_match_distances_and_decisions_vs_f64():
    """Lowe matching stated against f64: every returned match's distance and ratio
    against the f64 values of the same f32 descriptors (relative error within 1e-5:
    128 f32 products summed in order), and the f64 ratio test taking the same
    decisions for every query whose f64 ratio lies more than 1e-5 from the threshold."""
    rng = np.random.default_rng(5)
    t_desc = synth.sift_like_descriptors(3000, 71)
    q_desc = np.concatenate([synth.perturbed_queries(t_desc, 1500, 72, 0.05)[0], synth.sift_like_descriptors(1500, 73)])
    q_xy = rng.uniform(0, 1000, (len(q_desc), 2)).astype(np.float32)
    t_xy = rng.uniform(0, 1000, (len(t_desc), 2)).astype(np.float32)
    ratio = 0.8
    got = psift.match_arrays(q_desc, t_desc, q_xy, t_xy, psift.MatchOptions(ratio=ratio))
    # f64 nearest / second-nearest of every query
    q64, t64 = q_desc.astype(np.float64), t_desc.astype(np.float64)
    d2 = (q64 ** 2).sum(1)[:, None] + (t64 ** 2).sum(1)[None, :] - 2.0 * q64 @ t64.T
    d2 = np.maximum(d2, 0.0)
    order = np.argsort(d2, axis=1)[:, :2]
    best = np.sqrt(d2[np.arange(len(q64)), order[:, 0]])
    second = np.sqrt(d2[np.arange(len(q64)), order[:, 1]])
    r64 = best / second
    qi = got["query_index"].astype(np.int64)
    ti = got["target_index"].astype(np.int64)
    exact = np.sqrt(((q64[qi] - t64[ti]) ** 2).sum(1))
    rel_d = np.abs(got["distance"].astype(np.float64) - exact) / exact
    rel_r = np.abs(got["ratio"].astype(np.float64) - r64[qi]) / r64[qi]
    accepted64 = r64 < ratio
    clear = np.abs(r64 - ratio) > 1e-5
    gpu_acc = np.zeros(len(q64), bool)
    gpu_acc[qi] = True
    print(f"matching vs f64: {len(got)} matches, distance rel. error max {rel_d.max():.2e}, ratio rel. error max "
          f"{rel_r.max():.2e}; decisions equal on {int((gpu_acc == accepted64)[clear].sum())} of {int(clear.sum())} "
          f"queries clear of the threshold by 1e-5 ({int((~clear).sum())} within)")
    assert len(got) > 1000
    assert rel_d.max() <= 1e-5 and rel_r.max() <= 1e-5
    assert np.array_equal(gpu_acc[clear], accepted64[clear])
    assert (order[qi[clear[qi]], 0] == ti[clear[qi]]).all()
