"""RANSAC on the GPU returns the same inliers and model as the CPU restatement
for the same seed (src/pipeline.rs:1862-2755), including the reference's own
known-answer cases."""
import math

import numpy as np
import pytest

import oracle as O
import psift
import synth
from ransac_cases import (PTS_13, PTS_60, TRUE_H_13, TRUE_H_60, correspondences, homography_13,
                          homography_80pct_outliers, project, seeded_72, similarity_14)

pytestmark = pytest.mark.gpu


def _gpu_h(m, thr=3.0, seed=None):
    inl, H = psift.Homography.estimate(m, psift.RansacOptions(thr, seed))
    mask = np.isin(np.arange(len(m)), inl["query_index"]) if len(m) else np.zeros(0, bool)
    return inl, H


def _same_h(m, thr=3.0, seed=None):
    rmask, rH = O.homography_ransac(m, thr, seed)
    inl, H = psift.Homography.estimate(m, psift.RansacOptions(thr, seed))
    got_idx = inl["query_index"] if len(inl) else np.zeros(0, np.uint32)
    np.testing.assert_array_equal(got_idx, m["query_index"][rmask])
    assert (H is None) == (rH is None)
    if H is not None:
        np.testing.assert_array_equal(H, rH)


def _same_s(m, thr=3.0, seed=None):
    rmask, rmodel = O.similarity_ransac(m, thr, O.DEFAULT_SIMILARITY_RANSAC_SEED if seed is None else seed)
    inl, model = psift.Homography.estimate_similarity(m, psift.RansacOptions(thr, seed))
    np.testing.assert_array_equal(inl["query_index"], m["query_index"][rmask])
    assert (model is None) == (rmodel is None)
    if model is not None:
        np.testing.assert_array_equal(model[:5], rmodel[:5])
        assert abs(float(model[5]) - float(rmodel[5])) <= 1e-4  # rotation_deg: atan2f may differ by an ulp


def test_known_answer_similarity_14():
    _same_s(similarity_14())
    inl, model = psift.Homography.estimate_similarity(similarity_14())
    assert len(inl) == 10 and abs(model[2] + 341.0) < 1e-3


def test_known_answer_homography_13_and_80pct():
    for m, H_true, pts, n_in in ((homography_13(), TRUE_H_13, PTS_13, 10),
                                 (homography_80pct_outliers(), TRUE_H_60, PTS_60, 12)):
        _same_h(m)
        inl, H = psift.Homography.estimate(m)
        assert len(inl) == n_in
        for (x, y) in pts:
            tx, ty = project(H_true, x, y)
            px, py = project(H, x, y)
            assert math.hypot(tx - px, ty - py) < 0.05


def test_seeded_determinism_and_seeds():
    m = seeded_72()
    for seed in (None, 0x123456789ABCDEF0, 7):
        _same_h(m, seed=seed)
        _same_s(m, seed=seed)


def _synthetic(n, outlier_ratio, seed):
    H = synth.perspective_h(1920, 1080, 12.0, 1.1, 1e-4, -5e-5)
    q, t, r, _ = synth.correspondences(n, outlier_ratio, H, 1920, 1080, seed)
    rows = [(i, i, q[i, 0], q[i, 1], t[i, 0], t[i, 1], np.float32(0.1), r[i], t[i, 0] - q[i, 0], t[i, 1] - q[i, 1])
            for i in range(n)]
    return np.array(rows, dtype=O.MATCH_DTYPE)


@pytest.mark.parametrize("n,outliers", [(5, 0.0), (40, 0.3), (300, 0.5), (2000, 0.7), (6000, 0.2)])
def test_synthetic_equal_oracle(n, outliers):
    m = _synthetic(n, outliers, seed=n)
    _same_h(m)
    _same_s(m)


@pytest.mark.parametrize("n", [0, 1, 2, 3, 4])
def test_tiny_inputs(n):
    m = _synthetic(max(n, 1), 0.0, seed=3)[:n]
    _same_h(m)
    _same_s(m)


@pytest.mark.parametrize("case", range(6))
def test_degenerate_inputs_equal_oracle(case):
    rng = np.random.default_rng(case)
    pts = [((float(rng.uniform(-1e5, 1e5)), float(rng.uniform(-1e5, 1e5))),
            (float(rng.uniform(-1e5, 1e5)), float(rng.uniform(-1e5, 1e5)))) for _ in range(4 + case * 3)]
    for m in (correspondences(pts),
              correspondences([((i, 7.0), (3.0, i)) for i in (0.0, 1.0, 2.0, 3.0)]),
              correspondences([pts[0]] * 4)):
        _same_h(m)
        _same_s(m)
