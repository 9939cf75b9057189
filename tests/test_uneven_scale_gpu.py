"""Parity at the size of the batched uneven workload: the largest images of the
64-image uneven batch (the largest, 3486 x 6627, portrait; 3788 x 4396; and the
widest landscape image, 3719 x 1906), detected together in one call of the batch
entry with the feature cap off (the batched workload's setting, up to ~17k
features per image).

Against the f32 restatement: positions and responses identical, scale within
2 ulp, orientation within 1e-3 rad and descriptor relative L2 within 1e-4 for at
least 99.5 % of the features (the bar of the detect parity tests).  Against the
f64 run of the same pipeline: keypoints within 0.01 px / 0.01 scale and
descriptors within 1e-4 relative L2 (the f32 contract), with the fractions the
f64 error tests use."""
import numpy as np
import pytest

import fp64_error as E
import oracle as O
import psift
import synth

pytestmark = pytest.mark.gpu

PAIRS = (23, 54, 45)  # indices into synth.uneven_batch_shapes(64)


def _sift():
    return psift.Sift.new(psift.SiftConfig().with_octaves(4).with_contrast_threshold(0.015).max_features(0))


@pytest.fixture(scope="module")
def batch():
    imgs = [synth.uneven_pair(k)[0] for k in PAIRS]
    outs = _sift().detect_and_compute_batch_u8(imgs)
    return imgs, outs


def test_shapes_are_the_largest(batch):
    shapes = synth.uneven_batch_shapes(64)
    areas = sorted((h * w for h, w in shapes), reverse=True)
    imgs, outs = batch
    assert imgs[0].shape[0] * imgs[0].shape[1] == areas[0]
    assert imgs[2].shape[1] > 2 * imgs[2].shape[0] - 200  # landscape, aspect ~2
    assert max(len(f) for f in outs) > 10000


@pytest.mark.parametrize("j", range(len(PAIRS)))
def test_uncapped_batch_vs_f32_restatement(batch, j):
    imgs, outs = batch
    got = outs[j]
    meta, desc = O.detect_and_compute(O.luma_to_f32(imgs[j]), 4, 3, 0.015, True, 0, 0)
    assert len(got) == meta.shape[0] and len(got) > 3000
    np.testing.assert_array_equal(got.x, meta[:, 0])
    np.testing.assert_array_equal(got.y, meta[:, 1])
    np.testing.assert_allclose(got.scale, meta[:, 2], rtol=2.5e-7, atol=0)
    np.testing.assert_array_equal(got.response, meta[:, 3])
    dth = np.abs(got.orientation - meta[:, 4])
    dth = np.minimum(dth, 2 * np.pi - dth)
    rel = np.linalg.norm(got.descriptors - desc, axis=1) / np.maximum(np.linalg.norm(desc, axis=1), 1e-12)
    good = (dth <= 1e-3) & (rel <= 1e-4)
    print(f"uneven image {PAIRS[j]} {imgs[j].shape[1]}x{imgs[j].shape[0]}: {len(got)} features, "
          f"{good.mean() * 100:.3f} % within 1e-3 rad / 1e-4 rel. L2 of the f32 restatement")
    assert good.mean() >= 0.995


@pytest.mark.parametrize("j", range(len(PAIRS)))
def test_uncapped_batch_vs_f64(batch, j):
    imgs, outs = batch
    u8 = imgs[j]
    m64, d64 = O.detect_and_compute_f64(u8, 4, 3, 0.015, True, 0, 0)
    feats = outs[j]
    mg = np.stack([feats.x, feats.y, feats.scale, feats.response, feats.orientation], axis=1)
    ft = E.feature_error(mg, feats.descriptors, m64, d64)
    k64 = O.detect_keypoints_f64(u8, 4, 3, 0.015, True)
    kg = _sift().detect_keypoints(O.luma_to_f32(u8))
    kp = E.keypoint_error(kg["x"], kg["y"], kg["scale"], kg["octave"], kg["layer"], k64)
    print(E.statement(f"GPU uneven image {PAIRS[j]} ({u8.shape[1]}x{u8.shape[0]}, uncapped)", kp, ft))
    assert kp["paired"] >= 0.99 * max(kp["n_f32"], kp["n_f64"])
    assert kp["frac_within"] >= 0.995, kp
    assert ft["paired"] >= 0.99 * max(ft["n_f32"], ft["n_f64"])
    assert ft["frac_within"] >= 0.99, ft
