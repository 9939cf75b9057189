"""Parity of the CUDA detect/describe path with the CPU restatement (oracle).

Keypoints (pyramid, DoG, extrema, Taylor refinement, ordering, cap) must be
identical; features must agree within the stated tolerances:
  position/scale/response: identical to the oracle (scale within 2 ulp: the only
  libm call on that path, k^ds, is correctly rounded on the GPU and glibc's powf
  is not always),
  orientation: |d theta| <= 1e-3 rad,
  descriptor: relative L2 difference <= 1e-4,
for at least 99.5% of features, every feature within a looser bound (orientation
histograms are summed in a different order, and atan2f/expf differ from glibc by
an ulp, which can move a near-tied histogram peak).
"""
import numpy as np
import pytest

import oracle as O
import psift
import synth

pytestmark = pytest.mark.gpu


def _img640(seed=1):
    a, b, _ = synth.pair_640x480(seed)
    return a, b


def _cfg4():
    return psift.SiftConfig().with_octaves(4).with_contrast_threshold(0.015)


def test_keypoints_identical_640x480():
    a, _ = _img640()
    fa = O.luma_to_f32(a)
    ref = O.detect_keypoints(fa, 4, 3, 0.015, True)
    got = psift.Sift.new(_cfg4()).detect_keypoints(fa)
    assert len(got) == len(ref) and len(ref) > 50
    for f in ("x", "y", "response"):
        np.testing.assert_array_equal(got[f], ref[f], err_msg=f)
    np.testing.assert_array_equal(got["octave"], ref["octave"])
    np.testing.assert_array_equal(got["layer"], ref["layer"])
    np.testing.assert_allclose(got["scale"], ref["scale"], rtol=2.5e-7, atol=0)


@pytest.mark.parametrize("upsample", [True, False])
@pytest.mark.parametrize("octaves,scales", [(4, 3), (3, 5), (2, 10)])
def test_keypoints_identical_configs(upsample, octaves, scales):
    a = synth.blob_image(320, 240, 80, 2.0, 10.0, seed=7 + octaves)
    fa = O.luma_to_f32(a)
    ref = O.detect_keypoints(fa, octaves, scales, 0.015, upsample)
    cfg = psift.SiftConfig().with_octaves(octaves).with_scales(scales).upsample_first_octave(upsample)
    got = psift.Sift.new(cfg).detect_keypoints(fa)
    assert len(got) == len(ref)
    for f in ("x", "y", "response", "octave", "layer"):
        np.testing.assert_array_equal(got[f], ref[f], err_msg=f)
    np.testing.assert_allclose(got["scale"], ref["scale"], rtol=2.5e-7, atol=0)


def _compare_features(got: psift.Features, meta, desc, frac=0.995):
    assert len(got) == meta.shape[0]
    n = len(got)
    np.testing.assert_array_equal(got.x, meta[:, 0])
    np.testing.assert_array_equal(got.y, meta[:, 1])
    np.testing.assert_allclose(got.scale, meta[:, 2], rtol=2.5e-7, atol=0)
    np.testing.assert_array_equal(got.response, meta[:, 3])
    dth = np.abs(got.orientation - meta[:, 4])
    dth = np.minimum(dth, 2 * np.pi - dth)
    rel = np.linalg.norm(got.descriptors - desc, axis=1) / np.maximum(np.linalg.norm(desc, axis=1), 1e-12)
    good = (dth <= 1e-3) & (rel <= 1e-4)
    assert good.mean() >= frac, (good.mean(), np.sort(rel)[-5:], np.sort(dth)[-5:])
    return dth, rel


def test_features_parity_640x480():
    a, b = _img640()
    sift = psift.Sift.new(_cfg4())
    for img in (a, b):
        fa = O.luma_to_f32(img)
        meta, desc = O.detect_and_compute(fa, 4, 3, 0.015, True, 0, 4096)
        got = sift.detect_and_compute(fa)
        _compare_features(got, meta, desc)
        got8 = sift.detect_and_compute_u8(img)
        np.testing.assert_array_equal(got8.descriptors, got.descriptors)
        np.testing.assert_array_equal(got8.x, got.x)


@pytest.mark.parametrize("cap", [4096, 700])
def test_features_parity_1080p(cap):
    a, _, _ = synth.pair_1080p()
    fa = O.luma_to_f32(a)
    meta, desc = O.detect_and_compute(fa, 4, 3, 0.015, True, 0, cap)
    got = psift.Sift.new(_cfg4().max_features(cap)).detect_and_compute(fa)
    assert len(got) == meta.shape[0] and len(got) > 0
    _compare_features(got, meta, desc)


def test_rootsift_and_uncapped():
    a = synth.blob_image(400, 300, 120, 2.0, 10.0, seed=11)
    fa = O.luma_to_f32(a)
    meta, desc = O.detect_and_compute(fa, 3, 3, 0.015, True, 1, 0)
    got = psift.Sift.new(psift.SiftConfig().descriptor_kind(1).max_features(0)).detect_and_compute(fa)
    _compare_features(got, meta, desc)


def test_small_cap_selects_stable_topk():
    a = synth.blob_image(320, 240, 80, 2.0, 10.0, seed=5)
    fa = O.luma_to_f32(a)
    meta, desc = O.detect_and_compute(fa, 3, 3, 0.015, True, 0, 37)
    got = psift.Sift.new(psift.SiftConfig().max_features(37)).detect_and_compute(fa)
    _compare_features(got, meta, desc)


@pytest.mark.parametrize("shape", [(0, 0), (2, 2), (3, 3), (5, 700), (17, 9)])
def test_tiny_and_empty_images(shape):
    rng = np.random.default_rng(0)
    img = rng.random(shape).astype(np.float32)
    meta, desc = O.detect_and_compute(img, 3, 3, 0.015, True, 0, 4096)
    got = psift.Sift().detect_and_compute(img)
    assert len(got) == meta.shape[0]


def test_constant_image_has_no_features():
    img = np.full((64, 80), 0.5, np.float32)
    assert len(psift.Sift().detect_and_compute(img)) == 0
