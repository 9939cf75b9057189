"""The CPU restatement (oracle) passes the reference's own known-answer and
property tests for the hot path.  This pins the oracle to the reference: the
Rust reference cannot be built here and ships no numeric golden vectors."""
import math

import numpy as np
import pytest

import oracle as O
import synth
from ransac_cases import (PTS_13, PTS_60, TRUE_H_13, TRUE_H_60, correspondences, homography_13,
                          homography_80pct_outliers, project, seeded_72, similarity_14)


def checkerboard_512():
    """build_mock_checkerboard_512x512 (tests/pipeline_tests.rs:31-51)."""
    img = np.zeros((512, 512), np.float32)
    for y in range(64, 448):
        for x in range(64, 448):
            cy, cx = (y - 64) // 32, (x - 64) // 32
            if (cx + cy) % 2 == 0:
                ly, lx = (y - 64) % 32, (x - 64) % 32
                if 4 <= ly < 28 and 4 <= lx < 28:
                    img[y, x] = 1.0
    return img


def test_gaussian_kernel_properties():
    # tests/pipeline_tests.rs:192-226, :1067-1068
    k = O.gaussian_kernel_1d(1.6)
    assert len(k) % 2 == 1
    assert abs(float(k.astype(np.float64).sum()) - 1.0) < 1e-5
    assert np.allclose(k, k[::-1], atol=1e-6)
    assert len(O.gaussian_kernel_1d(4.0)) == 25
    blurred = O.gaussian_blur(np.full((64, 64), 0.75, np.float32), 1.6)
    assert np.abs(blurred - 0.75).max() < 1e-4


def test_octave_dimensions():
    # tests/pipeline_tests.rs:168-189 (generate_dog_space: no upsampling)
    pyr = O.Pyramid(checkerboard_512(), 3, 3, upsample=False)
    assert pyr.num_octaves == 3
    assert [pyr.octave_info(o)[:2] for o in range(3)] == [(512, 512), (256, 256), (128, 128)]


def test_checkerboard_keypoints_bounds_threshold_and_scale_bands():
    # tests/pipeline_tests.rs:54-165
    img = checkerboard_512()
    kps = O.detect_keypoints(img, 3, 3, 0.015, upsample=False)
    assert len(kps) > 0
    assert np.all((kps["x"] >= 0) & (kps["x"] < 512) & (kps["y"] >= 0) & (kps["y"] < 512))
    assert np.all(np.abs(kps["response"]) > 0.015) and np.all(kps["scale"] > 0)
    again = O.detect_keypoints(img, 3, 3, 0.015, upsample=False)
    np.testing.assert_array_equal(kps, again)
    k = np.float32(2.0) ** (np.float32(1.0) / np.float32(3.0))
    expected = [np.float32(1.6) * np.float32(2 ** o) * k ** s for o in range(3) for s in range(1, 4)]
    lo, hi = k ** np.float32(-0.5) - np.float32(1e-4), k ** np.float32(0.5) + np.float32(1e-4)
    for s in kps["scale"]:
        assert any(e * lo <= s <= e * hi for e in expected)


def test_taylor_subpixel_refinement_on_blob():
    # tests/pipeline_tests.rs:942-987: error < 0.12 px at (32.35, 28.65)
    cx, cy = np.float32(32.35), np.float32(28.65)
    sigma = np.float32(math.sqrt(2.0))
    two = np.float32(2.0) * sigma * sigma
    ys, xs = np.mgrid[0:64, 0:64].astype(np.float32)
    img = np.exp(-((xs - cx) ** 2 + (ys - cy) ** 2) / two).astype(np.float32)
    kps = O.detect_keypoints(img, 1, 3, 0.015, upsample=True)
    assert len(kps) > 0
    d = np.hypot(kps["x"] - cx, kps["y"] - cy)
    assert d.min() < 0.12


def test_secondary_orientation_splitting():
    # tests/pipeline_tests.rs:990-1033
    img = np.zeros((96, 96), np.float32)
    img[24:72, 42:54] = 1.0
    img[42:54, 24:72] = 1.0
    kps = O.detect_keypoints(img, 2, 3, 0.015, upsample=True)
    meta, _ = O.detect_and_compute(img, 2, 3, 0.015, True, 0, 4096)
    assert len(kps) > 0 and meta.shape[0] > len(kps)
    split = False
    for kp in kps:
        sel = meta[(np.abs(meta[:, 0] - kp["x"]) < 1e-5) & (np.abs(meta[:, 1] - kp["y"]) < 1e-5) &
                   (np.abs(meta[:, 2] - kp["scale"]) < 1e-5)]
        if len(sel) >= 2 and abs(sel[0, 4] - sel[1, 4]) > 0.1:
            split = True
    assert split


def test_descriptor_invariants():
    # tests/pipeline_tests.rs:255-279
    meta, desc = O.detect_and_compute(checkerboard_512(), 3, 3, 0.015, True, 0, 4096)
    assert meta.shape[0] > 0
    assert np.all((meta[:, 4] >= 0) & (meta[:, 4] < 2 * np.pi))
    assert np.all(np.abs(np.linalg.norm(desc, axis=1) - 1.0) < 1e-4)
    assert np.all((desc >= 0) & (desc <= 1))


def test_upsampling_coordinate_consistency_and_gain():
    # tests/pipeline_tests.rs:1139-1219; a fine-blob synthetic image stands in for the
    # sample JPEG in the "more features" half
    cx, cy = np.float32(32.35), np.float32(28.65)
    two = np.float32(2.0) * np.float32(2.2) * np.float32(2.2)
    ys, xs = np.mgrid[0:64, 0:64].astype(np.float32)
    img = np.exp(-((xs - cx) ** 2 + (ys - cy) ** 2) / two).astype(np.float32)
    nat = O.detect_keypoints(img, 2, 3, 0.015, upsample=False)
    up = O.detect_keypoints(img, 2, 3, 0.015, upsample=True)
    bn = nat[np.argmin(np.hypot(nat["x"] - cx, nat["y"] - cy))]
    bu = up[np.argmin(np.hypot(up["x"] - cx, up["y"] - cy))]
    assert math.hypot(bu["x"] - bn["x"], bu["y"] - bn["y"]) <= 0.5
    tex = O.luma_to_f32(synth.blob_image(420, 360, 400, 1.0, 3.0, seed=99))
    f_nat, _ = O.detect_and_compute(tex, 4, 3, 0.015, False, 0, 4096)
    f_up, d_up = O.detect_and_compute(tex, 4, 3, 0.015, True, 0, 4096)
    assert f_up.shape[0] > f_nat.shape[0]
    self_matches = O.match(d_up, d_up, f_up[:, :2], f_up[:, :2], 0.75, False)
    assert len(self_matches) > 100


def test_rootsift_and_u8_roundtrip():
    # tests/pipeline_tests.rs:1283-1332
    meta, desc = O.detect_and_compute(checkerboard_512(), 3, 3, 0.015, True, 1, 4096)
    assert np.all(np.abs(np.linalg.norm(desc, axis=1) - 1.0) < 1e-4)
    _, sift = O.detect_and_compute(checkerboard_512(), 3, 3, 0.015, True, 0, 4096)
    back = O.dequantize_u8(O.quantize_u8(sift))
    assert np.abs(back - sift).max() < 0.03


def test_mutual_nearest_neighbour_removes_many_to_one():
    # tests/pipeline_tests.rs:1222-1280: two queries near one target -> mutual keeps one
    t = synth.sift_like_descriptors(5, 7)
    q = np.stack([t[0] * 0.99 + 0.01 * t[1], t[0] * 0.98 + 0.02 * t[2], t[3]]).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    xy = np.zeros((5, 2), np.float32)
    fwd = O.match(q, t, xy[:3], xy, 0.9, False)
    mut = O.match(q, t, xy[:3], xy, 0.9, True)
    assert sum(fwd["target_index"] == 0) == 2
    assert sum(mut["target_index"] == 0) == 1


def test_similarity_ransac_keeps_10_of_14():
    # tests/pipeline_tests.rs:421-445
    m = similarity_14()
    mask, model = O.similarity_ransac(m, 3.0)
    assert mask.sum() == 10 and mask[:10].all()
    a, b, tx, ty, scale, rot = model
    assert abs(tx + 341.0) < 1e-3 and abs(ty) < 1e-3 and abs(scale - 1.0) < 1e-3 and abs(rot) < 1e-3
    s = O.summarize_tracking(m, np.full(14, 1.26), np.r_[np.ones(10), np.full(4, 2.5)],
                             np.r_[np.full(10, 1.26), np.full(4, 2.52)], np.r_[np.ones(10), np.full(4, 0.2)])
    assert (s.raw_match_count, s.match_count) == (14, 10)
    assert abs(s.mean_dx + 341.0) < 1e-3 and abs(s.mean_dy) < 1e-3
    assert abs(s.median_dx + 341.0) < 1e-3 and abs(s.median_dy) < 1e-3


def _reproj_ok(H, H_true, pts, tol):
    for (x, y) in pts:
        tx, ty = project(H_true, x, y)
        px, py = project(H, x, y)
        assert math.hypot(tx - px, ty - py) < tol


def test_homography_ransac_keeps_10_of_13():
    # tests/pipeline_tests.rs:448-524
    mask, H = O.homography_ransac(homography_13(), 3.0)
    assert mask.sum() == 10 and mask[:10].all()
    _reproj_ok(H, TRUE_H_13, PTS_13, 0.05)


def test_homography_ransac_under_80_percent_outliers():
    # tests/homography_properties.rs:71-149
    mask, H = O.homography_ransac(homography_80pct_outliers(), 3.0)
    assert mask.sum() == 12 and mask[:12].all()
    _reproj_ok(H, TRUE_H_60, PTS_60, 0.05)


def test_seeded_ransac_deterministic_and_default_seeds():
    # tests/homography_properties.rs:152-237
    m = seeded_72()
    seed = 0x123456789ABCDEF0
    a = O.homography_ransac(m, 3.0, seed)
    b = O.homography_ransac(m, 3.0, seed)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    d1 = O.homography_ransac(m, 3.0)
    d2 = O.homography_ransac(m, 3.0, None)
    np.testing.assert_array_equal(d1[0], d2[0])
    s1 = O.similarity_ransac(m, 3.0, seed)
    s2 = O.similarity_ransac(m, 3.0, seed)
    np.testing.assert_array_equal(s1[0], s2[0])


@pytest.mark.parametrize("case", range(16))
def test_ransac_never_panics_on_arbitrary_input(case):
    # tests/homography_properties.rs:30-68 (collinear, repeated, extreme coordinates)
    rng = np.random.default_rng(case)
    pts = [((float(rng.uniform(-1e5, 1e5)), float(rng.uniform(-1e5, 1e5))),
            (float(rng.uniform(-1e5, 1e5)), float(rng.uniform(-1e5, 1e5)))) for _ in range(4 + case % 17)]
    for m in (correspondences(pts),
              correspondences([((i, 7.0), (3.0, i)) for i in (0.0, 1.0, 2.0, 3.0)]),
              correspondences([pts[0]] * 4),
              correspondences([((np.float32(3.4e38) * (1 if i % 2 else -1), 1e30), p[1]) for i, p in enumerate(pts)])):
        mask, _ = O.homography_ransac(m, 3.0)
        assert mask.sum() <= len(m)


def test_splitmix64_matches_reference_constants():
    # splitmix64_next (src/pipeline.rs:1862-1868): first outputs for seed 0
    s = np.array([0], np.uint64)
    import ctypes as C
    out = [O.lib().oracle_splitmix64_next(s.ctypes.data_as(C.POINTER(C.c_uint64))) for _ in range(3)]
    r = synth.SplitMix64(0).next_u64(3)
    assert out == [int(v) for v in r]
    assert out[0] == 0xE220A8397B1DCDAF
