"""Pins of the fundamental-matrix restatement against the reference's own
tests (tests/geometry_tests.rs:99-123, :207-250), CPU only."""
import numpy as np

import oracle as O
from geometry_cases import K_720, euler_zyx_rotation, make_3d_correspondences, sampson


def test_oracle_8point_on_clean_subset():
    # tests/geometry_tests.rs:99-123: normalized 8-point on matches[..12], mean Sampson of the 80 inliers < 0.05
    m = make_3d_correspondences(80, 26, K_720, euler_zyx_rotation(12.0, -6.0, 4.0), (0.6, -0.15, 0.2))
    F = O.fit_fundamental_8point(m[:12])
    assert F is not None
    assert float(np.mean(np.sqrt(sampson(F, m[:80])))) < 0.05


def test_oracle_ransac_finds_the_inliers():
    m = make_3d_correspondences(80, 26, K_720, euler_zyx_rotation(12.0, -6.0, 4.0), (0.6, -0.15, 0.2))
    mask, F, iters = O.fundamental_ransac(m)
    assert F is not None and mask[:80].sum() >= 76 and mask[80:].sum() <= 3
    assert abs(np.linalg.norm(F) - 1.0) < 1e-12 and abs(np.linalg.det(F)) < 1e-9


def test_oracle_7point_generalises():
    # tests/geometry_tests.rs:207-250: some 7-point candidate fits the 5 held-out points (mean Sampson < 0.05)
    m = make_3d_correspondences(12, 0, K_720, euler_zyx_rotation(8.0, -4.0, 3.0), (0.5, 0.1, -0.15))
    cands = O.fit_fundamental_7point(m[:7])
    assert cands
    assert min(float(np.mean(np.sqrt(sampson(F, m[7:])))) for F in cands) < 0.05
    # with exactly 7 matches the RANSAC entry keeps one of them, all 7 points inliers
    mask, F, _ = O.fundamental_ransac(m[:7])
    assert F is not None and mask.all()
    assert min(float(np.abs(F - c).max()) for c in cands) == 0.0


def test_oracle_small_and_degenerate_inputs():
    m = make_3d_correspondences(6, 0, K_720, euler_zyx_rotation(8.0, -4.0, 3.0), (0.5, 0.1, -0.15))
    mask, F, _ = O.fundamental_ransac(m)
    assert F is None and not mask.any()  # fewer than 7
    same = np.repeat(m[:1], 30)
    mask, F, _ = O.fundamental_ransac(same)  # normalisation fails for every sample
    assert F is None and not mask.any()
