"""The reference's invariance sweeps (tests/invariance_sweeps.rs:83-217) on its own
sample image, run through the CPU restatement: the minimum similarity-inlier
counts and the 2 deg / 3 % model errors pin detection, description, matching
and similarity RANSAC together."""
import numpy as np
import pytest

import oracle as O
import sweep_cases as S


def _extract(u8):
    return O.detect_and_compute(O.luma_to_f32(u8), S.SWEEP_OCTAVES, S.SWEEP_SCALES, 0.015, True, 0, 4096)


def _match(a, b):
    return O.match(a[1], b[1], a[0][:, :2], b[0][:, :2], 0.75)


def _similarity(m):
    mask, model = O.similarity_ransac(m, 3.0)
    return int(mask.sum()), model


@pytest.mark.parametrize("which", ["scale", "rotation"])
def test_invariance_sweep_restatement(which):
    rows = S.run_sweeps(_extract, _match, _similarity, which=(which,))
    for r in rows:
        print("%-26s inliers %5d (min %4d)  scale %.4f  rotation %.2f" % r)


def test_sweep_warps():
    base = S.aerial_west_luma()
    assert base.shape == (720, 840)
    # rotation by 0 keeps every pixel; by 180 it flips both axes inside the border
    # (f32 sin(pi) is not 0, so border pixels map just outside the source and stay 0)
    np.testing.assert_array_equal(S.rotate_bilinear(base, 0.0), base)
    r180 = S.rotate_bilinear(base, 180.0)
    assert np.abs(r180[1:-1, 1:-1].astype(int) - base[::-1, ::-1][1:-1, 1:-1].astype(int)).max() <= 1
    # resizing to the same size is a copy; a constant image stays constant
    np.testing.assert_array_equal(S.resize_catmull_rom(base, 840, 720), base)
    c = np.full((64, 80), 77, np.uint8)
    for nw, nh in ((20, 16), (160, 128), (33, 47)):
        np.testing.assert_array_equal(S.resize_catmull_rom(c, nw, nh), np.full((nh, nw), 77, np.uint8))
