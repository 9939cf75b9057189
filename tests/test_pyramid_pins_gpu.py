"""The reference's pyramid-structure test (tests/pipeline_tests.rs:1366-1381) on the
CUDA path: the 512 x 512 checkerboard without first-octave upsampling gives
`octaves` octaves of scales + 3 Gaussian and scales + 2 DoG planes (512, 256, 128
on a side), and the extrema extracted from that pyramid are the restatement's."""
import numpy as np
import pytest

import oracle as O
import psift
from test_oracle_pins import checkerboard_512

pytestmark = pytest.mark.gpu


def test_checkerboard_pyramid_structure_and_extrema():
    img = checkerboard_512()
    cfg = psift.SiftConfig().upsample_first_octave(False)
    octs = psift.build_pyramid(img, cfg)
    assert len(octs) == cfg.octaves == 3
    for o, (g, d) in enumerate(octs):
        side = 512 >> o
        assert g.shape == (cfg.scales + 3, side, side) and d.shape == (cfg.scales + 2, side, side)
    got = psift.Sift.new(cfg).detect_keypoints(img)
    ref = O.detect_keypoints(img, cfg.octaves, cfg.scales, 0.015, False)
    assert len(got) == len(ref) > 0
    for f in ("x", "y", "response", "octave", "layer"):
        np.testing.assert_array_equal(got[f], ref[f], err_msg=f)
