"""The f32 restatement against the f64 run of the same pipeline: the error the
reference's own f32 arithmetic carries, the baseline for the GPU's statement
(tests/test_fp64_error_gpu.py).  Also checks that the f64 instantiation is the
same algorithm (same keypoint set on these images)."""
import numpy as np

import fp64_error as E
import oracle as O
import synth


def _check(label, u8):
    f = O.luma_to_f32(u8)
    k32 = O.detect_keypoints(f, 4, 3, 0.015, True)
    k64 = O.detect_keypoints_f64(u8, 4, 3, 0.015, True)
    kp = E.keypoint_error(k32["x"], k32["y"], k32["scale"], k32["octave"], k32["layer"], k64)
    m32, d32 = O.detect_and_compute(f, 4, 3, 0.015, True, 0, 4096)
    m64, d64 = O.detect_and_compute_f64(u8, 4, 3, 0.015, True, 0, 4096)
    ft = E.feature_error(m32, d32, m64, d64)
    print(E.statement(label, kp, ft))
    assert kp["paired"] >= 0.99 * max(kp["n_f32"], kp["n_f64"]) and kp["paired"] > 100
    assert kp["frac_within"] >= 0.995
    assert ft["paired"] >= 0.99 * max(ft["n_f32"], ft["n_f64"])
    assert ft["frac_within"] >= 0.99


def test_f32_restatement_vs_f64_640x480():
    a, b, _ = synth.pair_640x480(1)
    _check("640x480 A", a)
    _check("640x480 B", b)


def test_f32_restatement_vs_f64_1080p():
    a, _, _ = synth.pair_1080p(2)
    _check("1920x1080 A", a)


def test_f64_pipeline_matches_f32_on_constant_image():
    # No structure: both precisions find nothing (the reference's flat-image pin).
    u8 = np.full((120, 160), 128, np.uint8)
    assert len(O.detect_keypoints_f64(u8, 4, 3, 0.015, True)) == 0
    m, d = O.detect_and_compute_f64(u8, 4, 3, 0.015, True, 0, 4096)
    assert m.shape == (0, 5) and d.shape == (0, 128)
