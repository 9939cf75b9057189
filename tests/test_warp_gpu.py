"""warp_and_stitch (src/visualize.rs:379-483) on the GPU against the CPU
restatement: canvas bytes and origin bit-equal, and the reference's errors."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import psift

pytestmark = pytest.mark.gpu


def _rgba(rng, h, w):
    img = rng.integers(0, 256, (h, w, 4)).astype(np.uint8)
    img[..., 3] = np.where(rng.random((h, w)) < 0.8, 255, img[..., 3])
    return img


def _h(theta_deg, scale, tx, ty, p0=0.0, p1=0.0):
    th = np.deg2rad(theta_deg)
    return np.array([[scale * np.cos(th), -scale * np.sin(th), tx],
                     [scale * np.sin(th), scale * np.cos(th), ty],
                     [p0, p1, 1.0]], np.float32)


CASES = [
    ((60, 80), (50, 70), _h(0, 1, 0, 0)),
    ((60, 80), (50, 70), _h(7, 1.1, 12.5, -9.25)),
    ((121, 97), (88, 143), _h(-25, 0.8, -40.0, 30.0, 2e-4, -1e-4)),
    ((240, 320), (240, 320), _h(3, 1.02, 15.0, 4.0, 1e-5, 3e-5)),
    ((1, 1), (2, 3), _h(0, 1, 0.5, 0.5)),
    ((2, 3), (1, 1), _h(45, 2, 0, 0)),
    ((33, 17), (19, 41), _h(180, 1, 30, 20)),
]


@pytest.mark.parametrize("qshape,tshape,H", CASES)
def test_warp_and_stitch_bit_exact(qshape, tshape, H):
    rng = np.random.default_rng(qshape[0] * 131 + tshape[1])
    q, t = _rgba(rng, *qshape), _rgba(rng, *tshape)
    ref_canvas, ref_origin = O.warp_and_stitch(q, t, H)
    canvas, origin = psift.warp_and_stitch(q, t, H)
    assert origin == ref_origin
    assert canvas.shape == ref_canvas.shape
    np.testing.assert_array_equal(canvas, ref_canvas)


def test_warp_and_stitch_errors():
    rng = np.random.default_rng(5)
    q, t = _rgba(rng, 40, 50), _rgba(rng, 30, 30)
    with pytest.raises(ValueError, match="singular and cannot be inverted"):
        psift.warp_and_stitch(q, t, np.zeros((3, 3), np.float32))
    assert O.warp_and_stitch(q, t, np.zeros((3, 3), np.float32)) == -1
    # corner (w - 1, 0) projected to w = 0
    Hinf = np.array([[1, 0, 0], [0, 1, 0], [-1.0 / 49.0, 0, 1]], np.float32)
    with pytest.raises(ValueError, match="hit infinity"):
        psift.warp_and_stitch(q, t, Hinf)
    assert O.warp_and_stitch(q, t, Hinf) == -2
    big = _h(0, 300.0, 0, 0)
    with pytest.raises(ValueError, match="exceed safety limits"):
        psift.warp_and_stitch(q, t, big)
    assert O.warp_and_stitch(q, t, big) == -4


def test_warp_and_stitch_dev_matches_host():
    import torch
    rng = np.random.default_rng(6)
    q, t = _rgba(rng, 200, 300), _rgba(rng, 180, 260)
    H = _h(-8, 0.95, 20.0, -15.0, 5e-5, 1e-4)
    ref, _ = O.warp_and_stitch(q, t, H)
    ctx = psift.default_context()
    dq, dt = torch.from_numpy(q).cuda(), torch.from_numpy(t).cuda()
    out = torch.zeros(ref.size, dtype=torch.uint8, device="cuda")
    w, h = C.c_uint32(), C.c_uint32()
    h9 = np.ascontiguousarray(H.reshape(9))
    torch.cuda.synchronize()
    ctx.check(ctx.lib.psift_warp_and_stitch_dev(ctx.handle, C.c_void_p(dq.data_ptr()), 200, 300, 1200,
                                                C.c_void_p(dt.data_ptr()), 180, 260, 1040, h9.ctypes.data,
                                                C.c_void_p(out.data_ptr()), out.numel(), C.byref(w), C.byref(h)))
    ctx.synchronize()
    assert (h.value, w.value) == ref.shape[:2]
    np.testing.assert_array_equal(out.cpu().numpy().reshape(ref.shape), ref)
