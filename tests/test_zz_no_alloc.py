"""The allocation-free detect entry point against the regular one and the oracle.

psift_detect_and_compute_u8_noalloc_dev serves callers that cannot allocate
device memory (a plugin host that only lends a stream, a real-time loop that
cannot afford cudaMalloc's device-wide synchronisation): its scratch is a fixed
32 MiB device array inside the library.  This file is collected last so that a
failure here, in a run that stops at the first failure, comes after every other
test.  It must pass alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import psift
import synth

pytestmark = pytest.mark.gpu


def _noalloc(lib, d_img, h, w, cfg, cap, stream_ptr, expect=psift.PSIFT_OK):
    import torch
    out = {k: torch.full((cap,), -1.0, dtype=torch.float32, device="cuda") for k in ("x", "y", "s", "r", "o")}
    out["d"] = torch.full((cap, 128), -1.0, dtype=torch.float32, device="cuda")
    d_count = torch.zeros(1, dtype=torch.int32, device="cuda")
    cf = psift.CFeatures(cap, 0, out["x"].data_ptr(), out["y"].data_ptr(), out["s"].data_ptr(),
                         out["r"].data_ptr(), out["o"].data_ptr(), out["d"].data_ptr())
    c = cfg.to_c()
    st = lib.psift_detect_and_compute_u8_noalloc_dev(C.c_void_p(d_img.data_ptr()), h, w, w, C.byref(c),
                                                     C.byref(cf), C.c_void_p(d_count.data_ptr()),
                                                     C.c_void_p(stream_ptr))
    assert st == expect, st
    n = int(d_count.item())
    if expect != psift.PSIFT_OK:
        return n
    return psift.Features(out["x"][:n].cpu().numpy(), out["y"][:n].cpu().numpy(), out["s"][:n].cpu().numpy(),
                          out["r"][:n].cpu().numpy(), out["o"][:n].cpu().numpy(), out["d"][:n].cpu().numpy())


def _same(a: psift.Features, b: psift.Features):
    # Same kernels on the same input: identical results expected; the tolerance
    # is the one the parity tests use for descriptors (1e-4 relative L2).
    assert len(a) == len(b) and len(a) > 0
    np.testing.assert_array_equal(a.x, b.x)
    np.testing.assert_array_equal(a.y, b.y)
    np.testing.assert_array_equal(a.scale, b.scale)
    np.testing.assert_array_equal(a.response, b.response)
    np.testing.assert_allclose(a.orientation, b.orientation, rtol=0, atol=1e-6)
    rel = np.linalg.norm(a.descriptors - b.descriptors, axis=1) / np.linalg.norm(b.descriptors, axis=1)
    assert float(rel.max()) <= 1e-4


def test_noalloc_matches_regular_entry_point_twice():
    import torch
    lib = psift.load_library()
    cfg = psift.SiftConfig().with_octaves(4)
    stream = torch.cuda.Stream()
    imgs = [synth.blob_image(320, 240, 90, 2.0, 10.0, seed=21), synth.blob_image(300, 200, 70, 2.0, 9.0, seed=22)]
    for img in imgs:  # two calls in a row share (and must clear) the scratch array
        h, w = img.shape
        d_img = torch.from_numpy(img).cuda()
        torch.cuda.synchronize()
        got = _noalloc(lib, d_img, h, w, cfg, 4096, stream.cuda_stream)
        ref = psift.Sift.new(cfg).detect_and_compute_u8(img)
        _same(got, ref)
        _oracle_parity(got, img)


def _oracle_parity(got: psift.Features, img):
    """Independent of the GPU: the oracle's features on the same luma, at the bar of
    the detect parity tests (positions, responses identical, scale within 2 ulp,
    orientation within 1e-3 rad and descriptor relative L2 within 1e-4 for at least
    99.5 % of the features)."""
    meta, desc = O.detect_and_compute(O.luma_to_f32(img), 4, 3, 0.015, True, 0, 4096)
    assert len(got) == meta.shape[0]
    np.testing.assert_array_equal(got.x, meta[:, 0])
    np.testing.assert_array_equal(got.y, meta[:, 1])
    np.testing.assert_allclose(got.scale, meta[:, 2], rtol=2.5e-7, atol=0)
    np.testing.assert_array_equal(got.response, meta[:, 3])
    dth = np.abs(got.orientation - meta[:, 4])
    dth = np.minimum(dth, 2 * np.pi - dth)
    rel = np.linalg.norm(got.descriptors - desc, axis=1) / np.maximum(np.linalg.norm(desc, axis=1), 1e-12)
    assert ((dth <= 1e-3) & (rel <= 1e-4)).mean() >= 0.995


def test_noalloc_reports_a_short_output():
    """More features than the output holds: PSIFT_ERR_CAPACITY with the number
    needed in *d_count, as the regular entries report it."""
    import torch
    lib = psift.load_library()
    cfg = psift.SiftConfig().with_octaves(4)
    img = synth.blob_image(320, 240, 90, 2.0, 10.0, seed=21)
    full = psift.Sift.new(cfg).detect_and_compute_u8(img)
    assert len(full) > 8
    d_img = torch.from_numpy(img).cuda()
    torch.cuda.synchronize()
    needed = _noalloc(lib, d_img, 240, 320, cfg, 8, 0, expect=psift.PSIFT_ERR_CAPACITY)
    assert needed == len(full)


def test_noalloc_rejects_requests_beyond_its_scratch():
    import torch
    lib = psift.load_library()
    img = np.zeros((1080, 1920), np.uint8)
    d_img = torch.from_numpy(img).cuda()
    cap = 16
    bufs = [torch.zeros(cap, device="cuda") for _ in range(5)] + [torch.zeros((cap, 128), device="cuda")]
    cf = psift.CFeatures(cap, 0, *[b.data_ptr() for b in bufs])
    d_count = torch.zeros(1, dtype=torch.int32, device="cuda")
    c = psift.SiftConfig().to_c()
    st = lib.psift_detect_and_compute_u8_noalloc_dev(C.c_void_p(d_img.data_ptr()), 1080, 1920, 1920, C.byref(c),
                                                     C.byref(cf), C.c_void_p(d_count.data_ptr()), None)
    assert st == psift.PSIFT_ERR_CAPACITY
