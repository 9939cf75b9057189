"""JPEG input step on the GPU (psift_decode_jpeg_luma, psift_detect_and_compute_jpeg_batch).

* Decoded luma against PIL's decoder + the image crate's rgb_to_luma: the two
  decoders' IDCTs and chroma upsampling differ, so the bar is a tolerance (mean
  and maximum absolute difference in grey levels, written per case below), not
  equality.  Gray pixels go through the luma formula unchanged (checked exactly).
* The batch entry's features equal, bit for bit, the one-image u8 entry's
  features of the luma the GPU decoder returns (the decode feeds the same path).
* The reference's header checks: minimum 8x8, the enforced pixel cap, bad bytes.
"""
import numpy as np
import pytest

import jpeg_cases as J
import psift
import synth

pytestmark = pytest.mark.gpu


def _stats(a, b):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    return float(d.mean()), int(d.max())


# (label, image maker, subsampling, mean bound, max bound)
CASES = [
    ("gray 640x480 q92", lambda: J.gray_image(640, 480, 1), 2, 0.35, 3),
    ("color 4:4:4 640x480 q92", lambda: J.color_image(640, 480, 11), 0, 0.75, 4),
    ("color 4:2:0 640x480 q92", lambda: J.color_image(640, 480, 21), 2, 1.0, 24),
    ("color 4:2:0 1920x1080 q85", lambda: J.color_image(1920, 1080, 31), 2, 1.0, 24),
]


@pytest.mark.parametrize("label,make,sub,mean_tol,max_tol", CASES, ids=[c[0] for c in CASES])
def test_decoded_luma_against_cpu_decoder(label, make, sub, mean_tol, max_tol):
    img = make()
    blob = J.encode(img, 85 if "q85" in label else 92, sub)
    got = psift.decode_jpeg_luma(blob)
    ref = J.cpu_luma(blob)
    assert got.shape == ref.shape == img.shape[:2]
    mean, mx = _stats(got, ref)
    print(f"{label}: |GPU - CPU decoder| mean {mean:.3f}, max {mx}; nvJPEG backend "
          f"{psift.default_context().jpeg_backend}")
    assert mean <= mean_tol and mx <= max_tol


def test_single_call_mode_against_cpu_decoder():
    # threads = 1: one batched call (GPU-assisted backend) instead of shares on host threads
    ctx = psift.Context(0)
    try:
        ctx.set_jpeg_threads(1)
        img = J.color_image(800, 600, 41)
        blob = J.encode(img, 90, 2)
        one = psift.decode_jpeg_luma(blob, ctx=ctx)
        assert ctx.jpeg_backend in (2, 3)
        mean, mx = _stats(one, J.cpu_luma(blob))
        ctx.set_jpeg_threads(0)
        shared = psift.decode_jpeg_luma(blob, ctx=ctx)
        assert ctx.jpeg_backend == 1
        m2, x2 = _stats(one, shared)
        print(f"single call vs CPU decoder: mean {mean:.3f}, max {mx}; single call vs host-thread shares: "
              f"mean {m2:.3f}, max {x2}")
        assert mean <= 1.0 and mx <= 24
        with pytest.raises(psift.PsiftError):
            ctx.set_jpeg_threads(-1)
    finally:
        ctx.close()


def test_gray_rgb_pixels_keep_their_level():
    # a gray image stored as 4:4:4 colour: R = G = B up to the codec, luma = that level
    g = J.gray_image(320, 240, 5)
    blob = J.encode(np.stack([g, g, g], axis=2), 95, 0)
    got = psift.decode_jpeg_luma(blob)
    ref = J.cpu_luma(blob)
    assert _stats(got, ref)[0] <= 0.5
    levels = np.arange(256, dtype=np.uint8)
    np.testing.assert_array_equal(J.rgb_to_luma_u8(np.stack([levels] * 3, axis=1)), levels)


def test_batch_features_equal_single_image_path():
    imgs = [J.gray_image(640, 480, 2), J.color_image(800, 600, 3), J.color_image(333, 517, 4)]
    blobs = [J.encode(imgs[0]), J.encode(imgs[1], 90, 2), J.encode(imgs[2], 90, 0)]
    sift = psift.Sift.new(psift.SiftConfig().with_octaves(4).with_contrast_threshold(0.015))
    batch = sift.detect_and_compute_jpeg_batch(blobs)
    for blob, got in zip(blobs, batch):
        luma = psift.decode_jpeg_luma(blob)
        ref = sift.detect_and_compute_u8(luma)
        assert len(got) == len(ref) > 20
        for f in ("x", "y", "scale", "response", "orientation", "descriptors"):
            np.testing.assert_array_equal(getattr(got, f), getattr(ref, f), err_msg=f)
    # uncapped, as in the batched workload; a second call reuses the decoder state
    sift0 = psift.Sift.new(psift.SiftConfig().with_octaves(4).with_contrast_threshold(0.015).max_features(0))
    a = sift0.detect_and_compute_jpeg_batch(blobs)
    b = sift0.detect_and_compute_jpeg_batch(blobs[::-1])
    for x, y in zip(a, b[::-1]):
        np.testing.assert_array_equal(x.descriptors, y.descriptors)


def test_header_checks_and_errors():
    small = J.encode(synth.blob_image(7, 12, 2, 1.0, 2.0, 1))
    with pytest.raises(psift.PsiftError) as e:
        psift.decode_jpeg_luma(small)
    assert e.value.status == psift.PSIFT_ERR_INVALID_ARGUMENT and "are too small (minimum 8x8)" in str(e.value)
    wide = J.encode(np.full((16, 8200), 128, np.uint8))
    assert psift.jpeg_info(wide) == (8200, 16, 1)
    assert psift.decode_jpeg_luma(wide).shape == (16, 8200)
    with pytest.raises(psift.PsiftError) as e:
        psift.decode_jpeg_luma(wide, enforce_pixel_cap=True)
    assert "exceed maximum allowed (8192x8192, 25000000 px)" in str(e.value)
    with pytest.raises(psift.PsiftError) as e:
        psift.decode_jpeg_luma(b"\xff\xd8 not a jpeg at all" * 4)
    assert e.value.status == psift.PSIFT_ERR_FORMAT
    sift = psift.Sift.new(psift.SiftConfig())
    with pytest.raises(psift.PsiftError):
        sift.detect_and_compute_jpeg_batch([J.encode(J.gray_image(64, 64, 1)), small])
    # the context stays usable after the errors
    ok = sift.detect_and_compute_jpeg_batch([J.encode(J.gray_image(200, 150, 9))])
    assert len(ok) == 1


def test_large_batch_shares_and_thread_setting():
    # 60 JPEGs of 8 sizes: shares over host threads (automatic count, and 3) give,
    # per image, the features of the one-image path on the same decoded luma; one
    # batched call gives nearly the same feature counts.
    shapes = [(96, 128), (120, 160), (77, 203), (64, 64), (150, 100), (33, 250), (128, 96), (99, 101)]
    blobs = [J.encode(J.color_image(w, h, 500 + i) if i % 3 else J.gray_image(w, h, 500 + i), 90, i % 2 * 2)
             for i, (h, w) in enumerate(shapes[k % 8] for k in range(60))]
    ctx = psift.Context(0)
    try:
        sift = psift.Sift.new(psift.SiftConfig().with_octaves(3).with_contrast_threshold(0.015))
        counts = {}
        for threads in (0, 3):
            ctx.set_jpeg_threads(threads)
            got = sift.detect_and_compute_jpeg_batch(blobs, ctx=ctx)
            assert len(got) == 60 and ctx.jpeg_backend == 1
            counts[threads] = [len(f) for f in got]
            for k in (0, 7, 23, 59):
                ref = sift.detect_and_compute_u8(psift.decode_jpeg_luma(blobs[k], ctx=ctx), ctx=ctx)
                assert len(got[k]) == len(ref)
                np.testing.assert_array_equal(got[k].descriptors, ref.descriptors)
                np.testing.assert_array_equal(got[k].x, ref.x)
        assert counts[0] == counts[3]
        # one batched call (above 50 images nvJPEG decodes the Huffman stage on the GPU)
        ctx.set_jpeg_threads(1)
        one = sift.detect_and_compute_jpeg_batch(blobs, ctx=ctx)
        assert ctx.jpeg_backend in (2, 3)
        for a, b in zip(one, counts[0]):
            assert abs(len(a) - b) <= max(2, 0.1 * b)
    finally:
        ctx.close()
