"""psift_detect_and_compute_u8_batch: many host images per call, two chunks on
two streams.  Per image the features must equal the single-image entry's
exactly (same kernels, same order of operations)."""
import numpy as np
import pytest

import psift
import synth

pytestmark = pytest.mark.gpu


def _same(a: psift.Features, b: psift.Features):
    assert len(a) == len(b)
    for f in ("x", "y", "scale", "response", "orientation", "descriptors"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f)


def _images(shapes, seed=0):
    return [synth.blob_image(w, h, max(20, h * w // 2000), 1.5, 12.0, seed=seed + i) for i, (h, w) in enumerate(shapes)]


@pytest.mark.parametrize("n", [1, 2, 3, 6])
def test_batch_equals_single_image_calls(n):
    shapes = [(240 + 37 * i, 320 + 53 * (i % 3)) for i in range(n)]
    imgs = _images(shapes, seed=10 * n)
    sift = psift.Sift.new(psift.SiftConfig().with_octaves(4))
    got = sift.detect_and_compute_batch_u8(imgs)
    for im, g in zip(imgs, got):
        _same(g, sift.detect_and_compute_u8(im))


def test_batch_pinned_inputs_and_outputs_strided():
    shapes = [(300, 401), (257, 333), (480, 640), (100, 90)]
    imgs = _images(shapes, seed=5)
    sift = psift.Sift.new(psift.SiftConfig())
    pinned_in = []
    for k, im in enumerate(imgs):
        if k % 2 == 0:  # pinned, with a row stride wider than the image
            buf = psift.pinned_empty((im.shape[0], im.shape[1] + 24), np.uint8)
            buf[:, : im.shape[1]] = im
            pinned_in.append(buf[:, : im.shape[1]])
        else:
            pinned_in.append(im)
    outs = [psift.Features.pinned(4096) if k % 2 else psift.Features.empty(4096) for k in range(len(imgs))]
    got = sift.detect_and_compute_batch_u8(pinned_in, outs=outs)
    for im, g in zip(imgs, got):
        _same(g, sift.detect_and_compute_u8(im))


def test_batch_with_empty_and_tiny_images():
    imgs = [np.zeros((0, 0), np.uint8), synth.blob_image(200, 150, 40, 2.0, 8.0, seed=3), np.zeros((2, 2), np.uint8)]
    sift = psift.Sift.new(psift.SiftConfig())
    got = sift.detect_and_compute_batch_u8(imgs)
    assert len(got[0]) == 0 and len(got[2]) == 0
    _same(got[1], sift.detect_and_compute_u8(imgs[1]))


def test_batch_uncapped_grows_short_outputs():
    imgs = _images([(320, 480), (330, 470)], seed=77)
    sift = psift.Sift.new(psift.SiftConfig().max_features(0))
    outs = [psift.Features.empty(8), psift.Features.empty(8)]
    got = sift.detect_and_compute_batch_u8(imgs, outs=outs)
    for im, g in zip(imgs, got):
        assert len(g) > 8
        _same(g, sift.detect_and_compute_u8(im))
