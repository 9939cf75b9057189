"""PNG input step on the GPU (psift_decode_png_luma, psift_detect_and_compute_png_batch,
psift_detect_and_compute_image_batch).

PNG is lossless, so the bar is equality: the GPU's luma equals the image crate's
conversion of the file's samples (tests/png_cases.py) for every colour type and
bit depth, plain and Adam7-interlaced, with every row filter, and equals PIL's
decode + the conversion rule on files PIL wrote (its own filter choices, 1080p).
The batch entries' features equal the one-image u8 entry's on that luma, bit
for bit, and the reference's header checks and messages hold.
"""
import io
import struct
import zlib

import numpy as np
import pytest
from PIL import Image

import jpeg_cases as J
import png_cases as PC
import psift
import synth

pytestmark = pytest.mark.gpu

COMBOS = [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (2, 8), (2, 16), (3, 1), (3, 2), (3, 4), (3, 8),
          (4, 8), (4, 16), (6, 8), (6, 16)]


def _palette(depth, seed):
    return np.random.default_rng(seed).integers(0, 256, ((1 << depth), 3))


@pytest.mark.parametrize("color,depth", COMBOS)
@pytest.mark.parametrize("interlace", [False, True])
def test_luma_equals_conversion_of_samples(color, depth, interlace):
    # 70 rows: three 32-row groups of the wavefront, the last one partial
    h, w = (70, 53) if interlace else (70, 45)
    s = PC.random_samples(h, w, color, depth, seed=10 * color + depth + (1000 if interlace else 0))
    pal = _palette(depth, color + 3 * depth) if color == 3 else None
    blob = PC.encode_png(s, color, depth, interlace=interlace, palette=pal)
    assert psift.png_info(blob)[:2] == (w, h)
    np.testing.assert_array_equal(psift.decode_png_luma(blob), PC.expected_luma(s, color, depth, pal))


@pytest.mark.parametrize("filters", [(0,), (1,), (2,), (3,), (4,), (4, 3, 1, 2, 0)])
def test_each_filter_on_a_wide_rgb16_image(filters):
    s = PC.random_samples(97, 301, 2, 16, seed=sum(filters) + 11 * len(filters))
    blob = PC.encode_png(s, 2, 16, filters=filters)
    np.testing.assert_array_equal(psift.decode_png_luma(blob), PC.expected_luma(s, 2, 16))


@pytest.mark.parametrize("mode", ["L", "RGB", "RGBA"])
def test_1080p_pil_written_files(mode):
    rgb = np.stack([synth.blob_image(1920, 1080, 800, 1.5, 20.0, seed=50 + k) for k in range(3)], axis=2)
    im = Image.fromarray(rgb, "RGB")
    if mode != "RGB":
        im = im.convert(mode)
    buf = io.BytesIO()
    im.save(buf, format="PNG")
    blob = buf.getvalue()
    dec = np.asarray(Image.open(io.BytesIO(blob)).convert("RGB")).astype(np.uint64)
    want = PC.rgb_to_luma(dec[:, :, 0], dec[:, :, 1], dec[:, :, 2]).astype(np.uint8)
    np.testing.assert_array_equal(psift.decode_png_luma(blob), want)


def test_batch_features_equal_single_image_path():
    cases = [(PC.random_samples(480, 640, 2, 8, seed=1), 2, 8, False), (PC.random_samples(300, 411, 0, 16, seed=2), 0, 16, True),
             (synth.blob_image(800, 600, 300, 2.0, 12.0, seed=3), 0, 8, False)]
    blobs = [PC.encode_png(s, c, d, interlace=il, filters=(4, 1, 2, 3, 0)) for s, c, d, il in cases]
    sift = psift.Sift.new(psift.SiftConfig().with_octaves(4).with_contrast_threshold(0.015))
    batch = sift.detect_and_compute_png_batch(blobs)
    for blob, got in zip(blobs, batch):
        ref = sift.detect_and_compute_u8(psift.decode_png_luma(blob))
        assert len(got) == len(ref) > 10
        for f in ("x", "y", "scale", "response", "orientation", "descriptors"):
            np.testing.assert_array_equal(getattr(got, f), getattr(ref, f), err_msg=f)


def test_mixed_batch_keeps_order():
    png = PC.encode_png(synth.blob_image(640, 480, 300, 2.0, 12.0, seed=4), 0, 8)
    jpg = J.encode(J.color_image(640, 480, 5), 90, 2)
    png2 = PC.encode_png(PC.random_samples(200, 333, 6, 8, seed=6), 6, 8)
    sift = psift.Sift.new(psift.SiftConfig().with_octaves(4).with_contrast_threshold(0.015))
    mixed = sift.detect_and_compute_image_batch([png, jpg, png2])
    sep_png = sift.detect_and_compute_png_batch([png, png2])
    sep_jpg = sift.detect_and_compute_jpeg_batch([jpg])
    for got, want in zip(mixed, [sep_png[0], sep_jpg[0], sep_png[1]]):
        np.testing.assert_array_equal(got.descriptors, want.descriptors)
    np.testing.assert_array_equal(psift.decode_image_luma(png), psift.decode_png_luma(png))


def _rechunk(blob, tag, new_body=None, bad_crc=False):
    """Rewrites the first chunk `tag` of a PNG (new body and CRC, or a broken CRC)."""
    pos = 8
    while pos < len(blob):
        n = struct.unpack(">I", blob[pos:pos + 4])[0]
        if blob[pos + 4:pos + 8] == tag:
            body = blob[pos + 8:pos + 8 + n] if new_body is None else new_body
            crc = zlib.crc32(tag + body) & 0xFFFFFFFF
            if bad_crc:
                crc ^= 1
            return blob[:pos] + struct.pack(">I", len(body)) + tag + body + struct.pack(">I", crc) + blob[pos + 12 + n:]
        pos += 12 + n
    raise AssertionError(tag)


def test_header_checks_and_errors():
    s = PC.random_samples(40, 40, 0, 8, seed=9)
    good = PC.encode_png(s, 0, 8)
    with pytest.raises(psift.PsiftError, match="Invalid or unsupported image header"):
        psift.png_info(b"\x89PNG\r\n\x1a\x0a" + b"\x00" * 4)
    with pytest.raises(psift.PsiftError, match="too small"):
        psift.decode_png_luma(PC.encode_png(PC.random_samples(7, 20, 0, 8, seed=1), 0, 8))
    big = _rechunk(good, b"IHDR", struct.pack(">IIBBBBB", 9000, 40, 8, 0, 0, 0, 0))
    with pytest.raises(psift.PsiftError, match="exceed maximum allowed"):
        psift.png_info(big, enforce_pixel_cap=True)
    with pytest.raises(psift.PsiftError, match="CRC"):
        psift.decode_png_luma(_rechunk(good, b"IDAT", bad_crc=True))
    i = good.index(b"tEXt")
    n = struct.unpack(">I", good[i - 4:i])[0]
    body = good[i + 4:i + 4 + n]
    crit = good[:i] + b"XtXt" + body + struct.pack(">I", zlib.crc32(b"XtXt" + body) & 0xFFFFFFFF) + good[i + 8 + n:]
    with pytest.raises(psift.PsiftError, match="critical chunk"):
        psift.decode_png_luma(crit)
    raw = bytearray(zlib.decompress(good[good.index(b"IDAT") + 4:good.index(b"IDAT") + 4 +
                                         struct.unpack(">I", good[good.index(b"IDAT") - 4:good.index(b"IDAT")])[0]]))
    raw[0] = 7  # an unknown filter type
    with pytest.raises(psift.PsiftError, match="filter type"):
        psift.decode_png_luma(_rechunk(good, b"IDAT", zlib.compress(bytes(raw))))
    with pytest.raises(psift.PsiftError, match="truncated"):
        psift.decode_png_luma(_rechunk(good, b"IDAT", zlib.compress(bytes(raw[:100]))))
    # the context stays usable
    np.testing.assert_array_equal(psift.decode_png_luma(good), PC.expected_luma(s, 0, 8))
