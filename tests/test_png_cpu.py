"""The PNG restatement (oracle/png_oracle.py) pinned on the CPU.

* The test writer (tests/png_cases.py) is checked by PIL reading its files back
  equal to the samples (8-bit modes, 16-bit gray).
* The restatement's luma equals the image crate's conversion of the samples for
  every colour type and bit depth, plain and Adam7-interlaced, with every filter.
* On files written by PIL (its own filter choices) the restatement equals PIL's
  decode followed by the conversion rule.
"""
import io

import numpy as np
import pytest
from PIL import Image

import png_cases as PC
import png_oracle as PO

COMBOS = [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (2, 8), (2, 16), (3, 1), (3, 2), (3, 4), (3, 8),
          (4, 8), (4, 16), (6, 8), (6, 16)]


def _palette(depth, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, 256, ((1 << depth), 3))


@pytest.mark.parametrize("color,depth", COMBOS)
@pytest.mark.parametrize("interlace", [False, True])
def test_restatement_equals_conversion_rule(color, depth, interlace):
    h, w = (37, 23) if interlace else (19, 41)
    s = PC.random_samples(h, w, color, depth, seed=100 * color + depth)
    pal = _palette(depth, color + depth) if color == 3 else None
    blob = PC.encode_png(s, color, depth, interlace=interlace, palette=pal)
    np.testing.assert_array_equal(PO.luma(blob), PC.expected_luma(s, color, depth, pal))


@pytest.mark.parametrize("mode,color,depth", [("L", 0, 8), ("RGB", 2, 8), ("RGBA", 6, 8), ("LA", 4, 8),
                                              ("I;16", 0, 16), ("P", 3, 8), ("1", 0, 1)])
def test_writer_read_back_by_pil(mode, color, depth):
    s = PC.random_samples(21, 30, color, depth, seed=7)
    pal = _palette(depth, 3) if color == 3 else None
    for interlace in (False, True):
        im = Image.open(io.BytesIO(PC.encode_png(s, color, depth, interlace=interlace, palette=pal)))
        assert im.mode == mode
        got = np.asarray(im).astype(np.int64)
        want = s.astype(np.int64)
        if mode == "1":
            want = want.astype(bool)
            got = got.astype(bool)
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("mode", ["L", "RGB", "RGBA", "P"])
def test_restatement_on_pil_written_files(mode):
    rng = np.random.default_rng(5)
    base = rng.integers(0, 256, (29, 47, 3), dtype=np.uint8)
    im = Image.fromarray(base, "RGB")
    if mode == "L":
        im = im.convert("L")
    elif mode == "RGBA":
        im = im.convert("RGBA")
    elif mode == "P":
        im = im.quantize(64)
    buf = io.BytesIO()
    im.save(buf, format="PNG", optimize=False)
    blob = buf.getvalue()
    dec = Image.open(io.BytesIO(blob))
    rgb = np.asarray(dec.convert("RGB")).astype(np.uint64)
    want = PC.rgb_to_luma(rgb[:, :, 0], rgb[:, :, 1], rgb[:, :, 2]).astype(np.uint8)
    np.testing.assert_array_equal(PO.luma(blob), want)


def test_crc_and_filter_errors():
    s = PC.random_samples(9, 9, 0, 8, seed=1)
    blob = bytearray(PC.encode_png(s, 0, 8))
    bad = bytearray(blob)
    bad[-20] ^= 0xFF  # inside the last IDAT body or its CRC
    with pytest.raises(PO.PngError):
        PO.luma(bytes(bad))
    with pytest.raises(PO.PngError):
        PO.luma(b"not a png at all")
