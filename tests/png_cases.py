"""PNG inputs for the decode step (decode_validated_luma8, src/cli.rs:164-170).

`encode_png` writes PNG files from sample arrays with a chosen colour type, bit
depth, per-row filter types and optional Adam7 interlacing (ISO/IEC 15948), so
that every filter and layout the decoder must handle is exercised; PIL reading
these files back equal to the samples checks the writer.  `expected_luma` is
the image crate's DynamicImage::into_luma8 of the samples (image 0.25.10, not in
the tree), as published: rgb_to_luma = (2126 R + 7152 G + 722 B) / 10000 in u32
on the samples' own type, 16-bit results to u8 as (v + 128) // 257, low bit
depths expanded by v * 255 / (2^bits - 1), palettes to their colours, alpha
dropped.
"""
import struct
import zlib

import numpy as np

ADAM7 = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]
CHANNELS = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}


def _chunk(tag: bytes, body: bytes) -> bytes:
    return struct.pack(">I", len(body)) + tag + body + struct.pack(">I", zlib.crc32(tag + body) & 0xFFFFFFFF)


def _pack_row(samples: np.ndarray, depth: int) -> bytes:
    """One row of samples (w x channels, integers) as PNG bytes."""
    flat = samples.reshape(-1).astype(np.uint32)
    if depth == 16:
        return flat.astype(">u2").tobytes()
    if depth == 8:
        return flat.astype(np.uint8).tobytes()
    per = 8 // depth
    out = bytearray((len(flat) + per - 1) // per)
    for i, v in enumerate(flat):
        out[i // per] |= int(v) << (8 - depth - depth * (i % per))
    return bytes(out)


def _paeth(a: int, b: int, c: int) -> int:
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    return a if pa <= pb and pa <= pc else (b if pb <= pc else c)


def _filter_rows(rows, unit: int, filters):
    """Forward filters (type filters[r % len]) of a list of unfiltered byte rows."""
    out = bytearray()
    prior = bytes(len(rows[0])) if rows else b""
    for r, raw in enumerate(rows):
        f = filters[r % len(filters)]
        out.append(f)
        for i, x in enumerate(raw):
            a = raw[i - unit] if i >= unit else 0
            b = prior[i]
            c = prior[i - unit] if i >= unit else 0
            pred = [0, a, b, (a + b) >> 1, _paeth(a, b, c)][f]
            out.append((x - pred) & 0xFF)
        prior = raw
    return out


def encode_png(samples: np.ndarray, color: int, depth: int, filters=(0, 1, 2, 3, 4), interlace: bool = False,
               palette: np.ndarray | None = None, level: int = 6) -> bytes:
    """samples: (h, w) or (h, w, channels) integers within the bit depth."""
    s = samples if samples.ndim == 3 else samples[:, :, None]
    h, w, ch = s.shape
    assert ch == CHANNELS[color]
    unit = max(1, depth * ch // 8)
    stream = bytearray()
    passes = ADAM7 if interlace else [(0, 0, 1, 1)]
    for (x0, y0, dx, dy) in passes:
        sub = s[y0::dy, x0::dx]
        if sub.shape[0] == 0 or sub.shape[1] == 0:
            continue
        rows = [_pack_row(sub[r], depth) for r in range(sub.shape[0])]
        stream += _filter_rows(rows, unit, filters)
    out = b"\x89PNG\r\n\x1a\n"
    out += _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, color, 0, 0, 1 if interlace else 0))
    if palette is not None:
        out += _chunk(b"PLTE", np.asarray(palette, np.uint8).reshape(-1).tobytes())
    out += _chunk(b"tEXt", b"Comment\x00psift test image")  # an ancillary chunk to skip
    comp = zlib.compress(bytes(stream), level)
    # image data split over several IDAT chunks
    for k in range(0, len(comp), 4096):
        out += _chunk(b"IDAT", comp[k:k + 4096])
    out += _chunk(b"IEND", b"")
    return out


def rgb_to_luma(r, g, b):
    return (2126 * r.astype(np.uint64) + 7152 * g.astype(np.uint64) + 722 * b.astype(np.uint64)) // 10000


def expected_luma(samples: np.ndarray, color: int, depth: int, palette: np.ndarray | None = None) -> np.ndarray:
    s = samples if samples.ndim == 3 else samples[:, :, None]
    s = s.astype(np.uint64)
    if color == 3:
        pal = np.zeros((256, 3), np.uint64)
        pal[:len(palette)] = np.asarray(palette, np.uint64)
        c = pal[s[:, :, 0]]
        return rgb_to_luma(c[:, :, 0], c[:, :, 1], c[:, :, 2]).astype(np.uint8)
    if color in (0, 4):
        v = s[:, :, 0]
    else:
        v = rgb_to_luma(s[:, :, 0], s[:, :, 1], s[:, :, 2])
    if depth == 16:
        return ((v + 128) // 257).astype(np.uint8)
    if depth < 8:
        return (v * (255 // ((1 << depth) - 1))).astype(np.uint8)
    return v.astype(np.uint8)


def random_samples(h: int, w: int, color: int, depth: int, seed: int) -> np.ndarray:
    """Smooth fields plus noise (so every filter type sees real predictions)."""
    rng = np.random.default_rng(seed)
    ch = CHANNELS[color]
    top = (1 << depth) - 1  # palette images: indices into a palette of 2^depth entries
    yy, xx = np.mgrid[0:h, 0:w]
    out = np.empty((h, w, ch), np.int64)
    for c in range(ch):
        f = (np.sin(xx / (7.0 + 3 * c)) + np.cos(yy / (5.0 + 2 * c)) + 2.0) / 4.0
        out[:, :, c] = np.clip(f * top + rng.normal(0, top * 0.05, (h, w)), 0, top).astype(np.int64)
    return out if ch > 1 else out[:, :, 0]
