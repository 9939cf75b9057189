"""Test infrastructure only: CPU restatement of the PNG input step.

decode_validated_luma8 (src/cli.rs:129-170) decodes PNGs with the image crate
0.25.10 and its png 0.18.1 decoder (neither is in the reference tree) and
converts them with DynamicImage::into_luma8.  Restated here from the PNG
specification (ISO/IEC 15948: chunks with CRC-32, one zlib stream over the
IDAT chunks, per-row filters None / Sub / Up / Average / Paeth on bytes at a
distance of one complete pixel, Adam7 interlacing) and the image crate's
published conversion rule (rgb_to_luma = (2126 R + 7152 G + 722 B) / 10000 on
the samples' own integer type; 16-bit results to u8 by (v + 128) // 257; low
bit depths expanded by v * 255 / (2^bits - 1); palettes expanded; alpha
dropped).  Pure Python per byte for the filters: small images only.
"""
import struct
import zlib

import numpy as np

SIG = b"\x89PNG\r\n\x1a\n"
ADAM7 = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]
CHANNELS = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}


class PngError(ValueError):
    pass


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    return a if pa <= pb and pa <= pc else (b if pb <= pc else c)


def _unfilter(data: bytes, pos: int, rows: int, rb: int, unit: int):
    out = []
    prior = bytearray(rb)
    for _ in range(rows):
        f = data[pos]
        if f > 4:
            raise PngError(f"invalid filter type {f}")
        cur = bytearray(data[pos + 1:pos + 1 + rb])
        for i in range(rb):
            a = cur[i - unit] if i >= unit else 0
            b = prior[i]
            c = prior[i - unit] if i >= unit else 0
            pred = (0, a, b, (a + b) >> 1, _paeth(a, b, c) if f == 4 else 0)[f]
            cur[i] = (cur[i] + pred) & 0xFF
        out.append(bytes(cur))
        prior = cur
        pos += 1 + rb
    return out, pos


def _samples(row: bytes, w: int, ch: int, depth: int) -> np.ndarray:
    if depth == 16:
        return np.frombuffer(row, ">u2")[:w * ch].astype(np.uint64).reshape(w, ch)
    if depth == 8:
        return np.frombuffer(row, np.uint8)[:w * ch].astype(np.uint64).reshape(w, ch)
    bits = np.unpackbits(np.frombuffer(row, np.uint8))
    vals = bits[:w * depth].reshape(w, depth)
    weights = 1 << np.arange(depth - 1, -1, -1)
    return (vals * weights).sum(axis=1).astype(np.uint64).reshape(w, 1)


def decode(data: bytes):
    """Returns (samples (h, w, ch) uint64, colour type, bit depth, palette (n, 3) or None)."""
    if data[:8] != SIG:
        raise PngError("not a PNG signature")
    pos, ihdr, plte, idat = 8, None, None, bytearray()
    while pos + 12 <= len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if len(body) < n:
            raise PngError("truncated chunk")
        if struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0] != zlib.crc32(tag + body) & 0xFFFFFFFF:
            raise PngError("CRC error")
        if tag == b"IHDR":
            ihdr = struct.unpack(">IIBBBBB", body)
        elif tag == b"PLTE":
            plte = np.frombuffer(body, np.uint8).reshape(-1, 3)
        elif tag == b"IDAT":
            idat += body
        elif tag == b"IEND":
            break
        elif not (tag[0] & 0x20):
            raise PngError("unknown critical chunk")
        pos += 12 + n
    w, h, depth, color, _, _, interlace = ihdr
    ch = CHANNELS[color]
    unit = max(1, depth * ch // 8)
    raw = zlib.decompress(bytes(idat))
    out = np.zeros((h, w, ch), np.uint64)
    p = 0
    for (x0, y0, dx, dy) in (ADAM7 if interlace else [(0, 0, 1, 1)]):
        pw = (w - x0 + dx - 1) // dx if w > x0 else 0
        ph = (h - y0 + dy - 1) // dy if h > y0 else 0
        if pw == 0 or ph == 0:
            continue
        rb = (pw * depth * ch + 7) // 8
        rows, p = _unfilter(raw, p, ph, rb, unit)
        for r, row in enumerate(rows):
            out[y0 + r * dy, x0::dx][:pw] = _samples(row, pw, ch, depth)
    return out, color, depth, plte


def luma(data: bytes) -> np.ndarray:
    """decode_validated_luma8 of a PNG: the u8 luma plane."""
    s, color, depth, plte = decode(data)
    if color == 3:
        pal = np.zeros((256, 3), np.uint64)
        pal[:len(plte)] = plte
        c = pal[s[:, :, 0]]
        return ((2126 * c[:, :, 0] + 7152 * c[:, :, 1] + 722 * c[:, :, 2]) // 10000).astype(np.uint8)
    if color in (0, 4):
        v = s[:, :, 0]
    else:
        v = (2126 * s[:, :, 0] + 7152 * s[:, :, 1] + 722 * s[:, :, 2]) // 10000
    if depth == 16:
        return ((v + 128) // 257).astype(np.uint8)
    if depth < 8:
        return (v * (255 // ((1 << depth) - 1))).astype(np.uint8)
    return v.astype(np.uint8)
