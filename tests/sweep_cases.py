"""The reference's invariance sweeps (tests/invariance_sweeps.rs) over its own
sample image, for any detect / match / similarity-RANSAC implementation.

Inputs: tests/golden/aerial_west_luma.npz (the luma of docs/samples/aerial_west.jpg,
made by tests/golden/make_aerial_luma.py).  The rotation sweep's warp is the
test's own `rotate_bilinear` (:35-72), restated in f32 with glibc's cosf/sinf.
The scale sweep resizes with the image crate's (0.25.10) `imageops::resize` and
FilterType::CatmullRom, restated here from its published scheme: separable,
vertical pass to f32 then horizontal pass rounded to u8; output pixel centre
(o + 0.5) * ratio, support 2 widened by the downscale ratio, Mitchell-Netravali
cubic with B = 0, C = 0.5, weights normalised by their sequential sum.  That
restatement is not pinned to the crate bit for bit; the sweep's assertions
(minimum inlier counts, 2 deg rotation and 3 % scale error) do not depend on it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# tests/invariance_sweeps.rs:14-31 (scale or angle, minimum similarity inliers)
SCALE_SWEEP_BASELINES = [(0.25, 150), (0.35, 340), (0.50, 750), (0.70, 1400), (1.40, 900), (2.00, 800)]
ROTATION_SWEEP_BASELINES = [(0.0, 3000), (15.0, 1900), (30.0, 1500), (45.0, 1500), (90.0, 2500), (180.0, 2500)]
SWEEP_OCTAVES, SWEEP_SCALES = 4, 3

_libm = ctypes.CDLL("libm.so.6")
for _fn in ("cosf", "sinf"):
    getattr(_libm, _fn).restype = ctypes.c_float
    getattr(_libm, _fn).argtypes = [ctypes.c_float]

F = np.float32


def aerial_west_luma() -> np.ndarray:
    return np.load(os.path.join(HERE, "golden", "aerial_west_luma.npz"))["luma"]


def _round_half_away(v: np.ndarray) -> np.ndarray:
    """Rust `f32::round` for v >= 0: exact, halves away from zero."""
    fl = np.floor(v)
    return np.where(v - fl >= F(0.5), fl + F(1), fl).astype(F)


def rotate_bilinear(src: np.ndarray, angle_deg: float) -> np.ndarray:
    """tests/invariance_sweeps.rs:35-72: counter-clockwise rotation about the centre,
    bilinear, pixels that map outside the source stay 0."""
    h, w = src.shape
    cx = F(0.5) * (F(w) - F(1.0))
    cy = F(0.5) * (F(h) - F(1.0))
    rad = F(angle_deg) * (F(np.pi) / F(180.0))  # f32::to_radians
    cos_a, sin_a = F(_libm.cosf(rad)), F(_libm.sinf(rad))
    dy = (np.arange(h, dtype=F) - cy)[:, None]
    dx = (np.arange(w, dtype=F) - cx)[None, :]
    sx = (cx + dx * cos_a) + dy * sin_a
    sy = (cy - dx * sin_a) + dy * cos_a
    ok = (sx >= 0) & (sx <= F(w - 1)) & (sy >= 0) & (sy <= F(h - 1))
    sxc = np.where(ok, sx, F(0))
    syc = np.where(ok, sy, F(0))
    x0 = np.floor(sxc).astype(np.int64)
    y0 = np.floor(syc).astype(np.int64)
    x1 = np.minimum(x0 + 1, w - 1)
    y1 = np.minimum(y0 + 1, h - 1)
    fx = sxc - x0.astype(F)
    fy = syc - y0.astype(F)
    s = src.astype(F)
    p00, p10, p01, p11 = s[y0, x0], s[y0, x1], s[y1, x0], s[y1, x1]
    one = F(1.0)
    val = (one - fy) * ((one - fx) * p00 + fx * p10) + fy * ((one - fx) * p01 + fx * p11)
    out = np.clip(_round_half_away(val), 0, 255).astype(np.uint8)
    return np.where(ok, out, np.uint8(0))


def _catmull_rom(x: F) -> F:
    a = abs(F(x))
    b, c = F(0.0), F(0.5)
    if a < 1:
        k = (F(12) - F(9) * b - F(6) * c) * (a * a * a) + (F(-18) + F(12) * b + F(6) * c) * (a * a) + (F(6) - F(2) * b)
    elif a < 2:
        k = ((-b - F(6) * c) * (a * a * a) + (F(6) * b + F(30) * c) * (a * a) + (F(-12) * b - F(48) * c) * a
             + (F(8) * b + F(24) * c))
    else:
        k = F(0)
    return F(k / F(6))


def _weights(n_in: int, n_out: int):
    ratio = F(n_in) / F(n_out)
    sratio = F(1) if ratio < 1 else ratio
    support = F(2.0) * sratio
    rows = []
    for o in range(n_out):
        centre = (F(o) + F(0.5)) * ratio
        left = int(np.clip(np.floor(centre - support), 0, n_in - 1))
        right = int(np.clip(np.ceil(centre + support), left + 1, n_in))
        centre = centre - F(0.5)
        ws = [_catmull_rom((F(i) - centre) / sratio) for i in range(left, right)]
        total = F(0)
        for wv in ws:
            total = F(total + wv)
        rows.append((left, [F(wv / total) for wv in ws]))
    return rows


def resize_catmull_rom(src: np.ndarray, new_w: int, new_h: int) -> np.ndarray:
    h, w = src.shape
    if (new_w, new_h) == (w, h):
        return src.copy()
    s = src.astype(F)
    tmp = np.zeros((new_h, w), F)
    for o, (left, ws) in enumerate(_weights(h, new_h)):
        acc = np.zeros(w, F)
        for i, wv in enumerate(ws):
            acc = acc + s[left + i] * wv
        tmp[o] = acc
    out = np.zeros((new_h, new_w), np.uint8)
    for o, (left, ws) in enumerate(_weights(w, new_w)):
        acc = np.zeros(new_h, F)
        for i, wv in enumerate(ws):
            acc = acc + tmp[:, left + i] * wv
        out[:, o] = _round_half_away(np.clip(acc, F(0), F(255))).astype(np.uint8)
    return out


def angular_diff_deg(a: float, b: float) -> float:
    d = (a - b) % 360.0
    if d > 180.0:
        d -= 360.0
    return abs(d)


def run_sweeps(extract, match, similarity, which=("scale", "rotation")):
    """extract(u8 luma) -> features; match(base, target) -> matches (ratio 0.75);
    similarity(matches) -> (n_inliers, (a, b, tx, ty, scale, rotation_deg) or None).
    Returns the list of (label, inliers, minimum, scale, rotation) and asserts the
    reference's conditions."""
    base = aerial_west_luma()
    h, w = base.shape
    fb = extract(base)
    assert len(fb) > 0
    rows = []
    if "scale" in which:
        for s, need in SCALE_SWEEP_BASELINES:
            nw, nh = int(_round_half_away(np.array(F(w) * F(s)))), int(_round_half_away(np.array(F(h) * F(s))))
            ft = extract(resize_catmull_rom(base, nw, nh))
            n_in, sim = similarity(match(fb, ft))
            assert sim is not None, f"scale {s}: no similarity"
            rows.append((f"scale {s:.2f} ({nw}x{nh})", n_in, need, float(sim[4]), float(sim[5])))
            assert n_in >= need, rows[-1]
            assert abs(float(sim[4]) - s) / s <= 0.03, rows[-1]
            assert angular_diff_deg(float(sim[5]), 0.0) <= 2.0, rows[-1]
    if "rotation" in which:
        for ang, need in ROTATION_SWEEP_BASELINES:
            ft = extract(rotate_bilinear(base, ang))
            n_in, sim = similarity(match(fb, ft))
            assert sim is not None, f"rotation {ang}: no similarity"
            rows.append((f"rotation {ang:.0f} deg", n_in, need, float(sim[4]), float(sim[5])))
            assert n_in >= need, rows[-1]
            assert angular_diff_deg(float(sim[5]) % 360.0, ang % 360.0) <= 2.0, rows[-1]
            assert abs(float(sim[4]) - 1.0) <= 0.03, rows[-1]
    return rows
