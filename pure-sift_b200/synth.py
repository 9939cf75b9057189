"""Seeded synthetic workloads for the feature hot path (blob images, warps,
descriptor catalogs, putative correspondences).

No public dataset is used.  Every generator draws from one splitmix64 stream
(the reference's RNG, src/pipeline.rs:1862-1868) so inputs are reproducible.

Workloads:
  * blob image: mid-grey 128 background, Gaussian blobs (sigma ~ U(lo, hi),
    amplitude +/-U(40, 120), centres uniform), N(0, 3) noise (Box-Muller),
    rounded and clamped to u8.  Blobs are truncated at 4 sigma.
  * warped pair: image B = A warped bilinearly by a homography composed about
    the image centre; pixels mapping outside A are filled with 128 (the
    reference's own rotate helper fills 0, tests/invariance_sweeps.rs:35-73).
  * SIFT-like catalog descriptors: |N(0,1)| per element, L2-normalised, clipped
    at 0.2, renormalised; queries are copies of catalog descriptors with
    additive |N(0, 0.02)| noise, renormalised the same way.
"""
from __future__ import annotations

import math

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


class SplitMix64:
    """Vectorised splitmix64 stream (same sequence as calling next() repeatedly)."""

    def __init__(self, seed: int):
        self.state = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)

    def next_u64(self, n: int) -> np.ndarray:
        with np.errstate(over="ignore"):
            steps = (np.arange(1, n + 1, dtype=np.uint64) * GOLDEN)
            s = self.state + steps
            self.state = self.state + np.uint64(n) * GOLDEN
            z = s
            z = (z ^ (z >> np.uint64(30))) * _M1
            z = (z ^ (z >> np.uint64(27))) * _M2
            return z ^ (z >> np.uint64(31))

    def uniform(self, n: int) -> np.ndarray:
        """Uniform doubles in [0, 1) from the top 53 bits."""
        return (self.next_u64(n) >> np.uint64(11)).astype(np.float64) * (1.0 / float(1 << 53))

    def uniform_open(self, n: int) -> np.ndarray:
        """Uniform doubles in (0, 1]."""
        return ((self.next_u64(n) >> np.uint64(11)).astype(np.float64) + 1.0) * (1.0 / float(1 << 53))

    def normal(self, n: int) -> np.ndarray:
        m = (n + 1) // 2
        u1 = self.uniform_open(m)
        u2 = self.uniform(m)
        r = np.sqrt(-2.0 * np.log(u1))
        z = np.empty(2 * m)
        z[0::2] = r * np.cos(2.0 * np.pi * u2)
        z[1::2] = r * np.sin(2.0 * np.pi * u2)
        return z[:n]


def blob_image(width: int, height: int, n_blobs: int, sigma_lo: float, sigma_hi: float, seed: int,
               noise_sigma: float = 3.0) -> np.ndarray:
    """u8 luma image (height, width): 128 background + Gaussian blobs + noise."""
    rng = SplitMix64(seed)
    img = np.full((height, width), 128.0, np.float64)
    params = rng.uniform(5 * n_blobs).reshape(n_blobs, 5)
    for cx_u, cy_u, s_u, a_u, sign_u in params:
        cx, cy = cx_u * width, cy_u * height
        sigma = sigma_lo + (sigma_hi - sigma_lo) * s_u
        amp = (40.0 + 80.0 * a_u) * (1.0 if sign_u < 0.5 else -1.0)
        r = 4.0 * sigma
        x0, x1 = max(int(math.floor(cx - r)), 0), min(int(math.ceil(cx + r)) + 1, width)
        y0, y1 = max(int(math.floor(cy - r)), 0), min(int(math.ceil(cy + r)) + 1, height)
        if x0 >= x1 or y0 >= y1:
            continue
        xs = np.arange(x0, x1, dtype=np.float64) - cx
        ys = np.arange(y0, y1, dtype=np.float64) - cy
        inv = -1.0 / (2.0 * sigma * sigma)
        g = np.exp(ys[:, None] ** 2 * inv) * np.exp(xs[None, :] ** 2 * inv)
        img[y0:y1, x0:x1] += amp * g
    if noise_sigma > 0:
        img += noise_sigma * rng.normal(width * height).reshape(height, width)
    return np.clip(np.rint(img), 0, 255).astype(np.uint8)


def similarity_h(width: int, height: int, rot_deg: float, scale: float, tx: float, ty: float) -> np.ndarray:
    """Homography p' = s R (p - c) + c + t, c = image centre."""
    cx, cy = (width - 1) / 2.0, (height - 1) / 2.0
    th = math.radians(rot_deg)
    c, s = math.cos(th) * scale, math.sin(th) * scale
    T1 = np.array([[1, 0, -cx], [0, 1, -cy], [0, 0, 1]], np.float64)
    A = np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]], np.float64)
    T2 = np.array([[1, 0, cx + tx], [0, 1, cy + ty], [0, 0, 1]], np.float64)
    return T2 @ A @ T1


def perspective_h(width: int, height: int, rot_deg: float, scale: float, h31: float, h32: float) -> np.ndarray:
    """Homography T(c) P S R T(-c), P = [[1,0,0],[0,1,0],[h31,h32,1]] applied to centred coordinates."""
    cx, cy = (width - 1) / 2.0, (height - 1) / 2.0
    th = math.radians(rot_deg)
    c, s = math.cos(th) * scale, math.sin(th) * scale
    T1 = np.array([[1, 0, -cx], [0, 1, -cy], [0, 0, 1]], np.float64)
    A = np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]], np.float64)
    P = np.array([[1, 0, 0], [0, 1, 0], [h31, h32, 1]], np.float64)
    T2 = np.array([[1, 0, cx], [0, 1, cy], [0, 0, 1]], np.float64)
    return T2 @ P @ A @ T1


def warp_image(src: np.ndarray, H: np.ndarray, fill: float = 128.0) -> np.ndarray:
    """B(p') = A(H^-1 p'), bilinear, out-of-bounds = fill; returns u8."""
    h, w = src.shape
    Hi = np.linalg.inv(H)
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float64)
    den = Hi[2, 0] * xs + Hi[2, 1] * ys + Hi[2, 2]
    sx = (Hi[0, 0] * xs + Hi[0, 1] * ys + Hi[0, 2]) / den
    sy = (Hi[1, 0] * xs + Hi[1, 1] * ys + Hi[1, 2]) / den
    x0 = np.floor(sx)
    y0 = np.floor(sy)
    fx, fy = sx - x0, sy - y0
    x0 = x0.astype(np.int64)
    y0 = y0.astype(np.int64)
    inside = (x0 >= 0) & (y0 >= 0) & (x0 + 1 < w) & (y0 + 1 < h)
    x0c, y0c = np.clip(x0, 0, w - 2), np.clip(y0, 0, h - 2)
    a = src.astype(np.float64)
    v = (a[y0c, x0c] * (1 - fx) * (1 - fy) + a[y0c, x0c + 1] * fx * (1 - fy) +
         a[y0c + 1, x0c] * (1 - fx) * fy + a[y0c + 1, x0c + 1] * fx * fy)
    out = np.where(inside, v, fill)
    return np.clip(np.rint(out), 0, 255).astype(np.uint8)


def pair_640x480(seed: int = 1):
    """640x480 pair: 300 blobs sigma~U(2,12); B = rot 15 deg, scale 1.2, t (20,-15)."""
    a = blob_image(640, 480, 300, 2.0, 12.0, seed)
    H = similarity_h(640, 480, 15.0, 1.2, 20.0, -15.0)
    return a, warp_image(a, H), H


def pair_1080p(seed: int = 2):
    """1920x1080 pair: 2000 blobs sigma~U(1.5,20); B = perspective warp (h31,h32 ~ U(+-2e-4),
    rot U(+-30 deg), scale U(0.7,1.4)) about the centre."""
    a = blob_image(1920, 1080, 2000, 1.5, 20.0, seed)
    u = SplitMix64(seed ^ 0xABCDEF).uniform(4)
    H = perspective_h(1920, 1080, -30 + 60 * u[0], 0.7 + 0.7 * u[1], -2e-4 + 4e-4 * u[2], -2e-4 + 4e-4 * u[3])
    return a, warp_image(a, H), H


def uneven_batch_shapes(n: int, seed: int = 3):
    """(height, width) for n images: width ~ U(480, 3840), aspect ~ U(0.5, 2), h = round(w / aspect)."""
    u = SplitMix64(seed).uniform(2 * n).reshape(n, 2)
    shapes = []
    for uw, ua in u:
        w = int(round(480 + (3840 - 480) * uw))
        aspect = 0.5 + 1.5 * ua
        shapes.append((int(round(w / aspect)), w))
    return shapes


def uneven_pair(k: int, seed: int = 3):
    """Pair k of the uneven batch: A of shape uneven_batch_shapes(...)[k] with blobs in
    proportion to its area, B = A under a 1080p-pair-style perspective warp about its
    centre.  Returns (A, B).

    The density is 6000 blobs per 1920x1080 (three times the 1080p workload's): the
    detected features grow sub-linearly with the blob count (overlapping blobs), and
    this density puts the median image of the batch near 5k features, inside the
    workload's "~4k-20k keypoints each"; with the count in proportion to the area,
    the smallest images (0.14 Mpx) stay below that range and the largest (23 Mpx)
    above it."""
    h, w = uneven_batch_shapes(k + 1, seed)[k]
    n_blobs = max(1, int(round(6000 * (w * h) / (1920 * 1080))))
    a = blob_image(w, h, n_blobs, 1.5, 20.0, seed * 100003 + k)
    u = SplitMix64((seed * 7919 + k) ^ 0xABCDEF).uniform(4)
    H = perspective_h(w, h, -30 + 60 * u[0], 0.7 + 0.7 * u[1], -2e-4 + 4e-4 * u[2], -2e-4 + 4e-4 * u[3])
    return a, warp_image(a, H)


def sift_like_descriptors(n: int, seed: int) -> np.ndarray:
    """|N(0,1)| per element, L2-normalised, clipped at 0.2, renormalised (float32, n x 128)."""
    rng = SplitMix64(seed)
    d = np.abs(rng.normal(n * 128)).reshape(n, 128)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    np.minimum(d, 0.2, out=d)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d.astype(np.float32)


def perturbed_queries(cat: np.ndarray, n: int, seed: int, noise: float = 0.02):
    """Queries = catalog descriptors (uniformly chosen) + |N(0, noise)|, renormalised/clipped/renormalised."""
    rng = SplitMix64(seed)
    src = (rng.uniform(n) * cat.shape[0]).astype(np.int64)
    d = cat[src].astype(np.float64) + noise * np.abs(rng.normal(n * 128)).reshape(n, 128)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    np.minimum(d, 0.2, out=d)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d.astype(np.float32), src


def correspondences(n: int, outlier_ratio: float, H: np.ndarray, width: int, height: int, seed: int,
                    noise_px: float = 0.5):
    """Putative matches: inliers = H p + N(0, noise_px), outliers uniform in the target image.

    Returns (q_xy[n,2], t_xy[n,2], ratio[n], is_inlier[n]).  Lowe ratios are drawn
    lower for inliers (U(0.2, 0.8)) than for outliers (U(0.5, 1.0)).
    """
    rng = SplitMix64(seed)
    q = rng.uniform(2 * n).reshape(n, 2) * np.array([width, height])
    inl = rng.uniform(n) >= outlier_ratio
    ph = np.c_[q, np.ones(n)] @ H.T
    t = ph[:, :2] / ph[:, 2:3] + noise_px * rng.normal(2 * n).reshape(n, 2)
    t_out = rng.uniform(2 * n).reshape(n, 2) * np.array([width, height])
    t = np.where(inl[:, None], t, t_out)
    ru = rng.uniform(n)
    ratio = np.where(inl, 0.2 + 0.6 * ru, 0.5 + 0.5 * ru)
    return q.astype(np.float32), t.astype(np.float32), ratio.astype(np.float32), inl


def putative_matches(n: int, outlier_ratio: float, H: np.ndarray, width: int, height: int, seed: int):
    """Putative matches with per-match attributes for the learned sampler.

    Inliers: target = H p + N(0, 0.5 px); log scale ratio = log of H's local scale
    + N(0, 0.08); orientation difference = H's local rotation + N(0, 0.08) rad;
    best descriptor distance U(0.10, 0.40); Lowe ratio U(0.2, 0.8).
    Outliers: uniform target; log scale ratio N(0, 0.7); orientation difference
    U(-pi, pi); best distance U(0.25, 0.60); ratio U(0.5, 1.0).
    Returns (records with fields query_index, target_index, query_x, query_y,
    target_x, target_y, distance, ratio, displacement_x, displacement_y;
    features (n, 8) float32; is_inlier (n,) bool).
    """
    rng = SplitMix64(seed)
    q = rng.uniform(2 * n).reshape(n, 2) * np.array([width, height])
    inl = rng.uniform(n) >= outlier_ratio
    ph = np.c_[q, np.ones(n)] @ H.T
    t_in = ph[:, :2] / ph[:, 2:3] + 0.5 * rng.normal(2 * n).reshape(n, 2)
    t_out = rng.uniform(2 * n).reshape(n, 2) * np.array([width, height])
    t = np.where(inl[:, None], t_in, t_out)
    # local similarity of H at q (finite differences)
    eps = 1.0
    px = np.c_[q[:, 0] + eps, q[:, 1], np.ones(n)] @ H.T
    px = px[:, :2] / px[:, 2:3]
    jac = (px - ph[:, :2] / ph[:, 2:3]) / eps
    loc_scale = np.log(np.maximum(np.hypot(jac[:, 0], jac[:, 1]), 1e-6))
    loc_rot = np.arctan2(jac[:, 1], jac[:, 0])
    g = rng.normal(2 * n).reshape(n, 2)
    u = rng.uniform(4 * n).reshape(n, 4)
    lsr = np.where(inl, loc_scale + 0.08 * g[:, 0], 0.7 * g[:, 1])
    dori = np.where(inl, loc_rot + 0.08 * g[:, 1], -np.pi + 2 * np.pi * u[:, 0])
    dori = (dori + np.pi) % (2 * np.pi) - np.pi
    dist = np.where(inl, 0.10 + 0.30 * u[:, 1], 0.25 + 0.35 * u[:, 2])
    ratio = np.where(inl, 0.2 + 0.6 * u[:, 3], 0.5 + 0.5 * u[:, 3])
    rec = np.zeros(n, dtype=[("query_index", "<u4"), ("target_index", "<u4"), ("query_x", "<f4"),
                             ("query_y", "<f4"), ("target_x", "<f4"), ("target_y", "<f4"), ("distance", "<f4"),
                             ("ratio", "<f4"), ("displacement_x", "<f4"), ("displacement_y", "<f4")])
    rec["query_index"] = np.arange(n)
    rec["target_index"] = np.arange(n)
    rec["query_x"], rec["query_y"] = q[:, 0], q[:, 1]
    rec["target_x"], rec["target_y"] = t[:, 0], t[:, 1]
    rec["distance"] = dist
    rec["ratio"] = ratio
    rec["displacement_x"] = rec["target_x"] - rec["query_x"]
    rec["displacement_y"] = rec["target_y"] - rec["query_y"]
    feats = np.stack([ratio, lsr, dori, dist, q[:, 0] / width, q[:, 1] / height, t[:, 0] / width,
                      t[:, 1] / height], axis=1).astype(np.float32)
    return rec, feats, inl


def epipolar_matches(n: int, outlier_ratio: float, seed: int, width: int = 1920, height: int = 1080,
                     noise_px: float = 0.5):
    """Putative matches between two views of a 3-D scene (fundamental-matrix workload).

    Camera 1 = K [I | 0], camera 2 = K [R | t] with K = (focal 1200 px, centred
    principal point), R a rotation of up to 10 degrees about a random axis and t a
    baseline of length 1 (mostly sideways).  Query points are uniform in image 1 at
    depths U(4, 20); inliers are their projections in image 2 + N(0, noise_px);
    outliers are uniform in image 2.  Ratios as `correspondences`.  Returns
    (records with the match fields, is_inlier (n,) bool, F_true (3, 3))."""
    rng = SplitMix64(seed)
    u = rng.uniform(6)
    axis = np.array([u[0] - 0.5, u[1] - 0.5, u[2] - 0.5])
    axis /= max(np.linalg.norm(axis), 1e-9)
    ang = np.deg2rad(10.0) * (2 * u[3] - 1)
    Kx = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    R = np.eye(3) + np.sin(ang) * Kx + (1 - np.cos(ang)) * (Kx @ Kx)
    t = np.array([1.0, 0.2 * (u[4] - 0.5), 0.2 * (u[5] - 0.5)])
    t /= np.linalg.norm(t)
    K = np.array([[1200.0, 0, width / 2], [0, 1200.0, height / 2], [0, 0, 1]])
    q = rng.uniform(2 * n).reshape(n, 2) * np.array([width, height])
    z = 4.0 + 16.0 * rng.uniform(n)
    X = (np.linalg.inv(K) @ np.c_[q, np.ones(n)].T).T * z[:, None]
    Y = (R @ X.T).T + t
    p2 = (K @ Y.T).T
    t_in = p2[:, :2] / p2[:, 2:3] + noise_px * rng.normal(2 * n).reshape(n, 2)
    inl = rng.uniform(n) >= outlier_ratio
    t_out = rng.uniform(2 * n).reshape(n, 2) * np.array([width, height])
    tp = np.where(inl[:, None], t_in, t_out)
    ru = rng.uniform(n)
    ratio = np.where(inl, 0.2 + 0.6 * ru, 0.5 + 0.5 * ru)
    rec = np.zeros(n, dtype=[("query_index", "<u4"), ("target_index", "<u4"), ("query_x", "<f4"),
                             ("query_y", "<f4"), ("target_x", "<f4"), ("target_y", "<f4"), ("distance", "<f4"),
                             ("ratio", "<f4"), ("displacement_x", "<f4"), ("displacement_y", "<f4")])
    rec["query_index"] = np.arange(n)
    rec["target_index"] = np.arange(n)
    rec["query_x"], rec["query_y"] = q[:, 0], q[:, 1]
    rec["target_x"], rec["target_y"] = tp[:, 0], tp[:, 1]
    rec["distance"] = 0.3
    rec["ratio"] = ratio
    rec["displacement_x"] = rec["target_x"] - rec["query_x"]
    rec["displacement_y"] = rec["target_y"] - rec["query_y"]
    tx = np.array([[0, -t[2], t[1]], [t[2], 0, -t[0]], [-t[1], t[0], 0]])
    Kinv = np.linalg.inv(K)
    F = Kinv.T @ tx @ R @ Kinv
    return rec, inl, F / np.linalg.norm(F)


def c5_pair(k: int, seed0: int = 500):
    """Pair k of the learned-sampler workload: 1920x1080 geometry, random
    perspective homography (as for the 1080p pair), 2k-8k matches, outlier ratio U(0.1, 0.7)."""
    u = SplitMix64(seed0 + 7919 * k).uniform(6)
    H = perspective_h(1920, 1080, -30 + 60 * u[0], 0.7 + 0.7 * u[1], -2e-4 + 4e-4 * u[2], -2e-4 + 4e-4 * u[3])
    n = int(2000 + 6000 * u[4])
    return putative_matches(n, 0.1 + 0.6 * u[5], H, 1920, 1080, seed0 + 104729 * k)
