"""ctypes binding of the CPU restatement (``oracle/psift_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA build.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference leg import
this module.  The product library never calls it.

Parity pinning: the reference (Rust) cannot be built here and ships no numeric
golden vectors; the restatement is pinned by the reference's own known-answer and
property tests, ported in ``tests/test_oracle_pins.py``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libpsift_oracle.so")
_lock = threading.Lock()
_lib = None


class Keypoint(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("scale", C.c_float), ("response", C.c_float),
                ("octave", C.c_uint32), ("layer", C.c_uint32)]


class Match(C.Structure):
    _fields_ = [("query_index", C.c_uint32), ("target_index", C.c_uint32),
                ("qx", C.c_float), ("qy", C.c_float), ("tx", C.c_float), ("ty", C.c_float),
                ("distance", C.c_float), ("ratio", C.c_float), ("dx", C.c_float), ("dy", C.c_float)]


class Tracking(C.Structure):
    _fields_ = [("raw_match_count", C.c_uint32), ("match_count", C.c_uint32),
                ("inlier_ratio", C.c_float), ("mean_dx", C.c_float), ("mean_dy", C.c_float),
                ("median_dx", C.c_float), ("median_dy", C.c_float),
                ("mean_scale_ratio", C.c_float), ("mean_rotation_deg", C.c_float)]


KEYPOINT_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("scale", "<f4"), ("response", "<f4"),
                           ("octave", "<u4"), ("layer", "<u4")])
MATCH_DTYPE = np.dtype([("query_index", "<u4"), ("target_index", "<u4"), ("qx", "<f4"), ("qy", "<f4"),
                        ("tx", "<f4"), ("ty", "<f4"), ("distance", "<f4"), ("ratio", "<f4"),
                        ("dx", "<f4"), ("dy", "<f4")])

_fp = C.POINTER(C.c_float)
_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_i64p = C.POINTER(C.c_int64)
_ip = C.POINTER(C.c_int)


def build() -> str:
    """Compile the restatement with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            src = os.path.join(_HERE, "psift_oracle.cpp")
            if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
                build()
            L = C.CDLL(_LIB_PATH)
            L.oracle_gaussian_kernel_1d.argtypes = [C.c_float, _fp, C.c_int]
            L.oracle_gaussian_kernel_1d.restype = C.c_int
            L.oracle_gaussian_blur.argtypes = [_fp, C.c_int, C.c_int, C.c_float, _fp]
            L.oracle_upsample_2x.argtypes = [_fp, C.c_int, C.c_int, _fp]
            L.oracle_luma_to_f32.argtypes = [_u8p, C.c_size_t, _fp]
            L.oracle_pyramid_build.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
            L.oracle_pyramid_build.restype = C.c_void_p
            L.oracle_pyramid_num_octaves.argtypes = [C.c_void_p]
            L.oracle_pyramid_num_octaves.restype = C.c_int
            L.oracle_pyramid_octave_info.argtypes = [C.c_void_p, C.c_int, _ip, _ip, _fp]
            L.oracle_pyramid_copy_plane.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _fp]
            L.oracle_pyramid_extract_extrema.argtypes = [C.c_void_p, C.c_float, C.c_void_p, C.c_int]
            L.oracle_pyramid_extract_extrema.restype = C.c_int
            L.oracle_pyramid_free.argtypes = [C.c_void_p]
            L.oracle_detect_and_compute.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                                    C.c_int, C.c_int, C.c_int, _fp, _fp, C.c_int]
            L.oracle_detect_and_compute.restype = C.c_int
            L.oracle_detect_keypoints.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                                  C.c_int, C.c_void_p, C.c_int]
            L.oracle_detect_keypoints.restype = C.c_int
            _dp = C.POINTER(C.c_double)
            L.oracle_detect_and_compute_f64.argtypes = [_u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                                        C.c_int, C.c_int, C.c_int, _dp, _dp, C.c_int]
            L.oracle_detect_and_compute_f64.restype = C.c_int
            L.oracle_detect_keypoints_f64.argtypes = [_u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                                      C.c_int, _dp, C.c_int]
            L.oracle_detect_keypoints_f64.restype = C.c_int
            L.oracle_compute_descriptors.argtypes = [_fp, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                                     _fp, _fp, C.c_int]
            L.oracle_compute_descriptors.restype = C.c_int
            L.oracle_rootsift.argtypes = [_fp, _fp]
            L.oracle_quantize_u8.argtypes = [_fp, C.c_int, _u8p]
            L.oracle_dequantize_u8.argtypes = [_u8p, C.c_int, _fp]
            L.oracle_quantize_u128.argtypes = [_fp, C.c_int, _u64p]
            L.oracle_match_descriptors.argtypes = [_fp, C.c_int, _fp, C.c_int, _fp, _fp, C.c_float, C.c_int,
                                                   C.c_void_p, C.c_int]
            L.oracle_match_descriptors.restype = C.c_int
            L.oracle_similarity_ransac.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_uint64, _u8p, _fp, _ip]
            L.oracle_similarity_ransac.restype = C.c_int
            L.oracle_homography_ransac.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_uint64, C.c_uint64,
                                                   _u8p, _fp, _ip]
            L.oracle_homography_ransac.restype = C.c_int
            L.oracle_summarize_tracking.argtypes = [C.c_void_p, C.c_int, _fp, _fp, _fp, _fp,
                                                    C.POINTER(Tracking)]
            L.oracle_hamming_votes.argtypes = [_u64p, C.c_int, _u64p, _i64p, C.c_int, C.c_int, _u32p]
            L.oracle_mih_votes_tables.argtypes = [_u64p, C.c_int, _u64p, _i64p, C.c_int, _u32p]
            L.oracle_hamming_topk.argtypes = [_u64p, C.c_int, _u64p, C.c_int64, C.c_int, _u32p, _u32p]
            L.oracle_l2_rerank.argtypes = [_fp, C.c_int, _fp, _u32p, C.c_int, _u32p, _fp]
            L.oracle_warp_and_stitch.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.c_void_p, C.c_int,
                                                 C.c_int, C.c_size_t, _fp, C.c_void_p, _ip, _ip, C.c_void_p]
            L.oracle_warp_and_stitch.restype = C.c_int
            L.oracle_fundamental_ransac.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_double,
                                                    C.c_uint64, _u8p, C.POINTER(C.c_double), _ip, _ip]
            L.oracle_fundamental_ransac.restype = C.c_int
            L.oracle_fit_fundamental_8point.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
            L.oracle_fit_fundamental_8point.restype = C.c_int
            L.oracle_fit_fundamental_7point.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
            L.oracle_fit_fundamental_7point.restype = C.c_int
            L.oracle_sampson_distance_sq.argtypes = [C.POINTER(C.c_double), C.c_double, C.c_double, C.c_double,
                                                     C.c_double]
            L.oracle_sampson_distance_sq.restype = C.c_double
            L.oracle_warp_cylindrical.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.c_float, C.c_void_p]
            L.oracle_panorama_register.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                                   C.POINTER(PanoramaOptions), _ip, C.c_void_p, _fp,
                                                   C.c_void_p, C.c_void_p, C.c_void_p, _ip, _ip]
            L.oracle_panorama_register.restype = C.c_int
            L.oracle_panorama_composite.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, _fp,
                                                    C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                                    C.c_int, C.c_void_p]
            L.oracle_solve_exposure_gains.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double,
                                                      C.c_double, _fp]
            L.oracle_splitmix64_next.argtypes = [_u64p]
            L.oracle_splitmix64_next.restype = C.c_uint64
            _lib = L
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _p(a, t):
    return a.ctypes.data_as(t)


DEFAULT_SIMILARITY_RANSAC_SEED = 0xD1B54A32D192ED03
DEFAULT_HOMOGRAPHY_RANSAC_SEED = 0x517CC1B727220A95


def gaussian_kernel_1d(sigma: float) -> np.ndarray:
    out = np.zeros(4096, np.float32)
    n = lib().oracle_gaussian_kernel_1d(sigma, _p(out, _fp), out.size)
    return out[:n].copy()


def gaussian_blur(img, sigma: float) -> np.ndarray:
    img = _f32(img)
    out = np.empty_like(img)
    lib().oracle_gaussian_blur(_p(img, _fp), img.shape[0], img.shape[1], sigma, _p(out, _fp))
    return out


def upsample_2x(img) -> np.ndarray:
    img = _f32(img)
    out = np.empty((img.shape[0] * 2, img.shape[1] * 2), np.float32)
    lib().oracle_upsample_2x(_p(img, _fp), img.shape[0], img.shape[1], _p(out, _fp))
    return out


def luma_to_f32(u8) -> np.ndarray:
    u8 = np.ascontiguousarray(u8, dtype=np.uint8)
    out = np.empty(u8.shape, np.float32)
    lib().oracle_luma_to_f32(_p(u8, _u8p), u8.size, _p(out, _fp))
    return out


class Pyramid:
    """Gaussian/DoG pyramid exactly as the reference materialises it."""

    def __init__(self, img, octaves=3, scales=3, upsample=True):
        img = _f32(img)
        self.scales = scales
        self._h = lib().oracle_pyramid_build(_p(img, _fp), img.shape[0], img.shape[1], octaves, scales,
                                             int(bool(upsample)))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_pyramid_free(self._h)
            self._h = None

    @property
    def num_octaves(self) -> int:
        return lib().oracle_pyramid_num_octaves(self._h)

    def octave_info(self, o):
        h, w, sf = C.c_int(), C.c_int(), C.c_float()
        lib().oracle_pyramid_octave_info(self._h, o, C.byref(h), C.byref(w), C.byref(sf))
        return h.value, w.value, sf.value

    def plane(self, o, kind, idx) -> np.ndarray:
        h, w, _ = self.octave_info(o)
        out = np.empty((h, w), np.float32)
        lib().oracle_pyramid_copy_plane(self._h, o, 0 if kind == "g" else 1, idx, _p(out, _fp))
        return out

    def extract_extrema(self, threshold: float) -> np.ndarray:
        cap = 1 << 16
        while True:
            out = np.zeros(cap, KEYPOINT_DTYPE)
            n = lib().oracle_pyramid_extract_extrema(self._h, threshold, out.ctypes.data, cap)
            if n <= cap:
                return out[:n]
            cap = n


def detect_keypoints(img, octaves=3, scales=3, threshold=0.015, upsample=True) -> np.ndarray:
    img = _f32(img)
    cap = 1 << 16
    while True:
        out = np.zeros(cap, KEYPOINT_DTYPE)
        n = lib().oracle_detect_keypoints(_p(img, _fp), img.shape[0], img.shape[1], octaves, scales,
                                          threshold, int(bool(upsample)), out.ctypes.data, cap)
        if n <= cap:
            return out[:n]
        cap = n


def detect_and_compute(img, octaves=3, scales=3, threshold=0.015, upsample=True, kind=0,
                       max_features=4096):
    """Returns (meta[n,5] = x, y, scale, response, orientation; desc[n,128])."""
    img = _f32(img)
    cap = max(max_features, 1) if max_features > 0 else 1 << 15
    while True:
        meta = np.zeros((cap, 5), np.float32)
        desc = np.zeros((cap, 128), np.float32)
        n = lib().oracle_detect_and_compute(_p(img, _fp), img.shape[0], img.shape[1], octaves, scales,
                                            threshold, int(bool(upsample)), int(kind), int(max_features),
                                            _p(meta, _fp), _p(desc, _fp), cap)
        if n <= cap:
            return meta[:n].copy(), desc[:n].copy()
        cap = n


def detect_keypoints_f64(luma_u8, octaves=3, scales=3, threshold=0.015, upsample=True) -> np.ndarray:
    """The keypoints of the pipeline run in f64 from the u8 luma: (n, 6) float64
    rows (x, y, scale, response, octave, layer)."""
    u8 = np.ascontiguousarray(luma_u8, dtype=np.uint8)
    dp = C.POINTER(C.c_double)
    cap = 1 << 16
    while True:
        out = np.zeros((cap, 6), np.float64)
        n = lib().oracle_detect_keypoints_f64(_p(u8, _u8p), u8.shape[0], u8.shape[1], octaves, scales,
                                              threshold, int(bool(upsample)), _p(out, dp), cap)
        if n <= cap:
            return out[:n].copy()
        cap = n


def detect_and_compute_f64(luma_u8, octaves=3, scales=3, threshold=0.015, upsample=True, kind=0,
                           max_features=4096):
    """The pipeline run in f64 from the u8 luma: (meta[n,5], desc[n,128]) float64."""
    u8 = np.ascontiguousarray(luma_u8, dtype=np.uint8)
    dp = C.POINTER(C.c_double)
    cap = max(max_features, 1) if max_features > 0 else 1 << 15
    while True:
        meta = np.zeros((cap, 5), np.float64)
        desc = np.zeros((cap, 128), np.float64)
        n = lib().oracle_detect_and_compute_f64(_p(u8, _u8p), u8.shape[0], u8.shape[1], octaves, scales,
                                                threshold, int(bool(upsample)), int(kind), int(max_features),
                                                _p(meta, dp), _p(desc, dp), cap)
        if n <= cap:
            return meta[:n].copy(), desc[:n].copy()
        cap = n


def compute_descriptors(img, keypoints, kind=0):
    img = _f32(img)
    kps = np.ascontiguousarray(keypoints, dtype=KEYPOINT_DTYPE)
    cap = max(4 * len(kps), 1)
    meta = np.zeros((cap, 5), np.float32)
    desc = np.zeros((cap, 128), np.float32)
    n = lib().oracle_compute_descriptors(_p(img, _fp), img.shape[0], img.shape[1], kps.ctypes.data, len(kps),
                                         int(kind), _p(meta, _fp), _p(desc, _fp), cap)
    return meta[:n].copy(), desc[:n].copy()


def rootsift(desc) -> np.ndarray:
    d = _f32(desc).reshape(-1, 128)
    out = np.empty_like(d)
    for i in range(d.shape[0]):
        lib().oracle_rootsift(_p(d[i], _fp), _p(out[i], _fp))
    return out


def quantize_u8(desc) -> np.ndarray:
    d = _f32(desc).ravel()
    out = np.empty(d.size, np.uint8)
    lib().oracle_quantize_u8(_p(d, _fp), d.size, _p(out, _u8p))
    return out.reshape(np.shape(desc))


def dequantize_u8(q) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.uint8).reshape(-1, 128)
    out = np.empty(q.shape, np.float32)
    for i in range(q.shape[0]):
        lib().oracle_dequantize_u8(_p(q[i], _u8p), 128, _p(out[i], _fp))
    return out


def quantize_u128(desc) -> np.ndarray:
    d = _f32(desc).reshape(-1, 128)
    out = np.empty((d.shape[0], 2), np.uint64)
    lib().oracle_quantize_u128(_p(d, _fp), d.shape[0], _p(out, _u64p))
    return out


def match(q_desc, t_desc, q_xy, t_xy, ratio=0.75, mutual=False) -> np.ndarray:
    qd, td = _f32(q_desc).reshape(-1, 128), _f32(t_desc).reshape(-1, 128)
    qxy, txy = _f32(q_xy).reshape(-1, 2), _f32(t_xy).reshape(-1, 2)
    cap = max(qd.shape[0], 1)
    out = np.zeros(cap, MATCH_DTYPE)
    n = lib().oracle_match_descriptors(_p(qd, _fp), qd.shape[0], _p(td, _fp), td.shape[0], _p(qxy, _fp),
                                       _p(txy, _fp), ratio, int(bool(mutual)), out.ctypes.data, cap)
    return out[:n].copy()


def similarity_ransac(matches, thr=3.0, seed=DEFAULT_SIMILARITY_RANSAC_SEED):
    m = np.ascontiguousarray(matches, dtype=MATCH_DTYPE)
    mask = np.zeros(max(len(m), 1), np.uint8)
    model = np.zeros(6, np.float32)
    has = C.c_int()
    lib().oracle_similarity_ransac(m.ctypes.data, len(m), thr, seed, _p(mask, _u8p), _p(model, _fp),
                                   C.byref(has))
    return mask[:len(m)].astype(bool), (model if has.value else None)


def homography_ransac(matches, thr=3.0, seed=None):
    m = np.ascontiguousarray(matches, dtype=MATCH_DTYPE)
    if seed is None:
        s1, s2 = DEFAULT_SIMILARITY_RANSAC_SEED, DEFAULT_HOMOGRAPHY_RANSAC_SEED
    else:
        s1, s2 = seed, seed ^ 0x9E3779B97F4A7C15
    mask = np.zeros(max(len(m), 1), np.uint8)
    h9 = np.zeros(9, np.float32)
    has = C.c_int()
    lib().oracle_homography_ransac(m.ctypes.data, len(m), thr, s1, s2, _p(mask, _u8p), _p(h9, _fp),
                                   C.byref(has))
    return mask[:len(m)].astype(bool), (h9.reshape(3, 3) if has.value else None)


def summarize_tracking(matches, q_scale, q_ori, t_scale, t_ori) -> Tracking:
    m = np.ascontiguousarray(matches, dtype=MATCH_DTYPE)
    qs, qo, ts, to = (_f32(a) for a in (q_scale, q_ori, t_scale, t_ori))
    out = Tracking()
    lib().oracle_summarize_tracking(m.ctypes.data, len(m), _p(qs, _fp), _p(qo, _fp), _p(ts, _fp),
                                    _p(to, _fp), C.byref(out))
    return out


def hamming_votes(q_codes, cat_codes, offsets, mih: bool) -> np.ndarray:
    q = np.ascontiguousarray(q_codes, dtype=np.uint64).reshape(-1, 2)
    c = np.ascontiguousarray(cat_codes, dtype=np.uint64).reshape(-1, 2)
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    votes = np.zeros(len(off) - 1, np.uint32)
    lib().oracle_hamming_votes(_p(q, _u64p), q.shape[0], _p(c, _u64p), _p(off, _i64p), len(off) - 1,
                               int(bool(mih)), _p(votes, _u32p))
    return votes


def mih_votes_tables(q_codes, cat_codes, offsets) -> np.ndarray:
    """MIH votes by the reference's own table walk (inverted tables + seen_stamp)."""
    q = np.ascontiguousarray(q_codes, dtype=np.uint64).reshape(-1, 2)
    c = np.ascontiguousarray(cat_codes, dtype=np.uint64).reshape(-1, 2)
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    votes = np.zeros(len(off) - 1, np.uint32)
    lib().oracle_mih_votes_tables(_p(q, _u64p), q.shape[0], _p(c, _u64p), _p(off, _i64p), len(off) - 1,
                                  _p(votes, _u32p))
    return votes


def hamming_topk(q_codes, cat_codes, k: int):
    q = np.ascontiguousarray(q_codes, dtype=np.uint64).reshape(-1, 2)
    c = np.ascontiguousarray(cat_codes, dtype=np.uint64).reshape(-1, 2)
    idx = np.empty((q.shape[0], k), np.uint32)
    dist = np.empty((q.shape[0], k), np.uint32)
    lib().oracle_hamming_topk(_p(q, _u64p), q.shape[0], _p(c, _u64p), c.shape[0], k, _p(idx, _u32p),
                              _p(dist, _u32p))
    return idx, dist


def l2_rerank(q_desc, cat_desc, cand):
    qd, cd = _f32(q_desc).reshape(-1, 128), _f32(cat_desc).reshape(-1, 128)
    cand = np.ascontiguousarray(cand, dtype=np.uint32)
    k = cand.shape[1]
    out_idx = np.empty_like(cand)
    out_d2 = np.empty(cand.shape, np.float32)
    lib().oracle_l2_rerank(_p(qd, _fp), qd.shape[0], _p(cd, _fp), _p(cand, _u32p), k, _p(out_idx, _u32p),
                           _p(out_d2, _fp))
    return out_idx, out_d2


def warp_and_stitch(query, target, h9):
    """warp_and_stitch (src/visualize.rs:379-483): (canvas, (origin_x, origin_y)), or
    an int error code (-1 singular, -2 infinity, -3 non-finite, -4 too large)."""
    q = np.ascontiguousarray(query, dtype=np.uint8)
    t = np.ascontiguousarray(target, dtype=np.uint8)
    h = _f32(h9).reshape(9)
    w, hh = C.c_int(), C.c_int()
    origin = np.zeros(2, np.float64)
    rc = lib().oracle_warp_and_stitch(q.ctypes.data, q.shape[0], q.shape[1], q.shape[1] * 4, t.ctypes.data,
                                      t.shape[0], t.shape[1], t.shape[1] * 4, _p(h, _fp), None, C.byref(w),
                                      C.byref(hh), origin.ctypes.data)
    if rc != 0:
        return rc
    canvas = np.zeros((hh.value, w.value, 4), np.uint8)
    lib().oracle_warp_and_stitch(q.ctypes.data, q.shape[0], q.shape[1], q.shape[1] * 4, t.ctypes.data,
                                 t.shape[0], t.shape[1], t.shape[1] * 4, _p(h, _fp), canvas.ctypes.data,
                                 C.byref(w), C.byref(hh), origin.ctypes.data)
    return canvas, (float(origin[0]), float(origin[1]))


DEFAULT_FUNDAMENTAL_SEED = 0xF00DCAFE12345678


def _as_oracle_matches(matches) -> np.ndarray:
    m = np.ascontiguousarray(matches)
    return m if m.dtype == MATCH_DTYPE else m.view(MATCH_DTYPE)


def fundamental_ransac(matches, sampson_threshold=1.5, max_iters=2000, confidence=0.999,
                       seed=DEFAULT_FUNDAMENTAL_SEED):
    """estimate_fundamental_ransac_with_options (src/geometry.rs:868-1016):
    (inlier mask, F (3, 3) f64 or None, iterations)."""
    m = _as_oracle_matches(matches)
    n = len(m)
    mask = np.zeros(max(n, 1), np.uint8)
    f9 = np.zeros(9, np.float64)
    has, iters = C.c_int(), C.c_int()
    lib().oracle_fundamental_ransac(m.ctypes.data, n, sampson_threshold, max_iters, confidence,
                                    seed & 0xFFFFFFFFFFFFFFFF, _p(mask, _u8p), f9.ctypes.data_as(C.POINTER(C.c_double)),
                                    C.byref(has), C.byref(iters))
    return mask[:n].astype(bool), (f9.reshape(3, 3) if has.value else None), iters.value


def fit_fundamental_8point(matches):
    m = _as_oracle_matches(matches)
    f9 = np.zeros(9, np.float64)
    ok = lib().oracle_fit_fundamental_8point(m.ctypes.data, len(m), f9.ctypes.data_as(C.POINTER(C.c_double)))
    return f9.reshape(3, 3) if ok else None


def fit_fundamental_7point(matches):
    """fit_fundamental_7point (src/geometry.rs:727-806) of the first 7 matches: list of F."""
    m = _as_oracle_matches(matches)[:7]
    out = np.zeros(36, np.float64)
    k = lib().oracle_fit_fundamental_7point(m.ctypes.data, out.ctypes.data_as(C.POINTER(C.c_double)))
    return [out[9 * i:9 * i + 9].reshape(3, 3).copy() for i in range(k)]


# ---------------------------------------------------------------- stitch_panorama
class PanoramaOptions(C.Structure):
    """PanoramaOptions (src/stitch.rs:45-89); projection 0 planar / 1 cylindrical,
    blend 0 feather / 1 multi-band."""
    _fields_ = [("octaves", C.c_int), ("scales", C.c_int), ("threshold", C.c_float), ("ratio", C.c_float),
                ("ransac_threshold", C.c_float), ("projection", C.c_int), ("focal_px", C.c_float),
                ("blend", C.c_int), ("levels", C.c_int), ("exposure_compensation", C.c_int),
                ("max_canvas_dim", C.c_int), ("max_canvas_pixels", C.c_longlong), ("tile_size", C.c_int)]

    @classmethod
    def default(cls, **kw):
        o = cls(3, 3, 0.015, 0.75, 3.0, 0, 0.0, 1, 4, 1, 8192, 25_000_000, 512)
        for k, v in kw.items():
            setattr(o, k, v)
        return o


def warp_cylindrical(rgba, focal_px: float) -> np.ndarray:
    """warp_image_cylindrical (src/stitch.rs:166-201) on an H x W x 4 u8 image."""
    img = np.ascontiguousarray(rgba, dtype=np.uint8)
    h, w = img.shape[:2]
    out = np.zeros_like(img)
    lib().oracle_warp_cylindrical(img.ctypes.data, h, w, w * 4, float(focal_px), out.ctypes.data)
    return out


def _img_ptrs(imgs):
    imgs = [np.ascontiguousarray(im, dtype=np.uint8) for im in imgs]
    ptrs = (C.c_void_p * len(imgs))(*[im.ctypes.data for im in imgs])
    hs = np.array([im.shape[0] for im in imgs], np.int32)
    ws = np.array([im.shape[1] for im in imgs], np.int32)
    return imgs, ptrs, hs, ws


def panorama_register(prepared, opt: PanoramaOptions):
    """The registration half of stitch_panorama on prepared RGBA images: a dict with
    ref, registered, gains, h_to_ref (n, 3, 3), inv (n, 3, 3), origin, width, height,
    or an int error code (< 0)."""
    imgs, ptrs, hs, ws = _img_ptrs(prepared)
    n = len(imgs)
    ref = C.c_int()
    reg = np.zeros(n, np.uint8)
    gains = np.zeros(n, np.float32)
    H = np.zeros((n, 9), np.float64)
    inv = np.zeros((n, 9), np.float64)
    origin = np.zeros(2, np.float64)
    w, h = C.c_int(), C.c_int()
    rc = lib().oracle_panorama_register(ptrs, hs.ctypes.data, ws.ctypes.data, n, C.byref(opt), C.byref(ref),
                                        reg.ctypes.data, _p(gains, _fp), H.ctypes.data, inv.ctypes.data,
                                        origin.ctypes.data, C.byref(w), C.byref(h))
    if rc != 0:
        return rc
    return {"ref": ref.value, "registered": reg.astype(bool), "gains": gains, "h_to_ref": H.reshape(n, 3, 3),
            "inv": inv.reshape(n, 3, 3), "origin": origin, "width": w.value, "height": h.value}


def panorama_composite(prepared, reg: dict, blend: int, levels: int = 4, tile_size: int = 512) -> np.ndarray:
    """The blending half of stitch_panorama: the canvas (height, width, 4) u8."""
    imgs, ptrs, hs, ws = _img_ptrs(prepared)
    canvas = np.zeros((reg["height"], reg["width"], 4), np.uint8)
    regm = np.ascontiguousarray(reg["registered"], dtype=np.uint8)
    inv = np.ascontiguousarray(reg["inv"], dtype=np.float64)
    lib().oracle_panorama_composite(ptrs, hs.ctypes.data, ws.ctypes.data, len(imgs), regm.ctypes.data,
                                    _p(_f32(reg["gains"]), _fp), inv.ctypes.data,
                                    np.ascontiguousarray(reg["origin"], dtype=np.float64).ctypes.data,
                                    reg["width"], reg["height"], int(blend), int(levels), int(tile_size),
                                    canvas.ctypes.data)
    return canvas


def stitch_panorama(images, opt: PanoramaOptions):
    """stitch_panorama (src/stitch.rs:472-948) on H x W x 4 u8 images: (canvas, reg)
    or an int error code."""
    prepared = [np.ascontiguousarray(im, dtype=np.uint8) for im in images]
    if opt.projection == 1:
        prepared = [warp_cylindrical(im, opt.focal_px) for im in prepared]
    reg = panorama_register(prepared, opt)
    if isinstance(reg, int):
        return reg
    return panorama_composite(prepared, reg, opt.blend, opt.levels, opt.tile_size), reg


def solve_exposure_gains(pairs, n_images: int, ref_idx: int, sigma_n=10.0, sigma_g=0.25) -> np.ndarray:
    pr = np.ascontiguousarray(pairs, dtype=np.float64).reshape(-1, 5)
    out = np.zeros(n_images, np.float32)
    lib().oracle_solve_exposure_gains(pr.ctypes.data, pr.shape[0], n_images, ref_idx, sigma_n, sigma_g,
                                      _p(out, _fp))
    return out
