"""Python mirror of pure-sift's hot-path API over the sm_100a C ABI (libpsift_gpu.so).

Names, argument meaning and error behaviour follow the reference's Rust API
(src/lib.rs:26-52, src/pipeline.rs:22-247, src/catalog.rs:37-45, :576-702):

* ``SiftConfig`` builder + ``validate()``; ``Sift.new(config)`` raises
  ``ValueError`` with the reference's message where Rust returns ``Err(String)``.
* ``Sift.detect_and_compute(img)`` / ``detect_keypoints(img)`` take a float32
  ``(H, W)`` luma array in [0, 1] (the reference's ``Array2<f32>``); ``*_u8``
  variants take u8 luma (``luma_to_array2`` is fused on the device).
* Compute calls are infallible in the reference; here a device failure raises
  ``PsiftError`` (there is no CPU fallback).

Every compute call runs on the GPU through the C ABI; importing this module on
a machine without the built library raises ``ImportError``.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from dataclasses import dataclass, field, replace

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpsift_gpu.so")

BASE_SIGMA = 1.6
DEFAULT_CONTRAST_THRESHOLD = 0.015
DEFAULT_MATCH_RATIO = 0.75
DEFAULT_RANSAC_REPROJ_THRESHOLD = 3.0
MAX_FEATURES_PER_IMAGE = 4096
SIFT_DESCRIPTOR_LEN = 128
DEFAULT_SIMILARITY_RANSAC_SEED = 0xD1B54A32D192ED03
DEFAULT_HOMOGRAPHY_RANSAC_SEED = 0x517CC1B727220A95

PSIFT_OK = 0
PSIFT_ERR_INVALID_ARGUMENT = 1
PSIFT_ERR_INVALID_CONFIG = 2
PSIFT_ERR_CAPACITY = 3
PSIFT_ERR_IO = 9
PSIFT_ERR_FORMAT = 10
STATUS_NAMES = {0: "OK", 1: "INVALID_ARGUMENT", 2: "INVALID_CONFIG", 3: "CAPACITY", 4: "CUDA",
                5: "OUT_OF_MEMORY", 6: "TIMEOUT", 7: "NO_DEVICE", 8: "INTERNAL", 9: "IO", 10: "FORMAT"}


class PsiftError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"psift {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class CSiftConfig(C.Structure):
    _fields_ = [("octaves", C.c_uint32), ("scales", C.c_uint32), ("contrast_threshold", C.c_float),
                ("upsample_first_octave", C.c_int32), ("descriptor_kind", C.c_int32),
                ("max_features", C.c_uint32)]


class CKeypoint(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("scale", C.c_float), ("response", C.c_float),
                ("octave", C.c_uint32), ("layer", C.c_uint32)]


class CFeatures(C.Structure):
    _fields_ = [("capacity", C.c_uint32), ("count", C.c_uint32), ("x", C.c_void_p), ("y", C.c_void_p),
                ("scale", C.c_void_p), ("response", C.c_void_p), ("orientation", C.c_void_p),
                ("descriptors", C.c_void_p)]


class CImageU8(C.Structure):
    _fields_ = [("data", C.c_void_p), ("height", C.c_uint32), ("width", C.c_uint32), ("row_stride", C.c_size_t)]


class CMatchOptions(C.Structure):
    _fields_ = [("ratio", C.c_float), ("mutual", C.c_int32), ("precision", C.c_int32)]


class CMatchJob(C.Structure):
    _fields_ = [("query_descriptors", C.c_void_p), ("target_descriptors", C.c_void_p), ("query_xy", C.c_void_p),
                ("target_xy", C.c_void_p), ("nq", C.c_uint32), ("nt", C.c_uint32), ("out", C.c_void_p),
                ("capacity", C.c_uint32), ("d_count", C.c_void_p)]


MATCH_DTYPE = np.dtype([("query_index", "<u4"), ("target_index", "<u4"), ("query_x", "<f4"), ("query_y", "<f4"),
                        ("target_x", "<f4"), ("target_y", "<f4"), ("distance", "<f4"), ("ratio", "<f4"),
                        ("displacement_x", "<f4"), ("displacement_y", "<f4")])
PRECISION_FP32 = 0
PRECISION_BF16_RERANK = 1

class CRansacOptions(C.Structure):
    _fields_ = [("reproj_threshold", C.c_float), ("has_seed", C.c_int32), ("seed", C.c_uint64)]


class CRansacJob(C.Structure):
    _fields_ = [("matches", C.c_void_p), ("n", C.c_uint32), ("inlier_mask", C.c_void_p), ("model", C.c_void_p),
                ("has_model", C.c_void_p), ("inlier_count", C.c_void_p), ("sampling_weights", C.c_void_p),
                ("iterations", C.c_void_p)]


class CTracking(C.Structure):
    _fields_ = [("raw_match_count", C.c_uint32), ("match_count", C.c_uint32), ("inlier_ratio", C.c_float),
                ("mean_dx", C.c_float), ("mean_dy", C.c_float), ("median_dx", C.c_float),
                ("median_dy", C.c_float), ("mean_scale_ratio", C.c_float), ("mean_rotation_deg", C.c_float)]


class CFundamentalOptions(C.Structure):
    _fields_ = [("sampson_threshold", C.c_double), ("max_iters", C.c_uint32), ("confidence", C.c_double),
                ("seed", C.c_uint64)]


class CFundamentalJob(C.Structure):
    _fields_ = [("matches", C.c_void_p), ("n", C.c_uint32), ("inlier_mask", C.c_void_p), ("f9", C.c_void_p),
                ("has_f", C.c_void_p), ("inlier_count", C.c_void_p), ("iterations", C.c_void_p)]


class CCatalogParams(C.Structure):
    _fields_ = [("octaves", C.c_uint32), ("scales", C.c_uint32), ("threshold", C.c_float),
                ("descriptor_kind", C.c_int32)]


class CCatalogHit(C.Structure):
    _fields_ = [("entry", C.c_uint32), ("coarse_votes", C.c_uint32), ("tracking", CTracking),
                ("similarity", C.c_float * 6), ("has_similarity", C.c_int32), ("homography", C.c_float * 9),
                ("has_homography", C.c_int32)]


KEYPOINT_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("scale", "<f4"), ("response", "<f4"),
                           ("octave", "<u4"), ("layer", "<u4")])

# Every entry point declared in include/psift_gpu.h, with its ctypes signature.
_SIGS = {
    "psift_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "psift_ctx_destroy": (C.c_int, [C.c_void_p]),
    "psift_last_error": (C.c_char_p, [C.c_void_p]),
    "psift_ctx_launch_count": (C.c_uint64, [C.c_void_p]),
    "psift_ctx_stream": (C.c_void_p, [C.c_void_p]),
    "psift_ctx_synchronize": (C.c_int, [C.c_void_p]),
    "psift_ctx_enable_stage_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "psift_ctx_stage_times": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int]),
    "psift_sift_config_default": (None, [C.POINTER(CSiftConfig)]),
    "psift_sift_config_validate": (C.c_int, [C.POINTER(CSiftConfig), C.c_char_p, C.c_size_t]),
    "psift_detect_and_compute": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_size_t,
                                           C.POINTER(CSiftConfig), C.POINTER(CFeatures)]),
    "psift_detect_and_compute_u8": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_size_t,
                                              C.POINTER(CSiftConfig), C.POINTER(CFeatures)]),
    "psift_detect_keypoints": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_size_t,
                                         C.POINTER(CSiftConfig), C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]),
    "psift_detect_and_compute_batch_dev": (C.c_int, [C.c_void_p, C.POINTER(CImageU8), C.c_uint32,
                                                     C.POINTER(CSiftConfig), C.POINTER(CFeatures), C.c_void_p]),
    "psift_match_options_default": (None, [C.POINTER(CMatchOptions)]),
    "psift_match_options_validate": (C.c_int, [C.POINTER(CMatchOptions), C.c_char_p, C.c_size_t]),
    "psift_match_descriptors": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                          C.c_void_p, C.POINTER(CMatchOptions), C.c_void_p, C.c_uint32,
                                          C.POINTER(C.c_uint32)]),
    "psift_match_batch_dev": (C.c_int, [C.c_void_p, C.POINTER(CMatchJob), C.c_uint32, C.POINTER(CMatchOptions)]),
    "psift_ctx_rerank_fallbacks": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "psift_ransac_options_default": (None, [C.POINTER(CRansacOptions)]),
    "psift_ransac_options_validate": (C.c_int, [C.POINTER(CRansacOptions), C.c_char_p, C.c_size_t]),
    "psift_homography_estimate": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(CRansacOptions),
                                            C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_uint32)]),
    "psift_similarity_estimate": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(CRansacOptions),
                                            C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_uint32)]),
    "psift_ransac_batch_dev": (C.c_int, [C.c_void_p, C.POINTER(CRansacJob), C.c_uint32, C.POINTER(CRansacOptions),
                                         C.c_int32]),
    "psift_mlp_init": (None, [C.c_uint64, C.c_void_p]),
    "psift_mlp_infer": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "psift_mlp_infer_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "psift_mlp_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                      C.c_void_p]),
    "psift_mlp_gradients_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                          C.c_void_p]),
    "psift_mlp_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                  C.c_uint32, C.c_float, C.c_uint64, C.c_void_p]),
    "psift_mlp_train_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                      C.c_uint32, C.c_float, C.c_uint64, C.c_void_p]),
    "psift_gaussian_blur": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_size_t, C.c_float,
                                      C.c_void_p]),
    "psift_build_pyramid": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_size_t,
                                      C.POINTER(CSiftConfig), C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    "psift_jpeg_info": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int32, C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "psift_decode_jpeg_luma": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int32, C.c_void_p, C.c_size_t,
                                         C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "psift_detect_and_compute_jpeg_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int32,
                                                      C.POINTER(CSiftConfig), C.c_void_p]),
    "psift_png_info": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int32, C.POINTER(C.c_uint32),
                                 C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "psift_decode_png_luma": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int32, C.c_void_p, C.c_size_t,
                                        C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "psift_detect_and_compute_png_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int32,
                                                     C.POINTER(CSiftConfig), C.c_void_p]),
    "psift_detect_and_compute_image_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int32,
                                                       C.POINTER(CSiftConfig), C.c_void_p]),
    "psift_ctx_jpeg_backend": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "psift_ctx_set_jpeg_threads": (C.c_int, [C.c_void_p, C.c_int32]),
    "psift_detect_and_compute_u8_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(CSiftConfig),
                                                    C.c_void_p]),
    "psift_ctx_enable_graphs": (C.c_int, [C.c_void_p, C.c_int]),
    "psift_ctx_graph_replays": (C.c_uint64, [C.c_void_p]),
    "psift_host_alloc": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(C.c_void_p)]),
    "psift_host_free": (C.c_int, [C.c_void_p, C.c_void_p]),
    "psift_compute_descriptors": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_size_t, C.c_void_p,
                                            C.c_uint32, C.c_int32, C.POINTER(CFeatures)]),
    "psift_summarize_tracking": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                                           C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(CTracking)]),
    "psift_quantize_u128_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "psift_popc_throughput": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "psift_quantize_u128": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "psift_quantize_u8": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "psift_dequantize_u8": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "psift_hamming_votes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                                      C.c_int32, C.c_void_p]),
    "psift_hamming_topk": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.c_uint32,
                                     C.c_void_p, C.c_void_p]),
    "psift_hamming_topk_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.c_uint32,
                                         C.c_void_p, C.c_void_p]),
    "psift_l2_rerank": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p,
                                  C.c_uint32, C.c_void_p, C.c_void_p]),
    "psift_l2_rerank_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                                      C.c_void_p, C.c_void_p]),
    "psift_detect_and_compute_u8_noalloc_dev": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_size_t,
                                                          C.POINTER(CSiftConfig), C.POINTER(CFeatures), C.c_void_p,
                                                          C.c_void_p]),
    "psift_ctx_autotune": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(CSiftConfig),
                                     C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]),
    "psift_ctx_tuning_get": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "psift_ctx_tuning_set": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
    "psift_ctx_set_blur_rounding": (C.c_int, [C.c_void_p, C.c_int32]),
    "psift_panorama_options_default": (None, [C.c_void_p]),
    "psift_stitch_panorama": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_size_t,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "psift_warp_cylindrical": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p]),
    "psift_panorama_composite": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_double, C.c_double, C.c_uint32, C.c_uint32, C.c_int32, C.c_uint32,
                                           C.c_void_p]),
    "psift_fundamental_options_default": (None, [C.POINTER(CFundamentalOptions)]),
    "psift_fundamental_estimate": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(CFundamentalOptions),
                                             C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_uint32),
                                             C.POINTER(C.c_uint32)]),
    "psift_fundamental_batch_dev": (C.c_int, [C.c_void_p, C.POINTER(CFundamentalJob), C.c_uint32,
                                              C.POINTER(CFundamentalOptions)]),
    "psift_warp_and_stitch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_size_t, C.c_void_p,
                                        C.c_uint32, C.c_uint32, C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t,
                                        C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_void_p]),
    "psift_warp_and_stitch_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_size_t,
                                            C.c_void_p, C.c_uint32, C.c_uint32, C.c_size_t, C.c_void_p,
                                            C.c_void_p, C.c_size_t, C.POINTER(C.c_uint32),
                                            C.POINTER(C.c_uint32)]),
    "psift_catalog_create": (C.c_int, [C.c_void_p, C.POINTER(CCatalogParams), C.POINTER(C.c_void_p)]),
    "psift_catalog_destroy": (C.c_int, [C.c_void_p]),
    "psift_catalog_params_get": (C.c_int, [C.c_void_p, C.POINTER(CCatalogParams)]),
    "psift_catalog_size": (C.c_uint32, [C.c_void_p]),
    "psift_catalog_entry": (C.c_int, [C.c_void_p, C.c_uint32, C.c_char_p, C.c_size_t, C.POINTER(C.c_uint32),
                                      C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    "psift_catalog_find": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_uint32)]),
    "psift_catalog_upsert": (C.c_int, [C.c_void_p, C.c_char_p, C.c_uint32, C.c_uint32, C.POINTER(CFeatures)]),
    "psift_catalog_remove": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int32)]),
    "psift_catalog_features": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(CFeatures), C.c_void_p]),
    "psift_catalog_load_binary": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    "psift_catalog_save_binary": (C.c_int, [C.c_void_p, C.c_char_p]),
    "psift_catalog_votes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int32, C.c_void_p]),
    "psift_catalog_set_search_votes": (C.c_int, [C.c_void_p, C.c_int32]),
    "psift_catalog_search": (C.c_int, [C.c_void_p, C.POINTER(CFeatures), C.c_uint32, C.c_uint32, C.c_float,
                                       C.c_float, C.POINTER(CCatalogHit), C.c_uint32, C.POINTER(C.c_uint32)]),
}

_lib = None
_lib_lock = threading.Lock()


def load_library() -> C.CDLL:
    """Load libpsift_gpu.so (built in-tree by ``make -C pure-sift_b200``)."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(f"{LIB_PATH} is not built; run `make -C {_HERE}` (nvcc, sm_100a)")
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def exported_symbols():
    return list(_SIGS)


class Context:
    """One CUDA stream + workspace on one GPU (``psift_ctx``); not thread-safe."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        st = self.lib.psift_ctx_create(device, C.byref(h))
        if st != PSIFT_OK:
            raise PsiftError(st, "psift_ctx_create failed (no usable sm_100 device?)")
        self.handle = h
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            self.lib.psift_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, st: int):
        if st != PSIFT_OK:
            raise PsiftError(st, self.lib.psift_last_error(self.handle).decode())

    def set_jpeg_threads(self, threads: int):
        """JPEG batch decode: 0 = shares over host threads (default), 1 = one batched call."""
        self.check(self.lib.psift_ctx_set_jpeg_threads(self.handle, int(threads)))

    @property
    def jpeg_backend(self) -> int:
        """nvJPEG backend of the last decoded JPEG batch (3 hardware, 2 GPU-assisted, 1 hybrid
        on host threads, -1 none)."""
        b = C.c_int32()
        self.check(self.lib.psift_ctx_jpeg_backend(self.handle, C.byref(b)))
        return int(b.value)

    @property
    def launch_count(self) -> int:
        return int(self.lib.psift_ctx_launch_count(self.handle))

    @property
    def stream(self) -> int:
        return int(self.lib.psift_ctx_stream(self.handle) or 0)

    def synchronize(self):
        self.check(self.lib.psift_ctx_synchronize(self.handle))

    def enable_graphs(self, on: bool = True):
        self.check(self.lib.psift_ctx_enable_graphs(self.handle, int(on)))

    @property
    def graph_replays(self) -> int:
        return int(self.lib.psift_ctx_graph_replays(self.handle))

    STAGES = ("pyramid", "extrema", "select", "orientation", "descriptor", "match", "hamming", "ransac", "mlp")

    def enable_stage_timing(self, on: bool = True):
        self.check(self.lib.psift_ctx_enable_stage_timing(self.handle, int(on)))

    TUNE_BLUR, TUNE_MATCH_FP32, TUNE_MATCH_TC = 0, 1, 2
    # level-blur variants: 0-2 outputs per thread (4x8, 8x8, 4x4), 3 TMA tiles (persistent CTAs),
    # 4 128-row tiles of 512 threads
    BLUR_VARIANTS = 5

    def autotune(self, height: int, width: int, n_images: int, config: "SiftConfig" = None, n_desc: int = 4096,
                 n_pairs: int = 8) -> dict:
        """Times the candidate tile shapes (level-blur outputs per thread per radius,
        matcher work items per SM) on synthetic inputs of this geometry and keeps the
        fastest; returns {"blur": {radius: {"ms": [...], "variant": v}},
        "match_fp32" / "match_tc": {"ms": {items: ms}, "per_sm": m}}."""
        config = config or SiftConfig()
        c = config.to_c()
        rep = np.zeros(1024, np.float64)
        cnt = C.c_uint32()
        self.check(self.lib.psift_ctx_autotune(self.handle, height, width, n_images, C.byref(c), n_desc, n_pairs,
                                               rep.ctypes.data, len(rep), C.byref(cnt)))
        r = rep[:cnt.value].tolist()
        out = {"blur": {}}
        i = 0
        nv = self.BLUR_VARIANTS
        while i < len(r) and r[i] != -1.0:
            out["blur"][int(r[i])] = {"ms": r[i + 1:i + 1 + nv], "variant": int(r[i + 1 + nv])}
            i += 2 + nv
        i += 1
        while i + 6 <= len(r):
            key = "match_tc" if r[i] == 1.0 else "match_fp32"
            out[key] = {"ms": dict(zip((1, 2, 4, 8), r[i + 1:i + 5])), "per_sm": int(r[i + 5])}
            i += 6
        return out

    def tuning(self) -> dict:
        v = C.c_int32()
        blur = {}
        for rr in range(1, 16):
            self.check(self.lib.psift_ctx_tuning_get(self.handle, self.TUNE_BLUR, rr, C.byref(v)))
            blur[rr] = v.value
        self.check(self.lib.psift_ctx_tuning_get(self.handle, self.TUNE_MATCH_FP32, 0, C.byref(v)))
        fp32 = v.value
        self.check(self.lib.psift_ctx_tuning_get(self.handle, self.TUNE_MATCH_TC, 0, C.byref(v)))
        return {"blur": blur, "match_fp32_per_sm": fp32, "match_tc_per_sm": v.value}

    def set_tuning(self, what: int, index: int, value: int):
        self.check(self.lib.psift_ctx_tuning_set(self.handle, what, index, value))

    BLUR_REFERENCE, BLUR_FUSED = 0, 1

    def set_blur_rounding(self, mode: int):
        """BLUR_REFERENCE (default): the reference's two roundings per blur tap,
        bit-equal results.  BLUR_FUSED: one fused multiply-add per tap (faster; held
        to the f32 path's tolerances against an f64 run, not bit-equal)."""
        self.check(self.lib.psift_ctx_set_blur_rounding(self.handle, int(mode)))

    def stage_times(self, reset: bool = True) -> dict:
        """{stage: (total_ms, intervals)} accumulated since the last reset."""
        ms = np.zeros(16, np.float64)
        cnt = np.zeros(16, np.uint64)
        self.check(self.lib.psift_ctx_stage_times(self.handle, ms.ctypes.data, cnt.ctypes.data, 16, int(reset)))
        return {name: (float(ms[i]), int(cnt[i])) for i, name in enumerate(self.STAGES)}


class _PinnedBlock:
    """Page-locked host allocation (psift_host_alloc), freed with the last array using it."""

    def __init__(self, ctx: Context, nbytes: int):
        self.ctx = ctx
        p = C.c_void_p()
        ctx.check(ctx.lib.psift_host_alloc(ctx.handle, nbytes, C.byref(p)))
        self.ptr = int(p.value)
        self.__array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (self.ptr, False), "version": 3}

    def __del__(self):
        if getattr(self, "ptr", 0) and getattr(self.ctx, "handle", None):
            self.ctx.lib.psift_host_free(self.ctx.handle, C.c_void_p(self.ptr))
            self.ptr = 0


def pinned_empty(shape, dtype, ctx: Context | None = None) -> np.ndarray:
    """An uninitialised numpy array in page-locked host memory."""
    ctx = ctx or default_context()
    dtype = np.dtype(dtype)
    shape = tuple(shape) if isinstance(shape, (tuple, list)) else (int(shape),)
    nbytes = int(np.prod(shape)) * dtype.itemsize
    raw = np.asarray(_PinnedBlock(ctx, max(nbytes, 1)))
    return raw[:nbytes].view(dtype).reshape(shape)


_tls = threading.local()


def default_context() -> Context:
    ctx = getattr(_tls, "ctx", None)
    if ctx is None:
        ctx = Context(int(os.environ.get("PSIFT_DEVICE", "0")))
        _tls.ctx = ctx
    return ctx


@dataclass(frozen=True)
class SiftConfig:
    """``SiftConfig`` (src/pipeline.rs:22-104) with the builder methods."""
    octaves: int = 3
    scales: int = 3
    contrast_threshold: float = DEFAULT_CONTRAST_THRESHOLD
    upsample_first_octave_: bool = True
    descriptor_kind_: int = 0  # 0 = Sift, 1 = RootSift
    max_features_: int = MAX_FEATURES_PER_IMAGE

    @staticmethod
    def default() -> "SiftConfig":
        return SiftConfig()

    def with_octaves(self, n): return replace(self, octaves=n)
    def with_scales(self, n): return replace(self, scales=n)
    def with_contrast_threshold(self, t): return replace(self, contrast_threshold=t)
    def upsample_first_octave(self, up): return replace(self, upsample_first_octave_=bool(up))
    def descriptor_kind(self, kind): return replace(self, descriptor_kind_=int(kind))
    def max_features(self, n): return replace(self, max_features_=int(n))

    def to_c(self) -> CSiftConfig:
        return CSiftConfig(self.octaves, self.scales, self.contrast_threshold, int(self.upsample_first_octave_),
                           self.descriptor_kind_, self.max_features_)

    def validate(self):
        """Returns None when valid, else raises ValueError with the reference's message."""
        lib = load_library()
        buf = C.create_string_buffer(256)
        c = self.to_c()
        st = lib.psift_sift_config_validate(C.byref(c), buf, 256)
        if st != PSIFT_OK:
            raise ValueError(buf.value.decode())


@dataclass
class Features:
    """Structure-of-arrays ``Vec<SiftFeature>``."""
    x: np.ndarray
    y: np.ndarray
    scale: np.ndarray
    response: np.ndarray
    orientation: np.ndarray
    descriptors: np.ndarray  # (n, 128)

    def __len__(self):
        return int(self.x.shape[0])

    @property
    def xy(self) -> np.ndarray:
        return np.stack([self.x, self.y], axis=1)

    @staticmethod
    def empty(n: int) -> "Features":
        return Features(*(np.zeros(n, np.float32) for _ in range(5)), np.zeros((n, 128), np.float32))

    @staticmethod
    def uninitialized(n: int) -> "Features":
        """Capacity-n output arrays without a zero fill (the library writes them)."""
        return Features(*(np.empty(n, np.float32) for _ in range(5)), np.empty((n, 128), np.float32))

    @staticmethod
    def pinned(n: int, ctx: "Context | None" = None) -> "Features":
        """Capacity-n feature arrays in one page-locked block (direct device->host copies)."""
        blk = pinned_empty(((5 + 128) * max(n, 1),), np.float32, ctx)
        cols = [blk[i * n:(i + 1) * n] for i in range(5)]
        return Features(*cols, blk[5 * n:5 * n + 128 * n].reshape(n, 128))

    def view(self, n: int) -> "Features":
        """The first n features, without copying."""
        return Features(self.x[:n], self.y[:n], self.scale[:n], self.response[:n], self.orientation[:n],
                        self.descriptors[:n])

    def head(self, n: int) -> "Features":
        return Features(self.x[:n].copy(), self.y[:n].copy(), self.scale[:n].copy(), self.response[:n].copy(),
                        self.orientation[:n].copy(), self.descriptors[:n].copy())


def _c_features(f: Features) -> CFeatures:
    return CFeatures(len(f), 0, f.x.ctypes.data, f.y.ctypes.data, f.scale.ctypes.data, f.response.ctypes.data,
                     f.orientation.ctypes.data, f.descriptors.ctypes.data)


@dataclass(frozen=True)
class Sift:
    """``Sift`` (src/pipeline.rs:106-146)."""
    config: SiftConfig = field(default_factory=SiftConfig)

    @staticmethod
    def new(config: SiftConfig) -> "Sift":
        config.validate()
        return Sift(config)

    def _run(self, img: np.ndarray, u8: bool, ctx: Context | None) -> Features:
        ctx = ctx or default_context()
        dt = np.uint8 if u8 else np.float32
        img = np.ascontiguousarray(img, dtype=dt)
        if img.ndim != 2:
            raise ValueError("image must be 2-D (H, W)")
        h, w = img.shape
        cfg = self.config.to_c()
        cap = self.config.max_features_ or 16384
        fn = ctx.lib.psift_detect_and_compute_u8 if u8 else ctx.lib.psift_detect_and_compute
        while True:
            out = Features.uninitialized(cap)
            cf = _c_features(out)
            st = fn(ctx.handle, img.ctypes.data, h, w, w, C.byref(cfg), C.byref(cf))
            if st == PSIFT_ERR_CAPACITY and cf.count > cap:
                cap = int(cf.count)
                continue
            ctx.check(st)
            n = int(cf.count)
            # views when most of the block is used, else compact copies
            return out.view(n) if 2 * n >= cap else out.head(n)

    def detect_and_compute(self, img: np.ndarray, ctx: Context | None = None) -> Features:
        return self._run(img, False, ctx)

    def detect_and_compute_batch_u8(self, images, outs: "list[Features] | None" = None,
                                    ctx: Context | None = None) -> "list[Features]":
        """Many u8 images in one call (psift_detect_and_compute_u8_batch): one launch
        per stage for the batch, transfers overlapped with kernels.  Per image the
        result equals ``detect_and_compute_u8``.  Returns views into ``outs``
        (allocated here when not given; ``Features.pinned`` outputs and
        ``pinned_empty`` images are transferred without staging copies)."""
        ctx = ctx or default_context()
        imgs = [np.ascontiguousarray(im, dtype=np.uint8) for im in images]
        if any(im.ndim != 2 for im in imgs):
            raise ValueError("images must be 2-D (H, W)")
        n = len(imgs)
        if n == 0:
            return []
        cfg = self.config.to_c()
        cap = self.config.max_features_ or 16384
        outs = list(outs) if outs is not None else [Features.empty(cap) for _ in range(n)]
        cimgs = (CImageU8 * n)(*[CImageU8(im.ctypes.data, im.shape[0], im.shape[1], im.strides[0]) for im in imgs])
        while True:
            couts = (CFeatures * n)(*[_c_features(o) for o in outs])
            st = ctx.lib.psift_detect_and_compute_u8_batch(ctx.handle, cimgs, n, C.byref(cfg), couts)
            short = [i for i in range(n) if couts[i].count > len(outs[i])]
            if st == PSIFT_ERR_CAPACITY and short:
                for i in short:
                    outs[i] = Features.empty(int(couts[i].count))
                continue
            ctx.check(st)
            return [outs[i].view(int(couts[i].count)) for i in range(n)]

    def _bytes_batch(self, fn_name, blobs, enforce_pixel_cap, outs, ctx):
        ctx = ctx or default_context()
        bufs = [bytes(b) for b in blobs]
        n = len(bufs)
        if n == 0:
            return []
        ptrs = (C.c_char_p * n)(*bufs)
        lens = (C.c_size_t * n)(*[len(b) for b in bufs])
        cfg = self.config.to_c()
        cap = self.config.max_features_ or 16384
        outs = list(outs) if outs is not None else [Features.empty(cap) for _ in range(n)]
        fn = getattr(ctx.lib, fn_name)
        while True:
            couts = (CFeatures * n)(*[_c_features(o) for o in outs])
            st = fn(ctx.handle, ptrs, lens, n, int(bool(enforce_pixel_cap)), C.byref(cfg), couts)
            short = [i for i in range(n) if couts[i].count > len(outs[i])]
            if st == PSIFT_ERR_CAPACITY and short:
                for i in short:
                    outs[i] = Features.empty(int(couts[i].count))
                continue
            ctx.check(st)
            return [outs[i].view(int(couts[i].count)) for i in range(n)]

    def detect_and_compute_jpeg_batch(self, blobs, enforce_pixel_cap: bool = False, outs=None,
                                      ctx: Context | None = None) -> "list[Features]":
        """JPEG bytes -> features (psift_detect_and_compute_jpeg_batch): decoded on the
        GPU into the batch's inputs (decode_validated_luma8, src/cli.rs:164-170), then
        as ``detect_and_compute_batch_u8``."""
        return self._bytes_batch("psift_detect_and_compute_jpeg_batch", blobs, enforce_pixel_cap, outs, ctx)

    def detect_and_compute_png_batch(self, blobs, enforce_pixel_cap: bool = False, outs=None,
                                     ctx: Context | None = None) -> "list[Features]":
        """PNG bytes -> features (psift_detect_and_compute_png_batch): inflated on host
        threads, unfiltered and converted to luma on the GPU into the batch's inputs."""
        return self._bytes_batch("psift_detect_and_compute_png_batch", blobs, enforce_pixel_cap, outs, ctx)

    def detect_and_compute_image_batch(self, blobs, enforce_pixel_cap: bool = False, outs=None,
                                       ctx: Context | None = None) -> "list[Features]":
        """JPEG or PNG bytes (told apart by their leading bytes) -> features, in order
        (``run_extract_from_bytes``, src/cli.rs:173-185, for a batch)."""
        return self._bytes_batch("psift_detect_and_compute_image_batch", blobs, enforce_pixel_cap, outs, ctx)

    def detect_and_compute_u8(self, img: np.ndarray, ctx: Context | None = None) -> Features:
        return self._run(img, True, ctx)

    def detect_keypoints(self, img: np.ndarray, ctx: Context | None = None) -> np.ndarray:
        ctx = ctx or default_context()
        img = np.ascontiguousarray(img, dtype=np.float32)
        h, w = img.shape
        cfg = self.config.to_c()
        cap = 1 << 16
        while True:
            out = np.zeros(cap, KEYPOINT_DTYPE)
            n = C.c_uint32()
            st = ctx.lib.psift_detect_keypoints(ctx.handle, img.ctypes.data, h, w, w, C.byref(cfg), out.ctypes.data,
                                                cap, C.byref(n))
            if st == PSIFT_ERR_CAPACITY and n.value > cap:
                cap = n.value
                continue
            ctx.check(st)
            return out[:n.value].copy()


@dataclass(frozen=True)
class MatchOptions:
    """``MatchOptions`` (src/pipeline.rs:1721-1736) plus the arithmetic path.

    ``precision=PRECISION_BF16_RERANK`` (default) computes distances on the
    tensor cores in bf16 and re-ranks every query's candidates in exact f32; the
    match list is identical to ``PRECISION_FP32``.
    """
    ratio: float = DEFAULT_MATCH_RATIO
    mutual: bool = False
    precision: int = PRECISION_BF16_RERANK

    def to_c(self) -> CMatchOptions:
        return CMatchOptions(self.ratio, int(self.mutual), int(self.precision))


@dataclass(frozen=True)
class Matcher:
    """``Matcher`` (src/pipeline.rs:148-170)."""
    options: MatchOptions = field(default_factory=MatchOptions)

    @staticmethod
    def new(options: MatchOptions) -> "Matcher":
        lib = load_library()
        buf = C.create_string_buffer(256)
        c = options.to_c()
        if lib.psift_match_options_validate(C.byref(c), buf, 256) != PSIFT_OK:
            raise ValueError(buf.value.decode())
        return Matcher(options)

    def match_(self, query: Features, target: Features, ctx: Context | None = None) -> np.ndarray:
        return match_arrays(query.descriptors, target.descriptors, query.xy, target.xy, self.options, ctx)


def match_arrays(q_desc, t_desc, q_xy, t_xy, options: MatchOptions = MatchOptions(), ctx: Context | None = None):
    """Matches raw arrays (n x 128 descriptors, n x 2 coordinates); returns MATCH_DTYPE records."""
    ctx = ctx or default_context()
    qd = np.ascontiguousarray(q_desc, dtype=np.float32).reshape(-1, 128)
    td = np.ascontiguousarray(t_desc, dtype=np.float32).reshape(-1, 128)
    qxy = np.ascontiguousarray(q_xy, dtype=np.float32).reshape(-1, 2)
    txy = np.ascontiguousarray(t_xy, dtype=np.float32).reshape(-1, 2)
    nq, nt = qd.shape[0], td.shape[0]
    out = np.zeros(max(nq, 1), MATCH_DTYPE)
    n = C.c_uint32()
    c = options.to_c()
    ctx.check(ctx.lib.psift_match_descriptors(ctx.handle, qd.ctypes.data, nq, td.ctypes.data, nt, qxy.ctypes.data,
                                              txy.ctypes.data, C.byref(c), out.ctypes.data, out.shape[0],
                                              C.byref(n)))
    return out[:n.value].copy()


def match_descriptors(query: Features, target: Features, ratio_threshold: float, ctx: Context | None = None):
    """``match_descriptors`` (src/pipeline.rs:1845-1858)."""
    return Matcher.new(MatchOptions(ratio=ratio_threshold)).match_(query, target, ctx)


# ---------------------------------------------------------------- JPEG input
def jpeg_info(blob: bytes, enforce_pixel_cap: bool = False, ctx: Context | None = None):
    """(width, height, components) of a JPEG, with the reference's size checks."""
    ctx = ctx or default_context()
    w, h, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
    ctx.check(ctx.lib.psift_jpeg_info(ctx.handle, blob, len(blob), int(bool(enforce_pixel_cap)), C.byref(w),
                                      C.byref(h), C.byref(c)))
    return int(w.value), int(h.value), int(c.value)


def decode_jpeg_luma(blob: bytes, enforce_pixel_cap: bool = False, ctx: Context | None = None) -> np.ndarray:
    """``decode_validated_luma8`` (src/cli.rs:164-170) for a JPEG, decoded on the GPU."""
    ctx = ctx or default_context()
    w, h, _ = jpeg_info(blob, enforce_pixel_cap, ctx)
    out = np.zeros((h, w), np.uint8)
    ww, hh = C.c_uint32(), C.c_uint32()
    ctx.check(ctx.lib.psift_decode_jpeg_luma(ctx.handle, blob, len(blob), int(bool(enforce_pixel_cap)),
                                             out.ctypes.data, out.size, C.byref(ww), C.byref(hh)))
    return out


# ---------------------------------------------------------------- PNG input
def png_info(blob: bytes, enforce_pixel_cap: bool = False, ctx: Context | None = None):
    """(width, height, channels) of a PNG, with the reference's size checks."""
    ctx = ctx or default_context()
    w, h, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
    ctx.check(ctx.lib.psift_png_info(ctx.handle, blob, len(blob), int(bool(enforce_pixel_cap)), C.byref(w),
                                     C.byref(h), C.byref(c)))
    return int(w.value), int(h.value), int(c.value)


def decode_png_luma(blob: bytes, enforce_pixel_cap: bool = False, ctx: Context | None = None) -> np.ndarray:
    """``decode_validated_luma8`` (src/cli.rs:164-170) for a PNG: inflated on the host,
    row filters and the luma conversion on the GPU."""
    ctx = ctx or default_context()
    w, h, _ = png_info(blob, enforce_pixel_cap, ctx)
    out = np.zeros((h, w), np.uint8)
    ww, hh = C.c_uint32(), C.c_uint32()
    ctx.check(ctx.lib.psift_decode_png_luma(ctx.handle, blob, len(blob), int(bool(enforce_pixel_cap)),
                                            out.ctypes.data, out.size, C.byref(ww), C.byref(hh)))
    return out


def decode_image_luma(blob: bytes, enforce_pixel_cap: bool = False, ctx: Context | None = None) -> np.ndarray:
    """``decode_validated_luma8`` for either supported format (PNG signature, else JPEG)."""
    if bytes(blob[:8]) == b"\x89PNG\r\n\x1a\n":
        return decode_png_luma(blob, enforce_pixel_cap, ctx)
    return decode_jpeg_luma(blob, enforce_pixel_cap, ctx)


# ---------------------------------------------------------------- catalog codes
def quantize_descriptor_u128(desc, ctx: Context | None = None) -> np.ndarray:
    """``quantize_descriptor_u128`` (src/catalog.rs:37-45) for n descriptors -> (n, 2) u64 (lo, hi)."""
    ctx = ctx or default_context()
    d = np.ascontiguousarray(desc, dtype=np.float32).reshape(-1, 128)
    out = np.zeros((d.shape[0], 2), np.uint64)
    ctx.check(ctx.lib.psift_quantize_u128(ctx.handle, d.ctypes.data, d.shape[0], out.ctypes.data))
    return out


def quantize_descriptor_u8(desc, ctx: Context | None = None) -> np.ndarray:
    """``quantize_descriptor_u8`` (src/pipeline.rs:1024-1030)."""
    ctx = ctx or default_context()
    d = np.ascontiguousarray(desc, dtype=np.float32).reshape(-1, 128)
    out = np.zeros(d.shape, np.uint8)
    ctx.check(ctx.lib.psift_quantize_u8(ctx.handle, d.ctypes.data, d.shape[0], out.ctypes.data))
    return out


def dequantize_descriptor_u8(q, ctx: Context | None = None) -> np.ndarray:
    """``dequantize_descriptor_u8`` (src/pipeline.rs:1034-1044)."""
    ctx = ctx or default_context()
    qq = np.ascontiguousarray(q, dtype=np.uint8).reshape(-1, 128)
    out = np.zeros(qq.shape, np.float32)
    ctx.check(ctx.lib.psift_dequantize_u8(ctx.handle, qq.ctypes.data, qq.shape[0], out.ctypes.data))
    return out


def hamming_votes(query_codes, catalog_codes, entry_offsets, mih: bool, ctx: Context | None = None) -> np.ndarray:
    """Coarse votes per catalog entry (src/catalog.rs:596-633 MIH, :707-728 exhaustive)."""
    ctx = ctx or default_context()
    q = np.ascontiguousarray(query_codes, dtype=np.uint64).reshape(-1, 2)
    c = np.ascontiguousarray(catalog_codes, dtype=np.uint64).reshape(-1, 2)
    off = np.ascontiguousarray(entry_offsets, dtype=np.int64)
    votes = np.zeros(len(off) - 1, np.uint32)
    ctx.check(ctx.lib.psift_hamming_votes(ctx.handle, q.ctypes.data, q.shape[0], c.ctypes.data, off.ctypes.data,
                                          len(off) - 1, int(bool(mih)), votes.ctypes.data))
    return votes


def hamming_topk(query_codes, catalog_codes, k: int, ctx: Context | None = None):
    """Per query, the k nearest codes by (Hamming distance, index) -> (idx, dist) (nq, k) u32."""
    ctx = ctx or default_context()
    q = np.ascontiguousarray(query_codes, dtype=np.uint64).reshape(-1, 2)
    c = np.ascontiguousarray(catalog_codes, dtype=np.uint64).reshape(-1, 2)
    idx = np.zeros((q.shape[0], k), np.uint32)
    dist = np.zeros((q.shape[0], k), np.uint32)
    ctx.check(ctx.lib.psift_hamming_topk(ctx.handle, q.ctypes.data, q.shape[0], c.ctypes.data, c.shape[0], k,
                                         idx.ctypes.data, dist.ctypes.data))
    return idx, dist


def l2_rerank(query_desc, catalog_desc, candidates, ctx: Context | None = None):
    """Exact f32 L2^2 of each query to its candidates, sorted by (d2, index) -> (idx, d2)."""
    ctx = ctx or default_context()
    qd = np.ascontiguousarray(query_desc, dtype=np.float32).reshape(-1, 128)
    cd = np.ascontiguousarray(catalog_desc, dtype=np.float32).reshape(-1, 128)
    cand = np.ascontiguousarray(candidates, dtype=np.uint32)
    k = cand.shape[1]
    idx = np.zeros_like(cand)
    d2 = np.zeros(cand.shape, np.float32)
    ctx.check(ctx.lib.psift_l2_rerank(ctx.handle, qd.ctypes.data, qd.shape[0], cd.ctypes.data, cd.shape[0],
                                      cand.ctypes.data, k, idx.ctypes.data, d2.ctypes.data))
    return idx, d2


# ---------------------------------------------------------------- RANSAC
@dataclass(frozen=True)
class RansacOptions:
    """``RansacOptions`` (src/pipeline.rs:177-218)."""
    reproj_threshold: float = DEFAULT_RANSAC_REPROJ_THRESHOLD
    seed: int | None = None

    def to_c(self) -> CRansacOptions:
        return CRansacOptions(self.reproj_threshold, 0 if self.seed is None else 1,
                              0 if self.seed is None else (self.seed & 0xFFFFFFFFFFFFFFFF))

    def validate(self):
        lib = load_library()
        buf = C.create_string_buffer(256)
        c = self.to_c()
        if lib.psift_ransac_options_validate(C.byref(c), buf, 256) != PSIFT_OK:
            raise ValueError(buf.value.decode())


def _as_matches(matches) -> np.ndarray:
    m = np.asarray(matches)
    if m.dtype != MATCH_DTYPE:
        m = m.astype(MATCH_DTYPE) if m.dtype.names is None else np.array(
            [tuple(r) for r in m], dtype=MATCH_DTYPE)
    return np.ascontiguousarray(m)


class Homography:
    """``Homography`` (src/pipeline.rs:220-247): returns (inlier matches, model or None)."""

    @staticmethod
    def estimate(matches, options: RansacOptions = RansacOptions(), ctx: Context | None = None):
        ctx = ctx or default_context()
        m = _as_matches(matches)
        n = len(m)
        mask = np.zeros(max(n, 1), np.uint8)
        h9 = np.zeros(9, np.float32)
        has = C.c_int32()
        cnt = C.c_uint32()
        c = options.to_c()
        ctx.check(ctx.lib.psift_homography_estimate(ctx.handle, m.ctypes.data, n, C.byref(c), mask.ctypes.data,
                                                    h9.ctypes.data, C.byref(has), C.byref(cnt)))
        sel = mask[:n].astype(bool)
        return m[sel], (h9.reshape(3, 3) if has.value else None)

    @staticmethod
    def estimate_similarity(matches, options: RansacOptions = RansacOptions(), ctx: Context | None = None):
        """Returns (inlier matches, (a, b, tx, ty, scale, rotation_deg) or None)."""
        ctx = ctx or default_context()
        m = _as_matches(matches)
        n = len(m)
        mask = np.zeros(max(n, 1), np.uint8)
        m6 = np.zeros(9, np.float32)
        has = C.c_int32()
        cnt = C.c_uint32()
        c = options.to_c()
        ctx.check(ctx.lib.psift_similarity_estimate(ctx.handle, m.ctypes.data, n, C.byref(c), mask.ctypes.data,
                                                    m6.ctypes.data, C.byref(has), C.byref(cnt)))
        sel = mask[:n].astype(bool)
        return m[sel], (m6[:6].copy() if has.value else None)


def estimate_homography_ransac(matches, reproj_threshold: float, ctx: Context | None = None):
    """``estimate_homography_ransac`` (src/pipeline.rs:2635-2646)."""
    return Homography.estimate(matches, RansacOptions(reproj_threshold), ctx)


def filter_matches_ransac(matches, reproj_threshold: float, ctx: Context | None = None):
    """``filter_matches_ransac`` (src/pipeline.rs:2038-2044)."""
    return Homography.estimate_similarity(matches, RansacOptions(reproj_threshold), ctx)


# ---------------------------------------------------------------- learned sampler
MLP_NUM_PARAMS = 4801
MLP_NUM_FEATURES = 8


class InlierMLP:
    """The learned correspondence scorer (8-64-64-1, bf16 operands, f32 accumulation)."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0):
        if params is None:
            params = np.zeros(MLP_NUM_PARAMS, np.float32)
            load_library().psift_mlp_init(seed, params.ctypes.data)
        self.params = np.ascontiguousarray(params, dtype=np.float32).copy()

    def predict(self, features, ctx: Context | None = None) -> np.ndarray:
        ctx = ctx or default_context()
        x = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, MLP_NUM_FEATURES)
        out = np.zeros(x.shape[0], np.float32)
        ctx.check(ctx.lib.psift_mlp_infer(ctx.handle, self.params.ctypes.data, x.ctypes.data, x.shape[0],
                                          out.ctypes.data))
        return out

    def gradients(self, features, labels, ctx: Context | None = None):
        ctx = ctx or default_context()
        x = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, MLP_NUM_FEATURES)
        y = np.ascontiguousarray(labels, dtype=np.float32)
        g = np.zeros(MLP_NUM_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        ctx.check(ctx.lib.psift_mlp_gradients(ctx.handle, self.params.ctypes.data, x.ctypes.data, y.ctypes.data,
                                              x.shape[0], g.ctypes.data, loss.ctypes.data))
        return float(loss[0]), g

    def train(self, features, labels, steps=300, batch=4096, lr=3e-3, seed=1, ctx: Context | None = None):
        ctx = ctx or default_context()
        x = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, MLP_NUM_FEATURES)
        y = np.ascontiguousarray(labels, dtype=np.float32)
        losses = np.zeros(steps, np.float32)
        ctx.check(ctx.lib.psift_mlp_train(ctx.handle, self.params.ctypes.data, x.ctypes.data, y.ctypes.data,
                                          x.shape[0], steps, batch, lr, seed, losses.ctypes.data))
        return losses


def ransac_jobs(match_sets, weights=None):
    """Device-resident RANSAC jobs for psift_ransac_batch_dev (torch buffers)."""
    import torch
    dev = []
    jobs = (CRansacJob * len(match_sets))()
    for i, m in enumerate(match_sets):
        m = _as_matches(m)
        n = len(m)
        d_m = torch.from_numpy(m.view(np.uint8).copy()).cuda() if n else torch.zeros(40, dtype=torch.uint8,
                                                                                       device="cuda")
        mask = torch.zeros(max(n, 1), dtype=torch.uint8, device="cuda")
        out = torch.zeros(16, dtype=torch.int32, device="cuda")
        w = None
        if weights is not None:
            w = torch.from_numpy(np.ascontiguousarray(weights[i], dtype=np.float32)).cuda()
        dev.append((d_m, mask, out, w, n))
        # out (int32): [0] inlier count, [1] has model, [2] similarity iterations,
        # [3] homography iterations, [4..13) model floats
        jobs[i] = CRansacJob(d_m.data_ptr(), n, mask.data_ptr(), out.data_ptr() + 16, out.data_ptr() + 4,
                             out.data_ptr(), w.data_ptr() if w is not None else None, out.data_ptr() + 8)
    return jobs, dev


def ransac_results(dev, homography: bool = True):
    res = []
    for d_m, mask, out, w, n in dev:
        o = out.cpu().numpy()
        model = o[4:4 + (9 if homography else 6)].view(np.float32).copy()
        res.append((mask[:n].cpu().numpy().astype(bool), model if o[1] else None, (int(o[2]), int(o[3]))))
    return res


def ransac_batch(match_sets, options: RansacOptions = RansacOptions(), homography: bool = True,
                 weights=None, ctx: Context | None = None):
    """Runs many estimations in one launch (device-resident); returns
    [(inlier mask, model or None, (similarity iters, homography iters))]."""
    ctx = ctx or default_context()
    jobs, dev = ransac_jobs(match_sets, weights)
    c = options.to_c()
    ctx.check(ctx.lib.psift_ransac_batch_dev(ctx.handle, jobs, len(match_sets), C.byref(c), int(homography)))
    ctx.synchronize()
    return ransac_results(dev, homography)


@dataclass(frozen=True)
class FundamentalRansacOptions:
    """``FundamentalRansacOptions`` (src/geometry.rs:107-143)."""
    sampson_threshold: float = 1.5
    max_iters: int = 2000
    confidence: float = 0.999
    seed: int = 0xF00DCAFE12345678

    def to_c(self) -> CFundamentalOptions:
        return CFundamentalOptions(self.sampson_threshold, self.max_iters, self.confidence,
                                   self.seed & 0xFFFFFFFFFFFFFFFF)


def estimate_fundamental_ransac_with_options(matches, options: FundamentalRansacOptions = FundamentalRansacOptions(),
                                             ctx: Context | None = None):
    """``estimate_fundamental_ransac_with_options`` (src/geometry.rs:868-1016):
    (inlier matches, F (3, 3) f64 or None)."""
    ctx = ctx or default_context()
    m = _as_matches(matches)
    n = len(m)
    mask = np.zeros(max(n, 1), np.uint8)
    f9 = np.zeros(9, np.float64)
    has, cnt, it = C.c_int32(), C.c_uint32(), C.c_uint32()
    c = options.to_c()
    ctx.check(ctx.lib.psift_fundamental_estimate(ctx.handle, m.ctypes.data, n, C.byref(c), mask.ctypes.data,
                                                 f9.ctypes.data, C.byref(has), C.byref(cnt), C.byref(it)))
    return m[mask[:n].astype(bool)], (f9.reshape(3, 3) if has.value else None)


def estimate_fundamental_ransac(matches, sampson_threshold: float = 1.5, ctx: Context | None = None):
    """``estimate_fundamental_ransac`` (src/geometry.rs:857-866)."""
    return estimate_fundamental_ransac_with_options(matches, FundamentalRansacOptions(sampson_threshold), ctx)


def fundamental_batch(match_sets, options: FundamentalRansacOptions = FundamentalRansacOptions(),
                      ctx: Context | None = None, timing: bool = False):
    """Many fundamental-matrix estimations in one launch (device-resident); returns
    [(inlier mask, F or None, iterations)] and, with timing, the device ms."""
    import torch
    ctx = ctx or default_context()
    sizes = [len(m) for m in match_sets]
    allm = np.concatenate([_as_matches(m) for m in match_sets]) if sizes else np.zeros(0, MATCH_DTYPE)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    d_m = torch.from_numpy(allm.view(np.uint8)).cuda()
    d_mask = torch.zeros(max(int(off[-1]), 1), dtype=torch.uint8, device="cuda")
    d_f = torch.zeros((max(len(sizes), 1), 9), dtype=torch.float64, device="cuda")
    d_i = torch.zeros((max(len(sizes), 1), 4), dtype=torch.int32, device="cuda")  # has, count, iters
    jobs = (CFundamentalJob * max(len(sizes), 1))()
    rec = allm.dtype.itemsize
    for k, n in enumerate(sizes):
        jobs[k] = CFundamentalJob(d_m.data_ptr() + int(off[k]) * rec, n, d_mask.data_ptr() + int(off[k]),
                                  d_f.data_ptr() + 72 * k, d_i.data_ptr() + 16 * k, d_i.data_ptr() + 16 * k + 4,
                                  d_i.data_ptr() + 16 * k + 8)
    c = options.to_c()
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.check(ctx.lib.psift_fundamental_batch_dev(ctx.handle, jobs, len(sizes), C.byref(c)))
    e1.record(stream)
    ctx.synchronize()
    masks = d_mask.cpu().numpy().astype(bool)
    fs = d_f.cpu().numpy()
    info = d_i.cpu().numpy()
    out = [(masks[off[k]:off[k + 1]], fs[k].reshape(3, 3) if info[k, 0] else None, int(info[k, 2]))
           for k in range(len(sizes))]
    return (out, e0.elapsed_time(e1)) if timing else out


def compute_sift_descriptors(img: np.ndarray, keypoints, kind: int = 0, ctx: Context | None = None) -> Features:
    """``compute_sift_descriptors_with_kind`` (src/pipeline.rs:1585-1629): descriptors
    for given keypoints; the pyramid is rebuilt from what the keypoints imply."""
    ctx = ctx or default_context()
    img = np.ascontiguousarray(img, dtype=np.float32)
    kps = np.ascontiguousarray(keypoints, dtype=KEYPOINT_DTYPE)
    h, w = img.shape
    cap = max(4 * len(kps), 1)
    out = Features.empty(cap)
    cf = _c_features(out)
    ctx.check(ctx.lib.psift_compute_descriptors(ctx.handle, img.ctypes.data, h, w, w, kps.ctypes.data, len(kps),
                                                int(kind), C.byref(cf)))
    return out.head(int(cf.count))


@dataclass
class TrackingSummary:
    """``TrackingSummary`` (src/pipeline.rs:1137-1152)."""
    raw_match_count: int
    match_count: int
    inlier_ratio: float
    mean_displacement: tuple
    median_displacement: tuple
    mean_scale_ratio: float
    mean_rotation_deg: float


def summarize_tracking(query: Features, target: Features, matches, ctx: Context | None = None) -> TrackingSummary:
    """``summarize_tracking`` (src/pipeline.rs:2210-2272)."""
    ctx = ctx or default_context()
    m = _as_matches(matches)
    out = CTracking()
    ctx.check(ctx.lib.psift_summarize_tracking(ctx.handle, m.ctypes.data, len(m), query.scale.ctypes.data,
                                               query.orientation.ctypes.data, len(query), target.scale.ctypes.data,
                                               target.orientation.ctypes.data, len(target), C.byref(out)))
    return TrackingSummary(out.raw_match_count, out.match_count, out.inlier_ratio, (out.mean_dx, out.mean_dy),
                           (out.median_dx, out.median_dy), out.mean_scale_ratio, out.mean_rotation_deg)


DEFAULT_CATALOG_SHORTLIST = 16
# Coarse-vote computations of the device catalog (PSIFT_VOTES_*).
VOTES_AUTO, VOTES_MIH_SCAN, VOTES_MIH_INDEX, VOTES_EXHAUSTIVE = 0, 1, 2, 3
DEFAULT_CATALOG_TOP_K = 5


@dataclass
class CatalogEntry:
    """``CatalogEntry`` (src/catalog.rs:110-150)."""
    id: str
    width: int
    height: int
    features: Features
    signatures: np.ndarray  # (n, 2) u64


@dataclass
class CatalogSearchHit:
    """``CatalogSearchHit`` (src/catalog.rs:158-177)."""
    id: str
    width: int
    height: int
    feature_count: int
    coarse_votes: int
    tracking: TrackingSummary
    transform: object
    homography: object


class FeatureCatalog:
    """``FeatureCatalog`` (src/catalog.rs:182-702) with its search on the GPU.

    The index (entries, id lookup) is host data as in the reference; the coarse
    Hamming voting, Lowe matching, similarity / homography RANSAC and the tracking
    summary's RANSAC run through the C ABI.  The multi-index-hashing semantics
    apply above 32 entries, exactly where the reference switches to its tables.
    """

    def __init__(self, octaves: int = 3, scales: int = 3, threshold: float = DEFAULT_CONTRAST_THRESHOLD):
        self.octaves, self.scales, self.threshold = octaves, scales, threshold
        self.entries: list[CatalogEntry] = []
        self._index: dict[str, int] = {}

    def __len__(self):
        return len(self.entries)

    def upsert_entry(self, id: str, width: int, height: int, features: Features, ctx: Context | None = None):
        sig = quantize_descriptor_u128(features.descriptors, ctx) if len(features) else np.zeros((0, 2), np.uint64)
        e = CatalogEntry(id, width, height, features, sig)
        if id in self._index:
            self.entries[self._index[id]] = e
        else:
            self._index[id] = len(self.entries)
            self.entries.append(e)

    def remove(self, id: str) -> bool:
        """``remove`` (src/catalog.rs:343-352): swap_remove then reindex."""
        i = self._index.pop(id, None)
        if i is None:
            return False
        last = self.entries.pop()
        if i < len(self.entries):
            self.entries[i] = last
        self._index = {e.id: k for k, e in enumerate(self.entries)}
        return True

    def coarse_votes(self, query: Features, ctx: Context | None = None):
        qs = quantize_descriptor_u128(query.descriptors, ctx)
        sizes = [len(e.signatures) for e in self.entries]
        off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        cat = np.concatenate([e.signatures for e in self.entries]) if off[-1] else np.zeros((0, 2), np.uint64)
        mih = len(self.entries) > 32
        return hamming_votes(qs, cat, off, mih, ctx), mih

    def search_features(self, query: Features, top_k: int = DEFAULT_CATALOG_TOP_K,
                        shortlist_k: int = DEFAULT_CATALOG_SHORTLIST, ratio_threshold: float = DEFAULT_MATCH_RATIO,
                        ransac_threshold: float = DEFAULT_RANSAC_REPROJ_THRESHOLD,
                        ctx: Context | None = None) -> list:
        """``search_features`` (src/catalog.rs:576-702)."""
        if not self.entries or len(query) == 0 or top_k == 0:
            return []
        votes, mih = self.coarse_votes(query, ctx)
        cands = [(i, int(v)) for i, v in enumerate(votes) if (v > 0 or not mih)]
        if len(cands) > max(shortlist_k, 1):
            cands.sort(key=lambda c: (-c[1], self.entries[c[0]].id))
            cands = cands[:max(shortlist_k, 1)]
        hits = []
        opt = RansacOptions(ransac_threshold)
        for idx, v in cands:
            e = self.entries[idx]
            if len(e.features) < 2:
                continue
            raw = match_descriptors(query, e.features, ratio_threshold, ctx)
            if len(raw) == 0:
                continue
            tracking = summarize_tracking(query, e.features, raw, ctx)
            sim_in, sim_tf = Homography.estimate_similarity(raw, opt, ctx)
            hom_in, hom_tf = Homography.estimate(raw, opt, ctx)
            best = max(len(hom_in), len(sim_in))
            tracking.match_count = best
            if tracking.raw_match_count > 0:
                tracking.inlier_ratio = float(np.float32(best) / np.float32(tracking.raw_match_count))
            hits.append(CatalogSearchHit(e.id, e.width, e.height, len(e.features), v, tracking, sim_tf, hom_tf))
        hits.sort(key=lambda h: (-h.tracking.match_count, -h.tracking.inlier_ratio, -h.coarse_votes, h.id))
        return hits[:top_k]


@dataclass
class CatalogEntrySummary:
    """``CatalogEntrySummary`` (src/catalog.rs:47-58)."""
    id: str
    width: int
    height: int
    feature_count: int


BINARY_CATALOG_MAGIC = b"PSIFTCAT"
_KIND_NAMES = {0: "Sift", 1: "RootSift"}


def _c_features_count(f: Features) -> tuple:
    """CFeatures with count = capacity = len(f), and the contiguous f32 arrays it points into."""
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (f.x, f.y, f.scale, f.response, f.orientation)]
    d = np.ascontiguousarray(f.descriptors, dtype=np.float32).reshape(len(f), 128)
    n = len(f)
    return CFeatures(n, n, *(a.ctypes.data for a in arrs), d.ctypes.data), (arrs, d)


class DeviceCatalog:
    """``FeatureCatalog`` (src/catalog.rs:182-702) resident in device memory.

    Every entry's features, 128-bit codes and the entry table live on the GPU
    (``psift_catalog_*``).  ``search_features`` runs the coarse votes, the
    shortlist's Lowe matching and its similarity / homography RANSAC as batched
    launches; ``load_binary`` / ``save_binary`` move PSIFTCAT v1 files to and from
    device memory.  Entry order, upsert (replace in place or append) and remove
    (swap_remove) follow the reference."""

    def __init__(self, octaves: int = 3, scales: int = 3, threshold: float = DEFAULT_CONTRAST_THRESHOLD,
                 descriptor_kind: int = 0, ctx: Context | None = None, _handle=None):
        self.ctx = ctx or default_context()
        if _handle is None:
            prm = CCatalogParams(octaves, scales, threshold, descriptor_kind)
            _handle = C.c_void_p()
            self.ctx.check(self.ctx.lib.psift_catalog_create(self.ctx.handle, C.byref(prm), C.byref(_handle)))
        self.handle = _handle

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.ctx.lib.psift_catalog_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return int(self.ctx.lib.psift_catalog_size(self.handle))

    @property
    def params(self) -> CCatalogParams:
        p = CCatalogParams()
        self.ctx.check(self.ctx.lib.psift_catalog_params_get(self.handle, C.byref(p)))
        return p

    def entry(self, i: int) -> CatalogEntrySummary:
        lib = self.ctx.lib
        cap = 256
        while True:
            buf = C.create_string_buffer(cap)
            n, w, h, cnt = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint64()
            self.ctx.check(lib.psift_catalog_entry(self.handle, i, buf, cap, C.byref(n), C.byref(w), C.byref(h),
                                                   C.byref(cnt)))
            if n.value < cap:
                return CatalogEntrySummary(buf.raw[:n.value].decode("utf-8"), w.value, h.value, cnt.value)
            cap = n.value + 1

    def list_summaries(self) -> list:
        """``list_summaries`` (src/catalog.rs:355-366)."""
        return [self.entry(i) for i in range(len(self))]

    def index_of(self, id: str) -> int | None:
        i = C.c_uint32()
        st = self.ctx.lib.psift_catalog_find(self.handle, id.encode("utf-8"), C.byref(i))
        return int(i.value) if st == PSIFT_OK else None

    def entry_features(self, i: int):
        """Entry i's features and (n, 2) u64 codes, copied back from the device."""
        n = self.entry(i).feature_count
        f = Features.empty(n)
        codes = np.zeros((max(n, 1), 2), np.uint64)
        cf = CFeatures(n, 0, f.x.ctypes.data, f.y.ctypes.data, f.scale.ctypes.data, f.response.ctypes.data,
                       f.orientation.ctypes.data, f.descriptors.ctypes.data)
        self.ctx.check(self.ctx.lib.psift_catalog_features(self.handle, i, C.byref(cf), codes.ctypes.data))
        return f, codes[:n]

    def upsert_entry(self, id: str, width: int, height: int, features: Features):
        """``upsert_entry`` (src/catalog.rs:324-342)."""
        cf, keep = _c_features_count(features)
        self.ctx.check(self.ctx.lib.psift_catalog_upsert(self.handle, id.encode("utf-8"), width, height,
                                                         C.byref(cf)))
        del keep

    def remove(self, id: str) -> bool:
        """``remove`` (src/catalog.rs:345-353): swap_remove."""
        r = C.c_int32()
        self.ctx.check(self.ctx.lib.psift_catalog_remove(self.handle, id.encode("utf-8"), C.byref(r)))
        return bool(r.value)

    def search_features(self, query: Features, top_k: int = DEFAULT_CATALOG_TOP_K,
                        shortlist_k: int = DEFAULT_CATALOG_SHORTLIST, ratio_threshold: float = DEFAULT_MATCH_RATIO,
                        ransac_threshold: float = DEFAULT_RANSAC_REPROJ_THRESHOLD) -> list:
        """``search_features`` (src/catalog.rs:576-702)."""
        cap = max(int(top_k), 1)
        hits = (CCatalogHit * cap)()
        cnt = C.c_uint32()
        cf, keep = _c_features_count(query)
        self.ctx.check(self.ctx.lib.psift_catalog_search(self.handle, C.byref(cf), top_k, shortlist_k,
                                                         ratio_threshold, ransac_threshold, hits, cap,
                                                         C.byref(cnt)))
        del keep
        out = []
        for k in range(cnt.value):
            h = hits[k]
            e = self.entry(h.entry)
            t = h.tracking
            tr = TrackingSummary(t.raw_match_count, t.match_count, t.inlier_ratio, (t.mean_dx, t.mean_dy),
                                 (t.median_dx, t.median_dy), t.mean_scale_ratio, t.mean_rotation_deg)
            sim = np.array(h.similarity[:], np.float32) if h.has_similarity else None
            hom = np.array(h.homography[:], np.float32).reshape(3, 3) if h.has_homography else None
            out.append(CatalogSearchHit(e.id, e.width, e.height, e.feature_count, h.coarse_votes, tr, sim, hom))
        return out

    def votes(self, query_codes, path: int = 0) -> np.ndarray:
        """Coarse votes of ``search_features`` (src/catalog.rs:588-633) for u128
        query codes ((n, 2) u64) against the resident codes.  path: VOTES_AUTO
        (the search's choice), VOTES_MIH_SCAN, VOTES_MIH_INDEX (the device MIH
        tables, src/catalog.rs:291-321) or VOTES_EXHAUSTIVE."""
        q = np.ascontiguousarray(query_codes, dtype=np.uint64).reshape(-1, 2)
        out = np.zeros(len(self), np.uint32)
        self.ctx.check(self.ctx.lib.psift_catalog_votes(self.handle, q.ctypes.data, q.shape[0], int(path),
                                                        out.ctypes.data))
        return out

    def set_search_votes(self, path: int):
        """Votes computation of ``search_features``: VOTES_AUTO or VOTES_MIH_SCAN."""
        self.ctx.check(self.ctx.lib.psift_catalog_set_search_votes(self.handle, int(path)))

    # ---- persistence (src/catalog.rs:378-574)
    @classmethod
    def load_binary(cls, path: str, ctx: Context | None = None) -> "DeviceCatalog":
        """``load_binary`` (src/catalog.rs:447-540), straight into device memory."""
        ctx = ctx or default_context()
        h = C.c_void_p()
        ctx.check(ctx.lib.psift_catalog_load_binary(ctx.handle, os.fsencode(path), C.byref(h)))
        return cls(ctx=ctx, _handle=h)

    def save_binary(self, path: str):
        """``save_binary`` (src/catalog.rs:401-445), written atomically."""
        self.ctx.check(self.ctx.lib.psift_catalog_save_binary(self.handle, os.fsencode(path)))

    def to_json_obj(self) -> dict:
        p = self.params
        entries = []
        for i in range(len(self)):
            e = self.entry(i)
            f, _ = self.entry_features(i)
            feats = [{"x": float(f.x[j]), "y": float(f.y[j]), "scale": float(f.scale[j]),
                      "response": float(f.response[j]), "orientation": float(f.orientation[j]),
                      "descriptor": [float(v) for v in f.descriptors[j]]} for j in range(len(f))]
            entries.append({"id": e.id, "width": e.width, "height": e.height, "features": feats})
        return {"octaves": int(p.octaves), "scales": int(p.scales), "threshold": float(p.threshold),
                "descriptor_kind": _KIND_NAMES[int(p.descriptor_kind)], "entries": entries}

    def save_json(self, path: str, pretty: bool = False):
        """``save_json`` (src/catalog.rs:378-388): serde field names; temp file + rename."""
        import json
        text = json.dumps(self.to_json_obj(), indent=2 if pretty else None,
                          separators=None if pretty else (",", ":")) + "\n"
        d = os.path.dirname(path)
        if d:
            os.makedirs(d, exist_ok=True)
        tmp = os.path.join(d, f"{os.path.basename(path) or 'catalog'}.tmp.{os.getpid()}")
        with open(tmp, "w") as fh:
            fh.write(text)
        os.replace(tmp, path)

    @classmethod
    def load_json(cls, path: str, ctx: Context | None = None) -> "DeviceCatalog":
        """``load_json`` (src/catalog.rs:390-399): codes recomputed from the descriptors."""
        import json
        with open(path) as fh:
            obj = json.load(fh)
        kind = {"Sift": 0, "RootSift": 1}[obj.get("descriptor_kind", "Sift")]
        cat = cls(int(obj["octaves"]), int(obj["scales"]), float(obj["threshold"]), kind, ctx)
        for e in obj["entries"]:
            fs = e["features"]
            n = len(fs)
            col = lambda k: np.array([f[k] for f in fs], np.float32).reshape(n)
            desc = np.array([f["descriptor"] for f in fs], np.float32).reshape(n, 128) if n else \
                np.zeros((0, 128), np.float32)
            cat.upsert_entry(e["id"], int(e["width"]), int(e["height"]),
                             Features(col("x"), col("y"), col("scale"), col("response"), col("orientation"), desc))
        return cat

    def save_auto(self, path: str, pretty: bool = False):
        """``save_auto`` (src/catalog.rs:543-553): JSON for a .json extension, else binary."""
        if os.path.splitext(path)[1].lower() == ".json":
            self.save_json(path, pretty)
        else:
            self.save_binary(path)

    @classmethod
    def load_auto(cls, path: str, ctx: Context | None = None) -> "DeviceCatalog":
        """``load_auto`` (src/catalog.rs:556-574): PSIFTCAT magic -> binary, else JSON."""
        with open(path, "rb") as fh:
            head = fh.read(8)
        if head == BINARY_CATALOG_MAGIC:
            return cls.load_binary(path, ctx)
        return cls.load_json(path, ctx)


def warp_and_stitch(query: np.ndarray, target: np.ndarray, homography, ctx: Context | None = None):
    """``warp_and_stitch`` (src/visualize.rs:379-483) on the GPU.

    query, target: (h, w, 4) u8 RGBA; homography: 3x3 (query -> target).
    Returns (canvas (H, W, 4) u8, (origin_x, origin_y)); raises ValueError with
    the reference's message when it returns Err."""
    ctx = ctx or default_context()
    q = np.ascontiguousarray(query, dtype=np.uint8).reshape(query.shape[0], query.shape[1], 4)
    t = np.ascontiguousarray(target, dtype=np.uint8).reshape(target.shape[0], target.shape[1], 4)
    h9 = np.ascontiguousarray(homography, dtype=np.float32).reshape(9)
    w, h = C.c_uint32(), C.c_uint32()
    origin = np.zeros(2, np.float64)
    args = (q.ctypes.data, q.shape[0], q.shape[1], q.shape[1] * 4, t.ctypes.data, t.shape[0], t.shape[1],
            t.shape[1] * 4, h9.ctypes.data)
    st = ctx.lib.psift_warp_and_stitch(ctx.handle, *args, None, 0, C.byref(w), C.byref(h), origin.ctypes.data)
    if st == PSIFT_ERR_INVALID_ARGUMENT:
        raise ValueError(ctx.lib.psift_last_error(ctx.handle).decode())
    ctx.check(st)
    canvas = np.empty((h.value, w.value, 4), np.uint8)
    ctx.check(ctx.lib.psift_warp_and_stitch(ctx.handle, *args, canvas.ctypes.data, canvas.nbytes, C.byref(w),
                                            C.byref(h), None))
    return canvas, (float(origin[0]), float(origin[1]))


def gaussian_blur(img: np.ndarray, sigma: float, ctx: Context | None = None) -> np.ndarray:
    """``gaussian_blur`` (src/pipeline.rs:314-425) on the GPU."""
    ctx = ctx or default_context()
    img = np.ascontiguousarray(img, dtype=np.float32)
    out = np.empty_like(img)
    h, w = img.shape
    ctx.check(ctx.lib.psift_gaussian_blur(ctx.handle, img.ctypes.data, h, w, w, float(sigma), out.ctypes.data))
    return out


def build_pyramid(img: np.ndarray, config: "SiftConfig" = None, ctx: Context | None = None):
    """``build_scale_space_pyramid_with_options`` (src/pipeline.rs:550-638) on the GPU.

    Returns a list of (gaussian, dog) per octave: arrays of shape
    (scales+3, h, w) and (scales+2, h, w)."""
    ctx = ctx or default_context()
    config = config or SiftConfig()
    img = np.ascontiguousarray(img, dtype=np.float32)
    h, w = img.shape
    cc = config.to_c()
    dims = np.zeros(2 * max(cc.octaves, 1), np.uint32)
    n = C.c_uint32()
    ctx.check(ctx.lib.psift_build_pyramid(ctx.handle, img.ctypes.data, h, w, w, C.byref(cc), None, 0,
                                          dims.ctypes.data, C.byref(n)))
    S = cc.scales
    sizes = [(int(dims[2 * o]), int(dims[2 * o + 1])) for o in range(n.value)]
    total = sum((2 * S + 5) * a * b for a, b in sizes)
    buf = np.empty(max(total, 1), np.float32)
    ctx.check(ctx.lib.psift_build_pyramid(ctx.handle, img.ctypes.data, h, w, w, C.byref(cc), buf.ctypes.data, total,
                                          dims.ctypes.data, C.byref(n)))
    out, off = [], 0
    for a, b in sizes:
        blk = buf[off: off + (2 * S + 5) * a * b].reshape(2 * S + 5, a, b)
        out.append((blk[: S + 3], blk[S + 3:]))
        off += (2 * S + 5) * a * b
    return out


# ---------------------------------------------------------------- panorama
class CRgbaImage(C.Structure):
    _fields_ = [("data", C.c_void_p), ("height", C.c_uint32), ("width", C.c_uint32), ("row_stride", C.c_size_t)]


class PanoramaOptions(C.Structure):
    """``PanoramaOptions`` (src/stitch.rs:45-89).  projection: PROJECTION_PLANAR /
    PROJECTION_CYLINDRICAL (with focal_px); blend: BLEND_FEATHER / BLEND_MULTIBAND
    (with levels)."""
    _fields_ = [("octaves", C.c_uint32), ("scales", C.c_uint32), ("threshold", C.c_float), ("ratio", C.c_float),
                ("ransac_threshold", C.c_float), ("projection", C.c_int32), ("focal_px", C.c_float),
                ("blend", C.c_int32), ("levels", C.c_uint32), ("exposure_compensation", C.c_int32),
                ("max_canvas_dim", C.c_uint32), ("max_canvas_pixels", C.c_uint64), ("tile_size", C.c_uint32)]
    PROJECTION_PLANAR, PROJECTION_CYLINDRICAL = 0, 1
    BLEND_FEATHER, BLEND_MULTIBAND = 0, 1

    @classmethod
    def default(cls, **kw) -> "PanoramaOptions":
        o = cls()
        load_library().psift_panorama_options_default(C.byref(o))
        for k, v in kw.items():
            setattr(o, k, v)
        return o


class CPanoramaInfo(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("reference_index", C.c_int32),
                ("registered_count", C.c_int32), ("origin_x", C.c_double), ("origin_y", C.c_double)]


class PanoramaResult:
    """``PanoramaResult`` (src/stitch.rs:91-103): image (H, W, 4) u8, reference_index,
    registered_indices, gains (per input), homographies (per input: 3x3 f32 image ->
    reference, or None), plus the canvas origin in reference coordinates."""

    def __init__(self, image, reference_index, registered, gains, homographies, origin):
        self.image = image
        self.reference_index = reference_index
        self.registered_indices = [i for i, r in enumerate(registered) if r]
        self.gains = gains
        self.homographies = [homographies[i].reshape(3, 3) if r else None for i, r in enumerate(registered)]
        self.origin = origin


def _rgba_images(images):
    imgs = [np.ascontiguousarray(im, dtype=np.uint8).reshape(im.shape[0], im.shape[1], 4) for im in images]
    arr = (CRgbaImage * max(len(imgs), 1))(*[CRgbaImage(im.ctypes.data, im.shape[0], im.shape[1], im.shape[1] * 4)
                                             for im in imgs])
    return imgs, arr


def stitch_panorama(images, options: PanoramaOptions | None = None, ctx: Context | None = None) -> PanoramaResult:
    """``stitch_panorama`` (src/stitch.rs:472-948) on the GPU: images are (h, w, 4) u8
    RGBA.  Raises ValueError with the reference's message when it returns Err."""
    ctx = ctx or default_context()
    options = options or PanoramaOptions.default()
    imgs, arr = _rgba_images(images)
    n = len(imgs)
    info = CPanoramaInfo()
    reg = np.zeros(max(n, 1), np.uint8)
    gains = np.zeros(max(n, 1), np.float32)
    hs = np.zeros((max(n, 1), 9), np.float32)
    cap = sum(im.shape[0] * im.shape[1] for im in imgs) * 4 * 4 + 4096
    canvas = np.empty(cap, np.uint8)
    while True:
        st = ctx.lib.psift_stitch_panorama(ctx.handle, arr, n, C.byref(options), canvas.ctypes.data, canvas.nbytes,
                                           C.byref(info), reg.ctypes.data, gains.ctypes.data, hs.ctypes.data)
        if st == PSIFT_ERR_CAPACITY and info.width * info.height * 4 > canvas.nbytes:
            canvas = np.empty(info.width * info.height * 4, np.uint8)
            continue
        break
    if st == PSIFT_ERR_INVALID_ARGUMENT:
        raise ValueError(ctx.lib.psift_last_error(ctx.handle).decode())
    ctx.check(st)
    image = canvas[:info.width * info.height * 4].reshape(info.height, info.width, 4).copy()
    return PanoramaResult(image, info.reference_index, reg[:n].astype(bool), gains[:n], hs[:n],
                          (info.origin_x, info.origin_y))


def warp_cylindrical(image, focal_px: float, ctx: Context | None = None) -> np.ndarray:
    """``warp_image_cylindrical`` (src/stitch.rs:166-201) on the GPU."""
    ctx = ctx or default_context()
    imgs, arr = _rgba_images([image])
    out = np.zeros_like(imgs[0])
    ctx.check(ctx.lib.psift_warp_cylindrical(ctx.handle, arr, float(focal_px), out.ctypes.data))
    return out


def panorama_composite(images, registered, gains, inverses, origin, width: int, height: int, blend: int,
                       levels: int = 4, ctx: Context | None = None) -> np.ndarray:
    """The compositing half of ``stitch_panorama`` on given registration results:
    inverses (n, 3, 3) f64 reference -> image; returns the (height, width, 4) canvas."""
    ctx = ctx or default_context()
    imgs, arr = _rgba_images(images)
    regm = np.ascontiguousarray(registered, dtype=np.uint8)
    g = np.ascontiguousarray(gains, dtype=np.float32)
    inv = np.ascontiguousarray(inverses, dtype=np.float64).reshape(-1, 9)
    canvas = np.zeros((height, width, 4), np.uint8)
    ctx.check(ctx.lib.psift_panorama_composite(ctx.handle, arr, len(imgs), regm.ctypes.data, g.ctypes.data,
                                               inv.ctypes.data, float(origin[0]), float(origin[1]), width, height,
                                               int(blend), int(levels), canvas.ctypes.data))
    return canvas
