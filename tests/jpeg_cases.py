"""JPEG inputs for the decode step (decode_validated_luma8, src/cli.rs:164-170):
synthetic blob images encoded by PIL, and the CPU side of the comparison (PIL's
decoder followed by the image crate's u8 rgb_to_luma)."""
import io

import numpy as np
from PIL import Image

import synth


def rgb_to_luma_u8(rgb: np.ndarray) -> np.ndarray:
    """The image crate's rgb_to_luma for u8: (2126 R + 7152 G + 722 B) / 10000 in u32, truncated."""
    r, g, b = (rgb[..., i].astype(np.uint32) for i in range(3))
    return ((2126 * r + 7152 * g + 722 * b) // 10000).astype(np.uint8)


def gray_image(w: int, h: int, seed: int) -> np.ndarray:
    return synth.blob_image(w, h, max(1, int(300 * w * h / (640 * 480))), 2.0, 12.0, seed)


def color_image(w: int, h: int, seed: int) -> np.ndarray:
    """Three independent blob fields as R, G, B."""
    return np.stack([gray_image(w, h, seed + k) for k in range(3)], axis=2)


def encode(img: np.ndarray, quality: int = 92, subsampling: int = 2) -> bytes:
    """Baseline JPEG; subsampling 0 = 4:4:4, 1 = 4:2:2, 2 = 4:2:0 (ignored for gray)."""
    buf = io.BytesIO()
    im = Image.fromarray(img)
    if img.ndim == 2:
        im.save(buf, format="JPEG", quality=quality)
    else:
        im.save(buf, format="JPEG", quality=quality, subsampling=subsampling)
    return buf.getvalue()


def cpu_luma(blob: bytes) -> np.ndarray:
    im = Image.open(io.BytesIO(blob))
    if im.mode == "L":
        return np.asarray(im).copy()
    return rgb_to_luma_u8(np.asarray(im.convert("RGB")))
