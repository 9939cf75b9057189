"""Makes tests/golden/aerial_west_luma.npz: the luma of the reference's own test
sample docs/samples/aerial_west.jpg (840 x 720), which tests/invariance_sweeps.rs
loads with `image::open(..).into_luma8()`.

The JPEG is decoded here by PIL (libjpeg-turbo), not by the image crate (0.25.10)
the reference links, so pixels may differ from the reference's by a few levels;
the sweeps this fixture feeds assert minimum inlier counts and 2 deg / 3 %
model errors, which such differences do not reach.  RGB -> luma follows the
image crate's `rgb_to_luma` for u8: the Rec. 709 weights 2126, 7152, 722 in u32
arithmetic, divided by 10000 with truncation.

Run from the repository root in a checkout that has the reference tree:
    python tests/golden/make_aerial_luma.py /path/to/pure-sift
"""
import os
import sys

import numpy as np
from PIL import Image


def rgb_to_luma_u8(rgb: np.ndarray) -> np.ndarray:
    r, g, b = (rgb[..., i].astype(np.uint32) for i in range(3))
    return ((2126 * r + 7152 * g + 722 * b) // 10000).astype(np.uint8)


def main(ref_root: str):
    src = os.path.join(ref_root, "docs", "samples", "aerial_west.jpg")
    rgb = np.asarray(Image.open(src).convert("RGB"))
    luma = rgb_to_luma_u8(rgb)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "aerial_west_luma.npz")
    np.savez_compressed(out, luma=luma)
    print(out, luma.shape, luma.dtype, int(luma.min()), int(luma.max()))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_aerial_luma.py <root of the pure-sift source tree>")
    main(sys.argv[1])
