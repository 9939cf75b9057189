"""Panorama inputs shared by the CPU and GPU panorama tests.

aerial_tiles: the reference's 4-tile panorama test case
(tests/panorama_tests.rs:28-81): the sample docs/samples/aerial_west.jpg cut into
four overlapping tiles 42 % of its width wide, each scaled in exposure by
(0.85, 1.0, 1.18, 0.92) with round-and-clamp.  The committed fixture holds the
sample's luma only, so the tiles are grey RGBA (r = g = b = luma; its luma is
the same value again).

blob_tiles: three overlapping crops of a synthetic colour field (three
independent 2000-blob planes as R, G, B) at different exposures."""
import os

import numpy as np

import synth

HERE = os.path.dirname(os.path.abspath(__file__))
FACTORS = (0.85, 1.0, 1.18, 0.92)


def _rgba(v):
    return np.stack([v, v, v, np.full_like(v, 255)], axis=-1)


def aerial_tiles():
    L = np.load(os.path.join(HERE, "golden", "aerial_west_luma.npz"))["luma"]
    h, w = L.shape
    tile_w = (w * 42) // 100
    step = (w - tile_w) // 3
    tiles = []
    for i, f in enumerate(FACTORS):
        crop = L[:, i * step:i * step + tile_w].astype(np.float32)
        tiles.append(_rgba(np.clip(np.round(crop * np.float32(f)), 0, 255).astype(np.uint8)))
    return tiles, w


def blob_tiles(w=960, h=360, tile=420, factors=(1.0, 0.9, 1.1)):
    chans = [synth.blob_image(w, h, 700, 1.5, 12.0, seed=s) for s in (41, 42, 43)]
    rgb = np.stack(chans, axis=-1).astype(np.float32)
    step = (w - tile) // (len(factors) - 1)
    out = []
    for i, f in enumerate(factors):
        crop = rgb[:, i * step:i * step + tile]
        v = np.clip(np.round(crop * np.float32(f)), 0, 255).astype(np.uint8)
        out.append(np.concatenate([v, np.full(v.shape[:2] + (1,), 255, np.uint8)], axis=-1))
    return out
