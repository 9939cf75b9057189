"""The synthetic 220 x 220 scenes of the reference's catalog tests
(`render_synthetic_scene`, tests/pipeline_tests.rs:795-837): filled rectangles
(x0, y0, width, height, level) on black, shifted by (shift_x, shift_y) and
clipped to the image."""
import numpy as np

# tests/pipeline_tests.rs:797-823
_SHAPES = {
    0: [(25, 25, 28, 10, 255), (25, 25, 10, 28, 255), (90, 40, 22, 22, 220), (40, 110, 14, 30, 240),
        (54, 126, 20, 12, 255), (120, 95, 24, 10, 235), (134, 105, 10, 24, 210)],
    1: [(30, 35, 14, 14, 250), (60, 30, 12, 34, 215), (95, 65, 30, 12, 245), (135, 35, 16, 26, 230),
        (45, 130, 28, 12, 255), (115, 125, 22, 22, 200)],
    2: [(20, 50, 32, 8, 240), (44, 58, 8, 32, 240), (100, 25, 16, 16, 255), (140, 75, 24, 24, 190),
        (70, 120, 26, 10, 220), (30, 150, 18, 18, 250)],
}


def render_synthetic_scene(seed: int, shift_x: int = 0, shift_y: int = 0) -> np.ndarray:
    img = np.zeros((220, 220), np.uint8)
    for x0, y0, w, h, val in _SHAPES[seed if seed in (0, 1) else 2]:
        ys = slice(y0 + shift_y, min(y0 + h + shift_y, 220))
        xs = slice(x0 + shift_x, min(x0 + w + shift_x, 220))
        img[ys, xs] = val
    return img
