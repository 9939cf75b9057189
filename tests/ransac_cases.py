"""Correspondence sets restated from the reference's own RANSAC tests
(tests/pipeline_tests.rs:344-524, tests/homography_properties.rs:71-237),
built with the reference's f32 Homography2D::project (src/pipeline.rs:1114-1127)."""
import numpy as np

from oracle import MATCH_DTYPE


def project(H, x, y):
    H = np.asarray(H, np.float32)
    x, y = np.float32(x), np.float32(y)
    w = H[2, 0] * x + H[2, 1] * y + H[2, 2]
    inv = np.float32(1.0) / w
    return np.float32((H[0, 0] * x + H[0, 1] * y + H[0, 2]) * inv), np.float32((H[1, 0] * x + H[1, 1] * y + H[1, 2]) * inv)


def _m(i, q, t, distance, ratio):
    qx, qy = np.float32(q[0]), np.float32(q[1])
    tx, ty = np.float32(t[0]), np.float32(t[1])
    return (i, i, qx, qy, tx, ty, np.float32(distance), np.float32(ratio), tx - qx, ty - qy)


def similarity_14():
    """10 crop-offset inliers (-341, 0) + 4 gross outliers (tests/pipeline_tests.rs:344-445)."""
    rows = []
    for i in range(10):
        qx = np.float32(400.0) + np.float32(i) * np.float32(85.0)
        qy = np.float32(50.0) + np.float32((i * 73) % 600)
        rows.append((i, i, qx, qy, qx - np.float32(341.0), qy, np.float32(0.02), np.float32(0.10),
                     np.float32(-341.0), np.float32(0.0)))
    offs = [(220.0, 180.0), (-90.0, -310.0), (410.0, -95.0), (150.0, 260.0)]
    for k, (ox, oy) in enumerate(offs):
        qx = np.float32(500.0) + np.float32(k) * np.float32(60.0)
        qy = np.float32(200.0) + np.float32(k) * np.float32(50.0)
        rows.append((10 + k, 10 + k, qx, qy, qx + np.float32(ox), qy + np.float32(oy), np.float32(0.28),
                     np.float32(0.71), np.float32(ox), np.float32(oy)))
    return np.array(rows, dtype=MATCH_DTYPE)


TRUE_H_13 = [[1.08, -0.04, 35.0], [0.03, 0.96, -18.0], [0.00012, -0.00008, 1.0]]
PTS_13 = [(50.0, 60.0), (320.0, 45.0), (480.0, 110.0), (95.0, 240.0), (260.0, 275.0), (440.0, 310.0),
          (70.0, 460.0), (290.0, 490.0), (495.0, 470.0), (180.0, 170.0)]


def homography_13():
    """10 perspective inliers + 3 outliers (tests/pipeline_tests.rs:448-524)."""
    rows = [_m(i, p, project(TRUE_H_13, *p), 0.015, 0.08) for i, p in enumerate(PTS_13)]
    for k, (qx, qy, tx, ty) in enumerate([(120.0, 130.0, 490.0, 20.0), (350.0, 220.0, 15.0, 480.0),
                                           (200.0, 400.0, 420.0, 90.0)]):
        rows.append(_m(len(PTS_13) + k, (qx, qy), (tx, ty), 0.31, 0.72))
    return np.array(rows, dtype=MATCH_DTYPE)


TRUE_H_60 = [[1.12, -0.06, 42.0], [0.05, 0.94, -24.0], [0.00015, -0.0001, 1.0]]
PTS_60 = [(40.0, 50.0), (200.0, 40.0), (420.0, 75.0), (560.0, 110.0), (80.0, 210.0), (270.0, 240.0),
          (490.0, 280.0), (60.0, 410.0), (230.0, 450.0), (440.0, 430.0), (580.0, 470.0), (330.0, 340.0)]


def homography_80pct_outliers():
    """12 inliers + 48 outliers incl. 8 collinear distractors (tests/homography_properties.rs:71-149)."""
    rows = [_m(i, p, project(TRUE_H_60, *p), 0.02, 0.25) for i, p in enumerate(PTS_60)]
    for k in range(48):
        qx = 100.0 + k * 30.0 if k < 8 else float((k * 97) % 600)
        qy = 100.0 if k < 8 else float((k * 131) % 480)
        rows.append(_m(len(PTS_60) + k, (qx, qy), (float((k * 173 + 50) % 620), float((k * 211 + 80) % 490)), 0.35, 0.72))
    return np.array(rows, dtype=MATCH_DTYPE)


TRUE_H_72 = [[1.04, -0.08, 22.0], [0.06, 0.97, -14.0], [0.0002, -0.0001, 1.0]]


def seeded_72():
    """24 grid inliers + 48 outliers (tests/homography_properties.rs:152-214)."""
    rows = []
    for i in range(24):
        q = (40.0 + (i % 6) * 75.0, 35.0 + (i // 6) * 80.0)
        rows.append(_m(i, q, project(TRUE_H_72, *q), 0.15, 0.55))
    for k in range(48):
        rows.append(_m(24 + k, (float((k * 83 + 17) % 500), float((k * 127 + 29) % 400)),
                       (float((k * 191 + 41) % 520), float((k * 233 + 67) % 420)), 0.4, 0.78))
    return np.array(rows, dtype=MATCH_DTYPE)


def correspondences(pairs, ratio=0.5):
    """`correspondences` of tests/homography_properties.rs:10-24."""
    return np.array([_m(i, q, t, 0.0, ratio) for i, (q, t) in enumerate(pairs)], dtype=MATCH_DTYPE)
