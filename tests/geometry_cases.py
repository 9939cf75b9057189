"""Two-view correspondences of the reference's tests/geometry_tests.rs:10-95
(euler_zyx_rotation, project_point, make_3d_correspondences with its seeded
LCG), restated to build the same inputs for the fundamental-matrix pins."""
import math

import numpy as np

MATCH_FIELDS = [("query_index", "<u4"), ("target_index", "<u4"), ("query_x", "<f4"), ("query_y", "<f4"),
                ("target_x", "<f4"), ("target_y", "<f4"), ("distance", "<f4"), ("ratio", "<f4"),
                ("displacement_x", "<f4"), ("displacement_y", "<f4")]
K_720 = (720.0, 720.0, 400.0, 300.0)  # fx, fy, cx, cy


def euler_zyx_rotation(yaw_deg, pitch_deg, roll_deg):
    sz, cz = math.sin(math.radians(yaw_deg)), math.cos(math.radians(yaw_deg))
    sy, cy = math.sin(math.radians(pitch_deg)), math.cos(math.radians(pitch_deg))
    sx, cx = math.sin(math.radians(roll_deg)), math.cos(math.radians(roll_deg))
    rz = np.array([[cz, -sz, 0.0], [sz, cz, 0.0], [0.0, 0.0, 1.0]])
    ry = np.array([[cy, 0.0, sy], [0.0, 1.0, 0.0], [-sy, 0.0, cy]])
    rx = np.array([[1.0, 0.0, 0.0], [0.0, cx, -sx], [0.0, sx, cx]])
    return rz @ (ry @ rx)


def _project(k, r, t, pt):
    xc = r[0][0] * pt[0] + r[0][1] * pt[1] + r[0][2] * pt[2] + t[0]
    yc = r[1][0] * pt[0] + r[1][1] * pt[1] + r[1][2] * pt[2] + t[1]
    zc = r[2][0] * pt[0] + r[2][1] * pt[1] + r[2][2] * pt[2] + t[2]
    return k[0] * (xc / zc) + k[2], k[1] * (yc / zc) + k[3]


def make_3d_correspondences(n_inliers, n_outliers, k, r, t):
    """Inliers first (ratio 0.45), then outliers uniform in 800 x 600 (ratio 0.78)."""
    state = 0x1234ABCD567890EF
    mask64 = (1 << 64) - 1

    def u01():
        nonlocal state
        state = (state * 6364136223846793005 + 1) & mask64
        return (state >> 11) / float(1 << 53)

    rec = np.zeros(n_inliers + n_outliers, dtype=MATCH_FIELDS)
    ident = np.eye(3)
    for i in range(n_inliers):
        x = (u01() - 0.5) * 4.0
        y = (u01() - 0.5) * 3.5
        z = 4.0 + u01() * 5.0
        p1 = _project(k, ident, (0.0, 0.0, 0.0), (x, y, z))
        p2 = _project(k, r, t, (x, y, z))
        rec[i] = (i, i, p1[0], p1[1], p2[0], p2[1], 0.1, 0.45, p2[0] - p1[0], p2[1] - p1[1])
    for j in range(n_outliers):
        i = n_inliers + j
        x1, y1, x2, y2 = u01() * 800.0, u01() * 600.0, u01() * 800.0, u01() * 600.0
        rec[i] = (i, i, x1, y1, x2, y2, 0.4, 0.78, x2 - x1, y2 - y1)
    return rec


def sampson(F, m):
    """sampson_distance_sq (src/geometry.rs:617-636), vectorised (float64)."""
    x1, y1 = m["query_x"].astype(np.float64), m["query_y"].astype(np.float64)
    x2, y2 = m["target_x"].astype(np.float64), m["target_y"].astype(np.float64)
    a0 = F[0, 0] * x1 + F[0, 1] * y1 + F[0, 2]
    a1 = F[1, 0] * x1 + F[1, 1] * y1 + F[1, 2]
    a2 = F[2, 0] * x1 + F[2, 1] * y1 + F[2, 2]
    b0 = F[0, 0] * x2 + F[1, 0] * y2 + F[2, 0]
    b1 = F[0, 1] * x2 + F[1, 1] * y2 + F[2, 1]
    e = x2 * a0 + y2 * a1 + a2
    den = a0 * a0 + a1 * a1 + b0 * b0 + b1 * b1
    return np.where(den < 1e-18, np.inf, e * e / np.maximum(den, 1e-300))
