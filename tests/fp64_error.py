"""Error of an f32 detect/describe result against the same pipeline run in f64.

The yardstick is the oracle's f64 instantiation (every value, constant and libm
call in double, from the same u8 luma).  The tolerances are the ones the f32
path is held to: keypoint position within 0.01 px, scale within 0.01, and
descriptor relative L2 difference within 1e-4.  The reference's f32 arithmetic
itself does not meet them on every keypoint (a Taylor step that lands on the
other side of the +-0.5 offset test, an orientation-histogram pixel that changes
bin), so each statement is a fraction of the paired keypoints / features.
"""
import numpy as np

POS_TOL = 0.01      # px, base-image coordinates
SCALE_TOL = 0.01
DESC_TOL = 1e-4     # relative L2 of the 128-D descriptor


def pair_keypoints(x, y, octave, layer, k64, radius=0.5):
    """Pairs each f64 keypoint (rows x, y, scale, response, octave, layer) with
    the nearest f32 keypoint of the same octave and layer within `radius` px.
    Returns (index into k64, index into the f32 list) pairs."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    pairs = []
    for o in np.unique(k64[:, 4]):
        for l in np.unique(k64[k64[:, 4] == o, 5]):
            i64 = np.nonzero((k64[:, 4] == o) & (k64[:, 5] == l))[0]
            i32 = np.nonzero((np.asarray(octave) == o) & (np.asarray(layer) == l))[0]
            if len(i32) == 0:
                continue
            for c in range(0, len(i64), 512):
                a = i64[c:c + 512]
                d = np.hypot(k64[a, 0][:, None] - x[i32][None, :], k64[a, 1][:, None] - y[i32][None, :])
                j = np.argmin(d, axis=1)
                ok = d[np.arange(len(a)), j] < radius
                pairs.extend(zip(a[ok], i32[j[ok]]))
    return np.array(pairs, np.int64).reshape(-1, 2)


def keypoint_error(x, y, scale, octave, layer, k64):
    pr = pair_keypoints(x, y, octave, layer, k64)
    dxy = np.hypot(k64[pr[:, 0], 0] - np.asarray(x, np.float64)[pr[:, 1]],
                   k64[pr[:, 0], 1] - np.asarray(y, np.float64)[pr[:, 1]])
    dsc = np.abs(k64[pr[:, 0], 2] - np.asarray(scale, np.float64)[pr[:, 1]])
    return {
        "n_f32": int(len(x)), "n_f64": int(len(k64)), "paired": int(len(pr)),
        "pos_max": float(dxy.max()) if len(pr) else 0.0,
        "pos_p99": float(np.quantile(dxy, 0.99)) if len(pr) else 0.0,
        "scale_max": float(dsc.max()) if len(pr) else 0.0,
        "frac_within": float(((dxy <= POS_TOL) & (dsc <= SCALE_TOL)).mean()) if len(pr) else 1.0,
    }


def feature_error(meta32, desc32, meta64, desc64):
    """Pairs each f64 feature with the f32 feature at the nearest position
    (within 0.5 px) and, among those, the nearest orientation; returns the
    descriptor relative L2 differences and orientation differences."""
    m32 = np.asarray(meta32, np.float64)
    d32 = np.asarray(desc32, np.float64)
    rel, dth = [], []
    unpaired = 0
    for c in range(0, len(meta64), 256):
        a = np.arange(c, min(c + 256, len(meta64)))
        d = np.hypot(meta64[a, 0][:, None] - m32[None, :, 0], meta64[a, 1][:, None] - m32[None, :, 1])
        for r, i in enumerate(a):
            cand = np.nonzero(d[r] < 0.5)[0]
            if len(cand) == 0:
                unpaired += 1
                continue
            t = np.abs((m32[cand, 4] - meta64[i, 4] + np.pi) % (2 * np.pi) - np.pi)
            j = cand[int(np.argmin(t))]
            dth.append(float(t.min()))
            rel.append(float(np.linalg.norm(d32[j] - desc64[i]) / max(np.linalg.norm(desc64[i]), 1e-30)))
    rel = np.array(rel)
    dth = np.array(dth)
    return {
        "n_f32": int(len(meta32)), "n_f64": int(len(meta64)), "paired": int(len(rel)), "unpaired": unpaired,
        "desc_rel_max": float(rel.max()) if len(rel) else 0.0,
        "desc_rel_p99": float(np.quantile(rel, 0.99)) if len(rel) else 0.0,
        "frac_within": float((rel <= DESC_TOL).mean()) if len(rel) else 1.0,
        "theta_max": float(dth.max()) if len(dth) else 0.0,
    }


def statement(label, kp, ft):
    return (f"{label}: keypoints f32 {kp['n_f32']} / f64 {kp['n_f64']}, paired {kp['paired']}, "
            f"{100 * kp['frac_within']:.2f}% within {POS_TOL} px and {SCALE_TOL} scale "
            f"(position max {kp['pos_max']:.2e}, p99 {kp['pos_p99']:.2e}); features f32 {ft['n_f32']} / "
            f"f64 {ft['n_f64']}, {100 * ft['frac_within']:.2f}% within {DESC_TOL} descriptor rel. L2 "
            f"(max {ft['desc_rel_max']:.2e}, p99 {ft['desc_rel_p99']:.2e}; orientation max {ft['theta_max']:.2e} rad)")
