"""FP64 restatement of the learned sampler's forward/backward (test infrastructure).

Same network and the same bf16 rounding points as pure-sift_b200/csrc/mlp.cu:
x, W1, W2, W3, h1 and h2 are rounded to bf16 (nearest even) from their f32
values; all accumulation here is f64, so GPU gradients must agree to f32
accumulation error.
"""
import numpy as np

F, H = 8, 64
NP = H * F + H + H * H + H + H + 1


def bf16(x):
    x32 = np.asarray(x, dtype=np.float32)
    u = x32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    out = r.view(np.float32)
    special = (x32.view(np.uint32) & 0x7F800000) == 0x7F800000
    return np.where(special, x32, out).astype(np.float64)


def unpack(p):
    p = np.asarray(p) if np.asarray(p).dtype == np.float64 else np.asarray(p, np.float32)
    o = 0
    W1 = p[o:o + H * F].reshape(H, F); o += H * F
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def forward(p, X, rounding=True):
    """rounding=False gives the same network in plain f64 (for finite-difference checks:
    bf16 rounding makes the loss piecewise constant in small parameter steps)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    r = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    xb = r(X)
    z1 = xb @ r(W1).T + b1
    h1b = r(np.maximum(z1, 0) if not rounding else np.maximum(z1, 0).astype(np.float32))
    z2 = h1b @ r(W2).T + b2
    h2b = r(np.maximum(z2, 0) if not rounding else np.maximum(z2, 0).astype(np.float32))
    z3 = h2b @ r(W3) + float(b3)
    return xb, z1, h1b, z2, h2b, z3


def loss_and_grad(p, X, Y, rounding=True):
    xb, z1, h1b, z2, h2b, z3 = forward(p, X, rounding)
    W1, b1, W2, b2, W3, b3 = unpack(p)
    if not rounding:
        bf = lambda v: np.asarray(v, np.float64)  # noqa: E731
    else:
        bf = bf16
    B = X.shape[0]
    prob = 1.0 / (1.0 + np.exp(-z3))
    loss = np.mean(np.maximum(z3, 0) - z3 * Y + np.log1p(np.exp(-np.abs(z3))))
    dz3 = (prob - Y) / B
    dz2 = np.where(z2 > 0, dz3[:, None] * bf(W3)[None, :], 0.0)
    dz1 = np.where(z1 > 0, dz2 @ bf(W2), 0.0)
    g = np.concatenate([(dz1.T @ xb).ravel(), dz1.sum(0), (dz2.T @ h1b).ravel(), dz2.sum(0), dz3 @ h2b,
                        [dz3.sum()]])
    return loss, g


def predict(p, X):
    z3 = forward(p, X)[-1]
    return 1.0 / (1.0 + np.exp(-z3))
