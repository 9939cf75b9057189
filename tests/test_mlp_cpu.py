"""The FP64 restatement of the learned sampler is itself checked by finite
differences (so the GPU gradient check has a trustworthy reference)."""
import numpy as np

import mlp_oracle as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(M.NP) * 0.3
    X = rng.standard_normal((64, 8))
    Y = (rng.random(64) < 0.5).astype(np.float64)
    # unrounded f64 network: the same gradient formulas, checked by central differences
    _, g = M.loss_and_grad(p, X, Y, rounding=False)
    for idx in [0, 7, 300, 512, 520, 575, 600, 2000, 4607, 4672, 4700, 4735, 4800]:
        h = 1e-5
        pp, pm = p.copy(), p.copy()
        pp[idx] += h
        pm[idx] -= h
        fd = (M.loss_and_grad(pp, X, Y, rounding=False)[0] - M.loss_and_grad(pm, X, Y, rounding=False)[0]) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(g[idx])) + 1e-8, (idx, fd, g[idx])


def test_init_is_deterministic():
    import psift
    a = psift.InlierMLP(seed=5).params
    b = psift.InlierMLP(seed=5).params
    c = psift.InlierMLP(seed=6).params
    assert a.shape == (4801,) and np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.all(a[512:576] == 0) and abs(a[:512]).max() <= np.sqrt(6 / 8) + 1e-6
