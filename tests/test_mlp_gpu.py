"""The learned sampler on the GPU: forward and gradients against the FP64
restatement, training on plain-RANSAC labels, and what guided sampling gains
over the plain (reference) sampler at equal inlier count."""
import numpy as np
import pytest

import mlp_oracle as M
import psift
import synth

pytestmark = pytest.mark.gpu


def _data(n, seed):
    H = synth.perspective_h(1920, 1080, 20.0, 1.1, 1e-4, 5e-5)
    rec, feats, inl = synth.putative_matches(n, 0.5, H, 1920, 1080, seed)
    return feats, inl.astype(np.float32)


def test_forward_matches_fp64_oracle():
    X, _ = _data(3000, 1)
    mlp = psift.InlierMLP(seed=3)
    got = mlp.predict(X)
    ref = M.predict(mlp.params, X)
    assert np.abs(got - ref).max() < 2e-3


def test_gradients_match_fp64_oracle():
    X, Y = _data(4096, 2)
    mlp = psift.InlierMLP(seed=4)
    loss, g = mlp.gradients(X, Y)
    rloss, rg = M.loss_and_grad(mlp.params, X, Y)
    assert abs(loss - rloss) < 1e-4 * max(1.0, abs(rloss))
    rel = np.linalg.norm(g - rg) / np.linalg.norm(rg)
    assert rel < 2e-3, rel
    big = np.abs(rg) > 1e-2 * np.abs(rg).max()
    assert np.all(np.abs(g[big] - rg[big]) <= 1e-2 * np.abs(rg[big]) + 1e-6)


def _pairs(ks):
    return [synth.c5_pair(k) for k in ks]


def _plain_labels(recs):
    res = psift.ransac_batch([r for r, _, _ in recs])
    return [mask for mask, _, _ in res], res


def test_training_learns_plain_ransac_labels_and_guided_sampling_gains():
    train = _pairs(range(0, 24))
    labels, _ = _plain_labels(train)
    X = np.concatenate([f for _, f, _ in train])
    Y = np.concatenate(labels).astype(np.float32)
    mlp = psift.InlierMLP(seed=11)
    losses = mlp.train(X, Y, steps=400, batch=4096, lr=3e-3, seed=12)
    assert losses[-20:].mean() < 0.8 * losses[:20].mean()
    test = _pairs(range(100, 116))
    plain = psift.ransac_batch([r for r, _, _ in test])
    probs = [np.clip(mlp.predict(f), 0.02, 1.0) for _, f, _ in test]
    acc = np.mean(np.concatenate([(p > 0.5) == m for p, (m, _, _) in zip(probs, plain)]))
    assert acc > 0.9, acc
    guided = psift.ransac_batch([r for r, _, _ in test], weights=probs)
    plain_in = np.array([m.sum() for m, _, _ in plain])
    guided_in = np.array([m.sum() for m, _, _ in guided])
    plain_it = np.array([it[1] for _, _, it in plain])
    guided_it = np.array([it[1] for _, _, it in guided])
    assert np.all(guided_in >= np.floor(0.99 * plain_in)), (guided_in, plain_in)
    assert guided_it.sum() < plain_it.sum(), (guided_it, plain_it)
