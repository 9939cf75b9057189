"""The tile-shape autotuner (psift_ctx_autotune): every candidate it chooses
between computes the same results, so any choice is safe; the autotuner picks
valid entries and results after tuning equal the defaults."""
import numpy as np
import pytest

import oracle as O
import psift
import synth

pytestmark = pytest.mark.gpu


def _same_features(a, b):
    assert len(a) == len(b)
    for k in ("x", "y", "scale", "response", "orientation", "descriptors"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)


@pytest.mark.parametrize("variant", [1, 2, 3, 4])
def test_blur_variants_equal_default_and_oracle(variant):
    img = O.luma_to_f32(synth.blob_image(333, 251, 90, 1.5, 10.0, seed=41))
    cfg = psift.SiftConfig().with_octaves(4).with_scales(4)
    ctx = psift.Context(0)
    ref = psift.build_pyramid(img, cfg, ctx=ctx)
    for r in range(1, 16):
        ctx.set_tuning(ctx.TUNE_BLUR, r, variant)
    got = psift.build_pyramid(img, cfg, ctx=ctx)
    for (g0, d0), (g1, d1) in zip(ref, got):
        np.testing.assert_array_equal(g0, g1)
        np.testing.assert_array_equal(d0, d1)
    opy = O.Pyramid(img, 4, 4, True)
    np.testing.assert_array_equal(got[0][0][3], opy.plane(0, "g", 3))
    sift = psift.Sift.new(psift.SiftConfig())
    u8 = synth.blob_image(400, 300, 120, 2.0, 10.0, seed=42)
    eager = psift.Context(0)
    _same_features(sift.detect_and_compute_u8(u8, ctx=ctx), sift.detect_and_compute_u8(u8, ctx=eager))
    ctx.close()
    eager.close()


@pytest.mark.parametrize("per_sm", [1, 4, 8])
def test_matcher_work_split_keeps_match_lists(per_sm):
    q = synth.sift_like_descriptors(1500, seed=5)
    t = np.concatenate([q[:700] + 0.01 * synth.sift_like_descriptors(700, seed=6), synth.sift_like_descriptors(900, seed=7)])
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    rng = np.random.default_rng(3)
    qf = psift.Features(*(rng.random(1500).astype(np.float32) * 500 for _ in range(2)), np.ones(1500, np.float32),
                        np.zeros(1500, np.float32), np.zeros(1500, np.float32), q.astype(np.float32))
    tf = psift.Features(*(rng.random(1600).astype(np.float32) * 500 for _ in range(2)), np.ones(1600, np.float32),
                        np.zeros(1600, np.float32), np.zeros(1600, np.float32), t.astype(np.float32))
    base = psift.Context(0)
    ctx = psift.Context(0)
    ctx.set_tuning(ctx.TUNE_MATCH_FP32, 0, per_sm)
    ctx.set_tuning(ctx.TUNE_MATCH_TC, 0, per_sm)
    for prec in (psift.PRECISION_FP32, psift.PRECISION_BF16_RERANK):
        m = psift.Matcher.new(psift.MatchOptions(0.8, precision=prec))
        a, b = m.match_(qf, tf, ctx=ctx), m.match_(qf, tf, ctx=base)
        assert len(a) > 100
        np.testing.assert_array_equal(a, b)
    ctx.close()
    base.close()


def test_autotune_picks_valid_choices_and_keeps_results():
    ctx = psift.Context(0)
    cfg = psift.SiftConfig()
    rep = ctx.autotune(480, 640, 2, cfg, n_desc=1024, n_pairs=2)
    assert set(rep["blur"]) == {4, 5, 6, 8, 10}  # the default schedule's level radii
    for r, e in rep["blur"].items():
        assert e["variant"] in (0, 1, 2, 3, 4) and len(e["ms"]) == 5 and min(e["ms"]) > 0
        assert ctx.tuning()["blur"][r] == e["variant"]
    assert rep["match_fp32"]["per_sm"] in (1, 2, 4, 8) and rep["match_tc"]["per_sm"] in (1, 2, 4, 8)
    tun = ctx.tuning()
    assert tun["match_fp32_per_sm"] == rep["match_fp32"]["per_sm"]
    sift = psift.Sift.new(cfg)
    u8 = synth.blob_image(640, 480, 150, 2.0, 10.0, seed=43)
    plain = psift.Context(0)
    _same_features(sift.detect_and_compute_u8(u8, ctx=ctx), sift.detect_and_compute_u8(u8, ctx=plain))
    with pytest.raises(psift.PsiftError):
        ctx.set_tuning(ctx.TUNE_BLUR, 4, 7)
    with pytest.raises(psift.PsiftError):
        ctx.set_tuning(ctx.TUNE_MATCH_TC, 0, 0)
    ctx.close()
    plain.close()
