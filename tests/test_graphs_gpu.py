"""CUDA-graph replay of the device batch path: the first call with a geometry
runs eagerly, the second is captured, later ones replay.  Replays with other
image data and other output buffers must equal eager runs exactly."""
import ctypes as C

import numpy as np
import pytest

import psift
import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SHAPES = [(300, 420), (257, 333), (480, 640)]


def _run(ctx, host_imgs, cfg, cap=4096):
    B = len(host_imgs)
    d_imgs = [torch.from_numpy(np.ascontiguousarray(im)).cuda() for im in host_imgs]
    outs = [{k: torch.empty(cap, dtype=torch.float32, device="cuda") for k in "xysro"} for _ in range(B)]
    for o in outs:
        o["d"] = torch.empty((cap, 128), dtype=torch.float32, device="cuda")
    counts = torch.zeros(B, dtype=torch.int32, device="cuda")
    cimgs = (psift.CImageU8 * B)(*[psift.CImageU8(t.data_ptr(), t.shape[0], t.shape[1], t.shape[1]) for t in d_imgs])
    couts = (psift.CFeatures * B)(*[psift.CFeatures(cap, 0, o["x"].data_ptr(), o["y"].data_ptr(), o["s"].data_ptr(),
                                                    o["r"].data_ptr(), o["o"].data_ptr(), o["d"].data_ptr())
                                    for o in outs])
    ccfg = cfg.to_c()
    ctx.check(ctx.lib.psift_detect_and_compute_batch_dev(ctx.handle, cimgs, B, C.byref(ccfg), couts,
                                                         C.c_void_p(counts.data_ptr())))
    ctx.synchronize()
    res = []
    for i, o in enumerate(outs):
        c = int(counts[i].item())
        res.append({k: v[:c].cpu().numpy() for k, v in o.items()})
    return res


def _same(a, b):
    assert len(a) == len(b)
    for fa, fb in zip(a, b):
        assert fa.keys() == fb.keys()
        for k in fa:
            np.testing.assert_array_equal(fa[k], fb[k], err_msg=k)


def test_graph_replay_equals_eager():
    cfg = psift.SiftConfig().with_octaves(4)
    set_a = [synth.blob_image(w, h, 150, 1.5, 12.0, seed=100 + i) for i, (h, w) in enumerate(SHAPES)]
    set_b = [synth.blob_image(w, h, 150, 1.5, 12.0, seed=200 + i) for i, (h, w) in enumerate(SHAPES)]
    eager = psift.Context(0)
    eager.enable_graphs(False)
    ref_a, ref_b = _run(eager, set_a, cfg), _run(eager, set_b, cfg)
    assert eager.graph_replays == 0
    ctx = psift.Context(0)
    _same(_run(ctx, set_a, cfg), ref_a)  # eager (first sight of the geometry)
    _same(_run(ctx, set_b, cfg), ref_b)  # captured, then replayed
    _same(_run(ctx, set_a, cfg), ref_a)  # replay, other data and buffers
    _same(_run(ctx, set_b, cfg), ref_b)
    assert ctx.graph_replays == 3
    # another geometry gets its own graph
    small = [im[:200, :300] for im in set_a]
    ref_s = _run(eager, small, cfg)
    for _ in range(3):
        _same(_run(ctx, small, cfg), ref_s)
    assert ctx.graph_replays == 5
    ctx.close()
    eager.close()


def test_single_image_host_path_replays_graphs():
    # psift_detect_and_compute_u8 / psift_detect_and_compute (one image per call, host
    # buffers) share the geometry-keyed graph cache; u8 and f32 inputs get separate graphs
    cfg = psift.SiftConfig().with_octaves(4)
    sift = psift.Sift.new(cfg)
    imgs = [synth.blob_image(320, 240, 90, 2.0, 10.0, seed=300 + i) for i in range(3)]
    eager = psift.Context(0)
    eager.enable_graphs(False)
    ctx = psift.Context(0)
    ref = [sift.detect_and_compute_u8(im, ctx=eager) for im in imgs]
    ref_f = sift.detect_and_compute(imgs[0].astype(np.float32) / 255.0, ctx=eager)
    for _ in range(2):
        for im, r in zip(imgs, ref):
            got = sift.detect_and_compute_u8(im, ctx=ctx)
            for k in ("x", "y", "scale", "response", "orientation", "descriptors"):
                np.testing.assert_array_equal(getattr(got, k), getattr(r, k), err_msg=k)
    assert eager.graph_replays == 0 and ctx.graph_replays == 5
    for _ in range(3):
        got = sift.detect_and_compute(imgs[0].astype(np.float32) / 255.0, ctx=ctx)
        np.testing.assert_array_equal(got.descriptors, ref_f.descriptors)
        np.testing.assert_array_equal(got.x, ref_f.x)
    assert ctx.graph_replays == 7
    ctx.close()
    eager.close()
