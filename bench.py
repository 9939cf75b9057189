#!/usr/bin/env python
"""Headline benchmark: 1080p SIFT detect+describe images/s on B200.

Workload (one "step"): one pass of Sift::detect_and_compute over a batch of
synthetic 1920x1080 u8 luma images (2000 Gaussian blobs, sigma ~ U(1.5, 20),
N(0,3) noise) with SiftConfig::default().octaves(4).contrast_threshold(0.015),
first-octave upsampling, Lowe's 4096-feature cap.  Inputs are resident in HBM
for `value`; `e2e` runs the same images through the public host-pointer API
(psift_detect_and_compute_u8) with the host->device copy of every image and the
device->host copy of every feature list inside the timed region.

Multi-GPU: images are independent, so each rank processes its own batch (weak
scaling, no data-path collective); the step time is the max over ranks.

`--impl reference` times the CPU restatement of the reference path (the
reference itself is Rust and cannot be built here) on all host cores.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "pure-sift_b200"))

import numpy as np  # noqa: E402

import shard  # noqa: E402
import synth  # noqa: E402

WIDTH, HEIGHT = 1920, 1080
OCTAVES, SCALES, THRESH, MAX_FEATURES = 4, 3, 0.015, 4096
METRIC = "1080p SIFT detect+describe images/s"
WORKLOAD = ("1920x1080 u8 blob images (2000 blobs, sigma U(1.5,20), N(0,3) noise); "
            "SiftConfig octaves=4 scales=3 threshold=0.015 upsample=on, cap 4096")
L2_NOTE = "no flush: per-step working set (~0.5 GB of scale-space planes per image) >> 126 MB L2"
# DRAM bytes per blur_level_kernel launch, averaged over the 21 launches of one step:
# one ncu capture at batch 2 (826.2 MB read + written over 21 launches), scaled by 4 to
# the 8 images of a step here (traffic grows with the images processed).  Writes of the
# small octaves stay in L2 past the kernel's end, so this under-counts writes.
NCU_TRAFFIC_BLUR_LEVEL = 4 * 826.17e6 / 21


def peaks(key="hbm_gbs"):
    """Measured peak (HBM copy GB/s or cuBLAS bf16 TFLOP/s) and its kind; the
    pool's earlier measurement when the measured file is absent."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p[key]), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}[key], "fallback"


class ClockSampler:
    """nvidia-smi samples (200 ms) during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        time.sleep(0.25)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def make_images(n: int, seed0: int = 1, seeds=None):
    seeds = list(seeds) if seeds is not None else [seed0 + i for i in range(n)]
    return [synth.blob_image(WIDTH, HEIGHT, 2000, 1.5, 20.0, seed=sd) for sd in seeds[:n]]


def pyramid_bytes_per_image(h: int, w: int) -> tuple[float, int]:
    """Algorithmic HBM bytes of the pyramid stage for one image, and its launch count.

    Octave-0 base: read u8 image (W*H), write G0 (4 B/px).  Each blur level:
    read G[s-1], write G[s], write D[s-1] (12 B/px); the level that seeds the
    next octave also writes its base (4 B per next-octave px).
    """
    hh, ww = 2 * h, 2 * w
    total = float(h * w) + 4.0 * hh * ww
    launches = 1
    for o in range(OCTAVES):
        if hh < 3 or ww < 3:
            break
        p = hh * ww
        total += (SCALES + 2) * 12.0 * p
        launches += SCALES + 2
        nh, nw = hh // 2, ww // 2
        if o + 1 < OCTAVES and nh >= 3 and nw >= 3:
            total += 4.0 * nh * nw
        hh, ww = nh, nw
    return total, launches


def _blur_radius(sigma: float) -> int:
    # gaussian_kernel_1d's radius: ceil(3 sigma), at least 1 (f32 on the host)
    cs = float(np.float32(max(sigma, 1e-3)))
    return max(1, int(np.ceil(np.float32(3.0) * np.float32(cs))))


def pyramid_fp32_ops_per_image(h: int, w: int) -> tuple[float, float]:
    """FP32 lane operations of the pyramid stage for one image: (reference rounding,
    single rounding).  Each blur tap is a rounded multiply and a rounded add (one
    fused multiply-add in the single-rounding mode); the horizontal pass of a 64 x 64
    tile also covers the 2R halo rows, so it costs (64 + 2R) / 64 of the vertical
    one; the DoG is one subtraction per pixel; the octave base adds the bilinear
    upsampling's three adds and a multiply.  Radii of the schedule's incremental
    sigmas (base 1.6, the input's 0.5 doubled by the upsampling)."""
    k = np.float32(2.0) ** (np.float32(1.0) / np.float32(SCALES))
    radii, prev = [], np.float32(1.6)
    for s in range(1, SCALES + 3):
        target = np.float32(1.6) * k ** s
        radii.append(_blur_radius(np.sqrt(max(target * target - prev * prev, 1e-4))))
        prev = target
    r0 = _blur_radius(np.sqrt(max(1.6 * 1.6 - 1.0, 1e-4)))

    def per_px(r: int, fused: bool) -> float:
        taps = 2 * r + 1
        per_tap = 1.0 if fused else 2.0
        return per_tap * taps * (64 + 2 * r) / 64 + per_tap * taps

    ref = fused = 0.0
    hh, ww = 2 * h, 2 * w
    ref += hh * ww * (per_px(r0, False) + 4.0)
    fused += hh * ww * (per_px(r0, True) + 4.0)
    for o in range(OCTAVES):
        if hh < 3 or ww < 3:
            break
        for r in radii:
            ref += hh * ww * (per_px(r, False) + 1.0)
            fused += hh * ww * (per_px(r, True) + 1.0)
        hh, ww = hh // 2, ww // 2
    return ref, fused


def cpu_reference(steps: int, warmup: int, budget_s: float):
    """Time the CPU restatement (OpenMP over all host cores) on 1080p images."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    img = O.luma_to_f32(make_images(1, 0)[0])
    for _ in range(warmup):
        O.detect_and_compute(img, OCTAVES, SCALES, THRESH, True, 0, MAX_FEATURES)
    t0 = time.perf_counter()
    n = 0
    while n < steps and (time.perf_counter() - t0) < budget_s:
        O.detect_and_compute(img, OCTAVES, SCALES, THRESH, True, 0, MAX_FEATURES)
        n += 1
    dt = time.perf_counter() - t0
    return n / dt, n, dt, os.cpu_count()


def match_bench(ctx, torch, n_pairs: int = 32, n: int = 4096, reps: int = 5):
    """Pair matching, BF16 tensor-core + certified re-rank vs the exact FP32 kernel.

    32 pairs of 4096 x 4096 SIFT-like descriptors (|N(0,1)| normalised, clipped at
    0.2, renormalised; one third of the queries are perturbed copies of targets),
    ratio 0.8, all pairs in one batched call; device-resident inputs.
    """
    import psift
    qs, ts, qxy, txy, outs, counts = [], [], [], [], [], []
    for p in range(n_pairs):
        t = synth.sift_like_descriptors(n, 50_000 + p)
        q = synth.sift_like_descriptors(n, 60_000 + p)
        k = n // 3
        q[:k] = t[:k] + 0.02 * synth.sift_like_descriptors(k, 70_000 + p)
        qs.append(torch.from_numpy(q).cuda())
        ts.append(torch.from_numpy(t).cuda())
        xy = torch.rand((n, 2), device="cuda") * 1000
        qxy.append(xy)
        txy.append(xy.clone())
        outs.append(torch.zeros((n, 10), dtype=torch.float32, device="cuda"))
        counts.append(torch.zeros(1, dtype=torch.int32, device="cuda"))
    jobs = (psift.CMatchJob * n_pairs)(*[psift.CMatchJob(qs[i].data_ptr(), ts[i].data_ptr(), qxy[i].data_ptr(),
                                                         txy[i].data_ptr(), n, n, outs[i].data_ptr(), n,
                                                         counts[i].data_ptr()) for i in range(n_pairs)])
    stream = torch.cuda.ExternalStream(ctx.stream)
    res = {}
    lists = {}
    for name, prec in (("fp32", psift.PRECISION_FP32), ("bf16_rerank", psift.PRECISION_BF16_RERANK)):
        opt = psift.MatchOptions(0.8, False, prec).to_c()
        call = lambda: ctx.check(ctx.lib.psift_match_batch_dev(ctx.handle, jobs, n_pairs, C.byref(opt)))
        for _ in range(2):
            call()
        ctx.synchronize()
        fb0 = C.c_uint64()
        ctx.check(ctx.lib.psift_ctx_rerank_fallbacks(ctx.handle, C.byref(fb0)))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            call()
        e1.record(stream)
        ctx.synchronize()
        ms = e0.elapsed_time(e1) / reps
        res[name] = ms / n_pairs
        fb1 = C.c_uint64()
        ctx.check(ctx.lib.psift_ctx_rerank_fallbacks(ctx.handle, C.byref(fb1)))
        if name == "bf16_rerank":
            res["fallback_rows_per_call"] = (fb1.value - fb0.value) / reps
        lists[name] = [(int(c.item()), outs[i][: int(c.item())].cpu().numpy().tobytes()) for i, c in enumerate(counts)]
    flops = 2.0 * n * n * 128
    return {
        "workload": f"{n_pairs} pairs of {n}x{n} SIFT-like descriptors, ratio 0.8, one batched call",
        "fp32_ms_per_pair": res["fp32"], "bf16_rerank_ms_per_pair": res["bf16_rerank"],
        "speedup_bf16_vs_fp32": res["fp32"] / res["bf16_rerank"],
        "identical_match_lists": lists["fp32"] == lists["bf16_rerank"],
        "matches_per_pair": lists["fp32"][0][0],
        "bf16_tflops_effective": flops / (res["bf16_rerank"] * 1e-3) / 1e12,
        "rerank_exact_scan_rows_per_call": res["fallback_rows_per_call"],
    }


def _uneven_pair(k):
    sys.path.insert(0, os.path.join(ROOT, "pure-sift_b200"))
    import synth as S
    return S.uneven_pair(k)


def uneven_bench(ctx, torch, n_pairs: int = 32, reps: int = 3):
    """Uneven batch: 64 images (32 pairs A_i, B_i = perspective warp of A_i), widths
    U(480, 3840), aspect U(0.5, 2), blobs in proportion to area (6000 per 1080p
    area, synth.uneven_pair); SiftConfig octaves 4,
    threshold 0.015, upsampling, uncapped features.  All 64 images in one device
    batch call (one launch per stage; CUDA-graph replay), then the 32 pairs matched
    in one call with the exact FP32 kernel and with BF16 + certified re-rank."""
    import multiprocessing as mp
    import psift
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        pairs = pool.map(_uneven_pair, range(n_pairs))
    imgs = [im for ab in pairs for im in ab]
    B = len(imgs)
    cap = 65536
    d_imgs = [torch.from_numpy(im).cuda() for im in imgs]
    outs = [{k: torch.empty(cap, dtype=torch.float32, device="cuda") for k in "xysro"} for _ in range(B)]
    for o in outs:
        o["d"] = torch.empty((cap, 128), dtype=torch.float32, device="cuda")
    counts = torch.zeros(B, dtype=torch.int32, device="cuda")
    ccfg = psift.SiftConfig().with_octaves(OCTAVES).with_scales(SCALES).with_contrast_threshold(THRESH) \
        .max_features(0).to_c()
    cimgs = (psift.CImageU8 * B)(*[psift.CImageU8(t.data_ptr(), t.shape[0], t.shape[1], t.shape[1]) for t in d_imgs])
    couts = (psift.CFeatures * B)(*[psift.CFeatures(cap, 0, o["x"].data_ptr(), o["y"].data_ptr(), o["s"].data_ptr(),
                                                    o["r"].data_ptr(), o["o"].data_ptr(), o["d"].data_ptr())
                                    for o in outs])
    stream = torch.cuda.ExternalStream(ctx.stream)
    run = lambda: ctx.check(ctx.lib.psift_detect_and_compute_batch_dev(ctx.handle, cimgs, B, C.byref(ccfg), couts,
                                                                      C.c_void_p(counts.data_ptr())))
    for _ in range(2):
        run()
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        run()
    e1.record(stream)
    ctx.synchronize()
    det_ms = e0.elapsed_time(e1) / reps
    cnt = counts.cpu().numpy().astype(np.int64)
    mpx = sum(im.size for im in imgs) / 1e6
    # match A_i against B_i, all pairs in one call
    mouts = [torch.zeros((int(max(cnt[2 * i], 1)), 10), dtype=torch.float32, device="cuda") for i in range(n_pairs)]
    mcounts = [torch.zeros(1, dtype=torch.int32, device="cuda") for _ in range(n_pairs)]
    xy = [torch.stack([o["x"], o["y"]], dim=1).contiguous() for o in outs]
    jobs = (psift.CMatchJob * n_pairs)(*[psift.CMatchJob(outs[2 * i]["d"].data_ptr(), outs[2 * i + 1]["d"].data_ptr(),
                                                         xy[2 * i].data_ptr(), xy[2 * i + 1].data_ptr(),
                                                         int(cnt[2 * i]), int(cnt[2 * i + 1]),
                                                         mouts[i].data_ptr(), mouts[i].shape[0],
                                                         mcounts[i].data_ptr()) for i in range(n_pairs)])
    res, lists = {}, {}
    for name, prec in (("fp32", psift.PRECISION_FP32), ("bf16_rerank", psift.PRECISION_BF16_RERANK)):
        opt = psift.MatchOptions(0.8, False, prec).to_c()
        call = lambda: ctx.check(ctx.lib.psift_match_batch_dev(ctx.handle, jobs, n_pairs, C.byref(opt)))
        call()
        ctx.synchronize()
        e0.record(stream)
        call()
        e1.record(stream)
        ctx.synchronize()
        res[name] = e0.elapsed_time(e1)
        lists[name] = [mouts[i][: int(mcounts[i].item())].cpu().numpy().tobytes() for i in range(n_pairs)]
    flops = sum(2.0 * cnt[2 * i] * cnt[2 * i + 1] * 128 for i in range(n_pairs))
    return {
        "workload": f"{B} images (widths U(480,3840), aspect U(0.5,2), {mpx:.0f} Mpx total), uncapped; "
                    f"{n_pairs} pairs A_i vs warp(A_i), ratio 0.8",
        "detect_ms_batch": det_ms, "detect_images_per_s": B / (det_ms * 1e-3),
        "detect_mpx_per_s": mpx / (det_ms * 1e-3),
        "features_per_image": {"min": int(cnt.min()), "median": int(np.median(cnt)), "max": int(cnt.max()),
                               "fraction_within_4k_20k": float(((cnt >= 4000) & (cnt <= 20000)).mean())},
        "match_fp32_ms_32_pairs": res["fp32"], "match_bf16_rerank_ms_32_pairs": res["bf16_rerank"],
        "match_speedup_bf16_vs_fp32": res["fp32"] / res["bf16_rerank"],
        "identical_match_lists": lists["fp32"] == lists["bf16_rerank"],
        "matches_total": int(sum(int(m.item()) for m in mcounts)),
        "bf16_tflops_effective": flops / (res["bf16_rerank"] * 1e-3) / 1e12,
    }


def catalog_bench(ctx, torch, n_cat: int = 2_000_000, n_q: int = 4096, k: int = 64, reps: int = 5):
    """Catalog search: 2M SIFT-like catalog descriptors (10,000 images x 200;
    |N(0,1)| L2-normalised, clipped at 0.2, renormalised), binarised to 128-bit
    codes by the reference's scheme (bit i = desc[i] > 0.065), 4096 queries
    (perturbed catalog descriptors), XOR+POPCNT top-64 shortlist, exact FP32
    L2 re-rank of the 64.  Device-resident inputs; CUDA events per stage."""
    import psift
    g = torch.Generator(device="cuda")
    g.manual_seed(4)
    cat = torch.randn((n_cat, 128), generator=g, device="cuda").abs_()
    cat /= cat.norm(dim=1, keepdim=True)
    cat.clamp_(max=0.2)
    cat /= cat.norm(dim=1, keepdim=True)
    pick = torch.randint(0, n_cat, (n_q,), generator=g, device="cuda")
    q = cat[pick] + 0.02 * torch.randn((n_q, 128), generator=g, device="cuda").abs_()
    q /= q.norm(dim=1, keepdim=True)
    cat_codes = torch.empty((n_cat, 2), dtype=torch.int64, device="cuda")
    q_codes = torch.empty((n_q, 2), dtype=torch.int64, device="cuda")
    idx = torch.empty((n_q, k), dtype=torch.int32, device="cuda")
    dist = torch.empty((n_q, k), dtype=torch.int32, device="cuda")
    ridx = torch.empty((n_q, k), dtype=torch.int32, device="cuda")
    rd2 = torch.empty((n_q, k), dtype=torch.float32, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream)
    L = ctx.lib
    steps = {
        "quantize": lambda: ctx.check(L.psift_quantize_u128_dev(ctx.handle, C.c_void_p(cat.data_ptr()), n_cat,
                                                                 C.c_void_p(cat_codes.data_ptr()))),
        "topk": lambda: ctx.check(L.psift_hamming_topk_dev(ctx.handle, C.c_void_p(q_codes.data_ptr()), n_q,
                                                           C.c_void_p(cat_codes.data_ptr()), n_cat, k,
                                                           C.c_void_p(idx.data_ptr()), C.c_void_p(dist.data_ptr()))),
        "rerank": lambda: ctx.check(L.psift_l2_rerank_dev(ctx.handle, C.c_void_p(q.data_ptr()), n_q,
                                                          C.c_void_p(cat.data_ptr()), C.c_void_p(idx.data_ptr()), k,
                                                          C.c_void_p(ridx.data_ptr()), C.c_void_p(rd2.data_ptr()))),
    }
    ctx.check(L.psift_quantize_u128_dev(ctx.handle, C.c_void_p(q.data_ptr()), n_q, C.c_void_p(q_codes.data_ptr())))
    ms = {}
    for name, fn in steps.items():
        fn()
        ctx.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        ctx.synchronize()
        ms[name] = e0.elapsed_time(e1) / reps
    peak = C.c_double()
    ctx.check(L.psift_popc_throughput(ctx.handle, C.byref(peak)))
    pairs = float(n_q) * n_cat
    popc_s = pairs * 3 / (ms["topk"] * 1e-3)  # three popcounts per pair (carry-save step)
    # the query's own (perturbed) source descriptor should be found by the shortlist
    hit = float((idx == pick[:, None].int()).any(dim=1).float().mean().item())
    # outside the timed region: the whole top-64 and the re-rank against the CPU
    # restatement (OpenMP), bit for bit
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    hq = q_codes.cpu().numpy().view(np.uint64)
    hc = cat_codes.cpu().numpy().view(np.uint64)
    t_cpu = time.perf_counter()
    ci, cd = O.hamming_topk(hq, hc, k)
    cpu_topk_s = time.perf_counter() - t_cpu
    gi, gd = idx.cpu().numpy().view(np.uint32), dist.cpu().numpy().view(np.uint32)
    topk_exact = bool(np.array_equal(ci, gi) and np.array_equal(cd, gd))
    ri, rd = O.l2_rerank(q.cpu().numpy(), cat.cpu().numpy(), ci)
    rerank_exact = bool(np.array_equal(ri, ridx.cpu().numpy().view(np.uint32)) and
                        np.array_equal(rd.view(np.uint32), rd2.cpu().numpy().view(np.uint32)))
    return {
        "workload": f"{n_cat} catalog codes ({n_cat // 200:,} images x 200), {n_q} queries, top-{k} XOR+POPCNT shortlist "
                    f"+ exact FP32 L2 re-rank",
        "ms": {"quantize_2M": ms["quantize"], "topk": ms["topk"], "l2_rerank": ms["rerank"],
               "search_total": ms["topk"] + ms["rerank"]},
        "topk_pairs_per_s": pairs / (ms["topk"] * 1e-3),
        "roofline_topk": {"bound": "int (popc)", "achieved": popc_s, "peak": peak.value, "unit": "popc/s",
                          "frac": popc_s / peak.value, "popc_per_pair": 3,
                          "peak_source": "this library's own probe kernel psift_popc_throughput (popc+xor+add register "
                                         "chains); the measured-peaks file has no integer peak"},
        "quantize_gbs": n_cat * 512 / (ms["quantize"] * 1e-3) / 1e9,
        "source_in_shortlist": hit,
        "bit_exact_vs_cpu": {"topk": topk_exact, "l2_rerank": rerank_exact,
                             "cpu": f"CPU restatement, OpenMP {os.cpu_count()} threads, {cpu_topk_s:.1f} s for the top-k"},
    }


def _psiftcat_bytes(meta, codes, q, per_entry: int, w: int, h: int) -> bytes:
    """PSIFTCAT v1 file (FeatureCatalog::save_binary layout, src/catalog.rs:401-445)
    of len(meta) // per_entry entries named img00000, img00001, ..."""
    import struct
    n = len(meta)
    rec = np.zeros(n, np.dtype([("m", "<f4", 5), ("c", "<u8", 2), ("q", "u1", 128)]))
    rec["m"], rec["c"], rec["q"] = meta, codes, q
    raw = rec.tobytes()
    parts = [b"PSIFTCAT", struct.pack("<IIIfBQ", 1, 4, 3, 0.015, 0, n // per_entry)]
    for e in range(n // per_entry):
        ib = f"img{e:05d}".encode()
        parts.append(struct.pack("<I", len(ib)) + ib + struct.pack("<IIQ", w, h, per_entry))
        parts.append(raw[e * per_entry * 164:(e + 1) * per_entry * 164])
    return b"".join(parts)


def catalog_search_bench(ctx, torch, n_entries: int = 10_000, per_entry: int = 200, n_q: int = 4096,
                         reps: int = 10):
    """Device-resident catalog: a PSIFTCAT v1 file of 10,000 entries x 200 features
    (C4-style descriptors stored as the reference's u8 quantisation, codes of the
    f32 descriptors) is loaded into device memory, then search_features (top 5,
    shortlist 16, ratio 0.75, RANSAC 3 px) runs for a 4096-feature query whose
    first 200 features are the target entry's, perturbed and moved by a
    similarity (the rest are random).  Host API timing (wall clock of the call)."""
    import tempfile
    import psift
    rng = np.random.default_rng(21)
    n = n_entries * per_entry
    d = np.abs(rng.standard_normal((n, 128), dtype=np.float32))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    np.minimum(d, 0.2, out=d)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    q8 = np.clip(np.rint(d * 512.0), 0, 255).astype(np.uint8)
    codes = np.zeros((n, 2), np.uint64)
    bits = (d > 0.065)
    for wd in range(2):
        blk = bits[:, 64 * wd:64 * wd + 64].astype(np.uint64)
        codes[:, wd] = (blk << np.arange(64, dtype=np.uint64)).sum(axis=1, dtype=np.uint64)
    meta = np.zeros((n, 5), np.float32)
    meta[:, 0] = rng.uniform(0, 1920, n)
    meta[:, 1] = rng.uniform(0, 1080, n)
    meta[:, 2] = rng.uniform(1.6, 12.0, n)
    meta[:, 3] = rng.uniform(0.01, 0.1, n)
    meta[:, 4] = rng.uniform(0, 2 * np.pi, n)
    blob = _psiftcat_bytes(meta, codes, q8, per_entry, 1920, 1080)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "catalog.psiftcat")
        with open(path, "wb") as fh:
            fh.write(blob)
        psift.DeviceCatalog.load_binary(path, ctx).close()  # warm: page cache, allocations
        t0 = time.perf_counter()
        cat = psift.DeviceCatalog.load_binary(path, ctx)
        load_s = time.perf_counter() - t0
    target = 1234
    tf, _ = cat.entry_features(target)
    th = np.deg2rad(10.0)
    qx = 1.1 * (np.cos(th) * tf.x - np.sin(th) * tf.y) + 30.0
    qy = 1.1 * (np.sin(th) * tf.x + np.cos(th) * tf.y) - 20.0
    qd = np.abs(rng.standard_normal((n_q, 128), dtype=np.float32))
    qd[:per_entry] = tf.descriptors + 0.01 * np.abs(rng.standard_normal((per_entry, 128), dtype=np.float32))
    qd /= np.linalg.norm(qd, axis=1, keepdims=True)
    query = psift.Features(np.r_[qx, rng.uniform(0, 1920, n_q - per_entry)].astype(np.float32),
                           np.r_[qy, rng.uniform(0, 1080, n_q - per_entry)].astype(np.float32),
                           np.r_[tf.scale * 1.1, rng.uniform(1.6, 12, n_q - per_entry)].astype(np.float32),
                           np.full(n_q, 0.05, np.float32),
                           np.r_[tf.orientation + th, rng.uniform(0, 6.28, n_q - per_entry)].astype(np.float32), qd)
    t0 = time.perf_counter()
    hits = cat.search_features(query)  # first search after the load builds the MIH tables
    build_s = time.perf_counter() - t0
    hits = cat.search_features(query)
    t0 = time.perf_counter()
    hits = cat.search_features(query)
    build_s -= time.perf_counter() - t0
    l0 = ctx.launch_count
    t0 = time.perf_counter()
    for _ in range(reps):
        hits = cat.search_features(query)
    search_s = (time.perf_counter() - t0) / reps
    launches = (ctx.launch_count - l0) / reps
    ctx.enable_stage_timing(True)
    ctx.stage_times(reset=True)
    for _ in range(reps):
        cat.search_features(query)
    stages = {k: v[0] / reps for k, v in ctx.stage_times(reset=True).items() if v[1]}
    # Coarse votes alone (device time of the votes launches, query codes given):
    # the MIH rule through the device tables vs every code scanned; the search
    # with the scan path for comparison.
    qcodes = psift.quantize_descriptor_u128(qd, ctx)
    votes_ms = {}
    for name, path in (("mih_index", psift.VOTES_MIH_INDEX), ("mih_scan", psift.VOTES_MIH_SCAN)):
        ref = cat.votes(qcodes, path)
        ctx.stage_times(reset=True)
        for _ in range(reps):
            got = cat.votes(qcodes, path)
        votes_ms[name] = ctx.stage_times(reset=True)["hamming"][0] / reps
        assert np.array_equal(got, ref)
    same_votes = bool(np.array_equal(cat.votes(qcodes, psift.VOTES_MIH_INDEX), cat.votes(qcodes, psift.VOTES_MIH_SCAN)))
    # Pairs the MIH votes test: per band, queries x listed codes summed over the 256 keys.
    mih_pairs = 0
    for b in range(16):
        kc = ((codes[:, b // 8] >> np.uint64(8 * (b % 8))) & np.uint64(0xFF)).astype(np.int64)
        kq = ((qcodes[:, b // 8] >> np.uint64(8 * (b % 8))) & np.uint64(0xFF)).astype(np.int64)
        mih_pairs += int(np.dot(np.bincount(kc, minlength=256), np.bincount(kq, minlength=256)))
    ctx.enable_stage_timing(False)
    cat.set_search_votes(psift.VOTES_MIH_SCAN)
    t0 = time.perf_counter()
    for _ in range(reps):
        hits_scan = cat.search_features(query)
    search_scan_s = (time.perf_counter() - t0) / reps
    cat.set_search_votes(psift.VOTES_AUTO)
    same_hits = [(h.id, h.coarse_votes, h.tracking.match_count) for h in hits_scan] == \
                [(h.id, h.coarse_votes, h.tracking.match_count) for h in hits]
    cat.close()
    return {
        "workload": f"PSIFTCAT v1 catalog of {n_entries} entries x {per_entry} features ({len(blob) / 1e6:.0f} MB), "
                    f"{n_q}-feature query, top-5 / shortlist 16, host API wall clock",
        "load_binary_s": load_s, "load_binary_gbs": len(blob) / load_s / 1e9,
        "search_ms": search_s * 1e3, "launches_per_search": launches, "device_stage_ms_per_search": stages,
        "search_ms_votes_by_scan": search_scan_s * 1e3, "same_hits_either_votes_path": same_hits,
        "votes_device_ms": votes_ms, "same_votes_index_vs_scan": same_votes,
        "mih_pairs": mih_pairs, "scan_pairs": n_q * n,
        "mih_pairs_per_s": mih_pairs / (votes_ms["mih_index"] * 1e-3),
        "scan_pairs_per_s": n_q * n / (votes_ms["mih_scan"] * 1e-3),
        "mih_tables_build_s": build_s,
        "top_hit": hits[0].id if hits else None, "top_hit_inliers": hits[0].tracking.match_count if hits else 0,
        "expected_top_hit": f"img{target:05d}",
    }


def panorama_bench(ctx, torch, reps: int = 3):
    """stitch_panorama: four overlapping 1280x720 RGBA tiles of a synthetic colour
    field (three independent 2000-blob planes as R, G, B; tile step 900 px,
    exposures 0.9 / 1.0 / 1.1 / 0.95), multi-band blending with 4 levels and
    exposure compensation, through the host API (registration: detection,
    matching, RANSAC of the 6 pairs; compositing on the GPU); the compositing
    alone on the host API with the registration's results; the CPU restatement
    of both on the same tiles."""
    import psift
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    W, H, tile, step = 3980, 720, 1280, 900
    chans = [synth.blob_image(W, H, 4000, 1.5, 20.0, seed=s) for s in (91, 92, 93)]
    rgb = np.stack(chans, axis=-1).astype(np.float32)
    tiles = []
    for i, f in enumerate((0.9, 1.0, 1.1, 0.95)):
        v = np.clip(np.round(rgb[:, i * step:i * step + tile] * np.float32(f)), 0, 255).astype(np.uint8)
        tiles.append(np.concatenate([v, np.full(v.shape[:2] + (1,), 255, np.uint8)], axis=-1))
    opt = psift.PanoramaOptions.default()
    res = psift.stitch_panorama(tiles, opt, ctx=ctx)
    t0 = time.perf_counter()
    for _ in range(reps):
        res = psift.stitch_panorama(tiles, opt, ctx=ctx)
    full_s = (time.perf_counter() - t0) / reps
    reg = O.panorama_register(tiles, O.PanoramaOptions.default())
    comp = lambda: psift.panorama_composite(tiles, reg["registered"], reg["gains"], reg["inv"], reg["origin"],
                                            reg["width"], reg["height"], 1, 4, ctx=ctx)
    comp()
    t0 = time.perf_counter()
    for _ in range(reps):
        got = comp()
    comp_s = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    want = O.panorama_composite(tiles, reg, 1, 4)
    cpu_comp_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.panorama_register(tiles, O.PanoramaOptions.default())
    cpu_reg_s = time.perf_counter() - t0
    h, w = res.image.shape[:2]
    return {"workload": "4 overlapping 1280x720 RGBA tiles (synthetic colour field), multi-band 4 levels, "
                        "exposure compensation", "canvas": [w, h], "registered": len(res.registered_indices),
            "stitch_host_api_ms": full_s * 1e3, "composite_host_api_ms": comp_s * 1e3,
            "composite_mpx_per_s": w * h / comp_s / 1e6,
            "cpu_restatement_ms": {"registration": cpu_reg_s * 1e3, "composite": cpu_comp_s * 1e3},
            "composite_identical_to_restatement": bool(np.array_equal(got, want))}


def warp_bench(ctx, torch, reps: int = 50):
    """warp_and_stitch on a 1080p RGBA pair: the query warped by a C2-style
    homography (rotation, scale, perspective about the centre) onto the target's
    frame, feather-blended.  Device variant timed with CUDA events; host API
    (uploads and canvas download included) by wall clock; the CPU restatement
    (OpenMP, all host threads) on the same pair."""
    import psift
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    rng = np.random.default_rng(31)
    W, H = 1920, 1080
    q = rng.integers(0, 256, (H, W, 4)).astype(np.uint8)
    t = rng.integers(0, 256, (H, W, 4)).astype(np.uint8)
    th = np.deg2rad(8.0)
    A = np.array([[1.05 * np.cos(th), -1.05 * np.sin(th), 0], [1.05 * np.sin(th), 1.05 * np.cos(th), 0],
                  [4e-5, -3e-5, 1]])
    C0 = np.array([[1, 0, -W / 2], [0, 1, -H / 2], [0, 0, 1]])
    C1 = np.array([[1, 0, W / 2 + 60], [0, 1, H / 2 - 40], [0, 0, 1]])
    Hm = (C1 @ A @ C0).astype(np.float32)
    h9 = np.ascontiguousarray(Hm.reshape(9))
    canvas, origin = psift.warp_and_stitch(q, t, Hm, ctx)
    dq, dt = torch.from_numpy(q).cuda(), torch.from_numpy(t).cuda()
    out = torch.empty(canvas.size, dtype=torch.uint8, device="cuda")
    w, h = C.c_uint32(), C.c_uint32()
    stream = torch.cuda.ExternalStream(ctx.stream)

    def run():
        ctx.check(ctx.lib.psift_warp_and_stitch_dev(ctx.handle, C.c_void_p(dq.data_ptr()), H, W, 4 * W,
                                                    C.c_void_p(dt.data_ptr()), H, W, 4 * W, h9.ctypes.data,
                                                    C.c_void_p(out.data_ptr()), out.numel(), C.byref(w),
                                                    C.byref(h)))
    torch.cuda.synchronize()
    for _ in range(3):
        run()
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        run()
    e1.record(stream)
    ctx.synchronize()
    dev_ms = e0.elapsed_time(e1) / reps
    same = bool(np.array_equal(out.cpu().numpy().reshape(canvas.shape), canvas))
    t0 = time.perf_counter()
    for _ in range(5):
        psift.warp_and_stitch(q, t, Hm, ctx)
    host_ms = (time.perf_counter() - t0) / 5 * 1e3
    t0 = time.perf_counter()
    ref, _ = O.warp_and_stitch(q, t, Hm)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    px = canvas.shape[0] * canvas.shape[1]
    algo = 4 * px + 4 * q.shape[0] * q.shape[1] + 4 * t.shape[0] * t.shape[1]
    peak, _ = peaks()
    return {
        "workload": f"1080p RGBA query warped onto a 1080p RGBA target, canvas {canvas.shape[1]}x{canvas.shape[0]}",
        "device_ms": dev_ms, "canvas_mpx_per_s": px / (dev_ms * 1e-3) / 1e6,
        "roofline": {"bound": "hbm", "achieved": algo / (dev_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": algo / (dev_ms * 1e-3) / 1e9 / peak,
                     "algorithmic_bytes": algo, "note": "canvas write + each source texel once"},
        "host_api_ms": host_ms, "cpu_restatement_ms": cpu_ms, "cpu_threads": os.cpu_count(),
        "identical_to_restatement": same and bool(np.array_equal(ref, canvas)),
    }


def fundamental_bench(ctx, torch, n_sets: int = 256, cpu_sample: int = 8):
    """Fundamental-matrix LO-RANSAC over 256 two-view match sets (1920x1080 views
    of a 3-D scene, 2k-8k matches, outlier ratio U(0.1, 0.6)), one launch; the
    CPU restatement (one thread per set, as the reference runs it) on the first
    8 sets, scaled to the 256, and their inlier sets compared."""
    import psift
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    sets = []
    for k in range(n_sets):
        u = synth.SplitMix64(9000 + k).uniform(2)
        sets.append(synth.epipolar_matches(int(2000 + 6000 * u[0]), 0.1 + 0.5 * u[1], seed=9100 + k)[0])
    psift.fundamental_batch(sets[:4], ctx=ctx)  # warm-up
    res, dev_ms = psift.fundamental_batch(sets, ctx=ctx, timing=True)
    t0 = time.perf_counter()
    ref = [O.fundamental_ransac(m) for m in sets[:cpu_sample]]
    cpu_s = time.perf_counter() - t0
    same = all(np.array_equal(r[0], g[0]) and r[2] == g[2] for r, g in zip(ref, res[:cpu_sample]))
    n_matches = int(sum(len(m) for m in sets))
    iters = [g[2] for g in res]
    return {
        "workload": f"{n_sets} two-view sets, 2k-8k matches ({n_matches} total), outliers U(0.1, 0.6), one launch",
        "device_ms": dev_ms, "sets_per_s": n_sets / (dev_ms * 1e-3),
        "mean_iterations": float(np.mean(iters)), "max_iterations": int(np.max(iters)),
        "cpu_restatement_ms_per_set": cpu_s / cpu_sample * 1e3,
        "cpu_restatement_ms_256_sets_one_thread": cpu_s / cpu_sample * n_sets * 1e3,
        "identical_on_cpu_sample": same,
    }


def ransac_bench(ctx, torch, n_pairs: int = 1024, n_train: int = 64, reps: int = 3):
    """Learned RANSAC proposal: 1024 synthetic 1080p pairs with known perspective
    homographies, 2k-8k putative matches each, outlier ratio U(0.1, 0.7).  The MLP
    (8-64-64-1) is trained on the GPU on plain-RANSAC labels of 64 other pairs,
    then plain (uniform) and guided (MLP-weighted) homography RANSAC run over the
    1024 pairs in one launch each; iterations, ms, and inlier counts compared."""
    import psift
    train = [synth.c5_pair(k) for k in range(5000, 5000 + n_train)]
    pairs = [synth.c5_pair(k) for k in range(n_pairs)]
    labels = psift.ransac_batch([r for r, _, _ in train], ctx=ctx)
    X = np.concatenate([f for _, f, _ in train])
    Y = np.concatenate([m for m, _, _ in labels]).astype(np.float32)
    mlp = psift.InlierMLP(seed=11)
    t0 = time.perf_counter()
    mlp.train(X, Y, steps=400, batch=4096, lr=3e-3, seed=12, ctx=ctx)
    train_s = time.perf_counter() - t0
    feats = np.concatenate([f for _, f, _ in pairs])
    t0 = time.perf_counter()
    probs_all = np.clip(mlp.predict(feats, ctx=ctx), 0.02, 1.0)
    infer_s = time.perf_counter() - t0
    offs = np.cumsum([0] + [len(f) for _, f, _ in pairs])
    probs = [probs_all[offs[i]:offs[i + 1]] for i in range(n_pairs)]
    stream = torch.cuda.ExternalStream(ctx.stream)
    # device-resident inference (psift_mlp_infer_dev), CUDA events on the context's stream
    feats_d = torch.from_numpy(feats).cuda()
    params_d = torch.from_numpy(np.ascontiguousarray(mlp.params, dtype=np.float32)).cuda()
    prob_d = torch.empty(feats.shape[0], device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    infer = lambda: ctx.check(ctx.lib.psift_mlp_infer_dev(ctx.handle, params_d.data_ptr(), feats_d.data_ptr(),
                                                           feats.shape[0], prob_d.data_ptr()))
    infer()
    ctx.synchronize()
    i0, i1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    i0.record(stream)
    for _ in range(reps):
        infer()
    i1.record(stream)
    ctx.synchronize()
    infer_dev_ms = i0.elapsed_time(i1) / reps
    out = {}
    for name, w in (("plain", None), ("guided", probs)):
        jobs, keep = psift.ransac_jobs([r for r, _, _ in pairs], weights=w)
        opt = psift.RansacOptions().to_c()
        launch = lambda: ctx.check(ctx.lib.psift_ransac_batch_dev(ctx.handle, jobs, n_pairs, C.byref(opt), 1))
        launch()
        ctx.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            launch()
        e1.record(stream)
        ctx.synchronize()
        res = psift.ransac_results(keep, homography=True)
        out[name] = {"ms": e0.elapsed_time(e1) / reps,
                     "inliers": np.array([m.sum() for m, _, _ in res]),
                     "iters": np.array([it[1] for _, _, it in res])}
    p, gd = out["plain"], out["guided"]
    ok = gd["inliers"] >= np.floor(0.99 * p["inliers"])
    return {
        "workload": f"{n_pairs} pairs, 2k-8k matches, outlier ratio U(0.1,0.7); MLP trained on {n_train} other pairs",
        "plain_ms": p["ms"], "guided_ms": gd["ms"], "speedup": p["ms"] / gd["ms"],
        "plain_mean_iterations": float(p["iters"].mean()), "guided_mean_iterations": float(gd["iters"].mean()),
        "plain_total_inliers": int(p["inliers"].sum()), "guided_total_inliers": int(gd["inliers"].sum()),
        "pairs_guided_within_1pct_of_plain": float(ok.mean()),
        "mlp_train_s_400_steps": train_s, "mlp_infer_host_api_ms_all_matches": infer_s * 1e3,
        "mlp_infer_device_ms_all_matches": infer_dev_ms,
        "guided_plus_device_inference_ms": gd["ms"] + infer_dev_ms,
        "speedup_with_inference": p["ms"] / (gd["ms"] + infer_dev_ms),
        "matches_total": int(offs[-1]),
    }


def pyramid_bench(ctx, torch, blur: str = "reference", reps: int = 5, variant: int | None = None):
    """One 1080p image through psift.build_pyramid (the gaussian_blur chain, DoG and
    decimation of build_scale_space_pyramid_with_options, 4 octaves with the 2x
    upsampled base): device time of the call's launches with CUDA events on the
    context's stream, host wall clock with the planes' download; the rounding mode
    of the blur taps as given.  Also the profiling case of the level blur (the
    first launch per octave of each radius, e.g. the R = 10 level of octave 0).  With
    `variant`, every radius runs that level-blur variant (3 = TMA tiles)."""
    import psift
    img = synth.blob_image(WIDTH, HEIGHT, 2000, 1.5, 20.0, seed=7).astype(np.float32) / 255.0
    cfg = psift.SiftConfig().with_octaves(4).with_contrast_threshold(0.015)
    ctx.set_blur_rounding(ctx.BLUR_FUSED if blur == "fused" else ctx.BLUR_REFERENCE)
    if variant is not None:
        for r in range(1, 16):
            ctx.set_tuning(ctx.TUNE_BLUR, r, variant)
    try:
        for _ in range(2):
            psift.build_pyramid(img, cfg, ctx=ctx)
        stream = torch.cuda.ExternalStream(ctx.stream)
        ctx.enable_stage_timing(True)
        ctx.stage_times(reset=True)
        t0 = time.perf_counter()
        for _ in range(reps):
            psift.build_pyramid(img, cfg, ctx=ctx)
        wall = (time.perf_counter() - t0) / reps
        st = ctx.stage_times(reset=True)
        ctx.enable_stage_timing(False)
    finally:
        ctx.set_blur_rounding(ctx.BLUR_REFERENCE)
    del stream
    return {"workload": f"{WIDTH}x{HEIGHT} blob image, 4 octaves, scales 3, upsampled base (3840x2160 octave 0)",
            "blur": blur, "blur_variant": "autotuner default" if variant is None else variant,
            "device_pyramid_ms": st["pyramid"][0] / reps, "host_api_ms_with_download": wall * 1e3}


def png_bench(ctx, torch, n: int = 8, reps: int = 10):
    """Input step, PNG: 8 colour 1920x1080 PNGs (the JPEG section's images, written
    by PIL at its default compression, adaptive row filters) in host memory ->
    features in host memory through psift_detect_and_compute_png_batch (inflate on
    host threads, row filters and luma on the GPU into the batch's inputs), against
    the host u8 batch entry given the decoded luma, and the CPU decode (PIL + the
    image crate's luma formula, one thread) per image."""
    import io
    from PIL import Image
    import psift
    rgbs = [np.stack([synth.blob_image(WIDTH, HEIGHT, 2000, 1.5, 20.0, seed=900 + 3 * i + k) for k in range(3)],
                     axis=2) for i in range(n)]
    blobs = []
    for im in rgbs:
        buf = io.BytesIO()
        Image.fromarray(im).save(buf, format="PNG")
        blobs.append(buf.getvalue())
    sift = psift.Sift.new(psift.SiftConfig().with_octaves(4).with_contrast_threshold(0.015))
    outs = [psift.Features.pinned(4096, ctx) for _ in range(n)]
    for _ in range(2):
        sift.detect_and_compute_png_batch(blobs, outs=outs, ctx=ctx)
    t0 = time.perf_counter()
    for _ in range(reps):
        sift.detect_and_compute_png_batch(blobs, outs=outs, ctx=ctx)
    png_s = (time.perf_counter() - t0) / reps
    lumas = [psift.decode_png_luma(b, ctx=ctx) for b in blobs]
    t0 = time.perf_counter()
    for _ in range(reps):
        for b in blobs:
            psift.decode_png_luma(b, ctx=ctx)
    dec_s = (time.perf_counter() - t0) / reps / n
    t0 = time.perf_counter()
    for _ in range(reps):
        sift.detect_and_compute_batch_u8(lumas, outs=outs, ctx=ctx)
    u8_s = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    cpu = []
    for b in blobs[:2]:
        rgb = np.asarray(Image.open(io.BytesIO(b)).convert("RGB")).astype(np.uint32)
        cpu.append(((2126 * rgb[:, :, 0] + 7152 * rgb[:, :, 1] + 722 * rgb[:, :, 2]) // 10000).astype(np.uint8))
    cpu_s = (time.perf_counter() - t0) / 2
    return {
        "workload": f"{n} colour {WIDTH}x{HEIGHT} PNGs (PIL, default compression, {sum(map(len, blobs)) // n // 1024} KB "
                    "each), host bytes -> pinned host features, host API wall clock",
        "png_images_per_s": n / png_s, "u8_batch_images_per_s": n / u8_s,
        "png_minus_u8_input_ms_per_batch": (png_s - u8_s) * 1e3,
        "decode_png_luma_ms_per_image_host_api": dec_s * 1e3,
        "cpu_decode_ms_per_image_1_thread": cpu_s * 1e3,
        "luma_equal_to_cpu_decode": all(np.array_equal(c, l) for c, l in zip(cpu, lumas[:2])),
    }


def jpeg_bench(ctx, torch, n: int = 8, reps: int = 20):
    """Input step: 8 colour 1920x1080 JPEGs (three independent 2000-blob fields as
    R, G, B; 4:2:0, quality 90) in host memory -> features in host memory through
    psift_detect_and_compute_jpeg_batch (nvJPEG: Huffman stage on host threads, the
    rest on the GPU, into the batch's inputs), against the host u8 batch entry given
    the already decoded luma, and the CPU decode (PIL + the image crate's luma
    formula, one thread) per image; also 64-image batches and the single-call mode."""
    import io
    from PIL import Image
    import psift
    rgbs = [np.stack([synth.blob_image(WIDTH, HEIGHT, 2000, 1.5, 20.0, seed=900 + 3 * i + k) for k in range(3)],
                     axis=2) for i in range(n)]
    blobs = []
    for im in rgbs:
        buf = io.BytesIO()
        Image.fromarray(im).save(buf, format="JPEG", quality=90, subsampling=2)
        blobs.append(buf.getvalue())
    sift = psift.Sift.new(psift.SiftConfig().with_octaves(4).with_contrast_threshold(0.015))
    outs = [psift.Features.pinned(4096, ctx) for _ in range(n)]
    for _ in range(3):
        sift.detect_and_compute_jpeg_batch(blobs, outs=outs, ctx=ctx)
    t0 = time.perf_counter()
    for _ in range(reps):
        feats = sift.detect_and_compute_jpeg_batch(blobs, outs=outs, ctx=ctx)
    jpeg_s = (time.perf_counter() - t0) / reps
    backend = ctx.jpeg_backend
    # two host threads with a context each, alternate batches: one thread's Huffman
    # stage overlaps the other's GPU work
    ctx2 = psift.Context(ctx.device)
    outs2 = [psift.Features.pinned(4096, ctx2) for _ in range(n)]
    sift.detect_and_compute_jpeg_batch(blobs, outs=outs2, ctx=ctx2)
    pairs = [(ctx, outs), (ctx2, outs2)]

    def worker(wi):
        c, o = pairs[wi]
        for _ in range(wi, reps, 2):
            sift.detect_and_compute_jpeg_batch(blobs, outs=o, ctx=c)
    t0 = time.perf_counter()
    ths = [threading.Thread(target=worker, args=(wi,)) for wi in range(2)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    jpeg2_s = (time.perf_counter() - t0) / reps
    ctx2.close()
    lumas = [psift.decode_jpeg_luma(b, ctx=ctx) for b in blobs]
    pin = [psift.pinned_empty(l.shape, np.uint8, ctx) for l in lumas]
    for d, l in zip(pin, lumas):
        d[...] = l
    for _ in range(3):
        sift.detect_and_compute_batch_u8(pin, outs=outs, ctx=ctx)
    t0 = time.perf_counter()
    for _ in range(reps):
        sift.detect_and_compute_batch_u8(pin, outs=outs, ctx=ctx)
    u8_s = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    for b in blobs:
        rgb = np.asarray(Image.open(io.BytesIO(b)).convert("RGB"))
        r, g, bl = (rgb[..., k].astype(np.uint32) for k in range(3))
        _ = ((2126 * r + 7152 * g + 722 * bl) // 10000).astype(np.uint8)
    cpu_decode_ms = (time.perf_counter() - t0) / n * 1e3
    # 64 images (the same files repeated); and both batch sizes with one batched
    # call on the calling thread (nvJPEG's GPU-assisted backend, whose Huffman
    # stage runs on the GPU only for batches of more than 50 images)
    blobs8 = blobs * 8
    outs8 = outs + [psift.Features.pinned(4096, ctx) for _ in range(7 * n)]

    def timed(bl, ou, r):
        sift.detect_and_compute_jpeg_batch(bl, outs=ou, ctx=ctx)
        t = time.perf_counter()
        for _ in range(r):
            sift.detect_and_compute_jpeg_batch(bl, outs=ou, ctx=ctx)
        return (time.perf_counter() - t) / r
    jpeg8_s = timed(blobs8, outs8, reps // 4 or 1)
    ctx.set_jpeg_threads(1)
    single8_s = timed(blobs, outs, reps // 2 or 1)
    single64_s = timed(blobs8, outs8, reps // 4 or 1)
    single_backend = ctx.jpeg_backend
    ctx.set_jpeg_threads(0)
    return {
        "workload": f"{n} colour {WIDTH}x{HEIGHT} JPEGs (4:2:0, q90, {sum(map(len, blobs)) / n / 1e3:.0f} KB each), "
                    "host bytes -> pinned host features, host API wall clock",
        "jpeg_images_per_s": n / jpeg_s, "u8_batch_images_per_s": n / u8_s,
        "jpeg_images_per_s_batch_of_64": 8 * n / jpeg8_s,
        "jpeg_images_per_s_2_host_threads": n / jpeg2_s,
        "single_call_images_per_s": {"batch_8": n / single8_s, "batch_64": 8 * n / single64_s,
                                     "nvjpeg_backend": single_backend},
        "host_decode_threads": min(os.cpu_count() or 1, 16),
        "jpeg_minus_u8_input_ms_per_batch": (jpeg_s - u8_s) * 1e3, "cpu_decode_ms_per_image_1_thread": cpu_decode_ms,
        "nvjpeg_backend": backend, "features_per_image": [len(f) for f in feats[:4]],
    }


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    steps = max(args.steps, 1)
    ips, n, dt, cores = cpu_reference(steps, min(args.warmup, 1), budget_s=120.0)
    line = {
        "metric": METRIC, "value": ips, "unit": "images/s", "n_gpus": args.gpus, "steps": n,
        "warmup": min(args.warmup, 1), "ms_per_step": 1e3 * dt / max(n, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD, "batch_per_step": 1},
        "cpu_baseline": {"value": ips, "unit": "images/s", "cores": cores, "kind": "port",
                         "sample": f"{n} x 1080p detect+describe, CPU restatement of pure-sift 0.2.0 "
                                   "(OpenMP over the loops rayon parallelises)"},
        "e2e": {"value": ips, "unit": "images/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import psift

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    B = args.batch
    host_imgs = make_images(B, seeds=shard.rank_image_seeds(B, rank))
    d_imgs = [torch.from_numpy(im).cuda() for im in host_imgs]
    cap = MAX_FEATURES
    outs = [{k: torch.empty(cap, dtype=torch.float32, device="cuda") for k in ("x", "y", "s", "r", "o")}
            for _ in range(B)]
    for o in outs:
        o["d"] = torch.empty((cap, 128), dtype=torch.float32, device="cuda")
    d_counts = torch.zeros(B, dtype=torch.int32, device="cuda")
    ctx = psift.Context(local)
    if args.blur == "fused":
        ctx.set_blur_rounding(ctx.BLUR_FUSED)  # profiling case: the single-rounding blur in the main loop
    cfg = psift.SiftConfig().with_octaves(OCTAVES).with_scales(SCALES).with_contrast_threshold(THRESH)
    ccfg = cfg.to_c()
    # tile shapes: the library's autotuner on this geometry (one chunk of the batch;
    # the matcher on 4096 x 4096 problems), before any timing
    t_tune = time.perf_counter()
    tune = None if args.no_autotune else ctx.autotune(HEIGHT, WIDTH, (B + 1) // 2, cfg, n_desc=4096, n_pairs=8)
    tune_s = time.perf_counter() - t_tune
    cimgs = (psift.CImageU8 * B)(*[psift.CImageU8(t.data_ptr(), HEIGHT, WIDTH, WIDTH) for t in d_imgs])
    couts = (psift.CFeatures * B)(*[psift.CFeatures(cap, 0, o["x"].data_ptr(), o["y"].data_ptr(),
                                                    o["s"].data_ptr(), o["r"].data_ptr(), o["o"].data_ptr(),
                                                    o["d"].data_ptr()) for o in outs])
    stream = torch.cuda.ExternalStream(ctx.stream)

    def step():
        ctx.check(ctx.lib.psift_detect_and_compute_batch_dev(ctx.handle, cimgs, B, C.byref(ccfg), couts,
                                                             C.c_void_p(d_counts.data_ptr())))

    for _ in range(max(args.warmup, 3)):
        step()
    ctx.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launch_count
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = ctx.launch_count - launches0
    ms = shard.max_over_ranks(ms)
    if dist:
        dist.barrier()
    ms_per_step = ms / args.steps
    value = world * B * args.steps / (ms / 1e3)
    counts = d_counts.cpu().numpy()
    if args.only_device:
        # profiling case: the timed device path only
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "images/s", "ms_per_step": ms_per_step,
                              "batch_per_gpu": B, "gpu_launches": int(launches)}), flush=True)
        if dist:
            dist.destroy_process_group()
        ctx.close()
        return 0

    # Per-stage device times (separate pass; events around each stage).
    ctx.enable_stage_timing(True)
    ctx.stage_times(reset=True)
    reps = 3
    for _ in range(reps):
        step()
    st = ctx.stage_times(reset=True)
    ctx.enable_stage_timing(False)
    pyr_ms, pyr_intervals = st["pyramid"]
    bytes_img, blur_launches = pyramid_bytes_per_image(HEIGHT, WIDTH)
    # one pyramid interval = the init blur, or one octave's levels (all images of the batch)
    blur_launch_total = reps * blur_launches
    avg_launch_s = (pyr_ms / 1e3) / blur_launch_total
    bytes_per_launch = B * bytes_img / blur_launches
    achieved = bytes_per_launch / avg_launch_s / 1e9
    peak, peak_kind = peaks()
    # the same stage against the FP32 pipe: lane operations over the stage time,
    # peak = SMs x 128 FP32 lanes x the SM clock seen under load
    ops_ref, ops_fused = pyramid_fp32_ops_per_image(HEIGHT, WIDTH)
    n_sms = torch.cuda.get_device_properties(0).multi_processor_count

    # The single-rounding blur mode (PSIFT_BLUR_FUSED: one fused multiply-add per
    # tap; not bit-equal to the reference, held to the f32 path's tolerances
    # against an f64 run): the same step, device-timed the same way, and its
    # pyramid stage against the same algorithmic bytes.
    ctx.set_blur_rounding(ctx.BLUR_FUSED)
    for _ in range(max(args.warmup, 3)):
        step()
    ctx.synchronize()
    if dist:
        dist.barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        step()
    f1.record(stream)
    ctx.synchronize()
    fused_ms = shard.max_over_ranks(f0.elapsed_time(f1))
    ctx.enable_stage_timing(True)
    ctx.stage_times(reset=True)
    for _ in range(reps):
        step()
    st_f = ctx.stage_times(reset=True)
    ctx.enable_stage_timing(False)
    ctx.set_blur_rounding(ctx.BLUR_REFERENCE)
    fused_launch_s = (st_f["pyramid"][0] / 1e3) / blur_launch_total
    fused_achieved = bytes_per_launch / fused_launch_s / 1e9
    blur_fused = {
        "value": world * B * args.steps / (fused_ms / 1e3), "unit": "images/s", "ms_per_step": fused_ms / args.steps,
        "stage_ms_per_step": {k: v[0] / reps for k, v in st_f.items() if v[1]},
        "roofline": {"kernel": "blur_level_kernel, single-rounding taps", "bound": "hbm", "achieved": fused_achieved,
                     "peak": peak, "unit": "GB/s", "frac": fused_achieved / peak, "peak_source": peak_kind,
                     "avg_launch_ms": fused_launch_s * 1e3},
        "note": "PSIFT_BLUR_FUSED: one fused multiply-add per blur tap; error against an f64 run within 0.01 px / "
                "0.01 scale / 1e-4 descriptor L2 (tests/test_blur_fused_gpu.py), not bit-equal to the reference"}
    clocks = clk.summary()
    mhz = clocks.get("sm_mhz") or 1965.0
    fp32_peak = n_sms * 128 * mhz * 1e6 / 1e12

    def fp32_view(ops_img: float, stage_ms: float, kernel: str) -> dict:
        achieved_t = B * ops_img / (stage_ms / 1e3) / 1e12
        return {"kernel": kernel, "bound": "fp32", "achieved": achieved_t, "peak": fp32_peak,
                "unit": "T lane-ops/s", "frac": achieved_t / fp32_peak, "ops_per_image": ops_img,
                "peak_source": f"nominal: {n_sms} SMs x 128 FP32 lanes x {mhz:.0f} MHz (median SM clock in the "
                               "timed region)"}
    roofline_fp32 = fp32_view(ops_ref, pyr_ms / reps, "pyramid stage, reference rounding (2 rounded ops per tap)")
    blur_fused["roofline_fp32"] = fp32_view(ops_fused, st_f["pyramid"][0] / reps,
                                            "pyramid stage, single rounding (1 fused op per tap)")

    # End to end through the public host-pointer API: the batch entry with page-locked
    # images and outputs (every step uploads the 8 images and downloads all features).
    # Two host threads, each with its own context (stream + workspace), take
    # alternate steps, so one step's transfers overlap the other's kernels; the
    # single-thread figure is reported beside it.
    sift = psift.Sift.new(cfg)

    def pinned_set(c):
        ims = []
        for im in host_imgs:
            buf = psift.pinned_empty(im.shape, np.uint8, c)
            buf[...] = im
            ims.append(buf)
        return ims, [psift.Features.pinned(MAX_FEATURES, c) for _ in range(B)]

    ctx2 = psift.Context(local)
    if tune is not None:  # the second host thread's context runs the same tile shapes
        t = ctx.tuning()
        for r, v in t["blur"].items():
            ctx2.set_tuning(ctx2.TUNE_BLUR, r, v)
        ctx2.set_tuning(ctx2.TUNE_MATCH_FP32, 0, t["match_fp32_per_sm"])
        ctx2.set_tuning(ctx2.TUNE_MATCH_TC, 0, t["match_tc_per_sm"])
    workers = [(ctx,) + pinned_set(ctx), (ctx2,) + pinned_set(ctx2)]
    for c, ims, fo in workers:
        for _ in range(2):
            sift.detect_and_compute_batch_u8(ims, outs=fo, ctx=c)
    if dist:
        dist.barrier()
    e2e_steps = max(2, min(args.steps, 40))
    d2h_box = [0]

    def worker(wi):
        c, ims, fo = workers[wi]
        for _ in range(wi, e2e_steps, 2):
            feats = sift.detect_and_compute_batch_u8(ims, outs=fo, ctx=c)
            d2h_box[0] = sum(len(f) for f in feats) * (5 + 128) * 4 + 16 * B

    t0 = time.perf_counter()
    threads = [threading.Thread(target=worker, args=(wi,)) for wi in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    e2e_s = time.perf_counter() - t0
    d2h = d2h_box[0]
    c, ims, fo = workers[0]
    t1 = time.perf_counter()
    for _ in range(e2e_steps):
        sift.detect_and_compute_batch_u8(ims, outs=fo, ctx=c)
    e2e_single = B * e2e_steps / (time.perf_counter() - t1)
    # the same images one call per image (the reference's call pattern), for comparison
    for _ in range(3):  # warm the single-image path: eager, graph capture, replay
        sift.detect_and_compute_u8(ims[0], ctx=ctx)
    single_rounds = 3
    t1 = time.perf_counter()
    for _ in range(single_rounds):
        for im in ims:
            sift.detect_and_compute_u8(im, ctx=ctx)
    single_s = (time.perf_counter() - t1) / single_rounds
    # one call per image from 4 host threads with a context each (a drop-in wrapper
    # holding one context per rayon worker)
    n_callers = 4
    callers = [psift.Context(local) for _ in range(n_callers)]
    for c in callers:
        for _ in range(3):
            sift.detect_and_compute_u8(ims[0], ctx=c)

    def caller(ci):
        for _ in range(single_rounds):
            for k in range(ci, B, n_callers):
                sift.detect_and_compute_u8(ims[k], ctx=callers[ci])
    t1 = time.perf_counter()
    ths = [threading.Thread(target=caller, args=(ci,)) for ci in range(n_callers)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    single4_s = (time.perf_counter() - t1) / single_rounds
    for c in callers:
        c.close()
    e2e_s = shard.max_over_ranks(e2e_s)
    e2e_value = world * B * e2e_steps / e2e_s

    result = None
    if rank == 0:
        result = {
            "metric": METRIC, "value": value, "unit": "images/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "batch_per_gpu": B, "global_batch": world * B, "l2": L2_NOTE,
                       "features_per_image": [int(c) for c in counts[:4]],
                       "autotune": None if tune is None else {
                           "seconds": tune_s,
                           "blur_variant_per_radius": {r: e["variant"] for r, e in tune["blur"].items()},
                           "blur_ms_per_variant": {r: e["ms"] for r, e in tune["blur"].items()},
                           "match_fp32_items_per_sm": tune["match_fp32"]["per_sm"],
                           "match_tc_items_per_sm": tune["match_tc"]["per_sm"],
                           "variants": "blur 0: 4x8, 1: 8x8, 2: 4x4 outputs per thread (columns x rows); 3: TMA tiles, persistent CTAs; 4: 128-row tiles, 512 threads"}},
            "gpu_launches": int(launches),
            "e2e": {"value": e2e_value, "unit": "images/s", "h2d_bytes_per_step": B * WIDTH * HEIGHT,
                    "d2h_bytes_per_step": int(d2h),
                    "api": "psift_detect_and_compute_u8_batch (8 pinned host images -> pinned host features), "
                           "2 host threads with a context each, alternate steps",
                    "one_thread_images_per_s": e2e_single,
                    "single_image_api_images_per_s": B / single_s,
                    "single_image_api_4_host_threads_images_per_s": B / single4_s},
            "roofline": {"kernel": "blur_level_kernel (pyramid: blur + DoG + decimation)", "bound": "hbm",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "traffic": NCU_TRAFFIC_BLUR_LEVEL,
                         "algorithmic_bytes_per_launch": bytes_per_launch,
                         "avg_launch_ms": avg_launch_s * 1e3},
            "roofline_fp32": roofline_fp32,
            "stage_ms_per_step": {k: v[0] / reps for k, v in st.items() if v[1]},
            "blur_fused": blur_fused,
            "clocks": clocks,
        }
        for key, fn in (("uneven_batch", uneven_bench), ("catalog", catalog_bench),
                        ("catalog_search", catalog_search_bench), ("warp", warp_bench),
                        ("fundamental", fundamental_bench),
                        ("learned_ransac", ransac_bench), ("jpeg", jpeg_bench), ("png", png_bench),
                        ("panorama", panorama_bench)):
            if getattr(args, "no_" + key):
                continue
            try:
                result[key] = fn(ctx, torch)
            except Exception as exc:  # reported, not hidden
                result[key] = {"error": repr(exc)}
        try:
            result["match"] = match_bench(ctx, torch)
            bf16_peak, _ = peaks("bf16_tflops")
            result["match"]["tensor_frac_of_measured_bf16"] = result["match"]["bf16_tflops_effective"] / bf16_peak
        except Exception as exc:  # reported, not hidden
            result["match"] = {"error": repr(exc)}
        if world == 1 and not args.no_cpu_baseline:
            ips, n, dt, cores = cpu_reference(steps=30, warmup=1, budget_s=20.0)
            result["cpu_baseline"] = {
                "value": ips, "unit": "images/s", "cores": cores, "kind": "port",
                "sample": f"{n} x 1080p detect+describe of the same image, CPU restatement of pure-sift 0.2.0 "
                          f"(OpenMP, {cores} threads), {dt:.1f} s"}
        print(json.dumps(result), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    ctx2.close()
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only-device", action="store_true", help="time the device path only (profiling case)")
    ap.add_argument("--match-only", action="store_true", help="run only the pair-matching measurement")
    ap.add_argument("--match-pairs", type=int, default=32)
    ap.add_argument("--only-section", choices=["match", "catalog", "catalog_search", "warp", "fundamental",
                                               "learned_ransac", "uneven_batch", "jpeg", "png", "panorama", "pyramid"],
                    help="run one section alone (profiling case)")
    ap.add_argument("--ransac-pairs", type=int, default=1024, help="learned-RANSAC section: match sets")
    ap.add_argument("--blur", choices=["reference", "fused"], default="reference",
                    help="blur rounding of the main loop (profiling case; the default is the reference's)")
    ap.add_argument("--blur-variant", type=int, choices=[0, 1, 2, 3, 4], default=None,
                    help="pyramid section: run this level-blur variant at every radius (profiling case)")
    ap.add_argument("--catalog-codes", type=int, default=2_000_000, help="catalog section: catalog codes")
    ap.add_argument("--catalog-entries", type=int, default=10_000, help="catalog-search section: entries")
    ap.add_argument("--no-catalog", action="store_true")
    ap.add_argument("--no-catalog-search", dest="no_catalog_search", action="store_true")
    ap.add_argument("--no-warp", dest="no_warp", action="store_true")
    ap.add_argument("--no-autotune", dest="no_autotune", action="store_true",
                    help="run the default tile shapes instead of the autotuner's")
    ap.add_argument("--no-fundamental", dest="no_fundamental", action="store_true")
    ap.add_argument("--no-uneven-batch", dest="no_uneven_batch", action="store_true")
    ap.add_argument("--no-learned-ransac", dest="no_learned_ransac", action="store_true")
    ap.add_argument("--no-jpeg", dest="no_jpeg", action="store_true")
    ap.add_argument("--no-png", dest="no_png", action="store_true")
    ap.add_argument("--no-panorama", dest="no_panorama", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        # one process per GPU: --gpus N runs under torchrun with N ranks
        sys.exit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; launch N>1 with "
                 f"`python -m torch.distributed.run --nproc-per-node {args.gpus} bench.py --gpus {args.gpus}`")
    if args.impl == "reference":
        return run_reference(args)
    if args.match_only:
        args.only_section = "match"
    if args.only_section:
        # one section alone (profiling cases); sizes as in the full run
        import torch
        import psift
        ctx = psift.Context(int(os.environ.get("LOCAL_RANK", "0")))
        fns = {"match": lambda: match_bench(ctx, torch, n_pairs=args.match_pairs, reps=args.steps),
               "catalog": lambda: catalog_bench(ctx, torch, n_cat=args.catalog_codes),
               "learned_ransac": lambda: ransac_bench(ctx, torch, n_pairs=args.ransac_pairs),
               "catalog_search": lambda: catalog_search_bench(ctx, torch, n_entries=args.catalog_entries), "warp": lambda: warp_bench(ctx, torch),
               "fundamental": lambda: fundamental_bench(ctx, torch),
               "uneven_batch": lambda: uneven_bench(ctx, torch), "jpeg": lambda: jpeg_bench(ctx, torch),
               "png": lambda: png_bench(ctx, torch),
               "panorama": lambda: panorama_bench(ctx, torch),
               "pyramid": lambda: pyramid_bench(ctx, torch, blur=args.blur, reps=min(args.steps, 10),
                                                 variant=args.blur_variant)}
        print(json.dumps({args.only_section: fns[args.only_section]()}), flush=True)
        ctx.close()
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
