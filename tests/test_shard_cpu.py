"""The sharded catalog search's exchange and merge on CPU ranks (gloo, world
size 2 and 3): every rank must end with the single-process top-k.  The
per-shard search is the CPU restatement here (the GPU kernel's own parity is
tested against it in tests/test_catalog_gpu.py)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle as O
import shard
import synth


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q, cat, k, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        idx, dd = shard.sharded_topk(q, cat, k, topk_fn=O.hamming_topk)
        out[rank] = (idx, dd)
    finally:
        dist.destroy_process_group()


def _codes(n, seed):
    return O.quantize_u128(synth.sift_like_descriptors(n, seed))


@pytest.mark.parametrize("world,ncat,k", [(2, 5000, 16), (3, 4001, 64), (2, 40, 64)])
def test_sharded_topk_equals_single_process(world, ncat, k):
    cat = _codes(ncat, 11 + world)
    q = np.concatenate([cat[:20], _codes(44, 99)])  # exact hits and unrelated queries
    ref_idx, ref_dist = O.hamming_topk(q, cat, k)
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, q, cat, k, out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        idx, dd = out[r]
        np.testing.assert_array_equal(dd, ref_dist)
        np.testing.assert_array_equal(idx, ref_idx)


def test_shard_ranges_cover_catalog():
    for ncat in (0, 1, 7, 1000, 2_000_000):
        for world in (1, 2, 3, 8):
            rs = [shard.shard_range(ncat, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == ncat
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            assert max(h - l for l, h in rs) - min(h - l for l, h in rs) <= 1


def test_merge_handles_short_lists():
    # a shard with fewer codes than k pads with empty keys, which sort last
    idx = np.array([[3, 0xFFFFFFFF]], np.uint32)
    dd = np.array([[5, 0xFFFFFFFF]], np.uint32)
    keys = np.concatenate([shard.pack_keys(idx, dd, 100), shard.pack_keys(np.array([[1, 2]], np.uint32),
                                                                         np.array([[5, 7]], np.uint32), 0)], axis=1)
    i, d = shard.merge_keys(keys, 3)
    assert i.tolist() == [[1, 103, 2]] and d.tolist() == [[5, 5, 7]]


def _split_worker(rank, world, port, n_items, ms, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        items = shard.rank_items(n_items, rank, world)
        seeds = shard.rank_image_seeds(4, rank)
        slowest = shard.max_over_ranks(ms[rank])
        out[rank] = (items, seeds, slowest)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n_items", [(2, 64), (2, 7), (3, 32)])
def test_extraction_split_and_max_over_ranks(world, n_items):
    """Images (and pairs) are split round-robin with no exchange: every item on
    exactly one rank, shares within one item of each other; the weak-scaling
    bench gives every rank its own images (disjoint seeds); the timed region is
    the slowest rank's on every rank."""
    ms = [10.0 + 7.5 * r for r in range(world)][::-1]
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_split_worker, args=(world, port, n_items, ms, out), nprocs=world, start_method="spawn",
                       join=True)
    got = [out[r] for r in range(world)]
    every = sorted(i for items, _, _ in got for i in items)
    assert every == list(range(n_items))
    sizes = [len(items) for items, _, _ in got]
    assert max(sizes) - min(sizes) <= 1
    seeds = [s for _, ss, _ in got for s in ss]
    assert len(set(seeds)) == len(seeds) == 4 * world
    assert all(slowest == max(ms) for _, _, slowest in got)


def test_max_over_ranks_without_a_group():
    assert shard.max_over_ranks(3.25) == 3.25
