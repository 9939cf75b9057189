"""Work split over ranks (one process per GPU).

Extraction and matching: images and pairs are independent, so each rank takes
its own share (``rank_items``) with no exchange on the data path, and a timed
region is reported as the slowest rank's (``max_over_ranks``).

Catalog top-k search: sharded over ranks.

Each rank owns the contiguous code range ``shard_range(ncat, rank, world)`` and
computes the per-query top-k of its shard (``psift.hamming_topk`` on its GPU by
default).  The (distance, global index) lists are all-gathered with
``torch.distributed`` (NCCL for CUDA tensors, gloo for CPU tensors) and merged
with the same tiebreak the single-GPU kernel uses, so every rank ends with the
exact top-k of the whole catalog: the global top-k is contained in the union of
the shards' top-k lists.  Only the 4096 x k lists cross the interconnect
(k = 64: 2 MB per rank as int64 keys); codes never leave their GPU.
"""
from __future__ import annotations

import numpy as np


def rank_items(n_items: int, rank: int, world: int) -> list[int]:
    """Round-robin share of `rank` among n_items independent images or pairs:
    item i belongs to rank i mod world (shares differ in size by at most 1)."""
    return list(range(int(rank), int(n_items), int(world)))


def rank_image_seeds(batch: int, rank: int) -> list[int]:
    """Seeds of the `batch` synthetic images rank `rank` detects per step when the
    work scales weakly (every rank a full batch of its own, no image shared)."""
    return [1000 * int(rank) + 1 + i for i in range(int(batch))]


def max_over_ranks(value: float, group=None) -> float:
    """The largest of every rank's `value` (a timed region's milliseconds), on
    every rank; `value` itself when no process group is initialised."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def shard_range(ncat: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of the codes owned by `rank`; shards differ in size by at most 1."""
    base, extra = divmod(int(ncat), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def pack_keys(idx: np.ndarray, dist: np.ndarray, offset: int) -> np.ndarray:
    """Sort keys (distance << 32 | global index); empty slots (index 2^32-1) stay last."""
    idx = idx.astype(np.uint64)
    empty = idx == 0xFFFFFFFF
    g = idx + np.uint64(offset)
    keys = (dist.astype(np.uint64) << np.uint64(32)) | g
    keys[empty] = np.uint64(0xFFFFFFFFFFFFFFFF)
    return keys


def merge_keys(keys: np.ndarray, k: int) -> tuple[np.ndarray, np.ndarray]:
    """keys (nq, m) from all shards -> the k smallest per query as (idx, dist) u32."""
    top = np.sort(keys, axis=1)[:, :k]
    empty = top == np.uint64(0xFFFFFFFFFFFFFFFF)
    idx = (top & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    dist = (top >> np.uint64(32)).astype(np.uint32)
    idx[empty] = 0xFFFFFFFF
    dist[empty] = 0xFFFFFFFF
    return idx, dist


def sharded_topk(query_codes, catalog_codes, k: int, topk_fn=None, group=None):
    """Exact top-k of the whole catalog with the catalog split over the ranks of
    `group`.  `catalog_codes` is the FULL catalog's length-ncat view on every
    rank only for the range bookkeeping; each rank reads just its own slice.
    `topk_fn(q, shard, k) -> (idx, dist)` is the per-shard search (default: the
    GPU kernel).  Returns (idx, dist) (nq, k) u32 on every rank."""
    import torch
    import torch.distributed as dist

    if topk_fn is None:
        import psift
        topk_fn = psift.hamming_topk
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    codes = np.asarray(catalog_codes).reshape(-1, 2)
    lo, hi = shard_range(codes.shape[0], rank, world)
    q = np.ascontiguousarray(query_codes, dtype=np.uint64).reshape(-1, 2)
    if hi > lo:
        idx, dd = topk_fn(q, codes[lo:hi], k)
        keys = pack_keys(np.asarray(idx), np.asarray(dd), lo)
    else:
        keys = np.full((q.shape[0], k), 0xFFFFFFFFFFFFFFFF, np.uint64)
    local = torch.from_numpy(keys.view(np.int64).copy())
    backend = dist.get_backend(group)
    if backend == "nccl":
        local = local.cuda()
    parts = [torch.empty_like(local) for _ in range(world)]
    dist.all_gather(parts, local, group=group)
    allk = np.concatenate([p.cpu().numpy().view(np.uint64) for p in parts], axis=1)
    return merge_keys(allk, k)
