"""Catalog code sets for the multi-index-hashing votes (src/catalog.rs:291-321,
:596-633): entries of uneven size (empty ones included) and queries placed so
that every branch of the rule is taken — codes within 24 bits that share a byte
with the query (MIH and exhaustive votes), codes within 24 bits that share no
byte (one bit flipped in each of the 16 bytes: exhaustive votes only), codes
just outside (25 bits), repeated signatures inside one entry, and random codes.
"""
import numpy as np


def _random_codes(rng, n):
    return rng.integers(0, np.iinfo(np.uint64).max, size=(n, 2), dtype=np.uint64, endpoint=True)


def _flip(code, bits):
    out = code.copy()
    for b in bits:
        out[b // 64] ^= np.uint64(1) << np.uint64(b % 64)
    return out


def case(n_entries: int, n_queries: int, seed: int, max_per_entry: int = 60):
    """(query codes (nq, 2) u64, catalog codes (n, 2) u64, entry offsets (n_entries + 1) i64)."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(0, max_per_entry + 1, size=n_entries)
    sizes[rng.random(n_entries) < 0.1] = 0  # empty entries
    off = np.zeros(n_entries + 1, np.int64)
    off[1:] = np.cumsum(sizes)
    cat = _random_codes(rng, int(off[-1]))
    q = _random_codes(rng, n_queries)
    filled = np.nonzero(sizes)[0]
    for qi in range(n_queries):
        kind = qi % 5
        if kind == 4 or len(filled) == 0:
            continue  # random query: almost surely no vote
        e = int(rng.choice(filled))
        s = int(off[e] + rng.integers(0, sizes[e]))
        base = q[qi]
        if kind == 0:    # within 24 bits, some bytes untouched
            cat[s] = _flip(base, rng.choice(128, size=int(rng.integers(0, 25)), replace=False))
        elif kind == 1:  # 16 bits: one in every byte, no shared byte
            cat[s] = _flip(base, [8 * b + int(rng.integers(0, 8)) for b in range(16)])
        elif kind == 2:  # 25 bits: just outside
            cat[s] = _flip(base, rng.choice(128, size=25, replace=False))
        else:            # the same near code twice in the entry, plus one in another entry
            c = _flip(base, rng.choice(128, size=10, replace=False))
            cat[s] = c
            cat[int(off[e])] = c
            e2 = int(rng.choice(filled))
            cat[int(off[e2] + sizes[e2] - 1)] = _flip(base, rng.choice(128, size=24, replace=False))
    return q, cat, off
