"""Device MIH tables (src/catalog.rs:291-321) and the votes through them
(:596-621): equal to the reference's own table walk restated on the CPU
(oracle.mih_votes_tables), to the scan path with the MIH rule, and, for the
exhaustive rule, to count_coarse_hamming_votes (:707-728).  The tables follow
the catalog through upserts (replace and append) and removals, and the
catalog search gives the same hits with either votes computation."""
import numpy as np
import pytest

import mih_cases
import oracle as O
import psift
import synth

pytestmark = pytest.mark.gpu


def _features_for_codes(codes: np.ndarray, seed: int) -> psift.Features:
    """Features whose descriptors quantise to `codes` (bit set -> 0.1 > 0.065, else 0)."""
    n = codes.shape[0]
    bits = ((codes[:, :, None] >> np.arange(64, dtype=np.uint64)) & np.uint64(1)).astype(bool).reshape(n, 128)
    rng = np.random.default_rng(seed)
    d = np.where(bits, np.float32(0.1), np.float32(0.0)).astype(np.float32)
    return psift.Features(rng.uniform(0, 640, n).astype(np.float32), rng.uniform(0, 480, n).astype(np.float32),
                          np.full(n, 2.0, np.float32), np.full(n, 0.05, np.float32), np.zeros(n, np.float32), d)


def _catalog(cat_codes, off, seed=0):
    c = psift.DeviceCatalog()
    for e in range(len(off) - 1):
        c.upsert_entry(f"e{e:05d}", 640, 480, _features_for_codes(cat_codes[off[e]:off[e + 1]], seed + e))
    return c


def _check_all_paths(cat, q, cat_codes, off):
    walk = O.mih_votes_tables(q, cat_codes, off)
    np.testing.assert_array_equal(cat.votes(q, psift.VOTES_MIH_INDEX), walk)
    np.testing.assert_array_equal(cat.votes(q, psift.VOTES_MIH_SCAN), walk)
    np.testing.assert_array_equal(cat.votes(q, psift.VOTES_EXHAUSTIVE), O.hamming_votes(q, cat_codes, off, False))
    auto = walk if len(off) - 1 > 32 else O.hamming_votes(q, cat_codes, off, False)
    np.testing.assert_array_equal(cat.votes(q, psift.VOTES_AUTO), auto)
    return walk


@pytest.mark.parametrize("n_entries,n_queries,seed", [(40, 200, 1), (120, 500, 2), (300, 2000, 4), (20, 100, 6)])
def test_votes_through_tables_equal_table_walk(n_entries, n_queries, seed):
    q, cat_codes, off = mih_cases.case(n_entries, n_queries, seed)
    cat = _catalog(cat_codes, off)
    walk = _check_all_paths(cat, q, cat_codes, off)
    assert walk.sum() > 0
    # a second call reuses the tables and the scratch: same votes
    np.testing.assert_array_equal(cat.votes(q, psift.VOTES_MIH_INDEX), walk)
    cat.close()


def test_tables_follow_upsert_and_remove():
    q, cat_codes, off = mih_cases.case(60, 400, 7)
    cat = _catalog(cat_codes, off)
    _check_all_paths(cat, q, cat_codes, off)
    # replace entry 5 with the codes of queries 0..9 (every query 0..9 now votes for it)
    rep = q[:10].copy()
    cat.upsert_entry("e00005", 640, 480, _features_for_codes(rep, 99))
    codes2 = [cat_codes[off[e]:off[e + 1]] for e in range(60)]
    codes2[5] = rep
    off2 = np.zeros(61, np.int64)
    off2[1:] = np.cumsum([len(c) for c in codes2])
    flat2 = np.concatenate(codes2)
    v = _check_all_paths(cat, q, flat2, off2)
    assert v[5] >= 10
    # append, then swap_remove entry 3 (the last entry takes its place)
    cat.upsert_entry("zz_new", 640, 480, _features_for_codes(q[20:30], 98))
    codes2.append(q[20:30].copy())
    assert cat.remove("e00003")
    codes2[3] = codes2.pop()
    off3 = np.zeros(len(codes2) + 1, np.int64)
    off3[1:] = np.cumsum([len(c) for c in codes2])
    v = _check_all_paths(cat, q, np.concatenate(codes2), off3)
    assert v[3] >= 10
    cat.close()


def test_votes_edge_cases():
    q, cat_codes, off = mih_cases.case(50, 100, 8)
    cat = _catalog(cat_codes, off)
    assert cat.votes(q[:0], psift.VOTES_MIH_INDEX).sum() == 0
    # the same query many times: each copy votes once per entry
    qq = np.repeat(q[:1], 64, axis=0)
    np.testing.assert_array_equal(cat.votes(qq, psift.VOTES_MIH_INDEX), O.mih_votes_tables(qq, cat_codes, off))
    # a query equal to every signature of an entry with repeats (all 16 buckets hit)
    e = int(np.argmax(np.diff(off)))
    qe = cat_codes[off[e]:off[e] + 1]
    np.testing.assert_array_equal(cat.votes(qe, psift.VOTES_MIH_INDEX), O.mih_votes_tables(qe, cat_codes, off))
    with pytest.raises(psift.PsiftError):
        cat.votes(q, 7)
    cat.close()
    empty = psift.DeviceCatalog()
    assert empty.votes(q, psift.VOTES_MIH_INDEX).shape == (0,)
    empty.close()


def test_search_same_hits_with_either_votes_path():
    # 40 entries of SIFT-like features; the query holds entry 17's features moved
    # by a similarity, so the shortlist, matching and RANSAC all have work.
    rng = np.random.default_rng(3)
    cat = psift.DeviceCatalog()
    ents = []
    for e in range(40):
        n = int(rng.integers(30, 120))
        d = synth.sift_like_descriptors(n, 500 + e)
        f = psift.Features(rng.uniform(0, 640, n).astype(np.float32), rng.uniform(0, 480, n).astype(np.float32),
                           rng.uniform(1.6, 8, n).astype(np.float32), np.full(n, 0.05, np.float32),
                           rng.uniform(0, 6.28, n).astype(np.float32), d)
        ents.append(f)
        cat.upsert_entry(f"img{e:03d}", 640, 480, f)
    t = ents[17]
    th = np.deg2rad(12.0)
    qx = (1.05 * (np.cos(th) * t.x - np.sin(th) * t.y) + 15).astype(np.float32)
    qy = (1.05 * (np.sin(th) * t.x + np.cos(th) * t.y) - 10).astype(np.float32)
    query = psift.Features(qx, qy, t.scale * 1.05, t.response, t.orientation + th, t.descriptors.copy())
    cat.set_search_votes(psift.VOTES_MIH_SCAN)
    a = cat.search_features(query)
    cat.set_search_votes(psift.VOTES_AUTO)
    b = cat.search_features(query)
    assert len(a) == len(b) > 0 and a[0].id == "img017"
    for x, y in zip(a, b):
        assert (x.id, x.coarse_votes, x.tracking.match_count) == (y.id, y.coarse_votes, y.tracking.match_count)
    with pytest.raises(psift.PsiftError):
        cat.set_search_votes(psift.VOTES_MIH_INDEX)
    cat.close()


def test_reference_mih_indexed_search_and_remove():
    # tests/pipeline_tests.rs:1439-1489 through the device catalog: 40 entries, the
    # sample image's features at entry 17 among two synthetic scenes; the search
    # (MIH tables) ranks item_17 first; remove is a swap_remove.
    import scene_cases
    import sweep_cases
    sift = psift.Sift.new(psift.SiftConfig().with_octaves(3).with_scales(3).with_contrast_threshold(0.015))
    target = sift.detect_and_compute_u8(sweep_cases.aerial_west_luma())
    d1 = sift.detect_and_compute_u8(scene_cases.render_synthetic_scene(1))
    d2 = sift.detect_and_compute_u8(scene_cases.render_synthetic_scene(2))
    feats = [target if i == 17 else (d1 if i % 2 == 0 else d2) for i in range(40)]
    cat = psift.DeviceCatalog()
    for i, f in enumerate(feats):
        cat.upsert_entry(f"item_{i:02d}.png", 220, 220, f)
    hits = cat.search_features(target, top_k=3, shortlist_k=8)
    assert hits and hits[0].id == "item_17.png"
    qcodes = psift.quantize_descriptor_u128(target.descriptors)

    def walk(fs):
        sigs = [O.quantize_u128(f.descriptors) for f in fs]
        off = np.concatenate([[0], np.cumsum([len(s) for s in sigs])]).astype(np.int64)
        return O.mih_votes_tables(qcodes, np.concatenate(sigs), off)
    np.testing.assert_array_equal(cat.votes(qcodes, psift.VOTES_AUTO), walk(feats))
    assert cat.remove("item_17.png") and not cat.remove("item_17.png") and len(cat) == 39
    feats[17] = feats.pop()  # swap_remove
    np.testing.assert_array_equal(cat.votes(qcodes, psift.VOTES_AUTO), walk(feats))
    cat.close()
