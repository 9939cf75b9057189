"""The device-resident catalog (psift_catalog_*).

* PSIFTCAT v1 load / save against the byte layout of FeatureCatalog::save_binary
  and load_binary (src/catalog.rs:401-540), written here by `write_psiftcat`;
  the reference's format errors (:447-540).
* upsert / remove order (src/catalog.rs:324-353) against the host-side
  FeatureCatalog mirror.
* search_features (src/catalog.rs:576-702) against the same search composed
  from the CPU restatement's stages (votes, Lowe matching, similarity and
  homography RANSAC, tracking summary), on the same features.
"""
import os
import struct

import numpy as np
import pytest

import oracle as O
from catalog_oracle import oracle_search
import psift
import synth

pytestmark = pytest.mark.gpu


def write_psiftcat(path, octaves, scales, threshold, kind, entries) -> bytes:
    """entries: (id, width, height, meta (n, 5) f32 [x y scale response orientation],
    codes (n, 2) u64, q (n, 128) u8); the field order of save_binary."""
    b = bytearray(b"PSIFTCAT")
    b += struct.pack("<IIIfB", 1, octaves, scales, threshold, kind)
    b += struct.pack("<Q", len(entries))
    for id_, w, h, meta, codes, q in entries:
        ib = id_.encode("utf-8")
        b += struct.pack("<I", len(ib)) + ib + struct.pack("<IIQ", w, h, len(meta))
        for j in range(len(meta)):
            b += np.asarray(meta[j], "<f4").tobytes() + np.asarray(codes[j], "<u8").tobytes()
            b += np.asarray(q[j], np.uint8).tobytes()
    with open(path, "wb") as fh:
        fh.write(bytes(b))
    return bytes(b)


def random_entries(rng, sizes):
    out = []
    for k, n in enumerate(sizes):
        meta = rng.normal(size=(n, 5)).astype(np.float32) * 100
        codes = rng.integers(0, 2**63, size=(n, 2), dtype=np.uint64) ^ rng.integers(0, 2, (n, 2)).astype(np.uint64) << 63
        q = rng.integers(0, 256, size=(n, 128)).astype(np.uint8)
        q[: n // 3, 40:] = 0  # some sparse descriptors
        out.append((f"entry-{k}-é", 100 + k, 50 + k, meta, codes, q))
    return out


def test_psiftcat_load_matches_file(tmp_path):
    rng = np.random.default_rng(7)
    entries = random_entries(rng, [5, 0, 37, 1, 300])
    path = str(tmp_path / "c.psiftcat")
    write_psiftcat(path, 4, 5, 0.02, 1, entries)
    cat = psift.DeviceCatalog.load_binary(path)
    p = cat.params
    assert (p.octaves, p.scales, p.descriptor_kind) == (4, 5, 1) and np.float32(p.threshold) == np.float32(0.02)
    assert [(s.id, s.width, s.height, s.feature_count) for s in cat.list_summaries()] == \
        [(e[0], e[1], e[2], len(e[3])) for e in entries]
    for i, (_, _, _, meta, codes, q) in enumerate(entries):
        f, c = cat.entry_features(i)
        np.testing.assert_array_equal(np.stack([f.x, f.y, f.scale, f.response, f.orientation], 1).view(np.uint32),
                                      meta.view(np.uint32))
        np.testing.assert_array_equal(c, codes)  # stored codes kept, not recomputed
        if len(q):
            np.testing.assert_array_equal(f.descriptors.view(np.uint32), O.dequantize_u8(q).view(np.uint32))
    assert cat.index_of(entries[2][0]) == 2 and cat.index_of("absent") is None


def test_psiftcat_save_is_the_reference_layout(tmp_path):
    rng = np.random.default_rng(8)
    entries = random_entries(rng, [17, 0, 64])
    src = str(tmp_path / "a.psiftcat")
    write_psiftcat(src, 3, 3, 0.015, 0, entries)
    cat = psift.DeviceCatalog.load_binary(src)
    dst = str(tmp_path / "sub" / "dir" / "b.psiftcat")
    cat.save_binary(dst)
    # save_binary quantises the (dequantised) f32 descriptors again; codes are the stored ones
    requant = [(i, w, h, m, c, O.quantize_u8(O.dequantize_u8(q)) if len(q) else q) for i, w, h, m, c, q in entries]
    expect = write_psiftcat(str(tmp_path / "expect.psiftcat"), 3, 3, 0.015, 0, requant)
    assert open(dst, "rb").read() == expect
    assert not [n for n in os.listdir(tmp_path / "sub" / "dir") if ".tmp." in n]
    # and it loads back to the same catalog
    again = psift.DeviceCatalog.load_auto(dst)
    assert [s.id for s in again.list_summaries()] == [e[0] for e in entries]


@pytest.mark.parametrize("mutate,message", [
    (lambda b: b"PSIFTCAX" + b[8:], "Invalid binary catalog magic header"),
    (lambda b: b[:8] + struct.pack("<I", 2) + b[12:], "Unsupported binary catalog version 2"),
    (lambda b: b[:24] + bytes([7]) + b[25:], "Unknown descriptor kind 7"),
    (lambda b: b[:-1], "Unexpected EOF while reading binary catalog"),
    (lambda b: b[:35], "Unexpected EOF while reading binary catalog"),
    (lambda b: b[:40], "Truncated entry id in binary catalog"),
    (lambda b: b[:5], "Unexpected EOF while reading binary catalog"),
])
def test_psiftcat_format_errors(tmp_path, mutate, message):
    rng = np.random.default_rng(9)
    good = write_psiftcat(str(tmp_path / "g"), 3, 3, 0.015, 0, random_entries(rng, [3, 2]))
    bad = str(tmp_path / "bad")
    with open(bad, "wb") as fh:
        fh.write(mutate(good))
    with pytest.raises(psift.PsiftError) as ei:
        psift.DeviceCatalog.load_binary(bad)
    assert ei.value.status == psift.PSIFT_ERR_FORMAT and message in str(ei.value)


def test_psiftcat_bad_utf8_truncated_id_missing_file_and_empty(tmp_path):
    b = bytearray(b"PSIFTCAT") + struct.pack("<IIIfBQ", 1, 3, 3, 0.015, 0, 1)
    with open(tmp_path / "u", "wb") as fh:
        fh.write(bytes(b + struct.pack("<I", 2) + b"\xc3\x28" + struct.pack("<IIQ", 1, 1, 0)))
    with pytest.raises(psift.PsiftError, match="Invalid UTF-8 entry id"):
        psift.DeviceCatalog.load_binary(str(tmp_path / "u"))
    with open(tmp_path / "t", "wb") as fh:
        fh.write(bytes(b + struct.pack("<I", 9) + b"abc"))
    with pytest.raises(psift.PsiftError, match="Truncated entry id"):
        psift.DeviceCatalog.load_binary(str(tmp_path / "t"))
    with pytest.raises(psift.PsiftError) as ei:
        psift.DeviceCatalog.load_binary(str(tmp_path / "missing"))
    assert ei.value.status == psift.PSIFT_ERR_IO
    with open(tmp_path / "e", "wb") as fh:
        fh.write(bytes(bytearray(b"PSIFTCAT") + struct.pack("<IIIfBQ", 1, 3, 3, 0.015, 0, 0)))
    empty = psift.DeviceCatalog.load_binary(str(tmp_path / "e"))
    assert len(empty) == 0 and empty.search_features(psift.Features.empty(3)) == []


def _features(seed, n=None, w=256, h=192):
    sift = psift.Sift.new(psift.SiftConfig())
    f = sift.detect_and_compute_u8(synth.blob_image(w, h, 60, 2.0, 8.0, seed=seed))
    return f if n is None else f.head(min(n, len(f)))


def test_upsert_replace_and_swap_remove_order():
    host, dev = psift.FeatureCatalog(), psift.DeviceCatalog()
    feats = {f"e{k}": _features(500 + k) for k in range(6)}
    for k, (id_, f) in enumerate(feats.items()):
        host.upsert_entry(id_, 10 + k, 20 + k, f)
        dev.upsert_entry(id_, 10 + k, 20 + k, f)
    replacement = _features(999, 7)
    for c in (host, dev):
        c.upsert_entry("e2", 5, 6, replacement)  # replace keeps the position
        assert c.remove("e1") and not c.remove("e1")  # swap_remove: e5 moves to index 1
        c.upsert_entry("new", 1, 1, psift.Features.empty(0))
    ids = [s.id for s in dev.list_summaries()]
    assert ids == [e.id for e in host.entries] == ["e0", "e5", "e2", "e3", "e4", "new"]
    for i, e in enumerate(host.entries):
        f, codes = dev.entry_features(i)
        assert len(f) == len(e.features)
        np.testing.assert_array_equal(f.descriptors, e.features.descriptors)
        np.testing.assert_array_equal(f.x, e.features.x)
        np.testing.assert_array_equal(codes, e.signatures)


@pytest.mark.parametrize("n_entries,shortlist,thr", [(6, 16, 3.0), (40, 5, 3.0), (12, 4, 2.0)])
def test_search_equals_restatement_and_host_path(n_entries, shortlist, thr):
    sift = psift.Sift.new(psift.SiftConfig())
    host, dev = psift.FeatureCatalog(), psift.DeviceCatalog()
    imgs, entries = {}, []
    for i in range(n_entries):
        img = synth.blob_image(256, 192, 60, 2.0, 8.0, seed=2000 + i)
        imgs[i] = img
        f = sift.detect_and_compute_u8(img) if i != 1 else psift.Features.empty(1).head(1)
        entries.append((f"img{i:02d}", 256, 192, f))
        host.upsert_entry(*entries[-1])
        dev.upsert_entry(*entries[-1])
    target = 3
    query = sift.detect_and_compute_u8(
        synth.warp_image(imgs[target], synth.similarity_h(256, 192, 5.0, 1.05, 3.0, -2.0)))
    got = dev.search_features(query, top_k=5, shortlist_k=shortlist, ransac_threshold=thr)
    ref = oracle_search(query, entries, 5, shortlist, psift.DEFAULT_MATCH_RATIO, thr)
    hst = host.search_features(query, top_k=5, shortlist_k=shortlist, ransac_threshold=thr)
    assert got and got[0].id == f"img{target:02d}"
    assert [h.id for h in got] == [r[3] for r in ref] == [h.id for h in hst]
    for g, r, hh in zip(got, ref, hst):
        best, ratio_, votes, _, tr, sim, hom = r
        assert g.coarse_votes == votes == hh.coarse_votes
        t = g.tracking
        assert (t.match_count, t.raw_match_count) == (best, tr.raw_match_count)
        assert t.inlier_ratio == ratio_
        assert t.mean_displacement == (tr.mean_dx, tr.mean_dy)
        assert t.median_displacement == (tr.median_dx, tr.median_dy)
        assert t.mean_scale_ratio == tr.mean_scale_ratio and t.mean_rotation_deg == tr.mean_rotation_deg
        assert t == hh.tracking
        assert (g.transform is None) == (sim is None) and (g.homography is None) == (hom is None)
        if sim is not None:
            np.testing.assert_array_equal(g.transform[:5], sim[:5])
            assert abs(float(g.transform[5]) - float(sim[5])) <= 1e-4  # rotation_deg: atan2f may differ by an ulp
            np.testing.assert_array_equal(g.transform, hh.transform)
        if hom is not None:
            np.testing.assert_array_equal(g.homography, hom)


def test_search_edge_cases():
    dev = psift.DeviceCatalog()
    q = _features(77)
    assert dev.search_features(q) == []  # empty catalog
    dev.upsert_entry("a", 1, 1, _features(78))
    assert dev.search_features(psift.Features.empty(0)) == []
    assert dev.search_features(q, top_k=0) == []
    with pytest.raises(psift.PsiftError):
        dev.search_features(q, ratio_threshold=1.5)
