"""The reference's MIH catalog test (tests/pipeline_tests.rs:1439-1489) on the CPU
restatement: 40 entries (above the 32 that switch the coarse votes to multi-index
hashing), the sample image's features at entry 17 among two synthetic distractor
scenes; searching with the sample's own features ranks item_17 first.  The votes
also equal the reference's own table walk (inverted tables + seen_stamp)."""
import numpy as np

import oracle as O
import psift
import scene_cases
import sweep_cases
from catalog_oracle import oracle_search


def _features(u8):
    meta, desc = O.detect_and_compute(O.luma_to_f32(u8), 3, 3, 0.015, True, 0, 4096)
    return psift.Features(*(meta[:, i].copy() for i in range(5)), desc)


def test_mih_indexed_search_ranks_the_planted_entry_first():
    target = _features(sweep_cases.aerial_west_luma())
    d1 = _features(scene_cases.render_synthetic_scene(1))
    d2 = _features(scene_cases.render_synthetic_scene(2))
    entries = [(f"item_{i:02d}.png", 220, 220, target if i == 17 else (d1 if i % 2 == 0 else d2)) for i in range(40)]
    hits = oracle_search(target, entries, 3, 8, psift.DEFAULT_MATCH_RATIO, psift.DEFAULT_RANSAC_REPROJ_THRESHOLD)
    assert hits and hits[0][3] == "item_17.png"
    qs = O.quantize_u128(target.descriptors)
    sigs = [O.quantize_u128(f.descriptors) for _, _, _, f in entries]
    off = np.concatenate([[0], np.cumsum([len(s) for s in sigs])]).astype(np.int64)
    np.testing.assert_array_equal(O.hamming_votes(qs, np.concatenate(sigs), off, True),
                                  O.mih_votes_tables(qs, np.concatenate(sigs), off))
