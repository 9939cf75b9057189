"""The zero-byte rule that the oracle's MIH votes (and the GPU's scan path)
evaluate equals the reference's own table walk: the 16 x 256 inverted tables
and per-query seen_stamp (src/catalog.rs:291-321, :596-615), restated literally
in oracle_mih_votes_tables."""
import numpy as np
import pytest

import mih_cases
import oracle as O


@pytest.mark.parametrize("n_entries,n_queries,seed", [(40, 200, 1), (120, 500, 2), (33, 64, 3), (300, 1000, 4)])
def test_zero_byte_rule_equals_table_walk(n_entries, n_queries, seed):
    q, cat, off = mih_cases.case(n_entries, n_queries, seed)
    walk = O.mih_votes_tables(q, cat, off)
    rule = O.hamming_votes(q, cat, off, True)
    np.testing.assert_array_equal(rule, walk)
    assert walk.sum() > 0
    # the exhaustive rule counts the no-shared-byte codes the MIH walk cannot reach
    exh = O.hamming_votes(q, cat, off, False)
    assert (exh >= walk).all() and exh.sum() > walk.sum()


def test_table_walk_empty_inputs():
    q, cat, off = mih_cases.case(40, 10, 5)
    assert O.mih_votes_tables(q[:0], cat, off).sum() == 0
    off0 = np.zeros(41, np.int64)
    assert O.mih_votes_tables(q, cat[:0], off0).sum() == 0
