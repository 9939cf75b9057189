"""compute_sift_descriptors (the explicit-keypoint path), summarize_tracking and
FeatureCatalog::search_features on the GPU, against the CPU restatement."""
import numpy as np
import pytest

import oracle as O
import psift
import synth
from ransac_cases import similarity_14

pytestmark = pytest.mark.gpu


def test_compute_descriptors_equals_oracle():
    img = O.luma_to_f32(synth.blob_image(400, 300, 120, 2.0, 10.0, seed=31))
    kps = O.detect_keypoints(img, 4, 3, 0.015, True)
    ref_meta, ref_desc = O.compute_descriptors(img, kps, 0)
    got = psift.compute_sift_descriptors(img, kps)
    assert len(got) == ref_meta.shape[0] > 0
    np.testing.assert_array_equal(got.x, ref_meta[:, 0])
    rel = np.linalg.norm(got.descriptors - ref_desc, axis=1) / np.linalg.norm(ref_desc, axis=1)
    assert np.mean(rel <= 1e-4) >= 0.995
    # keypoints without layer information take the log2 fallback
    k2 = kps.copy()
    k2["layer"] = 0
    m2, d2 = O.compute_descriptors(img, k2, 1)
    g2 = psift.compute_sift_descriptors(img, k2, kind=1)
    assert len(g2) == m2.shape[0]


def test_summarize_tracking_known_answer():
    m = similarity_14()
    qs = np.full(14, 1.26, np.float32)
    qo = np.r_[np.ones(10), np.full(4, 2.5)].astype(np.float32)
    ts = np.r_[np.full(10, 1.26), np.full(4, 2.52)].astype(np.float32)
    to = np.r_[np.ones(10), np.full(4, 0.2)].astype(np.float32)
    q = psift.Features(np.zeros(14, np.float32), np.zeros(14, np.float32), qs, np.zeros(14, np.float32), qo,
                       np.zeros((14, 128), np.float32))
    t = psift.Features(np.zeros(14, np.float32), np.zeros(14, np.float32), ts, np.zeros(14, np.float32), to,
                       np.zeros((14, 128), np.float32))
    s = psift.summarize_tracking(q, t, m)
    r = O.summarize_tracking(m, qs, qo, ts, to)
    assert (s.raw_match_count, s.match_count) == (14, 10) == (r.raw_match_count, r.match_count)
    assert s.mean_displacement == (r.mean_dx, r.mean_dy)
    assert s.median_displacement == (r.median_dx, r.median_dy)
    assert s.mean_scale_ratio == r.mean_scale_ratio and s.mean_rotation_deg == r.mean_rotation_deg


@pytest.mark.parametrize("n_entries", [6, 40])
def test_catalog_search_ranks_the_matching_image_first(n_entries):
    # tests/coverage_gaps.rs:30-59 and tests/pipeline_tests.rs:840-877, :1439-1489 (MIH above 32 entries)
    sift = psift.Sift.new(psift.SiftConfig())
    cat = psift.FeatureCatalog()
    imgs = {}
    for i in range(n_entries):
        img = synth.blob_image(256, 192, 60, 2.0, 8.0, seed=1000 + i)
        imgs[f"img{i:02d}"] = img
        cat.upsert_entry(f"img{i:02d}", 256, 192, sift.detect_and_compute_u8(img))
    target = "img03"
    query = synth.warp_image(imgs[target], synth.similarity_h(256, 192, 5.0, 1.05, 3.0, -2.0))
    hits = cat.search_features(sift.detect_and_compute_u8(query))
    assert hits and hits[0].id == target
    # votes equal the restatement's for the same semantics
    qf = sift.detect_and_compute_u8(query)
    votes, mih = cat.coarse_votes(qf)
    qs = O.quantize_u128(qf.descriptors)
    sig = np.concatenate([e.signatures for e in cat.entries])
    off = np.concatenate([[0], np.cumsum([len(e.signatures) for e in cat.entries])])
    np.testing.assert_array_equal(votes, O.hamming_votes(qs, sig, off, mih))
    assert cat.remove(target) and not cat.remove(target)
    assert all(h.id != target for h in cat.search_features(qf))
