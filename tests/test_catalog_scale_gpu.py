"""Catalog search at the size of the 2M-code workload, bit for bit against the CPU
restatement: 2,000,000 SIFT-like catalog descriptors (|N(0,1)|, L2-normalised,
clipped at 0.2, renormalised; 10,000 images x 200), binarised by the reference's
quantize_descriptor_u128 (src/catalog.rs:37-45), 4096 queries that are perturbed
catalog descriptors, XOR+POPCNT top-64 with the (distance, index) tiebreak, then
the exact f32 L2 re-rank of the 64.  Codes, top-64 lists and re-ranked lists must
equal the restatement's (OpenMP over the queries) exactly."""
import numpy as np
import pytest

import oracle as O
import psift

pytestmark = pytest.mark.gpu


def _workload(torch, n_cat=2_000_000, n_q=4096):
    g = torch.Generator(device="cuda")
    g.manual_seed(4)
    cat = torch.randn((n_cat, 128), generator=g, device="cuda").abs_()
    cat /= cat.norm(dim=1, keepdim=True)
    cat.clamp_(max=0.2)
    cat /= cat.norm(dim=1, keepdim=True)
    pick = torch.randint(0, n_cat, (n_q,), generator=g, device="cuda")
    q = cat[pick] + 0.02 * torch.randn((n_q, 128), generator=g, device="cuda").abs_()
    q /= q.norm(dim=1, keepdim=True)
    return cat.cpu().numpy(), q.cpu().numpy(), pick.cpu().numpy()


def test_topk_2M_x_4096_bit_exact():
    import torch
    cat, q, pick = _workload(torch)
    cat_codes = psift.quantize_descriptor_u128(cat)
    q_codes = psift.quantize_descriptor_u128(q)
    np.testing.assert_array_equal(cat_codes, O.quantize_u128(cat))
    np.testing.assert_array_equal(q_codes, O.quantize_u128(q))
    gi, gd = psift.hamming_topk(q_codes, cat_codes, 64)
    ci, cd = O.hamming_topk(q_codes, cat_codes, 64)
    np.testing.assert_array_equal(gd, cd)
    np.testing.assert_array_equal(gi, ci)
    # the shortlist finds each query's source descriptor
    assert (gi == pick[:, None]).any(axis=1).mean() > 0.99
    ri, rd = psift.l2_rerank(q, cat, gi)
    ori, ord2 = O.l2_rerank(q, cat, ci)
    np.testing.assert_array_equal(ri, ori)
    np.testing.assert_array_equal(rd.view(np.uint32), ord2.view(np.uint32))
