"""search_features (src/catalog.rs:576-702) composed from the CPU restatement's
stages: the checker for the device-resident catalog's search."""
import numpy as np

import oracle as O


def oracle_search(query, entries, top_k, shortlist_k, ratio, thr):
    """search_features (src/catalog.rs:576-702) composed from the restatement's stages.
    entries: list of (id, width, height, Features)."""
    if not entries or len(query) == 0 or top_k == 0:
        return []
    qs = O.quantize_u128(query.descriptors)
    sigs = [O.quantize_u128(f.descriptors) if len(f) else np.zeros((0, 2), np.uint64) for _, _, _, f in entries]
    off = np.concatenate([[0], np.cumsum([len(s) for s in sigs])]).astype(np.int64)
    mih = len(entries) > 32
    votes = O.hamming_votes(qs, np.concatenate(sigs), off, mih)
    cands = [(i, int(v)) for i, v in enumerate(votes) if v > 0 or not mih]
    if len(cands) > max(shortlist_k, 1):
        cands.sort(key=lambda c: (-c[1], entries[c[0]][0].encode()))
        cands = cands[:max(shortlist_k, 1)]
    hits = []
    for i, v in cands:
        id_, w, h, f = entries[i]
        if len(f) < 2:
            continue
        raw = O.match(query.descriptors, f.descriptors, query.xy, f.xy, ratio)
        if len(raw) == 0:
            continue
        tr = O.summarize_tracking(raw, query.scale, query.orientation, f.scale, f.orientation)
        sim_mask, sim = O.similarity_ransac(raw, thr)
        hom_mask, hom = O.homography_ransac(raw, thr)
        best = max(int(hom_mask.sum()), int(sim_mask.sum()))
        ratio_ = float(np.float32(best) / np.float32(tr.raw_match_count))
        hits.append((best, ratio_, v, id_, tr, sim, hom))
    hits.sort(key=lambda t: (-t[0], -t[1], -t[2], t[3].encode()))
    return hits[:top_k]
