"""The reference's invariance sweeps (tests/invariance_sweeps.rs:83-217) on its own
sample image through the CUDA path (detect_and_compute_u8, Lowe matching, similarity
RANSAC): the reference's minimum inlier counts and model errors, and inlier counts
within 1 % of the CPU restatement's on the same warped images."""
import pytest

import oracle as O
import psift
import sweep_cases as S

pytestmark = pytest.mark.gpu


def _gpu_fns():
    sift = psift.Sift.new(psift.SiftConfig().with_octaves(S.SWEEP_OCTAVES).with_scales(S.SWEEP_SCALES)
                          .with_contrast_threshold(0.015))
    extract = sift.detect_and_compute_u8
    match = lambda a, b: psift.match_descriptors(a, b, 0.75)

    def similarity(m):
        inl, model = psift.filter_matches_ransac(m, 3.0)
        return len(inl), model
    return extract, match, similarity


def _cpu_fns():
    extract = lambda u8: O.detect_and_compute(O.luma_to_f32(u8), S.SWEEP_OCTAVES, S.SWEEP_SCALES, 0.015, True, 0, 4096)
    match = lambda a, b: O.match(a[1], b[1], a[0][:, :2], b[0][:, :2], 0.75)

    def similarity(m):
        mask, model = O.similarity_ransac(m, 3.0)
        return int(mask.sum()), model
    return extract, match, similarity


@pytest.mark.parametrize("which", ["scale", "rotation"])
def test_invariance_sweep_gpu(which):
    gpu = S.run_sweeps(*_gpu_fns(), which=(which,))
    cpu = S.run_sweeps(*_cpu_fns(), which=(which,))
    for g, c in zip(gpu, cpu):
        print("%-26s GPU inliers %5d  CPU restatement %5d (min %4d)  scale %.4f  rotation %.2f"
              % (g[0], g[1], c[1], g[2], g[3], g[4]))
        assert abs(g[1] - c[1]) <= 0.01 * c[1] + 2, (g, c)
