"""gaussian_blur and the scale-space pyramid on the GPU, plane by plane against
the CPU restatement: bit-identical (the blur is a fixed sequence of rounded f32
multiplies and adds, identical on both sides)."""
import numpy as np
import pytest

import oracle as O
import psift
import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("sigma", [0.5, 1.2489996, 1.6, 2.452, 3.09, 4.9])
@pytest.mark.parametrize("shape", [(480, 640), (67, 131), (5, 300), (300, 5), (1, 1), (2, 40)])
def test_gaussian_blur_bit_exact(sigma, shape):
    rng = np.random.default_rng(int(sigma * 100) + shape[0])
    img = rng.random(shape, dtype=np.float32)
    np.testing.assert_array_equal(psift.gaussian_blur(img, sigma), O.gaussian_blur(img, sigma))


def test_gaussian_blur_rejects_huge_sigma():
    with pytest.raises(psift.PsiftError):
        psift.gaussian_blur(np.zeros((8, 8), np.float32), 6.0)


@pytest.mark.parametrize("upsample", [True, False])
@pytest.mark.parametrize("octaves,scales,shape", [(4, 3, (480, 640)), (3, 5, (241, 163)), (2, 10, (100, 77))])
def test_pyramid_planes_bit_exact(upsample, octaves, scales, shape):
    img = O.luma_to_f32(synth.blob_image(shape[1], shape[0], 120, 1.5, 12.0, seed=shape[0]))
    ref = O.Pyramid(img, octaves, scales, upsample)
    cfg = psift.SiftConfig().with_octaves(octaves).with_scales(scales).upsample_first_octave(upsample)
    got = psift.build_pyramid(img, cfg)
    assert len(got) == ref.num_octaves
    for o, (g, d) in enumerate(got):
        assert g.shape[1:] == ref.octave_info(o)[:2]
        for i in range(scales + 3):
            np.testing.assert_array_equal(g[i], ref.plane(o, "g", i), err_msg=f"octave {o} gaussian {i}")
        for i in range(scales + 2):
            np.testing.assert_array_equal(d[i], ref.plane(o, "d", i), err_msg=f"octave {o} dog {i}")
