"""The CPU restatement of stitch_panorama (src/stitch.rs) pinned by the
reference's own panorama tests (tests/panorama_tests.rs): the 4-tile
exposure-compensated multi-band panorama registers every tile, spans more than
85 % of the source width, and its solved gains are within 0.15 of the inverse
exposure ratios relative to the reference tile; the cylindrical warp keeps the
image size and an opaque centre."""
import numpy as np
import pytest

import oracle as O
import panorama_cases as P


@pytest.mark.parametrize("blend", [1, 0])
def test_four_tile_panorama_pins(blend):
    tiles, w = P.aerial_tiles()
    out = O.stitch_panorama(tiles, O.PanoramaOptions.default(blend=blend))
    assert not isinstance(out, int), out
    canvas, reg = out
    assert reg["registered"].sum() == 4
    assert canvas.shape[1] > (w * 85) // 100
    ref_f = P.FACTORS[reg["ref"]]
    for i, f in enumerate(P.FACTORS):
        assert abs(reg["gains"][i] - ref_f / f) < 0.15, (i, reg["gains"])


def test_cylindrical_warp_pins():
    tiles, _ = P.aerial_tiles()
    img = tiles[1]
    cyl = O.warp_cylindrical(img, 650.0)
    assert cyl.shape == img.shape
    assert cyl[img.shape[0] // 2, img.shape[1] // 2, 3] == 255


def test_exposure_gains_known_answers():
    # no overlaps: the prior keeps every gain at 1
    assert np.array_equal(O.solve_exposure_gains(np.zeros((0, 5)), 3, 0), np.ones(3, np.float32))
    # two images, image 1 twice as bright in the overlap: its gain tends to 1/2
    g = O.solve_exposure_gains([[0, 1, 1e6, 100.0, 200.0]], 2, 0)
    assert g[0] == 1.0 and abs(g[1] - 0.5) < 1e-3
    # clamped to [0.4, 2.5]
    g = O.solve_exposure_gains([[0, 1, 1e6, 100.0, 1000.0]], 2, 0)
    assert g[1] == np.float32(0.4)


def test_too_few_images_is_an_error():
    tiles, _ = P.aerial_tiles()
    assert O.stitch_panorama(tiles[:1], O.PanoramaOptions.default()) == -1
