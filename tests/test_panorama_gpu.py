"""stitch_panorama on the GPU against the CPU restatement (src/stitch.rs).

Compositing (psift_panorama_composite) on the restatement's registration results
must give the restatement's canvas byte for byte: every kernel evaluates the
reference's per-pixel f64 / f32 expressions in its order and the images'
contributions are accumulated in the reference's image order.  The whole entry
(psift_stitch_panorama) must register the same images with the same reference,
gains and homographies (the features are the restatement's; matching and RANSAC
equal it) and then the same canvas.  The cylindrical warp evaluates cos / tan in
f64 with CUDA's functions rather than glibc's, so a pixel whose bilinear sum lies
within an ulp of a rounding boundary can differ by one level: at most 1 level,
on at most 0.1 % of the channel values."""
import numpy as np
import pytest

import oracle as O
import panorama_cases as P
import psift

pytestmark = pytest.mark.gpu


def _reg_case(tiles, blend):
    reg = O.panorama_register(tiles, O.PanoramaOptions.default(blend=blend))
    assert not isinstance(reg, int), reg
    return reg


@pytest.mark.parametrize("blend", [0, 1])
@pytest.mark.parametrize("case", ["aerial", "blobs"])
def test_composite_equals_restatement(case, blend):
    tiles = P.aerial_tiles()[0] if case == "aerial" else P.blob_tiles()
    reg = _reg_case(tiles, blend)
    want = O.panorama_composite(tiles, reg, blend, 4)
    got = psift.panorama_composite(tiles, reg["registered"], reg["gains"], reg["inv"], reg["origin"], reg["width"],
                                   reg["height"], blend, 4)
    assert got.shape == want.shape
    diff = np.abs(got.astype(int) - want.astype(int))
    assert diff.max() == 0, (int((diff > 0).sum()), int(diff.max()))


@pytest.mark.parametrize("levels", [1, 2, 6])
def test_composite_levels(levels):
    tiles = P.blob_tiles()
    reg = _reg_case(tiles, 1)
    want = O.panorama_composite(tiles, reg, 1, levels)
    got = psift.panorama_composite(tiles, reg["registered"], reg["gains"], reg["inv"], reg["origin"], reg["width"],
                                   reg["height"], 1, levels)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("blend", [1, 0])
def test_stitch_panorama_four_tiles(blend):
    """The reference's 4-tile test on the GPU entry, and equality with the restatement."""
    tiles, w = P.aerial_tiles()
    opt = psift.PanoramaOptions.default(blend=blend)
    res = psift.stitch_panorama(tiles, opt)
    assert len(res.registered_indices) == 4
    assert res.image.shape[1] > (w * 85) // 100
    ref_f = P.FACTORS[res.reference_index]
    for i, f in enumerate(P.FACTORS):
        assert abs(res.gains[i] - ref_f / f) < 0.15
    canvas, reg = O.stitch_panorama(tiles, O.PanoramaOptions.default(blend=blend))
    assert res.reference_index == reg["ref"]
    np.testing.assert_array_equal(np.array(res.registered_indices), np.nonzero(reg["registered"])[0])
    np.testing.assert_array_equal(res.gains, reg["gains"])
    for i in res.registered_indices:
        np.testing.assert_array_equal(res.homographies[i], reg["h_to_ref"][i].astype(np.float32))
    assert res.origin == tuple(reg["origin"])
    np.testing.assert_array_equal(res.image, canvas)


def test_stitch_panorama_blobs_cylindrical():
    tiles = P.blob_tiles()
    opt = psift.PanoramaOptions.default(projection=1, focal_px=900.0, blend=1)
    res = psift.stitch_panorama(tiles, opt)
    out = O.stitch_panorama(tiles, O.PanoramaOptions.default(projection=1, focal_px=900.0, blend=1))
    assert not isinstance(out, int)
    canvas, reg = out
    assert res.reference_index == reg["ref"] and len(res.registered_indices) == int(reg["registered"].sum())
    # the warped inputs may differ by a level on rare pixels (cos / tan), so the
    # registration can move by a hair; the canvases agree on all but a few pixels
    if res.image.shape == canvas.shape:
        diff = np.abs(res.image.astype(int) - canvas.astype(int))
        assert (diff > 2).mean() < 0.01


def test_cylindrical_warp_within_a_level():
    tiles, _ = P.aerial_tiles()
    for img in (tiles[0], P.blob_tiles()[1]):
        for f in (650.0, 0.0):
            got = psift.warp_cylindrical(img, f)
            want = O.warp_cylindrical(img, f)
            diff = np.abs(got.astype(int) - want.astype(int))
            assert diff.max() <= 1 and (diff > 0).mean() <= 1e-3, (diff.max(), (diff > 0).mean())
            assert got[img.shape[0] // 2, img.shape[1] // 2, 3] == 255


def test_panorama_errors_carry_the_reference_messages():
    tiles, _ = P.aerial_tiles()
    with pytest.raises(ValueError, match="at least 2 input images"):
        psift.stitch_panorama(tiles[:1])
    flat = [np.full((120, 160, 4), 128, np.uint8) for _ in range(3)]
    with pytest.raises(ValueError, match="No valid overlapping image pairs"):
        psift.stitch_panorama(flat)
    with pytest.raises(ValueError, match="exceeds safety limits"):
        psift.stitch_panorama(tiles, psift.PanoramaOptions.default(max_canvas_dim=300))
