"""The oracle against the reference's own golden render.

Tests/reference/regression-test.pbrt (a Cornell box of eight triangle meshes:
128 x 128, 64 samples per pixel, maximum depth 4, Gaussian filter radius 5 and
sigma 2.5, area light L = (17, 12, 4)) rendered by the reference is
Tests/reference/regression-test.exr; the reference's test accepts a render
whose normalised RMSE against it is below 0.1 (Tests/libgonzalesTests/
RenderRegressionTests.swift:40-62).  Both are committed as
tests/golden/regression_test.npz by tests/golden/make_regression_golden.py.

The golden image is the output of Film.writeImages, which always runs Open
Image Denoise on the film (Core/Film.swift:40-58): it is smooth where a raw
64-sample render is noisy, so a raw render meets the bound only once its own
noise is small.  The oracle's restatement of the loop that actually runs
(camera rays, the Mojo traversal, shade_core; Core/Tile.swift:19-223) is
checked at 256 samples per pixel: normalised RMSE below the reference's 0.1
and channel means within 2 %.
"""
import numpy as np

from gonzales_b200.tile import normalized
from oracle import pyoracle as O
from tests import helpers as H


def test_fixture_holds_the_reference_scene_and_image():
    z = H.regression_fixture()
    assert z["golden"].shape == (128, 128, 4)
    assert np.all(z["golden"][..., 3] == 1.0)
    assert int(z["spp"]) == 64 and int(z["max_depth"]) == 4
    assert list(z["mesh_materials"]) == ["Floor", "Ceiling", "BackWall", "RightWall", "LeftWall", "ShortBox",
                                         "TallBox", "Light"]
    sb, kw = H.regression_scene(z)
    hs = sb.build()
    assert hs.triangle_count == 5 * 2 + 2 * 12 + 2
    assert np.allclose(kw["eye"], (0.0, 1.0, 6.8)) and np.allclose(kw["target"], (0.0, 1.0, 5.8))


def test_oracle_tile_loop_matches_reference_golden_render():
    z = H.regression_fixture()
    sb, kw = H.regression_scene(z)
    hs = sb.build()
    kw = dict(kw, spp=256)
    light, weight = H.oracle_tile_loop(hs, O.render_params(**kw), seed=7)
    img = normalized(light, weight)
    golden = z["golden"][..., :3]
    rmse = H.normalised_rmse(img, golden)
    H.record("regression_oracle.json", {"spp": 256, "normalised_rmse": rmse})
    assert rmse < 0.1, rmse
    mean, gmean = img.mean((0, 1)), golden.mean((0, 1))
    assert np.all(np.abs(mean / gmean - 1.0) < 0.02), (mean, gmean)
