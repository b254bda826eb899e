"""The oracle's camera: PerspectiveCamera.generateRay with depthOfField
(Camera/PerspectiveCamera.swift:25-48).  A lens radius of 0 is the pinhole
exactly; a lens moves the ray origins over the lens disk while, as written,
the directions stay the pinhole ones: the image shifts slightly, its overall
brightness stays close."""
import numpy as np

from gonzales_b200 import scenes
from oracle import pyoracle as O


def test_zero_lens_radius_is_the_pinhole():
    hs = scenes.box_scene().build()
    a = O.render(hs, O.render_params(32, 32, 4, max_depth=3))
    b = O.render(hs, O.render_params(32, 32, 4, max_depth=3, lens_radius=0.0, focal_distance=5.0))
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])


def test_lens_moves_rays():
    hs = scenes.box_scene().build()
    a = O.render(hs, O.render_params(48, 48, 8, max_depth=3))
    c = O.render(hs, O.render_params(48, 48, 8, max_depth=3, lens_radius=0.05, focal_distance=1.5))
    assert not np.allclose(a[0], c[0])
    np.testing.assert_allclose(a[0].sum() / a[2].sum(), c[0].sum() / c[2].sum(), rtol=0.1)
    assert a[3]["camera"] == c[3]["camera"]
