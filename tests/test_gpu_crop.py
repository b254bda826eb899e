"""Crop windows (Film's crop, the pixels Film.getSampleBounds covers,
Core/Film.swift:7-27) and the two-level configuration at its full frame.

  - a crop window of a frame equals that window of the whole frame (same
    camera, same Z-Sobol samples per pixel), on the device and in the
    oracle's restatement;
  - the two-level configuration itself (16 meshes of 50,000 triangles, 4096
    instances, the 1024 x 512 sky map, the five material kinds, the medium
    box, depth 8, roulette from bounce 2, 1920 x 1080) rendered on a 160 x 90
    crop at the frame's centre at 16 spp agrees per pixel with the oracle's
    render of the same crop.
"""
import numpy as np
import pytest

from gonzales_b200 import GpuAccelerator, InstancedAccelerator, scenes
from gonzales_b200 import _ffi as F
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

MEDIUM = dict(box_min=(-10.0, -6.0, -10.0), box_max=(10.0, 6.0, 10.0), sigma_a=(0.05, 0.05, 0.05),
              sigma_s=(0.2, 0.2, 0.2), g=0.0)


def test_crop_equals_window_of_whole_frame():
    hs = scenes.box_scene().build()
    p = dict(width=64, height=48, spp=8, max_depth=5, rr_min_bounce=3, mis_corrected=1)
    with GpuAccelerator(hs) as acc:
        full = acc.render(F.render_params(**p))
        crop = acc.render(F.render_params(**p, crop=(12, 7, 40, 30)))
    assert crop[0].shape == (23, 28, 3)
    np.testing.assert_allclose(crop[0], full[0][7:30, 12:40], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(crop[2], full[2][7:30, 12:40], rtol=1e-6)
    assert crop[3]["camera_rays"] == 23 * 28 * 8
    o = O.render(hs, O.render_params(**p, crop=(12, 7, 40, 30)))
    np.testing.assert_allclose(crop[2], o[2], rtol=1e-4)


def test_bad_crop_is_rejected():
    from gonzales_b200 import GzgError

    hs = scenes.box_scene().build()
    with GpuAccelerator(hs) as acc:
        for bad in ((10, 10, 10, 20), (0, 0, 65, 10), (-1, 0, 5, 5)):
            with pytest.raises(GzgError):
                acc.render(F.render_params(64, 48, 1, crop=bad))


def _agree(g, o, spp):
    gm, om = g[0] / spp, o[0] / spp
    gse = np.sqrt(np.maximum(g[1] / spp - gm * gm, 0.0) / spp)
    ose = np.sqrt(np.maximum(o[1] / spp - om * om, 0.0) / spp)
    within = float((np.abs(gm - om) <= 3.0 * np.sqrt(gse ** 2 + ose ** 2) + 1e-4).mean())
    gi = g[0].sum(axis=(0, 1)) / g[2].sum()
    oi = o[0].sum(axis=(0, 1)) / o[2].sum()
    return within, gi, oi


def test_two_level_configuration_crop_matches_oracle():
    from tests import helpers

    blas_hosts, inst = scenes.instanced_scene(mixed=True)
    sky = scenes.sky_map()
    p = dict(width=1920, height=1080, spp=16, max_depth=8, rr_min_bounce=2, eye=(0.0, 6.0, 48.0),
             target=(0.0, 0.0, 0.0), crop=(880, 495, 1040, 585))
    blas = [GpuAccelerator(h) for h in blas_hosts]
    with InstancedAccelerator(blas, inst) as acc:
        acc.set_environment(sky, 1.0)
        acc.set_medium(MEDIUM)
        g = acc.render(F.render_params(**p))
        tlas, leaf = acc.tlas_nodes, acc.leaf_instance
        assert acc.error_word() == 0
    for b in blas:
        b.close()
    o = O.render(None, O.render_params(**p, medium=MEDIUM), env=O.Environment(sky, 1.0),
                 instances=dict(tlas_nodes=tlas, leaf_instance=leaf, instances=inst, blas=blas_hosts))
    within, gi, oi = _agree(g, o, p["spp"])
    helpers.record("two_level_crop_vs_oracle.json", {"crop": p["crop"], "spp": p["spp"], "within_3se": within,
                                                     "mean_gpu": gi.tolist(), "mean_oracle": oi.tolist()})
    assert g[0].shape == (90, 160, 3)
    assert within >= 0.99, within
    np.testing.assert_allclose(gi, oi, rtol=2e-2)
    np.testing.assert_allclose(g[2], o[2], rtol=1e-4)
