"""The oracle's homogeneous medium box (Medium/Homogeneous.swift,
Medium/HenyeyGreenstein.swift), on checks with known answers.

The reference's integrator never samples its media (VolumePathIntegrator.
swift:394 hard-codes the transmittance to white), so nothing the reference
ran pins these: parity unpinned.  The restatement runs the branch as meant.
Checks:
  - an emitter seen through a purely absorbing gray medium keeps exp(-sigma_a
    x length) of its radiance (no scattering event can add light);
  - a medium with zero coefficients leaves the image unchanged;
  - a scattering medium conserves energy in the sense that a white, purely
    scattering fog in front of a light changes the mean image only by the
    light it scatters out of view (the image stays within the no-fog image
    and the fully-absorbed one).
"""
import numpy as np

from gonzales_b200.scene import SceneBuilder
from gonzales_b200.tile import normalized
from oracle import pyoracle as O


def _emitter_scene():
    sb = SceneBuilder()
    sb.add_material((0.5, 0.5, 0.5))
    # a large quad at z = 0 facing +z (toward the camera)
    pts = np.array([(-2, -2, 0), (2, -2, 0), (2, 2, 0), (-2, 2, 0)], np.float32)
    sb.add_area_light(pts, np.array([0, 1, 2, 0, 2, 3]), (2.0, 1.0, 0.5))
    return sb.build()


def _render(hs, **kw):
    base = dict(width=24, height=24, spp=256, max_depth=3, rr_min_bounce=9, mis_corrected=1, eye=(0.0, 0.0, 5.0),
                target=(0.0, 0.0, 0.0), fov_deg=20.0)
    base.update(kw)
    r = O.render(hs, O.render_params(**base))
    return normalized(r[0].astype(np.float64), r[2].astype(np.float64))


def test_absorbing_medium_attenuates_by_beer_lambert():
    hs = _emitter_scene()
    clear = _render(hs)
    sa = 0.7
    fog = _render(hs, medium=dict(box_min=(-3, -3, 1.0), box_max=(3, 3, 2.0), sigma_a=(sa, sa, sa),
                                  sigma_s=(0, 0, 0), g=0.0))
    # camera rays cross the slab 1 <= z <= 2 over about 1 / cos(angle) ~ 1.0-1.01
    ratio = fog.mean((0, 1)) / clear.mean((0, 1))
    assert np.all(np.abs(ratio - np.exp(-sa * 1.005)) < 0.02), ratio


def test_zero_medium_leaves_image_unchanged():
    hs = _emitter_scene()
    clear = _render(hs)
    zero = _render(hs, medium=dict(box_min=(-3, -3, 1.0), box_max=(3, 3, 2.0), sigma_a=(0, 0, 0),
                                   sigma_s=(0, 0, 0), g=0.0))
    np.testing.assert_allclose(zero, clear, rtol=1e-6, atol=1e-7)


def test_scattering_medium_between_clear_and_absorbed():
    hs = _emitter_scene()
    box = dict(box_min=(-3, -3, 1.0), box_max=(3, 3, 2.0), g=0.5)
    clear = _render(hs).mean()
    scat = _render(hs, medium=dict(box, sigma_a=(0, 0, 0), sigma_s=(0.7, 0.7, 0.7))).mean()
    absorbed = _render(hs, medium=dict(box, sigma_a=(0.7, 0.7, 0.7), sigma_s=(0, 0, 0))).mean()
    assert absorbed < scat < clear, (absorbed, scat, clear)
