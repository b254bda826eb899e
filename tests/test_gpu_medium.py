"""The homogeneous medium box on the device against the oracle's restatement
(Medium/Homogeneous.swift:5-23, Medium/HenyeyGreenstein.swift:13-39, the
medium branch of VolumePathIntegrator.swift:286-323 and :394-408 run as
meant), at equal Z-Sobol indices.  Parity with the reference is unpinned:
its integrator never samples a medium (transmittance hard-coded to white).

  - the box scene with a fog box over its floor, MIS as written and corrected,
    forward-scattering phase function;
  - a two-level scene lit by the sky map with the configuration's medium
    coefficients (sigma_a 0.05, sigma_s 0.2) in a box around part of it;
  - a batch of two scenes, one with a medium, equals the scenes rendered
    alone.

Per pixel, GPU and oracle means agree within 3 combined standard errors on
>= 99.5 % of pixels; image means agree to 1 %.
"""
import numpy as np
import pytest

from gonzales_b200 import BatchRenderer, GpuAccelerator, GzgError, InstancedAccelerator, scenes
from gonzales_b200 import _ffi as F
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

FOG = dict(box_min=(0.05, 0.0, 0.05), box_max=(0.95, 0.55, 0.95), sigma_a=(0.4, 0.5, 0.6),
           sigma_s=(2.0, 1.6, 1.2), g=0.4)


def _agree(g, o, spp):
    gm, om = g[0] / spp, o[0] / spp
    gse = np.sqrt(np.maximum(g[1] / spp - gm * gm, 0.0) / spp)
    ose = np.sqrt(np.maximum(o[1] / spp - om * om, 0.0) / spp)
    within = float((np.abs(gm - om) <= 3.0 * np.sqrt(gse ** 2 + ose ** 2) + 1e-4).mean())
    gi = g[0].sum(axis=(0, 1)) / g[2].sum()
    oi = o[0].sum(axis=(0, 1)) / o[2].sum()
    return within, gi, oi


@pytest.mark.parametrize("mis", [0, 1])
def test_box_scene_with_fog_matches_oracle(mis):
    hs = scenes.box_scene().build()
    p = dict(width=64, height=64, spp=32, max_depth=6, rr_min_bounce=3, mis_corrected=mis)
    with GpuAccelerator(hs) as acc:
        plain = acc.render(F.render_params(**p))
        acc.set_medium(FOG)
        g = acc.render(F.render_params(**p))
        assert acc.error_word() == 0
    o = O.render(hs, O.render_params(**p, medium=FOG))
    within, gi, oi = _agree(g, o, p["spp"])
    assert within >= 0.995, within
    np.testing.assert_allclose(gi, oi, rtol=1e-2)
    np.testing.assert_allclose(g[2], o[2], rtol=1e-4)
    # the fog changes the image
    assert np.abs(g[0] / g[2][..., None] - plain[0] / plain[2][..., None]).mean() > 1e-3


def test_instanced_scene_with_environment_and_medium_matches_oracle():
    sky = scenes.sky_map(256, 128)
    blas_hosts, inst = scenes.instanced_scene(n_meshes=4, n_u=30, n_v=20, n_instances=96, extent=5.0,
                                              coloured=True)
    medium = dict(box_min=(-4.0, -2.0, -4.0), box_max=(4.0, 3.0, 4.0), sigma_a=(0.05, 0.05, 0.05),
                  sigma_s=(0.2, 0.2, 0.2), g=0.0)
    p = dict(width=64, height=48, spp=16, max_depth=5, rr_min_bounce=2, eye=(0.0, 2.0, 16.0),
             target=(0.0, 0.0, 0.0))
    blas = [GpuAccelerator(h) for h in blas_hosts]
    with InstancedAccelerator(blas, inst) as acc:
        acc.set_environment(sky, 1.0)
        acc.set_medium(medium)
        g = acc.render(F.render_params(**p))
        tlas, leaf = acc.tlas_nodes, acc.leaf_instance
        assert acc.error_word() == 0
    for b in blas:
        b.close()
    o = O.render(None, O.render_params(**p, medium=medium), env=O.Environment(sky, 1.0),
                 instances=dict(tlas_nodes=tlas, leaf_instance=leaf, instances=inst, blas=blas_hosts))
    within, gi, oi = _agree(g, o, p["spp"])
    assert within >= 0.995, within
    np.testing.assert_allclose(gi, oi, rtol=1e-2)


def test_batch_with_a_medium_scene_equals_solo_renders():
    import torch

    a_host = scenes.box_scene().build()
    b_host = scenes.batch_scene(21, 2_000).build()
    pa = F.render_params(40, 32, 8, max_depth=5, rr_min_bounce=3)
    pb = F.render_params(32, 32, 8, max_depth=4, rr_min_bounce=2)
    with GpuAccelerator(a_host) as a, GpuAccelerator(b_host) as b:
        a.set_medium(FOG)
        solo = [a.render(pa), b.render(pb)]
        with BatchRenderer([a, b], [pa, pb]) as r:
            rgb = torch.zeros((r.pixels, 3), device="cuda")
            w = torch.zeros((r.pixels,), device="cuda")
            r.render(rgb, w)
            torch.cuda.synchronize()
            parts = list(zip(r.split(rgb.cpu().numpy()), r.split(w.cpu().numpy())))
    for (img, wt), s in zip(parts, solo):
        np.testing.assert_allclose(img, s[0], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(wt, s[2], rtol=1e-6)


def test_medium_arguments_are_checked():
    hs = scenes.box_scene().build()
    with GpuAccelerator(hs) as acc:
        with pytest.raises(GzgError):
            acc.set_medium(dict(FOG, box_max=FOG["box_min"]))
        with pytest.raises(GzgError):
            acc.set_medium(dict(FOG, sigma_a=(-1.0, 0.0, 0.0)))
        with pytest.raises(GzgError):
            acc.set_medium(dict(FOG, g=1.0))
        acc.set_medium(FOG)
        acc.set_medium(None)
        p = F.render_params(16, 16, 4, max_depth=3)
        plain = acc.render(p)
        with GpuAccelerator(hs) as ref:
            np.testing.assert_allclose(plain[0], ref.render(p)[0], rtol=1e-6)
