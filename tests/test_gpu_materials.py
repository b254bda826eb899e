"""Dielectric and coated-diffuse materials on the device renderer against the
oracle's restatement (Bsdf/DielectricBsdf.swift, Bsdf/LayeredBsdf.swift,
the surface estimate of VolumePathIntegrator.swift:325-371 with a general
BSDF), at equal Z-Sobol indices:

  - the box scene with a coated box, a rough dielectric box, a smooth
    (specular) dielectric sphere, a coated sphere, a copper sphere and a
    coated-conductor box, MIS as written and corrected, with and without the
    sky map (specular paths reach the emitter and the environment);
  - a two-level scene of diffuse, coated-diffuse, dielectric, conductor and
    coated-conductor meshes (roughness uniform in [0.05, 0.5]) under the sky
    map;
  - a batch mixing the material scene with the diffuse box scene equals the
    solo renders;
  - first-hit albedo: white for a dielectric and the conductors, the base for
    a coated diffuse.

Per pixel, GPU and oracle means agree within 3 combined standard errors on
>= 99 % of pixels and image means agree to 1.5 %.  The coated BSDF's
stochastic layer walk seeds from quantised directions, so most evaluations
see the same stream on both sides and most pixels agree far more closely.
"""
import numpy as np
import pytest

from gonzales_b200 import BatchRenderer, GpuAccelerator, InstancedAccelerator, Renderer, scenes
from gonzales_b200 import _ffi as F
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu


def _mean_se(rgb, sq, n):
    mean = rgb / n
    var = np.maximum(sq / n - mean * mean, 0.0)
    return mean, np.sqrt(var / n)


def _agree(g, o, spp):
    gm, gse = _mean_se(g[0], g[1], spp)
    om, ose = _mean_se(o[0], o[1], spp)
    tol = 3.0 * np.sqrt(gse ** 2 + ose ** 2) + 1e-4
    within = float((np.abs(gm - om) <= tol).mean())
    close = float(np.isclose(gm, om, rtol=1e-3, atol=1e-5).mean())
    gi = g[0].sum(axis=(0, 1)) / g[2].sum()
    oi = o[0].sum(axis=(0, 1)) / o[2].sum()
    return within, close, gi, oi


@pytest.fixture(scope="module")
def mat_box():
    hs = scenes.materials_box_scene().build()
    assert hs.has_extended_materials
    return hs


@pytest.fixture(scope="module")
def sky():
    return scenes.sky_map(256, 128)


@pytest.mark.parametrize("mis", [0, 1])
def test_material_box_matches_oracle(mat_box, mis):
    p = dict(width=64, height=64, spp=32, max_depth=6, rr_min_bounce=3, mis_corrected=mis)
    with GpuAccelerator(mat_box) as acc:
        g = acc.render(F.render_params(**p))
        assert acc.error_word() == 0
    o = O.render(mat_box, O.render_params(**p))
    within, close, gi, oi = _agree(g, o, p["spp"])
    assert within >= 0.99, within
    assert close > 0.5, close
    np.testing.assert_allclose(gi, oi, rtol=1.5e-2)
    np.testing.assert_allclose(g[2], o[2], rtol=1e-4)
    assert g[3]["camera_rays"] == o[3]["camera"]
    assert np.isfinite(g[0]).all()


def test_material_box_with_environment_matches_oracle(mat_box, sky):
    p = dict(width=64, height=64, spp=32, max_depth=6, rr_min_bounce=3)
    with GpuAccelerator(mat_box) as acc:
        acc.set_environment(sky, 1.0)
        g = acc.render(F.render_params(**p))
    o = O.render(mat_box, O.render_params(**p), env=O.Environment(sky, 1.0))
    within, close, gi, oi = _agree(g, o, p["spp"])
    assert within >= 0.99, within
    np.testing.assert_allclose(gi, oi, rtol=1.5e-2)


def test_mixed_instanced_scene_matches_oracle(sky):
    blas_hosts, inst = scenes.instanced_scene(n_meshes=10, n_u=30, n_v=20, n_instances=128, extent=5.0, mixed=True)
    assert any(b.has_extended_materials for b in blas_hosts)
    p = dict(width=64, height=48, spp=32, max_depth=5, rr_min_bounce=2, eye=(0.0, 2.0, 16.0),
             target=(0.0, 0.0, 0.0))
    blas = [GpuAccelerator(h) for h in blas_hosts]
    with InstancedAccelerator(blas, inst) as acc:
        acc.set_environment(sky, 1.0)
        g = acc.render(F.render_params(**p))
        tlas, leaf = acc.tlas_nodes, acc.leaf_instance
        assert acc.error_word() == 0
    for b in blas:
        b.close()
    o = O.render(None, O.render_params(**p), env=O.Environment(sky, 1.0),
                 instances=dict(tlas_nodes=tlas, leaf_instance=leaf, instances=inst, blas=blas_hosts))
    within, close, gi, oi = _agree(g, o, p["spp"])
    assert within >= 0.99, within
    np.testing.assert_allclose(gi, oi, rtol=1.5e-2)
    assert g[3]["camera_rays"] == o[3]["camera"]


def test_batch_with_materials_equals_solo_renders(mat_box):
    import torch

    hs2 = scenes.box_scene().build()
    specs = [(mat_box, dict(width=48, height=40, spp=8, max_depth=5, rr_min_bounce=3)),
             (hs2, dict(width=32, height=32, spp=4, max_depth=4, rr_min_bounce=2, mis_corrected=1))]
    accs = [GpuAccelerator(h) for h, _ in specs]
    params = [F.render_params(**p) for _, p in specs]
    solo = [a.render(p) for a, p in zip(accs, params)]
    for sort_key in (F.SORT_NONE, F.SORT_MATERIAL):
        with BatchRenderer(accs, params, sort_key=sort_key) as r:
            rgb = torch.zeros((r.pixels, 3), device="cuda")
            sq = torch.zeros((r.pixels, 3), device="cuda")
            w = torch.zeros((r.pixels,), device="cuda")
            r.render(rgb, w, sq)
            torch.cuda.synchronize()
            parts = list(zip(r.split(rgb.cpu().numpy()), r.split(sq.cpu().numpy()), r.split(w.cpu().numpy())))
            assert r.error_word() == 0
        for (b_rgb, b_sq, b_w), (s_rgb, s_sq, s_w, _) in zip(parts, solo):
            np.testing.assert_allclose(b_rgb, s_rgb, rtol=1e-5, atol=1e-6)
            np.testing.assert_allclose(b_sq, s_sq, rtol=1e-5, atol=1e-6)
            np.testing.assert_allclose(b_w, s_w, rtol=1e-6)
    for a in accs:
        a.close()


def test_material_albedo_aov_matches_oracle(mat_box):
    import torch

    W, H, SPP = 48, 40, 4
    p = dict(max_depth=4, rr_min_bounce=2)
    rgb = torch.zeros((H, W, 3), device="cuda")
    w = torch.zeros((H, W), device="cuda")
    alb = torch.zeros((H, W, 3), device="cuda")
    nrm = torch.zeros((H, W, 3), device="cuda")
    with GpuAccelerator(mat_box) as acc, Renderer(acc, F.render_params(W, H, SPP, **p)) as r:
        r.render(rgb, w, film_albedo=alb, film_normal=nrm)
        torch.cuda.synchronize()
    o = O.render(mat_box, O.render_params(W, H, SPP, **p), aovs=True)
    np.testing.assert_allclose(alb.cpu().numpy(), o[4], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(nrm.cpu().numpy(), o[5], rtol=1e-5, atol=1e-5)
    # a dielectric's albedo is white: the pixels whose samples all hit one
    # average to (1, 1, 1) (the AOV films sum one value per sample)
    a = alb.cpu().numpy() / SPP
    white = np.all(np.abs(a - 1.0) < 1e-4, axis=-1)
    assert white.any()


def test_material_params_are_validated(mat_box):
    from gonzales_b200 import GzgError

    with GpuAccelerator(mat_box) as acc:
        with pytest.raises(GzgError):  # once per scene
            acc.set_material_params(mat_box.material_params)
    bad = scenes.materials_box_scene().build()
    bad.material_params = bad.material_params.copy()
    bad.material_params[1, 0] = -1.0  # eta of a coated material
    with pytest.raises(GzgError):
        GpuAccelerator(bad)


def test_material_render_is_repeatable(mat_box):
    # every material kind in one scene: lanes of one warp append to the
    # queues of different kinds at once; a repeat differs only by the order of
    # the film's atomic additions
    p = dict(width=48, height=48, spp=16, max_depth=5, rr_min_bounce=3)
    with GpuAccelerator(mat_box) as acc:
        a = acc.render(F.render_params(**p))
        b = acc.render(F.render_params(**p))
    np.testing.assert_allclose(a[0], b[0], rtol=1e-5, atol=1e-6)
    assert a[3] == b[3]
