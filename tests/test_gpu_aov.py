"""First-hit AOVs (albedo, normal: Tile.swift:157-205) and Film.add settings
(iso scaling, largest-component clamp: Film.swift:107-119) of the device
renderer against the oracle at equal Z-Sobol indices.  The AOVs come from the
camera ray's closest hit, which both sides find identically, so they agree to
rounding; the clamped beauty image agrees within Monte Carlo error."""
import numpy as np
import pytest

from gonzales_b200 import GpuAccelerator, Renderer, scenes
from gonzales_b200 import _ffi as F
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu
W, H, SPP = 48, 40, 8


def torch_mod():
    import torch

    return torch


def _device_render(acc, p, iso=100.0, max_component=0.0):
    torch = torch_mod()
    rgb = torch.zeros((H, W, 3), device="cuda")
    sq = torch.zeros((H, W, 3), device="cuda")
    w = torch.zeros((H, W), device="cuda")
    alb = torch.zeros((H, W, 3), device="cuda")
    nrm = torch.zeros((H, W, 3), device="cuda")
    with Renderer(acc, p) as r:
        r.set_film(iso, max_component)
        r.render(rgb, w, sq, film_albedo=alb, film_normal=nrm)
        torch.cuda.synchronize()
    return [t.cpu().numpy() for t in (rgb, sq, w, alb, nrm)]


@pytest.fixture(scope="module")
def box():
    hs = scenes.box_scene().build()
    acc = GpuAccelerator(hs)
    yield hs, acc
    acc.close()


def test_aovs_match_oracle(box):
    hs, acc = box
    p = dict(max_depth=4, rr_min_bounce=2)
    rgb, sq, w, alb, nrm = _device_render(acc, F.render_params(W, H, SPP, **p))
    o = O.render(hs, O.render_params(W, H, SPP, **p), aovs=True)
    np.testing.assert_allclose(w, o[2], rtol=1e-4)
    np.testing.assert_allclose(alb, o[4], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(nrm, o[5], rtol=1e-5, atol=1e-5)
    assert alb.max() > 0 and np.abs(nrm).max() > 0


def test_iso_scales_exactly_and_clamp_matches_oracle(box):
    hs, acc = box
    p = dict(max_depth=4, rr_min_bounce=2)
    base = _device_render(acc, F.render_params(W, H, SPP, **p))
    twice = _device_render(acc, F.render_params(W, H, SPP, **p), iso=200.0)
    np.testing.assert_allclose(twice[0], 2 * base[0], rtol=1e-6, atol=1e-6)
    g = _device_render(acc, F.render_params(W, H, SPP, **p), max_component=0.5)
    o = O.render(hs, O.render_params(W, H, SPP, max_component=0.5, **p))
    assert (g[0] <= 0.5 * SPP + 1e-4).all()
    gm, om = g[0] / SPP, o[0] / SPP
    gse = np.sqrt(np.maximum(g[1] / SPP - gm * gm, 0) / SPP)
    ose = np.sqrt(np.maximum(o[1] / SPP - om * om, 0) / SPP)
    within = (np.abs(gm - om) <= 3 * np.sqrt(gse ** 2 + ose ** 2) + 1e-4).mean()
    assert within >= 0.995, within
    np.testing.assert_allclose(g[0].sum(), o[0].sum(), rtol=1e-2)


def test_film_resolve_and_exr_output(box, tmp_path):
    """Film.writeImages: beauty, albedo and normal normalised by the film
    weights on the device, written as RGBA float EXR files."""
    from gonzales_b200 import film

    torch = torch_mod()
    hs, acc = box
    p = dict(max_depth=4, rr_min_bounce=2)
    rgb = torch.zeros((H, W, 3), device="cuda")
    w = torch.zeros((H, W), device="cuda")
    alb = torch.zeros((H, W, 3), device="cuda")
    nrm = torch.zeros((H, W, 3), device="cuda")
    with Renderer(acc, F.render_params(W, H, SPP, **p)) as r:
        r.render(rgb, w, film_albedo=alb, film_normal=nrm)
    torch.cuda.synchronize()
    wn = w.cpu().numpy()
    for name, sums in (("beauty", rgb), ("albedo", alb), ("normal", nrm)):
        img, zero = film.resolve(sums, w)
        assert zero == 0
        s = sums.cpu().numpy()
        black = np.all(s == 0, axis=-1, keepdims=True)
        expect = np.where(black, 0.0, s / np.where(wn == 0, 1, wn)[..., None])
        np.testing.assert_allclose(img.cpu().numpy(), expect, rtol=1e-6, atol=0)
        path = tmp_path / (name + ".exr")
        film.write_exr(path, img.cpu().numpy())
        back, _ = film.read_exr(path)
        assert np.array_equal(back[..., :3], img.cpu().numpy())
    # non-black light with zero weight is counted (the reference throws)
    rgb2 = torch.ones((2, 3), device="cuda")
    w2 = torch.tensor([1.0, 0.0], device="cuda")
    img, zero = film.resolve(rgb2, w2)
    assert zero == 1 and float(img[1].abs().sum()) == 0.0


def test_thin_lens_camera_matches_oracle():
    """PerspectiveCamera.depthOfField: camera rays leave from a point of the
    lens disk (concentric mapping of the lens sample); as written the
    direction keeps the pinhole direction.  GPU and oracle agree per pixel."""
    hs = scenes.box_scene().build()
    p = dict(max_depth=4, rr_min_bounce=2, lens_radius=0.05, focal_distance=1.5)
    with GpuAccelerator(hs) as acc:
        g = acc.render(F.render_params(W, H, SPP, **p))
        g0 = acc.render(F.render_params(W, H, SPP, max_depth=4, rr_min_bounce=2))
    o = O.render(hs, O.render_params(W, H, SPP, **p))
    gm, om = g[0] / SPP, o[0] / SPP
    assert np.isclose(gm, om, rtol=1e-3, atol=1e-5).mean() > 0.9
    np.testing.assert_allclose(g[0].sum((0, 1)) / g[2].sum(), o[0].sum((0, 1)) / o[2].sum(), rtol=1e-2)
    # the lens moves the rays: the image differs from the pinhole one
    assert not np.allclose(g[0], g0[0], rtol=1e-3)


def test_film_resolve_reference_pixel_cases():
    """Tests/libgonzalesTests/PixelTests.swift: light / weight; black with
    weight 0 stays black; non-black with weight 0 is the reference's error
    (counted here)."""
    from gonzales_b200 import film

    torch = torch_mod()
    rgb = torch.tensor([[4.0, 6.0, 8.0], [0.0, 0.0, 0.0], [1.0, 1.0, 1.0]], device="cuda")
    w = torch.tensor([2.0, 0.0, 0.0], device="cuda")
    img, zero = film.resolve(rgb, w)
    np.testing.assert_allclose(img.cpu().numpy(), [[2.0, 3.0, 4.0], [0, 0, 0], [0, 0, 0]], atol=1e-6)
    assert zero == 1
