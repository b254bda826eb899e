"""Batched wavefront renderer: many scenes in one renderer.

Every path of a batch computes exactly what it computes when its scene is
rendered alone (same tree under a root offset, same prims, materials and
lights under index offsets, same Z-Sobol indices), so a batch film window
must equal the scene's own render up to the order of the film atomics; the
same holds for every sort key, graph replay and wave size.  The single-scene
renderer is itself checked against the oracle's integrator (test_gpu_render).
"""
import numpy as np
import pytest

from gonzales_b200 import BatchRenderer, GpuAccelerator, GzgError, scenes
from gonzales_b200 import _ffi as F

pytestmark = pytest.mark.gpu


def torch_mod():
    import torch

    return torch


@pytest.fixture(scope="module")
def batch():
    specs = [
        (scenes.box_scene(), dict(width=48, height=40, spp=8, max_depth=5, rr_min_bounce=3)),
        (scenes.batch_scene(11, 3_000), dict(width=32, height=32, spp=4, max_depth=6, rr_min_bounce=2)),
        (scenes.batch_scene(12, 20_000), dict(width=40, height=24, spp=8, max_depth=3, rr_min_bounce=2)),
        (scenes.batch_scene(13, 1_500), dict(width=16, height=16, spp=16, max_depth=4, rr_min_bounce=2,
                                             mis_corrected=1, seed=99)),
    ]
    accs = [GpuAccelerator(sb.build()) for sb, _ in specs]
    params = [F.render_params(**p) for _, p in specs]
    solo = [a.render(p) for a, p in zip(accs, params)]
    yield accs, params, solo
    for a in accs:
        a.close()


def _render_batch(accs, params, **kw):
    torch = torch_mod()
    with BatchRenderer(accs, params, **kw) as r:
        rgb = torch.zeros((r.pixels, 3), device="cuda")
        sq = torch.zeros((r.pixels, 3), device="cuda")
        w = torch.zeros((r.pixels,), device="cuda")
        r.render(rgb, w, sq)
        torch.cuda.synchronize()
        parts = list(zip(r.split(rgb.cpu().numpy()), r.split(sq.cpu().numpy()), r.split(w.cpu().numpy())))
        return parts, r.stats(), r.error_word()


def _assert_same(parts, solo):
    for (rgb, sq, w), (s_rgb, s_sq, s_w, _) in zip(parts, solo):
        np.testing.assert_allclose(rgb, s_rgb, rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(sq, s_sq, rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(w, s_w, rtol=1e-6)


@pytest.mark.parametrize("sort_key", [F.SORT_NONE, F.SORT_MATERIAL, F.SORT_SCENE])
@pytest.mark.parametrize("use_graph", [0, 1])
def test_batch_windows_equal_solo_renders(batch, sort_key, use_graph):
    accs, params, solo = batch
    parts, stats, err = _render_batch(accs, params, use_graph=use_graph, sort_key=sort_key)
    assert err == 0
    _assert_same(parts, solo)
    assert stats["camera_rays"] == sum(p.width * p.height * p.spp for p in params)
    assert stats["extension_rays"] == sum(s[3]["extension_rays"] for s in solo)
    assert stats["shadow_rays"] == sum(s[3]["shadow_rays"] for s in solo)
    assert stats["probe_rays"] == sum(s[3]["probe_rays"] for s in solo)


@pytest.mark.parametrize("wave_paths", [1000, 4099])
def test_batch_small_waves(batch, wave_paths):
    accs, params, solo = batch
    parts, stats, err = _render_batch(accs, params, wave_paths=wave_paths, sort_key=F.SORT_MATERIAL)
    assert err == 0
    _assert_same(parts, solo)
    total = sum(p.width * p.height * p.spp for p in params)
    assert stats["waves"] == (total + wave_paths - 1) // wave_paths


def test_batch_of_one_equals_renderer(batch):
    accs, params, solo = batch
    for a, p, s in zip(accs, params, solo):
        parts, stats, err = _render_batch([a], [p], use_graph=1)
        assert err == 0
        _assert_same(parts, [s])
        assert stats["extension_rays"] == s[3]["extension_rays"]


def test_batch_autotune_keeps_the_image(batch):
    torch = torch_mod()
    accs, params, solo = batch
    with BatchRenderer(accs, params) as r:
        best, ms = r.autotune()
        assert ms > 0
        assert best["sort_key"] in (F.SORT_NONE, F.SORT_MATERIAL, F.SORT_SCENE)
        assert best["wave_paths"] > 0
        rgb = torch.zeros((r.pixels, 3), device="cuda")
        w = torch.zeros((r.pixels,), device="cuda")
        r.render(rgb, w)
        torch.cuda.synchronize()
        st = r.stats()
        for (img, wt), (s_rgb, _, s_w, _) in zip(zip(r.split(rgb.cpu().numpy()), r.split(w.cpu().numpy())), solo):
            np.testing.assert_allclose(img, s_rgb, rtol=1e-5, atol=1e-6)
            np.testing.assert_allclose(wt, s_w, rtol=1e-6)
        # autotuning resets the statistics; one render remains
        assert st["camera_rays"] == sum(p.width * p.height * p.spp for p in params)


def test_batch_rejects_bad_arguments(batch):
    accs, params, _ = batch
    with pytest.raises(GzgError):
        BatchRenderer(accs, params, sort_key=7)
    with pytest.raises(ValueError):
        BatchRenderer(accs, params[:2])
    bad = F.render_params(width=0, height=8, spp=1)
    with pytest.raises(GzgError):
        BatchRenderer(accs[:1], [bad])


def test_batch_configuration_subset_matches_oracle():
    """Four scenes of the scene-batch configuration itself (the first of each
    image side in the seeded 64-scene workload: 64^2, 128^2, 256^2 and 512^2,
    972 to 50,398 triangles) at its parameters (32 spp, depth 6, roulette from
    bounce 2), rendered in one batch and compared per pixel with the oracle's
    renders of the same scenes at equal Z-Sobol samples."""
    from oracle import pyoracle as O
    from tests import helpers

    torch = torch_mod()
    work = scenes.batch_workload(64, 0xC3)
    picks = {}
    for k, (_, side) in enumerate(work):
        picks.setdefault(side, k)
    chosen = [picks[s] for s in sorted(picks)]
    hosts = [work[k][0].build() for k in chosen]
    accs = [GpuAccelerator(h) for h in hosts]
    kw = [dict(width=work[k][1], height=work[k][1], spp=32, max_depth=6, rr_min_bounce=2) for k in chosen]
    params = [F.render_params(**p) for p in kw]
    record = []
    try:
        with BatchRenderer(accs, params, use_graph=1) as r:
            rgb = torch.zeros((r.pixels, 3), device="cuda")
            sq = torch.zeros((r.pixels, 3), device="cuda")
            w = torch.zeros((r.pixels,), device="cuda")
            r.render(rgb, w, sq)
            torch.cuda.synchronize()
            assert r.error_word() == 0
            parts = list(zip(r.split(rgb.cpu().numpy()), r.split(sq.cpu().numpy()), r.split(w.cpu().numpy())))
        for hs, p, (g_rgb, g_sq, g_w) in zip(hosts, kw, parts):
            o_rgb, o_sq, o_w, _ = O.render(hs, O.render_params(**p))
            n = p["spp"]
            side = p["width"]
            g_rgb, g_sq, g_w = (a.reshape(o.shape) for a, o in ((g_rgb, o_rgb), (g_sq, o_sq), (g_w, o_w)))
            gm, om = g_rgb / n, o_rgb / n
            gse = np.sqrt(np.maximum(g_sq / n - gm * gm, 0.0) / n)
            ose = np.sqrt(np.maximum(o_sq / n - om * om, 0.0) / n)
            within = float((np.abs(gm - om) <= 3.0 * np.sqrt(gse ** 2 + ose ** 2) + 1e-4).mean())
            record.append({"side": side, "triangles": hs.triangle_count, "within_3se": within})
            np.testing.assert_allclose(g_w, o_w, rtol=1e-4)
            assert within >= 0.997, record[-1]
            np.testing.assert_allclose(g_rgb.sum(axis=(0, 1)) / g_w.sum(), o_rgb.sum(axis=(0, 1)) / o_w.sum(),
                                       rtol=1e-2)
    finally:
        helpers.record("batch_subset_vs_oracle.json", record)
        for a in accs:
            a.close()
