"""GPU wavefront path integrator against the oracle's restatement of Gonzales'
MIS integrator, on the box scene, at equal Z-Sobol indices.

  - device Z-Sobol values are bit-identical to the oracle's (integer path);
  - per pixel, the GPU and oracle means agree within 3 combined Monte Carlo
    standard errors (the two draw identical random numbers, so they usually
    agree far more tightly; paths can still part ways after an ulp difference
    in cos/sin/sqrt);
  - film weights, ray counts and image means agree; graph replay and small
    waves give the same image as one large wave;
  - relMSE against a high-spp oracle render is reported.
"""
from pathlib import Path

import numpy as np
import pytest

from gonzales_b200 import GpuAccelerator, Renderer, scenes
from gonzales_b200 import _ffi as F
from oracle import pyoracle as O
from tests import helpers

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def torch_mod():
    import torch

    return torch


def device_zsobol(spp, rx, ry, px, py, index, kinds, seed=1234):
    torch = torch_mod()
    px_d = torch.as_tensor(np.asarray(px, np.int32)).cuda()
    py_d = torch.as_tensor(np.asarray(py, np.int32)).cuda()
    ix_d = torch.as_tensor(np.asarray(index, np.int64)).cuda()
    kinds = np.ascontiguousarray(kinds, np.int32)
    out = torch.zeros((len(px), int(kinds.sum())), dtype=torch.float32, device="cuda")
    F.check(F.lib().gzg_zsobol_fill_device(spp, rx, ry, seed, px_d.data_ptr(), py_d.data_ptr(), ix_d.data_ptr(),
                                           len(px), F.ptr(kinds), len(kinds), out.data_ptr(), None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_device_zsobol_matches_golden_fixture():
    g = np.load(GOLDEN / "zsobol_small.npz")
    vals = device_zsobol(16, 256, 256, g["px"], g["py"], g["index"], g["kinds"])
    assert vals.tobytes() == g["values"].tobytes()


@pytest.mark.parametrize("spp,res", [(1, (64, 64)), (2, (100, 37)), (4, (256, 256)), (8, (640, 480)),
                                     (32, (1920, 1080)), (64, (33, 33))])
def test_device_zsobol_matches_oracle(spp, res):
    rng = np.random.default_rng(spp)
    n = 2048
    px = rng.integers(0, res[0], n)
    py = rng.integers(0, res[1], n)
    idx = rng.integers(0, spp, n)
    kinds = [2, 2] + [1, 2, 3, 3, 1] * 8
    ours = device_zsobol(spp, res[0], res[1], px, py, idx, kinds)
    ref = O.zsobol_batch(spp, res[0], res[1], px, py, idx, kinds)
    assert ours.tobytes() == ref.tobytes()


@pytest.fixture(scope="module")
def box():
    hs = scenes.box_scene().build()
    acc = GpuAccelerator(hs)
    yield hs, acc
    acc.close()


def _params(**kw):
    base = dict(width=64, height=64, spp=16, max_depth=5, rr_min_bounce=3)
    base.update(kw)
    return base


def _mean_se(rgb, sq, n):
    mean = rgb / n
    var = np.maximum(sq / n - mean * mean, 0.0)
    return mean, np.sqrt(var / n)


def _compare(hs, acc, **kw):
    p = _params(**kw)
    g_rgb, g_sq, g_w, gstats = acc.render(F.render_params(**p))
    o_rgb, o_sq, o_w, ocnt = O.render(hs, O.render_params(**{k: v for k, v in p.items() if k not in
                                                             ("wave_paths", "use_graph")}))
    n = p["spp"]
    gm, gse = _mean_se(g_rgb, g_sq, n)
    om, ose = _mean_se(o_rgb, o_sq, n)
    tol = 3.0 * np.sqrt(gse ** 2 + ose ** 2) + 1e-4
    within = np.abs(gm - om) <= tol
    return dict(p=p, g=(g_rgb, g_sq, g_w, gstats), o=(o_rgb, o_sq, o_w, ocnt), within=within.mean(),
                exact_frac=float(np.isclose(gm, om, rtol=1e-4, atol=1e-6).mean()))


@pytest.mark.parametrize("mis", [0, 1])
def test_render_matches_oracle_per_pixel(box, mis):
    hs, acc = box
    r = _compare(hs, acc, mis_corrected=mis)
    g_rgb, g_sq, g_w, gstats = r["g"]
    o_rgb, o_sq, o_w, ocnt = r["o"]
    assert r["within"] >= 0.997, r["within"]
    # filter weights use erff/expf (library functions on each side) and rare
    # tail samples are clamped to the filter radius: agreement to 1e-4
    np.testing.assert_allclose(g_w, o_w, rtol=1e-4)
    assert gstats["camera_rays"] == ocnt["camera"] == 64 * 64 * 16
    # the GPU skips the reference's final extension (bounce == max_depth),
    # which can only add environment light; the oracle traces it
    assert 0.5 * ocnt["extension"] <= gstats["extension_rays"] <= ocnt["extension"]
    # the GPU also skips shadow rays whose contribution is zero (light behind
    # the surface as seen from the outgoing side); the oracle traces them
    assert 0.8 * ocnt["shadow"] <= gstats["shadow_rays"] <= ocnt["shadow"]
    if mis:
        assert gstats["probe_rays"] > 0
    else:
        assert gstats["probe_rays"] == 0
    gi = g_rgb.sum(axis=(0, 1)) / g_w.sum()
    oi = o_rgb.sum(axis=(0, 1)) / o_w.sum()
    np.testing.assert_allclose(gi, oi, rtol=5e-3)
    assert r["exact_frac"] > 0.9, r["exact_frac"]


def test_graph_replay_and_small_waves_match_one_wave(box):
    hs, acc = box
    base = dict(width=48, height=40, spp=8, max_depth=5, rr_min_bounce=3)
    a = acc.render(F.render_params(**base))
    b = acc.render(F.render_params(**base, wave_paths=1000, use_graph=1))
    c = acc.render(F.render_params(**base, wave_paths=777))
    for other in (b, c):
        np.testing.assert_allclose(other[0], a[0], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(other[2], a[2], rtol=1e-6)
    assert b[3]["waves"] == (48 * 40 * 8 + 999) // 1000


def test_renderer_device_films_accumulate(box):
    torch = torch_mod()
    hs, acc = box
    p = F.render_params(width=32, height=32, spp=4, max_depth=4, use_graph=1)
    rgb = torch.zeros((32, 32, 3), device="cuda")
    w = torch.zeros((32, 32), device="cuda")
    with Renderer(acc, p) as r:
        r.render(rgb, w)
        r.render(rgb, w)
        torch.cuda.synchronize()
        st = r.stats()
    once = acc.render(p)
    np.testing.assert_allclose(rgb.cpu().numpy(), 2 * once[0], rtol=1e-5, atol=1e-6)
    assert st["camera_rays"] == 2 * 32 * 32 * 4


def relmse(img, ref, eps=1e-2):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + eps)))


def test_relmse_against_high_spp_oracle(box):
    hs, acc = box
    W = H = 32
    ref_rgb, _, ref_w, _ = O.render(hs, O.render_params(W, H, 4096, max_depth=5, rr_min_bounce=3))
    ref = ref_rgb / ref_w[..., None]
    result = {}
    for spp in (16, 256, 1024):
        g = acc.render(F.render_params(W, H, spp, max_depth=5, rr_min_bounce=3))
        result[spp] = relmse(g[0] / g[2][..., None], ref)
    o16 = O.render(hs, O.render_params(W, H, 16, max_depth=5, rr_min_bounce=3))
    result["oracle16"] = relmse(o16[0] / o16[2][..., None], ref)
    helpers.record("relmse_box.json", {str(k): v for k, v in result.items()})
    assert result[1024] < result[256] < result[16]
    assert abs(result[16] - result["oracle16"]) <= 0.25 * result["oracle16"]
    assert result[1024] < 1e-2


def test_box_configuration_full_size_matches_oracle_and_meets_relmse_bar(box):
    """The box-scene configuration at its stated size (256 x 256, 16 spp,
    depth 5, roulette from bounce 3): per pixel against the oracle at equal
    Z-Sobol samples, then relMSE against a 4096-spp render.  The 4096-spp
    reference is a GPU render with another Z-Sobol seed: at equal samples the
    GPU render equals the oracle's (checked here at 16 spp over the full
    frame, and at 4096 spp on a 32 x 32 frame against the oracle's own 4096-spp
    render).  relMSE must reach 1e-3 by 1024 spp."""
    hs, acc = box
    r = _compare(hs, acc, width=256, height=256, spp=16, max_depth=5, rr_min_bounce=3)
    assert r["within"] >= 0.997, r["within"]
    assert r["exact_frac"] > 0.9, r["exact_frac"]
    g_rgb, _, g_w, _ = r["g"]
    o_rgb, _, o_w, _ = r["o"]
    np.testing.assert_allclose(g_w, o_w, rtol=1e-4)
    np.testing.assert_allclose(g_rgb.sum(axis=(0, 1)) / g_w.sum(), o_rgb.sum(axis=(0, 1)) / o_w.sum(), rtol=2e-3)
    # the GPU's 4096-spp image against the oracle's at equal samples (32 x 32)
    o4k = O.render(hs, O.render_params(32, 32, 4096, max_depth=5, rr_min_bounce=3))
    g4k = acc.render(F.render_params(32, 32, 4096, max_depth=5, rr_min_bounce=3))
    same = relmse(g4k[0] / g4k[2][..., None], o4k[0] / o4k[2][..., None])
    assert same < 1e-5, same
    # relMSE against the 4096-spp reference at the full size
    ref_rgb, _, ref_w, _ = acc.render(F.render_params(256, 256, 4096, max_depth=5, rr_min_bounce=3, seed=4321))
    ref = ref_rgb / ref_w[..., None]
    curve = {"16_oracle": relmse(o_rgb / o_w[..., None], ref)}
    for spp in (16, 64, 256, 1024):
        g = acc.render(F.render_params(256, 256, spp, max_depth=5, rr_min_bounce=3))
        curve[str(spp)] = relmse(g[0] / g[2][..., None], ref)
    curve["gpu_vs_oracle_4096_32x32"] = same
    helpers.record("relmse_box_full.json", curve)
    assert abs(curve["16"] - curve["16_oracle"]) <= 0.05 * curve["16_oracle"], curve
    assert curve["1024"] < curve["256"] < curve["64"] < curve["16"], curve
    assert curve["1024"] <= 1e-3, curve
