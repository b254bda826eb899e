"""gzg_gpu_shade_batch (drop-in for mojo_gpu_shade_batch) against the oracle's
restatement of shade_core (kernel.mojo:676-773) on identical path states and
intersections.  PCG32 state, activity, estimate and throughput are integer or
single-rounding arithmetic and must be bit-identical; the bounce direction goes
through cosf/sinf (library functions on each side) and agrees to a few ulps.
"""
import numpy as np
import pytest

from gonzales_b200 import GpuAccelerator, options, scenes
from gonzales_b200 import _ffi as F
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu


def camera_paths(n, seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(n, F.PATH_STATE_DTYPE)
    o = np.tile(np.array([0.5, 0.5, 2.2], np.float32), (n, 1))
    tgt = np.stack([rng.uniform(0.0, 1.0, n), rng.uniform(0.0, 1.0, n), np.zeros(n)], 1)
    d = tgt - o
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    p["ray"]["org"] = o
    p["ray"]["dir"] = d
    p["throughput"] = 1.0
    p["pcg_state"] = rng.integers(0, 2 ** 63, n, dtype=np.uint64)
    p["pcg_inc"] = rng.integers(0, 2 ** 63, n, dtype=np.uint64)
    p["active"] = 1
    return p


def rays_of(paths):
    r = np.zeros((len(paths), 6), np.float32)
    r[:, :3] = paths["ray"]["org"]
    r[:, 3:] = paths["ray"]["dir"]
    return r


def test_shade_batch_matches_shade_core():
    hs = scenes.box_scene().build()
    n = 50000
    paths = camera_paths(n, 3)
    with GpuAccelerator(hs) as acc:
        for bounce in range(3):
            tmax = np.full(n, np.inf, np.float32)
            isects = acc.intersect_batch(rays_of(paths), tmax, options(traversal=F.TRAVERSAL_BVH2))
            ora = O.shade_batch(hs, paths.view(O.PATH_DTYPE), isects)
            gpu = acc.shade_batch(paths.copy(), isects)
            ov = ora.view(F.PATH_STATE_DTYPE)
            assert np.array_equal(gpu["active"], ov["active"])
            assert np.array_equal(gpu["pcg_state"], ov["pcg_state"])
            assert np.array_equal(gpu["pcg_inc"], ov["pcg_inc"])
            assert gpu["estimate"].tobytes() == ov["estimate"].tobytes()
            assert gpu["throughput"].tobytes() == ov["throughput"].tobytes()
            np.testing.assert_allclose(gpu["ray"]["org"], ov["ray"]["org"], atol=2e-6)
            np.testing.assert_allclose(gpu["ray"]["dir"], ov["ray"]["dir"], atol=4e-6)
            assert acc.error_word() == 0
            paths = ov.copy()  # continue both from the oracle's state
        assert (paths["active"] == 0).mean() > 0.1
        assert paths["estimate"].max() > 0  # some paths reached the light


def test_shade_batch_reports_bad_material_index():
    hs = scenes.box_scene().build()
    paths = camera_paths(64, 4)
    with GpuAccelerator(hs) as acc:
        isects = acc.intersect_batch(rays_of(paths), np.full(64, np.inf, np.float32))
        hit = np.nonzero(isects["hit"])[0]
        isects["prim_id"]["material_index"][hit[0]] = 1000
        with pytest.raises(F.GzgError) as e:
            acc.shade_batch(paths, isects)
        assert e.value.status == 6
