"""CPU checks of the oracle's environment light (the checker of the device
environment light): the equal-area mapping round-trips, a sample's pdf equals
the light's pdf for the sampled direction, importance-sampled and uniform
estimates of the map's integral agree, and a two-level scene lit only by the
environment renders."""
import numpy as np

from gonzales_b200 import scenes
from gonzales_b200.accel import instance_bounds
from gonzales_b200.scene import build_bvh2
from oracle import pyoracle as O


def test_equal_area_mapping_round_trips():
    import ctypes as C

    L = O.lib()
    L.orc_equal_area_square_to_sphere.argtypes = [C.c_float, C.c_float, C.c_void_p]
    L.orc_equal_area_sphere_to_square.argtypes = [C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(3)
    for u, v in rng.random((500, 2)):
        d = np.zeros(3, np.float32)
        uv = np.zeros(2, np.float32)
        L.orc_equal_area_square_to_sphere(u, v, d.ctypes.data)
        # the reference's square-to-sphere omits the sqrt(2 - r^2) factor of
        # x and y, so its directions are shorter than 1 off the poles and the
        # equator; the inverse map only sees direction ratios and |z|
        r = 1 - abs(1 - (abs(2 * u - 1) + abs(2 * v - 1)))
        assert abs(np.linalg.norm(d) - np.sqrt(r * r + (1 - r * r) ** 2)) < 1e-5
        L.orc_equal_area_sphere_to_square(d.ctypes.data, uv.ctypes.data)
        assert np.allclose(uv, [u, v], atol=2e-5)
    # the numpy map builder uses the same mapping
    d = np.zeros(3, np.float32)
    L.orc_equal_area_square_to_sphere(0.3, 0.8, d.ctypes.data)
    assert np.allclose(scenes.equal_area_square_to_sphere(np.array(0.3), np.array(0.8)), d, atol=1e-6)


def test_environment_sample_pdf_and_integral():
    env = O.Environment(scenes.sky_map(256, 128), 1.0)
    rng = np.random.default_rng(0)
    n = 20000
    est = np.zeros(3)
    rel = []
    for u0, u1 in rng.random((n, 2)):
        d, c, pdf = env.sample(u0, u1)
        assert pdf > 0
        rel.append(abs(env.pdf(d) - pdf) / pdf)
        est += c / pdf
    est /= n
    # pdf0 * pdf1 against f / marginal integral: equal up to rounding, except
    # where the round trip through the mapping lands in a neighbouring cell
    rel = np.array(rel)
    assert np.mean(rel <= 1e-5) > 0.99 and rel.max() < 0.1
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    uni = np.mean([env.radiance(x.astype(np.float32)) for x in dirs], axis=0) * 4 * np.pi
    np.testing.assert_allclose(est, uni, rtol=0.03)
    t = env.tables()
    assert t["cdf"][:, -1].min() == 1.0 and t["marginal_cdf"][-1] == 1.0
    assert abs(env.power() - np.pi * 50.0 ** 2) < 1e-2


def test_instanced_environment_render_is_lit():
    blas, inst = scenes.instanced_scene(n_meshes=2, n_u=12, n_v=10, n_instances=40, extent=4.0, coloured=True)
    tlas, leaf = build_bvh2(instance_bounds(blas, inst))
    env = O.Environment(scenes.sky_map(64, 32), 1.0)
    p = O.render_params(24, 16, 4, max_depth=3, rr_min_bounce=3, eye=(0.0, 0.0, 14.0), target=(0.0, 0.0, 0.0))
    s, _, w, cnt = O.render(None, p, threads=4, env=env,
                            instances=dict(tlas_nodes=tlas, leaf_instance=leaf, instances=inst, blas=blas))
    img = s / w[..., None]
    assert np.isfinite(img).all() and img.mean() > 0.05
    assert cnt["shadow"] > 0 and cnt["probe"] > 0  # environment light: the BSDF strategy is traced
