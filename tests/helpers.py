"""Shared test helpers: scene construction and the parity classifier.

Parity rule (per ray, GPU vs oracle closest hit):
  exact            same prim, t/u/v bit-identical (or both miss)
  tie              different prim, same t bits, GPU prim is a valid MT hit at that t
                   (equal-t triangles resolved in a different visit order)
  reference-culled GPU t < oracle t (or oracle missed) and the GPU's triangle is
                   a valid MT hit with exactly the GPU's t/u/v: the reference's
                   non-conservative slab test (kernel.mojo:204) culled a node
  fail             anything else (in particular the GPU missing a hit or
                   returning a farther one)
"""
import json
import os
from pathlib import Path

import numpy as np

from gonzales_b200 import scenes
from oracle import pyoracle as O


def mesh_list(hs):
    return [(m.points, m.vertex_indices) for m in hs.meshes]


def prim_triangle(hs, k):
    p = hs.prims[k]
    if p["type"] == 0:
        mesh, base = int(p["id1"]), int(p["id2"])
    else:
        mesh, base = int(p["id2"]) >> 32, (int(p["id2"]) & 0xFFFFFFFF) * 3
    m = hs.meshes[mesh]
    idx = m.vertex_indices[base:base + 3]
    return [m.points[i, :3] for i in idx]


def oracle_closest(hs, o, d, t, watertight=False):
    r6 = scenes.pack_reference_rays(o, d)
    return O.traverse(hs.nodes, hs.prims, mesh_list(hs), r6, t, watertight=watertight)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def classify(hs, o, d, tmax, gpu_prim, gpu_t, gpu_u, gpu_v, ora_idx, ora_t, ora_u, ora_v, watertight=False):
    """Returns dict of counts and the indices of failures."""
    gpu_prim = np.asarray(gpu_prim, np.int64)
    ora_idx = np.asarray(ora_idx, np.int64)
    same = (gpu_prim == ora_idx)
    both_hit = same & (ora_idx >= 0)
    exact = (same & (ora_idx < 0)) | (both_hit & (bits(gpu_t) == bits(ora_t)) & (bits(gpu_u) == bits(ora_u))
                                      & (bits(gpu_v) == bits(ora_v)))
    counts = {"rays": len(gpu_prim), "exact": int(exact.sum()), "tie": 0, "reference_culled": 0, "fail": 0}
    fails = []
    for i in np.nonzero(~exact)[0]:
        g = int(gpu_prim[i])
        if g < 0:
            fails.append(i)
            continue
        p0, p1, p2 = prim_triangle(hs, g)
        if watertight:
            ok, t, b0, b1, b2 = O.watertight(o[i], d[i], p0, p1, p2, float(tmax[i]))
            u, v = b1, b2
        else:
            ok, t, u, v = O.mt(o[i], d[i], p0, p1, p2, float(tmax[i]))
        valid = ok and bits(t) == bits(gpu_t[i]) and bits(u) == bits(gpu_u[i]) and bits(v) == bits(gpu_v[i])
        if not valid:
            fails.append(i)
        elif ora_idx[i] >= 0 and bits(gpu_t[i]) == bits(ora_t[i]):
            counts["tie"] += 1
        elif ora_idx[i] < 0 or gpu_t[i] < ora_t[i]:
            counts["reference_culled"] += 1
        else:
            fails.append(i)
    counts["fail"] = len(fails)
    return counts, fails


def small_raycast(subdiv=4, n_side=48, n_incoherent=4096, seed=0xC1):
    sb = scenes.raycast_scene(subdiv=subdiv, seed=seed)
    hs = sb.build()
    o, d, t = scenes.raycast_rays(hs, n_side, n_side, n_incoherent, seed=seed)
    return hs, o, d, t


def record(name, data):
    """Writes a measurement record (JSON) into $GZG_RECORD_DIR when it is set."""
    d = os.environ.get("GZG_RECORD_DIR")
    if d and Path(d).is_dir():
        (Path(d) / name).write_text(json.dumps(data, default=lambda o: o.item() if hasattr(o, "item") else str(o)))


# ---------------------------------------------------------------- the reference's regression scene

GOLDEN_DIR = Path(__file__).resolve().parent / "golden"


def regression_fixture():
    """The arrays of tests/golden/regression_test.npz (made by
    tests/golden/make_regression_golden.py from the reference's
    Tests/reference/regression-test.pbrt and regression-test.exr)."""
    return np.load(GOLDEN_DIR / "regression_test.npz")


def regression_scene(z=None):
    """The regression scene as the reference's SceneDescription assembles it:
    every shape a mesh of GeometricPrimitives with its named diffuse material,
    the shape inside AreaLightSource an area light (radiance L); no mesh has
    more than 16 triangles, so all sit in the top-level BVH
    (Api/SceneDescription.swift:761-763).  Returns (SceneBuilder, render
    keyword arguments for gonzales_b200._ffi.render_params / the oracle's)."""
    from gonzales_b200.scene import SceneBuilder

    z = regression_fixture() if z is None else z
    sb = SceneBuilder()
    k = 0
    while "mesh%d_P" % k in z.files:
        pts, idx = z["mesh%d_P" % k], z["mesh%d_indices" % k]
        L = z["mesh%d_L" % k]
        if np.any(L > 0):
            sb.add_area_light(pts, idx, tuple(float(x) for x in L))
        else:
            mat = sb.add_material(tuple(float(x) for x in z["mesh%d_reflectance" % k]))
            sb.add_mesh(pts, idx, mat, normals=z["mesh%d_N" % k], uvs=z["mesh%d_uv" % k])
        k += 1
    # The PBRT Transform is camera-from-world, given column by column
    # (m[col*4 + row]); the camera sits at world_from_camera * (0, 0, 0) and
    # looks along world_from_camera * (0, 0, 1), with +y up.
    m = z["camera_transform"].reshape(4, 4).T
    inv = np.linalg.inv(m)
    eye = inv[:3, 3]
    fwd = inv[:3, :3] @ np.array([0.0, 0.0, 1.0])
    up = inv[:3, :3] @ np.array([0.0, 1.0, 0.0])
    W, H = (int(v) for v in z["resolution"])
    kw = dict(width=W, height=H, spp=int(z["spp"]), max_depth=int(z["max_depth"]),
              eye=tuple(eye), target=tuple(eye + fwd), up=tuple(up), fov_deg=float(z["fov"]),
              filter_radius=float(z["filter_radius"][0]), filter_sigma=float(z["filter_sigma"]))
    return sb, kw


def oracle_tile_loop(hs, params, seed=0):
    """The reference's live bounce loop (Core/Tile.swift:19-223) on the oracle:
    oracle camera rays, oracle traversal and the oracle's shade_core, with
    PCG seeds from a seeded generator.  Returns film sums (light, weight)."""
    from gonzales_b200 import _ffi as F
    from gonzales_b200.tile import normalized  # noqa: F401  (same normalisation)

    W, H, spp = params.width, params.height, params.spp
    n = W * H * spp
    rays, w, pixel = O.camera_rays(params, 0, n)
    paths = np.zeros(n, F.PATH_STATE_DTYPE)
    paths["ray"] = rays.view(F.RAY_DTYPE).reshape(-1)
    paths["throughput"] = 1.0
    rng = np.random.Generator(np.random.PCG64(seed))
    live = np.arange(n)
    for _ in range(params.max_depth + 1):
        if len(live) == 0:
            break
        state = paths[live]
        r6 = np.ascontiguousarray(state["ray"]).view(np.float32).reshape(-1, 6)
        isect, _, _ = O.traverse(hs.nodes, hs.prims, mesh_list(hs), r6, np.full(len(live), np.inf, np.float32))
        state["pcg_state"] = rng.integers(0, 2 ** 64, len(live), dtype=np.uint64, endpoint=False)
        state["pcg_inc"] = rng.integers(0, 2 ** 64, len(live), dtype=np.uint64, endpoint=False)
        state["active"] = 1
        state = O.shade_batch(hs, state, isect)
        paths[live] = state
        live = live[state["active"] != 0]
    light = np.zeros((H * W, 3))
    weight = np.zeros(H * W)
    np.add.at(light, pixel, paths["estimate"].astype(np.float64))
    np.add.at(weight, pixel, w.astype(np.float64))
    return light.reshape(H, W, 3), weight.reshape(H, W)


def normalised_rmse(img, golden):
    """The reference test's metric (`magick compare -metric RMSE`, normalised
    value, RenderRegressionTests.swift:40-62) on linear float RGB: the root
    mean square of the per-channel differences over all pixels (1.0 = white).
    The alpha channel, equal to 1 in both images, is left out."""
    d = np.asarray(img, np.float64)[..., :3] - np.asarray(golden, np.float64)[..., :3]
    return float(np.sqrt(np.mean(d * d)))
