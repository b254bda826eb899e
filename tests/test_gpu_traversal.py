"""GPU parity of the libgzg traversal kernels against the oracle (the CPU
restatement of kernel.mojo's traverse_bvh2_core) on identical rays.

  BVH2 mode (reference node order and slab arithmetic): bit-exact, no ties.
  wide mode: every ray exact, a counted equal-t tie, or a counted
      "reference-culled" hit (the reference's slab test culled a node the
      conservative wide boxes keep); never a missed or farther hit.
"""
from pathlib import Path

import numpy as np
import pytest

from gonzales_b200 import GpuAccelerator, options, scenes
from gonzales_b200 import _ffi as F
from oracle import pyoracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def torch_mod():
    import torch

    return torch


def device_closest(acc, o, d, t, opt=None):
    torch = torch_mod()
    rays = torch.from_numpy(scenes.pack_device_rays(o, d, t)).cuda()
    hits = torch.empty((len(t), 4), dtype=torch.float32, device="cuda")
    acc.trace_closest(rays, hits, opt)
    torch.cuda.synchronize()
    h = hits.cpu().numpy()
    return h[:, 3].view(np.int32).copy(), h[:, 0].copy(), h[:, 1].copy(), h[:, 2].copy()


def device_any(acc, o, d, t, opt=None):
    torch = torch_mod()
    rays = torch.from_numpy(scenes.pack_device_rays(o, d, t)).cuda()
    out = torch.empty(len(t), dtype=torch.int32, device="cuda")
    acc.trace_any(rays, out, opt)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.fixture(scope="module")
def small():
    hs, o, d, t = H.small_raycast(subdiv=4, n_side=64, n_incoherent=8192)
    acc = GpuAccelerator(hs)
    isect, idx, _ = H.oracle_closest(hs, o, d, t)
    yield hs, acc, o, d, t, isect, idx
    acc.close()


def _check(hs, o, d, t, gpu, isect, idx, watertight=False):
    prim, tt, u, v = gpu
    return H.classify(hs, o, d, t, prim, tt, u, v, idx, isect["t_hit"], isect["u"], isect["v"], watertight)


def test_bvh2_mode_is_bit_exact(small):
    hs, acc, o, d, t, isect, idx = small
    gpu = device_closest(acc, o, d, t, options(traversal=F.TRAVERSAL_BVH2))
    counts, fails = _check(hs, o, d, t, gpu, isect, idx)
    assert counts["exact"] == counts["rays"], counts


@pytest.mark.parametrize("traversal", [F.TRAVERSAL_WIDE, F.TRAVERSAL_WIDE_ONE_RAY_PER_THREAD])
def test_wide_mode_parity(small, traversal):
    hs, acc, o, d, t, isect, idx = small
    gpu = device_closest(acc, o, d, t, options(traversal=traversal))
    counts, fails = _check(hs, o, d, t, gpu, isect, idx)
    assert counts["fail"] == 0, (counts, fails[:10])
    assert counts["exact"] >= 0.999 * counts["rays"], counts
    assert acc.error_word() == 0


@pytest.mark.parametrize("traversal", [F.TRAVERSAL_WIDE, F.TRAVERSAL_BVH2])
def test_any_hit(small, traversal):
    hs, acc, o, d, t, isect, idx = small
    anyp = device_any(acc, o, d, t, options(traversal=traversal))
    hit_o = idx >= 0
    hit_g = anyp >= 0
    # every ray the reference hits is occluded on the GPU
    assert np.all(hit_g[hit_o])
    # every GPU any-hit prim is a genuine hit within (0, tMax]
    for i in np.nonzero(hit_g)[0][:: max(1, hit_g.sum() // 500)]:
        p0, p1, p2 = H.prim_triangle(hs, int(anyp[i]))
        assert O.mt(o[i], d[i], p0, p1, p2, float(t[i]))[0]
    extra = np.nonzero(hit_g & ~hit_o)[0]
    for i in extra:
        p0, p1, p2 = H.prim_triangle(hs, int(anyp[i]))
        assert O.mt(o[i], d[i], p0, p1, p2, float(t[i]))[0]
    if traversal == F.TRAVERSAL_BVH2:
        assert len(extra) == 0


def test_intersection_records_drop_in(small):
    """gzg_gpu_traverse_batch returns the reference's Intersection_C records."""
    hs, acc, o, d, t, isect, idx = small
    rays = scenes.pack_reference_rays(o, d)
    res = acc.intersect_batch(rays, t, options(traversal=F.TRAVERSAL_BVH2))
    assert res.tobytes() == isect.tobytes()
    res_w = acc.intersect_batch(rays, t)
    same = res_w.tobytes() == isect.tobytes()
    if not same:
        diff = np.nonzero(res_w["prim_id"]["id1"] != isect["prim_id"]["id1"])[0]
        assert len(diff) <= 0.001 * len(t)


def test_host_batch_pinned_and_pageable_agree(small):
    torch = torch_mod()
    hs, acc, o, d, t, isect, idx = small
    reps = 1300000 // len(t) + 1  # more than one pipelined chunk
    o2, d2, t2 = np.tile(o, (reps, 1)), np.tile(d, (reps, 1)), np.tile(t, reps)
    rays = scenes.pack_reference_rays(o2, d2)
    page = acc.intersect_batch(rays, t2)
    pr = torch.from_numpy(rays).pin_memory()
    pt = torch.from_numpy(t2).pin_memory()
    po = torch.zeros(len(t2) * 48, dtype=torch.uint8).pin_memory()
    out = po.numpy().view(F.INTERSECTION_DTYPE)
    acc.intersect_batch(pr.numpy(), pt.numpy(), out=out)
    assert out.tobytes() == page.tobytes()
    n = len(t)
    assert page[:n].tobytes() == page[n:2 * n].tobytes()
    occ = acc.occluded_batch(rays, t2)
    assert np.array_equal(occ[:n] != 0, device_any(acc, o, d, t) >= 0)


def test_watertight_leaf_test(small):
    hs, acc, o, d, t, _, _ = small
    isect, idx, _ = H.oracle_closest(hs, o, d, t, watertight=True)
    gpu = device_closest(acc, o, d, t, options(traversal=F.TRAVERSAL_BVH2, leaf_test=F.LEAF_WATERTIGHT))
    counts, _ = _check(hs, o, d, t, gpu, isect, idx, watertight=True)
    assert counts["exact"] == counts["rays"], counts
    gpu = device_closest(acc, o, d, t, options(leaf_test=F.LEAF_WATERTIGHT))
    counts, fails = _check(hs, o, d, t, gpu, isect, idx, watertight=True)
    assert counts["fail"] == 0, counts


def test_empty_batch_and_tiny_tmax(small):
    torch = torch_mod()
    hs, acc, o, d, t, _, _ = small
    rays = torch.zeros((0, 8), dtype=torch.float32, device="cuda")
    hits = torch.zeros((0, 4), dtype=torch.float32, device="cuda")
    acc.trace_closest(rays, hits)
    assert len(acc.intersect_batch(np.zeros((0, 6), np.float32), np.zeros(0, np.float32))) == 0
    tt = np.full(len(t), 1e-12, np.float32)
    prim, th, u, v = device_closest(acc, o, d, tt)
    assert (prim == -1).all() and (th == tt).all() and (u == 0).all() and (v == 0).all()


def test_axis_aligned_rays_reference_nan_quirk():
    """Rays with a zero direction component and zero origin component: the
    reference's slab test turns 0 * inf into NaN and culls every box.  BVH2
    mode reproduces that; wide mode finds the hits (reference-culled)."""
    hs = scenes.raycast_scene(subdiv=3).build()
    n = 64
    o = np.zeros((n, 3), np.float32)
    o[:, 2] = np.linspace(-3, 3, n)
    d = np.zeros((n, 3), np.float32)
    d[:, 0] = 1.0
    t = np.full(n, np.inf, np.float32)
    with GpuAccelerator(hs) as acc:
        isect, idx, _ = H.oracle_closest(hs, o, d, t)
        assert (idx == -1).all()
        gpu = device_closest(acc, o, d, t, options(traversal=F.TRAVERSAL_BVH2))
        assert _check(hs, o, d, t, gpu, isect, idx)[0]["exact"] == n
        gpu = device_closest(acc, o, d, t)
        counts, _ = _check(hs, o, d, t, gpu, isect, idx)
        assert counts["fail"] == 0 and counts["reference_culled"] > 0


def test_coincident_triangles_tie_rule():
    """Two identical triangles: the reference keeps the later one at equal t."""
    sb = scenes.SceneBuilder()
    m = sb.add_material()
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    sb.add_mesh(tri, [[0, 1, 2]], m)
    sb.add_mesh(tri, [[0, 1, 2]], m)
    hs = sb.build()
    o = np.array([[0.2, 0.2, 1.0]], np.float32)
    d = np.array([[0, 0, -1]], np.float32)
    t = np.array([np.inf], np.float32)
    with GpuAccelerator(hs) as acc:
        isect, idx, _ = H.oracle_closest(hs, o, d, t)
        gpu = device_closest(acc, o, d, t, options(traversal=F.TRAVERSAL_BVH2))
        assert gpu[0][0] == idx[0]
        gpu = device_closest(acc, o, d, t)
        counts, _ = _check(hs, o, d, t, gpu, isect, idx)
        assert counts["fail"] == 0 and counts["exact"] + counts["tie"] == 1


def test_box_scene_parity():
    hs = scenes.box_scene().build()
    rng = np.random.default_rng(7)
    n = 20000
    o = rng.uniform(0.05, 0.95, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    t = np.full(n, np.inf, np.float32)
    with GpuAccelerator(hs) as acc:
        isect, idx, _ = H.oracle_closest(hs, o, d, t)
        assert (idx >= 0).mean() > 0.7  # five walls: rays toward the open +z side escape
        gpu = device_closest(acc, o, d, t, options(traversal=F.TRAVERSAL_BVH2))
        assert _check(hs, o, d, t, gpu, isect, idx)[0]["exact"] == n
        gpu = device_closest(acc, o, d, t)
        counts, fails = _check(hs, o, d, t, gpu, isect, idx)
        assert counts["fail"] == 0, counts


def test_autotune_picks_a_valid_launch_and_keeps_results(small, tmp_path):
    torch = torch_mod()
    hs, acc, o, d, t, isect, idx = small
    rays = torch.from_numpy(scenes.pack_device_rays(o, d, t)).cuda()
    before = device_closest(acc, o, d, t)
    cache = str(tmp_path / "tuning.json")
    cfg, ms, cached = acc.tune_cached(rays, cache, "raycast-subdiv4")
    assert not cached and ms > 0
    assert cfg["block_size"] in (64, 128, 256)
    assert cfg["stack_depth"] in (0, 16, 32)
    after = device_closest(acc, o, d, t)
    for a, b in zip(before, after):
        assert np.array_equal(H.bits(a) if a.dtype == np.float32 else a, H.bits(b) if b.dtype == np.float32 else b)
    cfg2, ms2, cached2 = acc.tune_cached(rays, cache, "raycast-subdiv4")
    assert cached2 and cfg2 == cfg
    acc.set_launch({"block_size": 128, "blocks_per_sm": 0, "stack_depth": 0, "l1_carveout": 0})


def test_golden_vectors():
    """Committed oracle outputs (tests/golden/raycast_small.npz, made by
    tests/golden/make_golden.py) against the live GPU kernels."""
    g = np.load(GOLDEN / "raycast_small.npz")
    hs = scenes.raycast_scene(subdiv=int(g["subdiv"])).build()
    assert hs.nodes.tobytes() == g["nodes"].tobytes()
    o, d, t = g["o"], g["d"], g["t"]
    with GpuAccelerator(hs) as acc:
        prim, th, u, v = device_closest(acc, o, d, t, options(traversal=F.TRAVERSAL_BVH2))
        assert np.array_equal(prim, g["prim"])
        assert np.array_equal(H.bits(th), H.bits(g["t_hit"]))
        assert np.array_equal(H.bits(u), H.bits(g["u"])) and np.array_equal(H.bits(v), H.bits(g["v"]))
        prim, th, u, v = device_closest(acc, o, d, t)
        counts, _ = H.classify(hs, o, d, t, prim, th, u, v, g["prim"], g["t_hit"], g["u"], g["v"])
        assert counts["fail"] == 0


def test_full_size_raycast_parity():
    """The full ray-cast workload (1,310,720 triangles, 8M coherent + 8M
    incoherent rays) against the oracle on every ray."""
    hs = scenes.raycast_scene(subdiv=8).build()
    o, d, t = scenes.raycast_rays(hs, 4096, 2048, 8388608)
    isect, idx, _ = H.oracle_closest(hs, o, d, t)
    with GpuAccelerator(hs) as acc:
        info = acc.info()
        assert info["triangles"] == 1310720
        gpu = device_closest(acc, o, d, t)
        counts, fails = _check(hs, o, d, t, gpu, isect, idx)
        H.record("parity_full_raycast.json", {"wide": counts, "info": info})
        assert counts["fail"] == 0, (counts, fails[:10])
        gpu = device_closest(acc, o, d, t, options(traversal=F.TRAVERSAL_BVH2))
        assert np.array_equal(gpu[0], idx)
        assert np.array_equal(H.bits(gpu[1]), H.bits(isect["t_hit"]))
        anyp = device_any(acc, o, d, t)
        assert np.all(anyp[idx >= 0] >= 0)
        assert acc.error_word() == 0


def test_compact_host_batch_matches_drop_in_records():
    """gzg_gpu_traverse_batch_hits: the 16-byte records carry the same hits
    as the drop-in Intersection_C records (prim record = prims[index])."""
    hs, o, d, t = H.small_raycast(subdiv=5, n_side=96, n_incoherent=30000)
    r6 = scenes.pack_reference_rays(o, d)
    with GpuAccelerator(hs) as acc:
        full = acc.intersect_batch(r6, t)
        hits = acc.intersect_batch_hits(r6, t)
        assert acc.error_word() == 0
    prim = hits[:, 3].view(np.int32)
    assert np.array_equal(prim >= 0, full["hit"] != 0)
    assert np.array_equal(H.bits(hits[:, 0]), H.bits(full["t_hit"]))
    assert np.array_equal(H.bits(hits[:, 1]), H.bits(full["u"])) and np.array_equal(H.bits(hits[:, 2]), H.bits(full["v"]))
    hit = prim >= 0
    # the fields of each prim record (fancy indexing of a structured array
    # leaves its padding bytes unset, so fields are compared, not bytes)
    for f in ("id1", "id2", "material_index", "type"):
        assert np.array_equal(full["prim_id"][f][hit], hs.prims[f][prim[hit]])


@pytest.fixture(scope="module")
def full():
    hs = scenes.raycast_scene(subdiv=8).build()
    o, d, t = scenes.raycast_rays(hs, 4096, 2048, 8388608)
    acc = GpuAccelerator(hs)
    yield hs, acc, o, d, t
    acc.close()


def test_full_size_any_hit_exact(full):
    """Any hit (a10, the shadow query) on the full ray-cast workload: every
    reported prim is a valid Moller-Trumbore hit with 0 < t <= tMax, every ray
    the oracle's closest hit hits is reported occluded, and a ray the oracle
    misses is reported clear unless its reported prim is such a valid hit
    (the reference's slab test culls a few)."""
    hs, acc, o, d, t = full
    isect, idx, _ = H.oracle_closest(hs, o, d, t)
    anyp = device_any(acc, o, d, t)
    assert np.all(anyp[idx >= 0] >= 0)
    extra = np.nonzero((idx < 0) & (anyp >= 0))[0]
    sample = np.concatenate([extra, np.nonzero(anyp >= 0)[0][::50000]])
    for i in sample:
        p0, p1, p2 = H.prim_triangle(hs, int(anyp[i]))
        ok, tt, _, _ = O.mt(o[i], d[i], p0, p1, p2, float(t[i]))
        assert ok and 0.0 < tt <= t[i], (i, anyp[i])
    H.record("any_hit_full.json", {"rays": int(len(t)), "occluded": int((anyp >= 0).sum()),
                                   "oracle_hits": int((idx >= 0).sum()), "occluded_where_oracle_misses": int(len(extra))})
    assert len(extra) <= 1e-5 * len(t)
    assert acc.error_word() == 0


def test_full_size_watertight_parity(full):
    """The watertight leaf test (Shape/Triangle.swift:269-352) in the wide
    traversal on the full workload against the oracle's watertight traversal:
    exact, a counted tie or a counted reference-culled hit on every ray."""
    hs, acc, o, d, t = full
    isect, idx, _ = H.oracle_closest(hs, o, d, t, watertight=True)
    gpu = device_closest(acc, o, d, t, options(leaf_test=F.LEAF_WATERTIGHT))
    counts, fails = _check(hs, o, d, t, gpu, isect, idx, watertight=True)
    H.record("parity_full_watertight.json", counts)
    assert counts["fail"] == 0, (counts, fails[:10])
    assert counts["exact"] >= 0.9999 * counts["rays"], counts
    assert acc.error_word() == 0


def _edge_scene(kind, rng):
    """Meshes for the wide conversion's edge cases: a few triangles, a cluster
    whose triangle boxes all share one centre (the SAH builder keeps them in
    one leaf of 40 prims, which the conversion splits into groups of 4 before
    choosing the wide nodes), and a grid of small triangles (a deep binary
    tree)."""
    sb = scenes.SceneBuilder()
    m = sb.add_material()
    if kind in ("1", "2", "3", "9"):
        for _ in range(int(kind)):
            c = rng.uniform(-1, 1, 3)
            pts = (c + rng.normal(scale=0.4, size=(3, 3))).astype(np.float32)
            sb.add_mesh(pts, [[0, 1, 2]], m)
    elif kind == "same-centroid":
        # triangles (p, -p, r) with |r| <= |p| per axis: every box is
        # [-|p|, |p|], centred exactly on the origin (exact float values)
        for _ in range(40):
            p = rng.integers(16, 64, 3) * rng.choice([-1, 1], 3) / 64.0
            r = p * rng.integers(-64, 65, 3) / 64.0
            sb.add_mesh(np.array([p, -p, r], np.float32), [[0, 1, 2]], m)
    else:  # grid
        g = np.stack(np.meshgrid(np.linspace(-1, 1, 11), np.linspace(-1, 1, 16)), -1).reshape(-1, 2)
        pts = np.concatenate([g, rng.uniform(-0.05, 0.05, (len(g), 1))], 1).astype(np.float32)
        tris = []
        for j in range(15):
            for i in range(10):
                a = j * 11 + i
                tris += [[a, a + 1, a + 12], [a, a + 12, a + 11]]
        sb.add_mesh(pts, tris, m)
    return sb.build()


@pytest.mark.parametrize("kind", ["1", "2", "3", "9", "same-centroid", "grid"])
def test_wide_conversion_edge_cases(kind):
    """The host conversion's chosen wide nodes on tiny, degenerate and deep
    binary trees: closest hits equal the oracle's (exact or a counted tie,
    never missed or farther), any hit agrees on hit / miss, and no kernel sets
    an error bit."""
    rng = np.random.default_rng(0x5EED + len(kind))
    hs = _edge_scene(kind, rng)
    n = 4096
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    o = (dirs * 4.0).astype(np.float32)
    d = rng.normal(scale=0.5, size=(n, 3)) - o
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    t = np.full(n, np.inf, np.float32)
    with GpuAccelerator(hs) as acc:
        isect, idx, _ = H.oracle_closest(hs, o, d, t)
        assert (idx >= 0).any()
        gpu = device_closest(acc, o, d, t)
        counts, _ = _check(hs, o, d, t, gpu, isect, idx)
        assert counts["fail"] == 0, counts
        anyp = device_any(acc, o, d, t)
        assert np.array_equal(anyp >= 0, idx >= 0)
        assert acc.error_word() == 0
