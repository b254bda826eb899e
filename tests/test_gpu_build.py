"""The device tree build (gzg_gpu_build_scene: linear BVH over Morton codes,
radix tree, bottom-up bounds, collapse into the wide layout) against the
oracle's traversal of the host's SAH tree on the same rays.

Closest hits do not depend on the tree: every ray is exact, a counted
equal-t tie or a counted reference-culled hit (the parity classes of the
traversal tests), never a miss or a farther hit.  Prim ids index the prims as
given (any order).  Edge cases: one triangle, no intersectable prim, many
coincident centroids (equal Morton codes), leaves of 1 to 4 prims.  A
render of a device-built scene equals the render of the uploaded one.
"""
import numpy as np
import pytest

from gonzales_b200 import GpuAccelerator, scenes
from gonzales_b200 import _ffi as F
from gonzales_b200.scene import SceneBuilder
from tests import helpers as H
from tests.test_gpu_traversal import device_any, device_closest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    hs, o, d, t = H.small_raycast(subdiv=5, n_side=64, n_incoherent=16384)
    isect, idx, _ = H.oracle_closest(hs, o, d, t)
    return hs, o, d, t, isect, idx


@pytest.mark.parametrize("builder", [F.BUILD_PLOC, F.BUILD_LBVH])
@pytest.mark.parametrize("leaf_size", [1, 2, 4])
def test_device_built_tree_matches_oracle(small, leaf_size, builder):
    hs, o, d, t, isect, idx = small
    with GpuAccelerator(hs, device_build=True, leaf_size=leaf_size, builder=builder) as acc:
        assert acc.device_built
        info = acc.info()
        assert info["bvh2_nodes"] == 0 and info["triangles"] == len(hs.prims)
        gpu = device_closest(acc, o, d, t)
        counts, fails = H.classify(hs, o, d, t, *gpu, idx, isect["t_hit"], isect["u"], isect["v"])
        assert counts["fail"] == 0, (counts, fails[:10])
        assert counts["exact"] >= 0.999 * counts["rays"], counts
        anyp = device_any(acc, o, d, t)
        assert np.all(anyp[idx >= 0] >= 0)
        assert acc.build_time_ms() > 0.0
        cost = acc.tree_cost()
        assert np.isfinite(cost) and cost > 1.0
        assert acc.error_word() == 0
        # no reference BVH2: the reference-order kernel is refused
        from gonzales_b200 import GzgError, options

        with pytest.raises(GzgError):
            device_closest(acc, o, d, t, options(traversal=F.TRAVERSAL_BVH2))


def _identity(hs, prim):
    """A triangle's identity independent of prim order: (mesh << 32 | tri)."""
    prim = np.asarray(prim, np.int64)
    out = np.full(len(prim), -1, np.int64)
    ok = prim >= 0
    out[ok] = hs.prims["id2"][prim[ok]]
    return out


def test_prims_in_input_order(small):
    hs_sorted, o, d, t, isect, idx = small
    hs = scenes.raycast_scene(subdiv=5).build(host_bvh=False)
    with GpuAccelerator(hs) as acc:
        assert acc.device_built
        prim, tt, u, v = device_closest(acc, o, d, t)
    same_t = H.bits(tt) == H.bits(np.where(idx >= 0, isect["t_hit"], t))
    same_tri = _identity(hs, prim) == _identity(hs_sorted, idx)
    # equal t everywhere but where the oracle's slab test culled a nearer hit
    culled = (~same_t) & (tt < np.where(idx >= 0, isect["t_hit"], np.inf)) & (prim >= 0)
    assert np.all(same_t | culled)
    assert same_tri[same_t].mean() > 0.999


def _tri_builder(tris):
    sb = SceneBuilder()
    m = sb.add_material((0.5, 0.5, 0.5))
    pts = np.asarray(tris, np.float32).reshape(-1, 3)
    sb.add_mesh(pts, np.arange(len(pts)).reshape(-1, 3), m)
    return sb


def _tri_scene(tris):
    return _tri_builder(tris).build(host_bvh=False)


@pytest.mark.parametrize("builder", [F.BUILD_PLOC, F.BUILD_LBVH])
def test_single_triangle_and_coincident_centroids(builder):
    hs = _tri_scene([[[-1, -1, 0], [1, -1, 0], [0, 1, 0]]])
    o = np.array([[0, 0, 2], [5, 5, 2]], np.float32)
    d = np.array([[0, 0, -1], [0, 0, -1]], np.float32)
    t = np.full(2, np.inf, np.float32)
    with GpuAccelerator(hs, builder=builder) as acc:
        prim, tt, _, _ = device_closest(acc, o, d, t)
    assert prim.tolist() == [0, -1] and tt[0] == 2.0
    # 300 triangles tilted about the y axis by different amounts, all with
    # the box centre (0, 0, 0): the centroid bounds are a point, every Morton
    # code is 0, and the keys are ordered by prim index alone
    tris = []
    for h in np.linspace(-0.3, 0.3, 300):
        tris.append([[-1.0, -1.0, -h], [1.0, -1.0, h], [0.0, 1.0, 0.0]])
    sb = _tri_builder(tris)
    rng = np.random.default_rng(3)
    o = np.concatenate([rng.uniform(-1, 1, (2000, 2)), np.full((2000, 1), 1.0)], 1).astype(np.float32)
    d = np.tile(np.array([[0, 0, -1]], np.float32), (2000, 1))
    t = np.full(2000, np.inf, np.float32)
    isect, idx, _ = H.oracle_closest(sb.build(), o, d, t)
    with GpuAccelerator(sb.build(host_bvh=False), builder=builder) as acc:
        prim, tt, _, _ = device_closest(acc, o, d, t)
        assert acc.error_word() == 0
    hit = idx >= 0
    assert hit.any()
    assert np.array_equal(prim >= 0, hit)
    assert np.array_equal(H.bits(tt[hit]), H.bits(isect["t_hit"][hit]))


def test_no_intersectable_prim():
    # a transformed-primitive record (type 2) is never intersected
    hs = _tri_scene([[[-1, -1, 0], [1, -1, 0], [0, 1, 0]]])
    hs.prims["type"][0] = 2
    hs.prims["id2"][0] = -1
    o = np.array([[0, 0, 2]], np.float32)
    d = np.array([[0, 0, -1]], np.float32)
    t = np.full(1, np.inf, np.float32)
    with GpuAccelerator(hs) as acc:
        assert acc.info()["triangles"] == 0
        prim, tt, _, _ = device_closest(acc, o, d, t)
    assert prim[0] == -1


def test_device_built_render_equals_uploaded():
    sb = scenes.box_scene()
    hs_up, hs_dev = sb.build(), sb.build(host_bvh=False)
    p = F.render_params(64, 64, 16, max_depth=5, rr_min_bounce=3)
    with GpuAccelerator(hs_up) as a, GpuAccelerator(hs_dev) as b:
        ra = a.render(p)
        rb = b.render(p)
    np.testing.assert_allclose(ra[0], rb[0], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(ra[2], rb[2], rtol=1e-6)
    assert ra[3]["extension_rays"] == rb[3]["extension_rays"]


def test_full_size_device_build():
    """The ray-cast mesh (1,310,720 triangles): the device-built tree gives
    the host-built tree's closest-hit distances on all 16,777,216 rays."""
    torch = pytest.importorskip("torch")
    sb = scenes.raycast_scene(subdiv=8)
    hs = sb.build()
    o, d, t = scenes.raycast_rays(hs, 4096, 2048, 8388608)
    with GpuAccelerator(hs) as up:
        g_up = device_closest(up, o, d, t)
        cost_up = up.tree_cost()
    record = {"tree_cost_host": cost_up}
    for builder, name in ((F.BUILD_PLOC, "ploc"), (F.BUILD_LBVH, "lbvh")):
        with GpuAccelerator(hs, device_build=True, builder=builder) as dev:
            g_dev = device_closest(dev, o, d, t)
            build_ms = dev.build_time_ms()
            cost_dev = dev.tree_cost()
            info = dev.info()
            assert dev.error_word() == 0
        same_t = H.bits(g_up[1]) == H.bits(g_dev[1])
        assert same_t.all(), (name, int((~same_t).sum()))
        same_prim = g_up[0] == g_dev[0]
        assert same_prim.mean() > 0.99999
        assert build_ms > 0
        record[name] = {"build_ms": build_ms, "tree_cost": cost_dev, "prim_mismatch_equal_t": int((~same_prim).sum()),
                        "info": info}
    H.record("device_build_full.json", record)


# ---------------------------------------------------------------- ingestion fast path


def _arrays_of(sb):
    """(mesh arrays, materials) of a SceneBuilder: one entry per mesh with its
    prims' material; area-light meshes get one emissive material each."""
    hs = sb.build(host_bvh=False)
    mats = list(hs.materials[: len(sb._materials)])
    meshes = []
    for mesh_idx, ntri, ptype, material, first in sb._prims:
        m = sb.meshes[mesh_idx]
        pts = m.points[:, :3]
        idx = m.vertex_indices.reshape(-1, 3).astype(np.int32)
        if ptype == 3:
            le = sb._lights[first]
            mats.append((2, (0, 0, 0), le))
            mat = len(mats) - 1
        else:
            mat = material
        meshes.append((pts, idx, mat))
    arr = np.zeros(len(mats), F.MATERIAL_DTYPE)
    for k, m in enumerate(mats):
        arr[k] = tuple(m) if not isinstance(m, np.void) else m
    return meshes, arr, hs


def test_mesh_arrays_scene_matches_oracle(small, tmp_path):
    from gonzales_b200 import scene as S

    hs_sorted, o, d, t, isect, idx = small
    sb = scenes.raycast_scene(subdiv=5)
    m = sb.meshes[0]
    # through a PLY file: write, read, build
    path = tmp_path / "ico.ply"
    S.write_ply(path, m.points[:, :3], m.vertex_indices.reshape(-1, 3))
    ply = S.read_ply(path)
    mats = np.zeros(1, F.MATERIAL_DTYPE)
    mats[0] = (1, (0.5, 0.5, 0.5), (0, 0, 0))
    with GpuAccelerator.from_mesh_arrays([(ply["points"], ply["indices"], 0)], mats) as acc:
        info = acc.info()
        assert info["triangles"] == len(ply["indices"]) and acc.build_time_ms() > 0
        prim, tt, u, v = device_closest(acc, o, d, t)
        assert acc.error_word() == 0
    # prim k is triangle k of mesh 0 (id2 = 0 << 32 | k), the builder's convention
    gpu_tri = np.where(prim >= 0, prim, -1)
    ora_tri = _identity(hs_sorted, idx)
    same_t = H.bits(tt) == H.bits(np.where(idx >= 0, isect["t_hit"], t))
    culled = (~same_t) & (tt < np.where(idx >= 0, isect["t_hit"], np.inf)) & (prim >= 0)
    assert np.all(same_t | culled)
    assert (gpu_tri == ora_tri)[same_t].mean() > 0.999


def test_mesh_arrays_render_equals_builder_render():
    sb = scenes.box_scene()
    meshes, mats, hs = _arrays_of(sb)
    p = F.render_params(64, 64, 16, max_depth=5, rr_min_bounce=3)
    with GpuAccelerator(sb.build()) as a, GpuAccelerator.from_mesh_arrays(meshes, mats) as b:
        ra = a.render(p)
        rb = b.render(p)
    np.testing.assert_allclose(ra[0], rb[0], rtol=1e-5, atol=1e-6)
    assert ra[3]["shadow_rays"] == rb[3]["shadow_rays"]


def test_mesh_arrays_reject_out_of_range_index():
    from gonzales_b200 import GzgError

    mats = np.zeros(1, F.MATERIAL_DTYPE)
    mats[0] = (1, (0.5, 0.5, 0.5), (0, 0, 0))
    pts = np.zeros((3, 3), np.float32)
    with pytest.raises(GzgError) as e:
        GpuAccelerator.from_mesh_arrays([(pts, np.array([[0, 1, 3]], np.int32), 0)], mats)
    assert "out of" in str(e.value)


# ---------------------------------------------------------------- device-built scenes elsewhere


def test_device_built_blas_in_a_two_level_scene():
    """Bottom-level scenes built on the device (their host tree copies feed
    the two-level assembly) give the uploaded ones' closest hits."""
    from gonzales_b200 import InstancedAccelerator
    from tests.test_gpu_instanced import gpu_instanced

    blas_hosts, inst = scenes.instanced_scene(n_meshes=4, n_u=30, n_v=20, n_instances=64, extent=5.0)
    o, d, t = scenes.instanced_rays(200000, 5.0, 11)
    res = []
    for device in (False, True):
        blas = [GpuAccelerator(h, device_build=device) for h in blas_hosts]
        with InstancedAccelerator(blas, inst) as acc:
            res.append(gpu_instanced(acc, o, d, t))
            assert acc.error_word() == 0
        for b in blas:
            b.close()
    (p0, i0, t0, _, _, a0), (p1, i1, t1, _, _, a1) = res
    assert np.array_equal(H.bits(t0), H.bits(t1))
    assert ((p0 == p1) & (i0 == i1)).mean() > 0.9999
    assert np.array_equal(a0 >= 0, a1 >= 0)


def test_batch_of_device_built_scenes_equals_solo_renders():
    import torch

    from gonzales_b200 import BatchRenderer

    sb = scenes.box_scene()
    meshes, mats, _ = _arrays_of(sb)
    accs = [GpuAccelerator(sb.build(host_bvh=False)), GpuAccelerator.from_mesh_arrays(meshes, mats),
            GpuAccelerator(scenes.batch_scene(11, 3_000).build(host_bvh=False))]
    params = [F.render_params(48, 40, 8, max_depth=5, rr_min_bounce=3),
              F.render_params(32, 32, 4, max_depth=4, rr_min_bounce=2, mis_corrected=1),
              F.render_params(32, 32, 4, max_depth=6, rr_min_bounce=2)]
    solo = [a.render(p) for a, p in zip(accs, params)]
    with BatchRenderer(accs, params) as r:
        rgb = torch.zeros((r.pixels, 3), device="cuda")
        sq = torch.zeros((r.pixels, 3), device="cuda")
        w = torch.zeros((r.pixels,), device="cuda")
        r.render(rgb, w, sq)
        torch.cuda.synchronize()
        parts = list(zip(r.split(rgb.cpu().numpy()), r.split(w.cpu().numpy())))
        assert r.error_word() == 0
    for (b_rgb, b_w), (s_rgb, _, s_w, _) in zip(parts, solo):
        np.testing.assert_allclose(b_rgb, s_rgb, rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(b_w, s_w, rtol=1e-6)
    for a in accs:
        a.close()
