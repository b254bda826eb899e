"""CPU-only tests of the host side of libgzg: the library loads and exports
every declared entry point, the host SAH builder reproduces the reference
builder (via the oracle restatement) exactly, and argument errors are reported
as status codes."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from gonzales_b200 import _ffi as F
from gonzales_b200 import scene as S
from gonzales_b200 import scenes
from oracle import pyoracle as O

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        names |= set(re.findall(r"GZG_API\s+[\w\s\*]+?\b(gzg_\w+)\s*\(", h.read_text()))
    return names


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", str(F.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    declared = declared_symbols()
    assert declared, "no declarations parsed"
    missing = declared - exported
    assert not missing, missing
    # only declared gzg_ symbols are exported
    extra = {s for s in exported if s.startswith("gzg_")} - declared
    assert not extra, extra


def test_ffi_prototypes_cover_declarations():
    assert set(F.PROTOTYPES) == declared_symbols()
    F.lib()  # loads and binds every prototype


def test_record_layouts_match_reference_header():
    assert F.PRIM_ID_DTYPE.itemsize == 32
    assert F.INTERSECTION_DTYPE.itemsize == 48
    assert F.BVH2_NODE_DTYPE.itemsize == 32
    assert F.MATERIAL_DTYPE.itemsize == 28
    assert F.RAY_DTYPE.itemsize == 24


@pytest.mark.parametrize("subdiv", [0, 1, 3, 5])
def test_host_builder_matches_reference_builder(subdiv):
    hs = scenes.raycast_scene(subdiv=subdiv).build()
    b = S.triangle_bounds(hs.meshes[0])
    bo = O.triangle_bounds(hs.meshes[0].points, hs.meshes[0].vertex_indices)
    assert np.array_equal(b.view(np.uint32), bo.view(np.uint32))
    nodes, order = O.build_bvh2(b)
    assert nodes.tobytes() == hs.nodes.tobytes()
    assert np.array_equal(order, hs.prim_order)


def test_host_builder_box_scene_matches():
    hs = scenes.box_scene().build()
    bounds = np.concatenate([S.triangle_bounds(m) for m in hs.meshes])
    nodes, order = O.build_bvh2(bounds)
    assert nodes.tobytes() == hs.nodes.tobytes()
    assert np.array_equal(order, hs.prim_order)


def _rand_bounds(rng, n, degenerate=False):
    lo = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    if degenerate:
        lo[:] = lo[0]
    ext = rng.uniform(0, 0.2, (n, 3)).astype(np.float32)
    b = np.concatenate([lo, lo + ext], 1).astype(np.float32)
    if degenerate:
        b[:] = b[0]
    return b


@pytest.mark.parametrize("n,degenerate,threads", [(1, False, 1), (2, False, 1), (3, False, 2), (7, True, 4),
                                                  (1000, False, 8), (250000, False, 8), (250000, False, 1)])
def test_host_builder_edge_cases(n, degenerate, threads):
    rng = np.random.default_rng(n)
    b = _rand_bounds(rng, n, degenerate)
    if n == 3:
        b[1] = b[0]  # duplicate prims
    nodes, order = S.build_bvh2(b, threads=threads)
    onodes, oorder = O.build_bvh2(b)
    assert nodes.tobytes() == onodes.tobytes()
    assert np.array_equal(order, oorder)
    assert sorted(order.tolist()) == list(range(n))
    if degenerate:
        assert len(nodes) == 1 and nodes[0]["count"] == n  # identical centroids -> one leaf


def test_host_builder_zero_area_prims():
    # flat prims in a plane: bounds.surfaceArea() == 0 at the root -> one leaf
    b = np.zeros((5, 6), np.float32)
    b[:, 0] = np.arange(5)
    b[:, 3] = np.arange(5)
    nodes, order = S.build_bvh2(b)
    onodes, oorder = O.build_bvh2(b)
    assert nodes.tobytes() == onodes.tobytes() and np.array_equal(order, oorder)


def test_host_builder_argument_errors():
    L = F.lib()
    cnt = F.I64(0)
    assert L.gzg_host_build_bvh2(None, -1, None, C.byref(cnt), None, 0) == 1
    assert b"bad arguments" in L.gzg_last_error()
    assert L.gzg_host_build_bvh2(None, 0, None, C.byref(cnt), None, 0) == 0 and cnt.value == 0
    assert L.gzg_host_triangle_bounds(None, None, -5, None) == 1


def test_free_null_scene_is_noop():
    assert F.lib().gzg_gpu_free_scene(None) == 0


def test_upload_rejects_bad_arguments_before_touching_a_device():
    L = F.lib()
    h = C.c_void_p()
    assert L.gzg_gpu_upload_scene(None, 0, None, 0, None, 0, None, None, None, None, 0, C.byref(h)) == 1
    assert L.gzg_gpu_upload_scene(None, 1, None, 0, None, 0, None, None, None, None, 0, None) == 1


def _upload_status(hs):
    meshes = hs.mesh_structs()
    pts, fi, vi = hs.counts()
    h = C.c_void_p()
    st = F.lib().gzg_gpu_upload_scene(F.ptr(hs.nodes), len(hs.nodes), F.ptr(hs.prims), len(hs.prims),
                                      C.addressof(meshes), len(hs.meshes), F.ptr(pts), F.ptr(fi), F.ptr(vi),
                                      F.ptr(hs.materials), len(hs.materials), C.byref(h))
    if st == 0:
        F.lib().gzg_gpu_free_scene(h)
    return st, F.lib().gzg_last_error().decode()


def test_upload_rejects_cyclic_bvh():
    hs = scenes.raycast_scene(subdiv=1).build()
    hs.nodes[0]["offset"] = 0  # right child points back at the root
    st, msg = _upload_status(hs)
    assert st == 5 and "child link" in msg


def test_upload_rejects_out_of_range_vertex():
    hs = scenes.raycast_scene(subdiv=1).build()
    hs.meshes[0].vertex_indices[4] = 10 ** 9
    st, msg = _upload_status(hs)
    assert st == 5 and "out of range" in msg


def test_upload_rejects_bad_leaf_range():
    hs = scenes.raycast_scene(subdiv=1).build()
    leaf = np.nonzero(hs.nodes["count"] > 0)[0][0]
    hs.nodes[leaf]["offset"] = len(hs.prims)
    st, msg = _upload_status(hs)
    assert st == 5 and "leaf range" in msg


def test_upload_valid_scene_without_device_reports_no_device():
    from tests.conftest import HAS_GPU

    if HAS_GPU:
        pytest.skip("device present")
    st, _ = _upload_status(scenes.raycast_scene(subdiv=1).build())
    assert st == 2


def test_batch_renderer_rejects_bad_arguments_before_touching_a_device():
    L = F.lib()
    h = C.c_void_p()
    p = F.render_params(8, 8, 1)
    opts = F.BatchOptions(0, 0, 0, 0)
    assert L.gzg_batch_renderer_create(None, C.byref(p), 1, C.byref(opts), C.byref(h)) == 1
    assert L.gzg_batch_renderer_create(None, C.byref(p), 0, C.byref(opts), C.byref(h)) == 1
    assert L.gzg_batch_renderer_create(None, C.byref(p), 1, C.byref(opts), None) == 1
    bad = F.BatchOptions(0, 0, 9, 0)
    assert L.gzg_batch_renderer_create(None, C.byref(p), 1, C.byref(bad), C.byref(h)) == 1
    assert "sort key" in L.gzg_last_error().decode()
    assert L.gzg_renderer_film_layout(None, None) == 1
    assert L.gzg_renderer_autotune(None, None, None, None) == 1
    assert L.gzg_renderer_error_word(None, None, 0) == 1
    assert L.gzg_renderer_set_textures(None, None, 0, 0, None, 1.0) == 1
    assert L.gzg_renderer_render_f64(None, None, None, None, None) == 1
    assert L.gzg_renderer_adjoint(None, None, None, None, None, None) == 1
    assert L.gzg_renderer_destroy(None) == 0


def test_batch_workload_shapes():
    work = scenes.batch_workload(n_scenes=6, seed=5, tri_lo=1_000, tri_hi=4_000)
    assert len(work) == 6
    for sb, side in work:
        assert side in scenes.BATCH_SIDES
        n = sum(m.triangle_count for m in sb.meshes)
        assert 10 + 2 <= n <= 10 + 4_000 + 16
        assert 1 <= len(sb._lights) // 2 <= 8


def _build_status(hs, leaf_size=0):
    meshes = hs.mesh_structs()
    pts, fi, vi = hs.counts()
    h = C.c_void_p()
    opt = F.BuildOptions()
    opt.leaf_size = leaf_size
    st = F.lib().gzg_gpu_build_scene(F.ptr(hs.prims), len(hs.prims), C.addressof(meshes), len(hs.meshes),
                                     F.ptr(pts), F.ptr(fi), F.ptr(vi), F.ptr(hs.materials), len(hs.materials),
                                     C.byref(opt), C.byref(h))
    if st == 0:
        F.lib().gzg_gpu_free_scene(h)
    return st, F.lib().gzg_last_error().decode()


def test_device_build_rejects_bad_input_before_touching_a_device():
    L = F.lib()
    h = C.c_void_p()
    assert L.gzg_gpu_build_scene(None, 1, None, 0, None, None, None, None, 0, None, C.byref(h)) == 1
    assert L.gzg_gpu_build_scene(None, 0, None, 0, None, None, None, None, 0, None, None) == 1
    hs = scenes.raycast_scene(subdiv=1).build(host_bvh=False)
    assert hs.nodes is None and np.array_equal(hs.prim_order, np.arange(len(hs.prims)))
    st, msg = _build_status(hs, leaf_size=5)
    assert st == 1 and "leaf_size" in msg
    # every triangle prim is validated (no tree limits which are read)
    hs.meshes[0].vertex_indices[7] = 10 ** 9
    st, msg = _build_status(hs)
    assert st == 5 and "prim 2" in msg


def test_device_build_without_device_reports_no_device():
    from tests.conftest import HAS_GPU

    if HAS_GPU:
        pytest.skip("device present")
    st, _ = _build_status(scenes.raycast_scene(subdiv=1).build(host_bvh=False))
    assert st == 2


def test_root_bounds_without_a_host_tree():
    a = scenes.box_scene().build()
    b = scenes.box_scene().build(host_bvh=False)
    lo_a, hi_a = a.root_bounds()
    lo_b, hi_b = b.root_bounds()
    np.testing.assert_allclose(lo_a, lo_b, atol=1e-6)
    np.testing.assert_allclose(hi_a, hi_b, atol=1e-6)


# ---------------------------------------------------------------- PLY ingestion


def _ply_mesh():
    sb = scenes.raycast_scene(subdiv=2)
    m = sb.meshes[0]
    return m.points[:, :3].copy(), m.vertex_indices.reshape(-1, 3).astype(np.int32)


@pytest.mark.parametrize("big_endian", [False, True])
@pytest.mark.parametrize("list_type", ["uchar", "uint"])
@pytest.mark.parametrize("layout", ["p", "pn", "puv", "pnuv"])
def test_ply_round_trip(tmp_path, big_endian, list_type, layout):
    from gonzales_b200 import scene as S

    pts, idx = _ply_mesh()
    nrm = (pts / np.linalg.norm(pts, axis=1, keepdims=True)).astype(np.float32) if "n" in layout else None
    uv = pts[:, :2].copy() if "uv" in layout else None
    fi = np.arange(len(idx), dtype=np.int32) * 3 if layout == "pnuv" else None
    path = tmp_path / "m.ply"
    S.write_ply(path, pts, idx, normals=nrm, uvs=uv, big_endian=big_endian, list_type=list_type, face_indices=fi)
    r = S.read_ply(path)
    assert np.array_equal(r["points"], pts) and np.array_equal(r["indices"], idx)
    assert (r["normals"] is None) == (nrm is None) and (r["uvs"] is None) == (uv is None)
    if nrm is not None:
        assert np.array_equal(r["normals"], nrm)
    if uv is not None:
        assert np.array_equal(r["uvs"], uv)
    if fi is not None:
        assert np.array_equal(r["face_indices"], fi)
    # the same bytes parsed from memory
    r2 = S.read_ply(data=path.read_bytes())
    assert np.array_equal(r2["indices"], idx)


def _ply_error(data):
    from gonzales_b200 import GzgError, scene as S

    with pytest.raises(GzgError) as e:
        S.read_ply(data=data)
    return str(e.value)


def test_ply_rejects_malformed_files(tmp_path):
    from gonzales_b200 import scene as S

    pts, idx = _ply_mesh()
    path = tmp_path / "m.ply"
    S.write_ply(path, pts, idx)
    good = path.read_bytes()
    assert "ply" in _ply_error(b"plx\n" + good[4:])
    assert "format" in _ply_error(good.replace(b"binary_little_endian", b"ascii"))
    assert "shorter" in _ply_error(good[:-5])
    assert "vertex properties" in _ply_error(good.replace(b"property float z\n", b"property float w\n"))
    # a quad face
    head, body = good.split(b"end_header\n")
    nv = len(pts)
    quad = bytearray(body)
    off = nv * 12
    quad[off] = 4
    assert "not 3" in _ply_error(head + b"end_header\n" + bytes(quad))
    # an index out of range
    bad = bytearray(body)
    bad[off + 1:off + 5] = np.int32(nv).tobytes()
    assert "out of range" in _ply_error(head + b"end_header\n" + bytes(bad))


def test_mesh_arrays_build_rejects_bad_arguments_before_touching_a_device():
    from gonzales_b200 import GpuAccelerator, GzgError

    pts, idx = _ply_mesh()
    mats = np.zeros(1, F.MATERIAL_DTYPE)
    mats[0] = (1, (0.5, 0.5, 0.5), (0, 0, 0))
    with pytest.raises(GzgError) as e:
        GpuAccelerator.from_mesh_arrays([(pts, idx, 3)], mats)
    assert "material index" in str(e.value)


def test_exr_round_trip(tmp_path):
    from gonzales_b200 import film

    rng = np.random.default_rng(5)
    img = rng.random((7, 11, 3), dtype=np.float32) * 4
    film.write_exr(tmp_path / "a.exr", img)
    back, header = film.read_exr(tmp_path / "a.exr")
    assert back.shape == (7, 11, 4)
    assert np.array_equal(back[..., :3], img) and np.all(back[..., 3] == 1.0)
    for k in ("channels", "compression", "dataWindow", "displayWindow", "lineOrder", "pixelAspectRatio",
              "screenWindowCenter", "screenWindowWidth"):
        assert k in header
    raw = (tmp_path / "a.exr").read_bytes()
    assert raw[:4] == bytes([0x76, 0x2F, 0x31, 0x01])
    rgba = rng.random((3, 5, 4), dtype=np.float32)
    film.write_exr(tmp_path / "b.exr", rgba)
    assert np.array_equal(film.read_exr(tmp_path / "b.exr")[0], rgba)
    from gonzales_b200 import GzgError

    with pytest.raises(GzgError):
        film.write_exr(tmp_path / "c.exr", np.zeros((2, 2, 2), np.float32))
