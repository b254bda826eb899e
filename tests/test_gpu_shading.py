"""Vertex normals and UVs on the device (gzg_scene_set_vertex_attributes)
against the oracle's restatement of Triangle.computeSurfaceInteraction with
them, at equal Z-Sobol indices: a flat scene with a smooth UV-mapped coated
sphere and a smooth diffuse blob, MIS as written and corrected; a two-level
scene of smooth meshes; a batch holding the smooth scene equals its solo
render.  Per pixel, means agree within 3 combined standard errors on >= 99 %
of pixels and most pixels agree to 1e-3."""
import numpy as np
import pytest

from gonzales_b200 import BatchRenderer, GpuAccelerator, InstancedAccelerator, scenes
from gonzales_b200 import _ffi as F
from gonzales_b200.scene import SceneBuilder
from oracle import pyoracle as O
from tests.test_gpu_materials import _agree

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mis", [0, 1])
def test_smooth_scene_matches_oracle(mis):
    hs = scenes.smooth_box_scene().build()
    p = dict(width=64, height=64, spp=16, max_depth=5, rr_min_bounce=3, mis_corrected=mis)
    with GpuAccelerator(hs) as acc:
        g = acc.render(F.render_params(**p))
        assert acc.error_word() == 0
    o = O.render(hs, O.render_params(**p))
    within, close, gi, oi = _agree(g, o, p["spp"])
    assert within >= 0.99, within
    assert close > 0.8, close
    np.testing.assert_allclose(gi, oi, rtol=1e-2)
    # the normals matter: without them the device image differs
    for m in hs.meshes:
        m.normals = m.uvs = None
    with GpuAccelerator(hs) as acc:
        g2 = acc.render(F.render_params(**p))
    assert not np.allclose(g[0], g2[0], rtol=1e-3)


def test_smooth_two_level_scene_matches_oracle():
    blas = []
    for k in range(3):
        pts, tris = scenes.displaced_icosphere(2, amplitude=0.08, seed=20 + k)
        sb = SceneBuilder()
        sb.add_mesh(pts * 0.5, tris, sb.add_material((0.3 + 0.2 * k, 0.5, 0.6)),
                    normals=pts / np.linalg.norm(pts, axis=1, keepdims=True))
        blas.append(sb.build())
    inst = scenes.random_instances(48, 3, seed=5, extent=4.0)
    sky = scenes.sky_map(128, 64)
    p = dict(width=48, height=40, spp=16, max_depth=4, rr_min_bounce=2, eye=(0.0, 2.0, 14.0), target=(0.0, 0.0, 0.0))
    accs = [GpuAccelerator(h) for h in blas]
    with InstancedAccelerator(accs, inst) as acc:
        acc.set_environment(sky, 1.0)
        g = acc.render(F.render_params(**p))
        tlas, leaf = acc.tlas_nodes, acc.leaf_instance
    for a in accs:
        a.close()
    o = O.render(None, O.render_params(**p), env=O.Environment(sky, 1.0),
                 instances=dict(tlas_nodes=tlas, leaf_instance=leaf, instances=inst, blas=blas))
    within, close, gi, oi = _agree(g, o, p["spp"])
    assert within >= 0.99, within
    np.testing.assert_allclose(gi, oi, rtol=1e-2)


def test_batch_with_smooth_scene_equals_solo():
    import torch

    accs = [GpuAccelerator(scenes.smooth_box_scene().build()), GpuAccelerator(scenes.box_scene().build())]
    params = [F.render_params(40, 40, 8, max_depth=4, rr_min_bounce=2),
              F.render_params(32, 32, 4, max_depth=4, rr_min_bounce=2)]
    solo = [a.render(p) for a, p in zip(accs, params)]
    with BatchRenderer(accs, params) as r:
        rgb = torch.zeros((r.pixels, 3), device="cuda")
        w = torch.zeros((r.pixels,), device="cuda")
        r.render(rgb, w)
        torch.cuda.synchronize()
        parts = list(zip(r.split(rgb.cpu().numpy()), r.split(w.cpu().numpy())))
    for (b_rgb, b_w), (s_rgb, _, s_w, _) in zip(parts, solo):
        np.testing.assert_allclose(b_rgb, s_rgb, rtol=1e-5, atol=1e-6)
    for a in accs:
        a.close()


def test_vertex_attributes_are_validated():
    from gonzales_b200 import GzgError

    hs = scenes.box_scene().build()
    with GpuAccelerator(hs) as acc:
        with pytest.raises(GzgError):
            acc.set_vertex_attributes(0, normals=np.zeros((3, 3), np.float32))  # wrong vertex count
        with pytest.raises(GzgError):
            acc.set_vertex_attributes(99, normals=np.zeros((3, 3), np.float32))  # no such mesh


def test_ply_normals_through_the_fast_path(tmp_path):
    """A PLY mesh with vertex normals and UVs (x y z nx ny nz u v) read and
    built on the device shades like the same mesh through the builder."""
    from gonzales_b200 import scene as S

    pts, tris = scenes.icosphere(2)
    pts = pts * 0.2 + np.array([0.5, 0.2, 0.5])
    nrm = (pts - np.array([0.5, 0.2, 0.5])) / 0.2
    uv = pts[:, :2].copy()
    path = tmp_path / "s.ply"
    S.write_ply(path, pts, tris, normals=nrm, uvs=uv)
    ply = S.read_ply(path)
    sb = SceneBuilder()
    rng = np.random.default_rng(4)
    scenes._room(sb, rng)
    m = sb.add_material((0.6, 0.5, 0.4))
    sb.add_mesh(ply["points"], ply["indices"], m, normals=ply["normals"], uvs=ply["uvs"])
    lp, lt = scenes._quad((0.35, 0.999, 0.35), (0.65, 0.999, 0.35), (0.65, 0.999, 0.65), (0.35, 0.999, 0.65))
    sb.add_area_light(lp, lt, (15.0, 11.0, 4.0))
    hs = sb.build()
    room = hs.meshes[0]
    mats = np.zeros(3, F.MATERIAL_DTYPE)
    mats[0] = hs.materials[0]
    mats[1] = hs.materials[1]
    mats[2] = (2, (0, 0, 0), (15.0, 11.0, 4.0))
    light = hs.meshes[2]
    arrays = [(room.points[:, :3], room.vertex_indices.reshape(-1, 3), 0),
              (ply["points"], ply["indices"], 1, ply["normals"], ply["uvs"]),
              (light.points[:, :3], light.vertex_indices.reshape(-1, 3), 2)]
    p = F.render_params(48, 48, 8, max_depth=4, rr_min_bounce=3)
    with GpuAccelerator(hs) as a, GpuAccelerator.from_mesh_arrays(arrays, mats) as b:
        ra, rb = a.render(p), b.render(p)
    np.testing.assert_allclose(ra[0], rb[0], rtol=1e-5, atol=1e-6)
