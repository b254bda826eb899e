"""Two-level scenes (TransformedPrimitive semantics) on the GPU against the
oracle's restatement, on identical rays and the same host-built top-level BVH.

Per ray the (bottom-level prim, instance, t, u, v) is exact, a counted
equal-t tie, or a counted reference-culled hit (a valid nearer hit the
reference's slab test would cull); never a miss or a farther hit.
"""

import numpy as np
import pytest

from gonzales_b200 import GpuAccelerator, InstancedAccelerator, scenes
from gonzales_b200 import _ffi as F
from oracle import pyoracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu


def torch_mod():
    import torch

    return torch


def gpu_instanced(iacc, o, d, t):
    torch = torch_mod()
    rays = torch.from_numpy(scenes.pack_device_rays(o, d, t)).cuda()
    hits = torch.empty((len(t), 4), dtype=torch.float32, device="cuda")
    inst = torch.empty(len(t), dtype=torch.int32, device="cuda")
    iacc.trace_closest(rays, hits, inst)
    anyp = torch.empty(len(t), dtype=torch.int32, device="cuda")
    iacc.trace_any(rays, anyp)
    torch.cuda.synchronize()
    h = hits.cpu().numpy()
    return (h[:, 3].view(np.int32).copy(), inst.cpu().numpy(), h[:, 0].copy(), h[:, 1].copy(), h[:, 2].copy(),
            anyp.cpu().numpy())


def object_ray(inst, k, o, d):
    m = inst["world_to_object"][k].reshape(3, 4).astype(np.float32)
    oo = np.zeros(3, np.float32)
    dd = np.zeros(3, np.float32)
    for r in range(3):
        oo[r] = np.float32(np.float32(np.float32(m[r, 0] * o[0]) + np.float32(m[r, 1] * o[1])) + np.float32(m[r, 2] * o[2])) + m[r, 3]
        dd[r] = np.float32(np.float32(m[r, 0] * d[0]) + np.float32(m[r, 1] * d[1])) + np.float32(m[r, 2] * d[2])
    return oo, dd


def classify_instanced(blas, inst, o, d, tmax, gpu, ora):
    gp, gi, gt, gu, gv = gpu[:5]
    op, oi, ot, ou, ov = ora
    exact = (gp == op) & (gi == oi) & ((op < 0) | ((H.bits(gt) == H.bits(ot)) & (H.bits(gu) == H.bits(ou)) &
                                                     (H.bits(gv) == H.bits(ov))))
    counts = {"rays": len(gp), "exact": int(exact.sum()), "tie": 0, "reference_culled": 0, "fail": 0}
    fails = []
    for i in np.nonzero(~exact)[0]:
        if gp[i] < 0 or gi[i] < 0:
            fails.append(i)
            continue
        oo, dd = object_ray(inst, gi[i], o[i], d[i])
        p0, p1, p2 = H.prim_triangle(blas[inst["blas"][gi[i]]], int(gp[i]))
        ok, t, u, v = O.mt(oo, dd, p0, p1, p2, float(tmax[i]))
        valid = ok and H.bits(t) == H.bits(gt[i]) and H.bits(u) == H.bits(gu[i]) and H.bits(v) == H.bits(gv[i])
        if not valid:
            fails.append(i)
        elif op[i] >= 0 and H.bits(gt[i]) == H.bits(ot[i]):
            counts["tie"] += 1
        elif op[i] < 0 or gt[i] < ot[i]:
            counts["reference_culled"] += 1
        else:
            fails.append(i)
    counts["fail"] = len(fails)
    return counts, fails


def run_case(n_meshes, n_u, n_v, n_inst, extent, n_rays, seed):
    blas, inst = scenes.instanced_scene(n_meshes=n_meshes, n_u=n_u, n_v=n_v, n_instances=n_inst, extent=extent,
                                        seed=seed)
    accs = [GpuAccelerator(b) for b in blas]
    iacc = InstancedAccelerator(accs, inst)
    o, d, t = scenes.instanced_rays(n_rays, extent, seed + 1)
    gpu = gpu_instanced(iacc, o, d, t)
    ora = O.traverse_instanced(iacc.tlas_nodes, iacc.leaf_instance, inst["world_to_object"], inst["blas"], blas,
                               scenes.pack_reference_rays(o, d), t)
    counts, fails = classify_instanced(blas, inst, o, d, t, gpu, ora)
    anyp = gpu[5]
    assert np.all(anyp[ora[0] >= 0] >= 0)
    assert iacc.error_word() == 0
    info = iacc.info()
    iacc.close()
    for a in accs:
        a.close()
    return counts, fails, info, ora


def test_instanced_matches_oracle_small():
    counts, fails, info, ora = run_case(4, 30, 40, 64, 5.0, 20000, 0xC2)
    assert counts["fail"] == 0, (counts, fails[:10])
    assert counts["exact"] >= 0.999 * counts["rays"], counts
    assert (ora[0] >= 0).mean() > 0.1


def test_identity_instance_reproduces_single_level_scene():
    torch = torch_mod()
    hs, o, d, t = H.small_raycast(subdiv=4, n_side=48, n_incoherent=4096)
    inst = np.zeros(1, F.INSTANCE_DTYPE)
    eye = np.eye(4)[:3].reshape(12).astype(np.float32)
    inst["object_to_world"][0] = eye
    inst["world_to_object"][0] = eye
    with GpuAccelerator(hs) as acc:
        iacc = InstancedAccelerator([acc], inst)
        gp, gi, gt, gu, gv, _ = gpu_instanced(iacc, o, d, t)
        rays = torch.from_numpy(scenes.pack_device_rays(o, d, t)).cuda()
        hits = torch.empty((len(t), 4), dtype=torch.float32, device="cuda")
        acc.trace_closest(rays, hits)
        torch.cuda.synchronize()
        h = hits.cpu().numpy()
        assert np.array_equal(gp, h[:, 3].view(np.int32))
        assert np.array_equal(H.bits(gt), H.bits(h[:, 0]))
        assert np.all(gi[gp >= 0] == 0) and np.all(gi[gp < 0] == -1)
        iacc.close()


def test_instanced_full_size_parity():
    """16 meshes x 50,000 triangles, 4096 instances; 2M rays."""
    counts, fails, info, ora = run_case(16, 125, 200, 4096, 20.0, 1 << 21, 0xC2)
    H.record("parity_instanced.json", {"wide": counts, "info": info})
    assert counts["fail"] == 0, (counts, fails[:10])
    assert info["triangles"] == 16 * 50000


def test_instance_bounds_from_trees_contain_geometry_and_are_tighter():
    """gzg_host_instance_bounds_from_scenes: every vertex of every instance,
    carried to world space, lies inside its box, and the boxes are no larger
    than those from the bottom-level root box's corners (the reference's
    TransformedPrimitive.worldBound)."""
    from gonzales_b200.accel import instance_bounds

    blas_hosts, inst = scenes.instanced_scene(n_meshes=4, n_u=30, n_v=40, n_instances=256, extent=5.0, seed=0xB5)
    accs = [GpuAccelerator(b) for b in blas_hosts]
    try:
        iacc = InstancedAccelerator(accs, inst)
        tight = iacc.bounds
        loose = instance_bounds(blas_hosts, inst)
        for k in range(len(inst)):
            m = inst["object_to_world"][k].reshape(3, 4).astype(np.float64)
            pts = blas_hosts[inst["blas"][k]].meshes[0].points[:, :3].astype(np.float64)
            world = pts @ m[:, :3].T + m[:, 3]
            assert np.all(world >= tight[k, :3] - 1e-6) and np.all(world <= tight[k, 3:] + 1e-6), k
        vol_t = np.prod(tight[:, 3:] - tight[:, :3], axis=1)
        vol_l = np.prod(loose[:, 3:] - loose[:, :3], axis=1)
        assert np.all(vol_t <= vol_l * (1 + 1e-4))
        assert vol_t.sum() < 0.9 * vol_l.sum()
        iacc.close()
    finally:
        for a in accs:
            a.close()
