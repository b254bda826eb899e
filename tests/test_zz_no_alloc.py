"""gzg_gpu_traverse_batch_static: the closest-hit host batch for callers that
cannot allocate device or pinned memory on their render path (a renderer inside
a process whose GPU memory belongs to another allocator's pool, or a loop that
must not call cudaFree because it synchronises the device).  It stages through
a fixed array in the library's device image instead of allocating.

Checked against gzg_gpu_traverse_batch (the allocating entry point) on two
calls in a row with different rays: the records must be byte-identical (both
run the same kernel with the scene's tuned launch).  Checked against the
oracle's closest hits by the wide-mode parity rule (exact, or a counted
equal-t tie or reference-culled hit, never a failure).  Two-level scenes and
oversized calls are rejected with their errors.  The file is named to be
collected last.
"""
import numpy as np
import pytest

from gonzales_b200 import GpuAccelerator, InstancedAccelerator, scenes
from gonzales_b200 import _ffi as F
from tests import helpers as H

pytestmark = pytest.mark.gpu

MAX_RAYS = 65536


@pytest.fixture(scope="module")
def scene():
    hs = scenes.raycast_scene(subdiv=5).build()
    acc = GpuAccelerator(hs)
    yield hs, acc
    acc.close()


def call_static(handle, rays6, tmax):
    out = np.zeros(len(tmax), F.INTERSECTION_DTYPE)
    status = F.lib().gzg_gpu_traverse_batch_static(handle, F.ptr(rays6), F.ptr(tmax), len(tmax), F.ptr(out))
    return status, out


def test_static_batch_matches_allocating_batch_and_oracle_on_two_calls(scene):
    hs, acc = scene
    for seed, (w, h, inc) in ((0x51, (160, 160, 36000)), (0x52, (96, 64, 20000))):
        o, d, t = scenes.raycast_rays(hs, w, h, inc, seed=seed)
        assert len(t) <= MAX_RAYS
        rays6 = scenes.pack_reference_rays(o, d)
        status, out = call_static(acc.handle, rays6, t)
        assert status == 0, F.lib().gzg_last_error()
        ref = acc.intersect_batch(rays6, t)
        assert out.tobytes() == ref.tobytes()
        assert 0.1 < out["hit"].mean() < 1.0
        ora, ora_idx, _ = H.oracle_closest(hs, o, d, t)
        # the GPU record carries the prim-id record itself; every prim here is
        # a geometric prim with a unique id1, which maps it back to its index
        assert np.all(hs.prims["type"] == 1)
        lut = np.full(int(hs.prims["id1"].max()) + 1, -1, np.int64)
        lut[hs.prims["id1"]] = np.arange(len(hs.prims))
        gpu_idx = np.where(out["hit"] != 0, lut[np.maximum(out["prim_id"]["id1"], 0)], -1)
        counts, fails = H.classify(hs, o, d, t, gpu_idx, out["t_hit"], out["u"], out["v"], ora_idx,
                                   ora["t_hit"], ora["u"], ora["v"])
        assert counts["fail"] == 0, (counts, fails[:10])
        assert counts["exact"] >= 0.999 * counts["rays"], counts
    assert acc.error_word() == 0


def test_static_batch_rejects_more_than_capacity(scene):
    hs, acc = scene
    n = MAX_RAYS + 1
    rays6 = np.zeros((n, 6), np.float32)
    rays6[:, 5] = 1.0
    t = np.ones(n, np.float32)
    status, _ = call_static(acc.handle, rays6, t)
    assert status == 7
    assert b"65536" in F.lib().gzg_last_error()
    status, _ = call_static(acc.handle, rays6[:0], t[:0])
    assert status == 0


def test_static_batch_rejects_two_level_scene():
    blas, inst = scenes.instanced_scene(n_meshes=2, n_u=10, n_v=12, n_instances=8, extent=3.0, seed=0x5A)
    accs = [GpuAccelerator(b) for b in blas]
    try:
        with InstancedAccelerator(accs, inst) as iacc:
            o, d, t = scenes.instanced_rays(64, 3.0, 0x5B)
            status, out = call_static(iacc.handle, scenes.pack_reference_rays(o, d), t)
            assert status == 1
            assert b"two-level" in F.lib().gzg_last_error()
            assert iacc.error_word() == 0
    finally:
        for a in accs:
            a.close()
