"""gzg_gpu_traverse_batch_static: the closest-hit host batch for callers that
cannot allocate device or pinned memory on their render path (a renderer inside
a process whose GPU memory belongs to another allocator's pool, or a loop that
must not call cudaFree because it synchronises the device).  It stages through
a fixed array in the library's device image instead of allocating.

Checked against gzg_gpu_traverse_batch (the allocating entry point) on two
calls in a row with different rays: the records must be byte-identical (both
run the same kernel).  The file is named to be collected last.
"""
import numpy as np
import pytest

from gonzales_b200 import GpuAccelerator, scenes
from gonzales_b200 import _ffi as F

pytestmark = pytest.mark.gpu

MAX_RAYS = 65536


@pytest.fixture(scope="module")
def scene():
    hs = scenes.raycast_scene(subdiv=5).build()
    acc = GpuAccelerator(hs)
    yield hs, acc
    acc.close()


def call_static(acc, rays6, tmax):
    out = np.zeros(len(tmax), F.INTERSECTION_DTYPE)
    status = F.lib().gzg_gpu_traverse_batch_static(acc.handle, F.ptr(rays6), F.ptr(tmax), len(tmax), F.ptr(out))
    return status, out


def test_static_batch_matches_allocating_batch_on_two_calls(scene):
    hs, acc = scene
    for seed, (w, h, inc) in ((0x51, (160, 160, 36000)), (0x52, (96, 64, 20000))):
        o, d, t = scenes.raycast_rays(hs, w, h, inc, seed=seed)
        assert len(t) <= MAX_RAYS
        rays6 = scenes.pack_reference_rays(o, d)
        status, out = call_static(acc, rays6, t)
        assert status == 0, F.lib().gzg_last_error()
        ref = acc.intersect_batch(rays6, t)
        assert out.tobytes() == ref.tobytes()
        assert 0.1 < out["hit"].mean() < 1.0


def test_static_batch_rejects_more_than_capacity(scene):
    hs, acc = scene
    n = MAX_RAYS + 1
    rays6 = np.zeros((n, 6), np.float32)
    rays6[:, 5] = 1.0
    t = np.ones(n, np.float32)
    status, _ = call_static(acc, rays6, t)
    assert status == 7
    assert b"65536" in F.lib().gzg_last_error()
    status, _ = call_static(acc, rays6[:0], t[:0])
    assert status == 0
