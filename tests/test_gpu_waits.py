"""Bounded host waits.  Every host wait of the batch calls polls an event for
at most GZG_WAIT_LIMIT_US microseconds (default 300 s) and then returns
GZG_ERR_TIMEOUT instead of blocking; the call's queued work keeps running and
its staging buffers are left to it.  The limit is made to run out on the host
(1 us, far below the time a chunk of rays needs): nothing faults or hangs on
the GPU.  Afterwards the same scene handle serves new calls unchanged.
"""
import numpy as np
import pytest

from gonzales_b200 import GpuAccelerator, GzgError, scenes

pytestmark = pytest.mark.gpu

GZG_ERR_TIMEOUT = 8


def test_wait_limit_returns_timeout_and_scene_stays_usable(monkeypatch):
    import torch

    from gonzales_b200 import _ffi as F

    hs = scenes.raycast_scene(subdiv=6).build()
    o, d, t = scenes.raycast_rays(hs, 2048, 1024, 4_000_000, seed=0x77)
    # pinned buffers take the direct path: every chunk is queued before the
    # first wait, so the waits find work still in flight
    rays6 = torch.from_numpy(scenes.pack_reference_rays(o, d)).pin_memory().numpy()
    t = torch.from_numpy(t).pin_memory().numpy()
    out = torch.zeros(len(t) * F.INTERSECTION_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
    out = out.numpy().view(F.INTERSECTION_DTYPE)
    with GpuAccelerator(hs) as acc:
        ref = acc.intersect_batch(rays6[:5000], t[:5000])
        monkeypatch.setenv("GZG_WAIT_LIMIT_US", "1")
        with pytest.raises(GzgError) as e:
            acc.intersect_batch(rays6, t, out=out)
        assert e.value.status == GZG_ERR_TIMEOUT
        assert "GZG_WAIT_LIMIT_US" in str(e.value)
        monkeypatch.delenv("GZG_WAIT_LIMIT_US")
        torch.cuda.synchronize()  # the abandoned chunks run to the end (into `out`)
        again = acc.intersect_batch(rays6[:5000], t[:5000])
        assert again.tobytes() == ref.tobytes()
        full = acc.intersect_batch(rays6, t)
        assert full[:5000].tobytes() == ref.tobytes()
        assert acc.error_word() == 0
