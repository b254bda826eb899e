"""Thread safety of the host batch calls on one scene handle.

The reference's tile renderer runs up to cores-1 tile tasks at once
(Core/TileRenderer.swift:77-109), and every one of them calls the plugin's
batch trace on the same GPU scene handle (Core/Tile.swift:82-97).  The
drop-in calls must therefore give the same records when 8 host threads call
gzg_gpu_traverse_batch and gzg_gpu_occluded_batch on one handle at the same
time as when the calls run one after another.  ctypes releases the GIL for
the duration of each foreign call, so the calls really overlap.
"""
import threading

import numpy as np
import pytest

from gonzales_b200 import GpuAccelerator, scenes

pytestmark = pytest.mark.gpu

N_THREADS = 8
CALLS_PER_THREAD = 4


def test_concurrent_batches_on_one_handle_match_serial_calls():
    hs = scenes.raycast_scene(subdiv=6).build()
    with GpuAccelerator(hs) as acc:
        work = []
        for k in range(N_THREADS):
            # uneven sizes: some calls span several 512K-ray chunks, some are tiny
            w, h, inc = [(640, 480, 400000), (64, 64, 1000), (1024, 600, 700000), (32, 8, 17)][k % 4]
            o, d, t = scenes.raycast_rays(hs, w, h, inc, seed=0x7000 + k)
            work.append((scenes.pack_reference_rays(o, d), t))
        serial = [(acc.intersect_batch(r, t).tobytes(), acc.occluded_batch(r, t).tobytes()) for r, t in work]

        barrier = threading.Barrier(N_THREADS)
        results = [None] * N_THREADS
        errors = []

        def run(k):
            try:
                r, t = work[k]
                barrier.wait()
                out = []
                for c in range(CALLS_PER_THREAD):
                    if (k + c) % 2 == 0:
                        out.append(("closest", acc.intersect_batch(r, t).tobytes()))
                    else:
                        out.append(("any", acc.occluded_batch(r, t).tobytes()))
                results[k] = out
            except Exception as e:  # noqa: BLE001
                errors.append((k, repr(e)))

        threads = [threading.Thread(target=run, args=(k,)) for k in range(N_THREADS)]
        for th in threads:
            th.start()
        for th in threads:
            th.join(timeout=300)
        assert not any(th.is_alive() for th in threads), "a batch call did not return"
        assert not errors, errors
        for k in range(N_THREADS):
            for kind, blob in results[k]:
                want = serial[k][0] if kind == "closest" else serial[k][1]
                assert blob == want, (k, kind)
        assert acc.error_word() == 0
