"""The multi-GPU split on CPU: two gloo ranks (127.0.0.1) each render their
slice of a frame's Z-Sobol samples with the oracle integrator and all-reduce
the film sums; the result equals the single-process frame (the same samples,
summed in another order), and summed per-rank gradient buffers equal their
total.  The GPU path uses the same helpers with NCCL."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from gonzales_b200 import distributed as D


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sample_ranges_partition_the_frame():
    for spp in (1, 5, 16, 33):
        for world in (1, 2, 3, 8):
            got = []
            for r in range(world):
                first, count = D.sample_range(spp, r, world)
                got.extend(range(first, first + count))
            assert got == list(range(spp))
    with pytest.raises(ValueError):
        D.sample_range(8, 2, 2)


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from gonzales_b200 import scenes
    from oracle import pyoracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        hs = scenes.box_scene().build()
        params = O.render_params(24, 16, 6, max_depth=3, rr_min_bounce=2)
        rgb = torch.zeros((16, 24, 3), dtype=torch.float64)
        w = torch.zeros((16, 24), dtype=torch.float64)

        def render_slice(p, films):
            s, _, sw, _ = O.render(hs, p, threads=2)
            films[0] += torch.from_numpy(s.astype(np.float64))
            films[1] += torch.from_numpy(sw.astype(np.float64))

        D.render_frame(render_slice, params, [rgb, w])
        g = torch.full((4,), float(rank + 1), dtype=torch.float32)
        e = torch.tensor(0.5 * (rank + 1), dtype=torch.float64)
        D.allreduce_gradients(g, e)
        if rank == 0:
            np.save(os.path.join(out_dir, "rgb.npy"), rgb.numpy())
            np.save(os.path.join(out_dir, "w.npy"), w.numpy())
            np.save(os.path.join(out_dir, "grad.npy"), np.concatenate([g.numpy(), [e.item()]]))
    finally:
        dist.destroy_process_group()


def test_two_rank_frame_equals_single_frame(tmp_path):
    from gonzales_b200 import scenes
    from oracle import pyoracle as O

    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    hs = scenes.box_scene().build()
    s, _, sw, _ = O.render(hs, O.render_params(24, 16, 6, max_depth=3, rr_min_bounce=2), threads=2)
    np.testing.assert_allclose(np.load(tmp_path / "rgb.npy"), s, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(np.load(tmp_path / "w.npy"), sw, rtol=1e-6)
    np.testing.assert_allclose(np.load(tmp_path / "grad.npy"), [3, 3, 3, 3, 1.5])
