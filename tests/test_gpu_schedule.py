"""The persistent kernels' chunk schedule on the device calls.

A persistent traversal launch hands its rays out in 32-ray chunks through a
pull counter.  Launches on callers' streams take that counter from the
scene's ring of counters, each of which waits for the last launch that used
it, so launches that run at the same time on different streams must never
share one: a shared counter would skip chunks (rays left unwritten) or trace
some twice.  Launches of more than 2^30 rays are split
into consecutive launches over slices of the arrays; every slice must land
at its own offset.  A device call on a stream being captured into a CUDA
graph runs the static schedule; the graph's replays must equal the eager
call.
"""
import numpy as np
import pytest
import torch

from gonzales_b200 import GpuAccelerator, scenes

pytestmark = pytest.mark.gpu


def _ray_sets(hs, count):
    sets = []
    for k in range(count):
        o, d, t = scenes.raycast_rays(hs, 512 + 128 * k, 512, 600000 + 150000 * k, seed=0x5C00 + k)
        sets.append(torch.from_numpy(scenes.pack_device_rays(o, d, t)).cuda())
    return sets


def test_concurrent_streams_match_serial_launches():
    hs = scenes.raycast_scene(subdiv=6).build()
    with GpuAccelerator(hs) as acc:
        sets = _ray_sets(hs, 4)
        serial_hits, serial_any = [], []
        for rays in sets:
            h = torch.empty((rays.shape[0], 4), dtype=torch.float32, device="cuda")
            a = torch.empty(rays.shape[0], dtype=torch.int32, device="cuda")
            acc.trace_closest(rays, h)
            acc.trace_any(rays, a)
            serial_hits.append(h)
            serial_any.append(a)
        torch.cuda.synchronize()

        streams = [torch.cuda.Stream() for _ in sets]
        outs = []
        for rep in range(3):
            for k, (rays, st) in enumerate(zip(sets, streams)):
                # NaN / -2 sentinels: a ray the launch skipped keeps them
                h = torch.full((rays.shape[0], 4), float("nan"), dtype=torch.float32, device="cuda")
                a = torch.full((rays.shape[0],), -2, dtype=torch.int32, device="cuda")
                torch.cuda.synchronize()
                outs.append((k, h, a))
        torch.cuda.synchronize()
        # every stream's launches are queued back to back, all streams at once
        for rep in range(3):
            for k, st in enumerate(streams):
                _, h, a = outs[rep * len(sets) + k]
                acc.trace_closest(sets[k], h, stream=st)
                acc.trace_any(sets[k], a, stream=st)
        torch.cuda.synchronize()
        for k, h, a in outs:
            assert torch.equal(h.view(torch.int32), serial_hits[k].view(torch.int32)), k
            assert torch.equal(a, serial_any[k]), k
        assert acc.error_word() == 0


def test_launch_above_2_pow_30_rays_is_split_into_slices():
    n = (1 << 30) + 12345
    need = n * (32 + 16) + (1 << 30)
    free, _ = torch.cuda.mem_get_info()
    if free < need:
        pytest.skip(f"needs {need / 1e9:.1f} GB of free device memory, {free / 1e9:.1f} GB free")
    hs = scenes.raycast_scene(subdiv=4).build()
    with GpuAccelerator(hs) as acc:
        base_n = 1 << 16
        o, d, t = scenes.raycast_rays(hs, 128, 256, base_n - 128 * 256, seed=0x5D)
        base = torch.from_numpy(scenes.pack_device_rays(o, d, t)).cuda()
        want = torch.empty((base_n, 4), dtype=torch.float32, device="cuda")
        acc.trace_closest(base, want)
        reps = (n + base_n - 1) // base_n
        big = base.repeat(reps, 1)[:n]
        hits = torch.full((n, 4), float("nan"), dtype=torch.float32, device="cuda")
        acc.trace_closest(big, hits)
        torch.cuda.synchronize()
        del big
        rng = np.random.default_rng(7)
        idx = np.concatenate([
            np.arange(0, base_n),
            np.arange((1 << 30) - base_n, n),
            rng.integers(0, n, 20000),
        ])
        idx_t = torch.from_numpy(idx).cuda()
        got = hits[idx_t].view(torch.int32)
        exp = want[idx_t % base_n].view(torch.int32)
        assert torch.equal(got, exp)
        # no slot of the whole output was left unwritten
        assert not torch.isnan(hits[:, 0]).any().item()
        assert acc.error_word() == 0


def test_device_trace_captured_in_a_cuda_graph_matches_eager_launch():
    # a stream under capture gets the static schedule (no pull counter, no
    # event waits across the capture's boundary); replays equal the eager call
    hs = scenes.raycast_scene(subdiv=5).build()
    with GpuAccelerator(hs) as acc:
        o, d, t = scenes.raycast_rays(hs, 256, 256, 300000, seed=0x5E)
        rays = torch.from_numpy(scenes.pack_device_rays(o, d, t)).cuda()
        n = rays.shape[0]
        want = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        acc.trace_closest(rays, want)
        torch.cuda.synchronize()
        got = torch.full((n, 4), float("nan"), dtype=torch.float32, device="cuda")
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            acc.trace_closest(rays, got, stream=side)  # warm-up outside the capture
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        got.fill_(float("nan"))
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            acc.trace_closest(rays, got, stream=torch.cuda.current_stream())
        for _ in range(2):
            got.fill_(float("nan"))
            graph.replay()
            torch.cuda.synchronize()
            assert torch.equal(got.view(torch.int32), want.view(torch.int32))
        del graph
        assert acc.error_word() == 0
