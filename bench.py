#!/usr/bin/env python
"""Ray-cast throughput of libgzg on B200 (one JSON line on rank 0).

Workload (the headline single-GPU configuration): a displaced icosphere of
1,310,720 triangles (SAH BVH2, <= 4 prims per leaf, converted to 8-wide
quantised nodes) and 16,777,216 rays: 8,388,608 coherent pinhole rays at
4096 x 2048 and 8,388,608 incoherent rays (origins uniform in the bounds,
directions uniform on the sphere, tMax uniform in [0.1, 2] * diagonal).
A step is one closest-hit pass over all rays.  Inputs (512 MiB of rays) and
outputs (256 MiB of hits) are larger than the 126 MB L2, so no flush is done.

  value     closest-hit Mrays/s, rays resident in HBM, CUDA events around the
            K timed launches, max over ranks
  e2e       the same through gzg_gpu_traverse_batch (the drop-in call) from
            pinned host Ray_C + tMax to host Intersection_C records
  roofline  algorithmic bytes of the traversal kernel (48 B ray I/O + 80 B per
            wide node + 48 B per triangle, counts from an instrumented replay)
            over the average launch time, against the measured HBM copy
            bandwidth; `coherent` and `incoherent` give the same for each half
            of the rays launched alone; `io_lower_bound` the ray I/O alone
            (48 B per ray) and `reference_layout` the bytes the same launch
            time would move in the reference's layout (BVH2 records and
            triangle tests counted by an instrumented replay of the
            reference-order kernel, 104 B per triangle test, 76 B of ray I/O)
  cpu_baseline  the oracle (CPU restatement of the reference traversal, over
            a tree built by the oracle's own SAH builder) on the host cores
  render, batch, adjoint, instanced, device_build
            the renderer legs (box scene, 64-scene batch, adjoint step,
            two-level scene with the general materials) and the device tree
            build against the host's SAH build, each described in its entry

--impl reference times that CPU implementation alone over all rays per step
(the reference's own Swift/Mojo build cannot run here); it builds its tree
with the oracle, so libgzg.so is never loaded in that process.  Multi-GPU (torchrun): every rank traces
its own full ray set against a replica of the scene (weak scaling, no
collective on the data path).
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s (closest-hit/shadow) & spp/s, batched vs plain on B200 at equal relMSE"
FULL = dict(subdiv=8, width=4096, height=2048, incoherent=8388608)
SMALL = dict(subdiv=7, width=2048, height=1024, incoherent=2097152)  # profiler case, rays > L2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="small case for profiler captures")
    ap.add_argument("--skip-cpu", action="store_true", help="omit the CPU baseline leg")
    ap.add_argument("--skip-batch", action="store_true", help="omit the scene-batch and adjoint legs")
    ap.add_argument("--case", default=None,
                    choices=["instanced-small", "build", "incoherent", "coherent", "mixed", "render"],
                    help="run one small case alone (profiler captures) and print its own JSON line")
    return ap.parse_args()


def workload(small, rank):
    from gonzales_b200 import scenes

    cfg = SMALL if small else FULL
    hs = scenes.raycast_scene(subdiv=cfg["subdiv"]).build()
    o, d, t = scenes.raycast_rays(hs, cfg["width"], cfg["height"], cfg["incoherent"], seed=0xC1 + 7 * rank)
    name = "raycast_icosphere_%dtri_%dM_rays" % (hs.triangle_count, round(len(t) / 2 ** 20))
    return cfg, hs, o, d, t, name


def oracle_workload(small):
    """The same mesh, rays and SAH BVH2 built by the oracle alone (its own
    triangle bounds and builder), for the CPU legs: libgzg.so is never loaded
    for them.  The oracle's node array and prim order are byte-identical to
    the library builder's (tests/test_host.py)."""
    from types import SimpleNamespace

    from gonzales_b200 import scenes
    from gonzales_b200.scene import make_mesh
    from oracle import pyoracle as O

    cfg = SMALL if small else FULL
    pts, tris = scenes.displaced_icosphere(cfg["subdiv"], seed=0xC1)
    mesh = make_mesh(pts, tris)
    nodes, order = O.build_bvh2(O.triangle_bounds(mesh.points, mesh.vertex_indices))
    prims = np.zeros(len(order), O.PRIM_DTYPE)
    prims["id1"] = order
    prims["id2"] = order  # mesh 0 << 32 | triangle
    prims["type"] = 1     # geometric primitive
    hs = SimpleNamespace(meshes=[mesh], nodes=nodes, prims=prims, triangle_count=mesh.triangle_count)
    o, d, t = scenes.raycast_rays(hs, cfg["width"], cfg["height"], cfg["incoherent"], seed=0xC1)
    name = "raycast_icosphere_%dtri_%dM_rays" % (hs.triangle_count, round(len(t) / 2 ** 20))
    return cfg, hs, o, d, t, name


def workload_config(cfg, hs, name, world):
    """The `config` object both arms print (the workload, not the method)."""
    return {"workload": name, "triangles": int(hs.triangle_count), "rays": cfg["width"] * cfg["height"] +
            cfg["incoherent"], "coherent_rays": cfg["width"] * cfg["height"], "incoherent_rays": cfg["incoherent"],
            "query": "closest hit", "leaf_test": "moller_trumbore",
            "l2": "inputs 512 MiB + outputs 256 MiB > L2, no flush",
            "parallelism": "replica per GPU" if world > 1 else "single GPU"}


def measured_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle reasons from NVML every 20 ms in a thread."""

    def __init__(self, device_index):
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml

            pynvml.nvmlInit()
            import torch

            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
            self._h = pynvml.nvmlDeviceGetHandleByUUID(uuid.encode())
            self._nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # noqa: BLE001
            self.error = repr(e)

    def _run(self):
        nv = self._nv
        names = {
            "hw_slowdown": getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
            "hw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
            "sw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
            "sw_power_cap": getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4),
            "hw_power_brake_slowdown": getattr(nv, "nvmlClocksEventReasonHwPowerBrakeSlowdown", 0x80),
        }
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                    nv.nvmlDeviceGetCurrentClocksThrottleReasons
                r = fn(self._h)
                for k, bit in names.items():
                    if r & bit:
                        self.reasons.add(k)
            except Exception:  # noqa: BLE001
                pass
            time.sleep(0.02)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._h is not None:
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def cpu_baseline(small, budget_s=20.0):
    """The oracle traversal on all host threads over the oracle-built tree; a
    strided sample of the workload sized to roughly budget_s seconds of wall
    time."""
    from gonzales_b200 import scenes
    from oracle import pyoracle as O

    _, hs, o, d, t, _ = oracle_workload(small)

    cores = os.cpu_count() or 1
    meshes = [(m.points, m.vertex_indices) for m in hs.meshes]
    probe = np.arange(0, len(t), max(1, len(t) // 200000))
    r6 = scenes.pack_reference_rays(o[probe], d[probe])
    t0 = time.perf_counter()
    O.traverse(hs.nodes, hs.prims, meshes, r6, t[probe], threads=cores)
    rate = len(probe) / max(time.perf_counter() - t0, 1e-6)
    n = int(min(len(t), max(len(probe), rate * budget_s)))
    stride = max(1, len(t) // n)
    sel = np.arange(0, len(t), stride)
    r6 = scenes.pack_reference_rays(o[sel], d[sel])
    t0 = time.perf_counter()
    O.traverse(hs.nodes, hs.prims, meshes, r6, t[sel], threads=cores)
    el = time.perf_counter() - t0
    return {"value": len(sel) / el / 1e6, "unit": "Mrays/s", "cores": cores, "kind": "port",
            "sample": "every %d-th ray of the workload (%d rays, coherent and incoherent in proportion), "
                      "closest hit, oracle BVH2 + Moller-Trumbore, %d threads" % (stride, len(sel), cores)}


RENDER = dict(width=256, height=256, spp=16, max_depth=5, rr_min_bounce=3)


def render_leg(acc_box, args, stream, barrier):
    """The box-scene path tracer (256 x 256, 16 spp, depth 5, roulette from
    bounce 3): one frame per step through a graph-captured wavefront."""
    import torch

    from gonzales_b200 import GpuAccelerator, Renderer, scenes
    from gonzales_b200 import _ffi as F

    hs = scenes.box_scene().build()
    acc = GpuAccelerator(hs)
    p = F.render_params(**RENDER, use_graph=1)
    W, H = RENDER["width"], RENDER["height"]
    rgb = torch.zeros((H, W, 3), device="cuda")
    w = torch.zeros((H, W), device="cuda")
    steps = max(3, min(args.steps, 20))
    with Renderer(acc, p) as r:
        for _ in range(max(3, args.warmup)):
            r.render(rgb, w)
        barrier()
        s0 = r.stats()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            r.render(rgb, w)
        e1.record(stream)
        barrier()
        s1 = r.stats()
    acc.close()
    ms = e0.elapsed_time(e1) / steps
    rays = sum(s1[k] - s0[k] for k in ("camera_rays", "extension_rays", "shadow_rays", "probe_rays")) / steps
    spp = W * H * RENDER["spp"]
    return {"config": "box scene 36 tris, %dx%d, %d spp, max depth %d, roulette from bounce %d, MIS as written"
                      % (W, H, RENDER["spp"], RENDER["max_depth"], RENDER["rr_min_bounce"]),
            "spp_per_s": spp / ms * 1000.0, "ms_per_frame": ms, "mrays_per_s": rays / ms / 1000.0,
            "rays_per_frame": rays, "steps": steps, "graph": True}


BATCH = dict(n_scenes=64, seed=0xC3, spp=32, max_depth=6, rr_min_bounce=2, ref_spp=4096, ref_seed=4321,
             relmse_bar=1e-3)


def batch_leg(args, stream, barrier):
    """The scene batch: 64 scenes (triangles log-uniform in 1k-500k,
    displaced icospheres or box stacks; image sides among 64-512; 1-8 ceiling
    lights), depth 6, roulette from bounce 2.  Plain = one graph-captured
    renderer per scene, each scene's frame timed on its own and the times
    summed; batched = one autotuned renderer over all scenes.  Both compute
    the same per-path estimates, so their relMSE is equal by construction.
    Reference: a 4096-spp render of every scene with another Z-Sobol seed
    (the GPU renderer equals the oracle at equal samples; tests check it per
    pixel on a subset of these scenes).  Timed at the configuration's 32 spp
    and at the smallest power-of-two spp whose relMSE is at most 1e-3."""
    import torch

    from gonzales_b200 import BatchRenderer, GpuAccelerator, Renderer, scenes
    from gonzales_b200 import _ffi as F

    t0 = time.perf_counter()
    work = scenes.batch_workload(BATCH["n_scenes"], BATCH["seed"])
    hosts = [sb.build() for sb, _ in work]
    accs = [GpuAccelerator(h) for h in hosts]
    setup_s = time.perf_counter() - t0
    sides = [side for _, side in work]

    def params_at(spp, **kw):
        return [F.render_params(side, side, spp, max_depth=BATCH["max_depth"], rr_min_bounce=BATCH["rr_min_bounce"],
                                use_graph=1, **kw) for side in sides]

    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def timed(fn, steps, warm=1):
        for _ in range(warm):
            fn()
        barrier()
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        barrier()
        return e0.elapsed_time(e1) / steps

    def plain_ms(params, steps, film_rgb, film_w, offs):
        """Sum over scenes of one scene's frame time on its own renderer."""
        total = 0.0
        for k, (a, p) in enumerate(zip(accs, params)):
            with Renderer(a, p) as r:
                total += timed(lambda: r.render(film_rgb[offs[k]:offs[k + 1]], film_w[offs[k]:offs[k + 1]],
                                                stream=stream), steps)
        return total

    def image(rgb, w):
        return (rgb / w[:, None]).cpu().numpy()

    params = params_at(BATCH["spp"])
    paths = sum(p.width * p.height * p.spp for p in params)
    steps = max(3, min(args.steps, 5))
    with BatchRenderer(accs, params) as br:
        tuned, tuned_ms = br.autotune(stream)
        pix, offs = br.pixels, br.offsets
        rgb_b = torch.zeros((pix, 3), device="cuda")
        w_b = torch.zeros((pix,), device="cuda")
        ms_b = timed(lambda: br.render(rgb_b, w_b, stream=stream), steps)
        err = br.error_word()
    rgb_p = torch.zeros((pix, 3), device="cuda")
    w_p = torch.zeros((pix,), device="cuda")
    ms_p = plain_ms(params, steps, rgb_p, w_p, offs)
    # both films hold warm-up + timed frames of the same estimates
    img_b, img_p = image(rgb_b, w_b), image(rgb_p, w_p)

    with BatchRenderer(accs, params_at(BATCH["ref_spp"], seed=BATCH["ref_seed"]), use_graph=1,
                       sort_key=tuned["sort_key"]) as rr:
        rgb_r = torch.zeros((pix, 3), device="cuda")
        w_r = torch.zeros((pix,), device="cuda")
        rr.render(rgb_r, w_r, stream=stream)
        torch.cuda.synchronize()
        ref = image(rgb_r, w_r)
        del rgb_r, w_r

    def relmse(img):
        per = [float(np.mean((img[offs[k]:offs[k + 1]] - ref[offs[k]:offs[k + 1]]) ** 2 /
                             (ref[offs[k]:offs[k + 1]] ** 2 + 1e-2))) for k in range(len(params))]
        return float(np.mean(per))

    rel32 = relmse(img_b)
    # relMSE falls as 1 / spp: the smallest power of two predicted to reach the
    # bar, then measured (doubled until it does)
    spp_bar = BATCH["spp"]
    while spp_bar * 2 <= 4096 and rel32 * BATCH["spp"] / spp_bar > BATCH["relmse_bar"]:
        spp_bar *= 2
    bar = None
    while bar is None or (bar["relmse"]["batched"] > BATCH["relmse_bar"] and spp_bar < 2048):
        if bar is not None:
            spp_bar *= 2
        pb = params_at(spp_bar)
        with BatchRenderer(accs, pb, wave_paths=tuned["wave_paths"], sort_key=tuned["sort_key"]) as bs:
            rgb_b.zero_()
            w_b.zero_()
            ms_bs = timed(lambda: bs.render(rgb_b, w_b, stream=stream), 2)
        rgb_p.zero_()
        w_p.zero_()
        ms_ps = plain_ms(pb, 1, rgb_p, w_p, offs)
        paths_s = sum(p.width * p.height * p.spp for p in pb)
        bar = {"spp": spp_bar, "paths_per_frame": paths_s, "batched_ms": ms_bs, "plain_ms": ms_ps,
               "batched_spp_per_s": paths_s / ms_bs * 1000.0, "plain_spp_per_s": paths_s / ms_ps * 1000.0,
               "relmse": {"batched": relmse(image(rgb_b, w_b)), "plain": relmse(image(rgb_p, w_p))}}

    for a in accs:
        a.close()
    tris = [h.triangle_count for h in hosts]
    return {"config": "%d scenes, triangles %d-%d (total %d), sides %s, %d spp, depth %d, roulette from bounce %d"
                      % (len(params), min(tris), max(tris), sum(tris), sorted(set(sides)),
                         BATCH["spp"], BATCH["max_depth"], BATCH["rr_min_bounce"]),
            "paths_per_frame": paths, "steps": steps, "setup_s": setup_s,
            "batched_spp_per_s": paths / ms_b * 1000.0, "batched_ms": ms_b,
            "plain_spp_per_s": paths / ms_p * 1000.0, "plain_ms": ms_p,
            "plain_timing": "sum over scenes of each scene's frame on its own graph-captured renderer",
            "autotuned": {"wave_paths": tuned["wave_paths"],
                          "sort_key": ["none", "material", "scene"][tuned["sort_key"]], "ms": tuned_ms},
            "reference": "%d-spp GPU render of every scene, Z-Sobol seed %d" % (BATCH["ref_spp"], BATCH["ref_seed"]),
            "relmse_at_%dspp" % BATCH["spp"]: {"batched": rel32, "plain": relmse(img_p)},
            "at_relmse_bar": bar, "relmse_bar": BATCH["relmse_bar"],
            "max_abs_diff_batched_vs_plain": float(np.nanmax(np.abs(img_b - img_p))),
            "error_word": err}


INSTANCED_MEDIUM = dict(box_min=(-10.0, -6.0, -10.0), box_max=(10.0, 6.0, 10.0), sigma_a=(0.05, 0.05, 0.05),
                        sigma_s=(0.2, 0.2, 0.2), g=0.0)


def instanced_leg(args, stream, barrier):
    """The two-level scene lit by an environment map: 16 displaced tubes and
    spheres of 50,000 triangles each, 4096 instances under seeded affine
    transforms, a 1024 x 512 sky map with a sun lobe, materials mixed per
    mesh (diffuse, coated diffuse, dielectric, conductor, coated conductor;
    roughness uniform in [0.05, 0.5]), one homogeneous medium box (sigma_a
    0.05, sigma_s 0.2, isotropic) around the middle of the instance field,
    1920 x 1080, 64 spp, depth 8 (MIS as written; roulette from bounce 2).
    One frame per step through a graph-captured renderer."""
    import torch

    from gonzales_b200 import GpuAccelerator, InstancedAccelerator, Renderer, scenes
    from gonzales_b200 import _ffi as F

    t0 = time.perf_counter()
    blas_hosts, inst = scenes.instanced_scene(mixed=True)
    blas = [GpuAccelerator(h) for h in blas_hosts]
    acc = InstancedAccelerator(blas, inst)
    acc.set_environment(scenes.sky_map(), 1.0)
    acc.set_medium(INSTANCED_MEDIUM)
    setup_s = time.perf_counter() - t0
    W, H, spp = 1920, 1080, 64
    p = F.render_params(W, H, spp, max_depth=8, rr_min_bounce=2, eye=(0.0, 6.0, 48.0), target=(0.0, 0.0, 0.0),
                        use_graph=1)
    rgb = torch.zeros((H, W, 3), device="cuda")
    w = torch.zeros((H, W), device="cuda")
    steps = max(1, min(args.steps, 2))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Renderer(acc, p) as r:
        r.render(rgb, w, stream=stream)
        barrier()
        s0 = r.stats()
        e0.record(stream)
        for _ in range(steps):
            r.render(rgb, w, stream=stream)
        e1.record(stream)
        barrier()
        s1 = r.stats()
    err = acc.error_word()
    acc.close()
    for b in blas:
        b.close()
    ms = e0.elapsed_time(e1) / steps
    rays = sum(s1[k] - s0[k] for k in ("camera_rays", "extension_rays", "shadow_rays", "probe_rays")) / steps
    return {"config": "16 x 50k-triangle meshes, 4096 instances, sky map 1024x512 + sun lobe, diffuse / "
                      "coated diffuse / dielectric / conductor / coated conductor meshes (roughness "
                      "U[0.05,0.5]), homogeneous medium box [-10,10]x[-6,6]x[-10,10] sigma_a 0.05 sigma_s 0.2, "
                      "%dx%d, %d spp, depth 8, roulette from bounce 2" % (W, H, spp),
            "spp_per_s": W * H * spp / ms * 1000.0, "ms_per_frame": ms, "mrays_per_s": rays / ms / 1000.0,
            "rays_per_frame": rays, "steps": steps, "setup_s": setup_s, "error_word": err}


def build_leg(hs, rays_d, args, stream, barrier):
    """The ray-cast mesh's tree built on the device (gzg_gpu_build_scene)
    against the host's SAH build: build times, surface-area costs of the two
    wide trees, and closest-hit Mrays/s on each (same rays)."""
    import os

    import torch

    from gonzales_b200 import GpuAccelerator, scene as S

    n = rays_d.shape[0]
    hits = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    bounds = np.concatenate([S.triangle_bounds(m) for m in hs.meshes])
    S.build_bvh2(bounds, threads)
    host_sah_s = time.perf_counter() - t0

    def timed(acc):
        for _ in range(3):
            acc.trace_closest(rays_d, hits)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        steps = max(3, min(args.steps, 10))
        e0.record(stream)
        for _ in range(steps):
            acc.trace_closest(rays_d, hits)
        e1.record(stream)
        barrier()
        return n / (e0.elapsed_time(e1) / steps) / 1e3

    t0 = time.perf_counter()
    up = GpuAccelerator(hs)
    upload_s = time.perf_counter() - t0
    host_rate, host_cost = timed(up), up.tree_cost()
    up.close()
    from gonzales_b200 import _ffi as F

    res = {}
    for builder, name in ((F.BUILD_PLOC, "ploc"), (F.BUILD_LBVH, "lbvh")):
        ms = []
        for _ in range(3):
            t0 = time.perf_counter()
            dev = GpuAccelerator(hs, device_build=True, builder=builder)
            wall = time.perf_counter() - t0
            ms.append(dev.build_time_ms())
            if len(ms) < 3:
                dev.close()
        res[name] = {"build_ms": min(ms), "wall_s": wall, "tree_cost": dev.tree_cost(),
                     "closest_mrays": timed(dev), "wide_nodes": dev.info()["wide_nodes"], "error_word": dev.error_word()}
        dev.close()
    # ingestion fast path: packed float x3 points and int32 indices straight
    # to the device expansion and build (gzg_gpu_build_mesh_scene)
    packed = [(m.points[:, :3].copy(), m.vertex_indices.reshape(-1, 3).astype(np.int32), 0) for m in hs.meshes]
    mats = hs.materials[:1].copy()
    fast = []
    for _ in range(3):
        t0 = time.perf_counter()
        acc_f = GpuAccelerator.from_mesh_arrays(packed, mats)
        fast.append(time.perf_counter() - t0)
        fast_ms = acc_f.build_time_ms()
        acc_f.close()
    return {"config": "ray-cast mesh, %d triangles; closest hit on the %d bench rays" % (hs.triangle_count, n),
            "device_ploc": res["ploc"], "device_lbvh": res["lbvh"], "host_sah_build_s": host_sah_s,
            "host_sah_threads": threads, "upload_with_host_tree_s": upload_s, "tree_cost_host_sah": host_cost,
            "closest_mrays_host_tree": host_rate, "packed_arrays_to_scene_wall_s": min(fast),
            "packed_arrays_build_ms": fast_ms}


def adjoint_leg(args, stream, barrier):
    """The differentiable box scene (floor and back-wall albedo textures
    256 x 256 x 3 each, emission scale; 393,217 parameters): one step is a
    256 x 256, 16-spp forward render plus the path-replay adjoint of an L2
    loss against a 1024-spp target (depth 5, no roulette)."""
    import torch

    from gonzales_b200 import GpuAccelerator
    from gonzales_b200 import _ffi as F
    from gonzales_b200 import adjoint as A

    sb, mats = A.adjoint_box_scene()
    acc = GpuAccelerator(sb.build())
    gt = torch.as_tensor(A.ground_truth_textures()).cuda()
    depth = 5
    with A.DifferentiableRenderer(acc, F.render_params(256, 256, 1024, max_depth=depth, rr_min_bounce=depth),
                                  mats) as dt:
        target, _ = dt.forward(gt, 1.0)
    tex = torch.full_like(gt, 0.5)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2 = torch.cuda.Event(enable_timing=True)
    steps = max(3, min(args.steps, 10))
    with A.DifferentiableRenderer(acc, F.render_params(256, 256, 16, max_depth=depth, rr_min_bounce=depth),
                                  mats) as dr:
        for _ in range(max(3, args.warmup)):
            img, w = dr.forward(tex, 0.8, stream=stream)
            dr.backward(2.0 * (img - target) / img.numel(), w, tex, 0.8, stream=stream)
        barrier()
        fwd_ms = bwd_ms = 0.0
        for _ in range(steps):
            e0.record(stream)
            img, w = dr.forward(tex, 0.8, stream=stream)
            e1.record(stream)
            d_tex, d_em = dr.backward(2.0 * (img - target) / img.numel(), w, tex, 0.8, stream=stream)
            e2.record(stream)
            e2.synchronize()
            fwd_ms += e0.elapsed_time(e1)
            bwd_ms += e1.elapsed_time(e2)
        barrier()
    acc.close()
    return {"config": "adjoint box scene, 2 x 256x256x3 albedo textures + emission scale (393,217 parameters), "
                      "256x256, 16 spp, depth 5, no roulette, L2 loss vs 1024-spp target",
            "forward_ms": fwd_ms / steps, "adjoint_ms": bwd_ms / steps, "step_ms": (fwd_ms + bwd_ms) / steps,
            "gradient_nonzero": int((d_tex != 0).sum().item()), "d_emission": float(d_em.item()),
            "paths_per_step": 256 * 256 * 16, "steps": steps}


def cpu_render_baseline():
    """The oracle integrator on all host threads, the same full frame."""
    from gonzales_b200 import scenes
    from oracle import pyoracle as O

    hs = scenes.box_scene().build()
    p = O.render_params(RENDER["width"], RENDER["height"], RENDER["spp"], max_depth=RENDER["max_depth"],
                        rr_min_bounce=RENDER["rr_min_bounce"])
    t0 = time.perf_counter()
    O.render(hs, p)
    el = time.perf_counter() - t0
    return RENDER["width"] * RENDER["height"] * RENDER["spp"] / el


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args):
    """The reference's CPU implementation of the path (the oracle: the
    restated Mojo traversal, BVH2 + Moller-Trumbore) on all host threads,
    over the full ray set each step.  Only rank 0 runs; the tree is built by
    the oracle, so libgzg.so is not loaded."""
    world, rank, local = dist_setup(args)
    if rank != 0:
        return 0
    from gonzales_b200 import scenes
    from oracle import pyoracle as O

    cfg, hs, o, d, t, name = oracle_workload(args.small)
    cores = os.cpu_count() or 1
    meshes = [(m.points, m.vertex_indices) for m in hs.meshes]
    r6 = scenes.pack_reference_rays(o, d)
    for _ in range(args.warmup):
        O.traverse(hs.nodes, hs.prims, meshes, r6, t, threads=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.traverse(hs.nodes, hs.prims, meshes, r6, t, threads=cores)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = len(t) * args.steps / total / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural mesh and rays)",
        "config": workload_config(cfg, hs, name, 1),
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": cores, "kind": "port",
                         "sample": "all %d rays per step, closest hit, oracle SAH BVH2 + Moller-Trumbore "
                                   "(CPU restatement of the reference traversal; the Swift/Mojo reference has no "
                                   "toolchain here)" % len(t)},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    from gonzales_b200 import GpuAccelerator, options, scenes
    from gonzales_b200 import _ffi as F

    cfg, hs, o, d, t, name = workload(args.small, rank)
    n = len(t)
    acc = GpuAccelerator(hs)
    info = acc.info()
    stream = torch.cuda.current_stream()
    rays_d = torch.from_numpy(scenes.pack_device_rays(o, d, t)).cuda()
    hits_d = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    anyp_d = torch.empty(n, dtype=torch.int32, device="cuda")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # launch autotuning on these rays (untimed setup): becomes the scene default
    tuned_closest, _ = acc.autotune(rays_d)
    tuned_any, _ = acc.autotune(rays_d, any_hit=True)

    # instrumented replay (untimed): node / triangle fetch counts per launch
    cnt = torch.zeros(3, dtype=torch.int64, device="cuda")
    acc.trace_closest(rays_d, hits_d, options(fetch_counters=cnt.data_ptr()))
    torch.cuda.synchronize()
    nodes_per_launch, tris_per_launch, rays_counted = [int(x) for x in cnt.cpu()]
    assert rays_counted == n, (rays_counted, n)
    # the same rays through the reference's own node order and layout (k_bvh2,
    # untimed): 32-byte BVH2 records fetched (one per iteration, two per
    # interior step) and triangle tests, for the reference-layout bytes
    from gonzales_b200._ffi import TRAVERSAL_BVH2
    cnt.zero_()
    acc.trace_closest(rays_d, hits_d, options(traversal=TRAVERSAL_BVH2, fetch_counters=cnt.data_ptr()))
    torch.cuda.synchronize()
    bvh2_records, bvh2_tris, _ = [int(x) for x in cnt.cpu()]

    for _ in range(args.warmup):
        acc.trace_closest(rays_d, hits_d)
    barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    with sampler:
        barrier()
        t_first = torch.cuda.Event(enable_timing=True)
        t_last = torch.cuda.Event(enable_timing=True)
        t_first.record(stream)
        for k in range(args.steps):
            starts[k].record(stream)
            acc.trace_closest(rays_d, hits_d)
            ends[k].record(stream)
        t_last.record(stream)
        barrier()
    elapsed_ms = t_first.elapsed_time(t_last)
    launch_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    if dist is not None:
        tt = torch.tensor([elapsed_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        elapsed_ms = float(tt.item())
    assert acc.error_word() == 0

    # any-hit (shadow) pass, same rays
    for _ in range(args.warmup):
        acc.trace_any(rays_d, anyp_d)
    barrier()
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(args.steps):
        acc.trace_any(rays_d, anyp_d)
    a1.record(stream)
    barrier()
    any_ms = a0.elapsed_time(a1) / args.steps

    # each half alone (coherent camera rays, incoherent rays): its own
    # instrumented replay, timed launches and roofline
    nc = cfg["width"] * cfg["height"]
    halves = {}
    for label, sl in (("coherent", slice(0, nc)), ("incoherent", slice(nc, n))):
        rh, hh = rays_d[sl], hits_d[sl]
        cnt.zero_()
        acc.trace_closest(rh, hh, options(fetch_counters=cnt.data_ptr()))
        torch.cuda.synchronize()
        h_nodes, h_tris, h_rays = [int(x) for x in cnt.cpu()]
        for _ in range(args.warmup):
            acc.trace_closest(rh, hh)
        barrier()
        hs_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                 for _ in range(args.steps)]
        for e_start, e_end in hs_ev:
            e_start.record(stream)
            acc.trace_closest(rh, hh)
            e_end.record(stream)
        barrier()
        halves[label] = dict(rays=h_rays, nodes=h_nodes, tris=h_tris,
                             launch_s=statistics.mean(a.elapsed_time(b) for a, b in hs_ev) / 1000.0)

    # end to end through the drop-in C-ABI call, pinned host buffers
    rays_h = torch.from_numpy(scenes.pack_reference_rays(o, d)).pin_memory()
    tmax_h = torch.from_numpy(t).pin_memory()
    out_h = torch.zeros(n * 48, dtype=torch.uint8).pin_memory()
    out_np = out_h.numpy().view(F.INTERSECTION_DTYPE)
    e2e_steps = max(3, min(args.steps, 10))
    for _ in range(2):
        acc.intersect_batch(rays_h.numpy(), tmax_h.numpy(), out=out_np)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        acc.intersect_batch(rays_h.numpy(), tmax_h.numpy(), out=out_np)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if dist is not None:
        tt = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    # the same through the compact-result call (16-byte hits back)
    hits_h = torch.zeros((n, 4), dtype=torch.float32).pin_memory()
    for _ in range(2):
        acc.intersect_batch_hits(rays_h.numpy(), tmax_h.numpy(), out=hits_h.numpy())
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        acc.intersect_batch_hits(rays_h.numpy(), tmax_h.numpy(), out=hits_h.numpy())
    e2e_compact_s = (time.perf_counter() - t0) / e2e_steps
    if dist is not None:
        tt = torch.tensor([e2e_compact_s], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_compact_s = float(tt.item())

    render = render_leg(acc_box=None, args=args, stream=stream, barrier=barrier) if not args.small else None
    build = build_leg(hs, rays_d, args, stream, barrier) if not (args.small or args.skip_batch) else None
    batch = batch_leg(args, stream, barrier) if not (args.small or args.skip_batch) else None
    adjoint = adjoint_leg(args, stream, barrier) if not (args.small or args.skip_batch) else None
    instanced = instanced_leg(args, stream, barrier) if not (args.small or args.skip_batch) else None

    if rank == 0:
        ms_per_step = elapsed_ms / args.steps
        value = world * n / (ms_per_step / 1000.0) / 1e6
        avg_launch_s = statistics.mean(launch_ms) / 1000.0
        alg_bytes = n * 48 + nodes_per_launch * 80 + tris_per_launch * 48
        peak, peak_kind = measured_hbm()
        achieved = alg_bytes / avg_launch_s / 1e9
        traffic = None
        prof = ROOT / "profiles" / "k_wide_closest_raycast.json"
        if prof.exists() and not args.small:
            traffic = json.loads(prof.read_text()).get("dram_bytes_per_full_launch")
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                    "kernel": "k_wide_persistent (closest hit)",
                    "bytes_per_ray": alg_bytes / n, "nodes_per_ray": nodes_per_launch / n,
                    "tris_per_ray": tris_per_launch / n}
        # ray I/O alone (32 B device ray in, 16 B hit out): the lower bound of any layout
        roofline["io_lower_bound"] = {"bytes_per_ray": 48, "achieved": 48.0 * n / avg_launch_s / 1e9,
                                      "frac": 48.0 * n / avg_launch_s / 1e9 / peak}
        # the reference's layout for the same rays: 32 B BVH2 records, 104 B per
        # triangle test (32 B PrimId_C + 24 B int64 indices + 3 x 16 B points),
        # 76 B of ray I/O (Ray_C + tMax in, Intersection_C out); bytes that the
        # kernel's time would have to move in that layout
        ref_bytes = 76.0 * n + 32.0 * bvh2_records + 104.0 * bvh2_tris
        roofline["reference_layout"] = {
            "bytes_per_ray": ref_bytes / n, "node_records_per_ray": bvh2_records / n,
            "tris_per_ray": bvh2_tris / n, "equivalent_gbs": ref_bytes / avg_launch_s / 1e9}
        for label, hv in halves.items():
            hb = hv["rays"] * 48 + hv["nodes"] * 80 + hv["tris"] * 48
            ach = hb / hv["launch_s"] / 1e9
            h_traffic = None
            if prof.exists() and not args.small:
                h_traffic = json.loads(prof.read_text()).get("dram_bytes_per_full_launch_" + label)
            roofline[label] = {"rays": hv["rays"], "mrays_per_s": hv["rays"] / hv["launch_s"] / 1e6,
                               "ms_per_launch": hv["launch_s"] * 1000.0, "achieved": ach, "frac": ach / peak,
                               "traffic": h_traffic, "bytes_per_ray": hb / hv["rays"],
                               "nodes_per_ray": hv["nodes"] / hv["rays"], "tris_per_ray": hv["tris"] / hv["rays"]}
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural mesh and rays)",
            "config": workload_config(cfg, hs, name, world),
            "method": {"traversal": "wide8", "wide_nodes": info["wide_nodes"], "wide_depth": info["wide_depth"],
                       "bvh2_nodes": info["bvh2_nodes"], "launch_closest": tuned_closest,
                       "launch_any": tuned_any},
            "any_hit_mrays_s": world * n / any_ms * 1000.0 / 1e6,
            "roofline": roofline,
            "e2e": {"value": world * n / e2e_s / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": n * 28,
                    "d2h_bytes_per_step": n * 48, "call": "gzg_gpu_traverse_batch (pinned host Ray_C + tMax -> "
                                                         "Intersection_C)"},
            "e2e_compact": {"value": world * n / e2e_compact_s / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": n * 28,
                            "d2h_bytes_per_step": n * 16,
                            "call": "gzg_gpu_traverse_batch_hits (pinned host Ray_C + tMax -> 16-byte hits)"},
            "gpu_launches": args.steps,  # closest-hit launches in the timed region of `value`
            "clocks": sampler.summary(),
        }
        if render is not None:
            line["render"] = render
        if batch is not None:
            line["batch"] = batch
        if adjoint is not None:
            line["adjoint"] = adjoint
        if instanced is not None:
            line["instanced"] = instanced
        if build is not None:
            line["device_build"] = build
        if world == 1 and not args.skip_cpu:
            line["cpu_baseline"] = cpu_baseline(args.small)
            if render is not None:
                line["cpu_baseline"]["render_spp_per_s"] = cpu_render_baseline()
        print(json.dumps(line), flush=True)
    acc.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_case(args):
    """Small single cases for profiler captures (one GPU):
      instanced-small  one 640 x 360, 16-spp frame of the two-level scene with
                       the general materials and the medium, in 2^20-path
                       waves (after one warm-up frame)
      build            the device tree build of the ray-cast mesh (three builds)
      render           one frame of the box scene (256 x 256, 16 spp, depth 5)
                       after three warm-up frames
      incoherent       the ray-cast mesh's 8,388,608 incoherent rays alone:
      coherent         or its 8,388,608 coherent rays alone,
      mixed            or all 16,777,216 rays (the bench's launch); tuned
                       launch, two warm-up closest-hit launches, then three
                       timed ones inside a profiler range (384 MiB or 768 MiB
                       of rays and hits on the device)"""
    import torch

    from gonzales_b200 import GpuAccelerator, InstancedAccelerator, Renderer, scenes
    from gonzales_b200 import _ffi as F

    torch.cuda.set_device(0)
    if args.case == "instanced-small":
        blas_hosts, inst = scenes.instanced_scene(mixed=True)
        blas = [GpuAccelerator(h) for h in blas_hosts]
        acc = InstancedAccelerator(blas, inst)
        acc.set_environment(scenes.sky_map(), 1.0)
        acc.set_medium(INSTANCED_MEDIUM)
        W, H, spp = 640, 360, 16
        # a 2^20-path wave (about 0.37 GB) keeps profiler captures small
        p = F.render_params(W, H, spp, max_depth=8, rr_min_bounce=2, eye=(0.0, 6.0, 48.0), target=(0.0, 0.0, 0.0),
                            use_graph=1, wave_paths=1 << 20)
        rgb = torch.zeros((H, W, 3), device="cuda")
        w = torch.zeros((H, W), device="cuda")
        with Renderer(acc, p) as r:
            r.render(rgb, w)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.profiler.start()  # the timed frame only, for --profile-from-start off
            e0.record()
            r.render(rgb, w)
            e1.record()
            torch.cuda.synchronize()
            torch.cuda.profiler.stop()
            stats = r.stats()
        out = {"case": args.case, "ms_per_frame": e0.elapsed_time(e1), "stats": stats, "error_word": acc.error_word()}
        acc.close()
        for b in blas:
            b.close()
    elif args.case == "render":
        hs = scenes.box_scene().build()
        with GpuAccelerator(hs) as acc_box:
            p = F.render_params(**RENDER, use_graph=1)
            rgb = torch.zeros((RENDER["height"], RENDER["width"], 3), device="cuda")
            w = torch.zeros((RENDER["height"], RENDER["width"]), device="cuda")
            with Renderer(acc_box, p) as r:
                for _ in range(3):
                    r.render(rgb, w)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                torch.cuda.profiler.start()  # the timed frame only, for --profile-from-start off
                e0.record()
                r.render(rgb, w)
                e1.record()
                torch.cuda.synchronize()
                torch.cuda.profiler.stop()
            out = {"case": args.case, "ms_per_frame": e0.elapsed_time(e1), "error_word": acc_box.error_word()}
    elif args.case in ("incoherent", "coherent", "mixed"):
        cfg, hs, o, d, t, name = workload(False, 0)
        nc = cfg["width"] * cfg["height"]
        sl = {"incoherent": slice(nc, len(t)), "coherent": slice(0, nc), "mixed": slice(0, len(t))}[args.case]
        rays = torch.from_numpy(scenes.pack_device_rays(o[sl], d[sl], t[sl])).cuda()
        hits = torch.empty((rays.shape[0], 4), dtype=torch.float32, device="cuda")
        with GpuAccelerator(hs) as acc:
            tuned, _ = acc.autotune(rays)
            for _ in range(2):
                acc.trace_closest(rays, hits)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            # the profiler range (cudaProfilerStart / Stop) holds only these
            # launches, for captures with --profile-from-start off
            torch.cuda.profiler.start()
            e0.record()
            for _ in range(3):
                acc.trace_closest(rays, hits)
            e1.record()
            torch.cuda.synchronize()
            torch.cuda.profiler.stop()
            ms = e0.elapsed_time(e1) / 3
            out = {"case": args.case, "rays": int(rays.shape[0]), "ms_per_launch": ms,
                   "mrays_per_s": rays.shape[0] / ms / 1e3, "launch": tuned, "error_word": acc.error_word()}
    else:
        hs = scenes.raycast_scene(subdiv=8).build()
        ms = []
        for _ in range(3):
            with GpuAccelerator(hs, device_build=True) as a:
                ms.append(a.build_time_ms())
        out = {"case": args.case, "device_build_ms": ms}
    print(json.dumps(out), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.case:
        return run_case(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
