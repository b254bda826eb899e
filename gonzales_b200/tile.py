"""Host-side mirror of Gonzales' tile loop over the drop-in calls.

In the reference, TileRenderer (Core/TileRenderer.swift:77-109) runs
Tile.render (Core/Tile.swift:19-223) per tile: phase 1 generates one camera ray
per pixel sample (Tile.swift:27-59); phase 2 runs up to maxDepth + 1 rounds of
one batch trace through the native plugin (mojo_gpu_traverse_batch,
Tile.swift:82-97; tMax stays infinite because PathState.tHit is never
updated) and one batch shade (mojo_gpu_shade_batch, Tile.swift:137-155, with
fresh PCG32 seeds per path and bounce drawn from the integrator's xoshiro
generator, Tile.swift:122-123); every path ends as one Sample of its estimate
and ray weight, which Film.add accumulates into its pixel (Core/Film.swift:
107-119, Pixel sums of light and weight, Core/Pixel.swift:12-16).

Here the same loop calls libgzg's replacements: gzg_camera_rays (phase 1 on
the device), gzg_gpu_traverse_batch and gzg_gpu_shade_batch.  The PCG seeds
come from a seeded numpy generator (the reference's are system-seeded, so its
renders are not reproducible).  The film sums are accumulated on the host as
Film.add does.  There is no CPU fallback: every call goes through libgzg.
"""
import ctypes as C

import numpy as np

from . import _ffi as F


def camera_rays(params, first, count):
    """Camera rays of paths [first, first + count) of the frame in params
    (gzg_camera_rays): (rays (n, 6) float32 Ray_C, weights (n,) float32,
    pixels (n,) int32: the film pixel, (y - y0) * film width + (x - x0) within
    the crop window, y * width + x without one)."""
    rays = np.zeros((count, 6), np.float32)
    w = np.zeros(count, np.float32)
    px = np.zeros(count, np.int32)
    if count:
        F.check(F.lib().gzg_camera_rays(C.byref(params), int(first), int(count), F.ptr(rays), F.ptr(w), F.ptr(px)))
    return rays, w, px


def render_tile_loop(accel, params, seed=0, batch_paths=1 << 20, iso=100.0, max_component=0.0):
    """Renders the frame of `params` (width, height, spp, max_depth, camera,
    filter) with the reference's live bounce loop on `accel` (a
    GpuAccelerator of a scene uploaded with materials).  Paths run in batches
    of batch_paths (the reference sizes GPU tiles for about 1e6 rays per batch,
    Api/RenderConfiguration.swift:208-211).  Returns the film sums
    (light (H, W, 3) float64, weight (H, W) float64) and per-bounce counts of
    the rays traced."""
    W, H, spp = params.film_width, params.film_height, params.spp
    total = W * H * spp
    rng = np.random.Generator(np.random.PCG64(seed))
    light = np.zeros((H * W, 3), np.float64)
    weight = np.zeros(H * W, np.float64)
    traced = np.zeros(params.max_depth + 1, np.int64)
    scale = iso / 100.0
    for first in range(0, total, batch_paths):
        n = min(batch_paths, total - first)
        rays, w, pixel = camera_rays(params, first, n)
        paths = np.zeros(n, F.PATH_STATE_DTYPE)
        paths["ray"] = rays.view(F.RAY_DTYPE).reshape(-1)
        paths["throughput"] = 1.0
        live = np.arange(n)
        for bounce in range(params.max_depth + 1):
            if len(live) == 0:
                break
            traced[bounce] += len(live)
            state = paths[live]
            isect = accel.intersect_batch(state["ray"], np.full(len(live), np.inf, np.float32))
            state["pcg_state"] = rng.integers(0, 2 ** 64, len(live), dtype=np.uint64, endpoint=False)
            state["pcg_inc"] = rng.integers(0, 2 ** 64, len(live), dtype=np.uint64, endpoint=False)
            state["active"] = 1
            accel.shade_batch(state, isect)
            paths[live] = state
            live = live[state["active"] != 0]
        # Film.add: light scaled by iso / 100, optional clamp of the largest
        # component, then the pixel's light and weight sums
        est = paths["estimate"].astype(np.float64) * scale
        if max_component > 0:
            mv = est.max(1)
            over = mv > max_component
            est[over] *= (max_component / mv[over])[:, None]
        np.add.at(light, pixel, est)
        np.add.at(weight, pixel, w.astype(np.float64))
    return light.reshape(H, W, 3), weight.reshape(H, W), traced


def normalized(light, weight):
    """Pixel.normalized (Core/Pixel.swift:12-16): light / weight, and a black
    pixel stays black whatever its weight."""
    black = np.all(light == 0, axis=-1)
    out = np.zeros_like(light)
    ok = ~black
    out[ok] = light[ok] / weight[ok][:, None]
    return out
