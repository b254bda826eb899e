"""GPU accelerator: the host-facing mirror of Gonzales' Accelerator
(Sources/libgonzales/Accelerators/Accelerator.swift) on its GPU path.

  Accelerator.uploadToGPU      -> GpuAccelerator(host_scene)     (gzg_gpu_upload_scene)
  intersectBatchGPU            -> intersect_batch(rays, tmax)    (gzg_gpu_traverse_batch)
  Visibility.occluded          -> occluded_batch(rays, tmax)     (gzg_gpu_occluded_batch)
  BoundingHierarchy.deinit     -> close() / context manager      (gzg_gpu_free_scene)

plus device-resident calls on torch CUDA tensors (trace_closest / trace_any).
Rays on the host are Ray_C records (RAY_DTYPE or an (n, 6) float32 array);
device rays are (n, 8) float32 tensors: origin, tMax, direction, unused.
"""
import ctypes as C

import numpy as np

from . import _ffi as F
from .scene import HostScene


def gpu_available():
    return bool(F.lib().gzg_gpu_available())


def _host_rays(rays):
    rays = np.ascontiguousarray(rays)
    if rays.dtype == F.RAY_DTYPE:
        return rays
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
    return rays


def _set_medium(handle, medium):
    """gzg_scene_set_medium from a dict(box_min, box_max, sigma_a, sigma_s,
    g) or None (removes the medium)."""
    if medium is None:
        F.check(F.lib().gzg_scene_set_medium(handle, None))
        return
    m = F.Medium((C.c_float * 3)(*medium["box_min"]), (C.c_float * 3)(*medium["box_max"]),
                 (C.c_float * 3)(*medium["sigma_a"]), (C.c_float * 3)(*medium["sigma_s"]),
                 float(medium.get("g", 0.0)), 0)
    F.check(F.lib().gzg_scene_set_medium(handle, C.byref(m)))


def _stream_handle(stream):
    if stream is None:
        import torch

        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


class GpuAccelerator:
    def __init__(self, host_scene: HostScene, device_build=None, leaf_size=0, builder=0, radius=0):
        """Uploads the scene with the host's BVH2 (gzg_gpu_upload_scene), or
        builds its tree on the device (gzg_gpu_build_scene) when device_build
        is true or the scene has no BVH2 (SceneBuilder.build(host_bvh=False))."""
        self.host = host_scene
        meshes = host_scene.mesh_structs()
        pts, fi, vi = host_scene.counts()
        handle = C.c_void_p()
        if device_build is None:
            device_build = host_scene.nodes is None
        self.device_built = bool(device_build)
        if self.device_built:
            opt = F.BuildOptions()
            opt.leaf_size = int(leaf_size)
            opt.builder = int(builder)
            opt.radius = int(radius)
            F.check(F.lib().gzg_gpu_build_scene(
                F.ptr(host_scene.prims), len(host_scene.prims), C.addressof(meshes), len(host_scene.meshes),
                F.ptr(pts), F.ptr(fi), F.ptr(vi), F.ptr(host_scene.materials), len(host_scene.materials),
                C.byref(opt), C.byref(handle)))
        else:
            F.check(F.lib().gzg_gpu_upload_scene(
                F.ptr(host_scene.nodes), len(host_scene.nodes), F.ptr(host_scene.prims), len(host_scene.prims),
                C.addressof(meshes), len(host_scene.meshes), F.ptr(pts), F.ptr(fi), F.ptr(vi),
                F.ptr(host_scene.materials), len(host_scene.materials), C.byref(handle)))
        self.handle = handle
        try:
            if getattr(host_scene, "has_extended_materials", False) and host_scene.material_params is not None:
                self.set_material_params(host_scene.material_params)
            for k, m in enumerate(host_scene.meshes):
                if getattr(m, "normals", None) is not None or getattr(m, "uvs", None) is not None:
                    self.set_vertex_attributes(k, m.normals, m.uvs)
        except Exception:
            self.close()
            raise

    @classmethod
    def from_mesh_arrays(cls, meshes, materials, leaf_size=0, builder=0, radius=0):
        """The ingestion fast path (gzg_gpu_build_mesh_scene): meshes is a list
        of (points (n, 3) float32, indices (m, 3) int32, material index[,
        normals (n, 3) or None[, uvs (n, 2) or None]]); materials a
        MATERIAL_DTYPE array.  Prim k of the scene is triangle k in mesh order
        (id2 = mesh << 32 | triangle)."""
        self = cls.__new__(cls)
        keep = []
        arr = (F.MeshArrays * max(len(meshes), 1))()
        for k, entry in enumerate(meshes):
            pts, idx, mat = entry[:3]
            pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
            idx = np.ascontiguousarray(idx, np.int32).reshape(-1, 3)
            keep += [pts, idx]
            arr[k] = F.MeshArrays(pts.ctypes.data if len(pts) else None, len(pts),
                                  idx.ctypes.data if len(idx) else None, len(idx), int(mat))
        materials = np.ascontiguousarray(materials)
        opt = F.BuildOptions()
        opt.leaf_size = int(leaf_size)
        opt.builder = int(builder)
        opt.radius = int(radius)
        handle = C.c_void_p()
        F.check(F.lib().gzg_gpu_build_mesh_scene(C.addressof(arr), len(meshes), F.ptr(materials), len(materials),
                                                 C.byref(opt), C.byref(handle)))
        self.handle = handle
        self.device_built = True
        self.host = _ArraysHost(meshes, materials)
        try:
            for k, entry in enumerate(meshes):
                nrm = entry[3] if len(entry) > 3 else None
                uv = entry[4] if len(entry) > 4 else None
                if nrm is not None or uv is not None:
                    self.set_vertex_attributes(k, nrm, uv)
        except Exception:
            self.close()
            raise
        return self

    # ------------------------------------------------------------ lifetime
    def close(self):
        if self.handle:
            F.check(F.lib().gzg_gpu_free_scene(self.handle))
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ queries
    def info(self):
        info = F.SceneInfo()
        F.check(F.lib().gzg_scene_info_get(self.handle, C.byref(info)))
        return {name: getattr(info, name) for name, _ in F.SceneInfo._fields_}

    def error_word(self, clear=True):
        w = C.c_uint32(0)
        F.check(F.lib().gzg_scene_error_word(self.handle, C.byref(w), 1 if clear else 0))
        return w.value

    def build_time_ms(self):
        """Device time of the tree build (gzg_scene_build_time); -1 if uploaded."""
        ms = C.c_float(0.0)
        F.check(F.lib().gzg_scene_build_time(self.handle, C.byref(ms)))
        return ms.value

    def tree_cost(self):
        """Surface-area cost of the wide tree (gzg_scene_tree_cost)."""
        c = C.c_double(0.0)
        F.check(F.lib().gzg_scene_tree_cost(self.handle, C.byref(c)))
        return c.value

    def intersect_batch(self, rays, tmax, options=None, out=None):
        """Closest hit for host rays; returns INTERSECTION_DTYPE records."""
        rays = _host_rays(rays)
        tmax = np.ascontiguousarray(tmax, dtype=np.float32)
        n = len(tmax)
        if out is None:
            out = np.zeros(n, F.INTERSECTION_DTYPE)
        opt = C.byref(options) if options is not None else None
        F.check(F.lib().gzg_gpu_traverse_batch(self.handle, F.ptr(rays), F.ptr(tmax), n, F.ptr(out), opt))
        return out

    def intersect_batch_hits(self, rays, tmax, options=None, out=None):
        """Closest hit for host rays with compact results
        (gzg_gpu_traverse_batch_hits): (n, 4) float32 rows t, u, v, prim
        (prim as int32 bits: index into the prim-id array, -1 on a miss)."""
        rays = _host_rays(rays)
        tmax = np.ascontiguousarray(tmax, dtype=np.float32)
        n = len(tmax)
        if out is None:
            out = np.zeros((n, 4), np.float32)
        opt = C.byref(options) if options is not None else None
        F.check(F.lib().gzg_gpu_traverse_batch_hits(self.handle, F.ptr(rays), F.ptr(tmax), n, F.ptr(out), opt))
        return out

    def occluded_batch(self, rays, tmax, options=None, out=None):
        rays = _host_rays(rays)
        tmax = np.ascontiguousarray(tmax, dtype=np.float32)
        n = len(tmax)
        if out is None:
            out = np.zeros(n, np.uint8)
        opt = C.byref(options) if options is not None else None
        F.check(F.lib().gzg_gpu_occluded_batch(self.handle, F.ptr(rays), F.ptr(tmax), n, F.ptr(out), opt))
        return out

    def trace_closest(self, rays_d, hits_d, options=None, stream=None):
        """rays_d: (n, 8) float32 CUDA tensor; hits_d: (n, 4) float32 CUDA tensor
        receiving (t, u, v, prim-as-int32-bits)."""
        n = rays_d.shape[0]
        opt = C.byref(options) if options is not None else None
        F.check(F.lib().gzg_trace_closest_device(self.handle, rays_d.data_ptr(), n, hits_d.data_ptr(), opt,
                                                 _stream_handle(stream)))

    def trace_any(self, rays_d, hit_prim_d, options=None, stream=None):
        n = rays_d.shape[0]
        opt = C.byref(options) if options is not None else None
        F.check(F.lib().gzg_trace_any_device(self.handle, rays_d.data_ptr(), n, hit_prim_d.data_ptr(), opt,
                                             _stream_handle(stream)))

    def hits_to_intersections(self, hits_d, out_d, stream=None):
        F.check(F.lib().gzg_hits_to_intersections_device(self.handle, hits_d.data_ptr(), hits_d.shape[0],
                                                         out_d.data_ptr(), _stream_handle(stream)))

    def autotune(self, rays_d, any_hit=False, stream=None):
        """gzg_scene_autotune on device rays; returns (launch config dict, ms per launch)."""
        best = F.TraceOptions()
        ms = C.c_float(0.0)
        F.check(F.lib().gzg_scene_autotune(self.handle, rays_d.data_ptr(), rays_d.shape[0], 1 if any_hit else 0,
                                           C.byref(best), C.byref(ms), _stream_handle(stream)))
        cfg = {k: getattr(best, k) for k in ("block_size", "blocks_per_sm", "stack_depth", "l1_carveout")}
        return cfg, ms.value

    def set_launch(self, cfg, any_hit=False):
        opt = F.options(**cfg)
        F.check(F.lib().gzg_scene_set_launch(self.handle, 1 if any_hit else 0, C.byref(opt)))

    def tune_cached(self, rays_d, cache_path, key, any_hit=False):
        """Tuned launch from a JSON cache (keyed by GPU name, `key` and query
        kind) or, on a miss, from gzg_scene_autotune, written back to the cache."""
        import json
        import os

        import torch

        full_key = "%s|%s|%s" % (torch.cuda.get_device_name(), key, "any" if any_hit else "closest")
        cache = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                cache = json.load(f)
        if full_key in cache:
            self.set_launch(cache[full_key]["launch"], any_hit)
            return cache[full_key]["launch"], cache[full_key]["ms"], True
        cfg, ms = self.autotune(rays_d, any_hit)
        if cache_path:
            cache[full_key] = {"launch": cfg, "ms": ms}
            tmp = cache_path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(cache, f, indent=1, sort_keys=True)
            os.replace(tmp, cache_path)
        return cfg, ms, False

    def shade_batch(self, paths, intersections):
        """gzg_gpu_shade_batch on PATH_STATE_DTYPE records (updated in place)."""
        assert paths.dtype == F.PATH_STATE_DTYPE and intersections.dtype == F.INTERSECTION_DTYPE
        F.check(F.lib().gzg_gpu_shade_batch(self.handle, F.ptr(paths), len(paths), F.ptr(intersections)))
        return paths

    def render(self, params):
        """Renders on the device (gzg_render_image); returns host film sums
        (rgb (H, W, 3), squares (H, W, 3), weights (H, W)) and statistics."""
        W, H = params.film_width, params.film_height
        rgb = np.zeros((H, W, 3), np.float32)
        sq = np.zeros((H, W, 3), np.float32)
        w = np.zeros((H, W), np.float32)
        stats = F.RenderStats()
        F.check(F.lib().gzg_render_image(self.handle, C.byref(params), F.ptr(rgb), F.ptr(sq), F.ptr(w),
                                         C.byref(stats)))
        return rgb, sq, w, {name: getattr(stats, name) for name, _ in F.RenderStats._fields_}

    def set_vertex_attributes(self, mesh, normals=None, uvs=None):
        """Vertex normals (n, 3) and / or UVs (n, 2) of mesh `mesh`
        (gzg_scene_set_vertex_attributes); a HostScene's meshes set theirs on
        upload."""
        nrm = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        uv = None if uvs is None else np.ascontiguousarray(uvs, np.float32).reshape(-1, 2)
        n = len(nrm) if nrm is not None else len(uv)
        F.check(F.lib().gzg_scene_set_vertex_attributes(self.handle, int(mesh),
                                                        F.ptr(nrm) if nrm is not None else None,
                                                        F.ptr(uv) if uv is not None else None, n))

    def set_material_params(self, params):
        """Parameters of the dielectric, coated-diffuse, conductor and
        coated-conductor materials (gzg_scene_set_material_params):
        (n_materials, 12) float32 gzg_material_params rows.  A HostScene with
        such materials sets them on upload."""
        params = np.ascontiguousarray(params, np.float32).reshape(-1, 12)
        F.check(F.lib().gzg_scene_set_material_params(self.handle, F.ptr(params), len(params)))

    def set_environment(self, rgb, scale=1.0):
        """Adds the environment light (gzg_scene_set_environment): rgb (H, W, 3)
        float32 in the equal-area square layout."""
        rgb = np.ascontiguousarray(rgb, np.float32)
        F.check(F.lib().gzg_scene_set_environment(self.handle, F.ptr(rgb), rgb.shape[1], rgb.shape[0], float(scale)))

    def set_medium(self, medium):
        """Sets the homogeneous medium box (gzg_scene_set_medium):
        dict(box_min, box_max, sigma_a, sigma_s, g), or None to remove it."""
        _set_medium(self.handle, medium)


class _ArraysHost:
    """What the Python side reads of a scene built from mesh arrays."""

    def __init__(self, meshes, materials):
        # bounds of the vertices (a superset of the triangles' when some
        # vertices are unreferenced: still a valid instance bound)
        pts = [np.asarray(e[0], np.float32).reshape(-1, 3) for e in meshes]
        pts = [p for p in pts if len(p)]
        self._lo = np.min([p.min(0) for p in pts], 0) if pts else np.zeros(3, np.float32)
        self._hi = np.max([p.max(0) for p in pts], 0) if pts else np.zeros(3, np.float32)
        self.materials = materials
        self.nodes = None
        self.has_extended_materials = False

    def root_bounds(self):
        return self._lo, self._hi


def instance_bounds(blas_hosts, instances):
    """World bounds per instance (gzg_host_instance_bounds) from the bottom-level
    BVH2 root boxes."""
    bb = np.zeros((len(blas_hosts), 6), np.float32)
    for i, hs in enumerate(blas_hosts):
        bb[i, :3], bb[i, 3:] = hs.root_bounds()
    instances = np.ascontiguousarray(instances, F.INSTANCE_DTYPE)
    out = np.zeros((len(instances), 6), np.float32)
    F.check(F.lib().gzg_host_instance_bounds(F.ptr(bb), len(bb), F.ptr(instances), len(instances), F.ptr(out)))
    return out


class InstancedAccelerator:
    """A two-level scene (TransformedPrimitive, Primitive/TransformedPrimitive.swift):
    bottom-level GpuAccelerators, instances (INSTANCE_DTYPE) and a top-level
    SAH BVH2 the host builds over the instance bounds."""

    def __init__(self, blas_accels, instances):
        from .scene import build_bvh2

        self.blas = list(blas_accels)
        self.instances = np.ascontiguousarray(instances, F.INSTANCE_DTYPE)
        handles = (C.c_void_p * len(self.blas))(*[a.handle.value for a in self.blas])
        # the top-level tree over the instances' bounds from their bottom-level
        # trees (gzg_host_instance_bounds_from_scenes), as the scene uses them
        self.bounds = np.zeros((len(self.instances), 6), np.float32)
        F.check(F.lib().gzg_host_instance_bounds_from_scenes(handles, len(self.blas), F.ptr(self.instances),
                                                             len(self.instances), F.ptr(self.bounds)))
        self.tlas_nodes, self.leaf_instance = build_bvh2(self.bounds)
        h = C.c_void_p()
        F.check(F.lib().gzg_instanced_scene_create(handles, len(self.blas), F.ptr(self.instances),
                                                   len(self.instances), F.ptr(self.tlas_nodes),
                                                   len(self.tlas_nodes), F.ptr(self.leaf_instance),
                                                   len(self.leaf_instance), C.byref(h)))
        self.handle = h

    def close(self):
        if self.handle:
            F.check(F.lib().gzg_gpu_free_scene(self.handle))
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        info = F.SceneInfo()
        F.check(F.lib().gzg_scene_info_get(self.handle, C.byref(info)))
        return {name: getattr(info, name) for name, _ in F.SceneInfo._fields_}

    def error_word(self, clear=True):
        w = C.c_uint32(0)
        F.check(F.lib().gzg_scene_error_word(self.handle, C.byref(w), 1 if clear else 0))
        return w.value

    render = GpuAccelerator.render
    set_environment = GpuAccelerator.set_environment
    set_medium = GpuAccelerator.set_medium

    def trace_closest(self, rays_d, hits_d, inst_d, options=None, stream=None):
        opt = C.byref(options) if options is not None else None
        F.check(F.lib().gzg_trace_closest_instanced_device(self.handle, rays_d.data_ptr(), rays_d.shape[0],
                                                           hits_d.data_ptr(), inst_d.data_ptr(), opt,
                                                           _stream_handle(stream)))

    def trace_any(self, rays_d, hit_prim_d, options=None, stream=None):
        opt = C.byref(options) if options is not None else None
        F.check(F.lib().gzg_trace_any_device(self.handle, rays_d.data_ptr(), rays_d.shape[0], hit_prim_d.data_ptr(),
                                             opt, _stream_handle(stream)))

    def autotune(self, rays_d, any_hit=False, stream=None):
        best = F.TraceOptions()
        ms = C.c_float(0.0)
        F.check(F.lib().gzg_scene_autotune(self.handle, rays_d.data_ptr(), rays_d.shape[0], 1 if any_hit else 0,
                                           C.byref(best), C.byref(ms), _stream_handle(stream)))
        return {k: getattr(best, k) for k in ("block_size", "blocks_per_sm", "stack_depth", "l1_carveout")}, ms.value


class Renderer:
    """A wavefront renderer bound to one scene (gzg_renderer_*); renders into
    caller-owned device films (torch CUDA tensors)."""

    def __init__(self, accel, params):
        self.accel = accel
        self.params = params
        h = C.c_void_p()
        F.check(F.lib().gzg_renderer_create(accel.handle, C.byref(params), C.byref(h)))
        self.handle = h

    def render(self, film_rgb, film_w, film_sq=None, stream=None, film_albedo=None, film_normal=None):
        if film_albedo is None and film_normal is None:
            F.check(F.lib().gzg_renderer_render(self.handle, film_rgb.data_ptr(),
                                                film_sq.data_ptr() if film_sq is not None else None,
                                                film_w.data_ptr(), _stream_handle(stream)))
            return
        F.check(F.lib().gzg_renderer_render_aov(self.handle, film_rgb.data_ptr(),
                                                film_sq.data_ptr() if film_sq is not None else None,
                                                film_w.data_ptr(),
                                                film_albedo.data_ptr() if film_albedo is not None else None,
                                                film_normal.data_ptr() if film_normal is not None else None,
                                                _stream_handle(stream)))

    def set_film(self, iso=100.0, max_component=0.0):
        """Film.add settings: light scaled by iso / 100, optional clamp."""
        F.check(F.lib().gzg_renderer_set_film(self.handle, float(iso), float(max_component)))

    def stats(self):
        s = F.RenderStats()
        F.check(F.lib().gzg_renderer_stats(self.handle, C.byref(s)))
        return {name: getattr(s, name) for name, _ in F.RenderStats._fields_}

    def close(self):
        if self.handle:
            F.check(F.lib().gzg_renderer_destroy(self.handle))
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchRenderer(Renderer):
    """One renderer over many scenes (gzg_batch_renderer_create).  Scene k's
    image is the window film[offsets[k]:offsets[k+1]] of one batch film;
    `split` cuts a batch film into per-scene (H, W, ...) views."""

    def __init__(self, accels, params, wave_paths=0, use_graph=1, sort_key=F.SORT_NONE):
        self.accels = list(accels)
        self.params = list(params)
        if len(self.accels) != len(self.params) or not self.accels:
            raise ValueError("BatchRenderer: one params record per scene, at least one scene")
        self.handle = C.c_void_p()
        handles = (C.c_void_p * len(self.accels))(*[a.handle.value for a in self.accels])
        prm = (F.RenderParams * len(self.params))(*self.params)
        self.options = F.BatchOptions(wave_paths, use_graph, sort_key, 0)
        h = C.c_void_p()
        F.check(F.lib().gzg_batch_renderer_create(handles, prm, len(self.accels), C.byref(self.options),
                                                  C.byref(h)))
        self.handle = h
        offs = (C.c_int64 * (len(self.accels) + 1))()
        F.check(F.lib().gzg_renderer_film_layout(self.handle, offs))
        self.offsets = list(offs)

    @property
    def pixels(self):
        """Pixel count of the batch film."""
        return self.offsets[-1]

    def split(self, film):
        """Per-scene (H, W, ...) views of a batch film (pixels first)."""
        out = []
        for k, p in enumerate(self.params):
            part = film[self.offsets[k]:self.offsets[k + 1]]
            out.append(part.reshape((p.film_height, p.film_width) + tuple(part.shape[1:])))
        return out

    def autotune(self, stream=None):
        """Times renders over wave sizes and sort keys; keeps and returns the
        fastest (options dict, ms per render)."""
        best = F.BatchOptions()
        ms = C.c_float()
        F.check(F.lib().gzg_renderer_autotune(self.handle, C.byref(best), C.byref(ms), _stream_handle(stream)))
        self.options = best
        return {name: getattr(best, name) for name, _ in F.BatchOptions._fields_}, ms.value

    def error_word(self, clear=True):
        w = C.c_uint32()
        F.check(F.lib().gzg_renderer_error_word(self.handle, C.byref(w), int(clear)))
        return w.value
