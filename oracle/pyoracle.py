"""ctypes wrapper of liboracle.so, the CPU restatement of the Gonzales hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and bench.py's
CPU-baseline leg, as the checker.  The product library never uses it.
"""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SOBOL = HERE.parent / "gonzales_b200" / "data" / "sobol_1024x52.bin"

NODE_DTYPE = np.dtype({"names": ["bounds_min", "bounds_max", "offset", "count"],
                       "formats": [("<f4", 3), ("<f4", 3), "<i4", "<i4"], "offsets": [0, 12, 24, 28], "itemsize": 32})
PRIM_DTYPE = np.dtype({"names": ["id1", "id2", "material_index", "type"], "formats": ["<i8", "<i8", "<i8", "i1"],
                       "offsets": [0, 8, 16, 24], "itemsize": 32})
ISECT_DTYPE = np.dtype({"names": ["prim_id", "t_hit", "u", "v", "hit"],
                        "formats": [PRIM_DTYPE, "<f4", "<f4", "<f4", "i1"], "offsets": [0, 32, 36, 40, 44],
                        "itemsize": 48})


class _Mesh(C.Structure):
    _fields_ = [("points", C.c_void_p), ("face_indices", C.c_void_p), ("vertex_indices", C.c_void_p),
                ("normals", C.c_void_p), ("uvs", C.c_void_p)]


def _render_mesh(m, keep):
    """An orc_mesh for the renderer, with the mesh's vertex normals / UVs when it has them."""
    p4 = np.ascontiguousarray(m.points, np.float32)
    vi = np.ascontiguousarray(m.vertex_indices, np.int64)
    keep += [p4, vi]
    nrm = uvs = None
    if getattr(m, "normals", None) is not None:
        nrm = np.ascontiguousarray(m.normals, np.float32)
        keep.append(nrm)
    if getattr(m, "uvs", None) is not None:
        uvs = np.ascontiguousarray(m.uvs, np.float32)
        keep.append(uvs)
    return _Mesh(p4.ctypes.data, None, vi.ctypes.data, nrm.ctypes.data if nrm is not None else None,
                 uvs.ctypes.data if uvs is not None else None)


class ZSobolState(C.Structure):
    _fields_ = [("seed", C.c_int64), ("log2spp", C.c_int32), ("n_base4_digits", C.c_int32),
                ("morton_index", C.c_uint64), ("dimension", C.c_int32)]


_lib = None


def build():
    src = list(HERE.glob("*.cpp")) + [HERE / "oracle.h", HERE / "Makefile"]
    if not LIB.exists() or any(p.stat().st_mtime > LIB.stat().st_mtime for p in src):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        vp, i64, f32, i32, u32, u64 = C.c_void_p, C.c_int64, C.c_float, C.c_int32, C.c_uint32, C.c_uint64
        sig = {
            "orc_triangle_bounds": (None, [vp, vp, i64, vp]),
            "orc_build_bvh2": (i64, [vp, i64, vp, vp]),
            "orc_traverse_batch": (None, [vp, vp, vp, vp, vp, i64, C.c_int, vp, vp, vp, C.c_int]),
            "orc_intersect_triangle_mt": (C.c_int, [vp, vp, vp, vp, vp, f32, vp, vp, vp]),
            "orc_intersect_triangle_watertight": (C.c_int, [vp, vp, vp, vp, vp, vp, vp, vp, vp]),
            "orc_intersect_aabb": (C.c_int, [vp, vp, vp, vp, f32, vp]),
            "orc_bounds_intersects_swift": (C.c_int, [vp, vp, vp, vp, f32]),
            "orc_bounds_surface_area": (f32, [vp, vp]),
            "orc_bounds_maximum_extent": (C.c_int, [vp, vp]),
            "orc_sobol_set_matrices": (None, [vp]),
            "orc_reverse_bits32": (u32, [u32]),
            "orc_encode_morton2": (u64, [u32, u32]),
            "orc_mix_bits": (u32, [u64]),
            "orc_owen_scramble": (u32, [u32, u32]),
            "orc_next_power_of_two": (i64, [i64]),
            "orc_sobol_sample": (f32, [i64, C.c_int, u32]),
            "orc_zsobol_init": (None, [vp, i64, i32, i32, i64]),
            "orc_zsobol_start_pixel_sample": (None, [vp, i32, i32, i64, i32]),
            "orc_zsobol_sample_index": (u64, [vp]),
            "orc_zsobol_get1d": (f32, [vp]),
            "orc_zsobol_get2d": (None, [vp, vp]),
            "orc_zsobol_get3d": (None, [vp, vp]),
            "orc_zsobol_batch": (None, [i64, i32, i32, i64, vp, vp, vp, i64, vp, i32, vp]),
            "orc_power_heuristic": (f32, [f32, f32]),
            "orc_concentric_disk": (None, [f32, f32, vp]),
            "orc_cosine_hemisphere": (None, [f32, f32, vp]),
            "orc_offset_origin": (None, [vp, vp, vp, vp]),
            "orc_spawn_to": (f32, [vp, vp, vp, vp]),
            "orc_gaussian": (f32, [f32, f32]),
            "orc_gaussian_sample_1d": (None, [f32, f32, f32, vp, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        m = np.fromfile(SOBOL, dtype="<u4")
        L.orc_sobol_set_matrices(m.ctypes.data)
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def triangle_bounds(points4, vertex_indices):
    points4 = np.ascontiguousarray(points4, np.float32)
    vi = np.ascontiguousarray(vertex_indices, np.int64)
    n = len(vi) // 3
    out = np.empty((n, 6), np.float32)
    lib().orc_triangle_bounds(_p(points4), _p(vi), n, _p(out))
    return out


def build_bvh2(bounds6):
    bounds6 = np.ascontiguousarray(bounds6, np.float32)
    n = len(bounds6)
    nodes = np.zeros(max(2 * n, 1), NODE_DTYPE)
    order = np.zeros(max(n, 1), np.int64)
    cnt = lib().orc_build_bvh2(_p(bounds6), n, _p(nodes), _p(order))
    return nodes[:cnt].copy(), order[:n].copy()


def traverse(nodes, prims, meshes, rays6, tmax, watertight=False, counters=False, threads=0):
    """Closest hit per ray.  meshes: list of (points4 float32, vertex_indices int64).
    Returns (isect records, hit index into prims, counters or None)."""
    nodes = np.ascontiguousarray(nodes)
    prims = np.ascontiguousarray(prims)
    rays6 = np.ascontiguousarray(rays6, np.float32).reshape(-1, 6)
    tmax = np.ascontiguousarray(tmax, np.float32)
    n = len(tmax)
    keep = []
    arr = (_Mesh * max(len(meshes), 1))()
    for i, (p4, vi) in enumerate(meshes):
        p4 = np.ascontiguousarray(p4, np.float32)
        vi = np.ascontiguousarray(vi, np.int64)
        keep += [p4, vi]
        arr[i] = _Mesh(p4.ctypes.data, None, vi.ctypes.data)
    out = np.zeros(n, ISECT_DTYPE)
    hit_index = np.zeros(n, np.int32)
    cnt = np.zeros((n, 4), np.uint32) if counters else None
    if threads <= 0:
        threads = os.cpu_count() or 1
    lib().orc_traverse_batch(_p(nodes), _p(prims), C.addressof(arr), _p(rays6), _p(tmax), n, 1 if watertight else 0,
                             _p(out), _p(hit_index), _p(cnt), threads)
    return out, hit_index, cnt


def mt(o, d, p0, p1, p2, tmax):
    a = [np.ascontiguousarray(x, np.float32) for x in (o, d, p0, p1, p2)]
    t, u, v = C.c_float(), C.c_float(), C.c_float()
    hit = lib().orc_intersect_triangle_mt(*[_p(x) for x in a], tmax, C.byref(t), C.byref(u), C.byref(v))
    return bool(hit), t.value, u.value, v.value


def watertight(o, d, p0, p1, p2, thit):
    a = [np.ascontiguousarray(x, np.float32) for x in (o, d, p0, p1, p2)]
    th, b0, b1, b2 = C.c_float(thit), C.c_float(), C.c_float(), C.c_float()
    hit = lib().orc_intersect_triangle_watertight(*[_p(x) for x in a], C.byref(th), C.byref(b0), C.byref(b1),
                                                  C.byref(b2))
    return bool(hit), th.value, b0.value, b1.value, b2.value


def aabb(mn, mx, o, d, tmax):
    a = [np.ascontiguousarray(x, np.float32) for x in (mn, mx, o, d)]
    tn = C.c_float()
    hit = lib().orc_intersect_aabb(*[_p(x) for x in a], tmax, C.byref(tn))
    return bool(hit), tn.value


def bounds_intersects_swift(mn, mx, o, d, thit):
    a = [np.ascontiguousarray(x, np.float32) for x in (mn, mx, o, d)]
    return bool(lib().orc_bounds_intersects_swift(*[_p(x) for x in a], thit))


def surface_area(mn, mx):
    a = [np.ascontiguousarray(x, np.float32) for x in (mn, mx)]
    return lib().orc_bounds_surface_area(*[_p(x) for x in a])


def maximum_extent(mn, mx):
    a = [np.ascontiguousarray(x, np.float32) for x in (mn, mx)]
    return lib().orc_bounds_maximum_extent(*[_p(x) for x in a])


def zsobol_batch(spp, res_x, res_y, px, py, index, kinds, seed=1234):
    px = np.ascontiguousarray(px, np.int32)
    py = np.ascontiguousarray(py, np.int32)
    index = np.ascontiguousarray(index, np.int64)
    kinds = np.ascontiguousarray(kinds, np.int32)
    per = int(kinds.sum())
    out = np.zeros((len(px), per), np.float32)
    lib().orc_zsobol_batch(spp, res_x, res_y, seed, _p(px), _p(py), _p(index), len(px), _p(kinds), len(kinds),
                           _p(out))
    return out


class RenderParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_depth", C.c_int32),
                ("rr_min_bounce", C.c_int32), ("mis_corrected", C.c_int32), ("seed", C.c_int64),
                ("eye", C.c_float * 3), ("target", C.c_float * 3), ("up", C.c_float * 3), ("fov_deg", C.c_float),
                ("filter_radius", C.c_float), ("filter_sigma", C.c_float), ("first_sample", C.c_int32),
                ("sampler_spp", C.c_int32), ("iso", C.c_float), ("max_component", C.c_float),
                ("lens_radius", C.c_float), ("focal_distance", C.c_float), ("two_sided_emission", C.c_int32),
                ("has_medium", C.c_int32), ("medium_min", C.c_float * 3), ("medium_max", C.c_float * 3),
                ("sigma_a", C.c_float * 3), ("sigma_s", C.c_float * 3), ("medium_g", C.c_float),
                ("crop", C.c_int32 * 4)]


def render_params(width, height, spp, max_depth=5, rr_min_bounce=2, mis_corrected=0, seed=1234,
                  eye=(0.5, 0.5, 2.2), target=(0.5, 0.5, 0.0), up=(0.0, 1.0, 0.0), fov_deg=45.0,
                  filter_radius=2.0, filter_sigma=0.5, first_sample=0, sampler_spp=0, iso=100.0, max_component=0.0,
                  lens_radius=0.0, focal_distance=1e6, two_sided_emission=0, medium=None, crop=None):
    """medium: None or dict(box_min, box_max, sigma_a, sigma_s, g)."""
    m = medium or {}
    f3 = lambda k: (C.c_float * 3)(*m.get(k, (0.0, 0.0, 0.0)))  # noqa: E731
    return RenderParams(width, height, spp, max_depth, rr_min_bounce, mis_corrected, seed, (C.c_float * 3)(*eye),
                        (C.c_float * 3)(*target), (C.c_float * 3)(*up), fov_deg, filter_radius, filter_sigma,
                        first_sample, sampler_spp, iso, max_component, lens_radius, focal_distance,
                        two_sided_emission, 1 if medium else 0, f3("box_min"), f3("box_max"), f3("sigma_a"),
                        f3("sigma_s"), float(m.get("g", 0.0)), (C.c_int32 * 4)(*(crop or (0, 0, 0, 0))))


class _Textures(C.Structure):
    _fields_ = [("count", C.c_int32), ("resolution", C.c_int32), ("material_texture", C.c_void_p),
                ("maps", C.c_void_p), ("texels", C.c_void_p), ("emission_scale", C.c_float)]


class _RenderInstances(C.Structure):
    _fields_ = [("tlas", C.c_void_p), ("leaf_instance", C.c_void_p), ("w2o", C.c_void_p), ("o2w", C.c_void_p),
                ("blas_of", C.c_void_p), ("instance_count", C.c_int64), ("blas", C.c_void_p),
                ("blas_materials", C.c_void_p), ("blas_count", C.c_int64), ("blas_material_params", C.c_void_p)]


class Environment:
    """The oracle's environment light (orc_env): map rgb (H, W, 3) float32,
    scale (enters the light's power only)."""

    def __init__(self, rgb, scale=1.0):
        L = lib()
        if not getattr(L, "_env_bound", False):
            L.orc_env_create.restype = C.c_void_p
            L.orc_env_create.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_float]
            L.orc_env_destroy.argtypes = [C.c_void_p]
            L.orc_env_power.restype = C.c_float
            L.orc_env_power.argtypes = [C.c_void_p]
            L.orc_env_sample.restype = C.c_float
            L.orc_env_sample.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_void_p, C.c_void_p]
            L.orc_env_pdf.restype = C.c_float
            L.orc_env_pdf.argtypes = [C.c_void_p, C.c_void_p]
            L.orc_env_radiance.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
            L.orc_env_tables.argtypes = [C.c_void_p] * 7
            L._env_bound = True
        self.rgb = np.ascontiguousarray(rgb, np.float32)
        h, w = self.rgb.shape[:2]
        self.handle = L.orc_env_create(self.rgb.ctypes.data, w, h, float(scale))

    def __del__(self):
        if getattr(self, "handle", None):
            lib().orc_env_destroy(self.handle)
            self.handle = None

    def power(self):
        return float(lib().orc_env_power(self.handle))

    def sample(self, u0, u1):
        d = np.zeros(3, np.float32)
        c = np.zeros(3, np.float32)
        pdf = lib().orc_env_sample(self.handle, u0, u1, d.ctypes.data, c.ctypes.data)
        return d, c, float(pdf)

    def pdf(self, d):
        d = np.ascontiguousarray(d, np.float32)
        return float(lib().orc_env_pdf(self.handle, d.ctypes.data))

    def radiance(self, d):
        d = np.ascontiguousarray(d, np.float32)
        c = np.zeros(3, np.float32)
        lib().orc_env_radiance(self.handle, d.ctypes.data, c.ctypes.data)
        return c

    def tables(self):
        func = np.zeros((1024, 1024), np.float32)
        cdf = np.zeros((1024, 1025), np.float32)
        ri = np.zeros(1024, np.float32)
        mf = np.zeros(1024, np.float32)
        mc = np.zeros(1025, np.float32)
        mi = np.zeros(1, np.float32)
        lib().orc_env_tables(self.handle, func.ctypes.data, cdf.ctypes.data, ri.ctypes.data, mf.ctypes.data,
                             mc.ctypes.data, mi.ctypes.data)
        return dict(func=func, cdf=cdf, row_integral=ri, marginal_func=mf, marginal_cdf=mc,
                    marginal_integral=float(mi[0]))


def render(hs, params, threads=0, textures=None, env=None, instances=None, aovs=False):
    """Film sums of the oracle integrator: (sum_rgb (H,W,3), sum_sq (H,W,3),
    sum_w (H,W), counters {camera, extension, shadow, probe}).

    textures (optional): dict with material_texture (int32 per material, -1
    for none), maps (count x 9 float32: origin, u axis, v axis), texels
    (count x R x R x 3 float32) and emission_scale (float).
    env (optional): an Environment.
    instances (optional): dict with tlas_nodes, leaf_instance, instances
    (INSTANCE_DTYPE) and blas (HostScene list); hs is then unused (None).
    aovs: also return the albedo and normal sums (H,W,3) (Tile.swift:157-205)
    after the counters."""
    L = lib()
    if not getattr(L, "_render_bound", False):
        L.orc_render_ex.restype = None
        L.orc_render_ex.argtypes = [C.c_void_p] * 4 + [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                                       C.POINTER(RenderParams), C.c_void_p] + [C.c_void_p] * 6 + \
            [C.c_int]
        L._render_bound = True
    keep = []
    inst_struct = None
    if instances is not None:
        blas_scenes = instances["blas"]
        blas = (_Blas * len(blas_scenes))()
        mat_ptrs = (C.c_void_p * len(blas_scenes))()
        par_ptrs = (C.c_void_p * len(blas_scenes))()
        for i, b in enumerate(blas_scenes):
            marr = (_Mesh * max(len(b.meshes), 1))()
            for k, m in enumerate(b.meshes):
                marr[k] = _render_mesh(m, keep)
            nodes_b = np.ascontiguousarray(b.nodes)
            prims_b = np.ascontiguousarray(b.prims)
            mats_b = np.ascontiguousarray(b.materials)
            keep += [marr, nodes_b, prims_b, mats_b]
            blas[i] = _Blas(nodes_b.ctypes.data, prims_b.ctypes.data, C.addressof(marr))
            mat_ptrs[i] = mats_b.ctypes.data
            if getattr(b, "material_params", None) is not None:
                par_b = np.ascontiguousarray(b.material_params, np.float32)
                keep.append(par_b)
                par_ptrs[i] = par_b.ctypes.data
        inst = np.ascontiguousarray(instances["instances"])
        w2o = np.ascontiguousarray(inst["world_to_object"], np.float32)
        o2w = np.ascontiguousarray(inst["object_to_world"], np.float32)
        blas_of = np.ascontiguousarray(inst["blas"], np.int32)
        tlas = np.ascontiguousarray(instances["tlas_nodes"])
        leaf = np.ascontiguousarray(instances["leaf_instance"], np.int64)
        keep += [blas, mat_ptrs, par_ptrs, w2o, o2w, blas_of, tlas, leaf]
        inst_struct = _RenderInstances(tlas.ctypes.data, leaf.ctypes.data, w2o.ctypes.data, o2w.ctypes.data,
                                       blas_of.ctypes.data, len(inst), C.addressof(blas), C.addressof(mat_ptrs),
                                       len(blas_scenes), C.addressof(par_ptrs))
        hs = blas_scenes[0]  # flat arrays unused
    arr = (_Mesh * max(len(hs.meshes), 1))()
    for i, m in enumerate(hs.meshes):
        arr[i] = _render_mesh(m, keep)
    mats = np.ascontiguousarray(hs.materials)
    mparams = None
    if instances is None and getattr(hs, "material_params", None) is not None:
        mparams = np.ascontiguousarray(hs.material_params, np.float32)
        keep.append(mparams)
    W, H = params.width, params.height
    if any(params.crop):  # the film holds the crop window only
        W, H = params.crop[2] - params.crop[0], params.crop[3] - params.crop[1]
    s = np.zeros((H, W, 3), np.float32)
    s2 = np.zeros((H, W, 3), np.float32)
    sw = np.zeros((H, W), np.float32)
    cnt = np.zeros(4, np.uint64)
    alb = np.zeros((H, W, 3), np.float32)
    nrm = np.zeros((H, W, 3), np.float32)
    if threads <= 0:
        threads = os.cpu_count() or 1
    tex = None
    if textures is not None:
        mt = np.ascontiguousarray(textures["material_texture"], np.int32)
        maps = np.ascontiguousarray(textures["maps"], np.float32)
        tx = np.ascontiguousarray(textures["texels"], np.float32)
        if len(mt) != len(mats) or tx.ndim != 4 or tx.shape[1] != tx.shape[2] or tx.shape[3] != 3 \
                or maps.shape != (tx.shape[0], 9):
            raise ValueError("oracle render: inconsistent texture arrays")
        keep += [mt, maps, tx]
        tex = _Textures(tx.shape[0], tx.shape[1], mt.ctypes.data, maps.ctypes.data, tx.ctypes.data,
                        float(textures.get("emission_scale", 1.0)))
    L.orc_render_ex(_p(np.ascontiguousarray(hs.nodes)), _p(np.ascontiguousarray(hs.prims)), C.addressof(arr),
                    _p(mats), len(mats), len(hs.prims), C.byref(inst_struct) if inst_struct is not None else None,
                    env.handle if env is not None else None, _p(mparams) if mparams is not None else None,
                    C.byref(params),
                    C.byref(tex) if tex is not None else None, _p(s), _p(s2), _p(sw),
                    _p(alb) if aovs else None, _p(nrm) if aovs else None, _p(cnt), threads)
    counters = {"camera": int(cnt[0]), "extension": int(cnt[1]), "shadow": int(cnt[2]), "probe": int(cnt[3])}
    if aovs:
        return s, s2, sw, counters, alb, nrm
    return s, s2, sw, counters


PATH_DTYPE = np.dtype({"names": ["ray", "throughput", "estimate", "albedo", "pcg_state", "pcg_inc", "active"],
                       "formats": [("<f4", 6), ("<f4", 3), ("<f4", 3), ("<f4", 3), "<u8", "<u8", "i1"],
                       "offsets": [0, 24, 36, 48, 64, 72, 80], "itemsize": 88})


def camera_rays(params, first, count):
    """Camera rays of paths [first, first + count): (rays6 (n, 6) float32,
    weights (n,) float32, pixels (n,) int32)."""
    L = lib()
    if not getattr(L, "_camera_bound", False):
        L.orc_camera_rays.restype = None
        L.orc_camera_rays.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        L._camera_bound = True
    rays = np.zeros((count, 6), np.float32)
    w = np.zeros(count, np.float32)
    px = np.zeros(count, np.int32)
    L.orc_camera_rays(C.addressof(params), first, count, _p(rays), _p(w), _p(px))
    return rays, w, px


def shade_batch(hs, paths, isects):
    """shade_core over a batch (in place on a copy); returns the new paths."""
    L = lib()
    if not getattr(L, "_shade_bound", False):
        L.orc_shade_batch.restype = None
        L.orc_shade_batch.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        L._shade_bound = True
    out = np.ascontiguousarray(paths).copy()
    keep = []
    arr = (_Mesh * max(len(hs.meshes), 1))()
    for i, m in enumerate(hs.meshes):
        p4 = np.ascontiguousarray(m.points, np.float32)
        vi = np.ascontiguousarray(m.vertex_indices, np.int64)
        keep += [p4, vi]
        arr[i] = _Mesh(p4.ctypes.data, None, vi.ctypes.data)
    L.orc_shade_batch(_p(out), len(out), _p(np.ascontiguousarray(isects)), C.addressof(arr),
                      _p(np.ascontiguousarray(hs.materials)))
    return out


class _Blas(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("prims", C.c_void_p), ("meshes", C.c_void_p)]


def traverse_instanced(tlas_nodes, leaf_instance, w2o, blas_of, blas_scenes, rays6, tmax, threads=0):
    """Two-level closest hit.  blas_scenes: HostScene list; w2o: (n_inst, 12)
    float32; blas_of: (n_inst,) int32.  Returns prim, inst, t, u, v arrays."""
    L = lib()
    if not getattr(L, "_inst_bound", False):
        L.orc_traverse_instanced.restype = None
        L.orc_traverse_instanced.argtypes = [C.c_void_p] * 7 + [C.c_int64] + [C.c_void_p] * 5 + [C.c_int]
        L._inst_bound = True
    keep = []
    blas = (_Blas * len(blas_scenes))()
    for i, hs in enumerate(blas_scenes):
        arr = (_Mesh * max(len(hs.meshes), 1))()
        for k, m in enumerate(hs.meshes):
            p4 = np.ascontiguousarray(m.points, np.float32)
            vi = np.ascontiguousarray(m.vertex_indices, np.int64)
            keep += [p4, vi]
            arr[k] = _Mesh(p4.ctypes.data, None, vi.ctypes.data)
        nodes = np.ascontiguousarray(hs.nodes)
        prims = np.ascontiguousarray(hs.prims)
        keep += [arr, nodes, prims]
        blas[i] = _Blas(nodes.ctypes.data, prims.ctypes.data, C.addressof(arr))
    tlas_nodes = np.ascontiguousarray(tlas_nodes)
    leaf_instance = np.ascontiguousarray(leaf_instance, np.int64)
    w2o = np.ascontiguousarray(w2o, np.float32)
    blas_of = np.ascontiguousarray(blas_of, np.int32)
    rays6 = np.ascontiguousarray(rays6, np.float32).reshape(-1, 6)
    tmax = np.ascontiguousarray(tmax, np.float32)
    n = len(tmax)
    prim = np.zeros(n, np.int32)
    inst = np.zeros(n, np.int32)
    t = np.zeros(n, np.float32)
    u = np.zeros(n, np.float32)
    v = np.zeros(n, np.float32)
    if threads <= 0:
        threads = os.cpu_count() or 1
    L.orc_traverse_instanced(_p(tlas_nodes), _p(leaf_instance), _p(w2o), _p(blas_of), C.addressof(blas), _p(rays6),
                             _p(tmax), n, _p(prim), _p(inst), _p(t), _p(u), _p(v), threads)
    return prim, inst, t, u, v


class BsdfParams(C.Structure):
    _fields_ = [("type", C.c_int32), ("reflectance", C.c_float * 3), ("eta", C.c_float), ("roughness_u", C.c_float),
                ("roughness_v", C.c_float), ("thickness", C.c_float), ("conductor_eta", C.c_float * 3),
                ("conductor_k", C.c_float * 3), ("conductor_roughness_u", C.c_float),
                ("conductor_roughness_v", C.c_float)]


def bsdf_params(kind, reflectance=(0.5, 0.5, 0.5), eta=1.5, roughness=0.0, thickness=0.01,
                conductor_eta=(0.2, 0.92, 1.1), conductor_k=(3.9, 2.45, 2.14), conductor_roughness=0.0):
    """kind: 1 diffuse, 3 dielectric, 4 coated diffuse, 5 conductor, 6 coated
    conductor (Material_C.type values)."""
    p = BsdfParams()
    p.type = int(kind)
    for c in range(3):
        p.reflectance[c] = float(reflectance[c])
        p.conductor_eta[c] = float(conductor_eta[c])
        p.conductor_k[c] = float(conductor_k[c])
    p.eta, p.roughness_u, p.roughness_v, p.thickness = float(eta), float(roughness), float(roughness), float(thickness)
    p.conductor_roughness_u = p.conductor_roughness_v = float(conductor_roughness)
    return p


def _bsdf_lib():
    L = lib()
    if not getattr(L, "_bsdf_bound", False):
        L.orc_bsdf_eval.restype = None
        L.orc_bsdf_eval.argtypes = [C.POINTER(BsdfParams)] + [C.c_void_p] * 4
        L.orc_bsdf_sample.restype = C.c_int
        L.orc_bsdf_sample.argtypes = [C.POINTER(BsdfParams)] + [C.c_void_p] * 5
        L.orc_bsdf_is_specular.restype = C.c_int
        L.orc_bsdf_is_specular.argtypes = [C.POINTER(BsdfParams)]
        L._bsdf_bound = True
    return L


def bsdf_eval(p, wo, wi):
    """(f rgb, pdf) of directions in the shading frame."""
    L = _bsdf_lib()
    a = np.ascontiguousarray(wo, np.float32)
    b = np.ascontiguousarray(wi, np.float32)
    f = np.zeros(3, np.float32)
    pdf = np.zeros(1, np.float32)
    L.orc_bsdf_eval(C.byref(p), _p(a), _p(b), _p(f), _p(pdf))
    return f, float(pdf[0])


def bsdf_sample(p, wo, u):
    """(valid, f rgb, wi, pdf) for three uniform numbers u."""
    L = _bsdf_lib()
    a = np.ascontiguousarray(wo, np.float32)
    uu = np.ascontiguousarray(u, np.float32)
    f = np.zeros(3, np.float32)
    wi = np.zeros(3, np.float32)
    pdf = np.zeros(1, np.float32)
    ok = L.orc_bsdf_sample(C.byref(p), _p(a), _p(uu), _p(f), _p(wi), _p(pdf))
    return bool(ok), f, wi, float(pdf[0])


def bsdf_is_specular(p):
    return bool(_bsdf_lib().orc_bsdf_is_specular(C.byref(p)))


def power_heuristic(f, g):
    return float(lib().orc_power_heuristic(f, g))


def concentric_disk(u0, u1):
    out = np.zeros(2, np.float32)
    lib().orc_concentric_disk(u0, u1, out.ctypes.data)
    return out


def cosine_hemisphere(u0, u1):
    out = np.zeros(3, np.float32)
    lib().orc_cosine_hemisphere(u0, u1, out.ctypes.data)
    return out


def offset_origin(p, n, d):
    p, n, d = (np.ascontiguousarray(x, np.float32) for x in (p, n, d))
    out = np.zeros(3, np.float32)
    lib().orc_offset_origin(p.ctypes.data, n.ctypes.data, d.ctypes.data, out.ctypes.data)
    return out


def spawn_to(frm, target):
    """Shadow-ray spawn: (origin, direction, tHit)."""
    frm, target = (np.ascontiguousarray(x, np.float32) for x in (frm, target))
    o, d = np.zeros(3, np.float32), np.zeros(3, np.float32)
    t = lib().orc_spawn_to(frm.ctypes.data, target.ctypes.data, o.ctypes.data, d.ctypes.data)
    return o, d, float(t)


def gaussian_filter_evaluate(x, y, sigma):
    """GaussianFilter.evaluate: the separable product, each factor clamped at 0."""
    L = lib()
    return max(0.0, L.orc_gaussian(x, sigma)) * max(0.0, L.orc_gaussian(y, sigma))


def gaussian_filter_sample(u0, u1, radius, sigma):
    """GaussianFilter.sample: ((x, y), density)."""
    L = lib()
    xs, ds = [], []
    for u in (u0, u1):
        x, dn = C.c_float(), C.c_float()
        L.orc_gaussian_sample_1d(u, radius, sigma, C.byref(x), C.byref(dn))
        xs.append(x.value)
        ds.append(dn.value)
    return (xs[0], xs[1]), ds[0] * ds[1]
