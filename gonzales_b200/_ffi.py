"""ctypes binding of libgzg.so (include/gzg.h, include/gzg_host.h).

The library is loaded from the package directory.  There is no fallback: if
libgzg.so is missing or fails to load, every call raises GzgError.
"""
import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libgzg.so"

GZG_OK = 0
STATUS_NAMES = {
    0: "GZG_OK",
    1: "GZG_ERR_INVALID_ARGUMENT",
    2: "GZG_ERR_NO_DEVICE",
    3: "GZG_ERR_CUDA",
    4: "GZG_ERR_OUT_OF_MEMORY",
    5: "GZG_ERR_BAD_SCENE",
    6: "GZG_ERR_KERNEL_FAULT",
    7: "GZG_ERR_LIMIT",
    8: "GZG_ERR_TIMEOUT",
}

TRAVERSAL_WIDE = 0
TRAVERSAL_BVH2 = 1
TRAVERSAL_WIDE_ONE_RAY_PER_THREAD = 2
LEAF_MOLLER_TRUMBORE = 0
LEAF_WATERTIGHT = 1


class GzgError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


# ---------------------------------------------------------------- records
# numpy dtypes with the byte layouts of gzg.h (== mojo_kernel.h).

PRIM_ID_DTYPE = np.dtype(
    {"names": ["id1", "id2", "material_index", "type"], "formats": ["<i8", "<i8", "<i8", "i1"],
     "offsets": [0, 8, 16, 24], "itemsize": 32})
INTERSECTION_DTYPE = np.dtype(
    {"names": ["prim_id", "t_hit", "u", "v", "hit"], "formats": [PRIM_ID_DTYPE, "<f4", "<f4", "<f4", "i1"],
     "offsets": [0, 32, 36, 40, 44], "itemsize": 48})
BVH2_NODE_DTYPE = np.dtype(
    {"names": ["bounds_min", "bounds_max", "offset", "count"], "formats": [("<f4", 3), ("<f4", 3), "<i4", "<i4"],
     "offsets": [0, 12, 24, 28], "itemsize": 32})
MATERIAL_DTYPE = np.dtype(
    {"names": ["type", "albedo", "emission"], "formats": ["i1", ("<f4", 3), ("<f4", 3)],
     "offsets": [0, 4, 16], "itemsize": 28})
RAY_DTYPE = np.dtype([("org", "<f4", 3), ("dir", "<f4", 3)])  # Ray_C, 24 bytes
INSTANCE_DTYPE = np.dtype([("object_to_world", "<f4", 12), ("world_to_object", "<f4", 12), ("blas", "<i4"),
                           ("pad", "<i4")])  # gzg_instance, 104 bytes
PATH_STATE_DTYPE = np.dtype(
    {"names": ["ray", "throughput", "estimate", "albedo", "pcg_state", "pcg_inc", "active"],
     "formats": [RAY_DTYPE, ("<f4", 3), ("<f4", 3), ("<f4", 3), "<u8", "<u8", "i1"],
     "offsets": [0, 24, 36, 48, 64, 72, 80], "itemsize": 88})


class TriangleMeshC(C.Structure):
    _fields_ = [("points", C.c_void_p), ("face_indices", C.c_void_p), ("vertex_indices", C.c_void_p)]


class TraceOptions(C.Structure):
    _fields_ = [("traversal", C.c_int32), ("leaf_test", C.c_int32), ("block_size", C.c_int32),
                ("blocks_per_sm", C.c_int32), ("stack_depth", C.c_int32), ("l1_carveout", C.c_int32),
                ("fetch_counters", C.c_void_p)]


BUILD_DEFAULT, BUILD_LBVH, BUILD_PLOC = 0, 1, 2


class BuildOptions(C.Structure):
    _fields_ = [("leaf_size", C.c_int32), ("builder", C.c_int32), ("radius", C.c_int32), ("reserved", C.c_int32)]


class MeshArrays(C.Structure):
    _fields_ = [("points", C.c_void_p), ("vertex_count", C.c_int64), ("indices", C.c_void_p),
                ("triangle_count", C.c_int64), ("material", C.c_int64)]


class PlyMesh(C.Structure):
    _fields_ = [("vertex_count", C.c_int64), ("face_count", C.c_int64), ("points", C.POINTER(C.c_float)),
                ("normals", C.POINTER(C.c_float)), ("uvs", C.POINTER(C.c_float)),
                ("indices", C.POINTER(C.c_int32)), ("face_indices", C.POINTER(C.c_int32)), ("owner", C.c_void_p)]


class SceneInfo(C.Structure):
    _fields_ = [("bvh2_nodes", C.c_int64), ("prims", C.c_int64), ("triangles", C.c_int64),
                ("wide_nodes", C.c_int64), ("wide_depth", C.c_int32), ("bvh2_depth", C.c_int32),
                ("device_bytes", C.c_int64)]


class RenderParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_depth", C.c_int32),
                ("rr_min_bounce", C.c_int32), ("mis_corrected", C.c_int32), ("seed", C.c_int64),
                ("eye", C.c_float * 3), ("target", C.c_float * 3), ("up", C.c_float * 3), ("fov_deg", C.c_float),
                ("filter_radius", C.c_float), ("filter_sigma", C.c_float), ("first_sample", C.c_int32),
                ("sampler_spp", C.c_int32), ("wave_paths", C.c_int32), ("use_graph", C.c_int32),
                ("lens_radius", C.c_float), ("focal_distance", C.c_float), ("two_sided_emission", C.c_int32),
                ("crop", C.c_int32 * 4)]

    @property
    def film_width(self):
        """Width of the film: the crop window's, or the frame's."""
        return self.crop[2] - self.crop[0] if any(self.crop) else self.width

    @property
    def film_height(self):
        return self.crop[3] - self.crop[1] if any(self.crop) else self.height


class RenderStats(C.Structure):
    _fields_ = [("camera_rays", C.c_uint64), ("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("probe_rays", C.c_uint64), ("waves", C.c_uint64)]


def render_params(width, height, spp, max_depth=5, rr_min_bounce=2, mis_corrected=0, seed=1234,
                  eye=(0.5, 0.5, 2.2), target=(0.5, 0.5, 0.0), up=(0.0, 1.0, 0.0), fov_deg=45.0,
                  filter_radius=2.0, filter_sigma=0.5, first_sample=0, sampler_spp=0, wave_paths=0, use_graph=0,
                  lens_radius=0.0, focal_distance=1e6, two_sided_emission=0, crop=None):
    """gzg_render_params with the reference's defaults (Gaussian filter radius 2,
    sigma 0.5; Z-Sobol seed 1234; roulette from bounce 2; pinhole camera,
    focal distance 1e6)."""
    return RenderParams(width, height, spp, max_depth, rr_min_bounce, mis_corrected, seed, (C.c_float * 3)(*eye),
                        (C.c_float * 3)(*target), (C.c_float * 3)(*up), fov_deg, filter_radius, filter_sigma,
                        first_sample, sampler_spp, wave_paths, use_graph, lens_radius, focal_distance,
                        two_sided_emission, (C.c_int32 * 4)(*(crop or (0, 0, 0, 0))))


SORT_NONE, SORT_MATERIAL, SORT_SCENE = 0, 1, 2


class TextureBinding(C.Structure):
    _fields_ = [("material", C.c_int32), ("reserved", C.c_int32), ("origin", C.c_float * 3),
                ("u_axis", C.c_float * 3), ("v_axis", C.c_float * 3)]


class BatchOptions(C.Structure):
    _fields_ = [("wave_paths", C.c_int32), ("use_graph", C.c_int32), ("sort_key", C.c_int32),
                ("reserved", C.c_int32)]


class Medium(C.Structure):
    _fields_ = [("box_min", C.c_float * 3), ("box_max", C.c_float * 3), ("sigma_a", C.c_float * 3),
                ("sigma_s", C.c_float * 3), ("g", C.c_float), ("reserved", C.c_int32)]


VP = C.c_void_p
I64 = C.c_int64
ST = C.c_int32

# name -> (restype, argtypes); every symbol declared in include/gzg*.h.
PROTOTYPES = {
    "gzg_gpu_available": (C.c_bool, []),
    "gzg_last_error": (C.c_char_p, []),
    "gzg_gpu_upload_scene": (ST, [VP, I64, VP, I64, VP, I64, VP, VP, VP, VP, I64, C.POINTER(VP)]),
    "gzg_gpu_free_scene": (ST, [VP]),
    "gzg_gpu_traverse_batch": (ST, [VP, VP, VP, I64, VP, C.POINTER(TraceOptions)]),
    "gzg_gpu_traverse_batch_hits": (ST, [VP, VP, VP, I64, VP, C.POINTER(TraceOptions)]),
    "gzg_gpu_occluded_batch": (ST, [VP, VP, VP, I64, VP, C.POINTER(TraceOptions)]),
    "gzg_gpu_traverse_batch_static": (ST, [VP, VP, VP, I64, VP]),
    "gzg_gpu_shade_batch": (ST, [VP, VP, I64, VP]),
    "gzg_trace_closest_device": (ST, [VP, VP, I64, VP, C.POINTER(TraceOptions), VP]),
    "gzg_trace_any_device": (ST, [VP, VP, I64, VP, C.POINTER(TraceOptions), VP]),
    "gzg_hits_to_intersections_device": (ST, [VP, VP, I64, VP, VP]),
    "gzg_scene_autotune": (ST, [VP, VP, I64, C.c_int32, C.POINTER(TraceOptions), C.POINTER(C.c_float), VP]),
    "gzg_scene_set_launch": (ST, [VP, C.c_int32, C.POINTER(TraceOptions)]),
    "gzg_scene_set_environment": (ST, [VP, VP, C.c_int32, C.c_int32, C.c_float]),
    "gzg_scene_set_material_params": (ST, [VP, VP, I64]),
    "gzg_scene_set_vertex_attributes": (ST, [VP, I64, VP, VP, I64]),
    "gzg_gpu_build_scene": (ST, [VP, I64, VP, I64, VP, VP, VP, VP, I64, VP, C.POINTER(VP)]),
    "gzg_scene_build_time": (ST, [VP, C.POINTER(C.c_float)]),
    "gzg_gpu_build_mesh_scene": (ST, [VP, I64, VP, I64, VP, C.POINTER(VP)]),
    "gzg_ply_read": (ST, [C.c_char_p, C.POINTER(C.POINTER(PlyMesh))]),
    "gzg_ply_parse": (ST, [VP, I64, C.POINTER(C.POINTER(PlyMesh))]),
    "gzg_ply_free": (ST, [C.POINTER(PlyMesh)]),
    "gzg_film_resolve_device": (ST, [VP, VP, I64, VP, VP, VP]),
    "gzg_write_exr": (ST, [C.c_char_p, VP, C.c_int32, C.c_int32, C.c_int32]),
    "gzg_scene_tree_cost": (ST, [VP, C.POINTER(C.c_double)]),
    "gzg_host_instance_bounds": (ST, [VP, I64, VP, I64, VP]),
    "gzg_instanced_scene_create": (ST, [VP, I64, VP, I64, VP, I64, VP, I64, C.POINTER(VP)]),
    "gzg_trace_closest_instanced_device": (ST, [VP, VP, I64, VP, VP, C.POINTER(TraceOptions), VP]),
    "gzg_scene_info_get": (ST, [VP, C.POINTER(SceneInfo)]),
    "gzg_renderer_create": (ST, [VP, C.POINTER(RenderParams), C.POINTER(VP)]),
    "gzg_renderer_destroy": (ST, [VP]),
    "gzg_renderer_render": (ST, [VP, VP, VP, VP, VP]),
    "gzg_renderer_stats": (ST, [VP, C.POINTER(RenderStats)]),
    "gzg_batch_renderer_create": (ST, [VP, VP, I64, C.POINTER(BatchOptions), C.POINTER(VP)]),
    "gzg_renderer_film_layout": (ST, [VP, VP]),
    "gzg_renderer_autotune": (ST, [VP, C.POINTER(BatchOptions), C.POINTER(C.c_float), VP]),
    "gzg_renderer_error_word": (ST, [VP, C.POINTER(C.c_uint32), C.c_int32]),
    "gzg_renderer_set_textures": (ST, [VP, VP, C.c_int32, C.c_int32, VP, C.c_float]),
    "gzg_renderer_set_film": (ST, [VP, C.c_float, C.c_float]),
    "gzg_renderer_render_aov": (ST, [VP, VP, VP, VP, VP, VP, VP]),
    "gzg_renderer_render_f64": (ST, [VP, VP, VP, VP, VP]),
    "gzg_renderer_adjoint": (ST, [VP, VP, VP, VP, VP, VP]),
    "gzg_render_image": (ST, [VP, C.POINTER(RenderParams), VP, VP, VP, C.POINTER(RenderStats)]),
    "gzg_camera_rays": (ST, [C.POINTER(RenderParams), I64, I64, VP, VP, VP]),
    "gzg_host_instance_bounds_from_scenes": (ST, [VP, I64, VP, I64, VP]),
    "gzg_scene_set_medium": (ST, [VP, C.POINTER(Medium)]),
    "gzg_zsobol_fill_device": (ST, [I64, C.c_int32, C.c_int32, I64, VP, VP, VP, I64, VP, C.c_int32, VP, VP]),
    "gzg_scene_error_word": (ST, [VP, C.POINTER(C.c_uint32), C.c_int]),
    "gzg_host_triangle_bounds": (ST, [VP, VP, I64, VP]),
    "gzg_host_build_bvh2": (ST, [VP, I64, VP, C.POINTER(I64), VP, C.c_int32]),
}

_lib = None


def lib():
    """Loads libgzg.so once; raises GzgError if it is absent."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise GzgError(2, f"{LIB_PATH} is not built (run gonzales_b200/build.py)")
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status):
    if status != GZG_OK:
        msg = lib().gzg_last_error()
        raise GzgError(status, msg.decode() if msg else "")


def ptr(a):
    """Address of a numpy array's data (or None)."""
    if a is None:
        return None
    return a.ctypes.data


def options(traversal=TRAVERSAL_WIDE, leaf_test=LEAF_MOLLER_TRUMBORE, block_size=0, blocks_per_sm=0,
            stack_depth=0, l1_carveout=0, fetch_counters=None):
    """Trace options; 0 fields take the scene's tuned launch.  fetch_counters:
    device address (int) of 3 uint64 (nodes, triangles, rays) or None."""
    return TraceOptions(traversal, leaf_test, block_size, blocks_per_sm, stack_depth, l1_carveout, fetch_counters)
