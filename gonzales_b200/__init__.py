"""gonzales_b200: B200-native (sm_100a) BVH traversal for the Gonzales path tracer.

The compute path is libgzg.so (CUDA, built in-tree by gonzales_b200/build.py);
this package is its host-side mirror of the reference's Accelerator interface.
There is no CPU fallback: without libgzg.so or a B200, calls raise GzgError.
"""
from ._ffi import GzgError, LEAF_MOLLER_TRUMBORE, LEAF_WATERTIGHT, TRAVERSAL_BVH2, TRAVERSAL_WIDE, options
from .accel import BatchRenderer, GpuAccelerator, InstancedAccelerator, Renderer, gpu_available, instance_bounds
from .scene import HostScene, SceneBuilder, build_bvh2, make_mesh, triangle_bounds

__all__ = [
    "BatchRenderer", "GzgError", "GpuAccelerator", "HostScene", "Renderer", "SceneBuilder", "build_bvh2", "gpu_available", "make_mesh",
    "options", "triangle_bounds", "LEAF_MOLLER_TRUMBORE", "LEAF_WATERTIGHT", "TRAVERSAL_BVH2", "TRAVERSAL_WIDE",
]
