"""Host-side scene assembly: the part of Gonzales' Swift host that turns meshes
into the arrays its native plugin consumes.

Mirrors, in the reference:
  - TriangleMesh / cStruct        Sources/libgonzales/Shape/Triangle.swift:4-87
    (world-space float4 points, int64 vertex indices, int64 face indices)
  - shape batching into prims     Sources/libgonzales/Api/SceneDescription.swift:700-760
    (each triangle a GeometricPrimitive with a running idx; area lights as AreaLight prims)
  - prim-id packing               Sources/libgonzales/Accelerators/BoundingHierarchy.swift:21-56
    (type 1 geometric / 3 area light, id2 = mesh << 32 | tri)
  - materials for the plugin      Sources/libgonzales/Accelerators/BoundingHierarchy.swift:91-150
  - SAH BVH2 build                Sources/libgonzales/Accelerators/BoundingHierarchyBuilder.swift:66-339
    (run by libgzg's host builder, gzg_host_build_bvh2)
"""
from dataclasses import dataclass, field

import numpy as np

from . import _ffi as F

PRIM_TRIANGLE = 0
PRIM_GEOMETRIC = 1
PRIM_TRANSFORMED = 2
PRIM_AREA_LIGHT = 3

MATERIAL_NONE = 0
MATERIAL_DIFFUSE = 1
MATERIAL_AREA_LIGHT = 2
# renderer extensions (Material_C.type values the reference's plugin never sees)
MATERIAL_DIELECTRIC = 3         # Material/Dielectric.swift
MATERIAL_COATED_DIFFUSE = 4     # Material/CoatedDiffuse.swift
MATERIAL_CONDUCTOR = 5          # Material/Conductor.swift
MATERIAL_COATED_CONDUCTOR = 6   # Material/CoatedConductor.swift
EXTENDED_MATERIALS = (MATERIAL_DIELECTRIC, MATERIAL_COATED_DIFFUSE, MATERIAL_CONDUCTOR, MATERIAL_COATED_CONDUCTOR)
# gzg_material_params: eta, roughness u, v, thickness, conductor eta (3),
# conductor roughness u, conductor k (3), conductor roughness v
MATERIAL_PARAMS_WIDTH = 12
# copper's refractive index and extinction at the RGB primaries (approximate)
COPPER_ETA = (0.2, 0.92, 1.1)
COPPER_K = (3.9, 2.45, 2.14)


@dataclass
class Mesh:
    """A triangle mesh in world space (TriangleMesh, Shape/Triangle.swift:4-87)."""

    points: np.ndarray          # (n, 4) float32, w unused
    vertex_indices: np.ndarray  # (3 * ntri,) int64
    face_indices: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    normals: np.ndarray = None  # (n, 3) float32 vertex normals (renderer shading), or None
    uvs: np.ndarray = None      # (n, 2) float32 vertex UVs (renderer shading), or None

    @property
    def triangle_count(self):
        return len(self.vertex_indices) // 3


def make_mesh(points, triangles, normals=None, uvs=None):
    pts = np.asarray(points, dtype=np.float32).reshape(-1, 3)
    p4 = np.ones((len(pts), 4), np.float32)
    p4[:, :3] = pts
    vi = np.ascontiguousarray(np.asarray(triangles, dtype=np.int64).reshape(-1))
    nrm = None if normals is None else np.ascontiguousarray(np.asarray(normals, np.float32).reshape(len(pts), 3))
    uv = None if uvs is None else np.ascontiguousarray(np.asarray(uvs, np.float32).reshape(len(pts), 2))
    return Mesh(points=np.ascontiguousarray(p4), vertex_indices=vi, normals=nrm, uvs=uv)


def triangle_bounds(mesh):
    """Per-triangle bounds (Triangle.worldBound) via libgzg's host helper."""
    n = mesh.triangle_count
    out = np.empty((n, 6), np.float32)
    F.check(F.lib().gzg_host_triangle_bounds(F.ptr(mesh.points), F.ptr(mesh.vertex_indices), n, F.ptr(out)))
    return out


def build_bvh2(bounds6, threads=0):
    """SAH BVH2 over prim bounds; returns (nodes, order)."""
    bounds6 = np.ascontiguousarray(bounds6, dtype=np.float32)
    n = len(bounds6)
    nodes = np.zeros(max(2 * n, 1), F.BVH2_NODE_DTYPE)
    order = np.zeros(max(n, 1), np.int64)
    count = F.I64(0)
    F.check(F.lib().gzg_host_build_bvh2(F.ptr(bounds6), n, F.ptr(nodes), F.C.byref(count), F.ptr(order), threads))
    return nodes[: count.value].copy(), order[:n].copy()


@dataclass
class HostScene:
    """The arrays a Gonzales BoundingHierarchy hands to the native plugin."""

    meshes: list
    prims: np.ndarray      # PRIM_ID_DTYPE, in BVH leaf order
    nodes: np.ndarray      # BVH2_NODE_DTYPE
    materials: np.ndarray  # MATERIAL_DTYPE
    prim_order: np.ndarray  # k-th leaf prim = input prim prim_order[k]
    material_params: np.ndarray = None  # (n_materials, MATERIAL_PARAMS_WIDTH) float32

    def root_bounds(self):
        """(lo[3], hi[3]) of the scene: the BVH2 root's box, or the
        triangles' bounds when the tree is built on the device."""
        if self.nodes is not None:
            return self.nodes[0]["bounds_min"], self.nodes[0]["bounds_max"]
        lo = np.full(3, np.inf, np.float32)
        hi = np.full(3, -np.inf, np.float32)
        for m in self.meshes:
            p = np.asarray(m.points, np.float32).reshape(-1, 4)[:, :3]
            used = p[np.asarray(m.vertex_indices, np.int64).reshape(-1)]
            if len(used):
                lo = np.minimum(lo, used.min(0))
                hi = np.maximum(hi, used.max(0))
        return lo, hi

    @property
    def has_extended_materials(self):
        return bool(np.isin(self.materials["type"], EXTENDED_MATERIALS).any())

    def mesh_structs(self):
        arr = (F.TriangleMeshC * max(len(self.meshes), 1))()
        for i, m in enumerate(self.meshes):
            arr[i] = F.TriangleMeshC(m.points.ctypes.data,
                                     m.face_indices.ctypes.data if len(m.face_indices) else None,
                                     m.vertex_indices.ctypes.data)
        return arr

    def counts(self):
        pts = np.array([m.points.size for m in self.meshes], np.int64)
        fi = np.array([len(m.face_indices) for m in self.meshes], np.int64)
        vi = np.array([len(m.vertex_indices) for m in self.meshes], np.int64)
        return pts, fi, vi

    @property
    def triangle_count(self):
        return int(sum(m.triangle_count for m in self.meshes))


class SceneBuilder:
    """Collects meshes the way SceneDescription.worldEnd batches shapes.

    add_mesh(..., material) creates one GeometricPrimitive per triangle
    (type 1, id1 = running geometric-prim index, id2 = mesh << 32 | tri);
    add_area_light creates AreaLight prims (type 3, id1 = light index) whose
    material index is resolved like BoundingHierarchy.prepareMaterials
    (area-light materials follow the surface materials).
    """

    def __init__(self):
        self.meshes = []
        self._prims = []       # list of (mesh, first_tri, ntri, type, material or light)
        self._materials = []   # (type, albedo, emission)
        self._material_params = []  # MATERIAL_PARAMS_WIDTH floats per material
        self._lights = []      # emission per area light
        self._geometric = 0

    def add_material(self, albedo=(0.5, 0.5, 0.5), kind="diffuse", eta=1.5, roughness=0.0, thickness=0.01,
                     conductor_eta=COPPER_ETA, conductor_k=COPPER_K, conductor_roughness=0.0):
        """kind: "diffuse" (albedo), "dielectric" (eta, roughness; albedo
        unused), "coateddiffuse" (reflectance = albedo, coating eta and
        roughness, clear layer thickness), "conductor" (conductor eta / k per
        channel, conductor roughness used as alpha) or "coatedconductor"
        (coating eta and roughness over a conductor of reflectance = albedo,
        conductor eta / k / roughness, layer thickness).  Dielectric and
        coating roughness (and a coated conductor's) is remapped to alpha =
        sqrt(roughness) as the reference's remaproughness default does."""
        t = {"diffuse": MATERIAL_DIFFUSE, "dielectric": MATERIAL_DIELECTRIC,
             "coateddiffuse": MATERIAL_COATED_DIFFUSE, "conductor": MATERIAL_CONDUCTOR,
             "coatedconductor": MATERIAL_COATED_CONDUCTOR}[kind]
        self._materials.append((t, tuple(albedo), (0.0, 0.0, 0.0)))
        ce, ck = tuple(conductor_eta), tuple(conductor_k)
        self._material_params.append((eta, roughness, roughness, thickness) + ce + (conductor_roughness,) + ck +
                                     (conductor_roughness,))
        return len(self._materials) - 1

    def add_mesh(self, points, triangles, material=0, normals=None, uvs=None):
        """A mesh of diffuse (or `material`) triangles; optional vertex normals
        and UVs shade it as Triangle.computeSurfaceInteraction does."""
        mesh = make_mesh(points, triangles, normals, uvs)
        self.meshes.append(mesh)
        idx = len(self.meshes) - 1
        self._prims.append((idx, mesh.triangle_count, PRIM_GEOMETRIC, material, self._geometric))
        self._geometric += mesh.triangle_count
        return idx

    def add_area_light(self, points, triangles, emission):
        mesh = make_mesh(points, triangles)
        self.meshes.append(mesh)
        idx = len(self.meshes) - 1
        first_light = len(self._lights)
        for _ in range(mesh.triangle_count):
            self._lights.append(tuple(emission))
        self._prims.append((idx, mesh.triangle_count, PRIM_AREA_LIGHT, None, first_light))
        return idx

    def build(self, threads=0, host_bvh=True):
        """The HostScene.  host_bvh=False skips the host's SAH build: prims
        stay in input order and nodes is None, for the device build
        (GpuAccelerator builds the tree with gzg_gpu_build_scene)."""
        n_surface = len(self._materials)
        mats = np.zeros(n_surface + len(self._lights), F.MATERIAL_DTYPE)
        for i, (t, a, e) in enumerate(self._materials):
            mats[i] = (t, a, e)
        for j, e in enumerate(self._lights):
            mats[n_surface + j] = (MATERIAL_AREA_LIGHT, (0, 0, 0), e)

        total = sum(p[1] for p in self._prims)
        prims = np.zeros(total, F.PRIM_ID_DTYPE)
        bounds = np.zeros((total, 6), np.float32)
        k = 0
        for mesh_idx, ntri, ptype, material, first in self._prims:
            tri = np.arange(ntri, dtype=np.int64)
            sl = slice(k, k + ntri)
            prims["id1"][sl] = first + tri
            prims["id2"][sl] = (np.int64(mesh_idx) << 32) | tri
            prims["type"][sl] = ptype
            if ptype == PRIM_AREA_LIGHT:
                prims["material_index"][sl] = n_surface + first + tri
            else:
                prims["material_index"][sl] = material
            bounds[sl] = triangle_bounds(self.meshes[mesh_idx])
            k += ntri
        if host_bvh:
            nodes, order = build_bvh2(bounds, threads)
            # Reorder whole 32-byte records (a field-wise structured copy would
            # leave the padding bytes undefined).
            raw = prims.view(np.uint8).reshape(-1, F.PRIM_ID_DTYPE.itemsize)[order]
            sorted_prims = np.ascontiguousarray(raw).view(F.PRIM_ID_DTYPE).reshape(-1)
        else:
            nodes, order, sorted_prims = None, np.arange(total, dtype=np.int64), prims
        params = np.zeros((len(mats), MATERIAL_PARAMS_WIDTH), np.float32)
        if self._material_params:
            params[:n_surface] = np.asarray(self._material_params, np.float32)
        return HostScene(meshes=self.meshes, prims=sorted_prims, nodes=nodes, materials=mats,
                         prim_order=order, material_params=params)


def _ply_arrays(mesh_p):
    m = mesh_p.contents
    nv, nf = m.vertex_count, m.face_count

    def arr(ptr, n, cols, dtype):
        if not ptr or n == 0:
            return None if not ptr else np.zeros((0, cols), dtype)
        return np.ctypeslib.as_array(ptr, shape=(n * cols,)).reshape(n, cols).astype(dtype, copy=True)

    out = {"points": arr(m.points, nv, 3, np.float32), "indices": arr(m.indices, nf, 3, np.int32),
           "normals": arr(m.normals, nv, 3, np.float32), "uvs": arr(m.uvs, nv, 2, np.float32),
           "face_indices": None}
    if m.face_indices:
        out["face_indices"] = np.ctypeslib.as_array(m.face_indices, shape=(nf,)).astype(np.int32, copy=True)
    if out["points"] is None:
        out["points"] = np.zeros((0, 3), np.float32)
    if out["indices"] is None:
        out["indices"] = np.zeros((0, 3), np.int32)
    return out


def read_ply(path=None, data=None):
    """A PLY mesh (gzg_ply_read / gzg_ply_parse, the format of
    Shape/PlyMesh.swift) as numpy arrays: points (n, 3) float32, indices
    (m, 3) int32, normals / uvs / face_indices or None."""
    L = F.lib()
    mp = F.C.POINTER(F.PlyMesh)()
    if path is not None:
        F.check(L.gzg_ply_read(str(path).encode(), F.C.byref(mp)))
    else:
        buf = np.frombuffer(bytes(data), np.uint8)
        F.check(L.gzg_ply_parse(F.ptr(buf) if len(buf) else None, len(buf), F.C.byref(mp)))
    try:
        return _ply_arrays(mp)
    finally:
        L.gzg_ply_free(mp)


def write_ply(path, points, indices, normals=None, uvs=None, big_endian=False, list_type="uchar",
              face_indices=None):
    """Writes a binary PLY in one of the layouts read_ply accepts (test and
    tooling helper)."""
    points = np.asarray(points, np.float32).reshape(-1, 3)
    indices = np.asarray(indices, np.int32).reshape(-1, 3)
    end = ">" if big_endian else "<"
    cols = [points]
    props = ["x", "y", "z"]
    if normals is not None:
        cols.append(np.asarray(normals, np.float32).reshape(-1, 3))
        props += ["nx", "ny", "nz"]
    if uvs is not None:
        cols.append(np.asarray(uvs, np.float32).reshape(-1, 2))
        props += ["u", "v"]
    head = ["ply", "format binary_%s_endian 1.0" % ("big" if big_endian else "little"),
            "comment written by gonzales_b200", "element vertex %d" % len(points)]
    head += ["property float %s" % p for p in props]
    head += ["element face %d" % len(indices), "property list %s int vertex_indices" % list_type]
    if face_indices is not None:
        head.append("property int face_indices")
    head.append("end_header")
    vert = np.concatenate(cols, 1).astype(end + "f4")
    ct = np.dtype(end + ("u1" if list_type == "uchar" else "u4"))
    fields = [("n", ct), ("i", end + "i4", (3,))]
    if face_indices is not None:
        fields.append(("f", end + "i4"))
    faces = np.zeros(len(indices), np.dtype(fields))
    faces["n"] = 3
    faces["i"] = indices
    if face_indices is not None:
        faces["f"] = face_indices
    with open(path, "wb") as fh:
        fh.write(("\n".join(head) + "\n").encode())
        fh.write(vert.tobytes())
        fh.write(faces.tobytes())
