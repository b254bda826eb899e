"""Seeded synthetic workloads (no scene files are available offline).

  ray-cast workload:  an icosphere subdivided `subdiv` times (20 * 4**subdiv
      triangles; 1,310,720 at subdiv 8) displaced radially by 1 + 0.05 * n(p),
      n = 3-octave seeded value noise in [-1, 1]; coherent pinhole rays at
      width x height pixel centres with seeded jitter, plus incoherent rays with
      origins uniform in the mesh bounds, directions uniform on the sphere and
      tMax uniform in [0.1, 2] * |bounds diagonal|.
  box scene: five inward walls of the unit cube, two rotated boxes with seeded
      sizes in [0.2, 0.35], a ceiling area-light quad with radiance (15, 11, 4),
      diffuse albedo uniform in [0.1, 0.8]^3 per object.
"""
import math

import numpy as np

from .scene import SceneBuilder

# ---------------------------------------------------------------- icosphere


def icosphere(subdiv):
    """Unit icosphere: (points (V, 3) float64, triangles (F, 3) int64)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(subdiv):
        nv = len(v)
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        lo = np.minimum(e[:, 0], e[:, 1])
        hi = np.maximum(e[:, 0], e[:, 1])
        key = lo * nv + hi
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // nv, uniq % nv
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        v = np.concatenate([v, mid])
        nf = len(f)
        m01 = inv[:nf] + nv
        m12 = inv[nf:2 * nf] + nv
        m20 = inv[2 * nf:] + nv
        f = np.concatenate([
            np.stack([f[:, 0], m01, m20], 1),
            np.stack([f[:, 1], m12, m01], 1),
            np.stack([f[:, 2], m20, m12], 1),
            np.stack([m01, m12, m20], 1),
        ])
    return v, f


def _hash3(ix, iy, iz, seed):
    h = (ix.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)) ^ (iy.astype(np.uint64) * np.uint64(0xC2B2AE3D27D4EB4F))
    h ^= iz.astype(np.uint64) * np.uint64(0x165667B19E3779F9)
    h ^= np.uint64(seed) * np.uint64(0x27D4EB2F165667C5)
    h ^= h >> np.uint64(31)
    h *= np.uint64(0xBF58476D1CE4E5B9)
    h ^= h >> np.uint64(29)
    return (h >> np.uint64(11)).astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0  # [-1, 1)


def value_noise(p, seed, octaves=3, base_freq=4.0):
    """Seeded value noise: trilinear interpolation of lattice values with a
    smoothstep fade, summed over octaves (frequency x2, amplitude /2) and
    normalised to [-1, 1]."""
    total = np.zeros(len(p))
    norm = 0.0
    for o in range(octaves):
        freq = base_freq * (2 ** o)
        amp = 0.5 ** o
        q = p * freq
        i0 = np.floor(q).astype(np.int64)
        fr = q - i0
        w = fr * fr * (3 - 2 * fr)
        acc = np.zeros(len(p))
        with np.errstate(over="ignore"):
            for dx in (0, 1):
                for dy in (0, 1):
                    for dz in (0, 1):
                        val = _hash3(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz, seed * 131 + o)
                        wx = w[:, 0] if dx else 1 - w[:, 0]
                        wy = w[:, 1] if dy else 1 - w[:, 1]
                        wz = w[:, 2] if dz else 1 - w[:, 2]
                        acc += val * wx * wy * wz
        total += amp * acc
        norm += amp
    return total / norm


def displaced_icosphere(subdiv=8, amplitude=0.05, seed=0xC1):
    v, f = icosphere(subdiv)
    r = 1.0 + amplitude * value_noise(v, seed)
    return (v * r[:, None]).astype(np.float32), f


def raycast_scene(subdiv=8, seed=0xC1):
    """One displaced icosphere as a single mesh of geometric prims."""
    pts, tris = displaced_icosphere(subdiv, seed=seed)
    sb = SceneBuilder()
    mat = sb.add_material((0.5, 0.5, 0.5))
    sb.add_mesh(pts, tris, mat)
    return sb


# ---------------------------------------------------------------- rays


def _normalize(d):
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def coherent_rays(width, height, seed, eye=(0.0, 0.0, 3.2), fov_deg=45.0):
    """Pinhole rays through pixel centres + seeded jitter, looking at the origin."""
    rng = np.random.default_rng(seed)
    n = width * height
    px = np.arange(n, dtype=np.int64) % width
    py = np.arange(n, dtype=np.int64) // width
    jx = rng.uniform(-0.5, 0.5, n)
    jy = rng.uniform(-0.5, 0.5, n)
    tan_half = math.tan(math.radians(fov_deg) / 2.0)
    aspect = width / height
    sx = ((px + 0.5 + jx) / width * 2.0 - 1.0) * tan_half * aspect
    sy = (1.0 - (py + 0.5 + jy) / height * 2.0) * tan_half
    d = _normalize(np.stack([sx, sy, -np.ones(n)], 1))
    o = np.broadcast_to(np.asarray(eye, np.float64), (n, 3))
    t = np.full(n, np.inf)
    return o, d, t


def incoherent_rays(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    o = lo + (hi - lo) * rng.random((n, 3))
    d = _normalize(rng.normal(size=(n, 3)))
    diag = float(np.linalg.norm(hi - lo))
    t = rng.uniform(0.1, 2.0, n) * diag
    return o, d, t


def pack_device_rays(o, d, t):
    """(n, 8) float32: origin, tMax, direction, 0 (gzg_ray_d)."""
    n = len(t)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = t
    r[:, 4:7] = d
    return r


def pack_reference_rays(o, d):
    """(n, 6) float32 Ray_C records."""
    r = np.empty((len(o), 6), np.float32)
    r[:, 0:3] = o
    r[:, 3:6] = d
    return r


def raycast_rays(host_scene, n_coherent_w, n_coherent_h, n_incoherent, seed=0xC1):
    """Coherent rays then incoherent rays, as float32 arrays (o, d, tmax)."""
    o1, d1, t1 = coherent_rays(n_coherent_w, n_coherent_h, seed + 1)
    pts = np.concatenate([m.points[:, :3] for m in host_scene.meshes])
    o2, d2, t2 = incoherent_rays(n_incoherent, pts.min(0), pts.max(0), seed + 2)
    o = np.concatenate([o1, o2]).astype(np.float32)
    d = np.concatenate([d1, d2]).astype(np.float32)
    t = np.concatenate([t1, t2]).astype(np.float32)
    return o, d, t


# ---------------------------------------------------------------- instanced scene


def grid_mesh(kind, n_u, n_v, seed, amplitude=0.05):
    """A displaced tube (open cylinder, radius 0.3, height 1) or lat-long sphere
    (radius 0.5) with n_u x n_v quads (2 * n_u * n_v triangles)."""
    u = np.arange(n_u) / n_u * 2 * math.pi
    if kind == "tube":
        v = np.linspace(-0.5, 0.5, n_v + 1)
        uu, vv = np.meshgrid(u, v, indexing="ij")
        p = np.stack([0.3 * np.cos(uu), vv, 0.3 * np.sin(uu)], -1).reshape(-1, 3)
        normal = np.stack([np.cos(uu), np.zeros_like(uu), np.sin(uu)], -1).reshape(-1, 3)
    else:
        v = np.linspace(0.02, math.pi - 0.02, n_v + 1)
        uu, vv = np.meshgrid(u, v, indexing="ij")
        normal = np.stack([np.sin(vv) * np.cos(uu), np.cos(vv), np.sin(vv) * np.sin(uu)], -1).reshape(-1, 3)
        p = 0.5 * normal
    p = p + normal * (amplitude * value_noise(p * 2.0, seed))[:, None]
    i = np.arange(n_u)[:, None]
    j = np.arange(n_v)[None, :]
    a = i * (n_v + 1) + j
    b = ((i + 1) % n_u) * (n_v + 1) + j
    tris = np.stack([np.stack([a, b, a + 1], -1), np.stack([b, b + 1, a + 1], -1)], 2).reshape(-1, 3)
    return p.astype(np.float32), tris.astype(np.int64)


def random_instances(n, n_blas, seed, extent=20.0):
    """Instances with seeded affine transforms: uniform random rotation, uniform
    scale in [0.5, 2], translation uniform in [-extent, extent]^3."""
    from ._ffi import INSTANCE_DTYPE

    rng = np.random.default_rng(seed)
    inst = np.zeros(n, INSTANCE_DTYPE)
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)
    s = rng.uniform(0.5, 2.0, n)
    t = rng.uniform(-extent, extent, (n, 3))
    M = np.zeros((n, 4, 4))
    M[:, :3, :3] = R * s[:, None, None]
    M[:, :3, 3] = t
    M[:, 3, 3] = 1.0
    Minv = np.linalg.inv(M)
    inst["object_to_world"] = M[:, :3, :].reshape(n, 12).astype(np.float32)
    inst["world_to_object"] = Minv[:, :3, :].reshape(n, 12).astype(np.float32)
    inst["blas"] = rng.integers(0, n_blas, n)
    return inst


MIXED_KINDS = ("diffuse", "coateddiffuse", "dielectric", "conductor", "coatedconductor")


def instanced_scene(n_meshes=16, n_u=125, n_v=200, n_instances=4096, seed=0xC2, extent=20.0, coloured=False,
                    mixed=False):
    """Bottom-level scenes (one mesh each: tubes and spheres alternating) and
    instances; 2 * n_u * n_v triangles per mesh (50,000 at the defaults).
    coloured: a seeded diffuse albedo in [0.1, 0.8]^3 per mesh (else 0.5).
    mixed: mesh k is diffuse, coated diffuse, dielectric, conductor (copper)
    or coated conductor (k mod 5), eta 1.5, roughness uniform in [0.05, 0.5]
    (coating and conductor alike), coating thickness 0.01 (implies
    coloured)."""
    rng = np.random.default_rng(seed + 101)
    blas = []
    for k in range(n_meshes):
        pts, tris = grid_mesh("tube" if k % 2 == 0 else "sphere", n_u, n_v, seed + k)
        sb = SceneBuilder()
        albedo = rng.uniform(0.1, 0.8, 3) if (coloured or mixed) else (0.5, 0.5, 0.5)
        if mixed:
            rough = float(rng.uniform(0.05, 0.5))
            m = sb.add_material(albedo, kind=MIXED_KINDS[k % len(MIXED_KINDS)], eta=1.5, roughness=rough,
                                thickness=0.01, conductor_roughness=rough)
        else:
            m = sb.add_material(albedo)
        sb.add_mesh(pts, tris, m)
        blas.append(sb.build())
    return blas, random_instances(n_instances, n_meshes, seed, extent)


def equal_area_square_to_sphere(u, v):
    """numpy form of InfiniteLight.equalAreaSquareToSphere (for building maps)."""
    ru, rv = 2 * u - 1, 2 * v - 1
    au, av = np.abs(ru), np.abs(rv)
    sd = 1 - (au + av)
    r = 1 - np.abs(sd)
    with np.errstate(divide="ignore", invalid="ignore"):
        phi = np.where(r == 0, 1.0, (av - au) / np.where(r == 0, 1.0, r) + 1) * (np.pi / 4)
    z = np.copysign(np.maximum(0.0, 1 - r * r), sd)
    return np.stack([np.copysign(r * np.cos(phi), ru), np.copysign(r * np.sin(phi), rv), z], -1)


def sky_map(width=1024, height=512, seed=0xE1, sun_sigma_deg=3.0):
    """Seeded environment map in the equal-area square layout the environment
    light reads: a sky gradient over +y (horizon to zenith), a dim ground
    below the horizon, and a Gaussian sun lobe at a seeded direction."""
    rng = np.random.default_rng(seed)
    v, u = np.meshgrid((np.arange(height) + 0.5) / height, (np.arange(width) + 0.5) / width, indexing="ij")
    d = equal_area_square_to_sphere(u, v)
    d = d / np.linalg.norm(d, axis=-1, keepdims=True)  # the light looks maps up by unit direction
    up = d[..., 1]
    zenith = np.array([0.25, 0.45, 0.9])
    horizon = np.array([0.9, 0.95, 1.0])
    ground = np.array([0.12, 0.1, 0.08])
    t = np.clip(up, 0, 1)[..., None]
    sky = horizon * (1 - t) + zenith * t
    rgb = np.where(up[..., None] >= 0, sky, ground)
    el = rng.uniform(0.35, 0.9)
    az = rng.uniform(0, 2 * np.pi)
    sun = np.array([np.cos(el) * np.cos(az), np.sin(el), np.cos(el) * np.sin(az)])
    cosang = np.clip(d @ sun, -1, 1)
    ang = np.arccos(cosang)
    sigma = np.deg2rad(sun_sigma_deg)
    rgb = rgb + np.array([60.0, 55.0, 45.0]) * np.exp(-(ang ** 2) / (2 * sigma ** 2))[..., None]
    return rgb.astype(np.float32)


def instanced_rays(n, extent, seed):
    """Rays through the instance field: origins uniform in a box 1.2x the
    instance extent, directions uniform on the sphere, tMax = infinity."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(-1.2 * extent, 1.2 * extent, (n, 3))
    d = _normalize(rng.normal(size=(n, 3)))
    return o.astype(np.float32), d.astype(np.float32), np.full(n, np.inf, np.float32)


# ---------------------------------------------------------------- box scene


def _quad(p0, p1, p2, p3):
    return np.array([p0, p1, p2, p3], np.float64), np.array([[0, 1, 2], [0, 2, 3]], np.int64)


def _box(size, angle, center):
    s = size / 2.0
    c, si = math.cos(angle), math.sin(angle)
    corners = np.array([[x, y, z] for x in (-s, s) for y in (-s, s) for z in (-s, s)], np.float64)
    rot = np.array([[c, 0, si], [0, 1, 0], [-si, 0, c]])
    pts = corners @ rot.T + np.asarray(center)
    tris = np.array([[0, 1, 3], [0, 3, 2], [4, 6, 7], [4, 7, 5], [0, 4, 5], [0, 5, 1], [2, 3, 7], [2, 7, 6],
                     [0, 2, 6], [0, 6, 4], [1, 5, 7], [1, 7, 3]], np.int64)
    return pts, tris


def box_scene(seed=0xB0):
    """Unit cube [0,1]^3 open toward +z (camera side), two boxes, ceiling light."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    walls = [
        _quad((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1)),   # floor y=0
        _quad((0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0)),   # ceiling y=1
        _quad((0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0)),   # back z=0
        _quad((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0)),   # left x=0
        _quad((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1)),   # right x=1
    ]
    pts = np.concatenate([w[0] for w in walls])
    tris = np.concatenate([w[1] + 4 * i for i, w in enumerate(walls)])
    sb.add_mesh(pts, tris, sb.add_material(rng.uniform(0.1, 0.8, 3)))
    for cx, cz in ((0.3, 0.35), (0.68, 0.62)):
        size = rng.uniform(0.2, 0.35)
        ang = rng.uniform(0, math.pi / 2)
        bp, bt = _box(size, ang, (cx, size / 2.0 + 1e-4, cz))
        sb.add_mesh(bp, bt, sb.add_material(rng.uniform(0.1, 0.8, 3)))
    # wound so cross(p1 - p0, p2 - p0) points down (-y): area lights emit on
    # the side their geometric normal faces
    lp, lt = _quad((0.35, 0.999, 0.35), (0.65, 0.999, 0.35), (0.65, 0.999, 0.65), (0.35, 0.999, 0.65))
    sb.add_area_light(lp, lt, (15.0, 11.0, 4.0))
    return sb


def materials_box_scene(seed=0xB1):
    """The box scene with the renderer's other materials: a coated-diffuse box
    (roughness 0.2), a rough dielectric box (0.1), a smooth dielectric sphere
    (specular), a rough coated sphere (0.4), a copper sphere (alpha 0.15) and
    a coated-conductor box (coating 0.05, conductor 0.3), diffuse walls,
    ceiling light."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    _room(sb, rng)
    bp, bt = _box(0.25, 0.4, (0.3, 0.125 + 1e-4, 0.35))
    sb.add_mesh(bp, bt, sb.add_material(rng.uniform(0.1, 0.8, 3), kind="coateddiffuse", roughness=0.2,
                                        thickness=0.01))
    bp, bt = _box(0.3, 1.1, (0.7, 0.15 + 1e-4, 0.6))
    sb.add_mesh(bp, bt, sb.add_material(kind="dielectric", eta=1.5, roughness=0.1))
    sp, st = icosphere(3)
    sb.add_mesh(sp * 0.12 + np.array([0.62, 0.5, 0.75]), st, sb.add_material(kind="dielectric", eta=1.33,
                                                                               roughness=0.0))
    sb.add_mesh(sp * 0.1 + np.array([0.3, 0.36, 0.4]), st,
                sb.add_material(rng.uniform(0.1, 0.8, 3), kind="coateddiffuse", eta=1.5, roughness=0.4,
                                thickness=0.05))
    sb.add_mesh(sp * 0.09 + np.array([0.18, 0.09, 0.75]), st,
                sb.add_material(kind="conductor", conductor_roughness=0.15))
    bp, bt = _box(0.14, 0.7, (0.82, 0.07 + 1e-4, 0.25))
    sb.add_mesh(bp, bt, sb.add_material((0.9, 0.8, 0.5), kind="coatedconductor", eta=1.5, roughness=0.05,
                                        thickness=0.02, conductor_roughness=0.3))
    lp, lt = _quad((0.35, 0.999, 0.35), (0.65, 0.999, 0.35), (0.65, 0.999, 0.65), (0.35, 0.999, 0.65))
    sb.add_area_light(lp, lt, (15.0, 11.0, 4.0))
    return sb


def smooth_box_scene(seed=0xB2):
    """The box scene with two shaded-smooth meshes: an icosphere with vertex
    normals and spherical UVs (coated diffuse, roughness 0.3) and a coarse
    displaced sphere with vertex normals only (diffuse)."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    _room(sb, rng)
    sp, st = icosphere(2)
    nrm = sp / np.linalg.norm(sp, axis=1, keepdims=True)
    uv = np.stack([0.5 + np.arctan2(nrm[:, 2], nrm[:, 0]) / (2 * np.pi), np.arccos(np.clip(nrm[:, 1], -1, 1)) / np.pi], 1)
    sb.add_mesh(sp * 0.18 + np.array([0.35, 0.18, 0.45]), st,
                sb.add_material(rng.uniform(0.2, 0.8, 3), kind="coateddiffuse", roughness=0.3), normals=nrm, uvs=uv)
    pts, tris = displaced_icosphere(2, amplitude=0.1, seed=7)
    n2 = pts / np.linalg.norm(pts, axis=1, keepdims=True)
    sb.add_mesh(pts * 0.15 + np.array([0.7, 0.16, 0.55]), tris, sb.add_material(rng.uniform(0.2, 0.8, 3)), normals=n2)
    lp, lt = _quad((0.35, 0.999, 0.35), (0.65, 0.999, 0.35), (0.65, 0.999, 0.65), (0.35, 0.999, 0.65))
    sb.add_area_light(lp, lt, (15.0, 11.0, 4.0))
    return sb


# ---------------------------------------------------------------- scene batches

BATCH_SIDES = (64, 128, 256, 512)


def _room(sb, rng):
    """The box scene's five inward walls of the unit cube (10 triangles)."""
    walls = [
        _quad((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1)),
        _quad((0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0)),
        _quad((0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0)),
        _quad((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0)),
        _quad((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1)),
    ]
    pts = np.concatenate([w[0] for w in walls])
    tris = np.concatenate([w[1] + 4 * i for i, w in enumerate(walls)])
    sb.add_mesh(pts, tris, sb.add_material(rng.uniform(0.1, 0.8, 3)))


def _icosphere_cluster(sb, rng, target):
    """Displaced icospheres (20 * 4**s triangles each, s <= 7) whose triangle
    counts add up to about `target`, scattered in the lower half of the room."""
    left = int(target)
    sizes = []
    for s in range(7, 1, -1):
        n = 20 * 4 ** s
        while left >= n:
            sizes.append(s)
            left -= n
    if not sizes:
        sizes.append(2)
    for k, s in enumerate(sizes):
        pts, tris = displaced_icosphere(s, amplitude=0.08, seed=int(rng.integers(1 << 30)))
        radius = 0.09 + 0.16 * rng.random() / math.sqrt(1 + k)
        centre = (rng.uniform(0.2, 0.8), radius + 0.01 + rng.uniform(0.0, 0.3), rng.uniform(0.2, 0.8))
        sb.add_mesh(pts * np.float32(radius) + np.asarray(centre, np.float32), tris,
                    sb.add_material(rng.uniform(0.1, 0.8, 3)))


def _box_stacks(sb, rng, target):
    """About target / 12 small rotated boxes stacked in columns on the floor."""
    n_boxes = max(1, int(target) // 12)
    cols = max(1, int(math.ceil(math.sqrt(n_boxes / 6.0))))
    per_col = int(math.ceil(n_boxes / float(cols * cols)))
    pitch = 0.8 / cols
    size = 0.8 * pitch
    height = min(size, 0.7 / per_col)
    pts_all, tris_all = [], []
    k = 0
    for i in range(cols):
        for j in range(cols):
            for h in range(per_col):
                if k >= n_boxes:
                    break
                c = (0.1 + (i + 0.5) * pitch, (h + 0.5) * height + 1e-4, 0.1 + (j + 0.5) * pitch)
                bp, bt = _box(1.0, rng.uniform(0, math.pi / 2), (0.0, 0.0, 0.0))
                bp = bp * np.array([size * 0.9, height * 0.95, size * 0.9]) + np.asarray(c)
                pts_all.append(bp)
                tris_all.append(bt + 8 * k)
                k += 1
    sb.add_mesh(np.concatenate(pts_all).astype(np.float32), np.concatenate(tris_all),
                sb.add_material(rng.uniform(0.1, 0.8, 3)))


def _ceiling_lights(sb, rng, n_lights):
    """n_lights emissive ceiling quads, wound to face down, total power about
    that of the box scene's light."""
    sides = rng.uniform(0.08, 0.2, n_lights)
    scale = 0.09 / float(np.sum(sides ** 2))
    for s in sides:
        x, z = rng.uniform(0.05, 0.95 - s, 2)
        lp, lt = _quad((x, 0.999, z), (x + s, 0.999, z), (x + s, 0.999, z + s), (x, 0.999, z + s))
        colour = rng.uniform(0.5, 1.0, 3)
        sb.add_area_light(lp, lt, tuple(15.0 * scale * colour / colour.max()))


def batch_scene(seed, target_tris):
    """One scene of the batched workload: the room, about `target_tris`
    triangles of displaced icospheres or box stacks, 1-8 ceiling lights."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    _room(sb, rng)
    if rng.random() < 0.5:
        _icosphere_cluster(sb, rng, target_tris)
    else:
        _box_stacks(sb, rng, target_tris)
    _ceiling_lights(sb, rng, int(rng.integers(1, 9)))
    return sb


def batch_workload(n_scenes=64, seed=0xC3, tri_lo=1_000, tri_hi=500_000, sides=BATCH_SIDES):
    """The scene-batch workload: per scene (builder, image side).  Triangle
    counts are log-uniform in [tri_lo, tri_hi]; sides uniform among `sides`."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        target = math.exp(rng.uniform(math.log(tri_lo), math.log(tri_hi)))
        side = int(rng.choice(sides))
        out.append((batch_scene(int(rng.integers(1 << 62)), target), side))
    return out
