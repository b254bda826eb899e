// device.cuh - device-side scene view, leaf tests and ray/hit I/O shared by the
// traversal kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gzg.h"

namespace gzg {

// Error bits kernels OR into the scene's error word instead of trapping.
enum : uint32_t {
        kErrStackOverflow = 1u,
        kErrStepCap = 2u,
        kErrBadIndex = 4u,
};

struct DevScene {
        const uint4 *wide;        // WideNode records, 5 x uint4 each
        const float4 *tv0, *tv1, *tv2;  // leaf-order triangles (tv0.w = prim index bits)
        const float4 *bvh2;       // reference BVH2Node records, 2 x float4 each
        const float4 *pv0, *pv1, *pv2;  // triangles in prim-array order (pv0.w = 1 if intersectable)
        const gzg_prim_id *prims;
        int64_t bvh2_count;
        int64_t prim_count;
        uint32_t wide_count;
        uint32_t *err;
        unsigned long long *counters;  // optional fetch counters (nodes, triangles, rays)
        uint32_t *sched;               // persistent kernels: per-launch pull counter (zero at launch) or null
        const uint32_t *n_dev;         // optional device-side ray count (overrides the launch's n)
        // shading data (path integrator)
        const float4 *materials;       // 2 x float4 per material: albedo + type, emission
        const float4 *mat_params;      // per material 3 x float4 (gzg_material_params; null: none)
        // per prim 5 x float4: vertex normals n0, n1, n2 (n0.w = int 1 when
        // set), UVs (u0, v0, u1, v1), (u2, v2, int 1 when set, 0); null: none
        const float4 *attr;
        const float4 *lights;          // 4 x float4 per area light: p0 + area, p1 + power, p2, emission
        const float *light_cdf;        // running sum of light powers
        int32_t material_count;
        int32_t light_count;
        float light_total_power;
        // the host's meshes on the device (TriangleMesh_C with device pointers)
        const gzg_triangle_mesh *meshes;
        const int64_t *mesh_sizes;     // per mesh: point floats, vertex indices
        int64_t mesh_count;
        // two-level scenes: per instance 4 x float4 (world_to_object rows,
        // then bottom-level root node index and scene index as int bits)
        const float4 *instances;
        int64_t instance_count;
        int32_t *inst_out;             // per-launch output of hit instances (optional)
        // batches of scenes: a device ray's spare lane (gzg_ray_d.pad_) holds
        // the wide-node index its traversal starts at
        int32_t per_ray_root;
        // two-level shading: per instance object_to_world rows (3 x float4),
        // per bottom-level scene the first index of its prims in pv0/1/2 and
        // prims (materials already offset)
        const float4 *inst_o2w;
        const int32_t *blas_prim_base;
        // environment light (gzg_scene_set_environment): map env_w x env_h RGB,
        // 1024 x 1024 distribution (function, cdf 1025 per row, row integrals),
        // marginal function, cdf and integral, and the light's power
        const float *env_rgb;
        int32_t env_w, env_h;
        const float *env_func, *env_cdf, *env_row_int, *env_marg_func, *env_marg_cdf;
        float env_marg_int;
        float env_power;
};

// The launch's ray count: the device-side count when one is given.
__device__ __forceinline__ int64_t ray_count(const DevScene &s, int64_t n) {
        return s.n_dev ? (int64_t)*s.n_dev : n;
}

// Adds per-thread fetch counts into s.counters (one atomic per converged
// group of lanes; __reduce_add_sync is exact for any active mask).
__device__ __forceinline__ void add_counters(const DevScene &s, uint32_t nodes, uint32_t tris, uint32_t rays) {
        if (s.counters == nullptr) return;
        const unsigned mask = __activemask();
        const unsigned n = __reduce_add_sync(mask, nodes);
        const unsigned t = __reduce_add_sync(mask, tris);
        const unsigned r = __reduce_add_sync(mask, rays);
        if ((threadIdx.x & 31) == (unsigned)(__ffs(mask) - 1)) {
                atomicAdd(s.counters, (unsigned long long)n);
                atomicAdd(s.counters + 1, (unsigned long long)t);
                atomicAdd(s.counters + 2, (unsigned long long)r);
        }
}

// ------------------------------------------------------------ leaf tests

// Moller-Trumbore exactly as kernel.mojo:122-156: cross/dot of :84-95 with
// every product and sum rounded separately (the _rn intrinsics are never
// contracted into FMA), 1/det by IEEE division, |det| < 1e-7 rejected,
// t <= 0 or t > tMax rejected (so a later triangle at equal t wins).
__device__ __forceinline__ bool mt_test(float ox, float oy, float oz, float dx, float dy, float dz, const float4 &a,
                                        const float4 &b, const float4 &c, float tmax, float &t, float &u,
                                        float &v) {
        const float e1x = __fsub_rn(b.x, a.x), e1y = __fsub_rn(b.y, a.y), e1z = __fsub_rn(b.z, a.z);
        const float e2x = __fsub_rn(c.x, a.x), e2y = __fsub_rn(c.y, a.y), e2z = __fsub_rn(c.z, a.z);
        const float px = __fsub_rn(__fmul_rn(dy, e2z), __fmul_rn(dz, e2y));
        const float py = __fsub_rn(__fmul_rn(dz, e2x), __fmul_rn(dx, e2z));
        const float pz = __fsub_rn(__fmul_rn(dx, e2y), __fmul_rn(dy, e2x));
        const float det = __fadd_rn(__fadd_rn(__fmul_rn(e1x, px), __fmul_rn(e1y, py)), __fmul_rn(e1z, pz));
        if (det > -1e-7f && det < 1e-7f) return false;
        const float inv = __fdiv_rn(1.0f, det);
        const float tx = __fsub_rn(ox, a.x), ty = __fsub_rn(oy, a.y), tz = __fsub_rn(oz, a.z);
        const float uu = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(tx, px), __fmul_rn(ty, py)), __fmul_rn(tz, pz)), inv);
        if (uu < 0.0f || uu > 1.0f) return false;
        const float qx = __fsub_rn(__fmul_rn(ty, e1z), __fmul_rn(tz, e1y));
        const float qy = __fsub_rn(__fmul_rn(tz, e1x), __fmul_rn(tx, e1z));
        const float qz = __fsub_rn(__fmul_rn(tx, e1y), __fmul_rn(ty, e1x));
        const float vv = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, qx), __fmul_rn(dy, qy)), __fmul_rn(dz, qz)), inv);
        if (vv < 0.0f || __fadd_rn(uu, vv) > 1.0f) return false;
        const float tt =
            __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(e2x, qx), __fmul_rn(e2y, qy)), __fmul_rn(e2z, qz)), inv);
        if (tt <= 0.0f || tt > tmax) return false;
        t = tt;
        u = uu;
        v = vv;
        return true;
}

__device__ __forceinline__ float pick3(float x, float y, float z, int k) { return k == 0 ? x : (k == 1 ? y : z); }

// Watertight test as Triangle.getIntersectionData (Shape/Triangle.swift:269-352),
// in its operation order; (u, v) = (b1, b2) so b0 = 1 - u - v as MT.
__device__ __forceinline__ bool watertight_test(float ox, float oy, float oz, float dx, float dy, float dz,
                                                const float4 &a, const float4 &b, const float4 &c, float tmax,
                                                float &t, float &u, float &v) {
        const float adx = fabsf(dx), ady = fabsf(dy), adz = fabsf(dz);
        const int kz = (adx > ady) ? ((adx > adz) ? 0 : 2) : ((ady > adz) ? 1 : 2);
        const int kx = kz == 2 ? 0 : kz + 1;
        const int ky = kx == 2 ? 0 : kx + 1;
        const float a0x = __fsub_rn(a.x, ox), a0y = __fsub_rn(a.y, oy), a0z = __fsub_rn(a.z, oz);
        const float a1x = __fsub_rn(b.x, ox), a1y = __fsub_rn(b.y, oy), a1z = __fsub_rn(b.z, oz);
        const float a2x = __fsub_rn(c.x, ox), a2y = __fsub_rn(c.y, oy), a2z = __fsub_rn(c.z, oz);
        const float Dx = pick3(dx, dy, dz, kx), Dy = pick3(dx, dy, dz, ky), Dz = pick3(dx, dy, dz, kz);
        float q0x = pick3(a0x, a0y, a0z, kx), q0y = pick3(a0x, a0y, a0z, ky), q0z = pick3(a0x, a0y, a0z, kz);
        float q1x = pick3(a1x, a1y, a1z, kx), q1y = pick3(a1x, a1y, a1z, ky), q1z = pick3(a1x, a1y, a1z, kz);
        float q2x = pick3(a2x, a2y, a2z, kx), q2y = pick3(a2x, a2y, a2z, ky), q2z = pick3(a2x, a2y, a2z, kz);
        const float sx = __fdiv_rn(-Dx, Dz);
        const float sy = __fdiv_rn(-Dy, Dz);
        const float sz = __fdiv_rn(1.0f, Dz);
        q0x = __fadd_rn(q0x, __fmul_rn(sx, q0z));
        q0y = __fadd_rn(q0y, __fmul_rn(sy, q0z));
        q1x = __fadd_rn(q1x, __fmul_rn(sx, q1z));
        q1y = __fadd_rn(q1y, __fmul_rn(sy, q1z));
        q2x = __fadd_rn(q2x, __fmul_rn(sx, q2z));
        q2y = __fadd_rn(q2y, __fmul_rn(sy, q2z));
        const float e0 = __fsub_rn(__fmul_rn(q1x, q2y), __fmul_rn(q1y, q2x));
        const float e1 = __fsub_rn(__fmul_rn(q2x, q0y), __fmul_rn(q2y, q0x));
        const float e2 = __fsub_rn(__fmul_rn(q0x, q1y), __fmul_rn(q0y, q1x));
        if ((e0 < 0.0f || e1 < 0.0f || e2 < 0.0f) && (e0 > 0.0f || e1 > 0.0f || e2 > 0.0f)) return false;
        const float det = __fadd_rn(__fadd_rn(e0, e1), e2);
        if (det == 0.0f) return false;
        q0z = __fmul_rn(q0z, sz);
        q1z = __fmul_rn(q1z, sz);
        q2z = __fmul_rn(q2z, sz);
        const float ts = __fadd_rn(__fadd_rn(__fmul_rn(e0, q0z), __fmul_rn(e1, q1z)), __fmul_rn(e2, q2z));
        const float lim = __fmul_rn(tmax, det);
        if (det > 0.0f) {
                if (ts <= 0.0f || ts > lim) return false;
        } else {
                if (ts >= 0.0f || ts < lim) return false;
        }
        const float inv = __fdiv_rn(1.0f, det);
        u = __fmul_rn(e1, inv);
        v = __fmul_rn(e2, inv);
        t = __fmul_rn(ts, inv);
        return true;
}

template <int LEAF>
__device__ __forceinline__ bool leaf_test(float ox, float oy, float oz, float dx, float dy, float dz, const float4 &a,
                                          const float4 &b, const float4 &c, float tmax, float &t, float &u, float &v) {
        if (LEAF == GZG_LEAF_WATERTIGHT) return watertight_test(ox, oy, oz, dx, dy, dz, a, b, c, tmax, t, u, v);
        return mt_test(ox, oy, oz, dx, dy, dz, a, b, c, tmax, t, u, v);
}

// ------------------------------------------------------------ ray input

enum RayFormat { kRayDevice = 0, kRayReference = 1 };

struct RayIn {
        float ox, oy, oz, dx, dy, dz, tmax;
        uint32_t root;  // device rays: bits of the spare lane (traversal root in batches)
};

template <int FMT>
__device__ __forceinline__ RayIn load_ray(const void *rays, const float *tmax, int64_t i) {
        RayIn r;
        if (FMT == kRayDevice) {
                const float4 *p = reinterpret_cast<const float4 *>(rays) + 2 * i;
                const float4 a = __ldcs(p), b = __ldcs(p + 1);
                r.ox = a.x;
                r.oy = a.y;
                r.oz = a.z;
                r.tmax = a.w;
                r.dx = b.x;
                r.dy = b.y;
                r.dz = b.z;
                r.root = __float_as_uint(b.w);
        } else {
                const float2 *p = reinterpret_cast<const float2 *>(reinterpret_cast<const char *>(rays) + 24 * i);
                const float2 a = __ldcs(p), b = __ldcs(p + 1), c = __ldcs(p + 2);
                r.ox = a.x;
                r.oy = a.y;
                r.oz = b.x;
                r.dx = b.y;
                r.dy = c.x;
                r.dz = c.y;
                r.tmax = __ldcs(tmax + i);
                r.root = 0u;
        }
        return r;
}

// ------------------------------------------------------------ hit output

enum OutFormat { kOutHit = 0, kOutIntersection = 1, kOutAnyPrim = 2, kOutOccluded = 3 };

template <int FMT>
__device__ __forceinline__ void store_hit(const DevScene &s, void *out, int64_t i, int prim, float t, float u, float v) {
        if (FMT == kOutHit) {
                __stcs(reinterpret_cast<float4 *>(out) + i, make_float4(t, u, v, __int_as_float(prim)));
        } else if (FMT == kOutIntersection) {
                uint4 *o = reinterpret_cast<uint4 *>(reinterpret_cast<char *>(out) + 48 * i);
                uint4 w0, w1;
                if (prim >= 0) {
                        const uint4 *src = reinterpret_cast<const uint4 *>(s.prims + prim);
                        // the whole 32-byte PrimId_C, padding included, as the
                        // reference copies the struct (kernel.mojo:360-361)
                        w0 = __ldg(src);
                        w1 = __ldg(src + 1);
                } else {
                        w0 = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
                        w1 = make_uint4(0u, 0u, 0u, 0u);
                }
                __stcs(o, w0);
                __stcs(o + 1, w1);
                __stcs(o + 2, make_uint4(__float_as_uint(t), __float_as_uint(u), __float_as_uint(v), prim >= 0 ? 1u : 0u));
        } else if (FMT == kOutAnyPrim) {
                __stcs(reinterpret_cast<int *>(out) + i, prim);
        } else {
                reinterpret_cast<uint8_t *>(out)[i] = prim >= 0 ? 1 : 0;
        }
}

}  // namespace gzg
