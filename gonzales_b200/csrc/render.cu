// render.cu - the path integrator as a device-resident wavefront over a batch
// of scenes.
//
// Gonzales runs its bounce loop on the host, one tile at a time, shipping rays
// and path states to the plugin and back every bounce (Core/Tile.swift:66-209).
// Here a wave of paths lives in device memory for its whole life:
//
//   generate   Z-Sobol camera sample, Gaussian filter sample, pinhole ray
//   per bounce b = 0 .. max_depth-1:
//     extend   closest hit of the extension queue (k_wide_persistent)
//     [sort]   optional counting sort of the queue by material or scene
//     shade    emission, light choice + light sample (-> shadow queue),
//              MIS BSDF sample (-> probe queue, corrected MIS only),
//              continuation sample, Russian roulette (-> next extension queue)
//     shadow   any hit of the shadow queue, then add unoccluded contributions
//     probe    closest hit of the probe queue, then add emission it reaches
//   accumulate film sums (radiance, its square, filter weight) with atomics
//
// A renderer serves a batch of scenes: each scene has its own camera, film
// window, sampler, lights and BVH root in a per-scene constant table, every
// path carries its scene index, and traversal starts at a per-ray root in one
// concatenated node array.  A single scene is a batch of one that uses the
// scene's own device arrays.  Queue lengths live on the device; no stage waits
// for the host, so a whole wave can be captured as a CUDA graph and replayed.
// The shading arithmetic restates Integrator/VolumePathIntegrator.swift:67-463
// and the helpers it calls (same citations as the CPU oracle's integrator).
// The reference's last extension (bounce == max_depth) can only add
// environment light to camera or specular paths; these scenes have neither, so
// it is not traced.
//
// Differentiable rendering: single-scene renderers may bind albedo textures
// and an emission scale; gzg_renderer_adjoint replays each wave's paths
// (primal pass, then replay with the same samples) and accumulates
// dLoss/dtexel and dLoss/dscale.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "gzg_internal.h"
#include "kernels.h"
#include "sobol.cuh"

namespace gzg {

// An NVTX range (push on construction, pop on end() or destruction), marking
// one wavefront stage's launches for a profiler; a no-op without one.
struct NvtxRange {
        bool open = true;
        explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
        void end() {
                if (open) nvtxRangePop();
                open = false;
        }
        ~NvtxRange() { end(); }
};

}  // namespace gzg

namespace gzg {

const uint32_t *sobol_matrices(size_t *count);

namespace {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInf = __builtin_huge_valf();

// ------------------------------------------------------------ device math

struct V3 {
        float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 v3(const float4 &a) { return V3{a.x, a.y, a.z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 mulv(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 neg(V3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
        return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ V3 normalize(V3 a) {
        const float l = sqrtf(dot(a, a));
        return v3(a.x / l, a.y / l, a.z / l);
}
__device__ __forceinline__ bool is_black(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }

// powerHeuristic (Sampler/Sampling.swift:27-30).
__device__ __forceinline__ float power_heuristic(float f, float g) {
        if (f == 0.0f || g == 0.0f) return 0.0f;
        return (f * f) / (f * f + g * g);
}

// concentricSampleDisk + cosineSampleHemisphere (Sampler/Sampling.swift:3-25).
__device__ void concentric_disk(float u0, float u1, float &dx, float &dy) {
        const float ox = 2.0f * u0 - 1.0f, oy = 2.0f * u1 - 1.0f;
        dx = 0.0f;
        dy = 0.0f;
        if (!(ox == 0.0f && oy == 0.0f)) {
                float theta, r;
                if (fabsf(ox) > fabsf(oy)) {
                        r = ox;
                        theta = (kPi / 4.0f) * (oy / ox);
                } else {
                        r = oy;
                        theta = (kPi / 2.0f) - (kPi / 4.0f) * (ox / oy);
                }
                dx = r * cosf(theta);
                dy = r * sinf(theta);
        }
}

__device__ V3 cosine_hemisphere(float u0, float u1) {
        float dx, dy;
        concentric_disk(u0, u1, dx, dy);
        return v3(dx, dy, sqrtf(fmaxf(0.0f, 1.0f - dx * dx - dy * dy)));
}

// makeCoordinateSystem (Geometry/Geometry.swift:64-77).
__device__ void coordinate_system(V3 v1, V3 &v2, V3 &v3o) {
        if (fabsf(v1.x) > fabsf(v1.y)) {
                const float l = sqrtf(v1.x * v1.x + v1.z * v1.z);
                v2 = v3(-v1.z / l, 0.0f, v1.x / l);
        } else {
                const float l = sqrtf(v1.y * v1.y + v1.z * v1.z);
                v2 = v3(0.0f, v1.z / l, -v1.y / l);
        }
        v3o = cross(v1, v2);
}

struct Frame {
        V3 x, y, z;
        __device__ V3 to_local(V3 v) const { return v3(dot(v, x), dot(v, y), dot(v, z)); }
        __device__ V3 to_world(V3 v) const { return x * v.x + y * v.y + z * v.z; }
};

// The interaction's dpdu of a hit without UVs or vertex normals
// (Shape/Triangle.swift:395-452 with degenerate UVs): false for a degenerate
// triangle.
__device__ bool shading_dpdu(V3 p0, V3 p1, V3 p2, V3 ns, V3 &dpdu_out) {
        const V3 gn = cross(p2 - p0, p1 - p0);
        if (dot(gn, gn) == 0.0f) return false;
        V3 dpdu, dpdv;
        coordinate_system(normalize(gn), dpdu, dpdv);
        V3 s = normalize(dpdu);
        V3 t = cross(s, ns);
        if (dot(t, t) > 0.0f) {
                t = normalize(t);
                s = cross(t, ns);
        } else {
                coordinate_system(ns, s, t);
        }
        dpdu_out = s;
        return true;
}

// BsdfFrame from dpdu and the shading normal (Reflection/BsdfFrame.swift:13-21).
__device__ Frame frame_from(V3 dpdu, V3 ns) {
        Frame f;
        f.y = normalize(dpdu);
        f.z = ns;
        f.x = cross(f.y, f.z);
        return f;
}

__device__ bool make_frame(V3 p0, V3 p1, V3 p2, V3 ns, Frame &f) {
        V3 s;
        if (!shading_dpdu(p0, p1, p2, ns, s)) return false;
        f = frame_from(s, ns);
        return true;
}

// Triangle.computeSurfaceInteraction with vertex normals and / or UVs
// (Shape/Triangle.swift:386-452): dpdu from the UV parametrisation unless it
// is degenerate; the shading normal interpolated from the vertex normals
// (normalised, or (6, 6, 6) when it vanishes); shading tangent from dpdu
// made orthogonal to it.  a = the prim's 5 attribute records.  Returns the
// shading tangent and the shading normal (normalised as the interaction
// stores it), false when the triangle is degenerate.
__device__ bool attr_shading(V3 p0, V3 p1, V3 p2, float b0, float b1, float b2, V3 ng, const float4 a[5],
                             V3 &dpdu_out, V3 &ns_out) {
        const bool has_n = __float_as_int(a[0].w) != 0, has_uv = __float_as_int(a[4].z) != 0;
        const V3 dp02 = p0 - p2, dp12 = p1 - p2;
        const float u0 = has_uv ? a[3].x : 0.0f, v0 = has_uv ? a[3].y : 0.0f;
        const float u1 = has_uv ? a[3].z : 0.0f, v1 = has_uv ? a[3].w : 0.0f;
        const float u2 = has_uv ? a[4].x : 0.0f, v2 = has_uv ? a[4].y : 0.0f;
        const float du02 = u0 - u2, dv02 = v0 - v2, du12 = u1 - u2, dv12 = v1 - v2;
        const float det = du02 * dv12 - dv02 * du12;
        const bool degenerate = fabsf(det) < 1e-8f;
        V3 dpdu = v3(0.0f, 1.0f, 0.0f), dpdv = v3(0.0f, 1.0f, 0.0f);
        if (!degenerate) {
                const float inv = 1.0f / det;
                dpdu = (dp02 * dv12 - dp12 * dv02) * inv;
                dpdv = (dp02 * (-du12) - dp12 * du02) * inv;
        }
        const V3 cuv = cross(dpdu, dpdv);
        if (degenerate || dot(cuv, cuv) == 0.0f) {
                const V3 gn = cross(p2 - p0, p1 - p0);
                if (dot(gn, gn) == 0.0f) return false;
                coordinate_system(normalize(gn), dpdu, dpdv);
        }
        V3 ns = ng;
        if (has_n) {
                const V3 n0 = v3(a[0]), n1 = v3(a[1]), n2 = v3(a[2]);
                ns = n0 * b0 + n1 * b1 + n2 * b2;
                ns = dot(ns, ns) > 0.0f ? normalize(ns) : v3(6.0f, 6.0f, 6.0f);
        }
        V3 sv = normalize(dpdu);
        V3 t = cross(sv, ns);
        if (dot(t, t) > 0.0f) {
                t = normalize(t);
                sv = cross(t, ns);
        } else {
                coordinate_system(ns, sv, t);
        }
        dpdu_out = sv;
        ns_out = normalize(ns);
        return true;
}

// Transform * Point / Vector / Normal (Geometry/Transform.swift:31-65) with a
// 3x4 matrix given as three float4 rows; the normal uses the inverse's columns.
__device__ __forceinline__ V3 xf_pt(float4 a, float4 b, float4 c, V3 p) {
        return v3(__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(a.x, p.x), __fmul_rn(a.y, p.y)), __fmul_rn(a.z, p.z)), a.w),
                  __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(b.x, p.x), __fmul_rn(b.y, p.y)), __fmul_rn(b.z, p.z)), b.w),
                  __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(c.x, p.x), __fmul_rn(c.y, p.y)), __fmul_rn(c.z, p.z)), c.w));
}
__device__ __forceinline__ V3 xf_vec(float4 a, float4 b, float4 c, V3 p) {
        return v3(__fadd_rn(__fadd_rn(__fmul_rn(a.x, p.x), __fmul_rn(a.y, p.y)), __fmul_rn(a.z, p.z)),
                  __fadd_rn(__fadd_rn(__fmul_rn(b.x, p.x), __fmul_rn(b.y, p.y)), __fmul_rn(b.z, p.z)),
                  __fadd_rn(__fadd_rn(__fmul_rn(c.x, p.x), __fmul_rn(c.y, p.y)), __fmul_rn(c.z, p.z)));
}
__device__ __forceinline__ V3 xf_nrm(float4 a, float4 b, float4 c, V3 n) {
        return v3(__fadd_rn(__fadd_rn(__fmul_rn(a.x, n.x), __fmul_rn(b.x, n.y)), __fmul_rn(c.x, n.z)),
                  __fadd_rn(__fadd_rn(__fmul_rn(a.y, n.x), __fmul_rn(b.y, n.y)), __fmul_rn(c.y, n.z)),
                  __fadd_rn(__fadd_rn(__fmul_rn(a.z, n.x), __fmul_rn(b.z, n.y)), __fmul_rn(c.z, n.z)));
}

// erfinv of Filter/GaussianFilter.swift:27-91 (rational start, two Newton steps).
__device__ float erfinv_ref(float y) {
        const float ay = fabsf(y);
        const float two_over_sqrt_pi = 2.0f / sqrtf(kPi);
        float x;
        if (ay <= 0.7f) {
                const float z = y * y;
                float num = -0.140543331f * z + 0.914624893f;
                num = num * z + -1.645349621f;
                num = num * z + 0.886226899f;
                float den = 0.012229801f * z + -0.329097515f;
                den = den * z + 1.442710462f;
                den = den * z + -2.118377725f;
                den = den * z + 1.0f;
                x = y * num / den;
        } else if (ay < 1.0f) {
                const float z = sqrtf(-logf((1.0f - ay) / 2.0f));
                float num = 1.641345311f * z + 3.429567803f;
                num = num * z + -1.624906493f;
                num = num * z + -1.970840454f;
                float den = 1.637067800f * z + 3.543889200f;
                den = den * z + 1.0f;
                x = (signbit(y) ? -1.0f : 1.0f) * num / den;
        } else if (ay == 1.0f) {
                return signbit(y) ? -kInf : kInf;
        } else {
                return __int_as_float(0x7fc00000);
        }
        x -= (erff(x) - y) / (two_over_sqrt_pi * expf(-(x * x)));
        x -= (erff(x) - y) / (two_over_sqrt_pi * expf(-(x * x)));
        return x;
}

// GaussianFilter.sample's sample1D (GaussianFilter.swift:95-111).
__device__ void gaussian_sample_1d(float u, float radius, float sigma, float &x_out, float &density) {
        const float norm = 0.5f * (1.0f + erff(radius / (sigma * sqrtf(2.0f))));
        const float us = (1.0f - norm) + u * (2.0f * norm - 1.0f);
        const float x = sigma * sqrtf(2.0f) * erfinv_ref(2.0f * us - 1.0f);
        const float pdf = expf(-x * x / (2.0f * sigma * sigma)) / (sigma * sqrtf(2.0f * kPi));
        density = pdf / (2.0f * norm - 1.0f);
        x_out = fmaxf(-radius, fminf(radius, x));
}

// GaussianFilter.gaussian (GaussianFilter.swift:15-18).
__device__ float gaussian(float x, float sigma) {
        return 1.0f / sqrtf(2.0f * kPi * sigma * sigma) * expf(-(x * x) / (2.0f * sigma * sigma));
}

#include "bsdf.cuh"

// ------------------------------------------------------------ state

// Per-scene constants of a batch.
struct SceneConst {
        V3 eye, right, up, fwd;
        float tan_half, sx0, sx1, sy0, sy1;
        float filter_radius, filter_sigma;
        float lens_radius, focal_distance;  // thin lens (0: pinhole)
        int32_t width, height, spp, max_depth, rr_min, mis_corrected, first_sample;
        int32_t crop_x0, crop_y0, crop_w, crop_h;  // film window (the whole frame without a crop)
        int32_t light_begin, light_count;  // light_count includes the environment light
        float light_total;
        int32_t env_index;                 // scene-local index of the environment light or -1
        float env_power;
        float film_scale;                  // Film.add: iso / 100
        float max_component;               // clamp of a sample's largest component (0: none)
        int32_t two_sided;                 // area lights emit on both sides (the live shade step's rule)
        int32_t has_medium;                // homogeneous medium box (gzg_medium)
        V3 med_min, med_max, sigma_a, sigma_s;
        float med_g;
        int32_t material_begin;  // the scene's material 0 (area-light hits scatter with it)
        int32_t material_count;
        uint32_t root;            // wide-node root of the scene's tree
        uint32_t film_offset;     // first pixel of the scene in the batch film
        uint64_t path_begin;      // first batch-wide path index of the scene
        ZSobolConfig zs;
};

// ------------------------------------------------------------ medium
// A homogeneous medium filling an axis-aligned box (gzg_scene_set_medium;
// Medium/Homogeneous.swift:5-23, phase function Medium/HenyeyGreenstein.swift:
// 13-39).  The reference's integrator never samples it (VolumePathIntegrator.
// swift:394 hard-codes (white, nil)); these run the branch as meant: each
// segment's part inside the box is sampled for a scattering event before the
// segment is shaded, and shadow rays and MIS probes through the box carry its
// transmittance.  The box boundary scatters nothing (an interface).

// Parametric overlap [t0, t1] of o + t d (t in [0, tmax]) with the box.
__device__ bool medium_overlap(const SceneConst &sc, V3 o, V3 d, float tmax, float &t0, float &t1) {
        float lo = 0.0f, hi = tmax;
        const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
        const float mn[3] = {sc.med_min.x, sc.med_min.y, sc.med_min.z};
        const float mx[3] = {sc.med_max.x, sc.med_max.y, sc.med_max.z};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
                if (dd[a] == 0.0f) {
                        if (oo[a] < mn[a] || oo[a] > mx[a]) return false;
                        continue;
                }
                const float inv = 1.0f / dd[a];
                float tn = (mn[a] - oo[a]) * inv, tf = (mx[a] - oo[a]) * inv;
                if (tn > tf) {
                        const float t = tn;
                        tn = tf;
                        tf = t;
                }
                lo = fmaxf(lo, tn);
                hi = fminf(hi, tf);
        }
        t0 = lo;
        t1 = hi;
        return lo < hi;
}

// Transmittance along the part of [0, tmax] inside the box.
__device__ V3 medium_tr(const SceneConst &sc, V3 o, V3 d, float tmax) {
        float t0, t1;
        if (!sc.has_medium || !medium_overlap(sc, o, d, tmax, t0, t1)) return v3(1.0f, 1.0f, 1.0f);
        const V3 st = sc.sigma_a + sc.sigma_s;
        const float len = (t1 - t0) * sqrtf(dot(d, d));
        return v3(expf(-st.x * len), expf(-st.y * len), expf(-st.z * len));
}

// Homogeneous.sample on the in-box part of [0, tmax]: channel number uc,
// distance number ud.  True with the scattering parameter t when the medium
// is sampled; weight = transmittance x sigma_s / density there, else
// transmittance / density (Homogeneous.swift:19 writes sigma_t where the PBRT
// sampler it restates has sigma_s, which would scatter in a purely absorbing
// medium).
__device__ bool medium_sample(const SceneConst &sc, V3 o, V3 d, float tmax, float uc, float ud, float &t,
                              V3 &weight) {
        float t0, t1;
        weight = v3(1.0f, 1.0f, 1.0f);
        if (!medium_overlap(sc, o, d, tmax, t0, t1)) return false;
        const V3 st = sc.sigma_a + sc.sigma_s;
        const int channel = min((int)(uc * 3.0f), 2);
        const float stc = channel == 0 ? st.x : (channel == 1 ? st.y : st.z);
        const float distance = -logf(1.0f - ud) / stc;
        const float len = sqrtf(dot(d, d));
        const float seg = t1 - t0;
        const float param = fminf(distance / len, seg);
        const bool sampled = param < seg;
        const V3 tr = v3(expf(-st.x * param * len), expf(-st.y * param * len), expf(-st.z * param * len));
        const V3 density = sampled ? mulv(st, tr) : tr;
        const float pdf = (density.x + density.y + density.z) / 3.0f;
        weight = sampled ? mulv(tr, sc.sigma_s) * (1.0f / pdf) : tr * (1.0f / pdf);
        t = t0 + param;
        return sampled;
}

// HenyeyGreenstein.phase (HenyeyGreenstein.swift:13-16).
__device__ float hg_phase(float cos_theta, float g) {
        const float denom = 1.0f + g * g + 2.0f * g * cos_theta;
        return (1.0f / (4.0f * kPi)) * (1.0f - g * g) / (denom * sqrtf(denom));
}

// HenyeyGreenstein.samplePhase (HenyeyGreenstein.swift:18-36): incident
// direction in the frame (makeCoordinateSystem(outgoing), outgoing); value =
// density.
__device__ V3 hg_sample(V3 wo, float g, float u0, float u1, float &value) {
        float cos_theta;
        if (fabsf(g) < 1e-3f) {
                cos_theta = 1.0f - 2.0f * u0;
        } else {
                const float sqr = (1.0f - g * g) / (1.0f + g - 2.0f * g * u0);
                cos_theta = -(1.0f + g * g - sqr * sqr) / (2.0f * g);
        }
        const float sin_theta = sqrtf(fmaxf(0.0f, 1.0f - cos_theta * cos_theta));
        const float phi = 2.0f * kPi * u1;
        V3 v1, v2;
        coordinate_system(wo, v1, v2);
        value = hg_phase(cos_theta, g);
        return v1 * (sin_theta * cosf(phi)) + v2 * (sin_theta * sinf(phi)) + wo * cos_theta;
}

enum {
        kCountExt0 = 0, kCountExt1 = 1, kCountShadow = 2, kCountProbe = 3, kCountWaveBase = 4,
        kCountDielectric = 6, kCountCoated = 7, kCountConductor = 8, kCountCoatedConductor = 9,
        kCountSched = 10,  // pull counter of the wave's trace launches (one after another on its stream)
        kCountWords = 12
};
enum { kStatCamera = 0, kStatExt = 1, kStatShadow = 2, kStatProbe = 3, kStatWaves = 4, kStatWords = 8 };
enum SortKey { kSortNone = 0, kSortMaterial = 1, kSortScene = 2 };

// kRender: film accumulation; kPrimal: keep each path's radiance in Ltot;
// kReplay: path replay with gradients (Ltot from the primal pass of the wave).
enum Mode { kRender = 0, kPrimal = 1, kReplay = 2 };

struct Wave {
        uint32_t capacity;
        uint64_t total_paths;
        const SceneConst *scenes;
        int32_t scene_count;
        // path state, indexed by path slot in the wave
        uint64_t *zs_morton;
        int32_t *zs_dim;
        float4 *thr;
        float4 *L;
        uint32_t *pixel;  // batch film pixel
        uint32_t *scene;
        float *weight;
        // queues
        float4 *q_ray[2];  // gzg_ray_d, 2 x float4 per entry
        uint32_t *q_id[2];
        float4 *hits;
        float4 *sh_ray;
        uint32_t *sh_id;
        float4 *sh_contrib;
        int32_t *sh_occ;
        float4 *pr_ray;
        uint32_t *pr_id;
        float4 *pr_contrib;
        float4 *pr_hits;
        // sort of the extension queue before shading
        int32_t sort_key;
        int32_t key_count;
        uint32_t *key_hist;    // key_count counters, then key_count cursors
        uint32_t *order;       // sorted entry order, capacity
        // shade queues of the general BSDFs (2 x capacity): extension-queue
        // entries that hit a dielectric (from the front of the first half), a
        // coated diffuse (from its back), a conductor (from the front of the
        // second half) or a coated conductor (from its back)
        uint32_t *gen_q;
        uint32_t *counts;      // kCountWords words; wave base as 2 words at kCountWaveBase
        unsigned long long *stats;  // kStatWords
        // differentiable rendering (single-scene renderers)
        const float *tex;          // texels: count x tex_res x tex_res x 3 (row v, column u)
        const int32_t *mat_tex;    // per material: texture index or -1 (null: no textures)
        const float *tex_map;      // per texture: origin, u axis, v axis (9 floats)
        int32_t tex_res;
        float emission_scale;      // multiplies every emission
        int32_t mode;              // Mode
        float4 *Ltot;              // per path slot: radiance of the primal pass (replay input)
        const float *adj_rgb;      // dLoss/dImage per film pixel (3 floats)
        const float *adj_w;        // film weight sums per pixel (image = rgb / w)
        float *d_tex;              // dLoss/dtexel (accumulated)
        double *d_emission;        // dLoss/demission_scale (accumulated)
        // two-level scenes: the instance of each extension and probe hit
        int32_t *hit_inst;
        int32_t *pr_inst;
        // first-hit AOVs per path slot: BSDF albedo and geometric normal
        float4 *alb;
        float4 *nrm;
};

// Appends to a queue with one atomic per converged group of lanes.
// Lanes that reach this together may append to different queues (the shade
// queues of several material kinds from one call site): each group of lanes
// with the same counter takes one atomic and numbers its lanes in order.
__device__ __forceinline__ uint32_t queue_slot(uint32_t *count) {
        const unsigned mask = __activemask();
        const unsigned peers = __match_any_sync(mask, reinterpret_cast<unsigned long long>(count));
        const unsigned lane = threadIdx.x & 31u;
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if ((int)lane == leader) base = atomicAdd(count, (uint32_t)__popc(peers));
        base = __shfl_sync(mask, base, leader);
        return base + __popc(peers & ((1u << lane) - 1u));
}

// A queued ray; the spare lane carries the traversal root of the path's scene.
__device__ __forceinline__ void store_ray(float4 *q, uint32_t slot, V3 o, float tmax, V3 d, uint32_t root) {
        q[2 * slot] = make_float4(o.x, o.y, o.z, tmax);
        q[2 * slot + 1] = make_float4(d.x, d.y, d.z, __uint_as_float(root));
}

__device__ __forceinline__ uint64_t wave_base(const Wave &w) {
        return (uint64_t)w.counts[kCountWaveBase] | ((uint64_t)w.counts[kCountWaveBase + 1] << 32);
}

__device__ __forceinline__ uint32_t wave_count(const Wave &w) {
        const uint64_t base = wave_base(w);
        const uint64_t left = w.total_paths > base ? w.total_paths - base : 0;
        return (uint32_t)(left < w.capacity ? left : w.capacity);
}

// Triangle of a prim from the prim-order float4 streams.
__device__ __forceinline__ void prim_triangle_dev(const DevScene &s, int prim, V3 &p0, V3 &p1, V3 &p2) {
        p0 = v3(__ldg(s.pv0 + prim));
        p1 = v3(__ldg(s.pv1 + prim));
        p2 = v3(__ldg(s.pv2 + prim));
}

// type byte and material index of a PrimId_C record.
__device__ __forceinline__ void prim_info(const DevScene &s, int prim, int &type, int64_t &material) {
        const long long *r = reinterpret_cast<const long long *>(s.prims + prim);
        material = __ldg(r + 2);
        type = (int)(signed char)(__ldg(reinterpret_cast<const unsigned char *>(r + 3)));
}

// The surface interaction of a hit: Triangle.computeSurfaceInteraction
// (Shape/Triangle.swift:363-474); for an instance it is computed in object
// space and carried to world space (Core/Transform+SurfaceInteraction.swift:
// 3-14: position as a point, normals through the inverse, outgoing and dpdu
// as vectors).  gprim is the prim's index in the scene's shading arrays.
struct Surf {
        V3 pos, ng, wo;
        V3 ns;  // shading normal (ng without vertex normals)
        Frame fr;
        bool frame_ok;
        int gprim;
};

__device__ void surface(const DevScene &s, int prim, int inst, float bu, float bv, V3 d, Surf &o) {
        V3 p0, p1, p2;
        const float b0 = (1.0f - bu) - bv;
        if (!s.instances) {
                prim_triangle_dev(s, prim, p0, p1, p2);
                o.pos = p0 * b0 + p1 * bu + p2 * bv;
                o.ng = normalize(cross(p0 - p2, p1 - p2));
                o.wo = normalize(neg(d));
                o.gprim = prim;
                o.ns = o.ng;
                if (s.attr) {
                        float4 a[5];
                        for (int k = 0; k < 5; ++k) a[k] = __ldg(s.attr + 5 * (size_t)prim + k);
                        if (__float_as_int(a[0].w) != 0 || __float_as_int(a[4].z) != 0) {
                                V3 sv;
                                o.frame_ok = attr_shading(p0, p1, p2, b0, bu, bv, o.ng, a, sv, o.ns);
                                if (o.frame_ok) o.fr = frame_from(sv, o.ns);
                                return;
                        }
                }
                o.frame_ok = make_frame(p0, p1, p2, o.ng, o.fr);
                return;
        }
        const float4 w0 = __ldg(s.instances + 4 * inst), w1 = __ldg(s.instances + 4 * inst + 1),
                     w2 = __ldg(s.instances + 4 * inst + 2), w3 = __ldg(s.instances + 4 * inst + 3);
        const float4 o0 = __ldg(s.inst_o2w + 3 * inst), o1 = __ldg(s.inst_o2w + 3 * inst + 1),
                     o2 = __ldg(s.inst_o2w + 3 * inst + 2);
        o.gprim = __ldg(s.blas_prim_base + __float_as_int(w3.y)) + prim;
        prim_triangle_dev(s, o.gprim, p0, p1, p2);
        const V3 pos_o = p0 * b0 + p1 * bu + p2 * bv;
        const V3 n_o = normalize(cross(p0 - p2, p1 - p2));
        const V3 wo_o = normalize(neg(xf_vec(w0, w1, w2, d)));
        V3 s_o = v3(0.0f, 0.0f, 0.0f), ns_o = n_o;
        bool with_attr = false;
        if (s.attr) {
                float4 a[5];
                for (int k = 0; k < 5; ++k) a[k] = __ldg(s.attr + 5 * (size_t)o.gprim + k);
                with_attr = __float_as_int(a[0].w) != 0 || __float_as_int(a[4].z) != 0;
                if (with_attr) o.frame_ok = attr_shading(p0, p1, p2, b0, bu, bv, n_o, a, s_o, ns_o);
        }
        if (!with_attr) o.frame_ok = shading_dpdu(p0, p1, p2, n_o, s_o);
        o.pos = xf_pt(o0, o1, o2, pos_o);
        o.ng = normalize(xf_nrm(w0, w1, w2, n_o));
        o.ns = with_attr ? normalize(xf_nrm(w0, w1, w2, ns_o)) : o.ng;
        o.wo = normalize(xf_vec(o0, o1, o2, wo_o));
        if (o.frame_ok) o.fr = frame_from(xf_vec(o0, o1, o2, s_o), o.ns);
}

// Nearest texel of texture t at p (planar map), as a texel index.
__device__ __forceinline__ int texel_at(const Wave &w, int t, V3 p) {
        const float *mp = w.tex_map + 9 * t;
        const V3 d = p - v3(__ldg(mp), __ldg(mp + 1), __ldg(mp + 2));
        const float u = dot(d, v3(__ldg(mp + 3), __ldg(mp + 4), __ldg(mp + 5)));
        const float v = dot(d, v3(__ldg(mp + 6), __ldg(mp + 7), __ldg(mp + 8)));
        const int R = w.tex_res;
        const int ix = (int)fminf(fmaxf(u * (float)R, 0.0f), (float)(R - 1));
        const int iy = (int)fminf(fmaxf(v * (float)R, 0.0f), (float)(R - 1));
        return (t * R + iy) * R + ix;
}

// ------------------------------------------------------------ environment light
// Light/InfiniteLight.swift:7-160 with PiecewiseConstant1D/2D
// (Core/Distribution1D.swift, Core/Distribution2D.swift).  The map lookup is
// bilinear with clamped edges (the reference goes through OpenImageIO).

__device__ V3 env_lookup(const DevScene &s, float u, float v) {
        const float x = u * (float)s.env_w - 0.5f, y = v * (float)s.env_h - 0.5f;
        const float fx = floorf(x), fy = floorf(y);
        const float ax = x - fx, ay = y - fy;
        const int x0 = min(max((int)fx, 0), s.env_w - 1), x1 = min(max((int)fx + 1, 0), s.env_w - 1);
        const int y0 = min(max((int)fy, 0), s.env_h - 1), y1 = min(max((int)fy + 1, 0), s.env_h - 1);
        float out[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
                const float a = __ldg(s.env_rgb + ((size_t)y0 * s.env_w + x0) * 3 + c);
                const float b = __ldg(s.env_rgb + ((size_t)y0 * s.env_w + x1) * 3 + c);
                const float d = __ldg(s.env_rgb + ((size_t)y1 * s.env_w + x0) * 3 + c);
                const float e = __ldg(s.env_rgb + ((size_t)y1 * s.env_w + x1) * 3 + c);
                const float top = a + (b - a) * ax;
                const float bot = d + (e - d) * ax;
                out[c] = top + (bot - top) * ay;
        }
        return v3(out[0], out[1], out[2]);
}

// equalAreaSquareToSphere (InfiniteLight.swift:118-135): as in the reference,
// x and y lack the sqrt(2 - r^2) factor, so the direction is not unit length.
__device__ V3 env_square_to_sphere(float u, float v) {
        const float ru = 2.0f * u - 1.0f, rv = 2.0f * v - 1.0f;
        const float au = fabsf(ru), av = fabsf(rv);
        const float sd = 1.0f - (au + av);
        const float r = 1.0f - fabsf(sd);
        const float phi = (r == 0.0f ? 1.0f : (av - au) / r + 1.0f) * (kPi / 4.0f);
        const float z = copysignf(fmaxf(0.0f, 1.0f - r * r), sd);
        return v3(copysignf(r * cosf(phi), ru), copysignf(r * sinf(phi), rv), z);
}

// equalAreaSphereToSquare (InfiniteLight.swift:92-116).
__device__ void env_sphere_to_square(V3 d, float &u, float &v) {
        const float x = fabsf(d.x), y = fabsf(d.y), z = fabsf(d.z);
        const float radius = sqrtf(fmaxf(0.0f, 1.0f - z));
        const float a = fmaxf(x, y);
        float b = fminf(x, y);
        b = a == 0.0f ? 0.0f : b / a;
        float phi = atanf(b) * 2.0f / kPi;
        if (x < y) phi = 1.0f - phi;
        float vv = phi * radius;
        float uu = radius - vv;
        if (d.z < 0.0f) {
                const float t = uu;
                uu = 1.0f - vv;
                vv = 1.0f - t;
        }
        u = 0.5f * (copysignf(uu, d.x) + 1.0f);
        v = 0.5f * (copysignf(vv, d.y) + 1.0f);
}

// PiecewiseConstant1D.findInterval over cdf[0..n].
__device__ int env_find_interval(const float *cdf, int n, float u) {
        int lo = 0, hi = n;
        while (lo < hi) {
                const int mid = lo + (hi - lo) / 2;
                if (__ldg(cdf + mid) <= u)
                        lo = mid + 1;
                else
                        hi = mid;
        }
        return min(max(lo - 1, 0), n - 1);
}

// PiecewiseConstant1D.sampleContinuous: value, pdf(value), offset.
__device__ float env_sample_1d(const float *func, const float *cdf, float integral, int n, float u, float &pdf,
                               int &offset) {
        const int o = env_find_interval(cdf, n, u);
        float delta = u - __ldg(cdf + o);
        const float dist = __ldg(cdf + o + 1) - __ldg(cdf + o);
        if (dist > 0.0f) delta = delta / dist;
        const float value = ((float)o + delta) / (float)n;
        const int po = min(max((int)(value * (float)n), 0), n - 1);
        pdf = __ldg(func + po) / integral;
        offset = o;
        return value;
}

// InfiniteLight.sample: direction and map value; returns the solid-angle pdf
// (0: no sample).
__device__ float env_sample(const DevScene &s, float u0, float u1, V3 &dir, V3 &rgb) {
        constexpr int N = 1024;
        float pdf1, pdf0;
        int mo, co;
        const float mv = env_sample_1d(s.env_marg_func, s.env_marg_cdf, s.env_marg_int, N, u1, pdf1, mo);
        const float cv = env_sample_1d(s.env_func + (size_t)mo * N, s.env_cdf + (size_t)mo * (N + 1),
                                       __ldg(s.env_row_int + mo), N, u0, pdf0, co);
        const float map_pdf = pdf0 * pdf1;
        if (map_pdf == 0.0f) {
                dir = rgb = v3(0.0f, 0.0f, 0.0f);
                return 0.0f;
        }
        dir = env_square_to_sphere(cv, mv);
        rgb = env_lookup(s, cv, mv);
        return map_pdf / (4.0f * kPi);
}

// InfiniteLight.probabilityDensityFor: the direction is not normalised.
__device__ float env_pdf(const DevScene &s, V3 d) {
        constexpr int N = 1024;
        float u, v;
        env_sphere_to_square(d, u, v);
        const int col = min(max((int)(u * (float)N), 0), N - 1);
        const int row = min(max((int)(v * (float)N), 0), N - 1);
        return __ldg(s.env_func + (size_t)row * N + col) / s.env_marg_int / (4.0f * kPi);
}

// radianceFromInfinity: normalised direction (a zero vector stays as is).
__device__ V3 env_radiance(const DevScene &s, V3 d) {
        const float l = sqrtf(dot(d, d));
        const V3 n = l != 0.0f ? v3(d.x / l, d.y / l, d.z / l) : d;
        float u, v;
        env_sphere_to_square(n, u, v);
        return env_lookup(s, u, v);
}

// ------------------------------------------------------------ kernels

// Camera sample and ray of one path: Tile.render phase 1 (Core/Tile.swift:
// 27-59) with getCameraSample (Sampler/Sampler.swift:69-82), the Gaussian
// filter sample and PerspectiveCamera.generateRay.  Leaves z after the camera
// and lens dimensions; weight = filter value / filter pdf (Tile.swift:36-40).
__device__ void camera_ray(const SceneConst &sc, uint32_t px, uint32_t py, uint32_t sample, ZSobol &z, V3 &org,
                           V3 &dir, float &weight) {
        zs_start(sc.zs, z, px, py, sample);
        float u0, u1;
        zs_get2d(sc.zs, z, u0, u1);
        float dx, dy, denx, deny;
        gaussian_sample_1d(u0, sc.filter_radius, sc.filter_sigma, dx, denx);
        gaussian_sample_1d(u1, sc.filter_radius, sc.filter_sigma, dy, deny);
        const float fx = (float)px + 0.5f + dx, fy = (float)py + 0.5f + dy;
        float l0, l1;
        zs_get2d(sc.zs, z, l0, l1);  // lens sample (drawn also by a pinhole)
        // raster -> screen -> camera -> world
        const float scx = sc.sx0 + fx / (float)sc.width * (sc.sx1 - sc.sx0);
        const float scy = sc.sy1 - fy / (float)sc.height * (sc.sy1 - sc.sy0);
        V3 dcam = normalize(v3(scx * sc.tan_half, scy * sc.tan_half, 1.0f));
        org = sc.eye;
        if (sc.lens_radius > 0.0f) {
                // PerspectiveCamera.depthOfField (Camera/PerspectiveCamera.swift:25-35):
                // the origin moves to the lens point; as written the new
                // direction is taken from the pinhole origin, so it keeps the
                // pinhole direction (renormalised after scaling to the focal plane)
                float lx, ly;
                concentric_disk(l0, l1, lx, ly);
                lx = sc.lens_radius * lx;
                ly = sc.lens_radius * ly;
                const float ft = sc.focal_distance / dcam.z;
                dcam = normalize(dcam * ft);
                org = sc.eye + sc.right * lx + sc.up * ly;
        }
        dir = sc.right * dcam.x + sc.up * dcam.y + sc.fwd * dcam.z;
        const float ddx = fx - ((float)px + 0.5f), ddy = fy - ((float)py + 0.5f);
        const float fv = fmaxf(0.0f, gaussian(ddx, sc.filter_sigma)) * fmaxf(0.0f, gaussian(ddy, sc.filter_sigma));
        weight = fv / (denx * deny);
}

// generate: Tile.render phase 1 (Core/Tile.swift:27-59).  Batch path p belongs
// to the scene whose [path_begin, next path_begin) holds it; within the scene
// path q is sample q % spp of pixel q / spp.
__global__ void k_generate(Wave w) {
        const uint32_t count = wave_count(w);
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (threadIdx.x == 0 && blockIdx.x == 0) {
                w.counts[kCountExt0] = count;
                atomicAdd(w.stats + kStatCamera, (unsigned long long)count);
                atomicAdd(w.stats + kStatWaves, 1ull);
        }
        if (i >= count) return;
        const uint64_t path = wave_base(w) + i;
        int lo = 0, hi = w.scene_count - 1;
        while (lo < hi) {
                const int mid = (lo + hi + 1) / 2;
                if (w.scenes[mid].path_begin <= path)
                        lo = mid;
                else
                        hi = mid - 1;
        }
        const SceneConst &sc = w.scenes[lo];
        const uint64_t q = path - sc.path_begin;
        const uint32_t pixel = (uint32_t)(q / (uint64_t)sc.spp);
        const uint32_t sample = (uint32_t)(q % (uint64_t)sc.spp) + (uint32_t)sc.first_sample;
        const uint32_t px = (uint32_t)sc.crop_x0 + pixel % (uint32_t)sc.crop_w,
                       py = (uint32_t)sc.crop_y0 + pixel / (uint32_t)sc.crop_w;
        ZSobol z;
        V3 org, dir;
        float weight;
        camera_ray(sc, px, py, sample, z, org, dir, weight);
        w.zs_morton[i] = z.morton;
        w.zs_dim[i] = z.dim;
        w.thr[i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        w.L[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        w.alb[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        w.nrm[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        w.pixel[i] = sc.film_offset + pixel;
        w.scene[i] = (uint32_t)lo;
        w.weight[i] = weight;
        store_ray(w.q_ray[0], i, org, kInf, dir, sc.root);
        w.q_id[0][i] = i;
}

// Camera rays of paths [first, first + n) of one frame for host-driven bounce
// loops: Ray_C records (origin, direction), ray weights and pixel indices.
__global__ void k_camera_rays(SceneConst sc, uint64_t first, uint64_t n, float *rays6, float *weight,
                              int32_t *pixel_out) {
        const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n) return;
        const uint64_t q = first + i;
        const uint32_t pixel = (uint32_t)(q / (uint64_t)sc.spp);
        const uint32_t sample = (uint32_t)(q % (uint64_t)sc.spp) + (uint32_t)sc.first_sample;
        const uint32_t px = (uint32_t)sc.crop_x0 + pixel % (uint32_t)sc.crop_w,
                       py = (uint32_t)sc.crop_y0 + pixel / (uint32_t)sc.crop_w;
        ZSobol z;
        V3 org, dir;
        float w;
        camera_ray(sc, px, py, sample, z, org, dir, w);
        float *r = rays6 + 6 * i;
        r[0] = org.x;
        r[1] = org.y;
        r[2] = org.z;
        r[3] = dir.x;
        r[4] = dir.y;
        r[5] = dir.z;
        weight[i] = w;
        pixel_out[i] = (int32_t)pixel;
}

// Power light sampler over the scene's lights (area lights, then the
// environment light): lowerBound over the running power sum
// (Light/PowerLightSampler.swift:4-48).  Returns the scene-local index.
__device__ int choose_light(const DevScene &s, const SceneConst &sc, float u, float &pdf) {
        const float key = u * sc.light_total;
        int lo = 0, hi = sc.light_count;
        const float *cdf = s.light_cdf + sc.light_begin;
        while (lo < hi) {
                const int mid = lo + (hi - lo) / 2;
                const float c = __ldg(cdf + mid);
                if (c == key) {
                        lo = mid;
                        break;
                } else if (c < key) {
                        lo = mid + 1;
                } else {
                        hi = mid;
                }
        }
        if (lo >= sc.light_count) lo = sc.light_count - 1;
        pdf = (lo == sc.env_index ? sc.env_power : __ldg(s.lights + 4 * (sc.light_begin + lo) + 1).w) / sc.light_total;
        return lo;
}

// offsetRayOrigin(point:normal:direction:) (Core/Interaction.swift:26-35).
__device__ __forceinline__ V3 offset_origin(V3 p, V3 n, V3 dir) {
        const V3 off = n * 0.0001f;
        return dot(dir, n) > 0.0f ? p + off : p + neg(off);
}

// Sort key of an extension-queue entry: the hit's material (batch-wide) or
// the path's scene; misses get the last key.
__device__ __forceinline__ int entry_key(const Wave &w, const DevScene &s, int cur, uint32_t i) {
        const int prim = __float_as_int(w.hits[i].w);
        if (prim < 0) return w.key_count - 1;
        if (w.sort_key == kSortScene) return (int)w.scene[w.q_id[cur][i]];
        int gp = prim;
        if (s.instances) {
                const float4 w3 = __ldg(s.instances + 4 * w.hit_inst[i] + 3);
                gp = __ldg(s.blas_prim_base + __float_as_int(w3.y)) + prim;
        }
        int type;
        int64_t m;
        prim_info(s, gp, type, m);
        if (type == 3) m = w.scenes[w.scene[w.q_id[cur][i]]].material_begin;
        return m >= 0 && m < w.key_count - 1 ? (int)m : w.key_count - 1;
}

__global__ void k_sort_count(Wave w, DevScene s, int cur) {
        const uint32_t n = w.counts[cur];
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n) return;
        atomicAdd(w.key_hist + entry_key(w, s, cur, i), 1u);
}

// Exclusive scan of the key histogram into the cursors (one block of 1024).
__global__ void k_sort_scan(Wave w) {
        __shared__ uint32_t part[1024];
        const int per = (w.key_count + blockDim.x - 1) / blockDim.x;
        const int b0 = threadIdx.x * per;
        uint32_t sum = 0;
        for (int k = b0; k < b0 + per && k < w.key_count; ++k) sum += w.key_hist[k];
        part[threadIdx.x] = sum;
        __syncthreads();
        for (int off = 1; off < (int)blockDim.x; off <<= 1) {
                const uint32_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0u;
                __syncthreads();
                part[threadIdx.x] += v;
                __syncthreads();
        }
        uint32_t run = part[threadIdx.x] - sum;
        for (int k = b0; k < b0 + per && k < w.key_count; ++k) {
                const uint32_t c = w.key_hist[k];
                w.key_hist[w.key_count + k] = run;
                w.key_hist[k] = 0;  // ready for the next bounce
                run += c;
        }
}

__global__ void k_sort_scatter(Wave w, DevScene s, int cur) {
        const uint32_t n = w.counts[cur];
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n) return;
        const uint32_t pos = atomicAdd(w.key_hist + w.key_count + entry_key(w, s, cur, i), 1u);
        w.order[pos] = i;
}

// The general BSDF step of dielectric and coated-diffuse materials
// (surfaceEstimate, VolumePathIntegrator.swift:325-371, with the material's
// BSDF in place of the diffuse closed forms): the light sample is evaluated
// through the BSDF in the shading frame, reflection only in world space
// (FramedBsdf.swift:22-34); the BSDF strategy and the continuation sample it
// from three Z-Sobol dimensions each.  The path's specular flag (thr.w)
// records whether the continuation came from a specular BSDF.
template <int K>
__device__ void shade_generic(const Wave &w, const DevScene &s, const SceneConst &sc, uint32_t path, int bounce,
                              int cur, const BMat &bm, const Surf &sf, V3 thr, V3 L, ZSobol &z) {
        const V3 pos = sf.pos, ng = sf.ng, ns = sf.ns, wo = sf.wo;
        const Frame &fr = sf.fr;
        bool alive = sf.frame_ok;
        bool specular = false;
        if (alive && sc.light_count > 0) {
                const V3 wo_l = fr.to_local(wo);
                float choose_pdf;
                const int lo = choose_light(s, sc, zs_get1d(sc.zs, z), choose_pdf);
                const bool chose_env = lo == sc.env_index;
                const int li = sc.light_begin + lo;
                float u0, u1;
                zs_get2d(sc.zs, z, u0, u1);
                float light_pdf = 0.0f, area = 0.0f;
                V3 rad = v3(0, 0, 0), light_dir = v3(0, 0, 0), lp0, lp1, lp2, target;
                if (chose_env) {
                        V3 dv, r;
                        const float pdf = env_sample(s, u0, u1, dv, r);
                        target = pos + dv * 100.0f;
                        if (!is_black(r) && !isinf(pdf)) {
                                rad = r;
                                light_dir = dv;
                                light_pdf = pdf;
                        }
                } else {
                        const float4 l0 = __ldg(s.lights + 4 * li), l1 = __ldg(s.lights + 4 * li + 1),
                                     l2 = __ldg(s.lights + 4 * li + 2), le4 = __ldg(s.lights + 4 * li + 3);
                        lp0 = v3(l0);
                        lp1 = v3(l1);
                        lp2 = v3(l2);
                        area = l0.w;
                        const float su0 = sqrtf(u0);
                        const float lb0 = 1.0f - su0, lb1 = u1 * su0;
                        target = lp0 * lb0 + lp1 * lb1 + lp2 * ((1.0f - lb0) - lb1);
                        const V3 ln = normalize(cross(lp1 - lp0, lp2 - lp0));
                        const V3 inc = normalize(target - pos);
                        const V3 dl = pos - target;
                        const float pdf = (1.0f / area) * (dot(dl, dl) / fabsf(dot(ln, neg(inc))));
                        if ((sc.two_sided || dot(ln, neg(inc)) > 0.0f) && !isinf(pdf)) {
                                rad = v3(le4) * w.emission_scale;
                                light_dir = inc;
                                light_pdf = pdf;
                        }
                }
                if (light_pdf != 0.0f) {
                        const V3 wl = fr.to_local(light_dir);
                        const bool reflect = dot(light_dir, ng) * dot(wo, ng) > 0.0f;
                        const V3 f = reflect ? bmat_f<K>(bm, wo_l, wl) : v3(0, 0, 0);
                        const V3 light_est = mulv(f * fabsf(dot(light_dir, ns)), rad);
                        if (!is_black(light_est)) {
                                const float brdf_density = wo_l.z == 0.0f ? 0.0f : bmat_pdf<K>(bm, wo_l, wl);
                                const float light_w = power_heuristic(light_pdf, brdf_density);
                                const V3 so = pos + (target - pos) * 0.0001f;
                                const V3 sd = target - so;
                                const V3 c = mulv(mulv(thr, light_est * (light_w / light_pdf) * (1.0f / choose_pdf)),
                                                  medium_tr(sc, so, sd, 1.0f - 0.00001f));
                                const uint32_t q = queue_slot(w.counts + kCountShadow);
                                store_ray(w.sh_ray, q, so, 1.0f - 0.00001f, sd, sc.root);
                                w.sh_id[q] = path;
                                w.sh_contrib[q] = make_float4(c.x, c.y, c.z, 0.0f);
                        }
                }
                float v0, v1, v2;
                zs_get3d(sc.zs, z, v0, v1, v2);
                if (sc.mis_corrected || chose_env) {
                        const BsdfS bs = bmat_sample<K>(bm, wo_l, v0, v1, v2);
                        const float pdf_b = bs.pdf;
                        const V3 wi = fr.to_world(bs.wi);
                        const V3 est = bs.f * fabsf(dot(wi, ns));
                        if (!is_black(est) && pdf_b > 0.0f) {
                                const V3 po = offset_origin(pos, ng, wi);
                                float light_density = 0.0f;
                                if (chose_env) {
                                        light_density = env_pdf(s, wi);
                                } else {
                                        float tl, lu, lv;
                                        const float4 a4 = make_float4(lp0.x, lp0.y, lp0.z, 0.0f),
                                                     b4 = make_float4(lp1.x, lp1.y, lp1.z, 0.0f),
                                                     c4 = make_float4(lp2.x, lp2.y, lp2.z, 0.0f);
                                        if (watertight_test(po.x, po.y, po.z, wi.x, wi.y, wi.z, a4, b4, c4, kInf, tl, lu,
                                                            lv)) {
                                                const V3 hp = po + wi * tl;
                                                const V3 dq = pos - hp;
                                                const V3 lnn = normalize(cross(lp0 - lp2, lp1 - lp2));
                                                const float dens = dot(dq, dq) / (fabsf(dot(lnn, neg(wi))) * area);
                                                light_density = isinf(dens) ? 0.0f : dens;
                                        }
                                }
                                const float bw = power_heuristic(pdf_b, light_density);
                                if (bw > 0.0f) {
                                        const V3 c = mulv(thr, est * (bw / pdf_b) * (1.0f / choose_pdf));
                                        const uint32_t q = queue_slot(w.counts + kCountProbe);
                                        store_ray(w.pr_ray, q, po, kInf, wi, sc.root);
                                        w.pr_id[q] = path;
                                        w.pr_contrib[q] = make_float4(c.x, c.y, c.z, 0.0f);
                                }
                        }
                }
                zs_get3d(sc.zs, z, v0, v1, v2);
                const BsdfS bs = bmat_sample<K>(bm, wo_l, v0, v1, v2);
                const float pdf_c = bs.pdf;
                if (pdf_c == 0.0f || isnan(pdf_c)) {
                        alive = false;
                } else {
                        specular = bmat_specular<K>(bm);
                        const V3 wi = fr.to_world(bs.wi);
                        thr = mulv(thr, bs.f * (fabsf(dot(wi, ng)) / pdf_c));
                        const V3 o = offset_origin(pos, ng, wi);
                        const float mv = fmaxf(thr.x, fmaxf(thr.y, thr.z));
                        if (mv < 1.0f && bounce >= sc.rr_min) {
                                const float qq = fmaxf(0.0f, 1.0f - mv);
                                if (zs_get1d(sc.zs, z) < qq)
                                        alive = false;
                                else
                                        thr = thr * (1.0f / (1.0f - qq));
                        }
                        if (alive && bounce + 1 < sc.max_depth) {
                                const int nxt = cur ^ 1;
                                const uint32_t q = queue_slot(w.counts + nxt);
                                store_ray(w.q_ray[nxt], q, o, kInf, wi, sc.root);
                                w.q_id[nxt][q] = path;
                        }
                }
        }
        w.thr[path] = make_float4(thr.x, thr.y, thr.z, specular ? 1.0f : 0.0f);
        w.L[path] = make_float4(L.x, L.y, L.z, 0.0f);
        w.zs_dim[path] = z.dim;
}

enum ShadeKind {
        kShadeDiffuse = 0, kShadeSplit = 1, kShadeDielectric = 3, kShadeCoated = 4, kShadeConductor = 5,
        kShadeCoatedConductor = 6
};

// The shade queue of a general material kind: its counter and the gen_q
// position of its entry `slot` (two kinds share each half, from either end).
__device__ __forceinline__ uint32_t gen_counter(int kind) { return (uint32_t)(kCountDielectric + kind - 3); }
__device__ __forceinline__ uint32_t gen_pos(const Wave &w, int kind, uint32_t slot) {
        const uint32_t half = kind >= 5 ? w.capacity : 0u;
        return (kind == 3 || kind == 5) ? half + slot : half + w.capacity - 1u - slot;
}

// A scattering event in the medium at p (the oracle's shade_medium): light
// sample with MIS against the phase function (light choice 1D, light point
// 2D, phase sample 2D), then the phase sample (2D) that continues the path
// from p with its throughput unchanged (value / density = 1), then roulette.
__device__ void shade_medium(const Wave &w, const DevScene &s, const SceneConst &sc, uint32_t path, int bounce,
                             int cur, V3 p, V3 wo, V3 thr, V3 L, ZSobol &z) {
        const float g = sc.med_g;
        bool alive = true;
        if (sc.light_count > 0) {
                float choose_pdf;
                const int lo = choose_light(s, sc, zs_get1d(sc.zs, z), choose_pdf);
                const bool chose_env = lo == sc.env_index;
                const int li = sc.light_begin + lo;
                float u0, u1;
                zs_get2d(sc.zs, z, u0, u1);
                float light_pdf = 0.0f, area = 0.0f;
                V3 light_est = v3(0, 0, 0), light_dir = v3(0, 0, 0), lp0, lp1, lp2, target;
                if (chose_env) {
                        V3 dv, rad;
                        const float pdf = env_sample(s, u0, u1, dv, rad);
                        target = p + dv * 100.0f;
                        if (!is_black(rad) && !isinf(pdf)) {
                                light_est = rad * hg_phase(dot(wo, dv), g);
                                light_dir = dv;
                                light_pdf = pdf;
                        }
                } else {
                        const float4 l0 = __ldg(s.lights + 4 * li), l1 = __ldg(s.lights + 4 * li + 1),
                                     l2 = __ldg(s.lights + 4 * li + 2), le4 = __ldg(s.lights + 4 * li + 3);
                        lp0 = v3(l0);
                        lp1 = v3(l1);
                        lp2 = v3(l2);
                        area = l0.w;
                        const float su0 = sqrtf(u0);
                        const float lb0 = 1.0f - su0, lb1 = u1 * su0;
                        target = lp0 * lb0 + lp1 * lb1 + lp2 * ((1.0f - lb0) - lb1);
                        const V3 ln = normalize(cross(lp1 - lp0, lp2 - lp0));
                        const V3 inc = normalize(target - p);
                        const V3 dl = p - target;
                        const float pdf = (1.0f / area) * (dot(dl, dl) / fabsf(dot(ln, neg(inc))));
                        if ((sc.two_sided || dot(ln, neg(inc)) > 0.0f) && !isinf(pdf)) {
                                light_est = v3(le4) * w.emission_scale * hg_phase(dot(wo, inc), g);
                                light_dir = inc;
                                light_pdf = pdf;
                        }
                }
                const float phase_density = light_pdf == 0.0f ? 0.0f : hg_phase(dot(wo, light_dir), g);
                const float light_w = power_heuristic(light_pdf, phase_density);
                if (light_pdf != 0.0f && !is_black(light_est)) {
                        const V3 so = p + (target - p) * 0.0001f;
                        const V3 sd = target - so;
                        const V3 c = mulv(mulv(thr, light_est * (light_w / light_pdf) * (1.0f / choose_pdf)),
                                          medium_tr(sc, so, sd, 1.0f - 0.00001f));
                        const uint32_t q = queue_slot(w.counts + kCountShadow);
                        store_ray(w.sh_ray, q, so, 1.0f - 0.00001f, sd, sc.root);
                        w.sh_id[q] = path;
                        w.sh_contrib[q] = make_float4(c.x, c.y, c.z, 0.0f);
                }
                float v0, v1;
                zs_get2d(sc.zs, z, v0, v1);
                if (sc.mis_corrected || chose_env) {
                        float value;
                        const V3 wi = hg_sample(wo, g, v0, v1, value);
                        if (value > 0.0f) {
                                float light_density = 0.0f;
                                if (chose_env) {
                                        light_density = env_pdf(s, wi);
                                } else {
                                        float tl, lu, lv;
                                        const float4 a4 = make_float4(lp0.x, lp0.y, lp0.z, 0.0f),
                                                     b4 = make_float4(lp1.x, lp1.y, lp1.z, 0.0f),
                                                     c4 = make_float4(lp2.x, lp2.y, lp2.z, 0.0f);
                                        if (watertight_test(p.x, p.y, p.z, wi.x, wi.y, wi.z, a4, b4, c4, kInf, tl, lu, lv)) {
                                                const V3 hp = p + wi * tl;
                                                const V3 dq = p - hp;
                                                const V3 lnn = normalize(cross(lp0 - lp2, lp1 - lp2));
                                                const float dens = dot(dq, dq) / (fabsf(dot(lnn, neg(wi))) * area);
                                                light_density = isinf(dens) ? 0.0f : dens;
                                        }
                                }
                                const float bw = power_heuristic(value, light_density);
                                if (bw > 0.0f) {
                                        // value / density = 1; the probe's resolve applies the
                                        // medium's transmittance up to what it reaches
                                        const V3 c = thr * (bw / choose_pdf);
                                        const uint32_t q = queue_slot(w.counts + kCountProbe);
                                        store_ray(w.pr_ray, q, p, kInf, wi, sc.root);
                                        w.pr_id[q] = path;
                                        w.pr_contrib[q] = make_float4(c.x, c.y, c.z, 0.0f);
                                }
                        }
                }
        }
        float v0, v1;
        zs_get2d(sc.zs, z, v0, v1);
        float value;
        const V3 wi = hg_sample(wo, g, v0, v1, value);
        const float mv = fmaxf(thr.x, fmaxf(thr.y, thr.z));
        if (mv < 1.0f && bounce >= sc.rr_min) {
                const float qq = fmaxf(0.0f, 1.0f - mv);
                if (zs_get1d(sc.zs, z) < qq)
                        alive = false;
                else
                        thr = thr * (1.0f / (1.0f - qq));
        }
        if (alive && bounce + 1 < sc.max_depth) {
                const int nxt = cur ^ 1;
                const uint32_t q = queue_slot(w.counts + nxt);
                store_ray(w.q_ray[nxt], q, p, kInf, wi, sc.root);
                w.q_id[nxt][q] = path;
        }
        w.thr[path] = make_float4(thr.x, thr.y, thr.z, 0.0f);
        w.L[path] = make_float4(L.x, L.y, L.z, 0.0f);
        w.zs_dim[path] = z.dim;
}

// shade: VolumePathIntegrator.shadeBounce + surfaceEstimate (:325-430).
// kShadeDiffuse: a scene without general BSDFs.  kShadeSplit: shades diffuse
// hits and misses and queues hits on the general materials on their kind's
// shade queue, which the kShadeDielectric .. kShadeCoatedConductor launches
// then shade (one material kind per kernel: coherent warps, one BSDF's code).
// Register bounds per kind, blocks of 128 per SM: the layered kinds at 4
// (128 registers, 140-176 bytes of spills; 16-spp two-level frame 245.3 ->
// 242.1 ms against their natural 3, which won before the 32-bit sampler); the
// split kernel at 8 and the dielectric and conductor kinds at 6 (245.8 ->
// 244.0 ms with the split kernel at 7 against 6 and 5, 242.3 -> 241.2 ms at 8;
// the other two kinds at 7: 241.9 ms); the diffuse kind at 7 (72 registers, about 100
// bytes of spills: box-scene frame 1.508 -> 1.422 ms against 5 blocks; 6:
// 1.447, 8: 1.454).
template <int kKind>
__global__ void __launch_bounds__(128, kKind == kShadeSplit                                  ? 8
                                      : (kKind == kShadeCoated || kKind == kShadeCoatedConductor) ? 4
                                      : kKind == kShadeDiffuse                                    ? 7
                                                                                                  : 6)
    k_shade(Wave w, DevScene s, int bounce, int cur, int sorted) {
        const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
        uint32_t i;
        if (kKind >= kShadeDielectric) {
                const uint32_t n = w.counts[gen_counter(kKind)];
                if (slot >= n) return;
                i = w.gen_q[gen_pos(w, kKind, slot)];
        } else {
                const uint32_t n = w.counts[cur];
                if (slot >= n) return;
                i = sorted ? w.order[slot] : slot;
        }
        const uint32_t path = w.q_id[cur][i];
        const float4 hit = w.hits[i];
        const int prim = __float_as_int(hit.w);
        const float4 rd = w.q_ray[cur][2 * i + 1];
        const V3 d = v3(rd);
        if (kKind < kShadeDielectric) {
                const SceneConst &scm = w.scenes[w.scene[path]];
                if (scm.has_medium) {
                        // Homogeneous.sample on the segment before it is shaded (the
                        // branch of shadeBounce :394-408 as meant to run); its two
                        // numbers are drawn at every segment of a scene with a medium
                        ZSobol z;
                        z.morton = w.zs_morton[path];
                        z.dim = w.zs_dim[path];
                        const float uc = zs_get1d(scm.zs, z);
                        const float ud = zs_get1d(scm.zs, z);
                        const V3 o = v3(w.q_ray[cur][2 * i]);
                        float tm;
                        V3 wgt;
                        const bool scattered = medium_sample(scm, o, d, prim < 0 ? kInf : hit.x, uc, ud, tm, wgt);
                        const float4 t4 = w.thr[path];
                        const V3 thr = mulv(v3(t4), wgt);
                        if (scattered) {
                                if (is_black(thr) || bounce >= scm.max_depth) {
                                        w.thr[path] = make_float4(thr.x, thr.y, thr.z, 0.0f);
                                        w.zs_dim[path] = z.dim;
                                } else {
                                        shade_medium(w, s, scm, path, bounce, cur, o + d * tm, neg(d), thr, v3(w.L[path]), z);
                                }
                                return;
                        }
                        w.thr[path] = make_float4(thr.x, thr.y, thr.z, t4.w);
                        w.zs_dim[path] = z.dim;
                }
        }
        if (prim < 0) {
                // shadeBounce on a miss (:375-387): the environment light on
                // camera rays and after specular bounces
                const float4 t4 = w.thr[path];
                if ((bounce == 0 || t4.w != 0.0f) && s.env_rgb) {
                        const V3 thr = v3(t4);
                        const V3 le = env_radiance(s, d);
                        float4 L = w.L[path];
                        L.x += thr.x * le.x;
                        L.y += thr.y * le.y;
                        L.z += thr.z * le.z;
                        w.L[path] = L;
                }
                return;
        }
        const SceneConst &sc = w.scenes[w.scene[path]];
        const float4 t4 = w.thr[path];
        V3 thr = v3(t4);
        const bool after_specular = t4.w != 0.0f;
        if (is_black(thr)) return;
        if (bounce >= sc.max_depth) return;
        Surf sf;
        surface(s, prim, s.instances ? w.hit_inst[i] : -1, hit.y, hit.z, d, sf);
        const V3 pos = sf.pos, ng = sf.ng, wo = sf.wo;
        int type;
        int64_t mat_index;
        prim_info(s, sf.gprim, type, mat_index);
        const bool is_light = type == 3;
        V3 L = v3(w.L[path]);
        if ((bounce == 0 || after_specular) && is_light && mat_index >= 0 && mat_index < s.material_count) {
                const V3 le = v3(__ldg(s.materials + 2 * mat_index + 1)) * w.emission_scale;
                if (sc.two_sided || dot(ng, wo) > 0.0f) L = L + mulv(thr, le);
        }
        // Area-light hits scatter with the scene's material 0 (their interaction
        // keeps materialIndex 0, Core/SurfaceInteraction.swift:20).
        const int64_t mi = is_light ? (int64_t)sc.material_begin : mat_index;
        if (kKind != kShadeDiffuse && s.mat_params && mi >= 0 && mi < s.material_count) {
                const float4 m0 = __ldg(s.materials + 2 * mi);
                const int mt = (int)m0.w;
                if (kKind == kShadeSplit && mt >= 3 && mt <= 6) {
                        const uint32_t q = queue_slot(w.counts + gen_counter(mt));
                        w.gen_q[gen_pos(w, mt, q)] = i;
                        return;
                }
                if (kKind >= kShadeDielectric) {
                        const V3 base = v3(m0);
                        if (bounce == 0) {
                                // Bsdf.albedo(): the base reflectance of a coated diffuse,
                                // white for the dielectric and the conductors
                                const V3 a = kKind == kShadeCoated ? base : v3(1.0f, 1.0f, 1.0f);
                                w.alb[path] = make_float4(a.x, a.y, a.z, 0.0f);
                                w.nrm[path] = make_float4(ng.x, ng.y, ng.z, 0.0f);
                        }
                        const BMat bm = make_bmat<kKind>(base, __ldg(s.mat_params + 3 * mi), __ldg(s.mat_params + 3 * mi + 1),
                                                         __ldg(s.mat_params + 3 * mi + 2));
                        ZSobol z;
                        z.morton = w.zs_morton[path];
                        z.dim = w.zs_dim[path];
                        shade_generic<kKind>(w, s, sc, path, bounce, cur, bm, sf, thr, L, z);
                        return;
                }
        }
        if (kKind >= kShadeDielectric) return;  // not queued here
        V3 refl = (mi >= 0 && mi < s.material_count) ? v3(__ldg(s.materials + 2 * mi)) : v3(0.5f, 0.5f, 0.5f);
        if (w.mat_tex && mi >= 0 && mi < s.material_count) {
                const int t = __ldg(w.mat_tex + mi);
                if (t >= 0) {
                        const int texel = texel_at(w, t, pos);
                        refl = v3(__ldg(w.tex + 3 * texel), __ldg(w.tex + 3 * texel + 1), __ldg(w.tex + 3 * texel + 2));
                        if (w.mode == kReplay) {
                                // Path replay: every contribution still to come passes
                                // through this vertex's albedo once per channel, so
                                // dL/dalbedo = (Ltot - L so far) / albedo.
                                const V3 after = v3(w.Ltot[path]) - L;
                                const uint32_t px = w.pixel[path];
                                const float inv_w = 1.0f / w.adj_w[px];
                                const float *adj = w.adj_rgb + 3 * (size_t)px;
                                if (refl.x > 0.0f) atomicAdd(w.d_tex + 3 * texel, adj[0] * inv_w * (after.x / refl.x));
                                if (refl.y > 0.0f) atomicAdd(w.d_tex + 3 * texel + 1, adj[1] * inv_w * (after.y / refl.y));
                                if (refl.z > 0.0f) atomicAdd(w.d_tex + 3 * texel + 2, adj[2] * inv_w * (after.z / refl.z));
                        }
                }
        }
        const V3 f_val = refl * (1.0f / kPi);
        if (bounce == 0) {
                // surfaceEstimate (:341-344): state.albedo, state.firstNormal
                w.alb[path] = make_float4(refl.x, refl.y, refl.z, 0.0f);
                w.nrm[path] = make_float4(ng.x, ng.y, ng.z, 0.0f);
        }
        const Frame &fr = sf.fr;
        ZSobol z;
        z.morton = w.zs_morton[path];
        z.dim = w.zs_dim[path];
        bool alive = sf.frame_ok;
        if (alive && sc.light_count > 0) {
                const V3 wo_l = fr.to_local(wo);
                // ---- light choice and light sample (sampleLightSource, :67-89)
                float choose_pdf;
                const int lo = choose_light(s, sc, zs_get1d(sc.zs, z), choose_pdf);
                const bool chose_env = lo == sc.env_index;
                const int li = sc.light_begin + lo;
                float u0, u1;
                zs_get2d(sc.zs, z, u0, u1);
                float light_pdf = 0.0f, area = 0.0f;
                V3 light_est = v3(0, 0, 0), light_dir = v3(0, 0, 0), lp0, lp1, lp2, target;
                if (chose_env) {
                        // InfiniteLight.sample (InfiniteLight.swift:38-64); the
                        // shadow ray runs to a point 100 (sceneDiameter) away
                        V3 dv, rad;
                        const float pdf = env_sample(s, u0, u1, dv, rad);
                        target = pos + dv * 100.0f;
                        if (!is_black(rad) && !isinf(pdf)) {
                                const bool reflect = dot(dv, ng) * dot(wo, ng) > 0.0f;
                                const V3 f = reflect ? f_val : v3(0, 0, 0);
                                light_est = mulv(f * fabsf(dot(dv, sf.ns)), rad);
                                light_dir = dv;
                                light_pdf = pdf;
                        }
                } else {
                        const float4 l0 = __ldg(s.lights + 4 * li), l1 = __ldg(s.lights + 4 * li + 1),
                                     l2 = __ldg(s.lights + 4 * li + 2), le4 = __ldg(s.lights + 4 * li + 3);
                        const V3 le = v3(le4) * w.emission_scale;
                        lp0 = v3(l0);
                        lp1 = v3(l1);
                        lp2 = v3(l2);
                        area = l0.w;
                        const float su0 = sqrtf(u0);
                        const float lb0 = 1.0f - su0, lb1 = u1 * su0;
                        target = lp0 * lb0 + lp1 * lb1 + lp2 * ((1.0f - lb0) - lb1);
                        const V3 ln = normalize(cross(lp1 - lp0, lp2 - lp0));
                        const V3 inc = normalize(target - pos);
                        const V3 dl = pos - target;
                        const float pdf = (1.0f / area) * (dot(dl, dl) / fabsf(dot(ln, neg(inc))));
                        if ((sc.two_sided || dot(ln, neg(inc)) > 0.0f) && !isinf(pdf)) {
                                const bool reflect = dot(inc, ng) * dot(wo, ng) > 0.0f;
                                const V3 f = reflect ? f_val : v3(0, 0, 0);
                                light_est = mulv(f * fabsf(dot(inc, sf.ns)), le);
                                light_dir = inc;
                                light_pdf = pdf;
                        }
                }
                float brdf_density = 0.0f;
                {
                        const V3 wi_l = fr.to_local(light_dir);
                        if (wo_l.z != 0.0f && wo_l.z * wi_l.z > 0.0f) brdf_density = fabsf(wi_l.z) / kPi;
                }
                const float light_w = power_heuristic(light_pdf, brdf_density);
                if (light_pdf != 0.0f && !is_black(light_est)) {
                        // Visibility.occluded via spawnRay(from:target:) (Interaction.swift:15-24)
                        const V3 so = pos + (target - pos) * 0.0001f;
                        const V3 sd = target - so;
                        const V3 c = mulv(mulv(thr, light_est * (light_w / light_pdf) * (1.0f / choose_pdf)),
                                          medium_tr(sc, so, sd, 1.0f - 0.00001f));
                        const uint32_t q = queue_slot(w.counts + kCountShadow);
                        store_ray(w.sh_ray, q, so, 1.0f - 0.00001f, sd, sc.root);
                        w.sh_id[q] = path;
                        w.sh_contrib[q] = make_float4(c.x, c.y, c.z, 0.0f);
                }
                // ---- MIS BSDF sample (sampleDistributionFunction, :91-133).  The
                // chosen light's density along it: an environment light answers
                // from its map; an area light, as written, answers 0 (queried with
                // tHit = 0), so that strategy is traced only for corrected MIS.
                float v0, v1, v2;
                zs_get3d(sc.zs, z, v0, v1, v2);
                if (sc.mis_corrected || chose_env) {
                        V3 wi_l = cosine_hemisphere(v0, v1);
                        if (wo_l.z < 0.0f) wi_l.z = -wi_l.z;
                        const float pdf_b = (wo_l.z * wi_l.z > 0.0f) ? fabsf(wi_l.z) / kPi : 0.0f;
                        const V3 wi = fr.to_world(wi_l);
                        const V3 est = f_val * fabsf(dot(wi, sf.ns));
                        if (!is_black(est) && pdf_b > 0.0f) {
                                const V3 po = offset_origin(pos, ng, wi);
                                float light_density = 0.0f;
                                if (chose_env) {
                                        light_density = env_pdf(s, wi);
                                } else {
                                        // Sampleable.swift:47-68 with tHit = inf
                                        float tl, lu, lv;
                                        const float4 a4 = make_float4(lp0.x, lp0.y, lp0.z, 0.0f),
                                                     b4 = make_float4(lp1.x, lp1.y, lp1.z, 0.0f),
                                                     c4 = make_float4(lp2.x, lp2.y, lp2.z, 0.0f);
                                        if (watertight_test(po.x, po.y, po.z, wi.x, wi.y, wi.z, a4, b4, c4, kInf, tl, lu,
                                                            lv)) {
                                                const V3 hp = po + wi * tl;
                                                const V3 dq = pos - hp;
                                                const V3 lnn = normalize(cross(lp0 - lp2, lp1 - lp2));
                                                const float dens = dot(dq, dq) / (fabsf(dot(lnn, neg(wi))) * area);
                                                light_density = isinf(dens) ? 0.0f : dens;
                                        }
                                }
                                const float bw = power_heuristic(pdf_b, light_density);
                                if (bw > 0.0f) {
                                        const V3 c = mulv(thr, est * (bw / pdf_b) * (1.0f / choose_pdf));
                                        const uint32_t q = queue_slot(w.counts + kCountProbe);
                                        store_ray(w.pr_ray, q, po, kInf, wi, sc.root);
                                        w.pr_id[q] = path;
                                        w.pr_contrib[q] = make_float4(c.x, c.y, c.z, 0.0f);
                                }
                        }
                }
                // ---- continuation (bsdf.sampleWorldSpace, :358-369)
                zs_get3d(sc.zs, z, v0, v1, v2);
                V3 wi_l = cosine_hemisphere(v0, v1);
                if (wo_l.z < 0.0f) wi_l.z = -wi_l.z;
                const float pdf_c = (wo_l.z * wi_l.z > 0.0f) ? fabsf(wi_l.z) / kPi : 0.0f;
                if (pdf_c == 0.0f || isnan(pdf_c)) {
                        alive = false;
                } else {
                        const V3 wi = fr.to_world(wi_l);
                        thr = mulv(thr, f_val * (fabsf(dot(wi, ng)) / pdf_c));
                        const V3 o = offset_origin(pos, ng, wi);
                        // stopWithRussianRoulette (:269-283), roulette value from Z-Sobol
                        const float mv = fmaxf(thr.x, fmaxf(thr.y, thr.z));
                        if (mv < 1.0f && bounce >= sc.rr_min) {
                                const float qq = fmaxf(0.0f, 1.0f - mv);
                                if (zs_get1d(sc.zs, z) < qq)
                                        alive = false;
                                else
                                        thr = thr * (1.0f / (1.0f - qq));
                        }
                        if (alive && bounce + 1 < sc.max_depth) {
                                const int nxt = cur ^ 1;
                                const uint32_t q = queue_slot(w.counts + nxt);
                                store_ray(w.q_ray[nxt], q, o, kInf, wi, sc.root);
                                w.q_id[nxt][q] = path;
                        }
                }
        }
        w.thr[path] = make_float4(thr.x, thr.y, thr.z, 0.0f);
        w.L[path] = make_float4(L.x, L.y, L.z, 0.0f);
        w.zs_dim[path] = z.dim;
}

// Adds unoccluded shadow-ray contributions.
__global__ void k_shadow_resolve(Wave w) {
        const uint32_t n = w.counts[kCountShadow];
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n) return;
        if (w.sh_occ[i] >= 0) return;
        const uint32_t path = w.sh_id[i];
        const float4 c = w.sh_contrib[i];
        float4 L = w.L[path];
        L.x += c.x;
        L.y += c.y;
        L.z += c.z;
        w.L[path] = L;
}

// Adds the radiance a BSDF probe reaches: the emission of an area light whose
// normal faces back along the probe, or, on a miss, the environment light.
// any_only: the view has no area light and the probes were traced as any-hit
// queries (pr_hits holds one int32 prim or -1 per probe); a blocked probe
// reaches nothing, exactly as a closest hit on a non-emitting surface.
__global__ void k_probe_resolve(Wave w, DevScene s, int any_only) {
        const uint32_t n = w.counts[kCountProbe];
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n) return;
        const V3 wi = v3(w.pr_ray[2 * i + 1]);
        if (any_only && reinterpret_cast<const int32_t *>(w.pr_hits)[i] >= 0) return;
        const float4 h = any_only ? make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1)) : w.pr_hits[i];
        const int prim = __float_as_int(h.w);
        V3 le;
        if (prim < 0) {
                if (!s.env_rgb) return;
                le = env_radiance(s, wi);
        } else {
                Surf sf;
                surface(s, prim, s.instances ? w.pr_inst[i] : -1, h.y, h.z, wi, sf);
                int type;
                int64_t mat_index;
                prim_info(s, sf.gprim, type, mat_index);
                if (type != 3 || mat_index < 0 || mat_index >= s.material_count) return;
                if (!w.scenes[w.scene[w.pr_id[i]]].two_sided && !(dot(sf.ng, neg(wi)) > 0.0f)) return;
                le = v3(__ldg(s.materials + 2 * mat_index + 1)) * w.emission_scale;
        }
        const uint32_t path = w.pr_id[i];
        float4 c = w.pr_contrib[i];
        const SceneConst &sc = w.scenes[w.scene[path]];
        if (sc.has_medium) {
                // the medium's transmittance up to what the probe reaches
                const V3 tr = medium_tr(sc, v3(w.pr_ray[2 * i]), wi, prim < 0 ? kInf : h.x);
                c.x *= tr.x;
                c.y *= tr.y;
                c.z *= tr.z;
        }
        float4 L = w.L[path];
        L.x += c.x * le.x;
        L.y += c.y * le.y;
        L.z += c.z * le.z;
        w.L[path] = L;
}

// Per-bounce bookkeeping: ray statistics of the bounce.
__global__ void k_bounce_tally(Wave w, int cur) {
        atomicAdd(w.stats + kStatExt, (unsigned long long)w.counts[cur]);
        atomicAdd(w.stats + kStatShadow, (unsigned long long)w.counts[kCountShadow]);
        atomicAdd(w.stats + kStatProbe, (unsigned long long)w.counts[kCountProbe]);
}

// Clears the counters of the queues the next stages fill.
__global__ void k_clear_counts(Wave w, int next) {
        w.counts[next] = 0;
        w.counts[kCountShadow] = 0;
        w.counts[kCountProbe] = 0;
        w.counts[kCountDielectric] = 0;
        w.counts[kCountCoated] = 0;
        w.counts[kCountConductor] = 0;
        w.counts[kCountCoatedConductor] = 0;
}

// Film.add (Core/Film.swift:107-119): the sample's light scaled by iso / 100
// and, when a clamp is set, by max / its largest component.
__device__ __forceinline__ float4 film_light(const Wave &w, uint32_t i) {
        const SceneConst &sc = w.scenes[w.scene[i]];
        float4 L = w.L[i];
        L.x *= sc.film_scale;
        L.y *= sc.film_scale;
        L.z *= sc.film_scale;
        if (sc.max_component > 0.0f) {
                const float mv = fmaxf(L.x, fmaxf(L.y, L.z));
                if (mv > sc.max_component) {
                        const float k = sc.max_component / mv;
                        L.x *= k;
                        L.y *= k;
                        L.z *= k;
                }
        }
        return L;
}

// Film sums: radiance, its square, the filter weight and the first-hit AOVs
// (albedo, normal: Tile.swift:157-205), per pixel of the batch film.
__global__ void k_accumulate(Wave w, float *film_rgb, float *film_sq, float *film_w, float *film_alb,
                             float *film_nrm) {
        const uint32_t count = wave_count(w);
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= count) return;
        const uint32_t px = w.pixel[i];
        const float4 L = film_light(w, i);
        atomicAdd(film_rgb + 3 * (size_t)px, L.x);
        atomicAdd(film_rgb + 3 * (size_t)px + 1, L.y);
        atomicAdd(film_rgb + 3 * (size_t)px + 2, L.z);
        if (film_sq) {
                atomicAdd(film_sq + 3 * (size_t)px, L.x * L.x);
                atomicAdd(film_sq + 3 * (size_t)px + 1, L.y * L.y);
                atomicAdd(film_sq + 3 * (size_t)px + 2, L.z * L.z);
        }
        atomicAdd(film_w + px, w.weight[i]);
        if (film_alb) {
                const float4 a = w.alb[i];
                atomicAdd(film_alb + 3 * (size_t)px, a.x);
                atomicAdd(film_alb + 3 * (size_t)px + 1, a.y);
                atomicAdd(film_alb + 3 * (size_t)px + 2, a.z);
        }
        if (film_nrm) {
                const float4 nv = w.nrm[i];
                atomicAdd(film_nrm + 3 * (size_t)px, nv.x);
                atomicAdd(film_nrm + 3 * (size_t)px + 1, nv.y);
                atomicAdd(film_nrm + 3 * (size_t)px + 2, nv.z);
        }
}

// Double-precision film sums (finite differences need sums whose rounding
// does not depend on the order of the atomics).
__global__ void k_accumulate_f64(Wave w, double *film_rgb, double *film_sq, double *film_w) {
        const uint32_t count = wave_count(w);
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= count) return;
        const uint32_t px = w.pixel[i];
        const float4 L = film_light(w, i);
        atomicAdd(film_rgb + 3 * (size_t)px, (double)L.x);
        atomicAdd(film_rgb + 3 * (size_t)px + 1, (double)L.y);
        atomicAdd(film_rgb + 3 * (size_t)px + 2, (double)L.z);
        if (film_sq) {
                atomicAdd(film_sq + 3 * (size_t)px, (double)L.x * L.x);
                atomicAdd(film_sq + 3 * (size_t)px + 1, (double)L.y * L.y);
                atomicAdd(film_sq + 3 * (size_t)px + 2, (double)L.z * L.z);
        }
        atomicAdd(film_w + px, (double)w.weight[i]);
}

// Primal pass of a wave: keep each path's radiance for the replay.
__global__ void k_store_total(Wave w) {
        const uint32_t count = wave_count(w);
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= count) return;
        w.Ltot[i] = w.L[i];
}

// End of a replay: every emission is linear in the emission scale, so
// dLoss/dscale = sum over paths of <dLoss/dL, Ltot> / scale.
__global__ void k_emission_gradient(Wave w) {
        const uint32_t count = wave_count(w);
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        double v = 0.0;
        if (i < count) {
                const uint32_t px = w.pixel[i];
                const float4 Lt = w.Ltot[i];
                const float *adj = w.adj_rgb + 3 * (size_t)px;
                const double g = (double)adj[0] * Lt.x + (double)adj[1] * Lt.y + (double)adj[2] * Lt.z;
                v = g / ((double)w.adj_w[px] * (double)w.emission_scale);
        }
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, off);
        if ((threadIdx.x & 31u) == 0 && v != 0.0) atomicAdd(w.d_emission, v);
}

__global__ void k_advance_wave(Wave w) {
        const uint64_t next = wave_base(w) + wave_count(w);
        w.counts[kCountWaveBase] = (uint32_t)(next & 0xFFFFFFFFull);
        w.counts[kCountWaveBase + 1] = (uint32_t)(next >> 32);
}

__global__ void k_set_wave_base(Wave w, uint64_t base) {
        w.counts[kCountWaveBase] = (uint32_t)(base & 0xFFFFFFFFull);
        w.counts[kCountWaveBase + 1] = (uint32_t)(base >> 32);
}

struct KindList {
        int32_t k[64];
};

// Z-Sobol values for n pixel samples: the sequence of get1D/get2D/get3D
// calls in `kinds` (1, 2 or 3 each), starting at dimension 0.
__global__ void k_zsobol_fill(ZSobolConfig c, const int32_t *px, const int32_t *py, const int64_t *index, int64_t n,
                              KindList kinds, int nkinds, int per, float *out) {
        const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n) return;
        ZSobol z;
        zs_start(c, z, (uint32_t)px[i], (uint32_t)py[i], (uint32_t)index[i]);
        float *o = out + i * per;
        for (int k = 0; k < nkinds; ++k) {
                const int kind = kinds.k[k];
                if (kind == 1) {
                        *o++ = zs_get1d(c, z);
                } else if (kind == 2) {
                        zs_get2d(c, z, o[0], o[1]);
                        o += 2;
                } else {
                        zs_get3d(c, z, o[0], o[1], o[2]);
                        o += 3;
                }
        }
}

// ------------------------------------------------------------ host side

std::mutex g_sobol_mu;
const uint32_t *g_sobol_dev[64] = {};

gzg_status device_sobol(int dev, const uint32_t **out) {
        std::lock_guard<std::mutex> lk(g_sobol_mu);
        if (dev < 0 || dev >= 64) return set_error(GZG_ERR_LIMIT, "device ordinal above 63");
        if (!g_sobol_dev[dev]) {
                size_t count = 0;
                const uint32_t *host = sobol_matrices(&count);
                if (count != (size_t)kSobolDims * kSobolColumns)
                        return set_error(GZG_ERR_BAD_SCENE, "embedded Sobol table has the wrong size");
                void *p = nullptr;
                cudaError_t e = cudaMalloc(&p, count * 4);
                if (e != cudaSuccess) return set_error(GZG_ERR_OUT_OF_MEMORY, "Sobol table allocation");
                e = cudaMemcpy(p, host, count * 4, cudaMemcpyHostToDevice);
                if (e != cudaSuccess) return set_error(GZG_ERR_CUDA, "Sobol table upload");
                g_sobol_dev[dev] = static_cast<const uint32_t *>(p);
        }
        *out = g_sobol_dev[dev];
        return GZG_OK;
}

// ZSobolSampler.init (ZSobolSampler.swift:114-122).
ZSobolConfig make_zsobol(int64_t spp, int32_t res_x, int32_t res_y, int64_t seed, const uint32_t *matrices) {
        ZSobolConfig c{};
        c.matrices = matrices;
        c.seed = (uint64_t)seed;
        c.log2spp = __builtin_ctzll((uint64_t)spp);
        int64_t res = std::max(res_x, res_y);
        res -= 1;
        res |= res >> 1;
        res |= res >> 2;
        res |= res >> 4;
        res |= res >> 8;
        res |= res >> 16;
        res += 1;
        c.n_base4_digits = __builtin_ctzll((uint64_t)res) + (c.log2spp + 1) / 2;
        return c;
}

V3 hsub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 hcross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V3 hnorm(V3 a) {
        const float l = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
        return V3{a.x / l, a.y / l, a.z / l};
}

// Camera, film and sampler constants of one scene.
SceneConst make_scene_const(const gzg_render_params &P, const uint32_t *matrices) {
        SceneConst sc{};
        const V3 eye{P.eye[0], P.eye[1], P.eye[2]};
        const V3 fwd = hnorm(hsub(V3{P.target[0], P.target[1], P.target[2]}, eye));
        const V3 right = hnorm(hcross(fwd, V3{P.up[0], P.up[1], P.up[2]}));
        sc.eye = eye;
        sc.fwd = fwd;
        sc.right = right;
        sc.up = hcross(right, fwd);
        sc.tan_half = std::tan(P.fov_deg * 3.14159265358979323846f / 180.0f / 2.0f);
        const float aspect = (float)P.width / (float)P.height;
        sc.sx0 = aspect > 1.0f ? -aspect : -1.0f;
        sc.sx1 = -sc.sx0;
        sc.sy0 = aspect > 1.0f ? -1.0f : -1.0f / aspect;
        sc.sy1 = -sc.sy0;
        sc.filter_radius = P.filter_radius;
        sc.filter_sigma = P.filter_sigma;
        sc.width = P.width;
        sc.height = P.height;
        const bool cropped = P.crop[0] || P.crop[1] || P.crop[2] || P.crop[3];
        sc.crop_x0 = cropped ? P.crop[0] : 0;
        sc.crop_y0 = cropped ? P.crop[1] : 0;
        sc.crop_w = cropped ? P.crop[2] - P.crop[0] : P.width;
        sc.crop_h = cropped ? P.crop[3] - P.crop[1] : P.height;
        sc.spp = P.spp;
        sc.max_depth = P.max_depth;
        sc.rr_min = P.rr_min_bounce;
        sc.mis_corrected = P.mis_corrected;
        sc.first_sample = P.first_sample;
        sc.zs = make_zsobol(P.sampler_spp > 0 ? P.sampler_spp : P.spp, P.width, P.height, P.seed, matrices);
        sc.film_scale = 1.0f;  // iso 100
        sc.max_component = 0.0f;
        sc.lens_radius = P.lens_radius;
        sc.focal_distance = P.focal_distance;
        sc.two_sided = P.two_sided_emission != 0;
        return sc;
}

// Pixels of a frame's film: its crop window's, or the whole frame's.
int64_t film_pixels(const gzg_render_params &P) {
        if (P.crop[0] || P.crop[1] || P.crop[2] || P.crop[3])
                return (int64_t)(P.crop[2] - P.crop[0]) * (P.crop[3] - P.crop[1]);
        return (int64_t)P.width * P.height;
}

bool params_ok(const gzg_render_params &P) {
        const bool lens_ok = P.lens_radius == 0.0f ||
                             (std::isfinite(P.lens_radius) && P.lens_radius > 0.0f && std::isfinite(P.focal_distance) &&
                              P.focal_distance > 0.0f);
        const bool cropped = P.crop[0] || P.crop[1] || P.crop[2] || P.crop[3];
        const bool crop_ok = !cropped || (P.crop[0] >= 0 && P.crop[1] >= 0 && P.crop[0] < P.crop[2] &&
                                          P.crop[1] < P.crop[3] && P.crop[2] <= P.width && P.crop[3] <= P.height);
        return crop_ok && P.width > 0 && P.height > 0 && P.spp > 0 && P.max_depth >= 0 && P.fov_deg > 0.0f &&
               P.filter_sigma > 0.0f && P.filter_radius > 0.0f && P.first_sample >= 0 && P.sampler_spp >= 0 && lens_ok;
}

gzg_status cuda_err(cudaError_t e, const char *what) {
        if (e == cudaSuccess) return GZG_OK;
        return set_error(e == cudaErrorMemoryAllocation ? GZG_ERR_OUT_OF_MEMORY : GZG_ERR_CUDA,
                         std::string(what) + ": " + cudaGetErrorString(e));
}

// Paths per wave unless the caller sets one (about 350 device bytes per path:
// 5.9 GB at 2^24).  Larger waves keep the later, roulette-thinned bounces
// wide enough to fill the GPU: the two-level 1920 x 1080 x 64 spp frame takes
// 1522 / 1316 / 1230 / 1200 ms at 2^21 / 2^22 / 2^23 / 2^24 paths.
constexpr uint32_t kDefaultWave = 1u << 24;

}  // namespace
}  // namespace gzg

using namespace gzg;

struct gzg_renderer {
        int device = 0;
        std::vector<gzg_scene *> scenes;
        std::vector<gzg_render_params> params;
        gzg_batch_options opts{};
        std::vector<SceneConst> consts;
        std::vector<int64_t> film_offsets;  // scene count + 1 pixel offsets
        Wave w{};
        uint32_t max_capacity = 0;
        DevScene view{};
        int wide_depth = 0;
        // no prim of the view is an area light: a BSDF probe can only reach
        // the environment, so it is traced as an any-hit query
        bool probe_any = false;
        std::vector<void *> allocs;
        cudaGraphExec_t graph = nullptr;
        cudaGraph_t graph_def = nullptr;
        const void *graph_key[8] = {};
        // differentiable rendering
        int32_t *d_mat_tex = nullptr;
        float *d_tex_map = nullptr;
        int tex_slots = 0;

        ~gzg_renderer() {
                int prev = 0;
                cudaGetDevice(&prev);
                if (prev != device) cudaSetDevice(device);
                drop_graph();
                for (void *p : allocs) cudaFree(p);
                if (prev != device) cudaSetDevice(prev);
        }

        void drop_graph() {
                if (graph) cudaGraphExecDestroy(graph);
                if (graph_def) cudaGraphDestroy(graph_def);
                graph = nullptr;
                graph_def = nullptr;
        }

        template <class T>
        gzg_status alloc(T **p, size_t count) {
                void *d = nullptr;
                cudaError_t e = cudaMalloc(&d, std::max<size_t>(count * sizeof(T), 16));
                if (e != cudaSuccess) return set_error(GZG_ERR_OUT_OF_MEMORY, "renderer buffer allocation");
                allocs.push_back(d);
                *p = static_cast<T *>(d);
                return GZG_OK;
        }

        // Copies a host vector to a new device buffer of element type D.
        template <class D, class T>
        gzg_status upload(const D **p, const std::vector<T> &v) {
                static_assert(sizeof(T) % sizeof(D) == 0 || sizeof(D) % sizeof(T) == 0, "record size mismatch");
                const size_t bytes = v.size() * sizeof(T);
                D *d = nullptr;
                gzg_status st = alloc(&d, (bytes + sizeof(D) - 1) / sizeof(D));
                if (st) return st;
                if (bytes) {
                        st = cuda_err(cudaMemcpy(d, v.data(), bytes, cudaMemcpyHostToDevice), "batch upload");
                        if (st) return st;
                }
                *p = d;
                return GZG_OK;
        }

        // Film buffers of a pass: float sums, or double sums (d* set).
        struct Films {
                float *rgb, *sq, *w;
                double *drgb, *dsq, *dw;
                float *alb, *nrm;
        };

        // One wave: generate, bounces, then by w.mode accumulate + advance,
        // keep the primal radiance, or finish a replay + advance.  Enqueued on st.
        cudaError_t enqueue_wave(const Films &film, cudaStream_t st) {
                const int block = 128;
                const unsigned grid = (w.capacity + block - 1) / block;
                int max_depth = 0;
                bool corrected = view.env_rgb != nullptr;  // an environment light is probed as written too
                for (const gzg_render_params &P : params) {
                        max_depth = std::max(max_depth, (int)P.max_depth);
                        corrected = corrected || P.mis_corrected;
                }
                // the first scene's tuned launches (gzg_scene_autotune), read at
                // enqueue time so a later autotune takes effect
                LaunchParams lp_closest = scene_launch(scenes[0], false);
                LaunchParams lp_any = scene_launch(scenes[0], true);
                lp_closest.wide_depth = lp_any.wide_depth = wide_depth;
                // per-ray roots exist in the wide layout only
                if (view.per_ray_root) {
                        if (lp_closest.traversal == GZG_TRAVERSAL_BVH2) lp_closest.traversal = GZG_TRAVERSAL_WIDE;
                        if (lp_any.traversal == GZG_TRAVERSAL_BVH2) lp_any.traversal = GZG_TRAVERSAL_WIDE;
                }
                NvtxRange wave_range("gzg wave");
                {
                        NvtxRange r("gzg generate");
                        k_generate<<<grid, block, 0, st>>>(w);
                }
                int cur = 0;
                for (int b = 0; b < max_depth; ++b) {
                        k_clear_counts<<<1, 1, 0, st>>>(w, cur ^ 1);
                        LaunchParams lp = lp_closest, lpa = lp_any;
                        lp.sched = lpa.sched = w.counts + kCountSched;
                        lp.n_dev = w.counts + cur;
                        lp.inst_out = w.hit_inst;
                        NvtxRange extend_range("gzg extend");
                        cudaError_t e = launch_trace(view, lp, kRayDevice, kOutHit, w.q_ray[cur], nullptr, w.capacity,
                                                     w.hits, st);
                        if (e != cudaSuccess) return e;
                        extend_range.end();
                        NvtxRange shade_range("gzg shade");
                        const int sorted = w.sort_key != kSortNone;
                        if (sorted) {
                                k_sort_count<<<grid, block, 0, st>>>(w, view, cur);
                                k_sort_scan<<<1, 1024, 0, st>>>(w);
                                k_sort_scatter<<<grid, block, 0, st>>>(w, view, cur);
                        }
                        if (view.mat_params) {
                                k_shade<kShadeSplit><<<grid, block, 0, st>>>(w, view, b, cur, sorted);
                                k_shade<kShadeDielectric><<<grid, block, 0, st>>>(w, view, b, cur, sorted);
                                k_shade<kShadeCoated><<<grid, block, 0, st>>>(w, view, b, cur, sorted);
                                k_shade<kShadeConductor><<<grid, block, 0, st>>>(w, view, b, cur, sorted);
                                k_shade<kShadeCoatedConductor><<<grid, block, 0, st>>>(w, view, b, cur, sorted);
                        } else {
                                k_shade<kShadeDiffuse><<<grid, block, 0, st>>>(w, view, b, cur, sorted);
                        }
                        shade_range.end();
                        NvtxRange shadow_range("gzg shadow");
                        lpa.n_dev = w.counts + kCountShadow;
                        e = launch_trace(view, lpa, kRayDevice, kOutAnyPrim, w.sh_ray, nullptr, w.capacity, w.sh_occ, st);
                        if (e != cudaSuccess) return e;
                        k_shadow_resolve<<<grid, block, 0, st>>>(w);
                        shadow_range.end();
                        NvtxRange probe_range("gzg probe");
                        if (corrected) {
                                if (probe_any) {
                                        lpa.n_dev = w.counts + kCountProbe;
                                        e = launch_trace(view, lpa, kRayDevice, kOutAnyPrim, w.pr_ray, nullptr, w.capacity,
                                                         w.pr_hits, st);
                                } else {
                                        lp.n_dev = w.counts + kCountProbe;
                                        lp.inst_out = w.pr_inst;
                                        e = launch_trace(view, lp, kRayDevice, kOutHit, w.pr_ray, nullptr, w.capacity,
                                                         w.pr_hits, st);
                                }
                                if (e != cudaSuccess) return e;
                                k_probe_resolve<<<grid, block, 0, st>>>(w, view, probe_any ? 1 : 0);
                        }
                        k_bounce_tally<<<1, 1, 0, st>>>(w, cur);
                        cur ^= 1;
                }
                NvtxRange accumulate_range("gzg accumulate");
                if (w.mode == kPrimal) {
                        k_store_total<<<grid, block, 0, st>>>(w);  // the replay runs the same paths
                        return cudaGetLastError();
                }
                if (w.mode == kReplay) {
                        if (w.d_emission) k_emission_gradient<<<grid, block, 0, st>>>(w);
                } else if (film.drgb) {
                        k_accumulate_f64<<<grid, block, 0, st>>>(w, film.drgb, film.dsq, film.dw);
                } else {
                        k_accumulate<<<grid, block, 0, st>>>(w, film.rgb, film.sq, film.w, film.alb, film.nrm);
                }
                k_advance_wave<<<1, 1, 0, st>>>(w);
                return cudaGetLastError();
        }

        // Sets the wave capacity (clamped to the allocation) and the sort key.
        void configure(uint32_t capacity, int sort_key) {
                w.capacity = std::max<uint32_t>(1, std::min<uint32_t>(capacity, max_capacity));
                w.sort_key = sort_key;
                w.key_count = (sort_key == kSortScene ? (int32_t)scenes.size() : view.material_count) + 1;
                drop_graph();
        }

        uint64_t wave_total() const { return (w.total_paths + w.capacity - 1) / w.capacity; }

        // Double-precision films, direct launches.
        gzg_status render_f64(double *rgb, double *sq, double *wt, cudaStream_t st) {
                w.mode = kRender;
                k_set_wave_base<<<1, 1, 0, st>>>(w, 0ull);
                const Films f{nullptr, nullptr, nullptr, rgb, sq, wt, nullptr, nullptr};
                for (uint64_t k = 0; k < wave_total(); ++k) {
                        gzg_status status = cuda_err(enqueue_wave(f, st), "wave launch");
                        if (status) return status;
                }
                return GZG_OK;
        }

        // Path-replay adjoint: per wave a primal pass, then the replay.
        gzg_status adjoint(const float *adj_rgb, const float *adj_w, float *d_tex, double *d_emission, cudaStream_t st) {
                if (!w.Ltot) {
                        gzg_status status = alloc(&w.Ltot, max_capacity);
                        if (status) return status;
                }
                w.adj_rgb = adj_rgb;
                w.adj_w = adj_w;
                w.d_tex = d_tex;
                w.d_emission = d_emission;
                k_set_wave_base<<<1, 1, 0, st>>>(w, 0ull);
                const Films none{};
                gzg_status status = GZG_OK;
                for (uint64_t k = 0; k < wave_total() && !status; ++k) {
                        w.mode = kPrimal;
                        status = cuda_err(enqueue_wave(none, st), "primal wave launch");
                        if (status) break;
                        w.mode = kReplay;
                        status = cuda_err(enqueue_wave(none, st), "replay wave launch");
                }
                w.mode = kRender;
                w.adj_rgb = w.adj_w = nullptr;
                w.d_tex = nullptr;
                w.d_emission = nullptr;
                return status;
        }

        gzg_status render(float *film_rgb, float *film_sq, float *film_w, cudaStream_t st, float *film_alb = nullptr,
                          float *film_nrm = nullptr) {
                const uint64_t waves = wave_total();
                w.mode = kRender;
                const Films film{film_rgb, film_sq, film_w, nullptr, nullptr, nullptr, film_alb, film_nrm};
                k_set_wave_base<<<1, 1, 0, st>>>(w, 0ull);
                if (opts.use_graph) {
                        const void *key[8] = {film_rgb, film_sq, film_w, (const void *)(uintptr_t)w.capacity,
                                              (const void *)(uintptr_t)w.sort_key, (const void *)(uintptr_t)w.total_paths,
                                              film_alb, film_nrm};
                        if (!graph || !std::equal(key, key + 8, graph_key)) {
                                drop_graph();
                                cudaStream_t cap;
                                gzg_status status = cuda_err(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "graph stream");
                                if (status) return status;
                                status = cuda_err(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "graph capture");
                                if (!status) {
                                        cudaError_t e = enqueue_wave(film, cap);
                                        cudaError_t e2 = cudaStreamEndCapture(cap, &graph_def);
                                        status = cuda_err(e != cudaSuccess ? e : e2, "graph capture of a wave");
                                        if (!status) status = cuda_err(cudaGraphInstantiate(&graph, graph_def, 0), "graph instantiate");
                                }
                                cudaStreamDestroy(cap);
                                if (status) return status;
                                std::copy(key, key + 8, graph_key);
                        }
                        for (uint64_t k = 0; k < waves; ++k) {
                                gzg_status status = cuda_err(cudaGraphLaunch(graph, st), "graph launch");
                                if (status) return status;
                        }
                        return GZG_OK;
                }
                for (uint64_t k = 0; k < waves; ++k) {
                        gzg_status status = cuda_err(enqueue_wave(film, st), "wave launch");
                        if (status) return status;
                }
                return GZG_OK;
        }
};

namespace {

// Builds the batch: per-scene constants and, for more than one scene, one
// concatenated scene (nodes, leaf records with batch-wide prim indices,
// triangles, prim ids with batch-wide material indices, materials, lights).
gzg_status build_batch(gzg_renderer *r) {
        const size_t n = r->scenes.size();
        const uint32_t *matrices = nullptr;
        gzg_status st = device_sobol(r->device, &matrices);
        if (st) return st;
        r->consts.resize(n);
        r->film_offsets.assign(n + 1, 0);
        uint64_t paths = 0;
        for (size_t k = 0; k < n; ++k) {
                r->consts[k] = make_scene_const(r->params[k], matrices);
                r->consts[k].path_begin = paths;
                r->consts[k].film_offset = (uint32_t)r->film_offsets[k];
                r->film_offsets[k + 1] = r->film_offsets[k] + film_pixels(r->params[k]);
                paths += (uint64_t)film_pixels(r->params[k]) * r->params[k].spp;
        }
        if (r->film_offsets[n] >= (int64_t)0xFFFFFFFFll)
                return set_error(GZG_ERR_LIMIT, "renderer: more than 2^32 film pixels in a batch");
        r->w.total_paths = paths;
        for (size_t k = 0; k < n; ++k) {
                const HostShading &hs = scene_host_shading(r->scenes[k]);
                SceneConst &sc = r->consts[k];
                sc.has_medium = hs.has_medium ? 1 : 0;
                const gzg_medium &m = hs.medium;
                sc.med_min = V3{m.box_min[0], m.box_min[1], m.box_min[2]};
                sc.med_max = V3{m.box_max[0], m.box_max[1], m.box_max[2]};
                sc.sigma_a = V3{m.sigma_a[0], m.sigma_a[1], m.sigma_a[2]};
                sc.sigma_s = V3{m.sigma_s[0], m.sigma_s[1], m.sigma_s[2]};
                sc.med_g = m.g;
        }
        int wide_depth = 0;
        if (n == 1) {
                scene_view(r->scenes[0], &r->view, &r->device, &wide_depth);
                const HostShading &hs = scene_host_shading(r->scenes[0]);
                SceneConst &sc = r->consts[0];
                sc.root = 0;
                sc.material_begin = 0;
                sc.material_count = (int32_t)(hs.materials.size() / 2);
                sc.light_begin = 0;
                sc.light_count = (int32_t)(hs.lights.size() / 4) + (hs.has_env ? 1 : 0);
                sc.light_total = hs.has_env ? hs.light_total_env : hs.light_total;
                sc.env_index = hs.has_env ? (int32_t)(hs.lights.size() / 4) : -1;
                sc.env_power = hs.env_power;
                r->view.per_ray_root = 0;
        } else {
                std::vector<WideNode> nodes;
                std::vector<float4_> v0, v1, v2, pv0, pv1, pv2, mats, lights, mparams, attr;
                bool any_attr = false;
                for (size_t k = 0; k < n; ++k) any_attr = any_attr || !scene_host_shading(r->scenes[k]).attr.empty();
                bool any_params = false;
                for (size_t k = 0; k < n; ++k) any_params = any_params || !scene_host_shading(r->scenes[k]).mat_params.empty();
                std::vector<gzg_prim_id> prims;
                std::vector<float> cdf;
                uint64_t steps = 0;
                for (size_t k = 0; k < n; ++k) {
                        const WideBvh &wb = scene_host_wide(r->scenes[k]);
                        const HostShading &hs = scene_host_shading(r->scenes[k]);
                        const uint32_t noff = (uint32_t)nodes.size(), toff = (uint32_t)v0.size();
                        const int32_t poff = (int32_t)prims.size(), moff = (int32_t)(mats.size() / 2),
                                      loff = (int32_t)(lights.size() / 4);
                        for (WideNode nd : wb.nodes) {
                                nd.child_base += noff;
                                nd.tri_base += toff;
                                nodes.push_back(nd);
                        }
                        for (float4_ a : wb.v0) {
                                int32_t p;
                                std::memcpy(&p, &a.w, 4);
                                p += poff;
                                std::memcpy(&a.w, &p, 4);
                                v0.push_back(a);
                        }
                        v1.insert(v1.end(), wb.v1.begin(), wb.v1.end());
                        v2.insert(v2.end(), wb.v2.begin(), wb.v2.end());
                        pv0.insert(pv0.end(), hs.pv0.begin(), hs.pv0.end());
                        pv1.insert(pv1.end(), hs.pv1.begin(), hs.pv1.end());
                        pv2.insert(pv2.end(), hs.pv2.begin(), hs.pv2.end());
                        for (gzg_prim_id p : hs.prims) {
                                p.material_index += moff;
                                prims.push_back(p);
                        }
                        mats.insert(mats.end(), hs.materials.begin(), hs.materials.end());
                        if (any_attr) {
                                if (hs.attr.empty())
                                        attr.insert(attr.end(), 5 * hs.prims.size(), float4_{0, 0, 0, 0});
                                else
                                        attr.insert(attr.end(), hs.attr.begin(), hs.attr.end());
                        }
                        if (any_params) {
                                if (hs.mat_params.empty())
                                        mparams.insert(mparams.end(), 3 * (hs.materials.size() / 2), float4_{1, 0, 0, 0});
                                else
                                        mparams.insert(mparams.end(), hs.mat_params.begin(), hs.mat_params.end());
                        }
                        lights.insert(lights.end(), hs.lights.begin(), hs.lights.end());
                        cdf.insert(cdf.end(), hs.light_cdf.begin(), hs.light_cdf.end());
                        SceneConst &sc = r->consts[k];
                        sc.root = noff;
                        sc.material_begin = moff;
                        sc.material_count = (int32_t)(hs.materials.size() / 2);
                        sc.light_begin = loff;
                        sc.light_count = (int32_t)(hs.lights.size() / 4);
                        sc.light_total = hs.light_total;
                        sc.env_index = -1;
                        steps = std::max<uint64_t>(steps, wb.nodes.size());
                        wide_depth = std::max(wide_depth, (int)wb.depth);
                }
                if (nodes.size() >= 0x7FFFFFFFu || v0.size() >= 0x7FFFFFFFu || prims.size() >= 0x7FFFFFFFu)
                        return set_error(GZG_ERR_LIMIT, "renderer: batch exceeds 2^31 nodes, records or prims");
                DevScene &d = r->view;
                d = DevScene{};
                if ((st = r->upload(&d.wide, nodes)) || (st = r->upload(&d.tv0, v0)) || (st = r->upload(&d.tv1, v1)) ||
                    (st = r->upload(&d.tv2, v2)) || (st = r->upload(&d.pv0, pv0)) || (st = r->upload(&d.pv1, pv1)) ||
                    (st = r->upload(&d.pv2, pv2)) || (st = r->upload(&d.prims, prims)) ||
                    (st = r->upload(&d.materials, mats)) || (st = r->upload(&d.lights, lights)) ||
                    (st = r->upload(&d.light_cdf, cdf)))
                        return st;
                if (any_params && (st = r->upload(&d.mat_params, mparams))) return st;
                if (any_attr && (st = r->upload(&d.attr, attr))) return st;
                uint32_t *err = nullptr;
                if ((st = r->alloc(&err, 1))) return st;
                if ((st = cuda_err(cudaMemset(err, 0, 4), "batch error word"))) return st;
                d.err = err;
                d.prim_count = (int64_t)prims.size();
                d.wide_count = (uint32_t)std::min<uint64_t>(steps, 0xFFFFFFFFull);
                d.material_count = (int32_t)(mats.size() / 2);
                d.light_count = (int32_t)(lights.size() / 4);
                d.per_ray_root = 1;
        }
        r->wide_depth = wide_depth;
        r->probe_any = true;
        for (gzg_scene *sc : r->scenes)
                for (const gzg_prim_id &p : scene_host_shading(sc).prims)
                        if (p.type == 3) r->probe_any = false;
        return GZG_OK;
}

gzg_status renderer_create(gzg_scene *const *scenes, const gzg_render_params *params, int64_t n,
                           const gzg_batch_options *opts, gzg_renderer **out) {
        if (!out) return set_error(GZG_ERR_INVALID_ARGUMENT, "renderer: out is NULL");
        *out = nullptr;
        if (n <= 0 || !scenes || !params) return set_error(GZG_ERR_INVALID_ARGUMENT, "renderer: no scenes");
        auto r = std::make_unique<gzg_renderer>();
        for (int64_t k = 0; k < n; ++k) {
                if (!scenes[k]) return set_error(GZG_ERR_INVALID_ARGUMENT, "renderer: scene " + std::to_string(k) + " is NULL");
                if (n > 1 && (scene_is_instanced(scenes[k]) || scene_host_shading(scenes[k]).has_env))
                        return set_error(GZG_ERR_INVALID_ARGUMENT,
                                         "renderer: scene " + std::to_string(k) +
                                             " is two-level or has an environment light (single-scene renderers only)");
                if (!params_ok(params[k]))
                        return set_error(GZG_ERR_INVALID_ARGUMENT,
                                         "renderer: bad render parameters for scene " + std::to_string(k));
                DevScene v;
                int dev = 0, depth = 0;
                scene_view(scenes[k], &v, &dev, &depth);
                if (v.material_count <= 0)
                        return set_error(GZG_ERR_BAD_SCENE,
                                         "renderer: scene " + std::to_string(k) + " was uploaded without materials");
                if (k > 0 && dev != r->device)
                        return set_error(GZG_ERR_INVALID_ARGUMENT, "renderer: scenes on different devices");
                r->device = dev;
                r->scenes.push_back(scenes[k]);
                r->params.push_back(params[k]);
        }
        if (opts) r->opts = *opts;
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != r->device) cudaSetDevice(r->device);
        struct Restore {
                int prev, dev;
                ~Restore() {
                        if (prev != dev) cudaSetDevice(prev);
                }
        } restore{prev, r->device};
        gzg_status st = build_batch(r.get());
        if (st) return st;
        Wave &w = r->w;
        w.emission_scale = 1.0f;
        const uint64_t want = r->opts.wave_paths > 0 ? (uint64_t)r->opts.wave_paths : (uint64_t)kDefaultWave;
        r->max_capacity = (uint32_t)std::max<uint64_t>(
            1, std::min<uint64_t>(std::max<uint64_t>(want, kDefaultWave), w.total_paths));
        const size_t C = r->max_capacity;
        w.scene_count = (int32_t)n;
        const size_t keys = (size_t)std::max<int64_t>(n, r->view.material_count) + 1;
        if (keys > (1u << 20)) return set_error(GZG_ERR_LIMIT, "renderer: more than 2^20 sort keys");
        const SceneConst *scd = nullptr;
        if ((st = r->upload(&scd, r->consts))) return st;
        w.scenes = scd;
        if ((st = r->alloc(&w.zs_morton, C)) || (st = r->alloc(&w.zs_dim, C)) || (st = r->alloc(&w.thr, C)) ||
            (st = r->alloc(&w.L, C)) || (st = r->alloc(&w.pixel, C)) || (st = r->alloc(&w.scene, C)) ||
            (st = r->alloc(&w.weight, C)) || (st = r->alloc(&w.q_ray[0], 2 * C)) || (st = r->alloc(&w.q_ray[1], 2 * C)) ||
            (st = r->alloc(&w.q_id[0], C)) || (st = r->alloc(&w.q_id[1], C)) || (st = r->alloc(&w.hits, C)) ||
            (st = r->alloc(&w.sh_ray, 2 * C)) || (st = r->alloc(&w.sh_id, C)) || (st = r->alloc(&w.sh_contrib, C)) ||
            (st = r->alloc(&w.sh_occ, C)) || (st = r->alloc(&w.pr_ray, 2 * C)) || (st = r->alloc(&w.pr_id, C)) ||
            (st = r->alloc(&w.pr_contrib, C)) || (st = r->alloc(&w.pr_hits, C)) || (st = r->alloc(&w.order, C)) || (st = r->alloc(&w.gen_q, 2 * C)) ||
            (st = r->alloc(&w.alb, C)) || (st = r->alloc(&w.nrm, C)) ||
            (st = r->alloc(&w.key_hist, 2 * keys)) || (st = r->alloc(&w.counts, kCountWords)) ||
            (st = r->alloc(&w.stats, kStatWords)))
                return st;
        if (r->view.instances && ((st = r->alloc(&w.hit_inst, C)) || (st = r->alloc(&w.pr_inst, C)))) return st;
        if ((st = cuda_err(cudaMemset(w.key_hist, 0, 2 * keys * sizeof(uint32_t)), "sort histogram"))) return st;
        if ((st = cuda_err(cudaMemset(w.counts, 0, kCountWords * 4), "renderer counters"))) return st;
        if ((st = cuda_err(cudaMemset(w.stats, 0, kStatWords * 8), "renderer statistics"))) return st;
        r->configure((uint32_t)std::min<uint64_t>(want, w.total_paths), r->opts.sort_key);
        *out = r.release();
        return clear_error();
}

}  // namespace

extern "C" {

GZG_API gzg_status gzg_renderer_create(gzg_scene *scene, const gzg_render_params *params, gzg_renderer **out) {
        if (!params) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_create: null argument");
        gzg_batch_options o{};
        o.wave_paths = params->wave_paths;
        o.use_graph = params->use_graph;
        o.sort_key = GZG_SORT_NONE;
        return renderer_create(&scene, params, 1, &o, out);
}

GZG_API gzg_status gzg_batch_renderer_create(gzg_scene *const *scenes, const gzg_render_params *params,
                                             int64_t scene_count, const gzg_batch_options *options,
                                             gzg_renderer **out) {
        if (options && (options->sort_key < 0 || options->sort_key > 2))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_batch_renderer_create: unknown sort key");
        return renderer_create(scenes, params, scene_count, options, out);
}

GZG_API gzg_status gzg_renderer_film_layout(const gzg_renderer *r, int64_t *pixel_offsets) {
        if (!r || !pixel_offsets) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_film_layout: null argument");
        std::copy(r->film_offsets.begin(), r->film_offsets.end(), pixel_offsets);
        return clear_error();
}

GZG_API gzg_status gzg_renderer_destroy(gzg_renderer *renderer) {
        delete renderer;
        return clear_error();
}

GZG_API gzg_status gzg_renderer_render(gzg_renderer *r, float *film_rgb, float *film_sq, float *film_w, void *stream) {
        if (!r || !film_rgb || !film_w) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_render: null argument");
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != r->device) cudaSetDevice(r->device);
        const gzg_status st = r->render(film_rgb, film_sq, film_w, reinterpret_cast<cudaStream_t>(stream));
        if (prev != r->device) cudaSetDevice(prev);
        if (!st) clear_error();
        return st;
}

// Times whole renders over wave sizes and sort keys (into scratch films) and
// keeps the fastest configuration.
GZG_API gzg_status gzg_renderer_autotune(gzg_renderer *r, gzg_batch_options *best, float *best_ms, void *stream) {
        if (!r) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_autotune: null argument");
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != r->device) cudaSetDevice(r->device);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        const int64_t pix = r->film_offsets.back();
        float *rgb = nullptr, *wgt = nullptr;
        gzg_status status = r->alloc(&rgb, 3 * (size_t)pix);
        if (!status) status = r->alloc(&wgt, (size_t)pix);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        const uint32_t waves[] = {1u << 20, 1u << 21, 1u << 22, 1u << 23, 1u << 24};
        const int keys[] = {kSortNone, kSortMaterial, kSortScene};
        uint32_t best_cap = r->w.capacity;
        int best_key = r->w.sort_key;
        float best_t = 1e30f;
        const int saved_graph = r->opts.use_graph;
        r->opts.use_graph = 1;
        for (int key : keys)
                for (uint32_t cap : waves) {
                        if (status) break;
                        if (cap > r->max_capacity && cap != waves[0]) continue;
                        r->configure(cap, key);
                        status = r->render(rgb, nullptr, wgt, st);  // warm-up and graph capture
                        if (status) break;
                        cudaEventRecord(e0, st);
                        status = r->render(rgb, nullptr, wgt, st);
                        cudaEventRecord(e1, st);
                        if (!status) status = cuda_err(cudaEventSynchronize(e1), "renderer autotune");
                        float ms = 0;
                        cudaEventElapsedTime(&ms, e0, e1);
                        if (!status && ms < best_t) {
                                best_t = ms;
                                best_cap = r->w.capacity;
                                best_key = key;
                        }
                }
        r->opts.use_graph = saved_graph;
        if (!status) status = cuda_err(cudaMemsetAsync(r->w.stats, 0, kStatWords * 8, st), "renderer statistics");
        r->configure(best_cap, best_key);
        r->opts.wave_paths = (int32_t)best_cap;
        r->opts.sort_key = best_key;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (!status && best) *best = r->opts;
        if (!status && best_ms) *best_ms = best_t;
        if (prev != r->device) cudaSetDevice(prev);
        if (!status) clear_error();
        return status;
}

GZG_API gzg_status gzg_renderer_set_film(gzg_renderer *r, float iso, float max_component) {
        if (!r || !(iso > 0.0f) || !std::isfinite(iso) || !(max_component >= 0.0f) || !std::isfinite(max_component))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_set_film: bad arguments");
        for (SceneConst &sc : r->consts) {
                sc.film_scale = iso / 100.0f;
                sc.max_component = max_component;
        }
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != r->device) cudaSetDevice(r->device);
        const gzg_status st = cuda_err(cudaMemcpy(const_cast<SceneConst *>(r->w.scenes), r->consts.data(),
                                                  r->consts.size() * sizeof(SceneConst), cudaMemcpyHostToDevice),
                                       "film settings");
        if (prev != r->device) cudaSetDevice(prev);
        if (st) return st;
        r->drop_graph();
        return clear_error();
}

GZG_API gzg_status gzg_renderer_render_aov(gzg_renderer *r, float *film_rgb, float *film_sq, float *film_w,
                                           float *film_albedo, float *film_normal, void *stream) {
        if (!r || !film_rgb || !film_w)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_render_aov: null argument");
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != r->device) cudaSetDevice(r->device);
        const gzg_status st = r->render(film_rgb, film_sq, film_w, reinterpret_cast<cudaStream_t>(stream), film_albedo,
                                        film_normal);
        if (prev != r->device) cudaSetDevice(prev);
        if (!st) clear_error();
        return st;
}

GZG_API gzg_status gzg_renderer_set_textures(gzg_renderer *r, const gzg_texture_binding *bindings, int32_t count,
                                             int32_t resolution, const float *texels, float emission_scale) {
        if (!r) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_set_textures: null renderer");
        if (r->scenes.size() != 1)
                return set_error(GZG_ERR_INVALID_ARGUMENT,
                                 "gzg_renderer_set_textures: textures need a single-scene renderer");
        if (count < 0 || (count > 0 && (!bindings || !texels || resolution < 1 || resolution > 16384)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_set_textures: bad texture arguments");
        if (!std::isfinite(emission_scale))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_set_textures: emission scale not finite");
        if ((int64_t)count * resolution * resolution * 3 >= ((int64_t)1 << 31))
                return set_error(GZG_ERR_LIMIT, "gzg_renderer_set_textures: more than 2^31 texel values");
        const int32_t nm = r->view.material_count;
        std::vector<int32_t> mat_tex(nm, -1);
        std::vector<float> maps(9 * (size_t)count);
        for (int32_t t = 0; t < count; ++t) {
                const gzg_texture_binding &b = bindings[t];
                if (b.material < 0 || b.material >= nm)
                        return set_error(GZG_ERR_INVALID_ARGUMENT,
                                         "gzg_renderer_set_textures: binding " + std::to_string(t) + " names material " +
                                             std::to_string(b.material) + " of " + std::to_string(nm));
                mat_tex[b.material] = t;
                std::copy(b.origin, b.origin + 3, maps.begin() + 9 * t);
                std::copy(b.u_axis, b.u_axis + 3, maps.begin() + 9 * t + 3);
                std::copy(b.v_axis, b.v_axis + 3, maps.begin() + 9 * t + 6);
        }
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != r->device) cudaSetDevice(r->device);
        gzg_status st = GZG_OK;
        if (count > 0) {
                if (!r->d_mat_tex) st = r->alloc(&r->d_mat_tex, (size_t)nm);
                if (!st && count > r->tex_slots) {
                        st = r->alloc(&r->d_tex_map, 9 * (size_t)count);
                        if (!st) r->tex_slots = count;
                }
                if (!st)
                        st = cuda_err(cudaMemcpy(r->d_mat_tex, mat_tex.data(), 4 * (size_t)nm, cudaMemcpyHostToDevice),
                                      "texture bindings");
                if (!st)
                        st = cuda_err(cudaMemcpy(r->d_tex_map, maps.data(), 4 * maps.size(), cudaMemcpyHostToDevice),
                                      "texture maps");
        }
        if (prev != r->device) cudaSetDevice(prev);
        if (st) return st;
        r->w.tex = count > 0 ? texels : nullptr;
        r->w.mat_tex = count > 0 ? r->d_mat_tex : nullptr;
        r->w.tex_map = count > 0 ? r->d_tex_map : nullptr;
        r->w.tex_res = count > 0 ? resolution : 0;
        r->w.emission_scale = emission_scale;
        r->drop_graph();
        return clear_error();
}

GZG_API gzg_status gzg_renderer_render_f64(gzg_renderer *r, double *film_rgb, double *film_sq, double *film_w,
                                           void *stream) {
        if (!r || !film_rgb || !film_w)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_render_f64: null argument");
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != r->device) cudaSetDevice(r->device);
        const gzg_status st = r->render_f64(film_rgb, film_sq, film_w, reinterpret_cast<cudaStream_t>(stream));
        if (prev != r->device) cudaSetDevice(prev);
        if (!st) clear_error();
        return st;
}

GZG_API gzg_status gzg_renderer_adjoint(gzg_renderer *r, const float *adj_rgb, const float *film_w, float *d_texels,
                                        double *d_emission, void *stream) {
        if (!r || !adj_rgb || !film_w) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_adjoint: null argument");
        if (r->w.mat_tex && !d_texels)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_adjoint: textures bound but no texel gradient");
        if (d_emission && r->w.emission_scale == 0.0f)
                return set_error(GZG_ERR_INVALID_ARGUMENT,
                                 "gzg_renderer_adjoint: emission gradient needs a nonzero scale");
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != r->device) cudaSetDevice(r->device);
        const gzg_status st = r->adjoint(adj_rgb, film_w, d_texels, d_emission, reinterpret_cast<cudaStream_t>(stream));
        if (prev != r->device) cudaSetDevice(prev);
        if (!st) clear_error();
        return st;
}

GZG_API gzg_status gzg_renderer_error_word(gzg_renderer *r, uint32_t *word, int32_t clear) {
        if (!r || !word) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_error_word: null argument");
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != r->device) cudaSetDevice(r->device);
        gzg_status st = cuda_err(cudaMemcpy(word, r->view.err, 4, cudaMemcpyDeviceToHost), "error word read");
        if (!st && clear) st = cuda_err(cudaMemset(r->view.err, 0, 4), "error word clear");
        if (prev != r->device) cudaSetDevice(prev);
        if (!st) clear_error();
        return st;
}

GZG_API gzg_status gzg_renderer_stats(const gzg_renderer *r, gzg_render_stats *out) {
        if (!r || !out) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_stats: null argument");
        unsigned long long s[kStatWords];
        gzg_status st = cuda_err(cudaMemcpy(s, r->w.stats, sizeof(s), cudaMemcpyDeviceToHost), "renderer statistics");
        if (st) return st;
        out->camera_rays = s[kStatCamera];
        out->extension_rays = s[kStatExt];
        out->shadow_rays = s[kStatShadow];
        out->probe_rays = s[kStatProbe];
        out->waves = s[kStatWaves];
        return clear_error();
}

GZG_API gzg_status gzg_zsobol_fill_device(int64_t samples_per_pixel, int32_t res_x, int32_t res_y, int64_t seed,
                                          const int32_t *px, const int32_t *py, const int64_t *index, int64_t n,
                                          const int32_t *kinds, int32_t nkinds, float *out, void *stream) {
        if (samples_per_pixel <= 0 || res_x <= 0 || res_y <= 0 || n < 0 || nkinds < 0 || nkinds > 64 ||
            (n > 0 && (!px || !py || !index || !out)) || (nkinds > 0 && !kinds))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_zsobol_fill_device: bad arguments");
        int per = 0;
        for (int k = 0; k < nkinds; ++k) {
                if (kinds[k] < 1 || kinds[k] > 3)
                        return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_zsobol_fill_device: kind not 1, 2 or 3");
                per += kinds[k];
        }
        if (n == 0 || nkinds == 0) return clear_error();
        int dev = 0;
        cudaGetDevice(&dev);
        const uint32_t *matrices = nullptr;
        gzg_status st = device_sobol(dev, &matrices);
        if (st) return st;
        const ZSobolConfig c = make_zsobol(samples_per_pixel, res_x, res_y, seed, matrices);
        KindList kl{};
        for (int k = 0; k < nkinds; ++k) kl.k[k] = kinds[k];
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        k_zsobol_fill<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(c, px, py, index, n, kl, nkinds, per, out);
        st = cuda_err(cudaGetLastError(), "zsobol launch");
        if (!st) clear_error();
        return st;
}

GZG_API gzg_status gzg_camera_rays(const gzg_render_params *params, int64_t first_path, int64_t count, gzg_ray *rays,
                                   float *weights, int32_t *pixels) {
        if (!params || first_path < 0 || count < 0 || (count > 0 && (!rays || !weights || !pixels)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_camera_rays: null argument or negative range");
        if (!params_ok(*params)) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_camera_rays: bad render parameters");
        const int64_t total = film_pixels(*params) * params->spp;
        if (first_path > total || count > total - first_path)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_camera_rays: paths beyond the film's pixels x spp");
        if (count == 0) return clear_error();
        int dev = 0;
        cudaGetDevice(&dev);
        const uint32_t *matrices = nullptr;
        gzg_status st = device_sobol(dev, &matrices);
        if (st) return st;
        const SceneConst sc = make_scene_const(*params, matrices);
        const size_t bytes = (size_t)count * (6 * sizeof(float) + sizeof(float) + sizeof(int32_t));
        char *d = nullptr;
        if (cudaMalloc(&d, bytes) != cudaSuccess) {
                cudaGetLastError();
                return set_error(GZG_ERR_OUT_OF_MEMORY, "gzg_camera_rays: device buffer");
        }
        float *d_rays = reinterpret_cast<float *>(d);
        float *d_w = d_rays + 6 * count;
        int32_t *d_px = reinterpret_cast<int32_t *>(d_w + count);
        do {
                k_camera_rays<<<(unsigned)((count + 127) / 128), 128>>>(sc, (uint64_t)first_path, (uint64_t)count,
                                                                        d_rays, d_w, d_px);
                if ((st = cuda_err(cudaGetLastError(), "camera ray launch"))) break;
                if ((st = cuda_err(cudaMemcpy(rays, d_rays, (size_t)count * 24, cudaMemcpyDeviceToHost), "ray copy")))
                        break;
                if ((st = cuda_err(cudaMemcpy(weights, d_w, (size_t)count * 4, cudaMemcpyDeviceToHost), "weight copy")))
                        break;
                st = cuda_err(cudaMemcpy(pixels, d_px, (size_t)count * 4, cudaMemcpyDeviceToHost), "pixel copy");
        } while (false);
        cudaFree(d);
        if (!st) clear_error();
        return st;
}

GZG_API gzg_status gzg_render_image(gzg_scene *scene, const gzg_render_params *params, float *film_rgb, float *film_sq,
                                    float *film_w, gzg_render_stats *stats) {
        if (!scene || !params || !film_rgb || !film_w)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_render_image: null argument");
        gzg_renderer *r = nullptr;
        gzg_status st = gzg_renderer_create(scene, params, &r);
        if (st) return st;
        std::unique_ptr<gzg_renderer> hold(r);
        const size_t pix = (size_t)film_pixels(*params);
        float *d_rgb = nullptr, *d_sq = nullptr, *d_w = nullptr;
        if ((st = r->alloc(&d_rgb, 3 * pix)) || (st = r->alloc(&d_w, pix))) return st;
        if (film_sq && (st = r->alloc(&d_sq, 3 * pix))) return st;
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != r->device) cudaSetDevice(r->device);
        do {
                if ((st = cuda_err(cudaMemset(d_rgb, 0, 3 * pix * 4), "film clear"))) break;
                if ((st = cuda_err(cudaMemset(d_w, 0, pix * 4), "film clear"))) break;
                if (d_sq && (st = cuda_err(cudaMemset(d_sq, 0, 3 * pix * 4), "film clear"))) break;
                if ((st = r->render(d_rgb, d_sq, d_w, nullptr))) break;
                if ((st = wait_stream(nullptr, "gzg_render_image"))) break;
                if ((st = cuda_err(cudaMemcpy(film_rgb, d_rgb, 3 * pix * 4, cudaMemcpyDeviceToHost), "film copy"))) break;
                if ((st = cuda_err(cudaMemcpy(film_w, d_w, pix * 4, cudaMemcpyDeviceToHost), "film copy"))) break;
                if (d_sq && (st = cuda_err(cudaMemcpy(film_sq, d_sq, 3 * pix * 4, cudaMemcpyDeviceToHost), "film copy")))
                        break;
                if (stats && (st = gzg_renderer_stats(r, stats))) break;
                uint32_t word = 0;
                if ((st = gzg_scene_error_word(scene, &word, 1))) break;
                if (word) st = set_error(GZG_ERR_KERNEL_FAULT, "render: kernel error word " + std::to_string(word));
        } while (false);
        if (prev != r->device) cudaSetDevice(prev);
        // after a wait that ran out the frame is still rendering into the
        // renderer's buffers and the films: they are left to it
        if (st == GZG_ERR_TIMEOUT) hold.release();
        if (!st) clear_error();
        return st;
}

}  // extern "C"
