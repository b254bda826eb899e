// render.cu - the path integrator as a device-resident wavefront.
//
// Gonzales runs its bounce loop on the host, one tile at a time, shipping rays
// and path states to the plugin and back every bounce (Core/Tile.swift:66-209).
// Here a wave of paths lives in device memory for its whole life:
//
//   generate   Z-Sobol camera sample, Gaussian filter sample, pinhole ray
//   per bounce b = 0 .. max_depth-1:
//     extend   closest hit of the extension queue (k_wide_persistent)
//     shade    emission, light choice + light sample (-> shadow queue),
//              MIS BSDF sample (-> probe queue, corrected MIS only),
//              continuation sample, Russian roulette (-> next extension queue)
//     shadow   any hit of the shadow queue, then add unoccluded contributions
//     probe    closest hit of the probe queue, then add emission it reaches
//   accumulate film sums (radiance, its square, filter weight) with atomics
//
// Queue lengths live on the device; no stage waits for the host, so a whole
// wave can be captured once as a CUDA graph and replayed.  The shading
// arithmetic restates Integrator/VolumePathIntegrator.swift:67-463 and the
// helpers it calls (same citations as the CPU oracle's integrator).  The
// reference's last extension (bounce == max_depth) can only add environment
// light to camera or specular paths; these scenes have neither, so it is not
// traced.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "gzg_internal.h"
#include "kernels.h"
#include "sobol.cuh"

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
__device__ V3 cosine_hemisphere(float u0, float u1) {
        const float ox = 2.0f * u0 - 1.0f, oy = 2.0f * u1 - 1.0f;
        float dx = 0.0f, dy = 0.0f;
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

// Shading frame of a hit without UVs or vertex normals (Shape/Triangle.swift:
// 395-452 with degenerate UVs, Reflection/BsdfFrame.swift:13-21).
__device__ bool make_frame(V3 p0, V3 p1, V3 p2, V3 ns, Frame &f) {
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
        f.y = normalize(s);
        f.z = ns;
        f.x = cross(f.y, f.z);
        return true;
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

// ------------------------------------------------------------ state

struct RenderConst {
        V3 eye, right, up, fwd;
        float tan_half, sx0, sx1, sy0, sy1;
        int32_t width, height, spp, max_depth, rr_min, mis_corrected, first_sample;
        float filter_radius, filter_sigma;
        ZSobolConfig zs;
};

enum { kCountExt0 = 0, kCountExt1 = 1, kCountShadow = 2, kCountProbe = 3, kCountWaveBase = 4, kCountWords = 8 };
enum { kStatCamera = 0, kStatExt = 1, kStatShadow = 2, kStatProbe = 3, kStatWaves = 4, kStatWords = 8 };

struct Wave {
        uint32_t capacity;
        uint64_t total_paths;
        // path state, indexed by path slot in the wave
        uint64_t *zs_morton;
        int32_t *zs_dim;
        float4 *thr;
        float4 *L;
        uint32_t *pixel;
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
        uint32_t *counts;           // kCountWords words; wave base as 2 words at kCountWaveBase
        unsigned long long *stats;  // kStatWords
};

// Appends to a queue with one atomic per converged group of lanes.
__device__ __forceinline__ uint32_t queue_slot(uint32_t *count) {
        const unsigned mask = __activemask();
        const unsigned lane = threadIdx.x & 31u;
        const int leader = __ffs(mask) - 1;
        uint32_t base = 0;
        if ((int)lane == leader) base = atomicAdd(count, (uint32_t)__popc(mask));
        base = __shfl_sync(mask, base, leader);
        return base + __popc(mask & ((1u << lane) - 1u));
}

__device__ __forceinline__ void store_ray(float4 *q, uint32_t slot, V3 o, float tmax, V3 d) {
        q[2 * slot] = make_float4(o.x, o.y, o.z, tmax);
        q[2 * slot + 1] = make_float4(d.x, d.y, d.z, 0.0f);
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
__device__ __forceinline__ void prim_info(const DevScene &s, int prim, int &type, int64_t &material, int64_t &id1) {
        const long long *r = reinterpret_cast<const long long *>(s.prims + prim);
        id1 = __ldg(r);
        material = __ldg(r + 2);
        type = (int)(signed char)(__ldg(reinterpret_cast<const unsigned char *>(r + 3)));
}

// ------------------------------------------------------------ kernels

// generate: Tile.render phase 1 (Core/Tile.swift:27-59) for the paths
// [base, base + count) of the render; path p is sample p % spp of pixel p / spp.
__global__ void k_generate(RenderConst rc, Wave w) {
        const uint32_t count = wave_count(w);
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (threadIdx.x == 0 && blockIdx.x == 0) {
                w.counts[kCountExt0] = count;
                atomicAdd(w.stats + kStatCamera, (unsigned long long)count);
                atomicAdd(w.stats + kStatWaves, 1ull);
        }
        if (i >= count) return;
        const uint64_t path = wave_base(w) + i;
        const uint32_t pixel = (uint32_t)(path / (uint64_t)rc.spp);
        const uint32_t sample = (uint32_t)(path % (uint64_t)rc.spp) + (uint32_t)rc.first_sample;
        const uint32_t px = pixel % (uint32_t)rc.width, py = pixel / (uint32_t)rc.width;
        ZSobol z;
        zs_start(rc.zs, z, px, py, sample);
        // getCameraSample (Sampler/Sampler.swift:69-82)
        float u0, u1;
        zs_get2d(rc.zs, z, u0, u1);
        float dx, dy, denx, deny;
        gaussian_sample_1d(u0, rc.filter_radius, rc.filter_sigma, dx, denx);
        gaussian_sample_1d(u1, rc.filter_radius, rc.filter_sigma, dy, deny);
        const float fx = (float)px + 0.5f + dx, fy = (float)py + 0.5f + dy;
        float l0, l1;
        zs_get2d(rc.zs, z, l0, l1);  // lens sample: drawn, unused by a pinhole
        // raster -> screen -> camera -> world (pinhole)
        const float scx = rc.sx0 + fx / (float)rc.width * (rc.sx1 - rc.sx0);
        const float scy = rc.sy1 - fy / (float)rc.height * (rc.sy1 - rc.sy0);
        const V3 dcam = normalize(v3(scx * rc.tan_half, scy * rc.tan_half, 1.0f));
        const V3 dir = rc.right * dcam.x + rc.up * dcam.y + rc.fwd * dcam.z;
        // rayWeight = filter value / filter pdf (Tile.swift:36-40)
        const float ddx = fx - ((float)px + 0.5f), ddy = fy - ((float)py + 0.5f);
        const float fv = fmaxf(0.0f, gaussian(ddx, rc.filter_sigma)) * fmaxf(0.0f, gaussian(ddy, rc.filter_sigma));
        w.zs_morton[i] = z.morton;
        w.zs_dim[i] = z.dim;
        w.thr[i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        w.L[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        w.pixel[i] = pixel;
        w.weight[i] = fv / (denx * deny);
        store_ray(w.q_ray[0], i, rc.eye, kInf, dir);
        w.q_id[0][i] = i;
}

// Power light sampler: lowerBound over the running power sum
// (Light/PowerLightSampler.swift:4-48).
__device__ int choose_light(const DevScene &s, float u, float &pdf) {
        const float key = u * s.light_total_power;
        int lo = 0, hi = s.light_count;
        while (lo < hi) {
                const int mid = lo + (hi - lo) / 2;
                const float c = __ldg(s.light_cdf + mid);
                if (c == key) {
                        lo = mid;
                        break;
                } else if (c < key) {
                        lo = mid + 1;
                } else {
                        hi = mid;
                }
        }
        if (lo >= s.light_count) lo = s.light_count - 1;
        pdf = __ldg(s.lights + 4 * lo + 1).w / s.light_total_power;
        return lo;
}

// offsetRayOrigin(point:normal:direction:) (Core/Interaction.swift:26-35).
__device__ __forceinline__ V3 offset_origin(V3 p, V3 n, V3 dir) {
        const V3 off = n * 0.0001f;
        return dot(dir, n) > 0.0f ? p + off : p + neg(off);
}

// shade: VolumePathIntegrator.shadeBounce + surfaceEstimate (:325-430).
__global__ void k_shade(RenderConst rc, Wave w, DevScene s, int bounce, int cur) {
        const uint32_t n = w.counts[cur];
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n) return;
        const uint32_t path = w.q_id[cur][i];
        const float4 hit = w.hits[i];
        const int prim = __float_as_int(hit.w);
        if (prim < 0) return;  // miss: no environment light
        V3 thr = v3(w.thr[path]);
        if (is_black(thr)) return;
        if (bounce >= rc.max_depth) return;
        const float4 rd = w.q_ray[cur][2 * i + 1];
        const V3 d = v3(rd);
        V3 p0, p1, p2;
        prim_triangle_dev(s, prim, p0, p1, p2);
        const float b0 = (1.0f - hit.y) - hit.z;
        const V3 pos = p0 * b0 + p1 * hit.y + p2 * hit.z;
        const V3 ng = normalize(cross(p0 - p2, p1 - p2));
        const V3 wo = normalize(neg(d));
        int type;
        int64_t mat_index, id1;
        prim_info(s, prim, type, mat_index, id1);
        const bool is_light = type == 3;
        float4 Lacc = w.L[path];
        V3 L = v3(Lacc);
        if (bounce == 0 && is_light && mat_index >= 0 && mat_index < s.material_count) {
                const V3 le = v3(__ldg(s.materials + 2 * mat_index + 1));
                if (dot(ng, wo) > 0.0f) L = L + mulv(thr, le);
        }
        // Area-light hits scatter with material 0 (their interaction keeps
        // materialIndex 0, Core/SurfaceInteraction.swift:20).
        const int64_t mi = is_light ? 0 : mat_index;
        const V3 refl = (mi >= 0 && mi < s.material_count) ? v3(__ldg(s.materials + 2 * mi)) : v3(0.5f, 0.5f, 0.5f);
        const V3 f_val = refl * (1.0f / kPi);
        Frame fr;
        ZSobol z;
        z.morton = w.zs_morton[path];
        z.dim = w.zs_dim[path];
        bool alive = make_frame(p0, p1, p2, ng, fr);
        if (alive && s.light_count > 0) {
                const V3 wo_l = fr.to_local(wo);
                // ---- light choice and light sample (sampleLightSource, :67-89)
                float choose_pdf;
                const int li = choose_light(s, zs_get1d(rc.zs, z), choose_pdf);
                const float4 l0 = __ldg(s.lights + 4 * li), l1 = __ldg(s.lights + 4 * li + 1),
                             l2 = __ldg(s.lights + 4 * li + 2), le4 = __ldg(s.lights + 4 * li + 3);
                const V3 lp0 = v3(l0), lp1 = v3(l1), lp2 = v3(l2), le = v3(le4);
                const float area = l0.w;
                float u0, u1;
                zs_get2d(rc.zs, z, u0, u1);
                const float su0 = sqrtf(u0);
                const float lb0 = 1.0f - su0, lb1 = u1 * su0;
                const V3 lp = lp0 * lb0 + lp1 * lb1 + lp2 * ((1.0f - lb0) - lb1);
                const V3 ln = normalize(cross(lp1 - lp0, lp2 - lp0));
                const V3 inc = normalize(lp - pos);
                const V3 dl = pos - lp;
                const float pdf = (1.0f / area) * (dot(dl, dl) / fabsf(dot(ln, neg(inc))));
                float light_pdf = 0.0f;
                V3 light_est = v3(0, 0, 0), light_dir = v3(0, 0, 0);
                if (dot(ln, neg(inc)) > 0.0f && !isinf(pdf)) {
                        const bool reflect = dot(inc, ng) * dot(wo, ng) > 0.0f;
                        const V3 f = reflect ? f_val : v3(0, 0, 0);
                        light_est = mulv(f * fabsf(dot(inc, ng)), le);
                        light_dir = inc;
                        light_pdf = pdf;
                }
                float brdf_density = 0.0f;
                {
                        const V3 wi_l = fr.to_local(light_dir);
                        if (wo_l.z != 0.0f && wo_l.z * wi_l.z > 0.0f) brdf_density = fabsf(wi_l.z) / kPi;
                }
                const float light_w = power_heuristic(light_pdf, brdf_density);
                if (light_pdf != 0.0f && !is_black(light_est)) {
                        // Visibility.occluded via spawnRay(from:target:) (Interaction.swift:15-24)
                        const V3 so = pos + (lp - pos) * 0.0001f;
                        const V3 sd = lp - so;
                        const V3 c = mulv(thr, light_est * (light_w / light_pdf) * (1.0f / choose_pdf));
                        const uint32_t slot = queue_slot(w.counts + kCountShadow);
                        store_ray(w.sh_ray, slot, so, 1.0f - 0.00001f, sd);
                        w.sh_id[slot] = path;
                        w.sh_contrib[slot] = make_float4(c.x, c.y, c.z, 0.0f);
                }
                // ---- MIS BSDF sample (sampleDistributionFunction, :91-133)
                float v0, v1, v2;
                zs_get3d(rc.zs, z, v0, v1, v2);
                if (rc.mis_corrected) {
                        V3 wi_l = cosine_hemisphere(v0, v1);
                        if (wo_l.z < 0.0f) wi_l.z = -wi_l.z;
                        const float pdf_b = (wo_l.z * wi_l.z > 0.0f) ? fabsf(wi_l.z) / kPi : 0.0f;
                        const V3 wi = fr.to_world(wi_l);
                        const V3 est = f_val * fabsf(dot(wi, ng));
                        if (!is_black(est) && pdf_b > 0.0f) {
                                const V3 po = offset_origin(pos, ng, wi);
                                // light density of the chosen light along wi (Sampleable.swift:47-68 with tHit = inf)
                                float light_density = 0.0f;
                                float tl, lu, lv;
                                const float4 a4 = make_float4(lp0.x, lp0.y, lp0.z, 0.0f), b4 = make_float4(lp1.x, lp1.y, lp1.z, 0.0f),
                                             c4 = make_float4(lp2.x, lp2.y, lp2.z, 0.0f);
                                if (watertight_test(po.x, po.y, po.z, wi.x, wi.y, wi.z, a4, b4, c4, kInf, tl, lu, lv)) {
                                        const V3 hp = po + wi * tl;
                                        const V3 dq = pos - hp;
                                        const V3 lnn = normalize(cross(lp0 - lp2, lp1 - lp2));
                                        const float dens = dot(dq, dq) / (fabsf(dot(lnn, neg(wi))) * area);
                                        light_density = isinf(dens) ? 0.0f : dens;
                                }
                                const float bw = power_heuristic(pdf_b, light_density);
                                if (bw > 0.0f) {
                                        const V3 c = mulv(thr, est * (bw / pdf_b) * (1.0f / choose_pdf));
                                        const uint32_t slot = queue_slot(w.counts + kCountProbe);
                                        store_ray(w.pr_ray, slot, po, kInf, wi);
                                        w.pr_id[slot] = path;
                                        w.pr_contrib[slot] = make_float4(c.x, c.y, c.z, 0.0f);
                                }
                        }
                }
                // ---- continuation (bsdf.sampleWorldSpace, :358-369)
                zs_get3d(rc.zs, z, v0, v1, v2);
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
                        if (mv < 1.0f && bounce >= rc.rr_min) {
                                const float q = fmaxf(0.0f, 1.0f - mv);
                                if (zs_get1d(rc.zs, z) < q)
                                        alive = false;
                                else
                                        thr = thr * (1.0f / (1.0f - q));
                        }
                        if (alive && bounce + 1 < rc.max_depth) {
                                const int nxt = cur ^ 1;
                                const uint32_t slot = queue_slot(w.counts + nxt);
                                store_ray(w.q_ray[nxt], slot, o, kInf, wi);
                                w.q_id[nxt][slot] = path;
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

// Adds the emission a BSDF probe reaches (corrected MIS): the probe's closest
// hit must be an area light whose normal faces back along the probe.
__global__ void k_probe_resolve(Wave w, DevScene s) {
        const uint32_t n = w.counts[kCountProbe];
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n) return;
        const float4 h = w.pr_hits[i];
        const int prim = __float_as_int(h.w);
        if (prim < 0) return;
        int type;
        int64_t mat_index, id1;
        prim_info(s, prim, type, mat_index, id1);
        if (type != 3 || mat_index < 0 || mat_index >= s.material_count) return;
        V3 q0, q1, q2;
        prim_triangle_dev(s, prim, q0, q1, q2);
        const V3 qn = normalize(cross(q0 - q2, q1 - q2));
        const V3 wi = v3(w.pr_ray[2 * i + 1]);
        if (!(dot(qn, neg(wi)) > 0.0f)) return;
        const V3 le = v3(__ldg(s.materials + 2 * mat_index + 1));
        const uint32_t path = w.pr_id[i];
        const float4 c = w.pr_contrib[i];
        float4 L = w.L[path];
        L.x += c.x * le.x;
        L.y += c.y * le.y;
        L.z += c.z * le.z;
        w.L[path] = L;
}

// Per-bounce bookkeeping: ray statistics of this bounce, then the counters of
// the queues the next stages fill are cleared.
__global__ void k_bounce_tally(Wave w, int cur) {
        atomicAdd(w.stats + kStatExt, (unsigned long long)w.counts[cur]);
        atomicAdd(w.stats + kStatShadow, (unsigned long long)w.counts[kCountShadow]);
        atomicAdd(w.stats + kStatProbe, (unsigned long long)w.counts[kCountProbe]);
}

__global__ void k_clear_counts(Wave w, int next) {
        w.counts[next] = 0;
        w.counts[kCountShadow] = 0;
        w.counts[kCountProbe] = 0;
}

// Film sums (Core/Film.swift:107-119): radiance (iso 100 -> scale 1), its
// square, and the filter weight, per pixel; then advance the wave base.
__global__ void k_accumulate(Wave w, float *film_rgb, float *film_sq, float *film_w) {
        const uint32_t count = wave_count(w);
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i < count) {
                const uint32_t px = w.pixel[i];
                const float4 L = w.L[i];
                atomicAdd(film_rgb + 3 * (size_t)px, L.x);
                atomicAdd(film_rgb + 3 * (size_t)px + 1, L.y);
                atomicAdd(film_rgb + 3 * (size_t)px + 2, L.z);
                if (film_sq) {
                        atomicAdd(film_sq + 3 * (size_t)px, L.x * L.x);
                        atomicAdd(film_sq + 3 * (size_t)px + 1, L.y * L.y);
                        atomicAdd(film_sq + 3 * (size_t)px + 2, L.z * L.z);
                }
                atomicAdd(film_w + px, w.weight[i]);
        }
}

__global__ void k_advance_wave(Wave w) {
        const uint64_t next = wave_base(w) + wave_count(w);
        w.counts[kCountWaveBase] = (uint32_t)(next & 0xFFFFFFFFull);
        w.counts[kCountWaveBase + 1] = (uint32_t)(next >> 32);
}

// Z-Sobol values for n pixel samples: the sequence of get1D/get2D/get3D
// calls in `kinds` (1, 2 or 3 each), starting at dimension 0.
struct KindList {
        int32_t k[64];
};

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

__global__ void k_set_wave_base(Wave w, uint64_t base) {
        w.counts[kCountWaveBase] = (uint32_t)(base & 0xFFFFFFFFull);
        w.counts[kCountWaveBase + 1] = (uint32_t)(base >> 32);
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

V3 hv3(float x, float y, float z) { return V3{x, y, z}; }
V3 hsub(V3 a, V3 b) { return hv3(a.x - b.x, a.y - b.y, a.z - b.z); }
V3 hcross(V3 a, V3 b) { return hv3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
V3 hnorm(V3 a) {
        const float l = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
        return hv3(a.x / l, a.y / l, a.z / l);
}

}  // namespace
}  // namespace gzg

using namespace gzg;

struct gzg_renderer {
        gzg_scene *scene = nullptr;
        int device = 0;
        gzg_render_params params{};
        RenderConst rc{};
        Wave w{};
        DevScene view{};
        int wide_depth = 0;
        std::vector<void *> allocs;
        cudaGraphExec_t graph = nullptr;
        cudaGraph_t graph_def = nullptr;
        float *graph_film[3] = {nullptr, nullptr, nullptr};

        ~gzg_renderer() {
                int prev = 0;
                cudaGetDevice(&prev);
                if (prev != device) cudaSetDevice(device);
                if (graph) cudaGraphExecDestroy(graph);
                if (graph_def) cudaGraphDestroy(graph_def);
                for (void *p : allocs) cudaFree(p);
                if (prev != device) cudaSetDevice(prev);
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

        // One wave: generate, bounces, accumulate, advance.  Enqueued on st.
        cudaError_t enqueue_wave(float *film_rgb, float *film_sq, float *film_w, cudaStream_t st) {
                const int block = 128;
                const unsigned grid = (w.capacity + block - 1) / block;
                k_generate<<<grid, block, 0, st>>>(rc, w);
                int cur = 0;
                for (int b = 0; b < rc.max_depth; ++b) {
                        k_clear_counts<<<1, 1, 0, st>>>(w, cur ^ 1);
                        // the scene's tuned launches (gzg_scene_autotune)
                        LaunchParams lp = scene_launch(scene, false);
                        LaunchParams lpa = scene_launch(scene, true);
                        lp.n_dev = w.counts + cur;
                        cudaError_t e = launch_trace(view, lp, kRayDevice, kOutHit, w.q_ray[cur], nullptr, w.capacity,
                                                     w.hits, st);
                        if (e != cudaSuccess) return e;
                        k_shade<<<grid, block, 0, st>>>(rc, w, view, b, cur);
                        lpa.n_dev = w.counts + kCountShadow;
                        e = launch_trace(view, lpa, kRayDevice, kOutAnyPrim, w.sh_ray, nullptr, w.capacity, w.sh_occ, st);
                        if (e != cudaSuccess) return e;
                        k_shadow_resolve<<<grid, block, 0, st>>>(w);
                        if (rc.mis_corrected) {
                                lp.n_dev = w.counts + kCountProbe;
                                e = launch_trace(view, lp, kRayDevice, kOutHit, w.pr_ray, nullptr, w.capacity, w.pr_hits,
                                                 st);
                                if (e != cudaSuccess) return e;
                                k_probe_resolve<<<grid, block, 0, st>>>(w, view);
                        }
                        k_bounce_tally<<<1, 1, 0, st>>>(w, cur);
                        cur ^= 1;
                }
                k_accumulate<<<grid, block, 0, st>>>(w, film_rgb, film_sq, film_w);
                k_advance_wave<<<1, 1, 0, st>>>(w);
                return cudaGetLastError();
        }
};

namespace {

gzg_status cuda_err(cudaError_t e, const char *what) {
        if (e == cudaSuccess) return GZG_OK;
        return set_error(e == cudaErrorMemoryAllocation ? GZG_ERR_OUT_OF_MEMORY : GZG_ERR_CUDA,
                         std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" {

GZG_API gzg_status gzg_renderer_create(gzg_scene *scene, const gzg_render_params *params, gzg_renderer **out) {
        if (!out) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_create: out is NULL");
        *out = nullptr;
        if (!scene || !params) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_create: null argument");
        const gzg_render_params &P = *params;
        if (P.width <= 0 || P.height <= 0 || P.spp <= 0 || P.max_depth < 0 || P.fov_deg <= 0.0f ||
            P.filter_sigma <= 0.0f || P.filter_radius <= 0.0f || P.first_sample < 0 || P.sampler_spp < 0)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_renderer_create: bad render parameters");
        auto r = std::make_unique<gzg_renderer>();
        r->scene = scene;
        r->params = P;
        scene_view(scene, &r->view, &r->device, &r->wide_depth);
        if (r->view.material_count <= 0)
                return set_error(GZG_ERR_BAD_SCENE, "gzg_renderer_create: the scene was uploaded without materials");
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != r->device) cudaSetDevice(r->device);
        struct Restore {
                int prev, dev;
                ~Restore() {
                        if (prev != dev) cudaSetDevice(prev);
                }
        } restore{prev, r->device};

        RenderConst &rc = r->rc;
        const V3 eye = hv3(P.eye[0], P.eye[1], P.eye[2]);
        const V3 fwd = hnorm(hsub(hv3(P.target[0], P.target[1], P.target[2]), eye));
        const V3 right = hnorm(hcross(fwd, hv3(P.up[0], P.up[1], P.up[2])));
        rc.eye = eye;
        rc.fwd = fwd;
        rc.right = right;
        rc.up = hcross(right, fwd);
        rc.tan_half = std::tan(P.fov_deg * 3.14159265358979323846f / 180.0f / 2.0f);
        const float aspect = (float)P.width / (float)P.height;
        rc.sx0 = aspect > 1.0f ? -aspect : -1.0f;
        rc.sx1 = -rc.sx0;
        rc.sy0 = aspect > 1.0f ? -1.0f : -1.0f / aspect;
        rc.sy1 = -rc.sy0;
        rc.width = P.width;
        rc.height = P.height;
        rc.spp = P.spp;
        rc.max_depth = P.max_depth;
        rc.rr_min = P.rr_min_bounce;
        rc.mis_corrected = P.mis_corrected;
        rc.first_sample = P.first_sample;
        rc.filter_radius = P.filter_radius;
        rc.filter_sigma = P.filter_sigma;
        // ZSobolSampler.init (ZSobolSampler.swift:114-122)
        const int64_t sampler_spp = P.sampler_spp > 0 ? P.sampler_spp : P.spp;
        rc.zs.seed = (uint64_t)P.seed;
        rc.zs.log2spp = __builtin_ctzll((uint64_t)sampler_spp);
        int64_t res = std::max(P.width, P.height);
        res -= 1;
        res |= res >> 1;
        res |= res >> 2;
        res |= res >> 4;
        res |= res >> 8;
        res |= res >> 16;
        res += 1;
        rc.zs.n_base4_digits = __builtin_ctzll((uint64_t)res) + (rc.zs.log2spp + 1) / 2;
        gzg_status st = device_sobol(r->device, &rc.zs.matrices);
        if (st != GZG_OK) return st;

        Wave &w = r->w;
        w.total_paths = (uint64_t)P.width * P.height * P.spp;
        const uint64_t cap = P.wave_paths > 0 ? (uint64_t)P.wave_paths : (uint64_t)(1u << 21);
        w.capacity = (uint32_t)std::min<uint64_t>(cap, w.total_paths);
        const size_t C = w.capacity;
        if ((st = r->alloc(&w.zs_morton, C)) || (st = r->alloc(&w.zs_dim, C)) || (st = r->alloc(&w.thr, C)) ||
            (st = r->alloc(&w.L, C)) || (st = r->alloc(&w.pixel, C)) || (st = r->alloc(&w.weight, C)) ||
            (st = r->alloc(&w.q_ray[0], 2 * C)) || (st = r->alloc(&w.q_ray[1], 2 * C)) ||
            (st = r->alloc(&w.q_id[0], C)) || (st = r->alloc(&w.q_id[1], C)) || (st = r->alloc(&w.hits, C)) ||
            (st = r->alloc(&w.sh_ray, 2 * C)) || (st = r->alloc(&w.sh_id, C)) || (st = r->alloc(&w.sh_contrib, C)) ||
            (st = r->alloc(&w.sh_occ, C)) || (st = r->alloc(&w.pr_ray, 2 * C)) || (st = r->alloc(&w.pr_id, C)) ||
            (st = r->alloc(&w.pr_contrib, C)) || (st = r->alloc(&w.pr_hits, C)) ||
            (st = r->alloc(&w.counts, kCountWords)) || (st = r->alloc(&w.stats, kStatWords)))
                return st;
        st = cuda_err(cudaMemset(w.counts, 0, kCountWords * 4), "renderer counters");
        if (st) return st;
        st = cuda_err(cudaMemset(w.stats, 0, kStatWords * 8), "renderer statistics");
        if (st) return st;
        *out = r.release();
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
                if (kinds[k] < 1 || kinds[k] > 3) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_zsobol_fill_device: kind not 1, 2 or 3");
                per += kinds[k];
        }
        if (n == 0 || nkinds == 0) return clear_error();
        int dev = 0;
        cudaGetDevice(&dev);
        ZSobolConfig c{};
        gzg_status st = device_sobol(dev, &c.matrices);
        if (st) return st;
        c.seed = (uint64_t)seed;
        c.log2spp = __builtin_ctzll((uint64_t)samples_per_pixel);
        int64_t res = std::max(res_x, res_y);
        res -= 1;
        res |= res >> 1;
        res |= res >> 2;
        res |= res >> 4;
        res |= res >> 8;
        res |= res >> 16;
        res += 1;
        c.n_base4_digits = __builtin_ctzll((uint64_t)res) + (c.log2spp + 1) / 2;
        KindList kl{};
        for (int k = 0; k < nkinds; ++k) kl.k[k] = kinds[k];
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        k_zsobol_fill<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(c, px, py, index, n, kl, nkinds, per, out);
        st = cuda_err(cudaGetLastError(), "zsobol launch");
        if (!st) clear_error();
        return st;
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
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        gzg_status status = GZG_OK;
        const uint64_t waves = (r->w.total_paths + r->w.capacity - 1) / r->w.capacity;
        k_set_wave_base<<<1, 1, 0, st>>>(r->w, 0ull);
        if (r->params.use_graph) {
                const bool same_films =
                    r->graph && r->graph_film[0] == film_rgb && r->graph_film[1] == film_sq && r->graph_film[2] == film_w;
                if (!same_films) {
                        if (r->graph) cudaGraphExecDestroy(r->graph);
                        if (r->graph_def) cudaGraphDestroy(r->graph_def);
                        r->graph = nullptr;
                        r->graph_def = nullptr;
                        cudaStream_t cap;
                        status = cuda_err(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "graph stream");
                        if (!status) {
                                status = cuda_err(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "graph capture");
                                if (!status) {
                                        cudaError_t e = r->enqueue_wave(film_rgb, film_sq, film_w, cap);
                                        cudaError_t e2 = cudaStreamEndCapture(cap, &r->graph_def);
                                        status = cuda_err(e != cudaSuccess ? e : e2, "graph capture of a wave");
                                        if (!status)
                                                status = cuda_err(cudaGraphInstantiate(&r->graph, r->graph_def, 0),
                                                                  "graph instantiate");
                                }
                                cudaStreamDestroy(cap);
                        }
                        if (!status) {
                                r->graph_film[0] = film_rgb;
                                r->graph_film[1] = film_sq;
                                r->graph_film[2] = film_w;
                        }
                }
                for (uint64_t k = 0; k < waves && !status; ++k)
                        status = cuda_err(cudaGraphLaunch(r->graph, st), "graph launch");
        } else {
                for (uint64_t k = 0; k < waves && !status; ++k)
                        status = cuda_err(r->enqueue_wave(film_rgb, film_sq, film_w, st), "wave launch");
        }
        if (prev != r->device) cudaSetDevice(prev);
        if (!status) clear_error();
        return status;
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

GZG_API gzg_status gzg_render_image(gzg_scene *scene, const gzg_render_params *params, float *film_rgb, float *film_sq,
                                    float *film_w, gzg_render_stats *stats) {
        if (!scene || !params || !film_rgb || !film_w)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_render_image: null argument");
        gzg_renderer *r = nullptr;
        gzg_status st = gzg_renderer_create(scene, params, &r);
        if (st) return st;
        std::unique_ptr<gzg_renderer> hold(r);
        const size_t pix = (size_t)params->width * params->height;
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
                if ((st = gzg_renderer_render(r, d_rgb, d_sq, d_w, nullptr))) break;
                if ((st = cuda_err(cudaDeviceSynchronize(), "render"))) break;
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
        if (!st) clear_error();
        return st;
}

}  // extern "C"
