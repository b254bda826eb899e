// integrator.cpp - CPU restatement of Gonzales' MIS path integrator (test
// infrastructure: checker and CPU baseline).  Compiled with -ffp-contract=off.
//
// Restated from (paths relative to Sources/libgonzales):
//   bounce loop / shade       Integrator/VolumePathIntegrator.swift:325-463
//   MIS, light + BSDF sample  Integrator/VolumePathIntegrator.swift:67-266
//   Russian roulette          Integrator/VolumePathIntegrator.swift:269-283
//   power heuristic           Sampler/Sampling.swift:27-30
//   concentric disk / cosine  Sampler/Sampling.swift:3-25
//   light choice              Light/PowerLightSampler.swift:1-48
//   area light                Light/AreaLight.swift:13-49
//   triangle sample / area    Shape/Triangle.swift:517-544; Core/Sampleable.swift:33-68
//   hit interaction / frame   Shape/Triangle.swift:363-474; Geometry/Geometry.swift:64-77;
//                             Reflection/BsdfFrame.swift:13-21; Core/ShadingFrame.swift
//   diffuse BSDF              Bsdf/DiffuseBsdf.swift; Reflection/Bsdf.swift:20-52;
//                             Reflection/FramedBsdf.swift:16-83; Reflection/BsdfSample.swift:13-15
//   spawn / offsets           Core/Interaction.swift:15-54; Utility/Utility.swift:4
//   camera sample, weight     Core/Tile.swift:27-59; Sampler/Sampler.swift:69-82
//   Gaussian filter           Filter/GaussianFilter.swift:8-130
//   film sums                 Core/Film.swift:107-119; Core/Pixel.swift
//
// Decisions where the reference has no executing code (its MIS loop has no
// callers): every random dimension comes from the path's Z-Sobol sampler, in
// the order the Swift code draws them (camera 2D + lens 2D, then per bounce:
// light choice 1D, light point 2D, MIS BSDF sample 3D, continuation 3D,
// roulette 1D when it applies).  mis_corrected = 0 keeps the reference's
// arithmetic as written: the BSDF strategy's light density is queried with
// tHit = 0 (Core/Sampleable.swift:55-58), which rejects every hit, so that
// strategy's weight is 0; mis_corrected = 1 queries with tHit = infinity and
// evaluates the probe's emission toward the surface.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "oracle.h"

namespace {

const float kPi = 3.14159265358979323846f;
const float kInfF = std::numeric_limits<float>::infinity();

struct V3 {
        float x, y, z;
};
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 mul(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 mulv(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V3 neg(V3 a) { return v3(-a.x, -a.y, -a.z); }
inline float dot(V3 a, V3 b) {
        float s = a.x * b.x;
        s = s + a.y * b.y;
        return s + a.z * b.z;
}
inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline float length_sq(V3 a) { return dot(a, a); }
inline V3 normalize(V3 a) {
        float l = std::sqrt(dot(a, a));
        return v3(a.x / l, a.y / l, a.z / l);
}
inline float max_value(V3 a) { return std::max(a.x, std::max(a.y, a.z)); }
inline bool is_black(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }

// powerHeuristic (Sampler/Sampling.swift:27-30).
inline float power_heuristic(float f, float g) {
        if (f == 0.0f || g == 0.0f) return 0.0f;
        return (f * f) / (f * f + g * g);
}

// concentricSampleDisk / cosineSampleHemisphere (Sampler/Sampling.swift:3-25).
void concentric_disk(float u0, float u1, float *dx_out, float *dy_out) {
        float ox = 2.0f * u0 - 1.0f, oy = 2.0f * u1 - 1.0f;
        float dx = 0.0f, dy = 0.0f;
        if (!(ox == 0.0f && oy == 0.0f)) {
                float theta, r;
                if (std::fabs(ox) > std::fabs(oy)) {
                        r = ox;
                        theta = (kPi / 4.0f) * (oy / ox);
                } else {
                        r = oy;
                        theta = (kPi / 2.0f) - (kPi / 4.0f) * (ox / oy);
                }
                dx = r * std::cos(theta);
                dy = r * std::sin(theta);
        }
        *dx_out = dx;
        *dy_out = dy;
}

V3 cosine_hemisphere(float u0, float u1) {
        float dx, dy;
        concentric_disk(u0, u1, &dx, &dy);
        float z = std::sqrt(std::max(0.0f, 1.0f - dx * dx - dy * dy));
        return v3(dx, dy, z);
}

// makeCoordinateSystem (Geometry/Geometry.swift:64-77).
void coordinate_system(V3 v1, V3 *v2, V3 *v3o) {
        if (std::fabs(v1.x) > std::fabs(v1.y)) {
                float l = std::sqrt(v1.x * v1.x + v1.z * v1.z);
                *v2 = v3(-v1.z / l, 0.0f, v1.x / l);
        } else {
                float l = std::sqrt(v1.y * v1.y + v1.z * v1.z);
                *v2 = v3(0.0f, v1.z / l, -v1.y / l);
        }
        *v3o = cross(v1, *v2);
}

// Shading frame of a hit without UVs or vertex normals (Triangle.swift:395-452
// with degenerate UVs; BsdfFrame.swift:13-21; ShadingFrame(y:z:)).
struct Frame {
        V3 x, y, z;
        V3 to_local(V3 v) const { return v3(dot(v, x), dot(v, y), dot(v, z)); }
        V3 to_world(V3 v) const { return add(add(mul(x, v.x), mul(y, v.y)), mul(z, v.z)); }
};

// The interaction's dpdu (shading tangent) of Triangle.computeSurfaceInteraction.
bool shading_dpdu(V3 p0, V3 p1, V3 p2, V3 ns, V3 *dpdu_out) {
        V3 gn = cross(sub(p2, p0), sub(p1, p0));
        if (length_sq(gn) == 0.0f) return false;
        V3 dpdu, dpdv;
        coordinate_system(normalize(gn), &dpdu, &dpdv);
        V3 s = normalize(dpdu);
        V3 t = cross(s, ns);
        if (length_sq(t) > 0.0f) {
                t = normalize(t);
                s = cross(t, ns);
        } else {
                coordinate_system(ns, &s, &t);
        }
        *dpdu_out = s;
        return true;
}

// BsdfFrame from the interaction's dpdu and shading normal.
Frame frame_from(V3 dpdu, V3 ns) {
        Frame f;
        f.y = normalize(dpdu);
        f.z = ns;
        f.x = cross(f.y, f.z);
        return f;
}

bool make_frame(V3 p0, V3 p1, V3 p2, V3 ns, Frame *f) {
        V3 s;
        if (!shading_dpdu(p0, p1, p2, ns, &s)) return false;
        *f = frame_from(s, ns);
        return true;
}

// erfinv of GaussianFilter.swift:27-91.
float erfinv(float y) {
        const float center = 0.7f;
        const float a[4] = {0.886226899f, -1.645349621f, 0.914624893f, -0.140543331f};
        const float b[4] = {-2.118377725f, 1.442710462f, -0.329097515f, 0.012229801f};
        const float c[4] = {-1.970840454f, -1.624906493f, 3.429567803f, 1.641345311f};
        const float d[2] = {3.543889200f, 1.637067800f};
        const float ay = std::fabs(y);
        const float two_over_sqrt_pi = 2.0f / std::sqrt(kPi);
        float x;
        if (ay <= center) {
                float z = y * y;
                float num = a[3] * z + a[2];
                num = num * z + a[1];
                num = num * z + a[0];
                float den = b[3] * z + b[2];
                den = den * z + b[1];
                den = den * z + b[0];
                den = den * z + 1.0f;
                x = y * num / den;
        } else if (ay < 1.0f) {
                float z = std::sqrt(-std::log((1.0f - ay) / 2.0f));
                float num = c[3] * z + c[2];
                num = num * z + c[1];
                num = num * z + c[0];
                float den = d[1] * z + d[0];
                den = den * z + 1.0f;
                float sign = std::signbit(y) ? -1.0f : 1.0f;
                x = sign * num / den;
        } else if (ay == 1.0f) {
                return std::signbit(y) ? -kInfF : kInfF;
        } else {
                return std::numeric_limits<float>::quiet_NaN();
        }
        x -= (std::erf(x) - y) / (two_over_sqrt_pi * std::exp(-(x * x)));
        x -= (std::erf(x) - y) / (two_over_sqrt_pi * std::exp(-(x * x)));
        return x;
}

// GaussianFilter.sample's sample1D (GaussianFilter.swift:95-111).
void gaussian_sample_1d(float u, float radius, float sigma, float *x_out, float *density) {
        float norm = 0.5f * (1.0f + std::erf(radius / (sigma * std::sqrt(2.0f))));
        float us = (1.0f - norm) + u * (2.0f * norm - 1.0f);
        float x = sigma * std::sqrt(2.0f) * erfinv(2.0f * us - 1.0f);
        float pdf = std::exp(-x * x / (2.0f * sigma * sigma)) / (sigma * std::sqrt(2.0f * kPi));
        *density = pdf / (2.0f * norm - 1.0f);
        *x_out = std::max(-radius, std::min(radius, x));
}

// GaussianFilter.gaussian / evaluate (GaussianFilter.swift:15-25).
float gaussian(float x, float sigma) {
        return 1.0f / std::sqrt(2.0f * kPi * sigma * sigma) * std::exp(-(x * x) / (2.0f * sigma * sigma));
}

struct Light {
        V3 p0, p1, p2;
        V3 le;
        float area;
        float power;
        bool is_env = false;
};

struct Scene {
        const orc_node *nodes;
        const orc_prim_id *prims;
        const orc_mesh *meshes;
        const orc_material *materials;
        int64_t n_materials;
        std::vector<Light> lights;
        std::vector<float> cumulative;
        float total_power = 0.0f;
        const orc_render_params *p;
        const orc_textures *tex = nullptr;
        float escale = 1.0f;
        const orc_render_instances *inst = nullptr;
        const orc_env *env = nullptr;
        const float *mat_params = nullptr;  // 12 per material (orc_bsdf_params order from eta on)
};

// Emission times the scene's emission scale (1 without textures: exact).
V3 emitted(const Scene &sc, V3 e) { return v3(e.x * sc.escale, e.y * sc.escale, e.z * sc.escale); }

// Albedo of material m at p: its texture's nearest texel, else its constant.
V3 albedo_at(const Scene &sc, const orc_material *mats, int64_t m, V3 p) {
        const orc_material &mat = mats[m];
        if (sc.tex && !sc.inst && sc.tex->material_texture[m] >= 0) {
                const int t = sc.tex->material_texture[m];
                const int R = sc.tex->resolution;
                const float *mp = sc.tex->maps + 9 * t;
                const V3 d = sub(p, v3(mp[0], mp[1], mp[2]));
                const float u = dot(d, v3(mp[3], mp[4], mp[5])), v = dot(d, v3(mp[6], mp[7], mp[8]));
                // fmax/fmin: a NaN coordinate lands on texel 0
                const int ix = (int)std::fmin(std::fmax(u * (float)R, 0.0f), (float)(R - 1));
                const int iy = (int)std::fmin(std::fmax(v * (float)R, 0.0f), (float)(R - 1));
                const float *tx = sc.tex->texels + (((size_t)t * R + iy) * R + ix) * 3;
                return v3(tx[0], tx[1], tx[2]);
        }
        return v3(mat.albedo[0], mat.albedo[1], mat.albedo[2]);
}

bool prim_tri_of(const orc_prim_id *prims, const orc_mesh *meshes, int64_t k, V3 *p0, V3 *p1, V3 *p2) {
        const orc_prim_id &pr = prims[k];
        int64_t mesh, base;
        if (pr.type == 0) {
                mesh = pr.id1;
                base = pr.id2;
        } else if (pr.type >= 1 && pr.type <= 3 && pr.id2 != -1) {
                mesh = pr.id2 >> 32;
                base = (pr.id2 & 0xFFFFFFFFll) * 3;
        } else {
                return false;
        }
        const orc_mesh &m = meshes[mesh];
        const float *a = m.points + 4 * m.vertex_indices[base];
        const float *b = m.points + 4 * m.vertex_indices[base + 1];
        const float *c = m.points + 4 * m.vertex_indices[base + 2];
        *p0 = v3(a[0], a[1], a[2]);
        *p1 = v3(b[0], b[1], b[2]);
        *p2 = v3(c[0], c[1], c[2]);
        return true;
}

bool prim_tri(const Scene &sc, int64_t k, V3 *p0, V3 *p1, V3 *p2) {
        return prim_tri_of(sc.prims, sc.meshes, k, p0, p1, p2);
}

// The mesh and the vertex indices of prim k's triangle.
bool prim_vertices(const orc_prim_id *prims, const orc_mesh *meshes, int64_t k, const orc_mesh **m, int64_t v[3]) {
        const orc_prim_id &pr = prims[k];
        int64_t mesh, base;
        if (pr.type == 0) {
                mesh = pr.id1;
                base = pr.id2;
        } else if (pr.type >= 1 && pr.type <= 3 && pr.id2 != -1) {
                mesh = pr.id2 >> 32;
                base = (pr.id2 & 0xFFFFFFFFll) * 3;
        } else {
                return false;
        }
        *m = &meshes[mesh];
        for (int c = 0; c < 3; ++c) v[c] = (*m)->vertex_indices[base + c];
        return true;
}

// Triangle.computeSurfaceInteraction with vertex normals and / or UVs
// (Shape/Triangle.swift:386-452): dpdu from the UVs unless degenerate (then
// a coordinate system around the geometric normal), the shading normal
// interpolated from the vertex normals (normalised, (6, 6, 6) when it
// vanishes), the shading tangent made orthogonal to it.  Returns false for
// a degenerate triangle; ns = the interaction's (normalised) shading normal.
bool attr_shading(const orc_mesh &m, const int64_t v[3], V3 p0, V3 p1, V3 p2, float b0, float b1, float b2, V3 ng,
                  V3 *dpdu_out, V3 *ns_out) {
        const bool has_uv = m.uvs != nullptr, has_n = m.normals != nullptr;
        float uv[3][2] = {{0, 0}, {0, 0}, {0, 0}};
        if (has_uv)
                for (int c = 0; c < 3; ++c) {
                        uv[c][0] = m.uvs[2 * v[c]];
                        uv[c][1] = m.uvs[2 * v[c] + 1];
                }
        const V3 dp02 = sub(p0, p2), dp12 = sub(p1, p2);
        const float du02 = uv[0][0] - uv[2][0], dv02 = uv[0][1] - uv[2][1];
        const float du12 = uv[1][0] - uv[2][0], dv12 = uv[1][1] - uv[2][1];
        const float det = du02 * dv12 - dv02 * du12;
        const bool degenerate = std::fabs(det) < 1e-8f;
        V3 dpdu = v3(0, 1, 0), dpdv = v3(0, 1, 0);
        if (!degenerate) {
                const float inv = 1.0f / det;
                dpdu = mul(sub(mul(dp02, dv12), mul(dp12, dv02)), inv);
                dpdv = mul(sub(mul(dp02, -du12), mul(dp12, du02)), inv);
        }
        if (degenerate || length_sq(cross(dpdu, dpdv)) == 0.0f) {
                const V3 gn = cross(sub(p2, p0), sub(p1, p0));
                if (length_sq(gn) == 0.0f) return false;
                coordinate_system(normalize(gn), &dpdu, &dpdv);
        }
        V3 ns = ng;
        if (has_n) {
                V3 n[3];
                for (int c = 0; c < 3; ++c) n[c] = v3(m.normals[3 * v[c]], m.normals[3 * v[c] + 1], m.normals[3 * v[c] + 2]);
                ns = add(add(mul(n[0], b0), mul(n[1], b1)), mul(n[2], b2));
                ns = length_sq(ns) > 0.0f ? normalize(ns) : v3(6.0f, 6.0f, 6.0f);
        }
        V3 s = normalize(dpdu);
        V3 t = cross(s, ns);
        if (length_sq(t) > 0.0f) {
                t = normalize(t);
                s = cross(t, ns);
        } else {
                coordinate_system(ns, &s, &t);
        }
        *dpdu_out = s;
        *ns_out = normalize(ns);
        return true;
}

struct Hit {
        bool hit;
        int32_t prim, inst;
        float t, u, v;
};

Hit trace(const Scene &sc, V3 o, V3 d, float tmax) {
        orc_ray r{o.x, o.y, o.z, d.x, d.y, d.z};
        if (sc.inst) {
                Hit h;
                const orc_render_instances &I = *sc.inst;
                h.hit = orc_trace_instanced_one(I.tlas, I.leaf_instance, I.w2o, I.blas_of, I.blas, &r, tmax, &h.prim,
                                                &h.inst, &h.t, &h.u, &h.v) != 0;
                return h;
        }
        orc_isect is;
        int32_t idx;
        orc_trace_one(sc.nodes, sc.prims, sc.meshes, &r, tmax, &is, &idx);
        return Hit{is.hit != 0, idx, -1, is.t, is.u, is.v};
}

// Transform * Point / Vector / Normal (Geometry/Transform.swift:31-65) for a
// row-major 3x4 matrix m; the normal uses the inverse matrix's columns.
V3 xf_point(const float *m, V3 p) {
        return v3(((m[0] * p.x + m[1] * p.y) + m[2] * p.z) + m[3], ((m[4] * p.x + m[5] * p.y) + m[6] * p.z) + m[7],
                  ((m[8] * p.x + m[9] * p.y) + m[10] * p.z) + m[11]);
}
V3 xf_vector(const float *m, V3 v) {
        return v3((m[0] * v.x + m[1] * v.y) + m[2] * v.z, (m[4] * v.x + m[5] * v.y) + m[6] * v.z,
                  (m[8] * v.x + m[9] * v.y) + m[10] * v.z);
}
V3 xf_normal(const float *inv, V3 n) {
        return v3((inv[0] * n.x + inv[4] * n.y) + inv[8] * n.z, (inv[1] * n.x + inv[5] * n.y) + inv[9] * n.z,
                  (inv[2] * n.x + inv[6] * n.y) + inv[10] * n.z);
}

// The surface interaction of a hit (Triangle.computeSurfaceInteraction,
// Shape/Triangle.swift:363-474; for an instance in object space, then
// Transform * SurfaceInteraction, Core/Transform+SurfaceInteraction.swift:3-14).
struct Isect {
        V3 pos, ng, wo;
        V3 ns;  // shading normal (ng without vertex normals)
        Frame fr;
        bool frame_ok;
        const orc_prim_id *pr;
        const orc_material *mats;
        int blas;  // bottom-level scene of an instance hit, -1 for a flat scene
};

bool interaction(const Scene &sc, const Hit &h, V3 d, Isect *is) {
        V3 p0, p1, p2;
        const float b0 = (1.0f - h.u) - h.v;
        if (!sc.inst) {
                if (!prim_tri(sc, h.prim, &p0, &p1, &p2)) return false;
                is->pos = add(add(mul(p0, b0), mul(p1, h.u)), mul(p2, h.v));
                is->ng = normalize(cross(sub(p0, p2), sub(p1, p2)));
                is->wo = normalize(neg(d));
                is->ns = is->ng;
                const orc_mesh *m;
                int64_t vv[3];
                if (prim_vertices(sc.prims, sc.meshes, h.prim, &m, vv) && (m->normals || m->uvs)) {
                        V3 s;
                        is->frame_ok = attr_shading(*m, vv, p0, p1, p2, b0, h.u, h.v, is->ng, &s, &is->ns);
                        if (is->frame_ok) is->fr = frame_from(s, is->ns);
                } else {
                        is->frame_ok = make_frame(p0, p1, p2, is->ng, &is->fr);
                }
                is->pr = &sc.prims[h.prim];
                is->mats = sc.materials;
                is->blas = -1;
                return true;
        }
        const orc_render_instances &I = *sc.inst;
        const int32_t b = I.blas_of[h.inst];
        const orc_blas &B = I.blas[b];
        if (!prim_tri_of(B.prims, B.meshes, h.prim, &p0, &p1, &p2)) return false;
        const float *w2o = I.w2o + 12 * h.inst, *o2w = I.o2w + 12 * h.inst;
        const V3 pos_o = add(add(mul(p0, b0), mul(p1, h.u)), mul(p2, h.v));
        const V3 n_o = normalize(cross(sub(p0, p2), sub(p1, p2)));
        const V3 wo_o = normalize(neg(xf_vector(w2o, d)));
        V3 s_o = v3(0, 0, 0), ns_o = n_o;
        const orc_mesh *m;
        int64_t vv[3];
        const bool with_attr = prim_vertices(B.prims, B.meshes, h.prim, &m, vv) && (m->normals || m->uvs);
        if (with_attr)
                is->frame_ok = attr_shading(*m, vv, p0, p1, p2, b0, h.u, h.v, n_o, &s_o, &ns_o);
        else
                is->frame_ok = shading_dpdu(p0, p1, p2, n_o, &s_o);
        is->pos = xf_point(o2w, pos_o);
        is->ng = normalize(xf_normal(w2o, n_o));
        is->ns = with_attr ? normalize(xf_normal(w2o, ns_o)) : is->ng;
        is->wo = normalize(xf_vector(o2w, wo_o));
        if (is->frame_ok) is->fr = frame_from(xf_vector(o2w, s_o), is->ns);
        is->pr = &B.prims[h.prim];
        is->mats = I.blas_materials[b];
        is->blas = b;
        return true;
}

V3 env_radiance(const Scene &sc, V3 d) {
        const float dd[3] = {d.x, d.y, d.z};
        float c[3];
        orc_env_radiance(sc.env, dd, c);
        return v3(c[0], c[1], c[2]);
}

// offsetRayOrigin(point:normal:direction:) (Core/Interaction.swift:26-35).
V3 offset_origin(V3 p, V3 n, V3 dir) {
        V3 off = mul(n, 0.0001f);
        return dot(dir, n) > 0.0f ? add(p, off) : add(p, neg(off));
}

// ---- homogeneous medium in a box (Medium/Homogeneous.swift:5-23, phase
// function Medium/HenyeyGreenstein.swift:13-39).  The reference's integrator
// never samples it (VolumePathIntegrator.swift:394 hard-codes (white, nil));
// this is the branch as it evidently was meant to run: before a segment is
// shaded, the part of it inside the box is sampled for a scattering event;
// shadow rays and MIS probes through the box carry its transmittance.  The
// box boundary scatters nothing (an interface: Material/Interface.swift).

// Parametric overlap [t0, t1] of o + t d (t in [0, tmax]) with the medium
// box (slab test); false when empty.
bool medium_overlap(const orc_render_params &P, V3 o, V3 d, float tmax, float *t0, float *t1) {
        float lo = 0.0f, hi = tmax;
        const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
        for (int a = 0; a < 3; ++a) {
                if (dd[a] == 0.0f) {
                        if (oo[a] < P.medium_min[a] || oo[a] > P.medium_max[a]) return false;
                        continue;
                }
                const float inv = 1.0f / dd[a];
                float tn = (P.medium_min[a] - oo[a]) * inv, tf = (P.medium_max[a] - oo[a]) * inv;
                if (tn > tf) std::swap(tn, tf);
                lo = std::max(lo, tn);
                hi = std::min(hi, tf);
        }
        *t0 = lo;
        *t1 = hi;
        return lo < hi;
}

V3 sigma_t_of(const orc_render_params &P) {
        return v3(P.sigma_a[0] + P.sigma_s[0], P.sigma_a[1] + P.sigma_s[1], P.sigma_a[2] + P.sigma_s[2]);
}

// Transmittance exp(-sigma_t * length) along the part of [0, tmax] inside
// the box.
V3 medium_tr(const orc_render_params &P, V3 o, V3 d, float tmax) {
        float t0, t1;
        if (!P.has_medium || !medium_overlap(P, o, d, tmax, &t0, &t1)) return v3(1, 1, 1);
        const V3 st = sigma_t_of(P);
        const float len = (t1 - t0) * std::sqrt(dot(d, d));
        return v3(std::exp(-st.x * len), std::exp(-st.y * len), std::exp(-st.z * len));
}

// Homogeneous.sample on the segment [0, tmax] of the ray, restricted to its
// part inside the box, with the two uniform numbers uc (channel) and ud
// (distance).  Returns true with the scattering parameter t when the medium
// is sampled; `weight` is the throughput factor: transmittance x sigma_s /
// density at a scattering event and transmittance / density otherwise.
// Homogeneous.swift:19 writes sigma_t (`transmission`) where the PBRT
// sampler it restates has sigma_s; with sigma_t a purely absorbing medium
// would still scatter, so the scattering coefficient is used here.
bool medium_sample(const orc_render_params &P, V3 o, V3 d, float tmax, float uc, float ud, float *t, V3 *weight) {
        float t0, t1;
        *weight = v3(1, 1, 1);
        if (!medium_overlap(P, o, d, tmax, &t0, &t1)) return false;
        const V3 st = sigma_t_of(P);
        const float stc[3] = {st.x, st.y, st.z};
        const int channel = std::min((int)(uc * 3.0f), 2);
        const float distance = -std::log(1.0f - ud) / stc[channel];
        const float len = std::sqrt(dot(d, d));
        const float seg = t1 - t0;
        const float param = std::min(distance / len, seg);
        const bool sampled = param < seg;
        const V3 tr = v3(std::exp(-st.x * param * len), std::exp(-st.y * param * len), std::exp(-st.z * param * len));
        const V3 density = sampled ? mulv(st, tr) : tr;
        const float pdf = (density.x + density.y + density.z) / 3.0f;
        const V3 ss = v3(P.sigma_s[0], P.sigma_s[1], P.sigma_s[2]);
        *weight = sampled ? mul(mulv(tr, ss), 1.0f / pdf) : mul(tr, 1.0f / pdf);
        *t = t0 + param;
        return sampled;
}

// HenyeyGreenstein.phase (HenyeyGreenstein.swift:13-16).
float hg_phase(float cos_theta, float g) {
        const float denom = 1.0f + g * g + 2.0f * g * cos_theta;
        return (1.0f / (4.0f * kPi)) * (1.0f - g * g) / (denom * std::sqrt(denom));
}

// HenyeyGreenstein.samplePhase (HenyeyGreenstein.swift:18-36): the incident
// direction in the frame (makeCoordinateSystem(outgoing), outgoing) and the
// phase value, which is also its density.
V3 hg_sample(V3 wo, float g, float u0, float u1, float *value) {
        float cos_theta;
        if (std::fabs(g) < 1e-3f) {
                cos_theta = 1.0f - 2.0f * u0;
        } else {
                const float sqr = (1.0f - g * g) / (1.0f + g - 2.0f * g * u0);
                cos_theta = -(1.0f + g * g - sqr * sqr) / (2.0f * g);
        }
        const float sin_theta = std::sqrt(std::max(0.0f, 1.0f - cos_theta * cos_theta));
        const float phi = 2.0f * kPi * u1;
        V3 v1, v2;
        coordinate_system(wo, &v1, &v2);
        *value = hg_phase(cos_theta, g);
        return add(add(mul(v1, sin_theta * std::cos(phi)), mul(v2, sin_theta * std::sin(phi))), mul(wo, cos_theta));
}

// PowerLightSampler.chooseLight with the lowerBound search of
// PowerLightSampler.swift:4-18.
int choose_light(const Scene &sc, float u, float *pdf) {
        const float key = u * sc.total_power;
        int lo = 0, hi = (int)sc.cumulative.size();
        while (lo < hi) {
                int mid = lo + (hi - lo) / 2;
                if (sc.cumulative[mid] == key) {
                        lo = mid;
                        break;
                } else if (sc.cumulative[mid] < key) {
                        lo = mid + 1;
                } else {
                        hi = mid;
                }
        }
        if (lo >= (int)sc.lights.size()) lo = (int)sc.lights.size() - 1;
        *pdf = sc.lights[lo].power / sc.total_power;
        return lo;
}

// Watertight triangle intersection used by Triangle.intersect for the
// corrected MIS light density.
bool hit_light(const Light &l, V3 o, V3 d, float *t) {
        float th = kInfF, b0, b1, b2;
        const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
        const float a[3] = {l.p0.x, l.p0.y, l.p0.z}, b[3] = {l.p1.x, l.p1.y, l.p1.z}, c[3] = {l.p2.x, l.p2.y, l.p2.z};
        if (!orc_intersect_triangle_watertight(oo, dd, a, b, c, &th, &b0, &b1, &b2)) return false;
        *t = th;
        return true;
}

struct PathResult {
        V3 L;
        V3 albedo{0.0f, 0.0f, 0.0f}, normal{0.0f, 0.0f, 0.0f};  // first hit's BSDF albedo and normal (AOVs)
        uint64_t ext = 0, shadow = 0, probe = 0;
};

// The surface step for the non-diffuse materials (dielectric, coated
// diffuse): surfaceEstimate (VolumePathIntegrator.swift:325-371) through the
// FramedBsdf wrappers (Reflection/FramedBsdf.swift:16-83): light sample with
// MIS, BSDF sample with MIS, continuation.  Updates L, thr, the next ray and
// the specular flag; false ends the path.
bool shade_generic(const Scene &sc, orc_zsobol *smp, const orc_bsdf_params &bp, const Isect &is, int bounce, V3 &L,
                   V3 &thr, V3 &o, V3 &d, bool &specular, PathResult &res) {
        const orc_render_params &P = *sc.p;
        const V3 pos = is.pos, ng = is.ng, wo = is.wo;
        const Frame &fr = is.fr;
        const V3 wo_l = fr.to_local(wo);
        auto f_local = [&](V3 a, V3 b) {
                const float wa[3] = {a.x, a.y, a.z}, wb[3] = {b.x, b.y, b.z};
                float f[3], pdf;
                orc_bsdf_eval(&bp, wa, wb, f, &pdf);
                return v3(f[0], f[1], f[2]);
        };
        auto pdf_local = [&](V3 a, V3 b) {
                const float wa[3] = {a.x, a.y, a.z}, wb[3] = {b.x, b.y, b.z};
                float f[3], pdf;
                orc_bsdf_eval(&bp, wa, wb, f, &pdf);
                return pdf;
        };
        auto sample_local = [&](const float u[3], V3 &f, V3 &wi, float &pdf) {
                const float wa[3] = {wo_l.x, wo_l.y, wo_l.z};
                float fo[3], wio[3];
                orc_bsdf_sample(&bp, wa, u, fo, wio, &pdf);
                f = v3(fo[0], fo[1], fo[2]);
                wi = v3(wio[0], wio[1], wio[2]);
        };
        // evaluateDistributionFunction: reflection only (no BSDF here is
        // transmissive in world space), times |cos| with the shading normal
        auto f_world = [&](V3 wi) {
                const bool reflect = dot(wi, ng) * dot(wo, ng) > 0.0f;
                return reflect ? f_local(wo_l, fr.to_local(wi)) : v3(0, 0, 0);
        };

        float choose_pdf;
        const int li = choose_light(sc, orc_zsobol_get1d(smp), &choose_pdf);
        const Light &lt = sc.lights[li];
        float u2[2];
        orc_zsobol_get2d(smp, u2);
        V3 light_est = v3(0, 0, 0), light_dir = v3(0, 0, 0);
        float light_pdf = 0.0f;
        if (lt.is_env) {
                float dir[3], rgb[3];
                const float pdf = orc_env_sample(sc.env, u2[0], u2[1], dir, rgb);
                const V3 dv = v3(dir[0], dir[1], dir[2]), rad = v3(rgb[0], rgb[1], rgb[2]);
                if (!is_black(rad) && !std::isinf(pdf)) {
                        const V3 target = add(pos, mul(dv, 100.0f));
                        const V3 so = add(pos, mul(sub(target, pos), 0.0001f));
                        Hit sh = trace(sc, so, sub(target, so), 1.0f - 0.00001f);
                        ++res.shadow;
                        if (!sh.hit) {
                                light_est = mulv(mulv(mul(f_world(dv), std::fabs(dot(dv, is.ns))), rad),
                                                 medium_tr(P, so, sub(target, so), 1.0f - 0.00001f));
                                light_dir = dv;
                                light_pdf = pdf;
                        }
                }
        } else {
                const float su0 = std::sqrt(u2[0]);
                const float lb0 = 1.0f - su0, lb1 = u2[1] * su0;
                const V3 lp = add(add(mul(lt.p0, lb0), mul(lt.p1, lb1)), mul(lt.p2, (1.0f - lb0) - lb1));
                const V3 ln = normalize(cross(sub(lt.p1, lt.p0), sub(lt.p2, lt.p0)));
                const V3 inc = normalize(sub(lp, pos));
                const V3 dl = sub(pos, lp);
                const float pdf = (1.0f / lt.area) * (dot(dl, dl) / std::fabs(dot(ln, neg(inc))));
                if ((P.two_sided_emission || dot(ln, neg(inc)) > 0.0f) && !std::isinf(pdf)) {
                        const V3 so = add(pos, mul(sub(lp, pos), 0.0001f));
                        Hit sh = trace(sc, so, sub(lp, so), 1.0f - 0.00001f);
                        ++res.shadow;
                        if (!sh.hit) {
                                light_est = mulv(mulv(mul(f_world(inc), std::fabs(dot(inc, is.ns))), emitted(sc, lt.le)),
                                                 medium_tr(P, so, sub(lp, so), 1.0f - 0.00001f));
                                light_dir = inc;
                                light_pdf = pdf;
                        }
                }
        }
        const float brdf_density = wo_l.z == 0.0f ? 0.0f : pdf_local(wo_l, fr.to_local(light_dir));
        const float light_w = power_heuristic(light_pdf, brdf_density);
        V3 contrib = light_pdf == 0.0f ? v3(0, 0, 0) : mul(mul(light_est, light_w), 1.0f / light_pdf);

        float u3[3];
        orc_zsobol_get3d(smp, u3);
        {
                V3 fs, wi_l;
                float pdf_b;
                sample_local(u3, fs, wi_l, pdf_b);
                const V3 wi = fr.to_world(wi_l);
                V3 est = mul(fs, std::fabs(dot(wi, is.ns)));
                if ((P.mis_corrected || lt.is_env) && !is_black(est) && pdf_b > 0.0f) {
                        const V3 po = offset_origin(pos, ng, wi);
                        Hit ph = trace(sc, po, wi, kInfF);
                        ++res.probe;
                        V3 radiance = v3(0, 0, 0);
                        Isect pi;
                        if (ph.hit) {
                                if (interaction(sc, ph, wi, &pi) && pi.pr->type == 3) {
                                        const orc_material &lm = pi.mats[pi.pr->material_index];
                                        if (P.two_sided_emission || dot(pi.ng, neg(wi)) > 0.0f)
                                                radiance = emitted(sc, v3(lm.emission[0], lm.emission[1], lm.emission[2]));
                                }
                        } else if (sc.env) {
                                radiance = env_radiance(sc, wi);
                        }
                        est = mulv(mulv(est, radiance), medium_tr(P, po, wi, ph.hit ? ph.t : kInfF));
                        float light_density = 0.0f;
                        if (lt.is_env) {
                                const float dd[3] = {wi.x, wi.y, wi.z};
                                light_density = orc_env_pdf(sc.env, dd);
                        } else {
                                float tl;
                                if (hit_light(lt, po, wi, &tl)) {
                                        const V3 hp = add(po, mul(wi, tl));
                                        const V3 dq = sub(pos, hp);
                                        const V3 lnn = normalize(cross(sub(lt.p0, lt.p2), sub(lt.p1, lt.p2)));
                                        const float dens = dot(dq, dq) / (std::fabs(dot(lnn, neg(wi))) * lt.area);
                                        light_density = std::isinf(dens) ? 0.0f : dens;
                                }
                        }
                        const float bw = power_heuristic(pdf_b, light_density);
                        contrib = add(contrib, mul(mul(est, bw), 1.0f / pdf_b));
                }
        }
        L = add(L, mulv(thr, mul(contrib, 1.0f / choose_pdf)));

        // continuation: bsdf.sampleWorldSpace + throughputWeight(normal:)
        orc_zsobol_get3d(smp, u3);
        V3 fs, wi_l;
        float pdf_c;
        sample_local(u3, fs, wi_l, pdf_c);
        if (pdf_c == 0.0f || std::isnan(pdf_c)) return false;
        specular = orc_bsdf_is_specular(&bp) != 0;
        const V3 wi = fr.to_world(wi_l);
        thr = mulv(thr, mul(fs, std::fabs(dot(wi, ng)) / pdf_c));
        o = offset_origin(pos, ng, wi);
        d = wi;
        const float mv = max_value(thr);
        if (mv < 1.0f && bounce >= P.rr_min_bounce) {
                const float q = std::max(0.0f, 1.0f - mv);
                if (orc_zsobol_get1d(smp) < q) return false;
                thr = mul(thr, 1.0f / (1.0f - q));
        }
        return true;
}

// A scattering event in the medium at p: mediumEstimate / sampleMedium
// (VolumePathIntegrator.swift:286-323) with the Henyey-Greenstein phase
// function as the distribution model (PhaseFunction.swift: value without a
// cosine, density = value): sampleOneLight with MIS (light choice 1D, light
// point 2D, phase sample 2D), then the phase sample (2D) that continues the
// path with its throughput unchanged (value / density = 1), then roulette.
// The new ray starts at p itself (a medium interaction has no normal to
// offset along).  false ends the path.
bool shade_medium(const Scene &sc, orc_zsobol *smp, V3 p, V3 wo, int bounce, V3 &L, V3 &thr, V3 &o, V3 &d,
                  PathResult &res) {
        const orc_render_params &P = *sc.p;
        const float g = P.medium_g;
        if (!sc.lights.empty()) {
                float choose_pdf;
                const int li = choose_light(sc, orc_zsobol_get1d(smp), &choose_pdf);
                const Light &lt = sc.lights[li];
                float u2[2];
                orc_zsobol_get2d(smp, u2);
                V3 light_est = v3(0, 0, 0), light_dir = v3(0, 0, 0);
                float light_pdf = 0.0f;
                if (lt.is_env) {
                        float dir[3], rgb[3];
                        const float pdf = orc_env_sample(sc.env, u2[0], u2[1], dir, rgb);
                        const V3 dv = v3(dir[0], dir[1], dir[2]), rad = v3(rgb[0], rgb[1], rgb[2]);
                        if (!is_black(rad) && !std::isinf(pdf)) {
                                const V3 target = add(p, mul(dv, 100.0f));
                                const V3 so = add(p, mul(sub(target, p), 0.0001f));
                                const V3 sd = sub(target, so);
                                Hit sh = trace(sc, so, sd, 1.0f - 0.00001f);
                                ++res.shadow;
                                if (!sh.hit) {
                                        light_est = mulv(mul(rad, hg_phase(dot(wo, dv), g)),
                                                         medium_tr(P, so, sd, 1.0f - 0.00001f));
                                        light_dir = dv;
                                        light_pdf = pdf;
                                }
                        }
                } else {
                        const float su0 = std::sqrt(u2[0]);
                        const float lb0 = 1.0f - su0, lb1 = u2[1] * su0;
                        const V3 lp = add(add(mul(lt.p0, lb0), mul(lt.p1, lb1)), mul(lt.p2, (1.0f - lb0) - lb1));
                        const V3 ln = normalize(cross(sub(lt.p1, lt.p0), sub(lt.p2, lt.p0)));
                        const V3 inc = normalize(sub(lp, p));
                        const V3 dl = sub(p, lp);
                        const float pdf = (1.0f / lt.area) * (dot(dl, dl) / std::fabs(dot(ln, neg(inc))));
                        if ((P.two_sided_emission || dot(ln, neg(inc)) > 0.0f) && !std::isinf(pdf)) {
                                const V3 so = add(p, mul(sub(lp, p), 0.0001f));
                                const V3 sd = sub(lp, so);
                                Hit sh = trace(sc, so, sd, 1.0f - 0.00001f);
                                ++res.shadow;
                                if (!sh.hit) {
                                        light_est = mulv(mul(emitted(sc, lt.le), hg_phase(dot(wo, inc), g)),
                                                         medium_tr(P, so, sd, 1.0f - 0.00001f));
                                        light_dir = inc;
                                        light_pdf = pdf;
                                }
                        }
                }
                const float phase_density = light_pdf == 0.0f ? 0.0f : hg_phase(dot(wo, light_dir), g);
                const float light_w = power_heuristic(light_pdf, phase_density);
                V3 contrib = light_pdf == 0.0f ? v3(0, 0, 0) : mul(light_est, light_w / light_pdf);
                float u[2];
                orc_zsobol_get2d(smp, u);
                if (P.mis_corrected || lt.is_env) {
                        float value;
                        const V3 wi = hg_sample(wo, g, u[0], u[1], &value);
                        if (value > 0.0f) {
                                Hit ph = trace(sc, p, wi, kInfF);
                                ++res.probe;
                                V3 radiance = v3(0, 0, 0);
                                Isect pi;
                                if (ph.hit) {
                                        if (interaction(sc, ph, wi, &pi) && pi.pr->type == 3) {
                                                const orc_material &lm = pi.mats[pi.pr->material_index];
                                                if (P.two_sided_emission || dot(pi.ng, neg(wi)) > 0.0f)
                                                        radiance = emitted(sc, v3(lm.emission[0], lm.emission[1],
                                                                                  lm.emission[2]));
                                        }
                                } else if (sc.env) {
                                        radiance = env_radiance(sc, wi);
                                }
                                radiance = mulv(radiance, medium_tr(P, p, wi, ph.hit ? ph.t : kInfF));
                                float light_density = 0.0f;
                                if (lt.is_env) {
                                        const float dd[3] = {wi.x, wi.y, wi.z};
                                        light_density = orc_env_pdf(sc.env, dd);
                                } else {
                                        float tl;
                                        if (hit_light(lt, p, wi, &tl)) {
                                                const V3 hp = add(p, mul(wi, tl));
                                                const V3 dq = sub(p, hp);
                                                const V3 lnn = normalize(cross(sub(lt.p0, lt.p2), sub(lt.p1, lt.p2)));
                                                const float dens = dot(dq, dq) / (std::fabs(dot(lnn, neg(wi))) * lt.area);
                                                light_density = std::isinf(dens) ? 0.0f : dens;
                                        }
                                }
                                const float bw = power_heuristic(value, light_density);
                                contrib = add(contrib, mul(radiance, bw));  // value / density = 1
                        }
                }
                L = add(L, mulv(thr, mul(contrib, 1.0f / choose_pdf)));
        }
        float u[2];
        orc_zsobol_get2d(smp, u);
        float value;
        d = hg_sample(wo, g, u[0], u[1], &value);
        o = p;
        const float mv = max_value(thr);
        if (mv < 1.0f && bounce >= P.rr_min_bounce) {
                const float q = std::max(0.0f, 1.0f - mv);
                if (orc_zsobol_get1d(smp) < q) return false;
                thr = mul(thr, 1.0f / (1.0f - q));
        }
        return true;
}

// One path: VolumePathIntegrator.bounces (:448-463) with shadeBounce (:373-430)
// and surfaceEstimate (:325-371).
PathResult trace_path(const Scene &sc, orc_zsobol *smp, V3 o, V3 d) {
        const orc_render_params &P = *sc.p;
        PathResult res;
        V3 L = v3(0, 0, 0), thr = v3(1, 1, 1);
        bool specular = false;  // state.specularBounce
        for (int bounce = 0; bounce <= P.max_depth; ++bounce) {
                Hit h = trace(sc, o, d, kInfF);
                ++res.ext;
                if (P.has_medium) {
                        // Homogeneous.sample on the segment before it is shaded (the
                        // branch of shadeBounce :394-408 as meant to run); its two
                        // numbers are drawn at every segment of a scene with a medium
                        const float uc = orc_zsobol_get1d(smp);
                        const float ud = orc_zsobol_get1d(smp);
                        float tm;
                        V3 wgt;
                        const bool scattered = medium_sample(P, o, d, h.hit ? h.t : kInfF, uc, ud, &tm, &wgt);
                        thr = mulv(thr, wgt);
                        if (scattered) {
                                if (is_black(thr) || bounce >= P.max_depth) break;
                                if (!shade_medium(sc, smp, add(o, mul(d, tm)), neg(d), bounce, L, thr, o, d, res)) break;
                                specular = false;
                                continue;
                        }
                }
                if (!h.hit) {
                        // shadeBounce on a miss (:375-387): environment light on
                        // camera rays (no specular bounces in these scenes)
                        if ((bounce == 0 || specular) && sc.env) L = add(L, mulv(thr, env_radiance(sc, d)));
                        break;
                }
                if (is_black(thr)) break;
                if (bounce >= P.max_depth) break;
                Isect is;
                if (!interaction(sc, h, d, &is)) break;
                const V3 pos = is.pos, ng = is.ng, wo = is.wo;
                const orc_prim_id &pr = *is.pr;
                const bool is_light = pr.type == 3;
                if ((bounce == 0 || specular) && is_light) {
                        const orc_material &lm = is.mats[pr.material_index];
                        if (P.two_sided_emission || dot(ng, wo) > 0.0f)
                                L = add(L, mulv(thr, emitted(sc, v3(lm.emission[0], lm.emission[1], lm.emission[2]))));
                }
                // Area lights have materialIndex 0 in their interaction
                // (Core/SurfaceInteraction.swift:20): the scene's first material.
                // The material: a dielectric or coated diffuse takes the general
                // BSDF step; diffuse keeps its closed forms below.
                {
                        const orc_material *mset = is_light ? (sc.inst ? sc.inst->blas_materials[0] : sc.materials) : is.mats;
                        const int64_t mi = is_light ? 0 : pr.material_index;
                        const float *mp = nullptr;
                        if (sc.inst) {
                                const int b = is_light ? 0 : is.blas;
                                if (sc.inst->blas_material_params && sc.inst->blas_material_params[b])
                                        mp = sc.inst->blas_material_params[b] + 12 * mi;
                        } else if (sc.mat_params) {
                                mp = sc.mat_params + 12 * mi;
                        }
                        const orc_material &mm = mset[mi];
                        if (mm.type >= 3 && mm.type <= 6 && mp) {
                                // mp: eta, roughness u, v, thickness, conductor eta[3],
                                // conductor roughness u, conductor k[3], conductor roughness v
                                const orc_bsdf_params bp{mm.type,
                                                         {mm.albedo[0], mm.albedo[1], mm.albedo[2]},
                                                         mp[0],
                                                         mp[1],
                                                         mp[2],
                                                         mp[3],
                                                         {mp[4], mp[5], mp[6]},
                                                         {mp[8], mp[9], mp[10]},
                                                         mp[7],
                                                         mp[11]};
                                if (bounce == 0) {
                                        // Bsdf.albedo(): the diffuse base's reflectance for a coated
                                        // diffuse; white for the dielectric and for both conductors
                                        // (MicrofacetReflection.albedo)
                                        res.albedo = mm.type == 4 ? v3(mm.albedo[0], mm.albedo[1], mm.albedo[2]) : v3(1, 1, 1);
                                        res.normal = ng;
                                }
                                if (!is.frame_ok || sc.lights.empty()) break;
                                if (!shade_generic(sc, smp, bp, is, bounce, L, thr, o, d, specular, res)) break;
                                continue;
                        }
                }
                specular = false;
                const V3 refl = is_light ? albedo_at(sc, sc.inst ? sc.inst->blas_materials[0] : sc.materials, 0, pos)
                                         : albedo_at(sc, is.mats, pr.material_index, pos);
                const V3 f_val = mul(refl, 1.0f / kPi);
                if (bounce == 0) {
                        // surfaceEstimate (:341-344): state.albedo, state.firstNormal
                        res.albedo = refl;
                        res.normal = ng;
                }
                if (!is.frame_ok) break;
                if (sc.lights.empty()) break;
                const Frame &fr = is.fr;
                const V3 wo_l = fr.to_local(wo);

                // ---- sampleOneLight -> estimateDirect -> sampleMultipleImportance
                float choose_pdf;
                const int li = choose_light(sc, orc_zsobol_get1d(smp), &choose_pdf);
                const Light &lt = sc.lights[li];
                float u2[2];
                orc_zsobol_get2d(smp, u2);
                V3 light_est = v3(0, 0, 0);
                V3 light_dir = v3(0, 0, 0);
                float light_pdf = 0.0f;
                if (lt.is_env) {
                        // InfiniteLight.sample (InfiniteLight.swift:38-64)
                        float dir[3], rgb[3];
                        const float pdf = orc_env_sample(sc.env, u2[0], u2[1], dir, rgb);
                        const V3 dv = v3(dir[0], dir[1], dir[2]), rad = v3(rgb[0], rgb[1], rgb[2]);
                        if (!is_black(rad) && !std::isinf(pdf)) {
                                const V3 target = add(pos, mul(dv, 100.0f));  // sceneDiameter
                                const V3 so = add(pos, mul(sub(target, pos), 0.0001f));
                                const V3 sd = sub(target, so);
                                Hit sh = trace(sc, so, sd, 1.0f - 0.00001f);
                                ++res.shadow;
                                if (!sh.hit) {
                                        const bool reflect = dot(dv, ng) * dot(wo, ng) > 0.0f;
                                        const V3 f = reflect ? f_val : v3(0, 0, 0);
                                        light_est = mulv(mulv(mul(f, std::fabs(dot(dv, is.ns))), rad),
                                                         medium_tr(P, so, sd, 1.0f - 0.00001f));
                                        light_dir = dv;
                                        light_pdf = pdf;
                                }
                        }
                } else {
                        const float su0 = std::sqrt(u2[0]);
                        const float lb0 = 1.0f - su0, lb1 = u2[1] * su0;
                        const V3 lp = add(add(mul(lt.p0, lb0), mul(lt.p1, lb1)), mul(lt.p2, (1.0f - lb0) - lb1));
                        const V3 ln = normalize(cross(sub(lt.p1, lt.p0), sub(lt.p2, lt.p0)));
                        float pdf = 1.0f / lt.area;
                        const V3 inc = normalize(sub(lp, pos));
                        const V3 dl = sub(pos, lp);
                        const float d2 = dot(dl, dl);
                        const float angle = std::fabs(dot(ln, neg(inc)));
                        pdf = pdf * (d2 / angle);
                        const V3 dir = inc;
                        const bool lit = P.two_sided_emission || dot(ln, neg(dir)) > 0.0f;
                        if (lit && !std::isinf(pdf)) {
                                // Visibility.occluded: spawnRay(from:target:) (Interaction.swift:15-24)
                                const V3 so = add(pos, mul(sub(lp, pos), 0.0001f));
                                const V3 sd = sub(lp, so);
                                Hit sh = trace(sc, so, sd, 1.0f - 0.00001f);
                                ++res.shadow;
                                if (!sh.hit) {
                                        const bool reflect = dot(dir, ng) * dot(wo, ng) > 0.0f;
                                        const V3 f = reflect ? f_val : v3(0, 0, 0);
                                        const V3 scatter = mul(f, std::fabs(dot(dir, is.ns)));
                                        light_est = mulv(mulv(scatter, emitted(sc, lt.le)), medium_tr(P, so, sd, 1.0f - 0.00001f));
                                        light_dir = dir;
                                        light_pdf = pdf;
                                }
                        }
                }
                // brdfDensity: probabilityDensityWorldSpace (FramedBsdf.swift:36-43)
                float brdf_density = 0.0f;
                {
                        const V3 wi_l = fr.to_local(light_dir);
                        if (wo_l.z != 0.0f && wo_l.z * wi_l.z > 0.0f) brdf_density = std::fabs(wi_l.z) / kPi;
                }
                const float light_w = power_heuristic(light_pdf, brdf_density);
                V3 contrib = light_pdf == 0.0f ? v3(0, 0, 0) : mul(mul(light_est, light_w), 1.0f / light_pdf);

                // sampleDistributionFunction (VolumePathIntegrator.swift:91-133).
                // The light density of the chosen light along the BSDF sample:
                // an environment light answers from its map; an area light, as
                // written, is queried with tHit = 0 and answers 0 (weight 0).
                float u3[3];
                orc_zsobol_get3d(smp, u3);
                {
                        V3 wi_l = cosine_hemisphere(u3[0], u3[1]);
                        if (wo_l.z < 0.0f) wi_l.z = -wi_l.z;
                        const float pdf_b = (wo_l.z * wi_l.z > 0.0f) ? std::fabs(wi_l.z) / kPi : 0.0f;
                        const V3 wi = fr.to_world(wi_l);
                        V3 est = mul(f_val, std::fabs(dot(wi, is.ns)));
                        if ((P.mis_corrected || lt.is_env) && !is_black(est) && pdf_b > 0.0f) {
                                const V3 po = offset_origin(pos, ng, wi);
                                Hit ph = trace(sc, po, wi, kInfF);
                                ++res.probe;
                                V3 radiance = v3(0, 0, 0);
                                Isect pi;
                                if (ph.hit) {
                                        if (interaction(sc, ph, wi, &pi) && pi.pr->type == 3) {
                                                const orc_material &lm = pi.mats[pi.pr->material_index];
                                                if (P.two_sided_emission || dot(pi.ng, neg(wi)) > 0.0f)
                                                        radiance = emitted(sc, v3(lm.emission[0], lm.emission[1],
                                                                                  lm.emission[2]));
                                        }
                                } else if (sc.env) {
                                        radiance = env_radiance(sc, wi);
                                }
                                est = mulv(mulv(est, radiance), medium_tr(P, po, wi, ph.hit ? ph.t : kInfF));
                                float light_density = 0.0f;
                                if (lt.is_env) {
                                        const float dd[3] = {wi.x, wi.y, wi.z};
                                        light_density = orc_env_pdf(sc.env, dd);
                                } else {
                                        float tl;
                                        if (hit_light(lt, po, wi, &tl)) {
                                                const V3 hp = add(po, mul(wi, tl));
                                                const V3 dq = sub(pos, hp);
                                                const float dd2 = dot(dq, dq);
                                                const V3 lnn = normalize(cross(sub(lt.p0, lt.p2), sub(lt.p1, lt.p2)));
                                                const float ang = std::fabs(dot(lnn, neg(wi)));
                                                const float dens = dd2 / (ang * lt.area);
                                                light_density = std::isinf(dens) ? 0.0f : dens;
                                        }
                                }
                                const float bw = power_heuristic(pdf_b, light_density);
                                contrib = add(contrib, mul(mul(est, bw), 1.0f / pdf_b));
                        }
                }
                L = add(L, mulv(thr, mul(contrib, 1.0f / choose_pdf)));

                // continuation: bsdf.sampleWorldSpace(outgoing:uSample: get3D)
                orc_zsobol_get3d(smp, u3);
                V3 wi_l = cosine_hemisphere(u3[0], u3[1]);
                if (wo_l.z < 0.0f) wi_l.z = -wi_l.z;
                const float pdf_c = (wo_l.z * wi_l.z > 0.0f) ? std::fabs(wi_l.z) / kPi : 0.0f;
                if (pdf_c == 0.0f || std::isnan(pdf_c)) break;
                const V3 wi = fr.to_world(wi_l);
                thr = mulv(thr, mul(f_val, std::fabs(dot(wi, ng)) / pdf_c));
                o = offset_origin(pos, ng, wi);
                d = wi;
                // stopWithRussianRoulette (:269-283), roulette value from Z-Sobol
                const float mv = max_value(thr);
                if (mv < 1.0f && bounce >= P.rr_min_bounce) {
                        const float q = std::max(0.0f, 1.0f - mv);
                        if (orc_zsobol_get1d(smp) < q) break;
                        thr = mul(thr, 1.0f / (1.0f - q));
                }
        }
        res.L = L;
        return res;
}

// The camera of a frame and one path's camera ray: Tile.render phase 1
// (Core/Tile.swift:27-59) with Sampler.getCameraSample (Sampler/Sampler.swift:
// 69-82), GaussianFilter.sample and PerspectiveCamera.generateRay; the basis
// is right-handed (+x right, +y up in the image).
struct Camera {
        const orc_render_params &P;
        V3 eye, fwd, right, upv;
        float tan_half, sx0, sx1, sy0, sy1;
        int sampler_spp;
        explicit Camera(const orc_render_params &p) : P(p) {
                eye = v3(P.eye[0], P.eye[1], P.eye[2]);
                fwd = normalize(sub(v3(P.target[0], P.target[1], P.target[2]), eye));
                right = normalize(cross(fwd, v3(P.up[0], P.up[1], P.up[2])));
                upv = cross(right, fwd);
                tan_half = std::tan(P.fov_deg * kPi / 180.0f / 2.0f);
                const float aspect = (float)P.width / (float)P.height;
                sx0 = aspect > 1.0f ? -aspect : -1.0f;
                sx1 = -sx0;
                sy0 = aspect > 1.0f ? -1.0f : -1.0f / aspect;
                sy1 = -sy0;
                sampler_spp = P.sampler_spp > 0 ? P.sampler_spp : P.spp;
        }
        // Starts *smp at sample `sample` of pixel (px, py) and draws the
        // camera and lens dimensions; w = filter value / filter pdf
        // (Tile.swift:36-40).
        void ray(int px, int py, int sample, orc_zsobol *smp, V3 *org_out, V3 *dir_out, float *w_out) const {
                const int W = P.width, H = P.height;
                orc_zsobol_init(smp, sampler_spp, W, H, P.seed);
                orc_zsobol_start_pixel_sample(smp, px, py, sample, 0);
                float u2[2];
                orc_zsobol_get2d(smp, u2);
                float dx, dy, denx, deny;
                gaussian_sample_1d(u2[0], P.filter_radius, P.filter_sigma, &dx, &denx);
                gaussian_sample_1d(u2[1], P.filter_radius, P.filter_sigma, &dy, &deny);
                const float fx = (float)px + 0.5f + dx, fy = (float)py + 0.5f + dy;
                float lens[2];
                orc_zsobol_get2d(smp, lens);
                const float scx = sx0 + fx / (float)W * (sx1 - sx0);
                const float scy = sy1 - fy / (float)H * (sy1 - sy0);
                V3 dcam = normalize(v3(scx * tan_half, scy * tan_half, 1.0f));
                V3 org = eye;
                if (P.lens_radius > 0.0f) {
                        // PerspectiveCamera.depthOfField (Camera/PerspectiveCamera.swift:25-35):
                        // origin on the lens, direction from the pinhole origin to the
                        // focal point (the pinhole direction, renormalised)
                        float lx, ly;
                        concentric_disk(lens[0], lens[1], &lx, &ly);
                        lx = P.lens_radius * lx;
                        ly = P.lens_radius * ly;
                        const float ft = P.focal_distance / dcam.z;
                        dcam = normalize(mul(dcam, ft));
                        org = add(add(eye, mul(right, lx)), mul(upv, ly));
                }
                *dir_out = add(add(mul(right, dcam.x), mul(upv, dcam.y)), mul(fwd, dcam.z));
                *org_out = org;
                const float ddx = fx - ((float)px + 0.5f), ddy = fy - ((float)py + 0.5f);
                const float fv = std::max(0.0f, gaussian(ddx, P.filter_sigma)) *
                                 std::max(0.0f, gaussian(ddy, P.filter_sigma));
                *w_out = fv / (denx * deny);
        }
};

}  // namespace

extern "C" void orc_render_ex(const orc_node *nodes, const orc_prim_id *prims, const orc_mesh *meshes,
                              const orc_material *materials, int64_t n_materials, int64_t n_prims,
                              const orc_render_instances *instances, const orc_env *env, const float *material_params,
                              const orc_render_params *params, const orc_textures *textures, float *sum_rgb,
                              float *sum_sq, float *sum_w, float *sum_albedo, float *sum_normal, uint64_t *counters,
                              int threads) {
        Scene sc;
        sc.inst = instances;
        sc.env = env;
        sc.mat_params = material_params;
        if (instances) n_prims = 0;  // instanced emitters are not lights (objects add none)
        sc.tex = textures;
        sc.escale = textures ? textures->emission_scale : 1.0f;
        sc.nodes = nodes;
        sc.prims = prims;
        sc.meshes = meshes;
        sc.materials = materials;
        sc.n_materials = n_materials;
        sc.p = params;
        // Lights: area-light prims in light-index order (SceneDescription.worldEnd
        // appends one AreaLight per triangle; PowerLightSampler.init).
        std::vector<std::pair<int64_t, int64_t>> order;
        for (int64_t k = 0; k < n_prims; ++k)
                if (prims[k].type == 3) order.push_back({prims[k].id1, k});
        std::sort(order.begin(), order.end());
        for (auto &e : order) {
                Light l;
                prim_tri(sc, e.second, &l.p0, &l.p1, &l.p2);
                const orc_material &m = materials[prims[e.second].material_index];
                l.le = v3(m.emission[0], m.emission[1], m.emission[2]);
                l.area = 0.5f * std::sqrt(length_sq(cross(sub(l.p1, l.p0), sub(l.p2, l.p0))));
                const float avg = (l.le.x + l.le.y + l.le.z) / 3.0f;
                l.power = avg * l.area * kPi;
                sc.lights.push_back(l);
        }
        if (env) {
                // the environment light after the area lights
                Light l{};
                l.is_env = true;
                l.power = orc_env_power(env);
                sc.lights.push_back(l);
        }
        float run = 0.0f;
        for (size_t i = 0; i < sc.lights.size(); ++i) {
                run = i == 0 ? sc.lights[0].power : run + sc.lights[i].power;
                sc.cumulative.push_back(run);
        }
        sc.total_power = 0.0f;
        for (const Light &l : sc.lights) sc.total_power = sc.total_power + l.power;

        const orc_render_params &P = *params;
        const float film_scale = (P.iso > 0.0f ? P.iso : 100.0f) / 100.0f;
        // the film window: the crop (Film.getSampleBounds) or the whole frame
        const bool cropped = P.crop[0] || P.crop[1] || P.crop[2] || P.crop[3];
        const int x0 = cropped ? P.crop[0] : 0, y0 = cropped ? P.crop[1] : 0;
        const int x1 = cropped ? P.crop[2] : P.width, y1 = cropped ? P.crop[3] : P.height;
        const int FW = x1 - x0;
        const Camera cam(P);
        if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
        std::atomic<int> next_row{y0};
        std::vector<uint64_t> cnt(4 * threads, 0);
        std::vector<std::thread> pool;
        for (int ti = 0; ti < threads; ++ti)
                pool.emplace_back([&, ti]() {
                        for (;;) {
                                const int py = next_row.fetch_add(1);
                                if (py >= y1) break;
                                for (int px = x0; px < x1; ++px) {
                                        float acc[3] = {0, 0, 0}, acc2[3] = {0, 0, 0}, accw = 0.0f;
                                        float acca[3] = {0, 0, 0}, accn[3] = {0, 0, 0};
                                        for (int si = 0; si < P.spp; ++si) {
                                                orc_zsobol smp;
                                                V3 org, dir;
                                                float w;
                                                cam.ray(px, py, P.first_sample + si, &smp, &org, &dir, &w);
                                                PathResult pr = trace_path(sc, &smp, org, dir);
                                                cnt[4 * ti + 0] += 1;
                                                cnt[4 * ti + 1] += pr.ext;
                                                cnt[4 * ti + 2] += pr.shadow;
                                                cnt[4 * ti + 3] += pr.probe;
                                                // Film.add (Film.swift:107-119): iso scaling, then the
                                                // optional clamp of the largest component
                                                V3 sl = mul(pr.L, film_scale);
                                                if (P.max_component > 0.0f) {
                                                        const float mv = max_value(sl);
                                                        if (mv > P.max_component) sl = mul(sl, P.max_component / mv);
                                                }
                                                const float lv[3] = {sl.x, sl.y, sl.z};
                                                const float av[3] = {pr.albedo.x, pr.albedo.y, pr.albedo.z};
                                                const float nv[3] = {pr.normal.x, pr.normal.y, pr.normal.z};
                                                for (int c = 0; c < 3; ++c) {
                                                        acc[c] += lv[c];
                                                        acc2[c] += lv[c] * lv[c];
                                                        acca[c] += av[c];
                                                        accn[c] += nv[c];
                                                }
                                                accw += w;
                                        }
                                        const size_t pix = (size_t)(py - y0) * FW + (px - x0);
                                        for (int c = 0; c < 3; ++c) {
                                                sum_rgb[3 * pix + c] += acc[c];
                                                if (sum_sq) sum_sq[3 * pix + c] += acc2[c];
                                                if (sum_albedo) sum_albedo[3 * pix + c] += acca[c];
                                                if (sum_normal) sum_normal[3 * pix + c] += accn[c];
                                        }
                                        sum_w[pix] += accw;
                                }
                        }
                });
        for (auto &t : pool) t.join();
        if (counters)
                for (int ti = 0; ti < threads; ++ti)
                        for (int k = 0; k < 4; ++k) counters[k] += cnt[4 * ti + k];
}

extern "C" void orc_render(const orc_node *nodes, const orc_prim_id *prims, const orc_mesh *meshes,
                           const orc_material *materials, int64_t n_materials, int64_t n_prims,
                           const orc_render_params *params, float *sum_rgb, float *sum_sq, float *sum_w,
                           uint64_t *counters, int threads) {
        orc_render_ex(nodes, prims, meshes, materials, n_materials, n_prims, nullptr, nullptr, nullptr, params,
                      nullptr, sum_rgb, sum_sq, sum_w, nullptr, nullptr, counters, threads);
}

extern "C" void orc_render_textured(const orc_node *nodes, const orc_prim_id *prims, const orc_mesh *meshes,
                                    const orc_material *materials, int64_t n_materials, int64_t n_prims,
                                    const orc_render_params *params, const orc_textures *textures, float *sum_rgb,
                                    float *sum_sq, float *sum_w, uint64_t *counters, int threads) {
        orc_render_ex(nodes, prims, meshes, materials, n_materials, n_prims, nullptr, nullptr, nullptr, params,
                      textures, sum_rgb, sum_sq, sum_w, nullptr, nullptr, counters, threads);
}

// Sampling and interaction helpers, exported one by one so that tests can pin
// them on the reference's own unit tests (Tests/libgonzalesTests/
// SamplingTests.swift, InteractionTests.swift, FilterTests.swift).
extern "C" float orc_power_heuristic(float f, float g) { return power_heuristic(f, g); }

extern "C" void orc_concentric_disk(float u0, float u1, float *xy) { concentric_disk(u0, u1, &xy[0], &xy[1]); }

extern "C" void orc_cosine_hemisphere(float u0, float u1, float *d) {
        const V3 v = cosine_hemisphere(u0, u1);
        d[0] = v.x;
        d[1] = v.y;
        d[2] = v.z;
}

extern "C" void orc_offset_origin(const float *p, const float *n, const float *dir, float *out) {
        const V3 o = offset_origin(v3(p[0], p[1], p[2]), v3(n[0], n[1], n[2]), v3(dir[0], dir[1], dir[2]));
        out[0] = o.x;
        out[1] = o.y;
        out[2] = o.z;
}

// spawnRay(from:target:) as the shadow test uses it: origin nudged toward the
// target, direction to the target, tHit just below 1.
extern "C" float orc_spawn_to(const float *from, const float *target, float *origin, float *dir) {
        const V3 pf = v3(from[0], from[1], from[2]), pt = v3(target[0], target[1], target[2]);
        const V3 so = add(pf, mul(sub(pt, pf), 0.0001f));
        const V3 sd = sub(pt, so);
        origin[0] = so.x;
        origin[1] = so.y;
        origin[2] = so.z;
        dir[0] = sd.x;
        dir[1] = sd.y;
        dir[2] = sd.z;
        return 1.0f - 0.00001f;
}

extern "C" float orc_gaussian(float x, float sigma) { return gaussian(x, sigma); }

extern "C" void orc_gaussian_sample_1d(float u, float radius, float sigma, float *x, float *density) {
        gaussian_sample_1d(u, radius, sigma, x, density);
}

// Camera rays of paths [first, first + count) of a frame (path = pixel * spp
// + sample, pixel = y * width + x): Ray_C records, ray weights and pixels.
extern "C" void orc_camera_rays(const orc_render_params *params, int64_t first, int64_t count, float *rays6,
                                float *weights, int32_t *pixels) {
        const Camera cam(*params);
        const int32_t *cr = params->crop;
        const bool cropped = cr[0] || cr[1] || cr[2] || cr[3];
        const int x0 = cropped ? cr[0] : 0, y0 = cropped ? cr[1] : 0;
        const int fw = cropped ? cr[2] - cr[0] : params->width;
        for (int64_t i = 0; i < count; ++i) {
                const int64_t q = first + i;
                const int64_t pixel = q / params->spp;
                const int sample = (int)(q % params->spp) + params->first_sample;
                orc_zsobol smp;
                V3 org, dir;
                float w;
                cam.ray(x0 + (int)(pixel % fw), y0 + (int)(pixel / fw), sample, &smp, &org, &dir, &w);
                float *r = rays6 + 6 * i;
                r[0] = org.x;
                r[1] = org.y;
                r[2] = org.z;
                r[3] = dir.x;
                r[4] = dir.y;
                r[5] = dir.z;
                weights[i] = w;
                pixels[i] = (int32_t)pixel;
        }
}
