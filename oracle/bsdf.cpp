// bsdf.cpp - CPU restatement of Gonzales' dielectric, coated-diffuse,
// conductor and coated-conductor BSDFs
// (test infrastructure: checker and CPU baseline).  -ffp-contract=off.
//
// Restated from (paths relative to Sources/libgonzales):
//   Trowbridge-Reitz D, Lambda, G1, G, sample    Reflection/TrowbridgeReitzDistribution.swift:1-121,
//                                                Reflection/MicrofacetDistribution.swift:25-40
//   Fresnel (dielectric), refract, helpers       Reflection/FresnelDielectric.swift, Reflection/Reflection.swift
//   DielectricBsdf evaluate / sample / pdf       Bsdf/DielectricBsdf.swift:22-278
//   LayeredBsdf (coated diffuse: dielectric top, Bsdf/LayeredBsdf.swift:55-520, 847-855;
//     diffuse bottom, no medium)                 Bsdf/CoatedDiffuseBsdf.swift; Material/CoatedDiffuse.swift
//   diffuse, default cosine sampling              Bsdf/DiffuseBsdf.swift; Reflection/Bsdf.swift:20-60
//   conductor Fresnel, microfacet reflection      Reflection/FresnelConductor.swift, Bsdf/MicrofacetReflection.swift
//   coated conductor (dielectric over conductor)  Bsdf/CoatedConductorBsdf.swift; Material/CoatedConductor.swift
//
// The layered BSDF's random walks draw from a RandomSampler the reference
// seeds from the system (non-reproducible).  Here each evaluate / sample /
// pdf call seeds a PCG32 stream from a hash of its direction arguments, so
// calls are deterministic; the device does the same.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "oracle.h"

namespace {

const float kPi = 3.14159265358979323846f;

struct V {
        float x, y, z;
};
inline V v(float x, float y, float z) { return V{x, y, z}; }
inline V add(V a, V b) { return v(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V sub(V a, V b) { return v(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V mul(V a, float s) { return v(a.x * s, a.y * s, a.z * s); }
inline V neg(V a) { return v(-a.x, -a.y, -a.z); }
inline float dot(V a, V b) {
        float s = a.x * b.x;
        s = s + a.y * b.y;
        return s + a.z * b.z;
}
inline V normalize(V a) {
        const float l = std::sqrt(dot(a, a));
        return l == 0.0f ? a : v(a.x / l, a.y / l, a.z / l);
}
inline float sq(float x) { return x * x; }
inline float clampf(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }

// Reflection.swift helpers
inline float cos2_theta(V w) { return w.z * w.z; }
inline float sin2_theta(V w) { return std::max(0.0f, 1.0f - cos2_theta(w)); }
inline float sin_theta(V w) { return std::sqrt(sin2_theta(w)); }
inline float tan_theta(V w) { return sin_theta(w) / w.z; }
inline float tan2_theta(V w) { return sin2_theta(w) / cos2_theta(w); }
inline float cos_phi(V w) {
        const float st = sin_theta(w);
        return st == 0.0f ? 1.0f : clampf(w.x / st, -1.0f, 1.0f);
}
inline float sin_phi(V w) {
        const float st = sin_theta(w);
        return st == 0.0f ? 0.0f : clampf(w.y / st, -1.0f, 1.0f);
}
inline bool same_hemisphere(V a, V b) { return a.z * b.z > 0.0f; }

// ---------------------------------------------------------------- PCG32 stream

struct Rng {
        uint64_t state, inc;
        uint32_t next() {
                const uint64_t old = state;
                state = old * 6364136223846793005ull + inc;
                const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
                const uint32_t rot = (uint32_t)(old >> 59u);
                return (xs >> rot) | (xs << ((32u - rot) & 31u));
        }
        float get1d() { return (float)(next() >> 8) * 5.9604645e-08f; }  // [0, 1), 24 bits
};

uint64_t mix64(uint64_t z) {
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
}

// A component quantised to 1/4096 (a seed that an ulp of difference in a
// direction changes only near a quantisation step).
uint32_t qbits(float x) {
        if (!(std::fabs(x) < 1.0e6f)) return 0u;
        return (uint32_t)(int32_t)std::floor(x * 4096.0f);
}

// A stream seeded from up to two directions and a salt.
Rng rng_for(V a, V b, uint32_t salt) {
        uint64_t h = mix64(((uint64_t)qbits(a.x) << 32) ^ qbits(a.y) ^ ((uint64_t)salt << 48));
        h = mix64(h ^ (((uint64_t)qbits(a.z) << 32) | qbits(b.x)));
        h = mix64(h ^ (((uint64_t)qbits(b.y) << 32) | qbits(b.z)));
        Rng r;
        r.state = 0;
        r.inc = (h << 1u) | 1u;
        r.next();
        r.state += mix64(h + 0x9E3779B97F4A7C15ull);
        r.next();
        return r;
}

// ---------------------------------------------------------------- Trowbridge-Reitz

struct TR {
        float ax, ay;
        bool smooth() const { return std::max(ax, ay) < 0.001f; }
        float D(V wh) const {
                const float t2 = tan2_theta(wh);
                if (std::isinf(t2)) return 0.0f;
                const float cos4 = cos2_theta(wh) * cos2_theta(wh);
                const float e = t2 * (sq(cos_phi(wh) / ax) + sq(sin_phi(wh) / ay));
                return 1.0f / (kPi * ax * ay * cos4 * sq(1.0f + e));
        }
        float lambda(V w) const {
                const float att = std::fabs(tan_theta(w));
                if (std::isinf(att)) return 0.0f;
                const float cp = cos_phi(w), spv = sin_phi(w);
                const float at = std::sqrt(cp * cp * ax * ax + spv * spv * ay * ay);
                const float a2t2 = (at * att) * (at * att);
                return (-1.0f + std::sqrt(1.0f + a2t2)) / 2.0f;
        }
        float G1(V w) const { return 1.0f / (1.0f + lambda(w)); }
        float G(V wo, V wi) const { return 1.0f / (1.0f + lambda(wo) + lambda(wi)); }
        float pdf(V wo, V wh) const { return D(wh) * G1(wo) * std::fabs(dot(wo, wh)) / std::fabs(wo.z); }

        // trowbridgeReitzSample11 (TrowbridgeReitzDistribution.swift:40-88)
        void sample11(float cos_t, float u0, float u1, float &sx, float &sy) const {
                if (cos_t > 0.9999f) {
                        const float r = std::sqrt(u0 / (1.0f - u0));
                        const float phi = 2.0f * kPi * u1;
                        sx = r * std::cos(phi);
                        sy = r * std::sin(phi);
                        return;
                }
                const float sin_t = std::sqrt(std::max(0.0f, 1.0f - cos_t * cos_t));
                const float tan_t = sin_t / cos_t;
                const float inv_tan = 1.0f / tan_t;
                const float g1 = 2.0f / (1.0f + std::sqrt(1.0f + 1.0f / (inv_tan * inv_tan)));
                const float a = 2.0f * u0 / g1 - 1.0f;
                float tmp = 1.0f / (a * a - 1.0f);
                if (tmp > 1e10f) tmp = 1e10f;
                const float b = tan_t;
                const float d = std::sqrt(std::max(0.0f, b * b * tmp * tmp - (a * a - b * b) * tmp));
                const float x1 = b * tmp - d, x2 = b * tmp + d;
                sx = (a < 0.0f || x2 > 1.0f / tan_t) ? x1 : x2;
                float s, uu = u1;
                if (uu > 0.5f) {
                        s = 1.0f;
                        uu = 2.0f * (uu - 0.5f);
                } else {
                        s = -1.0f;
                        uu = 2.0f * (0.5f - uu);
                }
                const float z = (uu * (uu * (uu * 0.27385f - 0.73369f) + 0.46341f)) /
                                (uu * (uu * (uu * 0.093073f + 0.309420f) - 1.000000f) + 0.597999f);
                sy = s * z * std::sqrt(1.0f + sx * sx);
        }

        V sample_wh(V wo, float u0, float u1) const {
                const bool flip = wo.z < 0.0f;
                const V w = flip ? neg(wo) : wo;
                const V ws = normalize(v(ax * w.x, ay * w.y, w.z));
                float sx, sy;
                sample11(ws.z, u0, u1, sx, sy);
                const float cp = cos_phi(ws), spv = sin_phi(ws);
                const float tmp = cp * sx - spv * sy;
                sy = spv * sx + cp * sy;
                sx = tmp;
                sx = ax * sx;
                sy = ay * sy;
                const V h = normalize(v(-sx, -sy, 1.0f));
                return flip ? neg(h) : h;
        }
};

float fresnel_dielectric(float cos_i, float eta) {
        cos_i = clampf(cos_i, -1.0f, 1.0f);
        if (cos_i < 0.0f) {
                eta = 1.0f / eta;
                cos_i = -cos_i;
        }
        const float sin2_i = 1.0f - sq(cos_i);
        const float sin2_t = sin2_i / sq(eta);
        if (sin2_t >= 1.0f) return 1.0f;
        const float cos_t = std::sqrt(1.0f - sin2_t);
        const float ri = eta * cos_i, rt = eta * cos_t;
        const float par = (ri - cos_t) / (ri + cos_t);
        const float perp = (cos_i - rt) / (cos_i + rt);
        return (sq(par) + sq(perp)) / 2.0f;
}

// refract (Reflection.swift:13-30): false on total internal reflection.
bool refract(V wi, V n, float eta, V &wt, float &etap) {
        float c = dot(n, wi);
        V nf = n;
        if (c < 0.0f) {
                eta = 1.0f / eta;
                c = -c;
                nf = neg(nf);
        }
        const float s2i = std::max(0.0f, 1.0f - sq(c));
        const float s2t = s2i / sq(eta);
        if (s2t >= 1.0f) return false;
        const float ct = std::sqrt(1.0f - s2t);
        wt = add(v(-wi.x / eta, -wi.y / eta, -wi.z / eta), mul(nf, c / eta - ct));
        etap = eta;
        return true;
}

inline V face_forward_z(V w) { return w.z < 0.0f ? neg(w) : w; }

struct Sample {
        float f[3];
        V wi;
        float pdf;
        bool valid() const { return !(f[0] == 0.0f && f[1] == 0.0f && f[2] == 0.0f) && wi.z != 0.0f && pdf != 0.0f; }
};

Sample scalar_sample(float f, V wi, float pdf) { return Sample{{f, f, f}, wi, pdf}; }
Sample no_sample() { return Sample{{0, 0, 0}, v(0, 0, 0), 0.0f}; }

}  // namespace

namespace {

// DielectricBsdf (Bsdf/DielectricBsdf.swift).
struct Dielectric {
        TR d;
        float eta;
        bool specular() const { return eta == 1.0f || d.smooth(); }

        float f(V wo, V wi) const {
                if (specular()) return 0.0f;
                const float co = wo.z, ci = wi.z;
                const bool reflect = ci * co > 0.0f;
                float etap = 1.0f;
                if (!reflect) etap = co > 0.0f ? eta : 1.0f / eta;
                V h = add(mul(wi, etap), wo);
                if (ci == 0.0f || co == 0.0f || dot(h, h) == 0.0f) return 0.0f;
                h = face_forward_z(normalize(h));
                if (dot(h, wi) * ci < 0.0f || dot(h, wo) * co < 0.0f) return 0.0f;
                const float fr = fresnel_dielectric(dot(wo, h), eta);
                if (reflect) {
                        const float num = d.D(h) * d.G(wo, wi) * fr;
                        return num / std::fabs(4.0f * ci * co);
                }
                const float den = sq(dot(wi, h) + dot(wo, h) / etap) * std::fabs(ci) * std::fabs(co);
                const float ft = 1.0f - fr;
                float num = d.D(h) * ft * d.G(wo, wi) * (std::fabs(dot(wi, h)) * std::fabs(dot(wo, h)));
                num = num / sq(etap);
                return num / den;
        }

        // radiance = transport mode radiance (else importance)
        Sample sample(V wo, float u0, float u1, float u2, bool radiance) const {
                if (specular()) {
                        const float r = fresnel_dielectric(wo.z, eta), t = 1.0f - r;
                        const float pr = r / (r + t), pt = t / (r + t);
                        if (u0 < pr) {
                                const V wi = v(-wo.x, -wo.y, wo.z);
                                return scalar_sample(r / std::fabs(wi.z), wi, pr);
                        }
                        V wi;
                        float etap;
                        if (!refract(wo, v(0, 0, 1), eta, wi, etap)) return no_sample();
                        float fv = t / std::fabs(wi.z);
                        if (radiance) fv = fv / sq(etap);
                        return scalar_sample(fv, wi, pt);
                }
                const V h = d.sample_wh(wo, u0, u1);
                const float r = fresnel_dielectric(dot(wo, h), eta), t = 1.0f - r;
                const float pr = r / (r + t), pt = t / (r + t);
                if (u2 < pr) {
                        // reflect(vector:by:): -wo + 2 (wo . h) h
                        const V wi = add(neg(wo), mul(h, 2.0f * dot(wo, h)));
                        if (!same_hemisphere(wo, wi)) return no_sample();
                        const float pdf = d.pdf(wo, h) / (4.0f * std::fabs(dot(wo, h))) * pr;
                        const float num = d.D(h) * d.G(wo, wi) * r;
                        const float den = 4.0f * wi.z * wo.z;
                        return scalar_sample(num / den, wi, pdf);
                }
                V wi;
                float etap;
                if (!refract(wo, h, eta, wi, etap)) return no_sample();
                if (same_hemisphere(wo, wi) || wi.z == 0.0f) return no_sample();
                const float den = sq(dot(wi, h) + dot(wo, h) / etap);
                const float dwm = std::fabs(dot(wi, h)) / den;
                const float pdf = d.pdf(wo, h) * dwm * pt;
                float fv = t * d.D(h) * d.G(wo, wi) *
                           std::fabs(dot(wi, h) * dot(wo, h) / (std::fabs(wi.z) * std::fabs(wo.z) * den));
                if (radiance) fv = fv / sq(etap);
                return scalar_sample(fv, wi, pdf);
        }

        float pdf(V wo, V wi) const {
                if (eta == 1.0f || d.smooth()) return 0.0f;
                const float co = wo.z, ci = wi.z;
                const bool reflect = ci * co > 0.0f;
                float etap = 1.0f;
                if (!reflect) etap = co > 0.0f ? eta : 1.0f / eta;
                V h = add(mul(wi, etap), wo);
                if (co == 0.0f || ci == 0.0f || dot(h, h) == 0.0f) return 0.0f;
                h = face_forward_z(normalize(h));
                if (dot(h, wi) * ci < 0.0f || dot(h, wo) * co < 0.0f) return 0.0f;
                const float r = fresnel_dielectric(dot(wo, h), eta), t = 1.0f - r;
                if (reflect) return d.pdf(wo, h) / (4.0f * std::fabs(dot(wo, h))) * (r / (r + t));
                const float den = sq(dot(wi, h) + dot(wo, h) / etap);
                const float dwm = std::fabs(dot(wi, h)) / den;
                return d.pdf(wo, h) * dwm * t / (r + t);
        }
};

// DiffuseBsdf with the default cosine sampling of Reflection/Bsdf.swift.
struct Diffuse {
        float R[3];
        void f(float out[3]) const {
                for (int c = 0; c < 3; ++c) out[c] = R[c] / kPi;
        }
        float pdf(V wo, V wi) const { return same_hemisphere(wo, wi) ? std::fabs(wi.z) / kPi : 0.0f; }
        Sample sample(V wo, float u0, float u1) const {
                float dx = 0.0f, dy = 0.0f;
                const float ox = 2.0f * u0 - 1.0f, oy = 2.0f * u1 - 1.0f;
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
                V wi = v(dx, dy, std::sqrt(std::max(0.0f, 1.0f - dx * dx - dy * dy)));
                if (wo.z < 0.0f) wi.z = -wi.z;
                Sample s;
                f(s.f);
                s.wi = wi;
                s.pdf = pdf(wo, wi);
                return s;
        }
        // as a layer's base: the value ignores the directions (DiffuseBsdf.evaluate)
        void f(V, V, float out[3]) const { f(out); }
};

// FresnelConductor.fresnelConductor for one channel, etaI = 1
// (Reflection/FresnelConductor.swift:4-28).
float fresnel_conductor(float cos_theta, float eta, float etak) {
        const float c = clampf(cos_theta, -1.0f, 1.0f);
        const float cos2 = c * c;
        const float sin2 = 1.0f - cos2;
        const float eta2 = eta * eta;
        const float etak2 = etak * etak;
        const float t0 = eta2 - etak2 - sin2;
        const float a2pb2 = std::sqrt(t0 * t0 + 4.0f * eta2 * etak2);
        const float t1 = a2pb2 + cos2;
        const float a = std::sqrt(0.5f * (a2pb2 + t0));
        const float t2 = 2.0f * c * a;
        const float rs = (t1 - t2) / (t1 + t2);
        const float t3 = cos2 * a2pb2 + sin2 * sin2;
        const float t4 = t2 * sin2;
        const float rp = rs * (t3 - t4) / (t3 + t4);
        return 0.5f * (rp + rs);
}

// MicrofacetReflection with a conductor Fresnel term
// (Bsdf/MicrofacetReflection.swift:1-42): Conductor (reflectance white) and
// the base of CoatedConductor (reflectance from the material).
struct Conductor {
        TR d;
        float R[3];
        float eta[3], k[3];
        void f(V wo, V wi, float out[3]) const {
                out[0] = out[1] = out[2] = 0.0f;
                const float co = std::fabs(wo.z), ci = std::fabs(wi.z);
                V h = add(wo, wi);
                if (co == 0.0f || ci == 0.0f) return;
                if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return;
                h = normalize(h);
                const float cf = std::fabs(dot(wi, h));
                const float area = d.D(h);
                const float vis = d.G(wo, wi);
                const float den = 4.0f * ci * co;
                for (int c = 0; c < 3; ++c) out[c] = R[c] * area * vis * fresnel_conductor(cf, eta[c], k[c]) / den;
        }
        float pdf(V wo, V wi) const {
                if (!same_hemisphere(wo, wi)) return 0.0f;
                const V h = normalize(add(wo, wi));
                return d.pdf(wo, h) / (4.0f * dot(wo, h));
        }
        Sample sample(V wo, float u0, float u1) const {
                if (wo.z == 0.0f) return no_sample();
                const V h = d.sample_wh(wo, u0, u1);
                const V wi = add(neg(wo), mul(h, 2.0f * dot(wo, h)));
                Sample s;
                f(wo, wi, s.f);
                s.wi = wi;
                s.pdf = pdf(wo, wi);
                return s;
        }
};

inline float transmittance(float dz, V w) {
        if (std::fabs(dz) < 1.17549435e-38f) return 1.0f;
        return std::exp(-std::fabs(dz / w.z));
}

inline float max3(const float a[3]) { return std::max(a[0], std::max(a[1], a[2])); }

}  // namespace

namespace {

// LayeredBsdf<DielectricBsdf, Bottom> with a clear layer (albedo 0),
// two-sided (Bsdf/LayeredBsdf.swift): coated diffuse (Bottom = Diffuse,
// Bsdf/CoatedDiffuseBsdf.swift) and coated conductor (Bottom = Conductor,
// Bsdf/CoatedConductorBsdf.swift).
template <class Bottom>
struct Layered {
        Dielectric top;
        Bottom bottom;
        float thickness;
        int max_depth, nsamples;

        // evaluate (:55-299)
        void f(V wo, V wi, float out[3]) const {
                float res[3] = {0, 0, 0};
                if (wo.z < 0.0f) {
                        wo = neg(wo);
                        wi = neg(wi);
                }
                const bool same = same_hemisphere(wo, wi);
                const float exit_z = same ? thickness : 0.0f;  // entered at the top
                if (same) {
                        const float ft = top.f(wo, wi) * (float)nsamples;
                        for (int c = 0; c < 3; ++c) res[c] = ft;
                }
                Rng rng = rng_for(wo, wi, 1u);
                for (int s = 0; s < nsamples; ++s) {
                        const float a0 = rng.get1d(), a1 = rng.get1d(), a2 = rng.get1d();
                        const Sample wos = top.sample(wo, a0, a1, a2, true);
                        if (!wos.valid() || same_hemisphere(wos.wi, wo) || wos.wi.z == 0.0f) continue;
                        const float b0 = rng.get1d(), b1 = rng.get1d(), b2 = rng.get1d();
                        const Sample wis = same ? top.sample(wi, b0, b1, b2, false) : bottom.sample(wi, b0, b1);
                        if (!wis.valid() || same_hemisphere(wis.wi, wi) || wis.wi.z == 0.0f) continue;
                        float beta[3];
                        for (int c = 0; c < 3; ++c) beta[c] = wos.f[c] * std::fabs(wos.wi.z) / wos.pdf;
                        float z = thickness;
                        V w = wos.wi;
                        for (int depth = 0; depth < max_depth; ++depth) {
                                if (depth > 3 && max3(beta) < 0.25f) {
                                        const float q = std::max(0.0f, 1.0f - max3(beta));
                                        if (rng.get1d() < q) break;
                                        for (int c = 0; c < 3; ++c) beta[c] = beta[c] / (1.0f - q);
                                }
                                z = z == thickness ? 0.0f : thickness;
                                const float tr = transmittance(thickness, w);
                                for (int c = 0; c < 3; ++c) beta[c] = beta[c] * tr;
                                if (z == exit_z) {
                                        const float c0 = rng.get1d(), c1 = rng.get1d(), c2 = rng.get1d();
                                        const Sample bs = z == 0.0f ? bottom.sample(neg(w), c0, c1)
                                                                    : top.sample(neg(w), c0, c1, c2, true);
                                        if (!bs.valid() || bs.pdf == 0.0f || bs.wi.z == 0.0f) break;
                                        if (!same_hemisphere(bs.wi, neg(w))) break;
                                        for (int c = 0; c < 3; ++c)
                                                beta[c] = beta[c] * bs.f[c] * std::fabs(bs.wi.z) / bs.pdf;
                                        w = bs.wi;
                                } else {
                                        // NEE through the exit interface along wis
                                        float ne[3];
                                        float ne_pdf;
                                        if (z == 0.0f) {
                                                bottom.f(neg(w), neg(wis.wi), ne);
                                                ne_pdf = bottom.pdf(neg(w), neg(wis.wi));
                                        } else {
                                                const float ft = top.f(neg(w), neg(wis.wi));
                                                ne[0] = ne[1] = ne[2] = ft;
                                                ne_pdf = top.pdf(neg(w), neg(wis.wi));
                                        }
                                        const float wt = ne_pdf == 0.0f || wis.pdf == 0.0f
                                                                 ? 0.0f
                                                                 : (wis.pdf * wis.pdf) / (wis.pdf * wis.pdf + ne_pdf * ne_pdf);
                                        const float trw = transmittance(thickness, wis.wi);
                                        for (int c = 0; c < 3; ++c)
                                                res[c] = res[c] + beta[c] * ne[c] * std::fabs(wis.wi.z) * wt * trw *
                                                                      wis.f[c] / wis.pdf;
                                        const float c0 = rng.get1d(), c1 = rng.get1d(), c2 = rng.get1d();
                                        const Sample bs = z == 0.0f ? bottom.sample(neg(w), c0, c1)
                                                                    : top.sample(neg(w), c0, c1, c2, true);
                                        if (!bs.valid() || bs.pdf == 0.0f || bs.wi.z == 0.0f) break;
                                        if (!same_hemisphere(bs.wi, neg(w))) break;
                                        for (int c = 0; c < 3; ++c)
                                                beta[c] = beta[c] * bs.f[c] * std::fabs(bs.wi.z) / bs.pdf;
                                        w = bs.wi;
                                        // NEE of the exit interface along the new direction
                                        float fe[3];
                                        float fe_pdf;
                                        if (exit_z == 0.0f) {
                                                bottom.f(neg(w), wi, fe);
                                                fe_pdf = bottom.pdf(neg(w), wi);
                                        } else {
                                                const float ft = top.f(neg(w), wi);
                                                fe[0] = fe[1] = fe[2] = ft;
                                                fe_pdf = top.pdf(neg(w), wi);
                                        }
                                        if (!(fe[0] == 0.0f && fe[1] == 0.0f && fe[2] == 0.0f)) {
                                                const float we = fe_pdf == 0.0f || bs.pdf == 0.0f
                                                                         ? 0.0f
                                                                         : (bs.pdf * bs.pdf) / (bs.pdf * bs.pdf + fe_pdf * fe_pdf);
                                                const float tre = transmittance(thickness, bs.wi);
                                                for (int c = 0; c < 3; ++c) res[c] = res[c] + beta[c] * tre * fe[c] * we;
                                        }
                                }
                        }
                }
                for (int c = 0; c < 3; ++c) out[c] = res[c] / (float)nsamples;
        }

        // sample (:301-384).  As written, the walk ends after its first
        // interface sample: isTransmission is asked after the sampled
        // direction replaced the walk direction, and a direction is never in
        // the hemisphere of its own negation.
        Sample sample(V wo, float u0, float u1, float u2) const {
                bool flip = false;
                if (wo.z < 0.0f) {
                        wo = neg(wo);
                        flip = true;
                }
                const Sample st = top.sample(wo, u0, u1, u2, true);
                if (!st.valid() || st.pdf == 0.0f || st.wi.z == 0.0f) return no_sample();
                if (same_hemisphere(st.wi, wo)) {
                        Sample r = st;
                        if (flip) r.wi = neg(r.wi);
                        return r;
                }
                V w = st.wi;
                Rng rng = rng_for(wo, v(u0, u1, u2), 2u);
                float f[3];
                for (int c = 0; c < 3; ++c) f[c] = st.f[c] * std::fabs(w.z);
                float pdf = st.pdf;
                float z = thickness;
                for (int depth = 0; depth < max_depth; ++depth) {
                        const float rr = max3(f) / pdf;
                        if (depth > 3 && rr < 0.25f) {
                                const float q = std::max(0.0f, 1.0f - rr);
                                if (rng.get1d() < q) return no_sample();
                                pdf = pdf * (1.0f - q);
                        }
                        if (w.z == 0.0f) return no_sample();
                        z = z == thickness ? 0.0f : thickness;
                        const float c0 = rng.get1d(), c1 = rng.get1d(), c2 = rng.get1d();
                        const Sample bs = z == 0.0f ? bottom.sample(neg(w), c0, c1) : top.sample(neg(w), c0, c1, c2, true);
                        if (!bs.valid() || bs.pdf == 0.0f || bs.wi.z == 0.0f) return no_sample();
                        for (int c = 0; c < 3; ++c) f[c] = f[c] * bs.f[c];
                        pdf = pdf * bs.pdf;
                        w = bs.wi;
                        if (!same_hemisphere(bs.wi, neg(w))) {
                                Sample r;
                                for (int c = 0; c < 3; ++c) r.f[c] = f[c];
                                r.wi = flip ? neg(w) : w;
                                r.pdf = pdf;
                                return r;
                        }
                        for (int c = 0; c < 3; ++c) f[c] = f[c] * std::fabs(bs.wi.z);
                }
                return no_sample();
        }

        // probabilityDensity (:386-520)
        float pdf(V wo, V wi) const {
                if (wo.z < 0.0f) {
                        wo = neg(wo);
                        wi = neg(wi);
                }
                Rng rng = rng_for(wo, wi, 3u);
                float sum = 0.0f;
                const bool same = same_hemisphere(wo, wi);
                if (same) sum = sum + (float)nsamples * top.pdf(wo, wi);
                for (int s = 0; s < nsamples; ++s) {
                        if (same) {
                                const float a0 = rng.get1d(), a1 = rng.get1d(), a2 = rng.get1d();
                                const Sample wos = top.sample(wo, a0, a1, a2, true);
                                const float b0 = rng.get1d(), b1 = rng.get1d(), b2 = rng.get1d();
                                const Sample wis = top.sample(wi, b0, b1, b2, true);
                                if (wos.valid() && !same_hemisphere(wos.wi, wo) && wis.valid() &&
                                    !same_hemisphere(wis.wi, wi)) {
                                        const float c0 = rng.get1d(), c1 = rng.get1d();
                                        rng.get1d();
                                        const Sample rs = bottom.sample(neg(wos.wi), c0, c1);
                                        if (rs.valid() && rs.pdf > 0.0f) {
                                                const float rp = bottom.pdf(neg(wos.wi), neg(wis.wi));
                                                float wt = rp == 0.0f || wis.pdf == 0.0f
                                                                   ? 0.0f
                                                                   : (wis.pdf * wis.pdf) / (wis.pdf * wis.pdf + rp * rp);
                                                sum = sum + wt * rp;
                                                const float tp = top.pdf(neg(rs.wi), wi);
                                                wt = tp == 0.0f || rs.pdf == 0.0f ? 0.0f
                                                                                  : (rs.pdf * rs.pdf) / (rs.pdf * rs.pdf + tp * tp);
                                                sum = sum + wt * tp;
                                        }
                                }
                        } else {
                                const float a0 = rng.get1d(), a1 = rng.get1d(), a2 = rng.get1d();
                                const Sample wos = top.sample(wo, a0, a1, a2, true);
                                const float b0 = rng.get1d(), b1 = rng.get1d();
                                rng.get1d();
                                const Sample wis = bottom.sample(wi, b0, b1);
                                if (wos.valid() && !same_hemisphere(wos.wi, wo) && wis.valid() &&
                                    !same_hemisphere(wis.wi, wi)) {
                                        const float p1 = top.pdf(wo, neg(wis.wi));
                                        const float p2 = bottom.pdf(neg(wos.wi), wi);
                                        sum = sum + (p1 + p2) / 2.0f;
                                }
                        }
                }
                // lerp(0.9, 1 / (4 pi), sum / n) (Utility/Utility.swift:67-69)
                return (1.0f - 0.9f) * (1.0f / (4.0f * kPi)) + 0.9f * (sum / (float)nsamples);
        }
};

}  // namespace

// ---------------------------------------------------------------- materials

struct OrcMat {
        int type;  // 1 diffuse, 3 dielectric, 4 coated diffuse, 5 conductor, 6 coated conductor
        Diffuse diffuse;
        Dielectric diel;
        Layered<Diffuse> coated;
        Conductor conductor;
        Layered<Conductor> coated_conductor;
};

namespace {

// Dielectric.getBsdf, CoatedDiffuse.getBsdf, Conductor.getBsdf and
// CoatedConductor.getBsdf (Material/Dielectric.swift:3-14,
// Material/CoatedDiffuse.swift:23-58, Material/Conductor.swift:3-22,
// Material/CoatedConductor.swift:35-88): dielectric and coating roughness
// remapped to alpha = sqrt (a coating's alpha at least 0.001); a plain
// conductor's roughness is its alpha (at least 1e-3), a coated conductor's
// is remapped (at least 0.001); layers: thickness, depth 10, one sample.
OrcMat make_mat(const orc_bsdf_params &p) {
        OrcMat m;
        m.type = p.type;
        for (int c = 0; c < 3; ++c) m.diffuse.R[c] = p.reflectance[c];
        float ax = std::sqrt(p.roughness_u), ay = std::sqrt(p.roughness_v);
        if (p.type == 4 || p.type == 6) {
                ax = std::max(ax, 0.001f);
                ay = std::max(ay, 0.001f);
        }
        m.diel.d = TR{ax, ay};
        m.diel.eta = p.eta;
        const float thick = std::max(p.thickness, 1.17549435e-38f);
        m.coated.top = m.diel;
        m.coated.bottom = m.diffuse;
        m.coated.thickness = thick;
        m.coated.max_depth = 10;
        m.coated.nsamples = 1;
        float cx, cy;
        if (p.type == 6) {
                cx = std::max(std::sqrt(p.conductor_roughness_u), 0.001f);
                cy = std::max(std::sqrt(p.conductor_roughness_v), 0.001f);
        } else {
                cx = std::max(p.conductor_roughness_u, 1e-3f);
                cy = std::max(p.conductor_roughness_v, 1e-3f);
        }
        m.conductor.d = TR{cx, cy};
        for (int c = 0; c < 3; ++c) {
                m.conductor.R[c] = p.type == 6 ? p.reflectance[c] : 1.0f;
                m.conductor.eta[c] = p.conductor_eta[c];
                m.conductor.k[c] = p.conductor_k[c];
        }
        m.coated_conductor.top = m.diel;
        m.coated_conductor.bottom = m.conductor;
        m.coated_conductor.thickness = thick;
        m.coated_conductor.max_depth = 10;
        m.coated_conductor.nsamples = 1;
        return m;
}

void mat_f(const OrcMat &m, V wo, V wi, float out[3]) {
        if (m.type == 3) {
                out[0] = out[1] = out[2] = m.diel.f(wo, wi);
        } else if (m.type == 4) {
                m.coated.f(wo, wi, out);
        } else if (m.type == 5) {
                m.conductor.f(wo, wi, out);
        } else if (m.type == 6) {
                m.coated_conductor.f(wo, wi, out);
        } else {
                m.diffuse.f(out);
        }
}

float mat_pdf(const OrcMat &m, V wo, V wi) {
        if (m.type == 3) return m.diel.pdf(wo, wi);
        if (m.type == 4) return m.coated.pdf(wo, wi);
        if (m.type == 5) return m.conductor.pdf(wo, wi);
        if (m.type == 6) return m.coated_conductor.pdf(wo, wi);
        return m.diffuse.pdf(wo, wi);
}

Sample mat_sample(const OrcMat &m, V wo, float u0, float u1, float u2) {
        if (m.type == 3) return m.diel.sample(wo, u0, u1, u2, true);
        if (m.type == 4) return m.coated.sample(wo, u0, u1, u2);
        if (m.type == 5) return m.conductor.sample(wo, u0, u1);
        if (m.type == 6) return m.coated_conductor.sample(wo, u0, u1, u2);
        return m.diffuse.sample(wo, u0, u1);
}

}  // namespace

extern "C" void orc_bsdf_eval(const orc_bsdf_params *p, const float *wo, const float *wi, float *f, float *pdf) {
        const OrcMat m = make_mat(*p);
        mat_f(m, v(wo[0], wo[1], wo[2]), v(wi[0], wi[1], wi[2]), f);
        *pdf = mat_pdf(m, v(wo[0], wo[1], wo[2]), v(wi[0], wi[1], wi[2]));
}

extern "C" int orc_bsdf_sample(const orc_bsdf_params *p, const float *wo, const float *u, float *f, float *wi,
                               float *pdf) {
        const OrcMat m = make_mat(*p);
        const Sample s = mat_sample(m, v(wo[0], wo[1], wo[2]), u[0], u[1], u[2]);
        for (int c = 0; c < 3; ++c) f[c] = s.f[c];
        wi[0] = s.wi.x;
        wi[1] = s.wi.y;
        wi[2] = s.wi.z;
        *pdf = s.pdf;
        return s.valid() ? 1 : 0;
}

extern "C" int orc_bsdf_is_specular(const orc_bsdf_params *p) {
        const OrcMat m = make_mat(*p);
        return m.type == 3 && m.diel.specular() ? 1 : 0;
}
