// bsdf.cuh - dielectric, coated-diffuse, conductor and coated-conductor
// BSDFs on the device, in the shading frame (z = normal).  Included by
// render.cu inside its anonymous namespace, after its vector helpers (V3,
// dot, normalize, ...).
//
//   Trowbridge-Reitz D, Lambda, G, visible-normal sample
//       Reflection/TrowbridgeReitzDistribution.swift, Reflection/MicrofacetDistribution.swift
//   dielectric Fresnel, refract       Reflection/FresnelDielectric.swift, Reflection/Reflection.swift
//   DielectricBsdf                    Bsdf/DielectricBsdf.swift
//   LayeredBsdf<Dielectric, Diffuse> with a clear layer (coated diffuse)
//                                     Bsdf/LayeredBsdf.swift, Bsdf/CoatedDiffuseBsdf.swift
//   conductor Fresnel, MicrofacetReflection, coated conductor
//                                     Reflection/FresnelConductor.swift, Bsdf/MicrofacetReflection.swift,
//                                     Bsdf/CoatedConductorBsdf.swift
//
// The layered walks draw from a PCG32 stream seeded by a hash of the call's
// direction arguments (the reference seeds a RandomSampler from the system).
//
// The BSDF bodies and the larger microfacet and Fresnel helpers are kept out
// of line: the coated kernels were bound by instruction fetch (most stalls
// "no instruction"), and one copy of each body cut a mixed-material frame by
// 7 % against inlining them into every caller.

struct BsdfS {
        V3 f;
        V3 wi;
        float pdf;
        __device__ bool valid() const { return !is_black(f) && wi.z != 0.0f && pdf != 0.0f; }
};

__device__ __forceinline__ BsdfS bs_none() { return BsdfS{v3(0, 0, 0), v3(0, 0, 0), 0.0f}; }
__device__ __forceinline__ BsdfS bs_scalar(float f, V3 wi, float pdf) { return BsdfS{v3(f, f, f), wi, pdf}; }

__device__ __forceinline__ float b_sq(float x) { return x * x; }
__device__ __forceinline__ float b_clamp(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }
__device__ __forceinline__ float b_cos2(V3 w) { return w.z * w.z; }
__device__ __forceinline__ float b_sin2(V3 w) { return fmaxf(0.0f, 1.0f - b_cos2(w)); }
__device__ __forceinline__ float b_sin(V3 w) { return sqrtf(b_sin2(w)); }
__device__ __forceinline__ float b_cosphi(V3 w) {
        const float st = b_sin(w);
        return st == 0.0f ? 1.0f : b_clamp(w.x / st, -1.0f, 1.0f);
}
__device__ __forceinline__ float b_sinphi(V3 w) {
        const float st = b_sin(w);
        return st == 0.0f ? 0.0f : b_clamp(w.y / st, -1.0f, 1.0f);
}
__device__ __forceinline__ bool b_same(V3 a, V3 b) { return a.z * b.z > 0.0f; }
__device__ __forceinline__ V3 b_norm0(V3 a) {
        const float l = sqrtf(dot(a, a));
        return l == 0.0f ? a : v3(a.x / l, a.y / l, a.z / l);
}

// ---- PCG32 stream
struct BRng {
        unsigned long long state, inc;
        __device__ uint32_t next() {
                const unsigned long long old = state;
                state = old * 6364136223846793005ull + inc;
                const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
                const uint32_t rot = (uint32_t)(old >> 59u);
                return (xs >> rot) | (xs << ((32u - rot) & 31u));
        }
        __device__ float get1d() { return (float)(next() >> 8) * 5.9604645e-08f; }
};

__device__ __forceinline__ unsigned long long b_mix64(unsigned long long z) {
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
}

// A component quantised to 1/4096, so that an ulp of difference in a
// direction changes the seed only near a quantisation step.
__device__ __forceinline__ uint32_t b_qbits(float x) {
        if (!(fabsf(x) < 1.0e6f)) return 0u;
        return (uint32_t)(int32_t)floorf(x * 4096.0f);
}

// A stream seeded from up to two directions and a salt.
__device__ BRng b_rng(V3 a, V3 b, uint32_t salt) {
        unsigned long long h = b_mix64(((unsigned long long)b_qbits(a.x) << 32) ^ b_qbits(a.y) ^
                                       ((unsigned long long)salt << 48));
        h = b_mix64(h ^ (((unsigned long long)b_qbits(a.z) << 32) | b_qbits(b.x)));
        h = b_mix64(h ^ (((unsigned long long)b_qbits(b.y) << 32) | b_qbits(b.z)));
        BRng r;
        r.state = 0ull;
        r.inc = (h << 1u) | 1ull;
        r.next();
        r.state += b_mix64(h + 0x9E3779B97F4A7C15ull);
        r.next();
        return r;
}

// ---- Trowbridge-Reitz
struct BTR {
        float ax, ay;
        __device__ bool smooth() const { return fmaxf(ax, ay) < 0.001f; }
        __device__ __noinline__ float D(V3 h) const {
                const float t2 = b_sin2(h) / b_cos2(h);
                if (isinf(t2)) return 0.0f;
                const float cos4 = b_cos2(h) * b_cos2(h);
                const float e = t2 * (b_sq(b_cosphi(h) / ax) + b_sq(b_sinphi(h) / ay));
                return 1.0f / (kPi * ax * ay * cos4 * b_sq(1.0f + e));
        }
        __device__ __noinline__ float lambda(V3 w) const {
                const float att = fabsf(b_sin(w) / w.z);
                if (isinf(att)) return 0.0f;
                const float cp = b_cosphi(w), sp = b_sinphi(w);
                const float at = sqrtf(cp * cp * ax * ax + sp * sp * ay * ay);
                const float a2t2 = (at * att) * (at * att);
                return (-1.0f + sqrtf(1.0f + a2t2)) / 2.0f;
        }
        __device__ float G1(V3 w) const { return 1.0f / (1.0f + lambda(w)); }
        __device__ float G(V3 wo, V3 wi) const { return 1.0f / (1.0f + lambda(wo) + lambda(wi)); }
        __device__ float pdf(V3 wo, V3 h) const { return D(h) * G1(wo) * fabsf(dot(wo, h)) / fabsf(wo.z); }
        __device__ __noinline__ V3 sample_wh(V3 wo, float u0, float u1) const {
                const bool flip = wo.z < 0.0f;
                const V3 w = flip ? neg(wo) : wo;
                const V3 ws = b_norm0(v3(ax * w.x, ay * w.y, w.z));
                float sx, sy;
                const float cos_t = ws.z;
                if (cos_t > 0.9999f) {
                        const float r = sqrtf(u0 / (1.0f - u0));
                        const float phi = 2.0f * kPi * u1;
                        sx = r * cosf(phi);
                        sy = r * sinf(phi);
                } else {
                        const float sin_t = sqrtf(fmaxf(0.0f, 1.0f - cos_t * cos_t));
                        const float tan_t = sin_t / cos_t;
                        const float inv_tan = 1.0f / tan_t;
                        const float g1 = 2.0f / (1.0f + sqrtf(1.0f + 1.0f / (inv_tan * inv_tan)));
                        const float a = 2.0f * u0 / g1 - 1.0f;
                        float tmp = 1.0f / (a * a - 1.0f);
                        if (tmp > 1e10f) tmp = 1e10f;
                        const float b = tan_t;
                        const float d = sqrtf(fmaxf(0.0f, b * b * tmp * tmp - (a * a - b * b) * tmp));
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
                        sy = s * z * sqrtf(1.0f + sx * sx);
                }
                const float cp = b_cosphi(ws), sp = b_sinphi(ws);
                const float tmp = cp * sx - sp * sy;
                sy = sp * sx + cp * sy;
                sx = ax * tmp;
                sy = ay * sy;
                const V3 h = b_norm0(v3(-sx, -sy, 1.0f));
                return flip ? neg(h) : h;
        }
};

__device__ __noinline__ float b_fresnel(float ci, float eta) {
        ci = b_clamp(ci, -1.0f, 1.0f);
        if (ci < 0.0f) {
                eta = 1.0f / eta;
                ci = -ci;
        }
        const float s2i = 1.0f - b_sq(ci);
        const float s2t = s2i / b_sq(eta);
        if (s2t >= 1.0f) return 1.0f;
        const float ct = sqrtf(1.0f - s2t);
        const float ri = eta * ci, rt = eta * ct;
        const float par = (ri - ct) / (ri + ct);
        const float perp = (ci - rt) / (ci + rt);
        return (b_sq(par) + b_sq(perp)) / 2.0f;
}

__device__ bool b_refract(V3 wi, V3 n, float eta, V3 &wt, float &etap) {
        float c = dot(n, wi);
        V3 nf = n;
        if (c < 0.0f) {
                eta = 1.0f / eta;
                c = -c;
                nf = neg(nf);
        }
        const float s2i = fmaxf(0.0f, 1.0f - b_sq(c));
        const float s2t = s2i / b_sq(eta);
        if (s2t >= 1.0f) return false;
        const float ct = sqrtf(1.0f - s2t);
        wt = v3(-wi.x / eta, -wi.y / eta, -wi.z / eta) + nf * (c / eta - ct);
        etap = eta;
        return true;
}

// ---- DielectricBsdf
struct BDiel {
        BTR d;
        float eta;
        __device__ bool specular() const { return eta == 1.0f || d.smooth(); }
        __device__ __noinline__ float f(V3 wo, V3 wi) const {
                if (specular()) return 0.0f;
                const float co = wo.z, ci = wi.z;
                const bool reflect = ci * co > 0.0f;
                float etap = 1.0f;
                if (!reflect) etap = co > 0.0f ? eta : 1.0f / eta;
                V3 h = wi * etap + wo;
                if (ci == 0.0f || co == 0.0f || dot(h, h) == 0.0f) return 0.0f;
                h = b_norm0(h);
                if (h.z < 0.0f) h = neg(h);
                if (dot(h, wi) * ci < 0.0f || dot(h, wo) * co < 0.0f) return 0.0f;
                const float fr = b_fresnel(dot(wo, h), eta);
                if (reflect) return d.D(h) * d.G(wo, wi) * fr / fabsf(4.0f * ci * co);
                const float den = b_sq(dot(wi, h) + dot(wo, h) / etap) * fabsf(ci) * fabsf(co);
                float num = d.D(h) * (1.0f - fr) * d.G(wo, wi) * (fabsf(dot(wi, h)) * fabsf(dot(wo, h)));
                num = num / b_sq(etap);
                return num / den;
        }
        __device__ __noinline__ BsdfS sample(V3 wo, float u0, float u1, float u2, bool radiance) const {
                if (specular()) {
                        const float r = b_fresnel(wo.z, eta), t = 1.0f - r;
                        const float pr = r / (r + t), pt = t / (r + t);
                        if (u0 < pr) {
                                const V3 wi = v3(-wo.x, -wo.y, wo.z);
                                return bs_scalar(r / fabsf(wi.z), wi, pr);
                        }
                        V3 wi;
                        float etap;
                        if (!b_refract(wo, v3(0, 0, 1), eta, wi, etap)) return bs_none();
                        float fv = t / fabsf(wi.z);
                        if (radiance) fv = fv / b_sq(etap);
                        return bs_scalar(fv, wi, pt);
                }
                const V3 h = d.sample_wh(wo, u0, u1);
                const float r = b_fresnel(dot(wo, h), eta), t = 1.0f - r;
                const float pr = r / (r + t), pt = t / (r + t);
                if (u2 < pr) {
                        const V3 wi = neg(wo) + h * (2.0f * dot(wo, h));
                        if (!b_same(wo, wi)) return bs_none();
                        const float pdf = d.pdf(wo, h) / (4.0f * fabsf(dot(wo, h))) * pr;
                        return bs_scalar(d.D(h) * d.G(wo, wi) * r / (4.0f * wi.z * wo.z), wi, pdf);
                }
                V3 wi;
                float etap;
                if (!b_refract(wo, h, eta, wi, etap)) return bs_none();
                if (b_same(wo, wi) || wi.z == 0.0f) return bs_none();
                const float den = b_sq(dot(wi, h) + dot(wo, h) / etap);
                const float dwm = fabsf(dot(wi, h)) / den;
                const float pdf = d.pdf(wo, h) * dwm * pt;
                float fv = t * d.D(h) * d.G(wo, wi) * fabsf(dot(wi, h) * dot(wo, h) / (fabsf(wi.z) * fabsf(wo.z) * den));
                if (radiance) fv = fv / b_sq(etap);
                return bs_scalar(fv, wi, pdf);
        }
        __device__ __noinline__ float pdf(V3 wo, V3 wi) const {
                if (eta == 1.0f || d.smooth()) return 0.0f;
                const float co = wo.z, ci = wi.z;
                const bool reflect = ci * co > 0.0f;
                float etap = 1.0f;
                if (!reflect) etap = co > 0.0f ? eta : 1.0f / eta;
                V3 h = wi * etap + wo;
                if (co == 0.0f || ci == 0.0f || dot(h, h) == 0.0f) return 0.0f;
                h = b_norm0(h);
                if (h.z < 0.0f) h = neg(h);
                if (dot(h, wi) * ci < 0.0f || dot(h, wo) * co < 0.0f) return 0.0f;
                const float r = b_fresnel(dot(wo, h), eta), t = 1.0f - r;
                if (reflect) return d.pdf(wo, h) / (4.0f * fabsf(dot(wo, h))) * (r / (r + t));
                const float den = b_sq(dot(wi, h) + dot(wo, h) / etap);
                return d.pdf(wo, h) * (fabsf(dot(wi, h)) / den) * t / (r + t);
        }
};

// ---- DiffuseBsdf with the default cosine sampling (Reflection/Bsdf.swift)
struct BDiff {
        V3 R;
        __device__ V3 f() const { return v3(R.x / kPi, R.y / kPi, R.z / kPi); }
        __device__ float pdf(V3 wo, V3 wi) const { return b_same(wo, wi) ? fabsf(wi.z) / kPi : 0.0f; }
        __device__ BsdfS sample(V3 wo, float u0, float u1) const {
                V3 wi = cosine_hemisphere(u0, u1);
                if (wo.z < 0.0f) wi.z = -wi.z;
                return BsdfS{f(), wi, pdf(wo, wi)};
        }
        // as a layer's base: the value ignores the directions
        __device__ V3 f(V3, V3) const { return f(); }
};

// ---- conductor Fresnel term for one channel, etaI = 1 (Reflection/FresnelConductor.swift)
__device__ __noinline__ float b_fresnel_conductor(float cos_theta, float eta, float etak) {
        const float c = b_clamp(cos_theta, -1.0f, 1.0f);
        const float cos2 = c * c;
        const float sin2 = 1.0f - cos2;
        const float eta2 = eta * eta;
        const float etak2 = etak * etak;
        const float t0 = eta2 - etak2 - sin2;
        const float a2pb2 = sqrtf(t0 * t0 + 4.0f * eta2 * etak2);
        const float t1 = a2pb2 + cos2;
        const float a = sqrtf(0.5f * (a2pb2 + t0));
        const float t2 = 2.0f * c * a;
        const float rs = (t1 - t2) / (t1 + t2);
        const float t3 = cos2 * a2pb2 + sin2 * sin2;
        const float t4 = t2 * sin2;
        const float rp = rs * (t3 - t4) / (t3 + t4);
        return 0.5f * (rp + rs);
}

// ---- MicrofacetReflection with a conductor Fresnel term (Bsdf/MicrofacetReflection.swift)
struct BCond {
        BTR d;
        V3 R, eta, k;
        __device__ __noinline__ V3 f(V3 wo, V3 wi) const {
                const float co = fabsf(wo.z), ci = fabsf(wi.z);
                V3 h = wo + wi;
                if (co == 0.0f || ci == 0.0f) return v3(0, 0, 0);
                if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return v3(0, 0, 0);
                h = b_norm0(h);
                const float cf = fabsf(dot(wi, h));
                const float area = d.D(h);
                const float vis = d.G(wo, wi);
                const float den = 4.0f * ci * co;
                return v3(R.x * area * vis * b_fresnel_conductor(cf, eta.x, k.x) / den,
                          R.y * area * vis * b_fresnel_conductor(cf, eta.y, k.y) / den,
                          R.z * area * vis * b_fresnel_conductor(cf, eta.z, k.z) / den);
        }
        __device__ float pdf(V3 wo, V3 wi) const {
                if (!b_same(wo, wi)) return 0.0f;
                const V3 h = b_norm0(wo + wi);
                return d.pdf(wo, h) / (4.0f * dot(wo, h));
        }
        __device__ __noinline__ BsdfS sample(V3 wo, float u0, float u1) const {
                if (wo.z == 0.0f) return bs_none();
                const V3 h = d.sample_wh(wo, u0, u1);
                const V3 wi = neg(wo) + h * (2.0f * dot(wo, h));
                return BsdfS{f(wo, wi), wi, pdf(wo, wi)};
        }
};

__device__ __forceinline__ float b_tr(float dz, V3 w) {
        if (fabsf(dz) < 1.17549435e-38f) return 1.0f;
        return expf(-fabsf(dz / w.z));
}
__device__ __forceinline__ float b_max3(V3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
__device__ __forceinline__ float b_ph(float f, float g) {
        return (f == 0.0f || g == 0.0f) ? 0.0f : (f * f) / (f * f + g * g);
}

// ---- LayeredBsdf<Dielectric, Bottom>, clear layer, two-sided: coated
// diffuse (Bottom = BDiff) and coated conductor (Bottom = BCond)
template <class Bottom>
struct BLayered {
        BDiel top;
        Bottom bottom;
        float thickness;
        int max_depth, nsamples;

        __device__ __noinline__ V3 f(V3 wo, V3 wi) const {
                V3 res = v3(0, 0, 0);
                if (wo.z < 0.0f) {
                        wo = neg(wo);
                        wi = neg(wi);
                }
                const bool same = b_same(wo, wi);
                const float exit_z = same ? thickness : 0.0f;
                if (same) {
                        const float ft = top.f(wo, wi) * (float)nsamples;
                        res = v3(ft, ft, ft);
                }
                BRng rng = b_rng(wo, wi, 1u);
                for (int s = 0; s < nsamples; ++s) {
                        const float a0 = rng.get1d(), a1 = rng.get1d(), a2 = rng.get1d();
                        const BsdfS wos = top.sample(wo, a0, a1, a2, true);
                        if (!wos.valid() || b_same(wos.wi, wo) || wos.wi.z == 0.0f) continue;
                        const float c0 = rng.get1d(), c1 = rng.get1d(), c2 = rng.get1d();
                        const BsdfS wis = same ? top.sample(wi, c0, c1, c2, false) : bottom.sample(wi, c0, c1);
                        if (!wis.valid() || b_same(wis.wi, wi) || wis.wi.z == 0.0f) continue;
                        V3 beta = v3(wos.f.x * fabsf(wos.wi.z) / wos.pdf, wos.f.y * fabsf(wos.wi.z) / wos.pdf,
                                  wos.f.z * fabsf(wos.wi.z) / wos.pdf);
                        float z = thickness;
                        V3 w = wos.wi;
                        for (int depth = 0; depth < max_depth; ++depth) {
                                if (depth > 3 && b_max3(beta) < 0.25f) {
                                        const float q = fmaxf(0.0f, 1.0f - b_max3(beta));
                                        if (rng.get1d() < q) break;
                                        beta = v3(beta.x / (1.0f - q), beta.y / (1.0f - q), beta.z / (1.0f - q));
                                }
                                z = z == thickness ? 0.0f : thickness;
                                beta = beta * b_tr(thickness, w);
                                if (z == exit_z) {
                                        const float e0 = rng.get1d(), e1 = rng.get1d(), e2 = rng.get1d();
                                        const BsdfS bs = z == 0.0f ? bottom.sample(neg(w), e0, e1)
                                                                   : top.sample(neg(w), e0, e1, e2, true);
                                        if (!bs.valid() || bs.pdf == 0.0f || bs.wi.z == 0.0f) break;
                                        if (!b_same(bs.wi, neg(w))) break;
                                        beta = v3(beta.x * bs.f.x * fabsf(bs.wi.z) / bs.pdf,
                                                  beta.y * bs.f.y * fabsf(bs.wi.z) / bs.pdf,
                                                  beta.z * bs.f.z * fabsf(bs.wi.z) / bs.pdf);
                                        w = bs.wi;
                                } else {
                                        V3 ne;
                                        float ne_pdf;
                                        if (z == 0.0f) {
                                                ne = bottom.f(neg(w), neg(wis.wi));
                                                ne_pdf = bottom.pdf(neg(w), neg(wis.wi));
                                        } else {
                                                const float ft = top.f(neg(w), neg(wis.wi));
                                                ne = v3(ft, ft, ft);
                                                ne_pdf = top.pdf(neg(w), neg(wis.wi));
                                        }
                                        const float wt = b_ph(wis.pdf, ne_pdf);
                                        const float trw = b_tr(thickness, wis.wi);
                                        res = res + v3(beta.x * ne.x * fabsf(wis.wi.z) * wt * trw * wis.f.x / wis.pdf,
                                                       beta.y * ne.y * fabsf(wis.wi.z) * wt * trw * wis.f.y / wis.pdf,
                                                       beta.z * ne.z * fabsf(wis.wi.z) * wt * trw * wis.f.z / wis.pdf);
                                        const float e0 = rng.get1d(), e1 = rng.get1d(), e2 = rng.get1d();
                                        const BsdfS bs = z == 0.0f ? bottom.sample(neg(w), e0, e1)
                                                                   : top.sample(neg(w), e0, e1, e2, true);
                                        if (!bs.valid() || bs.pdf == 0.0f || bs.wi.z == 0.0f) break;
                                        if (!b_same(bs.wi, neg(w))) break;
                                        beta = v3(beta.x * bs.f.x * fabsf(bs.wi.z) / bs.pdf,
                                                  beta.y * bs.f.y * fabsf(bs.wi.z) / bs.pdf,
                                                  beta.z * bs.f.z * fabsf(bs.wi.z) / bs.pdf);
                                        w = bs.wi;
                                        V3 fe;
                                        float fe_pdf;
                                        if (exit_z == 0.0f) {
                                                fe = bottom.f(neg(w), wi);
                                                fe_pdf = bottom.pdf(neg(w), wi);
                                        } else {
                                                const float ft = top.f(neg(w), wi);
                                                fe = v3(ft, ft, ft);
                                                fe_pdf = top.pdf(neg(w), wi);
                                        }
                                        if (!is_black(fe)) {
                                                const float we = b_ph(bs.pdf, fe_pdf);
                                                const float tre = b_tr(thickness, bs.wi);
                                                res = res + v3(beta.x * tre * fe.x * we, beta.y * tre * fe.y * we,
                                                               beta.z * tre * fe.z * we);
                                        }
                                }
                        }
                }
                return v3(res.x / (float)nsamples, res.y / (float)nsamples, res.z / (float)nsamples);
        }

        // As written, the walk ends after its first interface sample (the
        // transmission test runs after the walk direction was replaced).
        __device__ __noinline__ BsdfS sample(V3 wo, float u0, float u1, float u2) const {
                bool flip = false;
                if (wo.z < 0.0f) {
                        wo = neg(wo);
                        flip = true;
                }
                const BsdfS st = top.sample(wo, u0, u1, u2, true);
                if (!st.valid() || st.pdf == 0.0f || st.wi.z == 0.0f) return bs_none();
                if (b_same(st.wi, wo)) {
                        BsdfS r = st;
                        if (flip) r.wi = neg(r.wi);
                        return r;
                }
                V3 w = st.wi;
                BRng rng = b_rng(wo, v3(u0, u1, u2), 2u);
                V3 f = st.f * fabsf(w.z);
                float pdf = st.pdf;
                float z = thickness;
                for (int depth = 0; depth < max_depth; ++depth) {
                        const float rr = b_max3(f) / pdf;
                        if (depth > 3 && rr < 0.25f) {
                                const float q = fmaxf(0.0f, 1.0f - rr);
                                if (rng.get1d() < q) return bs_none();
                                pdf = pdf * (1.0f - q);
                        }
                        if (w.z == 0.0f) return bs_none();
                        z = z == thickness ? 0.0f : thickness;
                        const float c0 = rng.get1d(), c1 = rng.get1d(), c2 = rng.get1d();
                        const BsdfS bs = z == 0.0f ? bottom.sample(neg(w), c0, c1) : top.sample(neg(w), c0, c1, c2, true);
                        if (!bs.valid() || bs.pdf == 0.0f || bs.wi.z == 0.0f) return bs_none();
                        f = mulv(f, bs.f);
                        pdf = pdf * bs.pdf;
                        w = bs.wi;
                        if (!b_same(bs.wi, neg(w))) return BsdfS{f, flip ? neg(w) : w, pdf};
                        f = f * fabsf(bs.wi.z);
                }
                return bs_none();
        }

        __device__ __noinline__ float pdf(V3 wo, V3 wi) const {
                if (wo.z < 0.0f) {
                        wo = neg(wo);
                        wi = neg(wi);
                }
                BRng rng = b_rng(wo, wi, 3u);
                float sum = 0.0f;
                const bool same = b_same(wo, wi);
                if (same) sum = sum + (float)nsamples * top.pdf(wo, wi);
                for (int s = 0; s < nsamples; ++s) {
                        if (same) {
                                const float a0 = rng.get1d(), a1 = rng.get1d(), a2 = rng.get1d();
                                const BsdfS wos = top.sample(wo, a0, a1, a2, true);
                                const float b0 = rng.get1d(), b1 = rng.get1d(), b2 = rng.get1d();
                                const BsdfS wis = top.sample(wi, b0, b1, b2, true);
                                if (wos.valid() && !b_same(wos.wi, wo) && wis.valid() && !b_same(wis.wi, wi)) {
                                        const float c0 = rng.get1d(), c1 = rng.get1d();
                                        rng.get1d();
                                        const BsdfS rs = bottom.sample(neg(wos.wi), c0, c1);
                                        if (rs.valid() && rs.pdf > 0.0f) {
                                                const float rp = bottom.pdf(neg(wos.wi), neg(wis.wi));
                                                sum = sum + b_ph(wis.pdf, rp) * rp;
                                                const float tp = top.pdf(neg(rs.wi), wi);
                                                sum = sum + b_ph(rs.pdf, tp) * tp;
                                        }
                                }
                        } else {
                                const float a0 = rng.get1d(), a1 = rng.get1d(), a2 = rng.get1d();
                                const BsdfS wos = top.sample(wo, a0, a1, a2, true);
                                const float b0 = rng.get1d(), b1 = rng.get1d();
                                rng.get1d();
                                const BsdfS wis = bottom.sample(wi, b0, b1);
                                if (wos.valid() && !b_same(wos.wi, wo) && wis.valid() && !b_same(wis.wi, wi)) {
                                        const float p1 = top.pdf(wo, neg(wis.wi));
                                        const float p2 = bottom.pdf(neg(wos.wi), wi);
                                        sum = sum + (p1 + p2) / 2.0f;
                                }
                        }
                }
                return (1.0f - 0.9f) * (1.0f / (4.0f * kPi)) + 0.9f * (sum / (float)nsamples);
        }
};

// A material's BSDF: type 3 dielectric, 4 coated diffuse, 5 conductor, 6
// coated conductor; p = the material's 3 parameter records (eta, roughness
// u, v, thickness; conductor eta, roughness u; conductor k, roughness v).
// Dielectric and coating roughness is remapped to alpha = sqrt (a coating's
// alpha at least 0.001); a conductor's roughness is its alpha (at least
// 1e-3), a coated conductor's is remapped (at least 0.001)
// (Material/Dielectric.swift:3-14, Material/CoatedDiffuse.swift:23-58,
// Material/Conductor.swift:3-22, Material/CoatedConductor.swift:35-88).
struct BMat {
        BDiel diel;
        BLayered<BDiff> coated;
        BCond cond;
        BLayered<BCond> coated_cond;
};

template <int K>
__device__ BMat make_bmat(V3 R, float4 p0, float4 p1, float4 p2) {
        BMat m;
        float ax = sqrtf(p0.y), ay = sqrtf(p0.z);
        if (K == 4 || K == 6) {
                ax = fmaxf(ax, 0.001f);
                ay = fmaxf(ay, 0.001f);
        }
        m.diel.d.ax = ax;
        m.diel.d.ay = ay;
        m.diel.eta = p0.x;
        const float thick = fmaxf(p0.w, 1.17549435e-38f);
        if (K == 4) {
                m.coated.top = m.diel;
                m.coated.bottom.R = R;
                m.coated.thickness = thick;
                m.coated.max_depth = 10;
                m.coated.nsamples = 1;
        }
        if (K == 5 || K == 6) {
                if (K == 6) {
                        m.cond.d.ax = fmaxf(sqrtf(p1.w), 0.001f);
                        m.cond.d.ay = fmaxf(sqrtf(p2.w), 0.001f);
                        m.cond.R = R;
                } else {
                        m.cond.d.ax = fmaxf(p1.w, 1e-3f);
                        m.cond.d.ay = fmaxf(p2.w, 1e-3f);
                        m.cond.R = v3(1.0f, 1.0f, 1.0f);
                }
                m.cond.eta = v3(p1.x, p1.y, p1.z);
                m.cond.k = v3(p2.x, p2.y, p2.z);
        }
        if (K == 6) {
                m.coated_cond.top = m.diel;
                m.coated_cond.bottom = m.cond;
                m.coated_cond.thickness = thick;
                m.coated_cond.max_depth = 10;
                m.coated_cond.nsamples = 1;
        }
        return m;
}

// Kind-specific dispatch (K = material type).
template <int K>
__device__ __forceinline__ V3 bmat_f(const BMat &m, V3 wo, V3 wi) {
        if (K == 3) {
                const float f = m.diel.f(wo, wi);
                return v3(f, f, f);
        }
        if (K == 4) return m.coated.f(wo, wi);
        if (K == 5) return m.cond.f(wo, wi);
        return m.coated_cond.f(wo, wi);
}
template <int K>
__device__ __forceinline__ float bmat_pdf(const BMat &m, V3 wo, V3 wi) {
        if (K == 3) return m.diel.pdf(wo, wi);
        if (K == 4) return m.coated.pdf(wo, wi);
        if (K == 5) return m.cond.pdf(wo, wi);
        return m.coated_cond.pdf(wo, wi);
}
template <int K>
__device__ __forceinline__ BsdfS bmat_sample(const BMat &m, V3 wo, float u0, float u1, float u2) {
        if (K == 3) return m.diel.sample(wo, u0, u1, u2, true);
        if (K == 4) return m.coated.sample(wo, u0, u1, u2);
        if (K == 5) return m.cond.sample(wo, u0, u1);
        return m.coated_cond.sample(wo, u0, u1, u2);
}
template <int K>
__device__ __forceinline__ bool bmat_specular(const BMat &m) {
        return K == 3 && m.diel.specular();
}
