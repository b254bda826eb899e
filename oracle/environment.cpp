// environment.cpp - CPU restatement of Gonzales' infinite (environment) light
// (test infrastructure: checker and CPU baseline).  -ffp-contract=off.
//
// Restated from (paths relative to Sources/libgonzales):
//   InfiniteLight init / sample / pdf / radiance   Light/InfiniteLight.swift:7-160
//   equal-area square <-> sphere                   Light/InfiniteLight.swift:85-135
//   PiecewiseConstant1D                            Core/Distribution1D.swift:1-79
//   PiecewiseConstant2D                            Core/Distribution2D.swift:1-39
//
// The reference builds the sampling distribution from the green channel of
// the map (`color.y` of an RgbSpectrum is its green component,
// Core/Spectrum.swift:246-254), at 1024 x 1024 points.  Its image lookup goes
// through OpenImageIO's texture system (third party, not restated); here the
// map is read with a plain bilinear lookup, clamped at the edges, the same
// on the device.  The light's `scale` enters only its power (light choice),
// as in the reference (`sample` and `radianceFromInfinity` return the map).
#include <algorithm>
#include <cmath>
#include <vector>

#include "oracle.h"

namespace {

const float kPi = 3.14159265358979323846f;

struct Dist1D {
        std::vector<float> func, cdf;
        float integral = 0.0f;
        int count = 0;

        void init(const float *values, int n) {
                count = n;
                func.assign(values, values + n);
                cdf.assign((size_t)n + 1, 0.0f);
                for (int i = 1; i <= n; ++i) cdf[i] = cdf[i - 1] + func[i - 1] / (float)n;
                integral = cdf[n];
                if (integral == 0.0f) {
                        for (int i = 1; i <= n; ++i) cdf[i] = (float)i / (float)n;
                } else {
                        for (int i = 1; i <= n; ++i) cdf[i] = cdf[i] / integral;
                }
        }

        int find_interval(float u) const {
                int lo = 0, hi = count;
                while (lo < hi) {
                        const int mid = lo + (hi - lo) / 2;
                        if (cdf[mid] <= u)
                                lo = mid + 1;
                        else
                                hi = mid;
                }
                return std::min(std::max(lo - 1, 0), count - 1);
        }

        float pdf(float value) const {
                const int o = std::min(std::max((int)(value * (float)count), 0), count - 1);
                return func[o] / integral;
        }

        // sampleContinuous: (value, pdf, offset)
        float sample(float u, float *pdf_out, int *offset) const {
                const int o = find_interval(u);
                float delta = u - cdf[o];
                const float dist = cdf[o + 1] - cdf[o];
                if (dist > 0.0f) delta = delta / dist;
                const float value = ((float)o + delta) / (float)count;
                *pdf_out = pdf(value);
                *offset = o;
                return value;
        }
};

struct Env {
        int w = 0, h = 0;
        std::vector<float> rgb;
        float scale = 1.0f;
        std::vector<Dist1D> rows;
        Dist1D marginal;
};

}  // namespace

// Bilinear lookup of an RGB map at uv in [0,1]^2 (texel centres at
// (i + 0.5) / size, clamped at the edges).
extern "C" void orc_env_lookup(const float *rgb, int32_t w, int32_t h, float u, float v, float *out) {
        const float x = u * (float)w - 0.5f, y = v * (float)h - 0.5f;
        const float fx0 = std::floor(x), fy0 = std::floor(y);
        const float ax = x - fx0, ay = y - fy0;
        int x0 = (int)fx0, y0 = (int)fy0;
        int x1 = x0 + 1, y1 = y0 + 1;
        x0 = std::min(std::max(x0, 0), w - 1);
        x1 = std::min(std::max(x1, 0), w - 1);
        y0 = std::min(std::max(y0, 0), h - 1);
        y1 = std::min(std::max(y1, 0), h - 1);
        for (int c = 0; c < 3; ++c) {
                const float a = rgb[((size_t)y0 * w + x0) * 3 + c], b = rgb[((size_t)y0 * w + x1) * 3 + c];
                const float d = rgb[((size_t)y1 * w + x0) * 3 + c], e = rgb[((size_t)y1 * w + x1) * 3 + c];
                const float top = a + (b - a) * ax;
                const float bot = d + (e - d) * ax;
                out[c] = top + (bot - top) * ay;
        }
}

// equalAreaSquareToSphere (InfiniteLight.swift:118-135).
extern "C" void orc_equal_area_square_to_sphere(float u, float v, float *dir) {
        const float ru = 2.0f * u - 1.0f, rv = 2.0f * v - 1.0f;
        const float au = std::fabs(ru), av = std::fabs(rv);
        const float sd = 1.0f - (au + av);
        const float ad = std::fabs(sd);
        const float r = 1.0f - ad;
        const float phi = (r == 0.0f ? 1.0f : (av - au) / r + 1.0f) * (kPi / 4.0f);
        const float z = std::copysign(std::max(0.0f, 1.0f - r * r), sd);
        const float cp = std::cos(phi), sp = std::sin(phi);
        dir[0] = std::copysign(r * cp, ru);
        dir[1] = std::copysign(r * sp, rv);
        dir[2] = z;
}

// equalAreaSphereToSquare (InfiniteLight.swift:92-116).
extern "C" void orc_equal_area_sphere_to_square(const float *d, float *uv) {
        const float x = std::fabs(d[0]), y = std::fabs(d[1]), z = std::fabs(d[2]);
        const float radius = std::sqrt(std::max(0.0f, 1.0f - z));
        const float a = std::max(x, y);
        float b = std::min(x, y);
        if (a == 0.0f)
                b = 0.0f;
        else
                b = b / a;
        float phi = std::atan(b) * 2.0f / kPi;
        if (x < y) phi = 1.0f - phi;
        float vv = phi * radius;
        float uu = radius - vv;
        if (d[2] < 0.0f) {
                std::swap(uu, vv);
                uu = 1.0f - uu;
                vv = 1.0f - vv;
        }
        uu = std::copysign(uu, d[0]);
        vv = std::copysign(vv, d[1]);
        uv[0] = 0.5f * (uu + 1.0f);
        uv[1] = 0.5f * (vv + 1.0f);
}

// The environment light: map, scale, 1024 x 1024 sampling distribution
// (InfiniteLight.init, InfiniteLight.swift:9-36).
struct orc_env {
        Env e;
};

extern "C" orc_env *orc_env_create(const float *rgb, int32_t w, int32_t h, float scale) {
        if (!rgb || w <= 0 || h <= 0) return nullptr;
        orc_env *env = new orc_env;
        Env &e = env->e;
        e.w = w;
        e.h = h;
        e.rgb.assign(rgb, rgb + (size_t)w * h * 3);
        e.scale = scale;
        const int W = 1024, H = 1024;
        std::vector<float> data((size_t)W * H);
        for (int row = 0; row < H; ++row)
                for (int col = 0; col < W; ++col) {
                        float c[3];
                        orc_env_lookup(rgb, w, h, ((float)col + 0.5f) / (float)W, ((float)row + 0.5f) / (float)H, c);
                        data[(size_t)row * W + col] = c[1];  // color.y: the green channel
                }
        e.rows.resize(H);
        std::vector<float> marg(H);
        for (int row = 0; row < H; ++row) {
                e.rows[row].init(data.data() + (size_t)row * W, W);
                marg[row] = e.rows[row].integral;
        }
        e.marginal.init(marg.data(), H);
        return env;
}

extern "C" void orc_env_destroy(orc_env *env) { delete env; }

// power (InfiniteLight.swift:141-144): pi * (sceneDiameter / 2)^2 * average(brightness).
extern "C" float orc_env_power(const orc_env *env) {
        const float radius = 100.0f / 2.0f;
        const float avg = (env->e.scale + env->e.scale + env->e.scale) / 3.0f;
        return kPi * (radius * radius) * avg;
}

// sample (InfiniteLight.swift:38-64): direction, map value, pdf (0 when the
// map density is 0).
extern "C" float orc_env_sample(const orc_env *env, float u0, float u1, float *dir, float *rgb) {
        const Env &e = env->e;
        float pdf1, pdf0;
        int mo, co;
        const float mv = e.marginal.sample(u1, &pdf1, &mo);
        const float cv = e.rows[mo].sample(u0, &pdf0, &co);
        const float map_pdf = pdf0 * pdf1;
        if (map_pdf == 0.0f) {
                dir[0] = dir[1] = dir[2] = 0.0f;
                rgb[0] = rgb[1] = rgb[2] = 0.0f;
                return 0.0f;
        }
        orc_equal_area_square_to_sphere(cv, mv, dir);
        orc_env_lookup(e.rgb.data(), e.w, e.h, cv, mv, rgb);
        return map_pdf / (4.0f * kPi);
}

// probabilityDensityFor (InfiniteLight.swift:66-76): the direction is not
// normalised before the mapping.
extern "C" float orc_env_pdf(const orc_env *env, const float *dir) {
        const Env &e = env->e;
        float uv[2];
        orc_equal_area_sphere_to_square(dir, uv);
        const int cols = e.rows[0].count, rows = e.marginal.count;
        const int col = std::min(std::max((int)(uv[0] * (float)cols), 0), cols - 1);
        const int row = std::min(std::max((int)(uv[1] * (float)rows), 0), rows - 1);
        return e.rows[row].func[col] / e.marginal.integral / (4.0f * kPi);
}

// radianceFromInfinity (InfiniteLight.swift:137-140): normalised direction.
extern "C" void orc_env_radiance(const orc_env *env, const float *dir, float *rgb) {
        const Env &e = env->e;
        const float l = std::sqrt((dir[0] * dir[0] + dir[1] * dir[1]) + dir[2] * dir[2]);
        float d[3] = {dir[0], dir[1], dir[2]};
        if (l != 0.0f) {
                d[0] = dir[0] / l;
                d[1] = dir[1] / l;
                d[2] = dir[2] / l;
        }
        float uv[2];
        orc_equal_area_sphere_to_square(d, uv);
        orc_env_lookup(e.rgb.data(), e.w, e.h, uv[0], uv[1], rgb);
}

// The distribution's tables: per row the function (1024) and cdf (1025), the
// row integrals, the marginal function, cdf and integral.
extern "C" void orc_env_tables(const orc_env *env, float *func, float *cdf, float *row_integral, float *marg_func,
                               float *marg_cdf, float *marg_integral) {
        const Env &e = env->e;
        for (int r = 0; r < e.marginal.count; ++r) {
                const Dist1D &d = e.rows[r];
                std::copy(d.func.begin(), d.func.end(), func + (size_t)r * d.count);
                std::copy(d.cdf.begin(), d.cdf.end(), cdf + (size_t)r * (d.count + 1));
                row_integral[r] = d.integral;
        }
        std::copy(e.marginal.func.begin(), e.marginal.func.end(), marg_func);
        std::copy(e.marginal.cdf.begin(), e.marginal.cdf.end(), marg_cdf);
        *marg_integral = e.marginal.integral;
}
