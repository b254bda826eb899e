// env.cpp - host side of the environment light: the bilinear map lookup and
// the 1024 x 1024 piecewise-constant sampling distribution of
// Light/InfiniteLight.swift:9-36 (PiecewiseConstant1D/2D,
// Core/Distribution1D.swift:1-79, Core/Distribution2D.swift:1-39).  The
// distribution is built from the map's green channel, as the reference's
// `color.y` is (Core/Spectrum.swift:246-254).
#include <algorithm>
#include <cmath>

#include "gzg_internal.h"

namespace gzg {

void env_lookup_host(const float *rgb, int w, int h, float u, float v, float *out) {
        const float x = u * (float)w - 0.5f, y = v * (float)h - 0.5f;
        const float fx = std::floor(x), fy = std::floor(y);
        const float ax = x - fx, ay = y - fy;
        const int x0 = std::min(std::max((int)fx, 0), w - 1), x1 = std::min(std::max((int)fx + 1, 0), w - 1);
        const int y0 = std::min(std::max((int)fy, 0), h - 1), y1 = std::min(std::max((int)fy + 1, 0), h - 1);
        for (int c = 0; c < 3; ++c) {
                const float a = rgb[((size_t)y0 * w + x0) * 3 + c], b = rgb[((size_t)y0 * w + x1) * 3 + c];
                const float d = rgb[((size_t)y1 * w + x0) * 3 + c], e = rgb[((size_t)y1 * w + x1) * 3 + c];
                const float top = a + (b - a) * ax;
                const float bot = d + (e - d) * ax;
                out[c] = top + (bot - top) * ay;
        }
}

namespace {

// One PiecewiseConstant1D: cdf (n + 1 entries, normalised) and integral.
float build_1d(const float *f, int n, float *cdf) {
        cdf[0] = 0.0f;
        for (int i = 1; i <= n; ++i) cdf[i] = cdf[i - 1] + f[i - 1] / (float)n;
        const float integral = cdf[n];
        for (int i = 1; i <= n; ++i) cdf[i] = integral == 0.0f ? (float)i / (float)n : cdf[i] / integral;
        return integral;
}

}  // namespace

void build_env_tables(const float *rgb, int w, int h, EnvTables *t) {
        const int N = kEnvDistSize;
        t->func.resize((size_t)N * N);
        t->cdf.resize((size_t)N * (N + 1));
        t->row_integral.resize(N);
        t->marg_func.resize(N);
        t->marg_cdf.resize(N + 1);
        for (int row = 0; row < N; ++row)
                for (int col = 0; col < N; ++col) {
                        float c[3];
                        env_lookup_host(rgb, w, h, ((float)col + 0.5f) / (float)N, ((float)row + 0.5f) / (float)N, c);
                        t->func[(size_t)row * N + col] = c[1];
                }
        for (int row = 0; row < N; ++row) {
                t->row_integral[row] = build_1d(&t->func[(size_t)row * N], N, &t->cdf[(size_t)row * (N + 1)]);
                t->marg_func[row] = t->row_integral[row];
        }
        t->marg_integral = build_1d(t->marg_func.data(), N, t->marg_cdf.data());
}

}  // namespace gzg
