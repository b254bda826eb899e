// film.cu - the film's last steps: normalising the device film sums into an
// image (Image.normalize / Pixel.normalized, Core/Pixel.swift:12-16) and
// writing images as OpenEXR files (the role of Image/OpenImageIOWriter.swift:
// RGBA 32-bit float, alpha 1).
//
// The writer emits the OpenEXR 2.0 single-part scanline layout without
// compression: magic and version, the required header attributes (channels,
// compression, dataWindow, displayWindow, lineOrder, pixelAspectRatio,
// screenWindowCenter, screenWindowWidth), the line offset table, then one
// chunk per scanline (y, byte count, the channels in name order: A, B, G, R).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gzg_internal.h"

namespace gzg {
namespace {

// A pixel's light / weight; black stays black; a weight of zero under
// non-black light (the reference throws PixelError.zeroWeight) gives black and
// is counted.
__global__ void k_resolve(const float *__restrict__ sums, const float *__restrict__ w, int64_t n,
                          float *__restrict__ out, unsigned long long *__restrict__ zero_weight) {
        const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (p >= n) return;
        const float r = sums[3 * p], g = sums[3 * p + 1], b = sums[3 * p + 2];
        const float wt = w[p];
        float o[3] = {r, g, b};
        if (!(r == 0.0f && g == 0.0f && b == 0.0f)) {
                if (wt == 0.0f) {
                        o[0] = o[1] = o[2] = 0.0f;
                        if (zero_weight) atomicAdd(zero_weight, 1ull);
                } else {
                        o[0] = r / wt;
                        o[1] = g / wt;
                        o[2] = b / wt;
                }
        }
        out[3 * p] = o[0];
        out[3 * p + 1] = o[1];
        out[3 * p + 2] = o[2];
}

void put_u32(std::vector<uint8_t> &b, uint32_t v) {
        for (int i = 0; i < 4; ++i) b.push_back((uint8_t)(v >> (8 * i)));
}
void put_u64(std::vector<uint8_t> &b, uint64_t v) {
        for (int i = 0; i < 8; ++i) b.push_back((uint8_t)(v >> (8 * i)));
}
void put_f32(std::vector<uint8_t> &b, float f) {
        uint32_t v;
        std::memcpy(&v, &f, 4);
        put_u32(b, v);
}
void put_str(std::vector<uint8_t> &b, const char *s) {
        b.insert(b.end(), s, s + std::strlen(s) + 1);
}
void attr(std::vector<uint8_t> &b, const char *name, const char *type, const std::vector<uint8_t> &value) {
        put_str(b, name);
        put_str(b, type);
        put_u32(b, (uint32_t)value.size());
        b.insert(b.end(), value.begin(), value.end());
}

}  // namespace
}  // namespace gzg

using namespace gzg;

GZG_API gzg_status gzg_film_resolve_device(const float *film_rgb, const float *film_w, int64_t pixels, float *image,
                                           unsigned long long *zero_weight_count, void *stream) {
        if (pixels < 0 || (pixels > 0 && (!film_rgb || !film_w || !image)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_film_resolve_device: bad arguments");
        if (pixels == 0) return clear_error();
        const int B = 256;
        k_resolve<<<(unsigned)((pixels + B - 1) / B), B, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
            film_rgb, film_w, pixels, image, zero_weight_count);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
                return set_error(GZG_ERR_CUDA, std::string("gzg_film_resolve_device: ") + cudaGetErrorString(e));
        return clear_error();
}

GZG_API gzg_status gzg_write_exr(const char *path, const float *pixels, int32_t width, int32_t height,
                                 int32_t channels) {
        // a scanline's byte count is a 32-bit field: width x 4 channels x 4 bytes
        if (!path || !pixels || width <= 0 || height <= 0 || (channels != 3 && channels != 4) ||
            (int64_t)width * height > ((int64_t)1 << 31) || (int64_t)width * 16 > (int64_t)UINT32_MAX)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_write_exr: bad arguments");
        std::vector<uint8_t> h;
        put_u32(h, 20000630u);  // magic 0x762f3101
        put_u32(h, 2u);         // version 2, single-part scanline
        {
                std::vector<uint8_t> v;
                for (const char *c : {"A", "B", "G", "R"}) {
                        put_str(v, c);
                        put_u32(v, 2u);  // FLOAT
                        v.push_back(0);  // pLinear
                        v.push_back(0);
                        v.push_back(0);
                        v.push_back(0);  // reserved
                        put_u32(v, 1u);  // x sampling
                        put_u32(v, 1u);  // y sampling
                }
                v.push_back(0);
                attr(h, "channels", "chlist", v);
        }
        attr(h, "compression", "compression", {0});
        {
                std::vector<uint8_t> v;
                put_u32(v, 0u);
                put_u32(v, 0u);
                put_u32(v, (uint32_t)(width - 1));
                put_u32(v, (uint32_t)(height - 1));
                attr(h, "dataWindow", "box2i", v);
                attr(h, "displayWindow", "box2i", v);
        }
        attr(h, "lineOrder", "lineOrder", {0});
        {
                std::vector<uint8_t> v;
                put_f32(v, 1.0f);
                attr(h, "pixelAspectRatio", "float", v);
        }
        {
                std::vector<uint8_t> v;
                put_f32(v, 0.0f);
                put_f32(v, 0.0f);
                attr(h, "screenWindowCenter", "v2f", v);
        }
        {
                std::vector<uint8_t> v;
                put_f32(v, 1.0f);
                attr(h, "screenWindowWidth", "float", v);
        }
        h.push_back(0);  // end of header
        const uint64_t line_bytes = 8 + (uint64_t)width * 4 * 4;
        const uint64_t table_end = h.size() + 8 * (uint64_t)height;
        for (int32_t y = 0; y < height; ++y) put_u64(h, table_end + (uint64_t)y * line_bytes);
        std::FILE *f = std::fopen(path, "wb");
        if (!f) return set_error(GZG_ERR_INVALID_ARGUMENT, std::string("gzg_write_exr: cannot open ") + path);
        bool ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
        std::vector<uint8_t> line;
        line.reserve((size_t)line_bytes);
        for (int32_t y = 0; ok && y < height; ++y) {
                line.clear();
                put_u32(line, (uint32_t)y);
                put_u32(line, (uint32_t)((int64_t)width * 16));
                const float *row = pixels + (size_t)y * width * channels;
                for (int c : {3, 2, 1, 0})  // A, B, G, R
                        for (int32_t x = 0; x < width; ++x)
                                put_f32(line, c == 3 && channels == 3 ? 1.0f : row[(size_t)x * channels + c]);
                ok = std::fwrite(line.data(), 1, line.size(), f) == line.size();
        }
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) return set_error(GZG_ERR_INVALID_ARGUMENT, std::string("gzg_write_exr: write failed for ") + path);
        return clear_error();
}
