// sobol.cuh - Z-Sobol sampler on the device (Sources/libgonzales/Sampler/
// ZSobolSampler.swift:6-280).  The integer path (Morton index, base-4 digit
// permutation, matrix product, Owen scramble) is bit-exact with the
// reference; the final value is (float)bits * 2^-32 clamped to 1 - 1e-6.
#pragma once

#include <stdint.h>

namespace gzg {

constexpr int kSobolDims = 1024;
constexpr int kSobolColumns = 52;

struct ZSobol {
        uint64_t morton;  // (Morton(px, py) << log2spp) | sample index
        int32_t dim;      // next dimension
};

struct ZSobolConfig {
        const uint32_t *matrices;  // kSobolDims x kSobolColumns
        uint64_t seed;             // sampler seed (1234, Sampler/Random.swift:66)
        int32_t log2spp;
        int32_t n_base4_digits;
};

__device__ __forceinline__ uint32_t zs_reverse_bits(uint32_t v) { return __brev(v); }

// mixBits (ZSobolSampler.swift:90-101): the 64-bit argument folded to 32
// bits by xor, then the 32-bit finaliser.
__device__ __forceinline__ uint32_t zs_mix_bits32(uint32_t x) {
        x ^= x >> 16;
        x *= 0x85ebca77u;
        x ^= x >> 13;
        x *= 0xc2b2ae35u;
        x ^= x >> 16;
        return x;
}
__device__ __forceinline__ uint32_t zs_mix_bits(uint64_t v) {
        return zs_mix_bits32((uint32_t)(v & 0xFFFFFFFFull) ^ (uint32_t)(v >> 32));
}

// FastOwenScrambler (ZSobolSampler.swift:43-67).
__device__ __forceinline__ uint32_t zs_owen(uint32_t v, uint32_t seed) {
        v = __brev(v);
        v ^= v * 0x3d20adeau;
        v += seed;
        v *= (seed >> 16) | 1u;
        v ^= v * 0x05526c56u;
        v ^= v * 0x53a22864u;
        return __brev(v);
}

// encodeMorton2 (ZSobolSampler.swift:70-88).
__device__ __forceinline__ uint64_t zs_morton2(uint32_t x, uint32_t y) {
        uint64_t a = x, b = y;
        a = (a | (a << 16)) & 0x0000FFFF0000FFFFull;
        a = (a | (a << 8)) & 0x00FF00FF00FF00FFull;
        a = (a | (a << 4)) & 0x0F0F0F0F0F0F0F0Full;
        a = (a | (a << 2)) & 0x3333333333333333ull;
        a = (a | (a << 1)) & 0x5555555555555555ull;
        b = (b | (b << 16)) & 0x0000FFFF0000FFFFull;
        b = (b | (b << 8)) & 0x00FF00FF00FF00FFull;
        b = (b | (b << 4)) & 0x0F0F0F0F0F0F0F0Full;
        b = (b | (b << 2)) & 0x3333333333333333ull;
        b = (b | (b << 1)) & 0x5555555555555555ull;
        return a | (b << 1);
}

__device__ __forceinline__ uint64_t zs_shr(uint64_t v, int s) { return s >= 64 ? 0ull : (v >> s); }

// The 24 permutations of ZSobolSampler.swift:105-112 packed two bits per
// entry, one byte per permutation, eight bytes per word (byte p & 7 of word
// p >> 3): perm[p][d] = (byte p >> (2 * d)) & 3.  Selected from registers
// rather than read from a local-memory array (box-scene frame 1.429 -> 1.407 ms).
__device__ __forceinline__ int zs_perm(int p, int digit) {
        const uint64_t word = p < 8 ? 0xB1E19C6C78D8B4E4ull : (p < 16 ? 0x72D236C68D2D39C9ull : 0x93634B1B87271E4Eull);
        const uint32_t entry = (uint32_t)(word >> (8 * (p & 7))) & 0xFFu;
        return (int)((entry >> (2 * digit)) & 3u);
}

__device__ __forceinline__ uint32_t zs_shr32(uint32_t v, int s) { return s >= 32 ? 0u : (v >> s); }

// getSampleIndex when the Morton index (pixel Morton code << log2 spp |
// sample) is below 2^32 and has at most 16 base-4 digits, as for 2048 x 2048
// pixels at up to 1024 spp: the same bits as the 64-bit form in 32-bit
// arithmetic.  mixBits folds its argument to 32 bits by xor, so for
// higher < 2^32, mixBits(higher ^ dim x 0x55555555) is
// mixBits32(higher ^ fold(dim x 0x55555555)).
__device__ __forceinline__ uint32_t zs_sample_index32(const ZSobolConfig &c, uint32_t morton, int dim) {
        const uint64_t dmul = 0x55555555ull * (uint64_t)(int64_t)dim;
        const uint32_t dfold = (uint32_t)(dmul & 0xFFFFFFFFull) ^ (uint32_t)(dmul >> 32);
        uint32_t idx = 0;
        const bool pow2 = (c.log2spp & 1) == 1;
        const int last = pow2 ? 1 : 0;
        for (int di = c.n_base4_digits - 1; di >= last; --di) {
                const int shift = 2 * di - (pow2 ? 1 : 0);
                const int digit = (int)(zs_shr32(morton, shift) & 3u);
                const uint32_t h = zs_mix_bits32(zs_shr32(morton, shift + 2) ^ dfold);
                idx |= (uint32_t)zs_perm((int)((h >> 24) % 24u), digit) << shift;
        }
        if (pow2) {
                int digit = (int)(morton & 1u);
                const uint32_t h = zs_mix_bits32((morton >> 1) ^ dfold);
                digit ^= (int)(h & 1u);
                idx |= (uint32_t)digit;
        }
        return idx;
}

// getSampleIndex (ZSobolSampler.swift:138-166).
__device__ __forceinline__ uint64_t zs_sample_index(const ZSobolConfig &c, const ZSobol &s) {
        if ((s.morton >> 32) == 0 && c.n_base4_digits <= 16) return zs_sample_index32(c, (uint32_t)s.morton, s.dim);
        uint64_t idx = 0;
        const bool pow2 = (c.log2spp & 1) == 1;
        const int last = pow2 ? 1 : 0;
        const uint64_t dmul = 0x55555555ull * (uint64_t)(int64_t)s.dim;
        for (int di = c.n_base4_digits - 1; di >= last; --di) {
                const int shift = 2 * di - (pow2 ? 1 : 0);
                const int digit = (int)(zs_shr(s.morton, shift) & 3u);
                const uint64_t higher = zs_shr(s.morton, shift + 2);
                const uint32_t h = zs_mix_bits(higher ^ dmul);
                idx |= (uint64_t)zs_perm((int)((h >> 24) % 24u), digit) << shift;
        }
        if (pow2) {
                int digit = (int)(s.morton & 1u);
                const uint32_t h = zs_mix_bits((s.morton >> 1) ^ dmul);
                digit ^= (int)(h & 1u);
                idx |= (uint64_t)digit;
        }
        return idx;
}

// sobolSample (ZSobolSampler.swift:6-31) of N consecutive dimensions d0.. for
// one index: the XOR of the matrix columns of the index's set bits, in one
// scan of those bits (the N columns of a bit are independent loads).
template <int N>
__device__ __forceinline__ void zs_sobol_bits(const ZSobolConfig &c, uint64_t index, int d0, uint32_t acc[N]) {
        const uint32_t *m = c.matrices + (size_t)d0 * kSobolColumns;
#pragma unroll
        for (int k = 0; k < N; ++k) acc[k] = 0u;
        if ((index >> 32) == 0) {
                uint32_t cur = (uint32_t)index;
                while (cur != 0u) {
                        const int bit = __ffs(cur) - 1;
#pragma unroll
                        for (int k = 0; k < N; ++k) acc[k] ^= __ldg(m + k * kSobolColumns + bit);
                        cur &= cur - 1u;
                }
        } else {
                uint64_t cur = index;
                while (cur != 0) {
                        const int bit = __ffsll((long long)cur) - 1;
                        if (bit >= kSobolColumns) break;
#pragma unroll
                        for (int k = 0; k < N; ++k) acc[k] ^= __ldg(m + k * kSobolColumns + bit);
                        cur &= cur - 1;
                }
        }
}

// Owen scramble, times 2^-32, clamped below 1 (the tail of sobolSample).
__device__ __forceinline__ float zs_finish(uint32_t acc, uint32_t scramble) {
        const uint32_t r = zs_owen(acc, scramble);
        const float f = __fmul_rn(__uint2float_rn(r), 2.32830643653869628906e-10f);
        const float one_minus_eps = 1.0f - 1e-6f;
        return one_minus_eps < f ? one_minus_eps : f;
}

// getSampleHash (ZSobolSampler.swift:188-199); the second hash is 0 because
// mixBits returns 32 bits.
__device__ __forceinline__ uint32_t zs_hash(const ZSobolConfig &c, int dim) {
        return zs_mix_bits((uint64_t)(int64_t)dim ^ c.seed);
}

// startPixelSample (ZSobolSampler.swift:130-136).
__device__ __forceinline__ void zs_start(const ZSobolConfig &c, ZSobol &s, uint32_t px, uint32_t py, uint32_t index) {
        s.dim = 0;
        s.morton = (zs_morton2(px, py) << c.log2spp) | (uint64_t)index;
}

// get1D (ZSobolSampler.swift:203-219).
__device__ __forceinline__ float zs_get1d(const ZSobolConfig &c, ZSobol &s) {
        const uint64_t idx = zs_sample_index(c, s);
        const uint32_t h = zs_hash(c, s.dim);
        if (s.dim >= kSobolDims) s.dim = 2;
        s.dim += 1;
        uint32_t acc[1];
        zs_sobol_bits<1>(c, idx, s.dim - 1, acc);
        return zs_finish(acc[0], h);
}

// get2D (ZSobolSampler.swift:221-244).
__device__ __forceinline__ void zs_get2d(const ZSobolConfig &c, ZSobol &s, float &a, float &b) {
        const uint64_t idx = zs_sample_index(c, s);
        const uint32_t h0 = zs_hash(c, s.dim);
        if (s.dim + 1 >= kSobolDims) s.dim = 2;
        s.dim += 2;
        uint32_t acc[2];
        zs_sobol_bits<2>(c, idx, s.dim - 2, acc);
        a = zs_finish(acc[0], h0);
        b = zs_finish(acc[1], 0u);
}

// get3D (ZSobolSampler.swift:249-280).
__device__ __forceinline__ void zs_get3d(const ZSobolConfig &c, ZSobol &s, float &a, float &b, float &d) {
        const uint64_t idx = zs_sample_index(c, s);
        const uint32_t h0 = zs_hash(c, s.dim);
        const uint32_t h2 = zs_hash(c, s.dim + 2);
        if (s.dim + 2 >= kSobolDims) s.dim = 2;
        s.dim += 3;
        uint32_t acc[3];
        zs_sobol_bits<3>(c, idx, s.dim - 3, acc);
        a = zs_finish(acc[0], h0);
        b = zs_finish(acc[1], 0u);
        d = zs_finish(acc[2], h2);
}

}  // namespace gzg
