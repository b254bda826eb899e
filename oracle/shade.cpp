// shade.cpp - CPU restatement of the reference's live shading step
// shade_core (Sources/mojoKernel/kernel.mojo:676-773) with its PCG32
// (kernel.mojo:99-118).  Test infrastructure only.  -ffp-contract=off.
#include <cmath>

#include "oracle.h"

namespace {

// PCG32 (kernel.mojo:99-118): the constructor reseeds from (initstate, initseq).
struct Pcg32 {
        uint64_t state, inc;
        Pcg32(uint64_t initstate, uint64_t initseq) {
                state = 0;
                inc = (initseq << 1) | 1u;
                next_uint();
                state += initstate;
                next_uint();
        }
        uint32_t next_uint() {
                const uint64_t old = state;
                state = old * 6364136223846793005ull + inc;
                const uint32_t xorshifted = (uint32_t)(((old >> 18) ^ old) >> 27);
                const uint32_t rot = (uint32_t)(old >> 59);
                return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
        }
        float next_float() { return (float)(next_uint() >> 8) * (1.0f / 16777216.0f); }
};

inline void cross3(const float a[3], const float b[3], float r[3]) {
        r[0] = a[1] * b[2] - a[2] * b[1];
        r[1] = a[2] * b[0] - a[0] * b[2];
        r[2] = a[0] * b[1] - a[1] * b[0];
}
inline float dot3(const float a[3], const float b[3]) {
        float s = a[0] * b[0];
        s = s + a[1] * b[1];
        return s + a[2] * b[2];
}

}  // namespace

extern "C" void orc_shade_batch(orc_path_state *paths, int64_t n, const orc_isect *isects, const orc_mesh *meshes,
                                const orc_material *materials) {
        for (int64_t tid = 0; tid < n; ++tid) {
                orc_path_state &p = paths[tid];
                if (p.active == 0) continue;
                const orc_isect &in = isects[tid];
                if (in.hit == 0) {
                        p.active = 0;
                        continue;
                }
                const orc_material &mat = materials[in.prim_id.material_index];
                if (mat.type == 2) {
                        for (int c = 0; c < 3; ++c) p.estimate[c] = p.estimate[c] + p.throughput[c] * mat.emission[c];
                        p.active = 0;
                        continue;
                }
                if (mat.type != 1) {
                        p.active = 0;
                        continue;
                }
                int64_t mesh, base;
                const orc_prim_id &pid = in.prim_id;
                if (pid.type == 0) {
                        mesh = pid.id1;
                        base = pid.id2;
                } else if (pid.type == 1 || pid.type == 2 || pid.type == 3) {
                        mesh = pid.id2 >> 32;
                        base = (pid.id2 & 0xFFFFFFFFll) * 3;
                } else {
                        p.active = 0;
                        continue;
                }
                const orc_mesh &m = meshes[mesh];
                const float *a = m.points + 4 * m.vertex_indices[base];
                const float *b = m.points + 4 * m.vertex_indices[base + 1];
                const float *c = m.points + 4 * m.vertex_indices[base + 2];
                const float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
                const float e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
                float nrm[3];
                cross3(e1, e2, nrm);
                const float nlen = dot3(nrm, nrm);
                if (nlen > 0) {
                        const float s = 1.0f / std::sqrt(nlen);
                        for (int k = 0; k < 3; ++k) nrm[k] = nrm[k] * s;
                }
                const float rd[3] = {p.ray.dx, p.ray.dy, p.ray.dz};
                if (dot3(nrm, rd) > 0)
                        for (int k = 0; k < 3; ++k) nrm[k] = nrm[k] * -1.0f;
                Pcg32 pcg(p.pcg_state, p.pcg_inc);
                const float u1 = pcg.next_float();
                const float u2 = pcg.next_float();
                p.pcg_state = pcg.state;
                const float r = std::sqrt(u1);
                const float theta = 2.0f * 3.14159265359f * u2;
                const float x = r * std::cos(theta);
                const float y = r * std::sin(theta);
                const float z2 = 1.0f - u1;
                const float z = std::sqrt(z2 > 0.0f ? z2 : 0.0f);
                const float sign = nrm[2] >= 0.0f ? 1.0f : -1.0f;
                const float aa = -1.0f / (sign + nrm[2]);
                const float bb = nrm[0] * nrm[1] * aa;
                const float t[3] = {1.0f + sign * nrm[0] * nrm[0] * aa, sign * bb, -sign * nrm[0]};
                const float bt[3] = {bb, sign + nrm[1] * nrm[1] * aa, -nrm[1]};
                float dir[3];
                for (int k = 0; k < 3; ++k) dir[k] = t[k] * x + bt[k] * y + nrm[k] * z;
                const float dlen = dot3(dir, dir);
                if (dlen > 0) {
                        const float s = 1.0f / std::sqrt(dlen);
                        for (int k = 0; k < 3; ++k) dir[k] = dir[k] * s;
                }
                const float ro[3] = {p.ray.ox, p.ray.oy, p.ray.oz};
                float org[3];
                for (int k = 0; k < 3; ++k) org[k] = ro[k] + rd[k] * in.t + nrm[k] * 0.0001f;
                p.ray.ox = org[0];
                p.ray.oy = org[1];
                p.ray.oz = org[2];
                p.ray.dx = dir[0];
                p.ray.dy = dir[1];
                p.ray.dz = dir[2];
                for (int k = 0; k < 3; ++k) p.throughput[k] = p.throughput[k] * mat.albedo[k];
        }
}
