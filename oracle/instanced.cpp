// instanced.cpp - CPU restatement of two-level traversal (test
// infrastructure only).  -ffp-contract=off.
//
// The top-level walk follows traverse_bvh2_core (kernel.mojo:223-364) with
// its slab test (:171-206); a leaf's prims are instances, and each is
// intersected as TransformedPrimitive.intersect does
// (Primitive/TransformedPrimitive.swift:5-22): the ray goes to object space
// through the inverse transform (Transform*Point / Transform*Vector,
// Geometry/Transform.swift:31-65; direction not renormalised), the bottom-level
// hierarchy is searched with the current tHit, and a hit lowers tHit.
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "oracle.h"

namespace {

struct Best {
        int32_t prim = -1, inst = -1;
        float t = 0, u = 0, v = 0;
};

inline float xf_point(const float *row, float x, float y, float z) {
        float s = row[0] * x;
        s = s + row[1] * y;
        s = s + row[2] * z;
        return s + row[3];
}
inline float xf_vector(const float *row, float x, float y, float z) {
        float s = row[0] * x;
        s = s + row[1] * y;
        return s + row[2] * z;
}

void intersect_instance(int64_t inst, const float *w2o, const int32_t *blas_of, const orc_blas *blas,
                        const orc_ray &ray, Best &best) {
        const float *m = w2o + 12 * inst;
        orc_ray local;
        local.ox = xf_point(m, ray.ox, ray.oy, ray.oz);
        local.oy = xf_point(m + 4, ray.ox, ray.oy, ray.oz);
        local.oz = xf_point(m + 8, ray.ox, ray.oy, ray.oz);
        local.dx = xf_vector(m, ray.dx, ray.dy, ray.dz);
        local.dy = xf_vector(m + 4, ray.dx, ray.dy, ray.dz);
        local.dz = xf_vector(m + 8, ray.dx, ray.dy, ray.dz);
        const orc_blas &b = blas[blas_of[inst]];
        orc_isect is;
        int32_t idx;
        orc_trace_one(b.nodes, b.prims, b.meshes, &local, best.t, &is, &idx);
        if (is.hit) {
                best.t = is.t;
                best.u = is.u;
                best.v = is.v;
                best.prim = idx;
                best.inst = (int32_t)inst;
        }
}

void traverse_top(const orc_node *nodes, const int64_t *leaf_instance, const float *w2o, const int32_t *blas_of,
                  const orc_blas *blas, const orc_ray &ray, float tmax, Best &best) {
        const float o[3] = {ray.ox, ray.oy, ray.oz}, d[3] = {ray.dx, ray.dy, ray.dz};
        best.t = tmax;
        int64_t stack[64];
        int sp = 0;
        int64_t current = 0;
        for (;;) {
                const orc_node &node = nodes[current];
                if (node.count > 0) {
                        for (int64_t j = 0; j < node.count; ++j)
                                intersect_instance(leaf_instance[node.offset + j], w2o, blas_of, blas, ray, best);
                        if (sp == 0) break;
                        current = stack[--sp];
                        continue;
                }
                const int64_t li = current + 1, ri = node.offset;
                float lt, rt;
                const bool lh = orc_intersect_aabb(nodes[li].mn, nodes[li].mx, o, d, best.t, &lt) != 0;
                const bool rh = orc_intersect_aabb(nodes[ri].mn, nodes[ri].mx, o, d, best.t, &rt) != 0;
                if (lh && rh) {
                        if (lt <= rt) {
                                current = li;
                                stack[sp++] = ri;
                        } else {
                                current = ri;
                                stack[sp++] = li;
                        }
                } else if (lh) {
                        current = li;
                } else if (rh) {
                        current = ri;
                } else {
                        if (sp == 0) break;
                        current = stack[--sp];
                }
        }
        if (best.prim < 0) {
                best.t = tmax;
                best.u = best.v = 0.0f;
                best.inst = -1;
        }
}

}  // namespace

extern "C" void orc_traverse_instanced(const orc_node *tlas, const int64_t *leaf_instance, const float *w2o,
                                       const int32_t *blas_of, const orc_blas *blas, const orc_ray *rays,
                                       const float *tmax, int64_t n, int32_t *prim, int32_t *inst, float *t,
                                       float *u, float *v, int threads) {
        if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
        std::atomic<int64_t> next{0};
        std::vector<std::thread> pool;
        for (int k = 0; k < threads; ++k)
                pool.emplace_back([&]() {
                        for (;;) {
                                const int64_t s = next.fetch_add(256);
                                if (s >= n) break;
                                const int64_t e = std::min(n, s + 256);
                                for (int64_t i = s; i < e; ++i) {
                                        Best b;
                                        traverse_top(tlas, leaf_instance, w2o, blas_of, blas, rays[i], tmax[i], b);
                                        prim[i] = b.prim;
                                        inst[i] = b.inst;
                                        t[i] = b.t;
                                        u[i] = b.u;
                                        v[i] = b.v;
                                }
                        }
                });
        for (auto &th : pool) th.join();
}

// One ray through the two-level scene (the renderer's trace); returns 1 on a
// hit.
extern "C" int orc_trace_instanced_one(const orc_node *tlas, const int64_t *leaf_instance, const float *w2o,
                                       const int32_t *blas_of, const orc_blas *blas, const orc_ray *ray, float tmax,
                                       int32_t *prim, int32_t *inst, float *t, float *u, float *v) {
        Best b;
        traverse_top(tlas, leaf_instance, w2o, blas_of, blas, *ray, tmax, b);
        *prim = b.prim;
        *inst = b.inst;
        *t = b.t;
        *u = b.u;
        *v = b.v;
        return b.prim >= 0 ? 1 : 0;
}
