// oracle.cpp - CPU restatement of the Gonzales hot path (test infrastructure:
// the checker and the timed CPU baseline; never linked by the product).
// Compile with -ffp-contract=off so each float operation rounds on its own,
// in the order the reference writes it.  File/line citations are relative to
// the Gonzales source tree.
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <thread>
#include <vector>

namespace {

const float kInf = std::numeric_limits<float>::infinity();

// Swift's global min/max (stdlib): min returns y < x ? y : x, max returns
// y >= x ? y : x.  The choice matters only for signed zeros, but it is kept.
inline float swift_min(float x, float y) { return y < x ? y : x; }
inline float swift_max(float x, float y) { return y >= x ? y : x; }

// Bounds3 (Geometry/Bounds3.swift).
struct Bounds {
        float mn[3], mx[3];
};

// Bounds3() : pMin = +inf, pMax = -inf (Bounds3.swift:56-59).
Bounds bounds_empty() { return Bounds{{kInf, kInf, kInf}, {-kInf, -kInf, -kInf}}; }

// Bounds3(first:second:) re-sorts its two corners (Bounds3.swift:3-12).
Bounds bounds_make(const float a[3], const float b[3]) {
        Bounds r;
        for (int i = 0; i < 3; ++i) {
                r.mn[i] = swift_min(a[i], b[i]);
                r.mx[i] = swift_max(a[i], b[i]);
        }
        return r;
}

// union(first:second:) (Bounds3.swift:104-114).  Note the re-sort of the
// result: the union of two empty boxes becomes the infinite box (-inf, +inf).
Bounds bounds_union(const Bounds &a, const Bounds &b) {
        float pmin[3], pmax[3];
        for (int i = 0; i < 3; ++i) {
                pmin[i] = swift_min(a.mn[i], b.mn[i]);
                pmax[i] = swift_max(a.mx[i], b.mx[i]);
        }
        return bounds_make(pmin, pmax);
}

// union(bound:point:) (Geometry/Geometry.swift:51-61).
Bounds bounds_union_point(const Bounds &a, const float p[3]) {
        float pmin[3], pmax[3];
        for (int i = 0; i < 3; ++i) {
                pmin[i] = swift_min(a.mn[i], p[i]);
                pmax[i] = swift_max(a.mx[i], p[i]);
        }
        return bounds_make(pmin, pmax);
}

// surfaceArea (Bounds3.swift:98-101): 2 * (x*y + x*z + y*z).
float bounds_sa(const Bounds &b) {
        float dx = b.mx[0] - b.mn[0], dy = b.mx[1] - b.mn[1], dz = b.mx[2] - b.mn[2];
        float s = dx * dy;
        s = s + dx * dz;
        s = s + dy * dz;
        return 2.0f * s;
}

// maximumExtent (Bounds3.swift:75-84).
int bounds_max_extent(const Bounds &b) {
        float dx = b.mx[0] - b.mn[0], dy = b.mx[1] - b.mn[1], dz = b.mx[2] - b.mn[2];
        if (dx > dy && dx > dz) return 0;
        if (dy > dz) return 1;
        return 2;
}

// center (Bounds3.swift:168-171) and CachedPrimitive.centroid()
// (BoundingHierarchyBuilder.swift:42-44): 0.5 * pMin + 0.5 * pMax.
void bounds_center(const Bounds &b, float c[3]) {
        for (int i = 0; i < 3; ++i) {
                float a = 0.5f * b.mn[i];
                float d = 0.5f * b.mx[i];
                c[i] = a + d;
        }
}

// offset(point:) (Bounds3.swift:90-96), one component.
float bounds_offset(const Bounds &b, const float p[3], int dim) {
        float r = p[dim] - b.mn[dim];
        if (b.mx[dim] > b.mn[dim]) r = r / (b.mx[dim] - b.mn[dim]);
        return r;
}

struct Prim {
        int64_t index;
        Bounds bound;
        float center[3];
};

struct BuildNode {
        Bounds bounds;
        int32_t left = -1, right = -1;
        int64_t first = 0, n = 0;
};

struct Builder {
        std::vector<Prim> buf;
        std::vector<BuildNode> nodes;

        // Swift MutableCollection.partition(by:) for bidirectional collections
        // (stdlib _partitionImpl): Hoare-style scan from both ends.
        template <class Pred>
        int64_t partition(int64_t lo, int64_t hi, Pred second) {
                for (;;) {
                        for (;;) {
                                if (!(lo < hi)) return lo;
                                if (second(buf[lo])) break;
                                ++lo;
                        }
                        for (;;) {
                                --hi;
                                if (!(lo < hi)) return lo;
                                if (!second(buf[hi])) break;
                        }
                        std::swap(buf[lo], buf[hi]);
                        ++lo;
                }
        }

        static int bucket_of(const Bounds &cb, const Prim &p, int dim) {
                float c[3];
                bounds_center(p.bound, c);
                float off = bounds_offset(cb, c, dim);
                int b = (int)(12.0f * off);
                if (b == 12) b = 11;
                return b;
        }

        // build(range:) (BoundingHierarchyBuilder.swift:266-339) with the SAH
        // split of :199-264.  Returns the build-node index.
        int32_t build(int64_t lo, int64_t hi) {
                BuildNode node;
                const int64_t count = hi - lo;
                if (count == 0) {
                        node.bounds = bounds_empty();
                        nodes.push_back(node);
                        return (int32_t)nodes.size() - 1;
                }
                Bounds bounds = bounds_empty();
                for (int64_t i = lo; i < hi; ++i) bounds = bounds_union(bounds, buf[i].bound);
                Bounds cb = bounds_empty();
                for (int64_t i = lo; i < hi; ++i) cb = bounds_union_point(cb, buf[i].center);
                const int dim = bounds_max_extent(cb);
                if (bounds_sa(bounds) == 0.0f || count == 1 || cb.mx[dim] == cb.mn[dim]) {
                        node.bounds = bounds;
                        node.first = lo;
                        node.n = count;
                        nodes.push_back(node);
                        return (int32_t)nodes.size() - 1;
                }
                int64_t mid;
                if (count <= 2) {
                        mid = lo + count / 2;
                        // sort(by: center[dim] <) of two elements: insertion sort.
                        if (buf[lo + 1].center[dim] < buf[lo].center[dim]) std::swap(buf[lo], buf[lo + 1]);
                } else {
                        const int nb = 12;
                        int64_t bcount[nb] = {0};
                        Bounds bb[nb];
                        for (int i = 0; i < nb; ++i) bb[i] = bounds_empty();
                        for (int64_t i = lo; i < hi; ++i) {
                                int b = bucket_of(cb, buf[i], dim);
                                bcount[b] += 1;
                                bb[b] = bounds_union(bb[b], buf[i].bound);
                        }
                        float costs[nb - 1];
                        for (int i = 0; i < nb - 1; ++i) costs[i] = 0.0f;
                        int64_t below = 0;
                        Bounds bbelow = bounds_empty();
                        for (int i = 0; i < nb - 1; ++i) {
                                bbelow = bounds_union(bbelow, bb[i]);
                                below += bcount[i];
                                costs[i] = costs[i] + (float)below * bounds_sa(bbelow);
                        }
                        int64_t above = 0;
                        Bounds babove = bounds_empty();
                        for (int i = nb - 1; i >= 1; --i) {
                                babove = bounds_union(babove, bb[i]);
                                above += bcount[i];
                                costs[i - 1] = costs[i - 1] + (float)above * bounds_sa(babove);
                        }
                        int split = -1;
                        float min_cost = kInf;
                        for (int i = 0; i < nb - 1; ++i)
                                if (costs[i] < min_cost) {
                                        min_cost = costs[i];
                                        split = i;
                                }
                        const float leaf_cost = (float)count;
                        min_cost = 0.5f + min_cost / bounds_sa(bounds);
                        if (count > 4 || min_cost < leaf_cost) {
                                mid = partition(lo, hi, [&](const Prim &p) { return bucket_of(cb, p, dim) > split; });
                        } else {
                                node.bounds = bounds;
                                node.first = lo;
                                node.n = count;
                                nodes.push_back(node);
                                return (int32_t)nodes.size() - 1;
                        }
                }
                int32_t l = build(lo, mid);
                int32_t r = build(mid, hi);
                node.left = l;
                node.right = r;
                node.bounds = bounds_union(nodes[l].bounds, nodes[r].bounds);
                nodes.push_back(node);
                return (int32_t)nodes.size() - 1;
        }

        // flatten2 (BoundingHierarchyBuilder.swift:122-156): depth-first,
        // left child at index + 1, right child index in offset.
        int64_t flatten(int32_t bi, orc_node *out, int64_t &used) {
                const int64_t me = used++;
                const BuildNode &b = nodes[bi];
                orc_node n;
                for (int i = 0; i < 3; ++i) {
                        n.mn[i] = b.bounds.mn[i];
                        n.mx[i] = b.bounds.mx[i];
                }
                if (b.n > 0) {
                        n.offset = (int32_t)b.first;
                        n.count = (int32_t)b.n;
                } else {
                        n.offset = 0;
                        if (b.left >= 0) flatten(b.left, out, used);
                        if (b.right >= 0) n.offset = (int32_t)flatten(b.right, out, used);
                        n.count = 0;
                }
                out[me] = n;
                return me;
        }
};

// ---------------------------------------------------------------- traversal

// cross / dot of kernel.mojo:84-95.
inline void cross3(const float a[3], const float b[3], float r[3]) {
        r[0] = a[1] * b[2] - a[2] * b[1];
        r[1] = a[2] * b[0] - a[0] * b[2];
        r[2] = a[0] * b[1] - a[1] * b[0];
}
inline float dot3(const float a[3], const float b[3]) {
        float s = a[0] * b[0];
        s = s + a[1] * b[1];
        s = s + a[2] * b[2];
        return s;
}

// intersect_triangle (kernel.mojo:122-156).
int mt_test(const float o[3], const float d[3], const float p0[3], const float p1[3], const float p2[3],
            float tmax, float *t_out, float *u_out, float *v_out) {
        float e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
        float e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
        float pvec[3];
        cross3(d, e2, pvec);
        float det = dot3(e1, pvec);
        if (det > -1e-7f && det < 1e-7f) return 0;
        float inv = 1.0f / det;
        float tvec[3] = {o[0] - p0[0], o[1] - p0[1], o[2] - p0[2]};
        float u = dot3(tvec, pvec) * inv;
        if (u < 0.0f || u > 1.0f) return 0;
        float qvec[3];
        cross3(tvec, e1, qvec);
        float v = dot3(d, qvec) * inv;
        if (v < 0.0f || u + v > 1.0f) return 0;
        float t = dot3(e2, qvec) * inv;
        if (t <= 0.0f || t > tmax) return 0;
        *t_out = t;
        *u_out = u;
        *v_out = v;
        return 1;
}

// Triangle.getIntersectionData (Shape/Triangle.swift:269-352).
int watertight_test(const float o[3], const float d[3], const float p0[3], const float p1[3],
                    const float p2[3], float *thit, float *b0o, float *b1o, float *b2o) {
        float a0[3], a1[3], a2[3];
        for (int i = 0; i < 3; ++i) {
                a0[i] = p0[i] - o[i];
                a1[i] = p1[i] - o[i];
                a2[i] = p2[i] - o[i];
        }
        float ad[3] = {std::fabs(d[0]), std::fabs(d[1]), std::fabs(d[2])};
        // maxDimension (Geometry/Geometry.swift:46-49)
        int kz = (ad[0] > ad[1]) ? ((ad[0] > ad[2]) ? 0 : 2) : ((ad[1] > ad[2]) ? 1 : 2);
        int kx = (kz + 1) % 3;
        int ky = (kx + 1) % 3;
        float dx = d[kx], dy = d[ky], dz = d[kz];
        float q0[3] = {a0[kx], a0[ky], a0[kz]};
        float q1[3] = {a1[kx], a1[ky], a1[kz]};
        float q2[3] = {a2[kx], a2[ky], a2[kz]};
        float sx = -dx / dz;
        float sy = -dy / dz;
        float sz = 1.0f / dz;
        q0[0] = q0[0] + sx * q0[2];
        q0[1] = q0[1] + sy * q0[2];
        q1[0] = q1[0] + sx * q1[2];
        q1[1] = q1[1] + sy * q1[2];
        q2[0] = q2[0] + sx * q2[2];
        q2[1] = q2[1] + sy * q2[2];
        float e0 = q1[0] * q2[1] - q1[1] * q2[0];
        float e1 = q2[0] * q0[1] - q2[1] * q0[0];
        float e2 = q0[0] * q1[1] - q0[1] * q1[0];
        if ((e0 < 0 || e1 < 0 || e2 < 0) && (e0 > 0 || e1 > 0 || e2 > 0)) return 0;
        float det = e0 + e1;
        det = det + e2;
        if (det == 0) return 0;
        q0[2] = q0[2] * sz;
        q1[2] = q1[2] * sz;
        q2[2] = q2[2] * sz;
        float ts = e0 * q0[2];
        ts = ts + e1 * q1[2];
        ts = ts + e2 * q2[2];
        bool pos = det > 0;
        if ((pos && (ts <= 0 || ts > *thit * det)) || (!pos && (ts >= 0 || ts < *thit * det))) return 0;
        float inv = 1 / det;
        *b0o = e0 * inv;
        *b1o = e1 * inv;
        *b2o = e2 * inv;
        *thit = ts * inv;
        return 1;
}

// intersect_aabb (kernel.mojo:171-206).
inline bool aabb_test(const float mn[3], const float mx[3], const float rdir[3], const float ordir[3],
                      const bool near_min[3], float tmax, float *tnear_out) {
        float tn[3], tf[3];
        for (int i = 0; i < 3; ++i) {
                float nr = near_min[i] ? mn[i] : mx[i];
                float fr = near_min[i] ? mx[i] : mn[i];
                tn[i] = nr * rdir[i] - ordir[i];
                tf[i] = fr * rdir[i] - ordir[i];
        }
        float tnear = tn[0] > tn[1] ? tn[0] : tn[1];
        tnear = tn[2] > tnear ? tn[2] : tnear;
        tnear = 0.0f > tnear ? 0.0f : tnear;
        float tfar = tf[0] < tf[1] ? tf[0] : tf[1];
        tfar = tf[2] < tfar ? tf[2] : tfar;
        tfar = tmax < tfar ? tmax : tfar;
        tfar = tfar * 1.0000003f;
        *tnear_out = tnear;
        return tnear <= tfar;
}

// traverse_bvh2_core (kernel.mojo:223-364).
void traverse_one(const orc_node *nodes, const orc_prim_id *prims, const orc_mesh *meshes, const orc_ray &ray,
                  float tmax, int watertight, orc_isect *res, int32_t *hit_index_out, uint32_t *cnt) {
        const float o[3] = {ray.ox, ray.oy, ray.oz};
        const float d[3] = {ray.dx, ray.dy, ray.dz};
        float rdir[3], ordir[3];
        bool near_min[3];
        for (int i = 0; i < 3; ++i) {
                rdir[i] = 1.0f / d[i];
                ordir[i] = o[i] * rdir[i];
                near_min[i] = rdir[i] >= 0.0f;
        }
        int64_t hit_index = -1;
        float t_hit = tmax, best_u = 0.0f, best_v = 0.0f;
        int64_t stack[64];
        int to_visit = 0;
        int64_t current = 0;
        uint32_t c_interior = 0, c_leaf = 0, c_tris = 0, c_fetch = 0;
        for (;;) {
                const orc_node &node = nodes[current];
                ++c_fetch;
                if (node.count > 0) {
                        ++c_leaf;
                        const int64_t off = node.offset;
                        for (int64_t j = 0; j < node.count; ++j) {
                                const orc_prim_id &p = prims[off + j];
                                int64_t mesh, base;
                                if (p.type == 0) {
                                        mesh = p.id1;
                                        base = p.id2;
                                } else if (p.type == 1 || p.type == 2 || p.type == 3) {
                                        if (p.id2 == -1) continue;
                                        mesh = p.id2 >> 32;
                                        base = (p.id2 & 0xFFFFFFFFll) * 3;
                                } else {
                                        continue;
                                }
                                const orc_mesh &m = meshes[mesh];
                                const int64_t i0 = m.vertex_indices[base], i1 = m.vertex_indices[base + 1],
                                              i2 = m.vertex_indices[base + 2];
                                const float p0[3] = {m.points[i0 * 4], m.points[i0 * 4 + 1], m.points[i0 * 4 + 2]};
                                const float p1[3] = {m.points[i1 * 4], m.points[i1 * 4 + 1], m.points[i1 * 4 + 2]};
                                const float p2[3] = {m.points[i2 * 4], m.points[i2 * 4 + 1], m.points[i2 * 4 + 2]};
                                ++c_tris;
                                if (watertight) {
                                        float th = t_hit, b0, b1, b2;
                                        if (watertight_test(o, d, p0, p1, p2, &th, &b0, &b1, &b2)) {
                                                t_hit = th;
                                                best_u = b1;
                                                best_v = b2;
                                                hit_index = off + j;
                                        }
                                } else {
                                        float t, u, v;
                                        if (mt_test(o, d, p0, p1, p2, t_hit, &t, &u, &v)) {
                                                t_hit = t;
                                                best_u = u;
                                                best_v = v;
                                                hit_index = off + j;
                                        }
                                }
                        }
                        if (to_visit == 0) break;
                        current = stack[--to_visit];
                } else {
                        ++c_interior;
                        const int64_t li = current + 1, ri = node.offset;
                        const orc_node &ln = nodes[li];
                        const orc_node &rn = nodes[ri];
                        c_fetch += 2;
                        float lt, rt;
                        bool lh = aabb_test(ln.mn, ln.mx, rdir, ordir, near_min, t_hit, &lt);
                        bool rh = aabb_test(rn.mn, rn.mx, rdir, ordir, near_min, t_hit, &rt);
                        if (lh && rh) {
                                if (lt <= rt) {
                                        current = li;
                                        stack[to_visit] = ri;
                                } else {
                                        current = ri;
                                        stack[to_visit] = li;
                                }
                                ++to_visit;
                        } else if (lh) {
                                current = li;
                        } else if (rh) {
                                current = ri;
                        } else {
                                if (to_visit == 0) break;
                                current = stack[--to_visit];
                        }
                }
        }
        std::memset(res, 0, sizeof(*res));
        if (hit_index != -1) {
                res->prim_id = prims[hit_index];
                res->t = t_hit;
                res->u = best_u;
                res->v = best_v;
                res->hit = 1;
        } else {
                res->prim_id.id1 = -1;
                res->prim_id.id2 = -1;
                res->prim_id.material_index = 0;
                res->prim_id.type = 0;
                res->t = tmax;
                res->u = 0.0f;
                res->v = 0.0f;
                res->hit = 0;
        }
        if (hit_index_out) *hit_index_out = (int32_t)hit_index;
        if (cnt) {
                cnt[0] = c_interior;
                cnt[1] = c_leaf;
                cnt[2] = c_tris;
                cnt[3] = c_fetch;
        }
}

template <class F>
void parallel_for(int64_t n, int threads, F f) {
        if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
        if (threads == 1 || n < 1024) {
                for (int64_t i = 0; i < n; ++i) f(i);
                return;
        }
        std::atomic<int64_t> next{0};
        const int64_t chunk = 256;
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t)
                pool.emplace_back([&]() {
                        for (;;) {
                                int64_t s = next.fetch_add(chunk);
                                if (s >= n) break;
                                int64_t e = std::min(n, s + chunk);
                                for (int64_t i = s; i < e; ++i) f(i);
                        }
                });
        for (auto &th : pool) th.join();
}

// ---------------------------------------------------------------- Z-Sobol

std::vector<uint32_t> g_sobol;  // 1024 x 52
const int kSobolDims = 1024;
const int kSobolSize = 52;

// ZSobolSampler.permutations (ZSobolSampler.swift:105-112).
const uint8_t kPerm[24][4] = {{0, 1, 2, 3}, {0, 1, 3, 2}, {0, 2, 1, 3}, {0, 2, 3, 1}, {0, 3, 2, 1}, {0, 3, 1, 2},
                              {1, 0, 2, 3}, {1, 0, 3, 2}, {1, 2, 0, 3}, {1, 2, 3, 0}, {1, 3, 2, 0}, {1, 3, 0, 2},
                              {2, 1, 0, 3}, {2, 1, 3, 0}, {2, 0, 1, 3}, {2, 0, 3, 1}, {2, 3, 0, 1}, {2, 3, 1, 0},
                              {3, 1, 2, 0}, {3, 1, 0, 2}, {3, 2, 1, 0}, {3, 2, 0, 1}, {3, 0, 2, 1}, {3, 0, 1, 2}};

inline uint64_t shr64(uint64_t v, int s) { return s >= 64 ? 0 : (v >> s); }

}  // namespace

extern "C" {

void orc_triangle_bounds(const float *pts, const int64_t *vi, int64_t ntri, float *out) {
        for (int64_t t = 0; t < ntri; ++t) {
                const float *p0 = pts + 4 * vi[3 * t], *p1 = pts + 4 * vi[3 * t + 1], *p2 = pts + 4 * vi[3 * t + 2];
                Bounds b = bounds_make(p0, p1);
                b = bounds_union_point(b, p2);
                std::memcpy(out + 6 * t, b.mn, 12);
                std::memcpy(out + 6 * t + 3, b.mx, 12);
        }
}

int64_t orc_build_bvh2(const float *bounds6, int64_t n, orc_node *nodes, int64_t *order) {
        if (n <= 0) return 0;
        Builder bld;
        bld.buf.resize(n);
        for (int64_t i = 0; i < n; ++i) {
                Prim &p = bld.buf[i];
                p.index = i;
                std::memcpy(p.bound.mn, bounds6 + 6 * i, 12);
                std::memcpy(p.bound.mx, bounds6 + 6 * i + 3, 12);
                bounds_center(p.bound, p.center);
        }
        bld.nodes.reserve(2 * n);
        int32_t root = bld.build(0, n);
        int64_t used = 0;
        bld.flatten(root, nodes, used);
        for (int64_t i = 0; i < n; ++i) order[i] = bld.buf[i].index;
        return used;
}

void orc_traverse_batch(const orc_node *nodes, const orc_prim_id *prims, const orc_mesh *meshes,
                        const orc_ray *rays, const float *tmax, int64_t n, int watertight, orc_isect *out,
                        int32_t *hit_index, uint32_t *counters, int threads) {
        parallel_for(n, threads, [&](int64_t i) {
                traverse_one(nodes, prims, meshes, rays[i], tmax[i], watertight, out + i,
                             hit_index ? hit_index + i : nullptr, counters ? counters + 4 * i : nullptr);
        });
}

void orc_trace_one(const orc_node *nodes, const orc_prim_id *prims, const orc_mesh *meshes, const orc_ray *ray,
                   float tmax, orc_isect *out, int32_t *hit_index) {
        traverse_one(nodes, prims, meshes, *ray, tmax, 0, out, hit_index, nullptr);
}

int orc_intersect_triangle_mt(const float *o, const float *d, const float *p0, const float *p1, const float *p2,
                              float tmax, float *t, float *u, float *v) {
        return mt_test(o, d, p0, p1, p2, tmax, t, u, v);
}

int orc_intersect_triangle_watertight(const float *o, const float *d, const float *p0, const float *p1,
                                      const float *p2, float *thit, float *b0, float *b1, float *b2) {
        return watertight_test(o, d, p0, p1, p2, thit, b0, b1, b2);
}

int orc_intersect_aabb(const float *mn, const float *mx, const float *o, const float *d, float tmax, float *tnear) {
        float rdir[3], ordir[3];
        bool nm[3];
        for (int i = 0; i < 3; ++i) {
                rdir[i] = 1.0f / d[i];
                ordir[i] = o[i] * rdir[i];
                nm[i] = rdir[i] >= 0.0f;
        }
        return aabb_test(mn, mx, rdir, ordir, nm, tmax, tnear) ? 1 : 0;
}

int orc_bounds_intersects_swift(const float *mn, const float *mx, const float *o, const float *d, float thit) {
        // Ray.inverseDirection = 1 / direction per component.
        float tmin[3], tmx[3], tentry[3], texit[3];
        for (int i = 0; i < 3; ++i) {
                float inv = 1.0f / d[i];
                tmin[i] = (mn[i] - o[i]) * inv;
                tmx[i] = (mx[i] - o[i]) * inv;
                tentry[i] = swift_min(tmin[i], tmx[i]);
                texit[i] = swift_max(tmin[i], tmx[i]);
        }
        // gamma(3) = 3 eps / (1 - 3 eps), eps = Float.ulpOfOne (Utility.swift:3, 24-26).
        const float eps = 1.1920928955078125e-07f;
        const float g3 = (3.0f * eps) / (1.0f - 3.0f * eps);
        const float corr = 1.0f + 2.0f * g3;
        for (int i = 0; i < 3; ++i) texit[i] = texit[i] * corr;
        float tnear = swift_max(tentry[0], tentry[1]);
        tnear = swift_max(tnear, tentry[2]);
        float tfar = swift_min(texit[0], texit[1]);
        tfar = swift_min(tfar, texit[2]);
        tnear = swift_max(tnear, 0.0f);
        tfar = swift_min(tfar, thit);
        return tnear <= tfar ? 1 : 0;
}

float orc_bounds_surface_area(const float *mn, const float *mx) {
        Bounds b = bounds_make(mn, mx);
        return bounds_sa(b);
}

int orc_bounds_maximum_extent(const float *mn, const float *mx) {
        Bounds b = bounds_make(mn, mx);
        return bounds_max_extent(b);
}

void orc_sobol_set_matrices(const uint32_t *m) { g_sobol.assign(m, m + kSobolDims * kSobolSize); }

// reverseBits32 (ZSobolSampler.swift:34-41).
uint32_t orc_reverse_bits32(uint32_t v) {
        v = ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
        v = ((v >> 2) & 0x33333333u) | ((v & 0x33333333u) << 2);
        v = ((v >> 4) & 0x0f0f0f0fu) | ((v & 0x0f0f0f0fu) << 4);
        v = ((v >> 8) & 0x00ff00ffu) | ((v & 0x00ff00ffu) << 8);
        return (v >> 16) | (v << 16);
}

// encodeMorton2 (ZSobolSampler.swift:70-88).
uint64_t orc_encode_morton2(uint32_t x, uint32_t y) {
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

// mixBits (ZSobolSampler.swift:90-101).
uint32_t orc_mix_bits(uint64_t v) {
        uint32_t x = (uint32_t)(v & 0xFFFFFFFFull);
        x ^= (uint32_t)(v >> 32);
        x ^= x >> 16;
        x *= 0x85ebca77u;
        x ^= x >> 13;
        x *= 0xc2b2ae35u;
        x ^= x >> 16;
        return x;
}

// FastOwenScrambler.callAsFunction (ZSobolSampler.swift:55-66).
uint32_t orc_owen_scramble(uint32_t v, uint32_t seed) {
        v = orc_reverse_bits32(v);
        v ^= v * 0x3d20adeau;
        v += seed;
        v *= (seed >> 16) | 1u;
        v ^= v * 0x05526c56u;
        v ^= v * 0x53a22864u;
        return orc_reverse_bits32(v);
}

// Int.nextPowerOfTwo (ZSobolSampler.swift:283-294).
int64_t orc_next_power_of_two(int64_t v) {
        v -= 1;
        v |= v >> 1;
        v |= v >> 2;
        v |= v >> 4;
        v |= v >> 8;
        v |= v >> 16;
        v += 1;
        return v;
}

// sobolSample (ZSobolSampler.swift:6-31).
float orc_sobol_sample(int64_t index, int dimension, uint32_t seed) {
        uint32_t acc = 0;
        uint64_t cur = (uint64_t)index;
        const uint32_t *m = g_sobol.data() + (size_t)dimension * kSobolSize;
        for (int bit = 0; bit < kSobolSize; ++bit) {
                if (cur & 1) acc ^= m[bit];
                cur >>= 1;
                if (cur == 0) break;
        }
        uint32_t r = orc_owen_scramble(acc, seed);
        float f = (float)r * 2.32830643653869628906e-10f;
        const float one_minus_eps = 1.0f - 1e-6f;
        return swift_min(f, one_minus_eps);
}

// ZSobolSampler.init(samplesPerPixel:fullResolution:seed:) (ZSobolSampler.swift:114-122).
void orc_zsobol_init(orc_zsobol *s, int64_t spp, int32_t res_x, int32_t res_y, int64_t seed) {
        int l2 = spp == 0 ? 64 : __builtin_ctzll((uint64_t)spp);
        s->log2spp = std::max(0, l2);
        s->seed = seed;
        int64_t res = orc_next_power_of_two(std::max(res_x, res_y));
        int log4 = (s->log2spp + 1) / 2;
        s->n_base4_digits = (res == 0 ? 64 : __builtin_ctzll((uint64_t)res)) + log4;
        s->morton_index = 0;
        s->dimension = 0;
}

// startPixelSample (ZSobolSampler.swift:130-136).
void orc_zsobol_start_pixel_sample(orc_zsobol *s, int32_t px, int32_t py, int64_t index, int32_t dim) {
        s->dimension = dim;
        uint64_t m = orc_encode_morton2((uint32_t)px, (uint32_t)py);
        s->morton_index = (m << s->log2spp) | (uint64_t)index;
}

// getSampleIndex (ZSobolSampler.swift:138-166).
uint64_t orc_zsobol_sample_index(const orc_zsobol *s) {
        uint64_t idx = 0;
        const bool pow2 = (s->log2spp & 1) == 1;
        const int last = pow2 ? 1 : 0;
        const uint64_t dmul = 0x55555555ull * (uint64_t)(int64_t)s->dimension;
        for (int di = s->n_base4_digits - 1; di >= last; --di) {
                const int shift = 2 * di - (pow2 ? 1 : 0);
                int digit = (int)(shr64(s->morton_index, shift) & 3);
                uint64_t higher = shr64(s->morton_index, shift + 2);
                uint32_t h = orc_mix_bits(higher ^ dmul);
                int p = (int)((h >> 24) % 24);
                digit = kPerm[p][digit];
                idx |= (uint64_t)digit << shift;
        }
        if (pow2) {
                int digit = (int)(s->morton_index & 1);
                uint32_t h = orc_mix_bits((s->morton_index >> 1) ^ dmul);
                digit ^= (int)(h & 1);
                idx |= (uint64_t)digit;
        }
        return idx;
}

// getSampleHash (ZSobolSampler.swift:188-199).  mixBits returns 32 bits, so
// the second hash is always 0.
static void zsobol_hash(const orc_zsobol *s, int off, uint32_t *h0, uint32_t *h1) {
        uint64_t dim = (uint64_t)(int64_t)(s->dimension + off);
        uint64_t bits = (uint64_t)orc_mix_bits(dim ^ (uint64_t)s->seed);
        *h0 = (uint32_t)(bits & 0xFFFFFFFFull);
        *h1 = (uint32_t)(bits >> 32);
}

// get1D (ZSobolSampler.swift:203-219).
float orc_zsobol_get1d(orc_zsobol *s) {
        int64_t idx = (int64_t)orc_zsobol_sample_index(s);
        uint32_t h0, h1;
        zsobol_hash(s, 0, &h0, &h1);
        if (s->dimension >= kSobolDims) s->dimension = 2;
        s->dimension += 1;
        return orc_sobol_sample(idx, s->dimension - 1, h0);
}

// get2D (ZSobolSampler.swift:221-244).
void orc_zsobol_get2d(orc_zsobol *s, float *out) {
        int64_t idx = (int64_t)orc_zsobol_sample_index(s);
        uint32_t h0, h1;
        zsobol_hash(s, 0, &h0, &h1);
        if (s->dimension + 1 >= kSobolDims) s->dimension = 2;
        s->dimension += 2;
        out[0] = orc_sobol_sample(idx, s->dimension - 2, h0);
        out[1] = orc_sobol_sample(idx, s->dimension - 1, h1);
}

// get3D (ZSobolSampler.swift:249-280).
void orc_zsobol_get3d(orc_zsobol *s, float *out) {
        int64_t idx = (int64_t)orc_zsobol_sample_index(s);
        uint32_t h0, h1, h2, unused;
        zsobol_hash(s, 0, &h0, &h1);
        zsobol_hash(s, 2, &h2, &unused);
        if (s->dimension + 2 >= kSobolDims) s->dimension = 2;
        s->dimension += 3;
        out[0] = orc_sobol_sample(idx, s->dimension - 3, h0);
        out[1] = orc_sobol_sample(idx, s->dimension - 2, h1);
        out[2] = orc_sobol_sample(idx, s->dimension - 1, h2);
}

void orc_zsobol_batch(int64_t spp, int32_t res_x, int32_t res_y, int64_t seed, const int32_t *px, const int32_t *py,
                      const int64_t *index, int64_t n, const int32_t *kinds, int32_t nkinds, float *out) {
        int32_t per = 0;
        for (int k = 0; k < nkinds; ++k) per += kinds[k];
        for (int64_t i = 0; i < n; ++i) {
                orc_zsobol s;
                orc_zsobol_init(&s, spp, res_x, res_y, seed);
                orc_zsobol_start_pixel_sample(&s, px[i], py[i], index[i], 0);
                float *o = out + i * per;
                for (int k = 0; k < nkinds; ++k) {
                        if (kinds[k] == 1) {
                                *o++ = orc_zsobol_get1d(&s);
                        } else if (kinds[k] == 2) {
                                orc_zsobol_get2d(&s, o);
                                o += 2;
                        } else {
                                orc_zsobol_get3d(&s, o);
                                o += 3;
                        }
                }
        }
}

}  // extern "C"
