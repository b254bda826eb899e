// host_bvh2.cpp - SAH BVH2 builder on the host, standing in for Gonzales'
// BoundingHierarchyBuilder (Sources/libgonzales/Accelerators/
// BoundingHierarchyBuilder.swift:66-339).  The output (node array and prim
// order) is the reference builder's exactly: same buckets, same float
// arithmetic order, same Swift partition scan, same depth-first flatten.  Like
// the reference, subtrees above 100k prims are built on a second thread
// (BoundingHierarchyBuilder.swift:313-332); ranges are disjoint, so the result
// does not depend on the thread count.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "gzg_internal.h"

namespace gzg {
namespace {

constexpr float kInf = std::numeric_limits<float>::infinity();
constexpr int kBuckets = 12;       // BoundingHierarchyBuilder.swift:214
constexpr int kLeafPrims = 4;      // BoundingHierarchyBuilder.swift:58
constexpr int64_t kParallel = 100000;  // BoundingHierarchyBuilder.swift:313

// Swift stdlib min/max: min(x, y) = y < x ? y : x; max(x, y) = y >= x ? y : x.
inline float smin(float x, float y) { return y < x ? y : x; }
inline float smax(float x, float y) { return y >= x ? y : x; }

struct Box {
        float lo[3], hi[3];
        static Box empty() { return Box{{kInf, kInf, kInf}, {-kInf, -kInf, -kInf}}; }
        // Bounds3(first:second:) sorts the corners (Geometry/Bounds3.swift:3-12);
        // union(first:second:) goes through it (Bounds3.swift:104-114).
        void merge(const Box &b) {
                for (int i = 0; i < 3; ++i) {
                        float a = smin(lo[i], b.lo[i]);
                        float c = smax(hi[i], b.hi[i]);
                        lo[i] = smin(a, c);
                        hi[i] = smax(a, c);
                }
        }
        // union(bound:point:) (Geometry/Geometry.swift:51-61).
        void merge_point(const float p[3]) {
                for (int i = 0; i < 3; ++i) {
                        float a = smin(lo[i], p[i]);
                        float c = smax(hi[i], p[i]);
                        lo[i] = smin(a, c);
                        hi[i] = smax(a, c);
                }
        }
        // surfaceArea (Bounds3.swift:98-101).
        float area() const {
                float x = hi[0] - lo[0], y = hi[1] - lo[1], z = hi[2] - lo[2];
                float s = x * y;
                s = s + x * z;
                s = s + y * z;
                return 2.0f * s;
        }
        // maximumExtent (Bounds3.swift:75-84).
        int widest() const {
                float x = hi[0] - lo[0], y = hi[1] - lo[1], z = hi[2] - lo[2];
                if (x > y && x > z) return 0;
                return y > z ? 1 : 2;
        }
};

struct PrimRec {
        Box box;
        float c[3];  // 0.5 * pMin + 0.5 * pMax (Bounds3.swift:168-171)
        int64_t index;
};

struct BNode {
        Box box;
        int32_t l = -1, r = -1;
        int64_t first = 0, n = 0;
};

class SahBuilder {
      public:
        explicit SahBuilder(std::vector<PrimRec> &prims) : p_(prims) {}

        int32_t build(std::vector<BNode> &out, int64_t lo, int64_t hi, int par_depth) {
                const int64_t count = hi - lo;
                BNode node;
                Box box = Box::empty();
                Box cbox = Box::empty();
                for (int64_t i = lo; i < hi; ++i) box.merge(p_[i].box);
                for (int64_t i = lo; i < hi; ++i) cbox.merge_point(p_[i].c);
                const int axis = cbox.widest();
                if (box.area() == 0.0f || count == 1 || cbox.hi[axis] == cbox.lo[axis]) return leaf(out, box, lo, count);

                int64_t mid;
                if (count <= 2) {
                        mid = lo + 1;
                        if (p_[lo + 1].c[axis] < p_[lo].c[axis]) std::swap(p_[lo], p_[lo + 1]);
                } else {
                        int split;
                        if (!choose_split(lo, hi, box, cbox, axis, &split)) return leaf(out, box, lo, count);
                        mid = partition(lo, hi, cbox, axis, split);
                }

                int32_t left, right;
                if (count > kParallel && par_depth > 0) {
                        std::vector<BNode> side;
                        int32_t side_root = -1;
                        std::thread worker([&] { side_root = build(side, lo, mid, par_depth - 1); });
                        right = build(out, mid, hi, par_depth - 1);
                        worker.join();
                        const int32_t base = (int32_t)out.size();
                        for (BNode n : side) {
                                if (n.l >= 0) n.l += base;
                                if (n.r >= 0) n.r += base;
                                out.push_back(n);
                        }
                        left = side_root + base;
                } else {
                        left = build(out, lo, mid, par_depth);
                        right = build(out, mid, hi, par_depth);
                }
                node.l = left;
                node.r = right;
                node.box = out[left].box;
                node.box.merge(out[right].box);
                out.push_back(node);
                return (int32_t)out.size() - 1;
        }

      private:
        std::vector<PrimRec> &p_;

        static int32_t leaf(std::vector<BNode> &out, const Box &box, int64_t first, int64_t n) {
                BNode node;
                node.box = box;
                node.first = first;
                node.n = n;
                out.push_back(node);
                return (int32_t)out.size() - 1;
        }

        // Bucket of a prim: Int(12 * centroidBounds.offset(centroid)[axis]),
        // clamped to 11 (BoundingHierarchyBuilder.swift:217-219).
        static int bucket(const Box &cbox, const float c[3], int axis) {
                float off = c[axis] - cbox.lo[axis];
                if (cbox.hi[axis] > cbox.lo[axis]) off = off / (cbox.hi[axis] - cbox.lo[axis]);
                int b = (int)(12.0f * off);
                return b == kBuckets ? kBuckets - 1 : b;
        }

        // splitSurfaceAreaHeuristic (BoundingHierarchyBuilder.swift:213-259).
        // Returns false when the range should become a leaf.
        bool choose_split(int64_t lo, int64_t hi, const Box &box, const Box &cbox, int axis, int *split) const {
                int64_t cnt[kBuckets] = {0};
                Box bb[kBuckets];
                for (auto &b : bb) b = Box::empty();
                for (int64_t i = lo; i < hi; ++i) {
                        const int b = bucket(cbox, p_[i].c, axis);
                        ++cnt[b];
                        bb[b].merge(p_[i].box);
                }
                float cost[kBuckets - 1];
                int64_t n_below = 0;
                Box below = Box::empty();
                for (int i = 0; i < kBuckets - 1; ++i) {
                        below.merge(bb[i]);
                        n_below += cnt[i];
                        cost[i] = 0.0f + (float)n_below * below.area();
                }
                int64_t n_above = 0;
                Box above = Box::empty();
                for (int i = kBuckets - 1; i >= 1; --i) {
                        above.merge(bb[i]);
                        n_above += cnt[i];
                        cost[i - 1] = cost[i - 1] + (float)n_above * above.area();
                }
                int best = -1;
                float best_cost = kInf;
                for (int i = 0; i < kBuckets - 1; ++i)
                        if (cost[i] < best_cost) {
                                best_cost = cost[i];
                                best = i;
                        }
                const float leaf_cost = (float)(hi - lo);
                best_cost = 0.5f + best_cost / box.area();
                *split = best;
                return (hi - lo) > kLeafPrims || best_cost < leaf_cost;
        }

        // MutableCollection.partition(by:) of the Swift stdlib for
        // bidirectional collections: advance lo past first-partition elements,
        // retreat hi past second-partition elements, swap, repeat.
        int64_t partition(int64_t lo, int64_t hi, const Box &cbox, int axis, int split) {
                auto second = [&](const PrimRec &r) { return bucket(cbox, r.c, axis) > split; };
                for (;;) {
                        while (true) {
                                if (lo >= hi) return lo;
                                if (second(p_[lo])) break;
                                ++lo;
                        }
                        while (true) {
                                --hi;
                                if (lo >= hi) return lo;
                                if (!second(p_[hi])) break;
                        }
                        std::swap(p_[lo], p_[hi]);
                        ++lo;
                }
        }
};

// flatten2 (BoundingHierarchyBuilder.swift:122-156), iterative pre-order.
int64_t flatten(const std::vector<BNode> &tree, int32_t root, gzg_bvh2_node *out) {
        struct Item {
                int32_t node;
                int64_t parent;  // flattened index of the parent whose right link this fills, or -1
        };
        std::vector<Item> todo;
        todo.push_back({root, -1});
        int64_t used = 0;
        while (!todo.empty()) {
                Item it = todo.back();
                todo.pop_back();
                const BNode &b = tree[it.node];
                const int64_t me = used++;
                gzg_bvh2_node &n = out[me];
                for (int i = 0; i < 3; ++i) {
                        n.bounds_min[i] = b.box.lo[i];
                        n.bounds_max[i] = b.box.hi[i];
                }
                if (it.parent >= 0) out[it.parent].offset = (int32_t)me;
                if (b.n > 0) {
                        n.offset = (int32_t)b.first;
                        n.count = (int32_t)b.n;
                } else {
                        n.offset = 0;
                        n.count = 0;
                        // Left is visited next (index me + 1); the right child's
                        // index is patched into this node when it is emitted.
                        if (b.r >= 0) todo.push_back({b.r, me});
                        if (b.l >= 0) todo.push_back({b.l, -1});
                }
        }
        return used;
}

}  // namespace
}  // namespace gzg

using namespace gzg;

extern "C" GZG_API gzg_status gzg_host_triangle_bounds(const float *points4, const int64_t *vi, int64_t ntri,
                                                        float *bounds6) {
        if (ntri < 0 || (ntri > 0 && (!points4 || !vi || !bounds6)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_host_triangle_bounds: bad arguments");
        for (int64_t t = 0; t < ntri; ++t) {
                const float *p0 = points4 + 4 * vi[3 * t];
                const float *p1 = points4 + 4 * vi[3 * t + 1];
                const float *p2 = points4 + 4 * vi[3 * t + 2];
                Box b;
                for (int i = 0; i < 3; ++i) {
                        b.lo[i] = smin(p0[i], p1[i]);
                        b.hi[i] = smax(p0[i], p1[i]);
                }
                b.merge_point(p2);
                std::memcpy(bounds6 + 6 * t, b.lo, 12);
                std::memcpy(bounds6 + 6 * t + 3, b.hi, 12);
        }
        return clear_error();
}

extern "C" GZG_API gzg_status gzg_host_build_bvh2(const float *bounds6, int64_t n, gzg_bvh2_node *nodes_out,
                                                   int64_t *node_count_out, int64_t *order_out, int32_t threads) {
        if (n < 0 || !node_count_out || (n > 0 && (!bounds6 || !nodes_out || !order_out)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_host_build_bvh2: bad arguments");
        if (n > (int64_t)INT32_MAX / 2)
                return set_error(GZG_ERR_LIMIT, "gzg_host_build_bvh2: more than 2^30 prims");
        *node_count_out = 0;
        if (n == 0) return clear_error();
        std::vector<PrimRec> prims((size_t)n);
        for (int64_t i = 0; i < n; ++i) {
                PrimRec &r = prims[i];
                std::memcpy(r.box.lo, bounds6 + 6 * i, 12);
                std::memcpy(r.box.hi, bounds6 + 6 * i + 3, 12);
                for (int k = 0; k < 3; ++k) {
                        float a = 0.5f * r.box.lo[k];
                        float b = 0.5f * r.box.hi[k];
                        r.c[k] = a + b;
                }
                r.index = i;
        }
        if (threads <= 0) threads = (int32_t)std::max(1u, std::thread::hardware_concurrency());
        int par_depth = 0;
        while ((1 << par_depth) < threads && par_depth < 6) ++par_depth;
        std::vector<BNode> tree;
        tree.reserve((size_t)(2 * n));
        SahBuilder builder(prims);
        const int32_t root = builder.build(tree, 0, n, par_depth);
        *node_count_out = flatten(tree, root, nodes_out);
        for (int64_t i = 0; i < n; ++i) order_out[i] = prims[i].index;
        return clear_error();
}
