// wide_bvh.cpp - validates the host's BVH2 (Gonzales layout, BVH2Node.swift:7-16)
// and converts it into the 8-wide quantised layout traversed on the device.
//
// Steps
//   1. Validate every reachable node link (left = i+1, i+1 < right < count),
//      leaf ranges and triangle/vertex indices.  Children always have larger
//      indices than their parent, so a validated tree has no cycles.
//   2. Lift the BVH2 into a binary tree whose leaves hold at most 4 triangles:
//      prims the reference never intersects (id2 == -1, kernel.mojo:273-275)
//      are dropped, larger leaves are split in order into groups of 4.  Node
//      boxes are the BVH2 boxes the host built.
//   3. Collapse: each wide node's children (at most 8 leaves or interior
//      binary nodes below it) are the ones that minimise the summed surface
//      area of the wide nodes beneath it, the SAH cost of node opens, by
//      dynamic programming over the binary tree (Ylitie, Karras and Laine
//      2017, without their leaf merging: leaves stay the lifted BVH2 leaves).
//   4. Assign children to slots by octant (front-to-back order for a ray is
//      slot ^ sign-bits) and quantise child boxes to 8 bits per plane,
//      rounding outward with a small extra margin.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>

#include "gzg_internal.h"

namespace gzg {
namespace {

// Triangles per leaf child: a BVH2 leaf with more is split in order into a
// balanced binary tree over groups of this size (each group gets its own
// quantised box).
constexpr int64_t kLeafTris = 4;

struct BinNode {
        float lo[3], hi[3];
        int32_t l = -1, r = -1;        // children (interior)
        int64_t tri_first = 0;         // leaf: range in the triangle list
        int32_t tri_count = 0;
        bool leaf() const { return l < 0; }
        double area() const {
                double x = (double)hi[0] - lo[0], y = (double)hi[1] - lo[1], z = (double)hi[2] - lo[2];
                return 2.0 * (x * y + x * z + y * z);
        }
};

// A leaf entry: a triangle (prim >= 0, the prim index) or, in a top-level
// tree, an instance (prim = -(instance + 1), vertices unused).
struct Tri {
        float p0[3], p1[3], p2[3];
        float lo[3], hi[3];
        int32_t prim;
};

class Converter {
      public:
        Converter(const gzg_bvh2_node *nodes, int64_t node_count, const gzg_prim_id *prims, int64_t prim_count,
                  const gzg_triangle_mesh *meshes, int64_t mesh_count, const int64_t *pts_counts,
                  const int64_t *vi_counts)
            : nodes_(nodes), node_count_(node_count), prims_(prims), prim_count_(prim_count), meshes_(meshes),
              mesh_count_(mesh_count), pts_counts_(pts_counts), vi_counts_(vi_counts) {}

        // Top-level mode: leaf prim k of the BVH2 is instance leaf_instance[k]
        // with world bounds inst_bounds[6 * instance ...].
        Converter(const gzg_bvh2_node *nodes, int64_t node_count, const int64_t *leaf_instance, int64_t leaf_count,
                  const float *inst_bounds, int64_t inst_count)
            : nodes_(nodes), node_count_(node_count), prims_(nullptr), prim_count_(leaf_count), meshes_(nullptr),
              mesh_count_(0), pts_counts_(nullptr), vi_counts_(nullptr), leaf_instance_(leaf_instance),
              inst_bounds_(inst_bounds), inst_count_(inst_count) {}

        gzg_status run(WideBvh *out, int32_t *bvh2_depth) {
                gzg_status st = lift(bvh2_depth);
                if (st != GZG_OK) return st;
                collapse(out);
                return GZG_OK;
        }

      private:
        const gzg_bvh2_node *nodes_;
        int64_t node_count_;
        const gzg_prim_id *prims_;
        int64_t prim_count_;
        const gzg_triangle_mesh *meshes_;
        int64_t mesh_count_;
        const int64_t *pts_counts_;
        const int64_t *vi_counts_;
        const int64_t *leaf_instance_ = nullptr;
        const float *inst_bounds_ = nullptr;
        int64_t inst_count_ = 0;

        std::vector<BinNode> bin_;
        std::vector<Tri> tris_;
        int32_t bin_root_ = -1;

        gzg_status bad(const std::string &m) { return set_error(GZG_ERR_BAD_SCENE, "gzg_gpu_upload_scene: " + m); }

        // Reads prim k's triangle into tris_ (if it is one).  Returns false on a bad index.
        bool read_prim(int64_t k, bool *is_tri, std::string *why) {
                if (leaf_instance_) {
                        const int64_t inst = leaf_instance_[k];
                        if (inst < 0 || inst >= inst_count_) {
                                *why = "top-level leaf " + std::to_string(k) + " references instance " + std::to_string(inst);
                                return false;
                        }
                        Tri t;
                        std::memset(&t, 0, sizeof(t));
                        std::memcpy(t.lo, inst_bounds_ + 6 * inst, 12);
                        std::memcpy(t.hi, inst_bounds_ + 6 * inst + 3, 12);
                        t.prim = -(int32_t)(inst + 1);
                        tris_.push_back(t);
                        *is_tri = true;
                        return true;
                }
                int64_t mesh, base;
                *is_tri = prim_triangle(prims_[k], &mesh, &base);
                if (!*is_tri) return true;
                if (mesh < 0 || mesh >= mesh_count_) {
                        *why = "prim " + std::to_string(k) + " references mesh " + std::to_string(mesh);
                        return false;
                }
                const gzg_triangle_mesh &m = meshes_[mesh];
                if (base < 0 || base + 2 >= vi_counts_[mesh] || !m.vertex_indices || !m.points) {
                        *why = "prim " + std::to_string(k) + " vertex-index slot out of range";
                        return false;
                }
                Tri t;
                float *dst[3] = {t.p0, t.p1, t.p2};
                for (int c = 0; c < 3; ++c) {
                        const int64_t v = m.vertex_indices[base + c];
                        if (v < 0 || v * 4 + 3 > pts_counts_[mesh]) {
                                *why = "prim " + std::to_string(k) + " vertex " + std::to_string(v) + " out of range";
                                return false;
                        }
                        dst[c][0] = m.points[v * 4 + 0];
                        dst[c][1] = m.points[v * 4 + 1];
                        dst[c][2] = m.points[v * 4 + 2];
                }
                for (int a = 0; a < 3; ++a) {
                        t.lo[a] = std::min({t.p0[a], t.p1[a], t.p2[a]});
                        t.hi[a] = std::max({t.p0[a], t.p1[a], t.p2[a]});
                }
                t.prim = (int32_t)k;
                tris_.push_back(t);
                return true;
        }

        int32_t new_bin(const float lo[3], const float hi[3]) {
                BinNode b;
                std::memcpy(b.lo, lo, 12);
                std::memcpy(b.hi, hi, 12);
                bin_.push_back(b);
                return (int32_t)bin_.size() - 1;
        }

        // Balanced binary tree over chunks [first, first+count) of tris_ with <= 4 each.
        int32_t split_leaf(int64_t first, int64_t count) {
                if (count <= kLeafTris) {
                        float lo[3], hi[3];
                        for (int a = 0; a < 3; ++a) {
                                lo[a] = std::numeric_limits<float>::infinity();
                                hi[a] = -lo[a];
                        }
                        for (int64_t i = first; i < first + count; ++i) {
                                const Tri &t = tris_[i];
                                for (int a = 0; a < 3; ++a) {
                                        lo[a] = std::min(lo[a], t.lo[a]);
                                        hi[a] = std::max(hi[a], t.hi[a]);
                                }
                        }
                        int32_t id = new_bin(lo, hi);
                        bin_[id].tri_first = first;
                        bin_[id].tri_count = (int32_t)count;
                        return id;
                }
                int64_t chunks = (count + kLeafTris - 1) / kLeafTris;
                int64_t left = (chunks / 2) * kLeafTris;
                int32_t l = split_leaf(first, left);
                int32_t r = split_leaf(first + left, count - left);
                float lo[3], hi[3];
                for (int a = 0; a < 3; ++a) {
                        lo[a] = std::min(bin_[l].lo[a], bin_[r].lo[a]);
                        hi[a] = std::max(bin_[l].hi[a], bin_[r].hi[a]);
                }
                int32_t id = new_bin(lo, hi);
                bin_[id].l = l;
                bin_[id].r = r;
                return id;
        }

        // Validation + lift of the BVH2 (iterative post-order).
        gzg_status lift(int32_t *bvh2_depth) {
                if (node_count_ <= 0) return bad("empty BVH2");
                struct Frame {
                        int64_t node;
                        int depth;
                        int state;  // 0 = new, 1 = children done
                        int32_t l = -1, r = -1;
                };
                std::vector<Frame> st;
                std::vector<int32_t> results;  // converted ids, stack of return values
                st.push_back({0, 1, 0});
                int64_t visits = 0;
                int max_depth = 0;
                std::string why;
                while (!st.empty()) {
                        Frame &f = st.back();
                        const gzg_bvh2_node &n = nodes_[f.node];
                        if (f.state == 0) {
                                if (++visits > node_count_) return bad("BVH2 visits more nodes than it has");
                                max_depth = std::max(max_depth, f.depth);
                                if (n.count < 0) return bad("negative leaf count at node " + std::to_string(f.node));
                                if (n.count > 0) {
                                        if (n.offset < 0 || (int64_t)n.offset + n.count > prim_count_)
                                                return bad("leaf range out of prim array at node " + std::to_string(f.node));
                                        const int64_t first = (int64_t)tris_.size();
                                        for (int64_t k = n.offset; k < (int64_t)n.offset + n.count; ++k) {
                                                bool is_tri;
                                                if (!read_prim(k, &is_tri, &why)) return bad(why);
                                        }
                                        const int64_t cnt = (int64_t)tris_.size() - first;
                                        int32_t id = -1;
                                        if (cnt > 0 && cnt <= kLeafTris) {
                                                id = new_bin(n.bounds_min, n.bounds_max);
                                                bin_[id].tri_first = first;
                                                bin_[id].tri_count = (int32_t)cnt;
                                        } else if (cnt > kLeafTris) {
                                                id = split_leaf(first, cnt);
                                        }
                                        results.push_back(id);
                                        st.pop_back();
                                        continue;
                                }
                                const int64_t li = f.node + 1, ri = n.offset;
                                if (li >= node_count_ || ri <= li || ri >= node_count_)
                                        return bad("bad child link at node " + std::to_string(f.node));
                                f.state = 1;
                                const int d = f.depth + 1;
                                st.push_back({ri, d, 0});
                                st.push_back({li, d, 0});
                                continue;
                        }
                        // children done: results has [.., left, right]
                        int32_t r = results.back();
                        results.pop_back();
                        int32_t l = results.back();
                        results.pop_back();
                        int32_t id;
                        if (l < 0)
                                id = r;
                        else if (r < 0)
                                id = l;
                        else {
                                id = new_bin(n.bounds_min, n.bounds_max);
                                bin_[id].l = l;
                                bin_[id].r = r;
                        }
                        results.push_back(id);
                        st.pop_back();
                }
                bin_root_ = results.back();
                *bvh2_depth = max_depth;
                return GZG_OK;
        }

        static void quantise_axis(const float *clo, const float *chi, int n, float *p_out, uint8_t *e_out,
                                  uint8_t *qlo, uint8_t *qhi) {
                double lo = std::numeric_limits<double>::infinity(), hi = -lo;
                for (int i = 0; i < n; ++i) {
                        lo = std::min(lo, (double)clo[i]);
                        hi = std::max(hi, (double)chi[i]);
                }
                const double mag = std::max(std::fabs(lo), std::fabs(hi));
                double margin = std::ldexp(std::max(mag, hi - lo), -18);
                if (!(margin > 0)) margin = 1e-30;
                float p = (float)(lo - margin);
                while ((double)p > lo - margin) p = std::nextafter(p, -std::numeric_limits<float>::infinity());
                const double span = (hi + margin) - (double)p;
                int k = (int)std::ceil(std::log2(span / 255.0));
                k = std::max(k, -126);
                while (std::ldexp(255.0, k) < span) ++k;
                k = std::min(k, 127);
                const double s = std::ldexp(1.0, k);
                *p_out = p;
                *e_out = (uint8_t)(k + 127);
                for (int i = 0; i < n; ++i) {
                        double a = std::floor(((double)clo[i] - margin - p) / s);
                        double b = std::ceil(((double)chi[i] + margin - p) / s);
                        qlo[i] = (uint8_t)std::min(255.0, std::max(0.0, a));
                        qhi[i] = (uint8_t)std::min(255.0, std::max(0.0, b));
                }
        }

        // Greedy octant slot assignment: slot s wants the child farthest along
        // (+-1,+-1,+-1) with bit i of s set meaning +.
        static void assign_slots(const std::vector<int32_t> &kids, const std::vector<BinNode> &bin, int slot_of[8]) {
                const int n = (int)kids.size();
                double pc[3] = {0, 0, 0};
                double cc[8][3];
                for (int k = 0; k < n; ++k)
                        for (int a = 0; a < 3; ++a) {
                                cc[k][a] = 0.5 * ((double)bin[kids[k]].lo[a] + bin[kids[k]].hi[a]);
                                pc[a] += cc[k][a] / n;
                        }
                struct Pair {
                        double cost;
                        int k, s;
                };
                std::vector<Pair> pairs;
                for (int k = 0; k < n; ++k)
                        for (int s = 0; s < 8; ++s) {
                                double d = 0;
                                for (int a = 0; a < 3; ++a) d += (cc[k][a] - pc[a]) * ((s >> a) & 1 ? 1.0 : -1.0);
                                pairs.push_back({-d, k, s});
                        }
                std::stable_sort(pairs.begin(), pairs.end(), [](const Pair &x, const Pair &y) { return x.cost < y.cost; });
                bool kdone[8] = {false}, sdone[8] = {false};
                for (int k = 0; k < 8; ++k) slot_of[k] = -1;
                for (const Pair &pr : pairs) {
                        if (kdone[pr.k] || sdone[pr.s]) continue;
                        kdone[pr.k] = sdone[pr.s] = true;
                        slot_of[pr.k] = pr.s;
                }
        }

        // area_[8b + i - 1] = least summed surface area of the wide nodes
        // needed to represent the subtree of binary node b by at most i
        // children of a wide node: a leaf costs nothing, an interior node
        // kept as one child becomes a wide node (its area plus its subtree
        // spread over 8 children), an interior node spread over j >= 2
        // children costs the best split of j between its two subtrees.
        // pick_ records the choice (0 = one child, j = spread over j), split_
        // the share of the left subtree when spread over j.  Children come
        // before parents in bin_, so one pass in index order fills the tables.
        std::vector<double> area_;
        std::vector<uint8_t> pick_, split_;
        void collapse_tables() {
                const size_t nb = bin_.size();
                area_.assign(nb * 8, 0.0);
                pick_.assign(nb * 8, 0);
                split_.assign(nb * 8, 0);
                for (size_t b = 0; b < nb; ++b) {
                        const BinNode &c = bin_[b];
                        if (c.leaf()) continue;
                        const double *al = &area_[(size_t)c.l * 8], *ar = &area_[(size_t)c.r * 8];
                        double spread[9];
                        for (int j = 2; j <= 8; ++j) {
                                spread[j] = std::numeric_limits<double>::infinity();
                                for (int k = 1; k < j; ++k) {
                                        const double v = al[k - 1] + ar[j - k - 1];
                                        if (v < spread[j]) {
                                                spread[j] = v;
                                                split_[b * 8 + (j - 1)] = (uint8_t)k;
                                        }
                                }
                        }
                        double best = c.area() + spread[8];
                        int best_pick = 0;
                        area_[b * 8] = best;
                        for (int i = 2; i <= 8; ++i) {
                                if (spread[i] < best) {
                                        best = spread[i];
                                        best_pick = i;
                                }
                                area_[b * 8 + (i - 1)] = best;
                                pick_[b * 8 + (i - 1)] = (uint8_t)best_pick;
                        }
                }
        }
        // Appends the children that represent binary node b with at most i.
        void collapse_children(int32_t b, int i, std::vector<int32_t> &kids) const {
                const int p = pick_[(size_t)b * 8 + (i - 1)];
                if (bin_[b].leaf() || p == 0) {
                        kids.push_back(b);
                        return;
                }
                const int k = split_[(size_t)b * 8 + (p - 1)];
                collapse_children(bin_[b].l, k, kids);
                collapse_children(bin_[b].r, p - k, kids);
        }

        void collapse(WideBvh *out) {
                collapse_tables();
                out->nodes.clear();
                out->v0.clear();
                out->v1.clear();
                out->v2.clear();
                struct Job {
                        std::vector<int32_t> kids;
                        uint32_t node;
                        int depth;
                };
                // the children of the wide node rooted at binary node b: its
                // two subtrees spread over 8 children by the tables' best split
                auto open_kids = [&](int32_t b) {
                        std::vector<int32_t> kids;
                        if (b < 0) return kids;
                        if (bin_[b].leaf()) {
                                kids.push_back(b);
                                return kids;
                        }
                        const int k = split_[(size_t)b * 8 + 7];
                        collapse_children(bin_[b].l, k, kids);
                        collapse_children(bin_[b].r, 8 - k, kids);
                        return kids;
                };
                std::vector<Job> queue;
                out->nodes.push_back(WideNode{});
                queue.push_back({open_kids(bin_root_), 0, 1});
                int32_t depth = 1;
                for (size_t qi = 0; qi < queue.size(); ++qi) {
                        Job job = queue[qi];
                        depth = std::max(depth, job.depth);
                        WideNode w;
                        std::memset(&w, 0, sizeof(w));
                        const int n = (int)job.kids.size();
                        int slot_of[8];
                        assign_slots(job.kids, bin_, slot_of);
                        int kid_in_slot[8];
                        for (int s = 0; s < 8; ++s) kid_in_slot[s] = -1;
                        for (int k = 0; k < n; ++k) kid_in_slot[slot_of[k]] = k;
                        // quantisation
                        float clo[3][8], chi[3][8];
                        int m = 0;
                        int order[8];
                        for (int s = 0; s < 8; ++s)
                                if (kid_in_slot[s] >= 0) {
                                        const BinNode &c = bin_[job.kids[kid_in_slot[s]]];
                                        for (int a = 0; a < 3; ++a) {
                                                clo[a][m] = c.lo[a];
                                                chi[a][m] = c.hi[a];
                                        }
                                        order[m++] = s;
                                }
                        float pxyz[3] = {0, 0, 0};
                        uint8_t ee[3] = {127, 127, 127};
                        for (int a = 0; a < 3; ++a) {
                                uint8_t ql[8], qh[8];
                                if (m > 0) quantise_axis(clo[a], chi[a], m, &pxyz[a], &ee[a], ql, qh);
                                for (int s = 0; s < 8; ++s) {
                                        w.qlo[a][s] = 255;
                                        w.qhi[a][s] = 0;
                                }
                                for (int i = 0; i < m; ++i) {
                                        w.qlo[a][order[i]] = ql[i];
                                        w.qhi[a][order[i]] = qh[i];
                                }
                        }
                        w.px = pxyz[0];
                        w.py = pxyz[1];
                        w.pz = pxyz[2];
                        w.ex = ee[0];
                        w.ey = ee[1];
                        w.ez = ee[2];
                        // interior children: contiguous, slot order
                        w.child_base = (uint32_t)out->nodes.size();
                        w.tri_base = (uint32_t)out->v0.size();
                        uint32_t tri_off = 0;
                        for (int s = 0; s < 8; ++s) {
                                const int k = kid_in_slot[s];
                                if (k < 0) continue;
                                const BinNode &c = bin_[job.kids[k]];
                                if (!c.leaf()) {
                                        w.imask |= (uint8_t)(1u << s);
                                        out->nodes.push_back(WideNode{});
                                        std::vector<int32_t> kids = open_kids(job.kids[k]);
                                        queue.push_back({kids, (uint32_t)out->nodes.size() - 1, job.depth + 1});
                                } else {
                                        w.meta[s] = (uint8_t)(0x80u | ((uint32_t)(c.tri_count - 1) << 5) | tri_off);
                                        for (int32_t t = 0; t < c.tri_count; ++t) {
                                                const Tri &tr = tris_[c.tri_first + t];
                                                float4_ a{tr.p0[0], tr.p0[1], tr.p0[2], 0.0f};
                                                std::memcpy(&a.w, &tr.prim, 4);
                                                out->v0.push_back(a);
                                                out->v1.push_back(float4_{tr.p1[0], tr.p1[1], tr.p1[2], 0.0f});
                                                out->v2.push_back(float4_{tr.p2[0], tr.p2[1], tr.p2[2], 0.0f});
                                        }
                                        tri_off += (uint32_t)c.tri_count;
                                }
                        }
                        out->nodes[job.node] = w;
                }
                out->depth = depth;
        }
};

}  // namespace

gzg_status build_wide_bvh(const gzg_bvh2_node *nodes, int64_t node_count, const gzg_prim_id *prims,
                          int64_t prim_count, const gzg_triangle_mesh *meshes, int64_t mesh_count,
                          const int64_t *points_counts, const int64_t *vertex_index_counts, WideBvh *out,
                          int32_t *bvh2_depth) {
        Converter c(nodes, node_count, prims, prim_count, meshes, mesh_count, points_counts, vertex_index_counts);
        return c.run(out, bvh2_depth);
}

gzg_status build_wide_tlas(const gzg_bvh2_node *nodes, int64_t node_count, const int64_t *leaf_instance,
                           int64_t leaf_count, const float *inst_bounds, int64_t inst_count, WideBvh *out,
                           int32_t *bvh2_depth) {
        Converter c(nodes, node_count, leaf_instance, leaf_count, inst_bounds, inst_count);
        return c.run(out, bvh2_depth);
}

}  // namespace gzg
