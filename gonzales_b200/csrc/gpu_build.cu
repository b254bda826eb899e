// gpu_build.cu - builds a scene's 8-wide quantised tree on the device.
//
// The reference builds its BVH2 on the host with a binned SAH
// (Accelerators/BoundingHierarchyBuilder.swift:199-339); this is the device
// alternative for scenes that arrive without one (a linear BVH):
//   1. per prim: bounds, centroid, and the scene's centroid bounds
//      (order-preserving integer atomics);
//   2. a 64-bit key per intersectable prim: 30-bit Morton code of the
//      centroid in the upper half, the prim index in the lower half (unique
//      keys, a deterministic order); other prims sort last;
//   3. a radix sort of the keys (CUB);
//   4. the binary tree, by default the radix tree over the sorted keys
//      (Karras 2012: one thread per internal node finds its range and split
//      from common-prefix lengths) with node bounds computed bottom-up (one
//      thread per leaf; the second of two children to arrive at a node
//      computes it); or PLOC (Meister and Bittner 2018: clusters merge with
//      their mutual nearest neighbour in Morton order, then compact), whose
//      lower surface-area cost did not traverse faster on the ray-cast mesh;
//   5. (bounds come with the tree)
//   6. collapse into wide nodes level by level: a wide node opens the
//      interior child of largest surface area until it has 8 children (a
//      greedy choice: the host converter, wide_bvh.cpp, minimises the summed
//      node area over the whole subtree instead, which needs the finished
//      binary tree's tables before the first wide node); a binary node
//      covering at most leaf_size prims is a leaf; children go to octant
//      slots and their boxes are quantised outward to 8 bits per plane as
//      the host converter does.
// The result uses the host converter's layout exactly (WideNode, leaf-order
// triangle records with the prim index in v0.w), so every traversal kernel
// runs on it unchanged.
#include <cub/cub.cuh>
#include <math_constants.h>

#include <cmath>
#include <cstring>
#include <string>

#include "device.cuh"
#include "gzg_internal.h"

namespace gzg {
namespace {

gzg_status build_fail(cudaError_t e, const char *what) {
        const gzg_status code = (e == cudaErrorMemoryAllocation) ? GZG_ERR_OUT_OF_MEMORY : GZG_ERR_CUDA;
        return set_error(code, std::string("gzg_gpu_build_scene: ") + what + ": " + cudaGetErrorString(e));
}

#define GZG_CK(call, what)                                   \
        do {                                                 \
                cudaError_t e_ = (call);                     \
                if (e_ != cudaSuccess) return build_fail(e_, what); \
        } while (0)

constexpr uint64_t kInvalidKey = ~0ull;

// float <-> int keeping the order of all non-NaN floats
__device__ __forceinline__ int ord_int(float f) {
        const int i = __float_as_int(f);
        return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float ord_float(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

__device__ __forceinline__ bool prim_valid(const float4 &a) { return __float_as_int(a.w) == 1; }

// Prim bounds (lo in .xyz of box[2k], hi in box[2k+1]) and the centroid
// bounds (6 ordered ints: lo xyz, -hi xyz ... stored as min of lo and min of
// -hi so one atomicMin serves both).
__global__ void k_prim_bounds(const float4 *__restrict__ pv0, const float4 *__restrict__ pv1,
                              const float4 *__restrict__ pv2, int64_t n, float4 *__restrict__ box,
                              int *__restrict__ cb, unsigned long long *__restrict__ n_valid) {
        const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        float c[3] = {0, 0, 0};
        bool ok = false;
        if (k < n) {
                const float4 a = pv0[k], b = pv1[k], d = pv2[k];
                ok = prim_valid(a);
                const float lo[3] = {fminf(a.x, fminf(b.x, d.x)), fminf(a.y, fminf(b.y, d.y)), fminf(a.z, fminf(b.z, d.z))};
                const float hi[3] = {fmaxf(a.x, fmaxf(b.x, d.x)), fmaxf(a.y, fmaxf(b.y, d.y)), fmaxf(a.z, fmaxf(b.z, d.z))};
                box[2 * k] = make_float4(lo[0], lo[1], lo[2], 0.0f);
                box[2 * k + 1] = make_float4(hi[0], hi[1], hi[2], 0.0f);
                for (int i = 0; i < 3; ++i) c[i] = 0.5f * lo[i] + 0.5f * hi[i];
        }
        // block reduction of the centroid bounds of valid prims
        typedef cub::BlockReduce<int, 256> Reduce;
        __shared__ typename Reduce::TempStorage tmp;
        __shared__ int res[6];
        unsigned cnt = __syncthreads_count(ok ? 1 : 0);
        for (int i = 0; i < 6; ++i) {
                const int v = ok ? (i < 3 ? ord_int(c[i]) : ord_int(-c[i - 3])) : INT_MAX;
                const int r = Reduce(tmp).Reduce(v, cub::Min());
                if (threadIdx.x == 0) res[i] = r;
                __syncthreads();
        }
        if (threadIdx.x == 0) {
                for (int i = 0; i < 6; ++i)
                        if (res[i] != INT_MAX) atomicMin(cb + i, res[i]);
                if (cnt) atomicAdd(n_valid, (unsigned long long)cnt);
        }
}

// Spreads the low 10 bits of v to every third bit.
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
        v &= 0x3FFu;
        v = (v | (v << 16)) & 0x030000FFu;
        v = (v | (v << 8)) & 0x0300F00Fu;
        v = (v | (v << 4)) & 0x030C30C3u;
        v = (v | (v << 2)) & 0x09249249u;
        return v;
}

__global__ void k_keys(const float4 *__restrict__ pv0, const float4 *__restrict__ box, int64_t n,
                       const int *__restrict__ cb, uint64_t *__restrict__ keys) {
        const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (k >= n) return;
        if (!prim_valid(pv0[k])) {
                keys[k] = kInvalidKey;
                return;
        }
        const float4 lo = box[2 * k], hi = box[2 * k + 1];
        const float c[3] = {0.5f * lo.x + 0.5f * hi.x, 0.5f * lo.y + 0.5f * hi.y, 0.5f * lo.z + 0.5f * hi.z};
        uint32_t q[3];
        for (int i = 0; i < 3; ++i) {
                const float a = ord_float(cb[i]), b = -ord_float(cb[3 + i]);
                const float ext = b - a;
                float t = ext > 0.0f ? (c[i] - a) / ext : 0.0f;
                t = fminf(fmaxf(t, 0.0f), 1.0f);
                q[i] = (uint32_t)fminf(t * 1024.0f, 1023.0f);
        }
        const uint32_t m = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
        keys[k] = ((uint64_t)m << 32) | (uint64_t)(uint32_t)k;
}

// Common-prefix length of sorted keys i and j (-1 outside [0, m)).
__device__ __forceinline__ int prefix(const uint64_t *__restrict__ k, int m, int i, int j) {
        if (j < 0 || j >= m) return -1;
        return __clzll(k[i] ^ k[j]);
}

// Binary radix tree: internal node i (0 .. m-2) gets children (>= 0:
// internal node, < 0: ~leaf) and the number of prims under it.
__global__ void k_radix_tree(const uint64_t *__restrict__ keys, const unsigned long long *__restrict__ m_dev,
                             int2 *__restrict__ child, int *__restrict__ count, int *__restrict__ parent_int,
                             int *__restrict__ parent_leaf) {
        const int m = (int)*m_dev;
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= m - 1) return;
        const int d = prefix(keys, m, i, i + 1) - prefix(keys, m, i, i - 1) >= 0 ? 1 : -1;
        const int dmin = prefix(keys, m, i, i - d);
        int lmax = 2;
        while (prefix(keys, m, i, i + lmax * d) > dmin) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
                if (prefix(keys, m, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = prefix(keys, m, i, j);
        int s = 0, t = l;
        do {
                t = (t + 1) >> 1;
                if (prefix(keys, m, i, i + (s + t) * d) > dnode) s += t;
        } while (t > 1);
        const int gamma = i + s * d + min(d, 0);
        const int first = min(i, j), last = max(i, j);
        const int left = first == gamma ? ~gamma : gamma;
        const int right = last == gamma + 1 ? ~(gamma + 1) : gamma + 1;
        child[i] = make_int2(left, right);
        count[i] = last - first + 1;
        if (left >= 0)
                parent_int[left] = i;
        else
                parent_leaf[~left] = i;
        if (right >= 0)
                parent_int[right] = i;
        else
                parent_leaf[~right] = i;
}

__device__ __forceinline__ void code_box(int code, const float4 *__restrict__ nbox, const float4 *__restrict__ pbox,
                                         const uint64_t *__restrict__ keys, float4 &lo, float4 &hi) {
        if (code >= 0) {
                lo = __ldcg(nbox + 2 * code);
                hi = __ldcg(nbox + 2 * code + 1);
        } else {
                const uint32_t p = (uint32_t)(keys[~code] & 0xFFFFFFFFu);
                lo = pbox[2 * (size_t)p];
                hi = pbox[2 * (size_t)p + 1];
        }
}

// Bottom-up node bounds: one thread per leaf climbs while it is the second
// child to arrive.  Every climb ends (each node admits one second arrival).
__global__ void k_refit(const uint64_t *__restrict__ keys, const unsigned long long *__restrict__ m_dev,
                        const int2 *__restrict__ child, const int *__restrict__ parent_int,
                        const int *__restrict__ parent_leaf, const float4 *__restrict__ pbox, float4 *__restrict__ nbox,
                        int *__restrict__ arrivals) {
        const int m = (int)*m_dev;
        const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
        if (leaf >= m || m < 2) return;
        int node = parent_leaf[leaf];
        for (int guard = 0; guard < m && node >= 0; ++guard) {
                __threadfence();
                if (atomicAdd(arrivals + node, 1) == 0) return;
                const int2 c = child[node];
                float4 l0, h0, l1, h1;
                code_box(c.x, nbox, pbox, keys, l0, h0);
                code_box(c.y, nbox, pbox, keys, l1, h1);
                nbox[2 * node] = make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.0f);
                nbox[2 * node + 1] = make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.0f);
                node = node == 0 ? -1 : parent_int[node];
        }
}

// ---- PLOC (Meister & Bittner 2018): clusters in Morton order repeatedly
// merge with their mutual nearest neighbour (surface area of the union box)
// within a window of +-radius, then the survivors are compacted.
struct alignas(16) Cluster {
        float lo[3];
        int code;  // >= 0 internal node, < 0 ~(sorted leaf position)
        float hi[3];
        int cnt;   // prims under the cluster
};

__device__ __forceinline__ float union_area(const Cluster &a, const Cluster &b) {
        const float x = fmaxf(a.hi[0], b.hi[0]) - fminf(a.lo[0], b.lo[0]);
        const float y = fmaxf(a.hi[1], b.hi[1]) - fminf(a.lo[1], b.lo[1]);
        const float z = fmaxf(a.hi[2], b.hi[2]) - fminf(a.lo[2], b.lo[2]);
        return x * y + x * z + y * z;
}

__global__ void k_ploc_init(const uint64_t *__restrict__ keys, const unsigned long long *__restrict__ m_dev,
                            const float4 *__restrict__ pbox, Cluster *__restrict__ cl) {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= (int)*m_dev) return;
        const uint32_t p = (uint32_t)(keys[i] & 0xFFFFFFFFu);
        const float4 lo = pbox[2 * (size_t)p], hi = pbox[2 * (size_t)p + 1];
        Cluster c;
        c.lo[0] = lo.x;
        c.lo[1] = lo.y;
        c.lo[2] = lo.z;
        c.hi[0] = hi.x;
        c.hi[1] = hi.y;
        c.hi[2] = hi.z;
        c.code = ~i;
        c.cnt = 1;
        cl[i] = c;
}

// nearest neighbour in the window (ties to the lower index); force: pair
// 2k with 2k + 1 (used after an iteration without a merge)
__global__ void k_ploc_nn(const Cluster *__restrict__ cl, int count, int radius, int force, int *__restrict__ nn) {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= count) return;
        if (force) {
                nn[i] = (i ^ 1) < count ? (i ^ 1) : i;
                return;
        }
        const Cluster a = cl[i];
        float best = CUDART_INF_F;
        int bj = i;
        const int j0 = max(0, i - radius), j1 = min(count - 1, i + radius);
        for (int j = j0; j <= j1; ++j) {
                if (j == i) continue;
                const float d = union_area(a, cl[j]);
                if (d < best) {
                        best = d;
                        bj = j;
                }
        }
        nn[i] = bj;
}

__global__ void k_ploc_merge(Cluster *__restrict__ cl, const int *__restrict__ nn, int count,
                             uint32_t *__restrict__ node_counter, uint32_t node_cap, int2 *__restrict__ child,
                             int *__restrict__ ncount, float4 *__restrict__ nbox, int *__restrict__ keep,
                             uint32_t *__restrict__ err) {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= count) return;
        const int j = nn[i];
        const bool mutual = j != i && nn[j] == i;
        if (!mutual) {
                keep[i] = 1;
                return;
        }
        if (i > j) {
                keep[i] = 0;
                return;
        }
        const uint32_t node = atomicAdd(node_counter, 1u);
        if (node >= node_cap) {
                atomicOr(err, 1u);
                keep[i] = 1;
                return;
        }
        const Cluster a = cl[i], b = cl[j];
        Cluster c;
        for (int k = 0; k < 3; ++k) {
                c.lo[k] = fminf(a.lo[k], b.lo[k]);
                c.hi[k] = fmaxf(a.hi[k], b.hi[k]);
        }
        c.code = (int)node;
        c.cnt = a.cnt + b.cnt;
        child[node] = make_int2(a.code, b.code);
        ncount[node] = c.cnt;
        nbox[2 * node] = make_float4(c.lo[0], c.lo[1], c.lo[2], 0.0f);
        nbox[2 * node + 1] = make_float4(c.hi[0], c.hi[1], c.hi[2], 0.0f);
        cl[i] = c;
        keep[i] = 1;
}

struct Tree {
        const uint64_t *keys;
        const unsigned long long *m_dev;  // intersectable prims (sorted first)
        const int2 *child;
        const int *count;                 // prims under each internal node
        const float4 *nbox, *pbox;
        const float4 *pv0, *pv1, *pv2;
        int leaf_size;
        const int *root;                  // the root's code
};

__device__ __forceinline__ int code_count(const Tree &t, int code) { return code < 0 ? 1 : t.count[code]; }

// The sorted-key positions of the leaves under a code (at most 4), left to
// right.
__device__ int code_leaves(const Tree &t, int code, int out[4]) {
        int stack[8], sp = 0, n = 0;
        stack[sp++] = code;
        while (sp > 0 && n < 4) {
                const int c = stack[--sp];
                if (c < 0) {
                        out[n++] = ~c;
                } else if (sp + 2 <= 8) {
                        const int2 ch = t.child[c];
                        stack[sp++] = ch.y;
                        stack[sp++] = ch.x;
                }
        }
        return n;
}
__device__ __forceinline__ bool code_leaf(const Tree &t, int code) { return code_count(t, code) <= t.leaf_size; }
__device__ __forceinline__ void code_bounds(const Tree &t, int code, double lo[3], double hi[3]) {
        float4 l, h;
        code_box(code, t.nbox, t.pbox, t.keys, l, h);
        lo[0] = l.x;
        lo[1] = l.y;
        lo[2] = l.z;
        hi[0] = h.x;
        hi[1] = h.y;
        hi[2] = h.z;
}
__device__ __forceinline__ double code_area(const Tree &t, int code) {
        double lo[3], hi[3];
        code_bounds(t, code, lo, hi);
        const double x = hi[0] - lo[0], y = hi[1] - lo[1], z = hi[2] - lo[2];
        return 2.0 * (x * y + x * z + y * z);
}

// quantise_axis of wide_bvh.cpp on the device (same arithmetic in double),
// in two parts: the axis's grid from the extent [lo, hi] of the node's
// children (origin p rounded down to a float, exponent e, margin, step), and
// one child plane quantised outward on that grid.
__device__ void axis_grid(double lo, double hi, float *p_out, int *e_out, double *margin_out, double *step_out) {
        const double mag = fmax(fabs(lo), fabs(hi));
        double margin = ldexp(fmax(mag, hi - lo), -18);
        if (!(margin > 0)) margin = 1e-30;
        float p = (float)(lo - margin);
        while ((double)p > lo - margin) p = nextafterf(p, -CUDART_INF_F);
        const double span = (hi + margin) - (double)p;
        int k = (int)ceil(log2(span / 255.0));
        k = max(k, -126);
        while (ldexp(255.0, k) < span) ++k;
        k = min(k, 127);
        *p_out = p;
        *e_out = k + 127;
        *margin_out = margin;
        *step_out = ldexp(1.0, k);
}

__device__ __forceinline__ uint8_t quantise_lo(double v, double margin, float p, double step) {
        return (uint8_t)fmin(255.0, fmax(0.0, floor((v - margin - (double)p) / step)));
}
__device__ __forceinline__ uint8_t quantise_hi(double v, double margin, float p, double step) {
        return (uint8_t)fmin(255.0, fmax(0.0, ceil((v + margin - (double)p) / step)));
}

constexpr int kRootItem = INT_MIN;  // the root's code, resolved on the device

// Reductions within an aligned group of 8 lanes (one wide node per group);
// every lane of the group gets the result.  argmax / argmin keep the lowest
// lane on ties.
__device__ __forceinline__ int g8_argmax(double v, int idx, double *best) {
#pragma unroll
        for (int off = 4; off > 0; off >>= 1) {
                const double ov = __shfl_xor_sync(0xFFFFFFFFu, v, off);
                const int oi = __shfl_xor_sync(0xFFFFFFFFu, idx, off);
                if (ov > v || (ov == v && oi < idx)) {
                        v = ov;
                        idx = oi;
                }
        }
        *best = v;
        return idx;
}
__device__ __forceinline__ int g8_argmin(float v, int idx, float *best) {
#pragma unroll
        for (int off = 4; off > 0; off >>= 1) {
                const float ov = __shfl_xor_sync(0xFFFFFFFFu, v, off);
                const int oi = __shfl_xor_sync(0xFFFFFFFFu, idx, off);
                if (ov < v || (ov == v && oi < idx)) {
                        v = ov;
                        idx = oi;
                }
        }
        *best = v;
        return idx;
}
__device__ __forceinline__ uint32_t g8_or(uint32_t v) {
#pragma unroll
        for (int off = 4; off > 0; off >>= 1) v |= __shfl_xor_sync(0xFFFFFFFFu, v, off);
        return v;
}
__device__ __forceinline__ uint32_t g8_sum(uint32_t v) {
#pragma unroll
        for (int off = 4; off > 0; off >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, off);
        return v;
}

// One level of the collapse, one group of 8 lanes per item (binary code, wide
// node index), four items per warp, with the serial loops of one node spread
// over the group's lanes (lane j of a group = child j or slot j):
//   - lane j < n holds child j while the node opens the interior child of
//     largest surface area (lowest index on ties) until it has 8 children;
//   - lane j loads child j's box and its 8 slot costs; each of n rounds gives
//     the lowest remaining cost (lowest child, then lowest slot, on ties) its
//     slot;
//   - lane s quantises the three axes of the child in slot s;
//   - lane j writes child j's slot fields and copies its triangles.
// The node is assembled in shared memory and stored as five 16-byte words.
// Every loop runs a fixed 8 steps (or until no group of the warp is still
// opening children) so that all 32 lanes take every shuffle.  One thread per
// node took about 85 us per node at the top of the tree (a chain of dependent
// loads and local-memory loops), so every level cost at least that however few
// nodes it held; a whole warp per node left most lanes idle on the wide levels.
__global__ void __launch_bounds__(128) k_collapse(Tree t, const int2 *__restrict__ items,
                                                  const uint32_t *__restrict__ n_items, int2 *__restrict__ next,
                                                  uint32_t *__restrict__ n_next, uint32_t *__restrict__ counters,
                                                  WideNode *__restrict__ nodes, float4 *__restrict__ tv0,
                                                  float4 *__restrict__ tv1, float4 *__restrict__ tv2, uint32_t node_cap,
                                                  uint32_t tri_cap, uint32_t *__restrict__ err) {
        const unsigned FULL = 0xFFFFFFFFu;
        __shared__ __align__(16) unsigned char s_node[16][80];
        const int lane = (int)(threadIdx.x & 31u);
        const int j = lane & 7;             // child / slot index within the group
        const int base = lane & ~7;         // the group's first lane
        unsigned char *wn = s_node[threadIdx.x >> 3];
        const uint32_t first = (blockIdx.x * blockDim.x + (threadIdx.x & ~31u)) >> 3;  // the warp's first item
        const uint32_t count = *n_items;
        if (first >= count) return;  // whole warps
        const uint32_t it = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
        const bool valid = it < count;
        const int m = (int)*t.m_dev;
        int2 item = valid ? items[it] : make_int2(0, 0);
        if (valid && item.x == kRootItem) item.x = m >= 2 ? *t.root : ~0;

        // ---- children: open the largest interior child until there are 8
        int kid = 0;
        double area = -1.0;  // -1: a leaf (never opened)
        int n = 0;
        bool opening = false;
        if (!valid || m == 0) {
                n = 0;
        } else if (code_leaf(t, item.x)) {
                kid = item.x;
                n = 1;
        } else {
                const int2 c = t.child[item.x];
                kid = j == 0 ? c.x : c.y;
                if (j < 2) area = code_leaf(t, kid) ? -1.0 : code_area(t, kid);
                n = 2;
                opening = true;
        }
        while (__any_sync(FULL, opening)) {
                double best_a;
                const int best = g8_argmax(opening && j < n ? area : -1.0, j, &best_a);
                if (!(best_a > -1.0)) opening = false;
                const int best_kid = __shfl_sync(FULL, kid, base + best);
                const int up_kid = __shfl_up_sync(FULL, kid, 1, 8);
                const double up_area = __shfl_up_sync(FULL, area, 1, 8);
                if (opening) {
                        const int2 c2 = t.child[best_kid];
                        if (j == best || j == best + 1) {
                                kid = j == best ? c2.x : c2.y;
                                area = code_leaf(t, kid) ? -1.0 : code_area(t, kid);
                        } else if (j > best + 1) {
                                kid = up_kid;
                                area = up_area;
                        }
                        ++n;
                        if (n == 8) opening = false;
                }
        }
        const bool mine = j < n;  // this lane holds a child

        // ---- boxes, centroid of the child centres (summed in child order)
        double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, term[3] = {0, 0, 0};
        if (mine) {
                code_bounds(t, kid, lo, hi);
                for (int a = 0; a < 3; ++a) term[a] = 0.5 * (lo[a] + hi[a]) / n;
        }
        double pc[3] = {0, 0, 0};
#pragma unroll
        for (int k = 0; k < 8; ++k)
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                        const double v = __shfl_sync(FULL, term[a], base + k);
                        if (k < n) pc[a] += v;
                }

        // ---- slots: slot s takes the child farthest along (+-1, +-1, +-1)
        float cost[8];
        {
                float cc[3];
                for (int a = 0; a < 3; ++a) cc[a] = mine ? (float)(0.5 * (lo[a] + hi[a]) - pc[a]) : 0.0f;
#pragma unroll
                for (int s2 = 0; s2 < 8; ++s2)
                        cost[s2] = -((s2 & 1 ? cc[0] : -cc[0]) + (s2 & 2 ? cc[1] : -cc[1]) + (s2 & 4 ? cc[2] : -cc[2]));
        }
        int my_slot = -1;
        unsigned sfree = 0xFFu;
        bool assigning = true;
#pragma unroll 1
        for (int round = 0; round < 8; ++round) {
                float lb = CUDART_INF_F;
                int ls = -1;
                if (mine && my_slot < 0) {
#pragma unroll
                        for (int s2 = 0; s2 < 8; ++s2)
                                if (((sfree >> s2) & 1u) && cost[s2] < lb) {
                                        lb = cost[s2];
                                        ls = s2;
                                }
                }
                float best_c;
                const int bk = g8_argmin(lb, j, &best_c);
                const int bs = __shfl_sync(FULL, ls, base + bk);
                if (round >= n || !(best_c < CUDART_INF_F)) assigning = false;
                if (assigning) {
                        if (j == bk) my_slot = bs;
                        sfree &= ~(1u << bs);
                }
        }
        // slot -> child + 1, four bits per slot
        const uint32_t slot_map = g8_or((mine && my_slot >= 0) ? (uint32_t)(j + 1) << (4 * my_slot) : 0u);

        // ---- zero the record, then quantise: lane s, three axes of slot s
        if (j < 5) reinterpret_cast<uint4 *>(wn)[j] = make_uint4(0u, 0u, 0u, 0u);
        __syncwarp();
        {
                const int k_in = (int)((slot_map >> (4 * j)) & 0xFu) - 1;  // child in slot j, or -1
                const int src = base + (k_in >= 0 ? k_in : 0);
#pragma unroll 1
                for (int a = 0; a < 3; ++a) {
                        // the axis's extent over every placed child
                        double alo = CUDART_INF, ahi = -CUDART_INF;
                        int nq = 0;
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                                const double l = __shfl_sync(FULL, a == 0 ? lo[0] : (a == 1 ? lo[1] : lo[2]), base + k);
                                const double h = __shfl_sync(FULL, a == 0 ? hi[0] : (a == 1 ? hi[1] : hi[2]), base + k);
                                const int ks = __shfl_sync(FULL, my_slot, base + k);
                                if (k < n && ks >= 0) {  // child k has a slot
                                        ++nq;
                                        alo = fmin(alo, l);
                                        ahi = fmax(ahi, h);
                                }
                        }
                        float p = 0.0f;
                        int e = 127;
                        double margin = 0.0, step = 1.0;
                        if (nq > 0) axis_grid(alo, ahi, &p, &e, &margin, &step);
                        const double cl = __shfl_sync(FULL, a == 0 ? lo[0] : (a == 1 ? lo[1] : lo[2]), src);
                        const double ch = __shfl_sync(FULL, a == 0 ? hi[0] : (a == 1 ? hi[1] : hi[2]), src);
                        uint8_t ql = 255, qh = 0;
                        if (k_in >= 0) {
                                ql = quantise_lo(cl, margin, p, step);
                                qh = quantise_hi(ch, margin, p, step);
                        }
                        wn[32 + 8 * a + j] = ql;
                        wn[56 + 8 * a + j] = qh;
                        if (j == 0) {
                                reinterpret_cast<float *>(wn)[a] = p;
                                wn[12 + a] = (uint8_t)e;
                        }
                }
        }

        // ---- interior children, leaf triangles
        const bool is_leaf = mine && code_leaf(t, kid);
        const bool is_int = mine && my_slot >= 0 && !is_leaf;
        int leaves[4];
        int cnt = 0;
        if (is_leaf && my_slot >= 0) cnt = code_leaves(t, kid, leaves);
        const uint32_t imask = g8_or(is_int ? 1u << my_slot : 0u);
        const uint32_t n_int = (uint32_t)__popc(imask);
        const uint32_t n_tri = g8_sum(is_leaf ? (uint32_t)code_count(t, kid) : 0u);
        uint32_t cbase = 0u, tbase = 0u, qbase = 0u;
        int overflow = valid ? 0 : 1;
        if (j == 0 && valid) {
                cbase = n_int ? atomicAdd(counters + 0, n_int) : 0u;
                tbase = n_tri ? atomicAdd(counters + 1, n_tri) : 0u;
                if (cbase + n_int > node_cap || tbase + n_tri > tri_cap) {
                        atomicOr(err, kErrBadIndex);
                        overflow = 1;
                } else if (n_int) {
                        qbase = atomicAdd(n_next, n_int);
                }
        }
        overflow = __shfl_sync(FULL, overflow, base);
        cbase = __shfl_sync(FULL, cbase, base);
        tbase = __shfl_sync(FULL, tbase, base);
        qbase = __shfl_sync(FULL, qbase, base);
        // a leaf child's triangles follow those of the leaf children in lower slots
        uint32_t tri_off = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
                const int ks = __shfl_sync(FULL, my_slot, base + k);
                const int kc = __shfl_sync(FULL, cnt, base + k);
                if (k < n && ks >= 0 && ks < my_slot) tri_off += (uint32_t)kc;
        }
        if (!overflow) {
                if (j == 0) {
                        wn[15] = (uint8_t)imask;
                        reinterpret_cast<uint32_t *>(wn)[4] = cbase;
                        reinterpret_cast<uint32_t *>(wn)[5] = tbase;
                }
                if (is_int) {
                        const uint32_t rank = (uint32_t)__popc(imask & ((1u << my_slot) - 1u));
                        next[qbase + rank] = make_int2(kid, (int)(cbase + rank));
                }
                if (cnt > 0) {
                        wn[24 + my_slot] = (uint8_t)(0x80u | ((uint32_t)(cnt - 1) << 5) | tri_off);
                        for (int q = 0; q < cnt; ++q) {
                                const uint32_t pidx = (uint32_t)(t.keys[leaves[q]] & 0xFFFFFFFFu);
                                float4 va = t.pv0[pidx];
                                va.w = __int_as_float((int)pidx);
                                float4 vb = t.pv1[pidx], vc = t.pv2[pidx];
                                vb.w = 0.0f;
                                vc.w = 0.0f;
                                tv0[tbase + tri_off + q] = va;
                                tv1[tbase + tri_off + q] = vb;
                                tv2[tbase + tri_off + q] = vc;
                        }
                }
        }
        __syncwarp();
        if (!overflow && j < 5) reinterpret_cast<uint4 *>(nodes + item.y)[j] = reinterpret_cast<const uint4 *>(wn)[j];
}

template <class T>
cudaError_t dalloc(T **p, size_t count, std::vector<void *> &tmp) {
        void *d = nullptr;
        cudaError_t e = cudaMalloc(&d, std::max<size_t>(count * sizeof(T), 16));
        if (e == cudaSuccess) tmp.push_back(d);
        *p = reinterpret_cast<T *>(d);
        return e;
}

}  // namespace

gzg_status gpu_build_wide(const float4_ *pv0, const float4_ *pv1, const float4_ *pv2, int64_t n, int leaf_size,
                          int builder, int radius, GpuWide *out, float *device_ms) {
        std::vector<void *> tmp;
        struct Free {
                std::vector<void *> &v;
                ~Free() {
                        for (void *p : v) cudaFree(p);
                }
        } free_tmp{tmp};
        *out = GpuWide{};
        if (n < 0 || n >= INT32_MAX) return set_error(GZG_ERR_LIMIT, "gzg_gpu_build_scene: prim count out of range");
        if (leaf_size < 1 || leaf_size > 4) leaf_size = 1;
        if (radius < 1 || radius > 64) radius = 16;
        const bool ploc = builder == GZG_BUILD_PLOC;
        cudaStream_t st = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        uint32_t *pinned = nullptr;  // level counts read back each level
        GZG_CK(cudaMallocHost(reinterpret_cast<void **>(&pinned), 16), "build: host counters");
        struct Ev {
                cudaEvent_t a, b;
                uint32_t *h;
                ~Ev() {
                        if (a) cudaEventDestroy(a);
                        if (b) cudaEventDestroy(b);
                        if (h) cudaFreeHost(h);
                }
        } ev{e0, e1, pinned};
        const float4 *d0 = reinterpret_cast<const float4 *>(pv0), *d1 = reinterpret_cast<const float4 *>(pv1),
                     *d2 = reinterpret_cast<const float4 *>(pv2);
        // every buffer up front (the intersectable count m <= n is known only
        // on the device), so the timed build holds no allocation
        const size_t N = (size_t)std::max<int64_t>(n, 1);
        float4 *pbox, *nbox;
        int *cb, *parent_int, *parent_leaf, *arrivals;
        unsigned long long *nvalid;
        uint64_t *keys, *sorted;
        int2 *child, *qa, *qb;
        int *ncount, *nn, *keep, *root, *n_sel;
        Cluster *ca, *cl_b;
        uint32_t *counts, *err;  // counts: [0] nodes used, [1] tris used, [2] items in, [3] items out
        GZG_CK(dalloc(&pbox, 2 * N, tmp), "build: prim bounds");
        GZG_CK(dalloc(&nbox, 2 * N, tmp), "build: node bounds");
        GZG_CK(dalloc(&cb, 6, tmp), "build: centroid bounds");
        GZG_CK(dalloc(&nvalid, 1, tmp), "build: prim count");
        GZG_CK(dalloc(&keys, N, tmp), "build: keys");
        GZG_CK(dalloc(&sorted, N, tmp), "build: keys");
        GZG_CK(dalloc(&child, N, tmp), "build: radix tree");
        GZG_CK(dalloc(&ncount, N, tmp), "build: radix tree");
        GZG_CK(dalloc(&root, 1, tmp), "build: root");
        GZG_CK(dalloc(&n_sel, 1, tmp), "build: cluster count");
        size_t sel_bytes = 0;
        if (ploc) {
                GZG_CK(dalloc(&ca, N, tmp), "build: clusters");
                GZG_CK(dalloc(&cl_b, N, tmp), "build: clusters");
                GZG_CK(dalloc(&nn, N, tmp), "build: clusters");
                GZG_CK(dalloc(&keep, N, tmp), "build: clusters");
                cub::DeviceSelect::Flagged(nullptr, sel_bytes, ca, keep, cl_b, n_sel, (int)N, st);
        }
        uint8_t *sel_temp;
        GZG_CK(dalloc(&sel_temp, sel_bytes, tmp), "build: cluster compaction scratch");
        GZG_CK(dalloc(&parent_int, N, tmp), "build: radix tree");
        GZG_CK(dalloc(&parent_leaf, N, tmp), "build: radix tree");
        GZG_CK(dalloc(&arrivals, N, tmp), "build: radix tree");
        GZG_CK(dalloc(&qa, N, tmp), "build: queue");
        GZG_CK(dalloc(&qb, N, tmp), "build: queue");
        GZG_CK(dalloc(&counts, 4, tmp), "build: counters");
        GZG_CK(dalloc(&err, 1, tmp), "build: error word");
        size_t temp_bytes = 0;
        if (n > 0) cub::DeviceRadixSort::SortKeys(nullptr, temp_bytes, keys, sorted, (int)n, 0, 64, st);
        uint8_t *temp;
        GZG_CK(dalloc(&temp, temp_bytes, tmp), "build: sort scratch");
        // outputs, at most one wide node per binary internal node (and the
        // root), one record per prim
        WideNode *nodes;
        float4 *tv0, *tv1, *tv2;
        GZG_CK(cudaMalloc(reinterpret_cast<void **>(&nodes), N * sizeof(WideNode)), "build: wide nodes");
        out->nodes = nodes;
        GZG_CK(cudaMalloc(reinterpret_cast<void **>(&tv0), N * sizeof(float4)), "build: triangles");
        out->tv0 = tv0;
        GZG_CK(cudaMalloc(reinterpret_cast<void **>(&tv1), N * sizeof(float4)), "build: triangles");
        out->tv1 = tv1;
        GZG_CK(cudaMalloc(reinterpret_cast<void **>(&tv2), N * sizeof(float4)), "build: triangles");
        out->tv2 = tv2;

        cudaEventRecord(e0, st);
        const int B = 256;
        const unsigned grid = (unsigned)((N + B - 1) / B);
        GZG_CK(cudaMemsetAsync(cb, 0x7F, 6 * sizeof(int), st), "build: reset");
        GZG_CK(cudaMemsetAsync(nvalid, 0, sizeof(unsigned long long), st), "build: reset");
        GZG_CK(cudaMemsetAsync(arrivals, 0, N * sizeof(int), st), "build: reset");
        const uint32_t init[4] = {1u, 0u, 1u, 0u};  // the root is node 0
        std::memcpy(pinned, init, sizeof(init));
        GZG_CK(cudaMemcpyAsync(counts, pinned, sizeof(init), cudaMemcpyHostToDevice, st), "build: counters");
        GZG_CK(cudaMemsetAsync(err, 0, 4, st), "build: error word");
        const int2 root_item = make_int2(kRootItem, 0);
        GZG_CK(cudaMemcpyAsync(qa, &root_item, sizeof(root_item), cudaMemcpyHostToDevice, st), "build: queue");
        if (n > 0) {
                k_prim_bounds<<<grid, B, 0, st>>>(d0, d1, d2, n, pbox, cb, nvalid);
                k_keys<<<grid, B, 0, st>>>(d0, pbox, n, cb, keys);
                GZG_CK(cub::DeviceRadixSort::SortKeys(temp, temp_bytes, keys, sorted, (int)n, 0, 64, st), "build: sort");
        }
        GZG_CK(cudaMemsetAsync(root, 0, sizeof(int), st), "build: root");
        if (n > 0 && !ploc) {
                k_radix_tree<<<grid, B, 0, st>>>(sorted, nvalid, child, ncount, parent_int, parent_leaf);
                k_refit<<<grid, B, 0, st>>>(sorted, nvalid, child, parent_int, parent_leaf, pbox, nbox, arrivals);
        } else if (n > 0) {
                unsigned long long hm = 0;
                GZG_CK(cudaMemcpyAsync(&hm, nvalid, sizeof(hm), cudaMemcpyDeviceToHost, st), "build: prim count");
                GZG_CK(cudaStreamSynchronize(st), "build: prim count");
                int count = (int)hm;
                k_ploc_init<<<grid, B, 0, st>>>(sorted, nvalid, pbox, ca);
                uint32_t *node_counter = counts + 3;  // borrowed until the collapse
                GZG_CK(cudaMemsetAsync(node_counter, 0, 4, st), "build: counters");
                int force = 0, iters = 0;
                while (count > 1) {
                        if (++iters > 4 * (int)hm + 64)
                                return set_error(GZG_ERR_KERNEL_FAULT, "gzg_gpu_build_scene: clustering did not converge");
                        const unsigned g = (unsigned)((count + B - 1) / B);
                        k_ploc_nn<<<g, B, 0, st>>>(ca, count, radius, force, nn);
                        k_ploc_merge<<<g, B, 0, st>>>(ca, nn, count, node_counter, (uint32_t)N, child, ncount, nbox, keep,
                                                       err);
                        GZG_CK(cub::DeviceSelect::Flagged(sel_temp, sel_bytes, ca, keep, cl_b, n_sel, count, st),
                               "build: cluster compaction");
                        GZG_CK(cudaMemcpyAsync(pinned + 3, n_sel, 4, cudaMemcpyDeviceToHost, st), "build: cluster count");
                        GZG_CK(cudaStreamSynchronize(st), "build: clustering");
                        const int next = (int)pinned[3];
                        force = next == count;  // no mutual pair this time: pair neighbours next
                        count = next;
                        std::swap(ca, cl_b);
                }
                GZG_CK(cudaMemcpyAsync(root, &ca[0].code, sizeof(int), cudaMemcpyDeviceToDevice, st), "build: root");
                // the collapse's counters start here
                GZG_CK(cudaMemcpyAsync(counts, pinned, 16, cudaMemcpyHostToDevice, st), "build: counters");
        }
        const uint32_t cap = (uint32_t)N;
        Tree t{sorted, nvalid, child, ncount, nbox, pbox, d0, d1, d2, leaf_size, root};
        uint32_t level_items = 1;
        int depth = 0;
        while (level_items > 0) {
                if (++depth > 64) return set_error(GZG_ERR_KERNEL_FAULT, "gzg_gpu_build_scene: tree deeper than 64 levels");
                GZG_CK(cudaMemsetAsync(counts + 3, 0, 4, st), "build: counters");
                k_collapse<<<(level_items + 15) / 16, 128, 0, st>>>(t, qa, counts + 2, qb, counts + 3, counts, nodes,
                                                                     tv0, tv1, tv2, cap, cap, err);
                GZG_CK(cudaMemcpyAsync(counts + 2, counts + 3, 4, cudaMemcpyDeviceToDevice, st), "build: counters");
                GZG_CK(cudaMemcpyAsync(pinned, counts + 3, 4, cudaMemcpyDeviceToHost, st), "build: counters");
                GZG_CK(cudaStreamSynchronize(st), "build: collapse");
                level_items = pinned[0];
                std::swap(qa, qb);
        }
        cudaEventRecord(e1, st);
        GZG_CK(cudaMemcpyAsync(pinned, counts, 8, cudaMemcpyDeviceToHost, st), "build: counters");
        GZG_CK(cudaMemcpyAsync(pinned + 2, err, 4, cudaMemcpyDeviceToHost, st), "build: error word");
        unsigned long long hv = 0;
        GZG_CK(cudaMemcpyAsync(&hv, nvalid, sizeof(hv), cudaMemcpyDeviceToHost, st), "build: prim count");
        GZG_CK(cudaStreamSynchronize(st), "build");
        if (pinned[2]) return set_error(GZG_ERR_KERNEL_FAULT, "gzg_gpu_build_scene: collapse ran out of node or triangle slots");
        if (pinned[1] != (uint32_t)hv)
                return set_error(GZG_ERR_KERNEL_FAULT, "gzg_gpu_build_scene: leaves do not cover every prim");
        out->node_count = pinned[0];
        out->tri_count = pinned[1];
        out->depth = depth;
        cudaEventElapsedTime(device_ms, e0, e1);
        return clear_error();
}

}  // namespace gzg

namespace gzg {
namespace {

__global__ void k_expand_points(const float *__restrict__ p3, int64_t n, float4 *__restrict__ p4) {
        const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (v >= n) return;
        p4[v] = make_float4(p3[3 * v], p3[3 * v + 1], p3[3 * v + 2], 0.0f);
}

__global__ void k_expand_tris(const float4 *__restrict__ p4, const int32_t *__restrict__ idx3,
                              const MeshRange *__restrict__ ranges, int mesh_count, int64_t n,
                              long long *__restrict__ vidx64, gzg_prim_id *__restrict__ prims, float4 *__restrict__ pv0,
                              float4 *__restrict__ pv1, float4 *__restrict__ pv2, uint32_t *__restrict__ bad) {
        const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= n) return;
        int lo = 0, hi = mesh_count - 1;
        while (lo < hi) {
                const int mid = (lo + hi + 1) / 2;
                if (ranges[mid].tri_off <= t)
                        lo = mid;
                else
                        hi = mid - 1;
        }
        const MeshRange r = ranges[lo];
        const int64_t lt = t - r.tri_off;
        bool ok = true;
        int32_t ix[3];
        for (int c = 0; c < 3; ++c) {
                ix[c] = idx3[3 * t + c];
                ok = ok && ix[c] >= 0 && (int64_t)ix[c] < r.vcount;
                vidx64[3 * t + c] = ok ? (long long)ix[c] : 0ll;
        }
        gzg_prim_id p;
        memset(&p, 0, sizeof(p));
        p.material_index = r.material;
        if (r.light_base >= 0) {
                p.type = 3;
                p.id1 = r.light_base + lt;
        } else {
                p.type = 1;
                p.id1 = 0;
        }
        p.id2 = ((int64_t)lo << 32) | lt;
        prims[t] = p;
        if (!ok) {
                atomicOr(bad, 1u);
                pv0[t] = pv1[t] = pv2[t] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                return;
        }
        float4 a = p4[r.vert_off + ix[0]];
        a.w = __int_as_float(1);
        pv0[t] = a;
        pv1[t] = p4[r.vert_off + ix[1]];
        pv2[t] = p4[r.vert_off + ix[2]];
}

}  // namespace

gzg_status gpu_expand_meshes(const float *points3, const int32_t *idx3, const MeshRange *ranges_dev, int mesh_count,
                             int64_t total_verts, int64_t total_tris, float *points4, int64_t *vidx64,
                             gzg_prim_id *prims, float4_ *pv0, float4_ *pv1, float4_ *pv2, bool *bad) {
        uint32_t *flag = nullptr;
        GZG_CK(cudaMalloc(reinterpret_cast<void **>(&flag), 4), "expand: flag");
        struct F {
                uint32_t *p;
                ~F() { cudaFree(p); }
        } fr{flag};
        GZG_CK(cudaMemset(flag, 0, 4), "expand: flag");
        const int B = 256;
        if (total_verts > 0)
                k_expand_points<<<(unsigned)((total_verts + B - 1) / B), B>>>(points3, total_verts,
                                                                             reinterpret_cast<float4 *>(points4));
        if (total_tris > 0)
                k_expand_tris<<<(unsigned)((total_tris + B - 1) / B), B>>>(
                    reinterpret_cast<const float4 *>(points4), idx3, ranges_dev, mesh_count, total_tris,
                    reinterpret_cast<long long *>(vidx64), prims, reinterpret_cast<float4 *>(pv0),
                    reinterpret_cast<float4 *>(pv1), reinterpret_cast<float4 *>(pv2), flag);
        GZG_CK(cudaGetLastError(), "expand: launch");
        uint32_t h = 0;
        GZG_CK(cudaMemcpy(&h, flag, 4, cudaMemcpyDeviceToHost), "expand: flag");
        *bad = h != 0;
        return clear_error();
}

}  // namespace gzg

namespace gzg {
namespace {

// Per prim of mesh `mesh`: its vertices' normals and UVs (5 float4 records,
// DevScene::attr layout).  Prims of other meshes keep their records.
__global__ void k_gather_attributes(const gzg_prim_id *__restrict__ prims, int64_t n,
                                    const gzg_triangle_mesh *__restrict__ meshes, int64_t mesh,
                                    const float *__restrict__ normals, const float *__restrict__ uvs, int64_t vcount,
                                    float4 *__restrict__ attr) {
        const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (k >= n) return;
        int64_t m, base;
        if (!prim_triangle(prims[k], &m, &base) || m != mesh) return;
        const int64_t *vi = meshes[m].vertex_indices;
        int64_t v[3];
        for (int c = 0; c < 3; ++c) {
                v[c] = vi[base + c];
                if (v[c] < 0 || v[c] >= vcount) return;
        }
        float4 *a = attr + 5 * k;
        if (normals) {
                for (int c = 0; c < 3; ++c)
                        a[c] = make_float4(normals[3 * v[c]], normals[3 * v[c] + 1], normals[3 * v[c] + 2],
                                           c == 0 ? __int_as_float(1) : 0.0f);
        }
        if (uvs) {
                a[3] = make_float4(uvs[2 * v[0]], uvs[2 * v[0] + 1], uvs[2 * v[1]], uvs[2 * v[1] + 1]);
                a[4] = make_float4(uvs[2 * v[2]], uvs[2 * v[2] + 1], __int_as_float(1), 0.0f);
        }
}

}  // namespace

gzg_status gpu_gather_attributes(const gzg_prim_id *prims, int64_t n, const gzg_triangle_mesh *meshes_dev,
                                 int64_t mesh, const float *normals, const float *uvs, int64_t vcount,
                                 float4_ *attr) {
        if (n <= 0) return clear_error();
        const int B = 256;
        k_gather_attributes<<<(unsigned)((n + B - 1) / B), B>>>(prims, n, meshes_dev, mesh, normals, uvs, vcount,
                                                                reinterpret_cast<float4 *>(attr));
        GZG_CK(cudaGetLastError(), "attributes: launch");
        GZG_CK(cudaDeviceSynchronize(), "attributes");
        return clear_error();
}

}  // namespace gzg
