// traverse.cu - closest-hit and any-hit traversal kernels for sm_100a.
//
// k_wide: 8-wide quantised nodes (layout in gzg_internal.h).  One ray per
//   thread.  The current "node group" (child base, 8-bit hit mask in
//   front-to-back key order, interior mask) lives in registers; groups still to
//   visit go to a short per-thread stack in shared memory laid out
//   [depth][blockDim] so consecutive threads hit consecutive banks.  Node
//   records are fetched as five 128-bit read-only loads; child planes are
//   8-bit offsets turned into floats with a byte permute and one add.  Leaf
//   triangles are tested as soon as their node is opened, in leaf order.
// k_bvh2: the host's BVH2 traversed exactly as the reference's
//   traverse_bvh2_core (kernel.mojo:223-364), one thread per ray, with the
//   reference's slab arithmetic (kernel.mojo:171-206) in _rn intrinsics.
//
// Both kernels are bounded: a step cap equal to the node count (each node is
// visited at most once per ray in a tree) and a stack-depth check set a bit in
// the scene's error word and end the ray instead of trapping.
#include "device.cuh"
#include "kernels.h"

namespace gzg {

// A persistent warp fetches new rays once at least this many of its lanes are
// idle (or all are): batching the divergent refill beats refilling every idle
// lane at once (ray-cast closest hit: 3,917 Mrays/s at 1, 4,011 at 4, 3,969
// at 8, 3,664 at 16).
constexpr int kRefillMin = 4;

// Fetch statistics of the persistent kernels (instrumented launches only,
// s.counters set): adds the lanes that reach the call to counter `which`
// (0 nodes opened, 1 triangles tested, 2 rays finished), one atomic per
// converged group.  Uninstrumented launches pay one uniform branch and keep no
// per-thread tallies (three registers under the 72-register cap).
__device__ __forceinline__ void count_lanes(const DevScene &s, int which) {
        if (s.counters == nullptr) return;
        const unsigned m = __activemask();
        if ((threadIdx.x & 31u) == (unsigned)(__ffs(m) - 1)) atomicAdd(s.counters + which, (unsigned long long)__popc(m));
}

// Chunk schedule of the persistent kernels.  Rays go out in 32-ray chunks;
// warp w of W starts with chunk w.  A warp that has used up its chunk pulls
// the next from the launch's pull counter (s.sched, cleared by launch_trace
// before the launch; one atomicAdd per 32 rays gives chunk W + the old value),
// or, without a counter, takes w + W,
// w + 2W, ...  Chunks differ in cost by the depth of their rays' traversals;
// the static sequence left the warps that drew costly chunks running alone at
// the launch's tail (ray-cast workload, closest hit: incoherent half 2,884 ->
// 3,148 Mrays/s, coherent half 7,097 -> 8,401 with the pull counter).
// 32-bit indices: launch_trace splits launches above kMaxLaunchRays.  (A
// reset of the word by the launch's last warp, instead of a clear before the
// launch, kept one more value live and spilled at the 72-register cap.)
struct ChunkCursor {
        uint32_t chunk, cursor, end;
};

__device__ __forceinline__ uint32_t grid_warps() { return (gridDim.x * blockDim.x) >> 5; }

__device__ __forceinline__ void chunk_first(ChunkCursor &c, uint32_t n) {
        c.chunk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        c.cursor = c.chunk * 32u;
        c.end = c.cursor + 32u < n ? c.cursor + 32u : n;
}

// Warp-uniform: moves the warp to its next chunk; false when none is left.
// A warp stops pulling once a pull lands past n, so the counter ends below
// n / 32 + 2W and every index stays below 2^32.
__device__ __forceinline__ bool chunk_next(ChunkCursor &c, uint32_t *sched, uint32_t n) {
        if (sched) {
                uint32_t k = 0u;
                if ((threadIdx.x & 31u) == 0u) k = atomicAdd(sched, 1u);
                c.chunk = grid_warps() + __shfl_sync(0xFFFFFFFFu, k, 0);
        } else {
                c.chunk += grid_warps();
        }
        c.cursor = c.chunk * 32u;
        c.end = c.cursor + 32u < n ? c.cursor + 32u : n;
        return c.cursor < n;
}

// 8-bit quantised plane -> float: 0x4B0000qq is 2^23 + q exactly.
__device__ __forceinline__ float qbyte(uint32_t word, uint32_t sel) {
        return __uint_as_float(__byte_perm(word, 0x4B000000u, sel)) - 8388608.0f;
}

// 1/d for the wide kernels' slab tests, kept finite: |d| <= 2^-64 (zero
// included) gives +-2^64 with d's sign.  Finite reciprocals keep every plane
// distance free of 0 * inf = NaN, which lets the slab test compare float bits
// as integers (below).  A plane then appears at distance |dx| * 2^64 instead of
// beyond it, still far past any hit distance of a scene with coordinates below
// about 1e12, so the test stays conservative.
__device__ __forceinline__ float wide_rcp(float d) {
        return fabsf(d) > 5.42101086e-20f ? __fdiv_rn(1.0f, d) : copysignf(1.8446744e19f, d);
}


// Packed FP32 pairs (sm_100a f32x2): each element rounds exactly as the
// scalar fadd / fmaf would, two elements per instruction.
struct F2 {
        float x, y;
};
__device__ __forceinline__ F2 add2(F2 a, F2 b) {
        F2 d;
        asm("{.reg .b64 ra, rb, rd;\n\t"
            "mov.b64 ra, {%2, %3};\n\t"
            "mov.b64 rb, {%4, %5};\n\t"
            "add.rn.f32x2 rd, ra, rb;\n\t"
            "mov.b64 {%0, %1}, rd;}"
            : "=f"(d.x), "=f"(d.y)
            : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
        return d;
}
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) {
        F2 d;
        asm("{.reg .b64 ra, rb, rc, rd;\n\t"
            "mov.b64 ra, {%2, %3};\n\t"
            "mov.b64 rb, {%4, %5};\n\t"
            "mov.b64 rc, {%6, %7};\n\t"
            "fma.rn.f32x2 rd, ra, rb, rc;\n\t"
            "mov.b64 {%0, %1}, rd;}"
            : "=f"(d.x), "=f"(d.y)
            : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
        return d;
}
// Two quantised planes as 2^23 + q floats.
__device__ __forceinline__ F2 qbytes(uint32_t wa, uint32_t wb, uint32_t sel) {
        return F2{__uint_as_float(__byte_perm(wa, 0x4B000000u, sel)), __uint_as_float(__byte_perm(wb, 0x4B000000u, sel))};
}

struct WideRay {
        float ox, oy, oz, dx, dy, dz;
        float rdx, rdy, rdz;
        uint32_t oct;  // sign bits of the inverse direction
};

// Tests the 8 child boxes of a wide node against [0, thit].  Produces the
// interior hit mask in key order (bit (slot ^ oct)), the node's interior mask,
// child base, and the triangle hit mask relative to tri_base.
__device__ __forceinline__ void open_node(const uint4 *__restrict__ node, const WideRay &r, float thit,
                                          uint32_t &node_hits, uint32_t &imask, uint32_t &child_base,
                                          uint32_t &tri_hits, uint32_t &tri_base) {
        const uint4 n0 = __ldg(node + 0);
        const uint4 n1 = __ldg(node + 1);
        const uint4 n2 = __ldg(node + 2);
        const uint4 n3 = __ldg(node + 3);
        const uint4 n4 = __ldg(node + 4);
        const float px = __uint_as_float(n0.x), py = __uint_as_float(n0.y), pz = __uint_as_float(n0.z);
        const uint32_t ew = n0.w;
        imask = ew >> 24;
        child_base = n1.x;
        tri_base = n1.y;
        // step * rdir (exact power-of-two scaling) and the grid origin in t.
        const float sx = __uint_as_float((ew & 0xFFu) << 23) * r.rdx;
        const float sy = __uint_as_float(((ew >> 8) & 0xFFu) << 23) * r.rdy;
        const float sz = __uint_as_float(((ew >> 16) & 0xFFu) << 23) * r.rdz;
        const float ax = (px - r.ox) * r.rdx;
        const float ay = (py - r.oy) * r.rdy;
        const float az = (pz - r.oz) * r.rdz;
        // Far planes carry the relative slack 1.0000003 of the reference's
        // tFar (kernel.mojo:204) in their per-node constants instead of one
        // multiply per child; thit is scaled the same way once.
        const float kSlack = 1.0000003f;
        const float fsx = sx * kSlack, fsy = sy * kSlack, fsz = sz * kSlack;
        const float fax = ax * kSlack, fay = ay * kSlack, faz = az * kSlack;
        const float thit_far = thit * kSlack;
        // near/far plane words by ray sign (lo planes are near for rdir >= 0)
        const bool nx = r.oct & 1u, ny = r.oct & 2u, nz = r.oct & 4u;
        const uint32_t lx0 = n2.x, lx1 = n2.y, ly0 = n2.z, ly1 = n2.w, lz0 = n3.x, lz1 = n3.y;
        const uint32_t hx0 = n3.z, hx1 = n3.w, hy0 = n4.x, hy1 = n4.y, hz0 = n4.z, hz1 = n4.w;
        const uint32_t nearx[2] = {nx ? hx0 : lx0, nx ? hx1 : lx1};
        const uint32_t farx[2] = {nx ? lx0 : hx0, nx ? lx1 : hx1};
        const uint32_t neary[2] = {ny ? hy0 : ly0, ny ? hy1 : ly1};
        const uint32_t fary[2] = {ny ? ly0 : hy0, ny ? ly1 : hy1};
        const uint32_t nearz[2] = {nz ? hz0 : lz0, nz ? hz1 : lz1};
        const uint32_t farz[2] = {nz ? lz0 : hz0, nz ? lz1 : hz1};
        const uint32_t meta[2] = {n1.z, n1.w};
        // The six planes of a child are computed as three packed pairs (near
        // x, y; far x, y; near z, far z), one f32x2 add and one f32x2 fma per
        // pair instead of two scalar ones, with the same rounding per plane:
        // incoherent rays 2,848 -> 2,891 Mrays/s, coherent 6,842 -> 7,089
        // (ray-cast workload, bit-identical hits).
        uint32_t nh = 0, th = 0;
        const F2 bias{-8388608.0f, -8388608.0f};
        const F2 s_nxy{sx, sy}, a_nxy{ax, ay}, s_fxy{fsx, fsy}, a_fxy{fax, fay}, s_z{sz, fsz}, a_z{az, faz};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
                const int w = k >> 2;
                const uint32_t sel = (uint32_t)(k & 3) | 0x7440u;
                const F2 tn = fma2(add2(qbytes(nearx[w], neary[w], sel), bias), s_nxy, a_nxy);
                const F2 tf = fma2(add2(qbytes(farx[w], fary[w], sel), bias), s_fxy, a_fxy);
                const F2 tz = fma2(add2(qbytes(nearz[w], farz[w], sel), bias), s_z, a_z);
                const float tnx = tn.x, tny = tn.y, tnz = tz.x;
                const float tfx = tf.x, tfy = tf.y, tfz = tz.y;
                // max(0, tn*) and min(tf*, thit) on the float bits as signed
                // integers: order-preserving for non-negative floats; tnear is
                // never negative, and a negative tfar (a negative integer)
                // rejects the box either way.  No NaN occurs (finite rdir).
                const int tnear = __vimax3_s32_relu(__float_as_int(tnx), __float_as_int(tny), __float_as_int(tnz));
                const int tfar = __vimin3_s32(__float_as_int(tfx), __float_as_int(tfy),
                                              min(__float_as_int(tfz), __float_as_int(thit_far)));
                if (tnear <= tfar) {
                        const uint32_t m = (meta[w] >> (8 * (k & 3))) & 0xFFu;
                        if ((imask >> k) & 1u) {
                                nh |= 1u << (k ^ r.oct);
                        } else if (m & 0x80u) {
                                const uint32_t cnt = ((m >> 5) & 3u) + 1u;
                                th |= ((1u << cnt) - 1u) << (m & 31u);
                        }
                }
        }
        node_hits = nh;
        tri_hits = th;
}

template <int RAYFMT, int OUTFMT, bool ANY, int STACK, int LEAF>
__global__ void __launch_bounds__(256) k_wide(DevScene s, const void *__restrict__ rays, const float *__restrict__ tmaxs,
                                              int64_t n, void *__restrict__ out) {
        extern __shared__ uint2 smem_stack[];
        const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        n = ray_count(s, n);
        if (i >= n) return;
        const RayIn in = load_ray<RAYFMT>(rays, tmaxs, i);
        WideRay r;
        r.ox = in.ox;
        r.oy = in.oy;
        r.oz = in.oz;
        r.dx = in.dx;
        r.dy = in.dy;
        r.dz = in.dz;
        r.rdx = wide_rcp(in.dx);
        r.rdy = wide_rcp(in.dy);
        r.rdz = wide_rcp(in.dz);
        r.oct = (__float_as_uint(r.rdx) >> 31) | ((__float_as_uint(r.rdy) >> 31) << 1) |
                ((__float_as_uint(r.rdz) >> 31) << 2);

        uint2 *stack = smem_stack + threadIdx.x;
        const int stride = blockDim.x;
        int sp = 0;
        float thit = in.tmax, bu = 0.0f, bv = 0.0f;
        int prim = -1;
        uint32_t steps = 0, n_nodes = 0, n_tris = 0;
        // The root is key 0 of a virtual parent whose only interior slot is oct.
        uint2 group = make_uint2(s.per_ray_root ? in.root : 0u, (1u << 24) | (1u << r.oct));
        for (;;) {
                uint32_t tri_hits = 0, tri_base = 0;
                uint32_t hits = group.y >> 24;
                if (hits) {
                        const uint32_t key = __ffs(hits) - 1;
                        hits &= hits - 1;
                        const uint32_t im = group.y & 0xFFu;
                        const uint32_t slot = key ^ r.oct;
                        const uint32_t node = group.x + __popc(im & ((1u << slot) - 1u));
                        if (hits) {
                                if (sp >= STACK) {
                                        atomicOr(s.err, kErrStackOverflow);
                                        break;
                                }
                                stack[sp * stride] = make_uint2(group.x, (hits << 24) | im);
                                ++sp;
                        }
                        if (++steps > s.wide_count) {
                                atomicOr(s.err, kErrStepCap);
                                break;
                        }
                        uint32_t nh, nim, cb;
                        open_node(s.wide + 5 * (size_t)node, r, thit, nh, nim, cb, tri_hits, tri_base);
                        ++n_nodes;
                        group = make_uint2(cb, (nh << 24) | nim);
                }
                bool done = false;
                while (tri_hits) {
                        const uint32_t b = __ffs(tri_hits) - 1;
                        tri_hits &= tri_hits - 1;
                        const uint32_t ti = tri_base + b;
                        ++n_tris;
                        const float4 a = __ldg(s.tv0 + ti);
                        const float4 bb = __ldg(s.tv1 + ti);
                        const float4 c = __ldg(s.tv2 + ti);
                        float t, u, v;
                        if (leaf_test<LEAF>(r.ox, r.oy, r.oz, r.dx, r.dy, r.dz, a, bb, c, thit, t, u, v)) {
                                thit = t;
                                bu = u;
                                bv = v;
                                prim = __float_as_int(a.w);
                                if (ANY) {
                                        done = true;
                                        break;
                                }
                        }
                }
                if (done) break;
                if ((group.y >> 24) == 0) {
                        if (sp == 0) break;
                        --sp;
                        group = stack[sp * stride];
                }
        }
        if (prim < 0) {
                thit = in.tmax;
                bu = 0.0f;
                bv = 0.0f;
        }
        store_hit<OUTFMT>(s, out, i, prim, thit, bu, bv);
        add_counters(s, n_nodes, n_tris, 1u);
}

// Persistent variant of k_wide.  The grid is sized to the resident capacity
// (SM count x blocks per SM); each warp takes 32-ray chunks by the chunk
// schedule above (the pull counter when the launch has one) and hands out the
// rays of its current chunk in order.  A lane whose ray finishes takes the
// next ray at the top of the next iteration, so lanes are not left idle while
// the slowest ray of a fixed 32-ray batch finishes.  Each iteration opens one
// node and tests its triangles.  A miss reads its tMax again at the end
// instead of keeping it in a register.
// Capped at 64 registers (8 blocks of 128 per SM).  With the pull counter the
// extra warps pay for closest hit's 28 bytes of spills: ray-cast halves
// against 7 blocks (72 registers, no spills), incoherent 3,170 -> 3,261
// Mrays/s closest and 3,827 -> 4,148 any hit, coherent 8,362 -> 8,456 closest
// and 9,692 -> 10,197 any hit.  9 blocks (56 registers, 84 bytes of spills)
// was slower than 7.  On the static schedule 8 blocks was slower than 7.
template <int RAYFMT, int OUTFMT, bool ANY, int STACK, int LEAF>
__global__ void __launch_bounds__(128, 8) k_wide_persistent(DevScene s, const void *__restrict__ rays,
                                                         const float *__restrict__ tmaxs, int64_t n,
                                                         void *__restrict__ out) {
        extern __shared__ uint2 smem_stack[];
        const unsigned FULL = 0xFFFFFFFFu;
        const uint32_t nr = (uint32_t)ray_count(s, n);
        const unsigned lane = threadIdx.x & 31u;
        const unsigned lt_mask = (1u << lane) - 1u;
        ChunkCursor cc;
        chunk_first(cc, nr);

        uint2 *stack = smem_stack + threadIdx.x;
        const int stride = blockDim.x;
        int ray_i = -1;
        WideRay r;
        float thit = 0.0f, bu = 0.0f, bv = 0.0f;
        int prim = -1, sp = 0;
        uint2 group = make_uint2(0u, 0u);
        uint32_t steps = 0;

        for (;;) {
                // ---- refill idle lanes from this warp's chunk sequence (warp-uniform cursor)
                unsigned need = __ballot_sync(FULL, ray_i < 0);
                if (__popc(need) < kRefillMin && need != FULL) need = 0u;
                while (need != 0u && cc.cursor < nr) {
                        if (cc.cursor >= cc.end && !chunk_next(cc, s.sched, nr)) break;
                        const int avail = (int)(cc.end - cc.cursor);
                        const int rank = __popc(need & lt_mask);
                        if (ray_i < 0 && rank < avail) {
                                ray_i = (int)(cc.cursor + (uint32_t)rank);
                                const RayIn in = load_ray<RAYFMT>(rays, tmaxs, ray_i);
                                r.ox = in.ox;
                                r.oy = in.oy;
                                r.oz = in.oz;
                                r.dx = in.dx;
                                r.dy = in.dy;
                                r.dz = in.dz;
                                r.rdx = wide_rcp(in.dx);
                                r.rdy = wide_rcp(in.dy);
                                r.rdz = wide_rcp(in.dz);
                                r.oct = (__float_as_uint(r.rdx) >> 31) | ((__float_as_uint(r.rdy) >> 31) << 1) |
                                        ((__float_as_uint(r.rdz) >> 31) << 2);
                                thit = in.tmax;
                                bu = bv = 0.0f;
                                prim = -1;
                                sp = 0;
                                steps = 0;
                                group = make_uint2(s.per_ray_root ? in.root : 0u, (1u << 24) | (1u << r.oct));
                        }
                        const int npop = __popc(need);
                        cc.cursor += (uint32_t)(npop < avail ? npop : avail);
                        need = __ballot_sync(FULL, ray_i < 0);
                }
                if (__all_sync(FULL, ray_i < 0)) break;
                if (ray_i < 0) continue;

                // ---- one traversal step: open one node, test its triangles
                bool finished = false;
                uint32_t tri_hits = 0, tri_base = 0;
                uint32_t hits = group.y >> 24;
                if (hits) {
                        const uint32_t key = __ffs(hits) - 1;
                        hits &= hits - 1;
                        const uint32_t im = group.y & 0xFFu;
                        const uint32_t slot = key ^ r.oct;
                        const uint32_t node = group.x + __popc(im & ((1u << slot) - 1u));
                        bool fault = false;
                        if (hits) {
                                if (sp >= STACK) {
                                        atomicOr(s.err, kErrStackOverflow);
                                        fault = true;
                                } else {
                                        stack[sp * stride] = make_uint2(group.x, (hits << 24) | im);
                                        ++sp;
                                }
                        }
                        if (++steps > s.wide_count) {
                                atomicOr(s.err, kErrStepCap);
                                fault = true;
                        }
                        if (fault) {
                                group.y = 0u;
                                sp = 0;
                        } else {
                                uint32_t nh, nim, cb;
                                open_node(s.wide + 5 * (size_t)node, r, thit, nh, nim, cb, tri_hits, tri_base);
                                count_lanes(s, 0);
                                group = make_uint2(cb, (nh << 24) | nim);
                        }
                }
                while (tri_hits) {
                        const uint32_t b = __ffs(tri_hits) - 1;
                        tri_hits &= tri_hits - 1;
                        const uint32_t ti = tri_base + b;
                        count_lanes(s, 1);
                        const float4 a = __ldg(s.tv0 + ti);
                        const float4 bb = __ldg(s.tv1 + ti);
                        const float4 c = __ldg(s.tv2 + ti);
                        float t, u, v;
                        if (leaf_test<LEAF>(r.ox, r.oy, r.oz, r.dx, r.dy, r.dz, a, bb, c, thit, t, u, v)) {
                                thit = t;
                                bu = u;
                                bv = v;
                                prim = __float_as_int(a.w);
                                if (ANY) {
                                        finished = true;
                                        break;
                                }
                        }
                }
                if (!finished && (group.y >> 24) == 0) {
                        if (sp == 0)
                                finished = true;
                        else {
                                --sp;
                                group = stack[sp * stride];
                        }
                }
                if (finished) {
                        if (prim < 0) {
                                // a miss reports the ray's tMax, read again
                                // rather than kept in a register
                                thit = load_ray<RAYFMT>(rays, tmaxs, ray_i).tmax;
                                bu = 0.0f;
                                bv = 0.0f;
                        }
                        store_hit<OUTFMT>(s, out, ray_i, prim, thit, bu, bv);
                        ray_i = -1;
                        count_lanes(s, 2);
                }
        }
}

__device__ __forceinline__ void set_ray_dirs(WideRay &r) {
        r.rdx = wide_rcp(r.dx);
        r.rdy = wide_rcp(r.dy);
        r.rdz = wide_rcp(r.dz);
        r.oct = (__float_as_uint(r.rdx) >> 31) | ((__float_as_uint(r.rdy) >> 31) << 1) |
                ((__float_as_uint(r.rdz) >> 31) << 2);
}

// The world-space ray of device-ray slot i, read again from the ray array (the
// two-level kernel keeps it out of registers: it is needed only when a ray
// enters or leaves an instance).
__device__ __forceinline__ void world_ray(const void *rays, int i, WideRay &r) {
        const float4 *p = reinterpret_cast<const float4 *>(rays) + 2 * (size_t)i;
        const float4 a = __ldg(p), b = __ldg(p + 1);
        r.ox = a.x;
        r.oy = a.y;
        r.oz = a.z;
        r.dx = b.x;
        r.dy = b.y;
        r.dz = b.z;
}

// Transform*Point / Transform*Vector of Geometry/Transform.swift:31-65 with a
// 3x4 affine matrix (w = 1, so the division is exact and omitted), each product
// and sum rounded separately in the reference's order.
__device__ __forceinline__ float xf_point(const float4 &row, float x, float y, float z) {
        return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(row.x, x), __fmul_rn(row.y, y)), __fmul_rn(row.z, z)), row.w);
}
__device__ __forceinline__ float xf_vector(const float4 &row, float x, float y, float z) {
        return __fadd_rn(__fadd_rn(__fmul_rn(row.x, x), __fmul_rn(row.y, y)), __fmul_rn(row.z, z));
}

// Two-level persistent traversal (TransformedPrimitive.intersect,
// Primitive/TransformedPrimitive.swift:5-22).  The top-level tree's leaf
// records are instances (v0.w = -(instance + 1)); reaching one pushes, in this
// order, the rest of the current node's children, the rest of its leaf
// records (0x80000000 | base, mask) and a return marker (0xFFFFFFFF), moves the
// ray to object space and descends into the bottom-level root.  Popping the
// marker restores the world ray.  Bottom-level trees are ordinary wide trees
// stored after the top-level nodes in the same arrays.
// The world ray is not kept in registers: it is read again from the ray
// array when a ray enters or leaves an instance.  Bounded to 128-thread
// blocks, 8 resident per SM (64 registers, 12-36 bytes of spills): the
// unbounded build's 99 registers left 4 blocks per SM; 6 blocks (80 registers)
// gave 1.6x its camera-ray rate and 7 another 2 % on the two-level frame
// (1,187 -> 1,162 ms); with the pull counter and the world ray out of
// registers, 8 blocks another 1.3 % (16-spp frame 265.5 -> 262.0 ms).
template <int OUTFMT, bool ANY, int STACK>
__global__ void __launch_bounds__(128, 8) k_wide_instanced(DevScene s, const void *__restrict__ rays,
                                                        const float *__restrict__ tmaxs, int64_t n,
                                                        void *__restrict__ out) {
        extern __shared__ uint2 smem_stack[];
        const unsigned FULL = 0xFFFFFFFFu;
        const uint32_t nr = (uint32_t)ray_count(s, n);
        const unsigned lane = threadIdx.x & 31u;
        const unsigned lt_mask = (1u << lane) - 1u;
        ChunkCursor cc;
        chunk_first(cc, nr);

        uint2 *stack = smem_stack + threadIdx.x;
        const int stride = blockDim.x;
        int ray_i = -1;
        WideRay r;
        float thit = 0.0f, bu = 0.0f, bv = 0.0f;
        int prim = -1, hit_inst = -1, cur_inst = -1, sp = 0;
        uint2 group = make_uint2(0u, 0u);
        uint32_t pend_base = 0, pend_mask = 0;
        uint32_t steps = 0;

        for (;;) {
                unsigned need = __ballot_sync(FULL, ray_i < 0);
                if (__popc(need) < kRefillMin && need != FULL) need = 0u;
                while (need != 0u && cc.cursor < nr) {
                        if (cc.cursor >= cc.end && !chunk_next(cc, s.sched, nr)) break;
                        const int avail = (int)(cc.end - cc.cursor);
                        const int rank = __popc(need & lt_mask);
                        if (ray_i < 0 && rank < avail) {
                                ray_i = (int)(cc.cursor + (uint32_t)rank);
                                const RayIn in = load_ray<kRayDevice>(rays, tmaxs, ray_i);
                                r.ox = in.ox;
                                r.oy = in.oy;
                                r.oz = in.oz;
                                r.dx = in.dx;
                                r.dy = in.dy;
                                r.dz = in.dz;
                                set_ray_dirs(r);
                                thit = in.tmax;
                                bu = bv = 0.0f;
                                prim = hit_inst = cur_inst = -1;
                                sp = 0;
                                steps = 0;
                                pend_mask = 0;
                                group = make_uint2(0u, (1u << 24) | (1u << r.oct));
                        }
                        const int npop = __popc(need);
                        cc.cursor += (uint32_t)(npop < avail ? npop : avail);
                        need = __ballot_sync(FULL, ray_i < 0);
                }
                if (__all_sync(FULL, ray_i < 0)) break;
                if (ray_i < 0) continue;

                bool finished = false, fault = false;
                if (pend_mask == 0) {
                        // pop until there is work: a world-ray marker restores the
                        // world ray and pops again in the same step
                        while ((group.y >> 24) == 0 && sp > 0) {
                                --sp;
                                const uint2 e = stack[sp * stride];
                                if (e.x == 0xFFFFFFFFu) {
                                        world_ray(rays, ray_i, r);
                                        set_ray_dirs(r);
                                        cur_inst = -1;
                                } else if (e.x & 0x80000000u) {
                                        pend_base = e.x & 0x7FFFFFFFu;
                                        pend_mask = e.y;
                                        break;
                                } else {
                                        group = e;
                                }
                        }
                        uint32_t hits = group.y >> 24;
                        if (pend_mask == 0 && hits) {
                                const uint32_t key = __ffs(hits) - 1;
                                hits &= hits - 1;
                                const uint32_t im = group.y & 0xFFu;
                                const uint32_t slot = key ^ r.oct;
                                const uint32_t node = group.x + __popc(im & ((1u << slot) - 1u));
                                if (hits) {
                                        if (sp >= STACK) {
                                                atomicOr(s.err, kErrStackOverflow);
                                                fault = true;
                                        } else {
                                                stack[sp * stride] = make_uint2(group.x, (hits << 24) | im);
                                                ++sp;
                                        }
                                }
                                if (++steps > s.wide_count) {
                                        atomicOr(s.err, kErrStepCap);
                                        fault = true;
                                }
                                if (!fault) {
                                        uint32_t nh, nim, cb;
                                        open_node(s.wide + 5 * (size_t)node, r, thit, nh, nim, cb, pend_mask, pend_base);
                                        count_lanes(s, 0);
                                        group = make_uint2(cb, (nh << 24) | nim);
                                }
                        }
                }
                while (!fault && pend_mask) {
                        const uint32_t b = __ffs(pend_mask) - 1;
                        pend_mask &= pend_mask - 1;
                        const uint32_t ti = pend_base + b;
                        const float4 a = __ldg(s.tv0 + ti);
                        const int tag = __float_as_int(a.w);
                        if (tag < 0) {
                                // instance record: save the resume state and descend
                                const int inst = -tag - 1;
                                const int need_slots = ((group.y >> 24) ? 1 : 0) + (pend_mask ? 1 : 0) + 1;
                                if (sp + need_slots > STACK || inst >= (int)s.instance_count) {
                                        atomicOr(s.err, inst >= (int)s.instance_count ? kErrBadIndex : kErrStackOverflow);
                                        fault = true;
                                        break;
                                }
                                if (group.y >> 24) {
                                        stack[sp * stride] = group;
                                        ++sp;
                                        group.y = 0u;
                                }
                                if (pend_mask) {
                                        stack[sp * stride] = make_uint2(0x80000000u | pend_base, pend_mask);
                                        ++sp;
                                        pend_mask = 0;
                                }
                                stack[sp * stride] = make_uint2(0xFFFFFFFFu, 0u);
                                ++sp;
                                const float4 m0 = __ldg(s.instances + 4 * inst), m1 = __ldg(s.instances + 4 * inst + 1),
                                             m2 = __ldg(s.instances + 4 * inst + 2), m3 = __ldg(s.instances + 4 * inst + 3);
                                WideRay w;
                                world_ray(rays, ray_i, w);
                                r.ox = xf_point(m0, w.ox, w.oy, w.oz);
                                r.oy = xf_point(m1, w.ox, w.oy, w.oz);
                                r.oz = xf_point(m2, w.ox, w.oy, w.oz);
                                r.dx = xf_vector(m0, w.dx, w.dy, w.dz);
                                r.dy = xf_vector(m1, w.dx, w.dy, w.dz);
                                r.dz = xf_vector(m2, w.dx, w.dy, w.dz);
                                set_ray_dirs(r);
                                cur_inst = inst;
                                group = make_uint2((uint32_t)__float_as_int(m3.x), (1u << 24) | (1u << r.oct));
                                break;
                        }
                        count_lanes(s, 1);
                        const float4 bb = __ldg(s.tv1 + ti);
                        const float4 c = __ldg(s.tv2 + ti);
                        float t, u, v;
                        if (mt_test(r.ox, r.oy, r.oz, r.dx, r.dy, r.dz, a, bb, c, thit, t, u, v)) {
                                thit = t;
                                bu = u;
                                bv = v;
                                prim = tag;
                                hit_inst = cur_inst;
                                if (ANY) {
                                        finished = true;
                                        break;
                                }
                        }
                }
                if (fault || (!finished && pend_mask == 0 && (group.y >> 24) == 0 && sp == 0)) finished = true;
                if (finished) {
                        if (prim < 0) {
                                thit = load_ray<kRayDevice>(rays, tmaxs, ray_i).tmax;
                                bu = 0.0f;
                                bv = 0.0f;
                                hit_inst = -1;
                        }
                        store_hit<OUTFMT>(s, out, ray_i, prim, thit, bu, bv);
                        if (s.inst_out) s.inst_out[ray_i] = hit_inst;
                        ray_i = -1;
                        count_lanes(s, 2);
                }
        }
}

// The reference's slab test (kernel.mojo:171-206), separately rounded.
__device__ __forceinline__ bool ref_aabb(const float4 &lo, const float4 &hi, const float rd[3], const float ord[3],
                                         const bool nm[3], float tmax, float &tnear_out) {
        const float mn[3] = {lo.x, lo.y, lo.z};
        const float mx[3] = {lo.w, hi.x, hi.y};
        float tn[3], tf[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
                const float nr = nm[k] ? mn[k] : mx[k];
                const float fr = nm[k] ? mx[k] : mn[k];
                tn[k] = __fsub_rn(__fmul_rn(nr, rd[k]), ord[k]);
                tf[k] = __fsub_rn(__fmul_rn(fr, rd[k]), ord[k]);
        }
        float tnear = tn[0] > tn[1] ? tn[0] : tn[1];
        tnear = tn[2] > tnear ? tn[2] : tnear;
        tnear = 0.0f > tnear ? 0.0f : tnear;
        float tfar = tf[0] < tf[1] ? tf[0] : tf[1];
        tfar = tf[2] < tfar ? tf[2] : tfar;
        tfar = tmax < tfar ? tmax : tfar;
        tfar = __fmul_rn(tfar, 1.0000003f);
        tnear_out = tnear;
        return tnear <= tfar;
}

template <int RAYFMT, int OUTFMT, bool ANY, int LEAF>
__global__ void __launch_bounds__(128) k_bvh2(DevScene s, const void *__restrict__ rays, const float *__restrict__ tmaxs,
                                              int64_t n, void *__restrict__ out) {
        const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        n = ray_count(s, n);
        if (i >= n) return;
        const RayIn in = load_ray<RAYFMT>(rays, tmaxs, i);
        const float rd[3] = {__fdiv_rn(1.0f, in.dx), __fdiv_rn(1.0f, in.dy), __fdiv_rn(1.0f, in.dz)};
        const float ord[3] = {__fmul_rn(in.ox, rd[0]), __fmul_rn(in.oy, rd[1]), __fmul_rn(in.oz, rd[2])};
        const bool nm[3] = {rd[0] >= 0.0f, rd[1] >= 0.0f, rd[2] >= 0.0f};
        int stack[64];
        int to_visit = 0;
        int64_t current = 0;
        int hit_index = -1;
        float thit = in.tmax, bu = 0.0f, bv = 0.0f;
        int64_t steps = 0;
        uint32_t n_nodes = 0, n_tris = 0;
        for (;;) {
                if (++steps > s.bvh2_count) {
                        atomicOr(s.err, kErrStepCap);
                        break;
                }
                const float4 *nd = s.bvh2 + 2 * current;
                const float4 hi = __ldg(nd + 1);
                const int count = __float_as_int(hi.w);
                ++n_nodes;
                if (count > 0) {
                        const int off = __float_as_int(hi.z);
                        for (int j = 0; j < count; ++j) {
                                const int k = off + j;
                                const float4 a = __ldg(s.pv0 + k);
                                if (__float_as_int(a.w) == 0) continue;  // id2 == -1 / not a triangle
                                const float4 b = __ldg(s.pv1 + k);
                                const float4 c = __ldg(s.pv2 + k);
                                ++n_tris;
                                float t, u, v;
                                if (leaf_test<LEAF>(in.ox, in.oy, in.oz, in.dx, in.dy, in.dz, a, b, c, thit, t, u, v)) {
                                        thit = t;
                                        bu = u;
                                        bv = v;
                                        hit_index = k;
                                }
                        }
                        if (ANY && hit_index >= 0) break;
                        if (to_visit == 0) break;
                        current = stack[--to_visit];
                } else {
                        const int64_t li = current + 1, ri = __float_as_int(hi.z);
                        const float4 l0 = __ldg(s.bvh2 + 2 * li), l1 = __ldg(s.bvh2 + 2 * li + 1);
                        const float4 r0 = __ldg(s.bvh2 + 2 * ri), r1 = __ldg(s.bvh2 + 2 * ri + 1);
                        n_nodes += 2;
                        float lt, rt;
                        const bool lh = ref_aabb(l0, l1, rd, ord, nm, thit, lt);
                        const bool rh = ref_aabb(r0, r1, rd, ord, nm, thit, rt);
                        if (lh && rh) {
                                if (to_visit >= 64) {
                                        atomicOr(s.err, kErrStackOverflow);
                                        break;
                                }
                                if (lt <= rt) {
                                        current = li;
                                        stack[to_visit] = (int)ri;
                                } else {
                                        current = ri;
                                        stack[to_visit] = (int)li;
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
        if (hit_index < 0) {
                thit = in.tmax;
                bu = 0.0f;
                bv = 0.0f;
        }
        store_hit<OUTFMT>(s, out, i, hit_index, thit, bu, bv);
        add_counters(s, n_nodes, n_tris, 1u);
}

__global__ void k_hits_to_isect(DevScene s, const float4 *__restrict__ hits, int64_t n, void *__restrict__ out) {
        const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n) return;
        const float4 h = __ldcs(hits + i);
        const int prim = __float_as_int(h.w);
        if (prim >= (int)s.prim_count) {
                atomicOr(s.err, kErrBadIndex);
                store_hit<kOutIntersection>(s, out, i, -1, h.x, 0.0f, 0.0f);
                return;
        }
        store_hit<kOutIntersection>(s, out, i, prim, h.x, h.y, h.z);
}

// ------------------------------------------------------------ launchers

namespace {

using TraceKernel = void (*)(DevScene, const void *, const float *, int64_t, void *);

// Launches a wide-node kernel with a STACK-deep shared-memory stack.  The
// persistent kernel gets one wave of resident blocks (SM count x blocks per
// SM, from the occupancy calculator unless blocks_per_sm is given), capped at
// the blocks the ray count needs; the one-ray-per-thread kernel one thread per
// ray.
cudaError_t launch_wide_kernel(TraceKernel k, int stack, bool persistent, const LaunchParams &p, const DevScene &s,
                               const void *rays, const float *tmax, int64_t n, void *out, cudaStream_t st) {
        // The persistent kernel is compiled for blocks of at most 128 threads
        // (measured faster for any-hit queries than a 256-thread bound).
        const int block = (p.block_size == 64 || (p.block_size == 256 && !persistent)) ? p.block_size : 128;
        const int blocks_per_sm = p.blocks_per_sm;
        const size_t smem = (size_t)stack * block * sizeof(uint2);
        if (smem > 48 * 1024) {
                cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                if (e != cudaSuccess) return e;
        }
        // L1 / shared split: explicit percent, or the driver's choice (-1).
        {
                const int carve = p.l1_carveout > 0 ? (p.l1_carveout > 100 ? 100 : p.l1_carveout) : -1;
                cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
                if (e != cudaSuccess) return e;
        }
        int64_t grid = (n + block - 1) / block;
        if (persistent) {
                int dev = 0, sms = 0, per_sm = blocks_per_sm;
                cudaGetDevice(&dev);
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                if (per_sm <= 0) {
                        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block, smem);
                        if (e != cudaSuccess) return e;
                        if (per_sm <= 0) per_sm = 1;
                }
                const int64_t wave = (int64_t)sms * per_sm;
                if (wave < grid) grid = wave;
                // The pull counter pays off once some warp has a second chunk
                // (with one chunk per warp both schedules are the same); it
                // starts every launch at zero.
                if (s.sched != nullptr) {
                        if (s.n_dev == nullptr && n <= grid * block) {
                                DevScene ws = s;
                                ws.sched = nullptr;
                                k<<<(unsigned)grid, block, smem, st>>>(ws, rays, tmax, n, out);
                                return cudaGetLastError();
                        }
                        const cudaError_t e = cudaMemsetAsync(s.sched, 0, sizeof(uint32_t), st);
                        if (e != cudaSuccess) return e;
                }
        }
        k<<<(unsigned)grid, block, smem, st>>>(s, rays, tmax, n, out);
        return cudaGetLastError();
}

template <int RAYFMT, int OUTFMT, bool ANY, int LEAF>
cudaError_t launch_wide_depth(const DevScene &s, const LaunchParams &p, const void *rays, const float *tmax, int64_t n,
                              void *out, cudaStream_t st) {
        const bool persistent = p.traversal == GZG_TRAVERSAL_WIDE;
        // A ray pushes at most one group (the rest of a node's interior hits)
        // per level whose nodes have interior children, so the stack holds at
        // most depth - 1 groups; a requested depth below that is raised so no
        // ray can overflow it (an overflow would set kErrStackOverflow).
        const int need = p.wide_depth > 2 ? p.wide_depth - 1 : 1;
        const int want = p.stack_depth > need ? p.stack_depth : need;
        if (want <= 8) {
                TraceKernel k = persistent ? k_wide_persistent<RAYFMT, OUTFMT, ANY, 8, LEAF> : k_wide<RAYFMT, OUTFMT, ANY, 8, LEAF>;
                return launch_wide_kernel(k, 8, persistent, p, s, rays, tmax, n, out, st);
        }
        if (want <= 16) {
                TraceKernel k = persistent ? k_wide_persistent<RAYFMT, OUTFMT, ANY, 16, LEAF> : k_wide<RAYFMT, OUTFMT, ANY, 16, LEAF>;
                return launch_wide_kernel(k, 16, persistent, p, s, rays, tmax, n, out, st);
        }
        if (want <= 32) {
                TraceKernel k = persistent ? k_wide_persistent<RAYFMT, OUTFMT, ANY, 32, LEAF> : k_wide<RAYFMT, OUTFMT, ANY, 32, LEAF>;
                return launch_wide_kernel(k, 32, persistent, p, s, rays, tmax, n, out, st);
        }
        TraceKernel k = persistent ? k_wide_persistent<RAYFMT, OUTFMT, ANY, 64, LEAF> : k_wide<RAYFMT, OUTFMT, ANY, 64, LEAF>;
        return launch_wide_kernel(k, 64, persistent, p, s, rays, tmax, n, out, st);
}

template <int RAYFMT, int OUTFMT, bool ANY>
cudaError_t launch_fmt(const DevScene &s, const LaunchParams &p, const void *rays, const float *tmax, int64_t n,
                       void *out, cudaStream_t st) {
        const int block = 128;
        if (p.traversal == GZG_TRAVERSAL_BVH2) {
                if (!s.bvh2) return cudaErrorInvalidValue;  // a device-built scene has no reference BVH2
                const int64_t grid = (n + block - 1) / block;
                if (p.leaf_test == GZG_LEAF_WATERTIGHT)
                        k_bvh2<RAYFMT, OUTFMT, ANY, GZG_LEAF_WATERTIGHT><<<(unsigned)grid, block, 0, st>>>(s, rays, tmax, n, out);
                else
                        k_bvh2<RAYFMT, OUTFMT, ANY, GZG_LEAF_MOLLER_TRUMBORE><<<(unsigned)grid, block, 0, st>>>(s, rays, tmax, n, out);
                return cudaGetLastError();
        }
        if (p.leaf_test == GZG_LEAF_WATERTIGHT)
                return launch_wide_depth<RAYFMT, OUTFMT, ANY, GZG_LEAF_WATERTIGHT>(s, p, rays, tmax, n, out, st);
        return launch_wide_depth<RAYFMT, OUTFMT, ANY, GZG_LEAF_MOLLER_TRUMBORE>(s, p, rays, tmax, n, out, st);
}

}  // namespace

cudaError_t launch_trace(const DevScene &scene, const LaunchParams &p, int ray_fmt, int out_fmt, const void *rays,
                         const float *tmax, int64_t n, void *out, cudaStream_t st) {
        if (n <= 0) return cudaSuccess;
        if (n > kMaxLaunchRays) {
                // consecutive launches over slices of the arrays
                if (p.n_dev) return cudaErrorInvalidValue;
                const size_t ray_bytes = ray_fmt == kRayDevice ? 32 : 24;
                const size_t out_bytes = out_fmt == kOutHit ? 16 : out_fmt == kOutIntersection ? 48 : out_fmt == kOutAnyPrim ? 4 : 1;
                LaunchParams q = p;
                for (int64_t off = 0; off < n; off += kMaxLaunchRays) {
                        const int64_t m = n - off < kMaxLaunchRays ? n - off : kMaxLaunchRays;
                        q.inst_out = p.inst_out ? p.inst_out + off : nullptr;
                        const cudaError_t e = launch_trace(scene, q, ray_fmt, out_fmt,
                                                           reinterpret_cast<const char *>(rays) + off * ray_bytes,
                                                           tmax ? tmax + off : nullptr, m,
                                                           reinterpret_cast<char *>(out) + off * out_bytes, st);
                        if (e != cudaSuccess) return e;
                }
                return cudaSuccess;
        }
        DevScene s = scene;
        s.counters = p.counters;
        s.n_dev = p.n_dev;
        s.inst_out = p.inst_out;
        s.sched = p.sched;
        if (s.instances) {
                // two-level scenes: persistent wide traversal only
                if (ray_fmt != kRayDevice || (out_fmt != kOutHit && out_fmt != kOutAnyPrim)) return cudaErrorNotSupported;
                const int need = p.wide_depth > 1 ? p.wide_depth : 1;
                const int want = p.stack_depth > need ? p.stack_depth : need;
                LaunchParams q = p;
                q.traversal = GZG_TRAVERSAL_WIDE;
                TraceKernel k;
                int stack;
                if (want <= 16) {
                        stack = 16;
                        k = out_fmt == kOutHit ? k_wide_instanced<kOutHit, false, 16> : k_wide_instanced<kOutAnyPrim, true, 16>;
                } else if (want <= 32) {
                        stack = 32;
                        k = out_fmt == kOutHit ? k_wide_instanced<kOutHit, false, 32> : k_wide_instanced<kOutAnyPrim, true, 32>;
                } else {
                        stack = 64;
                        k = out_fmt == kOutHit ? k_wide_instanced<kOutHit, false, 64> : k_wide_instanced<kOutAnyPrim, true, 64>;
                }
                return launch_wide_kernel(k, stack, true, q, s, rays, tmax, n, out, st);
        }
        if (ray_fmt == kRayDevice) {
                switch (out_fmt) {
                case kOutHit: return launch_fmt<kRayDevice, kOutHit, false>(s, p, rays, tmax, n, out, st);
                case kOutIntersection: return launch_fmt<kRayDevice, kOutIntersection, false>(s, p, rays, tmax, n, out, st);
                case kOutAnyPrim: return launch_fmt<kRayDevice, kOutAnyPrim, true>(s, p, rays, tmax, n, out, st);
                default: return launch_fmt<kRayDevice, kOutOccluded, true>(s, p, rays, tmax, n, out, st);
                }
        }
        switch (out_fmt) {
        case kOutHit: return launch_fmt<kRayReference, kOutHit, false>(s, p, rays, tmax, n, out, st);
        case kOutIntersection: return launch_fmt<kRayReference, kOutIntersection, false>(s, p, rays, tmax, n, out, st);
        case kOutAnyPrim: return launch_fmt<kRayReference, kOutAnyPrim, true>(s, p, rays, tmax, n, out, st);
        default: return launch_fmt<kRayReference, kOutOccluded, true>(s, p, rays, tmax, n, out, st);
        }
}

cudaError_t launch_hits_to_isect(const DevScene &s, const void *hits, int64_t n, void *out, cudaStream_t st) {
        if (n <= 0) return cudaSuccess;
        const int block = 256;
        k_hits_to_isect<<<(unsigned)((n + block - 1) / block), block, 0, st>>>(s, reinterpret_cast<const float4 *>(hits), n, out);
        return cudaGetLastError();
}

}  // namespace gzg
