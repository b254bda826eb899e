// shade_live.cu - gzg_gpu_shade_batch, the drop-in for mojo_gpu_shade_batch
// (Sources/mojoKernel/kernel.mojo:788-846): the live shading step of Gonzales'
// tile loop (Core/Tile.swift:137-155) on host PathState_C / Intersection_C
// arrays, one thread per path, restating shade_core (kernel.mojo:676-773):
// emission ends a path, a diffuse hit bounces with a cosine sample driven by
// PCG32 (kernel.mojo:99-118, reseeded from the path's state and increment on
// every call, only the state written back), anything else ends the path.
// Unlike the reference, a material or mesh index out of range ends the path
// and sets the scene's error word instead of reading out of bounds.
#include <cuda_runtime.h>

#include <string>

#include "gzg_internal.h"
#include "kernels.h"

namespace gzg {
namespace {

struct Pcg32 {
        uint64_t state, inc;
        __device__ Pcg32(uint64_t initstate, uint64_t initseq) {
                state = 0;
                inc = (initseq << 1) | 1ull;
                next_uint();
                state += initstate;
                next_uint();
        }
        __device__ uint32_t next_uint() {
                const uint64_t old = state;
                state = old * 6364136223846793005ull + inc;
                const uint32_t xorshifted = (uint32_t)(((old >> 18) ^ old) >> 27);
                const uint32_t rot = (uint32_t)(old >> 59);
                return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
        }
        __device__ float next_float() { return __fmul_rn((float)(next_uint() >> 8), 1.0f / 16777216.0f); }
};

__global__ void k_shade_live(DevScene s, gzg_path_state *paths, const gzg_intersection *isects, int64_t n) {
        const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (tid >= n) return;
        gzg_path_state p = paths[tid];
        if (p.active == 0) return;
        const gzg_intersection in = isects[tid];
        if (in.hit == 0) {
                paths[tid].active = 0;
                return;
        }
        const int64_t mi = in.prim_id.material_index;
        if (mi < 0 || mi >= s.material_count) {
                atomicOr(s.err, kErrBadIndex);
                paths[tid].active = 0;
                return;
        }
        const float4 alb = __ldg(s.materials + 2 * mi), em = __ldg(s.materials + 2 * mi + 1);
        const int type = (int)alb.w;
        if (type == 2) {
                p.estimate[0] = __fadd_rn(p.estimate[0], __fmul_rn(p.throughput[0], em.x));
                p.estimate[1] = __fadd_rn(p.estimate[1], __fmul_rn(p.throughput[1], em.y));
                p.estimate[2] = __fadd_rn(p.estimate[2], __fmul_rn(p.throughput[2], em.z));
                p.active = 0;
                paths[tid] = p;
                return;
        }
        if (type != 1) {
                paths[tid].active = 0;
                return;
        }
        int64_t mesh, base;
        if (!prim_triangle(in.prim_id, &mesh, &base) || mesh < 0 || mesh >= s.mesh_count || base < 0 ||
            base + 2 >= __ldg(s.mesh_sizes + 2 * mesh + 1)) {
                if (in.prim_id.type < 0 || in.prim_id.type > 3) {
                        paths[tid].active = 0;
                        return;
                }
                atomicOr(s.err, kErrBadIndex);
                paths[tid].active = 0;
                return;
        }
        const gzg_triangle_mesh m = s.meshes[mesh];
        const int64_t npts = __ldg(s.mesh_sizes + 2 * mesh);
        float v[3][3];
        for (int c = 0; c < 3; ++c) {
                const int64_t vi = __ldg(m.vertex_indices + base + c);
                if (vi < 0 || vi * 4 + 3 > npts) {
                        atomicOr(s.err, kErrBadIndex);
                        paths[tid].active = 0;
                        return;
                }
                v[c][0] = __ldg(m.points + vi * 4);
                v[c][1] = __ldg(m.points + vi * 4 + 1);
                v[c][2] = __ldg(m.points + vi * 4 + 2);
        }
        const float e1[3] = {__fsub_rn(v[1][0], v[0][0]), __fsub_rn(v[1][1], v[0][1]), __fsub_rn(v[1][2], v[0][2])};
        const float e2[3] = {__fsub_rn(v[2][0], v[0][0]), __fsub_rn(v[2][1], v[0][1]), __fsub_rn(v[2][2], v[0][2])};
        float nrm[3] = {__fsub_rn(__fmul_rn(e1[1], e2[2]), __fmul_rn(e1[2], e2[1])),
                        __fsub_rn(__fmul_rn(e1[2], e2[0]), __fmul_rn(e1[0], e2[2])),
                        __fsub_rn(__fmul_rn(e1[0], e2[1]), __fmul_rn(e1[1], e2[0]))};
        const float nlen = __fadd_rn(__fadd_rn(__fmul_rn(nrm[0], nrm[0]), __fmul_rn(nrm[1], nrm[1])), __fmul_rn(nrm[2], nrm[2]));
        if (nlen > 0.0f) {
                const float sc = __fdiv_rn(1.0f, sqrtf(nlen));
                for (int k = 0; k < 3; ++k) nrm[k] = __fmul_rn(nrm[k], sc);
        }
        const float rd[3] = {p.ray.dir_x, p.ray.dir_y, p.ray.dir_z};
        const float nd = __fadd_rn(__fadd_rn(__fmul_rn(nrm[0], rd[0]), __fmul_rn(nrm[1], rd[1])), __fmul_rn(nrm[2], rd[2]));
        if (nd > 0.0f)
                for (int k = 0; k < 3; ++k) nrm[k] = -nrm[k];
        Pcg32 pcg(p.pcg_state, p.pcg_inc);
        const float u1 = pcg.next_float();
        const float u2 = pcg.next_float();
        p.pcg_state = pcg.state;
        const float r = sqrtf(u1);
        const float theta = __fmul_rn(__fmul_rn(2.0f, 3.14159265359f), u2);
        const float x = __fmul_rn(r, cosf(theta));
        const float y = __fmul_rn(r, sinf(theta));
        const float z2 = __fsub_rn(1.0f, u1);
        const float z = sqrtf(z2 > 0.0f ? z2 : 0.0f);
        const float sign = nrm[2] >= 0.0f ? 1.0f : -1.0f;
        const float a = __fdiv_rn(-1.0f, __fadd_rn(sign, nrm[2]));
        const float b = __fmul_rn(__fmul_rn(nrm[0], nrm[1]), a);
        const float t[3] = {__fadd_rn(1.0f, __fmul_rn(__fmul_rn(__fmul_rn(sign, nrm[0]), nrm[0]), a)), __fmul_rn(sign, b),
                            __fmul_rn(-sign, nrm[0])};
        const float bt[3] = {b, __fadd_rn(sign, __fmul_rn(__fmul_rn(nrm[1], nrm[1]), a)), -nrm[1]};
        float dir[3];
        for (int k = 0; k < 3; ++k) dir[k] = __fadd_rn(__fadd_rn(__fmul_rn(t[k], x), __fmul_rn(bt[k], y)), __fmul_rn(nrm[k], z));
        const float dlen = __fadd_rn(__fadd_rn(__fmul_rn(dir[0], dir[0]), __fmul_rn(dir[1], dir[1])), __fmul_rn(dir[2], dir[2]));
        if (dlen > 0.0f) {
                const float sc = __fdiv_rn(1.0f, sqrtf(dlen));
                for (int k = 0; k < 3; ++k) dir[k] = __fmul_rn(dir[k], sc);
        }
        const float ro[3] = {p.ray.org_x, p.ray.org_y, p.ray.org_z};
        float org[3];
        for (int k = 0; k < 3; ++k) org[k] = __fadd_rn(__fadd_rn(ro[k], __fmul_rn(rd[k], in.t_hit)), __fmul_rn(nrm[k], 0.0001f));
        p.ray.org_x = org[0];
        p.ray.org_y = org[1];
        p.ray.org_z = org[2];
        p.ray.dir_x = dir[0];
        p.ray.dir_y = dir[1];
        p.ray.dir_z = dir[2];
        p.throughput[0] = __fmul_rn(p.throughput[0], alb.x);
        p.throughput[1] = __fmul_rn(p.throughput[1], alb.y);
        p.throughput[2] = __fmul_rn(p.throughput[2], alb.z);
        paths[tid] = p;
}

gzg_status cuda_fail2(cudaError_t e, const char *what) {
        return set_error(e == cudaErrorMemoryAllocation ? GZG_ERR_OUT_OF_MEMORY : GZG_ERR_CUDA,
                         std::string("gzg_gpu_shade_batch: ") + what + ": " + cudaGetErrorString(e));
}

}  // namespace
}  // namespace gzg

using namespace gzg;

extern "C" GZG_API gzg_status gzg_gpu_shade_batch(gzg_scene *scene, gzg_path_state *paths, int64_t count,
                                                  const gzg_intersection *intersections) {
        if (!scene || count < 0 || (count > 0 && (!paths || !intersections)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_gpu_shade_batch: null pointer or negative count");
        if (count == 0) return clear_error();
        DevScene view;
        int device = 0, depth = 0;
        scene_view(scene, &view, &device, &depth);
        if (view.material_count <= 0)
                return set_error(GZG_ERR_BAD_SCENE, "gzg_gpu_shade_batch: the scene was uploaded without materials");
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != device) cudaSetDevice(device);
        cudaStream_t st = nullptr;
        gzg_status status = GZG_OK;
        void *d_paths = nullptr, *d_isects = nullptr;
        const size_t pb = (size_t)count * sizeof(gzg_path_state), ib = (size_t)count * sizeof(gzg_intersection);
        do {
                cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
                if (e != cudaSuccess) {
                        status = cuda_fail2(e, "stream");
                        break;
                }
                if ((e = cudaMallocAsync(&d_paths, pb, st)) != cudaSuccess ||
                    (e = cudaMallocAsync(&d_isects, ib, st)) != cudaSuccess) {
                        status = cuda_fail2(e, "staging allocation");
                        break;
                }
                if ((e = cudaMemcpyAsync(d_paths, paths, pb, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
                    (e = cudaMemcpyAsync(d_isects, intersections, ib, cudaMemcpyHostToDevice, st)) != cudaSuccess) {
                        status = cuda_fail2(e, "upload");
                        break;
                }
                k_shade_live<<<(unsigned)((count + 127) / 128), 128, 0, st>>>(
                    view, static_cast<gzg_path_state *>(d_paths), static_cast<const gzg_intersection *>(d_isects), count);
                if ((e = cudaGetLastError()) != cudaSuccess ||
                    (e = cudaMemcpyAsync(paths, d_paths, pb, cudaMemcpyDeviceToHost, st)) != cudaSuccess) {
                        status = cuda_fail2(e, "shade");
                        break;
                }
                status = wait_stream(st, "gzg_gpu_shade_batch");
        } while (false);
        // stream-ordered frees: after a wait that ran out (the copy back may
        // still be writing `paths`) they run when the stream's work is done
        if (d_paths) cudaFreeAsync(d_paths, st);
        if (d_isects) cudaFreeAsync(d_isects, st);
        if (st) {
                if (status != GZG_ERR_TIMEOUT) cudaStreamSynchronize(st);
                cudaStreamDestroy(st);
        }
        if (!status) {
                uint32_t word = 0;
                status = gzg_scene_error_word(scene, &word, 1);
                if (!status && word)
                        status = set_error(GZG_ERR_KERNEL_FAULT, "gzg_gpu_shade_batch: index out of range (error word " +
                                                                     std::to_string(word) + ")");
        }
        if (prev != device) cudaSetDevice(prev);
        if (!status) clear_error();
        return status;
}
