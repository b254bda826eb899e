// static_batch.cu - gzg_gpu_traverse_batch_static: the closest-hit host batch
// without any allocation by the library.
//
// Who needs it: hosts that cannot call cudaMalloc / cudaFree / cudaHostAlloc on
// their render path.  Typical cases are a renderer embedded in a process whose
// device memory is owned by another allocator (a framework memory pool that
// reserves almost all of the GPU, so a fresh cudaMalloc fails or steals from
// the pool), and interactive loops that must not call cudaFree because it
// synchronises the whole device.  gzg_gpu_traverse_batch allocates its device
// and pinned staging buffers on first use; this entry point instead stages
// through one fixed array that lives in the library's own device image.
//
// The scratch: g_static_scratch, a file-scope __device__ array holding the
// rays (Ray_C, 24 B), their tMax (4 B) and the results (Intersection_C, 48 B)
// of at most kStaticMaxRays = 65,536 rays: 4,980,736 bytes.  Every GPU on which
// the library's device code is loaded keeps this array until the process exits.
// In host code `g_static_scratch` is only a host-side stand-in for the symbol,
// never a device address: the device address is obtained once per device with
// cudaGetSymbolAddress, with that device current, on the first call that runs
// on the device (so that first call should be made before any stream capture
// the caller might start on that device).
//
// Sharing: every call uses the same array, which keeps the last call's
// contents.  Nothing in it has to start at zero (each call overwrites the rays,
// tMax values and results it uses).  Calls that overlapped on the GPU would
// race on the array; calls through this entry point are serialised by a
// process-wide lock, so the array must not be touched by anything else.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "gzg_internal.h"
#include "kernels.h"

namespace gzg {
namespace {

constexpr int64_t kStaticMaxRays = 65536;
constexpr size_t kRayBytes = (size_t)kStaticMaxRays * sizeof(gzg_ray);
constexpr size_t kTmaxBytes = (size_t)kStaticMaxRays * sizeof(float);
constexpr size_t kOutBytes = (size_t)kStaticMaxRays * sizeof(gzg_intersection);
constexpr size_t kTmaxOffset = kRayBytes;
constexpr size_t kOutOffset = kRayBytes + kTmaxBytes;
static_assert(kTmaxOffset % 256 == 0 && kOutOffset % 256 == 0, "scratch sections must stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_static_scratch[kRayBytes + kTmaxBytes + kOutBytes];

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
void *g_static_addr[kMaxDevices] = {};

// Device address of g_static_scratch on `dev` (which must be current).
gzg_status static_scratch_address(int dev, unsigned char **out) {
        if (dev < 0 || dev >= kMaxDevices)
                return set_error(GZG_ERR_LIMIT, "gzg_gpu_traverse_batch_static: device ordinal above 63");
        if (!g_static_addr[dev]) {
                void *p = nullptr;
                cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
                if (e != cudaSuccess)
                        return set_error(GZG_ERR_CUDA, std::string("gzg_gpu_traverse_batch_static: cudaGetSymbolAddress: ") +
                                                           cudaGetErrorString(e));
                g_static_addr[dev] = p;
        }
        *out = static_cast<unsigned char *>(g_static_addr[dev]);
        return GZG_OK;
}

gzg_status cuda_step(cudaError_t e, const char *what) {
        if (e == cudaSuccess) return GZG_OK;
        return set_error(GZG_ERR_CUDA, std::string("gzg_gpu_traverse_batch_static: ") + what + ": " + cudaGetErrorString(e));
}

}  // namespace
}  // namespace gzg

using namespace gzg;

extern "C" GZG_API gzg_status gzg_gpu_traverse_batch_static(gzg_scene *scene, const gzg_ray *rays,
                                                             const float *t_max_values, int64_t count,
                                                             gzg_intersection *results) {
        if (!scene || count < 0 || (count > 0 && (!rays || !t_max_values || !results)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_gpu_traverse_batch_static: null pointer or negative count");
        if (count > kStaticMaxRays)
                return set_error(GZG_ERR_LIMIT, "gzg_gpu_traverse_batch_static: " + std::to_string(count) +
                                                    " rays exceed the static scratch capacity of 65536 rays per call");
        if (count == 0) return clear_error();

        std::lock_guard<std::mutex> lock(g_static_mu);
        DevScene view;
        int device = 0, wide_depth = 0;
        scene_view(scene, &view, &device, &wide_depth);
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != device) cudaSetDevice(device);
        gzg_status st = GZG_OK;
        unsigned char *base = nullptr;
        do {
                st = static_scratch_address(device, &base);
                if (st != GZG_OK) break;
                st = cuda_step(cudaMemcpy(base, rays, (size_t)count * sizeof(gzg_ray), cudaMemcpyHostToDevice), "ray copy");
                if (st != GZG_OK) break;
                st = cuda_step(cudaMemcpy(base + kTmaxOffset, t_max_values, (size_t)count * sizeof(float),
                                          cudaMemcpyHostToDevice),
                               "tMax copy");
                if (st != GZG_OK) break;
                LaunchParams p{};
                p.traversal = GZG_TRAVERSAL_WIDE;
                p.leaf_test = GZG_LEAF_MOLLER_TRUMBORE;
                p.wide_depth = wide_depth;
                st = cuda_step(launch_trace(view, p, kRayReference, kOutIntersection, base,
                                            reinterpret_cast<const float *>(base + kTmaxOffset), count,
                                            base + kOutOffset, /*legacy default stream*/ 0),
                               "trace launch");
                if (st != GZG_OK) break;
                st = cuda_step(cudaMemcpy(results, base + kOutOffset, (size_t)count * sizeof(gzg_intersection),
                                          cudaMemcpyDeviceToHost),
                               "result copy");
                if (st != GZG_OK) break;
                uint32_t word = 0;
                st = gzg_scene_error_word(scene, &word, 1);
                if (st == GZG_OK && word != 0)
                        st = set_error(GZG_ERR_KERNEL_FAULT,
                                       "gzg_gpu_traverse_batch_static: kernel error word " + std::to_string(word));
        } while (false);
        if (prev != device) cudaSetDevice(prev);
        if (st == GZG_OK) clear_error();
        return st;
}
