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
// of at most kStaticMaxRays = 65,536 rays, then the traversal kernel's pull
// counter in a 256-byte tail: 4,980,992 bytes.  Every GPU on which
// the library's device code is loaded keeps this array until the process exits.
// In host code `g_static_scratch` is only a host-side stand-in for the symbol,
// never a device address.  Every call looks the device address up again with
// cudaGetSymbolAddress, with the scene's device current, and checks the
// result: the lookup allocates nothing, and a fresh lookup stays right after
// the device's context was reset or recreated (the module is then reloaded and
// the array may sit at another address).
//
// Sharing: every call uses the same array, which keeps the last call's
// contents.  Nothing in it has to start at zero (each call overwrites the rays,
// tMax values and results it uses; the traversal launch clears its pull
// counter).  Calls that overlapped on the GPU would
// race on the array; calls through this entry point are serialised by a
// process-wide lock, so the array must not be touched by anything else.
//
// Stream: the copies and the launch run on the calling thread's per-thread
// default stream (cudaStreamPerThread), which does not wait for the caller's
// other streams unless those are the legacy default stream; the call returns
// after that stream has finished the result copy.
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
constexpr size_t kSchedOffset = kOutOffset + kOutBytes;
constexpr size_t kSchedBytes = 256;
static_assert(kTmaxOffset % 256 == 0 && kOutOffset % 256 == 0 && kSchedOffset % 256 == 0,
              "scratch sections must stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_static_scratch[kSchedOffset + kSchedBytes];

std::mutex g_static_mu;

gzg_status cuda_step(cudaError_t e, const char *what) {
        if (e == cudaSuccess) return GZG_OK;
        return set_error(GZG_ERR_CUDA, std::string("gzg_gpu_traverse_batch_static: ") + what + ": " + cudaGetErrorString(e));
}

// Device address of g_static_scratch on the current device.
gzg_status static_scratch_address(unsigned char **out) {
        void *p = nullptr;
        gzg_status st = cuda_step(cudaGetSymbolAddress(&p, g_static_scratch), "cudaGetSymbolAddress");
        if (st != GZG_OK) return st;
        *out = static_cast<unsigned char *>(p);
        return GZG_OK;
}

// Reads and clears the scene's device error word on `stream` (after the
// launch has been queued there).
gzg_status take_error_word(const DevScene &view, cudaStream_t stream, uint32_t *word) {
        gzg_status st = cuda_step(cudaMemcpyAsync(word, view.err, 4, cudaMemcpyDeviceToHost, stream), "error word read");
        if (st != GZG_OK) return st;
        st = cuda_step(cudaMemsetAsync(view.err, 0, 4, stream), "error word clear");
        if (st != GZG_OK) return st;
        return cuda_step(cudaStreamSynchronize(stream), "error word sync");
}

}  // namespace
}  // namespace gzg

using namespace gzg;

extern "C" GZG_API gzg_status gzg_gpu_traverse_batch_static(gzg_scene *scene, const gzg_ray *rays,
                                                             const float *t_max_values, int64_t count,
                                                             gzg_intersection *results) {
        if (!scene || count < 0 || (count > 0 && (!rays || !t_max_values || !results)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_gpu_traverse_batch_static: null pointer or negative count");
        if (scene_is_instanced(scene))
                return set_error(GZG_ERR_INVALID_ARGUMENT,
                                 "gzg_gpu_traverse_batch_static: two-level scenes take the device calls "
                                 "(gzg_trace_*_device)");
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
        const cudaStream_t stream = cudaStreamPerThread;
        gzg_status st = GZG_OK;
        bool launched = false;
        unsigned char *base = nullptr;
        do {
                st = static_scratch_address(&base);
                if (st != GZG_OK) break;
                st = cuda_step(cudaMemcpyAsync(base, rays, (size_t)count * sizeof(gzg_ray), cudaMemcpyHostToDevice, stream),
                               "ray copy");
                if (st != GZG_OK) break;
                st = cuda_step(cudaMemcpyAsync(base + kTmaxOffset, t_max_values, (size_t)count * sizeof(float),
                                               cudaMemcpyHostToDevice, stream),
                               "tMax copy");
                if (st != GZG_OK) break;
                // the scene's tuned closest-hit launch, as gzg_gpu_traverse_batch
                // uses with default options, with the scratch's pull counter
                LaunchParams p = scene_launch(scene, false);
                p.sched = reinterpret_cast<uint32_t *>(base + kSchedOffset);
                launched = true;
                st = cuda_step(launch_trace(view, p, kRayReference, kOutIntersection, base,
                                            reinterpret_cast<const float *>(base + kTmaxOffset), count,
                                            base + kOutOffset, stream),
                               "trace launch");
                if (st != GZG_OK) break;
                st = cuda_step(cudaMemcpyAsync(results, base + kOutOffset, (size_t)count * sizeof(gzg_intersection),
                                               cudaMemcpyDeviceToHost, stream),
                               "result copy");
                if (st != GZG_OK) break;
                st = cuda_step(cudaStreamSynchronize(stream), "stream sync");
        } while (false);
        // Every exit after the launch reads and clears the scene's error word,
        // so a fault of this call is reported here and never blamed on the
        // next call on the scene (the word is shared with the scene's other
        // entry points, which clear it the same way).
        if (launched) {
                uint32_t word = 0;
                const gzg_status ws = take_error_word(view, stream, &word);
                if (st == GZG_OK && ws != GZG_OK) st = ws;
                if (st == GZG_OK && word != 0) st = kernel_fault(word);
        }
        if (prev != device) cudaSetDevice(prev);
        if (st == GZG_OK) clear_error();
        return st;
}
