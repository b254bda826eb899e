// api.cu - the C ABI of libgzg.so (include/gzg.h): scene upload, host batch
// calls (drop-in for the reference's mojo_gpu_* exports, kernel.mojo:399-673)
// and device-resident trace calls.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <memory>
#include <chrono>
#include <cstdlib>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "gzg_internal.h"
#include "kernels.h"

namespace gzg {

namespace {
thread_local std::string g_last_error;
}

gzg_status set_error(gzg_status code, const std::string &msg) {
        g_last_error = msg;
        return code;
}
gzg_status clear_error() {
        g_last_error.clear();
        return GZG_OK;
}

namespace {

gzg_status cuda_fail(cudaError_t e, const char *what) {
        const gzg_status code = (e == cudaErrorMemoryAllocation) ? GZG_ERR_OUT_OF_MEMORY : GZG_ERR_CUDA;
        return set_error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define GZG_CK(call, what)                                  \
        do {                                                \
                cudaError_t e_ = (call);                    \
                if (e_ != cudaSuccess) return cuda_fail(e_, what); \
        } while (0)

// Switches to the scene's device for the duration of a call.
class DeviceGuard {
      public:
        explicit DeviceGuard(int dev) {
                cudaGetDevice(&prev_);
                if (prev_ != dev) cudaSetDevice(dev);
                dev_ = dev;
        }
        ~DeviceGuard() {
                if (prev_ != dev_) cudaSetDevice(prev_);
        }

      private:
        int prev_ = 0, dev_ = 0;
};

constexpr int kSlots = 4;
constexpr int64_t kChunk = 1 << 19;  // rays per pipelined chunk (512K x 4 streams: 2 % faster end to end than 1M x 3)

// Per-call staging: device buffers and pinned host buffers for kSlots chunks
// in flight, each slot with its own stream and its pull counter for the
// persistent kernel.
struct Staging {
        cudaStream_t st[kSlots] = {};
        void *d_in[kSlots] = {}, *d_tmax[kSlots] = {}, *d_out[kSlots] = {};
        void *h_in[kSlots] = {}, *h_tmax[kSlots] = {}, *h_out[kSlots] = {};
        uint32_t *d_sched = nullptr;  // one word per slot
        ~Staging() {
                cudaFree(d_sched);
                for (int k = 0; k < kSlots; ++k) {
                        if (st[k]) cudaStreamDestroy(st[k]);
                        cudaFree(d_in[k]);
                        cudaFree(d_tmax[k]);
                        cudaFree(d_out[k]);
                        cudaFreeHost(h_in[k]);
                        cudaFreeHost(h_tmax[k]);
                        cudaFreeHost(h_out[k]);
                }
        }
};

bool is_pinned(const void *p) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
                cudaGetLastError();
                return false;
        }
        return a.type == cudaMemoryTypeHost;
}

}  // namespace

// Pull counters of the persistent kernels for the device calls, which run on
// the callers' streams: kWords device words (one allocation, made by the first
// call that needs one), each with an event recorded after the last launch that
// used it.  A launch takes the next word, makes its stream wait for that
// word's previous launch, and records the word's event after itself, so
// launches that share a word run one after another whatever their streams,
// while up to kWords launches on different streams can run at once.
struct PullRing {
        static constexpr int kWords = 32;
        uint32_t *words = nullptr;
        cudaEvent_t ev[kWords] = {};
        bool recorded[kWords] = {};
        int next = 0;
        std::mutex mu;

        cudaError_t create() {
                cudaError_t e = cudaMalloc(&words, kWords * sizeof(uint32_t));
                for (int k = 0; e == cudaSuccess && k < kWords; ++k)
                        e = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming);
                if (e != cudaSuccess) release();
                return e;
        }
        void release() {
                for (cudaEvent_t &e : ev) {
                        if (e) cudaEventDestroy(e);
                        e = nullptr;
                }
                cudaFree(words);
                words = nullptr;
        }
};

// Launch configuration chosen by gzg_scene_autotune (or the defaults).
struct TunedLaunch {
        int block_size = 128;
        int blocks_per_sm = 0;  // occupancy limit
        int stack_depth = 0;    // by tree depth
        int l1_carveout = -1;   // driver default
};

}  // namespace gzg

using namespace gzg;

struct gzg_scene {
        int device = 0;
        DevScene dev{};
        std::vector<void *> allocs;
        gzg_scene_info info{};
        TunedLaunch tuned_closest, tuned_any;
        WideBvh host_wide;          // host copy of the wide tree (two-level assembly)
        float root_bounds[6] = {0, 0, 0, 0, 0, 0};
        bool instanced = false;
        float build_ms = -1.0f;     // device time of gzg_gpu_build_scene's tree build
        std::vector<int64_t> mesh_vertices;  // vertices per mesh (gzg_scene_set_vertex_attributes)
        // host copies of the shading arrays (batch assembly)
        HostShading host_shading;
        std::mutex pool_mu;
        std::vector<std::unique_ptr<Staging>> pool;
        PullRing pull;

        ~gzg_scene() {
                DeviceGuard g(device);
                pool.clear();
                pull.release();
                for (void *p : allocs) cudaFree(p);
        }

        template <class T>
        gzg_status upload(const T *host, size_t count, const T **dst, const char *what) {
                void *d = nullptr;
                const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
                GZG_CK(cudaMalloc(&d, bytes), what);
                allocs.push_back(d);
                if (count) GZG_CK(cudaMemcpy(d, host, count * sizeof(T), cudaMemcpyHostToDevice), what);
                info.device_bytes += (int64_t)bytes;
                *dst = reinterpret_cast<const T *>(d);
                return GZG_OK;
        }

        // A device array the scene owns, left uninitialised.
        template <class T>
        gzg_status alloc(T **dst, size_t count, const char *what) {
                void *d = nullptr;
                const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
                GZG_CK(cudaMalloc(&d, bytes), what);
                allocs.push_back(d);
                info.device_bytes += (int64_t)bytes;
                *dst = reinterpret_cast<T *>(d);
                return GZG_OK;
        }

        gzg_status acquire(std::unique_ptr<Staging> *out) {
                {
                        std::lock_guard<std::mutex> lk(pool_mu);
                        if (!pool.empty()) {
                                *out = std::move(pool.back());
                                pool.pop_back();
                                return GZG_OK;
                        }
                }
                auto s = std::make_unique<Staging>();
                GZG_CK(cudaMalloc(&s->d_sched, kSlots * sizeof(uint32_t)), "staging schedule words");
                for (int k = 0; k < kSlots; ++k) {
                        GZG_CK(cudaStreamCreateWithFlags(&s->st[k], cudaStreamNonBlocking), "staging stream");
                        GZG_CK(cudaMalloc(&s->d_in[k], kChunk * sizeof(gzg_ray_d)), "staging device buffer");
                        GZG_CK(cudaMalloc(&s->d_tmax[k], kChunk * sizeof(float)), "staging device buffer");
                        GZG_CK(cudaMalloc(&s->d_out[k], kChunk * sizeof(gzg_intersection)), "staging device buffer");
                        GZG_CK(cudaHostAlloc(&s->h_in[k], kChunk * sizeof(gzg_ray), cudaHostAllocDefault), "pinned buffer");
                        GZG_CK(cudaHostAlloc(&s->h_tmax[k], kChunk * sizeof(float), cudaHostAllocDefault), "pinned buffer");
                        GZG_CK(cudaHostAlloc(&s->h_out[k], kChunk * sizeof(gzg_intersection), cudaHostAllocDefault),
                               "pinned buffer");
                }
                *out = std::move(s);
                return GZG_OK;
        }
        void release(std::unique_ptr<Staging> s) {
                std::lock_guard<std::mutex> lk(pool_mu);
                pool.push_back(std::move(s));
        }
};

gzg_status gzg::wait_stream(void *stream, const char *what) {
        int64_t limit_us = 300000000;
        if (const char *env = std::getenv("GZG_WAIT_LIMIT_US")) limit_us = std::atoll(env);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        cudaEvent_t ev = nullptr;
        cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(ev, st);
        if (e != cudaSuccess) {
                if (ev) cudaEventDestroy(ev);
                return set_error(GZG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        }
        const auto t0 = std::chrono::steady_clock::now();
        gzg_status status = GZG_OK;
        for (;;) {
                e = cudaEventQuery(ev);
                if (e == cudaSuccess) break;
                if (e != cudaErrorNotReady) {
                        status = set_error(GZG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
                        break;
                }
                const int64_t us =
                    std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count();
                if (limit_us > 0 && us >= limit_us) {
                        status = set_error(GZG_ERR_TIMEOUT, std::string(what) + ": no completion within " +
                                                                std::to_string(limit_us) + " us (GZG_WAIT_LIMIT_US)");
                        break;
                }
                // spin with yields for the first 2 ms (batch chunks finish in
                // well under that), then poll every 50 us
                if (us < 2000)
                        std::this_thread::yield();
                else
                        std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
        cudaEventDestroy(ev);
        return status;
}

gzg_status gzg::kernel_fault(uint32_t w) {
        std::string m = "kernel error word " + std::to_string(w) + ":";
        if (w & kErrStackOverflow) m += " traversal stack overflow";
        if (w & kErrStepCap) m += " step cap exceeded (cyclic or corrupt tree)";
        if (w & kErrBadIndex) m += " index out of range";
        return set_error(GZG_ERR_KERNEL_FAULT, m);
}

namespace {

// Options fields left at 0 take the scene's tuned values (gzg_scene_autotune),
// separately for closest-hit and any-hit launches.
LaunchParams params_for(const gzg_scene *s, const gzg_trace_options *o, bool any) {
        const TunedLaunch &t = any ? s->tuned_any : s->tuned_closest;
        LaunchParams p;
        p.traversal = o ? o->traversal : GZG_TRAVERSAL_WIDE;
        p.leaf_test = o ? o->leaf_test : GZG_LEAF_MOLLER_TRUMBORE;
        p.block_size = (o && o->block_size) ? o->block_size : t.block_size;
        p.blocks_per_sm = (o && o->blocks_per_sm) ? o->blocks_per_sm : t.blocks_per_sm;
        p.stack_depth = (o && o->stack_depth) ? o->stack_depth : t.stack_depth;
        p.l1_carveout = (o && o->l1_carveout) ? o->l1_carveout : t.l1_carveout;
        p.wide_depth = s->info.wide_depth;
        p.counters = o ? reinterpret_cast<unsigned long long *>(o->fetch_counters) : nullptr;
        p.n_dev = nullptr;
        p.inst_out = nullptr;
        p.sched = nullptr;
        return p;
}

gzg_status check_options(const gzg_trace_options *o) {
        if (!o) return GZG_OK;
        if (o->traversal != GZG_TRAVERSAL_WIDE && o->traversal != GZG_TRAVERSAL_BVH2 &&
            o->traversal != GZG_TRAVERSAL_WIDE_ONE_RAY_PER_THREAD)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "unknown traversal");
        if (o->leaf_test != GZG_LEAF_MOLLER_TRUMBORE && o->leaf_test != GZG_LEAF_WATERTIGHT)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "unknown leaf test");
        return GZG_OK;
}

gzg_status read_error_word(gzg_scene *s, uint32_t *word, bool clear) {
        GZG_CK(cudaMemcpy(word, s->dev.err, 4, cudaMemcpyDeviceToHost), "error word read");
        if (clear) GZG_CK(cudaMemset(s->dev.err, 0, 4), "error word clear");
        return GZG_OK;
}


// launch_trace for the device calls, on the caller's stream, with one of the
// scene's pull counters.  A stream being captured into a graph gets the static
// schedule (no word, no event waits across the capture's boundary).
cudaError_t device_trace(gzg_scene *scene, LaunchParams p, int out_fmt, const void *rays, int64_t n, void *out,
                         cudaStream_t st) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
                cudaGetLastError();
                cs = cudaStreamCaptureStatusActive;
        }
        p.sched = nullptr;
        if (cs != cudaStreamCaptureStatusNone || n <= 0)
                return launch_trace(scene->dev, p, kRayDevice, out_fmt, rays, nullptr, n, out, st);
        PullRing &r = scene->pull;
        std::lock_guard<std::mutex> lk(r.mu);
        if (!r.words) {
                const cudaError_t e = r.create();
                if (e != cudaSuccess) return e;
        }
        const int k = r.next;
        r.next = (k + 1) % PullRing::kWords;
        if (r.recorded[k]) {
                const cudaError_t e = cudaStreamWaitEvent(st, r.ev[k], 0);
                if (e != cudaSuccess) return e;
        }
        p.sched = r.words + k;
        const cudaError_t e = launch_trace(scene->dev, p, kRayDevice, out_fmt, rays, nullptr, n, out, st);
        if (e != cudaSuccess) return e;
        r.recorded[k] = true;
        return cudaEventRecord(r.ev[k], st);
}

// Host batch: chunks of Ray_C + tMax through kSlots streams; results are
// `out_bytes` per ray in format `out_fmt`.
gzg_status host_batch(gzg_scene *s, const gzg_ray *rays, const float *tmax, int64_t count, void *results,
                      size_t out_bytes, int out_fmt, const gzg_trace_options *opt) {
        if (!s || count < 0 || (count > 0 && (!rays || !tmax || !results)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "batch call: null pointer or negative count");
        if (s->instanced)
                return set_error(GZG_ERR_INVALID_ARGUMENT,
                                 "batch call: two-level scenes take the device calls (gzg_trace_*_device)");
        gzg_status st = check_options(opt);
        if (st != GZG_OK) return st;
        if (count == 0) return clear_error();
        DeviceGuard g(s->device);
        std::unique_ptr<Staging> stg;
        st = s->acquire(&stg);
        if (st != GZG_OK) return st;
        LaunchParams p = params_for(s, opt, out_fmt == kOutAnyPrim || out_fmt == kOutOccluded);
        const bool direct = is_pinned(rays) && is_pinned(tmax) && is_pinned(results);
        const int64_t nchunks = (count + kChunk - 1) / kChunk;
        char *res = reinterpret_cast<char *>(results);
        // A wait that ran out leaves chunks in flight on the staging streams:
        // their buffers are left to them (never freed nor pooled again).
        auto abandon = [&](gzg_status s) -> gzg_status {
                if (s == GZG_ERR_TIMEOUT) stg.release();
                return s;
        };
        auto drain = [&](int64_t c) -> gzg_status {
                const int k = (int)(c % kSlots);
                const gzg_status ws = wait_stream(stg->st[k], "batch chunk");
                if (ws != GZG_OK) return ws;
                const int64_t off = c * kChunk, n = std::min(kChunk, count - off);
                std::memcpy(res + off * out_bytes, stg->h_out[k], (size_t)n * out_bytes);
                return GZG_OK;
        };
        for (int64_t c = 0; c < nchunks; ++c) {
                const int k = (int)(c % kSlots);
                const int64_t off = c * kChunk, n = std::min(kChunk, count - off);
                cudaStream_t stream = stg->st[k];
                const void *src_rays = rays + off;
                const void *src_tmax = tmax + off;
                if (!direct) {
                        if (c >= kSlots) {
                                st = drain(c - kSlots);
                                if (st != GZG_OK) return abandon(st);
                        }
                        std::memcpy(stg->h_in[k], rays + off, (size_t)n * sizeof(gzg_ray));
                        std::memcpy(stg->h_tmax[k], tmax + off, (size_t)n * sizeof(float));
                        src_rays = stg->h_in[k];
                        src_tmax = stg->h_tmax[k];
                }
                GZG_CK(cudaMemcpyAsync(stg->d_in[k], src_rays, (size_t)n * sizeof(gzg_ray), cudaMemcpyHostToDevice, stream),
                       "ray upload");
                GZG_CK(cudaMemcpyAsync(stg->d_tmax[k], src_tmax, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, stream),
                       "tMax upload");
                p.sched = stg->d_sched + k;  // this slot's stream orders its launches
                GZG_CK(launch_trace(s->dev, p, kRayReference, out_fmt, stg->d_in[k],
                                    reinterpret_cast<const float *>(stg->d_tmax[k]), n, stg->d_out[k], stream),
                       "trace launch");
                void *dst = direct ? (void *)(res + off * out_bytes) : stg->h_out[k];
                GZG_CK(cudaMemcpyAsync(dst, stg->d_out[k], (size_t)n * out_bytes, cudaMemcpyDeviceToHost, stream),
                       "result download");
        }
        if (!direct) {
                for (int64_t c = std::max<int64_t>(0, nchunks - kSlots); c < nchunks; ++c) {
                        st = drain(c);
                        if (st != GZG_OK) return abandon(st);
                }
        }
        for (int k = 0; k < kSlots; ++k) {
                st = wait_stream(stg->st[k], "batch sync");
                if (st != GZG_OK) return abandon(st);
        }
        s->release(std::move(stg));
        uint32_t w = 0;
        st = read_error_word(s, &w, true);
        if (st != GZG_OK) return st;
        if (w) return kernel_fault(w);
        return clear_error();
}

}  // namespace

extern "C" {

GZG_API bool gzg_gpu_available(void) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
                cudaGetLastError();
                return false;
        }
        int dev = 0, major = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
        return major == 10;
}

GZG_API const char *gzg_last_error(void) { return g_last_error.c_str(); }

namespace {

// Materials, area lights (from the prim-order triangles) and the host copies
// of a scene's shading arrays; the wide tree and pv0..2 move into the scene.
gzg_status attach_shading(gzg_scene *scene, WideBvh &&wide, const gzg_prim_id *prim_ids, int64_t prim_count,
                          std::vector<float4_> &&pv0, std::vector<float4_> &&pv1, std::vector<float4_> &&pv2,
                          const gzg_material *materials, int64_t material_count) {
        DevScene &d = scene->dev;
        const float4 *f;
        gzg_status st;
        // Shading data for the path integrator.  Materials: albedo + type,
        // emission (Material_C, mojo_kernel.h:11-15).  Lights: one per
        // area-light triangle prim, in light-index order (SceneDescription
        // creates one AreaLight per triangle), power = average radiance x area
        // x pi (AreaLight.swift:47-49), with the running power sum the power
        // light sampler searches (PowerLightSampler.swift:20-38).
        std::vector<float4_> mats((size_t)std::max<int64_t>(material_count, 0) * 2);
        for (int64_t k = 0; k < material_count; ++k) {
                const gzg_material &m = materials[k];
                mats[2 * k] = float4_{m.albedo[0], m.albedo[1], m.albedo[2], (float)m.type};
                mats[2 * k + 1] = float4_{m.emission[0], m.emission[1], m.emission[2], 0.0f};
        }
        std::vector<std::pair<int64_t, int64_t>> light_prims;
        for (int64_t k = 0; k < prim_count; ++k) {
                int64_t mesh, base;
                if (prim_ids[k].type == 3 && prim_triangle(prim_ids[k], &mesh, &base)) light_prims.push_back({prim_ids[k].id1, k});
        }
        std::sort(light_prims.begin(), light_prims.end());
        std::vector<float4_> lights;
        std::vector<float> cdf;
        float total = 0.0f, run = 0.0f;
        for (size_t i = 0; i < light_prims.size(); ++i) {
                const int64_t k = light_prims[i].second;
                const float4_ a = pv0[k], b = pv1[k], c = pv2[k];
                const float e1[3] = {b.x - a.x, b.y - a.y, b.z - a.z}, e2[3] = {c.x - a.x, c.y - a.y, c.z - a.z};
                const float cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2],
                            cz = e1[0] * e2[1] - e1[1] * e2[0];
                const float area = 0.5f * std::sqrt(cx * cx + cy * cy + cz * cz);
                float le[3] = {0, 0, 0};
                const int64_t mi = prim_ids[k].material_index;
                if (mi >= 0 && mi < material_count)
                        for (int j = 0; j < 3; ++j) le[j] = materials[mi].emission[j];
                const float power = (le[0] + le[1] + le[2]) / 3.0f * area * 3.14159265358979323846f;
                lights.push_back(float4_{a.x, a.y, a.z, area});
                lights.push_back(float4_{b.x, b.y, b.z, power});
                lights.push_back(float4_{c.x, c.y, c.z, 0.0f});
                lights.push_back(float4_{le[0], le[1], le[2], 0.0f});
                run = i == 0 ? power : run + power;
                cdf.push_back(run);
                total = total + power;
        }
        st = scene->upload(reinterpret_cast<const float4 *>(mats.data()), mats.size(), &f, "materials");
        if (st != GZG_OK) return st;
        d.materials = f;
        st = scene->upload(reinterpret_cast<const float4 *>(lights.data()), lights.size(), &f, "lights");
        if (st != GZG_OK) return st;
        d.lights = f;
        const float *cdf_d;
        st = scene->upload(cdf.data(), cdf.size(), &cdf_d, "light cdf");
        if (st != GZG_OK) return st;
        d.light_cdf = cdf_d;
        d.material_count = (int32_t)material_count;
        d.light_count = (int32_t)light_prims.size();
        d.light_total_power = total;

        scene->host_wide = std::move(wide);
        HostShading &hsd = scene->host_shading;
        hsd.pv0 = std::move(pv0);
        hsd.pv1 = std::move(pv1);
        hsd.pv2 = std::move(pv2);
        hsd.prims.assign(prim_ids, prim_ids + prim_count);
        hsd.materials = std::move(mats);
        hsd.lights = std::move(lights);
        hsd.light_cdf = std::move(cdf);
        hsd.light_total = total;
        return GZG_OK;
}

// gzg_gpu_upload_scene (bvh2_nodes given: the host's tree, converted on the
// host) and gzg_gpu_build_scene (build given: the tree built on the device).
gzg_status upload_scene(const gzg_bvh2_node *bvh2_nodes, int64_t bvh2_node_count, const gzg_prim_id *prim_ids,
                        int64_t prim_count, const gzg_triangle_mesh *meshes, int64_t mesh_count,
                        const int64_t *mesh_points_counts, const int64_t *mesh_vertex_indices_counts,
                        const gzg_material *materials, int64_t material_count, const gzg_build_options *build,
                        gzg_scene **out_scene, const char *fn) {
        const std::string name(fn);
        if (!out_scene) return set_error(GZG_ERR_INVALID_ARGUMENT, name + ": out_scene is NULL");
        *out_scene = nullptr;
        if ((!build && (bvh2_node_count <= 0 || !bvh2_nodes)) || prim_count < 0 || (prim_count > 0 && !prim_ids) ||
            mesh_count < 0 || (mesh_count > 0 && (!meshes || !mesh_points_counts || !mesh_vertex_indices_counts)) ||
            material_count < 0 || (material_count > 0 && !materials))
                return set_error(GZG_ERR_INVALID_ARGUMENT, name + ": bad arguments");
        if (build && (build->leaf_size < 0 || build->leaf_size > 4))
                return set_error(GZG_ERR_INVALID_ARGUMENT, name + ": leaf_size must be 0 (default 1) to 4");
        if (build && (build->builder < 0 || build->builder > GZG_BUILD_PLOC || build->radius < 0 || build->radius > 64))
                return set_error(GZG_ERR_INVALID_ARGUMENT, name + ": unknown builder or radius outside 0..64");
        if (prim_count > INT32_MAX - 1 || bvh2_node_count > INT32_MAX)
                return set_error(GZG_ERR_LIMIT, name + ": more than 2^31 prims or nodes");
        // Host-side validation and conversion first: a malformed scene is
        // reported as GZG_ERR_BAD_SCENE whether or not a device is present.
        WideBvh wide;
        int32_t bvh2_depth = 0;
        gzg_status st;
        if (!build) {
                st = build_wide_bvh(bvh2_nodes, bvh2_node_count, prim_ids, prim_count, meshes, mesh_count,
                                    mesh_points_counts, mesh_vertex_indices_counts, &wide, &bvh2_depth);
                if (st != GZG_OK) return st;
        } else {
                // every triangle prim must resolve (no tree limits which ones are read)
                for (int64_t k = 0; k < prim_count; ++k) {
                        int64_t mesh, base;
                        if (!prim_triangle(prim_ids[k], &mesh, &base)) continue;
                        bool ok = mesh >= 0 && mesh < mesh_count && base >= 0 &&
                                  base + 2 < mesh_vertex_indices_counts[mesh] && meshes[mesh].vertex_indices &&
                                  meshes[mesh].points;
                        for (int c = 0; ok && c < 3; ++c) {
                                const int64_t v = meshes[mesh].vertex_indices[base + c];
                                ok = v >= 0 && v * 4 + 3 <= mesh_points_counts[mesh];
                        }
                        if (!ok)
                                return set_error(GZG_ERR_BAD_SCENE,
                                                 name + ": prim " + std::to_string(k) + " has a mesh or vertex index out of range");
                }
        }
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
                cudaGetLastError();
                return set_error(GZG_ERR_NO_DEVICE, "gzg_gpu_upload_scene: no CUDA device");
        }
        if (wide.nodes.size() >= (size_t)UINT32_MAX || wide.v0.size() >= (size_t)INT32_MAX)
                return set_error(GZG_ERR_LIMIT, "gzg_gpu_upload_scene: wide tree exceeds 32-bit indexing");

        // Triangles in prim-array order for the reference-order BVH2 kernel.
        std::vector<float4_> pv0((size_t)prim_count), pv1((size_t)prim_count), pv2((size_t)prim_count);
        for (int64_t k = 0; k < prim_count; ++k) {
                int64_t mesh, base;
                float4_ z{0, 0, 0, 0};
                pv0[k] = pv1[k] = pv2[k] = z;
                if (!prim_triangle(prim_ids[k], &mesh, &base)) continue;
                if (mesh < 0 || mesh >= mesh_count || base < 0 || base + 2 >= mesh_vertex_indices_counts[mesh]) {
                        // Prims outside any leaf are not validated by the tree walk; keep them inert.
                        continue;
                }
                const gzg_triangle_mesh &m = meshes[mesh];
                float4_ *dst[3] = {&pv0[k], &pv1[k], &pv2[k]};
                bool ok = true;
                for (int c = 0; c < 3; ++c) {
                        const int64_t v = m.vertex_indices[base + c];
                        if (v < 0 || v * 4 + 3 > mesh_points_counts[mesh]) {
                                ok = false;
                                break;
                        }
                        *dst[c] = float4_{m.points[v * 4], m.points[v * 4 + 1], m.points[v * 4 + 2], 0.0f};
                }
                if (!ok) {
                        pv0[k] = pv1[k] = pv2[k] = z;
                        continue;
                }
                int one = 1;
                std::memcpy(&pv0[k].w, &one, 4);
        }

        auto scene = std::make_unique<gzg_scene>();
        cudaGetDevice(&scene->device);
        DevScene &d = scene->dev;
        const float4 *f;
        if (!build) {
                const uint4 *wn;
                st = scene->upload(reinterpret_cast<const uint4 *>(wide.nodes.data()), wide.nodes.size() * 5, &wn,
                                   "wide nodes");
                if (st != GZG_OK) return st;
                d.wide = wn;
                st = scene->upload(reinterpret_cast<const float4 *>(wide.v0.data()), wide.v0.size(), &f, "triangles");
                if (st != GZG_OK) return st;
                d.tv0 = f;
                st = scene->upload(reinterpret_cast<const float4 *>(wide.v1.data()), wide.v1.size(), &f, "triangles");
                if (st != GZG_OK) return st;
                d.tv1 = f;
                st = scene->upload(reinterpret_cast<const float4 *>(wide.v2.data()), wide.v2.size(), &f, "triangles");
                if (st != GZG_OK) return st;
                d.tv2 = f;
                st = scene->upload(reinterpret_cast<const float4 *>(bvh2_nodes), (size_t)bvh2_node_count * 2, &f,
                                   "bvh2 nodes");
                if (st != GZG_OK) return st;
                d.bvh2 = f;
        }
        st = scene->upload(reinterpret_cast<const float4 *>(pv0.data()), pv0.size(), &f, "prim triangles");
        if (st != GZG_OK) return st;
        d.pv0 = f;
        st = scene->upload(reinterpret_cast<const float4 *>(pv1.data()), pv1.size(), &f, "prim triangles");
        if (st != GZG_OK) return st;
        d.pv1 = f;
        st = scene->upload(reinterpret_cast<const float4 *>(pv2.data()), pv2.size(), &f, "prim triangles");
        if (st != GZG_OK) return st;
        d.pv2 = f;
        const gzg_prim_id *pp;
        st = scene->upload(prim_ids, (size_t)prim_count, &pp, "prim ids");
        if (st != GZG_OK) return st;
        d.prims = pp;
        const uint32_t zero = 0;
        const uint32_t *ew;
        st = scene->upload(&zero, 1, &ew, "error word");
        if (st != GZG_OK) return st;
        d.err = const_cast<uint32_t *>(ew);
        if (build) {
                // the tree, built on the device from the prim-order triangles
                GpuWide gw;
                float ms = 0.0f;
                st = gpu_build_wide(reinterpret_cast<const float4_ *>(d.pv0), reinterpret_cast<const float4_ *>(d.pv1),
                                    reinterpret_cast<const float4_ *>(d.pv2), prim_count, build->leaf_size,
                                    build->builder, build->radius, &gw, &ms);
                for (void *p : {gw.nodes, gw.tv0, gw.tv1, gw.tv2})
                        if (p) scene->allocs.push_back(p);
                if (st != GZG_OK) return st;
                d.wide = reinterpret_cast<const uint4 *>(gw.nodes);
                d.tv0 = reinterpret_cast<const float4 *>(gw.tv0);
                d.tv1 = reinterpret_cast<const float4 *>(gw.tv1);
                d.tv2 = reinterpret_cast<const float4 *>(gw.tv2);
                scene->info.device_bytes += (int64_t)gw.node_count * (int64_t)sizeof(WideNode) + 48 * (int64_t)gw.tri_count;
                scene->build_ms = ms;
                // host copy (two-level and batch assembly read it)
                wide.nodes.resize(gw.node_count);
                wide.v0.resize(gw.tri_count);
                wide.v1.resize(gw.tri_count);
                wide.v2.resize(gw.tri_count);
                wide.depth = gw.depth;
                GZG_CK(cudaMemcpy(wide.nodes.data(), gw.nodes, gw.node_count * sizeof(WideNode), cudaMemcpyDeviceToHost),
                       "gzg_gpu_build_scene: tree download");
                GZG_CK(cudaMemcpy(wide.v0.data(), gw.tv0, gw.tri_count * sizeof(float4_), cudaMemcpyDeviceToHost),
                       "gzg_gpu_build_scene: tree download");
                GZG_CK(cudaMemcpy(wide.v1.data(), gw.tv1, gw.tri_count * sizeof(float4_), cudaMemcpyDeviceToHost),
                       "gzg_gpu_build_scene: tree download");
                GZG_CK(cudaMemcpy(wide.v2.data(), gw.tv2, gw.tri_count * sizeof(float4_), cudaMemcpyDeviceToHost),
                       "gzg_gpu_build_scene: tree download");
        }
        d.bvh2_count = build ? 0 : bvh2_node_count;
        d.prim_count = prim_count;
        d.wide_count = (uint32_t)wide.nodes.size();

        gzg_scene_info &info = scene->info;
        info.bvh2_nodes = build ? 0 : bvh2_node_count;
        info.prims = prim_count;
        info.triangles = (int64_t)wide.v0.size();
        info.wide_nodes = (int64_t)wide.nodes.size();
        info.wide_depth = wide.depth;
        info.bvh2_depth = bvh2_depth;

        // Device copies of the meshes, for calls that take reference
        // Intersection_C records and decode (mesh, triangle) from the prim id
        // the way shade_core does (kernel.mojo:705-721).
        std::vector<gzg_triangle_mesh> dev_meshes((size_t)mesh_count);
        std::vector<int64_t> sizes((size_t)mesh_count * 2);
        for (int64_t k = 0; k < mesh_count; ++k) {
                const float *pts = nullptr;
                const int64_t *vi = nullptr;
                st = scene->upload(meshes[k].points, (size_t)std::max<int64_t>(mesh_points_counts[k], 0), &pts,
                                   "mesh points");
                if (st != GZG_OK) return st;
                st = scene->upload(meshes[k].vertex_indices, (size_t)std::max<int64_t>(mesh_vertex_indices_counts[k], 0),
                                   &vi, "mesh vertex indices");
                if (st != GZG_OK) return st;
                dev_meshes[k] = gzg_triangle_mesh{pts, nullptr, vi};
                sizes[2 * k] = mesh_points_counts[k];
                sizes[2 * k + 1] = mesh_vertex_indices_counts[k];
        }
        const gzg_triangle_mesh *dm;
        st = scene->upload(dev_meshes.data(), dev_meshes.size(), &dm, "mesh table");
        if (st != GZG_OK) return st;
        d.meshes = dm;
        const int64_t *ms;
        st = scene->upload(sizes.data(), sizes.size(), &ms, "mesh sizes");
        if (st != GZG_OK) return st;
        d.mesh_sizes = ms;
        d.mesh_count = mesh_count;
        scene->mesh_vertices.resize((size_t)mesh_count);
        for (int64_t k = 0; k < mesh_count; ++k) scene->mesh_vertices[k] = mesh_points_counts[k] / 4;
        if (!build) {
                for (int a = 0; a < 3; ++a) {
                        scene->root_bounds[a] = bvh2_nodes[0].bounds_min[a];
                        scene->root_bounds[3 + a] = bvh2_nodes[0].bounds_max[a];
                }
        } else {
                float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
                for (int64_t k = 0; k < prim_count; ++k) {
                        int flag;
                        std::memcpy(&flag, &pv0[k].w, 4);
                        if (flag != 1) continue;
                        const float4_ *v[3] = {&pv0[k], &pv1[k], &pv2[k]};
                        for (int c = 0; c < 3; ++c) {
                                const float xyz[3] = {v[c]->x, v[c]->y, v[c]->z};
                                for (int a = 0; a < 3; ++a) {
                                        lo[a] = std::min(lo[a], xyz[a]);
                                        hi[a] = std::max(hi[a], xyz[a]);
                                }
                        }
                }
                for (int a = 0; a < 3; ++a) {
                        scene->root_bounds[a] = lo[a];
                        scene->root_bounds[3 + a] = hi[a];
                }
        }
        st = attach_shading(scene.get(), std::move(wide), prim_ids, prim_count, std::move(pv0), std::move(pv1),
                            std::move(pv2), materials, material_count);
        if (st != GZG_OK) return st;
        *out_scene = scene.release();
        return clear_error();
}

}  // namespace

GZG_API gzg_status gzg_gpu_upload_scene(const gzg_bvh2_node *bvh2_nodes, int64_t bvh2_node_count,
                                        const gzg_prim_id *prim_ids, int64_t prim_count,
                                        const gzg_triangle_mesh *meshes, int64_t mesh_count,
                                        const int64_t *mesh_points_counts, const int64_t *mesh_face_indices_counts,
                                        const int64_t *mesh_vertex_indices_counts, const gzg_material *materials,
                                        int64_t material_count, gzg_scene **out_scene) {
        (void)mesh_face_indices_counts;
        return upload_scene(bvh2_nodes, bvh2_node_count, prim_ids, prim_count, meshes, mesh_count, mesh_points_counts,
                            mesh_vertex_indices_counts, materials, material_count, nullptr, out_scene,
                            "gzg_gpu_upload_scene");
}

GZG_API gzg_status gzg_gpu_build_scene(const gzg_prim_id *prim_ids, int64_t prim_count,
                                       const gzg_triangle_mesh *meshes, int64_t mesh_count,
                                       const int64_t *mesh_points_counts, const int64_t *mesh_face_indices_counts,
                                       const int64_t *mesh_vertex_indices_counts, const gzg_material *materials,
                                       int64_t material_count, const gzg_build_options *options,
                                       gzg_scene **out_scene) {
        (void)mesh_face_indices_counts;
        const gzg_build_options defaults{};
        return upload_scene(nullptr, 0, prim_ids, prim_count, meshes, mesh_count, mesh_points_counts,
                            mesh_vertex_indices_counts, materials, material_count, options ? options : &defaults,
                            out_scene, "gzg_gpu_build_scene");
}

GZG_API gzg_status gzg_gpu_build_mesh_scene(const gzg_mesh_arrays *meshes, int64_t mesh_count,
                                            const gzg_material *materials, int64_t material_count,
                                            const gzg_build_options *options, gzg_scene **out_scene) {
        const char *fn = "gzg_gpu_build_mesh_scene";
        if (!out_scene) return set_error(GZG_ERR_INVALID_ARGUMENT, std::string(fn) + ": out_scene is NULL");
        *out_scene = nullptr;
        if (mesh_count < 0 || (mesh_count > 0 && !meshes) || material_count < 0 || (material_count > 0 && !materials))
                return set_error(GZG_ERR_INVALID_ARGUMENT, std::string(fn) + ": bad arguments");
        const gzg_build_options defaults{};
        const gzg_build_options &opt = options ? *options : defaults;
        if (opt.leaf_size < 0 || opt.leaf_size > 4)
                return set_error(GZG_ERR_INVALID_ARGUMENT, std::string(fn) + ": leaf_size must be 0 (default 1) to 4");
        if (opt.builder < 0 || opt.builder > GZG_BUILD_PLOC || opt.radius < 0 || opt.radius > 64)
                return set_error(GZG_ERR_INVALID_ARGUMENT, std::string(fn) + ": unknown builder or radius outside 0..64");
        std::vector<MeshRange> ranges((size_t)mesh_count);
        int64_t nv = 0, nt = 0, lights = 0;
        for (int64_t k = 0; k < mesh_count; ++k) {
                const gzg_mesh_arrays &m = meshes[k];
                if (m.vertex_count < 0 || m.triangle_count < 0 || (m.vertex_count > 0 && !m.points) ||
                    (m.triangle_count > 0 && !m.indices) || m.material < 0 || m.material >= material_count)
                        return set_error(GZG_ERR_INVALID_ARGUMENT,
                                         std::string(fn) + ": bad arrays or material index for mesh " + std::to_string(k));
                const bool is_light = materials[m.material].type == 2;
                ranges[k] = MeshRange{nv, nt, m.vertex_count, m.triangle_count, m.material, is_light ? lights : -1};
                if (is_light) lights += m.triangle_count;
                nv += m.vertex_count;
                nt += m.triangle_count;
        }
        if (nt > INT32_MAX - 1 || nv > INT32_MAX) return set_error(GZG_ERR_LIMIT, std::string(fn) + ": more than 2^31 triangles or vertices");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
                cudaGetLastError();
                return set_error(GZG_ERR_NO_DEVICE, std::string(fn) + ": no CUDA device");
        }
        auto scene = std::make_unique<gzg_scene>();
        cudaGetDevice(&scene->device);
        DevScene &d = scene->dev;
        gzg_status st;
        // staging: the packed arrays as they are, then the device expansion
        float *p3 = nullptr;
        int32_t *i3 = nullptr;
        MeshRange *rd = nullptr;
        struct Tmp {
                std::vector<void *> v;
                ~Tmp() {
                        for (void *p : v) cudaFree(p);
                }
        } tmp;
        GZG_CK(cudaMalloc(reinterpret_cast<void **>(&p3), std::max<size_t>(12 * (size_t)nv, 16)), "gzg_gpu_build_mesh_scene: staging");
        tmp.v.push_back(p3);
        GZG_CK(cudaMalloc(reinterpret_cast<void **>(&i3), std::max<size_t>(12 * (size_t)nt, 16)), "gzg_gpu_build_mesh_scene: staging");
        tmp.v.push_back(i3);
        GZG_CK(cudaMalloc(reinterpret_cast<void **>(&rd), std::max<size_t>(sizeof(MeshRange) * ranges.size(), 16)),
               "gzg_gpu_build_mesh_scene: staging");
        tmp.v.push_back(rd);
        for (int64_t k = 0; k < mesh_count; ++k) {
                const gzg_mesh_arrays &m = meshes[k];
                if (m.vertex_count)
                        GZG_CK(cudaMemcpy(p3 + 3 * ranges[k].vert_off, m.points, 12 * (size_t)m.vertex_count, cudaMemcpyHostToDevice),
                               "gzg_gpu_build_mesh_scene: points");
                if (m.triangle_count)
                        GZG_CK(cudaMemcpy(i3 + 3 * ranges[k].tri_off, m.indices, 12 * (size_t)m.triangle_count,
                                          cudaMemcpyHostToDevice),
                               "gzg_gpu_build_mesh_scene: indices");
        }
        if (mesh_count)
                GZG_CK(cudaMemcpy(rd, ranges.data(), sizeof(MeshRange) * ranges.size(), cudaMemcpyHostToDevice),
                       "gzg_gpu_build_mesh_scene: mesh table");
        float *p4;
        int64_t *v64;
        gzg_prim_id *prims;
        float4_ *pv[3];
        if ((st = scene->alloc(&p4, 4 * (size_t)nv, "mesh points")) || (st = scene->alloc(&v64, 3 * (size_t)nt, "mesh vertex indices")) ||
            (st = scene->alloc(&prims, (size_t)nt, "prim ids")) || (st = scene->alloc(&pv[0], (size_t)nt, "prim triangles")) ||
            (st = scene->alloc(&pv[1], (size_t)nt, "prim triangles")) || (st = scene->alloc(&pv[2], (size_t)nt, "prim triangles")))
                return st;
        bool bad = false;
        if ((st = gpu_expand_meshes(p3, i3, rd, (int)mesh_count, nv, nt, p4, v64, prims, pv[0], pv[1], pv[2], &bad)))
                return st;
        if (bad) return set_error(GZG_ERR_BAD_SCENE, std::string(fn) + ": a triangle index is out of its mesh's vertices");
        d.pv0 = reinterpret_cast<const float4 *>(pv[0]);
        d.pv1 = reinterpret_cast<const float4 *>(pv[1]);
        d.pv2 = reinterpret_cast<const float4 *>(pv[2]);
        d.prims = prims;
        const uint32_t zero = 0;
        const uint32_t *ew;
        if ((st = scene->upload(&zero, 1, &ew, "error word"))) return st;
        d.err = const_cast<uint32_t *>(ew);
        GpuWide gw;
        float ms = 0.0f;
        st = gpu_build_wide(pv[0], pv[1], pv[2], nt, opt.leaf_size, opt.builder, opt.radius, &gw, &ms);
        for (void *p : {gw.nodes, gw.tv0, gw.tv1, gw.tv2})
                if (p) scene->allocs.push_back(p);
        if (st != GZG_OK) return st;
        d.wide = reinterpret_cast<const uint4 *>(gw.nodes);
        d.tv0 = reinterpret_cast<const float4 *>(gw.tv0);
        d.tv1 = reinterpret_cast<const float4 *>(gw.tv1);
        d.tv2 = reinterpret_cast<const float4 *>(gw.tv2);
        scene->info.device_bytes += (int64_t)gw.node_count * (int64_t)sizeof(WideNode) + 48 * (int64_t)gw.tri_count;
        scene->build_ms = ms;
        // host copies: the tree and the shading arrays (batches, two-level
        // scenes and the light list read them)
        WideBvh wide;
        wide.nodes.resize(gw.node_count);
        wide.v0.resize(gw.tri_count);
        wide.v1.resize(gw.tri_count);
        wide.v2.resize(gw.tri_count);
        wide.depth = gw.depth;
        std::vector<float4_> h0((size_t)nt), h1((size_t)nt), h2((size_t)nt);
        std::vector<gzg_prim_id> hp((size_t)nt);
        GZG_CK(cudaMemcpy(wide.nodes.data(), gw.nodes, gw.node_count * sizeof(WideNode), cudaMemcpyDeviceToHost), "tree download");
        GZG_CK(cudaMemcpy(wide.v0.data(), gw.tv0, gw.tri_count * sizeof(float4_), cudaMemcpyDeviceToHost), "tree download");
        GZG_CK(cudaMemcpy(wide.v1.data(), gw.tv1, gw.tri_count * sizeof(float4_), cudaMemcpyDeviceToHost), "tree download");
        GZG_CK(cudaMemcpy(wide.v2.data(), gw.tv2, gw.tri_count * sizeof(float4_), cudaMemcpyDeviceToHost), "tree download");
        GZG_CK(cudaMemcpy(h0.data(), pv[0], nt * sizeof(float4_), cudaMemcpyDeviceToHost), "shading download");
        GZG_CK(cudaMemcpy(h1.data(), pv[1], nt * sizeof(float4_), cudaMemcpyDeviceToHost), "shading download");
        GZG_CK(cudaMemcpy(h2.data(), pv[2], nt * sizeof(float4_), cudaMemcpyDeviceToHost), "shading download");
        GZG_CK(cudaMemcpy(hp.data(), prims, nt * sizeof(gzg_prim_id), cudaMemcpyDeviceToHost), "shading download");
        // the device mesh table (reference layout) over the expanded arrays
        std::vector<gzg_triangle_mesh> dev_meshes((size_t)mesh_count);
        std::vector<int64_t> sizes((size_t)mesh_count * 2);
        for (int64_t k = 0; k < mesh_count; ++k) {
                dev_meshes[k] = gzg_triangle_mesh{p4 + 4 * ranges[k].vert_off, nullptr, v64 + 3 * ranges[k].tri_off};
                sizes[2 * k] = 4 * ranges[k].vcount;
                sizes[2 * k + 1] = 3 * ranges[k].tcount;
        }
        const gzg_triangle_mesh *dm;
        if ((st = scene->upload(dev_meshes.data(), dev_meshes.size(), &dm, "mesh table"))) return st;
        d.meshes = dm;
        const int64_t *msz;
        if ((st = scene->upload(sizes.data(), sizes.size(), &msz, "mesh sizes"))) return st;
        d.mesh_sizes = msz;
        d.mesh_count = mesh_count;
        scene->mesh_vertices.resize((size_t)mesh_count);
        for (int64_t k = 0; k < mesh_count; ++k) scene->mesh_vertices[k] = ranges[k].vcount;
        d.bvh2_count = 0;
        d.prim_count = nt;
        d.wide_count = (uint32_t)wide.nodes.size();
        gzg_scene_info &info = scene->info;
        info.bvh2_nodes = 0;
        info.prims = nt;
        info.triangles = (int64_t)wide.v0.size();
        info.wide_nodes = (int64_t)wide.nodes.size();
        info.wide_depth = wide.depth;
        info.bvh2_depth = 0;
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (const std::vector<float4_> *v : {&h0, &h1, &h2})
                for (const float4_ &q : *v) {
                        lo[0] = std::min(lo[0], q.x);
                        lo[1] = std::min(lo[1], q.y);
                        lo[2] = std::min(lo[2], q.z);
                        hi[0] = std::max(hi[0], q.x);
                        hi[1] = std::max(hi[1], q.y);
                        hi[2] = std::max(hi[2], q.z);
                }
        for (int a = 0; a < 3; ++a) {
                scene->root_bounds[a] = lo[a];
                scene->root_bounds[3 + a] = hi[a];
        }
        st = attach_shading(scene.get(), std::move(wide), hp.data(), nt, std::move(h0), std::move(h1), std::move(h2),
                            materials, material_count);
        if (st != GZG_OK) return st;
        *out_scene = scene.release();
        return clear_error();
}

// Vertex normals and UVs of one mesh of a flat scene (the data
// Triangle.computeSurfaceInteraction reads from TriangleMesh, Shape/
// Triangle.swift:386-452); gathered per prim on the device.
GZG_API gzg_status gzg_scene_set_vertex_attributes(gzg_scene *scene, int64_t mesh, const float *normals,
                                                   const float *uvs, int64_t vertex_count) {
        const char *fn = "gzg_scene_set_vertex_attributes";
        if (!scene || (!normals && !uvs)) return set_error(GZG_ERR_INVALID_ARGUMENT, std::string(fn) + ": bad arguments");
        if (scene->instanced)
                return set_error(GZG_ERR_INVALID_ARGUMENT, std::string(fn) + ": set them on the bottom-level scenes");
        if (mesh < 0 || mesh >= (int64_t)scene->mesh_vertices.size() || vertex_count != scene->mesh_vertices[mesh])
                return set_error(GZG_ERR_INVALID_ARGUMENT,
                                 std::string(fn) + ": mesh index out of range or vertex count differs from the mesh's");
        for (int64_t i = 0; normals && i < 3 * vertex_count; ++i)
                if (!std::isfinite(normals[i]))
                        return set_error(GZG_ERR_INVALID_ARGUMENT, std::string(fn) + ": normals must be finite");
        for (int64_t i = 0; uvs && i < 2 * vertex_count; ++i)
                if (!std::isfinite(uvs[i])) return set_error(GZG_ERR_INVALID_ARGUMENT, std::string(fn) + ": UVs must be finite");
        DeviceGuard g(scene->device);
        DevScene &d = scene->dev;
        HostShading &hs = scene->host_shading;
        const int64_t n = d.prim_count;
        gzg_status st;
        if (!d.attr) {
                float4 *a;
                if ((st = scene->alloc(&a, 5 * (size_t)std::max<int64_t>(n, 1), "vertex attributes"))) return st;
                GZG_CK(cudaMemset(a, 0, 5 * sizeof(float4) * (size_t)std::max<int64_t>(n, 1)), "vertex attributes");
                d.attr = a;
        }
        struct Tmp {
                void *p = nullptr;
                ~Tmp() {
                        if (p) cudaFree(p);
                }
        } tn, tu;
        if (normals) {
                GZG_CK(cudaMalloc(&tn.p, 12 * (size_t)std::max<int64_t>(vertex_count, 1)), "vertex normals");
                GZG_CK(cudaMemcpy(tn.p, normals, 12 * (size_t)vertex_count, cudaMemcpyHostToDevice), "vertex normals");
        }
        if (uvs) {
                GZG_CK(cudaMalloc(&tu.p, 8 * (size_t)std::max<int64_t>(vertex_count, 1)), "vertex UVs");
                GZG_CK(cudaMemcpy(tu.p, uvs, 8 * (size_t)vertex_count, cudaMemcpyHostToDevice), "vertex UVs");
        }
        if ((st = gpu_gather_attributes(d.prims, n, d.meshes, mesh, static_cast<const float *>(tn.p),
                                        static_cast<const float *>(tu.p), vertex_count,
                                        reinterpret_cast<float4_ *>(const_cast<float4 *>(d.attr)))))
                return st;
        hs.attr.resize(5 * (size_t)n);
        if (n)
                GZG_CK(cudaMemcpy(hs.attr.data(), d.attr, 5 * sizeof(float4) * (size_t)n, cudaMemcpyDeviceToHost),
                       "vertex attributes");
        return clear_error();
}

GZG_API gzg_status gzg_scene_build_time(const gzg_scene *scene, float *device_ms) {
        if (!scene || !device_ms) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_scene_build_time: null argument");
        *device_ms = scene->build_ms;
        return clear_error();
}

// Surface-area cost of the wide tree (quantised boxes, relative to the
// root's box): interior children cost 1 per unit area, leaf triangles 1 each.
GZG_API gzg_status gzg_scene_tree_cost(const gzg_scene *scene, double *cost) {
        if (!scene || !cost) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_scene_tree_cost: null argument");
        const WideBvh &w = scene->host_wide;
        double root_area = 0.0, sum = 0.0;
        for (size_t i = 0; i < w.nodes.size(); ++i) {
                const WideNode &nd = w.nodes[i];
                const float p[3] = {nd.px, nd.py, nd.pz};
                const int e[3] = {nd.ex, nd.ey, nd.ez};
                double nlo[3] = {INFINITY, INFINITY, INFINITY}, nhi[3] = {-INFINITY, -INFINITY, -INFINITY};
                for (int s = 0; s < 8; ++s) {
                        const bool interior = (nd.imask >> s) & 1u, leaf = (nd.meta[s] & 0x80u) != 0;
                        if (!interior && !leaf) continue;
                        double lo[3], hi[3];
                        for (int a = 0; a < 3; ++a) {
                                const double step = std::ldexp(1.0, e[a] - 127);
                                lo[a] = p[a] + step * nd.qlo[a][s];
                                hi[a] = p[a] + step * nd.qhi[a][s];
                                nlo[a] = std::min(nlo[a], lo[a]);
                                nhi[a] = std::max(nhi[a], hi[a]);
                        }
                        const double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
                        const double area = 2.0 * (dx * dy + dx * dz + dy * dz);
                        sum += interior ? area : area * (double)(((nd.meta[s] >> 5) & 3u) + 1u);
                }
                if (i == 0) {
                        const double dx = nhi[0] - nlo[0], dy = nhi[1] - nlo[1], dz = nhi[2] - nlo[2];
                        root_area = 2.0 * (dx * dy + dx * dz + dy * dz);
                }
        }
        *cost = root_area > 0.0 ? 1.0 + sum / root_area : 0.0;
        return clear_error();
}

GZG_API gzg_status gzg_gpu_free_scene(gzg_scene *scene) {
        delete scene;
        return clear_error();
}

GZG_API gzg_status gzg_gpu_traverse_batch(gzg_scene *scene, const gzg_ray *rays, const float *t_max_values,
                                          int64_t count, gzg_intersection *results, const gzg_trace_options *options) {
        return host_batch(scene, rays, t_max_values, count, results, sizeof(gzg_intersection), kOutIntersection, options);
}

GZG_API gzg_status gzg_gpu_traverse_batch_hits(gzg_scene *scene, const gzg_ray *rays, const float *t_max_values,
                                               int64_t count, gzg_hit_d *hits, const gzg_trace_options *options) {
        return host_batch(scene, rays, t_max_values, count, hits, sizeof(gzg_hit_d), kOutHit, options);
}

GZG_API gzg_status gzg_gpu_occluded_batch(gzg_scene *scene, const gzg_ray *rays, const float *t_max_values,
                                          int64_t count, uint8_t *occluded, const gzg_trace_options *options) {
        return host_batch(scene, rays, t_max_values, count, occluded, 1, kOutOccluded, options);
}

GZG_API gzg_status gzg_trace_closest_device(gzg_scene *scene, const gzg_ray_d *rays, int64_t count, gzg_hit_d *hits,
                                            const gzg_trace_options *options, void *stream) {
        if (!scene || count < 0 || (count > 0 && (!rays || !hits)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_trace_closest_device: bad arguments");
        gzg_status st = check_options(options);
        if (st != GZG_OK) return st;
        DeviceGuard g(scene->device);
        GZG_CK(device_trace(scene, params_for(scene, options, false), kOutHit, rays, count, hits,
                            reinterpret_cast<cudaStream_t>(stream)),
               "gzg_trace_closest_device launch");
        return clear_error();
}

// Coordinate descent over the launch configuration of the persistent wide
// kernel on the caller's rays: L1 carveout, then blocks per SM, then block
// size, then stack depth; each candidate timed over three launches after one
// warm-up with CUDA events on `stream`.  The winner becomes the scene's
// default for that query kind.
GZG_API gzg_status gzg_scene_autotune(gzg_scene *scene, const gzg_ray_d *rays, int64_t count, int32_t any_hit,
                                      gzg_trace_options *best, float *best_ms, void *stream) {
        if (!scene || !rays || count <= 0)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_scene_autotune: bad arguments");
        DeviceGuard g(scene->device);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        void *out = nullptr;
        GZG_CK(cudaMalloc(&out, (size_t)count * 16), "gzg_scene_autotune output buffer");
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        gzg_status status = GZG_OK;
        auto time_config = [&](const TunedLaunch &t, float *ms) -> gzg_status {
                LaunchParams p = params_for(scene, nullptr, any_hit != 0);
                p.block_size = t.block_size;
                p.blocks_per_sm = t.blocks_per_sm;
                p.stack_depth = t.stack_depth;
                p.l1_carveout = t.l1_carveout;
                const int fmt = any_hit ? kOutAnyPrim : kOutHit;
                GZG_CK(device_trace(scene, p, fmt, rays, count, out, st), "autotune launch");
                // the faster of two timed batches of three launches (a single
                // batch let one noisy sample pick a slow configuration)
                float best_el = 0.0f;
                for (int rep = 0; rep < 2; ++rep) {
                        GZG_CK(cudaEventRecord(e0, st), "autotune event");
                        for (int k = 0; k < 3; ++k)
                                GZG_CK(device_trace(scene, p, fmt, rays, count, out, st),
                                       "autotune launch");
                        GZG_CK(cudaEventRecord(e1, st), "autotune event");
                        GZG_CK(cudaEventSynchronize(e1), "autotune sync");
                        float el = 0;
                        cudaEventElapsedTime(&el, e0, e1);
                        if (rep == 0 || el < best_el) best_el = el;
                }
                *ms = best_el / 3.0f;
                return GZG_OK;
        };
        TunedLaunch cur;
        float cur_ms = 0;
        status = time_config(cur, &cur_ms);
        auto try_set = [&](TunedLaunch cand) {
                if (status) return;
                float ms = 0;
                status = time_config(cand, &ms);
                if (!status && ms < cur_ms) {
                        cur = cand;
                        cur_ms = ms;
                }
        };
        // Joint grid over the coupled knobs (shared stack size, resident
        // blocks, L1/shared split), then block size around the winner.
        const int stacks[] = {0, 16};
        const int bps[] = {0, 4, 5, 6, 7, 8};
        const int carves[] = {-1, 25, 50};
        for (int sd : stacks)
                for (int b : bps)
                        for (int c : carves) {
                                TunedLaunch t;
                                t.stack_depth = sd;
                                t.blocks_per_sm = b;
                                t.l1_carveout = c;
                                try_set(t);
                        }
        const int blocks[] = {64, 256};
        const TunedLaunch base = cur;
        for (int bs : blocks) {
                TunedLaunch t = base;
                t.block_size = bs;
                t.blocks_per_sm = base.blocks_per_sm ? std::max(1, base.blocks_per_sm * 128 / bs) : 0;
                try_set(t);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(out);
        if (status) return status;
        (any_hit ? scene->tuned_any : scene->tuned_closest) = cur;
        if (best) {
                std::memset(best, 0, sizeof(*best));
                best->traversal = GZG_TRAVERSAL_WIDE;
                best->leaf_test = GZG_LEAF_MOLLER_TRUMBORE;
                best->block_size = cur.block_size;
                best->blocks_per_sm = cur.blocks_per_sm;
                best->stack_depth = cur.stack_depth;
                best->l1_carveout = cur.l1_carveout;
        }
        if (best_ms) *best_ms = cur_ms;
        return clear_error();
}

// transform * bound (Geometry/Bounds3.swift:61-69): the eight corners in the
// order of Bounds3.points (:31-42) through Transform*Point, the first two
// through Bounds3(first:second:), the rest through add(point:).
static void instance_world_bounds(const float *lo_hi, const float *m, float *out6) {
        float c[8][3];
        for (int i = 0; i < 8; ++i) {
                const float x = (i & 4) ? lo_hi[3] : lo_hi[0];
                const float y = (i & 2) ? lo_hi[4] : lo_hi[1];
                const float z = (i & 1) ? lo_hi[5] : lo_hi[2];
                for (int r = 0; r < 3; ++r) {
                        const float *row = m + 4 * r;
                        float v = row[0] * x;
                        v = v + row[1] * y;
                        v = v + row[2] * z;
                        c[i][r] = v + row[3];
                }
        }
        float lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
                lo[a] = c[1][a] < c[0][a] ? c[1][a] : c[0][a];
                hi[a] = c[1][a] >= c[0][a] ? c[1][a] : c[0][a];
        }
        for (int i = 2; i < 8; ++i)
                for (int a = 0; a < 3; ++a) {
                        if (c[i][a] < lo[a]) lo[a] = c[i][a];
                        if (c[i][a] > hi[a]) hi[a] = c[i][a];
                }
        std::memcpy(out6, lo, 12);
        std::memcpy(out6 + 3, hi, 12);
}

// World bounds of an instance from its bottom-level wide tree: the boxes of
// the root's children and, for interior children, of their children (up to
// 64 boxes, decoded in double precision and rounded outward), each carried to
// world space by its 8 corners, then united.  They contain the instance's
// geometry as the root box's transformed corners do (the reference's
// TransformedPrimitive.worldBound), but hug rotated shapes far more closely,
// so rays enter fewer instances.
static void instance_world_bounds_tree(const WideBvh &w, const float *root6, const float *m, float *out6) {
        std::vector<std::array<double, 6>> boxes;
        auto child_box = [](const WideNode &n, int s) {
                std::array<double, 6> b;
                const double p[3] = {n.px, n.py, n.pz};
                const int e[3] = {n.ex, n.ey, n.ez};
                for (int a = 0; a < 3; ++a) {
                        const double step = std::ldexp(1.0, e[a] - 127);
                        b[a] = p[a] + n.qlo[a][s] * step;
                        b[3 + a] = p[a] + n.qhi[a][s] * step;
                }
                return b;
        };
        auto used = [](const WideNode &n, int s) { return ((n.imask >> s) & 1u) || (n.meta[s] & 0x80u); };
        if (!w.nodes.empty()) {
                const WideNode &root = w.nodes[0];
                for (int s = 0; s < 8; ++s) {
                        if (!used(root, s)) continue;
                        if ((root.imask >> s) & 1u) {
                                const uint32_t ci = root.child_base + (uint32_t)__builtin_popcount(root.imask & ((1u << s) - 1u));
                                if (ci < w.nodes.size()) {
                                        const WideNode &c = w.nodes[ci];
                                        bool any = false;
                                        for (int t = 0; t < 8; ++t)
                                                if (used(c, t)) {
                                                        boxes.push_back(child_box(c, t));
                                                        any = true;
                                                }
                                        if (any) continue;
                                }
                        }
                        boxes.push_back(child_box(root, s));
                }
        }
        if (boxes.empty()) {
                instance_world_bounds(root6, m, out6);
                return;
        }
        double lo[3] = {HUGE_VAL, HUGE_VAL, HUGE_VAL}, hi[3] = {-HUGE_VAL, -HUGE_VAL, -HUGE_VAL};
        for (const auto &b : boxes)
                for (int i = 0; i < 8; ++i) {
                        const double x = (i & 4) ? b[3] : b[0], y = (i & 2) ? b[4] : b[1], z = (i & 1) ? b[5] : b[2];
                        for (int r = 0; r < 3; ++r) {
                                const float *row = m + 4 * r;
                                const double v = (double)row[0] * x + (double)row[1] * y + (double)row[2] * z + (double)row[3];
                                lo[r] = std::min(lo[r], v);
                                hi[r] = std::max(hi[r], v);
                        }
                }
        for (int a = 0; a < 3; ++a) {
                // outward to float, with a relative margin for the float
                // transform the traversal applies to rays
                const double mg = std::ldexp(std::max(std::fabs(lo[a]), std::fabs(hi[a])), -20);
                out6[a] = std::nextafter((float)(lo[a] - mg), -HUGE_VALF);
                out6[3 + a] = std::nextafter((float)(hi[a] + mg), HUGE_VALF);
        }
}

GZG_API gzg_status gzg_host_instance_bounds_from_scenes(gzg_scene *const *blas, int64_t blas_count,
                                                        const gzg_instance *inst, int64_t instance_count,
                                                        float *bounds6) {
        if (blas_count <= 0 || !blas || instance_count < 0 || (instance_count > 0 && (!inst || !bounds6)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_host_instance_bounds_from_scenes: bad arguments");
        for (int64_t b = 0; b < blas_count; ++b)
                if (!blas[b] || blas[b]->instanced)
                        return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_host_instance_bounds_from_scenes: bottom-level scene " +
                                                                       std::to_string(b) + " is NULL or two-level");
        for (int64_t k = 0; k < instance_count; ++k) {
                if (inst[k].blas < 0 || inst[k].blas >= blas_count)
                        return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_host_instance_bounds_from_scenes: instance " +
                                                                       std::to_string(k) + " references a missing bottom-level scene");
                const gzg_scene *s = blas[inst[k].blas];
                instance_world_bounds_tree(s->host_wide, s->root_bounds, inst[k].object_to_world, bounds6 + 6 * k);
        }
        return clear_error();
}

GZG_API gzg_status gzg_host_instance_bounds(const float *blas_bounds6, int64_t blas_count, const gzg_instance *inst,
                                            int64_t instance_count, float *bounds6) {
        if (blas_count < 0 || instance_count < 0 || (instance_count > 0 && (!blas_bounds6 || !inst || !bounds6)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_host_instance_bounds: bad arguments");
        for (int64_t k = 0; k < instance_count; ++k) {
                if (inst[k].blas < 0 || inst[k].blas >= blas_count)
                        return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_host_instance_bounds: instance " + std::to_string(k) +
                                                                       " references a missing bottom-level scene");
                instance_world_bounds(blas_bounds6 + 6 * inst[k].blas, inst[k].object_to_world, bounds6 + 6 * k);
        }
        return clear_error();
}

GZG_API gzg_status gzg_instanced_scene_create(gzg_scene *const *blas, int64_t blas_count, const gzg_instance *inst,
                                              int64_t instance_count, const gzg_bvh2_node *tlas_nodes,
                                              int64_t tlas_node_count, const int64_t *tlas_leaf_instance,
                                              int64_t tlas_leaf_count, gzg_scene **out_scene) {
        if (!out_scene) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_instanced_scene_create: out_scene is NULL");
        *out_scene = nullptr;
        if (blas_count <= 0 || !blas || instance_count <= 0 || !inst || tlas_node_count <= 0 || !tlas_nodes ||
            tlas_leaf_count < 0 || (tlas_leaf_count > 0 && !tlas_leaf_instance))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_instanced_scene_create: bad arguments");
        int device = -1;
        std::vector<float> blas_bounds((size_t)blas_count * 6);
        for (int64_t b = 0; b < blas_count; ++b) {
                if (!blas[b] || blas[b]->instanced)
                        return set_error(GZG_ERR_INVALID_ARGUMENT,
                                         "gzg_instanced_scene_create: bottom-level scene " + std::to_string(b) + " is NULL or two-level");
                if (device >= 0 && blas[b]->device != device)
                        return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_instanced_scene_create: scenes on different devices");
                device = blas[b]->device;
                std::memcpy(&blas_bounds[6 * b], blas[b]->root_bounds, 24);
        }
        std::vector<float> ib((size_t)instance_count * 6);
        gzg_status st = gzg_host_instance_bounds_from_scenes(blas, blas_count, inst, instance_count, ib.data());
        if (st) return st;
        WideBvh tlas;
        int32_t tlas_bvh2_depth = 0;
        st = build_wide_tlas(tlas_nodes, tlas_node_count, tlas_leaf_instance, tlas_leaf_count, ib.data(), instance_count,
                             &tlas, &tlas_bvh2_depth);
        if (st) return st;

        // One node array and one leaf-record array: top level first, then each
        // bottom-level tree with its child and leaf bases moved by its offsets.
        std::vector<WideNode> nodes = tlas.nodes;
        std::vector<float4_> v0 = tlas.v0, v1 = tlas.v1, v2 = tlas.v2;
        std::vector<uint32_t> root(blas_count);
        int32_t max_blas_depth = 0;
        for (int64_t b = 0; b < blas_count; ++b) {
                const WideBvh &w = blas[b]->host_wide;
                const uint32_t noff = (uint32_t)nodes.size(), toff = (uint32_t)v0.size();
                root[b] = noff;
                for (WideNode n : w.nodes) {
                        n.child_base += noff;
                        n.tri_base += toff;
                        nodes.push_back(n);
                }
                v0.insert(v0.end(), w.v0.begin(), w.v0.end());
                v1.insert(v1.end(), w.v1.begin(), w.v1.end());
                v2.insert(v2.end(), w.v2.begin(), w.v2.end());
                max_blas_depth = std::max(max_blas_depth, w.depth);
        }
        if (nodes.size() >= 0x7FFFFFFFu || v0.size() >= 0x7FFFFFFFu)
                return set_error(GZG_ERR_LIMIT, "gzg_instanced_scene_create: more than 2^31 nodes or leaf records");
        std::vector<float4_> table((size_t)instance_count * 4);
        uint64_t steps = tlas.nodes.size();
        for (int64_t k = 0; k < instance_count; ++k) {
                const float *m = inst[k].world_to_object;
                for (int r = 0; r < 3; ++r) table[4 * k + r] = float4_{m[4 * r], m[4 * r + 1], m[4 * r + 2], m[4 * r + 3]};
                float rf, bf;
                const int32_t rb = (int32_t)root[inst[k].blas], bb = inst[k].blas;
                std::memcpy(&rf, &rb, 4);
                std::memcpy(&bf, &bb, 4);
                table[4 * k + 3] = float4_{rf, bf, 0.0f, 0.0f};
                steps += blas[inst[k].blas]->host_wide.nodes.size();
        }

        // Shading arrays: the bottom-level scenes' prim-order triangles, prims
        // (material indices moved by each scene's material offset) and
        // materials, concatenated; per instance object_to_world rows.
        HostShading hsd;
        std::vector<int32_t> prim_base(blas_count);
        for (int64_t b = 0; b < blas_count; ++b) {
                const HostShading &bs = blas[b]->host_shading;
                prim_base[b] = (int32_t)hsd.prims.size();
                const int64_t moff = (int64_t)(hsd.materials.size() / 2);
                hsd.pv0.insert(hsd.pv0.end(), bs.pv0.begin(), bs.pv0.end());
                hsd.pv1.insert(hsd.pv1.end(), bs.pv1.begin(), bs.pv1.end());
                hsd.pv2.insert(hsd.pv2.end(), bs.pv2.begin(), bs.pv2.end());
                for (gzg_prim_id p : bs.prims) {
                        p.material_index += moff;
                        hsd.prims.push_back(p);
                }
                hsd.materials.insert(hsd.materials.end(), bs.materials.begin(), bs.materials.end());
        }
        bool any_attr = false;
        for (int64_t b = 0; b < blas_count; ++b) any_attr = any_attr || !blas[b]->host_shading.attr.empty();
        if (any_attr) {
                for (int64_t b = 0; b < blas_count; ++b) {
                        const HostShading &bs = blas[b]->host_shading;
                        if (bs.attr.empty())
                                hsd.attr.insert(hsd.attr.end(), 5 * bs.prims.size(), float4_{0, 0, 0, 0});
                        else
                                hsd.attr.insert(hsd.attr.end(), bs.attr.begin(), bs.attr.end());
                }
        }
        bool any_params = false;
        for (int64_t b = 0; b < blas_count; ++b) any_params = any_params || !blas[b]->host_shading.mat_params.empty();
        if (any_params) {
                for (int64_t b = 0; b < blas_count; ++b) {
                        const HostShading &bs = blas[b]->host_shading;
                        if (bs.mat_params.empty())
                                hsd.mat_params.insert(hsd.mat_params.end(), 3 * (bs.materials.size() / 2),
                                                      float4_{1, 0, 0, 0});
                        else
                                hsd.mat_params.insert(hsd.mat_params.end(), bs.mat_params.begin(), bs.mat_params.end());
                }
        }
        if (hsd.prims.size() >= 0x7FFFFFFFu)
                return set_error(GZG_ERR_LIMIT, "gzg_instanced_scene_create: more than 2^31 bottom-level prims");
        std::vector<float4_> o2w((size_t)instance_count * 3);
        for (int64_t k = 0; k < instance_count; ++k) {
                const float *m = inst[k].object_to_world;
                for (int r = 0; r < 3; ++r) o2w[3 * k + r] = float4_{m[4 * r], m[4 * r + 1], m[4 * r + 2], m[4 * r + 3]};
        }

        auto scene = std::make_unique<gzg_scene>();
        scene->device = device;
        scene->instanced = true;
        DeviceGuard g(device);
        DevScene &d = scene->dev;
        const uint4 *wn;
        st = scene->upload(reinterpret_cast<const uint4 *>(nodes.data()), nodes.size() * 5, &wn, "wide nodes");
        if (st) return st;
        d.wide = wn;
        const float4 *f;
        if ((st = scene->upload(reinterpret_cast<const float4 *>(v0.data()), v0.size(), &f, "leaf records"))) return st;
        d.tv0 = f;
        if ((st = scene->upload(reinterpret_cast<const float4 *>(v1.data()), v1.size(), &f, "leaf records"))) return st;
        d.tv1 = f;
        if ((st = scene->upload(reinterpret_cast<const float4 *>(v2.data()), v2.size(), &f, "leaf records"))) return st;
        d.tv2 = f;
        if ((st = scene->upload(reinterpret_cast<const float4 *>(table.data()), table.size(), &f, "instance table")))
                return st;
        d.instances = f;
        d.instance_count = instance_count;
        if ((st = scene->upload(reinterpret_cast<const float4 *>(o2w.data()), o2w.size(), &f, "instance transforms")))
                return st;
        d.inst_o2w = f;
        if (!hsd.prims.empty()) {
                if ((st = scene->upload(reinterpret_cast<const float4 *>(hsd.pv0.data()), hsd.pv0.size(), &f, "triangles")))
                        return st;
                d.pv0 = f;
                if ((st = scene->upload(reinterpret_cast<const float4 *>(hsd.pv1.data()), hsd.pv1.size(), &f, "triangles")))
                        return st;
                d.pv1 = f;
                if ((st = scene->upload(reinterpret_cast<const float4 *>(hsd.pv2.data()), hsd.pv2.size(), &f, "triangles")))
                        return st;
                d.pv2 = f;
                const gzg_prim_id *pd;
                if ((st = scene->upload(hsd.prims.data(), hsd.prims.size(), &pd, "prim ids"))) return st;
                d.prims = pd;
                d.prim_count = (int64_t)hsd.prims.size();
        }
        if (!hsd.materials.empty()) {
                if ((st = scene->upload(reinterpret_cast<const float4 *>(hsd.materials.data()), hsd.materials.size(), &f,
                                        "materials")))
                        return st;
                d.materials = f;
                d.material_count = (int32_t)(hsd.materials.size() / 2);
        }
        if (!hsd.mat_params.empty()) {
                if ((st = scene->upload(reinterpret_cast<const float4 *>(hsd.mat_params.data()), hsd.mat_params.size(),
                                        &f, "material parameters")))
                        return st;
                d.mat_params = f;
        }
        if (!hsd.attr.empty()) {
                if ((st = scene->upload(reinterpret_cast<const float4 *>(hsd.attr.data()), hsd.attr.size(), &f,
                                        "vertex attributes")))
                        return st;
                d.attr = f;
        }
        const int32_t *pb;
        if ((st = scene->upload(prim_base.data(), prim_base.size(), &pb, "prim bases"))) return st;
        d.blas_prim_base = pb;
        scene->host_shading = std::move(hsd);
        const uint32_t zero = 0;
        const uint32_t *ew;
        if ((st = scene->upload(&zero, 1, &ew, "error word"))) return st;
        d.err = const_cast<uint32_t *>(ew);
        d.wide_count = (uint32_t)std::min<uint64_t>(steps, 0xFFFFFFFFull);
        scene->info.wide_nodes = (int64_t)nodes.size();
        scene->info.triangles = (int64_t)(v0.size() - tlas.v0.size());
        scene->info.prims = instance_count;
        scene->info.bvh2_nodes = tlas_node_count;
        scene->info.bvh2_depth = tlas_bvh2_depth;
        scene->info.wide_depth = tlas.depth + max_blas_depth + 2;
        *out_scene = scene.release();
        return clear_error();
}

// Parameters of the general materials (types 3 to 6), one gzg_material_params
// record per material, kept on the device as 3 float4 (Material/
// Dielectric.swift:3-14, Material/CoatedDiffuse.swift:23-58,
// Material/Conductor.swift:3-22, Material/CoatedConductor.swift:35-88; the
// remapping of roughness to alpha happens when shading).  Once per flat
// scene, before it enters a two-level scene or a batch.
GZG_API gzg_status gzg_scene_set_material_params(gzg_scene *scene, const gzg_material_params *params,
                                                 int64_t count) {
        if (!scene || !params || count <= 0)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_scene_set_material_params: bad arguments");
        if (scene->instanced)
                return set_error(GZG_ERR_INVALID_ARGUMENT,
                                 "gzg_scene_set_material_params: set them on the bottom-level scenes");
        HostShading &hs = scene->host_shading;
        if (!hs.mat_params.empty())
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_scene_set_material_params: already set");
        if ((size_t)count != hs.materials.size() / 2)
                return set_error(GZG_ERR_INVALID_ARGUMENT,
                                 "gzg_scene_set_material_params: count differs from the scene's material count");
        static_assert(sizeof(gzg_material_params) == 48, "gzg_material_params is 3 x float4");
        auto fin = [](float x) { return std::isfinite(x) && x >= 0.0f; };
        std::vector<float4_> mp((size_t)count * 3);
        for (int64_t k = 0; k < count; ++k) {
                const gzg_material_params &q = params[k];
                const int type = (int)hs.materials[2 * k].w;
                bool ok = true;
                if (type == 3 || type == 4 || type == 6)
                        ok = ok && fin(q.eta) && q.eta > 0.0f && fin(q.roughness_u) && fin(q.roughness_v) &&
                             fin(q.thickness);
                if (type == 5 || type == 6)
                        for (int c = 0; c < 3; ++c)
                                ok = ok && fin(q.conductor_eta[c]) && fin(q.conductor_k[c]) &&
                                     fin(q.conductor_roughness_u) && fin(q.conductor_roughness_v);
                if (!ok)
                        return set_error(GZG_ERR_INVALID_ARGUMENT,
                                         "gzg_scene_set_material_params: eta must be > 0; roughness, thickness and "
                                         "conductor eta / k finite and >= 0");
                mp[3 * k] = float4_{q.eta, q.roughness_u, q.roughness_v, q.thickness};
                mp[3 * k + 1] = float4_{q.conductor_eta[0], q.conductor_eta[1], q.conductor_eta[2],
                                        q.conductor_roughness_u};
                mp[3 * k + 2] = float4_{q.conductor_k[0], q.conductor_k[1], q.conductor_k[2], q.conductor_roughness_v};
        }
        DeviceGuard g(scene->device);
        const float4 *f;
        gzg_status st;
        if ((st = scene->upload(reinterpret_cast<const float4 *>(mp.data()), mp.size(), &f, "material parameters")))
                return st;
        scene->dev.mat_params = f;
        hs.mat_params = std::move(mp);
        return clear_error();
}

// Environment light: the map, its sampling distribution (built on the host,
// env.cpp) and its place after the area lights in the light list: the
// running power sum gains one entry (Light/PowerLightSampler.swift) and the
// total the light's power pi * 50^2 * average(scale)
// (Light/InfiniteLight.swift:141-144).
GZG_API gzg_status gzg_scene_set_medium(gzg_scene *scene, const gzg_medium *medium) {
        if (!scene) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_scene_set_medium: null scene");
        if (!medium) {
                scene->host_shading.has_medium = false;
                return clear_error();
        }
        bool ok = std::isfinite(medium->g) && std::fabs(medium->g) < 1.0f && medium->reserved == 0;
        for (int a = 0; a < 3; ++a) {
                ok = ok && std::isfinite(medium->box_min[a]) && std::isfinite(medium->box_max[a]) &&
                     medium->box_min[a] < medium->box_max[a];
                ok = ok && std::isfinite(medium->sigma_a[a]) && medium->sigma_a[a] >= 0.0f &&
                     std::isfinite(medium->sigma_s[a]) && medium->sigma_s[a] >= 0.0f;
        }
        if (!ok)
                return set_error(GZG_ERR_INVALID_ARGUMENT,
                                 "gzg_scene_set_medium: empty box, negative or non-finite coefficient, or |g| >= 1");
        scene->host_shading.medium = *medium;
        scene->host_shading.has_medium = true;
        return clear_error();
}

GZG_API gzg_status gzg_scene_set_environment(gzg_scene *scene, const float *rgb, int32_t width, int32_t height,
                                             float scale) {
        if (!scene || !rgb || width <= 0 || height <= 0 || (int64_t)width * height > ((int64_t)1 << 28) ||
            !std::isfinite(scale) || scale < 0.0f)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_scene_set_environment: bad arguments");
        if (scene->host_shading.has_env)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_scene_set_environment: the scene has an environment");
        EnvTables t;
        build_env_tables(rgb, width, height, &t);
        DeviceGuard g(scene->device);
        DevScene &d = scene->dev;
        gzg_status st;
        const float *p;
        if ((st = scene->upload(rgb, (size_t)width * height * 3, &p, "environment map"))) return st;
        d.env_rgb = p;
        if ((st = scene->upload(t.func.data(), t.func.size(), &p, "environment distribution"))) return st;
        d.env_func = p;
        if ((st = scene->upload(t.cdf.data(), t.cdf.size(), &p, "environment distribution"))) return st;
        d.env_cdf = p;
        if ((st = scene->upload(t.row_integral.data(), t.row_integral.size(), &p, "environment distribution")))
                return st;
        d.env_row_int = p;
        if ((st = scene->upload(t.marg_func.data(), t.marg_func.size(), &p, "environment distribution"))) return st;
        d.env_marg_func = p;
        if ((st = scene->upload(t.marg_cdf.data(), t.marg_cdf.size(), &p, "environment distribution"))) return st;
        d.env_marg_cdf = p;
        d.env_marg_int = t.marg_integral;
        d.env_w = width;
        d.env_h = height;
        const float pi = 3.14159265358979323846f, radius = 100.0f / 2.0f;
        const float power = pi * (radius * radius) * ((scale + scale + scale) / 3.0f);
        d.env_power = power;
        HostShading &hs = scene->host_shading;
        std::vector<float> cdf = hs.light_cdf;
        cdf.push_back(cdf.empty() ? power : cdf.back() + power);
        if ((st = scene->upload(cdf.data(), cdf.size(), &p, "light cdf"))) return st;
        d.light_cdf = p;
        hs.has_env = true;
        hs.env_power = power;
        hs.light_total_env = hs.light_total + power;
        hs.light_cdf = std::move(cdf);
        return clear_error();
}

GZG_API gzg_status gzg_trace_closest_instanced_device(gzg_scene *scene, const gzg_ray_d *rays, int64_t count,
                                                      gzg_hit_d *hits, int32_t *instance,
                                                      const gzg_trace_options *options, void *stream) {
        if (!scene || count < 0 || (count > 0 && (!rays || !hits || !instance)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_trace_closest_instanced_device: bad arguments");
        if (!scene->instanced)
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_trace_closest_instanced_device: not a two-level scene");
        gzg_status st = check_options(options);
        if (st != GZG_OK) return st;
        DeviceGuard g(scene->device);
        LaunchParams p = params_for(scene, options, false);
        p.inst_out = instance;
        GZG_CK(device_trace(scene, p, kOutHit, rays, count, hits, reinterpret_cast<cudaStream_t>(stream)),
               "gzg_trace_closest_instanced_device launch");
        return clear_error();
}

// Installs a launch configuration (for example one read back from a tuning
// cache) as the scene's default for closest-hit (any_hit = 0) or any-hit queries.
GZG_API gzg_status gzg_scene_set_launch(gzg_scene *scene, int32_t any_hit, const gzg_trace_options *config) {
        if (!scene || !config) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_scene_set_launch: null argument");
        TunedLaunch t;
        if (config->block_size) t.block_size = config->block_size;
        t.blocks_per_sm = config->blocks_per_sm;
        t.stack_depth = config->stack_depth;
        t.l1_carveout = config->l1_carveout ? config->l1_carveout : -1;
        (any_hit ? scene->tuned_any : scene->tuned_closest) = t;
        return clear_error();
}

GZG_API gzg_status gzg_trace_any_device(gzg_scene *scene, const gzg_ray_d *rays, int64_t count, int32_t *hit_prim,
                                        const gzg_trace_options *options, void *stream) {
        if (!scene || count < 0 || (count > 0 && (!rays || !hit_prim)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_trace_any_device: bad arguments");
        gzg_status st = check_options(options);
        if (st != GZG_OK) return st;
        DeviceGuard g(scene->device);
        GZG_CK(device_trace(scene, params_for(scene, options, true), kOutAnyPrim, rays, count, hit_prim,
                            reinterpret_cast<cudaStream_t>(stream)),
               "gzg_trace_any_device launch");
        return clear_error();
}

GZG_API gzg_status gzg_hits_to_intersections_device(gzg_scene *scene, const gzg_hit_d *hits, int64_t count,
                                                    gzg_intersection *out, void *stream) {
        if (!scene || count < 0 || (count > 0 && (!hits || !out)))
                return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_hits_to_intersections_device: bad arguments");
        DeviceGuard g(scene->device);
        GZG_CK(launch_hits_to_isect(scene->dev, hits, count, out, reinterpret_cast<cudaStream_t>(stream)),
               "gzg_hits_to_intersections_device launch");
        return clear_error();
}

GZG_API gzg_status gzg_scene_info_get(const gzg_scene *scene, gzg_scene_info *info) {
        if (!scene || !info) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_scene_info_get: null pointer");
        *info = scene->info;
        return clear_error();
}

GZG_API gzg_status gzg_scene_error_word(gzg_scene *scene, uint32_t *word, int clear) {
        if (!scene || !word) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_scene_error_word: null pointer");
        DeviceGuard g(scene->device);
        gzg_status st = read_error_word(scene, word, clear != 0);
        if (st != GZG_OK) return st;
        return clear_error();
}

}  // extern "C"

namespace gzg {

void scene_view(const gzg_scene *scene, DevScene *view, int *device, int *wide_depth) {
        *view = scene->dev;
        *device = scene->device;
        *wide_depth = scene->info.wide_depth;
}

}  // namespace gzg

namespace gzg {

LaunchParams scene_launch(const gzg_scene *scene, bool any_hit) { return params_for(scene, nullptr, any_hit); }

const WideBvh &scene_host_wide(const gzg_scene *scene) { return scene->host_wide; }
const HostShading &scene_host_shading(const gzg_scene *scene) { return scene->host_shading; }
bool scene_is_instanced(const gzg_scene *scene) { return scene->instanced; }

}  // namespace gzg
