// kernels.h - host-callable launchers of the device kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device.cuh"

namespace gzg {

struct LaunchParams {
        int traversal;   // gzg_traversal
        int leaf_test;   // gzg_leaf_test
        int wide_depth;  // levels of the wide tree (selects the stack size)
        int block_size;     // 64, 128 or 256 (anything else: 128)
        int blocks_per_sm;  // persistent grid per SM; 0 = occupancy limit
        int stack_depth;    // shared stack entries; raised to the tree's need
        int l1_carveout;    // preferred shared-memory carveout percent; <= 0 = driver default
        unsigned long long *counters;  // optional fetch counters (device)
        const uint32_t *n_dev;         // optional device-side ray count; n is then the capacity
        int32_t *inst_out;             // two-level scenes: hit instance per ray (optional)
        // Persistent launches: the pull counter of the chunk schedule, a
        // device word that no launch running at the same time uses;
        // launch_trace clears it on the launch's stream first.  Null: the
        // static schedule.
        uint32_t *sched;
};

// Rays per kernel launch; launch_trace splits larger calls (32-bit chunk
// indices in the persistent kernels).
constexpr int64_t kMaxLaunchRays = int64_t(1) << 30;

// ray_fmt: RayFormat; out_fmt: OutFormat.  Asynchronous on `st`.
cudaError_t launch_trace(const DevScene &s, const LaunchParams &p, int ray_fmt, int out_fmt, const void *rays,
                         const float *tmax, int64_t n, void *out, cudaStream_t st);

cudaError_t launch_hits_to_isect(const DevScene &s, const void *hits, int64_t n, void *out, cudaStream_t st);

// Device view, device ordinal and wide-tree depth of an uploaded scene.
void scene_view(const gzg_scene *scene, DevScene *view, int *device, int *wide_depth);

// The scene's default (tuned) launch for closest-hit or any-hit queries.
LaunchParams scene_launch(const gzg_scene *scene, bool any_hit);

}  // namespace gzg
