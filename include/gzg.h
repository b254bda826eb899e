/*
 * gzg.h - C ABI of libgzg.so, the B200 (sm_100a) ray-traversal library for the
 * Gonzales path tracer.
 *
 * The library replaces the GPU half of Gonzales' native plugin
 * (Sources/mojoKernel/include/mojo_kernel.h, exported by libmojo.so).  The host
 * (Swift in Gonzales, Python in this repository's harness) keeps parsing scenes,
 * building the SAH BVH2 and owning the primitive arrays; it hands those arrays to
 * gzg_gpu_upload_scene, which copies them to the device, re-lays them out for
 * B200 (wide quantised nodes, leaf-ordered triangle records) and returns an
 * opaque scene handle.
 *
 * Conventions
 *   - Every entry point returns gzg_status (0 = success).  gzg_last_error()
 *     returns a message for the calling thread's most recent failure.
 *   - Pointers named host_* / passed to the *_batch calls are HOST memory and
 *     are only borrowed for the call.  Pointers passed to the *_device calls
 *     are DEVICE memory owned by the caller.
 *   - `stream` arguments are cudaStream_t values passed as void* (NULL = the
 *     legacy default stream).  *_device calls are asynchronous on that stream;
 *     *_batch calls are synchronous.
 *   - One scene handle may be used from several host threads at once (the
 *     Gonzales tile renderer calls from cores-1 tasks, TileRenderer.swift:77);
 *     each *_batch call takes its own staging buffers from a locked pool.
 *   - No entry point falls back to a CPU implementation: without a usable
 *     CUDA device they return GZG_ERR_NO_DEVICE.
 */
#ifndef GZG_H
#define GZG_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GZG_API __attribute__((visibility("default")))

typedef int32_t gzg_status;
enum {
        GZG_OK = 0,
        GZG_ERR_INVALID_ARGUMENT = 1, /* null pointer, negative count, bad enum          */
        GZG_ERR_NO_DEVICE = 2,        /* no CUDA device / driver                          */
        GZG_ERR_CUDA = 3,             /* a CUDA runtime call failed                       */
        GZG_ERR_OUT_OF_MEMORY = 4,    /* device or pinned-host allocation failed          */
        GZG_ERR_BAD_SCENE = 5,        /* malformed BVH / index out of range / cycle       */
        GZG_ERR_KERNEL_FAULT = 6,     /* a kernel reported an error through its flag word */
        GZG_ERR_LIMIT = 7,            /* scene exceeds a documented size limit            */
        GZG_ERR_TIMEOUT = 8           /* a bounded host wait ran out                      */
};

/* ------------------------------------------------------------------------- */
/* Reference-compatible records.  Byte-for-byte the layouts of                */
/* mojo_kernel.h:4-58 (and the padded Mojo structs of kernel.mojo:7-80), so a */
/* Swift caller passes its existing arrays by pointer cast.                   */
/* ------------------------------------------------------------------------- */

/* PrimId_C (mojo_kernel.h:4-9).  type 0: triangle, id1 = mesh, id2 = 3*tri.
 * type 1/3: geometric primitive / area light, id2 = mesh << 32 | tri.
 * type 2 (or id2 == -1): not a triangle; never intersected (kernel.mojo:273-275). */
typedef struct gzg_prim_id {
        int64_t id1;
        int64_t id2;
        int64_t material_index;
        int8_t type;
        int8_t pad_[7];
} gzg_prim_id;

/* Material_C (mojo_kernel.h:11-15): type 0 none, 1 diffuse, 2 area light. */
typedef struct gzg_material {
        int8_t type;
        int8_t pad_[3];
        float albedo[3];
        float emission[3];
} gzg_material;

/* TriangleMesh_C (mojo_kernel.h:17-21): points are float4 (x,y,z,pad) in world
 * space; vertex_indices hold 3 int64 per triangle. */
typedef struct gzg_triangle_mesh {
        const float *points;
        const int64_t *face_indices;
        const int64_t *vertex_indices;
} gzg_triangle_mesh;

/* Ray_C (mojo_kernel.h:23-26). */
typedef struct gzg_ray {
        float org_x, org_y, org_z;
        float dir_x, dir_y, dir_z;
} gzg_ray;

/* Intersection_C (mojo_kernel.h:28-34).  On a miss: prim_id = {-1,-1,0,0},
 * t_hit = tMax, u = v = 0, hit = 0 (kernel.mojo:360-364). */
typedef struct gzg_intersection {
        gzg_prim_id prim_id;
        float t_hit;
        float u;
        float v;
        int8_t hit;
        int8_t pad_[3];
} gzg_intersection;

/* PathState_C (mojo_kernel.h:36-44). */
typedef struct gzg_path_state {
        gzg_ray ray;
        float throughput[3];
        float estimate[3];
        float albedo[3];
        int32_t pad0_;
        uint64_t pcg_state;
        uint64_t pcg_inc;
        int8_t active;
        int8_t pad1_[7];
} gzg_path_state;

/* BVH2Node (mojo_kernel.h:46-51; BVH2Node.swift:7-16): depth-first layout,
 * left child = index + 1, interior: offset = right child, count = 0;
 * leaf: offset = first prim in the prim-id array, count > 0. */
typedef struct gzg_bvh2_node {
        float bounds_min[3];
        float bounds_max[3];
        int32_t offset;
        int32_t count;
} gzg_bvh2_node;

/* ------------------------------------------------------------------------- */
/* Device-resident records (the fast path; caller-owned device memory).       */
/* ------------------------------------------------------------------------- */

/* 32-byte ray: origin + tMax, direction + unused lane (two 16-byte loads). */
typedef struct gzg_ray_d {
        float org_x, org_y, org_z, t_max;
        float dir_x, dir_y, dir_z, pad_;
} gzg_ray_d;

/* 16-byte hit: prim = index into the uploaded prim-id array, -1 on a miss
 * (then t = tMax, u = v = 0, as the reference's miss record). */
typedef struct gzg_hit_d {
        float t, u, v;
        int32_t prim;
} gzg_hit_d;

/* ------------------------------------------------------------------------- */
/* Traversal options                                                          */
/* ------------------------------------------------------------------------- */

typedef enum gzg_traversal {
        /* Wide (8-ary) nodes with 8-bit child boxes quantised outward, leaf
         * triangles in leaf order, shared-memory short stack; persistent
         * warps that refill finished lanes from a static ray sequence.
         * Default. */
        GZG_TRAVERSAL_WIDE = 0,
        /* The uploaded BVH2 traversed in the reference's exact order and slab
         * arithmetic (kernel.mojo:171-206, 223-364), one thread per ray.
         * Bit-exact with the reference including ties. */
        GZG_TRAVERSAL_BVH2 = 1,
        /* The wide traversal with one thread per ray and no refill. */
        GZG_TRAVERSAL_WIDE_ONE_RAY_PER_THREAD = 2
} gzg_traversal;

typedef enum gzg_leaf_test {
        /* Moller-Trumbore in the reference's operation order without FMA
         * contraction (kernel.mojo:122-156). Default. */
        GZG_LEAF_MOLLER_TRUMBORE = 0,
        /* Watertight shear/edge-function test (Shape/Triangle.swift:269-352). */
        GZG_LEAF_WATERTIGHT = 1
} gzg_leaf_test;

typedef struct gzg_trace_options {
        int32_t traversal; /* gzg_traversal */
        int32_t leaf_test; /* gzg_leaf_test */
        int32_t block_size; /* 64, 128 or 256 threads; 0 = the scene's tuned value (default 128) */
        int32_t blocks_per_sm; /* persistent grid = SMs x this; 0 = tuned / occupancy limit */
        int32_t stack_depth; /* shared-memory stack entries (8, 16, 32, 64); 0 = tuned / by tree depth */
        int32_t l1_carveout; /* preferred shared-memory carveout in percent; -1 = driver default,
                                0 = tuned */
        /* Optional DEVICE pointer to 3 uint64 counters that the kernel adds to:
         * [0] nodes fetched (wide nodes, or BVH2 node records), [1] triangles
         * tested, [2] rays traced.  NULL = no counting. */
        uint64_t *fetch_counters;
} gzg_trace_options;

/* Scene summary filled by gzg_scene_info. */
typedef struct gzg_scene_info {
        int64_t bvh2_nodes;
        int64_t prims;
        int64_t triangles;     /* intersectable triangles after dropping id2 == -1 prims */
        int64_t wide_nodes;
        int32_t wide_depth;    /* levels of the wide tree (root = 1) */
        int32_t bvh2_depth;
        int64_t device_bytes;  /* bytes of device memory held by the scene */
} gzg_scene_info;

typedef struct gzg_scene gzg_scene;

/* ------------------------------------------------------------------------- */
/* Entry points                                                               */
/* ------------------------------------------------------------------------- */

/* Replaces mojo_gpu_available (kernel.mojo:399-401): true when a CUDA device
 * of compute capability 10.x is visible. */
GZG_API bool gzg_gpu_available(void);

/* Message for the calling thread's last failed call ("" if none). */
GZG_API const char *gzg_last_error(void);

/* Replaces mojo_gpu_upload_scene (kernel.mojo:430-587, mojo_kernel.h:67-71).
 * Same arguments; the counts are numbers of float / int64 elements per mesh
 * exactly as BoundingHierarchy.uploadToGPU passes them
 * (BoundingHierarchy.swift:160-173).  Unlike the reference it validates every
 * node link and index (GZG_ERR_BAD_SCENE) and returns a status instead of
 * printing and returning NULL. */
GZG_API gzg_status gzg_gpu_upload_scene(const gzg_bvh2_node *bvh2_nodes, int64_t bvh2_node_count,
                                        const gzg_prim_id *prim_ids, int64_t prim_count,
                                        const gzg_triangle_mesh *meshes, int64_t mesh_count,
                                        const int64_t *mesh_points_counts,
                                        const int64_t *mesh_face_indices_counts,
                                        const int64_t *mesh_vertex_indices_counts,
                                        const gzg_material *materials, int64_t material_count,
                                        gzg_scene **out_scene);

/* Replaces mojo_gpu_free_scene (kernel.mojo:848-854).  NULL is a no-op. */
GZG_API gzg_status gzg_gpu_free_scene(gzg_scene *scene);

/* Replaces mojo_gpu_traverse_batch (kernel.mojo:608-673): closest hit for
 * `count` host rays with per-ray tMax, results into host Intersection_C
 * records.  Synchronous; copies are pipelined in chunks over pinned staging
 * buffers.  options may be NULL (defaults). */
GZG_API gzg_status gzg_gpu_traverse_batch(gzg_scene *scene, const gzg_ray *rays,
                                          const float *t_max_values, int64_t count,
                                          gzg_intersection *results,
                                          const gzg_trace_options *options);

/* Closest hit for host rays like gzg_gpu_traverse_batch (default options),
 * for callers that must not allocate: it makes no cudaMalloc, cudaFree or
 * pinned-host allocation, and stages rays, tMax values and results through a
 * fixed array in the library's device image (a file-scope __device__ array of
 * 4,980,992 bytes, held on every GPU that loads the library until exit).
 * At most 65,536 rays per call (more: GZG_ERR_LIMIT); two-level scenes are
 * rejected (GZG_ERR_INVALID_ARGUMENT).  Every call looks up the array's device
 * address afresh, launches with the scene's tuned closest-hit parameters on
 * the calling thread's per-thread default stream (cudaStreamPerThread), waits
 * for that stream, then reads and clears the scene's device error word (as
 * gzg_gpu_traverse_batch does).  All calls share the one array, which keeps
 * the last call's contents; calls are serialised by a process-wide lock, and
 * nothing else may use the array (overlapping uses would race on it).
 * No counterpart in the reference: Gonzales' GPU batch call allocates device
 * buffers on every call. */
GZG_API gzg_status gzg_gpu_traverse_batch_static(gzg_scene *scene, const gzg_ray *rays,
                                                 const float *t_max_values, int64_t count,
                                                 gzg_intersection *results);

/* Replaces mojo_gpu_shade_batch (kernel.mojo:788-846, mojo_kernel.h:76-77):
 * the live shading step of the tile loop (Core/Tile.swift:137-155) on host
 * PathState_C and Intersection_C arrays (shade_core, kernel.mojo:676-773):
 * area-light hits add emission and end the path, diffuse hits bounce with a
 * PCG32-driven cosine sample, misses end the path.  Synchronous.  Needs the
 * scene's materials and meshes from gzg_gpu_upload_scene. */
GZG_API gzg_status gzg_gpu_shade_batch(gzg_scene *scene, gzg_path_state *paths, int64_t count,
                                       const gzg_intersection *intersections);

/* gzg_gpu_traverse_batch with compact results: one 16-byte gzg_hit_d per ray
 * (t, u, v, prim = index into the uploaded prim-id array, -1 on a miss with
 * t = tMax) instead of the 48-byte Intersection_C.  The host transfer is 28 +
 * 16 bytes per ray instead of 28 + 48; a caller that keeps its prim array
 * (as the Swift BoundingHierarchy does) reads the PrimId_C record from it by
 * index.  No counterpart in the reference (its batch call returns
 * Intersection_C records only). */
GZG_API gzg_status gzg_gpu_traverse_batch_hits(gzg_scene *scene, const gzg_ray *rays,
                                               const float *t_max_values, int64_t count,
                                               gzg_hit_d *hits, const gzg_trace_options *options);

/* Shadow / any-hit batch (new; Visibility.occluded, Core/Visibility.swift:5-24,
 * answers it with a closest-hit query, BoundingHierarchy.swift:348-384).
 * occluded[i] = 1 iff some triangle is hit with 0 < t <= tMax[i]. */
GZG_API gzg_status gzg_gpu_occluded_batch(gzg_scene *scene, const gzg_ray *rays,
                                          const float *t_max_values, int64_t count,
                                          uint8_t *occluded, const gzg_trace_options *options);

/* Device-resident closest hit: rays and hits are device pointers.  The
 * launch is queued on `stream` (null: the legacy default stream) and the call
 * returns without waiting.  Device calls on one scene may be queued from
 * several threads and on several streams at once.  Each launch takes one of
 * the scene's 32 pull counters and waits, on its own stream, for the last
 * launch that used the same counter.  The first device call on a scene
 * allocates those counters (128 bytes and 32 events).  A stream being
 * captured into a graph gets a launch without a counter. */
GZG_API gzg_status gzg_trace_closest_device(gzg_scene *scene, const gzg_ray_d *rays, int64_t count,
                                            gzg_hit_d *hits, const gzg_trace_options *options,
                                            void *stream);

/* Device-resident any hit: hit_prim[i] = index of a prim hit with
 * 0 < t <= tMax (the first one found), or -1. */
GZG_API gzg_status gzg_trace_any_device(gzg_scene *scene, const gzg_ray_d *rays, int64_t count,
                                        int32_t *hit_prim, const gzg_trace_options *options,
                                        void *stream);

/* ------------------------------------------------------------------------- */
/* Two-level scenes (TransformedPrimitive, Primitive/TransformedPrimitive.swift:5-57) */
/* ------------------------------------------------------------------------- */

/* An instance of a bottom-level scene.  Matrices are row-major 3x4 affine
 * transforms (the top three rows of the reference's 4x4 Transform); the ray is
 * taken to object space as world_to_object * ray (Core/Transform+Ray.swift,
 * Geometry/Transform.swift:31-65) without renormalising the direction, so the
 * ray parameter t is shared between levels. */
typedef struct gzg_instance {
        float object_to_world[12];
        float world_to_object[12];
        int32_t blas;  /* index into the bottom-level scene list */
        int32_t pad_;
} gzg_instance;

/* World bounds of each instance: the 8 corners of its bottom-level root box
 * (blas_bounds6: minx..maxz per bottom-level scene) through object_to_world
 * (Bounds3.swift:61-69), for building the top-level BVH on the host. */
GZG_API gzg_status gzg_host_instance_bounds(const float *blas_bounds6, int64_t blas_count,
                                            const gzg_instance *instances, int64_t instance_count,
                                            float *bounds6);

/* Tighter world bounds of each instance from its uploaded bottom-level scene:
 * the boxes of the top two levels of its wide tree (up to 64, rounded
 * outward) through object_to_world, united.  They contain the geometry like
 * the root box's corners do but hug rotated shapes, so fewer rays enter an
 * instance they miss; gzg_instanced_scene_create uses them for the top-level
 * tree's leaf boxes, and a host building the top-level BVH2 should too. */
GZG_API gzg_status gzg_host_instance_bounds_from_scenes(gzg_scene *const *blas, int64_t blas_count,
                                                        const gzg_instance *instances, int64_t instance_count,
                                                        float *bounds6);

/* Creates a two-level scene from uploaded bottom-level scenes (each from
 * gzg_gpu_upload_scene; they stay owned by the caller and must outlive the
 * new scene), the instances, and a top-level BVH2 the host built over the
 * instance bounds of gzg_host_instance_bounds_from_scenes (leaf prim k is
 * instance tlas_leaf_instance[k]).  Only the
 * wide traversal runs on a two-level scene; hits report the bottom-level prim
 * index and, through gzg_trace_closest_instanced_device, the instance. */
GZG_API gzg_status gzg_instanced_scene_create(gzg_scene *const *blas, int64_t blas_count,
                                              const gzg_instance *instances, int64_t instance_count,
                                              const gzg_bvh2_node *tlas_nodes, int64_t tlas_node_count,
                                              const int64_t *tlas_leaf_instance, int64_t tlas_leaf_count,
                                              gzg_scene **out_scene);

/* Closest hit on a two-level scene: hits as gzg_trace_closest_device (prim =
 * index into the hit instance's bottom-level prim array) and instance[i] =
 * the hit instance or -1. */
GZG_API gzg_status gzg_trace_closest_instanced_device(gzg_scene *scene, const gzg_ray_d *rays, int64_t count,
                                                      gzg_hit_d *hits, int32_t *instance,
                                                      const gzg_trace_options *options, void *stream);

/* Launch autotuner: times the persistent wide kernel on the caller's DEVICE
 * rays over L1 carveout, blocks per SM, block size and stack depth
 * (coordinate descent, CUDA events on `stream`), keeps the fastest as the
 * scene's default for closest-hit (any_hit = 0) or any-hit queries, and
 * returns it (and its time per launch in ms).  Synchronous. */
GZG_API gzg_status gzg_scene_autotune(gzg_scene *scene, const gzg_ray_d *rays, int64_t count, int32_t any_hit,
                                      gzg_trace_options *best, float *best_ms, void *stream);

/* Installs a launch configuration (e.g. from a tuning cache) as the scene's
 * default for closest-hit (any_hit = 0) or any-hit queries. */
GZG_API gzg_status gzg_scene_set_launch(gzg_scene *scene, int32_t any_hit, const gzg_trace_options *config);

/* A homogeneous participating medium (Medium/Homogeneous.swift) filling an
 * axis-aligned box whose boundary scatters nothing (an interface,
 * Material/Interface.swift), with a Henyey-Greenstein phase function
 * (Medium/HenyeyGreenstein.swift).  The reference's integrator never samples
 * its media (VolumePathIntegrator.swift:394 hard-codes the transmittance to
 * white); renderers run the branch as meant: each path segment samples a
 * scattering distance in the box (a random color channel, as
 * Homogeneous.sample), a scattering event shades with the phase function
 * (light sample with MIS, phase sample), and shadow rays and MIS probes carry
 * the box's transmittance. */
typedef struct gzg_medium {
        float box_min[3], box_max[3];
        float sigma_a[3];  /* absorption per unit length, per RGB channel */
        float sigma_s[3];  /* scattering per unit length, per RGB channel */
        float g;           /* Henyey-Greenstein asymmetry in (-1, 1) */
        int32_t reserved;  /* 0 */
} gzg_medium;

/* Sets (or, with medium NULL, removes) the scene's medium; flat or two-level
 * scenes.  Renderers created afterwards use it.  Rejects an empty box,
 * negative or non-finite coefficients and |g| >= 1. */
GZG_API gzg_status gzg_scene_set_medium(gzg_scene *scene, const gzg_medium *medium);

/* Adds an environment light (Light/InfiniteLight.swift) to an uploaded scene
 * (flat or two-level), after its area lights in the light list: the HOST map
 * rgb[height][width][3] (row v, column u) in the equal-area square layout the
 * reference reads, looked up bilinearly; its 1024 x 1024 sampling
 * distribution is built from the green channel, as the reference's is, and
 * `scale` enters only the light's power pi * 50^2 * scale (the light choice),
 * as in the reference.  Once per scene; renderers created afterwards use it
 * (single-scene renderers only). */
GZG_API gzg_status gzg_scene_set_environment(gzg_scene *scene, const float *rgb, int32_t width, int32_t height,
                                             float scale);

/* Options of gzg_gpu_build_scene and gzg_gpu_build_mesh_scene. */
enum { GZG_BUILD_DEFAULT = 0, GZG_BUILD_LBVH = 1, GZG_BUILD_PLOC = 2 };  /* DEFAULT = LBVH */
typedef struct gzg_build_options {
        int32_t leaf_size;   /* prims per leaf child, 1..4; 0 = 1 (measured fastest
                              * to traverse: 3,765 vs 3,031 Mrays/s at 4) */
        int32_t builder;     /* GZG_BUILD_LBVH (the default): the radix tree of the
                              * Morton codes; GZG_BUILD_PLOC: clusters in Morton
                              * order merged with their mutual nearest neighbour
                              * (union box area) within +-radius: a lower
                              * surface-area cost but slower to build and, on the
                              * ray-cast mesh, to traverse */
        int32_t radius;      /* PLOC search radius, 1..64; 0 = 16 */
        int32_t reserved;    /* zero */
} gzg_build_options;

/* Builds the scene's tree on the device instead of taking the host's BVH2
 * (the replacement of BoundingHierarchyBuilder.swift:66-339 for hosts that
 * would otherwise build it): the arguments of gzg_gpu_upload_scene without
 * the BVH2, prims in any order.  A binary tree over the prims sorted by the
 * 30-bit Morton codes of their centroids (PLOC clustering or the radix tree,
 * gzg_build_options.builder), collapsed on the device into the same 8-wide
 * quantised tree the upload path makes; every query and
 * renderer call accepts the scene, except traversal = GZG_TRAVERSAL_BVH2
 * (there is no reference BVH2: the call fails).  Hit prim ids index
 * prim_ids as given.  Every triangle prim must resolve to valid mesh and
 * vertex indices (GZG_ERR_BAD_SCENE otherwise).  options may be NULL. */
GZG_API gzg_status gzg_gpu_build_scene(const gzg_prim_id *prim_ids, int64_t prim_count,
                                       const gzg_triangle_mesh *meshes, int64_t mesh_count,
                                       const int64_t *mesh_points_counts, const int64_t *mesh_face_indices_counts,
                                       const int64_t *mesh_vertex_indices_counts, const gzg_material *materials,
                                       int64_t material_count, const gzg_build_options *options,
                                       gzg_scene **out_scene);

/* Device time in ms of the tree build of a gzg_gpu_build_scene scene (keys,
 * sort, radix tree, bounds, collapse); -1 for an uploaded scene. */
GZG_API gzg_status gzg_scene_build_time(const gzg_scene *scene, float *device_ms);

/* Surface-area cost of the scene's wide tree: 1 + sum over interior
 * children of their box area + sum over leaf children of area x triangles,
 * relative to the root's area (quantised boxes).  Compares trees built by
 * different builders over the same prims. */
GZG_API gzg_status gzg_scene_tree_cost(const gzg_scene *scene, double *cost);

/* ---- ingestion fast path ----------------------------------------------- */

/* One mesh of gzg_gpu_build_mesh_scene: packed arrays as a PLY file holds
 * them (12 B per vertex, 12 B per triangle, instead of the float4 points and
 * int64 indices of TriangleMesh_C). */
typedef struct gzg_mesh_arrays {
        const float *points;      /* vertex_count x 3 */
        int64_t vertex_count;
        const int32_t *indices;   /* triangle_count x 3, into this mesh's points */
        int64_t triangle_count;
        int64_t material;         /* index into materials; an area-light material
                                   * (type 2) makes every triangle an area light */
} gzg_mesh_arrays;

/* Builds a scene from packed HOST mesh arrays with no host-side per-triangle
 * work: the arrays are copied to the device as they are, expanded there into
 * the reference's records (prims: PrimId_C type 1, id2 = mesh << 32 | tri,
 * or type 3 area lights numbered in mesh order; TriangleMesh_C copies with
 * float4 points and int64 indices) and the tree is built on the device as
 * gzg_gpu_build_scene does.  Indices out of range give GZG_ERR_BAD_SCENE. */
GZG_API gzg_status gzg_gpu_build_mesh_scene(const gzg_mesh_arrays *meshes, int64_t mesh_count,
                                            const gzg_material *materials, int64_t material_count,
                                            const gzg_build_options *options, gzg_scene **out_scene);

/* A triangle mesh read from a PLY file (Shape/PlyMesh.swift): format
 * binary_little_endian / binary_big_endian 1.0; vertex float properties
 * x y z [u v | nx ny nz | nx ny nz u v (or s t) | u v nx ny nz]; faces as
 * "list uchar|uint int vertex_indices" [+ "int face_indices"].  Faces must
 * be triangles.  Arrays are library-owned until gzg_ply_free. */
typedef struct gzg_ply_mesh {
        int64_t vertex_count, face_count;
        const float *points;        /* vertex_count x 3 */
        const float *normals;       /* vertex_count x 3, or NULL */
        const float *uvs;           /* vertex_count x 2, or NULL */
        const int32_t *indices;     /* face_count x 3 */
        const int32_t *face_indices;/* face_count, or NULL */
        void *owner;
} gzg_ply_mesh;

GZG_API gzg_status gzg_ply_read(const char *path, gzg_ply_mesh **out);
GZG_API gzg_status gzg_ply_parse(const void *data, int64_t size, gzg_ply_mesh **out);
GZG_API gzg_status gzg_ply_free(gzg_ply_mesh *mesh);

/* Vertex normals (vertex_count x 3) and / or UVs (vertex_count x 2) of mesh
 * `mesh` of an uploaded flat scene (HOST arrays; either may be NULL;
 * vertex_count = the mesh's points count / 4).  The renderer then shades as
 * Triangle.computeSurfaceInteraction does with them (Shape/Triangle.swift:
 * 386-452): dpdu from the UVs unless degenerate, the shading normal
 * interpolated from the vertex normals; the shading normal weighs light
 * samples and BSDF samples, the geometric normal the path throughput.  Call
 * before the scene enters a renderer, batch or two-level scene. */
GZG_API gzg_status gzg_scene_set_vertex_attributes(gzg_scene *scene, int64_t mesh, const float *normals,
                                                   const float *uvs, int64_t vertex_count);

/* ---- film output ---------------------------------------------------------- */

/* Normalises device film sums into an image (Pixel.normalized,
 * Core/Pixel.swift:12-16): image = film_rgb / film_w per pixel (3 floats per
 * pixel), black stays black; non-black light with weight 0 (the reference
 * throws) gives black and adds 1 to *zero_weight_count (a device counter;
 * may be NULL).  The albedo and normal AOV sums resolve with the same film_w
 * (Film.writeImages adds them with the sample weights).  Asynchronous on
 * stream. */
GZG_API gzg_status gzg_film_resolve_device(const float *film_rgb, const float *film_w, int64_t pixels, float *image,
                                           unsigned long long *zero_weight_count, void *stream);

/* Writes a HOST image (height x width x channels floats, channels 3 or 4,
 * row 0 at the top) as an OpenEXR file with RGBA 32-bit float channels (alpha
 * 1 when channels = 3), as Image/OpenImageIOWriter.swift writes the beauty,
 * albedo and normal images: single-part scanlines, no compression. */
GZG_API gzg_status gzg_write_exr(const char *path, const float *pixels, int32_t width, int32_t height,
                                 int32_t channels);

/* Parameters of the renderer's general materials, by Material_C.type:
 *   3 dielectric        (Material/Dielectric.swift): eta, roughness u/v;
 *   4 coated diffuse    (Material/CoatedDiffuse.swift, base = albedo): eta,
 *                       roughness u/v of the coating, thickness;
 *   5 conductor         (Material/Conductor.swift): conductor eta/k per RGB
 *                       channel, conductor roughness u/v (used as alpha);
 *   6 coated conductor  (Material/CoatedConductor.swift, base reflectance =
 *                       albedo): coating eta, roughness u/v, thickness,
 *                       conductor eta/k and roughness.
 * Dielectric and coating roughness, and a coated conductor's conductor
 * roughness, are remapped to alpha = sqrt(roughness). */
typedef struct gzg_material_params {
        float eta, roughness_u, roughness_v, thickness;
        float conductor_eta[3], conductor_roughness_u;
        float conductor_k[3], conductor_roughness_v;
} gzg_material_params;

/* One HOST record per material of the flat scene (count = its material
 * count; records of other types are ignored).  Once per scene, before the
 * scene enters a two-level scene, a batch or a renderer; without it types 3
 * to 6 shade as diffuse. */
GZG_API gzg_status gzg_scene_set_material_params(gzg_scene *scene, const gzg_material_params *params,
                                                 int64_t count);

/* Expands device hits into reference Intersection_C records on the device
 * (prim-id lookup; the miss record of kernel.mojo:362-364). */
GZG_API gzg_status gzg_hits_to_intersections_device(gzg_scene *scene, const gzg_hit_d *hits,
                                                    int64_t count, gzg_intersection *out,
                                                    void *stream);

/* ------------------------------------------------------------------------- */
/* Path integrator (wavefront)                                                */
/* ------------------------------------------------------------------------- */

/* Parameters of a render.  The integrator is Gonzales' MIS path integrator
 * (Integrator/VolumePathIntegrator.swift:67-463) with every random dimension
 * drawn from the Z-Sobol sampler, restructured as a wavefront: generate ->
 * extend -> shade -> shadow (any hit) [-> BSDF probe] -> accumulate. */
typedef struct gzg_render_params {
        int32_t width, height, spp, max_depth;
        int32_t rr_min_bounce;   /* Russian roulette from this bounce (reference: 2, "bounce > 1") */
        int32_t mis_corrected;   /* 0: MIS as written (the BSDF strategy gets weight 0 because its
                                    light density is queried with tHit = 0, Core/Sampleable.swift:55);
                                    1: corrected MIS */
        int64_t seed;            /* Z-Sobol seed (reference: 1234, Sampler/Random.swift:66) */
        float eye[3], target[3], up[3];
        float fov_deg;           /* full field of view of the shorter image side */
        float filter_radius, filter_sigma; /* Gaussian pixel filter (reference default 2, 0.5) */
        int32_t first_sample;    /* render sample indices [first_sample, first_sample + spp) */
        int32_t sampler_spp;     /* ...of a Z-Sobol sampler with this many samples per pixel (0: spp) */
        int32_t wave_paths;      /* paths in flight per wave (0: library default, 2^24 paths or the
                                    frame's path count if smaller; about 350 device bytes per path) */
        int32_t use_graph;       /* capture one wave as a CUDA graph and replay it */
        float lens_radius;       /* thin lens (PerspectiveCamera.depthOfField); 0: pinhole */
        float focal_distance;    /* distance of the plane in focus (reference default 1e6) */
        int32_t two_sided_emission; /* 0: area lights emit on the side their geometric normal faces
                                       (AreaLight.emittedRadiance, Light/AreaLight.swift:13-19);
                                       1: on both sides, as the live shading step counts any hit
                                       on an emitter (shade_core, kernel.mojo:696-701) */
        int32_t crop[4];         /* crop window in pixels [x0, x1) x [y0, y1) as {x0, y0, x1, y1}
                                    (Film's crop, the pixels Film.getSampleBounds covers,
                                    Core/Film.swift:7-27); all 0: the whole frame.  The camera and
                                    the sampler keep the whole frame; films hold the window's
                                    pixels only, row-major, (x1 - x0) x (y1 - y0) */
} gzg_render_params;

typedef struct gzg_renderer gzg_renderer;

/* Render statistics (cumulative over the renderer's lifetime). */
typedef struct gzg_render_stats {
        uint64_t camera_rays, extension_rays, shadow_rays, probe_rays;
        uint64_t waves;
} gzg_render_stats;

/* Creates a renderer (device buffers for one wave) for a scene uploaded with
 * materials.  Replaces the Tile.render bounce loop (Core/Tile.swift:19-223). */
GZG_API gzg_status gzg_renderer_create(gzg_scene *scene, const gzg_render_params *params,
                                       gzg_renderer **out);
GZG_API gzg_status gzg_renderer_destroy(gzg_renderer *renderer);

/* Adds one render pass to DEVICE film buffers (caller-owned, row-major):
 * film_rgb[3*W*H] += sample radiance, film_sq[3*W*H] += its square (may be
 * NULL), film_w[W*H] += sample weight.  The image is film_rgb / film_w (the
 * reference's Pixel.normalized, Core/Pixel.swift:12-16).  Asynchronous on
 * `stream`. */
GZG_API gzg_status gzg_renderer_render(gzg_renderer *renderer, float *film_rgb, float *film_sq, float *film_w,
                                       void *stream);

GZG_API gzg_status gzg_renderer_stats(const gzg_renderer *renderer, gzg_render_stats *stats);

/* Film settings of Film.add (Core/Film.swift:107-119): each sample's light is
 * scaled by iso / 100 (default iso 100) and, when max_component > 0, scaled
 * down so its largest component is at most max_component. */
GZG_API gzg_status gzg_renderer_set_film(gzg_renderer *renderer, float iso, float max_component);

/* gzg_renderer_render plus the first-hit AOVs of Tile.render (Tile.swift:
 * 157-205): film_albedo[3*W*H] += the first hit's BSDF albedo, film_normal
 * [3*W*H] += its geometric normal (zero for camera rays that miss); either may
 * be NULL.  The AOV images are the sums / film_w, like the beauty image. */
GZG_API gzg_status gzg_renderer_render_aov(gzg_renderer *renderer, float *film_rgb, float *film_sq, float *film_w,
                                           float *film_albedo, float *film_normal, void *stream);

/* Sort of the extension queue before shading. */
typedef enum gzg_sort_key {
        GZG_SORT_NONE = 0,
        GZG_SORT_MATERIAL = 1,  /* by the hit's material (batch-wide index) */
        GZG_SORT_SCENE = 2      /* by the path's scene */
} gzg_sort_key;

/* Options of a batch renderer (the per-scene wave_paths / use_graph of
 * gzg_render_params are not used by a batch). */
typedef struct gzg_batch_options {
        int32_t wave_paths;  /* paths in flight per wave (0: library default, 2^24 paths; about 350
                                device bytes per path) */
        int32_t use_graph;   /* capture one wave as a CUDA graph and replay it */
        int32_t sort_key;    /* gzg_sort_key */
        int32_t reserved;
} gzg_batch_options;

/* Creates one renderer over many scenes (no reference counterpart: Gonzales
 * renders one scene per process).  Scene k is rendered with params[k] into
 * its window of one batch film: pixels [offset_k, offset_k + W_k*H_k) where
 * the offsets come from gzg_renderer_film_layout.  Paths of all scenes share
 * the waves; each path carries its scene and starts traversal at its scene's
 * root of one concatenated wide tree.  All scenes live on one device and were
 * uploaded with materials; two-level scenes are rejected. */
GZG_API gzg_status gzg_batch_renderer_create(gzg_scene *const *scenes, const gzg_render_params *params,
                                             int64_t scene_count, const gzg_batch_options *options,
                                             gzg_renderer **out);

/* Writes scene_count + 1 pixel offsets of the batch film (the last one is
 * the film's total pixel count). */
GZG_API gzg_status gzg_renderer_film_layout(const gzg_renderer *renderer, int64_t *pixel_offsets);

/* Times whole renders (into scratch films) over wave sizes and sort keys,
 * keeps the fastest configuration and returns it (and its time per render in
 * ms).  Synchronous; resets the renderer's statistics. */
GZG_API gzg_status gzg_renderer_autotune(gzg_renderer *renderer, gzg_batch_options *best, float *best_ms,
                                         void *stream);

/* Reads (and with clear != 0 resets) the device error word the renderer's
 * traversals report to. */
GZG_API gzg_status gzg_renderer_error_word(gzg_renderer *renderer, uint32_t *word, int32_t clear);

/* ------------------------------------------------------------------------- */
/* Differentiable rendering (path-replay adjoint)                             */
/* ------------------------------------------------------------------------- */

/* An albedo texture over material `material` (no reference counterpart: the
 * reference's GPU path has no textures or derivatives).  Nearest texel of a
 * resolution x resolution RGB grid laid over a plane through `origin`:
 * u = dot(p - origin, u_axis), v = dot(p - origin, v_axis), texel
 * (ix, iy) = (int)clamp((u, v) * resolution, 0, resolution - 1). */
typedef struct gzg_texture_binding {
        int32_t material;
        int32_t reserved;
        float origin[3], u_axis[3], v_axis[3];
} gzg_texture_binding;

/* Binds `count` textures (texture t uses bindings[t]) whose texels live in
 * the DEVICE array texels[count][resolution][resolution][3] (row iy, column
 * ix), borrowed and read at render time, and scales every emission by
 * emission_scale.  count = 0 removes the textures.  Single-scene renderers
 * only.  Russian roulette is not differentiated: adjoint renders should set
 * rr_min_bounce >= max_depth. */
GZG_API gzg_status gzg_renderer_set_textures(gzg_renderer *renderer, const gzg_texture_binding *bindings,
                                             int32_t count, int32_t resolution, const float *texels,
                                             float emission_scale);

/* gzg_renderer_render with double-precision DEVICE films (each path's
 * radiance is still computed in FP32; only the sums are FP64). */
GZG_API gzg_status gzg_renderer_render_f64(gzg_renderer *renderer, double *film_rgb, double *film_sq,
                                           double *film_w, void *stream);

/* Path-replay adjoint of one render pass: given adj_rgb = dLoss/dImage per
 * pixel (DEVICE, 3 floats per pixel, image = film_rgb / film_w) and the
 * pass's film_w (DEVICE), ADDS dLoss/dtexel to d_texels (DEVICE, the texel
 * layout) and dLoss/demission_scale to *d_emission (DEVICE, may be NULL).
 * Each wave is traced twice: a primal pass keeps each path's radiance, then
 * the replay draws the same samples and, at every textured vertex, adds
 * adj * (radiance still to come) / albedo.  Asynchronous on `stream`. */
GZG_API gzg_status gzg_renderer_adjoint(gzg_renderer *renderer, const float *adj_rgb, const float *film_w,
                                        float *d_texels, double *d_emission, void *stream);

/* Device Z-Sobol values (Sampler/ZSobolSampler.swift:6-280): for each of n
 * pixel samples (device arrays px, py, index) the values of the get1D / get2D /
 * get3D calls listed in the HOST array kinds (1, 2 or 3 each, at most 64),
 * starting at dimension 0, written row by row to the DEVICE array out.
 * The sampler is ZSobolSampler(samplesPerPixel:fullResolution:seed:). */
GZG_API gzg_status gzg_zsobol_fill_device(int64_t samples_per_pixel, int32_t res_x, int32_t res_y, int64_t seed,
                                          const int32_t *px, const int32_t *py, const int64_t *index, int64_t n,
                                          const int32_t *kinds, int32_t nkinds, float *out, void *stream);

/* Camera rays of Tile.render's first phase (Core/Tile.swift:27-59) for host
 * callers that drive the bounce loop through gzg_gpu_traverse_batch and
 * gzg_gpu_shade_batch themselves: for paths [first_path, first_path + count)
 * of the frame described by params (path = pixel * spp + sample, pixel = the
 * film pixel, row-major over the crop window or the whole frame; samples
 * first_sample + sample of the Z-Sobol sampler) writes
 * the Ray_C record (camera-space sample through the Gaussian filter and the
 * perspective camera, Sampler.getCameraSample + PerspectiveCamera.generateRay),
 * the ray weight (filter value / filter pdf, Tile.swift:36-40) and the pixel
 * index into HOST arrays.  Computed on the current device; synchronous. */
GZG_API gzg_status gzg_camera_rays(const gzg_render_params *params, int64_t first_path, int64_t count,
                                   gzg_ray *rays, float *weights, int32_t *pixels);

/* Convenience: renders into HOST films (overwritten); synchronous. */
GZG_API gzg_status gzg_render_image(gzg_scene *scene, const gzg_render_params *params, float *film_rgb,
                                    float *film_sq, float *film_w, gzg_render_stats *stats);

/* Scene statistics. */
GZG_API gzg_status gzg_scene_info_get(const gzg_scene *scene, gzg_scene_info *info);

/* Reads (and with clear != 0 resets) the scene's device error word, which
 * kernels set instead of trapping (stack overflow, step cap, bad index). */
GZG_API gzg_status gzg_scene_error_word(gzg_scene *scene, uint32_t *word, int clear);

#ifdef __cplusplus
}
#endif

#endif /* GZG_H */
