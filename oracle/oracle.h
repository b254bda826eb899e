/*
 * oracle.h - CPU restatement of the Gonzales hot path, used ONLY as the
 * correctness checker (tests, smoke check) and as the timed CPU baseline.
 * Nothing in the product library links or calls this code.
 *
 * Restated from the reference (paths relative to the Gonzales source tree):
 *   SAH BVH2 build + flatten   Sources/libgonzales/Accelerators/BoundingHierarchyBuilder.swift:66-339
 *   bounds helpers             Sources/libgonzales/Geometry/Bounds3.swift, Geometry/Geometry.swift:46-61
 *   triangle bound             Sources/libgonzales/Shape/Triangle.swift:248-256
 *   traversal + MT leaf test   Sources/mojoKernel/kernel.mojo:84-95, 122-156, 171-206, 223-364
 *   watertight leaf test       Sources/libgonzales/Shape/Triangle.swift:269-352
 *   Swift slab test (KATs)     Sources/libgonzales/Geometry/Bounds3.swift:143-164
 *   Z-Sobol sampler            Sources/libgonzales/Sampler/ZSobolSampler.swift:6-280
 *
 * Parity pins: the Sobol utilities against the reference's own KATs
 * (Tests/libgonzalesTests/SobolSamplerTests.swift), the bounds helpers and the
 * Swift slab test against Tests/libgonzalesTests/BoundsTests.swift, the Sobol
 * matrices against the published first dimensions of the Sobol sequence.  The
 * reference has no traversal or BVH tests and cannot run here (no Swift or Mojo
 * toolchain), so traversal parity is pinned by this restatement only.
 *
 * Built with -ffp-contract=off: every float operation rounds separately, in the
 * reference's source order.
 */
#ifndef GZG_ORACLE_H
#define GZG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Layouts identical to mojo_kernel.h:4-58 (and include/gzg.h). */
typedef struct orc_prim_id {
        int64_t id1, id2, material_index;
        int8_t type;
        int8_t pad_[7];
} orc_prim_id;
typedef struct orc_mesh {
        const float *points;
        const int64_t *face_indices;
        const int64_t *vertex_indices;
        const float *normals; /* per vertex x3, or NULL (renderer only) */
        const float *uvs;     /* per vertex x2, or NULL (renderer only) */
} orc_mesh;
typedef struct orc_ray {
        float ox, oy, oz, dx, dy, dz;
} orc_ray;
typedef struct orc_isect {
        orc_prim_id prim_id;
        float t, u, v;
        int8_t hit;
        int8_t pad_[3];
} orc_isect;
typedef struct orc_node {
        float mn[3], mx[3];
        int32_t offset, count;
} orc_node;

/* --- BVH build ---------------------------------------------------------- */

/* Bound of every triangle: union(Bounds3f(p0, p1), p2) with Swift min/max. */
void orc_triangle_bounds(const float *points4, const int64_t *vertex_indices, int64_t ntri,
                         float *bounds6);

/* SAH build over n prim bounds (minx,miny,minz,maxx,maxy,maxz per prim).
 * Writes the flattened nodes (capacity 2n) and the sorted prim order
 * (order[k] = input index of the k-th prim in the leaf order).
 * Returns the node count (0 for n == 0). */
int64_t orc_build_bvh2(const float *bounds6, int64_t n, orc_node *nodes, int64_t *order);

/* --- traversal ---------------------------------------------------------- */

/* counters (optional, may be NULL): per ray {interior steps, leaf visits,
 * triangle tests, node fetches}. */
void orc_traverse_batch(const orc_node *nodes, const orc_prim_id *prims, const orc_mesh *meshes,
                        const orc_ray *rays, const float *tmax, int64_t n, int watertight,
                        orc_isect *out, int32_t *hit_index, uint32_t *counters, int threads);

/* One closest-hit query (MT leaf test). */
void orc_trace_one(const orc_node *nodes, const orc_prim_id *prims, const orc_mesh *meshes, const orc_ray *ray,
                   float tmax, orc_isect *out, int32_t *hit_index);

/* --- path integrator ---------------------------------------------------- */

typedef struct orc_material {
        int8_t type;
        int8_t pad_[3];
        float albedo[3];
        float emission[3];
} orc_material;

typedef struct orc_render_params {
        int32_t width, height, spp, max_depth;
        int32_t rr_min_bounce;  /* Russian roulette when bounce >= this (reference: 2) */
        int32_t mis_corrected;  /* 0: as written (BSDF strategy weight 0), 1: corrected */
        int64_t seed;           /* Z-Sobol seed (reference: 1234) */
        float eye[3], target[3], up[3];
        float fov_deg;
        float filter_radius, filter_sigma;
        int32_t first_sample;   /* sample indices [first_sample, first_sample + spp) of a sampler */
        int32_t sampler_spp;    /* of sampler_spp samples per pixel (0: spp) */
        float iso;              /* film sensitivity: light scaled by iso / 100 (0: 100) */
        float max_component;    /* clamp of a sample's largest component (0: none) */
        float lens_radius;      /* thin lens (PerspectiveCamera.depthOfField); 0: pinhole */
        float focal_distance;
        int32_t two_sided_emission; /* 1: area lights emit on both sides (the live shade_core's rule) */
        /* a homogeneous medium (Medium/Homogeneous.swift) filling the box
         * medium_min..medium_max, whose boundary does not scatter (an
         * interface); phase function Henyey-Greenstein with asymmetry medium_g */
        int32_t has_medium;
        float medium_min[3], medium_max[3];
        float sigma_a[3], sigma_s[3];
        float medium_g;
        int32_t crop[4];  /* film window {x0, y0, x1, y1} in pixels; all 0: the whole frame */
} orc_render_params;

/* Renders the scene; per pixel (row-major) accumulates the film sums of the
 * reference's Pixel (light sum, weight sum; Core/Pixel.swift, Core/Film.swift:
 * 107-119) plus the per-channel sum of squares of the sample values.
 * counters (optional): {camera rays, extension rays, shadow rays, probe rays}. */
void orc_render(const orc_node *nodes, const orc_prim_id *prims, const orc_mesh *meshes,
                const orc_material *materials, int64_t n_materials, int64_t n_prims,
                const orc_render_params *params, float *sum_rgb, float *sum_sq, float *sum_w,
                uint64_t *counters, int threads);

/* Camera rays of paths [first, first + count) of the frame in params (path =
 * pixel * spp + sample, pixel = y * width + x): Ray_C records (6 floats),
 * ray weights (filter value / filter pdf) and pixel indices.  Tile.render
 * phase 1 (Core/Tile.swift:27-59). */
void orc_camera_rays(const orc_render_params *params, int64_t first, int64_t count, float *rays6, float *weights,
                     int32_t *pixels);

/* Albedo textures and an emission scale for the differentiable renderer's
 * scene: material m with material_texture[m] = t >= 0 takes its albedo from
 * texture t, a res x res RGB grid (texels[((t * res + iy) * res + ix) * 3 + c])
 * laid over a plane: u = dot(p - origin, u_axis), v = dot(p - origin, v_axis),
 * ix = (int)clamp(u * res, 0, res - 1), iy likewise (nearest texel).  Every
 * emission (emitted hits, light samples, probes) is multiplied by
 * emission_scale.  Not part of the reference, whose scenes carry no textures
 * on this path; the oracle's finite differences check the GPU adjoint. */
typedef struct orc_textures {
        int32_t count, resolution;
        const int32_t *material_texture; /* n_materials entries */
        const float *maps;               /* count x {origin[3], u_axis[3], v_axis[3]} */
        const float *texels;
        float emission_scale;
} orc_textures;

void orc_render_textured(const orc_node *nodes, const orc_prim_id *prims, const orc_mesh *meshes,
                         const orc_material *materials, int64_t n_materials, int64_t n_prims,
                         const orc_render_params *params, const orc_textures *textures, float *sum_rgb,
                         float *sum_sq, float *sum_w, uint64_t *counters, int threads);

typedef struct orc_env orc_env;
typedef struct orc_render_instances orc_render_instances;

/* The general form: a flat scene (nodes .. n_prims) or, with `instances`, a
 * two-level one (the flat arrays are then unused); an optional environment
 * light (appended last to the light list; its power enters the light
 * choice); optional material parameters (per material: eta, roughness u,
 * v, thickness, conductor eta[3], conductor roughness u,
 * conductor k[3], conductor roughness v: 12 floats) for materials of types 3
 * to 6; optional textures (flat scenes). */
void orc_render_ex(const orc_node *nodes, const orc_prim_id *prims, const orc_mesh *meshes,
                   const orc_material *materials, int64_t n_materials, int64_t n_prims,
                   const orc_render_instances *instances, const orc_env *env, const float *material_params,
                   const orc_render_params *params,
                   const orc_textures *textures, float *sum_rgb, float *sum_sq, float *sum_w, float *sum_albedo,
                   float *sum_normal, uint64_t *counters, int threads);

/* PathState_C (mojo_kernel.h:36-44). */
typedef struct orc_path_state {
        orc_ray ray;
        float throughput[3];
        float estimate[3];
        float albedo[3];
        int32_t pad0_;
        uint64_t pcg_state;
        uint64_t pcg_inc;
        int8_t active;
        int8_t pad1_[7];
} orc_path_state;

/* shade_core over a batch (kernel.mojo:676-773, mojo_cpu_shade_batch :378-390). */
void orc_shade_batch(orc_path_state *paths, int64_t n, const orc_isect *isects, const orc_mesh *meshes,
                     const orc_material *materials);

/* --- two-level scenes --------------------------------------------------- */

typedef struct orc_blas {
        const orc_node *nodes;
        const orc_prim_id *prims;
        const orc_mesh *meshes;
} orc_blas;

/* Closest hit through a top-level BVH2 whose leaf prim k is instance
 * leaf_instance[k]; instance i has world_to_object w2o[12 * i] (row-major
 * 3x4) and bottom-level scene blas_of[i].  Restates TransformedPrimitive.
 * intersect (Primitive/TransformedPrimitive.swift:5-22): ray = inverse * ray
 * (Core/Transform+Ray.swift, Geometry/Transform.swift:31-65), bottom-level
 * closest hit with the current tHit.  Outputs per ray: prim (bottom-level
 * prim index or -1), instance (or -1), t (tMax on a miss), u, v. */
void orc_traverse_instanced(const orc_node *tlas, const int64_t *leaf_instance, const float *w2o,
                            const int32_t *blas_of, const orc_blas *blas, const orc_ray *rays, const float *tmax,
                            int64_t n, int32_t *prim, int32_t *inst, float *t, float *u, float *v, int threads);

/* One ray of the above (the renderer's trace); returns 1 on a hit. */
int orc_trace_instanced_one(const orc_node *tlas, const int64_t *leaf_instance, const float *w2o,
                            const int32_t *blas_of, const orc_blas *blas, const orc_ray *ray, float tmax,
                            int32_t *prim, int32_t *inst, float *t, float *u, float *v);

/* A two-level scene for the renderer: the traversal arrays above plus
 * object_to_world o2w[12 * i] (row-major 3x4) and each bottom-level scene's
 * materials.  Hits are shaded in object space and carried to world space as
 * Transform * SurfaceInteraction does (Core/Transform+SurfaceInteraction.swift:3-14). */
typedef struct orc_render_instances {
        const orc_node *tlas;
        const int64_t *leaf_instance;
        const float *w2o, *o2w;
        const int32_t *blas_of;
        int64_t instance_count;
        const orc_blas *blas;
        const orc_material *const *blas_materials;
        int64_t blas_count;
        const float *const *blas_material_params; /* per bottom-level scene: 12 floats per material, or NULL */
} orc_render_instances;

/* The MT leaf test alone (kernel.mojo:122-156); returns 1 on a hit. */
int orc_intersect_triangle_mt(const float *o, const float *d, const float *p0, const float *p1,
                              const float *p2, float tmax, float *t, float *u, float *v);
/* The watertight leaf test alone (Triangle.swift:269-352), tHit in/out. */
int orc_intersect_triangle_watertight(const float *o, const float *d, const float *p0,
                                      const float *p1, const float *p2, float *thit, float *b0,
                                      float *b1, float *b2);
/* The reference's slab test (kernel.mojo:171-206) for one ray and box. */
int orc_intersect_aabb(const float *mn, const float *mx, const float *o, const float *d, float tmax,
                       float *tnear);
/* The Swift slab test Bounds3.intersects (Bounds3.swift:143-164). */
int orc_bounds_intersects_swift(const float *mn, const float *mx, const float *o, const float *d,
                                float thit);
float orc_bounds_surface_area(const float *mn, const float *mx);
int orc_bounds_maximum_extent(const float *mn, const float *mx);

/* --- BSDFs (Bsdf/DielectricBsdf.swift, Bsdf/LayeredBsdf.swift) ------------ */

/* type 1 diffuse (reflectance), 3 dielectric (eta, roughness u/v remapped to
 * alpha = sqrt), 4 coated diffuse (dielectric coating eta / roughness over a
 * diffuse base of `reflectance`, clear layer of `thickness`, depth 10, one
 * sample), 5 conductor (conductor eta / k per channel, conductor roughness
 * as alpha), 6 coated conductor (the coating over a conductor of
 * `reflectance`, its roughness remapped).  Directions are in the shading
 * frame (z = normal). */
typedef struct orc_bsdf_params {
        int32_t type;
        float reflectance[3];
        float eta, roughness_u, roughness_v, thickness;
        float conductor_eta[3], conductor_k[3];
        float conductor_roughness_u, conductor_roughness_v;
} orc_bsdf_params;

void orc_bsdf_eval(const orc_bsdf_params *p, const float *wo, const float *wi, float *f, float *pdf);
/* Returns 1 for a valid sample (BsdfSample.isValid). */
int orc_bsdf_sample(const orc_bsdf_params *p, const float *wo, const float *u, float *f, float *wi, float *pdf);
int orc_bsdf_is_specular(const orc_bsdf_params *p);

/* --- sampling and interaction helpers (Sampler/Sampling.swift,
 * Core/Interaction.swift, Filter/GaussianFilter.swift) ------------------- */

float orc_power_heuristic(float f, float g);
void orc_concentric_disk(float u0, float u1, float *xy);
void orc_cosine_hemisphere(float u0, float u1, float *dir);
void orc_offset_origin(const float *p, const float *n, const float *dir, float *out);
/* Shadow-ray spawn toward a target: writes origin and direction, returns tHit. */
float orc_spawn_to(const float *from, const float *target, float *origin, float *dir);
float orc_gaussian(float x, float sigma);
void orc_gaussian_sample_1d(float u, float radius, float sigma, float *x, float *density);

/* --- environment light (Light/InfiniteLight.swift) ----------------------- */

/* Map rgb[h][w][3] (row v, column u); scale enters the light's power only. */
orc_env *orc_env_create(const float *rgb, int32_t w, int32_t h, float scale);
void orc_env_destroy(orc_env *env);
float orc_env_power(const orc_env *env);
/* Light sample for (u0, u1): writes direction and map value, returns the
 * solid-angle pdf (0: no sample). */
float orc_env_sample(const orc_env *env, float u0, float u1, float *dir, float *rgb);
float orc_env_pdf(const orc_env *env, const float *dir);
void orc_env_radiance(const orc_env *env, const float *dir, float *rgb);
void orc_env_tables(const orc_env *env, float *func, float *cdf, float *row_integral, float *marg_func,
                    float *marg_cdf, float *marg_integral);
void orc_env_lookup(const float *rgb, int32_t w, int32_t h, float u, float v, float *out);
void orc_equal_area_square_to_sphere(float u, float v, float *dir);
void orc_equal_area_sphere_to_square(const float *d, float *uv);

/* --- Z-Sobol ------------------------------------------------------------ */

/* Matrices: 1024 dims x 52 uint32 (SobolGenerator/main.swift:11-76 output). */
void orc_sobol_set_matrices(const uint32_t *m);
uint32_t orc_reverse_bits32(uint32_t v);
uint64_t orc_encode_morton2(uint32_t x, uint32_t y);
uint32_t orc_mix_bits(uint64_t v);
uint32_t orc_owen_scramble(uint32_t v, uint32_t seed);
int64_t orc_next_power_of_two(int64_t v);
float orc_sobol_sample(int64_t index, int dimension, uint32_t seed);

typedef struct orc_zsobol {
        int64_t seed;
        int32_t log2spp;
        int32_t n_base4_digits;
        uint64_t morton_index;
        int32_t dimension;
} orc_zsobol;
void orc_zsobol_init(orc_zsobol *s, int64_t spp, int32_t res_x, int32_t res_y, int64_t seed);
void orc_zsobol_start_pixel_sample(orc_zsobol *s, int32_t px, int32_t py, int64_t index, int32_t dim);
uint64_t orc_zsobol_sample_index(const orc_zsobol *s);
float orc_zsobol_get1d(orc_zsobol *s);
void orc_zsobol_get2d(orc_zsobol *s, float *out2);
void orc_zsobol_get3d(orc_zsobol *s, float *out3);
/* Batch: for each pixel-sample (px, py, index) the first `ndims` values drawn
 * by the sequence of get calls in `kinds` (1/2/3 per call), dim starting at 0. */
void orc_zsobol_batch(int64_t spp, int32_t res_x, int32_t res_y, int64_t seed, const int32_t *px,
                      const int32_t *py, const int64_t *index, int64_t n, const int32_t *kinds,
                      int32_t nkinds, float *out);

#ifdef __cplusplus
}
#endif
#endif
