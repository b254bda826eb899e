// gzg_internal.h - shared declarations of libgzg's translation units.
#pragma once

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gzg.h"
#include "../../include/gzg_host.h"

namespace gzg {

// Thread-local last error (gzg_last_error).
gzg_status set_error(gzg_status code, const std::string &msg);
gzg_status clear_error();

// GZG_ERR_KERNEL_FAULT with the bits of a nonzero device error word decoded
// (stack overflow, step cap, index out of range) into the message.
gzg_status kernel_fault(uint32_t word);

// Host wait for the work queued so far on `stream` (a cudaStream_t; NULL =
// the legacy default stream): polls an event with cudaEventQuery, yielding
// between polls, for at most the wait limit, GZG_WAIT_LIMIT_US in the
// environment (microseconds; default 300 s; 0 = no limit).  GZG_ERR_TIMEOUT
// when the limit runs out: the queued work keeps running, so the caller must
// leave its buffers to it.
gzg_status wait_stream(void *stream, const char *what);

// ------------------------------------------------------------------ layouts

// Wide node: 8 children, 80 bytes, fetched as five 16-byte loads.
//   bytes  0-11  origin p (float x3) of the quantisation grid
//   bytes 12-14  per-axis exponent e (biased like IEEE binary32: step = 2^(e-127))
//   byte  15     imask: bit s set when child slot s is an interior node
//   bytes 16-19  child_base: node index of the first interior child; interior
//                children are stored contiguously in slot order
//   bytes 20-23  tri_base: first triangle record of this node's leaf children
//   bytes 24-31  meta[s]: 0 = empty or interior; leaf = 0x80 | (count-1) << 5 | offset,
//                triangles tri_base+offset .. +count-1 (count <= 4, offset < 32)
//   bytes 32-79  qlo_x[8] qlo_y[8] qlo_z[8] qhi_x[8] qhi_y[8] qhi_z[8]:
//                child box = p + q * 2^(e-127), rounded outward at build time
// Slot s holds the child lying farthest toward the octant whose sign bits are
// s (bit set = positive side), so a ray visits slots in the order key = s ^ oct
// (oct = sign bits of the direction) to go roughly front to back.
struct alignas(16) WideNode {
        float px, py, pz;
        uint8_t ex, ey, ez, imask;
        uint32_t child_base;
        uint32_t tri_base;
        uint8_t meta[8];
        uint8_t qlo[3][8];
        uint8_t qhi[3][8];
};
static_assert(sizeof(WideNode) == 80, "wide node must be 80 bytes");

// Triangle records in leaf order: three float4 streams (v0, v1, v2); v0.w holds
// the prim index (into the uploaded prim-id array) as int32 bits.
struct float4_ {
        float x, y, z, w;
};

struct WideBvh {
        std::vector<WideNode> nodes;
        std::vector<float4_> v0, v1, v2;
        int32_t depth = 0;
};

// Host copies of a scene's shading arrays, as uploaded (see DevScene).
struct HostShading {
        std::vector<float4_> pv0, pv1, pv2;  // triangles in prim order
        std::vector<gzg_prim_id> prims;
        std::vector<float4_> materials;      // 2 per material
        // per material 3 records (gzg_material_params: eta, roughness u, v,
        // thickness; conductor eta, roughness u; conductor k, roughness v);
        // empty when none were set
        std::vector<float4_> mat_params;
        // per prim 5 records of vertex normals and UVs (DevScene::attr); empty
        // when none were set
        std::vector<float4_> attr;
        std::vector<float4_> lights;         // 4 per light
        std::vector<float> light_cdf;
        float light_total = 0.0f;
        // homogeneous medium box (gzg_medium), when set
        bool has_medium = false;
        gzg_medium medium{};
        // environment light, after the area lights in the light list
        bool has_env = false;
        float env_power = 0.0f;
        float light_total_env = 0.0f;  // light_total + env_power
};

// A wide tree built on the device (gpu_build.cu): device arrays the caller
// takes ownership of (cudaFree), in the WideBvh layout.
struct GpuWide {
        void *nodes = nullptr;                      // node_count WideNode records
        void *tv0 = nullptr, *tv1 = nullptr, *tv2 = nullptr;  // tri_count leaf-order records
        uint32_t node_count = 0, tri_count = 0;
        int32_t depth = 0;
};

// Builds the wide tree over device prim-order triangles pv0/pv1/pv2 (pv0.w =
// int 1 for prims the traversal tests) with at most leaf_size (1..4) prims
// per leaf, by builder (GZG_BUILD_*) with the PLOC radius; device_ms = the
// build's device time.  On an error the arrays already allocated are in *out.
gzg_status gpu_build_wide(const float4_ *pv0, const float4_ *pv1, const float4_ *pv2, int64_t n, int leaf_size,
                          int builder, int radius, GpuWide *out, float *device_ms);

// Device expansion of packed meshes (gpu_build.cu): per mesh its first
// vertex and triangle in the concatenated arrays, counts, material and,
// for an area-light mesh, the light index of its first triangle (else -1).
struct MeshRange {
        int64_t vert_off, tri_off, vcount, tcount, material;
        int64_t light_base;
};
// points3 / idx3: concatenated packed arrays on the device; writes points4
// (x, y, z, 0), vidx64, prims (PrimId_C) and pv0/pv1/pv2 (pv0.w = int 1).
// Sets *bad when an index is out of range (that triangle is left inert).
gzg_status gpu_expand_meshes(const float *points3, const int32_t *idx3, const MeshRange *ranges_dev, int mesh_count,
                             int64_t total_verts, int64_t total_tris, float *points4, int64_t *vidx64,
                             gzg_prim_id *prims, float4_ *pv0, float4_ *pv1, float4_ *pv2, bool *bad);

// Writes the attribute records (DevScene::attr) of the prims of one mesh from
// device arrays of per-vertex normals (x3) and UVs (x2), either may be null.
gzg_status gpu_gather_attributes(const gzg_prim_id *prims, int64_t n, const gzg_triangle_mesh *meshes_dev,
                                 int64_t mesh, const float *normals, const float *uvs, int64_t vcount,
                                 float4_ *attr);

// Converts a validated reference BVH2 + prims + meshes into the wide layout.
// Returns GZG_OK or an error (with set_error called).
gzg_status build_wide_bvh(const gzg_bvh2_node *nodes, int64_t node_count, const gzg_prim_id *prims,
                          int64_t prim_count, const gzg_triangle_mesh *meshes, int64_t mesh_count,
                          const int64_t *points_counts, const int64_t *vertex_index_counts, WideBvh *out,
                          int32_t *bvh2_depth);

#ifdef __CUDACC__
#define GZG_HOST_DEVICE __host__ __device__
#else
#define GZG_HOST_DEVICE
#endif

// Environment light tables (env.cpp): kEnvDistSize x kEnvDistSize
// piecewise-constant distribution over the equal-area square.
constexpr int kEnvDistSize = 1024;
struct EnvTables {
        std::vector<float> func, cdf, row_integral, marg_func, marg_cdf;
        float marg_integral = 0.0f;
};
void build_env_tables(const float *rgb, int w, int h, EnvTables *t);
void env_lookup_host(const float *rgb, int w, int h, float u, float v, float *out);

// Host copies kept by an uploaded scene (batch assembly).
const WideBvh &scene_host_wide(const gzg_scene *scene);
const HostShading &scene_host_shading(const gzg_scene *scene);
bool scene_is_instanced(const gzg_scene *scene);

// Converts a top-level BVH2 whose leaf prim k is instance leaf_instance[k]
// (world bounds in inst_bounds, 6 floats per instance) into the wide layout;
// its leaf records are instance entries (v0.w = -(instance + 1)).
gzg_status build_wide_tlas(const gzg_bvh2_node *nodes, int64_t node_count, const int64_t *leaf_instance,
                           int64_t leaf_count, const float *inst_bounds, int64_t inst_count, WideBvh *out,
                           int32_t *bvh2_depth);

// Decodes PrimId_C to (mesh, first vertex-index slot) as kernel.mojo:270-279;
// returns false for prims the reference never intersects.
GZG_HOST_DEVICE inline bool prim_triangle(const gzg_prim_id &p, int64_t *mesh, int64_t *base) {
        if (p.type == 0) {
                *mesh = p.id1;
                *base = p.id2;
                return true;
        }
        if (p.type == 1 || p.type == 2 || p.type == 3) {
                if (p.id2 == -1) return false;
                *mesh = p.id2 >> 32;
                *base = (p.id2 & 0xFFFFFFFFll) * 3;
                return true;
        }
        return false;
}

}  // namespace gzg
