/*
 * gzg_host.h - host-side helpers of libgzg.so that stand in for the parts of the
 * Gonzales Swift host this library's own harness needs: the SAH BVH2 build and
 * the triangle bounds that feed it.  A Swift integration keeps using its own
 * BoundingHierarchyBuilder and does not need these.
 */
#ifndef GZG_HOST_H
#define GZG_HOST_H

#include "gzg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Triangle bounds as Triangle.worldBound computes them
 * (Shape/Triangle.swift:248-256: union(Bounds3f(p0, p1), p2)).
 * points4: float4 per vertex; vertex_indices: 3 per triangle;
 * bounds6 out: minx,miny,minz,maxx,maxy,maxz per triangle. */
GZG_API gzg_status gzg_host_triangle_bounds(const float *points4, const int64_t *vertex_indices,
                                            int64_t triangle_count, float *bounds6);

/* Binned-SAH BVH2 build and depth-first flatten, replacing
 * BoundingHierarchyBuilder (Accelerators/BoundingHierarchyBuilder.swift:66-339):
 * 12 buckets on the centroid's widest axis, cost 0.5 + sum(count*SA)/SA,
 * at most 4 prims per SAH leaf, Swift partition order, left child = i+1.
 * nodes_out needs room for 2*prim_count nodes; order_out[k] = input index of
 * the k-th prim in leaf order (the sortedPrimitives of
 * BoundingHierarchyBuilder.swift:102-107).  threads <= 0: all cores. */
GZG_API gzg_status gzg_host_build_bvh2(const float *bounds6, int64_t prim_count,
                                       gzg_bvh2_node *nodes_out, int64_t *node_count_out,
                                       int64_t *order_out, int32_t threads);

#ifdef __cplusplus
}
#endif
#endif
