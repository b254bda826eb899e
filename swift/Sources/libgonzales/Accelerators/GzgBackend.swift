import gzg
import mojoKernel

/// libgzg.so (the B200 traversal and wavefront library) behind Gonzales'
/// accelerator: the replacement of the GPU half of the native plugin.
///
/// Every record of the plugin's C header (Ray_C, Intersection_C,
/// PathState_C, PrimId_C, BVH2Node, TriangleMesh_C, Material_C) has the same
/// byte layout as its gzg_* counterpart, so the arrays Gonzales already
/// builds are passed by rebinding their memory; nothing is converted.
///
/// A GzgScene may be used from every tile task at once: each batch call
/// takes its own staging buffers.  Every call reports failure through its
/// status; `lastError` holds the message of the calling thread's last one.
///
/// Where it plugs in:
///   - SceneDescription, when `--gpu` is given: `GzgScene.isAvailable`
///     decides, as mojo_gpu_available does today.
///   - BoundingHierarchy.uploadToGPU: build the scene with `GzgScene(...)`
///     from the same arrays it hands to mojo_gpu_upload_scene, keep it where
///     gpuSceneHandle is kept (released with the hierarchy).
///   - BoundingHierarchy.intersectGPU / intersectBatchGPU: `intersect(...)`
///     in place of mojo_gpu_traverse_batch.
///   - Tile.render's shading step: `shade(...)` in place of
///     mojo_gpu_shade_batch.
///   - Visibility.occluded for batches of shadow rays: `occluded(...)`.
///   - Or the whole tile loop on the device: `render(...)` (the wavefront
///     integrator, gzg_render_image) returning the film sums Film.add
///     would accumulate.
final class GzgScene: @unchecked Sendable {

        let handle: OpaquePointer

        static var isAvailable: Bool { gzg_gpu_available() }

        static var lastError: String { String(cString: gzg_last_error()) }

        /// Uploads a scene from the arrays of BoundingHierarchy.uploadToGPU.
        /// The counts are element counts per mesh (floats of the float4
        /// points, int64 face and vertex indices).  Returns nil on failure
        /// (see lastError), where mojo_gpu_upload_scene returned a null handle.
        init?(
                nodes: UnsafeRawPointer, nodeCount: Int,
                primIds: UnsafeRawPointer, primCount: Int,
                meshes: UnsafeBufferPointer<TriangleMesh_C>,
                pointsCounts: [Int64], faceIndicesCounts: [Int64], vertexIndicesCounts: [Int64],
                materials: [Material_C]
        ) {
                var out: OpaquePointer? = nil
                let status = pointsCounts.withUnsafeBufferPointer { pts in
                        faceIndicesCounts.withUnsafeBufferPointer { fis in
                                vertexIndicesCounts.withUnsafeBufferPointer { vis in
                                        materials.withUnsafeBytes { mats in
                                                UnsafeRawPointer(meshes.baseAddress!).withMemoryRebound(
                                                        to: gzg_triangle_mesh.self, capacity: meshes.count
                                                ) { meshPtr in
                                                        gzg_gpu_upload_scene(
                                                                nodes.assumingMemoryBound(to: gzg_bvh2_node.self),
                                                                Int64(nodeCount),
                                                                primIds.assumingMemoryBound(to: gzg_prim_id.self),
                                                                Int64(primCount),
                                                                meshPtr, Int64(meshes.count),
                                                                pts.baseAddress, fis.baseAddress, vis.baseAddress,
                                                                mats.baseAddress?.assumingMemoryBound(
                                                                        to: gzg_material.self),
                                                                Int64(materials.count),
                                                                &out)
                                                }
                                        }
                                }
                        }
                }
                guard status == 0, let scene = out else { return nil }
                handle = scene
        }

        deinit {
                gzg_gpu_free_scene(handle)
        }

        /// Closest hits of `rays` within their tMax values into `results`
        /// (gzg_gpu_traverse_batch).  Misses are written as the plugin writes
        /// them (hit = 0, primId = {-1, -1}, tHit = tMax).
        @discardableResult
        func intersect(
                rays: UnsafeBufferPointer<Ray_C>, tMax: UnsafeBufferPointer<Float>,
                results: UnsafeMutableBufferPointer<Intersection_C>
        ) -> Bool {
                precondition(rays.count == tMax.count && results.count >= rays.count)
                return UnsafeRawPointer(rays.baseAddress!).withMemoryRebound(
                        to: gzg_ray.self, capacity: rays.count
                ) { r in
                        UnsafeMutableRawPointer(results.baseAddress!).withMemoryRebound(
                                to: gzg_intersection.self, capacity: rays.count
                        ) { out in
                                gzg_gpu_traverse_batch(handle, r, tMax.baseAddress, Int64(rays.count), out, nil) == 0
                        }
                }
        }

        /// One shading step of the tile loop on `paths` (gzg_gpu_shade_batch):
        /// emission ends a path, diffuse hits bounce, misses end the path.
        @discardableResult
        func shade(
                paths: UnsafeMutableBufferPointer<PathState_C>,
                intersections: UnsafeBufferPointer<Intersection_C>
        ) -> Bool {
                precondition(intersections.count >= paths.count)
                return UnsafeMutableRawPointer(paths.baseAddress!).withMemoryRebound(
                        to: gzg_path_state.self, capacity: paths.count
                ) { p in
                        UnsafeRawPointer(intersections.baseAddress!).withMemoryRebound(
                                to: gzg_intersection.self, capacity: paths.count
                        ) { hits in
                                gzg_gpu_shade_batch(handle, p, Int64(paths.count), hits) == 0
                        }
                }
        }

        /// Shadow queries (gzg_gpu_occluded_batch): occluded[i] = 1 when some
        /// triangle lies within (0, tMax[i]] along rays[i].
        @discardableResult
        func occluded(
                rays: UnsafeBufferPointer<Ray_C>, tMax: UnsafeBufferPointer<Float>,
                occluded: UnsafeMutableBufferPointer<UInt8>
        ) -> Bool {
                precondition(rays.count == tMax.count && occluded.count >= rays.count)
                return UnsafeRawPointer(rays.baseAddress!).withMemoryRebound(
                        to: gzg_ray.self, capacity: rays.count
                ) { r in
                        gzg_gpu_occluded_batch(
                                handle, r, tMax.baseAddress, Int64(rays.count), occluded.baseAddress, nil) == 0
                }
        }

        /// The whole frame on the device (gzg_render_image): per pixel, row
        /// major, the sums of sample light (3 floats) and of sample weight
        /// that Film.add accumulates; the image is light / weight
        /// (Pixel.normalized).  nil on failure.
        func render(parameters: gzg_render_params) -> (light: [Float], weight: [Float])? {
                var params = parameters
                let pixels = Int(params.width) * Int(params.height)
                var light = [Float](repeating: 0, count: 3 * pixels)
                var weight = [Float](repeating: 0, count: pixels)
                let status = light.withUnsafeMutableBufferPointer { l in
                        weight.withUnsafeMutableBufferPointer { w in
                                gzg_render_image(handle, &params, l.baseAddress, nil, w.baseAddress, nil)
                        }
                }
                return status == 0 ? (light, weight) : nil
        }
}
