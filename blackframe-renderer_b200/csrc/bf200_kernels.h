// Host-side launchers of the bf200 device kernels.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "bf200_device.cuh"

namespace bf200 {

cudaError_t launch_world_normals(const SceneView& s, uint32_t total, float4* out, uint32_t* failures,
                                 cudaStream_t stream);
// stage 0: k_regenerate; 1: k_trace; 2: route compaction, the per-route k_shade kernels, shadow
// compaction; 3: k_occlude. Adds the number of kernels launched to *launches. With `adjoint`, the
// shading and occlusion stages run as the path-replay adjoint's replay.
cudaError_t launch_stage(int stage, const SceneView& s, const Wavefront& w, const PathSource& src,
                         const TransportParams& p, uint32_t grid, cudaStream_t stream, uint32_t* launches,
                         const AdjointView* adjoint = nullptr);
// Stable compaction of n one-byte keys: the indices whose key is r < routes go to
// queue[offsets[r] .. offsets[r + 1]) in increasing order. tile_counts holds routes x
// ceil(n / kCompactTile) words of scratch. When total is given it receives the queue length; when
// reset_keys is given every one of its n bytes is set to kRouteNone. Three launches.
cudaError_t launch_compaction(const uint8_t* keys, uint32_t n, uint32_t routes, uint32_t* tile_counts,
                              uint32_t* queue, uint32_t* offsets, unsigned long long* total, uint8_t* reset_keys,
                              cudaStream_t stream, uint32_t* launches);
// Device BLAS build of one triangle geometry (bf200_lbvh.cu): a linear BVH whose BVH2 nodes (host
// builder format, node codes offset by node_base, leaf records by leaf_base) and leaf triangle
// records are appended to `nodes` and `leaf_tris`. Host arrays in; waits for the stream.
cudaError_t build_blas_lbvh(const float* positions, uint32_t vertex_count, const uint32_t* triangles, uint32_t n,
                            uint32_t node_base, uint32_t leaf_base, std::vector<BvhNode>& nodes,
                            std::vector<float4>& leaf_tris, cudaStream_t stream);
// Queues k_iteration_gate, which ends one iteration of a graph's device-side wavefront loop: it
// accumulates the shadow segments (counters[4]), counts iterations (counters[9]), clears the
// per-iteration counters and sets `loop` to continue until the wavefront drains or
// `max_iterations` is reached (then counters[10] = 1).
cudaError_t launch_gate(const Wavefront& w, uint64_t total, uint64_t max_iterations, cudaGraphConditionalHandle loop,
                        cudaStream_t stream);
// Retires the slots the last iteration finished (k_regenerate; nothing is left to claim).
cudaError_t launch_retire(const Wavefront& w, const PathSource& src, uint32_t grid, cudaStream_t stream);
cudaError_t launch_film(const float4* path_radiance, uint32_t pixels, uint32_t samples, const float* response12,
                        const float* pdf4, float normalization, uint32_t precision, float4* film32, double* film64,
                        unsigned long long* counts, unsigned long long* skipped, cudaStream_t stream);
// Per-pixel adjoint of the path-replay adjoint, from a target image (the loss, the sum of squared
// rgb differences, is added to *loss) or, with target null, from the caller's dLoss/d(image).
cudaError_t launch_adjoint_image(const float4* film32, const double* film64, const float* target,
                                 const float* image_adjoint, uint32_t pixels, uint32_t precision, float4* pixel_adjoint,
                                 double* loss, cudaStream_t stream);
cudaError_t launch_queries(const SceneView& s, const bf200_ray_v1* rays, uint64_t n, bf200_hit_v1* hits,
                           uint32_t* occluded, cudaStream_t stream);

// Primary rays of (pixel, sample) records through the camera of `src` (k_camera_rays): one ray and
// one lane status per record.
cudaError_t launch_camera_rays(const PathSource& src, const bf200_sample_index_v1* samples, uint64_t n,
                               bf200_ray_v1* rays, uint32_t* status, cudaStream_t stream);
// Environment-map light batches (bf200_envmap.cu).
struct EnvironmentView;
cudaError_t launch_environment_sample(const EnvironmentView& v, const float2* canonical, uint64_t n,
                                      bf200_environment_sample_v1* out, cudaStream_t stream);
cudaError_t launch_environment_pdf(const EnvironmentView& v, const float* directions, uint64_t n, float* pdf,
                                   uint32_t* status, cudaStream_t stream);
cudaError_t launch_environment_le(const EnvironmentView& v, const float* directions, uint64_t n, float4* radiance,
                                  uint32_t* status, cudaStream_t stream);

}  // namespace bf200
