// Shading kernels of traces that carry ray cones.
#include "bf200_kernels_body.cuh"

namespace bf200 {
template void launch_shading<false, true, false>(const SceneView&, const Wavefront&, const PathSource&,
                                             const TransportParams&, uint32_t, const AdjointView&, cudaStream_t);
}  // namespace bf200
