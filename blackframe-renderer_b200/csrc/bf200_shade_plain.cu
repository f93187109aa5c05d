// Shading kernels of traces without ray cones or a light tree.
#include "bf200_kernels_body.cuh"

namespace bf200 {
template void launch_shading<false, false, false>(const SceneView&, const Wavefront&, const PathSource&,
                                             const TransportParams&, uint32_t, const AdjointView&, cudaStream_t);
}  // namespace bf200
