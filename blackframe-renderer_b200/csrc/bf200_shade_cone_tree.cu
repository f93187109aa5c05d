// Shading kernels of cone-carrying traces of tree-selecting scenes.
#include "bf200_kernels_body.cuh"

namespace bf200 {
template void launch_shading<false, true, true>(const SceneView&, const Wavefront&, const PathSource&,
                                             const TransportParams&, uint32_t, const AdjointView&, cudaStream_t);
}  // namespace bf200
