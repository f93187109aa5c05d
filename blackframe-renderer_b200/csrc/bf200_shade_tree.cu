// Shading kernels of traces of scenes that select lights by the spatial tree.
#include "bf200_kernels_body.cuh"

namespace bf200 {
template void launch_shading<false, false, true>(const SceneView&, const Wavefront&, const PathSource&,
                                             const TransportParams&, uint32_t, const AdjointView&, cudaStream_t);
}  // namespace bf200
