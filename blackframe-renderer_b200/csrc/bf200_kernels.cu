// The wavefront's kernels and host-side launchers (bf200_kernels_body.cuh), except the shading
// kernels, which bf200_shade_*.cu instantiate.
#define BF200_KERNELS_MAIN_TU
#include "bf200_kernels_body.cuh"
