// Host-side Sobol directions (bf200_sobol.cu).
#pragma once

#include <cstdint>
#include <vector>

namespace bf200 {

// The 64 direction numbers of one Sobol dimension (0 .. 21200).
void sobol_directions(uint64_t dimension, uint64_t (&v)[64]);
// The 64-bit Sobol coordinate of a sample index.
uint64_t sobol_point(uint64_t sample_index, uint64_t dimension);
// Leading 32 bits of the 64 directions of Sobol dimensions 0 .. kDeviceSobolDimensions - 1, in
// dimension-major order: the table the device sampler reads.
const std::vector<uint32_t>& device_sobol_heads();

}  // namespace bf200
