// Sobol sequence and Owen scrambling on the host: the library functions behind bf200_sobol_bits
// and bf200_owen_sobol_bits, and the leading direction bits the device sampler reads.
//
// Sobol points follow SobolSampling.cpp:51-117: dimension 0 is the van der Corput sequence, every
// other dimension takes its Joe-Kuo D6 primitive polynomial and initial direction numbers and
// extends them with the Bratley-Fox recurrence; a point is the XOR of the directions selected by
// the Gray code of the sample index. The Owen scramble is OwenScrambling.cpp:8-44.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "bf200.h"
#include "bf200_sobol.h"
#include "bf200_device.cuh"

namespace bf200 {
namespace {

// Joe-Kuo D6 parameters of dimensions 1..21200, three little-endian 64-bit words per dimension:
// the polynomial coefficient bits (degree - 1), then m_1 .. m_degree with m_k taking k bits.
const uint64_t kJoeKuo[kSobolDimensions - 1][3] = {
#include "bf200_sobol_table.inc"
};

// Exclusive end row of each polynomial degree 1..18 in the table.
constexpr uint32_t kDegreeRowEnd[18] = {1,   2,   4,    6,    12,   18,   36,    52,    100,
                                        160, 336, 480, 1110, 1866, 3666, 5714, 13424, 21200};

uint32_t degree_of_row(uint64_t row) {
    uint32_t degree = 1;
    while (row >= kDegreeRowEnd[degree - 1]) {
        ++degree;
    }
    return degree;
}

uint64_t field(const uint64_t* words, uint32_t offset, uint32_t width) {
    if (width == 0) {
        return 0;
    }
    const uint32_t word = offset / 64U, shift = offset % 64U;
    uint64_t v = words[word] >> shift;
    if (shift + width > 64U) {
        v |= words[word + 1] << (64U - shift);
    }
    return v & ((width == 64U ? 0ULL : (1ULL << width)) - 1ULL);
}

}  // namespace

void sobol_directions(uint64_t dimension, uint64_t (&v)[64]) {
    if (dimension == 0) {
        for (uint32_t j = 0; j < 64; ++j) {
            v[j] = 1ULL << (63U - j);
        }
        return;
    }
    const uint64_t row = dimension - 1;
    const uint32_t s = degree_of_row(row);
    const uint64_t* words = kJoeKuo[row];
    const uint64_t a = field(words, 0, s - 1);
    uint32_t offset = s - 1;
    for (uint32_t j = 0; j < s; ++j) {
        v[j] = field(words, offset, j + 1) << (63U - j);
        offset += j + 1;
    }
    for (uint32_t j = s; j < 64; ++j) {
        uint64_t d = v[j - s] ^ (v[j - s] >> s);
        for (uint32_t k = 1; k < s; ++k) {
            if ((a >> (s - 1U - k)) & 1U) {
                d ^= v[j - k];
            }
        }
        v[j] = d;
    }
}

uint64_t sobol_point(uint64_t sample_index, uint64_t dimension) {
    uint64_t v[64];
    sobol_directions(dimension, v);
    uint64_t gray = sample_index ^ (sample_index >> 1U);
    uint64_t point = 0;
    while (gray != 0) {
        point ^= v[__builtin_ctzll(gray)];
        gray &= gray - 1U;
    }
    return point;
}

const std::vector<uint32_t>& device_sobol_heads() {
    static std::once_flag once;
    static std::vector<uint32_t> heads;
    std::call_once(once, [] {
        heads.resize(static_cast<size_t>(kDeviceSobolDimensions) * 64U);
        for (uint32_t d = 0; d < kDeviceSobolDimensions; ++d) {
            uint64_t v[64];
            sobol_directions(d, v);
            for (uint32_t j = 0; j < 64; ++j) {
                heads[64ULL * d + j] = static_cast<uint32_t>(v[j] >> 32U);
            }
        }
    });
    return heads;
}

}  // namespace bf200

extern "C" {

BF200_EXPORT blackframe_status bf200_sobol_bits(uint64_t sample_index, uint64_t sobol_dimension,
                                                uint64_t* out_bits) noexcept {
    if (out_bits == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    if (sobol_dimension >= bf200::kSobolDimensions) {
        return BLACKFRAME_STATUS_OUT_OF_RANGE;
    }
    *out_bits = bf200::sobol_point(sample_index, sobol_dimension);
    return BLACKFRAME_STATUS_SUCCESS;
}

BF200_EXPORT blackframe_status bf200_owen_sobol_bits(const bf200_sample_index_v1* index, uint64_t sobol_dimension,
                                                     uint64_t* out_bits) noexcept {
    if (index == nullptr || out_bits == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    if (sobol_dimension >= bf200::kSobolDimensions) {
        return BLACKFRAME_STATUS_OUT_OF_RANGE;
    }
    const uint64_t point = bf200::sobol_point(index->sample_index, sobol_dimension);
    const uint64_t key = bf200::owen_tree_key(bf200::owen_pixel_hash(index->pixel_x, index->pixel_y), index->seed,
                                              sobol_dimension);
    *out_bits = bf200::owen_scramble(point, key, 64U);
    return BLACKFRAME_STATUS_SUCCESS;
}

}  // extern "C"
