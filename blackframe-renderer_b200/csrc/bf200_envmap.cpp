// Host construction of the environment-map light (EnvironmentLights.hpp:468-733) and its power
// (:853-885), in float with every operation in the reference's order: the tables it builds are the
// reference's, value for value, so the device's sampling and lookups can be compared bit for bit.
// The file is compiled with floating-point contraction off.
#include "bf200_envmap.h"
#include "bf200_records.h"

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <limits>

namespace bf200 {
namespace {

constexpr float kPi = 3.14159265358979323846F;  // std::numbers::pi_v<float>
constexpr float kVisibleMin = 360.0F, kVisibleMax = 830.0F;

// std::midpoint of two floats of moderate magnitude (all partition boundaries here).
float midpoint(float a, float b) {
    constexpr float lo = std::numeric_limits<float>::min() * 2.0F;
    constexpr float hi = std::numeric_limits<float>::max() / 2.0F;
    const float abs_a = a < 0.0F ? -a : a, abs_b = b < 0.0F ? -b : b;
    if (abs_a <= hi && abs_b <= hi) {
        return (a + b) / 2.0F;
    }
    if (abs_a < lo) {
        return a + b / 2.0F;
    }
    if (abs_b < lo) {
        return a / 2.0F + b;
    }
    return a / 2.0F + b / 2.0F;
}

// representable_open_interval (:51-57).
bool open_interval(float lower, float upper) {
    if (!std::isfinite(lower) || !std::isfinite(upper) || !(lower < upper)) {
        return false;
    }
    const float m = midpoint(lower, upper);
    return m > lower && m < upper;
}

// add_compensated (:123-142).
bool add_compensated(float value, float& sum, float& correction) {
    if (!std::isfinite(value) || value < 0.0F) {
        return false;
    }
    const float next = sum + value;
    if (!std::isfinite(next)) {
        return false;
    }
    if (sum >= value) {
        correction += (sum - next) + value;
    } else {
        correction += (value - next) + sum;
    }
    if (!std::isfinite(correction)) {
        return false;
    }
    sum = next;
    return true;
}

// compensated_sum (:144-159): false when the sum is not representable.
bool compensated_sum(const float* values, size_t n, float& total) {
    float sum = 0.0F, correction = 0.0F;
    for (size_t i = 0; i < n; ++i) {
        if (!add_compensated(values[i], sum, correction)) {
            return false;
        }
    }
    total = sum + correction;
    if (!std::isfinite(total) || total < 0.0F) {
        return false;
    }
    if (total == 0.0F) {
        total = 0.0F;
    }
    return true;
}

// build_cdf (:161-219): returns -1 on error, 0 for an all-zero weight set, 1 for a CDF.
int build_cdf(const float* weights, float* cdf, size_t n) {
    if (n == 0) {
        return -1;
    }
    float total = 0.0F;
    if (!compensated_sum(weights, n, total)) {
        return -1;
    }
    if (total == 0.0F) {
        std::fill(cdf, cdf + n, 0.0F);
        return 0;
    }
    size_t last_positive = n;
    for (size_t index = n; index > 0; --index) {
        if (weights[index - 1] > 0.0F) {
            last_positive = index - 1;
            break;
        }
    }
    if (last_positive == n) {
        return -1;
    }
    float cumulative = 0.0F;
    for (size_t index = 0; index < n; ++index) {
        const float weight = weights[index];
        if (!std::isfinite(weight) || weight < 0.0F) {
            return -1;
        }
        if (weight == 0.0F) {
            cdf[index] = cumulative;
            continue;
        }
        const float probability = weight / total;
        const float candidate = cumulative + probability;
        if (!std::isfinite(probability) || !(probability > 0.0F) || !std::isfinite(candidate) ||
            !(candidate > cumulative)) {
            return -1;
        }
        float next = 1.0F;
        if (index != last_positive) {
            if (!(candidate < 1.0F)) {
                return -1;
            }
            next = candidate;
        }
        cdf[index] = next;
        cumulative = next;
    }
    return cdf[n - 1] == 1.0F ? 1 : -1;
}

int invalid(const char*& message, const char* text) {
    message = text;
    return kEnvironmentInvalid;
}

}  // namespace

int build_environment_tables(uint32_t width, uint32_t height, const float* texels, const float nanometers[4],
                             const float quaternion[4], EnvironmentTables& out, const char*& message) {
    message = nullptr;
    // checked_texel_count (:59-95); float indexes exactly up to 2^24
    if (width == 0U || height == 0U) {
        return invalid(message, "An environment map requires non-zero width and height.");
    }
    if (width > (1U << 24) || height > (1U << 24)) {
        return invalid(message, "Environment-map dimensions are not exactly indexable in the requested precision.");
    }
    const uint64_t count = static_cast<uint64_t>(width) * height;
    if (texels == nullptr) {
        return invalid(message, "Environment-map dimensions must match the row-major texel count exactly.");
    }
    // validate_light_wavelength_packet (PacketLightSpectrum.hpp:11-25): the nanometers part
    for (int lane = 0; lane < 4; ++lane) {
        if (!std::isfinite(nanometers[lane]) || nanometers[lane] < kVisibleMin || nanometers[lane] > kVisibleMax) {
            return invalid(message,
                           "Packet-bound lights require finite visible wavelengths with positive wavelength densities.");
        }
    }
    // AffineTransformT::rotation (Transforms.hpp:45-52): rotation_matrix, then from_matrix's inverse
    const float qx = quaternion[0], qy = quaternion[1], qz = quaternion[2], qw = quaternion[3];
    const float squared_length = qx * qx + qy * qy + qz * qz + qw * qw;
    const float unit_tolerance = std::numeric_limits<float>::epsilon() * 32.0F;
    if (!std::isfinite(qx) || !std::isfinite(qy) || !std::isfinite(qz) || !std::isfinite(qw) ||
        !std::isfinite(squared_length) || std::abs(squared_length - 1.0F) > unit_tolerance) {
        return invalid(message, "A rotation quaternion must be finite and normalized.");
    }
    const float xx = qx * qx, yy = qy * qy, zz = qz * qz;
    const float xy = qx * qy, xz = qx * qz, yz = qy * qz;
    const float wx = qw * qx, wy = qw * qy, wz = qw * qz;
    float m[16] = {1.0F, 0.0F, 0.0F, 0.0F, 0.0F, 1.0F, 0.0F, 0.0F, 0.0F, 0.0F, 1.0F, 0.0F, 0.0F, 0.0F, 0.0F, 1.0F};
    m[0] = 1.0F - 2.0F * (yy + zz);
    m[1] = 2.0F * (xy - wz);
    m[2] = 2.0F * (xz + wy);
    m[4] = 2.0F * (xy + wz);
    m[5] = 1.0F - 2.0F * (xx + zz);
    m[6] = 2.0F * (yz - wx);
    m[8] = 2.0F * (xz - wy);
    m[9] = 2.0F * (yz + wx);
    m[10] = 1.0F - 2.0F * (xx + yy);
    float inv[16];
    if (!invert_matrix4(m, inv)) {
        return invalid(message, "A singular matrix has no inverse.");
    }

    float global_peak = 0.0F;
    for (uint64_t i = 0; i < count * 4; ++i) {
        const float v = texels[i];
        if (!std::isfinite(v) || v < 0.0F) {
            return invalid(message, "Environment-map texels require finite non-negative spectral lanes.");
        }
        global_peak = std::max(global_peak, v);
    }

    const float theta_step = kPi / static_cast<float>(height);
    const float azimuth_step = (2.0F * kPi) / static_cast<float>(width);
    if (!std::isfinite(theta_step) || !(theta_step > 0.0F) || !std::isfinite(azimuth_step) ||
        !(azimuth_step > 0.0F)) {
        return invalid(message, "Environment-map angular resolution is not representable.");
    }

    EnvironmentTables t;
    t.width = width;
    t.height = height;
    t.texels.assign(texels, texels + count * 4);
    for (int lane = 0; lane < 4; ++lane) {
        t.nanometers[lane] = nanometers[lane];
        t.quaternion[lane] = quaternion[lane];
    }
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) {
            t.matrix[r * 3 + c] = m[r * 4 + c];
            t.inverse[r * 3 + c] = inv[r * 4 + c];
        }
    }
    t.azimuth.resize(static_cast<size_t>(width) + 1);
    t.cosine.resize(static_cast<size_t>(height) + 1);
    t.row_cdf.assign(height, 0.0F);
    t.column_cdfs.assign(count, 0.0F);
    t.density.assign(count, 0.0F);
    std::vector<float> azimuth_spans(width), cosine_spans(height), column_weights(width), row_weights(height),
        importances(count, 0.0F);

    const float full_azimuth = 2.0F * kPi;
    t.azimuth[0] = 0.0F;
    for (uint32_t column = 1; column < width; ++column) {
        const float boundary = static_cast<float>(column) * azimuth_step;
        if (!(boundary < full_azimuth) || !open_interval(t.azimuth[column - 1], boundary)) {
            return invalid(message, "Environment-map azimuth bins are not individually representable.");
        }
        t.azimuth[column] = boundary;
    }
    t.azimuth[width] = full_azimuth;
    if (!open_interval(t.azimuth[width - 1], full_azimuth)) {
        return invalid(message, "Environment-map azimuth bins are not individually representable.");
    }
    for (uint32_t column = 0; column < width; ++column) {
        azimuth_spans[column] = t.azimuth[column + 1] - t.azimuth[column];
    }
    t.cosine[0] = 1.0F;
    for (uint32_t row = 1; row < height; ++row) {
        const float boundary = std::cos(static_cast<float>(row) * theta_step);
        if (!open_interval(boundary, t.cosine[row - 1])) {
            return invalid(message, "Environment-map polar bins are not individually representable.");
        }
        t.cosine[row] = boundary;
    }
    t.cosine[height] = -1.0F;
    if (!open_interval(-1.0F, t.cosine[height - 1])) {
        return invalid(message, "Environment-map polar bins are not individually representable.");
    }
    for (uint32_t row = 0; row < height; ++row) {
        cosine_spans[row] = t.cosine[row] - t.cosine[row + 1];
    }

    if (global_peak > 0.0F) {
        for (uint64_t index = 0; index < count; ++index) {
            float ratios[4];
            for (int lane = 0; lane < 4; ++lane) {
                ratios[lane] = texels[index * 4 + lane] / global_peak;
                if (texels[index * 4 + lane] > 0.0F && !(ratios[lane] > 0.0F)) {
                    return invalid(message, "Environment-map spectral importance is not representable.");
                }
            }
            float ratio_sum = 0.0F;
            if (!compensated_sum(ratios, 4, ratio_sum)) {
                return invalid(message, "Environment-map spectral importance is not representable.");
            }
            const float importance = ratio_sum / 4.0F;
            if ((ratio_sum > 0.0F && !(importance > 0.0F)) || !std::isfinite(importance)) {
                return invalid(message, "Environment-map spectral importance is not representable.");
            }
            importances[index] = importance;
        }
        for (uint32_t row = 0; row < height; ++row) {
            for (uint32_t column = 0; column < width; ++column) {
                const uint64_t index = static_cast<uint64_t>(row) * width + column;
                column_weights[column] = importances[index] * azimuth_spans[column];
                if (importances[index] > 0.0F &&
                    (!std::isfinite(column_weights[column]) || !(column_weights[column] > 0.0F))) {
                    return invalid(message, "Environment-map texel probability is not representable.");
                }
            }
            float row_sum = 0.0F;
            if (!compensated_sum(column_weights.data(), width, row_sum)) {
                return invalid(message, "Environment-map row importance is not representable.");
            }
            row_weights[row] = row_sum * cosine_spans[row];
            if (row_sum > 0.0F && (!std::isfinite(row_weights[row]) || !(row_weights[row] > 0.0F))) {
                return invalid(message, "Environment-map row probability is not representable.");
            }
            const int built = build_cdf(column_weights.data(), t.column_cdfs.data() + static_cast<uint64_t>(row) * width,
                                        width);
            if (built < 0) {
                return invalid(message, "Environment-map conditional CDF is not representable.");
            }
            if ((row_sum > 0.0F) != (built == 1)) {
                return invalid(message, "Environment-map conditional CDF lost positive support.");
            }
        }
        const int rows_built = build_cdf(row_weights.data(), t.row_cdf.data(), height);
        if (rows_built < 0) {
            return invalid(message, "Environment-map marginal CDF is not representable.");
        }
        if (rows_built == 0) {
            return invalid(message, "A non-black environment map requires a positive sampling distribution.");
        }
        for (uint32_t row = 0; row < height; ++row) {
            const float row_previous = row == 0 ? 0.0F : t.row_cdf[row - 1];
            const float row_probability = t.row_cdf[row] - row_previous;
            for (uint32_t column = 0; column < width; ++column) {
                const uint64_t index = static_cast<uint64_t>(row) * width + column;
                if (importances[index] == 0.0F) {
                    t.density[index] = 0.0F;
                    continue;
                }
                const float column_previous = column == 0 ? 0.0F : t.column_cdfs[index - 1];
                const float column_probability = t.column_cdfs[index] - column_previous;
                const float texel_probability = row_probability * column_probability;
                const float solid_angle = cosine_spans[row] * azimuth_spans[column];
                const float density = texel_probability / solid_angle;
                if (!std::isfinite(row_probability) || !(row_probability > 0.0F) ||
                    !std::isfinite(column_probability) || !(column_probability > 0.0F) ||
                    !std::isfinite(texel_probability) || !(texel_probability > 0.0F) || !std::isfinite(solid_angle) ||
                    !(solid_angle > 0.0F) || !std::isfinite(density) || !(density > 0.0F)) {
                    return invalid(message, "Environment-map directional PDF is not representable.");
                }
                t.density[index] = density;
            }
        }
    }

    for (int lane = 0; lane < 4; ++lane) {
        float lane_peak = 0.0F;
        for (uint64_t index = 0; index < count; ++index) {
            lane_peak = std::max(lane_peak, texels[index * 4 + lane]);
        }
        t.lane_peak[lane] = lane_peak;
        if (lane_peak == 0.0F) {
            continue;
        }
        float sum = 0.0F, correction = 0.0F;
        for (uint32_t row = 0; row < height; ++row) {
            for (uint32_t column = 0; column < width; ++column) {
                const uint64_t index = static_cast<uint64_t>(row) * width + column;
                const float normalized = texels[index * 4 + lane] / lane_peak;
                const float solid_angle = cosine_spans[row] * azimuth_spans[column];
                const float contribution = normalized * solid_angle;
                if (texels[index * 4 + lane] > 0.0F && (!(normalized > 0.0F) || !std::isfinite(solid_angle) ||
                                                        !(solid_angle > 0.0F) || !(contribution > 0.0F))) {
                    return invalid(message, "Environment-map spectral integral is not representable.");
                }
                if (!add_compensated(contribution, sum, correction)) {
                    return invalid(message, "Environment-map spectral integral is not representable.");
                }
            }
        }
        const float integral = sum + correction;
        if (!std::isfinite(integral) || !(integral > 0.0F)) {
            return invalid(message, "Environment-map spectral integral is not representable.");
        }
        t.lane_integral[lane] = integral;
    }
    t.black = global_peak == 0.0F;
    out = std::move(t);
    return kEnvironmentOk;
}

namespace {

struct HalfExtent {
    float fraction;
    int exponent;
    bool zero;
};

// binary_half_extent (:322-351).
bool half_extent(float lower, float upper, HalfExtent& out) {
    if (lower == upper) {
        out = HalfExtent{0.0F, 0, true};
        return true;
    }
    const float full = upper - lower;
    int exponent = 0;
    if (std::isfinite(full)) {
        if (!(full > 0.0F)) {
            return false;
        }
        out.fraction = std::frexp(full, &exponent);
        out.exponent = exponent - 1;
        out.zero = false;
        return true;
    }
    const float half = upper / 2.0F - lower / 2.0F;
    if (!std::isfinite(half) || !(half > 0.0F)) {
        return false;
    }
    out.fraction = std::frexp(half, &exponent);
    out.exponent = exponent;
    out.zero = false;
    return true;
}

// scale_radiometric_value (:413-453) with the three factors of power().
bool scale_radiometric(float value, const float (&factors)[3], long long binary_exponent, float& out) {
    if (!std::isfinite(value) || value < 0.0F) {
        return false;
    }
    for (const float f : factors) {
        if (!std::isfinite(f) || !(f > 0.0F)) {
            return false;
        }
    }
    if (value == 0.0F) {
        out = 0.0F;
        return true;
    }
    int value_exponent = 0;
    float fraction = std::frexp(value, &value_exponent);
    long long accumulated = static_cast<long long>(value_exponent) + binary_exponent;
    for (const float f : factors) {
        int factor_exponent = 0;
        fraction *= std::frexp(f, &factor_exponent);
        accumulated += factor_exponent;
        int normalization = 0;
        fraction = std::frexp(fraction, &normalization);
        accumulated += normalization;
    }
    if (accumulated < INT_MIN || accumulated > INT_MAX) {
        return false;
    }
    out = std::scalbn(fraction, static_cast<int>(accumulated));
    return std::isfinite(out) && out > 0.0F;
}

}  // namespace

int environment_power(const EnvironmentTables& t, const float lo[3], const float hi[3], float out[4],
                      const char*& message) {
    message = nullptr;
    // bounding_sphere_scale (:359-411)
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(lo[a]) || !std::isfinite(hi[a]) || lo[a] > hi[a]) {
            return invalid(message, "Environment-light power requires explicit non-empty finite scene bounds.");
        }
    }
    HalfExtent e[3];
    for (int a = 0; a < 3; ++a) {
        if (!half_extent(lo[a], hi[a], e[a])) {
            return invalid(message, "Environment-light scene extent is not representable.");
        }
    }
    float result[4] = {0.0F, 0.0F, 0.0F, 0.0F};  // `out` is written only on success
    if ((e[0].zero && e[1].zero && e[2].zero) || t.black) {
        std::copy(result, result + 4, out);
        return kEnvironmentOk;
    }
    int maximum_exponent = INT_MIN;
    for (const HalfExtent& h : e) {
        if (!h.zero) {
            maximum_exponent = std::max(maximum_exponent, h.exponent);
        }
    }
    float s[3];
    for (int a = 0; a < 3; ++a) {
        s[a] = e[a].zero ? 0.0F : std::scalbn(e[a].fraction, e[a].exponent - maximum_exponent);
    }
    const float squared_radius = std::fma(s[0], s[0], std::fma(s[1], s[1], s[2] * s[2]));
    if (!std::isfinite(squared_radius) || !(squared_radius > 0.0F)) {
        return invalid(message, "Environment-light bounding sphere is not representable.");
    }
    const long long binary_exponent = static_cast<long long>(maximum_exponent) * 2;
    for (int lane = 0; lane < 4; ++lane) {
        if (t.lane_peak[lane] == 0.0F) {
            continue;
        }
        const float factors[3] = {t.lane_integral[lane], kPi, squared_radius};
        if (!scale_radiometric(t.lane_peak[lane], factors, binary_exponent, result[lane])) {
            return invalid(message, "Positive environment-light power is not representable.");
        }
    }
    std::copy(result, result + 4, out);
    return kEnvironmentOk;
}

}  // namespace bf200
