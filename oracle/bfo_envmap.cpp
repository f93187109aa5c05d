// Test infrastructure, not product code: the oracle's environment-map light. A CPU restatement of
// EnvironmentMapLightT<float>'s sample_li, pdf_li and le (EnvironmentLights.hpp:750-852,
// 967-1060) over the tables that blackframe-renderer_b200/csrc/bf200_envmap.cpp builds (its
// restatement of create(), :470-733, linked here as the light tree's construction is). Both are
// pinned on the compiled reference by tests/test_envmap.py (golden outputs of oracle/_ref); the
// device's batch kernels are compared with this file by tests/test_gpu_envmap.py.
//
// Rounding of sines, cosines and the arctangent: with device_trig 0 the C library's float
// functions, which the reference calls; with device_trig 1 the double-precision value rounded once
// to float, as the device computes them.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <new>

#include "../include/bf200.h"
#include "bf200_envmap.h"

namespace {

using bf200::EnvironmentTables;

struct V3 {
    float x, y, z;
};

struct Trig {
    bool device;
    float cos(float a) const { return device ? static_cast<float>(std::cos(static_cast<double>(a))) : std::cos(a); }
    float sin(float a) const { return device ? static_cast<float>(std::sin(static_cast<double>(a))) : std::sin(a); }
    float atan2(float y, float x) const {
        return device ? static_cast<float>(std::atan2(static_cast<double>(y), static_cast<double>(x)))
                      : std::atan2(y, x);
    }
};

// std::midpoint of two floats (libstdc++'s formula; the partition boundaries are all moderate).
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

bool unit_direction(V3 d) {
    const float squared = std::fma(d.x, d.x, std::fma(d.y, d.y, d.z * d.z));
    const float tolerance = 128.0F * std::numeric_limits<float>::epsilon();
    return std::isfinite(d.x) && std::isfinite(d.y) && std::isfinite(d.z) && std::isfinite(squared) &&
           std::abs(squared - 1.0F) <= tolerance;
}

// robust_unit_direction (:97-121)
bool robust_unit(V3 d, V3& out) {
    if (!std::isfinite(d.x) || !std::isfinite(d.y) || !std::isfinite(d.z)) {
        return false;
    }
    const float scale = std::max({std::abs(d.x), std::abs(d.y), std::abs(d.z)});
    if (!(scale > 0.0F) || !std::isfinite(scale)) {
        return false;
    }
    const V3 s{d.x / scale, d.y / scale, d.z / scale};
    const float squared = std::fma(s.x, s.x, std::fma(s.y, s.y, s.z * s.z));
    const float length = std::sqrt(squared);
    if (!std::isfinite(squared) || !(squared > 0.0F) || !std::isfinite(length) || !(length > 0.0F)) {
        return false;
    }
    out = V3{s.x / length, s.y / length, s.z / length};
    return unit_direction(out);
}

V3 apply(const float (&m)[9], V3 v) {
    return V3{m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
              m[6] * v.x + m[7] * v.y + m[8] * v.z};
}

struct Texel {
    size_t column, row, index;
};

// direction_texel (:264-314)
uint32_t direction_texel(const EnvironmentTables& t, const Trig& trig, V3 local, Texel& out) {
    V3 d;
    if (!robust_unit(local, d)) {
        return BF200_ENVIRONMENT_INVALID_DIRECTION;
    }
    const float equatorial = std::hypot(d.x, d.z);
    float azimuth = 0.0F;
    if (equatorial != 0.0F) {
        azimuth = trig.atan2(d.z, d.x);
        if (azimuth < 0.0F) {
            azimuth += t.azimuth.back();
        }
    }
    if (!std::isfinite(azimuth) || azimuth < 0.0F) {
        return BF200_ENVIRONMENT_NOT_REPRESENTABLE;
    }
    if (!(azimuth < t.azimuth.back())) {
        azimuth = 0.0F;
    }
    const auto column_end = std::upper_bound(t.azimuth.begin(), t.azimuth.end(), azimuth);
    const auto row_end = std::upper_bound(t.cosine.begin(), t.cosine.end(), d.y, std::greater<float>{});
    if (column_end == t.azimuth.begin() || row_end == t.cosine.begin()) {
        return BF200_ENVIRONMENT_ESCAPED;
    }
    out.column = std::min(static_cast<size_t>(column_end - t.azimuth.begin()) - 1, static_cast<size_t>(t.width) - 1);
    out.row = std::min(static_cast<size_t>(row_end - t.cosine.begin()) - 1, static_cast<size_t>(t.height) - 1);
    out.index = out.row * t.width + out.column;
    return BF200_ENVIRONMENT_OK;
}

uint32_t world_texel(const EnvironmentTables& t, const Trig& trig, V3 world, Texel& out) {
    V3 n;
    if (!robust_unit(world, n)) {
        return BF200_ENVIRONMENT_INVALID_DIRECTION;
    }
    return direction_texel(t, trig, apply(t.inverse, n), out);
}

struct Selection {
    size_t index;
    float probability, remapped;
};

// select_cdf_interval (:227-254)
bool select(const float* cdf, size_t n, float u, Selection& out) {
    const float* selected = std::upper_bound(cdf, cdf + n, u);
    if (selected == cdf + n) {
        return false;
    }
    const size_t index = static_cast<size_t>(selected - cdf);
    const float previous = index == 0 ? 0.0F : cdf[index - 1];
    const float probability = cdf[index] - previous;
    const float lower = u - previous;
    const float upper = cdf[index] - u;
    const float remapped = lower <= upper ? lower / probability : 1.0F - upper / probability;
    if (!std::isfinite(probability) || !(probability > 0.0F) || !std::isfinite(remapped) || !std::isfinite(lower) ||
        lower < 0.0F || !std::isfinite(upper) || !(upper > 0.0F) || remapped < 0.0F || !(remapped < 1.0F)) {
        return false;
    }
    out = Selection{index, probability, remapped};
    return true;
}

// sample_local_direction (:1017-1060)
uint32_t local_direction(const EnvironmentTables& t, const Trig& trig, size_t row, size_t column, float row_remapped,
                         float column_remapped, size_t row_steps, size_t column_steps, V3& out) {
    const float cosine0 = t.cosine[row], cosine1 = t.cosine[row + 1];
    const float cosine_span = cosine0 - cosine1;
    const float cosine_mid = midpoint(cosine0, cosine1);
    float cosine = std::fma(-row_remapped, cosine_span, cosine0);
    if (!(cosine < cosine0) || !(cosine > cosine1)) {
        cosine = row_remapped == 0.0F ? cosine_mid
                                      : (cosine >= cosine0 ? std::nextafter(cosine0, cosine1)
                                                           : std::nextafter(cosine1, cosine0));
        if (!(cosine < cosine0) || !(cosine > cosine1)) {
            return BF200_ENVIRONMENT_NOT_REPRESENTABLE;
        }
    }
    for (size_t step = 0; step < row_steps; ++step) {
        const float moved = std::nextafter(cosine, cosine_mid);
        if (moved == cosine || !(moved < cosine0) || !(moved > cosine1)) {
            return BF200_ENVIRONMENT_NOT_REPRESENTABLE;
        }
        cosine = moved;
    }
    if (!std::isfinite(cosine) || !(cosine > -1.0F) || !(cosine < 1.0F)) {
        return BF200_ENVIRONMENT_NOT_REPRESENTABLE;
    }
    const float radial_squared = (1.0F - cosine) * (1.0F + cosine);
    const float radial = std::sqrt(radial_squared);
    if (!std::isfinite(radial_squared) || !(radial_squared > 0.0F) || !std::isfinite(radial) || !(radial > 0.0F)) {
        return BF200_ENVIRONMENT_NOT_REPRESENTABLE;
    }
    const float azimuth0 = t.azimuth[column], azimuth1 = t.azimuth[column + 1];
    const float azimuth_span = azimuth1 - azimuth0;
    const float azimuth_mid = midpoint(azimuth0, azimuth1);
    float azimuth = std::fma(column_remapped, azimuth_span, azimuth0);
    if (!(azimuth > azimuth0) || !(azimuth < azimuth1)) {
        azimuth = column_remapped == 0.0F ? azimuth_mid
                                          : (azimuth <= azimuth0 ? std::nextafter(azimuth0, azimuth1)
                                                                 : std::nextafter(azimuth1, azimuth0));
        if (!(azimuth > azimuth0) || !(azimuth < azimuth1)) {
            return BF200_ENVIRONMENT_NOT_REPRESENTABLE;
        }
    }
    for (size_t step = 0; step < column_steps; ++step) {
        const float moved = std::nextafter(azimuth, azimuth_mid);
        if (moved == azimuth || !(moved > azimuth0) || !(moved < azimuth1)) {
            return BF200_ENVIRONMENT_NOT_REPRESENTABLE;
        }
        azimuth = moved;
    }
    if (!std::isfinite(azimuth) || azimuth < 0.0F || !(azimuth < t.azimuth.back())) {
        return BF200_ENVIRONMENT_NOT_REPRESENTABLE;
    }
    return robust_unit(V3{radial * trig.cos(azimuth), cosine, radial * trig.sin(azimuth)}, out)
               ? BF200_ENVIRONMENT_OK
               : BF200_ENVIRONMENT_NOT_REPRESENTABLE;
}

bf200_environment_sample_v1 sample_li(const EnvironmentTables& t, const Trig& trig, float u, float v) {
    bf200_environment_sample_v1 r{};
    if (!std::isfinite(u) || !std::isfinite(v) || u < 0.0F || u >= 1.0F || v < 0.0F || v >= 1.0F) {
        r.status = BF200_ENVIRONMENT_INVALID_SAMPLE;
        return r;
    }
    if (t.black) {
        return r;
    }
    Selection rs, cs;
    if (!select(t.row_cdf.data(), t.height, v, rs) ||
        !select(t.column_cdfs.data() + rs.index * t.width, t.width, u, cs)) {
        r.status = BF200_ENVIRONMENT_ESCAPED;
        return r;
    }
    const size_t index = rs.index * t.width + cs.index;
    constexpr size_t maximum = std::numeric_limits<float>::digits;
    size_t row_steps = 0, column_steps = 0;
    bool stable = false;
    V3 world{};
    for (size_t attempt = 0; attempt <= maximum * 2; ++attempt) {
        V3 local;
        uint32_t e = local_direction(t, trig, rs.index, cs.index, rs.remapped, cs.remapped, row_steps, column_steps,
                                     local);
        if (e != BF200_ENVIRONMENT_OK) {
            r.status = e;
            return r;
        }
        if (!robust_unit(apply(t.matrix, local), world)) {
            r.status = BF200_ENVIRONMENT_NOT_REPRESENTABLE;
            return r;
        }
        Texel replayed;
        e = world_texel(t, trig, world, replayed);
        if (e != BF200_ENVIRONMENT_OK) {
            r.status = e;
            return r;
        }
        if (replayed.index == index) {
            stable = true;
            break;
        }
        if (replayed.row != rs.index) {
            if (row_steps == maximum) {
                break;
            }
            ++row_steps;
        }
        if (replayed.column != cs.index) {
            if (column_steps == maximum) {
                break;
            }
            ++column_steps;
        }
    }
    if (!stable) {
        r.status = BF200_ENVIRONMENT_UNSTABLE;
        return r;
    }
    const float density = t.density[index];
    if (!std::isfinite(density) || !(density > 0.0F)) {
        r.status = BF200_ENVIRONMENT_NOT_REPRESENTABLE;
        return r;
    }
    r.direction[0] = world.x;
    r.direction[1] = world.y;
    r.direction[2] = world.z;
    for (int lane = 0; lane < 4; ++lane) {
        r.radiance[lane] = t.texels[index * 4 + lane];
    }
    r.pdf = density;
    r.valid = 1U;
    return r;
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) void* bfo_envmap_create(uint32_t width, uint32_t height, const float* texels,
                                                               const float nanometers[4], const float quaternion[4],
                                                               int* code, char* message, size_t capacity) {
    auto* t = new (std::nothrow) EnvironmentTables;
    if (t == nullptr) {
        *code = 2;
        return nullptr;
    }
    const char* text = nullptr;
    *code = bf200::build_environment_tables(width, height, texels, nanometers, quaternion, *t, text);
    if (*code != 0) {
        if (message != nullptr && capacity != 0 && text != nullptr) {
            std::strncpy(message, text, capacity - 1);
            message[capacity - 1] = '\0';
        }
        delete t;
        return nullptr;
    }
    return t;
}

__attribute__((visibility("default"))) void bfo_envmap_destroy(void* h) { delete static_cast<EnvironmentTables*>(h); }

__attribute__((visibility("default"))) void bfo_envmap_sample(const void* h, const float* canonical, uint64_t n,
                                                              int device_trig, bf200_environment_sample_v1* out) {
    const auto& t = *static_cast<const EnvironmentTables*>(h);
    const Trig trig{device_trig != 0};
    for (uint64_t i = 0; i < n; ++i) {
        out[i] = sample_li(t, trig, canonical[2 * i], canonical[2 * i + 1]);
    }
}

__attribute__((visibility("default"))) void bfo_envmap_pdf(const void* h, const float* directions, uint64_t n,
                                                           int device_trig, float* pdf, uint32_t* status) {
    const auto& t = *static_cast<const EnvironmentTables*>(h);
    const Trig trig{device_trig != 0};
    for (uint64_t i = 0; i < n; ++i) {
        const V3 d{directions[3 * i], directions[3 * i + 1], directions[3 * i + 2]};
        pdf[i] = 0.0F;
        status[i] = BF200_ENVIRONMENT_OK;
        if (!unit_direction(d)) {
            status[i] = BF200_ENVIRONMENT_INVALID_DIRECTION;
            continue;
        }
        if (t.black) {
            continue;
        }
        Texel texel;
        status[i] = world_texel(t, trig, d, texel);
        if (status[i] == BF200_ENVIRONMENT_OK) {
            pdf[i] = t.density[texel.index];
        }
    }
}

__attribute__((visibility("default"))) void bfo_envmap_le(const void* h, const float* directions, uint64_t n,
                                                          int device_trig, float* radiance, uint32_t* status) {
    const auto& t = *static_cast<const EnvironmentTables*>(h);
    const Trig trig{device_trig != 0};
    for (uint64_t i = 0; i < n; ++i) {
        const V3 d{directions[3 * i], directions[3 * i + 1], directions[3 * i + 2]};
        for (int lane = 0; lane < 4; ++lane) {
            radiance[4 * i + lane] = 0.0F;
        }
        Texel texel;
        status[i] = world_texel(t, trig, d, texel);
        if (status[i] == BF200_ENVIRONMENT_OK) {
            for (int lane = 0; lane < 4; ++lane) {
                radiance[4 * i + lane] = t.texels[texel.index * 4 + lane];
            }
        }
    }
}

__attribute__((visibility("default"))) int bfo_envmap_power(const void* h, const float lo[3], const float hi[3],
                                                            float out[4]) {
    const char* message = nullptr;
    return bf200::environment_power(*static_cast<const EnvironmentTables*>(h), lo, hi, out, message);
}

}  // extern "C"
