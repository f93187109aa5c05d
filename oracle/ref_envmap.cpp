// Test infrastructure, not product code: C entry points over the reference's own
// EnvironmentMapLightT<float> (Blackframe/Renderer/Include/Blackframe/Renderer/EnvironmentLights.hpp),
// compiled from the reference tree into oracle/_ref/libbfref.so. tests/golden/make_envmap_golden.py
// calls them to freeze golden outputs, which pin the oracle's restatement (oracle/bfo_envmap.cpp)
// and the host table construction of the product (csrc/bf200_envmap.cpp).
#include <Blackframe/Renderer/EnvironmentLights.hpp>

#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "../include/bf200.h"

namespace {

using namespace blackframe::renderer;
using Light = EnvironmentMapLightT<float>;

struct Holder {
    Light light;
    SampledWavelengthsT<float> wavelengths;
};

SampledWavelengthsT<float> packet(const float nanometers[4]) {
    SampledWavelengthsT<float> w{};
    for (int lane = 0; lane < 4; ++lane) {
        w.samples[lane].nanometers = nanometers[lane];
        w.samples[lane].probability.value = 1.0F / 470.0F;
        w.samples[lane].probability.measure = ProbabilityMeasure::wavelength;
    }
    return w;
}

void copy_message(const std::string& text, char* message, size_t capacity) {
    if (message != nullptr && capacity != 0) {
        std::strncpy(message, text.c_str(), capacity - 1);
        message[capacity - 1] = '\0';
    }
}

LightSampleContextT<float> any_context() {
    return LightSampleContextT<float>::create(Point3T<float>{}, 0.5F).value();
}

}  // namespace

extern "C" {

// Creates the light; returns null with *code (1 invalid, 2 exhausted) and the reference's message.
__attribute__((visibility("default"))) void* bfref_envmap_create(uint32_t width, uint32_t height, const float* texels,
                                                                 const float nanometers[4], const float quaternion[4],
                                                                 int* code, char* message, size_t capacity) {
    std::vector<LightSpectrumT<float>> spectra(static_cast<size_t>(width) * height);
    for (size_t i = 0; i < spectra.size(); ++i) {
        for (int lane = 0; lane < 4; ++lane) {
            spectra[i].values[lane] = texels[i * 4 + lane];
        }
    }
    const QuaternionT<float> q{.x = quaternion[0], .y = quaternion[1], .z = quaternion[2], .w = quaternion[3]};
    auto light = Light::create(width, height, std::move(spectra), packet(nanometers), q);
    if (!light) {
        *code = light.error().code == blackframe::core::StatusCode::resource_exhausted ? 2 : 1;
        copy_message(light.error().message, message, capacity);
        return nullptr;
    }
    *code = 0;
    return new Holder{std::move(*light), packet(nanometers)};
}

__attribute__((visibility("default"))) void bfref_envmap_destroy(void* h) { delete static_cast<Holder*>(h); }

// sample_li per canonical pair; a failed query has status 1 (the reference returned an error).
__attribute__((visibility("default"))) void bfref_envmap_sample(const void* h, const float* canonical, uint64_t n,
                                                                bf200_environment_sample_v1* out) {
    const Holder& holder = *static_cast<const Holder*>(h);
    const auto ctx = any_context();
    for (uint64_t i = 0; i < n; ++i) {
        bf200_environment_sample_v1 r{};
        const auto s = holder.light.sample_li(ctx, Point2T<float>{.x = canonical[2 * i], .y = canonical[2 * i + 1]},
                                              holder.wavelengths);
        if (!s) {
            r.status = 1U;
        } else if (s->has_value()) {
            const auto& v = **s;
            r.direction[0] = v.direction_to_light().x;
            r.direction[1] = v.direction_to_light().y;
            r.direction[2] = v.direction_to_light().z;
            for (int lane = 0; lane < 4; ++lane) {
                r.radiance[lane] = v.incident_radiance().values[lane];
            }
            r.pdf = v.probability().value;
            r.valid = 1U;
        }
        out[i] = r;
    }
}

__attribute__((visibility("default"))) void bfref_envmap_pdf(const void* h, const float* directions, uint64_t n,
                                                             float* pdf, uint32_t* status) {
    const Holder& holder = *static_cast<const Holder*>(h);
    const auto ctx = any_context();
    for (uint64_t i = 0; i < n; ++i) {
        const Vector3T<float> d{.x = directions[3 * i], .y = directions[3 * i + 1], .z = directions[3 * i + 2]};
        const auto p = holder.light.pdf_li(ctx, d, holder.wavelengths);
        pdf[i] = p ? p->value() : 0.0F;
        status[i] = p ? 0U : 1U;
    }
}

__attribute__((visibility("default"))) void bfref_envmap_le(const void* h, const float* directions, uint64_t n,
                                                            float* radiance, uint32_t* status) {
    const Holder& holder = *static_cast<const Holder*>(h);
    for (uint64_t i = 0; i < n; ++i) {
        const Vector3T<float> d{.x = directions[3 * i], .y = directions[3 * i + 1], .z = directions[3 * i + 2]};
        for (int lane = 0; lane < 4; ++lane) {
            radiance[4 * i + lane] = 0.0F;
        }
        const auto ray = RayT<float>::create(Point3T<float>{.x = 1.0F, .y = -2.0F, .z = 3.0F}, d, 0.0F,
                                             std::numeric_limits<float>::infinity(), 0.5F, AllRayVisibility,
                                             VacuumMedium);
        if (!ray) {
            status[i] = 2U;  // the reference cannot even form the escaped ray
            continue;
        }
        const auto e = holder.light.le(*ray, holder.wavelengths);
        status[i] = e ? 0U : 1U;
        if (e) {
            for (int lane = 0; lane < 4; ++lane) {
                radiance[4 * i + lane] = e->values[lane];
            }
        }
    }
}

__attribute__((visibility("default"))) int bfref_envmap_power(const void* h, const float lo[3], const float hi[3],
                                                              float out[4]) {
    const Holder& holder = *static_cast<const Holder*>(h);
    const auto bounds = Bounds3T<float>::from_minimum_maximum(Point3T<float>{.x = lo[0], .y = lo[1], .z = lo[2]},
                                                              Point3T<float>{.x = hi[0], .y = hi[1], .z = hi[2]});
    if (!bounds) {
        return 1;
    }
    const auto p = holder.light.power(*bounds, holder.wavelengths);
    if (!p) {
        return 1;
    }
    for (int lane = 0; lane < 4; ++lane) {
        out[lane] = p->values[lane];
    }
    return 0;
}

}  // extern "C"
