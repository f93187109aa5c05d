// Test-infrastructure harness around the reference implementation itself.
//
// This translation unit is compiled together with the reference's own Core, Renderer and
// Engine sources (see oracle/Makefile) into oracle/_ref/libbfref.so. It is never shipped and
// never called by the product: only tests, the golden-fixture generator and bench.py's
// reference arm load it, as the checker / CPU baseline. It turns the flat bf200 scene and path
// records into the reference's own objects and runs the reference's own scalar path tracer:
//
//   * FrameScene::create                   (Blackframe/Engine/Source/FrameScene.cpp:390-528)
//   * create_analytic_accel_backend        (Blackframe/Engine/Source/AccelBackend.cpp:348)
//   * LightSampler::create_uniform         (Blackframe/Renderer/Source/LightSampler.cpp:574)
//   * trace_scene_mis                      (Blackframe/Engine/Source/SceneMisPathLoop.cpp:1009)
//   * PinholeCamera::generate_primary_ray  (Blackframe/Renderer/Include/.../PinholeCamera.hpp)
//   * cie_1931_spectrum_to_xyz, xyz_to_linear_rgb, Film/ReferenceFilm::add_sample
//     (the caller-side film path of Tests/Backends/GPU/CUDA/CudaTransportParityTest.cpp:906-927)
//
// The CIE sensor source is included here (rather than linked) so the harness can read the
// colour-matching response at the frame's packet wavelengths.
#include "Cie1931Sensor.cpp"

#include "../include/bf200.h"
#include "ref_scene.hpp"

#include <Blackframe/Engine/AccelBackend.hpp>
#include <Blackframe/Engine/FrameScene.hpp>
#include <Blackframe/Engine/SceneMisPathLoop.hpp>
#include <Blackframe/Engine/TriangleMesh.hpp>
#include <Blackframe/Engine/TriangleMeshImport.hpp>
#include <Blackframe/Renderer/Color.hpp>
#include <Blackframe/Renderer/Film.hpp>
#include <Blackframe/Renderer/IndependentSampler.hpp>
#include <Blackframe/Renderer/LightSampler.hpp>
#include <Blackframe/Renderer/OwenScrambling.hpp>
#include <Blackframe/Renderer/PinholeCamera.hpp>
#include <Blackframe/Renderer/RayCone.hpp>
#include <Blackframe/Renderer/Sphere.hpp>
#include <Blackframe/Renderer/WavelengthSampling.hpp>

#include <atomic>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

using namespace blackframe;
using namespace bfref;

std::mutex g_error_mutex;
std::string g_last_error;

void set_error(const std::string& message) {
    std::lock_guard<std::mutex> lock{g_error_mutex};
    g_last_error = message;
}

struct RefScene {
    engine::FrameSceneHandle scene;
    std::unique_ptr<engine::AccelBackend> accel;
    std::unique_ptr<renderer::LightSampler> sampler;
    renderer::SampledWavelengths wavelengths{};
};

// Traces one path through the reference; lane_status 0 on success, 1 with the path zeroed when
// the reference itself returns an error for this path.
void trace_one(const RefScene& scene, const bf200_path_input_v1& input,
               const bf200_transport_options_v1& options,
               const renderer::RussianRoulettePolicy& policy, bf200_path_result_v1& out,
               std::string* error, const bf200_path_state_v1* initial = nullptr) {
    std::memset(&out, 0, sizeof(out));
    auto state = renderer::PathState::create_initial(scene.wavelengths, renderer::VacuumMedium);
    if (initial != nullptr) {
        renderer::TransportSpectrum beta{}, radiance{};
        for (std::size_t lane = 0; lane < 4; ++lane) {
            beta.values[lane] = initial->beta[lane];
            radiance.values[lane] = initial->radiance[lane];
        }
        state = renderer::PathState::create(beta, radiance, renderer::PathDepthCounters{}, initial->eta_scale,
                                            scene.wavelengths, renderer::PathDeltaFlags::none,
                                            renderer::VacuumMedium);
        if (!state) {
            out.lane_status = BF200_LANE_NUMERICAL_FAILURE;
            if (error != nullptr && error->empty()) {
                *error = state.error().message;
            }
            return;
        }
    }
    const auto stream = renderer::SampleStream{renderer::SampleStreamIndex{
        .pixel_x = input.sample.pixel_x,
        .pixel_y = input.sample.pixel_y,
        .sample_index = input.sample.sample_index,
        .seed = input.sample.seed,
    }};
    const auto limits = renderer::PathDepthLimits{
        .diffuse = options.depth_limits[0],
        .glossy = options.depth_limits[1],
        .specular = options.depth_limits[2],
        .transmission = options.depth_limits[3],
        .volume = options.depth_limits[4],
    };
    const auto result = engine::trace_scene_mis(
        make_ray(input.primary_ray), *state, stream, *scene.accel, *scene.sampler,
        options.mis_heuristic == 1 ? renderer::MisHeuristic::power : renderer::MisHeuristic::balance,
        limits, policy);
    if (!result) {
        out.lane_status = BF200_LANE_NUMERICAL_FAILURE;
        if (error != nullptr && error->empty()) {
            *error = result.error().message;
        }
        return;
    }
    const auto& path_state = result->state;
    for (std::size_t lane = 0; lane < 4; ++lane) {
        out.beta[lane] = path_state.beta()[lane];
        out.radiance[lane] = path_state.accumulated_radiance()[lane];
    }
    out.depth = path_state.depth();
    out.depth_counters[0] = path_state.depth_counters().diffuse;
    out.depth_counters[1] = path_state.depth_counters().glossy;
    out.depth_counters[2] = path_state.depth_counters().specular;
    out.depth_counters[3] = path_state.depth_counters().transmission;
    out.depth_counters[4] = path_state.depth_counters().volume;
    out.eta_scale = path_state.eta_scale();
    out.delta_flags = static_cast<uint32_t>(path_state.delta_flags());
    out.termination = static_cast<uint32_t>(result->termination);
    out.blocked_depth_limits = static_cast<uint32_t>(result->blocked_depth_limits);
    out.lane_status = BF200_LANE_OK;
    store_ray(result->terminal_ray, out.terminal_ray);
}

template <typename Body> void parallel_for(uint64_t count, int threads, Body body) {
    if (threads <= 1 || count < 2) {
        for (uint64_t index = 0; index < count; ++index) {
            body(index);
        }
        return;
    }
    std::atomic<uint64_t> next{0};
    std::vector<std::thread> pool;
    for (int worker = 0; worker < threads; ++worker) {
        pool.emplace_back([&] {
            for (uint64_t index = next.fetch_add(1); index < count; index = next.fetch_add(1)) {
                body(index);
            }
        });
    }
    for (auto& thread : pool) {
        thread.join();
    }
}

} // namespace

extern "C" {

__attribute__((visibility("default"))) const char* bfr_last_error() {
    return g_last_error.c_str();
}

__attribute__((visibility("default"))) int bfr_scene_create(const bf200_scene_desc_v1* desc,
                                                            void** out_scene) {
    if (desc == nullptr || out_scene == nullptr) {
        set_error("null argument");
        return 1;
    }
    std::string error;
    int code = 0;
    auto scene = bfref::make_frame_scene(desc, error, &code);
    if (!scene) {
        set_error(error);
        return code;
    }
    const auto wavelengths = bfref::make_wavelengths(desc->wavelength_nanometers, desc->wavelength_pdf);
    auto accel = engine::create_analytic_accel_backend(scene);
    if (!accel) {
        set_error("accel: " + accel.error().message);
        return 5;
    }
    auto sampler = renderer::LightSampler::create_uniform(scene->punctual_lights().size() +
                                                          scene->mesh_area_lights().size());
    if (!sampler) {
        set_error("light sampler: " + sampler.error().message);
        return 6;
    }
    auto* result = new RefScene{};
    result->scene = scene;
    result->accel = std::move(*accel);
    result->sampler = std::make_unique<renderer::LightSampler>(std::move(*sampler));
    result->wavelengths = wavelengths;
    *out_scene = result;
    return 0;
}

__attribute__((visibility("default"))) void bfr_scene_destroy(void* scene) {
    delete static_cast<RefScene*>(scene);
}

// Writes the committed world_to_object (inverse) matrix of instance `index` (sorted order).
__attribute__((visibility("default"))) int bfr_scene_world_to_object(void* handle, uint32_t index,
                                                                     float* out16) {
    const auto* scene = static_cast<RefScene*>(handle);
    const auto instances = scene->scene->instances();
    if (index >= instances.size()) {
        return 1;
    }
    const auto transform = scene->scene->world_transform(instances[index].id);
    if (!transform) {
        return 2;
    }
    for (std::size_t r = 0; r < 4; ++r) {
        for (std::size_t c = 0; c < 4; ++c) {
            out16[r * 4 + c] = transform->get().inverse_matrix()(r, c);
        }
    }
    return 0;
}

__attribute__((visibility("default"))) uint32_t bfr_scene_light_count(void* handle) {
    const auto* scene = static_cast<RefScene*>(handle);
    return static_cast<uint32_t>(scene->scene->mesh_area_lights().size() +
                                 scene->scene->punctual_lights().size());
}

// Runs trace_scene_mis for every input. Returns the number of paths the reference rejected
// with an error (those carry lane_status 1 and zeroed outputs).
__attribute__((visibility("default"))) int64_t
bfr_trace_paths(void* handle, const bf200_path_input_v1* inputs, uint64_t count,
                const bf200_transport_options_v1* options, bf200_path_result_v1* results,
                int threads) {
    const auto* scene = static_cast<RefScene*>(handle);
    const auto policy = make_policy(*options);
    if (!policy) {
        set_error(policy.error().message);
        return -1;
    }
    std::atomic<int64_t> failures{0};
    std::string first_error;
    std::mutex error_mutex;
    parallel_for(count, threads, [&](uint64_t index) {
        std::string error;
        trace_one(*scene, inputs[index], *options, *policy, results[index], &error);
        if (results[index].lane_status != 0) {
            failures.fetch_add(1);
            std::lock_guard<std::mutex> lock{error_mutex};
            if (first_error.empty()) {
                first_error = error;
            }
        }
    });
    if (!first_error.empty()) {
        set_error(first_error);
    }
    return failures.load();
}

// bfr_trace_paths with a depth-zero initial PathState per path (PathState::create with the
// given throughput, radiance and eta scale, no depth and no delta history).
__attribute__((visibility("default"))) int64_t
bfr_trace_paths_states(void* handle, const bf200_path_input_v1* inputs, const bf200_path_state_v1* states,
                       uint64_t count, const bf200_transport_options_v1* options, bf200_path_result_v1* results,
                       int threads) {
    const auto* scene = static_cast<RefScene*>(handle);
    const auto policy = make_policy(*options);
    if (!policy) {
        set_error(policy.error().message);
        return -1;
    }
    std::atomic<int64_t> failures{0};
    std::string first_error;
    std::mutex error_mutex;
    parallel_for(count, threads, [&](uint64_t index) {
        std::string error;
        trace_one(*scene, inputs[index], *options, *policy, results[index], &error, states + index);
        if (results[index].lane_status != 0) {
            failures.fetch_add(1);
            std::lock_guard<std::mutex> lock{error_mutex};
            if (first_error.empty()) {
                first_error = error;
            }
        }
    });
    if (!first_error.empty()) {
        set_error(first_error);
    }
    return failures.load();
}

// Builds the reference pinhole camera (origin, frame from normal + tangent seed, vertical fov)
// and reports the derived constants in bf200_camera_v1 form.
__attribute__((visibility("default"))) int bfr_camera(const float* origin, const float* normal,
                                                      const float* tangent, uint32_t width,
                                                      uint32_t height, float vfov, float t_min,
                                                      float t_max, float time, uint32_t mask,
                                                      bf200_camera_v1* out) {
    const auto frame = renderer::OrthonormalFrame::from_normal_and_tangent(
        renderer::Normal3{.x = normal[0], .y = normal[1], .z = normal[2]},
        renderer::Vector3{.x = tangent[0], .y = tangent[1], .z = tangent[2]});
    if (!frame) {
        set_error(frame.error().message);
        return 1;
    }
    const auto camera = renderer::PinholeCamera::create(
        renderer::Point3{.x = origin[0], .y = origin[1], .z = origin[2]}, *frame,
        renderer::RenderExtent{.width = width, .height = height}, vfov, t_min, t_max, mask,
        renderer::VacuumMedium);
    if (!camera) {
        set_error(camera.error().message);
        return 2;
    }
    std::memset(out, 0, sizeof(*out));
    for (int a = 0; a < 3; ++a) {
        out->origin[a] = origin[a];
    }
    out->tangent[0] = frame->tangent().x;
    out->tangent[1] = frame->tangent().y;
    out->tangent[2] = frame->tangent().z;
    out->bitangent[0] = frame->bitangent().x;
    out->bitangent[1] = frame->bitangent().y;
    out->bitangent[2] = frame->bitangent().z;
    out->normal[0] = frame->normal().x;
    out->normal[1] = frame->normal().y;
    out->normal[2] = frame->normal().z;
    const auto half_height = std::tan(vfov / 2.0F);
    out->half_height = half_height;
    out->half_width = half_height * (static_cast<float>(width) / static_cast<float>(height));
    out->t_min = t_min;
    out->t_max = t_max;
    out->time = time;
    out->mask = mask;
    out->width = width;
    out->height = height;
    out->jitter_mode = 1;
    return 0;
}

// Generates reference primary rays for (pixel, sample) indices with uniform jitter.
__attribute__((visibility("default"))) int
bfr_camera_rays(const float* origin, const float* normal, const float* tangent, uint32_t width,
                uint32_t height, float vfov, float time, const bf200_sample_index_v1* samples,
                uint64_t count, bf200_ray_v1* rays) {
    const auto frame = renderer::OrthonormalFrame::from_normal_and_tangent(
        renderer::Normal3{.x = normal[0], .y = normal[1], .z = normal[2]},
        renderer::Vector3{.x = tangent[0], .y = tangent[1], .z = tangent[2]});
    const auto camera = renderer::PinholeCamera::create(
        renderer::Point3{.x = origin[0], .y = origin[1], .z = origin[2]}, *frame,
        renderer::RenderExtent{.width = width, .height = height}, vfov, 0.0F,
        std::numeric_limits<float>::infinity(), renderer::AllRayVisibility,
        renderer::VacuumMedium);
    if (!camera) {
        set_error(camera.error().message);
        return 1;
    }
    for (uint64_t index = 0; index < count; ++index) {
        const auto pixel_sample = renderer::PixelSampleIndex{
            .pixel_x = samples[index].pixel_x,
            .pixel_y = samples[index].pixel_y,
            .sample_index = samples[index].sample_index,
            .seed = samples[index].seed,
        };
        const auto ray =
            camera->generate_primary_ray(pixel_sample, renderer::PixelJitterMode::uniform, time);
        if (!ray) {
            set_error(ray.error().message);
            return 2;
        }
        store_ray(*ray, rays[index]);
    }
    return 0;
}

// Reference primary ray cones (PinholeCamera::generate_primary_ray_cone through the ray
// differential, RayCone.hpp:194-220) for (pixel, sample) indices with uniform jitter: 2 floats
// (width, spread) per sample.
__attribute__((visibility("default"))) int
bfr_camera_cones(const float* origin, const float* normal, const float* tangent, uint32_t width,
                 uint32_t height, float vfov, float time, const bf200_sample_index_v1* samples,
                 uint64_t count, float* cones) {
    const auto frame = renderer::OrthonormalFrame::from_normal_and_tangent(
        renderer::Normal3{.x = normal[0], .y = normal[1], .z = normal[2]},
        renderer::Vector3{.x = tangent[0], .y = tangent[1], .z = tangent[2]});
    const auto camera = renderer::PinholeCamera::create(
        renderer::Point3{.x = origin[0], .y = origin[1], .z = origin[2]}, *frame,
        renderer::RenderExtent{.width = width, .height = height}, vfov, 0.0F,
        std::numeric_limits<float>::infinity(), renderer::AllRayVisibility,
        renderer::VacuumMedium);
    if (!camera) {
        set_error(camera.error().message);
        return 1;
    }
    for (uint64_t index = 0; index < count; ++index) {
        const auto pixel_sample = renderer::PixelSampleIndex{
            .pixel_x = samples[index].pixel_x,
            .pixel_y = samples[index].pixel_y,
            .sample_index = samples[index].sample_index,
            .seed = samples[index].seed,
        };
        const auto sample = renderer::generate_pixel_sample<float>(pixel_sample, renderer::PixelJitterMode::uniform);
        if (!sample) {
            set_error(sample.error().message);
            return 2;
        }
        const auto cone = camera->generate_primary_ray_cone(*sample, time);
        if (!cone) {
            set_error(cone.error().message);
            return 3;
        }
        cones[2 * index] = cone->width();
        cones[2 * index + 1] = cone->spread();
    }
    return 0;
}

// renderer::advance_ray_cone(cone, distance) (RayCone.hpp:222-241) per case: the advanced width,
// NaN where the reference returns an error. Returns the number of errors.
__attribute__((visibility("default"))) int64_t bfr_cone_advance(const float* cones, const float* distances,
                                                                uint64_t count, float* widths) {
    int64_t failures = 0;
    for (uint64_t i = 0; i < count; ++i) {
        widths[i] = std::numeric_limits<float>::quiet_NaN();
        const auto cone = renderer::RayCone::create(cones[2 * i], cones[2 * i + 1]);
        if (!cone) {
            ++failures;
            continue;
        }
        const auto advanced = renderer::advance_ray_cone(*cone, distances[i]);
        if (!advanced) {
            ++failures;
            continue;
        }
        widths[i] = advanced->width();
    }
    return failures;
}

// renderer::propagate_ray_cone_scattering (RayCone.hpp:316-437) per case: closure kind, lobes
// and 10 parameters, event lobes, local wo and wi; (width, spread), NaN where the reference
// returns an error. Returns the number of errors.
__attribute__((visibility("default"))) int64_t bfr_cone_scatter(const float* cones, const uint32_t* kinds,
                                                                const float* parameters, const uint32_t* events,
                                                                const float* wo, const float* wi, uint64_t count,
                                                                float* out) {
    int64_t failures = 0;
    for (uint64_t i = 0; i < count; ++i) {
        out[2 * i] = out[2 * i + 1] = std::numeric_limits<float>::quiet_NaN();
        const auto cone = renderer::RayCone::create(cones[2 * i], cones[2 * i + 1]);
        if (!cone) {
            ++failures;
            continue;
        }
        renderer::Closure closure{};
        closure.kind = static_cast<renderer::ClosureKind>(kinds[i]);
        for (std::size_t k = 0; k < 10; ++k) {
            closure.parameters[k] = parameters[10 * i + k];
        }
        const auto scattered = renderer::propagate_ray_cone_scattering(
            *cone, closure, static_cast<renderer::ScatteringLobe>(events[i]),
            renderer::Vector3{.x = wo[3 * i], .y = wo[3 * i + 1], .z = wo[3 * i + 2]},
            renderer::Vector3{.x = wi[3 * i], .y = wi[3 * i + 1], .z = wi[3 * i + 2]});
        if (!scattered) {
            ++failures;
            continue;
        }
        out[2 * i] = scattered->width();
        out[2 * i + 1] = scattered->spread();
    }
    return failures;
}

// CIE 1931 sensor constants at a packet: response at each lane, lane pdf, normalisation.
__attribute__((visibility("default"))) int bfr_sensor(const float* nm, const float* pdf,
                                                      bf200_sensor_v1* out) {
    std::memset(out, 0, sizeof(*out));
    for (std::size_t lane = 0; lane < 4; ++lane) {
        const auto response = renderer::color_matching_functions<float>(nm[lane]);
        out->response_xyz[lane][0] = response.x;
        out->response_xyz[lane][1] = response.y;
        out->response_xyz[lane][2] = response.z;
        out->wavelength_pdf[lane] = pdf[lane];
    }
    constexpr auto inverse_lane_count = 1.0F / 4.0F;
    out->normalization = inverse_lane_count / static_cast<float>(renderer::Cie1931YIntegralNanometers);
    return 0;
}

// LightSampler::create_power_weighted over 4-lane spectral powers: probability(i) of every light
// into `probabilities`, and sample(u_k) (index, probability) for every u in `samples`. Returns 0,
// or the reference StatusCode when it refuses the powers.
__attribute__((visibility("default"))) int bfr_power_sampler(const float* powers, uint32_t count, float* probabilities,
                                                             const float* samples, uint32_t sample_count,
                                                             uint32_t* selected, float* selected_probability) {
    std::vector<renderer::LightSpectrumT<renderer::TransportScalar>> spectra(count);
    for (uint32_t i = 0; i < count; ++i) {
        for (int l = 0; l < 4; ++l) {
            spectra[i].values[l] = powers[4 * i + l];
        }
    }
    auto sampler = renderer::LightSampler::create_power_weighted(spectra);
    if (!sampler) {
        set_error(sampler.error().message);
        return static_cast<int>(sampler.error().code);
    }
    for (uint32_t i = 0; i < count; ++i) {
        probabilities[i] = sampler->probability(i)->value();
    }
    for (uint32_t k = 0; k < sample_count; ++k) {
        const auto selection = sampler->sample(samples[k]);
        selected[k] = selection ? selection->light_index() : 0xFFFFFFFFU;
        selected_probability[k] = selection ? selection->probability().value() : -1.0F;
    }
    return 0;
}

// The reference's spatial light tree (LightSampler::create_spatial_tree) queried at points:
// mode 0 samples (samples[q] -> selected[q], probability[q]), mode 1 evaluates the probability of
// selected[q]. A refused query gives 0xFFFFFFFF / -1; a refused tree returns its StatusCode.
__attribute__((visibility("default"))) int bfr_light_tree(const float* bounds_min, const float* bounds_max,
                                                          const float* powers, uint32_t count, int mode,
                                                          const float* positions, const float* samples,
                                                          uint64_t query_count, uint32_t* selected,
                                                          float* probabilities) {
    std::vector<renderer::LightTreeInputT<renderer::TransportScalar>> lights;
    lights.reserve(count);
    for (uint32_t i = 0; i < count; ++i) {
        const auto bounds = renderer::Bounds3::from_minimum_maximum(
            renderer::Point3{.x = bounds_min[3 * i], .y = bounds_min[3 * i + 1], .z = bounds_min[3 * i + 2]},
            renderer::Point3{.x = bounds_max[3 * i], .y = bounds_max[3 * i + 1], .z = bounds_max[3 * i + 2]});
        if (!bounds) {
            set_error(bounds.error().message);
            return static_cast<int>(bounds.error().code);
        }
        renderer::LightSpectrumT<renderer::TransportScalar> power{};
        for (int l = 0; l < 4; ++l) {
            power.values[l] = powers[4 * i + l];
        }
        lights.push_back({.bounds = *bounds, .spectral_power = power});
    }
    auto sampler = renderer::LightSampler::create_spatial_tree(lights);
    if (!sampler) {
        set_error(sampler.error().message);
        return static_cast<int>(sampler.error().code);
    }
    for (uint64_t q = 0; q < query_count; ++q) {
        const auto context = renderer::LightSampleContext::create(
            renderer::Point3{.x = positions[3 * q], .y = positions[3 * q + 1], .z = positions[3 * q + 2]}, 0.5F);
        if (!context) {
            if (mode == 0) {
                selected[q] = 0xFFFFFFFFU;
            }
            probabilities[q] = -1.0F;
            continue;
        }
        if (mode == 0) {
            const auto selection = sampler->sample(*context, samples[q]);
            selected[q] = selection ? selection->light_index() : 0xFFFFFFFFU;
            probabilities[q] = selection ? selection->probability().value() : -1.0F;
        } else {
            const auto probability = sampler->probability(*context, selected[q]);
            probabilities[q] = probability ? probability->value() : -1.0F;
        }
    }
    return 0;
}

// Replaces a scene's light sampler by the spatial light tree of the given per-light bounds and
// spectral powers (registry order); traces then select by the tree.
__attribute__((visibility("default"))) int bfr_scene_set_light_tree(void* handle, const bf200_light_tree_input_v1* in,
                                                                    uint32_t count) {
    auto* scene = static_cast<RefScene*>(handle);
    std::vector<renderer::LightTreeInputT<renderer::TransportScalar>> lights;
    for (uint32_t i = 0; i < count; ++i) {
        const auto bounds = renderer::Bounds3::from_minimum_maximum(
            renderer::Point3{.x = in[i].bounds_min[0], .y = in[i].bounds_min[1], .z = in[i].bounds_min[2]},
            renderer::Point3{.x = in[i].bounds_max[0], .y = in[i].bounds_max[1], .z = in[i].bounds_max[2]});
        if (!bounds) {
            set_error(bounds.error().message);
            return static_cast<int>(bounds.error().code);
        }
        renderer::LightSpectrumT<renderer::TransportScalar> power{};
        for (int l = 0; l < 4; ++l) {
            power.values[l] = in[i].spectral_power[l];
        }
        lights.push_back({.bounds = *bounds, .spectral_power = power});
    }
    auto sampler = renderer::LightSampler::create_spatial_tree(lights);
    if (!sampler) {
        set_error(sampler.error().message);
        return static_cast<int>(sampler.error().code);
    }
    scene->sampler = std::make_unique<renderer::LightSampler>(std::move(*sampler));
    return 0;
}

// Replaces a scene's light sampler by the power-weighted one (traces then select by power).
__attribute__((visibility("default"))) int bfr_scene_set_light_powers(void* handle, const float* powers,
                                                                      uint32_t count) {
    auto* scene = static_cast<RefScene*>(handle);
    std::vector<renderer::LightSpectrumT<renderer::TransportScalar>> spectra(count);
    for (uint32_t i = 0; i < count; ++i) {
        for (int l = 0; l < 4; ++l) {
            spectra[i].values[l] = powers[4 * i + l];
        }
    }
    auto sampler = renderer::LightSampler::create_power_weighted(spectra);
    if (!sampler) {
        set_error(sampler.error().message);
        return static_cast<int>(sampler.error().code);
    }
    scene->sampler = std::make_unique<renderer::LightSampler>(std::move(*sampler));
    return 0;
}

// engine::load_obj_triangle_mesh / load_ply_triangle_mesh (by the path's extension). Returns a
// handle (null on failure, with *code = the reference's StatusCode and the message in
// bfr_last_error); bfr_mesh_counts and bfr_mesh_copy read it, bfr_mesh_free releases it.
__attribute__((visibility("default"))) void* bfr_mesh_load(const char* path, int* code) {
    const std::string p(path);
    const bool ply = p.size() >= 4 && p.compare(p.size() - 4, 4, ".ply") == 0;
    auto mesh = ply ? engine::load_ply_triangle_mesh(p) : engine::load_obj_triangle_mesh(p);
    if (!mesh) {
        *code = static_cast<int>(mesh.error().code);
        set_error(mesh.error().message);
        return nullptr;
    }
    *code = 0;
    return new engine::TriangleMesh(std::move(*mesh));
}

__attribute__((visibility("default"))) void bfr_mesh_counts(void* handle, uint32_t* vertices, uint32_t* triangles) {
    const auto* m = static_cast<const engine::TriangleMesh*>(handle);
    *vertices = static_cast<uint32_t>(m->positions().size());
    *triangles = static_cast<uint32_t>(m->triangles().size());
}

__attribute__((visibility("default"))) void bfr_mesh_copy(void* handle, float* positions, float* normals, float* uvs,
                                                          uint32_t* triangles) {
    const auto* m = static_cast<const engine::TriangleMesh*>(handle);
    for (size_t i = 0; i < m->positions().size(); ++i) {
        positions[3 * i] = m->positions()[i].x;
        positions[3 * i + 1] = m->positions()[i].y;
        positions[3 * i + 2] = m->positions()[i].z;
        normals[3 * i] = m->normals()[i].x;
        normals[3 * i + 1] = m->normals()[i].y;
        normals[3 * i + 2] = m->normals()[i].z;
        uvs[2 * i] = m->texture_coordinates()[i].x;
        uvs[2 * i + 1] = m->texture_coordinates()[i].y;
    }
    for (size_t t = 0; t < m->triangles().size(); ++t) {
        for (int k = 0; k < 3; ++k) {
            triangles[3 * t + k] = m->triangles()[t].vertices[k];
        }
    }
}

__attribute__((visibility("default"))) void bfr_mesh_free(void* handle) {
    delete static_cast<engine::TriangleMesh*>(handle);
}

// renderer::Sphere (float) on ray k against sphere k (centre xyz, radius). Per ray, out receives
// 8 floats: status (0 miss, 1 hit, 2 the reference reported an error), t, outward normal xyz,
// hit position xyz.
__attribute__((visibility("default"))) int
bfr_sphere_intersect(const float* spheres, const bf200_ray_v1* rays, uint64_t count, float* out) {
    for (uint64_t k = 0; k < count; ++k) {
        float* o = out + 8 * k;
        for (int i = 0; i < 8; ++i) {
            o[i] = 0.0F;
        }
        const float* sp = spheres + 4 * k;
        const auto sphere = renderer::Sphere::create(renderer::Point3{.x = sp[0], .y = sp[1], .z = sp[2]}, sp[3]);
        const auto& r = rays[k];
        const auto ray = renderer::Ray::create(
            renderer::Point3{.x = r.origin[0], .y = r.origin[1], .z = r.origin[2]},
            renderer::Vector3{.x = r.direction[0], .y = r.direction[1], .z = r.direction[2]}, r.t_min, r.t_max,
            r.time, r.mask, renderer::MediumId{.value = r.medium});
        if (!sphere.has_value() || !ray.has_value()) {
            o[0] = 2.0F;
            continue;
        }
        const auto hit = sphere->intersect(*ray);
        if (!hit.has_value()) {
            o[0] = 2.0F;
            continue;
        }
        if (!hit->has_value()) {
            continue;
        }
        const auto& h = **hit;
        o[0] = 1.0F;
        o[1] = h.parameter;
        o[2] = h.geometric_normal.x;
        o[3] = h.geometric_normal.y;
        o[4] = h.geometric_normal.z;
        o[5] = h.position.x;
        o[6] = h.position.y;
        o[7] = h.position.z;
    }
    return 0;
}

// Reference caller-side film path: spectrum -> XYZ -> linear RGB -> add_sample(x, y, rgb, 1).
// Radiance lanes per path; pixels and samples given per path in the order they are added.
// precision 0: renderer::Film (float32), 1: renderer::ReferenceFilm (float64, Neumaier).
// out_sums receives the resolved snapshot sums (r, g, b, weight) per pixel as double.
__attribute__((visibility("default"))) int
bfr_film_accumulate(const float* radiance, const bf200_sample_index_v1* samples, uint64_t count,
                    const float* nm, const float* pdf, uint32_t width, uint32_t height,
                    uint32_t precision, double* out_sums, uint64_t* out_counts) {
    const auto wavelengths = make_wavelengths(nm, pdf);
    auto run = [&](auto& film) -> int {
        for (uint64_t index = 0; index < count; ++index) {
            const auto spectrum = spectrum4(radiance + 4 * index);
            const auto xyz = renderer::cie_1931_spectrum_to_xyz(spectrum, wavelengths);
            if (!xyz) {
                set_error(xyz.error().message);
                return 2;
            }
            const auto rgb = renderer::xyz_to_linear_rgb(*xyz);
            if (!rgb) {
                set_error(rgb.error().message);
                return 3;
            }
            using Film = std::remove_reference_t<decltype(film)>;
            const auto status = film.add_sample(
                samples[index].pixel_x, samples[index].pixel_y,
                typename Film::Color{.red = static_cast<typename Film::Scalar>(rgb->red),
                                     .green = static_cast<typename Film::Scalar>(rgb->green),
                                     .blue = static_cast<typename Film::Scalar>(rgb->blue)},
                typename Film::Scalar{1});
            if (!status) {
                set_error(status.error().message);
                return 4;
            }
        }
        for (uint32_t y = 0; y < height; ++y) {
            for (uint32_t x = 0; x < width; ++x) {
                const auto pixel = film.pixel(x, y);
                const auto i = static_cast<std::size_t>(y) * width + x;
                out_sums[4 * i + 0] = static_cast<double>(pixel->weighted_sum.red);
                out_sums[4 * i + 1] = static_cast<double>(pixel->weighted_sum.green);
                out_sums[4 * i + 2] = static_cast<double>(pixel->weighted_sum.blue);
                out_sums[4 * i + 3] = static_cast<double>(pixel->weight_sum);
                out_counts[i] = pixel->sample_count;
            }
        }
        return 0;
    };
    const auto extent = renderer::RenderExtent{.width = width, .height = height};
    if (precision == 0) {
        auto film = renderer::Film::create(extent);
        if (!film) {
            set_error(film.error().message);
            return 1;
        }
        return run(*film);
    }
    auto film = renderer::ReferenceFilm::create(extent);
    if (!film) {
        set_error(film.error().message);
        return 1;
    }
    return run(*film);
}

// sobol_sample_bits / owen_scrambled_sobol_bits of the reference library; 0 on success, 1 when the
// dimension is outside the table.
__attribute__((visibility("default"))) int bfr_sobol_bits(std::uint64_t sample_index, std::uint64_t dimension,
                                                          std::uint64_t* out) {
    const auto bits = renderer::sobol_sample_bits(sample_index, dimension);
    if (!bits) {
        set_error(bits.error().message);
        return 1;
    }
    *out = *bits;
    return 0;
}

__attribute__((visibility("default"))) int bfr_owen_sobol_bits(std::uint32_t pixel_x, std::uint32_t pixel_y,
                                                               std::uint64_t sample_index, std::uint64_t seed,
                                                               std::uint64_t dimension, std::uint64_t* out) {
    const auto index = renderer::SampleStreamIndex{
        .pixel_x = pixel_x, .pixel_y = pixel_y, .sample_index = sample_index, .seed = seed};
    const auto bits = renderer::owen_scrambled_sobol_bits(index, dimension);
    if (!bits) {
        set_error(bits.error().message);
        return 1;
    }
    *out = *bits;
    return 0;
}

} // extern "C"
