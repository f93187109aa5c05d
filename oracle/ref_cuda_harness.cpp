// Test-infrastructure harness around the reference's own CUDA backend.
//
// Compiled by oracle/Makefile (target `refcuda`) together with the reference's CUDA sources,
// unchanged, for sm_100a (Blackframe/XPU/CUDA/Source/*.cu, Blackframe/XPU/CUDA/Host/Source,
// Blackframe/Backends/GPU/CUDA/Source) and the reference Core/Renderer/Engine objects of the
// `ref` target, into oracle/_ref/libbfrefcuda.so. Never shipped, never called by the product:
// the GPU tests use it as the hit-identifier checker, bench.py as the reference CUDA arm. It
// drives the reference's public entry points exactly as its benchmark does
// (Benchmarks/Renderer/CudaWavefrontTransportBenchmark.cpp:163-393):
//
//   * CudaSceneSoA::upload            (Blackframe/Backends/GPU/CUDA/Source/SceneSoA.cpp)
//   * CudaSceneBvh::build             (Blackframe/Backends/GPU/CUDA/Source/SceneBvh.cpp:1109)
//   * trace_cuda_closest_hits         (Blackframe/Backends/GPU/CUDA/Include/.../ClosestHit.hpp:21-28)
//   * CudaWavefrontTransportWorkspace::create + trace_cuda_wavefront_transport
//                                     (WavefrontTransport.hpp:147-208), with a reused workspace
#include "ref_scene.hpp"

#include <Blackframe/Backends/GPU/CUDA/ClosestHit.hpp>
#include <Blackframe/Backends/GPU/CUDA/SceneBvh.hpp>
#include <Blackframe/Backends/GPU/CUDA/SceneSoA.hpp>
#include <Blackframe/Backends/GPU/CUDA/WavefrontTransport.hpp>
#include <Blackframe/Renderer/LightSampler.hpp>
#include <Blackframe/Renderer/PathState.hpp>

#include <cuda_runtime_api.h>

#include <chrono>
#include <cstring>
#include <memory>
#include <optional>
#include <string>
#include <vector>

namespace {

using namespace blackframe;
using namespace bfref;

std::string g_last_error;

struct RefCudaScene {
    engine::FrameSceneHandle scene;
    std::unique_ptr<renderer::LightSampler> sampler;
    std::optional<engine::CudaSceneSoA> soa;
    std::optional<engine::CudaSceneBvh> bvh;
    std::optional<engine::CudaWavefrontTransportWorkspace> workspace;
    std::size_t workspace_paths = 0;
    renderer::SampledWavelengths wavelengths{};
    std::vector<uint32_t> instance_ids;  // committed order
    double upload_ms = 0.0;
    double build_ms = 0.0;
};

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

engine::CudaWavefrontTransportOptions make_options(const bf200_transport_options_v1& o,
                                                   const renderer::RussianRoulettePolicy& policy) {
    auto options = engine::CudaWavefrontTransportOptions{};
    options.heuristic = o.mis_heuristic == 1 ? renderer::MisHeuristic::power : renderer::MisHeuristic::balance;
    options.depth_limits = renderer::PathDepthLimits{
        .diffuse = o.depth_limits[0],
        .glossy = o.depth_limits[1],
        .specular = o.depth_limits[2],
        .transmission = o.depth_limits[3],
        .volume = o.depth_limits[4],
    };
    options.roulette_policy = policy;
    options.transfer_mode = engine::CudaWavefrontTransferMode::synchronous;
    return options;
}

// The reference's per-path inputs: the primary ray, its cone (the caller's, or a zero-width cone of
// slope `spread`), PathState::create_initial and the sample stream index.
bool make_inputs(const RefCudaScene& s, const bf200_path_input_v1* inputs, const float* cones, uint64_t n,
                 std::vector<engine::CudaWavefrontPathInput>& out) {
    const auto initial = renderer::PathState::create_initial(s.wavelengths, renderer::VacuumMedium);
    if (!initial) {
        g_last_error = "initial state: " + initial.error().message;
        return false;
    }
    out.clear();
    out.reserve(n);
    for (uint64_t k = 0; k < n; ++k) {
        const float width = cones != nullptr ? cones[2 * k] : 0.0F;
        const float spread = cones != nullptr ? cones[2 * k + 1] : 0.0F;
        const auto cone = renderer::RayCone::create(width, spread);
        if (!cone) {
            g_last_error = "primary cone: " + cone.error().message;
            return false;
        }
        out.push_back(engine::CudaWavefrontPathInput{
            .primary_ray = make_ray(inputs[k].primary_ray),
            .primary_cone = *cone,
            .initial_state = *initial,
            .sample = renderer::SampleStreamIndex{.pixel_x = inputs[k].sample.pixel_x,
                                                  .pixel_y = inputs[k].sample.pixel_y,
                                                  .sample_index = inputs[k].sample.sample_index,
                                                  .seed = inputs[k].sample.seed},
        });
    }
    return true;
}

bool ensure_workspace(RefCudaScene& s, std::size_t paths) {
    if (s.workspace && s.workspace_paths >= paths) {
        return true;
    }
    if (s.workspace) {
        static_cast<void>(s.workspace->close());
        s.workspace.reset();
    }
    auto created = engine::CudaWavefrontTransportWorkspace::create(paths, xpu::cuda::DeviceMemoryBudget{},
                                                                   engine::CudaWavefrontTransferMode::synchronous);
    if (!created) {
        g_last_error = "workspace: " + created.error().message;
        return false;
    }
    s.workspace.emplace(std::move(*created));
    s.workspace_paths = paths;
    return true;
}

void store_result(const engine::CudaWavefrontPathResult& r, bf200_path_result_v1& out) {
    std::memset(&out, 0, sizeof(out));
    const auto& st = r.state;
    for (std::size_t lane = 0; lane < 4; ++lane) {
        out.beta[lane] = st.beta()[lane];
        out.radiance[lane] = st.accumulated_radiance()[lane];
    }
    out.depth = st.depth();
    out.depth_counters[0] = st.depth_counters().diffuse;
    out.depth_counters[1] = st.depth_counters().glossy;
    out.depth_counters[2] = st.depth_counters().specular;
    out.depth_counters[3] = st.depth_counters().transmission;
    out.depth_counters[4] = st.depth_counters().volume;
    out.eta_scale = st.eta_scale();
    out.delta_flags = static_cast<uint32_t>(st.delta_flags());
    // CudaWavefrontPathTermination numbers zero throughput 2 and outside-support 3; bf200 follows
    // BsdfOnlyPathTermination (outside-support 2, zero throughput 3)
    switch (r.termination) {
    case engine::CudaWavefrontPathTermination::escaped_environment:
        out.termination = BF200_TERMINATION_ESCAPED_ENVIRONMENT;
        break;
    case engine::CudaWavefrontPathTermination::depth_limit:
        out.termination = BF200_TERMINATION_DEPTH_LIMIT;
        break;
    case engine::CudaWavefrontPathTermination::zero_throughput:
        out.termination = BF200_TERMINATION_ZERO_THROUGHPUT;
        break;
    case engine::CudaWavefrontPathTermination::outside_bsdf_support:
        out.termination = BF200_TERMINATION_OUTSIDE_BSDF_SUPPORT;
        break;
    case engine::CudaWavefrontPathTermination::russian_roulette:
        out.termination = BF200_TERMINATION_RUSSIAN_ROULETTE;
        break;
    }
    out.blocked_depth_limits = static_cast<uint32_t>(r.blocked_depth_limits);
    out.lane_status = BF200_LANE_OK;
    store_ray(r.terminal_ray, out.terminal_ray);
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) const char* bfrc_last_error() { return g_last_error.c_str(); }

// Builds the FrameScene of `desc`, the uniform light sampler, the device scene blob and its BVH.
// Returns 0, or a non-zero stage code with the reference's message in bfrc_last_error().
__attribute__((visibility("default"))) int bfrc_scene_create(const bf200_scene_desc_v1* desc, void** out_scene) {
    if (desc == nullptr || out_scene == nullptr) {
        g_last_error = "null argument";
        return 1;
    }
    std::string error;
    int code = 0;
    auto scene = make_frame_scene(desc, error, &code);
    if (!scene) {
        g_last_error = error;
        return code;
    }
    auto sampler = renderer::LightSampler::create_uniform(scene->punctual_lights().size() +
                                                          scene->mesh_area_lights().size());
    if (!sampler) {
        g_last_error = "light sampler: " + sampler.error().message;
        return 6;
    }
    auto result = std::make_unique<RefCudaScene>();
    result->scene = scene;
    result->sampler = std::make_unique<renderer::LightSampler>(std::move(*sampler));
    result->wavelengths = make_wavelengths(desc->wavelength_nanometers, desc->wavelength_pdf);
    for (const auto& instance : scene->instances()) {
        result->instance_ids.push_back(instance.id.value);
    }
    double t0 = now_ms();
    auto soa = engine::CudaSceneSoA::upload(*scene);
    if (!soa) {
        g_last_error = "CudaSceneSoA::upload: " + soa.error().message;
        return 7;
    }
    result->upload_ms = now_ms() - t0;
    result->soa.emplace(std::move(*soa));
    t0 = now_ms();
    auto bvh = engine::CudaSceneBvh::build(*result->soa);
    if (!bvh) {
        g_last_error = "CudaSceneBvh::build: " + bvh.error().message;
        return 8;
    }
    result->build_ms = now_ms() - t0;
    result->bvh.emplace(std::move(*bvh));
    *out_scene = result.release();
    return 0;
}

__attribute__((visibility("default"))) void bfrc_scene_destroy(void* handle) {
    auto* s = static_cast<RefCudaScene*>(handle);
    if (s == nullptr) {
        return;
    }
    if (s->workspace) {
        static_cast<void>(s->workspace->close());
    }
    if (s->bvh) {
        static_cast<void>(s->bvh->close());
    }
    if (s->soa) {
        static_cast<void>(s->soa->close());
    }
    delete s;
}

// Host milliseconds of the scene upload and of the BVH build, and the device bytes of each.
__attribute__((visibility("default"))) void bfrc_scene_stats(void* handle, double* upload_ms, double* build_ms,
                                                             uint64_t* scene_bytes, uint64_t* bvh_bytes) {
    const auto* s = static_cast<RefCudaScene*>(handle);
    *upload_ms = s->upload_ms;
    *build_ms = s->build_ms;
    *scene_bytes = s->soa->size_bytes();
    *bvh_bytes = s->bvh->size_bytes();
}

// Closest hits of world rays through the reference CUDA traversal; per ray t, barycentrics, the
// committed instance index and the primitive index (both 0xffffffff on a miss), status 0.
__attribute__((visibility("default"))) int bfrc_closest_hits(void* handle, const bf200_ray_v1* rays, uint64_t n,
                                                             bf200_hit_v1* hits) {
    auto* s = static_cast<RefCudaScene*>(handle);
    std::vector<renderer::Ray> batch;
    batch.reserve(n);
    for (uint64_t k = 0; k < n; ++k) {
        batch.push_back(make_ray(rays[k]));
    }
    auto result = engine::trace_cuda_closest_hits(*s->soa, *s->bvh, batch);
    if (!result) {
        g_last_error = "trace_cuda_closest_hits: " + result.error().message;
        return 1;
    }
    for (uint64_t k = 0; k < n; ++k) {
        std::memset(&hits[k], 0, sizeof(hits[k]));
        const auto& hit = (*result)[k];
        if (!hit) {
            hits[k].instance_index = 0xFFFFFFFFU;
            hits[k].primitive_index = 0xFFFFFFFFU;
            continue;
        }
        hits[k].t = hit->triangle.parameter;
        hits[k].barycentrics[0] = hit->triangle.barycentrics.vertex0;
        hits[k].barycentrics[1] = hit->triangle.barycentrics.vertex1;
        hits[k].barycentrics[2] = hit->triangle.barycentrics.vertex2;
        hits[k].instance_index = 0xFFFFFFFFU;
        for (uint32_t i = 0; i < s->instance_ids.size(); ++i) {
            if (s->instance_ids[i] == hit->identifiers.instance.value) {
                hits[k].instance_index = i;
                break;
            }
        }
        hits[k].primitive_index = hit->identifiers.primitive.value;
    }
    return 0;
}

// One trace_cuda_wavefront_transport call over `n` paths on the scene's reused workspace (grown to
// n paths when smaller). cones: 2 floats per path or null (zero cones). Results and the report's
// counts are written when the pointers are given; *milliseconds receives the host wall time of
// the call (which returns after its device work and result download).
__attribute__((visibility("default"))) int bfrc_trace(void* handle, const bf200_path_input_v1* inputs,
                                                      const float* cones, uint64_t n,
                                                      const bf200_transport_options_v1* options,
                                                      bf200_path_result_v1* results, bf200_report_v1* report,
                                                      double* milliseconds) {
    auto* s = static_cast<RefCudaScene*>(handle);
    auto policy = make_policy(*options);
    if (!policy) {
        g_last_error = "roulette: " + policy.error().message;
        return 1;
    }
    std::vector<engine::CudaWavefrontPathInput> batch;
    if (!make_inputs(*s, inputs, cones, n, batch) || !ensure_workspace(*s, n)) {
        return 2;
    }
    const auto o = make_options(*options, *policy);
    cudaDeviceSynchronize();
    const double t0 = now_ms();
    auto traced = engine::trace_cuda_wavefront_transport(*s->workspace, *s->soa, *s->bvh, batch,
                                                         engine::CudaWavefrontLightSampler{std::cref(*s->sampler)}, o);
    cudaDeviceSynchronize();
    if (milliseconds != nullptr) {
        *milliseconds = now_ms() - t0;
    }
    if (!traced) {
        g_last_error = "trace_cuda_wavefront_transport: " + traced.error().message;
        return 3;
    }
    if (results != nullptr) {
        for (uint64_t k = 0; k < n; ++k) {
            store_result(traced->paths[k], results[k]);
        }
    }
    if (report != nullptr) {
        std::memset(report, 0, sizeof(*report));
        report->struct_size = sizeof(*report);
        report->registered_light_count = traced->report.registered_light_count;
        report->path_count = traced->report.path_count;
        report->extension_segments = traced->report.stage_lanes.intersection;
        report->shadow_segments = traced->report.stage_lanes.shadow;
        report->closure_samples = traced->report.closure_samples;
        report->light_samples = traced->report.light_samples;
        report->terminated_paths = traced->report.terminated_paths;
        report->miss_segments = traced->report.stage_lanes.miss;
        report->continuation_segments = traced->report.stage_lanes.continuation;
    }
    return 0;
}

}  // extern "C"
