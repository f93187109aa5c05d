// The reference's CUDA wavefront transport entry points, implemented over the bf200 C ABI.
//
// This translation unit replaces Blackframe/Backends/GPU/CUDA/Source/WavefrontTransport.cpp in a
// Blackframe build: it defines every member that Blackframe/Backends/GPU/CUDA/Include/Blackframe/
// Backends/GPU/CUDA/WavefrontTransport.hpp declares (CudaWavefrontTransportWorkspace and both
// trace_cuda_wavefront_transport overloads, WavefrontTransport.hpp:150-208) with the same argument
// meaning and the same refusals, so callers and the reference's own tests link against it
// unchanged. The work is done by libbf200.so (include/bf200.h):
//
//   * the workspace owns one bf200 context (bf200_context_create) with the workspace capacity as
//     its path capacity;
//   * the CudaSceneSoA's device blob is copied to the host once per distinct blob and uploaded
//     with bf200_scene_create_from_soa, which validates the v4 header and content hash and builds
//     bf200's own BLAS/TLAS; the serialized CudaSceneBvh is therefore only checked for presence
//     and device, never read;
//   * every batch goes through bf200_trace_paths_with_cones, which carries each path's depth-zero
//     initial state (throughput, radiance, eta scale) and primary ray cone, and returns the
//     terminal cones.
//
// Beyond the reference's own refusals (validate_options_and_inputs and validate_light_sampler,
// WavefrontTransport.cpp:481-626) this backend refuses, with StatusCode::unavailable and without
// substitution: input wavelength packets other than the scene blob's, and scenes
// bf200_scene_create_from_soa refuses (punctual lights, normal or bump maps, textures). Lane
// failures fail the batch as the reference's stage audits do (stage_failure,
// WavefrontTransport.cpp:875-922): numerical failures map to internal_error, unsupported lanes
// to unavailable, traversal failures to incompatible.
//
// The report fills every counting field: schema, light registry and sampler, the echoed options,
// path count, the stage lanes (camera, intersection, hit, miss, shade, shadow, continuation),
// closure and light samples, shadow queries and terminated paths. The per-stage metrics
// (dispatches, lanes and GPU time of the reference's own stage kernels) describe a kernel
// structure bf200 does not have and stay zero; device_size_bytes() is the context's device arena
// and workspaces (bf200_context_device_bytes).
#include <Blackframe/Backends/GPU/CUDA/WavefrontTransport.hpp>

#include <cuda_runtime_api.h>

#include "bf200.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <utility>
#include <vector>

namespace blackframe::engine {
namespace {

[[nodiscard]] core::Error adapter_error(const core::StatusCode code, std::string message) {
    return core::Error{.code = code, .message = std::move(message)};
}

[[nodiscard]] core::StatusCode status_code(const blackframe_status status) noexcept {
    switch (status) {
    case BLACKFRAME_STATUS_SUCCESS:
        return core::StatusCode::success;
    case BLACKFRAME_STATUS_INVALID_ARGUMENT:
        return core::StatusCode::invalid_argument;
    case BLACKFRAME_STATUS_UNSUPPORTED_ABI:
    case BLACKFRAME_STATUS_INVALID_STATE:
        return core::StatusCode::unavailable;
    case BLACKFRAME_STATUS_OUT_OF_RANGE:
        return core::StatusCode::resource_exhausted;
    case BLACKFRAME_STATUS_INTERFACE_NOT_FOUND:
        return core::StatusCode::not_found;
    default:
        return core::StatusCode::platform_error;
    }
}

[[nodiscard]] core::Error bf200_error(bf200_context* context, const blackframe_status status,
                                      const std::string& operation) {
    const char* text = context != nullptr ? bf200_context_last_error(context) : nullptr;
    return adapter_error(status_code(status), "bf200 " + operation + " failed: " +
                                                  (text != nullptr ? text : "no detail"));
}

[[nodiscard]] bool valid_transfer_mode(const CudaWavefrontTransferMode mode) noexcept {
    return mode == CudaWavefrontTransferMode::synchronous ||
           mode == CudaWavefrontTransferMode::asynchronous;
}

[[nodiscard]] bool valid_instrumentation_mode(const CudaWavefrontInstrumentationMode mode) noexcept {
    return mode == CudaWavefrontInstrumentationMode::disabled ||
           mode == CudaWavefrontInstrumentationMode::nsight;
}

// The reference's own preflight (WavefrontTransport.cpp:481-567).
[[nodiscard]] core::Status validate_options_and_inputs(const std::span<const CudaWavefrontPathInput> inputs,
                                                       const CudaWavefrontTransportOptions& options) {
    if (!valid_transfer_mode(options.transfer_mode)) {
        return std::unexpected(adapter_error(
            core::StatusCode::invalid_argument,
            "CUDA wavefront transport requires an explicit synchronous or asynchronous transfer mode."));
    }
    if (!valid_instrumentation_mode(options.instrumentation_mode)) {
        return std::unexpected(adapter_error(
            core::StatusCode::invalid_argument,
            "CUDA wavefront transport requires instrumentation to be explicitly disabled or set to Nsight."));
    }
    if (inputs.empty()) {
        return std::unexpected(adapter_error(core::StatusCode::invalid_argument,
                                             "CUDA wavefront transport requires at least one explicit path input."));
    }
    if (inputs.size() > std::numeric_limits<std::uint32_t>::max()) {
        return std::unexpected(adapter_error(
            core::StatusCode::resource_exhausted,
            "CUDA wavefront transport path count exceeds its fixed 32-bit device domain."));
    }
    if (options.heuristic != renderer::MisHeuristic::balance && options.heuristic != renderer::MisHeuristic::power) {
        return std::unexpected(adapter_error(core::StatusCode::invalid_argument,
                                             "CUDA wavefront transport requires the balance or power MIS heuristic."));
    }
    if (auto status = renderer::validate_russian_roulette_policy(options.roulette_policy); !status) {
        return std::unexpected(adapter_error(
            status.error().code,
            "CUDA wavefront transport rejected its Russian roulette policy: " + status.error().message));
    }
    for (std::size_t index = 0; index < inputs.size(); ++index) {
        const auto& input = inputs[index];
        const auto at = std::to_string(index);
        if (!std::isfinite(input.primary_cone.width()) || input.primary_cone.width() < 0.0F ||
            !std::isfinite(input.primary_cone.spread()) || input.primary_cone.spread() < 0.0F) {
            return std::unexpected(adapter_error(
                core::StatusCode::invalid_argument,
                "CUDA wavefront transport requires an explicit finite non-negative ray cone at path " + at + "."));
        }
        if (input.primary_ray.current_medium() != input.initial_state.current_medium()) {
            return std::unexpected(adapter_error(
                core::StatusCode::incompatible,
                "CUDA wavefront transport path and ray medium identities disagree at path " + at + "."));
        }
        if (input.initial_state.current_medium() != renderer::VacuumMedium) {
            return std::unexpected(adapter_error(
                core::StatusCode::invalid_argument,
                "CUDA wavefront transport currently requires vacuum rays and path states; path " + at +
                    " selected another medium."));
        }
        if (input.initial_state.depth() != 0U) {
            return std::unexpected(adapter_error(
                core::StatusCode::incompatible,
                "CUDA wavefront transport must begin at primary path depth zero; path " + at +
                    " supplied a resumed state."));
        }
        if (auto status = renderer::validate_path_depth_state(
                options.depth_limits, input.initial_state.depth_counters(), input.initial_state.depth());
            !status) {
            return std::unexpected(adapter_error(
                status.error().code,
                "CUDA wavefront transport rejected depth state at path " + at + ": " + status.error().message));
        }
        const auto finite_nonnegative = [](const renderer::TransportSpectrum& spectrum) {
            return std::ranges::all_of(spectrum.values,
                                       [](const auto value) { return std::isfinite(value) && value >= 0.0F; });
        };
        if (!finite_nonnegative(input.initial_state.beta()) ||
            !finite_nonnegative(input.initial_state.accumulated_radiance())) {
            return std::unexpected(adapter_error(
                core::StatusCode::invalid_argument,
                "CUDA wavefront transport requires finite non-negative path spectra at path " + at + "."));
        }
    }
    return {};
}

// validate_light_sampler (WavefrontTransport.cpp:575-626): the sampler is absent exactly when the
// serialized registry is empty, uniform, and sized like the registry.
[[nodiscard]] core::Result<std::uint32_t> validate_light_sampler(const xpu::shared::SceneSoaHeader& scene,
                                                                const CudaWavefrontLightSampler& light_sampler) {
    if (scene.punctual_light_count > std::numeric_limits<std::uint64_t>::max() - scene.mesh_area_light_count) {
        return std::unexpected(adapter_error(core::StatusCode::resource_exhausted,
                                             "CUDA wavefront light-registry size overflowed its serialized domain."));
    }
    const auto expected = scene.punctual_light_count + scene.mesh_area_light_count;
    if (expected == 0U) {
        if (light_sampler.has_value()) {
            return std::unexpected(adapter_error(
                core::StatusCode::incompatible,
                "CUDA wavefront transport requires the light sampler to be explicitly absent when the "
                "serialized scene light registry is empty."));
        }
        return 0U;
    }
    if (expected > std::numeric_limits<std::uint32_t>::max()) {
        return std::unexpected(adapter_error(core::StatusCode::resource_exhausted,
                                             "CUDA wavefront light registry exceeds its fixed 32-bit device domain."));
    }
    if (!light_sampler.has_value()) {
        return std::unexpected(adapter_error(
            core::StatusCode::incompatible,
            "CUDA wavefront transport requires an explicit light sampler for a non-empty serialized scene "
            "light registry."));
    }
    const auto& sampler = light_sampler->get();
    if (sampler.strategy() != renderer::LightSamplingStrategy::uniform) {
        return std::unexpected(adapter_error(
            core::StatusCode::unavailable,
            "CUDA wavefront transport currently requires an explicit uniform light sampler; the requested "
            "strategy is not ported and will not be substituted."));
    }
    if (sampler.light_count() != expected) {
        return std::unexpected(adapter_error(
            core::StatusCode::incompatible,
            "CUDA wavefront light sampler count does not match the serialized punctual and mesh-area registry."));
    }
    return static_cast<std::uint32_t>(expected);
}

// The wavelength packet of the blob's first material (material_wavelength_nanometers and
// material_wavelength_pdf, one column per lane): bf200 resolves every material at it.
[[nodiscard]] bool blob_packet(const std::vector<std::uint8_t>& blob, const xpu::shared::SceneSoaHeader& header,
                               float (&nanometers)[4], float (&pdfs)[4]) {
    if (header.material_count == 0U) {
        return false;
    }
    for (std::uint32_t lane = 0; lane < 4U; ++lane) {
        const auto& nm = header.columns[xpu::shared::scene_soa_column::material_wavelength_nanometers + lane];
        const auto& pdf = header.columns[xpu::shared::scene_soa_column::material_wavelength_pdf + lane];
        if (nm.element_size != sizeof(float) || pdf.element_size != sizeof(float) || nm.element_count == 0U ||
            pdf.element_count == 0U || nm.offset_bytes > blob.size() - sizeof(float) ||
            pdf.offset_bytes > blob.size() - sizeof(float)) {
            return false;
        }
        std::memcpy(&nanometers[lane], blob.data() + nm.offset_bytes, sizeof(float));
        std::memcpy(&pdfs[lane], blob.data() + pdf.offset_bytes, sizeof(float));
    }
    return true;
}

[[nodiscard]] CudaWavefrontPathTermination termination_of(const std::uint32_t code) noexcept {
    switch (code) {
    case BF200_TERMINATION_DEPTH_LIMIT:
        return CudaWavefrontPathTermination::depth_limit;
    case BF200_TERMINATION_OUTSIDE_BSDF_SUPPORT:
        return CudaWavefrontPathTermination::outside_bsdf_support;
    case BF200_TERMINATION_ZERO_THROUGHPUT:
        return CudaWavefrontPathTermination::zero_throughput;
    case BF200_TERMINATION_RUSSIAN_ROULETTE:
        return CudaWavefrontPathTermination::russian_roulette;
    default:
        return CudaWavefrontPathTermination::escaped_environment;
    }
}

[[nodiscard]] core::StatusCode lane_status_code(const std::uint32_t lane_status) noexcept {
    switch (lane_status) {
    case BF200_LANE_UNSUPPORTED:
        return core::StatusCode::unavailable;
    case BF200_LANE_TRAVERSAL_FAILURE:
        return core::StatusCode::incompatible;
    default:
        return core::StatusCode::internal_error;
    }
}

}  // namespace

struct CudaWavefrontTransportWorkspace::Storage final {
    bf200_context* context{};
    std::size_t capacity{};
    std::int32_t device{};
    CudaWavefrontTransferMode transfer_mode{CudaWavefrontTransferMode::synchronous};
    CudaWavefrontInstrumentationMode instrumentation_mode{CudaWavefrontInstrumentationMode::disabled};
    // the bf200 scene of the last CudaSceneSoA, keyed by its device bytes, size and content hash
    bf200_scene* scene{};
    const std::uint8_t* scene_bytes{};
    std::size_t scene_size{};
    std::uint64_t scene_hash{};
    float scene_nanometers[4]{};
    float scene_pdfs[4]{};
    // host staging reused across batches
    std::vector<std::uint8_t> blob;
    std::vector<bf200_path_input_v1> inputs;
    std::vector<bf200_path_state_v1> states;
    std::vector<bf200_ray_cone_v1> primary_cones;
    std::vector<bf200_ray_cone_v1> terminal_cones;
    std::vector<bf200_path_result_v1> results;

    [[nodiscard]] core::Status release() {
        core::Status first{};
        if (scene != nullptr) {
            if (const auto status = bf200_scene_destroy(scene); status != BLACKFRAME_STATUS_SUCCESS) {
                first = std::unexpected(bf200_error(context, status, "scene destroy"));
            }
            scene = nullptr;
        }
        if (context != nullptr) {
            if (const auto status = bf200_context_destroy(context); status != BLACKFRAME_STATUS_SUCCESS && first) {
                first = std::unexpected(adapter_error(status_code(status), "bf200 context destroy failed"));
            }
            context = nullptr;
        }
        return first;
    }
};

CudaWavefrontTransportWorkspace::CudaWavefrontTransportWorkspace(std::unique_ptr<Storage> storage) noexcept
    : storage_{std::move(storage)} {}

CudaWavefrontTransportWorkspace::CudaWavefrontTransportWorkspace(CudaWavefrontTransportWorkspace&& other) noexcept
    : storage_{std::move(other.storage_)} {}

CudaWavefrontTransportWorkspace::~CudaWavefrontTransportWorkspace() noexcept {
    if (storage_ != nullptr) {
        static_cast<void>(storage_->release());
    }
}

core::Result<CudaWavefrontTransportWorkspace>
CudaWavefrontTransportWorkspace::create(const std::size_t capacity, const xpu::cuda::DeviceMemoryBudget device_memory_budget,
                                        const CudaWavefrontTransferMode transfer_mode,
                                        const CudaWavefrontInstrumentationMode instrumentation_mode) try {
    static_cast<void>(device_memory_budget);  // bf200 sizes its own arena from the capacity
    if (!valid_transfer_mode(transfer_mode)) {
        return std::unexpected(adapter_error(
            core::StatusCode::invalid_argument,
            "CUDA wavefront workspace requires an explicit synchronous or asynchronous transfer mode."));
    }
    if (!valid_instrumentation_mode(instrumentation_mode)) {
        return std::unexpected(adapter_error(
            core::StatusCode::invalid_argument,
            "CUDA wavefront workspace requires instrumentation to be explicitly disabled or set to Nsight."));
    }
    if (capacity == 0U) {
        return std::unexpected(adapter_error(core::StatusCode::invalid_argument,
                                             "CUDA wavefront transport workspace capacity must be non-zero."));
    }
    if (capacity > std::numeric_limits<std::uint32_t>::max()) {
        return std::unexpected(adapter_error(
            core::StatusCode::resource_exhausted,
            "CUDA wavefront transport workspace capacity exceeds its 32-bit device domain."));
    }
    auto storage = std::make_unique<Storage>();
    if (cudaGetDevice(&storage->device) != cudaSuccess) {
        return std::unexpected(adapter_error(core::StatusCode::platform_error, "no current CUDA device"));
    }
    storage->capacity = capacity;
    storage->transfer_mode = transfer_mode;
    storage->instrumentation_mode = instrumentation_mode;
    if (const auto status = bf200_context_create(storage->device, capacity, &storage->context);
        status != BLACKFRAME_STATUS_SUCCESS) {
        return std::unexpected(adapter_error(status_code(status), "bf200 context creation failed"));
    }
    return CudaWavefrontTransportWorkspace{std::move(storage)};
} catch (const std::bad_alloc&) {
    return std::unexpected(adapter_error(core::StatusCode::resource_exhausted,
                                         "CUDA wavefront workspace exhausted host memory."));
}

std::size_t CudaWavefrontTransportWorkspace::capacity() const noexcept {
    return storage_ != nullptr ? storage_->capacity : 0U;
}

std::size_t CudaWavefrontTransportWorkspace::device_size_bytes() const noexcept {
    std::uint64_t bytes = 0;
    if (storage_ == nullptr || storage_->context == nullptr ||
        bf200_context_device_bytes(storage_->context, &bytes) != BLACKFRAME_STATUS_SUCCESS) {
        return 0U;
    }
    return static_cast<std::size_t>(bytes);
}

std::int32_t CudaWavefrontTransportWorkspace::device_ordinal() const noexcept {
    return storage_ != nullptr ? storage_->device : -1;
}

CudaWavefrontTransferMode CudaWavefrontTransportWorkspace::transfer_mode() const noexcept {
    return storage_ != nullptr ? storage_->transfer_mode : CudaWavefrontTransferMode::synchronous;
}

CudaWavefrontInstrumentationMode CudaWavefrontTransportWorkspace::instrumentation_mode() const noexcept {
    return storage_ != nullptr ? storage_->instrumentation_mode : CudaWavefrontInstrumentationMode::disabled;
}

CudaWavefrontTransportWorkspace::operator bool() const noexcept {
    return storage_ != nullptr && storage_->context != nullptr;
}

core::Status CudaWavefrontTransportWorkspace::close() {
    if (storage_ == nullptr) {
        return {};
    }
    auto status = storage_->release();
    storage_.reset();
    return status;
}

core::Result<CudaWavefrontTransportBatch>
trace_cuda_wavefront_transport(CudaWavefrontTransportWorkspace& workspace, const CudaSceneSoA& scene,
                               const CudaSceneBvh& bvh, const std::span<const CudaWavefrontPathInput> inputs,
                               const CudaWavefrontLightSampler light_sampler,
                               const CudaWavefrontTransportOptions options) try {
    if (!workspace) {
        return std::unexpected(adapter_error(core::StatusCode::invalid_argument,
                                             "CUDA wavefront transport requires an open workspace."));
    }
    auto& storage = *workspace.storage_;
    if (!scene || !bvh || scene.device_ordinal() != storage.device || bvh.device_ordinal() != storage.device) {
        return std::unexpected(adapter_error(
            core::StatusCode::incompatible,
            "CUDA wavefront transport requires a scene and BVH resident on the workspace's device."));
    }
    if (auto status = validate_options_and_inputs(inputs, options); !status) {
        return std::unexpected(std::move(status.error()));
    }
    const auto light_count = validate_light_sampler(scene.header(), light_sampler);
    if (!light_count) {
        return std::unexpected(light_count.error());
    }
    if (storage.transfer_mode != options.transfer_mode ||
        storage.instrumentation_mode != options.instrumentation_mode) {
        return std::unexpected(adapter_error(
            core::StatusCode::incompatible,
            "CUDA wavefront transport modes do not match its reusable workspace; the requested mode was not "
            "substituted."));
    }
    if (inputs.size() > storage.capacity) {
        return std::unexpected(adapter_error(core::StatusCode::resource_exhausted,
                                             "CUDA wavefront transport path count exceeds the reusable workspace capacity."));
    }

    // the bf200 scene of this blob (uploaded once per distinct blob)
    const auto& header = scene.header();
    if (storage.scene == nullptr || storage.scene_bytes != scene.device_data() ||
        storage.scene_size != scene.size_bytes() || storage.scene_hash != header.content_hash) {
        if (storage.scene != nullptr) {
            static_cast<void>(bf200_scene_destroy(storage.scene));
            storage.scene = nullptr;
        }
        storage.blob.resize(scene.size_bytes());
        if (const auto e = cudaMemcpy(storage.blob.data(), scene.device_data(), scene.size_bytes(),
                                      cudaMemcpyDeviceToHost);
            e != cudaSuccess) {
            return std::unexpected(adapter_error(core::StatusCode::platform_error,
                                                 std::string{"scene blob download failed: "} + cudaGetErrorString(e)));
        }
        char message[512] = {};
        if (const auto status = bf200_scene_create_from_soa(storage.context, storage.blob.data(), storage.blob.size(),
                                                            &storage.scene, message, sizeof(message));
            status != BLACKFRAME_STATUS_SUCCESS) {
            storage.scene = nullptr;
            return std::unexpected(adapter_error(status_code(status), std::string{"bf200 scene upload: "} + message));
        }
        if (!blob_packet(storage.blob, header, storage.scene_nanometers, storage.scene_pdfs)) {
            std::fill(std::begin(storage.scene_nanometers), std::end(storage.scene_nanometers), 0.0F);
        }
        storage.scene_bytes = scene.device_data();
        storage.scene_size = scene.size_bytes();
        storage.scene_hash = header.content_hash;
    }

    // inputs: primary ray, sample, cone and the depth-zero initial state
    const auto n = inputs.size();
    storage.inputs.assign(n, bf200_path_input_v1{});
    storage.states.assign(n, bf200_path_state_v1{});
    storage.primary_cones.resize(n);
    storage.terminal_cones.resize(n);
    storage.results.resize(n);
    for (std::size_t i = 0; i < n; ++i) {
        const auto& input = inputs[i];
        const auto& state = input.initial_state;
        auto& initial = storage.states[i];
        initial.eta_scale = state.eta_scale();
        for (std::size_t lane = 0; lane < 4; ++lane) {
            initial.beta[lane] = state.beta().values[lane];
            initial.radiance[lane] = state.accumulated_radiance().values[lane];
            const auto& w = state.wavelengths()[lane];
            if (storage.scene_nanometers[lane] != 0.0F &&
                (w.nanometers != storage.scene_nanometers[lane] || w.probability.value != storage.scene_pdfs[lane])) {
                return std::unexpected(adapter_error(
                    core::StatusCode::unavailable,
                    "bf200 resolves the scene at the blob's wavelength packet; path " + std::to_string(i) +
                        " carries another packet, which is not substituted."));
            }
        }
        auto& out = storage.inputs[i];
        const auto& ray = input.primary_ray;
        out.primary_ray.origin[0] = ray.origin().x;
        out.primary_ray.origin[1] = ray.origin().y;
        out.primary_ray.origin[2] = ray.origin().z;
        out.primary_ray.direction[0] = ray.direction().x;
        out.primary_ray.direction[1] = ray.direction().y;
        out.primary_ray.direction[2] = ray.direction().z;
        out.primary_ray.t_min = ray.t_min();
        out.primary_ray.t_max = ray.t_max();
        out.primary_ray.time = ray.time();
        out.primary_ray.mask = ray.mask();
        out.primary_ray.medium = ray.current_medium().value;
        out.sample.pixel_x = input.sample.pixel_x;
        out.sample.pixel_y = input.sample.pixel_y;
        out.sample.sample_index = input.sample.sample_index;
        out.sample.seed = input.sample.seed;
        storage.primary_cones[i] = bf200_ray_cone_v1{input.primary_cone.width(), input.primary_cone.spread()};
    }

    bf200_transport_options_v1 bf{};
    bf.struct_size = sizeof(bf);
    bf.mis_heuristic = options.heuristic == renderer::MisHeuristic::power ? 1U : 0U;
    bf.depth_limits[0] = options.depth_limits.diffuse;
    bf.depth_limits[1] = options.depth_limits.glossy;
    bf.depth_limits[2] = options.depth_limits.specular;
    bf.depth_limits[3] = options.depth_limits.transmission;
    bf.depth_limits[4] = options.depth_limits.volume;
    bf.roulette_enabled = options.roulette_policy.is_enabled() ? 1U : 0U;
    bf.roulette_first_eligible_depth = options.roulette_policy.first_eligible_depth();
    bf.roulette_minimum_survival = options.roulette_policy.minimum_survival_probability();
    bf.roulette_maximum_survival = options.roulette_policy.maximum_survival_probability();
    bf.instrumentation = options.instrumentation_mode == CudaWavefrontInstrumentationMode::nsight ? 1U : 0U;
    bf.sampler = BF200_SAMPLER_HASH;

    bf200_report_v1 report{};
    report.struct_size = sizeof(report);
    if (const auto status = bf200_trace_paths_with_cones(storage.context, storage.scene, storage.inputs.data(),
                                                         storage.states.data(), storage.primary_cones.data(), n, &bf,
                                                         storage.results.data(), storage.terminal_cones.data(),
                                                         &report);
        status != BLACKFRAME_STATUS_SUCCESS) {
        return std::unexpected(bf200_error(storage.context, status, "trace"));
    }
    if (report.failed_lanes != 0U) {
        const auto path = report.first_failure_path;
        return std::unexpected(adapter_error(
            lane_status_code(report.first_failure_status),
            "CUDA wavefront transport failed at path " + std::to_string(path) + " (bf200 lane status " +
                std::to_string(report.first_failure_status) + ", " + std::to_string(report.failed_lanes) +
                " failed lanes)."));
    }

    CudaWavefrontTransportBatch batch;
    batch.paths.reserve(n);
    batch.terminal_cones.reserve(n);
    for (std::size_t i = 0; i < n; ++i) {
        const auto& r = storage.results[i];
        const auto& input = inputs[i];
        renderer::TransportSpectrum beta{}, radiance{};
        for (std::size_t lane = 0; lane < 4; ++lane) {
            beta.values[lane] = r.beta[lane];
            radiance.values[lane] = r.radiance[lane];
        }
        const renderer::PathDepthCounters counters{.diffuse = r.depth_counters[0],
                                                   .glossy = r.depth_counters[1],
                                                   .specular = r.depth_counters[2],
                                                   .transmission = r.depth_counters[3],
                                                   .volume = r.depth_counters[4]};
        auto state = renderer::PathState::create(beta, radiance, counters, r.eta_scale,
                                                 input.initial_state.wavelengths(),
                                                 static_cast<renderer::PathDeltaFlags>(r.delta_flags),
                                                 input.initial_state.current_medium());
        if (!state) {
            return std::unexpected(adapter_error(core::StatusCode::internal_error,
                                                 "CUDA wavefront terminal state " + std::to_string(i) +
                                                     " is not representable: " + state.error().message));
        }
        const auto& t = r.terminal_ray;
        auto terminal = renderer::Ray::create(
            renderer::Point3{.x = t.origin[0], .y = t.origin[1], .z = t.origin[2]},
            renderer::Vector3{.x = t.direction[0], .y = t.direction[1], .z = t.direction[2]}, t.t_min, t.t_max,
            t.time, t.mask, renderer::MediumId{.value = t.medium});
        if (!terminal) {
            return std::unexpected(adapter_error(core::StatusCode::internal_error,
                                                 "CUDA wavefront terminal ray " + std::to_string(i) +
                                                     " is not representable: " + terminal.error().message));
        }
        auto cone = renderer::RayCone::create(storage.terminal_cones[i].width, storage.terminal_cones[i].spread);
        if (!cone) {
            return std::unexpected(adapter_error(core::StatusCode::internal_error,
                                                 "CUDA wavefront terminal ray cone " + std::to_string(i) +
                                                     " is not representable: " + cone.error().message));
        }
        batch.paths.push_back(CudaWavefrontPathResult{
            .state = *state,
            .terminal_ray = *terminal,
            .termination = termination_of(r.termination),
            .blocked_depth_limits = static_cast<renderer::ScatteringLobe>(r.blocked_depth_limits),
        });
        batch.terminal_cones.push_back(*cone);
    }

    auto& out = batch.report;
    out.schema_version = CurrentCudaWavefrontTransportReportSchemaVersion;
    out.has_light_sampler = light_sampler.has_value();
    out.registered_light_count = *light_count;
    out.heuristic = options.heuristic;
    out.light_sampling_strategy = renderer::LightSamplingStrategy::uniform;
    out.depth_limits = options.depth_limits;
    out.roulette_policy = options.roulette_policy;
    out.path_count = n;
    out.transfer_mode = options.transfer_mode;
    out.instrumentation_mode = options.instrumentation_mode;
    // every traced extension segment either hit (and was shaded) or missed
    out.stage_lanes.camera = n;
    out.stage_lanes.intersection = report.extension_segments;
    out.stage_lanes.miss = report.miss_segments;
    out.stage_lanes.hit = report.extension_segments - std::min(report.extension_segments, report.miss_segments);
    out.stage_lanes.shade = out.stage_lanes.hit;
    out.stage_lanes.shadow = report.shadow_segments;
    out.stage_lanes.continuation = report.continuation_segments;
    out.closure_samples = report.closure_samples;
    out.light_samples = report.light_samples;
    out.shadow_queries = report.shadow_segments;
    out.terminated_paths = report.terminated_paths;
    return batch;
} catch (const std::bad_alloc&) {
    return std::unexpected(adapter_error(core::StatusCode::resource_exhausted,
                                         "CUDA wavefront transport exhausted host memory."));
}

core::Result<CudaWavefrontTransportBatch>
trace_cuda_wavefront_transport(const CudaSceneSoA& scene, const CudaSceneBvh& bvh,
                               const std::span<const CudaWavefrontPathInput> inputs,
                               const CudaWavefrontLightSampler light_sampler,
                               const CudaWavefrontTransportOptions options) {
    // the reference's preflight before any per-call storage (WavefrontTransport.cpp:2836-2856)
    if (auto status = validate_options_and_inputs(inputs, options); !status) {
        return std::unexpected(std::move(status.error()));
    }
    if (scene) {
        if (auto count = validate_light_sampler(scene.header(), light_sampler); !count) {
            return std::unexpected(count.error());
        }
    }
    auto workspace = CudaWavefrontTransportWorkspace::create(inputs.size(), options.device_memory_budget,
                                                             options.transfer_mode, options.instrumentation_mode);
    if (!workspace) {
        return std::unexpected(std::move(workspace.error()));
    }
    auto traced = trace_cuda_wavefront_transport(*workspace, scene, bvh, inputs, light_sampler, options);
    auto closed = workspace->close();
    if (!traced) {
        return traced;
    }
    if (!closed) {
        return std::unexpected(std::move(closed.error()));
    }
    return traced;
}

}  // namespace blackframe::engine
