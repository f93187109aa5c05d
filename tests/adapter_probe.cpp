// CPU checks of the C++ adapter's own logic (blackframe-renderer_b200/adapter/WavefrontTransport.cpp),
// built by tests/test_adapter.py against the reference headers and the reference's compiled CPU
// libraries: the preflight of the reference (codes and message fragments), the light-sampler
// checks against a serialized header, the status and termination mappings, and a workspace that
// cannot be created without a CUDA device. The adapter source is included so its internal
// functions can be called; nothing here touches a GPU. Prints one line per check and exits
// non-zero when one fails.
#include "../blackframe-renderer_b200/adapter/WavefrontTransport.cpp"

#include <cstdio>
#include <string_view>

namespace {

using namespace blackframe;
using engine::CudaWavefrontPathInput;
using engine::CudaWavefrontTransportOptions;

int failures = 0;

void check(bool ok, const char* name) {
    std::printf("%s %s\n", ok ? "ok" : "FAIL", name);
    failures += ok ? 0 : 1;
}

template <typename Result>
bool refused(const Result& r, core::StatusCode code, std::string_view fragment) {
    return !r.has_value() && r.error().code == code && r.error().message.find(fragment) != std::string::npos;
}

CudaWavefrontPathInput input(float cone_width = 0.0F, std::uint32_t medium = 0U) {
    const auto wavelengths = renderer::sample_uniform_visible_wavelengths(0.25F);
    const auto ray = renderer::Ray::create(renderer::Point3{.z = 1.0F}, renderer::Vector3{.z = -1.0F}, 0.0F,
                                           std::numeric_limits<float>::infinity(), 0.5F, renderer::AllRayVisibility,
                                           renderer::MediumId{.value = medium});
    const auto cone = renderer::RayCone::create(cone_width, 0.25F);
    const auto state = renderer::PathState::create_initial(*wavelengths, renderer::MediumId{.value = medium});
    return CudaWavefrontPathInput{.primary_ray = *ray,
                                  .primary_cone = *cone,
                                  .initial_state = *state,
                                  .sample = renderer::SampleStreamIndex{.pixel_x = 1, .pixel_y = 2}};
}

}  // namespace

int main() {
    using engine::validate_options_and_inputs;
    const CudaWavefrontTransportOptions options{};
    const std::vector<CudaWavefrontPathInput> one{input()};
    check(validate_options_and_inputs(one, options).has_value(), "preflight accepts a primary path");
    check(refused(validate_options_and_inputs({}, options), core::StatusCode::invalid_argument,
                  "at least one explicit path input"),
          "preflight refuses an empty batch");
    const std::vector<CudaWavefrontPathInput> medium{input(0.0F, 3U)};
    check(refused(validate_options_and_inputs(medium, options), core::StatusCode::invalid_argument,
                  "requires vacuum rays"),
          "preflight refuses a non-vacuum path");
    auto bad_transfer = options;
    bad_transfer.transfer_mode = static_cast<engine::CudaWavefrontTransferMode>(7);
    check(refused(validate_options_and_inputs(one, bad_transfer), core::StatusCode::invalid_argument,
                  "transfer mode"),
          "preflight refuses an unknown transfer mode");
    auto bad_mis = options;
    bad_mis.heuristic = static_cast<renderer::MisHeuristic>(9);
    check(refused(validate_options_and_inputs(one, bad_mis), core::StatusCode::invalid_argument, "MIS heuristic"),
          "preflight refuses an unknown MIS heuristic");

    // light samplers against a serialized registry
    xpu::shared::SceneSoaHeader header{};
    const auto uniform2 = renderer::LightSampler::create_uniform(2);
    const auto uniform3 = renderer::LightSampler::create_uniform(3);
    using Spectrum = renderer::LightSpectrumT<renderer::TransportScalar>;
    const std::vector<Spectrum> powers(2, Spectrum{.values = {1, 1, 1, 1}});
    const auto power2 = renderer::LightSampler::create_power_weighted(powers);
    check(engine::validate_light_sampler(header, std::nullopt).value_or(99U) == 0U, "an empty registry takes no sampler");
    check(refused(engine::validate_light_sampler(header, std::cref(*uniform2)), core::StatusCode::incompatible,
                  "explicitly absent"),
          "an empty registry refuses a sampler");
    header.mesh_area_light_count = 2;
    check(engine::validate_light_sampler(header, std::cref(*uniform2)).value_or(99U) == 2U,
          "two mesh lights take a uniform sampler of two");
    check(refused(engine::validate_light_sampler(header, std::nullopt), core::StatusCode::incompatible,
                  "explicit light sampler"),
          "a registry refuses a missing sampler");
    check(refused(engine::validate_light_sampler(header, std::cref(*uniform3)), core::StatusCode::incompatible,
                  "count does not match"),
          "a sampler of the wrong size is refused");
    check(refused(engine::validate_light_sampler(header, std::cref(*power2)), core::StatusCode::unavailable,
                  "not ported"),
          "a power-weighted sampler is refused without substitution");

    // mappings
    check(engine::termination_of(BF200_TERMINATION_ZERO_THROUGHPUT) ==
                  engine::CudaWavefrontPathTermination::zero_throughput &&
              engine::termination_of(BF200_TERMINATION_OUTSIDE_BSDF_SUPPORT) ==
                  engine::CudaWavefrontPathTermination::outside_bsdf_support &&
              engine::termination_of(BF200_TERMINATION_RUSSIAN_ROULETTE) ==
                  engine::CudaWavefrontPathTermination::russian_roulette &&
              engine::termination_of(BF200_TERMINATION_DEPTH_LIMIT) == engine::CudaWavefrontPathTermination::depth_limit &&
              engine::termination_of(BF200_TERMINATION_ESCAPED_ENVIRONMENT) ==
                  engine::CudaWavefrontPathTermination::escaped_environment,
          "terminations map onto the reference's codes");
    check(engine::lane_status_code(BF200_LANE_NUMERICAL_FAILURE) == core::StatusCode::internal_error &&
              engine::lane_status_code(BF200_LANE_UNSUPPORTED) == core::StatusCode::unavailable &&
              engine::lane_status_code(BF200_LANE_TRAVERSAL_FAILURE) == core::StatusCode::incompatible,
          "lane failures map onto the reference's stage-audit codes");
    check(engine::status_code(BLACKFRAME_STATUS_INVALID_STATE) == core::StatusCode::unavailable &&
              engine::status_code(BLACKFRAME_STATUS_INVALID_ARGUMENT) == core::StatusCode::invalid_argument &&
              engine::status_code(BLACKFRAME_STATUS_OUT_OF_RANGE) == core::StatusCode::resource_exhausted,
          "C ABI statuses map onto core status codes");

    // workspaces
    check(refused(engine::CudaWavefrontTransportWorkspace::create(0), core::StatusCode::invalid_argument, "non-zero"),
          "a workspace of no capacity is refused");
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
        const auto no_device = engine::CudaWavefrontTransportWorkspace::create(64);
        check(!no_device.has_value(), "without a CUDA device no workspace is created");
    } else {
        auto workspace = engine::CudaWavefrontTransportWorkspace::create(64);
        check(workspace.has_value() && workspace->capacity() == 64U && workspace->close().has_value(),
              "a workspace opens and closes on a CUDA device");
    }
    return failures == 0 ? 0 : 1;
}
