// Shared by the reference harnesses (test infrastructure only): the flat bf200 scene and path
// records turned into the reference's own objects (FrameSceneDescription -> FrameScene::create,
// Blackframe/Engine/Source/FrameScene.cpp:390-528; ClosureSet appends, ClosureSet.hpp; Ray::create).
#pragma once

#include "../include/bf200.h"

#include <Blackframe/Engine/FrameScene.hpp>
#include <Blackframe/Engine/TriangleMesh.hpp>
#include <Blackframe/Renderer/ClosureSet.hpp>
#include <Blackframe/Renderer/Ray.hpp>
#include <Blackframe/Renderer/RussianRoulette.hpp>
#include <Blackframe/Renderer/WavelengthSampling.hpp>

#include <algorithm>
#include <memory>
#include <span>
#include <string>
#include <vector>

namespace bfref {

using namespace blackframe;

inline renderer::SampledWavelengths make_wavelengths(const float* nm, const float* pdf) {
    auto result = renderer::SampledWavelengths{};
    for (std::size_t lane = 0; lane < 4; ++lane) {
        result[lane].nanometers = nm[lane];
        result[lane].probability.value = pdf[lane];
        result[lane].probability.measure = renderer::ProbabilityMeasure::wavelength;
    }
    return result;
}

inline renderer::TransportSpectrum spectrum4(const float* values) {
    auto result = renderer::TransportSpectrum{};
    for (std::size_t lane = 0; lane < 4; ++lane) {
        result.values[lane] = values[lane];
    }
    return result;
}

inline core::Result<engine::SceneClosureMixture> make_mixture(const bf200_material_v1& material,
                                                       const bf200_closure_v1* closures) {
    auto set = renderer::ClosureSet{};
    for (uint32_t index = 0; index < material.closure_count; ++index) {
        const auto& record = closures[material.closure_offset + index];
        const auto weight = spectrum4(record.weight);
        auto status = renderer::ClosureAppendStatus::invalid_payload;
        switch (record.kind) {
        case BF200_CLOSURE_LAMBERTIAN_REFLECTION:
            status = set.append_lambertian_reflection(weight);
            break;
        case BF200_CLOSURE_ROUGH_CONDUCTOR_REFLECTION:
            status = set.append_rough_conductor_reflection(weight, spectrum4(record.parameters),
                                                           spectrum4(record.parameters + 4),
                                                           record.parameters[8],
                                                           record.parameters[9]);
            break;
        case BF200_CLOSURE_ROUGH_DIELECTRIC:
            status = set.append_rough_dielectric(weight, record.parameters[0],
                                                 record.parameters[1], record.parameters[2],
                                                 record.parameters[3]);
            break;
        case BF200_CLOSURE_ROUGH_DIFFUSE_REFLECTION:
            status = set.append_rough_diffuse_reflection(weight, record.parameters[0]);
            break;
        case BF200_CLOSURE_SPECULAR_REFLECTION:
            status = set.append_specular_reflection(weight);
            break;
        case BF200_CLOSURE_SPECULAR_TRANSMISSION:
            status = set.append_specular_transmission(weight, record.parameters[0], record.parameters[1]);
            break;
        default:
            break;
        }
        if (status != renderer::ClosureAppendStatus::appended) {
            return std::unexpected(core::Error{.code = core::StatusCode::invalid_argument,
                                               .message = "closure record rejected"});
        }
    }
    return engine::SceneClosureMixture::create(
        set,
        std::span<const float>{material.component_probabilities, material.closure_count},
        material.frame_mode == 1 ? engine::SceneClosureFrameMode::surface_tangent
                                 : engine::SceneClosureFrameMode::shading_normal,
        material.tangent_rotation_radians);
}

inline renderer::Ray make_ray(const bf200_ray_v1& ray) {
    const auto created = renderer::Ray::create(
        renderer::Point3{.x = ray.origin[0], .y = ray.origin[1], .z = ray.origin[2]},
        renderer::Vector3{.x = ray.direction[0], .y = ray.direction[1], .z = ray.direction[2]},
        ray.t_min, ray.t_max, ray.time, ray.mask, renderer::MediumId{.value = ray.medium});
    return *created;
}

inline void store_ray(const renderer::Ray& ray, bf200_ray_v1& out) {
    out.origin[0] = ray.origin().x;
    out.origin[1] = ray.origin().y;
    out.origin[2] = ray.origin().z;
    out.direction[0] = ray.direction().x;
    out.direction[1] = ray.direction().y;
    out.direction[2] = ray.direction().z;
    out.t_min = ray.t_min();
    out.t_max = ray.t_max();
    out.time = ray.time();
    out.mask = ray.mask();
    out.medium = ray.current_medium().value;
    out.reserved = 0;
}

inline core::Result<renderer::RussianRoulettePolicy> make_policy(const bf200_transport_options_v1& o) {
    if (o.roulette_enabled == 0) {
        return renderer::RussianRoulettePolicy::disabled();
    }
    return renderer::RussianRoulettePolicy::create_enabled(o.roulette_first_eligible_depth,
                                                           o.roulette_minimum_survival,
                                                           o.roulette_maximum_survival);
}

// The committed FrameScene of a bf200 scene description; on failure, the stage and the reference's
// message in `error` and a null handle.
inline engine::FrameSceneHandle make_frame_scene(const bf200_scene_desc_v1* desc, std::string& error,
                                                 int* code = nullptr) {
    auto set_error = [&](const std::string& m) { error = m; };
    auto fail_code = [&](int c) -> engine::FrameSceneHandle {
        if (code != nullptr) {
            *code = c;
        }
        return nullptr;
    };
    auto description = engine::FrameSceneDescription{};
    const auto wavelengths = make_wavelengths(desc->wavelength_nanometers, desc->wavelength_pdf);
    for (uint32_t g = 0; g < desc->geometry_count; ++g) {
        const auto& geometry = desc->geometries[g];
        auto positions = std::vector<renderer::Point3>{};
        auto normals = std::vector<renderer::Normal3>{};
        auto uvs = std::vector<renderer::Point2>{};
        for (uint32_t v = 0; v < geometry.vertex_count; ++v) {
            const auto i = geometry.vertex_offset + v;
            positions.push_back(renderer::Point3{.x = desc->positions[3 * i],
                                                 .y = desc->positions[3 * i + 1],
                                                 .z = desc->positions[3 * i + 2]});
            normals.push_back(renderer::Normal3{.x = desc->normals[3 * i],
                                                .y = desc->normals[3 * i + 1],
                                                .z = desc->normals[3 * i + 2]});
            uvs.push_back(renderer::Point2{.x = desc->texture_coordinates[2 * i],
                                           .y = desc->texture_coordinates[2 * i + 1]});
        }
        auto triangles = std::vector<engine::TriangleVertexIndices>{};
        for (uint32_t t = 0; t < geometry.triangle_count; ++t) {
            const auto i = geometry.triangle_offset + t;
            triangles.push_back(engine::TriangleVertexIndices{
                .vertices = {desc->triangles[3 * i], desc->triangles[3 * i + 1],
                             desc->triangles[3 * i + 2]}});
        }
        auto mesh = engine::TriangleMesh::create(std::move(positions), std::move(normals),
                                                 std::move(uvs), std::move(triangles));
        if (!mesh) {
            set_error("mesh: " + mesh.error().message);
            return fail_code(2);
        }
        description.geometries.push_back(engine::SceneGeometry{
            .id = {.value = geometry.geometry_id},
            .mesh = std::make_shared<const engine::TriangleMesh>(std::move(*mesh))});
    }
    for (uint32_t m = 0; m < desc->material_count; ++m) {
        const auto& material = desc->materials[m];
        auto mixture = make_mixture(material, desc->closures);
        if (!mixture) {
            set_error("material: " + mixture.error().message);
            return fail_code(3);
        }
        description.materials.push_back(engine::SceneMaterial{
            .id = {.value = material.material_id},
            .spectral =
                engine::SceneSpectralMaterial{
                    .wavelengths = wavelengths,
                    .closure_mixture = *mixture,
                    .emitted_radiance = spectrum4(material.emitted_radiance),
                },
        });
    }
    auto object_ids = std::vector<uint32_t>{};
    for (uint32_t i = 0; i < desc->instance_count; ++i) {
        const auto& instance = desc->instances[i];
        if (std::find(object_ids.begin(), object_ids.end(), instance.object_id) ==
            object_ids.end()) {
            object_ids.push_back(instance.object_id);
            description.objects.push_back(engine::SceneObject{.id = {.value = instance.object_id}});
        }
        auto matrix = renderer::Matrix4{};
        for (std::size_t r = 0; r < 4; ++r) {
            for (std::size_t c = 0; c < 4; ++c) {
                matrix(r, c) = instance.object_to_world[r * 4 + c];
            }
        }
        description.instances.push_back(engine::SceneInstance{
            .id = {.value = instance.instance_id},
            .parent = std::nullopt,
            .object = {.value = instance.object_id},
            .geometry = {.value = desc->geometries[instance.geometry_index].geometry_id},
            .material = {.value = desc->materials[instance.material_index].material_id},
            .local_to_parent = matrix,
            .visibility_mask = instance.visibility_mask,
        });
    }
    const uint32_t punctual_count =
        desc->struct_size >= sizeof(bf200_scene_desc_v1) && desc->punctual_lights != nullptr ? desc->punctual_light_count : 0U;
    for (uint32_t k = 0; k < punctual_count; ++k) {
        const auto& light = desc->punctual_lights[k];
        const auto position = renderer::Point3{.x = light.position[0], .y = light.position[1], .z = light.position[2]};
        const auto error =
            renderer::Vector3{.x = light.position_error[0], .y = light.position_error[1], .z = light.position_error[2]};
        const auto direction = renderer::Vector3{.x = light.direction[0], .y = light.direction[1], .z = light.direction[2]};
        if (light.kind == BF200_PUNCTUAL_POINT) {
            description.punctual_lights.emplace_back(engine::ScenePointLight{
                .position = position, .absolute_position_error = error, .spectral_radiant_intensity = spectrum4(light.spectrum)});
        } else if (light.kind == BF200_PUNCTUAL_DIRECTIONAL) {
            description.punctual_lights.emplace_back(engine::SceneDirectionalLight{
                .propagation_direction = direction, .spectral_irradiance = spectrum4(light.spectrum)});
        } else {
            description.punctual_lights.emplace_back(engine::SceneSpotLight{
                .position = position,
                .absolute_position_error = error,
                .emission_direction = direction,
                .inner_half_angle_radians = light.inner_half_angle,
                .outer_half_angle_radians = light.outer_half_angle,
                .on_axis_spectral_radiant_intensity = spectrum4(light.spectrum)});
        }
    }
    description.spectral_environment = engine::SceneSpectralEnvironment{
        .wavelengths = wavelengths,
        .radiance = spectrum4(desc->environment_radiance),
    };
    auto scene = engine::FrameScene::create(std::move(description));
    if (!scene) {
        set_error("frame scene: " + scene.error().message);
        return fail_code(4);
    }
    return *scene;
}

}  // namespace bfref
