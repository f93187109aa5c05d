// Test infrastructure, not product code: C entry points over the reference's own scene JSON codec
// (Blackframe/Engine/Source/SceneDescriptionJsonReader.cpp, SceneDescriptionJsonWriter.cpp,
// SceneDescription.cpp) and FrameScene::create (FrameScene.cpp), compiled from the reference tree
// into oracle/_ref/libbfref.so. tests/golden/make_scene_json_golden.py and tests/test_scene_json.py
// call them to pin the product's codec (csrc/bf200_scene_json.cpp): the same documents must be
// accepted or refused with the same status code, and an accepted document must serialize to the
// same canonical bytes and commit the same instance transforms and light registry.
#include <Blackframe/Engine/FrameScene.hpp>
#include <Blackframe/Engine/SceneDescription.hpp>
#include <Blackframe/Engine/SceneDescriptionJson.hpp>

#include <cstdint>
#include <cstring>
#include <string>
#include <string_view>
#include <variant>

namespace {

using namespace blackframe;

void copy_message(const std::string& text, char* message, uint64_t capacity) {
    if (message != nullptr && capacity != 0) {
        std::strncpy(message, text.c_str(), capacity - 1);
        message[capacity - 1] = '\0';
    }
}

engine::SceneDescriptionJsonLimits limits_from(const uint64_t* values) {
    auto limits = engine::SceneDescriptionJsonLimits{};
    if (values != nullptr) {
        limits.maximum_encoded_bytes = values[0];
        limits.maximum_nesting_depth = static_cast<uint32_t>(values[1]);
        limits.maximum_total_values = values[2];
        limits.maximum_total_string_bytes = values[3];
        limits.maximum_records_per_registry = static_cast<uint32_t>(values[4]);
        limits.maximum_mesh_vertices = values[5];
        limits.maximum_mesh_triangles = values[6];
        limits.maximum_image_scalar_values = values[7];
        limits.maximum_decoded_bytes = values[8];
    }
    return limits;
}

}  // namespace

extern "C" {

// deserialize_scene_description_json, then serialize_scene_description_json of the result.
// Returns the StatusCode of the first call that failed (0: both succeeded) with its message; on
// success the canonical bytes go to `out` when they fit (*out_size is their length either way).
__attribute__((visibility("default"))) int bfref_scene_json_canonical(const char* bytes, uint64_t size,
                                                                      const uint64_t* limits, char* out,
                                                                      uint64_t capacity, uint64_t* out_size,
                                                                      char* message, uint64_t message_capacity) {
    const auto decoded = engine::deserialize_scene_description_json(std::string_view{bytes, size}, limits_from(limits));
    if (!decoded) {
        copy_message(decoded.error().message, message, message_capacity);
        return static_cast<int>(decoded.error().code);
    }
    const auto encoded = engine::serialize_scene_description_json(*decoded, limits_from(limits));
    if (!encoded) {
        copy_message("serialize: " + encoded.error().message, message, message_capacity);
        return static_cast<int>(encoded.error().code);
    }
    *out_size = encoded->size();
    if (out != nullptr && encoded->size() <= capacity) {
        std::memcpy(out, encoded->data(), encoded->size());
    }
    copy_message("", message, message_capacity);
    return 0;
}

// deserialize_scene_description_json alone (default limits): its StatusCode. For timing the
// reference's reader beside the product's.
__attribute__((visibility("default"))) int bfref_scene_json_parse_only(const char* bytes, uint64_t size) {
    const auto decoded = engine::deserialize_scene_description_json(std::string_view{bytes, size});
    return decoded ? 0 : static_cast<int>(decoded.error().code);
}

// The frame a caller commits from a decoded description: FrameScene::create over its textures,
// objects, geometries, materials and instances, its punctual lights in registry order and its
// spectral environment. Per committed instance (identifier order): the identifier and the world
// transform's matrix and inverse (row-major); then the instance identifiers of the mesh area
// lights. Returns the StatusCode of the first failure (0: success).
__attribute__((visibility("default"))) int bfref_scene_json_frame(const char* bytes, uint64_t size, uint32_t* ids,
                                                                  float* world, float* inverse, uint64_t capacity,
                                                                  uint64_t* count, uint32_t* light_ids,
                                                                  uint64_t light_capacity, uint64_t* light_count,
                                                                  char* message, uint64_t message_capacity) {
    const auto decoded = engine::deserialize_scene_description_json(std::string_view{bytes, size});
    if (!decoded) {
        copy_message(decoded.error().message, message, message_capacity);
        return static_cast<int>(decoded.error().code);
    }
    auto frame = engine::FrameSceneDescription{};
    frame.constant_textures.assign(decoded->constant_textures().begin(), decoded->constant_textures().end());
    frame.host_image_textures.assign(decoded->host_image_textures().begin(), decoded->host_image_textures().end());
    frame.objects.assign(decoded->objects().begin(), decoded->objects().end());
    frame.geometries.assign(decoded->geometries().begin(), decoded->geometries().end());
    frame.materials.assign(decoded->materials().begin(), decoded->materials().end());
    frame.instances.assign(decoded->instances().begin(), decoded->instances().end());
    for (const auto& record : decoded->lights()) {
        std::visit(
            [&](const auto& light) {
                using Light = std::remove_cvref_t<decltype(light)>;
                if constexpr (std::is_same_v<Light, engine::SceneSpectralEnvironment>) {
                    frame.spectral_environment = light;
                } else {
                    frame.punctual_lights.emplace_back(light);
                }
            },
            record.light);
    }
    const auto scene = engine::FrameScene::create(std::move(frame));
    if (!scene) {
        copy_message("frame: " + scene.error().message, message, message_capacity);
        return static_cast<int>(scene.error().code);
    }
    const auto instances = (*scene)->instances();
    *count = instances.size();
    for (size_t i = 0; i < instances.size() && i < capacity; ++i) {
        ids[i] = instances[i].id.value;
        const auto transform = (*scene)->world_transform(instances[i].id);
        if (!transform) {
            copy_message("world transform: " + transform.error().message, message, message_capacity);
            return static_cast<int>(transform.error().code);
        }
        for (size_t r = 0; r < 4; ++r) {
            for (size_t c = 0; c < 4; ++c) {
                world[i * 16 + r * 4 + c] = transform->get().matrix()(r, c);
                inverse[i * 16 + r * 4 + c] = transform->get().inverse_matrix()(r, c);
            }
        }
    }
    const auto lights = (*scene)->mesh_area_light_instance_ids();
    *light_count = lights.size();
    for (size_t i = 0; i < lights.size() && i < light_capacity; ++i) {
        light_ids[i] = lights[i].value;
    }
    copy_message("", message, message_capacity);
    return 0;
}

// The byte sizes the reference's decoded-scene budget charges per record (the sizeof of each
// registry record and mesh element), in the order films, cameras, render options, constant
// textures, host-image textures, objects, geometries, materials, instances, lights, mesh
// position, normal, texture coordinate and triangle.
__attribute__((visibility("default"))) void bfref_scene_json_record_sizes(uint64_t* out) {
    out[0] = sizeof(engine::SceneFilmDescription);
    out[1] = sizeof(engine::SceneCameraDescription);
    out[2] = sizeof(engine::SceneRenderOptionsDescription);
    out[3] = sizeof(engine::SceneConstantTexture);
    out[4] = sizeof(engine::SceneHostImageTexture);
    out[5] = sizeof(engine::SceneObject);
    out[6] = sizeof(engine::SceneGeometry);
    out[7] = sizeof(engine::SceneMaterial);
    out[8] = sizeof(engine::SceneInstance);
    out[9] = sizeof(engine::SceneLightDescription);
    out[10] = sizeof(renderer::Point3);
    out[11] = sizeof(renderer::Normal3);
    out[12] = sizeof(renderer::Point2);
    out[13] = sizeof(engine::TriangleVertexIndices);
}

}  // extern "C"
