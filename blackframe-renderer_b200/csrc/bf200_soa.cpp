// Scene upload from the reference's scene SoA blob, ABI v4 (the canonical column layout a Blackframe
// host serialises a FrameScene into for its CUDA backend: SceneSoaHeader + 194 columns,
// Blackframe/XPU/Shared/Include/Blackframe/XPU/Shared/SceneSoaAbi.hpp:11-398, written by
// CudaSceneSoA::upload, Blackframe/Backends/GPU/CUDA/Source/SceneSoA.cpp:334-1160). The header is
// validated as validate_scene_soa_header does, the content hash is checked (FNV-1a 64 over the
// blob with the hash field read as zero), and the columns become a bf200_scene_desc_v1 for
// bf200_scene_create.
//
// Kept alike with the reference, because a blob is an interchange format: the magic, version,
// header size (4,848 bytes), column numbering, element sizes, the 16-byte column alignment, and
// the hash. What the backend does not render is refused (no substitution):
// normal and bump maps, materials whose spectral packets differ.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "bf200.h"

namespace {

constexpr uint64_t kMagic = 0x34414F53464B4C42ULL;  // "BLKFSOA4"
constexpr uint32_t kColumns = 194U;
constexpr uint64_t kHeaderBytes = 4848U;
constexpr uint64_t kHashOffset = 32U;

// column numbers (SceneSoaAbi.hpp:23-125)
enum Column : uint32_t {
    object_id = 0, geometry_id = 1, geometry_vertex_offset = 2, geometry_vertex_count = 3,
    geometry_triangle_offset = 4, geometry_triangle_count = 5, position_x = 6, normal_x = 9,
    texture_coordinate_x = 12, triangle_vertex_0 = 14, material_id = 17, material_spectral_present = 18,
    material_wavelength_nanometers = 19, material_wavelength_pdf = 23, material_wavelength_measure = 27,
    material_closure_offset = 31, material_closure_count = 32, material_closure_frame_mode = 33,
    material_closure_tangent_rotation_radians = 34, material_emitted_radiance = 35, closure_kind = 39,
    closure_lobes = 40, closure_weight = 41, closure_parameters = 45, closure_probability = 55,
    instance_id = 56, instance_parent_present = 57, instance_parent_id = 58, instance_object_id = 59,
    instance_geometry_id = 60, instance_material_id = 61, instance_visibility_mask = 62,
    instance_local_to_parent = 63, instance_parent_to_local = 79, instance_local_to_world = 95,
    instance_world_to_local = 111, punctual_kind = 127, mesh_area_light_instance_id = 143,
    environment_wavelength_nanometers = 144, environment_wavelength_pdf = 148,
    environment_wavelength_measure = 152, environment_radiance = 156, texture_id = 160,
    material_normal_map_present = 166, material_bump_map_present = 176, image_texture_id = 184,
    image_mip_width = 189, image_texel_value = 193,
};

struct Header {
    uint64_t magic;
    uint16_t abi_major, abi_minor;
    uint32_t header_size, column_count, hash_algorithm;
    uint64_t total_size_bytes, content_hash;
    uint64_t object_count, geometry_count, vertex_count, triangle_count, material_count, closure_count,
        instance_count, punctual_light_count, mesh_area_light_count, environment_count, texture_count,
        image_texture_count, image_mip_count, image_texel_count;
    struct Column {
        uint64_t offset_bytes, element_count;
        uint32_t element_size, reserved;
    } columns[kColumns];
    uint64_t reserved[5];
};
static_assert(sizeof(Header) == kHeaderBytes, "SceneSoaHeader layout");

// scene_soa_column_count (SceneSoaAbi.hpp:186-228)
uint64_t column_count(const Header& h, uint32_t c) {
    if (c == object_id) return h.object_count;
    if (c >= geometry_id && c <= geometry_triangle_count) return h.geometry_count;
    if (c >= position_x && c <= 13) return h.vertex_count;
    if (c >= triangle_vertex_0 && c <= 16) return h.triangle_count;
    if (c >= material_id && c < closure_kind) return h.material_count;
    if (c >= closure_kind && c < instance_id) return h.closure_count;
    if (c >= instance_id && c < punctual_kind) return h.instance_count;
    if (c >= punctual_kind && c < mesh_area_light_instance_id) return h.punctual_light_count;
    if (c == mesh_area_light_instance_id) return h.mesh_area_light_count;
    if (c >= environment_wavelength_nanometers && c < texture_id) return h.environment_count;
    if (c >= texture_id && c < material_normal_map_present) return h.texture_count;
    if (c >= material_normal_map_present && c < image_texture_id) return h.material_count;
    if (c >= image_texture_id && c < image_mip_width) return h.image_texture_count;
    if (c >= image_mip_width && c < image_texel_value) return h.image_mip_count;
    if (c == image_texel_value) return h.image_texel_count;
    return 0;
}

// scene_soa_column_element_size (SceneSoaAbi.hpp:230-262)
uint32_t element_size(uint32_t c) {
    if (c >= kColumns) return 0;
    if ((c >= geometry_vertex_offset && c <= geometry_triangle_count) || c == material_closure_offset ||
        c == material_closure_count) {
        return 8;
    }
    if (c == material_spectral_present || (c >= material_wavelength_measure && c < material_closure_offset) ||
        c == material_closure_frame_mode || c == instance_parent_present || c == material_normal_map_present ||
        c == material_bump_map_present || (c >= environment_wavelength_measure && c < environment_radiance)) {
        return 1;
    }
    if ((c >= position_x && c <= 13) || (c >= material_wavelength_nanometers && c < material_wavelength_measure) ||
        c == material_closure_tangent_rotation_radians || (c >= material_emitted_radiance && c < closure_kind) ||
        (c >= closure_weight && c < instance_id) || (c >= instance_local_to_parent && c < punctual_kind) ||
        (c >= 128 && c < mesh_area_light_instance_id) ||
        (c >= environment_wavelength_nanometers && c < environment_wavelength_measure) ||
        (c >= environment_radiance && c < texture_id) || (c >= 162 && c < material_normal_map_present) ||
        c == 179 || c == image_texel_value) {
        return 4;
    }
    if (c == 185 || c == 186 || c == 191 || c == 192) {
        return 8;
    }
    return 4;
}

uint64_t align16(uint64_t v) { return (v + 15U) & ~uint64_t(15); }

// validate_scene_soa_header (SceneSoaAbi.hpp:283-340); empty string when valid
std::string validate_header(const Header& h) {
    if (h.magic != kMagic) return "bad magic";
    if (h.abi_major != 4 || h.abi_minor != 0) return "incompatible version";
    if (h.header_size != kHeaderBytes) return "bad header size";
    if (h.column_count != kColumns) return "bad column count";
    if (h.hash_algorithm != 1) return "unsupported hash algorithm";
    for (uint64_t r : h.reserved) {
        if (r != 0) return "nonzero reserved";
    }
    if (h.environment_count > 1) return "invalid environment count";
    if (h.total_size_bytes < kHeaderBytes) return "bad total size";
    uint64_t cursor = align16(kHeaderBytes);
    for (uint32_t c = 0; c < kColumns; ++c) {
        const auto& d = h.columns[c];
        const uint64_t count = column_count(h, c);
        const uint32_t size = element_size(c);
        if (d.element_count != count || d.element_size != size || d.reserved != 0) return "invalid column descriptor";
        if (count == 0) {
            if (d.offset_bytes != 0) return "invalid column descriptor";
            continue;
        }
        cursor = align16(cursor);
        if (d.offset_bytes != cursor) return "invalid column descriptor";
        if (count > UINT64_MAX / size || cursor > UINT64_MAX - count * size) return "size overflow";
        cursor += count * size;
    }
    if (h.total_size_bytes != cursor) return "bad total size";
    return "";
}

template <typename T>
T read(const unsigned char* blob, const Header& h, uint32_t column, uint64_t index) {
    T v;
    std::memcpy(&v, blob + h.columns[column].offset_bytes + index * sizeof(T), sizeof(T));
    return v;
}

}  // namespace

extern "C" {

BF200_EXPORT blackframe_status bf200_scene_create_from_soa(bf200_context* context, const void* blob_bytes,
                                                           uint64_t size, bf200_scene** out_scene,
                                                           char* message, uint64_t message_capacity) noexcept {
    auto refuse = [&](blackframe_status st, const std::string& why) {
        if (message != nullptr && message_capacity != 0) {
            const size_t n = std::min<uint64_t>(why.size(), message_capacity - 1);
            std::memcpy(message, why.data(), n);
            message[n] = '\0';
        }
        return st;
    };
    if (blob_bytes == nullptr || out_scene == nullptr) {
        return refuse(BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    *out_scene = nullptr;
    if (size < kHeaderBytes) {
        return refuse(BLACKFRAME_STATUS_INVALID_ARGUMENT, "scene SoA blob shorter than its header");
    }
    const auto* blob = static_cast<const unsigned char*>(blob_bytes);
    try {
        Header h;
        std::memcpy(&h, blob, sizeof(h));
        if (const std::string why = validate_header(h); !why.empty()) {
            return refuse(BLACKFRAME_STATUS_INVALID_ARGUMENT, "scene SoA header: " + why);
        }
        if (h.total_size_bytes != size) {
            return refuse(BLACKFRAME_STATUS_INVALID_ARGUMENT, "scene SoA blob size differs from its header");
        }
        uint64_t hash = 14695981039346656037ULL;  // normalized_hash (SceneSoA.cpp:229-239)
        for (uint64_t i = 0; i < size; ++i) {
            const unsigned char b = (i >= kHashOffset && i < kHashOffset + 8) ? 0 : blob[i];
            hash = (hash ^ b) * 1099511628211ULL;
        }
        if (hash != h.content_hash) {
            return refuse(BLACKFRAME_STATUS_INVALID_ARGUMENT, "scene SoA content hash mismatch");
        }
        for (uint64_t m = 0; m < h.material_count; ++m) {
            if (read<uint8_t>(blob, h, material_normal_map_present, m) != 0 ||
                read<uint8_t>(blob, h, material_bump_map_present, m) != 0) {
                return refuse(BLACKFRAME_STATUS_INVALID_STATE, "normal and bump maps are not supported (no substitution)");
            }
        }
        if (h.geometry_count > UINT32_MAX || h.vertex_count > UINT32_MAX || h.triangle_count > UINT32_MAX ||
            h.material_count > UINT32_MAX || h.closure_count > UINT32_MAX || h.instance_count > UINT32_MAX) {
            return refuse(BLACKFRAME_STATUS_OUT_OF_RANGE, "scene SoA counts exceed the 32-bit descriptor");
        }
        // geometry
        std::vector<bf200_geometry_v1> geometries(h.geometry_count);
        std::unordered_map<uint32_t, uint32_t> geometry_index;
        for (uint64_t g = 0; g < h.geometry_count; ++g) {
            bf200_geometry_v1& out = geometries[g];
            std::memset(&out, 0, sizeof(out));
            out.geometry_id = read<uint32_t>(blob, h, geometry_id, g);
            const uint64_t vo = read<uint64_t>(blob, h, geometry_vertex_offset, g);
            const uint64_t vc = read<uint64_t>(blob, h, geometry_vertex_count, g);
            const uint64_t to = read<uint64_t>(blob, h, geometry_triangle_offset, g);
            const uint64_t tc = read<uint64_t>(blob, h, geometry_triangle_count, g);
            if (vo + vc > h.vertex_count || to + tc > h.triangle_count) {
                return refuse(BLACKFRAME_STATUS_OUT_OF_RANGE, "scene SoA geometry range outside its columns");
            }
            out.vertex_offset = static_cast<uint32_t>(vo);
            out.vertex_count = static_cast<uint32_t>(vc);
            out.triangle_offset = static_cast<uint32_t>(to);
            out.triangle_count = static_cast<uint32_t>(tc);
            geometry_index[out.geometry_id] = static_cast<uint32_t>(g);
        }
        std::vector<float> positions(3 * h.vertex_count), normals(3 * h.vertex_count), uvs(2 * h.vertex_count);
        for (uint64_t v = 0; v < h.vertex_count; ++v) {
            for (uint32_t a = 0; a < 3; ++a) {
                positions[3 * v + a] = read<float>(blob, h, position_x + a, v);
                normals[3 * v + a] = read<float>(blob, h, normal_x + a, v);
            }
            for (uint32_t a = 0; a < 2; ++a) {
                uvs[2 * v + a] = read<float>(blob, h, texture_coordinate_x + a, v);
            }
        }
        std::vector<uint32_t> triangles(3 * h.triangle_count);
        for (uint64_t t = 0; t < h.triangle_count; ++t) {
            for (uint32_t k = 0; k < 3; ++k) {
                triangles[3 * t + k] = read<uint32_t>(blob, h, triangle_vertex_0 + k, t);
            }
        }
        // materials and closures; one spectral packet for the whole frame
        bf200_scene_desc_v1 desc{};
        bool packet_seen = false;
        auto take_packet = [&](const float* nm, const float* pdf) {
            if (!packet_seen) {
                std::memcpy(desc.wavelength_nanometers, nm, 16);
                std::memcpy(desc.wavelength_pdf, pdf, 16);
                packet_seen = true;
                return true;
            }
            return std::memcmp(desc.wavelength_nanometers, nm, 16) == 0 && std::memcmp(desc.wavelength_pdf, pdf, 16) == 0;
        };
        std::vector<bf200_material_v1> materials(h.material_count);
        std::unordered_map<uint32_t, uint32_t> material_index;
        std::vector<bf200_closure_v1> closures(h.closure_count);
        for (uint64_t k = 0; k < h.closure_count; ++k) {
            bf200_closure_v1& c = closures[k];
            c.kind = read<uint32_t>(blob, h, closure_kind, k);
            c.lobes = read<uint32_t>(blob, h, closure_lobes, k);
            for (uint32_t l = 0; l < 4; ++l) c.weight[l] = read<float>(blob, h, closure_weight + l, k);
            for (uint32_t p = 0; p < 10; ++p) c.parameters[p] = read<float>(blob, h, closure_parameters + p, k);
        }
        for (uint64_t m = 0; m < h.material_count; ++m) {
            bf200_material_v1& out = materials[m];
            std::memset(&out, 0, sizeof(out));
            out.material_id = read<uint32_t>(blob, h, material_id, m);
            const uint64_t co = read<uint64_t>(blob, h, material_closure_offset, m);
            const uint64_t cc = read<uint64_t>(blob, h, material_closure_count, m);
            if (co + cc > h.closure_count || cc > 8) {
                return refuse(BLACKFRAME_STATUS_OUT_OF_RANGE, "scene SoA material closures outside their column");
            }
            out.closure_offset = static_cast<uint32_t>(co);
            out.closure_count = static_cast<uint32_t>(cc);
            out.frame_mode = read<uint8_t>(blob, h, material_closure_frame_mode, m);
            out.tangent_rotation_radians = read<float>(blob, h, material_closure_tangent_rotation_radians, m);
            for (uint32_t l = 0; l < 4; ++l) {
                out.emitted_radiance[l] = read<float>(blob, h, material_emitted_radiance + l, m);
            }
            for (uint64_t k = 0; k < cc; ++k) {
                out.component_probabilities[k] = read<float>(blob, h, closure_probability, co + k);
            }
            if (read<uint8_t>(blob, h, material_spectral_present, m) != 0) {
                float nm[4], pdf[4];
                for (uint32_t l = 0; l < 4; ++l) {
                    nm[l] = read<float>(blob, h, material_wavelength_nanometers + l, m);
                    pdf[l] = read<float>(blob, h, material_wavelength_pdf + l, m);
                }
                if (!take_packet(nm, pdf)) {
                    return refuse(BLACKFRAME_STATUS_INVALID_STATE, "materials resolved at different wavelength packets");
                }
            }
            material_index[out.material_id] = static_cast<uint32_t>(m);
        }
        if (h.environment_count == 1) {
            float nm[4], pdf[4];
            for (uint32_t l = 0; l < 4; ++l) {
                nm[l] = read<float>(blob, h, environment_wavelength_nanometers + l, 0);
                pdf[l] = read<float>(blob, h, environment_wavelength_pdf + l, 0);
                desc.environment_radiance[l] = read<float>(blob, h, environment_radiance + l, 0);
            }
            if (!take_packet(nm, pdf)) {
                return refuse(BLACKFRAME_STATUS_INVALID_STATE, "the environment is resolved at another wavelength packet");
            }
        }
        // instances: resolved world transforms, ids mapped to indices
        std::vector<bf200_instance_v1> instances(h.instance_count);
        std::vector<uint32_t> emissive_ids;
        for (uint64_t i = 0; i < h.instance_count; ++i) {
            bf200_instance_v1& out = instances[i];
            std::memset(&out, 0, sizeof(out));
            out.instance_id = read<uint32_t>(blob, h, instance_id, i);
            out.object_id = read<uint32_t>(blob, h, instance_object_id, i);
            const auto g = geometry_index.find(read<uint32_t>(blob, h, instance_geometry_id, i));
            const auto m = material_index.find(read<uint32_t>(blob, h, instance_material_id, i));
            if (g == geometry_index.end() || m == material_index.end()) {
                return refuse(BLACKFRAME_STATUS_OUT_OF_RANGE, "scene SoA instance names an unknown geometry or material");
            }
            out.geometry_index = g->second;
            out.material_index = m->second;
            out.visibility_mask = read<uint32_t>(blob, h, instance_visibility_mask, i);
            for (uint32_t e = 0; e < 16; ++e) {
                out.object_to_world[e] = read<float>(blob, h, instance_local_to_world + e, i);
                out.world_to_object[e] = read<float>(blob, h, instance_world_to_local + e, i);
            }
            const float* le = materials[out.material_index].emitted_radiance;
            if (le[0] != 0.0F || le[1] != 0.0F || le[2] != 0.0F || le[3] != 0.0F) {
                emissive_ids.push_back(out.instance_id);
            }
        }
        // the mesh-light registry must be the emissive instances in instance order (FrameScene.cpp:201-261)
        if (emissive_ids.size() != h.mesh_area_light_count) {
            return refuse(BLACKFRAME_STATUS_INVALID_STATE, "scene SoA mesh lights differ from its emissive instances");
        }
        for (uint64_t k = 0; k < h.mesh_area_light_count; ++k) {
            if (read<uint32_t>(blob, h, mesh_area_light_instance_id, k) != emissive_ids[k]) {
                return refuse(BLACKFRAME_STATUS_INVALID_STATE, "scene SoA mesh lights differ from its emissive instances");
            }
        }
        // punctual lights (SceneSoA.cpp:241-300: kind 0 point, 1 directional, 2 spot), first in the
        // light registry
        if (h.punctual_light_count > UINT32_MAX) {
            return refuse(BLACKFRAME_STATUS_OUT_OF_RANGE, "scene SoA counts exceed the 32-bit descriptor");
        }
        std::vector<bf200_punctual_light_v1> punctual(h.punctual_light_count);
        for (uint64_t k = 0; k < h.punctual_light_count; ++k) {
            bf200_punctual_light_v1& out = punctual[k];
            std::memset(&out, 0, sizeof(out));
            const uint32_t kind = read<uint32_t>(blob, h, punctual_kind, k);
            if (kind > 2U) {
                return refuse(BLACKFRAME_STATUS_INVALID_ARGUMENT, "scene SoA punctual light of an unknown kind");
            }
            out.kind = kind == 0U ? BF200_PUNCTUAL_POINT : (kind == 1U ? BF200_PUNCTUAL_DIRECTIONAL : BF200_PUNCTUAL_SPOT);
            for (uint32_t a = 0; a < 3; ++a) {
                out.position[a] = read<float>(blob, h, punctual_kind + 1 + a, k);
                out.position_error[a] = read<float>(blob, h, punctual_kind + 4 + a, k);
                out.direction[a] = read<float>(blob, h, punctual_kind + 7 + a, k);
            }
            out.inner_half_angle = read<float>(blob, h, punctual_kind + 10, k);
            out.outer_half_angle = read<float>(blob, h, punctual_kind + 11, k);
            for (uint32_t l = 0; l < 4; ++l) {
                out.spectrum[l] = read<float>(blob, h, punctual_kind + 12 + l, k);
            }
        }
        desc.struct_size = sizeof(desc);
        desc.punctual_lights = punctual.empty() ? nullptr : punctual.data();
        desc.geometry_count = static_cast<uint32_t>(h.geometry_count);
        desc.vertex_count = static_cast<uint32_t>(h.vertex_count);
        desc.triangle_count = static_cast<uint32_t>(h.triangle_count);
        desc.material_count = static_cast<uint32_t>(h.material_count);
        desc.closure_count = static_cast<uint32_t>(h.closure_count);
        desc.instance_count = static_cast<uint32_t>(h.instance_count);
        desc.punctual_light_count = static_cast<uint32_t>(h.punctual_light_count);
        desc.geometries = geometries.data();
        desc.positions = positions.data();
        desc.normals = normals.data();
        desc.texture_coordinates = uvs.data();
        desc.triangles = triangles.data();
        desc.materials = materials.data();
        desc.closures = closures.data();
        desc.instances = instances.data();
        if (context == nullptr) {  // the blob is valid; a scene needs a context
            return refuse(BLACKFRAME_STATUS_INVALID_ARGUMENT, "null context");
        }
        const blackframe_status st = bf200_scene_create(context, &desc, out_scene);
        if (st != BLACKFRAME_STATUS_SUCCESS) {
            const char* why = bf200_context_last_error(context);
            return refuse(st, why != nullptr ? why : "scene creation failed");
        }
        return refuse(BLACKFRAME_STATUS_SUCCESS, "");
    } catch (const std::bad_alloc&) {
        return refuse(BLACKFRAME_STATUS_OUT_OF_RANGE, "scene SoA upload exhausted host memory");
    }
}

}  // extern "C"
