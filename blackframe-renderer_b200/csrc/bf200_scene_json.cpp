// The native scene JSON codec (schema "blackframe.scene" v1): the reference's
// deserialize_scene_description_json and serialize_scene_description_json
// (Blackframe/Engine/Source/SceneDescriptionJsonReader.cpp, SceneDescriptionJsonWriter.cpp,
// SceneJsonSyntax.cpp) and the checks of SceneDescription::create (SceneDescription.cpp:379-552)
// over the same bytes, plus the commit of the active selection into this backend's scene, camera
// and transport options.
//
// Reading is one forward pass over the bytes, in the reference's order, so the first violation it
// meets (syntax, schema, budget) is the one the reference reports and carries the same status
// code. The schema is closed: unknown keys, duplicate keys, missing required keys, wrong shapes
// and out-of-domain integers are refused. Numbers are parsed as correctly rounded doubles and
// narrowed to float as renderer::to_transport_scalar narrows them. Host-image textures and
// normal/bump maps are refused as unavailable (this backend has no image textures).
//
// The document keeps the validated description with every registry sorted by identifier, the
// instance world transforms resolved through the hierarchy, and the committed arrays that
// bf200_scene_json_frame hands to bf200_scene_create. The file is compiled with floating-point
// contraction off, like the reference's scalar build.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <new>
#include <set>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

#include "bf200.h"
#include "bf200_records.h"

namespace bf200 {
namespace scene_json {

enum Code : uint32_t {
    kOk = BF200_SCENE_JSON_OK,
    kInvalid = BF200_SCENE_JSON_INVALID_ARGUMENT,
    kUnavailable = BF200_SCENE_JSON_UNAVAILABLE,
    kIncompatible = BF200_SCENE_JSON_INCOMPATIBLE,
    kExhausted = BF200_SCENE_JSON_RESOURCE_EXHAUSTED,
    kInternal = BF200_SCENE_JSON_INTERNAL_ERROR,
};

struct Refusal {
    uint32_t code;
    std::string message;
};

[[noreturn]] void refuse(uint32_t code, std::string message) {
    throw Refusal{code, std::move(message)};
}

// SceneDescriptionJsonLimits and its default and hard-maximum values (SceneDescriptionJson.hpp:18-44).
struct Limits {
    uint64_t encoded = 64ULL << 20;
    uint64_t values = 64'000'000ULL;
    uint64_t string_bytes = 16ULL << 20;
    uint64_t mesh_vertices = 4'000'000ULL;
    uint64_t mesh_triangles = 4'000'000ULL;
    uint64_t image_scalars = 16'000'000ULL;
    uint64_t decoded = 512ULL << 20;
    uint32_t depth = 64;
    uint32_t records = 1'000'000;
};

constexpr Limits kMaximumLimits{256ULL << 20, 128'000'000ULL, 64ULL << 20, 16'000'000ULL, 16'000'000ULL,
                                64'000'000ULL, 2ULL << 30, 128, 4'000'000};

Limits limits_from(const bf200_scene_json_limits_v1* in) {
    Limits l;
    if (in != nullptr) {
        l = Limits{in->maximum_encoded_bytes, in->maximum_total_values, in->maximum_total_string_bytes,
                   in->maximum_mesh_vertices, in->maximum_mesh_triangles, in->maximum_image_scalar_values,
                   in->maximum_decoded_bytes, in->maximum_nesting_depth, in->maximum_records_per_registry};
    }
    return l;
}

// validate_limits (SceneJsonSyntax.cpp:133-149).
void validate_limits(const Limits& l) {
    const auto bad = [](uint64_t value, uint64_t maximum) { return value == 0 || value > maximum; };
    const Limits& m = kMaximumLimits;
    if (bad(l.encoded, m.encoded) || bad(l.depth, m.depth) || bad(l.values, m.values) ||
        bad(l.string_bytes, m.string_bytes) || bad(l.records, m.records) || bad(l.mesh_vertices, m.mesh_vertices) ||
        bad(l.mesh_triangles, m.mesh_triangles) || bad(l.image_scalars, m.image_scalars) ||
        bad(l.decoded, m.decoded)) {
        refuse(kInvalid, "Every scene JSON limit must be non-zero and no greater than its hard maximum.");
    }
}

// The bytes the decoded-scene budget charges per record: the sizes of the reference's records
// (SceneDescription.hpp, FrameScene.hpp) on a 64-bit host, which the budget arithmetic depends on.
constexpr uint64_t kFilmBytes = 32, kCameraBytes = 80, kRenderOptionsBytes = 72, kConstantTextureBytes = 24,
                   kHostImageTextureBytes = 24, kObjectBytes = 4, kGeometryBytes = 24, kMaterialBytes = 712,
                   kInstanceBytes = 92, kLightBytes = 72, kPositionBytes = 12, kNormalBytes = 12,
                   kTextureCoordinateBytes = 8, kTriangleBytes = 12;

constexpr std::string_view kSchemaName = "blackframe.scene";
constexpr uint64_t kSchemaVersion = 1;
constexpr float kPi = 3.14159265358979323846F;  // std::numbers::pi_v<float>

// ---------------------------------------------------------------------------------------------
// Syntax: a strict pull reader over the bytes (SceneJsonSyntax.cpp:151-724).

bool json_space(char c) {
    return c == ' ' || c == '\t' || c == '\r' || c == '\n';
}

bool continuation(unsigned char c) {
    return c >= 0x80U && c <= 0xBFU;
}

// Length of one shortest-form UTF-8 scalar at `at`, 0 when malformed.
size_t utf8_length(std::string_view s, size_t at) {
    const auto byte = [&](size_t k) { return static_cast<unsigned char>(s[at + k]); };
    const unsigned char first = byte(0);
    if (first <= 0x7FU) {
        return 1;
    }
    if (first >= 0xC2U && first <= 0xDFU) {
        return at + 1 < s.size() && continuation(byte(1)) ? 2 : 0;
    }
    if (first >= 0xE0U && first <= 0xEFU) {
        if (at + 2 >= s.size()) {
            return 0;
        }
        const unsigned char second = byte(1);
        const bool ok = first == 0xE0U   ? second >= 0xA0U && second <= 0xBFU
                        : first == 0xEDU ? second >= 0x80U && second <= 0x9FU
                                         : continuation(second);
        return ok && continuation(byte(2)) ? 3 : 0;
    }
    if (first >= 0xF0U && first <= 0xF4U) {
        if (at + 3 >= s.size()) {
            return 0;
        }
        const unsigned char second = byte(1);
        const bool ok = first == 0xF0U   ? second >= 0x90U && second <= 0xBFU
                        : first == 0xF4U ? second >= 0x80U && second <= 0x8FU
                                         : continuation(second);
        return ok && continuation(byte(2)) && continuation(byte(3)) ? 4 : 0;
    }
    return 0;
}

void append_utf8(std::string& out, uint32_t cp) {
    if (cp <= 0x7FU) {
        out.push_back(static_cast<char>(cp));
    } else if (cp <= 0x7FFU) {
        out.push_back(static_cast<char>(0xC0U | (cp >> 6)));
        out.push_back(static_cast<char>(0x80U | (cp & 0x3FU)));
    } else if (cp <= 0xFFFFU) {
        out.push_back(static_cast<char>(0xE0U | (cp >> 12)));
        out.push_back(static_cast<char>(0x80U | ((cp >> 6) & 0x3FU)));
        out.push_back(static_cast<char>(0x80U | (cp & 0x3FU)));
    } else {
        out.push_back(static_cast<char>(0xF0U | (cp >> 18)));
        out.push_back(static_cast<char>(0x80U | ((cp >> 12) & 0x3FU)));
        out.push_back(static_cast<char>(0x80U | ((cp >> 6) & 0x3FU)));
        out.push_back(static_cast<char>(0x80U | (cp & 0x3FU)));
    }
}

class Cursor {
  public:
    Cursor(std::string_view input, const Limits& limits) : in_(input), lim_(limits) {}

    // An object: `on_key(key)` consumes the key's value.
    template <typename F> void object(F&& on_key) {
        open('{');
        if (consume('}')) {
            --depth_;
            return;
        }
        std::set<std::string, std::less<>> keys;
        for (;;) {
            std::string key = string_token();
            const auto inserted = keys.insert(key);
            if (!inserted.second) {
                syntax("Duplicate decoded JSON object key '" + key + "'");
            }
            if (!consume(':')) {
                syntax("Expected ':' after JSON object key");
            }
            on_key(std::string_view(*inserted.first));
            if (consume('}')) {
                --depth_;
                return;
            }
            if (!consume(',')) {
                syntax("Expected ',' or '}' after JSON object value");
            }
        }
    }

    // An array: `on_element(index)` consumes element `index`.
    template <typename F> void array(F&& on_element) {
        open('[');
        if (consume(']')) {
            --depth_;
            return;
        }
        for (uint64_t index = 0;; ++index) {
            on_element(index);
            if (consume(']')) {
                --depth_;
                return;
            }
            if (!consume(',')) {
                syntax("Expected ',' or ']' after JSON array value");
            }
        }
    }

    std::string string() {
        claim();
        return string_token();
    }

    uint64_t u64() {
        claim();
        const std::string_view t = number_token(true, true);
        uint64_t v = 0;
        const auto r = std::from_chars(t.data(), t.data() + t.size(), v, 10);
        if (r.ec != std::errc{} || r.ptr != t.data() + t.size()) {
            syntax("Unsigned JSON integer is outside uint64 range");
        }
        return v;
    }

    // renderer::to_transport_scalar of the correctly rounded double (NumericConversion.cpp:17-37).
    float real() {
        claim();
        const std::string_view t = number_token(false, false);
        double v = 0.0;
        const auto r = std::from_chars(t.data(), t.data() + t.size(), v, std::chars_format::general);
        if (r.ec != std::errc{} || r.ptr != t.data() + t.size() || !std::isfinite(v)) {
            syntax("JSON number is not a finite representable scalar");
        }
        if (v < static_cast<double>(std::numeric_limits<float>::lowest()) ||
            v > static_cast<double>(std::numeric_limits<float>::max())) {
            refuse(kInvalid, "A reference scalar exceeds the finite transport range.");
        }
        const float f = static_cast<float>(v);
        if (v != 0.0 && f == 0.0F) {
            refuse(kInvalid, "A reference scalar underflows to zero in transport precision.");
        }
        return f;
    }

    void null() {
        claim();
        ws();
        if (in_.size() - pos_ < 4 || in_.substr(pos_, 4) != "null" || !boundary_at(pos_ + 4)) {
            syntax("Expected JSON null");
        }
        pos_ += 4;
    }

    bool peek_null() {
        ws();
        return in_.size() - pos_ >= 4 && in_.substr(pos_, 4) == "null" && boundary_at(pos_ + 4);
    }

    bool peek_array() {
        ws();
        return pos_ < in_.size() && in_[pos_] == '[';
    }

    // An object whose values are any JSON values, checked for syntax and budgets only: the
    // records this backend refuses as unavailable (host images, normal and bump maps) are read
    // this way, so malformed bytes are still refused as the reference refuses them.
    void skip_object() {
        object([&](std::string_view) { skip_value(); });
    }

    // Exactly one complete root value followed by JSON whitespace.
    void finish() {
        if (depth_ != 0 || values_ == 0) {
            syntax("Scene JSON must contain exactly one complete root value");
        }
        ws();
        if (pos_ != in_.size()) {
            syntax("Unexpected data after scene JSON root value");
        }
    }

  private:
    [[noreturn]] void syntax(const std::string& message) const {
        refuse(kInvalid, message + " At byte " + std::to_string(pos_) + ".");
    }
    [[noreturn]] void budget(const std::string& message) const {
        refuse(kExhausted, message + " At byte " + std::to_string(pos_) + ".");
    }

    void ws() {
        while (pos_ < in_.size() && json_space(in_[pos_])) {
            ++pos_;
        }
    }

    bool consume(char c) {
        ws();
        if (pos_ < in_.size() && in_[pos_] == c) {
            ++pos_;
            return true;
        }
        return false;
    }

    bool boundary_at(size_t at) const {
        if (at == in_.size()) {
            return true;
        }
        const char c = in_[at];
        return json_space(c) || c == ',' || c == ']' || c == '}';
    }

    void claim() {
        if (values_ == lim_.values) {
            budget("Scene JSON exceeds its total-value budget");
        }
        ++values_;
    }

    void open(char c) {
        claim();
        if (depth_ == lim_.depth) {
            budget("Scene JSON exceeds its nesting-depth budget");
        }
        if (!consume(c)) {
            syntax(std::string("Expected '") + c + "'");
        }
        ++depth_;
    }

    void skip_value() {
        ws();
        const char c = pos_ < in_.size() ? in_[pos_] : '\0';
        if (c == '{') {
            skip_object();
        } else if (c == '[') {
            array([&](uint64_t) { skip_value(); });
        } else if (c == '"') {
            string();
        } else if (c == 't' || c == 'f' || c == 'n') {
            claim();
            for (const char* literal : {"true", "false", "null"}) {
                const size_t n = std::strlen(literal);
                if (in_.size() - pos_ >= n && in_.compare(pos_, n, literal) == 0 && boundary_at(pos_ + n)) {
                    pos_ += n;
                    return;
                }
            }
            syntax("Expected a JSON value");
        } else {
            claim();
            number_token(false, false);
        }
    }

    void add_string_bytes(std::string& out, std::string_view bytes) {
        const uint64_t remaining = lim_.string_bytes - string_bytes_;
        if (out.size() > remaining || bytes.size() > remaining - out.size()) {
            budget("Scene JSON exceeds its decoded-string byte budget");
        }
        out.append(bytes.data(), bytes.size());
    }

    uint32_t hex_quad() {
        if (in_.size() - pos_ < 4) {
            syntax("Incomplete JSON Unicode escape");
        }
        uint32_t v = 0;
        for (int k = 0; k < 4; ++k) {
            const char c = in_[pos_++];
            v <<= 4;
            if (c >= '0' && c <= '9') {
                v |= static_cast<uint32_t>(c - '0');
            } else if (c >= 'a' && c <= 'f') {
                v |= static_cast<uint32_t>(c - 'a' + 10);
            } else if (c >= 'A' && c <= 'F') {
                v |= static_cast<uint32_t>(c - 'A' + 10);
            } else {
                syntax("Invalid JSON Unicode escape");
            }
        }
        return v;
    }

    std::string string_token() {
        ws();
        if (pos_ >= in_.size() || in_[pos_] != '"') {
            syntax("Expected a JSON string");
        }
        ++pos_;
        std::string out;
        while (pos_ < in_.size()) {
            const size_t at = pos_;
            const auto c = static_cast<unsigned char>(in_[pos_++]);
            if (c == '"') {
                string_bytes_ += out.size();
                return out;
            }
            if (c < 0x20U) {
                syntax("JSON strings cannot contain raw control bytes");
            }
            if (c == '\\') {
                if (pos_ >= in_.size()) {
                    syntax("Unterminated JSON escape sequence");
                }
                const char e = in_[pos_++];
                char single = 0;
                switch (e) {
                case '"': case '\\': case '/': single = e; break;
                case 'b': single = '\b'; break;
                case 'f': single = '\f'; break;
                case 'n': single = '\n'; break;
                case 'r': single = '\r'; break;
                case 't': single = '\t'; break;
                case 'u': {
                    const uint32_t first = hex_quad();
                    if (first >= 0xDC00U && first <= 0xDFFFU) {
                        syntax("Unexpected low Unicode surrogate");
                    }
                    uint32_t cp = first;
                    if (first >= 0xD800U && first <= 0xDBFFU) {
                        if (in_.size() - pos_ < 2 || in_[pos_] != '\\' || in_[pos_ + 1] != 'u') {
                            syntax("Missing low Unicode surrogate");
                        }
                        pos_ += 2;
                        const uint32_t second = hex_quad();
                        if (second < 0xDC00U || second > 0xDFFFU) {
                            syntax("Invalid low Unicode surrogate");
                        }
                        cp = 0x10000U + ((first - 0xD800U) << 10) + (second - 0xDC00U);
                    }
                    std::string encoded;
                    append_utf8(encoded, cp);
                    add_string_bytes(out, encoded);
                    continue;
                }
                default:
                    syntax("Unknown JSON escape sequence");
                }
                add_string_bytes(out, std::string_view(&single, 1));
                continue;
            }
            if (c <= 0x7FU) {
                add_string_bytes(out, in_.substr(at, 1));
                continue;
            }
            const size_t n = utf8_length(in_, at);
            if (n == 0) {
                syntax("JSON string contains malformed UTF-8");
            }
            pos_ = at + n;
            add_string_bytes(out, in_.substr(at, n));
        }
        syntax("Unterminated JSON string");
    }

    std::string_view number_token(bool integer_only, bool unsigned_only) {
        ws();
        const size_t start = pos_;
        const auto digit = [&](size_t at) { return at < in_.size() && in_[at] >= '0' && in_[at] <= '9'; };
        if (pos_ < in_.size() && in_[pos_] == '-') {
            if (unsigned_only) {
                syntax("Expected an unsigned JSON integer");
            }
            ++pos_;
        }
        if (!digit(pos_)) {
            syntax(integer_only ? "Expected a JSON integer" : "Expected a JSON number");
        }
        if (in_[pos_] == '0') {
            ++pos_;
            if (digit(pos_)) {
                syntax("JSON numbers cannot contain leading zeroes");
            }
        } else {
            while (digit(pos_)) {
                ++pos_;
            }
        }
        if (pos_ < in_.size() && in_[pos_] == '.') {
            if (integer_only) {
                syntax("Expected an integer without a fraction");
            }
            ++pos_;
            const size_t fraction = pos_;
            while (digit(pos_)) {
                ++pos_;
            }
            if (pos_ == fraction) {
                syntax("A JSON fraction requires at least one digit");
            }
        }
        if (pos_ < in_.size() && (in_[pos_] == 'e' || in_[pos_] == 'E')) {
            if (integer_only) {
                syntax("Expected an integer without an exponent");
            }
            ++pos_;
            if (pos_ < in_.size() && (in_[pos_] == '+' || in_[pos_] == '-')) {
                ++pos_;
            }
            const size_t exponent = pos_;
            while (digit(pos_)) {
                ++pos_;
            }
            if (pos_ == exponent) {
                syntax("A JSON exponent requires at least one digit");
            }
        }
        if (!boundary_at(pos_)) {
            syntax("Invalid byte after JSON number");
        }
        return in_.substr(start, pos_ - start);
    }

    std::string_view in_;
    const Limits& lim_;
    size_t pos_ = 0;
    uint64_t values_ = 0;
    uint64_t string_bytes_ = 0;
    uint32_t depth_ = 0;
};

// ---------------------------------------------------------------------------------------------
// The decoded description (SceneDescriptionInput, SceneDescription.hpp; records of FrameScene.hpp).

struct Film {
    uint32_t id = 0, width = 0, height = 0;
    uint32_t crop[4] = {};
    uint32_t precision = 0;  // AccumulationPrecision: 0 float32, 1 float64
};

struct Camera {
    uint32_t id = 0, film = 0;
    float origin[3] = {}, normal[3] = {}, tangent[3] = {}, bitangent[3] = {};
    float vfov = 0, t_min = 0, t_max = 0;
    uint32_t mask = 0, medium = 0;
};

struct RenderOptions {
    uint32_t id = 0, film = 0;
    uint32_t spp = 1, max_depth = 4, tile = 16;
    uint64_t seed = 0;
    uint32_t jitter = 1, mis = 1, strategy = 0;  // PixelJitterMode, MisHeuristic, LightSamplingStrategy
    uint32_t depth[5] = {4, 4, 4, 4, 4};
    bool roulette = false;
    uint32_t roulette_first = 0;
    float roulette_min = 0, roulette_max = 0;
};

struct ConstantTexture {
    uint32_t id = 0;
    uint32_t kind = 0;  // 0 float, 1 color, 2 spectrum
    float value[4] = {};
};

struct Geometry {
    uint32_t id = 0;
    std::vector<float> positions, normals, uvs;
    std::vector<uint32_t> triangles;
};

struct Packet {
    float nanometers[4] = {};
    float pdf[4] = {};
    bool operator==(const Packet& o) const {
        for (int l = 0; l < 4; ++l) {
            if (!(nanometers[l] == o.nanometers[l]) || !(pdf[l] == o.pdf[l])) {
                return false;
            }
        }
        return true;
    }
};

struct Material {
    uint32_t id = 0;
    bool spectral = false;
    Packet packet;
    uint32_t frame_mode = 0;
    float rotation = 0;
    std::vector<bf200_closure_v1> closures;
    float probabilities[kClosureCapacity] = {};
    float emission[4] = {};
};

struct Instance {
    uint32_t id = 0;
    bool has_parent = false;
    uint32_t parent = 0, object = 0, geometry = 0, material = 0;
    float local[16] = {};
    uint32_t mask = 0;
};

enum LightKind : uint32_t { kPoint = 1, kDirectional = 2, kSpot = 3, kEnvironment = 4 };

struct Light {
    uint32_t id = 0;
    uint32_t kind = 0;
    float position[3] = {}, error[3] = {}, direction[3] = {};
    float inner = 0, outer = 0;
    float spectrum[4] = {};  // intensity, irradiance, on-axis intensity or environment radiance
    Packet packet;           // environment
};

}  // namespace scene_json
}  // namespace bf200

struct bf200_scene_json {
    uint32_t active_film = 0, active_camera = 0, active_options = 0;
    std::vector<bf200::scene_json::Film> films;
    std::vector<bf200::scene_json::Camera> cameras;
    std::vector<bf200::scene_json::RenderOptions> options;
    std::vector<bf200::scene_json::ConstantTexture> constant_textures;
    std::vector<uint32_t> objects;
    std::vector<bf200::scene_json::Geometry> geometries;
    std::vector<bf200::scene_json::Material> materials;
    std::vector<bf200::scene_json::Instance> instances;
    std::vector<bf200::scene_json::Light> lights;
    // Resolved world transforms (AffineTransform::from_matrix) of the sorted instances.
    std::vector<float> world, world_inverse;
    // Committed arrays of bf200_scene_json_frame, built once.
    bool committed = false;
    std::vector<bf200_geometry_v1> c_geometries;
    std::vector<float> c_positions, c_normals, c_uvs;
    std::vector<uint32_t> c_triangles;
    std::vector<bf200_material_v1> c_materials;
    std::vector<bf200_closure_v1> c_closures;
    std::vector<bf200_instance_v1> c_instances;
    std::vector<bf200_punctual_light_v1> c_punctual;
};

namespace bf200 {
namespace scene_json {
namespace {

// The decoded-scene budget (SceneDescriptionJsonReader.cpp:69-135).
class Budget {
  public:
    explicit Budget(const Limits& l) : lim_(l) {}
    void bytes(uint64_t n, const std::string& what) {
        if (n > lim_.decoded - used_) {
            refuse(kExhausted, what + " exceeds the decoded scene byte budget.");
        }
        used_ += n;
    }
    void vertex() {
        if (1 > lim_.mesh_vertices - vertices_) {
            refuse(kExhausted, "Scene geometry exceeds the configured mesh-vertex limit.");
        }
        ++vertices_;
    }
    void triangle() {
        if (1 > lim_.mesh_triangles - triangles_) {
            refuse(kExhausted, "Scene geometry exceeds the configured mesh-triangle limit.");
        }
        ++triangles_;
    }
    const Limits& limits() const { return lim_; }

  private:
    const Limits& lim_;
    uint64_t used_ = 0, vertices_ = 0, triangles_ = 0;
};

[[noreturn]] void unknown(const char* context, std::string_view key) {
    refuse(kInvalid, std::string("Unknown ") + context + " key '" + std::string(key) + "'.");
}

// An object whose keys must include every bit of `required` (read_closed_object).
template <typename F> void closed(Cursor& c, uint64_t required, const char* context, F&& field) {
    uint64_t seen = 0;
    c.object([&](std::string_view key) { field(key, seen); });
    if ((seen & required) != required) {
        refuse(kInvalid, std::string(context) + " is missing one or more required keys.");
    }
}

// An array of exactly N elements (read_fixed_array).
template <size_t N, typename F> void fixed(Cursor& c, const char* what, F&& element) {
    uint64_t count = 0;
    c.array([&](uint64_t index) {
        if (index >= N) {
            refuse(kInvalid, std::string(what) + " contains too many elements.");
        }
        element(static_cast<size_t>(index));
        count = index + 1;
    });
    if (count != N) {
        refuse(kInvalid, std::string(what) + " must contain exactly " + std::to_string(N) + " elements.");
    }
}

uint32_t u32(Cursor& c, const char* what) {
    const uint64_t v = c.u64();
    if (v > std::numeric_limits<uint32_t>::max()) {
        refuse(kInvalid, std::string(what) + " exceeds the 32-bit unsigned domain.");
    }
    return static_cast<uint32_t>(v);
}

uint32_t identifier(Cursor& c, const char* what) {
    const uint64_t v = c.u64();
    if (v > std::numeric_limits<uint32_t>::max()) {
        refuse(kInvalid, std::string(what) + " exceeds the 32-bit identifier domain.");
    }
    return static_cast<uint32_t>(v);
}

void floats3(Cursor& c, const char* what, float* out) {
    fixed<3>(c, what, [&](size_t i) { out[i] = c.real(); });
}

void spectrum(Cursor& c, const char* what, float* out) {
    fixed<4>(c, what, [&](size_t i) { out[i] = c.real(); });
}

// A string among `names` (read_named_enum): its index.
template <size_t N> uint32_t named(Cursor& c, const char* what, const char* const (&names)[N]) {
    const std::string s = c.string();
    for (size_t i = 0; i < N; ++i) {
        if (s == names[i]) {
            return static_cast<uint32_t>(i);
        }
    }
    refuse(kInvalid, std::string(what) + " has unsupported value '" + s + "'.");
}

// The registry of one root key (read_registry).
template <typename F> void registry(Cursor& c, Budget& budget, uint64_t record_bytes, const char* what, F&& record) {
    c.array([&](uint64_t index) {
        if (index >= budget.limits().records) {
            refuse(kExhausted, std::string(what) + " exceeds the configured registry-record limit.");
        }
        budget.bytes(record_bytes, what);
        record();
    });
}

Film read_film(Cursor& c) {
    Film f;
    closed(c, 0x0F, "Scene film", [&](std::string_view key, uint64_t& seen) {
        if (key == "id") {
            f.id = identifier(c, "Film identifier");
            seen |= 1U;
        } else if (key == "extent") {
            uint32_t v[2];
            fixed<2>(c, "Film extent", [&](size_t i) { v[i] = u32(c, "Film extent"); });
            f.width = v[0], f.height = v[1];
            seen |= 2U;
        } else if (key == "crop") {
            uint32_t v[4];
            fixed<4>(c, "Film crop", [&](size_t i) { v[i] = u32(c, "Film crop"); });
            std::copy(v, v + 4, f.crop);
            seen |= 4U;
        } else if (key == "accumulation") {
            static const char* const names[] = {"float32", "float64"};
            f.precision = named(c, "Film accumulation precision", names);
            seen |= 8U;
        } else {
            unknown("scene film", key);
        }
    });
    return f;
}

float squared(const float* v) {
    return v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
}

float dot3(const float* a, const float* b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// local_frame_detail::orthonormal (LocalFrame.hpp:73-85).
bool orthonormal(const float* t, const float* b, const float* n) {
    const float tolerance = std::numeric_limits<float>::epsilon() * 128.0F;
    const float cross[3] = {t[1] * b[2] - t[2] * b[1], t[2] * b[0] - t[0] * b[2], t[0] * b[1] - t[1] * b[0]};
    return std::abs(squared(t) - 1.0F) <= tolerance && std::abs(squared(b) - 1.0F) <= tolerance &&
           std::abs(squared(n) - 1.0F) <= tolerance && std::abs(dot3(t, b)) <= tolerance &&
           std::abs(dot3(n, t)) <= tolerance && std::abs(dot3(b, n)) <= tolerance &&
           std::abs(dot3(cross, n) - 1.0F) <= tolerance;
}

Camera read_camera(Cursor& c) {
    Camera cam;
    closed(c, 0x07, "Scene camera", [&](std::string_view key, uint64_t& seen) {
        if (key == "id") {
            cam.id = identifier(c, "Camera identifier");
            seen |= 1U;
        } else if (key == "film") {
            cam.film = identifier(c, "Camera film identifier");
            seen |= 2U;
        } else if (key == "model") {
            std::string type;
            closed(c, 0x3FF, "Scene camera model", [&](std::string_view k, uint64_t& s) {
                if (k == "type") {
                    type = c.string();
                    s |= 1U;
                } else if (k == "origin") {
                    floats3(c, "Camera origin", cam.origin);
                    s |= 2U;
                } else if (k == "normal") {
                    floats3(c, "Camera normal", cam.normal);
                    s |= 4U;
                } else if (k == "tangent") {
                    floats3(c, "Camera tangent", cam.tangent);
                    s |= 8U;
                } else if (k == "bitangent") {
                    floats3(c, "Camera bitangent", cam.bitangent);
                    s |= 16U;
                } else if (k == "vertical_fov_radians") {
                    cam.vfov = c.real();
                    s |= 32U;
                } else if (k == "t_min") {
                    cam.t_min = c.real();
                    s |= 64U;
                } else if (k == "t_max") {
                    cam.t_max = c.real();
                    s |= 128U;
                } else if (k == "visibility_mask") {
                    cam.mask = u32(c, "Camera visibility mask");
                    s |= 256U;
                } else if (k == "current_medium") {
                    cam.medium = identifier(c, "Camera medium");
                    s |= 512U;
                } else {
                    unknown("scene camera model", k);
                }
            });
            if (type != "pinhole") {
                refuse(kInvalid, "Scene camera model type is unsupported.");
            }
            if (!orthonormal(cam.tangent, cam.bitangent, cam.normal)) {
                refuse(kInvalid, "Snapshot frame axes must be finite, orthonormal, and right-handed.");
            }
            seen |= 4U;
        } else {
            unknown("scene camera", key);
        }
    });
    return cam;
}

void read_roulette(Cursor& c, RenderOptions& o) {
    std::string mode;
    uint64_t seen = 0;
    c.object([&](std::string_view key) {
        if (key == "mode") {
            mode = c.string();
            seen |= 1U;
        } else if (key == "first_eligible_depth") {
            o.roulette_first = u32(c, "Russian roulette first eligible depth");
            seen |= 2U;
        } else if (key == "minimum_survival_probability") {
            o.roulette_min = c.real();
            seen |= 4U;
        } else if (key == "maximum_survival_probability") {
            o.roulette_max = c.real();
            seen |= 8U;
        } else {
            unknown("Russian roulette", key);
        }
    });
    if ((seen & 1U) == 0) {
        refuse(kInvalid, "Russian roulette is missing its mode.");
    }
    if (mode == "disabled") {
        if (seen != 1U) {
            refuse(kInvalid, "Disabled Russian roulette cannot contain enabled-mode parameters.");
        }
        o.roulette = false, o.roulette_first = 0, o.roulette_min = 0.0F, o.roulette_max = 0.0F;
        return;
    }
    if (mode != "enabled") {
        refuse(kInvalid, "Russian roulette mode is unsupported.");
    }
    if (seen != 0x0FU) {
        refuse(kInvalid, "Enabled Russian roulette requires every survival parameter.");
    }
    // RussianRoulettePolicy::create_enabled (RussianRoulette.hpp:41-70)
    if (o.roulette_first == 0) {
        refuse(kInvalid, "Russian roulette requires a strictly positive first eligible depth.");
    }
    const float lo = o.roulette_min, hi = o.roulette_max;
    if (!std::isfinite(lo) || !std::isfinite(hi) || !(lo > 0.0F) || !(lo < 1.0F) || hi < lo || hi > 1.0F) {
        refuse(kInvalid, "Russian roulette survival bounds must be finite and satisfy 0 < minimum < 1 and "
                         "minimum <= maximum <= 1.");
    }
    o.roulette = true;
}

RenderOptions read_render_options(Cursor& c) {
    RenderOptions o;
    closed(c, 0x7FF, "Scene render options", [&](std::string_view key, uint64_t& seen) {
        if (key == "id") {
            o.id = identifier(c, "Render-options identifier");
            seen |= 1U;
        } else if (key == "film") {
            o.film = identifier(c, "Render-options film identifier");
            seen |= 2U;
        } else if (key == "samples_per_pixel") {
            o.spp = u32(c, "Samples per pixel");
            seen |= 4U;
        } else if (key == "maximum_path_depth") {
            o.max_depth = u32(c, "Maximum path depth");
            seen |= 8U;
        } else if (key == "tile_edge_length") {
            o.tile = u32(c, "Tile edge length");
            seen |= 16U;
        } else if (key == "seed") {
            o.seed = c.u64();
            seen |= 32U;
        } else if (key == "pixel_jitter") {
            static const char* const names[] = {"center", "uniform"};
            o.jitter = named(c, "Pixel-jitter mode", names);
            seen |= 64U;
        } else if (key == "mis_heuristic") {
            static const char* const names[] = {"balance", "power"};
            o.mis = named(c, "MIS heuristic", names);
            seen |= 128U;
        } else if (key == "light_sampling_strategy") {
            static const char* const names[] = {"uniform", "power_weighted", "spatial_tree"};
            o.strategy = named(c, "Light-sampling strategy", names);
            seen |= 256U;
        } else if (key == "depth_limits") {
            closed(c, 0x1F, "Path depth limits", [&](std::string_view k, uint64_t& s) {
                static const char* const names[] = {"diffuse", "glossy", "specular", "transmission", "volume"};
                for (int i = 0; i < 5; ++i) {
                    if (k == names[i]) {
                        o.depth[i] = u32(c, "Path depth limit");
                        s |= 1U << i;
                        return;
                    }
                }
                unknown("path depth limits", k);
            });
            seen |= 512U;
        } else if (key == "russian_roulette") {
            read_roulette(c, o);
            seen |= 1024U;
        } else {
            unknown("scene render options", key);
        }
    });
    return o;
}

ConstantTexture read_constant_texture(Cursor& c) {
    ConstantTexture t;
    std::string type;
    int shape = -1;  // 0 scalar, 1 three values, 2 four values
    closed(c, 0x07, "Scene constant texture", [&](std::string_view key, uint64_t& seen) {
        if (key == "id") {
            t.id = identifier(c, "Texture identifier");
            seen |= 1U;
        } else if (key == "type") {
            type = c.string();
            seen |= 2U;
        } else if (key == "value") {
            if (!c.peek_array()) {
                t.value[0] = c.real();
                shape = 0;
            } else {
                uint64_t count = 0;
                float v[4] = {};
                c.array([&](uint64_t index) {
                    if (index >= 4) {
                        refuse(kInvalid, "A constant texture value contains too many elements.");
                    }
                    v[index] = c.real();
                    count = index + 1;
                });
                if (count != 3 && count != 4) {
                    refuse(kInvalid, "A constant texture array must contain exactly three or four values.");
                }
                std::copy(v, v + 4, t.value);
                shape = count == 3 ? 1 : 2;
            }
            seen |= 4U;
        } else {
            unknown("scene constant texture", key);
        }
    });
    // ConstantFloat/Color/SpectrumTexture::create only require finite values, which every
    // decoded number is.
    if (type == "float" && shape == 0) {
        t.kind = 0;
    } else if (type == "color" && shape == 1) {
        t.kind = 1;
    } else if (type == "spectrum" && shape == 2) {
        t.kind = 2;
    } else {
        refuse(kInvalid, "A scene constant texture has an unsupported type or mismatched value shape.");
    }
    return t;
}

Geometry read_geometry(Cursor& c, Budget& budget) {
    Geometry g;
    closed(c, 0x03, "Scene geometry", [&](std::string_view key, uint64_t& seen) {
        if (key == "id") {
            g.id = identifier(c, "Geometry identifier");
            seen |= 1U;
        } else if (key == "mesh") {
            closed(c, 0x0F, "Scene triangle mesh", [&](std::string_view k, uint64_t& s) {
                const uint64_t vertex_limit = budget.limits().mesh_vertices;
                if (k == "positions") {
                    c.array([&](uint64_t) {
                        budget.vertex();
                        budget.bytes(kPositionBytes, "Mesh positions");
                        float p[3];
                        floats3(c, "Mesh position", p);
                        g.positions.insert(g.positions.end(), p, p + 3);
                    });
                    s |= 1U;
                } else if (k == "normals") {
                    c.array([&](uint64_t index) {
                        if (index >= vertex_limit) {
                            refuse(kExhausted, "Mesh normals exceed the configured mesh-vertex limit.");
                        }
                        if (index >= g.positions.size() / 3 && !g.positions.empty()) {
                            refuse(kInvalid, "A mesh contains more normals than positions.");
                        }
                        budget.bytes(kNormalBytes, "Mesh normals");
                        float n[3];
                        floats3(c, "Mesh normal", n);
                        g.normals.insert(g.normals.end(), n, n + 3);
                    });
                    s |= 2U;
                } else if (k == "texture_coordinates") {
                    c.array([&](uint64_t index) {
                        if (index >= vertex_limit) {
                            refuse(kExhausted, "Mesh texture coordinates exceed the configured mesh-vertex limit.");
                        }
                        if (index >= g.positions.size() / 3 && !g.positions.empty()) {
                            refuse(kInvalid, "A mesh contains more texture coordinates than positions.");
                        }
                        budget.bytes(kTextureCoordinateBytes, "Mesh texture coordinates");
                        float uv[2];
                        fixed<2>(c, "Mesh texture coordinate", [&](size_t i) { uv[i] = c.real(); });
                        g.uvs.insert(g.uvs.end(), uv, uv + 2);
                    });
                    s |= 4U;
                } else if (k == "triangles") {
                    c.array([&](uint64_t) {
                        budget.triangle();
                        budget.bytes(kTriangleBytes, "Mesh triangles");
                        uint32_t t[3];
                        fixed<3>(c, "Triangle indices", [&](size_t i) { t[i] = u32(c, "Triangle vertex index"); });
                        g.triangles.insert(g.triangles.end(), t, t + 3);
                    });
                    s |= 8U;
                } else {
                    unknown("scene triangle mesh", k);
                }
            });
            // TriangleMesh::create (TriangleMesh.cpp:60-130)
            const uint64_t vertices = g.positions.size() / 3, triangles = g.triangles.size() / 3;
            if (vertices == 0) {
                refuse(kInvalid, "A triangle mesh requires at least one aligned vertex.");
            }
            if (triangles == 0) {
                refuse(kInvalid, "A triangle mesh requires at least one indexed triangle.");
            }
            if (g.normals.size() / 3 != vertices || g.uvs.size() / 2 != vertices) {
                refuse(kInvalid, "Triangle mesh positions, normals, and texture coordinates must be aligned.");
            }
            if (vertices > std::numeric_limits<uint32_t>::max() || triangles > std::numeric_limits<uint32_t>::max()) {
                refuse(kExhausted, "Triangle mesh counts exceed the supported 32-bit index domain.");
            }
            if (const char* problem = triangle_mesh_problem(g.positions.data(), g.normals.data(), g.uvs.data(),
                                                            vertices, g.triangles.data(), triangles)) {
                refuse(kInvalid, problem);
            }
            seen |= 2U;
        } else {
            unknown("scene geometry", key);
        }
    });
    return g;
}

void read_packet(Cursor& c, Packet& p) {
    closed(c, 0x03, "Sampled wavelengths", [&](std::string_view key, uint64_t& seen) {
        if (key == "nanometers") {
            spectrum(c, "Wavelength nanometers", p.nanometers);
            seen |= 1U;
        } else if (key == "pdf") {
            spectrum(c, "Wavelength PDFs", p.pdf);
            seen |= 2U;
        } else {
            unknown("sampled wavelengths", key);
        }
    });
}

// One closure component (read_closure_component, append_closure).
bf200_closure_v1 read_component(Cursor& c, float& probability) {
    std::string type;
    float weight[4] = {}, eta[4] = {}, k[4] = {};
    float roughness = 0, exterior = 0, interior = 0, ax = 0, ay = 0;
    uint64_t seen = 0;
    c.object([&](std::string_view key) {
        if (key == "probability") {
            probability = c.real();
            seen |= 1U;
        } else if (key == "type") {
            type = c.string();
            seen |= 2U;
        } else if (key == "weight") {
            spectrum(c, "Closure weight", weight);
            seen |= 4U;
        } else if (key == "roughness") {
            roughness = c.real();
            seen |= 8U;
        } else if (key == "eta") {
            spectrum(c, "Closure eta", eta);
            seen |= 16U;
        } else if (key == "k") {
            spectrum(c, "Closure k", k);
            seen |= 32U;
        } else if (key == "exterior_eta") {
            exterior = c.real();
            seen |= 64U;
        } else if (key == "interior_eta") {
            interior = c.real();
            seen |= 128U;
        } else if (key == "alpha_x") {
            ax = c.real();
            seen |= 256U;
        } else if (key == "alpha_y") {
            ay = c.real();
            seen |= 512U;
        } else {
            unknown("closure component", key);
        }
    });
    if ((seen & 0x07U) != 0x07U) {
        refuse(kInvalid, "A closure component is missing probability, type, or weight.");
    }
    bf200_closure_v1 out{};
    uint64_t expected = 0x07U;
    if (type == "lambertian_reflection") {
        out.kind = BF200_CLOSURE_LAMBERTIAN_REFLECTION;
    } else if (type == "rough_diffuse_reflection") {
        out.kind = BF200_CLOSURE_ROUGH_DIFFUSE_REFLECTION;
        expected |= 8U;
        out.parameters[0] = roughness;
    } else if (type == "rough_conductor_reflection") {
        out.kind = BF200_CLOSURE_ROUGH_CONDUCTOR_REFLECTION;
        expected |= 16U | 32U | 256U | 512U;
        std::copy(eta, eta + 4, out.parameters);
        std::copy(k, k + 4, out.parameters + 4);
        out.parameters[8] = ax, out.parameters[9] = ay;
    } else if (type == "rough_dielectric") {
        out.kind = BF200_CLOSURE_ROUGH_DIELECTRIC;
        expected |= 64U | 128U | 256U | 512U;
        out.parameters[0] = exterior, out.parameters[1] = interior, out.parameters[2] = ax, out.parameters[3] = ay;
    } else if (type == "specular_reflection") {
        out.kind = BF200_CLOSURE_SPECULAR_REFLECTION;
    } else if (type == "specular_transmission") {
        out.kind = BF200_CLOSURE_SPECULAR_TRANSMISSION;
        expected |= 64U | 128U;
        out.parameters[0] = exterior, out.parameters[1] = interior;
    } else {
        refuse(kInvalid, "A closure component type is unsupported.");
    }
    if (seen != expected) {
        refuse(kInvalid, "A closure component has missing or type-incompatible parameters.");
    }
    out.lobes = closure_lobes(out.kind);
    std::copy(weight, weight + 4, out.weight);
    if (!valid_closure_payload(out)) {
        refuse(kInvalid, "A closure component payload cannot be represented without repair.");
    }
    return out;
}

void read_spectral(Cursor& c, Material& m) {
    closed(c, 0x1F, "Scene spectral material", [&](std::string_view key, uint64_t& seen) {
        if (key == "wavelengths") {
            read_packet(c, m.packet);
            seen |= 1U;
        } else if (key == "closures") {
            float given[kClosureCapacity] = {};
            m.closures.clear();
            closed(c, 0x07, "Scene closure mixture", [&](std::string_view k, uint64_t& s) {
                if (k == "frame_mode") {
                    static const char* const names[] = {"shading_normal", "surface_tangent"};
                    m.frame_mode = named(c, "Closure frame mode", names);
                    s |= 1U;
                } else if (k == "tangent_rotation_radians") {
                    m.rotation = c.real();
                    s |= 2U;
                } else if (k == "components") {
                    m.closures.clear();
                    c.array([&](uint64_t index) {
                        if (index >= kClosureCapacity) {
                            refuse(kExhausted, "A closure mixture exceeds its fixed component capacity.");
                        }
                        m.closures.push_back(read_component(c, given[index]));
                    });
                    s |= 4U;
                } else {
                    unknown("scene closure mixture", k);
                }
            });
            // SceneClosureMixture::create (FrameScene.cpp:355-384)
            if (!(std::isfinite(m.rotation) && m.rotation >= -kPi && m.rotation < kPi)) {
                refuse(kInvalid, "A scene closure mixture requires a finite tangent rotation in [-pi, pi).");
            }
            float cdf[kClosureCapacity + 1];
            if (!project_component_distribution(given, static_cast<uint32_t>(m.closures.size()), m.probabilities, cdf)) {
                refuse(kInvalid, "A closure mixture's component probabilities do not form a distribution.");
            }
            seen |= 2U;
        } else if (key == "emission") {
            spectrum(c, "Material emission", m.emission);
            seen |= 4U;
        } else if (key == "normal_map" || key == "bump_map") {
            if (!c.peek_null()) {
                c.skip_object();
                refuse(kUnavailable, "Normal and bump maps are unavailable: this backend has no image textures.");
            }
            c.null();
            seen |= key == "normal_map" ? 8U : 16U;
        } else {
            unknown("scene spectral material", key);
        }
    });
}

Material read_material(Cursor& c) {
    Material m;
    closed(c, 0x03, "Scene material", [&](std::string_view key, uint64_t& seen) {
        if (key == "id") {
            m.id = identifier(c, "Material identifier");
            seen |= 1U;
        } else if (key == "spectral") {
            if (c.peek_null()) {
                c.null();
                const uint32_t id = m.id;
                m = Material();
                m.id = id;
            } else {
                read_spectral(c, m);
                m.spectral = true;
            }
            seen |= 2U;
        } else {
            unknown("scene material", key);
        }
    });
    return m;
}

Instance read_instance(Cursor& c) {
    Instance in;
    closed(c, 0x7F, "Scene instance", [&](std::string_view key, uint64_t& seen) {
        if (key == "id") {
            in.id = identifier(c, "Instance identifier");
            seen |= 1U;
        } else if (key == "parent") {
            if (c.peek_null()) {
                c.null();
                in.has_parent = false;
            } else {
                in.parent = identifier(c, "Parent instance identifier");
                in.has_parent = true;
            }
            seen |= 2U;
        } else if (key == "object") {
            in.object = identifier(c, "Object identifier");
            seen |= 4U;
        } else if (key == "geometry") {
            in.geometry = identifier(c, "Geometry identifier");
            seen |= 8U;
        } else if (key == "material") {
            in.material = identifier(c, "Material identifier");
            seen |= 16U;
        } else if (key == "local_to_parent") {
            fixed<16>(c, "Instance local-to-parent matrix", [&](size_t i) { in.local[i] = c.real(); });
            seen |= 32U;
        } else if (key == "visibility_mask") {
            in.mask = u32(c, "Instance visibility mask");
            seen |= 64U;
        } else {
            unknown("scene instance", key);
        }
    });
    return in;
}

Light read_light(Cursor& c) {
    Light l;
    std::string type;
    uint64_t seen = 0;
    float point_intensity[4] = {}, irradiance[4] = {}, on_axis[4] = {}, radiance[4] = {};
    float propagation[3] = {}, emission_direction[3] = {};
    c.object([&](std::string_view key) {
        if (key == "id") {
            l.id = identifier(c, "Light identifier");
            seen |= 1U;
        } else if (key == "type") {
            type = c.string();
            seen |= 2U;
        } else if (key == "position") {
            floats3(c, "Light position", l.position);
            seen |= 4U;
        } else if (key == "absolute_position_error") {
            floats3(c, "Light absolute position error", l.error);
            seen |= 8U;
        } else if (key == "spectral_radiant_intensity") {
            spectrum(c, "Point-light spectral radiant intensity", point_intensity);
            seen |= 16U;
        } else if (key == "propagation_direction") {
            floats3(c, "Directional-light propagation direction", propagation);
            seen |= 32U;
        } else if (key == "spectral_irradiance") {
            spectrum(c, "Directional-light spectral irradiance", irradiance);
            seen |= 64U;
        } else if (key == "emission_direction") {
            floats3(c, "Spot-light emission direction", emission_direction);
            seen |= 128U;
        } else if (key == "inner_half_angle_radians") {
            l.inner = c.real();
            seen |= 256U;
        } else if (key == "outer_half_angle_radians") {
            l.outer = c.real();
            seen |= 512U;
        } else if (key == "on_axis_spectral_radiant_intensity") {
            spectrum(c, "Spot-light on-axis spectral radiant intensity", on_axis);
            seen |= 1024U;
        } else if (key == "wavelengths") {
            read_packet(c, l.packet);
            seen |= 2048U;
        } else if (key == "radiance") {
            spectrum(c, "Environment radiance", radiance);
            seen |= 4096U;
        } else {
            unknown("scene light", key);
        }
    });
    if ((seen & 0x03U) != 0x03U) {
        refuse(kInvalid, "A scene light is missing its identifier or explicit type.");
    }
    uint64_t expected = 0x03U;
    if (type == "point") {
        l.kind = kPoint;
        expected |= 4U | 8U | 16U;
        std::copy(point_intensity, point_intensity + 4, l.spectrum);
    } else if (type == "directional") {
        l.kind = kDirectional;
        expected |= 32U | 64U;
        std::copy(propagation, propagation + 3, l.direction);
        std::copy(irradiance, irradiance + 4, l.spectrum);
    } else if (type == "spot") {
        l.kind = kSpot;
        expected |= 4U | 8U | 128U | 256U | 512U | 1024U;
        std::copy(emission_direction, emission_direction + 3, l.direction);
        std::copy(on_axis, on_axis + 4, l.spectrum);
    } else if (type == "environment") {
        l.kind = kEnvironment;
        expected |= 2048U | 4096U;
        std::copy(radiance, radiance + 4, l.spectrum);
    } else {
        refuse(kInvalid, "A scene light type is unsupported.");
    }
    if (seen != expected) {
        refuse(kInvalid, "A scene light has missing or type-incompatible parameters.");
    }
    return l;
}

// read_scene (SceneDescriptionJsonReader.cpp:2277-2428).
void read_root(Cursor& c, Budget& budget, bf200_scene_json& d) {
    closed(c, 0x1FFF, "Scene JSON root", [&](std::string_view key, uint64_t& seen) {
        if (key == "schema") {
            if (c.string() != kSchemaName) {
                refuse(kIncompatible, "The native scene schema identifier is incompatible with Blackframe.");
            }
            seen |= 1U;
        } else if (key == "schema_version") {
            if (c.u64() != kSchemaVersion) {
                refuse(kIncompatible, "The native scene schema version is incompatible with Blackframe.");
            }
            seen |= 2U;
        } else if (key == "active") {
            closed(c, 0x07, "Active scene selection", [&](std::string_view k, uint64_t& s) {
                if (k == "film") {
                    d.active_film = identifier(c, "Active film identifier");
                    s |= 1U;
                } else if (k == "camera") {
                    d.active_camera = identifier(c, "Active camera identifier");
                    s |= 2U;
                } else if (k == "render_options") {
                    d.active_options = identifier(c, "Active render-options identifier");
                    s |= 4U;
                } else {
                    unknown("active scene selection", k);
                }
            });
            seen |= 4U;
        } else if (key == "films") {
            registry(c, budget, kFilmBytes, "Scene films", [&] { d.films.push_back(read_film(c)); });
            seen |= 8U;
        } else if (key == "cameras") {
            registry(c, budget, kCameraBytes, "Scene cameras", [&] { d.cameras.push_back(read_camera(c)); });
            seen |= 16U;
        } else if (key == "render_options") {
            registry(c, budget, kRenderOptionsBytes, "Scene render options",
                     [&] { d.options.push_back(read_render_options(c)); });
            seen |= 32U;
        } else if (key == "constant_textures") {
            registry(c, budget, kConstantTextureBytes, "Scene constant textures",
                     [&] { d.constant_textures.push_back(read_constant_texture(c)); });
            seen |= 64U;
        } else if (key == "host_image_textures") {
            registry(c, budget, kHostImageTextureBytes, "Scene host-image textures", [&]() {
                c.skip_object();
                refuse(kUnavailable, "Host-image textures are unavailable: this backend has no image textures.");
            });
            seen |= 128U;
        } else if (key == "objects") {
            registry(c, budget, kObjectBytes, "Scene objects", [&] {
                uint32_t id = 0;
                closed(c, 0x01, "Scene object", [&](std::string_view k, uint64_t& s) {
                    if (k != "id") {
                        unknown("scene object", k);
                    }
                    id = identifier(c, "Object identifier");
                    s |= 1U;
                });
                d.objects.push_back(id);
            });
            seen |= 256U;
        } else if (key == "geometries") {
            registry(c, budget, kGeometryBytes, "Scene geometries",
                     [&] { d.geometries.push_back(read_geometry(c, budget)); });
            seen |= 512U;
        } else if (key == "materials") {
            registry(c, budget, kMaterialBytes, "Scene materials", [&] { d.materials.push_back(read_material(c)); });
            seen |= 1024U;
        } else if (key == "instances") {
            registry(c, budget, kInstanceBytes, "Scene instances", [&] { d.instances.push_back(read_instance(c)); });
            seen |= 2048U;
        } else if (key == "lights") {
            registry(c, budget, kLightBytes, "Scene lights", [&] { d.lights.push_back(read_light(c)); });
            seen |= 4096U;
        } else {
            unknown("scene JSON root", key);
        }
    });
}

// ---------------------------------------------------------------------------------------------
// SceneDescription::create (SceneDescription.cpp:379-552) and the checks it calls.

template <typename R> uint32_t id_of(const R& r) {
    return r.id;
}
uint32_t id_of(uint32_t object) {
    return object;
}

template <typename R> void sort_and_check(std::vector<R>& records, const char* domain) {
    std::stable_sort(records.begin(), records.end(), [](const R& a, const R& b) { return id_of(a) < id_of(b); });
    for (size_t i = 1; i < records.size(); ++i) {
        if (id_of(records[i - 1]) == id_of(records[i])) {
            refuse(kInvalid, std::string("A scene description contains duplicate ") + domain + " identifiers.");
        }
    }
}

template <typename R> long find(const std::vector<R>& records, uint32_t id) {
    const auto it = std::lower_bound(records.begin(), records.end(), id,
                                     [](const R& r, uint32_t v) { return id_of(r) < v; });
    return it != records.end() && id_of(*it) == id ? static_cast<long>(it - records.begin()) : -1;
}

constexpr uint32_t kMaximumDimension = 1U << 20;
constexpr uint64_t kMaximumPixels = std::numeric_limits<uint32_t>::max();

// validate_render_extent (RenderConfiguration.cpp:22-45).
void validate_extent(uint32_t width, uint32_t height) {
    if (width == 0) {
        refuse(kInvalid, "Render extent width must be greater than zero.");
    }
    if (height == 0) {
        refuse(kInvalid, "Render extent height must be greater than zero.");
    }
    if (width > kMaximumDimension || height > kMaximumDimension) {
        refuse(kExhausted, "Render dimensions exceed the configured safety limit.");
    }
    if (static_cast<uint64_t>(width) * height > kMaximumPixels) {
        refuse(kExhausted, "The requested image contains too many pixels.");
    }
}

bool product_exceeds(uint64_t left, uint64_t right, uint64_t limit) {
    return left != 0 && right > limit / left;
}

// validate_render_configuration (RenderConfiguration.cpp:47-118) and the scene-level checks of
// validate_render_options (SceneDescription.cpp:128-173).
void validate_options(const RenderOptions& o, const Film& film) {
    validate_extent(film.width, film.height);
    const uint64_t pixels = static_cast<uint64_t>(film.width) * film.height;
    if (o.spp == 0) {
        refuse(kInvalid, "Render configuration key 'samples_per_pixel' must be greater than zero.");
    }
    if (o.max_depth == 0) {
        refuse(kInvalid, "Render configuration key 'maximum_path_depth' must be greater than zero.");
    }
    if (o.tile == 0) {
        refuse(kInvalid, "Render configuration key 'tile_edge_length' must be greater than zero.");
    }
    if (o.spp > (1U << 24)) {
        refuse(kExhausted, "Samples per pixel exceed the configured safety limit.");
    }
    if (o.max_depth > 4096U) {
        refuse(kExhausted, "Path depth exceeds the configured safety limit.");
    }
    if (o.tile > 4096U) {
        refuse(kExhausted, "Tile dimensions exceed the configured safety limit.");
    }
    if (product_exceeds(pixels, o.spp, 1ULL << 48)) {
        refuse(kExhausted, "The requested sample workload exceeds the safety limit.");
    }
    if (product_exceeds(pixels * o.spp, o.max_depth, 1ULL << 56)) {
        refuse(kExhausted, "The requested transport workload exceeds the safety limit.");
    }
    if (product_exceeds(o.tile, o.tile, kMaximumPixels)) {
        refuse(kExhausted, "The requested tile contains too many pixels.");
    }
    for (uint32_t limit : o.depth) {
        if (limit > o.max_depth) {
            refuse(kInvalid, "A scene path-category limit cannot exceed the global path-depth limit.");
        }
    }
}

// PinholeCamera::create (PinholeCamera.hpp:58-96) after the scene's medium check.
void validate_camera(const Camera& cam, const Film& film, float& half_width, float& half_height) {
    if (cam.medium != 0) {
        refuse(kInvalid, "A scene pinhole camera cannot reference a medium because this scene description has no "
                         "medium registry.");
    }
    validate_extent(film.width, film.height);
    if (!std::isfinite(cam.origin[0]) || !std::isfinite(cam.origin[1]) || !std::isfinite(cam.origin[2])) {
        refuse(kInvalid, "A pinhole camera origin must be finite.");
    }
    if (!std::isfinite(cam.vfov) || cam.vfov <= 0.0F || cam.vfov >= kPi) {
        refuse(kInvalid, "A pinhole vertical field of view must be finite and inside (0, pi).");
    }
    if (!std::isfinite(cam.t_min) || cam.t_min < 0.0F || std::isnan(cam.t_max) || cam.t_max < cam.t_min) {
        refuse(kInvalid, "Pinhole ray bounds must form an ordered non-negative interval.");
    }
    half_height = std::tan(cam.vfov / 2.0F);
    const float aspect = static_cast<float>(film.width) / static_cast<float>(film.height);
    half_width = half_height * aspect;
    if (!std::isfinite(half_height) || !std::isfinite(half_width) || half_height <= 0.0F || half_width <= 0.0F) {
        refuse(kInvalid, "Pinhole projection dimensions are not representable.");
    }
}

// Matrix product of the reference's operator* (MatrixTypes.hpp:41-52): each entry summed from
// zero in component order.
void multiply4(const float* a, const float* b, float* out) {
    for (int r = 0; r < 4; ++r) {
        for (int c = 0; c < 4; ++c) {
            float sum = 0.0F;
            for (int k = 0; k < 4; ++k) {
                sum += a[r * 4 + k] * b[k * 4 + c];
            }
            out[r * 4 + c] = sum;
        }
    }
}

// AffineTransform::from_matrix (Transforms.hpp:14-27).
bool affine(const float* m, float* inverse) {
    if (m[12] != 0.0F || m[13] != 0.0F || m[14] != 0.0F || m[15] != 1.0F) {
        return false;
    }
    float in[16], out[16];
    std::copy(m, m + 16, in);
    if (!invert_matrix4(in, out)) {
        return false;
    }
    std::copy(out, out + 16, inverse);
    return true;
}

// resolve_instance_transforms (SceneHierarchyValidation.cpp:38-130).
void resolve_hierarchy(bf200_scene_json& d) {
    const size_t n = d.instances.size();
    std::vector<float> local_inverse(16 * n);
    for (size_t i = 0; i < n; ++i) {
        if (!affine(d.instances[i].local, &local_inverse[16 * i])) {
            refuse(kInvalid, "A frame scene instance local transform must be finite, affine, and invertible.");
        }
    }
    d.world.assign(16 * n, 0.0F);
    d.world_inverse.assign(16 * n, 0.0F);
    std::vector<uint8_t> state(n, 0);  // 0 unresolved, 1 resolving, 2 resolved
    std::vector<size_t> chain;
    for (size_t start = 0; start < n; ++start) {
        if (state[start] == 2) {
            continue;
        }
        chain.clear();
        size_t current = start;
        while (state[current] != 2) {
            if (state[current] == 1) {
                refuse(kInvalid, "A frame scene instance hierarchy contains a cycle.");
            }
            state[current] = 1;
            chain.push_back(current);
            if (!d.instances[current].has_parent) {
                break;
            }
            const long parent = find(d.instances, d.instances[current].parent);
            if (parent < 0) {
                refuse(kInvalid, "A frame scene instance references an unknown parent instance.");
            }
            current = static_cast<size_t>(parent);
        }
        while (!chain.empty()) {
            const size_t i = chain.back();
            chain.pop_back();
            const Instance& in = d.instances[i];
            if (in.has_parent) {
                const size_t p = static_cast<size_t>(find(d.instances, in.parent));
                multiply4(&d.world[16 * p], in.local, &d.world[16 * i]);
                if (!affine(&d.world[16 * i], &d.world_inverse[16 * i])) {
                    refuse(kInvalid, "A frame scene hierarchy produced an invalid world transform.");
                }
            } else {
                std::copy(in.local, in.local + 16, &d.world[16 * i]);
                std::copy(&local_inverse[16 * i], &local_inverse[16 * i] + 16, &d.world_inverse[16 * i]);
            }
            state[i] = 2;
        }
    }
}

bool finite_nonnegative4(const float* v) {
    for (int l = 0; l < 4; ++l) {
        if (!std::isfinite(v[l]) || v[l] < 0.0F) {
            return false;
        }
    }
    return true;
}

// PathState::create_initial's wavelength checks (PathState.hpp:106-120).
bool valid_packet(const Packet& p) {
    for (int l = 0; l < 4; ++l) {
        if (!std::isfinite(p.nanometers[l]) || p.nanometers[l] < 360.0F || p.nanometers[l] > 830.0F ||
            !std::isfinite(p.pdf[l]) || !(p.pdf[l] > 0.0F)) {
            return false;
        }
    }
    return true;
}

bf200_punctual_light_v1 punctual_record(const Light& l) {
    bf200_punctual_light_v1 p{};
    p.kind = l.kind;
    std::copy(l.position, l.position + 3, p.position);
    std::copy(l.error, l.error + 3, p.position_error);
    std::copy(l.direction, l.direction + 3, p.direction);
    p.inner_half_angle = l.inner;
    p.outer_half_angle = l.outer;
    std::copy(l.spectrum, l.spectrum + 4, p.spectrum);
    return p;
}

// validate_spectral_records (SceneDescription.cpp:265-376).
void validate_spectral(const bf200_scene_json& d) {
    const Light* environment = nullptr;
    for (const Light& l : d.lights) {
        if (l.kind == kEnvironment) {
            if (environment != nullptr) {
                refuse(kInvalid, "A scene description supports at most one spectral environment light.");
            }
            environment = &l;
        }
    }
    bool requires_environment = false;
    for (const Material& m : d.materials) {
        requires_environment = requires_environment || m.spectral;
    }
    for (const Light& l : d.lights) {
        requires_environment = requires_environment || l.kind != kEnvironment;
    }
    if (environment == nullptr) {
        if (!requires_environment) {
            return;
        }
        refuse(kInvalid, "Spectral materials and punctual lights require one explicit environment wavelength packet.");
    }
    if (!valid_packet(environment->packet) || !finite_nonnegative4(environment->spectrum)) {
        refuse(kInvalid, "A scene spectral environment requires valid wavelengths and finite non-negative radiance.");
    }
    for (const Light& l : d.lights) {
        if (l.kind == kEnvironment) {
            continue;
        }
        float cos_inner = 0, cos_outer = 0;
        if (!punctual_light_checks(punctual_record(l), cos_inner, cos_outer)) {
            refuse(kInvalid, l.kind == kPoint         ? "A scene point light contains invalid transport data."
                             : l.kind == kDirectional ? "A scene directional light contains invalid transport data."
                                                      : "A scene spot light contains invalid transport data.");
        }
    }
    for (const Material& m : d.materials) {
        if (!m.spectral) {
            refuse(kInvalid, "Every material in a spectral scene requires explicit spectral data.");
        }
        if (!(m.packet == environment->packet)) {
            refuse(kInvalid, "Scene materials and lights must share one wavelength packet.");
        }
        if (!finite_nonnegative4(m.emission)) {
            refuse(kInvalid, "A scene material contains invalid spectral emission data.");
        }
    }
}

void create_description(bf200_scene_json& d) {
    sort_and_check(d.films, "film");
    sort_and_check(d.cameras, "camera");
    sort_and_check(d.options, "render-options");
    sort_and_check(d.constant_textures, "constant-texture");
    sort_and_check(d.objects, "object");
    sort_and_check(d.geometries, "geometry");
    sort_and_check(d.materials, "material");
    sort_and_check(d.instances, "instance");
    sort_and_check(d.lights, "light");
    const long film = find(d.films, d.active_film);
    const long camera = find(d.cameras, d.active_camera);
    const long options = find(d.options, d.active_options);
    if (film < 0) {
        refuse(kInvalid, "A scene description references an unknown active film identifier.");
    }
    if (camera < 0) {
        refuse(kInvalid, "A scene description references an unknown active camera identifier.");
    }
    if (options < 0) {
        refuse(kInvalid, "A scene description references unknown active render-options.");
    }
    for (const Film& f : d.films) {
        validate_extent(f.width, f.height);  // validate_film_crop (Film.hpp:48-67)
        if (f.crop[0] >= f.crop[2] || f.crop[1] >= f.crop[3]) {
            refuse(kInvalid, "A film crop must have a non-empty half-open pixel range.");
        }
        if (f.crop[2] > f.width || f.crop[3] > f.height) {
            refuse(kInvalid, "A film crop must remain inside the full image extent.");
        }
    }
    for (const Camera& cam : d.cameras) {
        const long f = find(d.films, cam.film);
        if (f < 0) {
            refuse(kInvalid, "A scene camera references an unknown film identifier.");
        }
        float hw = 0, hh = 0;
        validate_camera(cam, d.films[f], hw, hh);
    }
    for (const RenderOptions& o : d.options) {
        const long f = find(d.films, o.film);
        if (f < 0) {
            refuse(kInvalid, "Scene render options reference an unknown film identifier.");
        }
        validate_options(o, d.films[f]);
    }
    if (d.cameras[camera].film != d.active_film) {
        refuse(kInvalid, "The active scene camera must reference the active film.");
    }
    if (d.options[options].film != d.active_film) {
        refuse(kInvalid, "The active scene render-options must reference the active film.");
    }
    for (const Instance& in : d.instances) {
        if (find(d.objects, in.object) < 0) {
            refuse(kInvalid, "A scene instance references an unknown object identifier.");
        }
        if (find(d.geometries, in.geometry) < 0) {
            refuse(kInvalid, "A scene instance references an unknown geometry identifier.");
        }
        if (find(d.materials, in.material) < 0) {
            refuse(kInvalid, "A scene instance references an unknown material identifier.");
        }
        if (in.has_parent && find(d.instances, in.parent) < 0) {
            refuse(kInvalid, "A scene instance references an unknown parent identifier.");
        }
    }
    resolve_hierarchy(d);
    validate_spectral(d);
}

// ---------------------------------------------------------------------------------------------
// Canonical writer (SceneJsonSyntax.cpp:726-1139, SceneDescriptionJsonWriter.cpp).

class Writer {
  public:
    explicit Writer(const Limits& l) : lim_(l) {}

    void begin_object() { open('{'); }
    void end_object() { close('}'); }
    void begin_array() { open('['); }
    void end_array() { close(']'); }

    void key(std::string_view k) {
        count_string(k.size());
        Frame& f = stack_.back();
        if (f.count > 0) {
            append(",");
        }
        escaped(k);
        append(":");
        f.awaiting = true;
    }
    void null() {
        value();
        append("null");
    }
    void string(std::string_view s) {
        value();
        count_string(s.size());
        escaped(s);
    }
    void u64(uint64_t v) {
        value();
        char buf[32];
        const auto r = std::to_chars(buf, buf + sizeof buf, v);
        append(std::string_view(buf, static_cast<size_t>(r.ptr - buf)));
    }
    void real(float v) {
        if (!std::isfinite(v)) {
            refuse(kInvalid, "Canonical scene JSON floats must be finite.");
        }
        value();
        char buf[64];
        const auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::general,
                                     std::numeric_limits<float>::max_digits10);
        append(std::string_view(buf, static_cast<size_t>(r.ptr - buf)));
    }
    // key + value shorthands
    void u64(std::string_view k, uint64_t v) {
        key(k);
        u64(v);
    }
    void real(std::string_view k, float v) {
        key(k);
        real(v);
    }
    void string(std::string_view k, std::string_view v) {
        key(k);
        string(v);
    }
    void reals(const float* v, size_t n) {
        begin_array();
        for (size_t i = 0; i < n; ++i) {
            real(v[i]);
        }
        end_array();
    }
    void reals(std::string_view k, const float* v, size_t n) {
        key(k);
        reals(v, n);
    }
    std::string take() { return std::move(out_); }

  private:
    struct Frame {
        uint64_t count = 0;
        bool object = false;
        bool awaiting = false;
    };
    [[noreturn]] void budget(const char* message) const { refuse(kExhausted, std::string(message) + " At byte " + std::to_string(out_.size()) + "."); }

    void append(std::string_view bytes) {
        if (out_.size() > lim_.encoded || bytes.size() > lim_.encoded - out_.size()) {
            budget("Canonical scene JSON exceeds its output budget.");
        }
        out_.append(bytes.data(), bytes.size());
    }
    void count_string(size_t n) {
        if (strings_ > lim_.string_bytes || n > lim_.string_bytes - strings_) {
            budget("Canonical scene JSON exceeds its decoded-string byte budget.");
        }
        strings_ += n;
    }
    void value() {
        if (values_ == lim_.values) {
            budget("Canonical scene JSON exceeds its total-value budget.");
        }
        ++values_;
        if (stack_.empty()) {
            return;
        }
        Frame& f = stack_.back();
        if (f.object) {
            f.awaiting = false;
            ++f.count;
            return;
        }
        if (f.count > 0) {
            append(",");
        }
        ++f.count;
    }
    void open(char c) {
        value();
        if (stack_.size() == lim_.depth) {
            budget("Canonical scene JSON exceeds its nesting-depth budget.");
        }
        append(std::string_view(&c, 1));
        stack_.push_back(Frame{0, c == '{', false});
    }
    void close(char c) {
        stack_.pop_back();
        append(std::string_view(&c, 1));
    }
    void escaped(std::string_view s) {
        static const char hex[] = "0123456789abcdef";
        append("\"");
        for (size_t i = 0; i < s.size();) {
            const auto c = static_cast<unsigned char>(s[i]);
            if (c > 0x7FU) {
                const size_t n = utf8_length(s, i);
                append(s.substr(i, n));
                i += n;
                continue;
            }
            ++i;
            switch (c) {
            case '"': append("\\\""); break;
            case '\\': append("\\\\"); break;
            case '\b': append("\\b"); break;
            case '\f': append("\\f"); break;
            case '\n': append("\\n"); break;
            case '\r': append("\\r"); break;
            case '\t': append("\\t"); break;
            default:
                if (c < 0x20U) {
                    const char e[6] = {'\\', 'u', '0', '0', hex[(c >> 4) & 0xF], hex[c & 0xF]};
                    append(std::string_view(e, 6));
                } else {
                    const char b = static_cast<char>(c);
                    append(std::string_view(&b, 1));
                }
            }
        }
        append("\"");
    }

    const Limits& lim_;
    std::string out_;
    std::vector<Frame> stack_;
    uint64_t values_ = 0, strings_ = 0;
};

const char* closure_type_name(uint32_t kind) {
    switch (kind) {
    case BF200_CLOSURE_LAMBERTIAN_REFLECTION: return "lambertian_reflection";
    case BF200_CLOSURE_ROUGH_DIFFUSE_REFLECTION: return "rough_diffuse_reflection";
    case BF200_CLOSURE_ROUGH_CONDUCTOR_REFLECTION: return "rough_conductor_reflection";
    case BF200_CLOSURE_ROUGH_DIELECTRIC: return "rough_dielectric";
    case BF200_CLOSURE_SPECULAR_REFLECTION: return "specular_reflection";
    default: return "specular_transmission";
    }
}

void write_packet(Writer& w, const Packet& p) {
    w.begin_object();
    w.reals("nanometers", p.nanometers, 4);
    w.reals("pdf", p.pdf, 4);
    w.end_object();
}

// preflight_description (SceneDescriptionJsonWriter.cpp:65-190): record counts and decoded bytes.
void preflight(const bf200_scene_json& d, const Limits& l) {
    uint64_t decoded = 0;
    const auto add = [&](uint64_t& current, uint64_t amount, uint64_t maximum, const char* message) {
        if (amount > maximum - current) {
            refuse(kExhausted, message);
        }
        current += amount;
    };
    const auto registry_bytes = [&](size_t count, uint64_t record_bytes) {
        if (count > l.records) {
            refuse(kExhausted, "A scene JSON registry exceeds the configured record-count limit.");
        }
        add(decoded, count * record_bytes, l.decoded, "A scene JSON description exceeds the configured decoded-byte limit.");
    };
    registry_bytes(d.films.size(), kFilmBytes);
    registry_bytes(d.cameras.size(), kCameraBytes);
    registry_bytes(d.options.size(), kRenderOptionsBytes);
    registry_bytes(d.constant_textures.size(), kConstantTextureBytes);
    registry_bytes(0, kHostImageTextureBytes);
    registry_bytes(d.objects.size(), kObjectBytes);
    registry_bytes(d.geometries.size(), kGeometryBytes);
    registry_bytes(d.materials.size(), kMaterialBytes);
    registry_bytes(d.instances.size(), kInstanceBytes);
    registry_bytes(d.lights.size(), kLightBytes);
    uint64_t vertices = 0, triangles = 0;
    for (const Geometry& g : d.geometries) {
        const uint64_t v = g.positions.size() / 3, t = g.triangles.size() / 3;
        add(vertices, v, l.mesh_vertices, "Scene JSON meshes exceed the configured vertex limit.");
        add(triangles, t, l.mesh_triangles, "Scene JSON meshes exceed the configured triangle limit.");
        add(decoded, v * (kPositionBytes + kNormalBytes + kTextureCoordinateBytes) + t * kTriangleBytes, l.decoded,
            "A scene JSON description exceeds the configured decoded-byte limit.");
    }
}

std::string write_document(const bf200_scene_json& d, const Limits& l) {
    validate_limits(l);
    preflight(d, l);
    Writer w(l);
    w.begin_object();
    w.string("schema", kSchemaName);
    w.u64("schema_version", kSchemaVersion);
    w.key("active");
    w.begin_object();
    w.u64("film", d.active_film);
    w.u64("camera", d.active_camera);
    w.u64("render_options", d.active_options);
    w.end_object();
    static const char* const precision[] = {"float32", "float64"};
    static const char* const jitter[] = {"center", "uniform"};
    static const char* const mis[] = {"balance", "power"};
    static const char* const strategy[] = {"uniform", "power_weighted", "spatial_tree"};
    static const char* const depth[] = {"diffuse", "glossy", "specular", "transmission", "volume"};
    w.key("films");
    w.begin_array();
    for (const Film& f : d.films) {
        w.begin_object();
        w.u64("id", f.id);
        w.key("extent");
        w.begin_array();
        w.u64(f.width);
        w.u64(f.height);
        w.end_array();
        w.key("crop");
        w.begin_array();
        for (uint32_t v : f.crop) {
            w.u64(v);
        }
        w.end_array();
        w.string("accumulation", precision[f.precision]);
        w.end_object();
    }
    w.end_array();
    w.key("cameras");
    w.begin_array();
    for (const Camera& c : d.cameras) {
        w.begin_object();
        w.u64("id", c.id);
        w.u64("film", c.film);
        w.key("model");
        w.begin_object();
        w.string("type", "pinhole");
        w.reals("origin", c.origin, 3);
        w.reals("normal", c.normal, 3);
        w.reals("tangent", c.tangent, 3);
        w.reals("bitangent", c.bitangent, 3);
        w.real("vertical_fov_radians", c.vfov);
        w.real("t_min", c.t_min);
        w.real("t_max", c.t_max);
        w.u64("visibility_mask", c.mask);
        w.u64("current_medium", c.medium);
        w.end_object();
        w.end_object();
    }
    w.end_array();
    w.key("render_options");
    w.begin_array();
    for (const RenderOptions& o : d.options) {
        w.begin_object();
        w.u64("id", o.id);
        w.u64("film", o.film);
        w.u64("samples_per_pixel", o.spp);
        w.u64("maximum_path_depth", o.max_depth);
        w.u64("tile_edge_length", o.tile);
        w.u64("seed", o.seed);
        w.string("pixel_jitter", jitter[o.jitter]);
        w.string("mis_heuristic", mis[o.mis]);
        w.string("light_sampling_strategy", strategy[o.strategy]);
        w.key("depth_limits");
        w.begin_object();
        for (int i = 0; i < 5; ++i) {
            w.u64(depth[i], o.depth[i]);
        }
        w.end_object();
        w.key("russian_roulette");
        w.begin_object();
        if (!o.roulette) {
            w.string("mode", "disabled");
        } else {
            w.string("mode", "enabled");
            w.u64("first_eligible_depth", o.roulette_first);
            w.real("minimum_survival_probability", o.roulette_min);
            w.real("maximum_survival_probability", o.roulette_max);
        }
        w.end_object();
        w.end_object();
    }
    w.end_array();
    w.key("constant_textures");
    w.begin_array();
    for (const ConstantTexture& t : d.constant_textures) {
        w.begin_object();
        w.u64("id", t.id);
        if (t.kind == 0) {
            w.string("type", "float");
            w.real("value", t.value[0]);
        } else {
            w.string("type", t.kind == 1 ? "color" : "spectrum");
            w.reals("value", t.value, t.kind == 1 ? 3 : 4);
        }
        w.end_object();
    }
    w.end_array();
    w.key("host_image_textures");
    w.begin_array();
    w.end_array();
    w.key("objects");
    w.begin_array();
    for (uint32_t id : d.objects) {
        w.begin_object();
        w.u64("id", id);
        w.end_object();
    }
    w.end_array();
    w.key("geometries");
    w.begin_array();
    for (const Geometry& g : d.geometries) {
        w.begin_object();
        w.u64("id", g.id);
        w.key("mesh");
        w.begin_object();
        const size_t v = g.positions.size() / 3;
        w.key("positions");
        w.begin_array();
        for (size_t i = 0; i < v; ++i) {
            w.reals(&g.positions[3 * i], 3);
        }
        w.end_array();
        w.key("normals");
        w.begin_array();
        for (size_t i = 0; i < v; ++i) {
            w.reals(&g.normals[3 * i], 3);
        }
        w.end_array();
        w.key("texture_coordinates");
        w.begin_array();
        for (size_t i = 0; i < v; ++i) {
            w.reals(&g.uvs[2 * i], 2);
        }
        w.end_array();
        w.key("triangles");
        w.begin_array();
        for (size_t t = 0; t < g.triangles.size() / 3; ++t) {
            w.begin_array();
            for (int k = 0; k < 3; ++k) {
                w.u64(g.triangles[3 * t + k]);
            }
            w.end_array();
        }
        w.end_array();
        w.end_object();
        w.end_object();
    }
    w.end_array();
    w.key("materials");
    w.begin_array();
    for (const Material& m : d.materials) {
        w.begin_object();
        w.u64("id", m.id);
        w.key("spectral");
        if (!m.spectral) {
            w.null();
        } else {
            w.begin_object();
            w.key("wavelengths");
            write_packet(w, m.packet);
            w.key("closures");
            w.begin_object();
            static const char* const frame[] = {"shading_normal", "surface_tangent"};
            w.string("frame_mode", frame[m.frame_mode]);
            w.real("tangent_rotation_radians", m.rotation);
            w.key("components");
            w.begin_array();
            for (size_t i = 0; i < m.closures.size(); ++i) {
                const bf200_closure_v1& c = m.closures[i];
                const float* p = c.parameters;
                w.begin_object();
                w.real("probability", m.probabilities[i]);
                w.string("type", closure_type_name(c.kind));
                w.reals("weight", c.weight, 4);
                switch (c.kind) {
                case BF200_CLOSURE_ROUGH_DIFFUSE_REFLECTION:
                    w.real("roughness", p[0]);
                    break;
                case BF200_CLOSURE_ROUGH_CONDUCTOR_REFLECTION:
                    w.reals("eta", p, 4);
                    w.reals("k", p + 4, 4);
                    w.real("alpha_x", p[8]);
                    w.real("alpha_y", p[9]);
                    break;
                case BF200_CLOSURE_ROUGH_DIELECTRIC:
                    w.real("exterior_eta", p[0]);
                    w.real("interior_eta", p[1]);
                    w.real("alpha_x", p[2]);
                    w.real("alpha_y", p[3]);
                    break;
                case BF200_CLOSURE_SPECULAR_TRANSMISSION:
                    w.real("exterior_eta", p[0]);
                    w.real("interior_eta", p[1]);
                    break;
                default:
                    break;
                }
                w.end_object();
            }
            w.end_array();
            w.end_object();
            w.reals("emission", m.emission, 4);
            w.key("normal_map");
            w.null();
            w.key("bump_map");
            w.null();
            w.end_object();
        }
        w.end_object();
    }
    w.end_array();
    w.key("instances");
    w.begin_array();
    for (const Instance& in : d.instances) {
        w.begin_object();
        w.u64("id", in.id);
        w.key("parent");
        if (in.has_parent) {
            w.u64(in.parent);
        } else {
            w.null();
        }
        w.u64("object", in.object);
        w.u64("geometry", in.geometry);
        w.u64("material", in.material);
        w.reals("local_to_parent", in.local, 16);
        w.u64("visibility_mask", in.mask);
        w.end_object();
    }
    w.end_array();
    w.key("lights");
    w.begin_array();
    for (const Light& l : d.lights) {
        w.begin_object();
        w.u64("id", l.id);
        switch (l.kind) {
        case kPoint:
            w.string("type", "point");
            w.reals("position", l.position, 3);
            w.reals("absolute_position_error", l.error, 3);
            w.reals("spectral_radiant_intensity", l.spectrum, 4);
            break;
        case kDirectional:
            w.string("type", "directional");
            w.reals("propagation_direction", l.direction, 3);
            w.reals("spectral_irradiance", l.spectrum, 4);
            break;
        case kSpot:
            w.string("type", "spot");
            w.reals("position", l.position, 3);
            w.reals("absolute_position_error", l.error, 3);
            w.reals("emission_direction", l.direction, 3);
            w.real("inner_half_angle_radians", l.inner);
            w.real("outer_half_angle_radians", l.outer);
            w.reals("on_axis_spectral_radiant_intensity", l.spectrum, 4);
            break;
        default:
            w.string("type", "environment");
            w.key("wavelengths");
            write_packet(w, l.packet);
            w.reals("radiance", l.spectrum, 4);
            break;
        }
        w.end_object();
    }
    w.end_array();
    w.end_object();
    return w.take();
}

// ---------------------------------------------------------------------------------------------
// The committed frame (FrameScene::create over the description's registries).

void commit(bf200_scene_json& d) {
    if (d.committed) {
        return;
    }
    for (const Geometry& g : d.geometries) {
        bf200_geometry_v1 out{};
        out.geometry_id = g.id;
        out.vertex_offset = static_cast<uint32_t>(d.c_positions.size() / 3);
        out.vertex_count = static_cast<uint32_t>(g.positions.size() / 3);
        out.triangle_offset = static_cast<uint32_t>(d.c_triangles.size() / 3);
        out.triangle_count = static_cast<uint32_t>(g.triangles.size() / 3);
        out.kind = BF200_GEOMETRY_TRIANGLES;
        d.c_geometries.push_back(out);
        d.c_positions.insert(d.c_positions.end(), g.positions.begin(), g.positions.end());
        d.c_normals.insert(d.c_normals.end(), g.normals.begin(), g.normals.end());
        d.c_uvs.insert(d.c_uvs.end(), g.uvs.begin(), g.uvs.end());
        d.c_triangles.insert(d.c_triangles.end(), g.triangles.begin(), g.triangles.end());
    }
    for (const Material& m : d.materials) {
        bf200_material_v1 out{};
        out.material_id = m.id;
        out.closure_offset = static_cast<uint32_t>(d.c_closures.size());
        out.closure_count = static_cast<uint32_t>(m.closures.size());
        out.frame_mode = m.frame_mode;
        out.tangent_rotation_radians = m.rotation;
        std::copy(m.probabilities, m.probabilities + kClosureCapacity, out.component_probabilities);
        std::copy(m.emission, m.emission + 4, out.emitted_radiance);
        d.c_materials.push_back(out);
        d.c_closures.insert(d.c_closures.end(), m.closures.begin(), m.closures.end());
    }
    for (size_t i = 0; i < d.instances.size(); ++i) {
        const Instance& in = d.instances[i];
        bf200_instance_v1 out{};
        out.instance_id = in.id;
        out.object_id = in.object;
        out.geometry_index = static_cast<uint32_t>(find(d.geometries, in.geometry));
        out.material_index = static_cast<uint32_t>(find(d.materials, in.material));
        out.visibility_mask = in.mask;
        std::copy(&d.world[16 * i], &d.world[16 * i] + 16, out.object_to_world);
        std::copy(&d.world_inverse[16 * i], &d.world_inverse[16 * i] + 16, out.world_to_object);
        d.c_instances.push_back(out);
    }
    for (const Light& l : d.lights) {
        if (l.kind != kEnvironment) {
            d.c_punctual.push_back(punctual_record(l));
        }
    }
    d.committed = true;
}

void frame(bf200_scene_json& d, bf200_scene_json_frame_v1& out) {
    const Light* environment = nullptr;
    for (const Light& l : d.lights) {
        if (l.kind == kEnvironment) {
            environment = &l;
        }
    }
    if (environment == nullptr) {
        refuse(kUnavailable, "A render needs the scene's spectral environment light (its wavelength packet).");
    }
    if (d.instances.empty()) {
        refuse(kUnavailable, "A render needs at least one instance.");
    }
    commit(d);
    const Film& film = d.films[find(d.films, d.active_film)];
    const Camera& cam = d.cameras[find(d.cameras, d.active_camera)];
    const RenderOptions& o = d.options[find(d.options, d.active_options)];
    out = bf200_scene_json_frame_v1{};
    out.struct_size = sizeof(bf200_scene_json_frame_v1);
    out.film_id = film.id, out.camera_id = cam.id, out.render_options_id = o.id;
    out.width = film.width, out.height = film.height;
    std::copy(film.crop, film.crop + 4, out.crop);
    out.precision = film.precision;
    out.samples_per_pixel = o.spp, out.maximum_path_depth = o.max_depth, out.tile_edge_length = o.tile;
    out.light_sampling_strategy = o.strategy;
    out.seed = o.seed;
    bf200_camera_v1& c = out.camera;
    std::copy(cam.origin, cam.origin + 3, c.origin);
    std::copy(cam.tangent, cam.tangent + 3, c.tangent);
    std::copy(cam.bitangent, cam.bitangent + 3, c.bitangent);
    std::copy(cam.normal, cam.normal + 3, c.normal);
    validate_camera(cam, film, c.half_width, c.half_height);
    c.t_min = cam.t_min, c.t_max = cam.t_max, c.time = 0.0F, c.mask = cam.mask;
    c.width = film.width, c.height = film.height, c.jitter_mode = o.jitter;
    bf200_transport_options_v1& t = out.options;
    t.struct_size = sizeof(bf200_transport_options_v1);
    t.mis_heuristic = o.mis;
    std::copy(o.depth, o.depth + 5, t.depth_limits);
    t.roulette_enabled = o.roulette ? 1U : 0U;
    t.roulette_first_eligible_depth = o.roulette_first;
    t.roulette_minimum_survival = o.roulette_min;
    t.roulette_maximum_survival = o.roulette_max;
    t.sampler = BF200_SAMPLER_HASH;
    bf200_scene_desc_v1& s = out.scene;
    s.struct_size = sizeof(bf200_scene_desc_v1);
    s.geometry_count = static_cast<uint32_t>(d.c_geometries.size());
    s.vertex_count = static_cast<uint32_t>(d.c_positions.size() / 3);
    s.triangle_count = static_cast<uint32_t>(d.c_triangles.size() / 3);
    s.material_count = static_cast<uint32_t>(d.c_materials.size());
    s.closure_count = static_cast<uint32_t>(d.c_closures.size());
    s.instance_count = static_cast<uint32_t>(d.c_instances.size());
    s.punctual_light_count = static_cast<uint32_t>(d.c_punctual.size());
    s.geometries = d.c_geometries.data();
    s.positions = d.c_positions.data();
    s.normals = d.c_normals.data();
    s.texture_coordinates = d.c_uvs.data();
    s.triangles = d.c_triangles.data();
    s.materials = d.c_materials.data();
    s.closures = d.c_closures.data();
    s.instances = d.c_instances.data();
    s.punctual_lights = d.c_punctual.empty() ? nullptr : d.c_punctual.data();
    std::copy(environment->packet.nanometers, environment->packet.nanometers + 4, s.wavelength_nanometers);
    std::copy(environment->packet.pdf, environment->packet.pdf + 4, s.wavelength_pdf);
    std::copy(environment->spectrum, environment->spectrum + 4, s.environment_radiance);
}

void store(const std::string& text, char* message, uint64_t capacity) {
    if (message != nullptr && capacity != 0) {
        const size_t n = std::min<size_t>(text.size(), capacity - 1);
        std::memcpy(message, text.data(), n);
        message[n] = '\0';
    }
}

template <typename F> uint32_t guarded(char* message, uint64_t capacity, F&& body) noexcept {
    try {
        body();
        store("", message, capacity);
        return kOk;
    } catch (const Refusal& r) {
        store(r.message, message, capacity);
        return r.code;
    } catch (const std::bad_alloc&) {
        store("Scene JSON decoding exhausted memory.", message, capacity);
        return kExhausted;
    } catch (const std::length_error&) {
        store("A scene JSON decoded allocation size is not representable.", message, capacity);
        return kExhausted;
    } catch (...) {
        store("Scene JSON processing failed.", message, capacity);
        return kInternal;
    }
}

}  // namespace
}  // namespace scene_json
}  // namespace bf200

using namespace bf200::scene_json;

extern "C" {

BF200_EXPORT uint32_t bf200_scene_json_parse(const char* bytes, uint64_t size, const bf200_scene_json_limits_v1* limits,
                                             bf200_scene_json** out_document, char* message,
                                             uint64_t message_capacity) noexcept {
    if (out_document != nullptr) {
        *out_document = nullptr;
    }
    bf200_scene_json* created = nullptr;
    const uint32_t code = guarded(message, message_capacity, [&] {
        if (out_document == nullptr || (bytes == nullptr && size != 0)) {
            refuse(kInvalid, "bf200_scene_json_parse needs the bytes and an output pointer.");
        }
        const Limits l = limits_from(limits);
        validate_limits(l);
        if (size > l.encoded) {
            refuse(kExhausted, "Encoded scene JSON exceeds its byte budget.");
        }
        auto document = std::make_unique<bf200_scene_json>();
        Cursor cursor(std::string_view(bytes == nullptr ? "" : bytes, size), l);
        Budget budget(l);
        read_root(cursor, budget, *document);
        cursor.finish();
        create_description(*document);
        created = document.release();
    });
    if (code == kOk) {
        *out_document = created;
    }
    return code;
}

BF200_EXPORT void bf200_scene_json_destroy(bf200_scene_json* document) noexcept {
    delete document;
}

BF200_EXPORT uint32_t bf200_scene_json_write(const bf200_scene_json* document, const bf200_scene_json_limits_v1* limits,
                                             char* out, uint64_t capacity, uint64_t* out_size, char* message,
                                             uint64_t message_capacity) noexcept {
    return guarded(message, message_capacity, [&] {
        if (document == nullptr || out_size == nullptr) {
            refuse(kInvalid, "bf200_scene_json_write needs a document and an output size.");
        }
        const std::string text = write_document(*document, limits_from(limits));
        *out_size = text.size();
        if (out != nullptr) {
            if (capacity < text.size()) {
                refuse(kExhausted, "The output buffer cannot hold the canonical scene JSON.");
            }
            std::memcpy(out, text.data(), text.size());
        }
    });
}

BF200_EXPORT uint32_t bf200_scene_json_frame(const bf200_scene_json* document, bf200_scene_json_frame_v1* out,
                                             char* message, uint64_t message_capacity) noexcept {
    return guarded(message, message_capacity, [&] {
        if (document == nullptr || out == nullptr) {
            refuse(kInvalid, "bf200_scene_json_frame needs a document and an output record.");
        }
        // The committed arrays are built on first use and owned by the document.
        frame(*const_cast<bf200_scene_json*>(document), *out);
    });
}

}  // extern "C"
