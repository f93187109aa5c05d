// Triangle-mesh import for callers that hold meshes as files: OBJ and ASCII PLY, accepted and
// rejected as engine::load_obj_triangle_mesh / load_ply_triangle_mesh accept and reject them
// (Blackframe/Engine/Include/Blackframe/Engine/TriangleMeshImport.hpp:9-17,
// Blackframe/Engine/Source/TriangleMeshImport.cpp), into the aligned vertex arrays a
// bf200_scene_desc_v1 geometry takes.
//
// The rules kept alike, because a caller must get the same mesh or the same refusal:
// * paths are absolute with the lower-case extension; files are at most 256 MiB;
// * OBJ: v / vn / vt records with exactly 3 / 3 / 2 scalars (vn unit length within 256 epsilon),
//   f with exactly three complete v/vt/vn corners (1-based, or negative relative indices), g with at
//   most one name, o / s / usemtl / mtllib with exactly one value, '#' comments; every other record
//   is refused. A corner's (v, vt, vn) triple becomes one aligned vertex, numbered in order of
//   first use;
// * PLY: "ply", "format ascii 1.0", then element vertex (x/y/z, nx/ny/nz, u/v in any order, aliases
//   s/t and texture_u/texture_v, scalar types char..double) followed by element face with one
//   integer vertex_indices list of exactly 3; comment and obj_info lines; nothing after the data;
// * scalars: an optional leading '+', then a complete decimal or scientific number parsed to double
//   (correctly rounded) and rounded to float; non-finite values, values beyond the float range and
//   nonzero values that round to zero are refused;
// * the mesh: at least one vertex and triangle, finite positions and texture coordinates, unit
//   normals, indices in range, and no triangle whose vertices are exactly collinear.
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <string>
#include <string_view>
#include <sys/stat.h>
#include <vector>

#include "bf200.h"
#include "bf200_records.h"

struct bf200_mesh {
    std::vector<float> positions, normals, uvs;
    std::vector<uint32_t> triangles;
};

namespace {

constexpr uint64_t kMaximumFileBytes = 256ULL * 1024 * 1024;
constexpr uint64_t kMaximumStorageBytes = 256ULL * 1024 * 1024;
constexpr uint64_t kMaximumEntries = std::numeric_limits<uint32_t>::max();

struct ImportError {
    blackframe_status status = BLACKFRAME_STATUS_SUCCESS;
    std::string message;
};

bool failure(ImportError& e, blackframe_status status, std::string message) {
    e.status = status;
    e.message = std::move(message);
    return false;
}

bool line_failure(ImportError& e, const char* format, size_t line, const char* detail,
                  blackframe_status status = BLACKFRAME_STATUS_INVALID_ARGUMENT) {
    return failure(e, status, std::string(format) + " line " + std::to_string(line) + ": " + detail);
}

bool space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// Lines split at '\n' with one trailing '\r' removed, numbered from 1.
struct Lines {
    std::string_view text;
    size_t offset = 0, number = 0;
    bool next(std::string_view& line) {
        if (offset == text.size()) {
            return false;
        }
        const size_t end = text.find('\n', offset);
        const size_t stop = end == std::string_view::npos ? text.size() : end;
        line = text.substr(offset, stop - offset);
        if (!line.empty() && line.back() == '\r') {
            line.remove_suffix(1);
        }
        offset = end == std::string_view::npos ? text.size() : end + 1;
        ++number;
        return true;
    }
};

// Whitespace-separated fields, at most `limit` of them (so a longer line shows as `limit` fields).
size_t fields(std::string_view line, bool comments, size_t limit, std::string_view* out) {
    if (comments) {
        const size_t hash = line.find('#');
        if (hash != std::string_view::npos) {
            line = line.substr(0, hash);
        }
    }
    size_t n = 0, i = 0;
    while (i < line.size()) {
        while (i < line.size() && space(line[i])) {
            ++i;
        }
        if (i == line.size()) {
            break;
        }
        const size_t begin = i;
        while (i < line.size() && !space(line[i])) {
            ++i;
        }
        if (n == limit) {
            break;
        }
        out[n++] = line.substr(begin, i - begin);
    }
    return n;
}

std::string_view strip_plus(std::string_view t) {
    if (!t.empty() && t.front() == '+') {
        t.remove_prefix(1);
    }
    return t;
}

// Complete decimal integers (std::from_chars, base 10) after one optional leading '+'.
bool parse_int(std::string_view t, int64_t& out) {
    t = strip_plus(t);
    const auto parsed = std::from_chars(t.data(), t.data() + t.size(), out, 10);
    return !t.empty() && parsed.ec == std::errc{} && parsed.ptr == t.data() + t.size();
}

bool parse_uint(std::string_view t, uint64_t& out) {
    t = strip_plus(t);
    const auto parsed = std::from_chars(t.data(), t.data() + t.size(), out, 10);
    return !t.empty() && parsed.ec == std::errc{} && parsed.ptr == t.data() + t.size();
}

// A complete decimal or scientific scalar (std::from_chars, general format: correctly rounded to
// double, no leading whitespace, sign '-' only after the one optional '+' is removed), then to
// float (to_transport_scalar: finite, within the float range, nonzero values must stay nonzero).
bool parse_scalar(std::string_view t, float& out, const char*& problem) {
    t = strip_plus(t);
    problem = "expected a complete locale-independent scalar.";
    double value = 0.0;
    const auto parsed = std::from_chars(t.data(), t.data() + t.size(), value, std::chars_format::general);
    if (t.empty() || parsed.ec != std::errc{} || parsed.ptr != t.data() + t.size()) {
        return false;
    }
    if (!std::isfinite(value)) {
        problem = "A reference scalar must be finite before transport conversion.";
        return false;
    }
    if (value < -static_cast<double>(std::numeric_limits<float>::max()) ||
        value > static_cast<double>(std::numeric_limits<float>::max())) {
        problem = "A reference scalar exceeds the finite transport range.";
        return false;
    }
    const float f = static_cast<float>(value);
    if (value != 0.0 && f == 0.0F) {
        problem = "A reference scalar underflows to zero in transport precision.";
        return false;
    }
    out = f;
    return true;
}

// TriangleMesh::create (Blackframe/Engine/Source/TriangleMesh.cpp:60-130)
bool validate_mesh(const bf200_mesh& m, ImportError& e) {
    const char* problem = bf200::triangle_mesh_problem(m.positions.data(), m.normals.data(), m.uvs.data(),
                                                       m.positions.size() / 3, m.triangles.data(),
                                                       m.triangles.size() / 3);
    return problem == nullptr || failure(e, BLACKFRAME_STATUS_INVALID_ARGUMENT, problem);
}

// Aligned OBJ vertices by their (v, vt, vn) corner: an open-addressing table sized for every
// corner of the file, so each lookup is one probe sequence over flat arrays.
struct CornerTable {
    std::vector<uint32_t> v, t, n, index;  // index UINT32_MAX: empty
    uint64_t mask = 0;
    explicit CornerTable(uint64_t corners) {
        uint64_t size = 16;
        while (size < 2 * corners) {
            size <<= 1;
        }
        v.resize(size);
        t.resize(size);
        n.resize(size);
        index.assign(size, 0xFFFFFFFFU);
        mask = size - 1;
    }
    // The slot of the corner: holding it, or empty where it belongs.
    uint64_t slot(uint32_t vi, uint32_t ti, uint32_t ni) const {
        uint64_t h = (static_cast<uint64_t>(vi) * 0x9E3779B97F4A7C15ULL) ^ (static_cast<uint64_t>(ti) * 0xC2B2AE3D27D4EB4FULL) ^
                     (static_cast<uint64_t>(ni) * 0x165667B19E3779F9ULL);
        h ^= h >> 29;
        for (uint64_t s = h & mask;; s = (s + 1) & mask) {
            if (index[s] == 0xFFFFFFFFU || (v[s] == vi && t[s] == ti && n[s] == ni)) {
                return s;
            }
        }
    }
};

bool take_storage(uint64_t& remaining, uint64_t count, uint64_t bytes) {
    if (bytes != 0 && count > remaining / bytes) {
        return false;
    }
    remaining -= count * bytes;
    return true;
}

// An OBJ index: 1-based, or negative relative to the records seen so far.
bool obj_index(std::string_view t, size_t count, size_t line, uint32_t& out, ImportError& e) {
    int64_t v = 0;
    if (!parse_int(t, v)) {
        return line_failure(e, "OBJ", line, "expected a complete signed decimal integer.");
    }
    if (v == 0) {
        return line_failure(e, "OBJ", line, "index zero is not valid.");
    }
    const int64_t n = static_cast<int64_t>(count);
    const int64_t resolved = v > 0 ? v - 1 : n + v;
    if (resolved < 0 || resolved >= n) {
        return line_failure(e, "OBJ", line, "index references an attribute outside its current domain.");
    }
    out = static_cast<uint32_t>(resolved);
    return true;
}

bool parse_obj(std::string_view text, bf200_mesh& m, ImportError& e) {
    if (text.find('\0') != std::string_view::npos) {
        return failure(e, BLACKFRAME_STATUS_INVALID_ARGUMENT, "OBJ text contains an embedded null byte.");
    }
    // record counts bound the decoded storage before anything is stored
    uint64_t counts[4] = {0, 0, 0, 0};  // v, vn, vt, f
    {
        Lines lines{text};
        std::string_view line, first[1];
        while (lines.next(line)) {
            if (fields(line, true, 1, first) == 0) {
                continue;
            }
            const int k = first[0] == "v" ? 0 : first[0] == "vn" ? 1 : first[0] == "vt" ? 2 : first[0] == "f" ? 3 : -1;
            if (k < 0) {
                continue;
            }
            if (counts[k] == kMaximumEntries) {
                return failure(e, BLACKFRAME_STATUS_OUT_OF_RANGE,
                               "OBJ record count exceeds the supported 32-bit index domain.");
            }
            ++counts[k];
        }
        if (counts[3] > kMaximumEntries / 3) {
            return failure(e, BLACKFRAME_STATUS_OUT_OF_RANGE,
                           "OBJ faces can exceed the supported 32-bit aligned-vertex domain.");
        }
        const uint64_t aligned = counts[3] * 3;
        uint64_t remaining = kMaximumStorageBytes;
        if (!take_storage(remaining, counts[0], 12) || !take_storage(remaining, counts[1], 12) ||
            !take_storage(remaining, counts[2], 8) || !take_storage(remaining, aligned, 12) ||
            !take_storage(remaining, aligned, 12) || !take_storage(remaining, aligned, 8) ||
            !take_storage(remaining, counts[3], 12) || !take_storage(remaining, aligned, 128)) {
            return failure(e, BLACKFRAME_STATUS_OUT_OF_RANGE,
                           "OBJ records exceed the conservative 256 MiB decoded mesh-storage limit.");
        }
    }
    std::vector<float> src_p, src_n, src_t;
    src_p.reserve(3 * counts[0]);
    src_n.reserve(3 * counts[1]);
    src_t.reserve(2 * counts[2]);
    m.triangles.reserve(3 * counts[3]);
    CornerTable aligned(3 * counts[3]);
    Lines lines{text};
    std::string_view line, f[5];
    const char* problem = nullptr;
    while (lines.next(line)) {
        const size_t n = fields(line, true, 5, f);
        if (n == 0) {
            continue;
        }
        const size_t number = lines.number;
        if (f[0] == "v" || f[0] == "vn") {
            const bool normal = f[0] == "vn";
            if (n != 4) {
                return line_failure(e, "OBJ", number,
                                    normal ? "normals require exactly x, y, and z." : "positions require exactly x, y, and z.");
            }
            float xyz[3];
            for (int k = 0; k < 3; ++k) {
                if (!parse_scalar(f[1 + k], xyz[k], problem)) {
                    return line_failure(e, "OBJ", number, problem);
                }
            }
            if (normal && !bf200::unit_normal(xyz[0], xyz[1], xyz[2])) {
                return line_failure(e, "OBJ", number, "normals must be finite unit-length values.");
            }
            (normal ? src_n : src_p).insert((normal ? src_n : src_p).end(), xyz, xyz + 3);
            continue;
        }
        if (f[0] == "vt") {
            if (n != 3) {
                return line_failure(e, "OBJ", number, "texture coordinates require exactly u and v.");
            }
            float uv[2];
            for (int k = 0; k < 2; ++k) {
                if (!parse_scalar(f[1 + k], uv[k], problem)) {
                    return line_failure(e, "OBJ", number, problem);
                }
            }
            src_t.insert(src_t.end(), uv, uv + 2);
            continue;
        }
        if (f[0] == "f") {
            if (n != 4) {
                return line_failure(e, "OBJ", number,
                                    "only explicitly triangulated faces with three corners are supported.");
            }
            for (int corner = 0; corner < 3; ++corner) {
                const std::string_view t = f[1 + corner];
                const size_t s1 = t.find('/');
                const size_t s2 = s1 == std::string_view::npos ? std::string_view::npos : t.find('/', s1 + 1);
                if (s1 == std::string_view::npos || s2 == std::string_view::npos ||
                    t.find('/', s2 + 1) != std::string_view::npos || s1 == 0 || s2 == s1 + 1 || s2 + 1 == t.size()) {
                    return line_failure(e, "OBJ", number, "triangle corners must use complete v/vt/vn indices.");
                }
                uint32_t vi = 0, ti = 0, ni = 0;
                if (!obj_index(t.substr(0, s1), src_p.size() / 3, number, vi, e) ||
                    !obj_index(t.substr(s1 + 1, s2 - s1 - 1), src_t.size() / 2, number, ti, e) ||
                    !obj_index(t.substr(s2 + 1), src_n.size() / 3, number, ni, e)) {
                    return false;
                }
                const uint64_t slot = aligned.slot(vi, ti, ni);
                if (aligned.index[slot] != 0xFFFFFFFFU) {
                    m.triangles.push_back(aligned.index[slot]);
                    continue;
                }
                const uint32_t index = static_cast<uint32_t>(m.positions.size() / 3);
                aligned.v[slot] = vi;
                aligned.t[slot] = ti;
                aligned.n[slot] = ni;
                aligned.index[slot] = index;
                m.positions.insert(m.positions.end(), &src_p[3ULL * vi], &src_p[3ULL * vi] + 3);
                m.normals.insert(m.normals.end(), &src_n[3ULL * ni], &src_n[3ULL * ni] + 3);
                m.uvs.insert(m.uvs.end(), &src_t[2ULL * ti], &src_t[2ULL * ti] + 2);
                m.triangles.push_back(index);
            }
            continue;
        }
        if (f[0] == "g") {
            if (n > 2) {
                return line_failure(e, "OBJ", number, "at most one opaque group name is supported by this importer.");
            }
            continue;
        }
        if (f[0] == "o" || f[0] == "s" || f[0] == "usemtl" || f[0] == "mtllib") {
            if (n != 2) {
                return line_failure(e, "OBJ", number,
                                    "opaque object, smoothing, and material metadata requires one value.");
            }
            continue;
        }
        return line_failure(e, "OBJ", number, "record is not supported by the triangle importer.");
    }
    return validate_mesh(m, e);
}

enum class PlyType { int8, uint8, int16, uint16, int32, uint32, float32, float64, none };

PlyType ply_type(std::string_view n) {
    if (n == "char" || n == "int8") return PlyType::int8;
    if (n == "uchar" || n == "uint8") return PlyType::uint8;
    if (n == "short" || n == "int16") return PlyType::int16;
    if (n == "ushort" || n == "uint16") return PlyType::uint16;
    if (n == "int" || n == "int32") return PlyType::int32;
    if (n == "uint" || n == "uint32") return PlyType::uint32;
    if (n == "float" || n == "float32") return PlyType::float32;
    if (n == "double" || n == "float64") return PlyType::float64;
    return PlyType::none;
}

bool ply_integer(PlyType t) { return t != PlyType::float32 && t != PlyType::float64 && t != PlyType::none; }
bool ply_signed(PlyType t) { return t == PlyType::int8 || t == PlyType::int16 || t == PlyType::int32; }

// A PLY integer within its declared type; `negative_ok` false for list counts and indices.
bool ply_int_value(std::string_view tok, PlyType t, size_t line, bool negative_ok, int64_t& out, ImportError& e) {
    if (ply_signed(t)) {
        int64_t v = 0;
        if (!parse_int(tok, v)) {
            return line_failure(e, "PLY", line, "expected a complete signed decimal integer.");
        }
        const int64_t lo = t == PlyType::int8 ? -128 : t == PlyType::int16 ? -32768 : INT32_MIN;
        const int64_t hi = t == PlyType::int8 ? 127 : t == PlyType::int16 ? 32767 : INT32_MAX;
        if (v < lo || v > hi) {
            return line_failure(e, "PLY", line, "integer value exceeds its declared scalar type.");
        }
        if (!negative_ok && v < 0) {
            return line_failure(e, "PLY", line, "list counts and indices cannot be negative.");
        }
        out = v;
        return true;
    }
    uint64_t v = 0;
    if (!parse_uint(tok, v)) {
        return line_failure(e, "PLY", line, "expected a complete unsigned decimal integer.");
    }
    const uint64_t hi = t == PlyType::uint8 ? 255U : t == PlyType::uint16 ? 65535U : 4294967295ULL;
    if (v > hi) {
        return line_failure(e, "PLY", line, "integer value exceeds its declared scalar type.");
    }
    out = static_cast<int64_t>(v);
    return true;
}

int ply_semantic(std::string_view n) {  // x y z nx ny nz u v
    if (n == "x") return 0;
    if (n == "y") return 1;
    if (n == "z") return 2;
    if (n == "nx") return 3;
    if (n == "ny") return 4;
    if (n == "nz") return 5;
    if (n == "u" || n == "s" || n == "texture_u") return 6;
    if (n == "v" || n == "t" || n == "texture_v") return 7;
    return -1;
}

bool parse_ply(std::string_view text, bf200_mesh& m, ImportError& e) {
    Lines lines{text};
    std::string_view line, f[6];
    if (!lines.next(line)) {
        return line_failure(e, "PLY", 1, "file is empty.");
    }
    if (fields(line, false, 2, f) != 1 || f[0] != "ply") {
        return line_failure(e, "PLY", lines.number, "missing ply magic.");
    }
    bool format_seen = false, vertex_seen = false, face_seen = false, end_seen = false;
    int element = 0;  // 0 none, 1 vertex, 2 face
    uint64_t vertex_count = 0, face_count = 0;
    std::vector<std::pair<int, PlyType>> properties;
    bool seen[8] = {};
    PlyType count_type = PlyType::none, index_type = PlyType::none;
    while (lines.next(line)) {
        const size_t n = fields(line, false, 6, f);
        const size_t number = lines.number;
        if (n == 0 || f[0] == "comment" || f[0] == "obj_info") {
            continue;
        }
        if (f[0] == "format") {
            if (format_seen || n != 3) {
                return line_failure(e, "PLY", number, "format declaration is malformed or repeated.");
            }
            format_seen = true;
            if (f[1] != "ascii" || f[2] != "1.0") {
                return line_failure(e, "PLY", number,
                                    "only the ASCII 1.0 encoding is supported; no encoding fallback is available.",
                                    BLACKFRAME_STATUS_INVALID_STATE);
            }
            continue;
        }
        if (f[0] == "element") {
            if (!format_seen || n != 3) {
                return line_failure(e, "PLY", number, "element declaration is malformed.");
            }
            uint64_t count = 0;
            if (!parse_uint(f[2], count)) {
                return line_failure(e, "PLY", number, "expected a complete unsigned decimal integer.");
            }
            if (count > kMaximumEntries) {
                return line_failure(e, "PLY", number, "element count exceeds the 32-bit mesh domain.",
                                    BLACKFRAME_STATUS_OUT_OF_RANGE);
            }
            if (f[1] == "vertex") {
                if (vertex_seen || face_seen) {
                    return line_failure(e, "PLY", number, "vertex must be the first and only vertex element.");
                }
                vertex_seen = true;
                element = 1;
                vertex_count = count;
                continue;
            }
            if (f[1] == "face") {
                if (!vertex_seen || face_seen) {
                    return line_failure(e, "PLY", number, "face must follow exactly one vertex element.");
                }
                face_seen = true;
                element = 2;
                face_count = count;
                continue;
            }
            return line_failure(e, "PLY", number, "element is not supported by the triangle importer.",
                                BLACKFRAME_STATUS_INVALID_STATE);
        }
        if (f[0] == "property") {
            if (element == 1) {
                if (n != 3 || f[1] == "list") {
                    return line_failure(e, "PLY", number, "vertex properties must be supported scalar values.");
                }
                const PlyType t = ply_type(f[1]);
                const int sem = ply_semantic(f[2]);
                if (t == PlyType::none || sem < 0) {
                    return line_failure(e, "PLY", number, "vertex property type or semantic is not supported.",
                                        BLACKFRAME_STATUS_INVALID_STATE);
                }
                if (seen[sem]) {
                    return line_failure(e, "PLY", number, "vertex property semantic is duplicated or aliased twice.");
                }
                seen[sem] = true;
                properties.emplace_back(sem, t);
                continue;
            }
            if (element == 2) {
                if (n != 5 || f[1] != "list" || (f[4] != "vertex_indices" && f[4] != "vertex_index")) {
                    return line_failure(e, "PLY", number, "faces require exactly one vertex_indices list property.",
                                        BLACKFRAME_STATUS_INVALID_STATE);
                }
                if (count_type != PlyType::none || index_type != PlyType::none) {
                    return line_failure(e, "PLY", number, "face index property is duplicated.");
                }
                const PlyType ct = ply_type(f[2]), it = ply_type(f[3]);
                if (!ply_integer(ct) || !ply_integer(it)) {
                    return line_failure(e, "PLY", number, "face list counts and indices require supported integer types.",
                                        BLACKFRAME_STATUS_INVALID_STATE);
                }
                count_type = ct;
                index_type = it;
                continue;
            }
            return line_failure(e, "PLY", number, "property appears before an element.");
        }
        if (f[0] == "end_header") {
            if (n != 1) {
                return line_failure(e, "PLY", number, "end_header cannot carry extra fields.");
            }
            end_seen = true;
            break;
        }
        return line_failure(e, "PLY", number, "header directive is not supported.", BLACKFRAME_STATUS_INVALID_STATE);
    }
    bool every = true;
    for (bool s : seen) {
        every = every && s;
    }
    if (!end_seen) {
        return line_failure(e, "PLY", lines.number + 1, "header is truncated.");
    }
    if (!format_seen || !vertex_seen || !face_seen || !every || count_type == PlyType::none) {
        return line_failure(e, "PLY", lines.number + 1,
                            "header must define vertices with x/y/z, nx/ny/nz, u/v and triangular faces.");
    }
    if (vertex_count == 0 || face_count == 0) {
        return line_failure(e, "PLY", lines.number + 1, "vertex and face elements must be non-empty.");
    }
    if (text.find('\0') != std::string_view::npos) {
        return failure(e, BLACKFRAME_STATUS_INVALID_ARGUMENT, "PLY ASCII data contains an embedded null byte.");
    }
    const uint64_t vertex_bytes = vertex_count * 32, triangle_bytes = face_count * 12;
    if (vertex_bytes > kMaximumStorageBytes || triangle_bytes > kMaximumStorageBytes - vertex_bytes) {
        return failure(e, BLACKFRAME_STATUS_OUT_OF_RANGE, "PLY declarations exceed the 256 MiB decoded mesh-storage limit.");
    }
    if (vertex_count * 15 > text.size() || face_count * 7 > text.size() - vertex_count * 15) {
        return failure(e, BLACKFRAME_STATUS_INVALID_ARGUMENT,
                       "PLY declared element counts cannot fit in the available source data.");
    }
    m.positions.resize(3 * vertex_count);
    m.normals.resize(3 * vertex_count);
    m.uvs.resize(2 * vertex_count);
    m.triangles.reserve(3 * face_count);
    std::vector<std::string_view> vf(properties.size() + 1);
    const char* problem = nullptr;
    for (uint64_t v = 0; v < vertex_count; ++v) {
        if (!lines.next(line)) {
            return line_failure(e, "PLY", lines.number + 1, "vertex records are truncated.");
        }
        if (fields(line, false, properties.size() + 1, vf.data()) != properties.size()) {
            return line_failure(e, "PLY", lines.number, "vertex record does not match the declared property count and order.");
        }
        float value[8] = {};
        for (size_t k = 0; k < properties.size(); ++k) {
            const PlyType t = properties[k].second;
            float x = 0.0F;
            if (t == PlyType::float32 || t == PlyType::float64) {
                if (!parse_scalar(vf[k], x, problem)) {
                    return line_failure(e, "PLY", lines.number, problem);
                }
            } else {
                int64_t iv = 0;
                if (!ply_int_value(vf[k], t, lines.number, true, iv, e)) {
                    return false;
                }
                x = static_cast<float>(static_cast<double>(iv));  // to_transport_scalar of an integer
            }
            value[properties[k].first] = x;
        }
        float* p = &m.positions[3 * v];
        float* nrm = &m.normals[3 * v];
        float* uv = &m.uvs[2 * v];
        p[0] = value[0], p[1] = value[1], p[2] = value[2];
        nrm[0] = value[3], nrm[1] = value[4], nrm[2] = value[5];
        uv[0] = value[6], uv[1] = value[7];
    }
    for (uint64_t t = 0; t < face_count; ++t) {
        if (!lines.next(line)) {
            return line_failure(e, "PLY", lines.number + 1, "face records are truncated.");
        }
        std::string_view ff[5];
        const size_t n = fields(line, false, 5, ff);
        if (n == 0) {
            return line_failure(e, "PLY", lines.number, "face record cannot be empty.");
        }
        int64_t list = 0;
        if (!ply_int_value(ff[0], count_type, lines.number, false, list, e)) {
            return false;
        }
        if (n != static_cast<size_t>(list) + 1) {
            return line_failure(e, "PLY", lines.number, "face record does not match its declared list count.");
        }
        if (list != 3) {
            return line_failure(e, "PLY", lines.number, "only explicitly triangulated faces with three indices are supported.");
        }
        for (int corner = 0; corner < 3; ++corner) {
            int64_t index = 0;
            if (!ply_int_value(ff[1 + corner], index_type, lines.number, false, index, e)) {
                return false;
            }
            if (static_cast<uint64_t>(index) >= vertex_count) {
                return line_failure(e, "PLY", lines.number, "face index references an unknown vertex.");
            }
            m.triangles.push_back(static_cast<uint32_t>(index));
        }
    }
    std::string_view rest[1];
    while (lines.next(line)) {
        if (fields(line, false, 1, rest) != 0) {
            return line_failure(e, "PLY", lines.number, "unexpected data follows the declared elements.");
        }
    }
    return validate_mesh(m, e);
}

// read_mesh_text_file (TriangleMeshImport.cpp:1105-1180)
bool read_file(const char* path, const char* extension, const char* format, std::string& out, ImportError& e) {
    const std::string p = path == nullptr ? std::string() : std::string(path);
    if (p.empty() || p[0] != '/') {
        return failure(e, BLACKFRAME_STATUS_INVALID_ARGUMENT, std::string(format) + " mesh paths must be explicit absolute paths.");
    }
    struct stat st {};
    if (stat(p.c_str(), &st) != 0) {
        return failure(e, BLACKFRAME_STATUS_INVALID_ARGUMENT, std::string(format) + " mesh file was not found.");
    }
    if (!S_ISREG(st.st_mode)) {
        return failure(e, BLACKFRAME_STATUS_INVALID_ARGUMENT, std::string(format) + " mesh path must identify a regular file.");
    }
    if (static_cast<uint64_t>(st.st_size) > kMaximumFileBytes) {
        return failure(e, BLACKFRAME_STATUS_OUT_OF_RANGE, std::string(format) + " mesh file exceeds the 256 MiB import limit.");
    }
    std::ifstream in(p, std::ios::binary);
    if (!in.is_open()) {
        return failure(e, BLACKFRAME_STATUS_EXTENSION_FAILURE, std::string(format) + " mesh file could not be opened for reading.");
    }
    out.resize(static_cast<size_t>(st.st_size));
    if (!out.empty()) {
        in.read(&out[0], static_cast<std::streamsize>(out.size()));
        if (in.gcount() != static_cast<std::streamsize>(out.size())) {
            return failure(e, BLACKFRAME_STATUS_EXTENSION_FAILURE, std::string(format) + " mesh file could not be read completely.");
        }
    }
    (void)extension;
    return true;
}

bool ends_with(const std::string& s, const char* suffix) {
    const size_t n = std::strlen(suffix);
    return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

void store_message(const std::string& message, char* out, uint64_t capacity) {
    if (out == nullptr || capacity == 0) {
        return;
    }
    const size_t n = std::min<uint64_t>(message.size(), capacity - 1);
    std::memcpy(out, message.data(), n);
    out[n] = '\0';
}

}  // namespace

extern "C" {

BF200_EXPORT blackframe_status bf200_mesh_load(const char* absolute_path, bf200_mesh** out, char* message,
                                               uint64_t message_capacity) noexcept {
    ImportError e;
    if (out == nullptr) {
        store_message("null argument", message, message_capacity);
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    *out = nullptr;
    try {
        const std::string path = absolute_path == nullptr ? std::string() : std::string(absolute_path);
        const bool obj = ends_with(path, ".obj"), ply = ends_with(path, ".ply");
        const char* format = ply ? "PLY" : "OBJ";
        if (path.empty() || path[0] != '/') {
            failure(e, BLACKFRAME_STATUS_INVALID_ARGUMENT, std::string(format) + " mesh paths must be explicit absolute paths.");
        } else if (!obj && !ply) {
            failure(e, BLACKFRAME_STATUS_INVALID_ARGUMENT, "mesh path has no lower-case .obj or .ply extension.");
        } else {
            std::string text;
            auto mesh = new bf200_mesh();
            const bool ok = read_file(absolute_path, obj ? ".obj" : ".ply", format, text, e) &&
                            (obj ? parse_obj(text, *mesh, e) : parse_ply(text, *mesh, e));
            if (ok) {
                *out = mesh;
                store_message("", message, message_capacity);
                return BLACKFRAME_STATUS_SUCCESS;
            }
            delete mesh;
        }
    } catch (const std::bad_alloc&) {
        failure(e, BLACKFRAME_STATUS_OUT_OF_RANGE, "mesh import exhausted host memory.");
    } catch (const std::length_error&) {
        failure(e, BLACKFRAME_STATUS_OUT_OF_RANGE, "mesh import exceeded host container limits.");
    }
    store_message(e.message, message, message_capacity);
    return e.status;
}

BF200_EXPORT blackframe_status bf200_mesh_view(const bf200_mesh* mesh, bf200_mesh_view_v1* out) noexcept {
    if (mesh == nullptr || out == nullptr || out->struct_size < sizeof(bf200_mesh_view_v1)) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    out->vertex_count = static_cast<uint32_t>(mesh->positions.size() / 3);
    out->triangle_count = static_cast<uint32_t>(mesh->triangles.size() / 3);
    out->reserved = 0;
    out->positions = mesh->positions.data();
    out->normals = mesh->normals.data();
    out->texture_coordinates = mesh->uvs.data();
    out->triangles = mesh->triangles.data();
    return BLACKFRAME_STATUS_SUCCESS;
}

BF200_EXPORT void bf200_mesh_destroy(bf200_mesh* mesh) noexcept { delete mesh; }

}  // extern "C"
