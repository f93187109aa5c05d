// Oracle (test infrastructure only): a CPU restatement of the reference's scalar path tracer.
//
// This file is never linked into, loaded by, or called from the product. Tests, the golden
// fixture generator and bench.py's CPU arm load oracle/liboracle.so as the checker. It restates,
// function by function, the reference's one-sample NEE + MIS scalar loop
//   trace_scene_mis -> trace_lambertian_mis_with_query
//   (Blackframe/Engine/Source/SceneMisPathLoop.cpp:632-1016)
// for the scene contract of include/bf200.h (triangle meshes, root instances, one closure per
// material: Lambertian, GGX rough conductor, GGX rough dielectric; mesh area lights with a
// uniform light sampler; constant environment). Every helper cites the reference lines it
// follows. Arithmetic is float in the reference's operation order (compiled without FMA
// contraction); std::fma appears exactly where the reference calls it.
//
// Parity of this restatement is pinned against the reference itself (oracle/_ref, built from the
// reference sources by oracle/Makefile) by tests/test_oracle_vs_reference.py and by the committed
// fixtures in tests/golden/.
#include "bfo_exact.h"

#include "../include/bf200.h"
#include "bf200_light_tree.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace bfo {
namespace {

constexpr float kInfinity = std::numeric_limits<float>::infinity();
constexpr float kEpsilon = std::numeric_limits<float>::epsilon();
constexpr float kDenormMin = std::numeric_limits<float>::denorm_min();
constexpr float kInvPi = 0.318309886183790671538F;  // std::numbers::inv_pi_v<float>
constexpr float kPi = 3.14159265358979323846F;      // std::numbers::pi_v<float>

using Spectrum = std::array<float, 4>;

// Rounding of the sine and cosine of sampled angles. 0: the C library's float functions, which the
// reference calls (std::sin / std::cos of a float); 1: the float nearest to the double-precision
// value, which is how the device computes them. The two differ by an ulp on a small share of
// angles, which can send a path in a direction one ulp apart. Set before a call, never during one.
std::atomic<int> g_device_trig{0};

float sin_f(float a) {
    return g_device_trig.load(std::memory_order_relaxed) != 0 ? static_cast<float>(std::sin(static_cast<double>(a)))
                                                              : std::sin(a);
}
float cos_f(float a) {
    return g_device_trig.load(std::memory_order_relaxed) != 0 ? static_cast<float>(std::cos(static_cast<double>(a)))
                                                              : std::cos(a);
}
float atan2_f(float y, float x) {
    return g_device_trig.load(std::memory_order_relaxed) != 0
               ? static_cast<float>(std::atan2(static_cast<double>(y), static_cast<double>(x)))
               : std::atan2(y, x);
}

// Failure of one path: the reference returns std::unexpected for the whole path.
struct Failure {
    const char* message;
};

[[noreturn]] void fail(const char* message) { throw Failure{message}; }

// ---------------------------------------------------------------------------------------------
// Sample stream (SampleStream.hpp:23-67) and dimension map (SampleDimensionMap.cpp:47-68)
// ---------------------------------------------------------------------------------------------

uint64_t mix_bits(uint64_t v) {
    v ^= v >> 30U;
    v *= 0xBF58476D1CE4E5B9ULL;
    v ^= v >> 27U;
    v *= 0x94D049BB133111EBULL;
    return v ^ (v >> 31U);
}

// Sobol coordinates (SobolSampling.cpp:51-117) over the Joe-Kuo D6 parameters, and the nested
// binary Owen scramble (OwenScrambling.cpp:8-44).
const uint64_t kJoeKuoRows[21200][3] = {
#include "bf200_sobol_table.inc"
};

uint64_t sobol_coordinate(uint64_t sample_index, uint64_t dimension) {
    uint64_t v[64];
    if (dimension == 0) {
        for (uint32_t j = 0; j < 64; ++j) {
            v[j] = 1ULL << (63U - j);
        }
    } else {
        static const uint32_t row_end[18] = {1,   2,   4,   6,    12,   18,   36,   52,    100,
                                             160, 336, 480, 1110, 1866, 3666, 5714, 13424, 21200};
        const uint64_t row = dimension - 1;
        uint32_t degree = 1;
        while (row >= row_end[degree - 1]) {
            ++degree;
        }
        // the row's three words as one 192-bit little-endian integer
        auto bits = [&](uint32_t offset, uint32_t width) -> uint64_t {
            uint64_t value = 0;
            for (uint32_t k = 0; k < width; ++k) {
                const uint32_t pos = offset + k;
                value |= ((kJoeKuoRows[row][pos / 64U] >> (pos % 64U)) & 1ULL) << k;
            }
            return value;
        };
        const uint64_t a = bits(0, degree - 1);
        uint32_t offset = degree - 1;
        for (uint32_t j = 0; j < degree; ++j) {
            v[j] = bits(offset, j + 1) << (63U - j);
            offset += j + 1;
        }
        for (uint32_t j = degree; j < 64; ++j) {
            uint64_t d = v[j - degree] ^ (v[j - degree] >> degree);
            for (uint32_t k = 1; k < degree; ++k) {
                if ((a >> (degree - 1U - k)) & 1U) {
                    d ^= v[j - k];
                }
            }
            v[j] = d;
        }
    }
    uint64_t gray = sample_index ^ (sample_index >> 1U);
    uint64_t point = 0;
    for (uint32_t j = 0; gray != 0; ++j, gray >>= 1U) {
        if (gray & 1U) {
            point ^= v[j];
        }
    }
    return point;
}

uint64_t owen_coordinate(uint32_t px, uint32_t py, uint64_t sample_index, uint64_t seed, uint64_t dimension) {
    const uint64_t packed = (uint64_t(px) << 32U) | uint64_t(py);
    const uint64_t key = mix_bits(seed ^ mix_bits(dimension + 1U)) ^ mix_bits(packed);
    const uint64_t input = sobol_coordinate(sample_index, dimension);
    uint64_t prefix = 0, output = 0;
    for (uint32_t depth = 0; depth < 64; ++depth) {
        const uint64_t bit = (input >> (63U - depth)) & 1U;
        const uint64_t flip = mix_bits(key ^ ((1ULL << depth) | prefix)) >> 63U;
        output |= (bit ^ flip) << (63U - depth);
        prefix = (prefix << 1U) | bit;
    }
    return output;
}

// The transport's Sobol dimension of a sample dimension (the mapping of BF200_SAMPLER_OWEN_SOBOL):
// camera raster x, y -> 0, 1; every other dimension d -> d + 2.
uint64_t transport_sobol_dimension(uint64_t d) {
    return d == 0xA24BAED4963EE407ULL ? 0U : (d == 0x9FB21C651E98DF25ULL ? 1U : d + 2U);
}

struct Stream {
    uint32_t px, py;
    uint64_t sample, seed;
    bool owen = false;  // Owen-scrambled Sobol instead of the hash stream
    float sample_1d(uint64_t dimension) const {
        if (owen) {
            const uint64_t bits = owen_coordinate(px, py, sample, seed, transport_sobol_dimension(dimension));
            return static_cast<float>(bits >> 40U) * 0x1p-24F;
        }
        const uint64_t packed = (uint64_t(px) << 32U) | uint64_t(py);
        uint64_t state = mix_bits(seed ^ 0x9E3779B97F4A7C15ULL);
        state = mix_bits(state ^ packed ^ 0xD1B54A32D192ED03ULL);
        state = mix_bits(state ^ sample ^ 0x8CB92BA72F3D8DD7ULL);
        const uint64_t bits = mix_bits(state ^ dimension);
        return static_cast<float>(bits >> 40U) * 0x1p-24F;
    }
};

struct Dims {
    uint64_t light_selection, light_u, light_v, bsdf_component, bsdf_u, bsdf_v, russian_roulette;
};

Dims dims_for_bounce(uint64_t bounce) {
    const uint64_t first = 4 + bounce * 10;
    return Dims{first + 0, first + 1, first + 2, first + 3, first + 4, first + 5, first + 9};
}

// ---------------------------------------------------------------------------------------------
// Scene records
// ---------------------------------------------------------------------------------------------

struct Mat4 {
    float m[16];
    float operator()(int r, int c) const { return m[r * 4 + c]; }
};

// Transforms.hpp:93-119: point and vector transforms, left-to-right sums.
V3 transform_point(const Mat4& m, V3 p) {
    return {m(0, 0) * p.x + m(0, 1) * p.y + m(0, 2) * p.z + m(0, 3),
            m(1, 0) * p.x + m(1, 1) * p.y + m(1, 2) * p.z + m(1, 3),
            m(2, 0) * p.x + m(2, 1) * p.y + m(2, 2) * p.z + m(2, 3)};
}
V3 transform_vector(const Mat4& m, V3 v) {
    return {m(0, 0) * v.x + m(0, 1) * v.y + m(0, 2) * v.z,
            m(1, 0) * v.x + m(1, 1) * v.y + m(1, 2) * v.z,
            m(2, 0) * v.x + m(2, 1) * v.y + m(2, 2) * v.z};
}

struct Closure {
    uint32_t kind, lobes;
    Spectrum weight;
    float p[10];
};

constexpr uint32_t kMaxClosures = 8;  // MaximumClosureCount (ClosureSet.hpp:15)

struct Material {
    Closure closures[kMaxClosures];
    uint32_t closure_count;
    float probability[kMaxClosures];  // the mixture's projected component distribution
    float cdf[kMaxClosures + 1];
    uint32_t frame_mode;
    float rotation;
    Spectrum emission;
};

struct MeshLight {
    uint32_t instance;
    std::vector<V3> positions;  // world space
    std::vector<uint32_t> tris; // 3 per triangle
    std::vector<V3> normals;    // per-triangle geometric normal
    std::vector<float> areas, cdf;
    V3 position_error;
    float area, inverse_area;
    Spectrum radiance;
};

struct Instance {
    uint32_t geometry, material, mask, instance_id;
    Mat4 to_world, to_object;
    std::vector<V3> world_vertices;  // 3 per triangle
    std::vector<V3> world_normals;   // per triangle
};

// A punctual light of the registry (FrameScene.hpp:191-215) with the constants its sampling uses.
struct Punctual {
    uint32_t kind;
    V3 position, error, direction;
    float cos_inner, cos_outer;
    bool hard;
    Spectrum spectrum;
};

struct Scene {
    std::vector<Punctual> punctual;  // registry slots [0, punctual.size())
    std::vector<bf200_geometry_v1> geometries;
    std::vector<V3> positions, normals;
    std::vector<float> uvs;
    std::vector<uint32_t> triangles;
    std::vector<Material> materials;
    std::vector<Instance> instances;
    std::vector<MeshLight> lights;
    std::vector<float> light_cdf;  // uniform boundaries, size light_count + 1
    // spatial light tree (LightSampler::create_spatial_tree), when installed: selection and MIS
    // probabilities then depend on the shading / previous vertex position
    bf200::LightTree tree;
    bool use_tree = false;
    std::vector<int32_t> light_of_instance;
    Spectrum environment;
    float nm[4], pdf[4];
    bool prefilter = true;
};

V3 load3(const float* a, uint64_t i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }

// FrameScene.cpp:138-195: world positions of an emissive mesh and their absolute error bound.
bool transform_mesh_positions(const Scene& scene, const Instance& inst, MeshLight& light) {
    const auto& g = scene.geometries[inst.geometry];
    constexpr double eps = static_cast<double>(kEpsilon);
    constexpr double gamma7 = (7.0 * eps) / (1.0 - 7.0 * eps);
    constexpr double underflow = 7.0 * static_cast<double>(kDenormMin);
    constexpr double maximum = static_cast<double>(std::numeric_limits<float>::max());
    float max_error[3] = {0.0F, 0.0F, 0.0F};
    for (uint32_t v = 0; v < g.vertex_count; ++v) {
        const V3 source = scene.positions[g.vertex_offset + v];
        const V3 world = transform_point(inst.to_world, source);
        const float s[3] = {source.x, source.y, source.z};
        const float w[3] = {world.x, world.y, world.z};
        for (int row = 0; row < 3; ++row) {
            double magnitude = std::abs(static_cast<double>(inst.to_world(row, 3)));
            for (int col = 0; col < 3; ++col) {
                magnitude += std::abs(static_cast<double>(inst.to_world(row, col))) *
                             std::abs(static_cast<double>(s[col]));
            }
            const double bound = std::fma(gamma7, magnitude, underflow);
            if (!std::isfinite(static_cast<double>(w[row])) || !std::isfinite(bound) ||
                bound < 0.0 || bound > maximum) {
                return false;
            }
            float rounded = static_cast<float>(bound);
            if (static_cast<double>(rounded) < bound) {
                rounded = std::nextafter(rounded, kInfinity);
            }
            max_error[row] = std::max(max_error[row], rounded);
        }
        light.positions.push_back(world);
    }
    light.position_error = V3{max_error[0], max_error[1], max_error[2]};
    return true;
}

// AreaLights.hpp:1023-1183: mesh-light construction (areas, compensated total, float CDF).
bool build_mesh_light(MeshLight& light) {
    float sum = 0.0F, comp = 0.0F;
    const size_t n = light.tris.size() / 3;
    for (size_t t = 0; t < n; ++t) {
        const V3 a = light.positions[light.tris[3 * t]], b = light.positions[light.tris[3 * t + 1]],
                 c = light.positions[light.tris[3 * t + 2]];
        V3 normal;
        float area;
        if (!triangle_normal(a, b, c, normal) || !triangle_area(a, b, c, area)) {
            return false;
        }
        light.normals.push_back(normal);
        const float next = sum + area;
        if (std::abs(sum) >= std::abs(area)) {
            comp += (sum - next) + area;
        } else {
            comp += (area - next) + sum;
        }
        sum = next;
        light.areas.push_back(area);
    }
    const float total = sum + comp;
    if (!std::isfinite(total) || !(total > 0.0F)) {
        return false;
    }
    light.area = total;
    light.inverse_area = 1.0F / total;
    float cumulative = 0.0F;
    for (size_t t = 0; t < n; ++t) {
        float next = 1.0F;
        if (t + 1 != n) {
            const float selection = light.areas[t] / light.area;
            next = cumulative + selection;
            if (!(selection > 0.0F) || !(next > cumulative) || !(next < 1.0F)) {
                return false;
            }
        }
        cumulative = next;
        light.cdf.push_back(cumulative);
    }
    return true;
}

// ---------------------------------------------------------------------------------------------
// Acceleration queries: the analytic backend (AccelBackend.cpp:43-147)
// ---------------------------------------------------------------------------------------------

struct Hit {
    float t;
    float b0, b1, b2;
    uint32_t instance, primitive;
    V3 position, normal;
};

// ---------------------------------------------------------------------------------------------
// Analytic spheres: renderer::SphereT::intersect (Sphere.hpp:321-437) restated in float. The
// constant term and the discriminant are exact float expansions (add_component :48-81,
// add_product :83-95, multiply_expansions :109-122); their values are the in-order float sums of
// the components, the roots q / a and c / q, as in the reference.
// ---------------------------------------------------------------------------------------------

struct FloatExpansion {
    float c[128];
    int n = 0;
};

bool is_normal_float(float x) { return std::isnormal(x); }

bool fe_add(FloatExpansion& e, float component) {
    float accumulated = component;
    int out = 0;
    const int n = e.n;
    for (int i = 0; i < n; ++i) {
        const float existing = e.c[i];
        const float sum = accumulated + existing;
        const float existing_from_sum = sum - accumulated;
        const float accumulated_from_sum = sum - existing_from_sum;
        const float error = (existing - existing_from_sum) + (accumulated - accumulated_from_sum);
        if (!std::isfinite(sum) || !std::isfinite(error)) {
            return false;
        }
        if (error != 0.0F) {
            if (out == 128) {
                return false;
            }
            e.c[out++] = error;
        }
        accumulated = sum;
    }
    if (accumulated != 0.0F || out == 0) {
        if (out == 128) {
            return false;
        }
        e.c[out++] = accumulated;
    }
    e.n = out;
    return true;
}

bool fe_add_product(FloatExpansion& e, float left, float right, float sign = 1.0F) {
    const float rounded = left * right;
    const float error = std::fma(left, right, -rounded);
    if (!std::isfinite(rounded) || !std::isfinite(error) ||
        (left != 0.0F && right != 0.0F && !is_normal_float(rounded)) ||
        (error != 0.0F && !is_normal_float(error))) {
        return false;
    }
    return fe_add(e, sign * error) && fe_add(e, sign * rounded);
}

bool fe_add_expansion(FloatExpansion& destination, const FloatExpansion& source, float sign = 1.0F) {
    for (int i = 0; i < source.n; ++i) {
        if (!fe_add(destination, sign * source.c[i])) {
            return false;
        }
    }
    return true;
}

bool fe_multiply(const FloatExpansion& left, const FloatExpansion& right, FloatExpansion& product) {
    product = FloatExpansion{};
    for (int i = 0; i < left.n; ++i) {
        for (int j = 0; j < right.n; ++j) {
            if (!fe_add_product(product, left.c[i], right.c[j])) {
                return false;
            }
        }
    }
    return true;
}

int fe_sign(const FloatExpansion& e) {
    for (int i = e.n; i > 0; --i) {
        if (e.c[i - 1] != 0.0F) {
            return e.c[i - 1] > 0.0F ? 1 : -1;
        }
    }
    return 0;
}

float fe_value(const FloatExpansion& e) {
    float value = 0.0F;
    for (int i = 0; i < e.n; ++i) {
        value += e.c[i];
    }
    return value;
}

bool fe_squared_norm(V3 v, FloatExpansion& out) {
    out = FloatExpansion{};
    return fe_add_product(out, v.x, v.x) && fe_add_product(out, v.y, v.y) && fe_add_product(out, v.z, v.z);
}

float fused_dot(V3 a, V3 b) { return std::fma(a.x, b.x, std::fma(a.y, b.y, a.z * b.z)); }

// robust_outward_normal (Sphere.hpp:245-267)
bool sphere_outward_normal(V3 outward, V3& normal) {
    if (!std::isfinite(outward.x) || !std::isfinite(outward.y) || !std::isfinite(outward.z)) {
        return false;
    }
    const float m = std::max({std::abs(outward.x), std::abs(outward.y), std::abs(outward.z)});
    if (m == 0.0F) {
        return false;
    }
    const V3 scaled{outward.x / m, outward.y / m, outward.z / m};
    const float magnitude = std::sqrt(fused_dot(scaled, scaled));
    if (!std::isfinite(magnitude) || magnitude <= 0.0F) {
        return false;
    }
    normal = V3{scaled.x / magnitude, scaled.y / magnitude, scaled.z / magnitude};
    return true;
}

enum class SphereResult { miss, hit, failure };

SphereResult intersect_sphere(V3 centre, float radius, V3 o, V3 d, float t_min, float t_max, float& t_out,
                              V3& normal) {
    const V3 rel{o.x - centre.x, o.y - centre.y, o.z - centre.z};
    if (!std::isfinite(rel.x) || !std::isfinite(rel.y) || !std::isfinite(rel.z)) {
        return SphereResult::failure;
    }
    const float spatial_maximum = std::max({std::abs(rel.x), std::abs(rel.y), std::abs(rel.z), radius});
    const float direction_maximum = std::max({std::abs(d.x), std::abs(d.y), std::abs(d.z)});
    int se = 0, de = 0;
    static_cast<void>(std::frexp(spatial_maximum, &se));
    static_cast<void>(std::frexp(direction_maximum, &de));
    const V3 srel{std::ldexp(rel.x, -se), std::ldexp(rel.y, -se), std::ldexp(rel.z, -se)};
    const V3 sd{std::ldexp(d.x, -de), std::ldexp(d.y, -de), std::ldexp(d.z, -de)};
    const float sr = std::ldexp(radius, -se);
    auto preserved = [](float original, float scaled) { return original == 0.0F || std::isnormal(scaled); };
    if (!std::isfinite(direction_maximum) || direction_maximum <= 0.0F || !preserved(rel.x, srel.x) ||
        !preserved(rel.y, srel.y) || !preserved(rel.z, srel.z) || !preserved(d.x, sd.x) ||
        !preserved(d.y, sd.y) || !preserved(d.z, sd.z) || !preserved(radius, sr)) {
        return SphereResult::failure;
    }
    const float a = fused_dot(sd, sd);
    const float half_b = fused_dot(srel, sd);
    // exact_quadratic_constant (:147-181)
    float c = 0.0F;
    {
        FloatExpansion origin_squared, radius_squared;
        if (!fe_squared_norm(srel, origin_squared) || !fe_add_product(radius_squared, sr, sr) ||
            !fe_add_expansion(origin_squared, radius_squared, -1.0F)) {
            return SphereResult::failure;
        }
        const int sign = fe_sign(origin_squared);
        if (sign != 0) {
            c = fe_value(origin_squared);
            if (!std::isfinite(c) || c == 0.0F || (c > 0.0F ? 1 : -1) != sign) {
                return SphereResult::failure;
            }
        }
    }
    // exact_discriminant (:183-243)
    int disc_sign = 0;
    float disc = 0.0F;
    {
        FloatExpansion direction_squared, radius_squared, radial;
        if (!fe_squared_norm(sd, direction_squared) || !fe_add_product(radius_squared, sr, sr) ||
            !fe_multiply(direction_squared, radius_squared, radial)) {
            return SphereResult::failure;
        }
        const float terms[3][4] = {{srel.y, sd.z, srel.z, sd.y}, {srel.z, sd.x, srel.x, sd.z},
                                   {srel.x, sd.y, srel.y, sd.x}};
        FloatExpansion perpendicular;
        for (const auto& t : terms) {
            FloatExpansion cross, cross_squared;
            if (!fe_add_product(cross, t[0], t[1]) || !fe_add_product(cross, t[2], t[3], -1.0F) ||
                !fe_multiply(cross, cross, cross_squared) || !fe_add_expansion(perpendicular, cross_squared)) {
                return SphereResult::failure;
            }
        }
        if (!fe_add_expansion(radial, perpendicular, -1.0F)) {
            return SphereResult::failure;
        }
        disc_sign = fe_sign(radial);
        if (disc_sign > 0) {
            disc = fe_value(radial);
            if (!std::isfinite(disc) || disc <= 0.0F) {
                return SphereResult::failure;
            }
        }
    }
    if (!std::isfinite(a) || !std::isfinite(half_b) || !std::isfinite(c) || a <= 0.0F || sr <= 0.0F) {
        return SphereResult::failure;
    }
    if (disc_sign < 0) {
        return SphereResult::miss;
    }
    float r0, r1;
    if (disc_sign == 0) {
        r0 = -half_b / a;
        r1 = r0;
    } else {
        const float root = std::sqrt(disc);
        const float q = -half_b - std::copysign(root, half_b);
        if (!std::isfinite(root) || !std::isfinite(q) || q == 0.0F) {
            return SphereResult::failure;
        }
        r0 = q / a;
        r1 = c / q;
        if (r0 > r1) {
            std::swap(r0, r1);
        }
    }
    const float t0 = std::ldexp(r0, se - de), t1 = std::ldexp(r1, se - de);
    if (!std::isfinite(t0) || !std::isfinite(t1) || (r0 != 0.0F && t0 == 0.0F) || (r1 != 0.0F && t1 == 0.0F)) {
        return SphereResult::failure;
    }
    float t;
    if (!std::isnan(t0) && t0 >= t_min && t0 <= t_max) {
        t = t0;
    } else if (!std::isnan(t1) && t1 >= t_min && t1 <= t_max) {
        t = t1;
    } else {
        return SphereResult::miss;
    }
    const V3 position = o + d * t;  // Ray::at (Ray.hpp:81-95)
    if (!std::isfinite(position.x) || !std::isfinite(position.y) || !std::isfinite(position.z) ||
        !sphere_outward_normal(V3{position.x - centre.x, position.y - centre.y, position.z - centre.z}, normal)) {
        return SphereResult::failure;
    }
    t_out = t;
    return SphereResult::hit;
}

// Conservative double prefilter: true only when the three edge functions certainly have mixed
// signs, in which case the exact test is certain to report a miss (or a coplanar skip).
bool certainly_missed(V3 v0, V3 v1, V3 v2, V3 o, V3 d) {
    const double ox = o.x, oy = o.y, oz = o.z;
    const double p[3][3] = {{v0.x - ox, v0.y - oy, v0.z - oz},
                            {v1.x - ox, v1.y - oy, v1.z - oz},
                            {v2.x - ox, v2.y - oy, v2.z - oz}};
    const double dx = d.x, dy = d.y, dz = d.z;
    int signs[3];
    const int pairs[3][2] = {{1, 2}, {2, 0}, {0, 1}};
    for (int e = 0; e < 3; ++e) {
        const double* a = p[pairs[e][0]];
        const double* b = p[pairs[e][1]];
        const double t1 = a[0] * b[1] * dz, t2 = a[1] * b[2] * dx, t3 = a[2] * b[0] * dy;
        const double t4 = a[2] * b[1] * dx, t5 = a[1] * b[0] * dz, t6 = a[0] * b[2] * dy;
        const double value = ((t1 + t2) + t3) - ((t4 + t5) + t6);
        const double permanent = std::abs(t1) + std::abs(t2) + std::abs(t3) + std::abs(t4) +
                                 std::abs(t5) + std::abs(t6);
        const double bound = 32.0 * 0x1p-53 * permanent;
        if (value > bound) {
            signs[e] = 1;
        } else if (value < -bound) {
            signs[e] = -1;
        } else {
            signs[e] = 0;
        }
    }
    const bool has_pos = signs[0] > 0 || signs[1] > 0 || signs[2] > 0;
    const bool has_neg = signs[0] < 0 || signs[1] < 0 || signs[2] < 0;
    return has_pos && has_neg;
}

// Closest hit over every instance and triangle in committed order; ties keep the earlier one.
bool closest_hit(const Scene& scene, V3 origin, V3 dir, float t_min, float t_max, uint32_t mask,
                 Hit& best) {
    bool found = false;
    for (uint32_t i = 0; i < scene.instances.size(); ++i) {
        const Instance& inst = scene.instances[i];
        if ((mask & inst.mask) == 0U) {
            continue;
        }
        const V3 lo = transform_point(inst.to_object, origin);
        const V3 ld = transform_vector(inst.to_object, dir);
        const auto& g = scene.geometries[inst.geometry];
        if (g.kind == BF200_GEOMETRY_SPHERE) {
            float t = 0.0F;
            V3 n{};
            const SphereResult r = intersect_sphere(scene.positions[g.vertex_offset], g.radius, lo, ld, t_min,
                                                    found ? best.t : t_max, t, n);
            if (r == SphereResult::failure) {
                fail("A sphere intersection is not representable.");
            }
            if (r != SphereResult::hit || (found && best.t <= t)) {
                continue;
            }
            best.t = t;
            best.b0 = n.x;  // the object-space outward normal
            best.b1 = n.y;
            best.b2 = n.z;
            best.instance = i;
            best.primitive = 0;
            best.position = origin + dir * t;  // Ray::at (Ray.hpp:81-95)
            found = true;
            continue;
        }
        for (uint32_t t = 0; t < g.triangle_count; ++t) {
            const uint32_t* tri = &scene.triangles[3 * (g.triangle_offset + t)];
            const V3 v0 = scene.positions[g.vertex_offset + tri[0]];
            const V3 v1 = scene.positions[g.vertex_offset + tri[1]];
            const V3 v2 = scene.positions[g.vertex_offset + tri[2]];
            if (scene.prefilter && certainly_missed(v0, v1, v2, lo, ld)) {
                continue;
            }
            TriHit th;
            const TriResult r = intersect_triangle(v0, v1, v2, lo, ld, t_min, t_max, th);
            if (r == TriResult::failure) {
                fail("A triangle intersection is not representable.");
            }
            if (r != TriResult::hit) {
                continue;
            }
            if (found && best.t <= th.t) {
                continue;
            }
            best.t = th.t;
            best.b0 = th.b0;
            best.b1 = th.b1;
            best.b2 = th.b2;
            best.instance = i;
            best.primitive = t;
            best.normal = inst.world_normals[t];
            best.position = origin + dir * th.t;  // Ray::at (Ray.hpp:81-95)
            found = true;
        }
    }
    return found;
}

bool occluded(const Scene& scene, V3 origin, V3 dir, float t_min, float t_max, uint32_t mask) {
    for (uint32_t i = 0; i < scene.instances.size(); ++i) {
        const Instance& inst = scene.instances[i];
        if ((mask & inst.mask) == 0U) {
            continue;
        }
        const V3 lo = transform_point(inst.to_object, origin);
        const V3 ld = transform_vector(inst.to_object, dir);
        const auto& g = scene.geometries[inst.geometry];
        if (g.kind == BF200_GEOMETRY_SPHERE) {
            float t = 0.0F;
            V3 n{};
            const SphereResult r =
                intersect_sphere(scene.positions[g.vertex_offset], g.radius, lo, ld, t_min, t_max, t, n);
            if (r == SphereResult::failure) {
                fail("A sphere intersection is not representable.");
            }
            if (r == SphereResult::hit) {
                return true;
            }
            continue;
        }
        for (uint32_t t = 0; t < g.triangle_count; ++t) {
            const uint32_t* tri = &scene.triangles[3 * (g.triangle_offset + t)];
            const V3 v0 = scene.positions[g.vertex_offset + tri[0]];
            const V3 v1 = scene.positions[g.vertex_offset + tri[1]];
            const V3 v2 = scene.positions[g.vertex_offset + tri[2]];
            if (scene.prefilter && certainly_missed(v0, v1, v2, lo, ld)) {
                continue;
            }
            TriHit th;
            const TriResult r = intersect_triangle(v0, v1, v2, lo, ld, t_min, t_max, th);
            if (r == TriResult::failure) {
                fail("A triangle intersection is not representable.");
            }
            if (r == TriResult::hit) {
                return true;
            }
        }
    }
    return false;
}

// ---------------------------------------------------------------------------------------------
// Geometry helpers
// ---------------------------------------------------------------------------------------------

float max_abs3(V3 v) { return std::max({std::abs(v.x), std::abs(v.y), std::abs(v.z)}); }

// BsdfOnlyPathLoop.hpp:190-209 / PinholeCamera.hpp:27-46: scale by the largest component, then
// divide by the square root of the scaled length squared.
V3 robust_unit(V3 d) {
    if (!finite3(d)) {
        fail("A path direction must remain finite.");
    }
    const float m = max_abs3(d);
    if (m == 0.0F) {
        fail("A path direction must remain non-zero.");
    }
    const V3 s = d / m;
    const float magnitude = std::sqrt(dot(s, s));
    const V3 r = s / magnitude;
    if (!finite3(r)) {
        fail("Path normalization is not representable.");
    }
    return r;
}

bool unit_length(V3 d) {  // ClosureMixture.hpp:56-64 and its twins
    if (!finite3(d)) {
        return false;
    }
    const float sq = std::fma(d.x, d.x, std::fma(d.y, d.y, d.z * d.z));
    return std::isfinite(sq) && std::abs(sq - 1.0F) <= kEpsilon * 128.0F;
}

struct Frame {
    V3 t, b, n;
    V3 to_local(V3 w) const { return {dot(w, t), dot(w, b), dot(w, n)}; }
    // LocalFrame.hpp:160-163: tangent*x + bitangent*y + normal*z, per component.
    V3 to_world(V3 l) const {
        return {t.x * l.x + b.x * l.y + n.x * l.z, t.y * l.x + b.y * l.y + n.y * l.z,
                t.z * l.x + b.z * l.y + n.z * l.z};
    }
};

// LocalFrame.hpp:8-30.
V3 robust_unit_normal(V3 v) {
    const float m = max_abs3(v);
    if (!finite3(v) || m == 0.0F) {
        fail("A frame normal must be finite and non-zero.");
    }
    const V3 s{v.x / m, v.y / m, v.z / m};
    const float magnitude = std::sqrt(s.x * s.x + s.y * s.y + s.z * s.z);
    return V3{s.x / magnitude, s.y / magnitude, s.z / magnitude};
}

V3 robust_unit_vector(V3 v) {  // LocalFrame.hpp:32-48
    const float m = max_abs3(v);
    if (!finite3(v) || m == 0.0F) {
        fail("A frame tangent must be finite and non-parallel to its normal.");
    }
    const V3 s = v / m;
    const float magnitude = std::sqrt(dot(s, s));
    return s / magnitude;
}

bool orthonormal(V3 t, V3 b, V3 n) {  // LocalFrame.hpp:50-62
    constexpr float tol = kEpsilon * 128.0F;
    return std::abs(dot(t, t) - 1.0F) <= tol && std::abs(dot(b, b) - 1.0F) <= tol &&
           std::abs(dot(n, n) - 1.0F) <= tol && std::abs(dot(t, b)) <= tol &&
           std::abs(dot(t, n)) <= tol && std::abs(dot(b, n)) <= tol &&
           std::abs(dot(cross(t, b), n) - 1.0F) <= tol;
}

// LocalFrame.hpp:188-219 (from_unit_normal_and_tangent).
Frame frame_from_unit_normal_and_tangent(V3 n, V3 tangent) {
    const V3 td = robust_unit_vector(tangent);
    const V3 projected = td - n * dot(td, n);
    V3 ut = robust_unit_vector(projected);
    const V3 ub = robust_unit_vector(cross(n, ut));
    ut = robust_unit_vector(cross(ub, n));
    if (!orthonormal(ut, ub, n)) {
        fail("The supplied directions cannot form a stable orthonormal frame.");
    }
    return Frame{ut, ub, n};
}

// LocalFrame.hpp:66-80 (from_normal).
Frame frame_from_normal(V3 normal) {
    const V3 n = robust_unit_normal(normal);
    const float sign = std::copysign(1.0F, n.z);
    const float coefficient = -1.0F / (sign + n.z);
    const float product = n.x * n.y * coefficient;
    const V3 seed{1.0F + sign * n.x * n.x * coefficient, sign * product, -sign * n.x};
    return frame_from_unit_normal_and_tangent(n, seed);
}

// LocalFrame.hpp:116-135 (rotated_about_normal).
Frame rotated_about_normal(const Frame& f, float angle) {
    const float reduced = std::remainder(angle, 2.0F * kPi);
    const float c = cos_f(reduced);
    const float s = sin_f(reduced);
    const V3 rotated = f.t * c + f.b * s;
    return frame_from_unit_normal_and_tangent(f.n, rotated);
}

// RayOriginOffset.hpp:58-117 (offset_ray_origin).
V3 offset_ray_origin(V3 p, V3 err, V3 ng, V3 w) {
    const float m = max_abs3(ng);
    const V3 sn = ng / m;
    const V3 n = sn / std::sqrt(dot(sn, sn));
    const float d = std::abs(n.x) * err.x + std::abs(n.y) * err.y + std::abs(n.z) * err.z;
    if (!std::isfinite(d)) {
        fail("The projected ray origin error is not finite.");
    }
    const float ds = max_abs3(w);
    const V3 sw = w / ds;
    V3 offset{n.x * d, n.y * d, n.z * d};
    if (dot(n, sw) < 0.0F) {
        offset = -offset;
    }
    auto outward = [](float value, float off) {
        if (off > 0.0F) {
            return std::nextafter(value, kInfinity);
        }
        if (off < 0.0F) {
            return std::nextafter(value, -kInfinity);
        }
        return value;
    };
    const V3 shifted{outward(p.x + offset.x, offset.x), outward(p.y + offset.y, offset.y),
                     outward(p.z + offset.z, offset.z)};
    if (!finite3(shifted)) {
        fail("The ray origin offset exceeds the finite coordinate range.");
    }
    return shifted;
}

// ShadowRay.hpp:15-48 (offset_surface_point).
V3 offset_surface_point(V3 p, V3 err, V3 ng, V3 w) {
    const V3 offset = offset_ray_origin(p, err, ng, w);
    if (offset != p) {
        return offset;
    }
    V3 oriented = ng;
    if (dot(ng, w) < 0.0F) {
        oriented = -oriented;
    }
    V3 shifted = p;
    if (oriented.x != 0.0F) {
        shifted.x = std::nextafter(p.x, oriented.x > 0.0F ? kInfinity : -kInfinity);
    }
    if (oriented.y != 0.0F) {
        shifted.y = std::nextafter(p.y, oriented.y > 0.0F ? kInfinity : -kInfinity);
    }
    if (oriented.z != 0.0F) {
        shifted.z = std::nextafter(p.z, oriented.z > 0.0F ? kInfinity : -kInfinity);
    }
    if (!finite3(shifted) || shifted == p) {
        fail("A shadow-ray surface offset is not representable in the requested precision.");
    }
    return shifted;
}

// ShadowRay.hpp:107-135 (unit_segment).
void unit_segment(V3 origin, V3 endpoint, V3 expected, V3& direction, float& length) {
    const V3 disp = endpoint - origin;
    const float scale = max_abs3(disp);
    if (!(scale > 0.0F) || !std::isfinite(scale)) {
        fail("A finite shadow-ray segment must have positive length.");
    }
    const V3 s = disp / scale;
    const float sq = std::fma(s.x, s.x, std::fma(s.y, s.y, s.z * s.z));
    const float sl = std::sqrt(sq);
    length = scale * sl;
    if (!(sl > 0.0F) || !std::isfinite(sl) || !(length > 0.0F) || !std::isfinite(length)) {
        fail("A finite shadow-ray length is not representable.");
    }
    direction = s / sl;
    const float alignment = dot(direction, expected);
    if (!std::isfinite(alignment) || !(alignment > 0.0F)) {
        fail("Shadow-ray endpoint contraction reversed the sampled light direction.");
    }
}

// ---------------------------------------------------------------------------------------------
// Checked products (frexp/scalbn forms of the reference)
// ---------------------------------------------------------------------------------------------

// DirectLighting.hpp:21-62 (checked_product_quotient).
float checked_product_quotient(const float* num, int nn, const float* den, int nd) {
    float significand = 1.0F;
    int exponent = 0;
    for (int i = 0; i < nn; ++i) {
        const float v = num[i];
        if (!std::isfinite(v) || v < 0.0F) {
            fail("Direct-lighting numerator factors must be finite and non-negative.");
        }
        if (v == 0.0F) {
            return 0.0F;
        }
        int e = 0;
        significand *= std::frexp(v, &e);
        exponent += e;
    }
    for (int i = 0; i < nd; ++i) {
        const float v = den[i];
        if (!std::isfinite(v) || !(v > 0.0F)) {
            fail("Direct-lighting PDF factors must be finite and strictly positive.");
        }
        int e = 0;
        significand /= std::frexp(v, &e);
        exponent -= e;
    }
    int ne = 0;
    significand = std::frexp(significand, &ne);
    const float result = std::scalbn(significand, exponent + ne);
    if (!std::isfinite(result) || !(result > 0.0F)) {
        fail("Direct-lighting contribution is not representable in the requested precision.");
    }
    return result;
}

// RoughDielectric.hpp:52-86 (checked_product_ratio: renormalises after every factor).
float checked_product_ratio(const float* num, int nn, const float* den, int nd) {
    bool zero = false;
    for (int i = 0; i < nn; ++i) {
        if (!std::isfinite(num[i]) || num[i] < 0.0F) {
            fail("A rough-dielectric product is not representable.");
        }
        zero = zero || num[i] == 0.0F;
    }
    for (int i = 0; i < nd; ++i) {
        if (!std::isfinite(den[i]) || !(den[i] > 0.0F)) {
            fail("A rough-dielectric product is not representable.");
        }
    }
    if (zero) {
        return 0.0F;
    }
    float significand = 1.0F;
    int exponent = 0;
    for (int i = 0; i < nn; ++i) {
        int ve = 0, ne = 0;
        const float vs = std::frexp(num[i], &ve);
        significand = std::frexp(significand * vs, &ne);
        exponent += ve + ne;
    }
    for (int i = 0; i < nd; ++i) {
        int ve = 0, ne = 0;
        const float vs = std::frexp(den[i], &ve);
        significand = std::frexp(significand / vs, &ne);
        exponent += ne - ve;
    }
    const float result = std::scalbn(significand, exponent);
    if (!std::isfinite(result) || !(result > 0.0F)) {
        fail("A rough-dielectric product is not representable.");
    }
    return result;
}

// MisHeuristics.hpp:142-172 and ClosureMixture.hpp:249-268: a positive product of two factors.
float positive_product2(float a, float b) {
    if (b == 0.0F) {
        return 0.0F;
    }
    int ea = 0, eb = 0, en = 0;
    const float sa = std::frexp(a, &ea);
    const float sb = std::frexp(b, &eb);
    const float n = std::frexp(sa * sb, &en);
    const float r = std::scalbn(n, ea + eb + en);
    if (!std::isfinite(r) || !(r > 0.0F)) {
        fail("A positive probability product is not representable.");
    }
    return r;
}

// MisHeuristics.hpp:44-72.
float ratio_at_most_one(float n, float d) {
    int ne = 0, de = 0;
    const float ns = std::frexp(n, &ne);
    const float ds = std::frexp(d, &de);
    return std::scalbn(ns / ds, ne - de);
}
float squared_ratio_at_most_one(float n, float d) {
    int ne = 0, de = 0;
    const float ns = std::frexp(n, &ne);
    const float ds = std::frexp(d, &de);
    const float r = ns / ds;
    return std::scalbn(r * r, 2 * (ne - de));
}
float checked_small_weight(float ratio) {
    if (!(ratio > 0.0F)) {
        fail("The positive MIS weight is not representable in the requested precision.");
    }
    const float w = ratio / (1.0F + ratio);
    if (!std::isfinite(w) || !(w > 0.0F)) {
        fail("The positive MIS weight is not representable in the requested precision.");
    }
    return w;
}

// MisHeuristics.hpp:75-141 (balance/power with validate_pdfs).
float mis_weight(uint32_t heuristic, float sampled, float competing) {
    if (!std::isfinite(sampled) || !(sampled > 0.0F)) {
        fail("The sampled-technique MIS PDF must be finite and strictly positive.");
    }
    if (!std::isfinite(competing) || competing < 0.0F) {
        fail("The competing-technique MIS PDF must be finite and non-negative.");
    }
    if (competing == 0.0F) {
        return 1.0F;
    }
    if (heuristic == 0) {
        if (sampled < competing) {
            return checked_small_weight(ratio_at_most_one(sampled, competing));
        }
        return 1.0F / (1.0F + ratio_at_most_one(competing, sampled));
    }
    if (sampled < competing) {
        return checked_small_weight(squared_ratio_at_most_one(sampled, competing));
    }
    return 1.0F / (1.0F + squared_ratio_at_most_one(competing, sampled));
}

// MisHeuristics.hpp:143-172 (joint_light_pdf).
float joint_light_pdf(float selection, float conditional) {
    if (!std::isfinite(selection) || !(selection > 0.0F) || selection > 1.0F) {
        fail("A joint light PDF requires a discrete selection probability in (0, 1].");
    }
    if (!std::isfinite(conditional) || conditional < 0.0F) {
        fail("A joint light PDF requires a finite non-negative conditional PDF.");
    }
    if (conditional == 0.0F) {
        return 0.0F;
    }
    return positive_product2(selection, conditional);
}

// ---------------------------------------------------------------------------------------------
// Emission (Emission.hpp:42-108)
// ---------------------------------------------------------------------------------------------

bool unit_normal(V3 n) {
    const float sq = std::fma(n.x, n.x, std::fma(n.y, n.y, n.z * n.z));
    return finite3(n) && std::isfinite(sq) && std::abs(sq - 1.0F) <= kEpsilon * 128.0F;
}

// Returns +1 (emitting side), 0 (back side / tangent-orthogonal), fails when ambiguous.
int emission_side(V3 ng, V3 wo) {
    if (!unit_normal(ng) || !finite3(wo) || (wo.x == 0.0F && wo.y == 0.0F && wo.z == 0.0F)) {
        fail("Surface emission evaluation requires a unit normal and a non-zero direction.");
    }
    const float m = max_abs3(wo);
    const V3 s = wo / m;
    const float alignment = std::fma(ng.x, s.x, std::fma(ng.y, s.y, ng.z * s.z));
    if (!std::isfinite(alignment)) {
        fail("Surface emission orientation is not representable.");
    }
    const bool orthogonal = (ng.x == 0.0F || wo.x == 0.0F) && (ng.y == 0.0F || wo.y == 0.0F) &&
                            (ng.z == 0.0F || wo.z == 0.0F);
    if (alignment == 0.0F && orthogonal) {
        return 0;
    }
    const float abs_sum =
        std::fma(std::abs(ng.x), std::abs(s.x),
                 std::fma(std::abs(ng.y), std::abs(s.y), std::abs(ng.z) * std::abs(s.z)));
    const float uncertainty = std::fma(4.0F * kEpsilon, abs_sum, 4.0F * kDenormMin);
    if (std::abs(alignment) <= uncertainty) {
        fail("Surface emission orientation is not representable.");
    }
    return alignment > 0.0F ? 1 : 0;
}

bool is_black(const Spectrum& s) { return s[0] == 0 && s[1] == 0 && s[2] == 0 && s[3] == 0; }

// ---------------------------------------------------------------------------------------------
// Area-light pdf conversion (Light.hpp:75-163, 593-620) and mesh-light sampling
// ---------------------------------------------------------------------------------------------

float area_to_solid_angle(float area_pdf, V3 ref, V3 surf, V3 ng) {
    if (!unit_normal(ng)) {
        fail("Light PDF conversion requires a finite unit surface geometric normal.");
    }
    const V3 disp = surf - ref;
    const float scale = max_abs3(disp);
    if (!(scale > 0.0F) || !std::isfinite(scale)) {
        fail("Light PDF conversion requires two distinct positions.");
    }
    const V3 s = disp / scale;
    const float sq = std::fma(s.x, s.x, std::fma(s.y, s.y, s.z * s.z));
    const float sl = std::sqrt(sq);
    const float cubed = sq * sl;
    if (!std::isfinite(sq) || !(sq > 0.0F) || !std::isfinite(cubed) || !(cubed > 0.0F)) {
        fail("Light PDF conversion distance is not representable.");
    }
    const float signed_alignment = std::fma(ng.x, -s.x, std::fma(ng.y, -s.y, ng.z * -s.z));
    const float alignment = std::abs(signed_alignment);
    const float term_sum =
        std::fma(std::abs(ng.x), std::abs(s.x),
                 std::fma(std::abs(ng.y), std::abs(s.y), std::abs(ng.z) * std::abs(s.z)));
    const float uncertainty = std::fma(4.0F * kEpsilon, term_sum, 4.0F * kDenormMin);
    if (!std::isfinite(alignment) || !std::isfinite(term_sum) || alignment <= uncertainty) {
        fail("Light PDF conversion Jacobian is singular or numerically ambiguous.");
    }
    if (area_pdf == 0.0F) {
        return 0.0F;
    }
    int es = 0, ed = 0, ec = 0, ea = 0, en = 0;
    const float fs = std::frexp(area_pdf, &es);
    const float fd = std::frexp(scale, &ed);
    const float fc = std::frexp(cubed, &ec);
    const float fa = std::frexp(alignment, &ea);
    const float combined = fs * fd * fd * fc / fa;
    const int exponent = es + 2 * ed + ec - ea;
    const float normalized = std::frexp(combined, &en);
    const float converted = std::scalbn(normalized, exponent + en);
    if (!std::isfinite(converted) || !(converted > 0.0F)) {
        fail("Converted light PDF is not representable in the requested precision.");
    }
    return converted;
}

struct LightSample {
    bool valid = false;
    V3 position, error, normal;
    V3 direction;
    float distance;
    float pdf;  // solid angle, or the discrete mass of a punctual light
    Spectrum radiance;
    bool discrete = false;  // punctual: the pdf is a discrete probability
    bool point = false;     // finite point endpoint (point and spot lights)
    bool infinite = false;  // directional light: no endpoint
};

// IncidentLightSample::create_finite (Light.hpp:401-441): direction and distance.
void incident_direction(V3 context, V3 endpoint, V3& direction, float& distance) {
    const V3 disp = endpoint - context;
    const float scale = max_abs3(disp);
    if (!(scale > 0.0F) || !std::isfinite(scale)) {
        fail("A finite incident light sample requires distinct positions.");
    }
    const V3 s = disp / scale;
    const float sq = std::fma(s.x, s.x, std::fma(s.y, s.y, s.z * s.z));
    const float sl = std::sqrt(sq);
    distance = scale * sl;
    if (!std::isfinite(sl) || !(sl > 0.0F) || !std::isfinite(distance) || !(distance > 0.0F)) {
        fail("Finite incident light sample distance is not representable.");
    }
    direction = s / sl;
    if (!unit_length(direction)) {
        fail("An incident light sample requires a finite unit direction.");
    }
}

// MeshAreaLight::sample_li (AreaLights.hpp:1184-1243) with finish_sample (AreaLights.hpp:329-371).
LightSample sample_mesh_light(const MeshLight& light, V3 context, float u, float v) {
    LightSample out;
    if (!(u >= 0.0F && u < 1.0F && v >= 0.0F && v < 1.0F)) {
        fail("Area-light sampling requires a canonical sample.");
    }
    const auto it = std::upper_bound(light.cdf.begin(), light.cdf.end(), u);
    if (it == light.cdf.end()) {
        fail("Mesh area-light selection escaped its cumulative distribution.");
    }
    const size_t index = static_cast<size_t>(it - light.cdf.begin());
    const float previous = index == 0 ? 0.0F : light.cdf[index - 1];
    const float selection = light.cdf[index] - previous;
    const float remapped = (u - previous) / selection;
    if (!std::isfinite(selection) || !(selection > 0.0F) || !std::isfinite(remapped) ||
        remapped < 0.0F || !(remapped < 1.0F)) {
        fail("Mesh area-light canonical remapping is not representable.");
    }
    const float density = selection / light.areas[index];
    if (!std::isfinite(density) || !(density > 0.0F)) {
        fail("Mesh area-light triangle density is not representable.");
    }
    const float root = std::sqrt(remapped);
    const float bary[3] = {1.0F - root, root * (1.0F - v), root * v};
    const V3 p[3] = {light.positions[light.tris[3 * index]], light.positions[light.tris[3 * index + 1]],
                     light.positions[light.tris[3 * index + 2]]};
    // triangle_position_with_error (AreaLights.hpp:260-301).
    constexpr float gamma12 = (12.0F * kEpsilon) / (1.0F - 12.0F * kEpsilon);
    constexpr float underflow = 12.0F * kDenormMin;
    const float base[3] = {light.position_error.x, light.position_error.y, light.position_error.z};
    float point[3], error[3];
    for (int axis = 0; axis < 3; ++axis) {
        const float c0 = axis == 0 ? p[0].x : axis == 1 ? p[0].y : p[0].z;
        const float c1 = axis == 0 ? p[1].x : axis == 1 ? p[1].y : p[1].z;
        const float c2 = axis == 0 ? p[2].x : axis == 1 ? p[2].y : p[2].z;
        const float prod0 = bary[0] * c0, prod1 = bary[1] * c1, prod2 = bary[2] * c2;
        point[axis] = std::fma(bary[0], c0, std::fma(bary[1], c1, prod2));
        const float magnitude = std::abs(prod0) + std::abs(prod1) + std::abs(prod2);
        const float arithmetic = std::fma(gamma12, magnitude, underflow);
        error[axis] = std::nextafter(base[axis] + arithmetic, kInfinity);
    }
    out.position = V3{point[0], point[1], point[2]};
    out.error = V3{error[0], error[1], error[2]};
    out.normal = light.normals[index];
    // one-sided support, then the solid-angle conversion of the triangle's area density.
    if (emission_side(out.normal, context - out.position) <= 0) {
        return out;  // no sample
    }
    out.pdf = area_to_solid_angle(density, context, out.position, out.normal);
    incident_direction(context, out.position, out.direction, out.distance);
    if (!std::isfinite(out.pdf) || !(out.pdf > 0.0F)) {
        fail("A finite surface light sample requires a solid-angle density.");
    }
    out.radiance = light.radiance;
    out.valid = !is_black(light.radiance);
    return out;
}

// MeshAreaLight::pdf_li_at_surface (AreaLights.hpp:1296-1309) via finish_pdf (AreaLights.hpp:373-403).
float mesh_light_pdf_at_surface(const MeshLight& light, V3 context, V3 surface, V3 ng) {
    if (emission_side(ng, context - surface) <= 0) {
        return 0.0F;
    }
    const float pdf = area_to_solid_angle(light.inverse_area, context, surface, ng);
    if (is_black(light.radiance)) {
        return 0.0F;
    }
    return pdf;
}

// scale_radiometric_value (PunctualLights.hpp:131-183): value x numerators / denominators, each
// factor taken as a significand and an exponent so no partial product under- or overflows.
float scale_radiometric(float value, const float* num, int nn, const float* den, int nd) {
    if (!std::isfinite(value) || value < 0.0F) {
        fail("Punctual light radiometric values must be finite and non-negative.");
    }
    for (int i = 0; i < nn; ++i) {
        if (!std::isfinite(num[i]) || !(num[i] > 0.0F)) {
            fail("A punctual light radiometric numerator is not representable.");
        }
    }
    for (int i = 0; i < nd; ++i) {
        if (!std::isfinite(den[i]) || !(den[i] > 0.0F)) {
            fail("A punctual light radiometric denominator is not representable.");
        }
    }
    if (value == 0.0F) {
        return 0.0F;
    }
    int exponent = 0;
    float fraction = std::frexp(value, &exponent);
    long long accumulated = exponent;
    for (int i = 0; i < nn; ++i) {
        int e = 0;
        fraction *= std::frexp(num[i], &e);
        accumulated += e;
    }
    for (int i = 0; i < nd; ++i) {
        int e = 0;
        fraction /= std::frexp(den[i], &e);
        accumulated -= e;
    }
    int ne = 0;
    fraction = std::frexp(fraction, &ne);
    accumulated += ne;
    const float result = std::scalbn(fraction, static_cast<int>(accumulated));
    if (!std::isfinite(result) || !(result > 0.0F)) {
        fail("A positive punctual light result is not representable in the requested precision.");
    }
    return result;
}

// PointLight / DirectionalLight / SpotLight::sample_li (PunctualLights.hpp:390-430, 510-530,
// 654-720) with IncidentLightSample::create_finite / create_infinite (Light.hpp:404-456).
LightSample sample_punctual_light(const Punctual& light, V3 context, float u, float v) {
    LightSample out;
    if (!std::isfinite(u) || !std::isfinite(v) || u < 0.0F || u >= 1.0F || v < 0.0F || v >= 1.0F) {
        fail("Punctual light sampling requires a finite canonical sample in [0, 1)^2.");
    }
    out.discrete = true;
    out.pdf = 1.0F;
    if (light.kind == BF200_PUNCTUAL_DIRECTIONAL) {
        if (is_black(light.spectrum)) {
            return out;
        }
        out.direction = V3{-light.direction.x, -light.direction.y, -light.direction.z};
        if (!unit_length(out.direction)) {
            fail("An incident light sample requires a finite unit direction.");
        }
        out.distance = kInfinity;
        out.radiance = light.spectrum;
        out.infinite = true;
        out.valid = true;
        return out;
    }
    // finite_light_geometry (PunctualLights.hpp:102-129)
    const V3 disp = light.position - context;
    if (!std::isfinite(disp.x) || !std::isfinite(disp.y) || !std::isfinite(disp.z)) {
        fail("Finite punctual light separation is not representable in the requested precision.");
    }
    const float scale = max_abs3(disp);
    if (!(scale > 0.0F) || !std::isfinite(scale)) {
        fail("A finite punctual light cannot be sampled at its own position.");
    }
    const V3 scaled = disp / scale;
    const float squared = std::fma(scaled.x, scaled.x, std::fma(scaled.y, scaled.y, scaled.z * scaled.z));
    const float root = std::sqrt(squared);
    const float distance = scale * root;
    if (!std::isfinite(squared) || !(squared > 0.0F) || !std::isfinite(root) || !(root > 0.0F) ||
        !std::isfinite(distance) || !(distance > 0.0F)) {
        fail("Finite punctual light distance is not representable in the requested precision.");
    }
    const V3 to_light = scaled / root;
    if (!unit_length(to_light)) {
        fail("Finite punctual light direction is not representable as a unit vector.");
    }
    float falloff[3] = {1.0F, 1.0F, 1.0F};
    int falloff_count = 0;
    if (light.kind == BF200_PUNCTUAL_SPOT) {
        const V3 from_light{-to_light.x, -to_light.y, -to_light.z};
        const float cone = std::fma(light.direction.x, from_light.x,
                                    std::fma(light.direction.y, from_light.y, light.direction.z * from_light.z));
        if (!std::isfinite(cone)) {
            fail("Spot light cone evaluation is not representable.");
        }
        if (cone <= light.cos_outer) {
            return out;
        }
        falloff_count = 3;
        if (!light.hard && cone < light.cos_inner) {
            const float transition = (cone - light.cos_outer) / (light.cos_inner - light.cos_outer);
            const float smooth = 3.0F - 2.0F * transition;
            if (!std::isfinite(transition) || !(transition > 0.0F) || !(transition < 1.0F) ||
                !std::isfinite(smooth) || !(smooth > 0.0F)) {
                fail("Spot light smooth falloff is not representable.");
            }
            falloff[0] = transition;
            falloff[1] = transition;
            falloff[2] = smooth;
        }
    }
    const float den[3] = {scale, scale, squared};
    for (int lane = 0; lane < 4; ++lane) {
        out.radiance[lane] = scale_radiometric(light.spectrum[lane], falloff, falloff_count, den, 3);
    }
    if (is_black(light.spectrum)) {
        return out;
    }
    incident_direction(context, light.position, out.direction, out.distance);
    out.position = light.position;
    out.error = light.error;
    out.point = true;
    out.valid = true;
    return out;
}

// contract_point_endpoint (ShadowRay.hpp:66-113): the point light's endpoint moved toward the
// shading point past its position error, so the shadow ray's interval excludes the light.
V3 contract_point_endpoint(V3 point, V3 error, V3 to_light) {
    float contraction = 0.0F;
    auto support = [&](float direction, float e) {
        const float candidate = std::fma(std::abs(direction), e, contraction);
        if (!std::isfinite(candidate) || candidate < contraction) {
            fail("A shadow-ray point-endpoint contraction is not representable.");
        }
        if (direction != 0.0F && e != 0.0F) {
            contraction = std::nextafter(candidate, kInfinity);
            if (!std::isfinite(contraction)) {
                fail("A shadow-ray point-endpoint contraction is not representable.");
            }
        } else {
            contraction = candidate;
        }
    };
    support(to_light.x, error.x);
    support(to_light.y, error.y);
    support(to_light.z, error.z);
    if (contraction == 0.0F) {
        return point;
    }
    V3 c{std::fma(-to_light.x, contraction, point.x), std::fma(-to_light.y, contraction, point.y),
         std::fma(-to_light.z, contraction, point.z)};
    if (to_light.x != 0.0F) {
        c.x = std::nextafter(c.x, to_light.x > 0.0F ? -kInfinity : kInfinity);
    }
    if (to_light.y != 0.0F) {
        c.y = std::nextafter(c.y, to_light.y > 0.0F ? -kInfinity : kInfinity);
    }
    if (to_light.z != 0.0F) {
        c.z = std::nextafter(c.z, to_light.z > 0.0F ? -kInfinity : kInfinity);
    }
    if (!std::isfinite(c.x) || !std::isfinite(c.y) || !std::isfinite(c.z)) {
        fail("A shadow-ray point endpoint exceeds the finite coordinate range.");
    }
    return c;
}

// ---------------------------------------------------------------------------------------------
// Closures
// ---------------------------------------------------------------------------------------------

struct BsdfSample {
    bool valid = false;
    V3 wi;
    Spectrum value{};
    float pdf = 0.0F;
    bool delta = false;  // pdf is a discrete (delta) mass rather than a solid-angle density
    uint32_t lobes = 0;
    float eta_scale = 1.0F;
    uint32_t selected = 0;  // the source index of the sampled closure
};

// SamplingMappings.hpp:33-60 and 128-141 (concentric disk, cosine hemisphere).
V3 map_cosine_hemisphere(float u, float v) {
    const float ox = 2.0F * u - 1.0F;
    const float oy = 2.0F * v - 1.0F;
    float px = 0.0F, py = 0.0F, radius = 0.0F;
    if (!(ox == 0.0F && oy == 0.0F)) {
        constexpr float quarter_pi = kPi / 4.0F;
        float r, phi;
        if (std::abs(ox) > std::abs(oy)) {
            r = ox;
            phi = quarter_pi * (oy / ox);
        } else {
            r = oy;
            phi = 2.0F * quarter_pi - quarter_pi * (ox / oy);
        }
        px = r * cos_f(phi);
        py = r * sin_f(phi);
        radius = std::abs(r);
    }
    const float z = std::sqrt((1.0F - radius) * (1.0F + radius));
    return V3{px, py, z};
}

// GGX (GgxMicrofacet.hpp).
struct Ggx {
    float ax, ay;
};

struct SmithTerms {
    float normal, tangent, radius, normal_over_radius;
};

// GgxMicrofacet.hpp:134-184.
SmithTerms smith_terms(const Ggx& g, V3 w) {
    SmithTerms t{};
    if (g.ax == g.ay) {
        const float alpha = g.ax;
        const float sine = std::hypot(w.x, w.y);
        const float inverse_alpha = 1.0F / alpha;
        t.normal = alpha <= 1.0F ? w.z : w.z * inverse_alpha;
        t.tangent = alpha <= 1.0F ? alpha * sine : sine;
        t.radius = std::hypot(t.normal, t.tangent);
    } else {
        const float common = std::max({1.0F, g.ax, g.ay});
        t.normal = w.z / common;
        const float tx = (g.ax / common) * w.x;
        const float ty = (g.ay / common) * w.y;
        t.tangent = std::hypot(tx, ty);
        t.radius = std::hypot(t.normal, t.tangent);
    }
    if (!std::isfinite(t.normal) || !std::isfinite(t.tangent) || !std::isfinite(t.radius) ||
        !(t.normal > 0.0F) || !(t.radius > 0.0F)) {
        fail("GGX Smith geometry is not representable for the supplied direction.");
    }
    t.normal_over_radius = t.normal / t.radius;
    if (!std::isfinite(t.normal_over_radius) || !(t.normal_over_radius > 0.0F) ||
        t.normal_over_radius > 1.0F) {
        fail("GGX Smith geometry is not representable for the supplied direction.");
    }
    return t;
}

// GgxMicrofacet.hpp:232-270 (normal_distribution).
float ggx_d(const Ggx& g, V3 m) {
    if (!unit_length(m)) {
        fail("GGX microfacet normals must be finite unit normals.");
    }
    if (!(m.z > 0.0F)) {
        return 0.0F;
    }
    float denominator_root, density_root;
    if (g.ax == g.ay) {
        const float radial = std::hypot(m.x, m.y);
        if (g.ax <= 1.0F) {
            denominator_root = std::hypot(radial, g.ax * m.z);
            density_root = (g.ax / denominator_root) / denominator_root;
        } else {
            const float inverse_alpha = 1.0F / g.ax;
            denominator_root = std::hypot(radial * inverse_alpha, m.z);
            density_root = (inverse_alpha / denominator_root) / denominator_root;
        }
        density_root *= std::sqrt(kInvPi);
    } else {
        denominator_root = std::hypot(m.x / g.ax, m.y / g.ay, m.z);
        const float normalization_root = std::sqrt(kInvPi) / (std::sqrt(g.ax) * std::sqrt(g.ay));
        density_root = (normalization_root / denominator_root) / denominator_root;
    }
    const float value = density_root * density_root;
    if (!std::isfinite(denominator_root) || !(denominator_root > 0.0F) || !std::isfinite(value) ||
        !(value > 0.0F)) {
        fail("The GGX normal distribution value is not representable.");
    }
    return value;
}

// GgxMicrofacet.hpp:320-353 (smith_g2).
float ggx_g2(const Ggx& g, V3 wo, V3 wi) {
    if (!unit_length(wo) || !unit_length(wi)) {
        fail("GGX Smith directions must be finite unit vectors.");
    }
    if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
        return 0.0F;
    }
    const SmithTerms o = smith_terms(g, wo);
    const SmithTerms i = smith_terms(g, wi);
    const float smaller = std::min(o.normal_over_radius, i.normal_over_radius);
    const float larger = std::max(o.normal_over_radius, i.normal_over_radius);
    const float value = 2.0F * smaller / (1.0F + smaller / larger);
    if (!std::isfinite(value) || !(value > 0.0F) || value > 1.0F) {
        fail("GGX Smith G2 is not representable for the supplied directions.");
    }
    return value;
}

// GgxMicrofacet.hpp:355-388 (visible_normal_pdf).
float ggx_vndf_pdf(const Ggx& g, V3 wo, V3 m) {
    if (!unit_length(wo) || !unit_length(m)) {
        fail("GGX VNDF queries require finite unit directions and normals.");
    }
    const float visible_dot = dot(wo, m);
    if (!(wo.z > 0.0F) || !(m.z > 0.0F) || !(visible_dot > 0.0F)) {
        return 0.0F;
    }
    const float d = ggx_d(g, m);
    const float physical_radius = g.ax == g.ay
                                      ? std::hypot(wo.z, g.ax * std::hypot(wo.x, wo.y))
                                      : std::hypot(wo.z, g.ax * wo.x, g.ay * wo.y);
    const float physical_denominator = wo.z + physical_radius;
    const float visible_factor = 2.0F * visible_dot / physical_denominator;
    const float value = d * visible_factor;
    if (!std::isfinite(physical_denominator) || !(physical_denominator > 0.0F) ||
        !std::isfinite(value) || !(value > 0.0F)) {
        fail("The GGX visible-normal PDF is not representable.");
    }
    return value;
}

// GgxMicrofacet.hpp:71-103 (normalize_vector / normalize_normal).
V3 ggx_normalize(V3 v) {
    const float length = std::hypot(std::hypot(v.x, v.y), v.z);
    if (!std::isfinite(length) || !(length > 0.0F)) {
        fail("A GGX VNDF intermediate vector is not normalizable.");
    }
    const V3 r{v.x / length, v.y / length, v.z / length};
    if (!unit_length(r)) {
        fail("A GGX VNDF intermediate direction is not representable.");
    }
    return r;
}

float nonnegative_roundoff(float value, float scale) {  // GgxMicrofacet.hpp:186-197
    if (value >= 0.0F) {
        return value;
    }
    const float bound = kEpsilon * 16.0F * std::max(1.0F, std::abs(scale));
    if (-value <= bound) {
        return 0.0F;
    }
    fail("A GGX VNDF square-root argument is negative beyond round-off.");
}

// GgxMicrofacet.hpp:390-525 (sample_visible_normal). Returns false when wo.z <= 0.
bool ggx_sample_vndf(const Ggx& g, V3 wo, float u, float v, V3& m_out, float& pdf_out) {
    if (!unit_length(wo)) {
        fail("GGX VNDF sampling requires a finite unit outgoing direction.");
    }
    if (!(wo.z > 0.0F)) {
        return false;
    }
    const bool iso = g.ax == g.ay;
    const float inverse_alpha = 1.0F / g.ax;
    const float common = std::max({1.0F, g.ax, g.ay});
    const float sax = g.ax / common, say = g.ay / common;
    V3 st;
    if (iso) {
        st = g.ax <= 1.0F ? V3{g.ax * wo.x, g.ax * wo.y, wo.z}
                          : V3{wo.x, wo.y, wo.z * inverse_alpha};
    } else {
        st = V3{sax * wo.x, say * wo.y, wo.z / common};
    }
    if ((iso && g.ax <= 1.0F && ((wo.x != 0.0F && st.x == 0.0F) || (wo.y != 0.0F && st.y == 0.0F))) ||
        (iso && g.ax > 1.0F && st.z == 0.0F) ||
        (!iso && ((wo.x != 0.0F && st.x == 0.0F) || (wo.y != 0.0F && st.y == 0.0F) || st.z == 0.0F))) {
        fail("The GGX VNDF view stretch is not representable.");
    }
    const V3 hv = ggx_normalize(st);
    const float tl = std::hypot(hv.x, hv.y);
    const V3 tangent = tl > 0.0F ? V3{-hv.y / tl, hv.x / tl, 0.0F} : V3{1.0F, 0.0F, 0.0F};
    const V3 bitangent = cross(hv, tangent);
    const float disk_radius = std::sqrt(u);
    const float azimuth = 2.0F * kPi * v;
    const float disk_x = disk_radius * cos_f(azimuth);
    const float initial_disk_y = disk_radius * sin_f(azimuth);
    const float limit_sq = (1.0F - disk_x) * (1.0F + disk_x);
    const float checked_limit_sq = nonnegative_roundoff(limit_sq, 1.0F + std::abs(disk_x));
    const float disk_y_limit = std::sqrt(checked_limit_sq);
    const float projection = 0.5F * (1.0F + hv.z);
    const float disk_y = std::fma(projection, initial_disk_y, (1.0F - projection) * disk_y_limit);
    const float hz_sq = std::fma(-disk_y, disk_y, checked_limit_sq);
    const float checked_hz_sq = nonnegative_roundoff(hz_sq, checked_limit_sq + std::abs(disk_y * disk_y));
    const float hz = std::sqrt(checked_hz_sq);
    const V3 hn{std::fma(disk_x, tangent.x, std::fma(disk_y, bitangent.x, hz * hv.x)),
                std::fma(disk_x, tangent.y, std::fma(disk_y, bitangent.y, hz * hv.y)),
                std::fma(disk_x, tangent.z, std::fma(disk_y, bitangent.z, hz * hv.z))};
    if (!(hn.z > 0.0F)) {
        fail("The GGX VNDF hemisphere sample is outside its open support.");
    }
    V3 un;
    if (iso) {
        un = g.ax <= 1.0F ? V3{g.ax * hn.x, g.ax * hn.y, hn.z} : V3{hn.x, hn.y, hn.z * inverse_alpha};
    } else {
        un = V3{sax * hn.x, say * hn.y, hn.z / common};
    }
    if ((iso && g.ax <= 1.0F && ((hn.x != 0.0F && un.x == 0.0F) || (hn.y != 0.0F && un.y == 0.0F))) ||
        (iso && g.ax > 1.0F && un.z == 0.0F) ||
        (!iso && ((hn.x != 0.0F && un.x == 0.0F) || (hn.y != 0.0F && un.y == 0.0F) || un.z == 0.0F))) {
        fail("The GGX visible-normal unstretch is not representable.");
    }
    const V3 m = ggx_normalize(un);
    if (!(m.z > 0.0F) || !(dot(wo, m) > 0.0F)) {
        fail("The GGX VNDF sample is outside its visible support.");
    }
    m_out = m;
    pdf_out = ggx_vndf_pdf(g, wo, m);
    return true;
}

// Fresnel.hpp:27-104 (conductor, one lane).
float squared_magnitude_ratio(float nr, float ni, float dr, float di) {
    const float n = std::hypot(nr, ni);
    const float d = std::hypot(dr, di);
    if (!std::isfinite(n) || !std::isfinite(d) || !(d > 0.0F)) {
        fail("A conductor Fresnel polarization ratio is not representable.");
    }
    const float amplitude = n / d;
    const float r = amplitude * amplitude;
    if (!std::isfinite(r) || r < 0.0F || r > 1.0F) {
        fail("A conductor Fresnel polarization ratio is not representable.");
    }
    return r;
}

float conductor_fresnel_lane(float cosine, float eta, float k) {
    if (eta == 1.0F && k == 0.0F) {
        return 0.0F;
    }
    if (cosine == 0.0F) {
        return 1.0F;
    }
    const float scale = std::max({1.0F, eta, k});
    const float nie = 1.0F / scale;
    const float ne = eta / scale;
    const float nk = k / scale;
    if (cosine == 1.0F) {
        const float r = squared_magnitude_ratio(ne - nie, nk, ne + nie, nk);
        if (!(r > 0.0F)) {
            fail("Conductor Fresnel reflectance is not representable.");
        }
        return r;
    }
    const float sin_sq = (1.0F - cosine) * (1.0F + cosine);
    const float scaled_sin_sq = nie * nie * sin_sq;
    const float x = std::fma(ne, ne, -std::fma(nk, nk, scaled_sin_sq));
    const float y = 2.0F * ne * nk;
    const float magnitude = std::hypot(x, y);
    float rr, ri;
    if (x >= 0.0F) {
        rr = std::sqrt(0.5F * (magnitude + x));
        ri = rr == 0.0F ? 0.0F : y / (2.0F * rr);
    } else {
        ri = std::sqrt(0.5F * (magnitude - x));
        rr = ri == 0.0F ? 0.0F : y / (2.0F * ri);
    }
    const float sc = nie * cosine;
    const float perpendicular = squared_magnitude_ratio(sc - rr, -ri, sc + rr, ri);
    const float ser = std::fma(ne, ne, -(nk * nk));
    const float sei = y;
    const float srr = nie * rr;
    const float sri = nie * ri;
    const float pbr = cosine * ser;
    const float pbi = cosine * sei;
    const float parallel = squared_magnitude_ratio(pbr - srr, pbi - sri, pbr + srr, pbi + sri);
    const float r = 0.5F * (perpendicular + parallel);
    if (!std::isfinite(r) || !(r > 0.0F) || r > 1.0F) {
        fail("Conductor Fresnel reflectance is not representable.");
    }
    return r;
}

// Fresnel.hpp:107-170 (dielectric).
float dielectric_fresnel(float cosine, float eta_i, float eta_t) {
    if (!std::isfinite(cosine) || cosine < 0.0F || cosine > 1.0F) {
        fail("Dielectric Fresnel requires an incident-cosine magnitude in [0, 1].");
    }
    if (eta_i == eta_t) {
        return 0.0F;
    }
    if (cosine == 0.0F) {
        return 1.0F;
    }
    const bool denser = eta_i > eta_t;
    const float ne = denser ? eta_t / eta_i : eta_i / eta_t;
    if (cosine == 1.0F) {
        const float a = (1.0F - ne) / (1.0F + ne);
        const float r = a * a;
        if (!std::isfinite(r) || !(r > 0.0F) || r > 1.0F) {
            fail("Dielectric Fresnel reflectance is not representable.");
        }
        return r;
    }
    const float sin_i = std::sqrt((1.0F - cosine) * (1.0F + cosine));
    float sin_t;
    if (denser) {
        if (ne == 0.0F || sin_i >= ne) {
            return 1.0F;
        }
        sin_t = sin_i / ne;
    } else {
        sin_t = ne * sin_i;
    }
    if (!(sin_t < 1.0F)) {
        return 1.0F;
    }
    const float cos_t = std::sqrt((1.0F - sin_t) * (1.0F + sin_t));
    const float fec = ne * cos_t;
    const float fa = (cosine - fec) / (cosine + fec);
    const float sec = ne * cosine;
    const float sa = (sec - cos_t) / (sec + cos_t);
    const float r = 0.5F * std::fma(fa, fa, sa * sa);
    if (!std::isfinite(r) || !(r > 0.0F) || r > 1.0F) {
        fail("Dielectric Fresnel reflectance is not representable.");
    }
    return r;
}

// RoughConductorReflection.hpp:68-106 (reflection_geometry: half vector and its cosine).
void half_vector_geometry(V3 wo, V3 wi, V3& m, float& half_cos) {
    const V3 h{wo.x + wi.x, wo.y + wi.y, wo.z + wi.z};
    const float length = std::hypot(std::hypot(h.x, h.y), h.z);
    if (!std::isfinite(length) || !(length > 0.0F)) {
        fail("The reflection half-vector is not normalizable.");
    }
    m = V3{h.x / length, h.y / length, h.z / length};
    if (!unit_length(m) || !(m.z > 0.0F)) {
        fail("The reflection half-vector is not representable.");
    }
    half_cos = 0.5F * length;
    if (!std::isfinite(half_cos) || !(half_cos > 0.0F) || half_cos > 1.0F) {
        fail("The reflection half-angle cosine is outside [0, 1].");
    }
}

// RoughConductorReflection.hpp:167-209 (eval).
Spectrum conductor_eval(const Closure& c, V3 wo, V3 wi) {
    Spectrum r{};
    if (!unit_length(wo) || !unit_length(wi)) {
        fail("Rough-conductor directions must be finite unit vectors.");
    }
    if (!(wo.z > 0.0F) || !(wi.z > 0.0F) || is_black(c.weight)) {
        return r;
    }
    const Ggx g{c.p[8], c.p[9]};
    V3 m;
    float hc;
    half_vector_geometry(wo, wi, m, hc);
    const float d = ggx_d(g, m);
    const float g2 = ggx_g2(g, wo, wi);
    float fresnel[4];
    for (int lane = 0; lane < 4; ++lane) {
        fresnel[lane] = conductor_fresnel_lane(hc, c.p[lane], c.p[4 + lane]);
    }
    const float denominator = 4.0F * wo.z * wi.z;
    const float scale = (d * g2) / denominator;
    if (!std::isfinite(denominator) || !(denominator > 0.0F) || !std::isfinite(scale) ||
        !(scale > 0.0F)) {
        fail("The rough-conductor GGX reflection value is not representable.");
    }
    for (int lane = 0; lane < 4; ++lane) {
        r[lane] = c.weight[lane] * fresnel[lane] * scale;
    }
    return r;
}

// RoughConductorReflection.hpp:211-238 (pdf).
float conductor_pdf(const Closure& c, V3 wo, V3 wi) {
    if (!unit_length(wo) || !unit_length(wi)) {
        fail("Rough-conductor directions must be finite unit vectors.");
    }
    if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
        return 0.0F;
    }
    V3 m;
    float hc;
    half_vector_geometry(wo, wi, m, hc);
    const float visible = ggx_vndf_pdf(Ggx{c.p[8], c.p[9]}, wo, m);
    const float value = visible / (4.0F * hc);
    if (!std::isfinite(value) || !(value > 0.0F)) {
        fail("The rough-conductor reflected-direction PDF is not representable.");
    }
    return value;
}

// RoughConductorReflection.hpp:240-288 (sample).
BsdfSample conductor_sample(const Closure& c, V3 wo, float u, float v) {
    BsdfSample s;
    V3 m;
    float vpdf;
    if (!ggx_sample_vndf(Ggx{c.p[8], c.p[9]}, wo, u, v, m, vpdf)) {
        return s;
    }
    const float hc = dot(wo, m);
    if (!std::isfinite(hc) || !(hc > 0.0F) || hc > 1.0F) {
        fail("The sampled rough-conductor half-angle cosine is outside [0, 1].");
    }
    const V3 wi{2.0F * hc * m.x - wo.x, 2.0F * hc * m.y - wo.y, 2.0F * hc * m.z - wo.z};
    if (!unit_length(wi)) {
        fail("The sampled rough-conductor reflection direction is not representable.");
    }
    if (!(wi.z > 0.0F)) {
        return s;
    }
    s.wi = wi;
    s.value = conductor_eval(c, wo, wi);
    s.pdf = conductor_pdf(c, wo, wi);
    s.lobes = c.lobes;
    s.valid = true;
    return s;
}

// RoughDielectric.hpp:114-134 (interface_for).
struct Interface {
    float face_sign, incident_eta, transmitted_eta, nie, nte;
};
Interface interface_for(V3 wo, float ext, float in) {
    Interface f;
    f.face_sign = wo.z > 0.0F ? 1.0F : -1.0F;
    f.incident_eta = f.face_sign > 0.0F ? ext : in;
    f.transmitted_eta = f.face_sign > 0.0F ? in : ext;
    const float mx = std::max(f.incident_eta, f.transmitted_eta);
    f.nie = f.incident_eta / mx;
    f.nte = f.transmitted_eta / mx;
    return f;
}

V3 scaled_dir(V3 d, float s) { return {s * d.x, s * d.y, s * d.z}; }

struct TransmissionGeometry {
    bool valid;
    V3 m;
    float o_dot_m, i_dot_m, length;
};

// RoughDielectric.hpp:172-223 (transmission_geometry).
TransmissionGeometry transmission_geometry(V3 of, V3 inf, const Interface& f) {
    TransmissionGeometry g{};
    V3 h{std::fma(f.nie, of.x, f.nte * inf.x), std::fma(f.nie, of.y, f.nte * inf.y),
         std::fma(f.nie, of.z, f.nte * inf.z)};
    const float length = std::hypot(std::hypot(h.x, h.y), h.z);
    if (!std::isfinite(length) || !(length > 0.0F)) {
        fail("The rough-dielectric transmission half-vector is not normalizable.");
    }
    h = scaled_dir(h, 1.0F / length);
    if (h.z < 0.0F) {
        h = scaled_dir(h, -1.0F);
    }
    if (h.z == 0.0F) {
        return g;
    }
    if (!unit_length(h)) {
        fail("The rough-dielectric transmission half-vector is not representable.");
    }
    const float od = dot(of, h);
    const float id = dot(inf, h);
    if (!std::isfinite(od) || !std::isfinite(id)) {
        fail("The rough-dielectric transmission half-angle cosines are not representable.");
    }
    if (!(od > 0.0F) || !(id < 0.0F)) {
        return g;
    }
    if (od > 1.0F || id < -1.0F) {
        fail("The rough-dielectric transmission half-angle cosines are outside [-1, 1].");
    }
    g.valid = true;
    g.m = h;
    g.o_dot_m = od;
    g.i_dot_m = id;
    g.length = length;
    return g;
}

Spectrum scale_spectrum(const Spectrum& c, float scale) {  // RoughDielectric.hpp:88-103
    Spectrum r{};
    for (int lane = 0; lane < 4; ++lane) {
        const float num[2] = {c[lane], scale};
        const float den[1] = {1.0F};
        r[lane] = checked_product_ratio(num, 2, den, 1);
    }
    return r;
}

// RoughDielectric.hpp:299-381 (eval, radiance mode).
Spectrum dielectric_eval(const Closure& c, V3 wo, V3 wi) {
    Spectrum r{};
    if (!unit_length(wo) || !unit_length(wi)) {
        fail("Rough-dielectric directions must be finite unit vectors.");
    }
    if (wo.z == 0.0F || wi.z == 0.0F) {
        return r;
    }
    const Ggx g{c.p[2], c.p[3]};
    const Interface f = interface_for(wo, c.p[0], c.p[1]);
    const V3 of = scaled_dir(wo, f.face_sign);
    const V3 inf = scaled_dir(wi, f.face_sign);
    if (inf.z > 0.0F) {
        V3 m;
        float od;
        half_vector_geometry(of, inf, m, od);
        const float fr = dielectric_fresnel(od, f.incident_eta, f.transmitted_eta);
        const float d = ggx_d(g, m);
        const float g2 = ggx_g2(g, of, inf);
        const float num[3] = {fr, d, g2};
        const float den[3] = {4.0F, of.z, inf.z};
        return scale_spectrum(c.weight, checked_product_ratio(num, 3, den, 3));
    }
    const TransmissionGeometry tg = transmission_geometry(of, inf, f);
    if (!tg.valid) {
        return r;
    }
    const float fr = dielectric_fresnel(tg.o_dot_m, f.incident_eta, f.transmitted_eta);
    if (fr == 1.0F) {
        return r;
    }
    if (!(tg.length > 0.0F)) {
        fail("The rough-dielectric transmission Jacobian denominator is zero.");
    }
    const float d = ggx_d(g, tg.m);
    const float g2 = ggx_g2(g, of, scaled_dir(inf, -1.0F));
    const float eta = f.nie;  // radiance mode
    const float num[7] = {1.0F - fr, d, g2, eta, eta, tg.o_dot_m, -tg.i_dot_m};
    const float den[4] = {of.z, -inf.z, tg.length, tg.length};
    return scale_spectrum(c.weight, checked_product_ratio(num, 7, den, 4));
}

// RoughDielectric.hpp:383-467 (pdf).
float dielectric_pdf(const Closure& c, V3 wo, V3 wi) {
    if (!unit_length(wo) || !unit_length(wi)) {
        fail("Rough-dielectric directions must be finite unit vectors.");
    }
    if (wo.z == 0.0F || wi.z == 0.0F) {
        return 0.0F;
    }
    const Ggx g{c.p[2], c.p[3]};
    const Interface f = interface_for(wo, c.p[0], c.p[1]);
    const V3 of = scaled_dir(wo, f.face_sign);
    const V3 inf = scaled_dir(wi, f.face_sign);
    if (inf.z > 0.0F) {
        V3 m;
        float od;
        half_vector_geometry(of, inf, m, od);
        const float fr = dielectric_fresnel(od, f.incident_eta, f.transmitted_eta);
        const float visible = ggx_vndf_pdf(g, of, m);
        const float num[2] = {fr, visible};
        const float den[2] = {4.0F, od};
        return checked_product_ratio(num, 2, den, 2);
    }
    const TransmissionGeometry tg = transmission_geometry(of, inf, f);
    if (!tg.valid) {
        return 0.0F;
    }
    const float fr = dielectric_fresnel(tg.o_dot_m, f.incident_eta, f.transmitted_eta);
    if (fr == 1.0F) {
        return 0.0F;
    }
    if (!(tg.length > 0.0F)) {
        fail("The rough-dielectric transmission Jacobian denominator is zero.");
    }
    const float visible = ggx_vndf_pdf(g, of, tg.m);
    const float num[5] = {1.0F - fr, visible, f.nte, f.nte, -tg.i_dot_m};
    const float den[2] = {tg.length, tg.length};
    return checked_product_ratio(num, 5, den, 2);
}

// RoughDielectric.hpp:469-632 (sample, radiance mode).
BsdfSample dielectric_sample(const Closure& c, V3 wo, float event, float u, float v) {
    BsdfSample s;
    if (!unit_length(wo)) {
        fail("Rough-dielectric directions must be finite unit vectors.");
    }
    if (!(event >= 0.0F && event < 1.0F)) {
        fail("Rough-dielectric event selection requires a finite sample in [0, 1).");
    }
    if (wo.z == 0.0F) {
        return s;
    }
    const Ggx g{c.p[2], c.p[3]};
    const Interface f = interface_for(wo, c.p[0], c.p[1]);
    const V3 of = scaled_dir(wo, f.face_sign);
    V3 m;
    float vpdf;
    if (!ggx_sample_vndf(g, of, u, v, m, vpdf)) {
        return s;
    }
    const float od = dot(of, m);
    if (!std::isfinite(od) || !(od > 0.0F) || od > 1.0F) {
        fail("The sampled rough-dielectric half-angle cosine is outside [0, 1].");
    }
    const float fr = dielectric_fresnel(od, f.incident_eta, f.transmitted_eta);
    V3 inf;
    uint32_t lobes;
    float eta_scale = 1.0F;
    if (event < fr) {
        inf = V3{2.0F * od * m.x - of.x, 2.0F * od * m.y - of.y, 2.0F * od * m.z - of.z};
        lobes = BF200_LOBE_GLOSSY | BF200_LOBE_REFLECTION;
        if (!unit_length(inf)) {
            fail("The sampled rough-dielectric reflection direction is not representable.");
        }
        if (!(inf.z > 0.0F)) {
            return s;
        }
    } else {
        const V3 tangent{of.x - od * m.x, of.y - od * m.y, of.z - od * m.z};
        const float incident_sine = std::hypot(std::hypot(tangent.x, tangent.y), tangent.z);
        if (!std::isfinite(incident_sine) || incident_sine > 1.0F) {
            fail("The sampled rough-dielectric incident sine is not representable.");
        }
        float incoming_cosine = 1.0F, tangent_scale = 0.0F;
        if (incident_sine > 0.0F) {
            float transmitted_sine;
            if (f.incident_eta > f.transmitted_eta) {
                const float critical = f.transmitted_eta / f.incident_eta;
                if (critical == 0.0F || incident_sine >= critical) {
                    fail("Fresnel selected transmission at total internal reflection.");
                }
                transmitted_sine = incident_sine / critical;
            } else {
                const float ratio = f.incident_eta / f.transmitted_eta;
                if (ratio == 0.0F) {
                    fail("The rough-dielectric refraction ratio is not representable.");
                }
                transmitted_sine = ratio * incident_sine;
            }
            if (!std::isfinite(transmitted_sine) || !(transmitted_sine < 1.0F)) {
                fail("A subcritical rough-dielectric transmission sine is not representable.");
            }
            incoming_cosine = std::sqrt((1.0F - transmitted_sine) * (1.0F + transmitted_sine));
            tangent_scale = transmitted_sine / incident_sine;
            if (!std::isfinite(incoming_cosine) || !(incoming_cosine > 0.0F) ||
                !std::isfinite(tangent_scale) || !(tangent_scale > 0.0F)) {
                fail("The sampled rough-dielectric transmission direction is not representable.");
            }
        }
        inf = V3{std::fma(-tangent_scale, tangent.x, -incoming_cosine * m.x),
                 std::fma(-tangent_scale, tangent.y, -incoming_cosine * m.y),
                 std::fma(-tangent_scale, tangent.z, -incoming_cosine * m.z)};
        lobes = BF200_LOBE_GLOSSY | BF200_LOBE_TRANSMISSION;
        if (!unit_length(inf)) {
            fail("The sampled rough-dielectric transmission direction is not a unit vector.");
        }
        if (!(inf.z < 0.0F)) {
            return s;
        }
        const float num[2] = {f.nte, f.nte};
        const float den[2] = {f.nie, f.nie};
        eta_scale = checked_product_ratio(num, 2, den, 2);
    }
    const V3 wi = scaled_dir(inf, f.face_sign);
    s.wi = wi;
    s.value = dielectric_eval(c, wo, wi);
    s.pdf = dielectric_pdf(c, wo, wi);
    s.lobes = lobes;
    s.eta_scale = eta_scale;
    s.valid = true;
    return s;
}

// DepthFilteredClosureMixture.hpp:48-133: a dielectric restricted to one direction has the
// branch-conditional pdf base / P(branch).
float dielectric_pdf_masked(const Closure& c, uint32_t allowed, V3 wo, V3 wi) {
    const float base = dielectric_pdf(c, wo, wi);
    if (wo.z == 0.0F || wi.z == 0.0F || base == 0.0F) {
        return base;
    }
    const bool reflection = (wo.z > 0.0F) == (wi.z > 0.0F);
    const uint32_t direction = reflection ? BF200_LOBE_REFLECTION : BF200_LOBE_TRANSMISSION;
    if ((allowed & direction) == 0U) {
        return 0.0F;
    }
    if (allowed == (BF200_LOBE_REFLECTION | BF200_LOBE_TRANSMISSION)) {
        return base;
    }
    const Interface f = interface_for(wo, c.p[0], c.p[1]);
    const V3 of = scaled_dir(wo, f.face_sign);
    const V3 inf = scaled_dir(wi, f.face_sign);
    float branch;
    if (reflection) {
        V3 m;
        float od;
        half_vector_geometry(of, inf, m, od);
        branch = dielectric_fresnel(od, f.incident_eta, f.transmitted_eta);
    } else {
        const TransmissionGeometry tg = transmission_geometry(of, inf, f);
        if (!tg.valid) {
            return 0.0F;
        }
        branch = 1.0F - dielectric_fresnel(tg.o_dot_m, f.incident_eta, f.transmitted_eta);
    }
    if (!std::isfinite(branch) || !(branch > 0.0F) || branch > 1.0F) {
        fail("A filtered rough-dielectric branch probability is not representable.");
    }
    const float num[1] = {base};
    const float den[1] = {branch};
    return checked_product_ratio(num, 1, den, 1);
}

Spectrum dielectric_eval_masked(const Closure& c, uint32_t allowed, V3 wo, V3 wi) {
    const Spectrum value = dielectric_eval(c, wo, wi);
    if (wo.z == 0.0F || wi.z == 0.0F) {
        return value;
    }
    const uint32_t direction =
        (wo.z > 0.0F) == (wi.z > 0.0F) ? BF200_LOBE_REFLECTION : BF200_LOBE_TRANSMISSION;
    return (allowed & direction) != 0U ? value : Spectrum{};
}

// ---------------------------------------------------------------------------------------------
// Depth limits (PathDepthLimits.cpp) and the single-closure depth filter
// ---------------------------------------------------------------------------------------------

struct Depth {
    uint32_t c[5];  // diffuse, glossy, specular, transmission, volume
    uint32_t total() const { return c[0] + c[1] + c[2] + c[4]; }
};


// ---------------------------------------------------------------------------------------------
// Energy-preserving Oren-Nayar rough diffuse reflection (RoughDiffuseReflection.hpp:62-283)
// ---------------------------------------------------------------------------------------------

constexpr float kFonCoefficient = 0.5F - 2.0F * kInvPi / 3.0F;
constexpr float kFonAverageCoefficient = 2.0F / 3.0F - 28.0F * kInvPi / 15.0F;
constexpr float kFonAverageLossCoefficient = kFonCoefficient - kFonAverageCoefficient;

// directional_loss_shape: 1 - E_FON for unit albedo without the factor A_F * r.
float eon_loss_shape(V3 d) {
    const float sine = std::hypot(d.x, d.y);
    const float cosine = d.z;
    const float angle = atan2_f(sine, cosine);
    const float stable_ratio = sine * cosine * (1.0F + sine + sine * sine) / (1.0F + sine);
    const float g = sine * (angle - sine * cosine) + (2.0F / 3.0F) * (stable_ratio - sine);
    const float loss = kFonCoefficient - g * kInvPi;
    if (!std::isfinite(loss) || loss < 0.0F) {
        fail("The rough-diffuse directional albedo is not representable for the supplied direction.");
    }
    return loss;
}

Spectrum eon_eval(const Closure& c, V3 wo, V3 wi) {
    if (!unit_length(wo) || !unit_length(wi)) {
        fail("Rough-diffuse directions must be finite unit vectors.");
    }
    if (!(wo.z > 0.0F) || !(wi.z > 0.0F) || is_black(c.weight)) {
        return Spectrum{};
    }
    const float r = c.p[0];
    if (r == 0.0F) {
        return Spectrum{c.weight[0] * kInvPi, c.weight[1] * kInvPi, c.weight[2] * kInvPi, c.weight[3] * kInvPi};
    }
    const float tangent_dot = std::fma(wo.x, wi.x, wo.y * wi.y);
    const float s_over_t = tangent_dot > 0.0F ? tangent_dot / std::max(wo.z, wi.z) : tangent_dot;
    const float a = 1.0F / (1.0F + kFonCoefficient * r);
    const float single = kInvPi * a * (1.0F + r * s_over_t);
    if (!std::isfinite(single) || single < 0.0F) {
        fail("The rough-diffuse single-scattering value is not representable.");
    }
    const float outgoing_loss = eon_loss_shape(wo);
    const float incoming_loss = eon_loss_shape(wi);
    const float average = a * (1.0F + kFonAverageCoefficient * r);
    const float loss_over_average = a * r * incoming_loss * outgoing_loss / kFonAverageLossCoefficient;
    if (!std::isfinite(average) || !(average > 0.0F) || average > 1.0F || !std::isfinite(loss_over_average) ||
        loss_over_average < 0.0F) {
        fail("The rough-diffuse energy compensation is not representable.");
    }
    Spectrum out{};
    for (int lane = 0; lane < 4; ++lane) {
        const float rho = c.weight[lane];
        const float den = (1.0F - rho) + rho * average;
        if (!std::isfinite(den) || !(den > 0.0F)) {
            fail("The rough-diffuse multiple-scattering albedo is not representable.");
        }
        const float ms = rho * rho * average / den;
        const float value = rho * single + ms * kInvPi * loss_over_average;
        if (!std::isfinite(value) || value < 0.0F) {
            fail("The rough-diffuse BRDF value is not representable.");
        }
        out[lane] = value;
    }
    return out;
}

float cosine_pdf(V3 wo, V3 wi, const char* message) {  // Lambertian / rough-diffuse pdf
    if (!unit_length(wo) || !unit_length(wi)) {
        fail(message);
    }
    if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
        return 0.0F;
    }
    const float v = wi.z * kInvPi;
    if (!(v > 0.0F) || !std::isfinite(v)) {
        fail("A diffuse PDF is not representable for the supplied direction.");
    }
    return v;
}

// ---------------------------------------------------------------------------------------------
// Ideal specular reflection and transmission (SpecularDelta.hpp:85-495). Directional eval/pdf
// queries exclude the Dirac atom (zero value, zero solid-angle density); only sample() exposes
// the discrete mass.
// ---------------------------------------------------------------------------------------------

float delta_product_quotient(float left, float right, float den) {  // checked_positive_product_quotient
    if (left == 0.0F) {
        return 0.0F;
    }
    if (!std::isfinite(left) || !(left > 0.0F) || !std::isfinite(right) || !(right > 0.0F) ||
        !std::isfinite(den) || !(den > 0.0F)) {
        fail("A specular delta value is not representable in the requested precision.");
    }
    int le = 0, re = 0, de = 0, ne = 0;
    const float ls = std::frexp(left, &le), rs = std::frexp(right, &re), ds = std::frexp(den, &de);
    const float normalized = std::frexp((ls * rs) / ds, &ne);
    const float result = std::scalbn(normalized, le + re - de + ne);
    if (!std::isfinite(result) || !(result > 0.0F)) {
        fail("A specular delta value is not representable in the requested precision.");
    }
    return result;
}

float delta_squared_ratio(float num, float den) {  // checked_squared_ratio
    if (!std::isfinite(num) || !(num > 0.0F) || !std::isfinite(den) || !(den > 0.0F)) {
        fail("A specular transmission factor is not representable.");
    }
    int ne = 0, de = 0, re = 0;
    const float ns = std::frexp(num, &ne), ds = std::frexp(den, &de);
    const float ratio = ns / ds;
    const float normalized = std::frexp(ratio * ratio, &re);
    const float result = std::scalbn(normalized, 2 * (ne - de) + re);
    if (!std::isfinite(result) || !(result > 0.0F)) {
        fail("A specular transmission factor is not representable.");
    }
    return result;
}

BsdfSample specular_reflection_sample(const Closure& c, V3 wo) {
    BsdfSample s;
    if (!unit_length(wo)) {
        fail("Specular delta directions must be finite unit vectors.");
    }
    if (wo.z == 0.0F) {
        return s;
    }
    s.wi = V3{-wo.x, -wo.y, wo.z};
    for (int lane = 0; lane < 4; ++lane) {
        s.value[lane] = delta_product_quotient(c.weight[lane], 1.0F, std::abs(s.wi.z));
    }
    s.pdf = 1.0F;
    s.delta = true;
    s.lobes = BF200_LOBE_SPECULAR | BF200_LOBE_REFLECTION;
    s.valid = true;
    return s;
}

BsdfSample specular_transmission_sample(const Closure& c, V3 wo) {
    BsdfSample s;
    if (!unit_length(wo)) {
        fail("Specular delta directions must be finite unit vectors.");
    }
    if (wo.z == 0.0F) {
        return s;
    }
    const bool entering = wo.z > 0.0F;
    const float incident = entering ? c.p[0] : c.p[1];
    const float transmitted = entering ? c.p[1] : c.p[0];
    s.lobes = BF200_LOBE_SPECULAR | BF200_LOBE_TRANSMISSION;
    s.delta = true;
    s.pdf = 1.0F;
    if (incident == transmitted) {
        s.wi = V3{-wo.x, -wo.y, -wo.z};
        for (int lane = 0; lane < 4; ++lane) {
            s.value[lane] = delta_product_quotient(c.weight[lane], 1.0F, std::abs(s.wi.z));
        }
        s.valid = true;
        return s;
    }
    const float raw_sine = std::hypot(wo.x, wo.y);
    if (!std::isfinite(raw_sine)) {
        fail("The specular transmission incident sine is not representable.");
    }
    float sine = raw_sine, normalization = 1.0F;
    if (raw_sine > 1.0F) {
        const float cosine = std::abs(wo.z);
        if (cosine > 1.0F) {
            fail("The specular transmission incident direction is inconsistent.");
        }
        sine = std::sqrt((1.0F - cosine) * (1.0F + cosine));
        normalization = sine / raw_sine;
        if (!std::isfinite(sine) || !std::isfinite(normalization) || !(normalization > 0.0F)) {
            fail("The specular transmission incident sine is not representable.");
        }
    }
    if (sine > 0.0F) {
        const float critical = transmitted / incident;
        if (critical <= 1.0F && sine >= critical) {
            return BsdfSample{};
        }
    }
    const float ratio = incident / transmitted;
    if (!std::isfinite(ratio) || !(ratio > 0.0F)) {
        fail("The specular transmission relative index is not representable.");
    }
    const float ix = -ratio * normalization * wo.x;
    const float iy = -ratio * normalization * wo.y;
    if (!std::isfinite(ix) || !std::isfinite(iy) || (wo.x != 0.0F && ix == 0.0F) || (wo.y != 0.0F && iy == 0.0F)) {
        fail("The specular transmission tangent is not representable.");
    }
    const float transmitted_sine = std::hypot(ix, iy);
    if (!std::isfinite(transmitted_sine)) {
        fail("The specular transmission sine is not representable.");
    }
    if (transmitted_sine >= 1.0F) {
        fail("A subcritical specular transmission direction is not representable.");
    }
    const float transmitted_cosine = std::sqrt((1.0F - transmitted_sine) * (1.0F + transmitted_sine));
    if (!std::isfinite(transmitted_cosine) || !(transmitted_cosine > 0.0F)) {
        fail("The specular transmission cosine is not representable.");
    }
    s.wi = V3{ix, iy, entering ? -transmitted_cosine : transmitted_cosine};
    if (!unit_length(s.wi)) {
        fail("The refracted specular direction is not a representable unit vector.");
    }
    const float adjoint = delta_squared_ratio(incident, transmitted);  // radiance mode
    s.eta_scale = delta_squared_ratio(transmitted, incident);
    for (int lane = 0; lane < 4; ++lane) {
        s.value[lane] = delta_product_quotient(c.weight[lane], adjoint, transmitted_cosine);
    }
    s.valid = true;
    return s;
}

// ---------------------------------------------------------------------------------------------
// Depth limits (PathDepthLimits.cpp) and the depth-filtered closure mixture
// (DepthFilteredClosureMixture.hpp:254-552, ClosureMixture.hpp:79-334, 760-876)
// ---------------------------------------------------------------------------------------------

bool valid_surface_event(uint32_t lobes) {  // TransportConventions.hpp:101-109
    const uint32_t family = lobes & (BF200_LOBE_DIFFUSE | BF200_LOBE_GLOSSY | BF200_LOBE_SPECULAR);
    const uint32_t direction = lobes & (BF200_LOBE_REFLECTION | BF200_LOBE_TRANSMISSION);
    return lobes != 0U && (lobes & ~0x3FU) == 0U && (lobes & BF200_LOBE_VOLUME) == 0U &&
           (family == BF200_LOBE_DIFFUSE || family == BF200_LOBE_GLOSSY || family == BF200_LOBE_SPECULAR) &&
           (direction == BF200_LOBE_REFLECTION || direction == BF200_LOBE_TRANSMISSION);
}

bool is_delta_kind(uint32_t kind) {
    return kind == BF200_CLOSURE_SPECULAR_REFLECTION || kind == BF200_CLOSURE_SPECULAR_TRANSMISSION;
}

// add_compensated (ClosureMixture.hpp:78-99): a Neumaier step over non-negative values.
bool add_compensated(float value, float& sum, float& correction) {
    if (!std::isfinite(value) || value < 0.0F) {
        return false;
    }
    const float next = sum + value;
    if (!std::isfinite(next)) {
        return false;
    }
    if (sum >= value) {
        correction += (sum - next) + value;
    } else {
        correction += (value - next) + sum;
    }
    if (!std::isfinite(correction)) {
        return false;
    }
    sum = next;
    return true;
}

float compensated_sum(const float* values, uint32_t n) {  // ClosureMixture.hpp:105-120
    float sum = 0.0F, correction = 0.0F;
    for (uint32_t i = 0; i < n; ++i) {
        if (!add_compensated(values[i], sum, correction)) {
            fail("Closure-mixture probability accumulation is not representable.");
        }
    }
    const float total = sum + correction;
    if (!std::isfinite(total) || total < 0.0F) {
        fail("Closure-mixture probability accumulation is not representable.");
    }
    return total == 0.0F ? 0.0F : total;
}

// build_component_distribution (ClosureMixture.hpp:122-234): the probabilities projected onto the
// 2^-24 sampler grid (largest remainders first) and their CDF. Returns false with `error` set
// instead of failing, so scene creation can report it.
bool component_distribution(const float* probabilities, uint32_t n, bool allow_empty, float* out_p, float* out_cdf,
                            const char** error) {
    for (uint32_t i = 0; i <= kMaxClosures; ++i) {
        out_cdf[i] = 0.0F;
        if (i < kMaxClosures) {
            out_p[i] = 0.0F;
        }
    }
    if (n > kMaxClosures) {
        *error = "Closure-mixture probabilities must match the active closure count.";
        return false;
    }
    if (n == 0U) {
        if (!allow_empty) {
            *error = "A probability mixture requires at least one component.";
        }
        return allow_empty;
    }
    if (n == 1U) {
        if (probabilities[0] != 1.0F) {
            *error = "A singleton closure mixture requires probability one.";
            return false;
        }
        out_p[0] = 1.0F;
        out_cdf[1] = 1.0F;
        return true;
    }
    for (uint32_t i = 0; i < n; ++i) {
        if (!std::isfinite(probabilities[i]) || !(probabilities[i] > 0.0F) || !(probabilities[i] < 1.0F)) {
            *error = "A multi-closure mixture requires finite probabilities strictly between zero and one.";
            return false;
        }
    }
    constexpr int digits = std::numeric_limits<float>::digits;
    constexpr uint64_t scale = uint64_t{1} << digits;
    uint64_t masses[kMaxClosures] = {};
    float remainders[kMaxClosures] = {};
    uint64_t base_mass = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const float scaled = std::ldexp(probabilities[i], digits);
        const float base = std::floor(scaled);
        if (!std::isfinite(scaled) || !(scaled > 0.0F) || base < 0.0F || base > static_cast<float>(scale)) {
            *error = "A closure-mixture probability cannot be projected onto the sampler grid.";
            return false;
        }
        masses[i] = static_cast<uint64_t>(base);
        remainders[i] = scaled - base;
        if (!std::isfinite(remainders[i]) || remainders[i] < 0.0F || remainders[i] >= 1.0F) {
            *error = "A closure-mixture probability cannot be projected onto the sampler grid.";
            return false;
        }
        base_mass += masses[i];
    }
    if (base_mass > scale) {
        *error = "Closure-mixture probabilities exceed one on the sampler grid.";
        return false;
    }
    float remainder_sum = 0.0F, remainder_correction = 0.0F;
    for (uint32_t i = 0; i < n; ++i) {
        if (!add_compensated(remainders[i], remainder_sum, remainder_correction)) {
            *error = "Closure-mixture probability accumulation is not representable.";
            return false;
        }
    }
    float remainder_total = remainder_sum + remainder_correction;
    if (!std::isfinite(remainder_total) || remainder_total < 0.0F) {
        *error = "Closure-mixture probability accumulation is not representable.";
        return false;
    }
    if (remainder_total == 0.0F) {
        remainder_total = 0.0F;
    }
    const uint64_t missing = scale - base_mass;
    if (missing > n) {
        *error = "Closure-mixture probabilities do not sum to one at sampler precision.";
        return false;
    }
    constexpr float tolerance = std::numeric_limits<float>::epsilon() * 16.0F;
    if (std::abs(remainder_total - static_cast<float>(missing)) > 0.5F + tolerance) {
        *error = "Closure-mixture probabilities do not round to one at sampler precision.";
        return false;
    }
    bool received[kMaxClosures] = {};
    for (uint64_t unit = 0; unit < missing; ++unit) {
        uint32_t selected = n;
        for (uint32_t i = 0; i < n; ++i) {
            if (received[i] || !(remainders[i] > 0.0F)) {
                continue;
            }
            if (selected == n || remainders[i] > remainders[selected]) {
                selected = i;
            }
        }
        if (selected == n) {
            *error = "Closure-mixture rounding cannot preserve every positive component.";
            return false;
        }
        ++masses[selected];
        received[selected] = true;
    }
    uint64_t cumulative = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (masses[i] == 0U || cumulative > scale - masses[i]) {
            *error = "A positive closure-mixture probability is not representable on the sampler grid.";
            return false;
        }
        cumulative += masses[i];
        out_p[i] = std::ldexp(static_cast<float>(masses[i]), -digits);
        out_cdf[i + 1] = std::ldexp(static_cast<float>(cumulative), -digits);
    }
    if (cumulative != scale || out_cdf[n] != 1.0F) {
        *error = "The closure-mixture CDF does not terminate at one.";
        return false;
    }
    return true;
}

// positive_probability_product (ClosureMixture.hpp:249-268)
float positive_probability_product(float selection, float conditional) {
    if (conditional == 0.0F) {
        return 0.0F;
    }
    int se = 0, ce = 0, ne = 0;
    const float ss = std::frexp(selection, &se), cs = std::frexp(conditional, &ce);
    const float normalized = std::frexp(ss * cs, &ne);
    const float product = std::scalbn(normalized, se + ce + ne);
    if (!std::isfinite(product) || !(product > 0.0F)) {
        fail("A positive weighted closure PDF is not representable in the requested precision.");
    }
    return product;
}

// mix_probability_densities (ClosureMixture.hpp:270-334) over solid-angle densities.
float mix_densities(const float* probabilities, const float* conditional, uint32_t n) {
    if (n == 0U) {
        fail("Closure PDF components require a non-empty matching sampling distribution.");
    }
    float maximum = 0.0F;
    for (uint32_t i = 0; i < n; ++i) {
        if (!std::isfinite(conditional[i]) || conditional[i] < 0.0F) {
            fail("Closure PDF components require finite non-negative solid-angle densities.");
        }
        maximum = std::max(maximum, conditional[i]);
    }
    if (n == 1U) {
        return conditional[0];
    }
    if (maximum == 0.0F) {
        return 0.0F;
    }
    float sum = 0.0F, correction = 0.0F;
    for (uint32_t i = 0; i < n; ++i) {
        const float density = conditional[i];
        const float ratio = density / maximum;
        if (density > 0.0F && (!std::isfinite(ratio) || !(ratio > 0.0F))) {
            fail("A positive normalized closure PDF is not representable in the requested precision.");
        }
        const float contribution = positive_probability_product(probabilities[i], ratio);
        if (!add_compensated(contribution, sum, correction)) {
            fail("The weighted closure PDF sum is not representable in the requested precision.");
        }
    }
    const float normalized = sum + correction;
    if (!std::isfinite(normalized) || !(normalized > 0.0F) || normalized > 1.0F) {
        fail("The normalized closure PDF sum is not representable in the requested precision.");
    }
    return positive_probability_product(normalized, maximum);
}

uint32_t blocked_limits(const uint32_t* limits, const Depth& d, uint32_t lobes) {
    uint32_t blocked = 0;
    if ((lobes & BF200_LOBE_DIFFUSE) && d.c[0] >= limits[0]) blocked |= BF200_LOBE_DIFFUSE;
    if ((lobes & BF200_LOBE_GLOSSY) && d.c[1] >= limits[1]) blocked |= BF200_LOBE_GLOSSY;
    if ((lobes & BF200_LOBE_SPECULAR) && d.c[2] >= limits[2]) blocked |= BF200_LOBE_SPECULAR;
    if ((lobes & BF200_LOBE_TRANSMISSION) && d.c[3] >= limits[3]) blocked |= BF200_LOBE_TRANSMISSION;
    if ((lobes & BF200_LOBE_VOLUME) && d.c[4] >= limits[4]) blocked |= BF200_LOBE_VOLUME;
    return blocked;
}

Depth advanced(const Depth& d, uint32_t lobes) {
    Depth r = d;
    if (lobes & BF200_LOBE_DIFFUSE) ++r.c[0];
    if (lobes & BF200_LOBE_GLOSSY) ++r.c[1];
    if (lobes & BF200_LOBE_SPECULAR) ++r.c[2];
    if (lobes & BF200_LOBE_TRANSMISSION) ++r.c[3];
    if (lobes & BF200_LOBE_VOLUME) ++r.c[4];
    return r;
}

// One material's closures after the depth filter: the active closures (source order), their
// allowed directions and their renormalised component distribution.
struct Mixture {
    uint32_t count = 0;
    uint32_t source[kMaxClosures] = {};
    uint32_t allowed[kMaxClosures] = {};
    float p[kMaxClosures] = {};
    float cdf[kMaxClosures + 1] = {};
    uint32_t blocked = 0;
    const Material* material = nullptr;
    const Closure& closure(uint32_t i) const { return material->closures[source[i]]; }
};

// DepthFilteredClosureMixture::create (DepthFilteredClosureMixture.hpp:262-364)
Mixture depth_filter(const Material& material, const uint32_t* limits, const Depth& d) {
    Mixture m;
    m.material = &material;
    for (uint32_t i = 0; i < material.closure_count; ++i) {
        const Closure& c = material.closures[i];
        uint32_t allowed = 0;
        auto consider = [&](uint32_t event, uint32_t direction) {
            const uint32_t b = blocked_limits(limits, d, event);
            if (b == 0U) {
                allowed |= direction;
            } else {
                m.blocked |= b;
            }
        };
        if (c.kind == BF200_CLOSURE_ROUGH_DIELECTRIC) {
            consider(BF200_LOBE_GLOSSY | BF200_LOBE_REFLECTION, BF200_LOBE_REFLECTION);
            consider(BF200_LOBE_GLOSSY | BF200_LOBE_TRANSMISSION, BF200_LOBE_TRANSMISSION);
        } else {
            if (!valid_surface_event(c.lobes)) {
                fail("A depth-filtered closure record requires a concrete surface event.");
            }
            consider(c.lobes, c.lobes & (BF200_LOBE_REFLECTION | BF200_LOBE_TRANSMISSION));
        }
        if (allowed == 0U) {
            continue;
        }
        m.source[m.count] = i;
        m.allowed[m.count] = allowed;
        m.p[m.count] = material.probability[i];
        ++m.count;
    }
    if (m.count == 0U) {
        return m;
    }
    if (m.count == material.closure_count) {
        for (uint32_t i = 0; i < m.count; ++i) {
            m.p[i] = material.probability[i];
        }
        for (uint32_t i = 0; i <= m.count; ++i) {
            m.cdf[i] = material.cdf[i];
        }
        return m;
    }
    if (m.count == 1U) {
        m.p[0] = 1.0F;
        m.cdf[0] = 0.0F;
        m.cdf[1] = 1.0F;
        return m;
    }
    const float total = compensated_sum(m.p, m.count);
    if (!std::isfinite(total) || !(total > 0.0F)) {
        fail("Active depth-filtered closure probabilities have no representable mass.");
    }
    float normalized[kMaxClosures] = {};
    for (uint32_t i = 0; i < m.count; ++i) {
        normalized[i] = m.p[i] / total;
    }
    const char* error = nullptr;
    if (!component_distribution(normalized, m.count, false, m.p, m.cdf, &error)) {
        fail(error);
    }
    return m;
}

// eval / pdf / sample of one closure record, the rough dielectric restricted to `allowed`
// (DepthFilteredClosureMixture.hpp:182-252, ClosureMixture.hpp:527-748)
Spectrum record_eval(const Closure& c, uint32_t allowed, V3 wo, V3 wi) {
    switch (c.kind) {
    case BF200_CLOSURE_LAMBERTIAN_REFLECTION: {  // LambertianReflection.hpp:76-85
        if (!unit_length(wo) || !unit_length(wi)) {
            fail("Lambertian directions must be finite unit vectors.");
        }
        if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
            return Spectrum{};
        }
        return Spectrum{c.weight[0] * kInvPi, c.weight[1] * kInvPi, c.weight[2] * kInvPi,
                        c.weight[3] * kInvPi};
    }
    case BF200_CLOSURE_ROUGH_DIFFUSE_REFLECTION:
        return eon_eval(c, wo, wi);
    case BF200_CLOSURE_ROUGH_CONDUCTOR_REFLECTION:
        return conductor_eval(c, wo, wi);
    case BF200_CLOSURE_ROUGH_DIELECTRIC:
        return dielectric_eval_masked(c, allowed, wo, wi);
    case BF200_CLOSURE_SPECULAR_REFLECTION:
    case BF200_CLOSURE_SPECULAR_TRANSMISSION:
        if (!unit_length(wo) || !unit_length(wi)) {
            fail("Specular delta directions must be finite unit vectors.");
        }
        return Spectrum{};
    default:
        fail("unsupported closure");
    }
}

float record_pdf(const Closure& c, uint32_t allowed, V3 wo, V3 wi) {
    switch (c.kind) {
    case BF200_CLOSURE_LAMBERTIAN_REFLECTION:  // LambertianReflection.hpp:87-106
        return cosine_pdf(wo, wi, "Lambertian directions must be finite unit vectors.");
    case BF200_CLOSURE_ROUGH_DIFFUSE_REFLECTION:
        return cosine_pdf(wo, wi, "Rough-diffuse directions must be finite unit vectors.");
    case BF200_CLOSURE_ROUGH_CONDUCTOR_REFLECTION:
        return conductor_pdf(c, wo, wi);
    case BF200_CLOSURE_ROUGH_DIELECTRIC:
        return dielectric_pdf_masked(c, allowed, wo, wi);
    case BF200_CLOSURE_SPECULAR_REFLECTION:
    case BF200_CLOSURE_SPECULAR_TRANSMISSION:
        if (!unit_length(wo) || !unit_length(wi)) {
            fail("Specular delta directions must be finite unit vectors.");
        }
        return 0.0F;
    default:
        fail("unsupported closure");
    }
}

BsdfSample record_sample(const Closure& c, uint32_t allowed, V3 wo, float event, float u, float v) {
    switch (c.kind) {
    case BF200_CLOSURE_LAMBERTIAN_REFLECTION:  // LambertianReflection.hpp:108-140
    case BF200_CLOSURE_ROUGH_DIFFUSE_REFLECTION: {  // RoughDiffuseReflection.hpp:235-266
        if (!unit_length(wo)) {
            fail(c.kind == BF200_CLOSURE_LAMBERTIAN_REFLECTION ? "Lambertian directions must be finite unit vectors."
                                                                : "Rough-diffuse directions must be finite unit vectors.");
        }
        BsdfSample s;
        const V3 wi = map_cosine_hemisphere(u, v);
        if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
            return s;
        }
        s.wi = wi;
        s.value = record_eval(c, allowed, wo, wi);
        s.pdf = record_pdf(c, allowed, wo, wi);
        s.lobes = c.lobes;
        s.valid = true;
        return s;
    }
    case BF200_CLOSURE_ROUGH_CONDUCTOR_REFLECTION:
        return conductor_sample(c, wo, u, v);
    case BF200_CLOSURE_ROUGH_DIELECTRIC: {  // DepthFilteredClosureMixture.hpp:135-180
        float e = event;
        if (allowed == BF200_LOBE_REFLECTION) {
            e = 0.0F;
        } else if (allowed == BF200_LOBE_TRANSMISSION) {
            e = std::nextafter(1.0F, 0.0F);
        }
        BsdfSample s = dielectric_sample(c, wo, e, u, v);
        if (!s.valid) {
            return s;
        }
        if ((s.lobes & allowed) == 0U) {
            return BsdfSample{};
        }
        s.pdf = dielectric_pdf_masked(c, allowed, wo, s.wi);
        return s;
    }
    case BF200_CLOSURE_SPECULAR_REFLECTION:
        return specular_reflection_sample(c, wo);
    case BF200_CLOSURE_SPECULAR_TRANSMISSION:
        return specular_transmission_sample(c, wo);
    default:
        fail("unsupported closure");
    }
}

void require_unit_queries(V3 wo, V3 wi) {
    if (!unit_length(wo) || !unit_length(wi)) {
        fail("Depth-filtered closure queries require finite unit directions and a supported transport mode.");
    }
}

Spectrum mixture_eval(const Mixture& m, V3 wo, V3 wi) {
    require_unit_queries(wo, wi);
    Spectrum result{};
    for (uint32_t i = 0; i < m.count; ++i) {
        const Spectrum component = record_eval(m.closure(i), m.allowed[i], wo, wi);
        for (int lane = 0; lane < 4; ++lane) {
            const float sum = result[lane] + component[lane];
            if (!std::isfinite(sum)) {
                fail("A depth-filtered closure value is not representable.");
            }
            result[lane] = sum;
        }
    }
    return result;
}

float mixture_pdf(const Mixture& m, V3 wo, V3 wi) {
    require_unit_queries(wo, wi);
    if (m.count == 0U) {
        return 0.0F;
    }
    float conditional[kMaxClosures] = {};
    for (uint32_t i = 0; i < m.count; ++i) {
        conditional[i] = record_pdf(m.closure(i), m.allowed[i], wo, wi);
    }
    return mix_densities(m.p, conditional, m.count);
}

// aggregate_delta_atom (ClosureMixture.hpp:760-870): the discrete mass and value of every active
// delta closure whose deterministic direction is exactly `wi`.
void aggregate_delta_atom(const Mixture& m, V3 wo, V3 wi, Spectrum& value, float& probability) {
    float value_sum[4] = {}, value_correction[4] = {};
    float p_sum = 0.0F, p_correction = 0.0F;
    uint32_t matching = 0;
    for (uint32_t i = 0; i < m.count; ++i) {
        const Closure& c = m.closure(i);
        if (!is_delta_kind(c.kind)) {
            continue;
        }
        const BsdfSample candidate = record_sample(c, BF200_LOBE_REFLECTION | BF200_LOBE_TRANSMISSION, wo, 0.0F, 0.0F, 0.0F);
        if (!candidate.valid || candidate.wi.x != wi.x || candidate.wi.y != wi.y || candidate.wi.z != wi.z) {
            continue;
        }
        if (!candidate.delta || !std::isfinite(candidate.pdf) || !(candidate.pdf > 0.0F) || candidate.pdf > 1.0F) {
            fail("A sampled delta closure requires a finite positive discrete probability.");
        }
        for (int lane = 0; lane < 4; ++lane) {
            if (!add_compensated(candidate.value[lane], value_sum[lane], value_correction[lane])) {
                fail("A coincident delta value is not representable in the requested precision.");
            }
        }
        if (!add_compensated(positive_probability_product(m.p[i], candidate.pdf), p_sum, p_correction)) {
            fail("A coincident delta probability is not representable in the requested precision.");
        }
        ++matching;
    }
    probability = p_sum + p_correction;
    if (matching == 0U || !std::isfinite(probability) || !(probability > 0.0F) || probability > 1.0F) {
        fail("The sampled delta atom is absent from the closure mixture.");
    }
    for (int lane = 0; lane < 4; ++lane) {
        value[lane] = value_sum[lane] + value_correction[lane];
        if (!std::isfinite(value[lane]) || value[lane] < 0.0F) {
            fail("A coincident delta value is not representable in the requested precision.");
        }
    }
}

// DepthFilteredClosureMixture::sample (DepthFilteredClosureMixture.hpp:460-552)
BsdfSample mixture_sample(const Mixture& m, V3 wo, float component, float u, float v) {
    if (!unit_length(wo) || !(component >= 0.0F && component < 1.0F) || !(u >= 0.0F && u < 1.0F) ||
        !(v >= 0.0F && v < 1.0F)) {
        fail("Depth-filtered closure sampling requires canonical samples, a finite unit direction, and a supported "
             "transport mode.");
    }
    if (m.count == 0U) {
        return BsdfSample{};
    }
    uint32_t selected = m.count;
    for (uint32_t i = 0; i < m.count; ++i) {
        if (component < m.cdf[i + 1]) {
            selected = i;
            break;
        }
    }
    if (selected == m.count) {
        fail("The depth-filtered closure CDF did not select a component.");
    }
    const float event = (component - m.cdf[selected]) / m.p[selected];
    if (!std::isfinite(event) || event < 0.0F || !(event < 1.0F)) {
        fail("The depth-filtered closure sample cannot be remapped to [0, 1).");
    }
    BsdfSample s = record_sample(m.closure(selected), m.allowed[selected], wo, event, u, v);
    if (!s.valid) {
        return s;
    }
    if (m.count > 1U) {
        if (!s.delta) {
            s.value = mixture_eval(m, wo, s.wi);
            s.pdf = mixture_pdf(m, wo, s.wi);
        } else {
            aggregate_delta_atom(m, wo, s.wi, s.value, s.pdf);
        }
    }
    s.selected = m.source[selected];
    return s;
}

// ---------------------------------------------------------------------------------------------
// Surface reconstruction (SceneSurfaceInteraction.cpp:54-350, 804-937)
// ---------------------------------------------------------------------------------------------

struct Surface {
    V3 position, error, ng, ns;
    Frame frame;
    const Material* material;
};

// Surface of an analytic sphere hit, the backend's design (the reference has no scene-level
// spheres): the outward normal of the object-space hit point (robust_outward_normal), the point
// moved onto the sphere along it with a 7-ulp bound of |centre| + r per axis, carried into world
// space as transform_position_with_error does; geometric normal = shading normal = the world
// normal through the inverse transpose (robust_transformed_normal).
Surface resolve_sphere_surface(const Scene& scene, const Instance& inst, const bf200_geometry_v1& g, const Hit& hit,
                               Surface s) {
    const V3 centre = scene.positions[g.vertex_offset];
    const float radius = g.radius;
    const V3 local = transform_point(inst.to_object, hit.position);
    V3 n{};
    if (!sphere_outward_normal(V3{local.x - centre.x, local.y - centre.y, local.z - centre.z}, n)) {
        fail("A sphere hit normal is not representable.");
    }
    constexpr float gamma7 = (7.0F * kEpsilon) / (1.0F - 7.0F * kEpsilon);
    const float c[3] = {centre.x, centre.y, centre.z}, nv[3] = {n.x, n.y, n.z};
    float point[3], perr[3];
    for (int a = 0; a < 3; ++a) {
        point[a] = c[a] + nv[a] * radius;
        perr[a] = gamma7 * (std::abs(c[a]) + radius);
    }
    const V3 world = transform_point(inst.to_world, V3{point[0], point[1], point[2]});
    const float w[3] = {world.x, world.y, world.z};
    const float h[3] = {hit.position.x, hit.position.y, hit.position.z};
    constexpr double eps = static_cast<double>(kEpsilon);
    constexpr double g7 = (7.0 * eps) / (1.0 - 7.0 * eps);
    float err[3];
    for (int row = 0; row < 3; ++row) {
        double magnitude = std::abs(static_cast<double>(inst.to_world(row, 3)));
        double propagated = 0.0;
        for (int col = 0; col < 3; ++col) {
            const double coefficient = std::abs(static_cast<double>(inst.to_world(row, col)));
            magnitude += coefficient * std::abs(static_cast<double>(point[col]));
            propagated += coefficient * static_cast<double>(perr[col]);
        }
        const double discrepancy = std::abs(static_cast<double>(w[row]) - static_cast<double>(h[row]));
        const double bound = g7 * magnitude + (1.0 + g7) * propagated + discrepancy;
        if (!std::isfinite(bound) || bound < 0.0 || bound > static_cast<double>(std::numeric_limits<float>::max())) {
            fail("A transformed sphere position error is not representable.");
        }
        err[row] = static_cast<float>(bound);
        if (static_cast<double>(err[row]) < bound) {
            err[row] = std::nextafter(err[row], kInfinity);
        }
    }
    s.position = world;
    s.error = V3{err[0], err[1], err[2]};
    const Mat4& inv = inst.to_object;
    const double nd[3] = {n.x, n.y, n.z};
    const double tr[3] = {
        std::fma(double(inv(0, 0)), nd[0], std::fma(double(inv(1, 0)), nd[1], double(inv(2, 0)) * nd[2])),
        std::fma(double(inv(0, 1)), nd[0], std::fma(double(inv(1, 1)), nd[1], double(inv(2, 1)) * nd[2])),
        std::fma(double(inv(0, 2)), nd[0], std::fma(double(inv(1, 2)), nd[1], double(inv(2, 2)) * nd[2]))};
    const double mc = std::max({std::abs(tr[0]), std::abs(tr[1]), std::abs(tr[2])});
    if (!std::isfinite(mc) || mc == 0.0) {
        fail("A sphere normal cannot be normalized.");
    }
    const double sc[3] = {tr[0] / mc, tr[1] / mc, tr[2] / mc};
    const double magnitude = std::sqrt(std::fma(sc[0], sc[0], std::fma(sc[1], sc[1], sc[2] * sc[2])));
    const V3 ng{static_cast<float>(sc[0] / magnitude), static_cast<float>(sc[1] / magnitude),
                static_cast<float>(sc[2] / magnitude)};
    s.ng = ng;
    s.ns = ng;
    if (s.material->frame_mode != 0) {
        fail("surface-tangent closure frames are not part of this restatement");
    }
    s.frame = rotated_about_normal(frame_from_normal(ng), s.material->rotation);
    return s;
}

Surface resolve_surface(const Scene& scene, const Hit& hit) {
    Surface s{};
    const Instance& inst = scene.instances[hit.instance];
    const auto& g = scene.geometries[inst.geometry];
    s.material = &scene.materials[inst.material];
    if (g.kind == BF200_GEOMETRY_SPHERE) {
        return resolve_sphere_surface(scene, inst, g, hit, s);
    }
    // validate_barycentrics (:54-76)
    constexpr float tolerance = 32.0F * kEpsilon;
    const float bs[3] = {hit.b0, hit.b1, hit.b2};
    for (float b : bs) {
        if (!std::isfinite(b) || b < -tolerance || b > 1.0F + tolerance) {
            fail("An acceleration hit contains invalid triangle barycentric coordinates.");
        }
    }
    const float sum = bs[0] + bs[1] + bs[2];
    if (!std::isfinite(sum) || std::abs(sum - 1.0F) > tolerance) {
        fail("An acceleration hit contains barycentric coordinates that do not sum to one.");
    }
    const uint32_t* tri = &scene.triangles[3 * (g.triangle_offset + hit.primitive)];
    V3 op[3], on[3];
    for (int k = 0; k < 3; ++k) {
        op[k] = scene.positions[g.vertex_offset + tri[k]];
        on[k] = scene.normals[g.vertex_offset + tri[k]];
    }
    // interpolate_position_with_error (:82-133)
    constexpr float gamma7 = (7.0F * kEpsilon) / (1.0F - 7.0F * kEpsilon);
    float scale = 0.0F;
    const float coords[3][3] = {{op[0].x, op[0].y, op[0].z}, {op[1].x, op[1].y, op[1].z},
                                {op[2].x, op[2].y, op[2].z}};
    for (int axis = 0; axis < 3; ++axis) {
        scale = std::max({scale, std::abs(coords[1][axis] - coords[0][axis]),
                          std::abs(coords[2][axis] - coords[0][axis])});
    }
    const float floor_error = kEpsilon * scale;
    if (!std::isfinite(scale) || !std::isfinite(floor_error) || !(floor_error > 0.0F)) {
        fail("A scene triangle position-error scale is not representable.");
    }
    float point[3], perr[3];
    for (int axis = 0; axis < 3; ++axis) {
        const float p0 = bs[0] * coords[0][axis], p1 = bs[1] * coords[1][axis],
                    p2 = bs[2] * coords[2][axis];
        point[axis] = std::fma(bs[0], coords[0][axis], std::fma(bs[1], coords[1][axis], p2));
        const float magnitude = std::abs(p0) + std::abs(p1) + std::abs(p2);
        perr[axis] = std::max(gamma7 * magnitude, floor_error);
    }
    // transform_position_with_error (:135-189)
    const V3 object_point{point[0], point[1], point[2]};
    const V3 world = transform_point(inst.to_world, object_point);
    {
        const float src[3] = {point[0], point[1], point[2]};
        const float w[3] = {world.x, world.y, world.z};
        const float h[3] = {hit.position.x, hit.position.y, hit.position.z};
        constexpr double eps = static_cast<double>(kEpsilon);
        constexpr double g7 = (7.0 * eps) / (1.0 - 7.0 * eps);
        constexpr double maximum = static_cast<double>(std::numeric_limits<float>::max());
        float err[3];
        for (int row = 0; row < 3; ++row) {
            double magnitude = std::abs(static_cast<double>(inst.to_world(row, 3)));
            double propagated = 0.0;
            for (int col = 0; col < 3; ++col) {
                const double coefficient = std::abs(static_cast<double>(inst.to_world(row, col)));
                magnitude += coefficient * std::abs(static_cast<double>(src[col]));
                propagated += coefficient * static_cast<double>(perr[col]);
            }
            const double discrepancy = std::abs(static_cast<double>(w[row]) - static_cast<double>(h[row]));
            const double bound = g7 * magnitude + (1.0 + g7) * propagated + discrepancy;
            if (!std::isfinite(bound) || bound < 0.0 || bound > maximum) {
                fail("A transformed scene triangle position error is not representable.");
            }
            err[row] = static_cast<float>(bound);
            if (static_cast<double>(err[row]) < bound) {
                err[row] = std::nextafter(err[row], kInfinity);
            }
        }
        s.error = V3{err[0], err[1], err[2]};
    }
    s.position = world;
    s.ng = hit.normal;
    // interpolate_shading_normal (:305-349) with robust_transformed_normal (:252-295)
    const V3 obj_n{std::fma(bs[0], on[0].x, std::fma(bs[1], on[1].x, bs[2] * on[2].x)),
                   std::fma(bs[0], on[0].y, std::fma(bs[1], on[1].y, bs[2] * on[2].y)),
                   std::fma(bs[0], on[0].z, std::fma(bs[1], on[1].z, bs[2] * on[2].z))};
    const Mat4& inv = inst.to_object;
    const double n[3] = {obj_n.x, obj_n.y, obj_n.z};
    const double tr[3] = {
        std::fma(double(inv(0, 0)), n[0], std::fma(double(inv(1, 0)), n[1], double(inv(2, 0)) * n[2])),
        std::fma(double(inv(0, 1)), n[0], std::fma(double(inv(1, 1)), n[1], double(inv(2, 1)) * n[2])),
        std::fma(double(inv(0, 2)), n[0], std::fma(double(inv(1, 2)), n[1], double(inv(2, 2)) * n[2]))};
    const double mc = std::max({std::abs(tr[0]), std::abs(tr[1]), std::abs(tr[2])});
    if (!std::isfinite(mc) || mc == 0.0) {
        fail("A scene shading normal cannot be normalized.");
    }
    const double sc[3] = {tr[0] / mc, tr[1] / mc, tr[2] / mc};
    const double magnitude = std::sqrt(std::fma(sc[0], sc[0], std::fma(sc[1], sc[1], sc[2] * sc[2])));
    V3 ns{static_cast<float>(sc[0] / magnitude), static_cast<float>(sc[1] / magnitude),
          static_cast<float>(sc[2] / magnitude)};
    // transform_orientation (:204-250): sign of det of the upper 3x3 by partial pivoting.
    {
        double m[9];
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 3; ++c) {
                m[r * 3 + c] = static_cast<double>(inst.to_world(r, c));
            }
        }
        int orientation = 1;
        for (int col = 0; col < 3; ++col) {
            int pr = col;
            double pm = std::abs(m[col * 3 + col]);
            for (int cand = col + 1; cand < 3; ++cand) {
                const double cm = std::abs(m[cand * 3 + col]);
                if (cm > pm) {
                    pm = cm;
                    pr = cand;
                }
            }
            if (!std::isfinite(pm) || pm == 0.0) {
                fail("A scene instance transform orientation is not representable.");
            }
            if (pr != col) {
                for (int sc2 = col; sc2 < 3; ++sc2) {
                    std::swap(m[col * 3 + sc2], m[pr * 3 + sc2]);
                }
                orientation = -orientation;
            }
            const double pivot = m[col * 3 + col];
            orientation = pivot < 0.0 ? -orientation : orientation;
            for (int row = col + 1; row < 3; ++row) {
                const double factor = m[row * 3 + col] / pivot;
                for (int uc = col + 1; uc < 3; ++uc) {
                    m[row * 3 + uc] -= factor * m[col * 3 + uc];
                }
            }
        }
        if (orientation < 0) {
            ns = -ns;
        }
    }
    if (!(dot(s.ng, ns) > 0.0F)) {
        fail("A scene shading normal lies outside the geometric-normal hemisphere.");
    }
    s.ns = ns;
    if (s.material->frame_mode != 0) {
        fail("surface-tangent closure frames are not part of this restatement");
    }
    s.frame = rotated_about_normal(frame_from_normal(ns), s.material->rotation);
    return s;
}

// ---------------------------------------------------------------------------------------------
// The path loop (SceneMisPathLoop.cpp:632-917)
// ---------------------------------------------------------------------------------------------

struct Options {
    uint32_t sampler;
    uint32_t heuristic;
    uint32_t limits[5];
    bool roulette;
    uint32_t roulette_first;
    float roulette_min, roulette_max;
};

struct PrevBsdf {
    bool valid = false;
    V3 position;
    float pdf;
    V3 direction;
};

void add_spectrum_product(Spectrum& acc, const Spectrum& a, const Spectrum& b) {
    // accumulate_emission (BsdfOnlyPathLoop.hpp:148-168) with checked_product (:47-62).
    for (int lane = 0; lane < 4; ++lane) {
        const float product = a[lane] * b[lane];
        if (!std::isfinite(product) || (a[lane] != 0.0F && b[lane] != 0.0F && product == 0.0F)) {
            fail("Emitted-radiance multiplication is not representable.");
        }
        acc[lane] = acc[lane] + product;
        if (!std::isfinite(acc[lane])) {
            fail("Radiance accumulation is not representable.");
        }
    }
}

// SceneMisPathLoop.cpp:481-528 (accumulate_weighted_emission).
void add_weighted_emission(Spectrum& acc, const Spectrum& beta, const Spectrum& le, float w) {
    if (!std::isfinite(w) || w < 0.0F || w > 1.0F) {
        fail("An emitted-radiance MIS weight must lie in [0, 1].");
    }
    if (w == 1.0F) {
        add_spectrum_product(acc, beta, le);
        return;
    }
    for (int lane = 0; lane < 4; ++lane) {
        if (beta[lane] == 0.0F || le[lane] == 0.0F || w == 0.0F) {
            continue;
        }
        int e1 = 0, e2 = 0, e3 = 0, en = 0;
        const float significand = std::frexp(beta[lane], &e1) * std::frexp(le[lane], &e2) *
                                  std::frexp(w, &e3);
        const float normalized = std::frexp(significand, &en);
        const float contribution = std::scalbn(normalized, e1 + e2 + e3 + en);
        if (!std::isfinite(contribution) || !(contribution > 0.0F)) {
            fail("A weighted emitted-radiance contribution is not representable.");
        }
        acc[lane] = acc[lane] + contribution;
        if (!std::isfinite(acc[lane])) {
            fail("MIS radiance accumulation is not representable.");
        }
    }
}

// LightSampler.cpp:1023-1056 (uniform sample) and :1133-1149 (probability).
uint32_t select_light(const Scene& scene, float u, float& probability, V3 position) {
    if (scene.use_tree) {  // LightSampler::sample(context, u) (LightSampler.cpp:1058-1129)
        const float p[3] = {position.x, position.y, position.z};
        uint32_t light = 0;
        std::string error;
        if (bf200::light_tree_sample(scene.tree, p, u, light, probability, error) != BLACKFRAME_STATUS_SUCCESS) {
            fail("The light tree refused a selection.");
        }
        return light;
    }
    const auto begin = scene.light_cdf.begin() + 1;
    const auto it = std::upper_bound(begin, scene.light_cdf.end(), u);
    if (it == scene.light_cdf.end()) {
        fail("Light-selection CDF could not classify a canonical sample.");
    }
    const size_t index = static_cast<size_t>(it - scene.light_cdf.begin()) - 1;
    probability = scene.light_cdf[index + 1] - scene.light_cdf[index];
    return static_cast<uint32_t>(index);
}

float light_probability(const Scene& scene, uint32_t index, V3 position) {
    if (scene.use_tree) {  // LightSampler::probability(context, i) (LightSampler.cpp:1151-1225)
        const float p[3] = {position.x, position.y, position.z};
        float probability = 0.0F;
        std::string error;
        if (bf200::light_tree_probability(scene.tree, p, index, probability, error) != BLACKFRAME_STATUS_SUCCESS) {
            fail("The light tree refused a selection probability.");
        }
        return probability;
    }
    return scene.light_cdf[index + 1] - scene.light_cdf[index];
}

// validate_sampler_support (SceneMisPathLoop.cpp:397-430) under the light tree: every mesh light
// must have a representable, positive selection probability at the shading point.
void validate_tree_support(const Scene& scene, V3 position) {
    if (!scene.use_tree) {
        return;
    }
    for (uint32_t i = 0; i < scene.punctual.size(); ++i) {
        if (!is_black(scene.punctual[i].spectrum) && !(light_probability(scene, i, position) > 0.0F)) {
            fail("The light sampler gives zero support to a non-black punctual light.");
        }
    }
    for (uint32_t i = 0; i < scene.lights.size(); ++i) {
        const uint32_t slot = static_cast<uint32_t>(scene.punctual.size()) + i;
        if (!(light_probability(scene, slot, position) > 0.0F)) {
            fail("The light sampler gives zero support to a non-black mesh area light.");
        }
    }
}

// RussianRoulette.cpp (evaluate): returns false when the path terminates.
bool russian_roulette(Spectrum& beta, float eta_scale, float u, const Options& o) {
    float maximum_throughput = 0.0F;
    for (float lane : beta) {
        if (!std::isfinite(lane) || lane < 0.0F) {
            fail("Russian roulette throughput must be finite and non-negative.");
        }
        maximum_throughput = std::max(maximum_throughput, lane);
    }
    if (maximum_throughput == 0.0F) {
        fail("Russian roulette cannot evaluate an all-zero continuation throughput.");
    }
    float survival;
    if (maximum_throughput >= o.roulette_max / eta_scale) {
        survival = o.roulette_max;
    } else if (maximum_throughput <= o.roulette_min / eta_scale) {
        survival = o.roulette_min;
    } else {
        survival = std::clamp(maximum_throughput * eta_scale, o.roulette_min, o.roulette_max);
    }
    if (!(u < survival)) {
        return false;
    }
    for (int lane = 0; lane < 4; ++lane) {
        const float c = beta[lane] / survival;
        if (!std::isfinite(c) || (beta[lane] != 0.0F && c == 0.0F)) {
            fail("Russian roulette compensation is not representable.");
        }
        beta[lane] = c;
    }
    return true;
}

// ShadingNormalCorrection.hpp:65-121 in radiance mode: 1 when both directions lie on the same
// side of both normals, otherwise 0.
float shading_correction(V3 ng, V3 ns, V3 wo, V3 wi) {
    const float og = dot(ng, wo), os = dot(ns, wo), ig = dot(ng, wi), is = dot(ns, wi);
    if (og == 0.0F || os == 0.0F || ig == 0.0F || is == 0.0F ||
        std::signbit(og) != std::signbit(os) || std::signbit(ig) != std::signbit(is)) {
        return 0.0F;
    }
    return 1.0F;
}

struct PathOut {
    Spectrum beta, radiance;
    Depth depth;
    float eta_scale;
    uint32_t delta_flags, termination, blocked, segments;
    V3 ray_o, ray_d;
    float ray_tmin, ray_tmax;
    float cone_width = 0.0F, cone_spread = 0.0F;  // the ray cone at ray_o (traced with cones only)
};

// ---------------------------------------------------------------------------------------------
// Ray cones of the reference's wavefront (CudaWavefrontStages.cu:540-543, 2816-2870, 3675-3781;
// the CPU twin is RayCone.hpp:133-156, 222-240, 316-437, which measures the direction with
// std::hypot and tests unit directions to 256 ulp where the wavefront uses max|d| * |d / max|d||
// and 128 ulp). Every product and ratio is checked: not finite, or non-zero factors whose
// product underflows to zero, is a failure.
// ---------------------------------------------------------------------------------------------

bool cone_valid(float width, float spread) {
    return std::isfinite(width) && width >= 0.0F && std::isfinite(spread) && spread >= 0.0F;
}

bool cone_product(float left, float right, float& product) {  // checked_ray_cone_product
    product = left * right;
    return std::isfinite(product) && !(left != 0.0F && right != 0.0F && product == 0.0F);
}

bool cone_ratio(float numerator, float denominator, float& ratio) {  // checked_ray_cone_ratio
    if (!std::isfinite(numerator) || !(numerator > 0.0F) || !std::isfinite(denominator) ||
        !(denominator > 0.0F)) {
        return false;
    }
    ratio = numerator / denominator;
    return std::isfinite(ratio) && ratio > 0.0F;
}

// advance_ray_cone_to_hit (CudaWavefrontStages.cu:2832-2870)
bool cone_advance(float width, float spread, V3 d, float t, float& out_width) {
    if (!cone_valid(width, spread) || !std::isfinite(t) || t < 0.0F) {
        return false;
    }
    const float scale = std::fmax(std::fabs(d.x), std::fmax(std::fabs(d.y), std::fabs(d.z)));
    if (!std::isfinite(scale) || !(scale > 0.0F)) {
        return false;
    }
    const float inverse = 1.0F / scale;
    const float sx = d.x * inverse, sy = d.y * inverse, sz = d.z * inverse;
    const float normalized_length = std::sqrt(std::fma(sx, sx, std::fma(sy, sy, sz * sz)));
    float length = 0.0F, distance = 0.0F, growth = 0.0F;
    if (!std::isfinite(normalized_length) || !(normalized_length > 0.0F) ||
        !cone_product(scale, normalized_length, length) || !(length > 0.0F)) {
        return false;
    }
    if (!cone_product(t, length, distance) || distance < 0.0F || !cone_product(spread, distance, growth)) {
        return false;
    }
    const float advanced = std::fma(spread, distance, width);
    if (!std::isfinite(advanced) || advanced < width || (growth != 0.0F && advanced == width)) {
        return false;
    }
    out_width = advanced;
    return cone_valid(advanced, spread);
}

// transport::unit_vector (TransportDevice.cuh:325-333)
bool cone_unit(V3 v) {
    if (!std::isfinite(v.x) || !std::isfinite(v.y) || !std::isfinite(v.z)) {
        return false;
    }
    const float squared = std::fma(v.x, v.x, std::fma(v.y, v.y, v.z * v.z));
    return std::isfinite(squared) && std::fabs(squared - 1.0F) <= 128.0F * kEpsilon;
}

// valid_surface_event (CudaWavefrontStages.cu:2803-2814)
bool cone_surface_event(uint32_t bits) {
    const uint32_t family = bits & 0x07U, direction = bits & 0x18U;
    return bits != 0U && (bits & ~0x3FU) == 0U && (bits & 0x20U) == 0U &&
           (family == 0x01U || family == 0x02U || family == 0x04U) && (direction == 0x08U || direction == 0x10U);
}

// propagate_ray_cone_scattering (CudaWavefrontStages.cu:3675-3781). Closure kinds follow
// ClosureKind: 1 lambertian, 2 rough diffuse, 3 rough conductor, 4 rough dielectric,
// 5 specular reflection, 6 specular transmission.
bool cone_scatter(float width, float spread, uint32_t kind, const float* p, uint32_t event, V3 wo, V3 wi,
                  float& out_width, float& out_spread) {
    if (!cone_valid(width, spread) || !cone_surface_event(event) || !cone_unit(wo) || !cone_unit(wi) ||
        wo.z == 0.0F || wi.z == 0.0F) {
        return false;
    }
    const bool reflection = (event & 0x08U) != 0U, transmission = (event & 0x10U) != 0U;
    const bool same_hemisphere = (wo.z > 0.0F) == (wi.z > 0.0F);
    if ((reflection && !same_hemisphere) || (transmission && same_hemisphere)) {
        return false;
    }
    float spread_floor = 0.0F, transmission_scale = 1.0F, width_scale = 1.0F;
    switch (kind) {
    case 1U:
    case 2U:
        if (!reflection || (event & 0x01U) == 0U) {
            return false;
        }
        spread_floor = 1.0F;
        break;
    case 3U:
        if (!reflection || (event & 0x02U) == 0U || !std::isfinite(p[8]) || p[8] < 0.0F ||
            !std::isfinite(p[9]) || p[9] < 0.0F) {
            return false;
        }
        spread_floor = std::fmax(p[8], p[9]);
        break;
    case 4U:
        if ((event & 0x02U) == 0U || !std::isfinite(p[2]) || p[2] < 0.0F || !std::isfinite(p[3]) || p[3] < 0.0F) {
            return false;
        }
        spread_floor = std::fmax(p[2], p[3]);
        break;
    case 5U:
        if (!reflection || (event & 0x04U) == 0U) {
            return false;
        }
        break;
    case 6U:
        if (!transmission || (event & 0x04U) == 0U) {
            return false;
        }
        break;
    default:
        return false;
    }
    if (transmission) {
        if (kind != 4U && kind != 6U) {
            return false;
        }
        const float incident = wo.z > 0.0F ? p[0] : p[1];
        const float transmitted = wo.z > 0.0F ? p[1] : p[0];
        float eta_ratio = 0.0F, cosine_ratio = 0.0F, inverse_cosine_ratio = 0.0F, meridional = 0.0F;
        if (!cone_ratio(incident, transmitted, eta_ratio) ||
            !cone_ratio(std::fabs(wo.z), std::fabs(wi.z), cosine_ratio) ||
            !cone_ratio(std::fabs(wi.z), std::fabs(wo.z), inverse_cosine_ratio) ||
            !cone_product(eta_ratio, cosine_ratio, meridional)) {
            return false;
        }
        transmission_scale = std::fmax(eta_ratio, meridional);
        width_scale = std::fmax(1.0F, inverse_cosine_ratio);
    }
    float scattered_width = 0.0F, scattered_spread = 0.0F;
    if (!cone_product(width, width_scale, scattered_width) ||
        !cone_product(spread, transmission_scale, scattered_spread)) {
        return false;
    }
    out_width = scattered_width;
    out_spread = std::fmax(scattered_spread, spread_floor);
    return cone_valid(out_width, out_spread);
}

// SceneMisPathLoop.cpp:136-275 (estimate): the direct contribution of one light sample, its
// shadow ray traced.
Spectrum direct_lighting(const Scene& scene, const Options& opt, const Surface& surf, const Mixture& mix,
                         const Spectrum& beta, V3 wo_world, const Dims& dims, const Stream& stream, uint32_t mask,
                         float time) {
    const Spectrum zero{};
    if (is_black(beta)) {
        return zero;
    }
    bool all_black = true;
    for (uint32_t i = 0; i < mix.count; ++i) {
        all_black = all_black && is_black(mix.closure(i).weight);
    }
    if (all_black) {
        return zero;
    }
    float selection;
    validate_tree_support(scene, surf.position);
    const uint32_t light_index = select_light(scene, stream.sample_1d(dims.light_selection), selection, surf.position);
    const float lu = stream.sample_1d(dims.light_u), lv = stream.sample_1d(dims.light_v);
    LightSample ls;
    if (light_index < scene.punctual.size()) {
        ls = sample_punctual_light(scene.punctual[light_index], surf.position, lu, lv);
    } else {
        const MeshLight& light = scene.lights[light_index - scene.punctual.size()];
        if ((scene.instances[light.instance].mask & mask) == 0U) {
            return zero;
        }
        ls = sample_mesh_light(light, surf.position, lu, lv);
    }
    if (!ls.valid) {
        return zero;
    }
    const V3 wo = surf.frame.to_local(wo_world);
    const V3 wi = surf.frame.to_local(ls.direction);
    if (wo.z == 0.0F || wi.z == 0.0F) {
        return zero;
    }
    const bool lambert = mix.count == 1U && mix.closure(0).kind == BF200_CLOSURE_LAMBERTIAN_REFLECTION;
    Spectrum f{};
    if (!lambert) {
        f = mixture_eval(mix, wo, wi);
        if (is_black(f)) {
            return zero;
        }
    }
    const float correction = shading_correction(surf.ng, surf.ns, wo_world, ls.direction);
    if (correction == 0.0F) {
        return zero;
    }
    float weight = 1.0F;
    if (!ls.discrete) {
        const float bsdf_pdf = mixture_pdf(mix, wo, wi);
        const float light_pdf = joint_light_pdf(selection, ls.pdf);
        weight = mis_weight(opt.heuristic, light_pdf, bsdf_pdf);
    }
    // make_shadow_ray (ShadowRay.hpp:181-253)
    const V3 origin = offset_surface_point(surf.position, surf.error, surf.ng, ls.direction);
    V3 sd = ls.direction;
    float t_max = kInfinity;
    if (!ls.infinite) {
        V3 endpoint;
        if (ls.point) {
            V3 nominal;
            float nominal_length;
            unit_segment(origin, ls.position, ls.direction, nominal, nominal_length);
            endpoint = contract_point_endpoint(ls.position, ls.error, nominal);
        } else {
            endpoint = offset_surface_point(ls.position, ls.error, ls.normal, origin - ls.position);
        }
        float length;
        unit_segment(origin, endpoint, ls.direction, sd, length);
        t_max = std::nextafter(length, 0.0F);
        if (!(t_max > 0.0F) || !std::isfinite(t_max)) {
            fail("A finite shadow-ray interval is not representable in the requested precision.");
        }
    }
    (void)time;
    const bool blocked = occluded(scene, origin, sd, 0.0F, t_max, mask);
    const float transmittance = blocked ? 0.0F : 1.0F;
    Spectrum out{};
    for (int lane = 0; lane < 4; ++lane) {
        const Closure& closure = mix.closure(0);
        if (lambert) {
            // evaluate_lambertian_direct_lighting (DirectLighting.hpp:171-236)
            if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
                return zero;
            }
            if (weight == 1.0F) {
                const float num[6] = {beta[lane], closure.weight[lane], kInvPi, ls.radiance[lane], wi.z,
                                      transmittance};
                const float den[2] = {selection, ls.pdf};
                out[lane] = checked_product_quotient(num, 6, den, 2);
            } else {
                const float num[7] = {beta[lane], closure.weight[lane], kInvPi, ls.radiance[lane], wi.z,
                                      transmittance, weight};
                const float den[2] = {selection, ls.pdf};
                out[lane] = checked_product_quotient(num, 7, den, 2);
            }
        } else {
            // evaluate_bsdf_direct_lighting (DirectLighting.hpp:66-145)
            const float cosine = std::abs(wi.z);
            if (weight == 1.0F) {
                const float num[5] = {beta[lane], f[lane], ls.radiance[lane], cosine, transmittance};
                const float den[2] = {selection, ls.pdf};
                out[lane] = checked_product_quotient(num, 5, den, 2);
            } else {
                const float num[6] = {beta[lane], f[lane], ls.radiance[lane], cosine, transmittance,
                                      weight};
                const float den[2] = {selection, ls.pdf};
                out[lane] = checked_product_quotient(num, 6, den, 2);
            }
        }
        out[lane] = out[lane] * correction;
    }
    return out;
}

// cone: null, or the path's primary ray cone (width, spread), carried as the reference's wavefront
// carries it (CudaWavefrontStages.cu:4602-4624) and returned in PathOut::cone_*.
// state: null (PathState::create_initial), or a depth-zero initial state whose throughput,
// radiance and eta scale the path starts from (trace_scene_mis takes any such PathState).
// The radiance contributions of one path as the float transport adds them, for the float64
// gradient (bfo_weight_gradients): each contribution's value, the closure vertices whose weights
// multiply into it (the first `vertices` entries of `materials`), and whether an emitter's radiance
// is one of its factors (emission hits and light samples; not the environment).
struct PathRecord {
    struct Contribution {
        std::array<double, 4> value;
        uint32_t vertices;
        bool emitter;
    };
    std::vector<Contribution> contributions;
    std::vector<uint32_t> materials;  // material of every scattering vertex, in path order
};

PathOut trace(const Scene& scene, const bf200_path_input_v1& input, const Options& opt,
              const float* cone = nullptr, const bf200_path_state_v1* state = nullptr,
              PathRecord* record = nullptr) {
    PathOut out{};
    out.beta = Spectrum{1.0F, 1.0F, 1.0F, 1.0F};
    out.radiance = Spectrum{};
    if (state != nullptr) {
        for (int lane = 0; lane < 4; ++lane) {
            out.beta[lane] = state->beta[lane];
            out.radiance[lane] = state->radiance[lane];
        }
    }
    out.depth = Depth{{0, 0, 0, 0, 0}};
    out.eta_scale = state != nullptr ? state->eta_scale : 1.0F;
    if (state != nullptr) {  // PathState::create's checks (PathState.hpp:84-96)
        for (int lane = 0; lane < 4; ++lane) {
            if (!std::isfinite(out.beta[lane]) || out.beta[lane] < 0.0F || !std::isfinite(out.radiance[lane]) ||
                out.radiance[lane] < 0.0F) {
                fail("An initial path spectrum must be finite and non-negative.");
            }
        }
        if (!std::isfinite(out.eta_scale) || !(out.eta_scale > 0.0F)) {
            fail("Path eta scale must be finite and strictly positive.");
        }
    }
    out.delta_flags = 0;
    out.blocked = 0;
    out.segments = 0;
    const Stream stream{input.sample.pixel_x, input.sample.pixel_y, input.sample.sample_index,
                        input.sample.seed, opt.sampler == 1U};
    V3 ro{input.primary_ray.origin[0], input.primary_ray.origin[1], input.primary_ray.origin[2]};
    V3 rd{input.primary_ray.direction[0], input.primary_ray.direction[1],
          input.primary_ray.direction[2]};
    float tmin = input.primary_ray.t_min, tmax = input.primary_ray.t_max;
    const uint32_t mask = input.primary_ray.mask;
    const float time = input.primary_ray.time;
    if (cone != nullptr) {
        out.cone_width = cone[0];
        out.cone_spread = cone[1];
        if (!cone_valid(out.cone_width, out.cone_spread)) {
            fail("A primary ray cone must be finite and non-negative.");
        }
    }
    PrevBsdf prev;
    auto finish = [&](uint32_t termination) {
        out.termination = termination;
        out.ray_o = ro;
        out.ray_d = rd;
        out.ray_tmin = tmin;
        out.ray_tmax = tmax;
        return out;
    };
    while (true) {
        Hit hit{};
        ++out.segments;
        if (!closest_hit(scene, ro, rd, tmin, tmax, mask, hit)) {
            if (record != nullptr) {
                std::array<double, 4> c{};
                for (int lane = 0; lane < 4; ++lane) {
                    c[lane] = static_cast<double>(out.beta[lane]) * scene.environment[lane];
                }
                record->contributions.push_back({c, static_cast<uint32_t>(record->materials.size()), false});
            }
            add_spectrum_product(out.radiance, out.beta, scene.environment);
            return finish(BF200_TERMINATION_ESCAPED_ENVIRONMENT);
        }
        const Surface surf = resolve_surface(scene, hit);
        const Material& material = *surf.material;
        // Surface emission and its MIS weight (SceneMisPathLoop.cpp:277-356).
        Spectrum emitted{};
        if (emission_side(surf.ng, -rd) > 0) {
            emitted = material.emission;
        }
        float emission_weight = 1.0F;
        if (!is_black(emitted) && prev.valid) {
            if (rd != prev.direction) {
                fail("The emissive hit direction does not match the recorded BSDF sample.");
            }
            const int32_t light_index = scene.light_of_instance[hit.instance];
            if (light_index < 0) {
                fail("A non-black emissive hit is absent from the committed mesh-light registry.");
            }
            const uint32_t slot = static_cast<uint32_t>(scene.punctual.size()) + static_cast<uint32_t>(light_index);
            const float selection = light_probability(scene, slot, prev.position);
            const float conditional = mesh_light_pdf_at_surface(scene.lights[light_index], prev.position,
                                                                surf.position, surf.ng);
            const float light_pdf = joint_light_pdf(selection, conditional);
            emission_weight = mis_weight(opt.heuristic, prev.pdf, light_pdf);
        }
        if (record != nullptr && !is_black(emitted)) {
            std::array<double, 4> c{};
            for (int lane = 0; lane < 4; ++lane) {
                c[lane] = static_cast<double>(out.beta[lane]) * emitted[lane] * emission_weight;
            }
            record->contributions.push_back({c, static_cast<uint32_t>(record->materials.size()), true});
        }
        add_weighted_emission(out.radiance, out.beta, emitted, emission_weight);
        if (is_black(out.beta)) {
            return finish(BF200_TERMINATION_ZERO_THROUGHPUT);
        }
        const Mixture mix = depth_filter(material, opt.limits, out.depth);
        if (mix.count == 0U) {
            if (material.closure_count == 0U) {
                return finish(BF200_TERMINATION_OUTSIDE_BSDF_SUPPORT);
            }
            out.blocked = mix.blocked;
            return finish(BF200_TERMINATION_DEPTH_LIMIT);
        }
        const V3 wo_world = robust_unit(-rd);
        const V3 wo = surf.frame.to_local(wo_world);
        const Dims dims = dims_for_bounce(out.depth.total());
        const float bu = stream.sample_1d(dims.bsdf_u);
        const float bv = stream.sample_1d(dims.bsdf_v);
        const float bc = stream.sample_1d(dims.bsdf_component);
        const BsdfSample bs = mixture_sample(mix, wo, bc, bu, bv);
        Depth next_depth = out.depth;
        if (bs.valid) {
            bool finite_value = true;
            for (int lane = 0; lane < 4; ++lane) {
                finite_value = finite_value && std::isfinite(bs.value[lane]) && bs.value[lane] >= 0.0F;
            }
            if (!valid_surface_event(bs.lobes) || !finite_value || !std::isfinite(bs.pdf) || !(bs.pdf > 0.0F) ||
                bs.wi.z == 0.0F) {
                fail("The closure mixture returned an invalid MIS continuation sample.");
            }
            if (blocked_limits(opt.limits, out.depth, bs.lobes) != 0U) {
                fail("A depth-filtered closure selected a blocked MIS continuation event.");
            }
            next_depth = advanced(out.depth, bs.lobes);
        }
        const Spectrum direct = direct_lighting(scene, opt, surf, mix, out.beta, wo_world, dims, stream, mask, time);
        for (int lane = 0; lane < 4; ++lane) {
            if (!std::isfinite(direct[lane]) || direct[lane] < 0.0F) {
                fail("A direct-lighting contribution must be finite and non-negative.");
            }
            out.radiance[lane] = out.radiance[lane] + direct[lane];
        }
        if (record != nullptr) {
            record->materials.push_back(scene.instances[hit.instance].material);
            if (!is_black(direct)) {
                std::array<double, 4> c{};
                for (int lane = 0; lane < 4; ++lane) {
                    c[lane] = direct[lane];
                }
                record->contributions.push_back({c, static_cast<uint32_t>(record->materials.size()), true});
            }
        }
        if (!bs.valid) {
            return finish(BF200_TERMINATION_OUTSIDE_BSDF_SUPPORT);
        }
        const V3 wi_world = robust_unit(surf.frame.to_world(bs.wi));
        const float correction = shading_correction(surf.ng, surf.ns, wo_world, wi_world);
        if (correction == 0.0F) {
            return finish(BF200_TERMINATION_OUTSIDE_BSDF_SUPPORT);
        }
        // update_closure_throughput (BsdfOnlyPathLoop.hpp:64-131)
        const bool delta = (bs.lobes & BF200_LOBE_SPECULAR) != 0U;
        if (bs.delta != delta || (delta && bs.pdf > 1.0F)) {
            fail("A closure sample uses an incompatible probability measure.");
        }
        Spectrum next_beta{};
        const float cosine = std::abs(bs.wi.z);
        if (!std::isfinite(cosine) || !(cosine > 0.0F)) {
            fail("A closure direction has no representable projected measure.");
        }
        if (mix.count == 1U && mix.closure(0).kind == BF200_CLOSURE_LAMBERTIAN_REFLECTION && correction == 1.0F) {
            const Closure& closure = mix.closure(0);
            for (int lane = 0; lane < 4; ++lane) {
                next_beta[lane] = out.beta[lane] * closure.weight[lane];
                if (!std::isfinite(next_beta[lane]) ||
                    (out.beta[lane] != 0.0F && closure.weight[lane] != 0.0F && next_beta[lane] == 0.0F)) {
                    fail("Lambertian path throughput is not representable.");
                }
            }
        } else {
            for (int lane = 0; lane < 4; ++lane) {
                const float num[4] = {out.beta[lane], bs.value[lane], cosine, correction};
                float significand = 1.0F;
                int exponent = 0;
                bool zero = false;
                for (float factor : num) {
                    if (!std::isfinite(factor) || factor < 0.0F) {
                        fail("Closure factors must be finite and non-negative.");
                    }
                    if (factor == 0.0F) {
                        zero = true;
                        break;
                    }
                    int fe = 0;
                    significand *= std::frexp(factor, &fe);
                    exponent += fe;
                }
                if (zero) {
                    next_beta[lane] = 0.0F;
                    continue;
                }
                int pe = 0, ne = 0;
                significand /= std::frexp(bs.pdf, &pe);
                exponent -= pe;
                significand = std::frexp(significand, &ne);
                const float value = std::scalbn(significand, exponent + ne);
                if (!std::isfinite(value) || !(value > 0.0F)) {
                    fail("Closure throughput is not representable.");
                }
                next_beta[lane] = value;
            }
        }
        const float next_eta = out.eta_scale * bs.eta_scale;
        if (!std::isfinite(next_eta) || !(next_eta > 0.0F)) {
            fail("A closure eta-scale update is not representable.");
        }
        const V3 origin = offset_ray_origin(surf.position, surf.error, surf.ng, wi_world);
        if (origin == surf.position) {
            fail("The derived triangle error did not move the MIS continuation-ray origin.");
        }
        if (cone != nullptr) {
            float advanced = 0.0F;
            const Closure& closure = material.closures[bs.selected];
            if (!cone_advance(out.cone_width, out.cone_spread, rd, hit.t, advanced) ||
                !cone_scatter(advanced, out.cone_spread, closure.kind, closure.p, bs.lobes, wo, bs.wi,
                              out.cone_width, out.cone_spread)) {
                fail("A scattered ray cone is not representable.");
            }
        }
        // record_bsdf_sample (SceneMisPathLoop.cpp:358-390): a delta continuation leaves no density
        // for the next emissive hit's MIS weight
        prev.valid = !delta;
        prev.position = surf.position;
        prev.pdf = bs.pdf;
        prev.direction = wi_world;
        out.beta = next_beta;
        out.depth = next_depth;
        out.eta_scale = next_eta;
        // next_delta_flags (SceneMisPathLoop.cpp:39-52): previous_bounce_was_delta 1,
        // any_non_delta_bounces 2
        out.delta_flags = (out.delta_flags & 2U) | (delta ? 1U : 2U);
        ro = origin;
        rd = wi_world;
        tmin = 0.0F;
        tmax = kInfinity;
        if (is_black(out.beta)) {
            return finish(BF200_TERMINATION_ZERO_THROUGHPUT);
        }
        if (opt.roulette && out.depth.total() >= opt.roulette_first) {
            if (!russian_roulette(out.beta, out.eta_scale, stream.sample_1d(dims.russian_roulette), opt)) {
                return finish(BF200_TERMINATION_RUSSIAN_ROULETTE);
            }
        }
    }
}

std::mutex g_error_mutex;
std::string g_error;

void set_error(const char* message) {
    std::lock_guard<std::mutex> lock{g_error_mutex};
    g_error = message;
}

Options make_options(const bf200_transport_options_v1& o) {
    Options r{};
    r.sampler = o.sampler;
    r.heuristic = o.mis_heuristic;
    for (int i = 0; i < 5; ++i) {
        r.limits[i] = o.depth_limits[i];
    }
    r.roulette = o.roulette_enabled != 0;
    r.roulette_first = o.roulette_first_eligible_depth;
    r.roulette_min = o.roulette_minimum_survival;
    r.roulette_max = o.roulette_maximum_survival;
    return r;
}

void store_result(const PathOut& p, bf200_path_result_v1& r, float time, uint32_t mask) {
    std::memset(&r, 0, sizeof(r));
    for (int lane = 0; lane < 4; ++lane) {
        r.beta[lane] = p.beta[lane];
        r.radiance[lane] = p.radiance[lane];
    }
    r.depth = p.depth.total();
    for (int i = 0; i < 5; ++i) {
        r.depth_counters[i] = p.depth.c[i];
    }
    r.eta_scale = p.eta_scale;
    r.delta_flags = p.delta_flags;
    r.termination = p.termination;
    r.blocked_depth_limits = p.blocked;
    r.lane_status = BF200_LANE_OK;
    r.segments = p.segments;
    r.terminal_ray.origin[0] = p.ray_o.x;
    r.terminal_ray.origin[1] = p.ray_o.y;
    r.terminal_ray.origin[2] = p.ray_o.z;
    r.terminal_ray.direction[0] = p.ray_d.x;
    r.terminal_ray.direction[1] = p.ray_d.y;
    r.terminal_ray.direction[2] = p.ray_d.z;
    r.terminal_ray.t_min = p.ray_tmin;
    r.terminal_ray.t_max = p.ray_tmax;
    r.terminal_ray.time = time;
    r.terminal_ray.mask = mask;
}

}  // namespace
}  // namespace bfo

using namespace bfo;

extern "C" {

__attribute__((visibility("default"))) const char* bfo_last_error() { return g_error.c_str(); }

// 1: sampled-angle sines and cosines rounded as the device rounds them; 0: as the reference does.
__attribute__((visibility("default"))) void bfo_set_device_trig(int enabled) { g_device_trig.store(enabled != 0); }

__attribute__((visibility("default"))) int bfo_scene_create(const bf200_scene_desc_v1* d, void** out) {
    try {
        auto* s = new Scene{};
        s->geometries.assign(d->geometries, d->geometries + d->geometry_count);
        for (uint32_t v = 0; v < d->vertex_count; ++v) {
            s->positions.push_back(load3(d->positions, v));
            s->normals.push_back(load3(d->normals, v));
        }
        s->uvs.assign(d->texture_coordinates, d->texture_coordinates + 2 * d->vertex_count);
        s->triangles.assign(d->triangles, d->triangles + 3 * d->triangle_count);
        for (uint32_t m = 0; m < d->material_count; ++m) {
            const auto& src = d->materials[m];
            Material mat{};
            mat.closure_count = src.closure_count;
            mat.frame_mode = src.frame_mode;
            mat.rotation = src.tangent_rotation_radians;
            for (int lane = 0; lane < 4; ++lane) {
                mat.emission[lane] = src.emitted_radiance[lane];
            }
            if (src.closure_count > kMaxClosures) {
                set_error("A closure mixture contains an invalid active closure count.");
                delete s;
                return 6;
            }
            for (uint32_t k = 0; k < src.closure_count; ++k) {
                const auto& c = d->closures[src.closure_offset + k];
                Closure& dst = mat.closures[k];
                dst.kind = c.kind;
                dst.lobes = c.lobes;
                for (int lane = 0; lane < 4; ++lane) {
                    dst.weight[lane] = c.weight[lane];
                }
                std::memcpy(dst.p, c.parameters, sizeof(dst.p));
            }
            const char* error = nullptr;
            if (!component_distribution(src.component_probabilities, src.closure_count, true, mat.probability,
                                        mat.cdf, &error)) {
                set_error(error);
                delete s;
                return 6;
            }
            s->materials.push_back(mat);
        }
        for (uint32_t i = 0; i < d->instance_count; ++i) {
            const auto& src = d->instances[i];
            Instance inst{};
            inst.geometry = src.geometry_index;
            inst.material = src.material_index;
            inst.mask = src.visibility_mask;
            inst.instance_id = src.instance_id;
            std::memcpy(inst.to_world.m, src.object_to_world, sizeof(inst.to_world.m));
            std::memcpy(inst.to_object.m, src.world_to_object, sizeof(inst.to_object.m));
            const auto& g = s->geometries[inst.geometry];
            for (uint32_t t = 0; t < g.triangle_count; ++t) {
                const uint32_t* tri = &s->triangles[3 * (g.triangle_offset + t)];
                V3 w[3];
                for (int k = 0; k < 3; ++k) {
                    w[k] = transform_point(inst.to_world, s->positions[g.vertex_offset + tri[k]]);
                    inst.world_vertices.push_back(w[k]);
                }
                V3 n;
                if (!triangle_normal(w[0], w[1], w[2], n)) {
                    set_error("A world-space triangle normal is not representable.");
                    delete s;
                    return 2;
                }
                inst.world_normals.push_back(n);
            }
            s->instances.push_back(std::move(inst));
        }
        // Punctual lights, first in the registry (PunctualLights.hpp create checks).
        const uint32_t punctual_count =
            d->struct_size >= sizeof(bf200_scene_desc_v1) && d->punctual_lights != nullptr ? d->punctual_light_count : 0U;
        if (punctual_count != d->punctual_light_count) {
            set_error("punctual lights require the full scene description layout");
            delete s;
            return 7;
        }
        for (uint32_t k = 0; k < punctual_count; ++k) {
            const auto& src = d->punctual_lights[k];
            Punctual light{};
            light.kind = src.kind;
            light.position = load3(src.position, 0);
            light.error = load3(src.position_error, 0);
            light.direction = load3(src.direction, 0);
            for (int lane = 0; lane < 4; ++lane) {
                light.spectrum[lane] = src.spectrum[lane];
                if (!std::isfinite(light.spectrum[lane]) || light.spectrum[lane] < 0.0F) {
                    set_error("A punctual light spectrum must be finite and non-negative.");
                    delete s;
                    return 7;
                }
            }
            const bool finite_point = std::isfinite(light.position.x) && std::isfinite(light.position.y) &&
                                      std::isfinite(light.position.z) && std::isfinite(light.error.x) &&
                                      std::isfinite(light.error.y) && std::isfinite(light.error.z) &&
                                      light.error.x >= 0.0F && light.error.y >= 0.0F && light.error.z >= 0.0F;
            if (src.kind == BF200_PUNCTUAL_POINT) {
                if (!finite_point) {
                    set_error("A finite punctual light requires a finite position and non-negative error.");
                    delete s;
                    return 7;
                }
            } else if (src.kind == BF200_PUNCTUAL_DIRECTIONAL) {
                if (!unit_length(light.direction)) {
                    set_error("A directional light requires a finite unit propagation direction.");
                    delete s;
                    return 7;
                }
            } else if (src.kind == BF200_PUNCTUAL_SPOT) {
                const float inner = src.inner_half_angle, outer = src.outer_half_angle;
                if (!finite_point || !unit_length(light.direction) || !std::isfinite(inner) || !std::isfinite(outer) ||
                    inner < 0.0F || inner > outer || !(outer > 0.0F) || outer >= kPi) {
                    set_error("Spot half angles require 0 <= inner <= outer < pi and a positive outer cone.");
                    delete s;
                    return 7;
                }
                // exact_special_cosine (PunctualLights.hpp:186-197)
                auto special_cosine = [](float angle) {
                    if (angle == 0.0F) return 1.0F;
                    if (angle == kPi / 2.0F) return 0.0F;
                    if (angle == kPi) return -1.0F;
                    return std::cos(angle);
                };
                light.cos_inner = special_cosine(inner);
                light.cos_outer = special_cosine(outer);
                light.hard = inner == outer;
                if (!std::isfinite(light.cos_inner) || !std::isfinite(light.cos_outer) || light.cos_outer == 1.0F ||
                    light.cos_outer == -1.0F || (inner > 0.0F && light.cos_inner == 1.0F) ||
                    light.cos_inner < light.cos_outer || (inner < outer && light.cos_inner == light.cos_outer)) {
                    set_error("Spot cone cosines are not distinguishable in the requested precision.");
                    delete s;
                    return 7;
                }
            } else {
                set_error("unknown punctual light kind");
                delete s;
                return 7;
            }
            s->punctual.push_back(light);
        }
        // Mesh-light registry (FrameScene.cpp:201-261): one light per emissive instance.
        s->light_of_instance.assign(d->instance_count, -1);
        for (uint32_t i = 0; i < d->instance_count; ++i) {
            const Material& mat = s->materials[s->instances[i].material];
            if (is_black(mat.emission)) {
                continue;
            }
            if (s->geometries[s->instances[i].geometry].kind == BF200_GEOMETRY_SPHERE) {
                set_error("emissive analytic spheres are not supported: lights are meshes");
                delete s;
                return 3;
            }
            MeshLight light{};
            light.instance = i;
            if (!transform_mesh_positions(*s, s->instances[i], light)) {
                set_error("An emissive mesh world position is not representable.");
                delete s;
                return 3;
            }
            const auto& g = s->geometries[s->instances[i].geometry];
            light.tris.assign(&s->triangles[3 * g.triangle_offset],
                              &s->triangles[3 * (g.triangle_offset + g.triangle_count)]);
            if (!build_mesh_light(light)) {
                set_error("A mesh area light could not be built.");
                delete s;
                return 4;
            }
            light.radiance = mat.emission;
            s->light_of_instance[i] = static_cast<int32_t>(s->lights.size());
            s->lights.push_back(std::move(light));
        }
        // LightSampler::create_uniform (LightSampler.cpp:574-602) over the registry: punctual
        // lights, then mesh lights.
        const size_t count = s->punctual.size() + s->lights.size();
        if (count == 0) {
            set_error("MIS requires at least one punctual or emissive mesh light in the committed scene.");
            delete s;
            return 5;
        }
        s->light_cdf.assign(count + 1, 0.0F);
        for (size_t k = 1; k < count; ++k) {
            s->light_cdf[k] = static_cast<float>(k) / static_cast<float>(count);
        }
        s->light_cdf[count] = 1.0F;
        for (int lane = 0; lane < 4; ++lane) {
            s->environment[lane] = d->environment_radiance[lane];
            s->nm[lane] = d->wavelength_nanometers[lane];
            s->pdf[lane] = d->wavelength_pdf[lane];
        }
        *out = s;
        return 0;
    } catch (const Failure& f) {
        set_error(f.message);
        return 1;
    }
}

__attribute__((visibility("default"))) void bfo_scene_destroy(void* s) { delete static_cast<Scene*>(s); }

__attribute__((visibility("default"))) void bfo_scene_set_prefilter(void* s, int enabled) {
    static_cast<Scene*>(s)->prefilter = enabled != 0;
}

// Writes the world-space geometric normal of (instance, primitive) as the backend resolves it.
__attribute__((visibility("default"))) int bfo_scene_world_normal(void* h, uint32_t instance,
                                                                  uint32_t primitive, float* out3) {
    const auto* s = static_cast<Scene*>(h);
    if (instance >= s->instances.size() || primitive >= s->instances[instance].world_normals.size()) {
        return 1;
    }
    const V3 n = s->instances[instance].world_normals[primitive];
    out3[0] = n.x;
    out3[1] = n.y;
    out3[2] = n.z;
    return 0;
}

// Traces paths; returns how many failed (lane_status 1, first message in bfo_last_error()).
// cones_in / cones_out (both or neither, 2 floats per path) carry the ray cones.
static int64_t trace_batch(void* h, const bf200_path_input_v1* in, const bf200_path_state_v1* states,
                           const float* cones_in, uint64_t n, const bf200_transport_options_v1* o,
                           bf200_path_result_v1* res, float* cones_out, int threads) {
    const auto* s = static_cast<Scene*>(h);
    const Options opt = make_options(*o);
    std::atomic<uint64_t> next{0};
    std::atomic<int64_t> failures{0};
    auto worker = [&] {
        for (uint64_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) {
            try {
                const PathOut p = trace(*s, in[i], opt, cones_in != nullptr ? cones_in + 2 * i : nullptr,
                                        states != nullptr ? states + i : nullptr);
                store_result(p, res[i], in[i].primary_ray.time, in[i].primary_ray.mask);
                if (cones_out != nullptr) {
                    cones_out[2 * i] = p.cone_width;
                    cones_out[2 * i + 1] = p.cone_spread;
                }
            } catch (const Failure& f) {
                std::memset(&res[i], 0, sizeof(res[i]));
                res[i].lane_status = BF200_LANE_NUMERICAL_FAILURE;
                if (cones_out != nullptr) {
                    cones_out[2 * i] = cones_out[2 * i + 1] = 0.0F;
                }
                if (failures.fetch_add(1) == 0) {
                    set_error(f.message);
                }
            }
        }
    };
    if (threads <= 1) {
        worker();
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) {
            pool.emplace_back(worker);
        }
        for (auto& t : pool) {
            t.join();
        }
    }
    return failures.load();
}

__attribute__((visibility("default"))) int64_t bfo_trace_paths(void* h, const bf200_path_input_v1* in,
                                                               uint64_t n,
                                                               const bf200_transport_options_v1* o,
                                                               bf200_path_result_v1* res, int threads) {
    return trace_batch(h, in, nullptr, nullptr, n, o, res, nullptr, threads);
}

// Float64 gradient of a loss with respect to every material's closure weight (per packet lane) and
// a common emitter radiance scale, along the float transport's own paths. path_adjoint holds
// dLoss/dL per path and lane. With the sampled directions fixed every radiance contribution is a
// product in which the closure weight of each scattering vertex before it appears once (Lambert: in
// the throughput update; GGX and specular: in the BSDF value) and an emitter's radiance at most
// once, so its derivative with respect to material m's lane-l weight is value * (vertices of m) /
// weight. The sums run in double over the recorded contributions; they restate the derivative
// independently of the device replay's per-vertex "radiance after this vertex" bookkeeping.
// Materials must be single closures. Returns the number of failed paths (left out).
__attribute__((visibility("default"))) int64_t bfo_weight_gradients(void* h, const bf200_path_input_v1* in, uint64_t n,
                                                                    const bf200_transport_options_v1* o,
                                                                    const double* path_adjoint, double* gradients,
                                                                    double* emission_gradient) {
    const auto* s = static_cast<Scene*>(h);
    const Options opt = make_options(*o);
    const size_t materials = s->materials.size();
    std::vector<double> g(materials * 4, 0.0);
    double e = 0.0;
    int64_t failures = 0;
    for (uint64_t i = 0; i < n; ++i) {
        PathRecord record;
        try {
            trace(*s, in[i], opt, nullptr, nullptr, &record);
        } catch (const Failure&) {
            ++failures;
            continue;
        }
        const double* adj = path_adjoint + 4 * i;
        for (const auto& c : record.contributions) {
            for (int lane = 0; lane < 4; ++lane) {
                const double weighted = adj[lane] * c.value[lane];
                if (weighted == 0.0) {
                    continue;
                }
                if (c.emitter) {
                    e += weighted;
                }
                for (uint32_t v = 0; v < c.vertices; ++v) {
                    const uint32_t m = record.materials[v];
                    const float w = s->materials[m].closures[0].weight[lane];
                    if (w != 0.0F) {
                        g[4 * m + lane] += weighted / w;
                    }
                }
            }
        }
    }
    std::memcpy(gradients, g.data(), g.size() * sizeof(double));
    *emission_gradient = e;
    return failures;
}

// bfo_trace_paths with ray cones (width, spread per path) in and at every terminal-ray origin out,
// and optional depth-zero initial states (null: PathState::create_initial).
__attribute__((visibility("default"))) int64_t bfo_trace_paths_cones(void* h, const bf200_path_input_v1* in,
                                                                     const bf200_path_state_v1* states,
                                                                     const float* cones_in, uint64_t n,
                                                                     const bf200_transport_options_v1* o,
                                                                     bf200_path_result_v1* res, float* cones_out,
                                                                     int threads) {
    return trace_batch(h, in, states, cones_in, n, o, res, cones_out, threads);
}

// One ray-cone advance per case: cones (width, spread), ray directions, hit parameters; writes the
// advanced width (NaN where the advance fails). Returns the number of failures.
__attribute__((visibility("default"))) int64_t bfo_cone_advance(const float* cones, const float* directions,
                                                                const float* parameters, uint64_t n,
                                                                float* widths) {
    int64_t failures = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const V3 d{directions[3 * i], directions[3 * i + 1], directions[3 * i + 2]};
        float width = 0.0F;
        if (!cone_advance(cones[2 * i], cones[2 * i + 1], d, parameters[i], width)) {
            width = std::numeric_limits<float>::quiet_NaN();
            ++failures;
        }
        widths[i] = width;
    }
    return failures;
}

// One ray-cone scattering per case: cone (width, spread), closure kind and its 10 parameters, the
// event lobes, local wo and wi; writes (width, spread), NaN where it fails. Returns the failures.
__attribute__((visibility("default"))) int64_t bfo_cone_scatter(const float* cones, const uint32_t* kinds,
                                                                const float* parameters, const uint32_t* events,
                                                                const float* wo, const float* wi, uint64_t n,
                                                                float* out) {
    int64_t failures = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const V3 o{wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]};
        const V3 w{wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]};
        float width = 0.0F, spread = 0.0F;
        if (!cone_scatter(cones[2 * i], cones[2 * i + 1], kinds[i], parameters + 10 * i, events[i], o, w, width,
                          spread)) {
            width = spread = std::numeric_limits<float>::quiet_NaN();
            ++failures;
        }
        out[2 * i] = width;
        out[2 * i + 1] = spread;
    }
    return failures;
}

// Closest hits for world rays (the accel contract; AccelBackend.cpp:43-112).
__attribute__((visibility("default"))) int bfo_closest_hits(void* h, const bf200_ray_v1* rays, uint64_t n,
                                                            bf200_hit_v1* hits) {
    const auto* s = static_cast<Scene*>(h);
    for (uint64_t i = 0; i < n; ++i) {
        std::memset(&hits[i], 0, sizeof(hits[i]));
        hits[i].instance_index = 0xFFFFFFFFU;
        hits[i].primitive_index = 0xFFFFFFFFU;
        try {
            Hit hit{};
            const V3 o{rays[i].origin[0], rays[i].origin[1], rays[i].origin[2]};
            const V3 d{rays[i].direction[0], rays[i].direction[1], rays[i].direction[2]};
            if (closest_hit(*s, o, d, rays[i].t_min, rays[i].t_max, rays[i].mask, hit)) {
                hits[i].t = hit.t;
                hits[i].barycentrics[0] = hit.b0;
                hits[i].barycentrics[1] = hit.b1;
                hits[i].barycentrics[2] = hit.b2;
                hits[i].instance_index = hit.instance;
                hits[i].primitive_index = hit.primitive;
            }
        } catch (const Failure& f) {
            hits[i].status = BF200_LANE_NUMERICAL_FAILURE;
            set_error(f.message);
        }
    }
    return 0;
}

// PinholeCamera::generate_primary_ray with uniform pixel jitter (PinholeCamera.hpp:144-283,
// PixelJitter.hpp:47-64) for a camera whose frame and half extents are given.
// `sampler` selects the jitter's sampler (BF200_SAMPLER_*).
__attribute__((visibility("default"))) int bfo_camera_rays_sampled(const bf200_camera_v1* cam,
                                                                   const bf200_sample_index_v1* samples, uint64_t n,
                                                                   uint32_t sampler, bf200_ray_v1* rays) {
    try {
        for (uint64_t i = 0; i < n; ++i) {
            const Stream stream{samples[i].pixel_x, samples[i].pixel_y, samples[i].sample_index, samples[i].seed,
                                sampler == 1U};
            float ox = 0.5F, oy = 0.5F;
            if (cam->jitter_mode != 0) {
                ox = stream.sample_1d(0xA24BAED4963EE407ULL);
                oy = stream.sample_1d(0x9FB21C651E98DF25ULL);
            }
            const float rw = static_cast<float>(cam->width), rh = static_cast<float>(cam->height);
            const float tpx = 2.0F * static_cast<float>(samples[i].pixel_x);
            const float tpy = 2.0F * static_cast<float>(samples[i].pixel_y);
            const float nx = (tpx + 2.0F * ox) / rw - 1.0F;
            const float ny = 1.0F - (tpy + 2.0F * oy) / rh;
            const V3 local = robust_unit(V3{nx * cam->half_width, ny * cam->half_height, -1.0F});
            const Frame frame{V3{cam->tangent[0], cam->tangent[1], cam->tangent[2]},
                              V3{cam->bitangent[0], cam->bitangent[1], cam->bitangent[2]},
                              V3{cam->normal[0], cam->normal[1], cam->normal[2]}};
            const V3 d = robust_unit(frame.to_world(local));
            std::memset(&rays[i], 0, sizeof(rays[i]));
            for (int a = 0; a < 3; ++a) {
                rays[i].origin[a] = cam->origin[a];
            }
            rays[i].direction[0] = d.x;
            rays[i].direction[1] = d.y;
            rays[i].direction[2] = d.z;
            rays[i].t_min = cam->t_min;
            rays[i].t_max = cam->t_max;
            rays[i].time = cam->time;
            rays[i].mask = cam->mask;
        }
        return 0;
    } catch (const Failure& f) {
        set_error(f.message);
        return 1;
    }
}

__attribute__((visibility("default"))) int bfo_camera_rays(const bf200_camera_v1* cam,
                                                           const bf200_sample_index_v1* samples, uint64_t n,
                                                           bf200_ray_v1* rays) {
    return bfo_camera_rays_sampled(cam, samples, n, 0U, rays);
}

__attribute__((visibility("default"))) uint64_t bfo_sobol_bits(uint64_t sample_index, uint64_t dimension) {
    return sobol_coordinate(sample_index, dimension);
}

__attribute__((visibility("default"))) uint64_t bfo_owen_sobol_bits(uint32_t px, uint32_t py, uint64_t sample_index,
                                                                    uint64_t seed, uint64_t dimension) {
    return owen_coordinate(px, py, sample_index, seed, dimension);
}

// Float32 or Neumaier float64 film of the caller-side path: CIE XYZ (Cie1931Sensor.cpp:104-176),
// linear sRGB (Color.hpp:77-88), add_sample(x, y, rgb, 1) (Film.hpp:150-182). `sums` holds
// (r, g, b, weight) per pixel as double; for precision 1 also the compensations are applied.
// LightSampler::create_power_weighted (LightSampler.cpp:605-625, power_weights :200-245,
// build_power_cdf :117-190, add_compensated :78-95) restated: the scene's selection CDF from four-
// lane spectral powers. Returns 0, or 1 with the reason in last_error.
bool neumaier_add(float value, float& sum, float& correction) {
    if (!std::isfinite(value) || value < 0.0F) {
        return false;
    }
    const float next = sum + value;
    if (!std::isfinite(next)) {
        return false;
    }
    correction += sum >= value ? (sum - next) + value : (value - next) + sum;
    if (!std::isfinite(correction)) {
        return false;
    }
    sum = next;
    return true;
}

// Installs the spatial light tree of the scene's mesh lights (bounds and spectral power per light,
// in registry order); selection and MIS then follow the tree.
__attribute__((visibility("default"))) int bfo_scene_set_light_tree(void* handle,
                                                                    const bf200_light_tree_input_v1* lights,
                                                                    uint32_t count) {
    auto* s = static_cast<Scene*>(handle);
    if (count != s->punctual.size() + s->lights.size()) {
        set_error("one light-tree input per scene light is required");
        return 1;
    }
    std::string error;
    if (bf200::build_light_tree(lights, count, s->tree, error) != BLACKFRAME_STATUS_SUCCESS) {
        set_error(error.c_str());
        return 1;
    }
    s->use_tree = true;
    return 0;
}

__attribute__((visibility("default"))) int bfo_scene_set_light_powers(void* handle, const float* powers,
                                                                      uint32_t count) {
    auto* s = static_cast<Scene*>(handle);
    if (count == 0 || count != s->punctual.size() + s->lights.size()) {
        set_error("one spectral power per scene light is required");
        return 1;
    }
    float peak = 0.0F;
    for (uint64_t i = 0; i < 4ULL * count; ++i) {
        if (!std::isfinite(powers[i]) || powers[i] < 0.0F) {
            set_error("Power-weighted light sampling requires finite non-negative spectral lanes.");
            return 1;
        }
        peak = std::max(peak, powers[i]);
    }
    if (peak == 0.0F) {
        set_error("Power-weighted light sampling requires positive spectral power.");
        return 1;
    }
    std::vector<float> weights(count);
    for (uint32_t i = 0; i < count; ++i) {
        float sum = 0.0F, correction = 0.0F;
        for (int l = 0; l < 4; ++l) {
            if (!neumaier_add(powers[4 * i + l] / peak, sum, correction)) {
                set_error("A spectral light-selection weight is not representable.");
                return 1;
            }
        }
        weights[i] = sum + correction;
    }
    float ts = 0.0F, tc = 0.0F;
    for (float w : weights) {
        if (!neumaier_add(w, ts, tc)) {
            set_error("Light-selection power accumulation is not representable.");
            return 1;
        }
    }
    const float total = ts + tc;
    if (!(total > 0.0F)) {
        set_error("Power-weighted light sampling requires positive spectral power.");
        return 1;
    }
    uint32_t last = count;
    for (uint32_t i = count; i > 0; --i) {
        if (weights[i - 1] > 0.0F) {
            last = i - 1;
            break;
        }
    }
    std::vector<float> cdf(count + 1, 0.0F);
    float ps = 0.0F, pc = 0.0F, previous = 0.0F;
    for (uint32_t i = 0; i < count; ++i) {
        if (weights[i] == 0.0F) {
            cdf[i + 1] = previous;
            continue;
        }
        if (!neumaier_add(weights[i], ps, pc)) {
            set_error("Light-selection power prefix is not representable.");
            return 1;
        }
        const float boundary = i != last ? (ps + pc) / total : 1.0F;
        if (i != last && !(boundary > previous && boundary < 1.0F)) {
            set_error("A positive light-selection probability is not representable.");
            return 1;
        }
        cdf[i + 1] = boundary;
        previous = boundary;
    }
    s->light_cdf = cdf;
    return 0;
}

// intersect_sphere on ray k against sphere k (centre xyz, radius), in world space. Per ray, out
// receives 8 floats: status (0 miss, 1 hit, 2 not representable), t, outward normal xyz, position xyz.
__attribute__((visibility("default"))) int bfo_sphere_intersect(const float* spheres, const bf200_ray_v1* rays,
                                                                uint64_t count, float* out) {
    for (uint64_t k = 0; k < count; ++k) {
        float* o = out + 8 * k;
        for (int i = 0; i < 8; ++i) {
            o[i] = 0.0F;
        }
        const float* sp = spheres + 4 * k;
        const auto& r = rays[k];
        const V3 origin{r.origin[0], r.origin[1], r.origin[2]}, dir{r.direction[0], r.direction[1], r.direction[2]};
        if (!std::isfinite(sp[0]) || !std::isfinite(sp[1]) || !std::isfinite(sp[2]) || !std::isfinite(sp[3]) ||
            sp[3] <= 0.0F) {
            o[0] = 2.0F;
            continue;
        }
        float t = 0.0F;
        V3 n{};
        const SphereResult res = intersect_sphere(V3{sp[0], sp[1], sp[2]}, sp[3], origin, dir, r.t_min, r.t_max, t, n);
        if (res == SphereResult::failure) {
            o[0] = 2.0F;
            continue;
        }
        if (res == SphereResult::miss) {
            continue;
        }
        const V3 p = origin + dir * t;
        o[0] = 1.0F;
        o[1] = t;
        o[2] = n.x;
        o[3] = n.y;
        o[4] = n.z;
        o[5] = p.x;
        o[6] = p.y;
        o[7] = p.z;
    }
    return 0;
}

__attribute__((visibility("default"))) int bfo_film_accumulate(const float* radiance,
                                                               const bf200_sample_index_v1* samples,
                                                               uint64_t n, const bf200_sensor_v1* sensor,
                                                               uint32_t width, uint32_t height,
                                                               uint32_t precision, double* out_sums,
                                                               uint64_t* out_counts) {
    const size_t pixels = size_t(width) * height;
    std::vector<float> f32(4 * pixels, 0.0F);
    std::vector<double> f64(8 * pixels, 0.0);
    std::vector<uint64_t> counts(pixels, 0);
    for (uint64_t i = 0; i < n; ++i) {
        float xyz[3] = {0.0F, 0.0F, 0.0F};
        for (int lane = 0; lane < 4; ++lane) {
            const float c = radiance[4 * i + lane];
            for (int k = 0; k < 3; ++k) {
                const float r = sensor->response_xyz[lane][k];
                float term = 0.0F;
                if (c != 0.0F && r != 0.0F) {
                    int ec = 0, er = 0, en = 0, ep = 0;
                    const float mc = std::frexp(c, &ec);
                    const float mr = std::frexp(r, &er);
                    const float mn = std::frexp(sensor->normalization, &en);
                    const float mp = std::frexp(sensor->wavelength_pdf[lane], &ep);
                    const float mantissa = mc * mr * mn / mp;
                    term = std::ldexp(mantissa, ec + er + en - ep);
                }
                xyz[k] += term;
            }
        }
        const float red = 3.2404542F * xyz[0] - 1.5371385F * xyz[1] - 0.4985314F * xyz[2];
        const float green = -0.9692660F * xyz[0] + 1.8760108F * xyz[1] + 0.0415560F * xyz[2];
        const float blue = 0.0556434F * xyz[0] - 0.2040259F * xyz[1] + 1.0572252F * xyz[2];
        const size_t p = size_t(samples[i].pixel_y) * width + samples[i].pixel_x;
        if (precision == 0) {
            f32[4 * p + 0] += red * 1.0F;
            f32[4 * p + 1] += green * 1.0F;
            f32[4 * p + 2] += blue * 1.0F;
            f32[4 * p + 3] += 1.0F;
        } else {
            const double values[4] = {double(red) * 1.0, double(green) * 1.0, double(blue) * 1.0, 1.0};
            for (int k = 0; k < 4; ++k) {
                double& sum = f64[8 * p + k];
                double& comp = f64[8 * p + 4 + k];
                const double updated = sum + values[k];
                if (std::abs(sum) >= std::abs(values[k])) {
                    comp += (sum - updated) + values[k];
                } else {
                    comp += (values[k] - updated) + sum;
                }
                sum = updated;
            }
        }
        ++counts[p];
    }
    for (size_t p = 0; p < pixels; ++p) {
        for (int k = 0; k < 4; ++k) {
            out_sums[4 * p + k] = precision == 0 ? double(f32[4 * p + k]) : f64[8 * p + k] + f64[8 * p + 4 + k];
        }
        out_counts[p] = counts[p];
    }
    return 0;
}

}  // extern "C"
