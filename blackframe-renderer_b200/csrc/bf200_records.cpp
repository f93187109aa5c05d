// Host checks of scene records (see bf200_records.h). Compiled with floating-point contraction
// off, like the reference's scalar build.
#include "bf200_records.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <utility>

namespace bf200 {
namespace {

// Exactly collinear vertices: every component of (v1 - v0) x (v2 - v0) is zero. The edges and
// products are formed in long double arithmetic from exact double differences where they are exact.
bool collinear(const float* a, const float* b, const float* c) {
    const long double e1[3] = {static_cast<long double>(b[0]) - a[0], static_cast<long double>(b[1]) - a[1],
                               static_cast<long double>(b[2]) - a[2]};
    const long double e2[3] = {static_cast<long double>(c[0]) - a[0], static_cast<long double>(c[1]) - a[1],
                               static_cast<long double>(c[2]) - a[2]};
    return e1[1] * e2[2] == e1[2] * e2[1] && e1[2] * e2[0] == e1[0] * e2[2] && e1[0] * e2[1] == e1[1] * e2[0];
}

}  // namespace

bool unit_normal(float x, float y, float z) {
    const float squared = std::fma(x, x, std::fma(y, y, z * z));
    const float tolerance = std::numeric_limits<float>::epsilon() * 256.0F;
    return std::isfinite(squared) && std::abs(squared - 1.0F) <= tolerance;
}

// The payload checks of ClosureSet's append_* (ClosureSet.hpp:76-111, 140-260): reflectances in
// [0, 1], conductor eta > 0 and k >= 0, dielectric etas > 0 and distinct, a representable GGX
// alpha pair (GgxMicrofacet.hpp:62-104), and the lobes each kind is appended with.
bool unit_interval4(const float* v) {
    for (int i = 0; i < 4; ++i) {
        if (!std::isfinite(v[i]) || v[i] < 0.0F || v[i] > 1.0F) {
            return false;
        }
    }
    return true;
}

bool representable_alpha_pair(float alpha_x, float alpha_y) {
    if (!std::isfinite(alpha_x) || !(alpha_x > 0.0F) || !std::isfinite(alpha_y) || !(alpha_y > 0.0F)) {
        return false;
    }
    const float maximum_alpha = std::sqrt(std::numeric_limits<float>::max()) * std::sqrt(3.14159265358979323846F);
    const float minimum_alpha = 1.0F / maximum_alpha;
    if (alpha_x < minimum_alpha || alpha_x > maximum_alpha || alpha_y < minimum_alpha || alpha_y > maximum_alpha) {
        return false;
    }
    if (alpha_x == alpha_y) {
        return true;
    }
    // D = 1 / (pi ax ay q^4) with q between min and max of {1, 1/ax, 1/ay}: both extremes of the
    // density must stay inside float range (evaluated in logs, in long double)
    using Wide = long double;
    const Wide ax = alpha_x, ay = alpha_y;
    const Wide min_q = std::min({Wide{1}, Wide{1} / ax, Wide{1} / ay});
    const Wide max_q = std::max({Wide{1}, Wide{1} / ax, Wide{1} / ay});
    const Wide log_scale = std::log(Wide{1} / Wide{3.141592653589793238462643383279502884L}) - std::log(ax) -
                           std::log(ay);
    const Wide max_log_density = log_scale - Wide{4} * std::log(min_q);
    const Wide min_log_density = log_scale - Wide{4} * std::log(max_q);
    return std::isfinite(max_log_density) && std::isfinite(min_log_density) &&
           max_log_density <= std::log(static_cast<Wide>(std::numeric_limits<float>::max())) &&
           min_log_density >= std::log(static_cast<Wide>(std::numeric_limits<float>::denorm_min()));
}

bool valid_closure_payload(const bf200_closure_v1& c) {
    const float* p = c.parameters;
    if (!unit_interval4(c.weight)) {
        return false;
    }
    switch (c.kind) {
    case BF200_CLOSURE_LAMBERTIAN_REFLECTION:
        return c.lobes == (BF200_LOBE_DIFFUSE | BF200_LOBE_REFLECTION);
    case BF200_CLOSURE_ROUGH_CONDUCTOR_REFLECTION:
        for (int i = 0; i < 4; ++i) {
            if (!std::isfinite(p[i]) || !(p[i] > 0.0F) || !std::isfinite(p[4 + i]) || p[4 + i] < 0.0F) {
                return false;
            }
        }
        return c.lobes == (BF200_LOBE_GLOSSY | BF200_LOBE_REFLECTION) && representable_alpha_pair(p[8], p[9]);
    case BF200_CLOSURE_ROUGH_DIELECTRIC:
        return c.lobes == (BF200_LOBE_GLOSSY | BF200_LOBE_REFLECTION | BF200_LOBE_TRANSMISSION) &&
               std::isfinite(p[0]) && p[0] > 0.0F && std::isfinite(p[1]) && p[1] > 0.0F && p[0] != p[1] &&
               representable_alpha_pair(p[2], p[3]);
    case BF200_CLOSURE_ROUGH_DIFFUSE_REFLECTION:  // append_rough_diffuse_reflection: roughness in [0, 1]
        for (int i = 1; i < 10; ++i) {
            if (p[i] != 0.0F) {
                return false;
            }
        }
        return c.lobes == (BF200_LOBE_DIFFUSE | BF200_LOBE_REFLECTION) && std::isfinite(p[0]) && p[0] >= 0.0F &&
               p[0] <= 1.0F;
    case BF200_CLOSURE_SPECULAR_REFLECTION:
        for (int i = 0; i < 10; ++i) {
            if (p[i] != 0.0F) {
                return false;
            }
        }
        return c.lobes == (BF200_LOBE_SPECULAR | BF200_LOBE_REFLECTION);
    case BF200_CLOSURE_SPECULAR_TRANSMISSION:  // append_specular_transmission: finite positive indices
        for (int i = 2; i < 10; ++i) {
            if (p[i] != 0.0F) {
                return false;
            }
        }
        return c.lobes == (BF200_LOBE_SPECULAR | BF200_LOBE_TRANSMISSION) && std::isfinite(p[0]) && p[0] > 0.0F &&
               std::isfinite(p[1]) && p[1] > 0.0F;
    default:
        return false;
    }
}

// build_component_distribution (ClosureMixture.hpp:122-234): the component probabilities of a
// closure mixture projected onto the 2^-24 sampler grid (largest remainders first) and their CDF.
// False when the probabilities do not form a distribution at that precision.
bool project_component_distribution(const float* probabilities, uint32_t n, float* out_p, float* out_cdf) {
    for (uint32_t i = 0; i <= kClosureCapacity; ++i) {
        out_cdf[i] = 0.0F;
        if (i < kClosureCapacity) {
            out_p[i] = 0.0F;
        }
    }
    if (n == 0U) {
        return true;
    }
    if (n > kClosureCapacity) {
        return false;
    }
    if (n == 1U) {
        out_p[0] = 1.0F;
        out_cdf[1] = 1.0F;
        return probabilities[0] == 1.0F;
    }
    constexpr int digits = 24;
    constexpr uint64_t scale = uint64_t{1} << digits;
    uint64_t masses[kClosureCapacity] = {};
    float remainders[kClosureCapacity] = {};
    uint64_t base_mass = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const float q = probabilities[i];
        if (!std::isfinite(q) || !(q > 0.0F) || !(q < 1.0F)) {
            return false;
        }
        const float scaled = std::ldexp(q, digits);
        const float base = std::floor(scaled);
        masses[i] = static_cast<uint64_t>(base);
        remainders[i] = scaled - base;
        base_mass += masses[i];
    }
    if (base_mass > scale) {
        return false;
    }
    float sum = 0.0F, correction = 0.0F;  // add_compensated over non-negative remainders
    for (uint32_t i = 0; i < n; ++i) {
        const float next = sum + remainders[i];
        correction += sum >= remainders[i] ? (sum - next) + remainders[i] : (remainders[i] - next) + sum;
        sum = next;
    }
    const uint64_t missing = scale - base_mass;
    if (missing > n ||
        std::fabs((sum + correction) - static_cast<float>(missing)) > 0.5F + std::numeric_limits<float>::epsilon() * 16.0F) {
        return false;
    }
    bool received[kClosureCapacity] = {};
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
            return false;
        }
        ++masses[selected];
        received[selected] = true;
    }
    uint64_t cumulative = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (masses[i] == 0U || cumulative > scale - masses[i]) {
            return false;
        }
        cumulative += masses[i];
        out_p[i] = std::ldexp(static_cast<float>(masses[i]), -digits);
        out_cdf[i + 1] = std::ldexp(static_cast<float>(cumulative), -digits);
    }
    return cumulative == scale && out_cdf[n] == 1.0F;
}

bool unit_direction3(const float* d) {  // unit_direction: squared length within 128 ulp of one
    if (!std::isfinite(d[0]) || !std::isfinite(d[1]) || !std::isfinite(d[2])) {
        return false;
    }
    const float squared = std::fma(d[0], d[0], std::fma(d[1], d[1], d[2] * d[2]));
    return std::isfinite(squared) && std::fabs(squared - 1.0F) <= 128.0F * std::numeric_limits<float>::epsilon();
}

// exact_special_cosine (PunctualLights.hpp:186-197)
float special_cosine(float angle) {
    constexpr float pi = 3.14159265358979323846F;
    if (angle == 0.0F) {
        return 1.0F;
    }
    if (angle == pi / 2.0F) {
        return 0.0F;
    }
    if (angle == pi) {
        return -1.0F;
    }
    return std::cos(angle);
}


uint32_t closure_lobes(uint32_t kind) {
    switch (kind) {
    case BF200_CLOSURE_LAMBERTIAN_REFLECTION:
    case BF200_CLOSURE_ROUGH_DIFFUSE_REFLECTION:
        return BF200_LOBE_DIFFUSE | BF200_LOBE_REFLECTION;
    case BF200_CLOSURE_ROUGH_CONDUCTOR_REFLECTION:
        return BF200_LOBE_GLOSSY | BF200_LOBE_REFLECTION;
    case BF200_CLOSURE_ROUGH_DIELECTRIC:
        return BF200_LOBE_GLOSSY | BF200_LOBE_REFLECTION | BF200_LOBE_TRANSMISSION;
    case BF200_CLOSURE_SPECULAR_REFLECTION:
        return BF200_LOBE_SPECULAR | BF200_LOBE_REFLECTION;
    case BF200_CLOSURE_SPECULAR_TRANSMISSION:
        return BF200_LOBE_SPECULAR | BF200_LOBE_TRANSMISSION;
    default:
        return 0U;
    }
}

bool punctual_light_checks(const bf200_punctual_light_v1& src, float& cos_inner, float& cos_outer) {
    constexpr float pi = 3.14159265358979323846F;
    for (int l = 0; l < 4; ++l) {
        if (!std::isfinite(src.spectrum[l]) || src.spectrum[l] < 0.0F) {
            return false;
        }
    }
    if (src.reserved != 0U) {
        return false;
    }
    bool finite_point = true;
    for (int a = 0; a < 3; ++a) {
        finite_point = finite_point && std::isfinite(src.position[a]) && std::isfinite(src.position_error[a]) &&
                       src.position_error[a] >= 0.0F;
    }
    if (src.kind == BF200_PUNCTUAL_POINT) {
        return finite_point;
    }
    if (src.kind == BF200_PUNCTUAL_DIRECTIONAL) {
        return unit_direction3(src.direction);
    }
    if (src.kind != BF200_PUNCTUAL_SPOT || !finite_point || !unit_direction3(src.direction)) {
        return false;
    }
    const float inner = src.inner_half_angle, outer = src.outer_half_angle;
    if (!std::isfinite(inner) || !std::isfinite(outer) || inner < 0.0F || inner > outer || !(outer > 0.0F) ||
        outer >= pi) {
        return false;
    }
    cos_inner = special_cosine(inner);
    cos_outer = special_cosine(outer);
    return std::isfinite(cos_inner) && std::isfinite(cos_outer) && cos_outer != 1.0F && cos_outer != -1.0F &&
           !(inner > 0.0F && cos_inner == 1.0F) && !(cos_inner < cos_outer) &&
           !(inner < outer && cos_inner == cos_outer);
}

bool invert_matrix4(const float (&m)[16], float (&out)[16]) {
    float a[32];
    for (int r = 0; r < 4; ++r) {
        for (int c = 0; c < 4; ++c) {
            if (!std::isfinite(m[r * 4 + c])) {
                return false;
            }
            a[r * 8 + c] = m[r * 4 + c];
            a[r * 8 + c + 4] = r == c ? 1.0F : 0.0F;
        }
    }
    for (int pc = 0; pc < 4; ++pc) {
        int pr = pc;
        float magnitude = std::abs(a[pr * 8 + pc]);
        for (int cand = pc + 1; cand < 4; ++cand) {
            const float cm = std::abs(a[cand * 8 + pc]);
            if (cm > magnitude) {
                magnitude = cm;
                pr = cand;
            }
        }
        if (magnitude == 0.0F) {
            return false;
        }
        if (pr != pc) {
            for (int c = 0; c < 8; ++c) {
                std::swap(a[pc * 8 + c], a[pr * 8 + c]);
            }
        }
        const float pivot = a[pc * 8 + pc];
        for (int c = 0; c < 8; ++c) {
            a[pc * 8 + c] /= pivot;
        }
        for (int r = 0; r < 4; ++r) {
            if (r == pc) {
                continue;
            }
            const float factor = a[r * 8 + pc];
            for (int c = 0; c < 8; ++c) {
                a[r * 8 + c] -= factor * a[pc * 8 + c];
            }
        }
    }
    for (int r = 0; r < 4; ++r) {
        for (int c = 0; c < 4; ++c) {
            out[r * 4 + c] = a[r * 8 + c + 4];
            if (!std::isfinite(out[r * 4 + c])) {
                return false;
            }
        }
    }
    return true;
}

const char* triangle_mesh_problem(const float* positions, const float* normals, const float* uvs,
                                  uint64_t vertices, const uint32_t* triangles, uint64_t triangle_count) {
    if (vertices == 0) {
        return "A triangle mesh requires at least one aligned vertex.";
    }
    if (triangle_count == 0) {
        return "A triangle mesh requires at least one indexed triangle.";
    }
    for (uint64_t i = 0; i < 3 * vertices; ++i) {
        if (!std::isfinite(positions[i])) {
            return "Triangle mesh positions must contain only finite values.";
        }
    }
    for (uint64_t i = 0; i < vertices; ++i) {
        if (!unit_normal(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2])) {
            return "Triangle mesh normals must be finite unit-length values.";
        }
    }
    for (uint64_t i = 0; i < 2 * vertices; ++i) {
        if (!std::isfinite(uvs[i])) {
            return "Triangle mesh texture coordinates must contain only finite values.";
        }
    }
    for (uint64_t t = 0; t < triangle_count; ++t) {
        const uint32_t* tri = &triangles[3 * t];
        if (tri[0] >= vertices || tri[1] >= vertices || tri[2] >= vertices) {
            return "A triangle mesh index references an unknown aligned vertex.";
        }
        if (collinear(&positions[3ULL * tri[0]], &positions[3ULL * tri[1]], &positions[3ULL * tri[2]])) {
            return "A triangle mesh contains a degenerate or unrepresentable triangle.";
        }
    }
    return nullptr;
}

}  // namespace bf200
