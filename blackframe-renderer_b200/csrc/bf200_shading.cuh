// Device numerics of the transport: sampler, frames, closures, lights, MIS, Russian roulette.
//
// Every function keeps the operation order of the reference's scalar loop so that a lane's float
// results match the scalar oracle bit for bit; the file is compiled without FMA contraction and
// fmaf() appears exactly where the reference calls std::fma. References are to the reference
// repository (Blackframe/Renderer/Include/Blackframe/Renderer/...). A failed check sets the
// lane's error code (the reference returns an error for the whole path); the wavefront then
// retires the lane with that status instead of substituting a value.
#pragma once

#include "bf200_geometry.cuh"

namespace bf200 {

constexpr float kInf = __builtin_huge_valf();
constexpr float kEps = 1.1920928955078125e-7F;
constexpr float kDenormMin = 1.40129846e-45F;
constexpr float kInvPi = 0.318309886183790671538F;
constexpr float kPi = 3.14159265358979323846F;

constexpr uint32_t kLobeDiffuse = 0x01U, kLobeGlossy = 0x02U, kLobeSpecular = 0x04U;
constexpr uint32_t kLobeReflection = 0x08U, kLobeTransmission = 0x10U, kLobeVolume = 0x20U;
constexpr uint32_t kClosureLambert = 1U, kClosureRoughDiffuse = 2U, kClosureConductor = 3U, kClosureDielectric = 4U;
constexpr uint32_t kClosureSpecularReflection = 5U, kClosureSpecularTransmission = 6U;
constexpr uint32_t kMaxClosures = 8U;  // MaximumClosureCount (ClosureSet.hpp:15)

// Lane failure codes (include/bf200.h BF200_LANE_*)
constexpr uint32_t kLaneNumerical = 1U, kLaneUnsupported = 2U, kLaneTraversal = 3U;

struct Lane {
    uint32_t err = 0;
    __device__ __forceinline__ void fail(uint32_t code = kLaneNumerical) {
        if (err == 0) {
            err = code;
        }
    }
};

__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 operator-(F3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ F3 operator/(F3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ bool operator==(F3 a, F3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
__device__ __forceinline__ bool operator!=(F3 a, F3 b) { return !(a == b); }
__device__ __forceinline__ float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ bool finite3(F3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
__device__ __forceinline__ float max_abs3(F3 v) {
    return bf_max(bf_max(fabsf(v.x), fabsf(v.y)), fabsf(v.z));
}
__device__ __forceinline__ F3 ld3(const float4 v) { return {v.x, v.y, v.z}; }

// Sine and cosine of a float angle: the double-precision values rounded once to float. One
// out-of-line copy shared by every call site (one argument reduction for both values).
static __device__ __noinline__ float2 sincos_f(float a) {
    double s = 0.0, c = 0.0;
    sincos(static_cast<double>(a), &s, &c);
    return make_float2(static_cast<float>(s), static_cast<float>(c));
}

// ------------------------------------------------------------------------------------------------
// SampleStream (SampleStream.hpp:23-67) and SampleDimensionMap (SampleDimensionMap.cpp:47-68)
// ------------------------------------------------------------------------------------------------

BF_HD uint64_t mix_bits(uint64_t v) {
    v ^= v >> 30U;
    v *= 0xBF58476D1CE4E5B9ULL;
    v ^= v >> 27U;
    v *= 0x94D049BB133111EBULL;
    return v ^ (v >> 31U);
}

// ------------------------------------------------------------------------------------------------
// Owen-scrambled Sobol (SobolSampling.cpp:51-117, OwenScrambling.cpp:8-44). No reference transport
// draws from it; as a selectable transport sampler its dimension mapping is this backend's own:
// the two hashed camera-raster dimensions take Sobol dimensions 0 and 1, and every other sample
// dimension d (lens, time, wavelength 0..3; bounce b at 4 + 10 b + offset) takes Sobol dimension
// d + 2.
// ------------------------------------------------------------------------------------------------

constexpr uint64_t kSobolDimensions = 21201;

BF_HD uint64_t owen_pixel_hash(uint32_t px, uint32_t py) {
    return mix_bits((static_cast<uint64_t>(px) << 32U) | static_cast<uint64_t>(py));
}

// Key of the nested permutation of one (seed, pixel, Sobol dimension) (OwenScrambling.cpp:10-17).
BF_HD uint64_t owen_tree_key(uint64_t pixel_hash, uint64_t seed, uint64_t sobol_dimension) {
    return mix_bits(seed ^ mix_bits(sobol_dimension + 1U)) ^ pixel_hash;
}

// Nested binary scramble of the leading `depths` bits of a 64-bit coordinate (OwenScrambling.cpp:
// 19-33): the output bit at depth k flips with the hash of the tree node addressed by the input's
// first k bits. Output bits below the scrambled depths are zero.
BF_HD uint64_t owen_scramble(uint64_t input, uint64_t key, uint32_t depths) {
    uint64_t prefix = 0, output = 0;
    for (uint32_t depth = 0; depth < depths; ++depth) {
        const uint32_t shift = 63U - depth;
        const uint64_t bit = (input >> shift) & 1U;
        const uint64_t node = (1ULL << depth) | prefix;
        const uint64_t flip = mix_bits(key ^ node) >> 63U;
        output |= (bit ^ flip) << shift;
        prefix = (prefix << 1U) | bit;
    }
    return output;
}

constexpr uint64_t kCameraRasterX = 0xA24BAED4963EE407ULL;
constexpr uint64_t kCameraRasterY = 0x9FB21C651E98DF25ULL;

BF_HD uint64_t transport_sobol_dimension(uint64_t dimension) {
    return dimension == kCameraRasterX ? 0U : (dimension == kCameraRasterY ? 1U : dimension + 2U);
}

// Per-path sampler. The hash stream draws indexed_bits(seed, pixel, sample, dimension)
// (SampleStream.hpp:31-67); with `sobol` set it draws the Owen-scrambled Sobol coordinate of the
// path's sample index instead. `sobol` holds, per Sobol dimension, the leading 32 bits of the 64
// direction numbers: the 24 bits a float sample keeps (bits >> 40 of the 64-bit coordinate) depend
// only on the directions' leading bits, so only those and the first 24 scramble depths are
// evaluated, which leaves every float sample identical to the 64-bit computation.
struct Stream {
    uint64_t state;  // the (seed, pixel, sample) prefix of indexed_bits
    const uint32_t* sobol;
    uint64_t sample, seed, pixel_hash;
    __device__ __forceinline__ static Stream make(uint32_t px, uint32_t py, uint64_t sample, uint64_t seed,
                                                  const uint32_t* sobol) {
        const uint64_t packed = (static_cast<uint64_t>(px) << 32U) | static_cast<uint64_t>(py);
        uint64_t s = mix_bits(seed ^ 0x9E3779B97F4A7C15ULL);
        s = mix_bits(s ^ packed ^ 0xD1B54A32D192ED03ULL);
        s = mix_bits(s ^ sample ^ 0x8CB92BA72F3D8DD7ULL);
        Stream r;
        r.state = s;
        r.sobol = sobol;
        r.sample = sample;
        r.seed = seed;
        r.pixel_hash = sobol != nullptr ? owen_pixel_hash(px, py) : 0U;
        return r;
    }
    __device__ __forceinline__ float sample_1d(uint64_t dimension) const {
        if (sobol == nullptr) {
            const uint64_t bits = mix_bits(state ^ dimension);
            return static_cast<float>(bits >> 40U) * 0x1p-24F;
        }
        const uint64_t sd = transport_sobol_dimension(dimension);
        const uint32_t* heads = sobol + 64ULL * sd;
        uint64_t gray = sample ^ (sample >> 1U);
        uint32_t point = 0U;
        while (gray != 0U) {
            point ^= heads[__ffsll(static_cast<long long>(gray)) - 1];
            gray &= gray - 1U;
        }
        const uint64_t bits = owen_scramble(static_cast<uint64_t>(point) << 32U,
                                            owen_tree_key(pixel_hash, seed, sd), 24U);
        return static_cast<float>(bits >> 40U) * 0x1p-24F;
    }
};

__device__ __forceinline__ uint64_t bounce_base(uint32_t bounce) { return 4ULL + 10ULL * bounce; }

// ------------------------------------------------------------------------------------------------
// Frames and directions (LocalFrame.hpp, BsdfOnlyPathLoop.hpp:190-209)
// ------------------------------------------------------------------------------------------------

__device__ __forceinline__ F3 robust_unit(F3 d, Lane& lane) {
    if (!finite3(d)) {
        lane.fail();
        return d;
    }
    const float m = max_abs3(d);
    if (m == 0.0F) {
        lane.fail();
        return d;
    }
    const F3 s = d / m;
    const float magnitude = sqrtf(dot(s, s));
    const F3 r = s / magnitude;
    if (!finite3(r)) {
        lane.fail();
    }
    return r;
}

__device__ __forceinline__ bool unit_length(F3 d) {
    if (!finite3(d)) {
        return false;
    }
    const float sq = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
    return isfinite(sq) && fabsf(sq - 1.0F) <= kEps * 128.0F;
}

struct Frame {
    F3 t, b, n;
    __device__ __forceinline__ F3 to_local(F3 w) const { return {dot(w, t), dot(w, b), dot(w, n)}; }
    __device__ __forceinline__ F3 to_world(F3 l) const {
        return {t.x * l.x + b.x * l.y + n.x * l.z, t.y * l.x + b.y * l.y + n.y * l.z,
                t.z * l.x + b.z * l.y + n.z * l.z};
    }
};

__device__ __forceinline__ F3 robust_unit_vector(F3 v, Lane& lane) {
    const float m = max_abs3(v);
    if (!finite3(v) || m == 0.0F) {
        lane.fail();
        return v;
    }
    const F3 s = v / m;
    const float magnitude = sqrtf(dot(s, s));
    return s / magnitude;
}

__device__ __forceinline__ bool orthonormal(F3 t, F3 b, F3 n) {
    const float tol = kEps * 128.0F;
    return fabsf(dot(t, t) - 1.0F) <= tol && fabsf(dot(b, b) - 1.0F) <= tol &&
           fabsf(dot(n, n) - 1.0F) <= tol && fabsf(dot(t, b)) <= tol && fabsf(dot(t, n)) <= tol &&
           fabsf(dot(b, n)) <= tol && fabsf(dot(cross(t, b), n) - 1.0F) <= tol;
}

// LocalFrame.hpp:188-219
__device__ __forceinline__ Frame frame_from_unit_normal_and_tangent(F3 n, F3 tangent, Lane& lane) {
    const F3 td = robust_unit_vector(tangent, lane);
    const F3 projected = td - n * dot(td, n);
    F3 ut = robust_unit_vector(projected, lane);
    const F3 ub = robust_unit_vector(cross(n, ut), lane);
    ut = robust_unit_vector(cross(ub, n), lane);
    if (!orthonormal(ut, ub, n)) {
        lane.fail();
    }
    return Frame{ut, ub, n};
}

// LocalFrame.hpp:66-80 (from_normal), LocalFrame.hpp:8-30 (robust_unit_normal)
__device__ __forceinline__ Frame frame_from_normal(F3 v, Lane& lane) {
    const float m = max_abs3(v);
    if (!finite3(v) || m == 0.0F) {
        lane.fail();
        return Frame{};
    }
    const F3 s{v.x / m, v.y / m, v.z / m};
    const float magnitude = sqrtf(s.x * s.x + s.y * s.y + s.z * s.z);
    const F3 n{s.x / magnitude, s.y / magnitude, s.z / magnitude};
    const float sign = copysignf(1.0F, n.z);
    const float coefficient = -1.0F / (sign + n.z);
    const float product = n.x * n.y * coefficient;
    const F3 seed{1.0F + sign * n.x * n.x * coefficient, sign * product, -sign * n.x};
    return frame_from_unit_normal_and_tangent(n, seed, lane);
}

// LocalFrame.hpp:116-135
__device__ __forceinline__ Frame rotated_about_normal(const Frame& f, float angle, Lane& lane) {
    const float reduced = remainderf(angle, 2.0F * kPi);
    const float2 sc = sincos_f(reduced);
    const float c = sc.y;
    const float s = sc.x;
    const F3 rotated = f.t * c + f.b * s;
    return frame_from_unit_normal_and_tangent(f.n, rotated, lane);
}

// RayOriginOffset.hpp:58-117
__device__ __forceinline__ float outward(float value, float off) {
    if (off > 0.0F) {
        return nextafterf(value, kInf);
    }
    if (off < 0.0F) {
        return nextafterf(value, -kInf);
    }
    return value;
}

__device__ __forceinline__ F3 offset_ray_origin(F3 p, F3 err, F3 ng, F3 w, Lane& lane) {
    const float m = max_abs3(ng);
    const F3 sn = ng / m;
    const F3 n = sn / sqrtf(dot(sn, sn));
    const float d = fabsf(n.x) * err.x + fabsf(n.y) * err.y + fabsf(n.z) * err.z;
    if (!isfinite(d)) {
        lane.fail();
    }
    const float ds = max_abs3(w);
    const F3 sw = w / ds;
    F3 offset{n.x * d, n.y * d, n.z * d};
    if (dot(n, sw) < 0.0F) {
        offset = -offset;
    }
    const F3 shifted{outward(p.x + offset.x, offset.x), outward(p.y + offset.y, offset.y),
                     outward(p.z + offset.z, offset.z)};
    if (!finite3(shifted)) {
        lane.fail();
    }
    return shifted;
}

// ShadowRay.hpp:15-48
__device__ __forceinline__ F3 offset_surface_point(F3 p, F3 err, F3 ng, F3 w, Lane& lane) {
    const F3 offset = offset_ray_origin(p, err, ng, w, lane);
    if (offset != p) {
        return offset;
    }
    F3 oriented = ng;
    if (dot(ng, w) < 0.0F) {
        oriented = -oriented;
    }
    F3 s = p;
    if (oriented.x != 0.0F) s.x = nextafterf(p.x, oriented.x > 0.0F ? kInf : -kInf);
    if (oriented.y != 0.0F) s.y = nextafterf(p.y, oriented.y > 0.0F ? kInf : -kInf);
    if (oriented.z != 0.0F) s.z = nextafterf(p.z, oriented.z > 0.0F ? kInf : -kInf);
    if (!finite3(s) || s == p) {
        lane.fail();
    }
    return s;
}

// ShadowRay.hpp:107-135
__device__ __forceinline__ void unit_segment(F3 origin, F3 endpoint, F3 expected, F3& direction,
                                             float& length, Lane& lane) {
    const F3 disp = endpoint - origin;
    const float scale = max_abs3(disp);
    if (!(scale > 0.0F) || !isfinite(scale)) {
        lane.fail();
        return;
    }
    const F3 s = disp / scale;
    const float sq = fmaf(s.x, s.x, fmaf(s.y, s.y, s.z * s.z));
    const float sl = sqrtf(sq);
    length = scale * sl;
    if (!(sl > 0.0F) || !isfinite(sl) || !(length > 0.0F) || !isfinite(length)) {
        lane.fail();
        return;
    }
    direction = s / sl;
    const float alignment = dot(direction, expected);
    if (!isfinite(alignment) || !(alignment > 0.0F)) {
        lane.fail();
    }
}

// ------------------------------------------------------------------------------------------------
// Checked products (frexp / scalbn forms)
// ------------------------------------------------------------------------------------------------

// DirectLighting.hpp:21-62
template <int NN, int ND>
__device__ __forceinline__ float checked_product_quotient(const float (&num)[NN], const float (&den)[ND],
                                                          Lane& lane) {
    float significand = 1.0F;
    int exponent = 0;
#pragma unroll
    for (int i = 0; i < NN; ++i) {
        const float v = num[i];
        if (!isfinite(v) || v < 0.0F) {
            lane.fail();
            return 0.0F;
        }
        if (v == 0.0F) {
            return 0.0F;
        }
        int e = 0;
        significand *= frexpf(v, &e);
        exponent += e;
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) {
        const float v = den[i];
        if (!isfinite(v) || !(v > 0.0F)) {
            lane.fail();
            return 0.0F;
        }
        int e = 0;
        significand /= frexpf(v, &e);
        exponent -= e;
    }
    int ne = 0;
    significand = frexpf(significand, &ne);
    const float result = scalbnf(significand, exponent + ne);
    if (!isfinite(result) || !(result > 0.0F)) {
        lane.fail();
    }
    return result;
}

// RoughDielectric.hpp:52-86
template <int NN, int ND>
__device__ __forceinline__ float checked_product_ratio(const float (&num)[NN], const float (&den)[ND],
                                                       Lane& lane) {
    bool zero = false;
#pragma unroll
    for (int i = 0; i < NN; ++i) {
        if (!isfinite(num[i]) || num[i] < 0.0F) {
            lane.fail();
            return 0.0F;
        }
        zero = zero || num[i] == 0.0F;
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) {
        if (!isfinite(den[i]) || !(den[i] > 0.0F)) {
            lane.fail();
            return 0.0F;
        }
    }
    if (zero) {
        return 0.0F;
    }
    float significand = 1.0F;
    int exponent = 0;
#pragma unroll
    for (int i = 0; i < NN; ++i) {
        int ve = 0, ne = 0;
        const float vs = frexpf(num[i], &ve);
        significand = frexpf(significand * vs, &ne);
        exponent += ve + ne;
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) {
        int ve = 0, ne = 0;
        const float vs = frexpf(den[i], &ve);
        significand = frexpf(significand / vs, &ne);
        exponent += ne - ve;
    }
    const float result = scalbnf(significand, exponent);
    if (!isfinite(result) || !(result > 0.0F)) {
        lane.fail();
    }
    return result;
}

// MisHeuristics.hpp:142-172
__device__ __forceinline__ float positive_product2(float a, float b, Lane& lane) {
    if (b == 0.0F) {
        return 0.0F;
    }
    int ea = 0, eb = 0, en = 0;
    const float sa = frexpf(a, &ea);
    const float sb = frexpf(b, &eb);
    const float n = frexpf(sa * sb, &en);
    const float r = scalbnf(n, ea + eb + en);
    if (!isfinite(r) || !(r > 0.0F)) {
        lane.fail();
    }
    return r;
}

// MisHeuristics.hpp:44-141
__device__ __forceinline__ float mis_weight(uint32_t heuristic, float sampled, float competing, Lane& lane) {
    if (!isfinite(sampled) || !(sampled > 0.0F) || !isfinite(competing) || competing < 0.0F) {
        lane.fail();
        return 1.0F;
    }
    if (competing == 0.0F) {
        return 1.0F;
    }
    const bool small = sampled < competing;
    const float n = small ? sampled : competing;
    const float d = small ? competing : sampled;
    int ne = 0, de = 0;
    const float ns = frexpf(n, &ne);
    const float ds = frexpf(d, &de);
    float ratio;
    if (heuristic == 0U) {
        ratio = scalbnf(ns / ds, ne - de);
    } else {
        const float r = ns / ds;
        ratio = scalbnf(r * r, 2 * (ne - de));
    }
    if (small) {
        if (!(ratio > 0.0F)) {
            lane.fail();
            return 1.0F;
        }
        const float w = ratio / (1.0F + ratio);
        if (!isfinite(w) || !(w > 0.0F)) {
            lane.fail();
        }
        return w;
    }
    return 1.0F / (1.0F + ratio);
}

// MisHeuristics.hpp:143-172
__device__ __forceinline__ float joint_light_pdf(float selection, float conditional, Lane& lane) {
    if (!isfinite(selection) || !(selection > 0.0F) || selection > 1.0F || !isfinite(conditional) ||
        conditional < 0.0F) {
        lane.fail();
        return 0.0F;
    }
    if (conditional == 0.0F) {
        return 0.0F;
    }
    return positive_product2(selection, conditional, lane);
}

// ------------------------------------------------------------------------------------------------
// Emission (Emission.hpp:42-108) and area-pdf conversion (Light.hpp:75-163, 593-620)
// ------------------------------------------------------------------------------------------------

__device__ __forceinline__ bool unit_normal(F3 n) {
    const float sq = fmaf(n.x, n.x, fmaf(n.y, n.y, n.z * n.z));
    return finite3(n) && isfinite(sq) && fabsf(sq - 1.0F) <= kEps * 128.0F;
}

// +1 emitting side, 0 back side or exactly tangent; fails when the orientation is ambiguous.
__device__ __forceinline__ int emission_side(F3 ng, F3 wo, Lane& lane) {
    if (!unit_normal(ng) || !finite3(wo) || (wo.x == 0.0F && wo.y == 0.0F && wo.z == 0.0F)) {
        lane.fail();
        return 0;
    }
    const float m = max_abs3(wo);
    const F3 s = wo / m;
    const float alignment = fmaf(ng.x, s.x, fmaf(ng.y, s.y, ng.z * s.z));
    if (!isfinite(alignment)) {
        lane.fail();
        return 0;
    }
    const bool orthogonal = (ng.x == 0.0F || wo.x == 0.0F) && (ng.y == 0.0F || wo.y == 0.0F) &&
                            (ng.z == 0.0F || wo.z == 0.0F);
    if (alignment == 0.0F && orthogonal) {
        return 0;
    }
    const float abs_sum = fmaf(fabsf(ng.x), fabsf(s.x), fmaf(fabsf(ng.y), fabsf(s.y), fabsf(ng.z) * fabsf(s.z)));
    const float uncertainty = fmaf(4.0F * kEps, abs_sum, 4.0F * kDenormMin);
    if (fabsf(alignment) <= uncertainty) {
        lane.fail();
        return 0;
    }
    return alignment > 0.0F ? 1 : 0;
}

__device__ __forceinline__ float area_to_solid_angle(float area_pdf, F3 ref, F3 surf, F3 ng, Lane& lane) {
    if (!unit_normal(ng)) {
        lane.fail();
        return 0.0F;
    }
    const F3 disp = surf - ref;
    const float scale = max_abs3(disp);
    if (!(scale > 0.0F) || !isfinite(scale)) {
        lane.fail();
        return 0.0F;
    }
    const F3 s = disp / scale;
    const float sq = fmaf(s.x, s.x, fmaf(s.y, s.y, s.z * s.z));
    const float sl = sqrtf(sq);
    const float cubed = sq * sl;
    if (!isfinite(sq) || !(sq > 0.0F) || !isfinite(cubed) || !(cubed > 0.0F)) {
        lane.fail();
        return 0.0F;
    }
    const float signed_alignment = fmaf(ng.x, -s.x, fmaf(ng.y, -s.y, ng.z * -s.z));
    const float alignment = fabsf(signed_alignment);
    const float term_sum = fmaf(fabsf(ng.x), fabsf(s.x), fmaf(fabsf(ng.y), fabsf(s.y), fabsf(ng.z) * fabsf(s.z)));
    const float uncertainty = fmaf(4.0F * kEps, term_sum, 4.0F * kDenormMin);
    if (!isfinite(alignment) || !isfinite(term_sum) || alignment <= uncertainty) {
        lane.fail();
        return 0.0F;
    }
    if (area_pdf == 0.0F) {
        return 0.0F;
    }
    int es = 0, ed = 0, ec = 0, ea = 0, en = 0;
    const float fs = frexpf(area_pdf, &es);
    const float fd = frexpf(scale, &ed);
    const float fc = frexpf(cubed, &ec);
    const float fa = frexpf(alignment, &ea);
    const float combined = fs * fd * fd * fc / fa;
    const int exponent = es + 2 * ed + ec - ea;
    const float normalized = frexpf(combined, &en);
    const float converted = scalbnf(normalized, exponent + en);
    if (!isfinite(converted) || !(converted > 0.0F)) {
        lane.fail();
    }
    return converted;
}

// ------------------------------------------------------------------------------------------------
// Closures
// ------------------------------------------------------------------------------------------------

struct ClosureData {
    uint32_t kind, lobes;
    float w[4];
    float p[10];
};

struct BsdfSample {
    bool valid;
    F3 wi;
    float value[4];
    float pdf;
    uint32_t lobes;
    float eta_scale;
    bool delta;         // pdf is a discrete mass (specular), not a solid-angle density
    uint32_t selected;  // the sampled closure, as an index into the depth-filtered mixture
};

// SamplingMappings.hpp:33-60, 128-141
__device__ __forceinline__ F3 map_cosine_hemisphere(float u, float v) {
    const float ox = 2.0F * u - 1.0F;
    const float oy = 2.0F * v - 1.0F;
    float px = 0.0F, py = 0.0F, radius = 0.0F;
    if (!(ox == 0.0F && oy == 0.0F)) {
        const float quarter_pi = kPi / 4.0F;
        float r, phi;
        if (fabsf(ox) > fabsf(oy)) {
            r = ox;
            phi = quarter_pi * (oy / ox);
        } else {
            r = oy;
            phi = 2.0F * quarter_pi - quarter_pi * (ox / oy);
        }
        const float2 sc = sincos_f(phi);
        px = r * sc.y;
        py = r * sc.x;
        radius = fabsf(r);
    }
    const float z = sqrtf((1.0F - radius) * (1.0F + radius));
    return F3{px, py, z};
}

struct Smith {
    float normal, tangent, radius, nor;
};

// GgxMicrofacet.hpp:134-184
__device__ __forceinline__ Smith smith_terms(float ax, float ay, F3 w, Lane& lane) {
    Smith t;
    if (ax == ay) {
        const float sine = hypot2f(w.x, w.y);
        const float inverse_alpha = 1.0F / ax;
        t.normal = ax <= 1.0F ? w.z : w.z * inverse_alpha;
        t.tangent = ax <= 1.0F ? ax * sine : sine;
        t.radius = hypot2f(t.normal, t.tangent);
    } else {
        const float common = bf_max(bf_max(1.0F, ax), ay);
        t.normal = w.z / common;
        const float tx = (ax / common) * w.x;
        const float ty = (ay / common) * w.y;
        t.tangent = hypot2f(tx, ty);
        t.radius = hypot2f(t.normal, t.tangent);
    }
    if (!isfinite(t.normal) || !isfinite(t.tangent) || !isfinite(t.radius) || !(t.normal > 0.0F) ||
        !(t.radius > 0.0F)) {
        lane.fail();
        t.nor = 1.0F;
        return t;
    }
    t.nor = t.normal / t.radius;
    if (!isfinite(t.nor) || !(t.nor > 0.0F) || t.nor > 1.0F) {
        lane.fail();
    }
    return t;
}

// GgxMicrofacet.hpp:232-270
__device__ __forceinline__ float ggx_d(float ax, float ay, F3 m, Lane& lane) {
    if (!unit_length(m)) {
        lane.fail();
        return 0.0F;
    }
    if (!(m.z > 0.0F)) {
        return 0.0F;
    }
    float denominator_root, density_root;
    if (ax == ay) {
        const float radial = hypot2f(m.x, m.y);
        if (ax <= 1.0F) {
            denominator_root = hypot2f(radial, ax * m.z);
            density_root = (ax / denominator_root) / denominator_root;
        } else {
            const float inverse_alpha = 1.0F / ax;
            denominator_root = hypot2f(radial * inverse_alpha, m.z);
            density_root = (inverse_alpha / denominator_root) / denominator_root;
        }
        density_root *= sqrtf(kInvPi);
    } else {
        denominator_root = hypot3f(m.x / ax, m.y / ay, m.z);
        const float normalization_root = sqrtf(kInvPi) / (sqrtf(ax) * sqrtf(ay));
        density_root = (normalization_root / denominator_root) / denominator_root;
    }
    const float value = density_root * density_root;
    if (!isfinite(denominator_root) || !(denominator_root > 0.0F) || !isfinite(value) || !(value > 0.0F)) {
        lane.fail();
    }
    return value;
}

// GgxMicrofacet.hpp:320-353
__device__ __forceinline__ float ggx_g2(float ax, float ay, F3 wo, F3 wi, Lane& lane) {
    if (!unit_length(wo) || !unit_length(wi)) {
        lane.fail();
        return 0.0F;
    }
    if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
        return 0.0F;
    }
    const Smith o = smith_terms(ax, ay, wo, lane);
    const Smith i = smith_terms(ax, ay, wi, lane);
    const float smaller = bf_min(o.nor, i.nor);
    const float larger = bf_max(o.nor, i.nor);
    const float value = 2.0F * smaller / (1.0F + smaller / larger);
    if (!isfinite(value) || !(value > 0.0F) || value > 1.0F) {
        lane.fail();
    }
    return value;
}

// GgxMicrofacet.hpp:355-388
__device__ __forceinline__ float ggx_vndf_pdf(float ax, float ay, F3 wo, F3 m, Lane& lane) {
    if (!unit_length(wo) || !unit_length(m)) {
        lane.fail();
        return 0.0F;
    }
    const float visible_dot = dot(wo, m);
    if (!(wo.z > 0.0F) || !(m.z > 0.0F) || !(visible_dot > 0.0F)) {
        return 0.0F;
    }
    const float d = ggx_d(ax, ay, m, lane);
    const float physical_radius = ax == ay ? hypot2f(wo.z, ax * hypot2f(wo.x, wo.y))
                                           : hypot3f(wo.z, ax * wo.x, ay * wo.y);
    const float physical_denominator = wo.z + physical_radius;
    const float visible_factor = 2.0F * visible_dot / physical_denominator;
    const float value = d * visible_factor;
    if (!isfinite(physical_denominator) || !(physical_denominator > 0.0F) || !isfinite(value) ||
        !(value > 0.0F)) {
        lane.fail();
    }
    return value;
}

// GgxMicrofacet.hpp:71-103
__device__ __forceinline__ F3 ggx_normalize(F3 v, Lane& lane) {
    const float length = hypot2f(hypot2f(v.x, v.y), v.z);
    if (!isfinite(length) || !(length > 0.0F)) {
        lane.fail();
        return F3{0.0F, 0.0F, 1.0F};
    }
    const F3 r{v.x / length, v.y / length, v.z / length};
    if (!unit_length(r)) {
        lane.fail();
    }
    return r;
}

__device__ __forceinline__ float nonnegative_roundoff(float value, float scale, Lane& lane) {
    if (value >= 0.0F) {
        return value;
    }
    const float bound = kEps * 16.0F * bf_max(1.0F, fabsf(scale));
    if (-value <= bound) {
        return 0.0F;
    }
    lane.fail();
    return 0.0F;
}

// GgxMicrofacet.hpp:390-525
static __device__ bool ggx_sample_vndf(float ax, float ay, F3 wo, float u, float v, F3& m_out, Lane& lane) {
    if (!unit_length(wo)) {
        lane.fail();
        return false;
    }
    if (!(wo.z > 0.0F)) {
        return false;
    }
    const bool iso = ax == ay;
    const float inverse_alpha = 1.0F / ax;
    const float common = bf_max(bf_max(1.0F, ax), ay);
    const float sax = ax / common, say = ay / common;
    F3 st;
    if (iso) {
        st = ax <= 1.0F ? F3{ax * wo.x, ax * wo.y, wo.z} : F3{wo.x, wo.y, wo.z * inverse_alpha};
    } else {
        st = F3{sax * wo.x, say * wo.y, wo.z / common};
    }
    if ((iso && ax <= 1.0F && ((wo.x != 0.0F && st.x == 0.0F) || (wo.y != 0.0F && st.y == 0.0F))) ||
        (iso && ax > 1.0F && st.z == 0.0F) ||
        (!iso && ((wo.x != 0.0F && st.x == 0.0F) || (wo.y != 0.0F && st.y == 0.0F) || st.z == 0.0F))) {
        lane.fail();
        return false;
    }
    const F3 hv = ggx_normalize(st, lane);
    const float tl = hypot2f(hv.x, hv.y);
    const F3 tangent = tl > 0.0F ? F3{-hv.y / tl, hv.x / tl, 0.0F} : F3{1.0F, 0.0F, 0.0F};
    const F3 bitangent = cross(hv, tangent);
    const float disk_radius = sqrtf(u);
    const float azimuth = 2.0F * kPi * v;
    const float2 sc = sincos_f(azimuth);
    const float disk_x = disk_radius * sc.y;
    const float initial_disk_y = disk_radius * sc.x;
    const float limit_sq = (1.0F - disk_x) * (1.0F + disk_x);
    const float checked_limit_sq = nonnegative_roundoff(limit_sq, 1.0F + fabsf(disk_x), lane);
    const float disk_y_limit = sqrtf(checked_limit_sq);
    const float projection = 0.5F * (1.0F + hv.z);
    const float disk_y = fmaf(projection, initial_disk_y, (1.0F - projection) * disk_y_limit);
    const float hz_sq = fmaf(-disk_y, disk_y, checked_limit_sq);
    const float checked_hz_sq = nonnegative_roundoff(hz_sq, checked_limit_sq + fabsf(disk_y * disk_y), lane);
    const float hz = sqrtf(checked_hz_sq);
    const F3 hn{fmaf(disk_x, tangent.x, fmaf(disk_y, bitangent.x, hz * hv.x)),
                fmaf(disk_x, tangent.y, fmaf(disk_y, bitangent.y, hz * hv.y)),
                fmaf(disk_x, tangent.z, fmaf(disk_y, bitangent.z, hz * hv.z))};
    if (!(hn.z > 0.0F)) {
        lane.fail();
        return false;
    }
    F3 un;
    if (iso) {
        un = ax <= 1.0F ? F3{ax * hn.x, ax * hn.y, hn.z} : F3{hn.x, hn.y, hn.z * inverse_alpha};
    } else {
        un = F3{sax * hn.x, say * hn.y, hn.z / common};
    }
    if ((iso && ax <= 1.0F && ((hn.x != 0.0F && un.x == 0.0F) || (hn.y != 0.0F && un.y == 0.0F))) ||
        (iso && ax > 1.0F && un.z == 0.0F) ||
        (!iso && ((hn.x != 0.0F && un.x == 0.0F) || (hn.y != 0.0F && un.y == 0.0F) || un.z == 0.0F))) {
        lane.fail();
        return false;
    }
    const F3 m = ggx_normalize(un, lane);
    if (!(m.z > 0.0F) || !(dot(wo, m) > 0.0F)) {
        lane.fail();
        return false;
    }
    m_out = m;
    return true;
}

// Fresnel.hpp:27-104
__device__ __forceinline__ float squared_magnitude_ratio(float nr, float ni, float dr, float di, Lane& lane) {
    const float n = hypot2f(nr, ni);
    const float d = hypot2f(dr, di);
    if (!isfinite(n) || !isfinite(d) || !(d > 0.0F)) {
        lane.fail();
        return 0.0F;
    }
    const float amplitude = n / d;
    const float r = amplitude * amplitude;
    if (!isfinite(r) || r < 0.0F || r > 1.0F) {
        lane.fail();
    }
    return r;
}

// Out of line, as is dielectric_fresnel: each is called per packet lane from several evaluation
// sites, and inlined copies made the shading kernels stall on instruction fetch (measured: shading
// 4 % faster on the BVH-stress frame out of line).
static __device__ __noinline__ float conductor_fresnel_lane(float cosine, float eta, float k, Lane& lane) {
    if (eta == 1.0F && k == 0.0F) {
        return 0.0F;
    }
    if (cosine == 0.0F) {
        return 1.0F;
    }
    const float scale = bf_max(bf_max(1.0F, eta), k);
    const float nie = 1.0F / scale;
    const float ne = eta / scale;
    const float nk = k / scale;
    if (cosine == 1.0F) {
        const float r = squared_magnitude_ratio(ne - nie, nk, ne + nie, nk, lane);
        if (!(r > 0.0F)) {
            lane.fail();
        }
        return r;
    }
    const float sin_sq = (1.0F - cosine) * (1.0F + cosine);
    const float scaled_sin_sq = nie * nie * sin_sq;
    const float x = fmaf(ne, ne, -fmaf(nk, nk, scaled_sin_sq));
    const float y = 2.0F * ne * nk;
    const float magnitude = hypot2f(x, y);
    float rr, ri;
    if (x >= 0.0F) {
        rr = sqrtf(0.5F * (magnitude + x));
        ri = rr == 0.0F ? 0.0F : y / (2.0F * rr);
    } else {
        ri = sqrtf(0.5F * (magnitude - x));
        rr = ri == 0.0F ? 0.0F : y / (2.0F * ri);
    }
    const float sc = nie * cosine;
    const float perpendicular = squared_magnitude_ratio(sc - rr, -ri, sc + rr, ri, lane);
    const float ser = fmaf(ne, ne, -(nk * nk));
    const float sei = y;
    const float srr = nie * rr;
    const float sri = nie * ri;
    const float pbr = cosine * ser;
    const float pbi = cosine * sei;
    const float parallel = squared_magnitude_ratio(pbr - srr, pbi - sri, pbr + srr, pbi + sri, lane);
    const float r = 0.5F * (perpendicular + parallel);
    if (!isfinite(r) || !(r > 0.0F) || r > 1.0F) {
        lane.fail();
    }
    return r;
}

// Fresnel.hpp:107-170
static __device__ __noinline__ float dielectric_fresnel(float cosine, float eta_i, float eta_t, Lane& lane) {
    if (!isfinite(cosine) || cosine < 0.0F || cosine > 1.0F) {
        lane.fail();
        return 1.0F;
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
        if (!isfinite(r) || !(r > 0.0F) || r > 1.0F) {
            lane.fail();
        }
        return r;
    }
    const float sin_i = sqrtf((1.0F - cosine) * (1.0F + cosine));
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
    const float cos_t = sqrtf((1.0F - sin_t) * (1.0F + sin_t));
    const float fec = ne * cos_t;
    const float fa = (cosine - fec) / (cosine + fec);
    const float sec = ne * cosine;
    const float sa = (sec - cos_t) / (sec + cos_t);
    const float r = 0.5F * fmaf(fa, fa, sa * sa);
    if (!isfinite(r) || !(r > 0.0F) || r > 1.0F) {
        lane.fail();
    }
    return r;
}

// RoughConductorReflection.hpp:68-106 / RoughDielectric.hpp:136-170
__device__ __forceinline__ void half_vector_geometry(F3 wo, F3 wi, F3& m, float& half_cos, Lane& lane) {
    const F3 h{wo.x + wi.x, wo.y + wi.y, wo.z + wi.z};
    const float length = hypot2f(hypot2f(h.x, h.y), h.z);
    if (!isfinite(length) || !(length > 0.0F)) {
        lane.fail();
        m = F3{0.0F, 0.0F, 1.0F};
        half_cos = 1.0F;
        return;
    }
    m = F3{h.x / length, h.y / length, h.z / length};
    if (!unit_length(m) || !(m.z > 0.0F)) {
        lane.fail();
    }
    half_cos = 0.5F * length;
    if (!isfinite(half_cos) || !(half_cos > 0.0F) || half_cos > 1.0F) {
        lane.fail();
    }
}

// RoughConductorReflection.hpp:167-238
static __device__ void conductor_eval(const ClosureData& c, F3 wo, F3 wi, float (&out)[4], Lane& lane) {
    out[0] = out[1] = out[2] = out[3] = 0.0F;
    if (!unit_length(wo) || !unit_length(wi)) {
        lane.fail();
        return;
    }
    if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
        return;
    }
    if (c.w[0] == 0.0F && c.w[1] == 0.0F && c.w[2] == 0.0F && c.w[3] == 0.0F) {
        return;
    }
    F3 m;
    float hc;
    half_vector_geometry(wo, wi, m, hc, lane);
    const float d = ggx_d(c.p[8], c.p[9], m, lane);
    const float g2 = ggx_g2(c.p[8], c.p[9], wo, wi, lane);
    float fresnel[4];
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        fresnel[l] = conductor_fresnel_lane(hc, c.p[l], c.p[4 + l], lane);
    }
    const float denominator = 4.0F * wo.z * wi.z;
    const float scale = (d * g2) / denominator;
    if (!isfinite(denominator) || !(denominator > 0.0F) || !isfinite(scale) || !(scale > 0.0F)) {
        lane.fail();
        return;
    }
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        out[l] = c.w[l] * fresnel[l] * scale;
    }
}

static __device__ float conductor_pdf(const ClosureData& c, F3 wo, F3 wi, Lane& lane) {
    if (!unit_length(wo) || !unit_length(wi)) {
        lane.fail();
        return 0.0F;
    }
    if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
        return 0.0F;
    }
    F3 m;
    float hc;
    half_vector_geometry(wo, wi, m, hc, lane);
    const float visible = ggx_vndf_pdf(c.p[8], c.p[9], wo, m, lane);
    const float value = visible / (4.0F * hc);
    if (!isfinite(value) || !(value > 0.0F)) {
        lane.fail();
    }
    return value;
}

struct Interface {
    float face_sign, incident_eta, transmitted_eta, nie, nte;
};

// RoughDielectric.hpp:114-134
__device__ __forceinline__ Interface interface_for(F3 wo, float ext, float in) {
    Interface f;
    f.face_sign = wo.z > 0.0F ? 1.0F : -1.0F;
    f.incident_eta = f.face_sign > 0.0F ? ext : in;
    f.transmitted_eta = f.face_sign > 0.0F ? in : ext;
    const float mx = bf_max(f.incident_eta, f.transmitted_eta);
    f.nie = f.incident_eta / mx;
    f.nte = f.transmitted_eta / mx;
    return f;
}

__device__ __forceinline__ F3 scaled_dir(F3 d, float s) { return {s * d.x, s * d.y, s * d.z}; }

struct TransmissionGeometry {
    bool valid;
    F3 m;
    float od, id, length;
};

// RoughDielectric.hpp:172-223
static __device__ TransmissionGeometry transmission_geometry(F3 of, F3 inf, const Interface& f, Lane& lane) {
    TransmissionGeometry g{};
    g.valid = false;
    F3 h{fmaf(f.nie, of.x, f.nte * inf.x), fmaf(f.nie, of.y, f.nte * inf.y), fmaf(f.nie, of.z, f.nte * inf.z)};
    const float length = hypot2f(hypot2f(h.x, h.y), h.z);
    if (!isfinite(length) || !(length > 0.0F)) {
        lane.fail();
        return g;
    }
    h = scaled_dir(h, 1.0F / length);
    if (h.z < 0.0F) {
        h = scaled_dir(h, -1.0F);
    }
    if (h.z == 0.0F) {
        return g;
    }
    if (!unit_length(h)) {
        lane.fail();
        return g;
    }
    const float od = dot(of, h);
    const float id = dot(inf, h);
    if (!isfinite(od) || !isfinite(id)) {
        lane.fail();
        return g;
    }
    if (!(od > 0.0F) || !(id < 0.0F)) {
        return g;
    }
    if (od > 1.0F || id < -1.0F) {
        lane.fail();
        return g;
    }
    g.valid = true;
    g.m = h;
    g.od = od;
    g.id = id;
    g.length = length;
    return g;
}

__device__ __forceinline__ void scale_spectrum(const float (&c)[4], float scale, float (&out)[4], Lane& lane) {
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        const float num[2] = {c[l], scale};
        const float den[1] = {1.0F};
        out[l] = checked_product_ratio(num, den, lane);
    }
}

// RoughDielectric.hpp:299-381 (radiance mode)
static __device__ void dielectric_eval(const ClosureData& c, F3 wo, F3 wi, float (&out)[4], Lane& lane) {
    out[0] = out[1] = out[2] = out[3] = 0.0F;
    if (!unit_length(wo) || !unit_length(wi)) {
        lane.fail();
        return;
    }
    if (wo.z == 0.0F || wi.z == 0.0F) {
        return;
    }
    const float ax = c.p[2], ay = c.p[3];
    const Interface f = interface_for(wo, c.p[0], c.p[1]);
    const F3 of = scaled_dir(wo, f.face_sign);
    const F3 inf = scaled_dir(wi, f.face_sign);
    if (inf.z > 0.0F) {
        F3 m;
        float od;
        half_vector_geometry(of, inf, m, od, lane);
        const float fr = dielectric_fresnel(od, f.incident_eta, f.transmitted_eta, lane);
        const float d = ggx_d(ax, ay, m, lane);
        const float g2 = ggx_g2(ax, ay, of, inf, lane);
        const float num[3] = {fr, d, g2};
        const float den[3] = {4.0F, of.z, inf.z};
        scale_spectrum(c.w, checked_product_ratio(num, den, lane), out, lane);
        return;
    }
    const TransmissionGeometry tg = transmission_geometry(of, inf, f, lane);
    if (!tg.valid) {
        return;
    }
    const float fr = dielectric_fresnel(tg.od, f.incident_eta, f.transmitted_eta, lane);
    if (fr == 1.0F) {
        return;
    }
    if (!(tg.length > 0.0F)) {
        lane.fail();
        return;
    }
    const float d = ggx_d(ax, ay, tg.m, lane);
    const float g2 = ggx_g2(ax, ay, of, scaled_dir(inf, -1.0F), lane);
    const float eta = f.nie;
    const float num[7] = {1.0F - fr, d, g2, eta, eta, tg.od, -tg.id};
    const float den[4] = {of.z, -inf.z, tg.length, tg.length};
    scale_spectrum(c.w, checked_product_ratio(num, den, lane), out, lane);
}

// RoughDielectric.hpp:383-467
static __device__ float dielectric_pdf(const ClosureData& c, F3 wo, F3 wi, Lane& lane) {
    if (!unit_length(wo) || !unit_length(wi)) {
        lane.fail();
        return 0.0F;
    }
    if (wo.z == 0.0F || wi.z == 0.0F) {
        return 0.0F;
    }
    const float ax = c.p[2], ay = c.p[3];
    const Interface f = interface_for(wo, c.p[0], c.p[1]);
    const F3 of = scaled_dir(wo, f.face_sign);
    const F3 inf = scaled_dir(wi, f.face_sign);
    if (inf.z > 0.0F) {
        F3 m;
        float od;
        half_vector_geometry(of, inf, m, od, lane);
        const float fr = dielectric_fresnel(od, f.incident_eta, f.transmitted_eta, lane);
        const float visible = ggx_vndf_pdf(ax, ay, of, m, lane);
        const float num[2] = {fr, visible};
        const float den[2] = {4.0F, od};
        return checked_product_ratio(num, den, lane);
    }
    const TransmissionGeometry tg = transmission_geometry(of, inf, f, lane);
    if (!tg.valid) {
        return 0.0F;
    }
    const float fr = dielectric_fresnel(tg.od, f.incident_eta, f.transmitted_eta, lane);
    if (fr == 1.0F) {
        return 0.0F;
    }
    if (!(tg.length > 0.0F)) {
        lane.fail();
        return 0.0F;
    }
    const float visible = ggx_vndf_pdf(ax, ay, of, tg.m, lane);
    const float num[5] = {1.0F - fr, visible, f.nte, f.nte, -tg.id};
    const float den[2] = {tg.length, tg.length};
    return checked_product_ratio(num, den, lane);
}

// DepthFilteredClosureMixture.hpp:48-133
static __device__ float dielectric_pdf_masked(const ClosureData& c, uint32_t allowed, F3 wo, F3 wi, Lane& lane) {
    const float base = dielectric_pdf(c, wo, wi, lane);
    if (wo.z == 0.0F || wi.z == 0.0F || base == 0.0F) {
        return base;
    }
    const bool reflection = (wo.z > 0.0F) == (wi.z > 0.0F);
    const uint32_t direction = reflection ? kLobeReflection : kLobeTransmission;
    if ((allowed & direction) == 0U) {
        return 0.0F;
    }
    if (allowed == (kLobeReflection | kLobeTransmission)) {
        return base;
    }
    const Interface f = interface_for(wo, c.p[0], c.p[1]);
    const F3 of = scaled_dir(wo, f.face_sign);
    const F3 inf = scaled_dir(wi, f.face_sign);
    float branch;
    if (reflection) {
        F3 m;
        float od;
        half_vector_geometry(of, inf, m, od, lane);
        branch = dielectric_fresnel(od, f.incident_eta, f.transmitted_eta, lane);
    } else {
        const TransmissionGeometry tg = transmission_geometry(of, inf, f, lane);
        if (!tg.valid) {
            return 0.0F;
        }
        branch = 1.0F - dielectric_fresnel(tg.od, f.incident_eta, f.transmitted_eta, lane);
    }
    if (!isfinite(branch) || !(branch > 0.0F) || branch > 1.0F) {
        lane.fail();
        return 0.0F;
    }
    const float num[1] = {base};
    const float den[1] = {branch};
    return checked_product_ratio(num, den, lane);
}

// Closure kind fixed at compile time (K = the kind) or read from the record (K = 0). The shading
// kernels are instantiated per kind so each one carries only its own closure's code.
template <int K>
__device__ __forceinline__ bool kind_is(const ClosureData& c, uint32_t kind) {
    if constexpr (K == 0) {
        return c.kind == kind;
    } else {
        return static_cast<uint32_t>(K) == kind;
    }
}

// ------------------------------------------------------------------------------------------------
// Ray cones of the wavefront transport (CudaWavefrontStages.cu:540-543, 2803-2870, 3675-3781; the
// CPU twin is RayCone.hpp). A cone is (width, spread): its radius at the ray origin and its radial
// slope. It advances to a hit as width + spread * distance and is re-spread at every scattering
// event by the selected closure's footprint policy (unit slope for diffuse, max(alpha_x, alpha_y)
// for GGX, Snell's singular values through a refraction). Every product and ratio is checked as
// the reference checks it: a non-finite result, or two non-zero factors whose product underflows
// to zero, fails the lane.
// ------------------------------------------------------------------------------------------------

__device__ __forceinline__ bool cone_valid(float2 cone) {
    return isfinite(cone.x) && cone.x >= 0.0F && isfinite(cone.y) && cone.y >= 0.0F;
}

__device__ __forceinline__ bool cone_product(float left, float right, float& product) {
    product = left * right;
    return isfinite(product) && !(left != 0.0F && right != 0.0F && product == 0.0F);
}

__device__ __forceinline__ bool cone_ratio(float numerator, float denominator, float& ratio) {
    if (!isfinite(numerator) || !(numerator > 0.0F) || !isfinite(denominator) || !(denominator > 0.0F)) {
        return false;
    }
    ratio = numerator / denominator;
    return isfinite(ratio) && ratio > 0.0F;
}

// advance_ray_cone_to_hit: the cone carried from the ray origin to the hit at parameter t of a ray
// whose direction d need not be unit (its length taken as max|d| * |d / max|d||).
static __device__ bool cone_advance(float2 cone, F3 d, float t, float2& out) {
    if (!cone_valid(cone) || !isfinite(t) || t < 0.0F) {
        return false;
    }
    const float scale = fmaxf(fabsf(d.x), fmaxf(fabsf(d.y), fabsf(d.z)));
    if (!isfinite(scale) || !(scale > 0.0F)) {
        return false;
    }
    const float inverse = 1.0F / scale;
    const float sx = d.x * inverse, sy = d.y * inverse, sz = d.z * inverse;
    const float normalized_length = sqrtf(fmaf(sx, sx, fmaf(sy, sy, sz * sz)));
    float length = 0.0F, distance = 0.0F, growth = 0.0F;
    if (!isfinite(normalized_length) || !(normalized_length > 0.0F) ||
        !cone_product(scale, normalized_length, length) || !(length > 0.0F)) {
        return false;
    }
    if (!cone_product(t, length, distance) || distance < 0.0F || !cone_product(cone.y, distance, growth)) {
        return false;
    }
    const float width = fmaf(cone.y, distance, cone.x);
    if (!isfinite(width) || width < cone.x || (growth != 0.0F && width == cone.x)) {
        return false;
    }
    out = make_float2(width, cone.y);
    return cone_valid(out);
}

// unit_vector (TransportDevice.cuh:325-333): squared length within 128 ulp of one
__device__ __forceinline__ bool cone_unit(F3 v) {
    if (!finite3(v)) {
        return false;
    }
    const float squared = fmaf(v.x, v.x, fmaf(v.y, v.y, v.z * v.z));
    return isfinite(squared) && fabsf(squared - 1.0F) <= 128.0F * kEps;
}

// valid_surface_event: exactly one lobe family and one direction, no volume lobe
__device__ __forceinline__ bool cone_surface_event(uint32_t bits) {
    const uint32_t family = bits & (kLobeDiffuse | kLobeGlossy | kLobeSpecular);
    const uint32_t direction = bits & (kLobeReflection | kLobeTransmission);
    return bits != 0U && (bits & ~0x3FU) == 0U && (bits & kLobeVolume) == 0U &&
           (family == kLobeDiffuse || family == kLobeGlossy || family == kLobeSpecular) &&
           (direction == kLobeReflection || direction == kLobeTransmission);
}

// propagate_ray_cone_scattering: the cone after the closure `c` scattered wo (local, outgoing)
// into wi (local, incoming) with the sampled event lobes.
template <int K>
__device__ bool cone_scatter(float2 cone, const ClosureData& c, uint32_t event, F3 wo, F3 wi, float2& out) {
    if (!cone_valid(cone) || !cone_surface_event(event) || !cone_unit(wo) || !cone_unit(wi) || wo.z == 0.0F ||
        wi.z == 0.0F) {
        return false;
    }
    const bool reflection = (event & kLobeReflection) != 0U;
    const bool transmission = (event & kLobeTransmission) != 0U;
    const bool same_hemisphere = (wo.z > 0.0F) == (wi.z > 0.0F);
    if ((reflection && !same_hemisphere) || (transmission && same_hemisphere)) {
        return false;
    }
    float spread_floor = 0.0F, transmission_scale = 1.0F, width_scale = 1.0F;
    bool dielectric = false;
    if (kind_is<K>(c, kClosureLambert) || kind_is<K>(c, kClosureRoughDiffuse)) {
        if (!reflection || (event & kLobeDiffuse) == 0U) {
            return false;
        }
        spread_floor = 1.0F;
    } else if (kind_is<K>(c, kClosureSpecularReflection)) {
        if (!reflection || (event & kLobeSpecular) == 0U) {
            return false;
        }
    } else if (kind_is<K>(c, kClosureSpecularTransmission)) {
        if (!transmission || (event & kLobeSpecular) == 0U) {
            return false;
        }
        dielectric = true;
    } else if (kind_is<K>(c, kClosureConductor)) {
        if (!reflection || (event & kLobeGlossy) == 0U || !isfinite(c.p[8]) || c.p[8] < 0.0F ||
            !isfinite(c.p[9]) || c.p[9] < 0.0F) {
            return false;
        }
        spread_floor = fmaxf(c.p[8], c.p[9]);
    } else if (kind_is<K>(c, kClosureDielectric)) {
        if ((event & kLobeGlossy) == 0U || !isfinite(c.p[2]) || c.p[2] < 0.0F || !isfinite(c.p[3]) ||
            c.p[3] < 0.0F) {
            return false;
        }
        spread_floor = fmaxf(c.p[2], c.p[3]);
        dielectric = true;
    } else {
        return false;
    }
    if (transmission) {
        if (!dielectric) {
            return false;
        }
        const float incident = wo.z > 0.0F ? c.p[0] : c.p[1];
        const float transmitted = wo.z > 0.0F ? c.p[1] : c.p[0];
        float eta_ratio = 0.0F, cosine_ratio = 0.0F, inverse_cosine_ratio = 0.0F, meridional = 0.0F;
        if (!cone_ratio(incident, transmitted, eta_ratio) || !cone_ratio(fabsf(wo.z), fabsf(wi.z), cosine_ratio) ||
            !cone_ratio(fabsf(wi.z), fabsf(wo.z), inverse_cosine_ratio) ||
            !cone_product(eta_ratio, cosine_ratio, meridional)) {
            return false;
        }
        transmission_scale = fmaxf(eta_ratio, meridional);
        width_scale = fmaxf(1.0F, inverse_cosine_ratio);
    }
    float width = 0.0F, spread = 0.0F;
    if (!cone_product(cone.x, width_scale, width) || !cone_product(cone.y, transmission_scale, spread)) {
        return false;
    }
    out = make_float2(width, fmaxf(spread, spread_floor));
    return cone_valid(out);
}

template <int K>
static __device__ void closure_eval(const ClosureData& c, uint32_t allowed, F3 wo, F3 wi, float (&out)[4], Lane& lane) {
    if (kind_is<K>(c, kClosureLambert)) {  // LambertianReflection.hpp:76-85
        out[0] = out[1] = out[2] = out[3] = 0.0F;
        if (!unit_length(wo) || !unit_length(wi)) {
            lane.fail();
            return;
        }
        if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
            return;
        }
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            out[l] = c.w[l] * kInvPi;
        }
        return;
    }
    if (kind_is<K>(c, kClosureConductor)) {
        conductor_eval(c, wo, wi, out, lane);
        return;
    }
    dielectric_eval(c, wo, wi, out, lane);
    if (wo.z == 0.0F || wi.z == 0.0F) {
        return;
    }
    const uint32_t direction = (wo.z > 0.0F) == (wi.z > 0.0F) ? kLobeReflection : kLobeTransmission;
    if ((allowed & direction) == 0U) {
        out[0] = out[1] = out[2] = out[3] = 0.0F;
    }
}

template <int K>
static __device__ float closure_pdf(const ClosureData& c, uint32_t allowed, F3 wo, F3 wi, Lane& lane) {
    if (kind_is<K>(c, kClosureLambert)) {  // LambertianReflection.hpp:87-106
        if (!unit_length(wo) || !unit_length(wi)) {
            lane.fail();
            return 0.0F;
        }
        if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
            return 0.0F;
        }
        return wi.z * kInvPi;
    }
    if (kind_is<K>(c, kClosureConductor)) {
        return conductor_pdf(c, wo, wi, lane);
    }
    return dielectric_pdf_masked(c, allowed, wo, wi, lane);
}

// RoughDielectric.hpp:469-632 (radiance mode)
static __device__ void dielectric_sample(const ClosureData& c, F3 wo, float event, float u, float v, BsdfSample& s,
                                  Lane& lane) {
    s.valid = false;
    if (!unit_length(wo) || !(event >= 0.0F && event < 1.0F)) {
        lane.fail();
        return;
    }
    if (wo.z == 0.0F) {
        return;
    }
    const float ax = c.p[2], ay = c.p[3];
    const Interface f = interface_for(wo, c.p[0], c.p[1]);
    const F3 of = scaled_dir(wo, f.face_sign);
    F3 m;
    if (!ggx_sample_vndf(ax, ay, of, u, v, m, lane)) {
        return;
    }
    const float od = dot(of, m);
    if (!isfinite(od) || !(od > 0.0F) || od > 1.0F) {
        lane.fail();
        return;
    }
    const float fr = dielectric_fresnel(od, f.incident_eta, f.transmitted_eta, lane);
    F3 inf;
    uint32_t lobes;
    float eta_scale = 1.0F;
    if (event < fr) {
        inf = F3{2.0F * od * m.x - of.x, 2.0F * od * m.y - of.y, 2.0F * od * m.z - of.z};
        lobes = kLobeGlossy | kLobeReflection;
        if (!unit_length(inf)) {
            lane.fail();
            return;
        }
        if (!(inf.z > 0.0F)) {
            return;
        }
    } else {
        const F3 tangent{of.x - od * m.x, of.y - od * m.y, of.z - od * m.z};
        const float incident_sine = hypot2f(hypot2f(tangent.x, tangent.y), tangent.z);
        if (!isfinite(incident_sine) || incident_sine > 1.0F) {
            lane.fail();
            return;
        }
        float incoming_cosine = 1.0F, tangent_scale = 0.0F;
        if (incident_sine > 0.0F) {
            float transmitted_sine;
            if (f.incident_eta > f.transmitted_eta) {
                const float critical = f.transmitted_eta / f.incident_eta;
                if (critical == 0.0F || incident_sine >= critical) {
                    lane.fail();
                    return;
                }
                transmitted_sine = incident_sine / critical;
            } else {
                const float ratio = f.incident_eta / f.transmitted_eta;
                if (ratio == 0.0F) {
                    lane.fail();
                    return;
                }
                transmitted_sine = ratio * incident_sine;
            }
            if (!isfinite(transmitted_sine) || !(transmitted_sine < 1.0F)) {
                lane.fail();
                return;
            }
            incoming_cosine = sqrtf((1.0F - transmitted_sine) * (1.0F + transmitted_sine));
            tangent_scale = transmitted_sine / incident_sine;
            if (!isfinite(incoming_cosine) || !(incoming_cosine > 0.0F) || !isfinite(tangent_scale) ||
                !(tangent_scale > 0.0F)) {
                lane.fail();
                return;
            }
        }
        inf = F3{fmaf(-tangent_scale, tangent.x, -incoming_cosine * m.x),
                 fmaf(-tangent_scale, tangent.y, -incoming_cosine * m.y),
                 fmaf(-tangent_scale, tangent.z, -incoming_cosine * m.z)};
        lobes = kLobeGlossy | kLobeTransmission;
        if (!unit_length(inf)) {
            lane.fail();
            return;
        }
        if (!(inf.z < 0.0F)) {
            return;
        }
        const float num[2] = {f.nte, f.nte};
        const float den[2] = {f.nie, f.nie};
        eta_scale = checked_product_ratio(num, den, lane);
    }
    s.wi = scaled_dir(inf, f.face_sign);
    dielectric_eval(c, wo, s.wi, s.value, lane);
    s.pdf = dielectric_pdf(c, wo, s.wi, lane);
    s.lobes = lobes;
    s.eta_scale = eta_scale;
    s.valid = true;
}

// DepthFilteredClosureMixture.hpp:460-552 for a single active closure.
template <int K>
static __device__ void closure_sample(const ClosureData& c, uint32_t allowed, F3 wo, float component, float u, float v,
                               BsdfSample& s, Lane& lane) {
    s.valid = false;
    s.eta_scale = 1.0F;
    s.lobes = c.lobes;
    if (!unit_length(wo)) {
        lane.fail();
        return;
    }
    if (kind_is<K>(c, kClosureLambert)) {  // LambertianReflection.hpp:108-140
        const F3 wi = map_cosine_hemisphere(u, v);
        if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
            return;
        }
        s.wi = wi;
        closure_eval<K>(c, allowed, wo, wi, s.value, lane);
        s.pdf = closure_pdf<K>(c, allowed, wo, wi, lane);
        s.valid = true;
        return;
    }
    if (kind_is<K>(c, kClosureConductor)) {  // RoughConductorReflection.hpp:240-288
        F3 m;
        if (!ggx_sample_vndf(c.p[8], c.p[9], wo, u, v, m, lane)) {
            return;
        }
        const float hc = dot(wo, m);
        if (!isfinite(hc) || !(hc > 0.0F) || hc > 1.0F) {
            lane.fail();
            return;
        }
        const F3 wi{2.0F * hc * m.x - wo.x, 2.0F * hc * m.y - wo.y, 2.0F * hc * m.z - wo.z};
        if (!unit_length(wi)) {
            lane.fail();
            return;
        }
        if (!(wi.z > 0.0F)) {
            return;
        }
        s.wi = wi;
        conductor_eval(c, wo, wi, s.value, lane);
        s.pdf = conductor_pdf(c, wo, wi, lane);
        s.valid = true;
        return;
    }
    // rough dielectric with a depth-restricted direction (DepthFilteredClosureMixture.hpp:135-180)
    float event = component;
    if (allowed == kLobeReflection) {
        event = 0.0F;
    } else if (allowed == kLobeTransmission) {
        event = nextafterf(1.0F, 0.0F);
    }
    dielectric_sample(c, wo, event, u, v, s, lane);
    if (!s.valid) {
        return;
    }
    if ((s.lobes & allowed) == 0U) {
        s.valid = false;
        return;
    }
    s.pdf = dielectric_pdf_masked(c, allowed, wo, s.wi, lane);
}

// ------------------------------------------------------------------------------------------------
// Energy-preserving Oren-Nayar rough diffuse reflection (RoughDiffuseReflection.hpp:62-283). The
// arctangent is the double-precision value rounded once to float.
// ------------------------------------------------------------------------------------------------

constexpr float kFonCoefficient = 0.5F - 2.0F * kInvPi / 3.0F;
constexpr float kFonAverageCoefficient = 2.0F / 3.0F - 28.0F * kInvPi / 15.0F;
constexpr float kFonAverageLossCoefficient = kFonCoefficient - kFonAverageCoefficient;

static __device__ __noinline__ float atan2_f(float y, float x) {
    return static_cast<float>(atan2(static_cast<double>(y), static_cast<double>(x)));
}

// directional_loss_shape: 1 - E_FON for unit albedo without the factor A_F * r
static __device__ float eon_loss_shape(F3 d, Lane& lane) {
    const float sine = hypot2f(d.x, d.y);
    const float cosine = d.z;
    const float angle = atan2_f(sine, cosine);
    const float stable_ratio = sine * cosine * (1.0F + sine + sine * sine) / (1.0F + sine);
    const float g = sine * (angle - sine * cosine) + (2.0F / 3.0F) * (stable_ratio - sine);
    const float loss = kFonCoefficient - g * kInvPi;
    if (!isfinite(loss) || loss < 0.0F) {
        lane.fail();
    }
    return loss;
}

static __device__ void eon_eval(const ClosureData& c, F3 wo, F3 wi, float (&out)[4], Lane& lane) {
    out[0] = out[1] = out[2] = out[3] = 0.0F;
    if (!unit_length(wo) || !unit_length(wi)) {
        lane.fail();
        return;
    }
    if (!(wo.z > 0.0F) || !(wi.z > 0.0F) || (c.w[0] == 0.0F && c.w[1] == 0.0F && c.w[2] == 0.0F && c.w[3] == 0.0F)) {
        return;
    }
    const float r = c.p[0];
    if (r == 0.0F) {
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            out[l] = c.w[l] * kInvPi;
        }
        return;
    }
    const float tangent_dot = fmaf(wo.x, wi.x, wo.y * wi.y);
    const float s_over_t = tangent_dot > 0.0F ? tangent_dot / bf_max(wo.z, wi.z) : tangent_dot;
    const float a = 1.0F / (1.0F + kFonCoefficient * r);
    const float single = kInvPi * a * (1.0F + r * s_over_t);
    if (!isfinite(single) || single < 0.0F) {
        lane.fail();
        return;
    }
    const float outgoing_loss = eon_loss_shape(wo, lane);
    const float incoming_loss = eon_loss_shape(wi, lane);
    const float average = a * (1.0F + kFonAverageCoefficient * r);
    const float loss_over_average = a * r * incoming_loss * outgoing_loss / kFonAverageLossCoefficient;
    if (!isfinite(average) || !(average > 0.0F) || average > 1.0F || !isfinite(loss_over_average) ||
        loss_over_average < 0.0F) {
        lane.fail();
        return;
    }
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        const float rho = c.w[l];
        const float den = (1.0F - rho) + rho * average;
        if (!isfinite(den) || !(den > 0.0F)) {
            lane.fail();
        }
        const float ms = rho * rho * average / den;
        const float value = rho * single + ms * kInvPi * loss_over_average;
        if (!isfinite(value) || value < 0.0F) {
            lane.fail();
        }
        out[l] = value;
    }
}

// ------------------------------------------------------------------------------------------------
// Ideal specular reflection and transmission (SpecularDelta.hpp:85-495): eval and pdf queries
// exclude the Dirac atom, sample() returns it with a discrete mass of one.
// ------------------------------------------------------------------------------------------------

// checked_positive_product_quotient
__device__ __forceinline__ float delta_product_quotient(float left, float right, float den, Lane& lane) {
    if (left == 0.0F) {
        return 0.0F;
    }
    if (!isfinite(left) || !(left > 0.0F) || !isfinite(right) || !(right > 0.0F) || !isfinite(den) || !(den > 0.0F)) {
        lane.fail();
        return 0.0F;
    }
    int le = 0, re = 0, de = 0, ne = 0;
    const float ls = frexpf(left, &le), rs = frexpf(right, &re), ds = frexpf(den, &de);
    const float normalized = frexpf((ls * rs) / ds, &ne);
    const float result = scalbnf(normalized, le + re - de + ne);
    if (!isfinite(result) || !(result > 0.0F)) {
        lane.fail();
    }
    return result;
}

// checked_squared_ratio
__device__ __forceinline__ float delta_squared_ratio(float num, float den, Lane& lane) {
    if (!isfinite(num) || !(num > 0.0F) || !isfinite(den) || !(den > 0.0F)) {
        lane.fail();
        return 1.0F;
    }
    int ne = 0, de = 0, re = 0;
    const float ns = frexpf(num, &ne), ds = frexpf(den, &de);
    const float ratio = ns / ds;
    const float normalized = frexpf(ratio * ratio, &re);
    const float result = scalbnf(normalized, 2 * (ne - de) + re);
    if (!isfinite(result) || !(result > 0.0F)) {
        lane.fail();
    }
    return result;
}

static __device__ void specular_sample(const ClosureData& c, F3 wo, BsdfSample& s, Lane& lane) {
    s.valid = false;
    s.delta = true;
    s.pdf = 1.0F;
    s.eta_scale = 1.0F;
    if (!unit_length(wo)) {
        lane.fail();
        return;
    }
    if (wo.z == 0.0F) {
        return;
    }
    if (c.kind == kClosureSpecularReflection) {
        s.wi = F3{-wo.x, -wo.y, wo.z};
        s.lobes = kLobeSpecular | kLobeReflection;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            s.value[l] = delta_product_quotient(c.w[l], 1.0F, fabsf(s.wi.z), lane);
        }
        s.valid = true;
        return;
    }
    const bool entering = wo.z > 0.0F;
    const float incident = entering ? c.p[0] : c.p[1];
    const float transmitted = entering ? c.p[1] : c.p[0];
    s.lobes = kLobeSpecular | kLobeTransmission;
    if (incident == transmitted) {
        s.wi = F3{-wo.x, -wo.y, -wo.z};
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            s.value[l] = delta_product_quotient(c.w[l], 1.0F, fabsf(s.wi.z), lane);
        }
        s.valid = true;
        return;
    }
    const float raw_sine = hypot2f(wo.x, wo.y);
    if (!isfinite(raw_sine)) {
        lane.fail();
        return;
    }
    float sine = raw_sine, normalization = 1.0F;
    if (raw_sine > 1.0F) {
        const float cosine = fabsf(wo.z);
        if (cosine > 1.0F) {
            lane.fail();
            return;
        }
        sine = sqrtf((1.0F - cosine) * (1.0F + cosine));
        normalization = sine / raw_sine;
        if (!isfinite(sine) || !isfinite(normalization) || !(normalization > 0.0F)) {
            lane.fail();
            return;
        }
    }
    if (sine > 0.0F) {
        const float critical = transmitted / incident;
        if (critical <= 1.0F && sine >= critical) {
            return;  // total internal reflection: no transmission support
        }
    }
    const float ratio = incident / transmitted;
    if (!isfinite(ratio) || !(ratio > 0.0F)) {
        lane.fail();
        return;
    }
    const float ix = -ratio * normalization * wo.x;
    const float iy = -ratio * normalization * wo.y;
    if (!isfinite(ix) || !isfinite(iy) || (wo.x != 0.0F && ix == 0.0F) || (wo.y != 0.0F && iy == 0.0F)) {
        lane.fail();
        return;
    }
    const float transmitted_sine = hypot2f(ix, iy);
    if (!isfinite(transmitted_sine) || transmitted_sine >= 1.0F) {
        lane.fail();
        return;
    }
    const float transmitted_cosine = sqrtf((1.0F - transmitted_sine) * (1.0F + transmitted_sine));
    if (!isfinite(transmitted_cosine) || !(transmitted_cosine > 0.0F)) {
        lane.fail();
        return;
    }
    s.wi = F3{ix, iy, entering ? -transmitted_cosine : transmitted_cosine};
    if (!unit_length(s.wi)) {
        lane.fail();
        return;
    }
    const float adjoint = delta_squared_ratio(incident, transmitted, lane);  // radiance mode
    s.eta_scale = delta_squared_ratio(transmitted, incident, lane);
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        s.value[l] = delta_product_quotient(c.w[l], adjoint, transmitted_cosine, lane);
    }
    s.valid = true;
}

// ------------------------------------------------------------------------------------------------
// One closure record of any kind, the rough dielectric restricted to `allowed`
// (DepthFilteredClosureMixture.hpp:182-252, ClosureMixture.hpp:527-748)
// ------------------------------------------------------------------------------------------------

__device__ __forceinline__ bool is_delta_kind(uint32_t kind) {
    return kind == kClosureSpecularReflection || kind == kClosureSpecularTransmission;
}

static __device__ void record_eval(const ClosureData& c, uint32_t allowed, F3 wo, F3 wi, float (&out)[4], Lane& lane) {
    if (c.kind == kClosureRoughDiffuse) {
        eon_eval(c, wo, wi, out, lane);
    } else if (is_delta_kind(c.kind)) {
        out[0] = out[1] = out[2] = out[3] = 0.0F;
        if (!unit_length(wo) || !unit_length(wi)) {
            lane.fail();
        }
    } else {
        closure_eval<0>(c, allowed, wo, wi, out, lane);
    }
}

static __device__ float record_pdf(const ClosureData& c, uint32_t allowed, F3 wo, F3 wi, Lane& lane) {
    if (c.kind == kClosureRoughDiffuse || is_delta_kind(c.kind)) {
        if (!unit_length(wo) || !unit_length(wi)) {
            lane.fail();
            return 0.0F;
        }
        if (is_delta_kind(c.kind) || !(wo.z > 0.0F) || !(wi.z > 0.0F)) {
            return 0.0F;
        }
        return wi.z * kInvPi;
    }
    return closure_pdf<0>(c, allowed, wo, wi, lane);
}

static __device__ void record_sample(const ClosureData& c, uint32_t allowed, F3 wo, float event, float u, float v,
                                     BsdfSample& s, Lane& lane) {
    s.delta = false;
    s.valid = false;
    if (is_delta_kind(c.kind)) {
        specular_sample(c, wo, s, lane);
        return;
    }
    if (c.kind == kClosureRoughDiffuse) {  // RoughDiffuseReflection.hpp:235-266
        s.eta_scale = 1.0F;
        s.lobes = c.lobes;
        if (!unit_length(wo)) {
            lane.fail();
            return;
        }
        const F3 wi = map_cosine_hemisphere(u, v);
        if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
            return;
        }
        s.wi = wi;
        eon_eval(c, wo, wi, s.value, lane);
        s.pdf = record_pdf(c, allowed, wo, wi, lane);
        s.valid = true;
        return;
    }
    closure_sample<0>(c, allowed, wo, event, u, v, s, lane);
}

// ------------------------------------------------------------------------------------------------
// Depth-filtered closure mixtures (DepthFilteredClosureMixture.hpp:254-552; ClosureMixture.hpp:
// 79-334, 760-876). A material's closures are filtered by the depth limits; the survivors keep
// their component probabilities, renormalised on the sampler grid when some were dropped.
// ------------------------------------------------------------------------------------------------

// A material's projected component distribution (build_component_distribution at upload).
struct MixDistribution {
    float p[kMaxClosures];
    float cdf[kMaxClosures + 1];
    uint32_t closure_offset;  // first closure in SceneView::mix_closures
    uint32_t pad[2];
};

struct Mix {
    ClosureData first;             // single-closure routes (K != 0): the closure itself
    const ClosureData* closures;   // generic route (K == 0): the material's closures
    uint32_t count, blocked;
    uint8_t source[kMaxClosures], allowed[kMaxClosures];
    float p[kMaxClosures];
    float cdf[kMaxClosures + 1];
};

template <int K>
__device__ __forceinline__ ClosureData mix_closure(const Mix& m, uint32_t i) {
    if constexpr (K != 0) {
        return m.first;
    } else {
        return m.closures[m.source[i]];
    }
}

// add_compensated (ClosureMixture.hpp:78-99)
__device__ __forceinline__ bool add_compensated(float value, float& sum, float& correction) {
    if (!isfinite(value) || value < 0.0F) {
        return false;
    }
    const float next = sum + value;
    if (!isfinite(next)) {
        return false;
    }
    if (sum >= value) {
        correction += (sum - next) + value;
    } else {
        correction += (value - next) + sum;
    }
    if (!isfinite(correction)) {
        return false;
    }
    sum = next;
    return true;
}

// build_component_distribution (ClosureMixture.hpp:122-234) for n >= 2 renormalised probabilities
static __device__ bool component_distribution(const float* probabilities, uint32_t n, float* out_p, float* out_cdf) {
#pragma unroll
    for (uint32_t i = 0; i <= kMaxClosures; ++i) {
        out_cdf[i] = 0.0F;
    }
    for (uint32_t i = 0; i < n; ++i) {
        if (!isfinite(probabilities[i]) || !(probabilities[i] > 0.0F) || !(probabilities[i] < 1.0F)) {
            return false;
        }
    }
    constexpr int digits = 24;
    constexpr uint64_t scale = 1ULL << digits;
    uint64_t masses[kMaxClosures];
    float remainders[kMaxClosures];
    uint64_t base_mass = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const float scaled = ldexpf(probabilities[i], digits);
        const float base = floorf(scaled);
        if (!isfinite(scaled) || !(scaled > 0.0F) || base < 0.0F || base > static_cast<float>(scale)) {
            return false;
        }
        masses[i] = static_cast<uint64_t>(base);
        remainders[i] = scaled - base;
        if (!isfinite(remainders[i]) || remainders[i] < 0.0F || remainders[i] >= 1.0F) {
            return false;
        }
        base_mass += masses[i];
    }
    if (base_mass > scale) {
        return false;
    }
    float rs = 0.0F, rc = 0.0F;
    for (uint32_t i = 0; i < n; ++i) {
        if (!add_compensated(remainders[i], rs, rc)) {
            return false;
        }
    }
    const float remainder_total = rs + rc;
    if (!isfinite(remainder_total) || remainder_total < 0.0F) {
        return false;
    }
    const uint64_t missing = scale - base_mass;
    if (missing > n || fabsf(remainder_total - static_cast<float>(missing)) > 0.5F + kEps * 16.0F) {
        return false;
    }
    uint32_t received = 0U;
    for (uint64_t unit = 0; unit < missing; ++unit) {
        uint32_t selected = n;
        for (uint32_t i = 0; i < n; ++i) {
            if ((received >> i) & 1U || !(remainders[i] > 0.0F)) {
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
        received |= 1U << selected;
    }
    uint64_t cumulative = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (masses[i] == 0U || cumulative > scale - masses[i]) {
            return false;
        }
        cumulative += masses[i];
        out_p[i] = ldexpf(static_cast<float>(masses[i]), -digits);
        out_cdf[i + 1] = ldexpf(static_cast<float>(cumulative), -digits);
    }
    return cumulative == scale && out_cdf[n] == 1.0F;
}


// positive_probability_product (ClosureMixture.hpp:249-268)
__device__ __forceinline__ float positive_probability_product(float selection, float conditional, Lane& lane) {
    if (conditional == 0.0F) {
        return 0.0F;
    }
    int se = 0, ce = 0, ne = 0;
    const float ss = frexpf(selection, &se), cs = frexpf(conditional, &ce);
    const float normalized = frexpf(ss * cs, &ne);
    const float product = scalbnf(normalized, se + ce + ne);
    if (!isfinite(product) || !(product > 0.0F)) {
        lane.fail();
    }
    return product;
}

// mix_probability_densities (ClosureMixture.hpp:270-334)
static __device__ float mix_densities(const float* probabilities, const float* conditional, uint32_t n, Lane& lane) {
    float maximum = 0.0F;
    for (uint32_t i = 0; i < n; ++i) {
        if (!isfinite(conditional[i]) || conditional[i] < 0.0F) {
            lane.fail();
            return 0.0F;
        }
        maximum = bf_max(maximum, conditional[i]);
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
        if (density > 0.0F && (!isfinite(ratio) || !(ratio > 0.0F))) {
            lane.fail();
            return 0.0F;
        }
        if (!add_compensated(positive_probability_product(probabilities[i], ratio, lane), sum, correction)) {
            lane.fail();
            return 0.0F;
        }
    }
    const float normalized = sum + correction;
    if (!isfinite(normalized) || !(normalized > 0.0F) || normalized > 1.0F) {
        lane.fail();
        return 0.0F;
    }
    return positive_probability_product(normalized, maximum, lane);
}

template <int K>
__device__ void mix_eval(const Mix& m, F3 wo, F3 wi, float (&out)[4], Lane& lane) {
    if constexpr (K != 0) {
        closure_eval<K>(m.first, m.allowed[0], wo, wi, out, lane);
    } else {
        out[0] = out[1] = out[2] = out[3] = 0.0F;
        if (!unit_length(wo) || !unit_length(wi)) {
            lane.fail();
            return;
        }
        for (uint32_t i = 0; i < m.count; ++i) {
            float component[4];
            record_eval(m.closures[m.source[i]], m.allowed[i], wo, wi, component, lane);
#pragma unroll
            for (int l = 0; l < 4; ++l) {
                out[l] = out[l] + component[l];
                if (!isfinite(out[l])) {
                    lane.fail();
                }
            }
        }
    }
}

template <int K>
__device__ float mix_pdf(const Mix& m, F3 wo, F3 wi, Lane& lane) {
    if constexpr (K != 0) {
        return closure_pdf<K>(m.first, m.allowed[0], wo, wi, lane);
    } else {
        if (!unit_length(wo) || !unit_length(wi)) {
            lane.fail();
            return 0.0F;
        }
        float conditional[kMaxClosures];
        for (uint32_t i = 0; i < m.count; ++i) {
            conditional[i] = record_pdf(m.closures[m.source[i]], m.allowed[i], wo, wi, lane);
        }
        return mix_densities(m.p, conditional, m.count, lane);
    }
}

// aggregate_delta_atom (ClosureMixture.hpp:760-870)
static __device__ void aggregate_delta_atom(const Mix& m, F3 wo, F3 wi, float (&value)[4], float& probability,
                                            Lane& lane) {
    float vs[4] = {0.0F, 0.0F, 0.0F, 0.0F}, vc[4] = {0.0F, 0.0F, 0.0F, 0.0F};
    float ps = 0.0F, pc = 0.0F;
    uint32_t matching = 0;
    for (uint32_t i = 0; i < m.count; ++i) {
        const ClosureData c = m.closures[m.source[i]];
        if (!is_delta_kind(c.kind)) {
            continue;
        }
        BsdfSample candidate;
        specular_sample(c, wo, candidate, lane);
        if (!candidate.valid || candidate.wi.x != wi.x || candidate.wi.y != wi.y || candidate.wi.z != wi.z) {
            continue;
        }
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            if (!add_compensated(candidate.value[l], vs[l], vc[l])) {
                lane.fail();
            }
        }
        if (!add_compensated(positive_probability_product(m.p[i], candidate.pdf, lane), ps, pc)) {
            lane.fail();
        }
        ++matching;
    }
    probability = ps + pc;
    if (matching == 0U || !isfinite(probability) || !(probability > 0.0F) || probability > 1.0F) {
        lane.fail();
    }
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        value[l] = vs[l] + vc[l];
        if (!isfinite(value[l]) || value[l] < 0.0F) {
            lane.fail();
        }
    }
}

// DepthFilteredClosureMixture::sample (DepthFilteredClosureMixture.hpp:460-552)
template <int K>
__device__ void mix_sample(const Mix& m, F3 wo, float component, float u, float v, BsdfSample& s, Lane& lane) {
    s.valid = false;
    s.delta = false;
    s.selected = 0U;
    if constexpr (K != 0) {
        closure_sample<K>(m.first, m.allowed[0], wo, component, u, v, s, lane);
    } else {
        if (!unit_length(wo) || !(component >= 0.0F && component < 1.0F) || !(u >= 0.0F && u < 1.0F) ||
            !(v >= 0.0F && v < 1.0F)) {
            lane.fail();
            return;
        }
        uint32_t selected = m.count;
        for (uint32_t i = 0; i < m.count; ++i) {
            if (component < m.cdf[i + 1]) {
                selected = i;
                break;
            }
        }
        if (selected == m.count) {
            lane.fail();
            return;
        }
        const float event = (component - m.cdf[selected]) / m.p[selected];
        if (!isfinite(event) || event < 0.0F || !(event < 1.0F)) {
            lane.fail();
            return;
        }
        record_sample(m.closures[m.source[selected]], m.allowed[selected], wo, event, u, v, s, lane);
        if (!s.valid) {
            return;
        }
        if (m.count > 1U) {
            if (!s.delta) {
                mix_eval<0>(m, wo, s.wi, s.value, lane);
                s.pdf = mix_pdf<0>(m, wo, s.wi, lane);
            } else {
                aggregate_delta_atom(m, wo, s.wi, s.value, s.pdf, lane);
            }
        }
        s.selected = selected;
    }
}

}  // namespace bf200
