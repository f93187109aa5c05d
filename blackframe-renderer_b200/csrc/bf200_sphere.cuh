// Analytic sphere intersection: the exact quadratic of renderer::SphereT::intersect
// (Blackframe/Renderer/Include/Blackframe/Renderer/Sphere.hpp:321-437), in float.
//
// The quadratic's constant term c = |o - centre|^2 - r^2 and its discriminant
// |d|^2 r^2 - |(o - centre) x d|^2 are evaluated exactly as nonoverlapping float expansions (Two-Sum
// chains with zero elimination). Their signs are exact, and their values are the in-order float sums
// of the expansion components, as the reference computes them. The expansion steps, their order and
// every failure check follow the reference, because the values, and hence the roots, must match it
// bit for bit. Each expansion holds as many components as its inputs can produce here; the
// reference's capacity of 128 is never reached for these inputs, so its capacity failure cannot
// occur in either.
#pragma once

#include <cstdint>

#include "bf200_device.cuh"
#include "bf200_shading.cuh"

namespace bf200 {

enum SphereOutcome : int { kSphereMiss = 0, kSphereHit = 1, kSphereFailure = 2 };

template <int N>
struct FloatExpansion {
    float c[N];
    int n;
};

__device__ __forceinline__ bool is_normal_float(float x) { return isfinite(x) && fabsf(x) >= 1.17549435e-38F; }

// add_component (Sphere.hpp:48-81)
template <int N>
__device__ bool expansion_add(FloatExpansion<N>& e, float component) {
    float accumulated = component;
    int out = 0;
    const int n = e.n;
    for (int i = 0; i < n; ++i) {
        const float existing = e.c[i];
        const float sum = accumulated + existing;
        const float existing_from_sum = sum - accumulated;
        const float accumulated_from_sum = sum - existing_from_sum;
        const float error = (existing - existing_from_sum) + (accumulated - accumulated_from_sum);
        if (!isfinite(sum) || !isfinite(error)) {
            return false;
        }
        if (error != 0.0F) {
            if (out == N) {
                return false;
            }
            e.c[out++] = error;
        }
        accumulated = sum;
    }
    if (accumulated != 0.0F || out == 0) {
        if (out == N) {
            return false;
        }
        e.c[out++] = accumulated;
    }
    e.n = out;
    return true;
}

// add_product (Sphere.hpp:83-95): the exact product as (error, rounded) components
template <int N>
__device__ bool expansion_add_product(FloatExpansion<N>& e, float left, float right, float sign) {
    const float rounded = left * right;
    const float error = fmaf(left, right, -rounded);
    if (!isfinite(rounded) || !isfinite(error) || (left != 0.0F && right != 0.0F && !is_normal_float(rounded)) ||
        (error != 0.0F && !is_normal_float(error))) {
        return false;
    }
    return expansion_add(e, sign * error) && expansion_add(e, sign * rounded);
}

// add_expansion (Sphere.hpp:97-107)
template <int N, int M>
__device__ bool expansion_add_expansion(FloatExpansion<N>& destination, const FloatExpansion<M>& source, float sign) {
    for (int i = 0; i < source.n; ++i) {
        if (!expansion_add(destination, sign * source.c[i])) {
            return false;
        }
    }
    return true;
}

// multiply_expansions (Sphere.hpp:109-122)
template <int N, int L, int R>
__device__ bool expansion_multiply(const FloatExpansion<L>& left, const FloatExpansion<R>& right, FloatExpansion<N>& product) {
    product.n = 0;
    for (int i = 0; i < left.n; ++i) {
        for (int j = 0; j < right.n; ++j) {
            if (!expansion_add_product(product, left.c[i], right.c[j], 1.0F)) {
                return false;
            }
        }
    }
    return true;
}

template <int N>
__device__ __forceinline__ int expansion_sign(const FloatExpansion<N>& e) {
    for (int i = e.n; i > 0; --i) {
        const float component = e.c[i - 1];
        if (component != 0.0F) {
            return component > 0.0F ? 1 : -1;
        }
    }
    return 0;
}

template <int N>
__device__ __forceinline__ float expansion_value(const FloatExpansion<N>& e) {
    float value = 0.0F;
    for (int i = 0; i < e.n; ++i) {
        value += e.c[i];
    }
    return value;
}

// squared_norm_expansion (Sphere.hpp:124-130)
template <int N>
__device__ bool expansion_squared_norm(F3 v, FloatExpansion<N>& out) {
    out.n = 0;
    return expansion_add_product(out, v.x, v.x, 1.0F) && expansion_add_product(out, v.y, v.y, 1.0F) &&
           expansion_add_product(out, v.z, v.z, 1.0F);
}

// exact_quadratic_constant (Sphere.hpp:147-181): false when not representable
static __device__ bool sphere_constant(F3 rel, float radius, float& value) {
    FloatExpansion<8> origin_squared;
    FloatExpansion<2> radius_squared;
    radius_squared.n = 0;
    if (!expansion_squared_norm(rel, origin_squared) ||
        !expansion_add_product(radius_squared, radius, radius, 1.0F) ||
        !expansion_add_expansion(origin_squared, radius_squared, -1.0F)) {
        return false;
    }
    const int sign = expansion_sign(origin_squared);
    if (sign == 0) {
        value = 0.0F;
        return true;
    }
    value = expansion_value(origin_squared);
    return isfinite(value) && value != 0.0F && (value > 0.0F ? 1 : -1) == sign;
}

// exact_discriminant (Sphere.hpp:183-243): false when not representable; sign and value otherwise
static __device__ bool sphere_discriminant(F3 rel, F3 d, float radius, int& sign, float& value) {
    FloatExpansion<6> direction_squared;
    FloatExpansion<2> radius_squared;
    radius_squared.n = 0;
    if (!expansion_squared_norm(d, direction_squared) ||
        !expansion_add_product(radius_squared, radius, radius, 1.0F)) {
        return false;
    }
    FloatExpansion<120> radial;
    if (!expansion_multiply(direction_squared, radius_squared, radial)) {
        return false;
    }
    const float terms[3][4] = {{rel.y, d.z, rel.z, d.y}, {rel.z, d.x, rel.x, d.z}, {rel.x, d.y, rel.y, d.x}};
    FloatExpansion<96> perpendicular;
    perpendicular.n = 0;
    for (int k = 0; k < 3; ++k) {
        FloatExpansion<4> cross;
        cross.n = 0;
        FloatExpansion<32> cross_squared;
        if (!expansion_add_product(cross, terms[k][0], terms[k][1], 1.0F) ||
            !expansion_add_product(cross, terms[k][2], terms[k][3], -1.0F) ||
            !expansion_multiply(cross, cross, cross_squared) ||
            !expansion_add_expansion(perpendicular, cross_squared, 1.0F)) {
            return false;
        }
    }
    if (!expansion_add_expansion(radial, perpendicular, -1.0F)) {
        return false;
    }
    sign = expansion_sign(radial);
    if (sign <= 0) {
        value = 0.0F;
        return true;
    }
    value = expansion_value(radial);
    return isfinite(value) && value > 0.0F;
}

__device__ __forceinline__ float fused_dot3(F3 a, F3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }

// ------------------------------------------------------------------------------------------------
// Fast path for the two expansion values. Two facts make it exact:
// * With every scaled input component 0 or of magnitude >= 2^-8 (least significant bit
//   >= 2^-31), every nonzero product and product error the expansions form is a multiple of at
//   least 2^-124, so none is subnormal and the reference's representability checks all pass.
// * Summing a nonoverlapping expansion from its smallest component up, as the reference does,
//   lands within about 2 u_f ulp of its exact value X (u_f = 2^-24). So when X lies farther than
//   2^-12 ulp from every float rounding boundary, that sum is the float nearest to X.
// X is evaluated in double-double with an error bound; anything uncertain takes the expansions.
// ------------------------------------------------------------------------------------------------

struct DoubleDouble {
    double hi, lo;
};

__device__ __forceinline__ DoubleDouble dd_two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}

__device__ __forceinline__ DoubleDouble dd_add(DoubleDouble x, DoubleDouble y) {
    DoubleDouble s = dd_two_sum(x.hi, y.hi);
    s.lo += x.lo + y.lo;
    return dd_two_sum(s.hi, s.lo);
}

__device__ __forceinline__ DoubleDouble dd_square(DoubleDouble x) {
    const double p = x.hi * x.hi;
    const double e = fma(x.hi, x.hi, -p) + (2.0 * x.hi * x.lo + x.lo * x.lo);
    return dd_two_sum(p, e);
}

__device__ __forceinline__ DoubleDouble dd_scale(DoubleDouble x, double y) {
    const double p = x.hi * y;
    const double e = fma(x.hi, y, -p) + x.lo * y;
    return dd_two_sum(p, e);
}

__device__ __forceinline__ bool coarse_component(float x) { return x == 0.0F || fabsf(x) >= 0.00390625F; }

// The float nearest to X = x.hi + x.lo (known to within err) when X is certainly farther than
// 2^-12 ulp from each rounding boundary of that float; false otherwise.
__device__ __forceinline__ bool certified_nearest(DoubleDouble x, double err, float& out) {
    const float f = __double2float_rn(x.hi);
    if (!isfinite(f) || fabsf(f) < 1.17549435e-38F) {
        return false;
    }
    const double fd = f;
    const double up = static_cast<double>(nextafterf(f, kInf)) - fd;
    const double down = fd - static_cast<double>(nextafterf(f, -kInf));
    const double dist = (x.hi - fd) + x.lo;
    const double margin = 0x1p-12;
    if (dist + err + margin * up < 0.5 * up && err - dist + margin * down < 0.5 * down) {
        out = f;
        return true;
    }
    return false;
}

// c = |rel|^2 - r^2 and the discriminant |d|^2 r^2 - |rel x d|^2 of the scaled inputs by the fast
// path; false when the fast path is not certain (the expansions then decide).
__device__ __forceinline__ bool sphere_values_fast(F3 srel, F3 sd, float sr, float& c, int& disc_sign, float& disc) {
    if (!coarse_component(srel.x) || !coarse_component(srel.y) || !coarse_component(srel.z) ||
        !coarse_component(sd.x) || !coarse_component(sd.y) || !coarse_component(sd.z) || !coarse_component(sr)) {
        return false;
    }
    const double rx = srel.x, ry = srel.y, rz = srel.z, dx = sd.x, dy = sd.y, dz = sd.z, r2 = double(sr) * sr;
    const double ox2 = rx * rx, oy2 = ry * ry, oz2 = rz * rz;
    const DoubleDouble cc = dd_add(dd_add(dd_two_sum(ox2, oy2), DoubleDouble{oz2, 0.0}), DoubleDouble{-r2, 0.0});
    const double c_err = 0x1p-100 * (ox2 + oy2 + oz2 + r2);
    if (!(fabs(cc.hi) > 2.0 * c_err) || !certified_nearest(cc, c_err, c)) {
        return false;
    }
    const DoubleDouble dir2 = dd_add(dd_two_sum(dx * dx, dy * dy), DoubleDouble{dz * dz, 0.0});
    const DoubleDouble radial = dd_scale(dir2, r2);
    const DoubleDouble cx = dd_two_sum(ry * dz, -(rz * dy));
    const DoubleDouble cy = dd_two_sum(rz * dx, -(rx * dz));
    const DoubleDouble cz = dd_two_sum(rx * dy, -(ry * dx));
    const DoubleDouble perpendicular = dd_add(dd_add(dd_square(cx), dd_square(cy)), dd_square(cz));
    const DoubleDouble x = dd_add(radial, DoubleDouble{-perpendicular.hi, -perpendicular.lo});
    const double err = 0x1p-98 * (fabs(radial.hi) + fabs(perpendicular.hi));
    if (x.hi < -2.0 * err) {
        disc_sign = -1;
        disc = 0.0F;
        return true;
    }
    if (!(x.hi > 2.0 * err)) {
        return false;
    }
    disc_sign = 1;
    return certified_nearest(x, err, disc);
}

// robust_outward_normal (Sphere.hpp:245-267)
__device__ __forceinline__ bool sphere_outward_normal(F3 outward, F3& normal) {
    if (!finite3(outward)) {
        return false;
    }
    const float m = bf_max(bf_max(fabsf(outward.x), fabsf(outward.y)), fabsf(outward.z));
    if (m == 0.0F) {
        return false;
    }
    const F3 scaled{outward.x / m, outward.y / m, outward.z / m};
    const float magnitude = sqrtf(fused_dot3(scaled, scaled));
    if (!isfinite(magnitude) || magnitude <= 0.0F) {
        return false;
    }
    normal = F3{scaled.x / magnitude, scaled.y / magnitude, scaled.z / magnitude};
    return true;
}

struct SphereHit {
    int outcome;  // SphereOutcome
    float t;
    F3 normal;
};

// SphereT::intersect (Sphere.hpp:321-437) for the ray (o, d) restricted to [t_min, t_max]: the
// nearer root inside the interval, else the farther one. The surface point (Ray::at) and the
// outward normal are formed too, as the reference does before it reports a hit. Out of line, with
// every operand and the result by value: the expansions live in this call's frame, and no state of
// the calling walk needs an address (which would move it out of registers).
static __device__ __noinline__ SphereHit sphere_intersect(float4 centre4, float radius, F3 o, F3 d, float t_min,
                                                   float t_max) {
    SphereHit out{kSphereMiss, 0.0F, F3{0.0F, 0.0F, 0.0F}};
    const F3 centre{centre4.x, centre4.y, centre4.z};
    const F3 rel = o - centre;
    if (!finite3(rel)) {
        return SphereHit{kSphereFailure, 0.0F, F3{0.0F, 0.0F, 0.0F}};
    }
    const float spatial_maximum =
        bf_max(bf_max(bf_max(fabsf(rel.x), fabsf(rel.y)), fabsf(rel.z)), radius);
    const float direction_maximum = bf_max(bf_max(fabsf(d.x), fabsf(d.y)), fabsf(d.z));
    int spatial_exponent = 0, direction_exponent = 0;
    frexpf(spatial_maximum, &spatial_exponent);
    frexpf(direction_maximum, &direction_exponent);
    const F3 srel{ldexpf(rel.x, -spatial_exponent), ldexpf(rel.y, -spatial_exponent),
                  ldexpf(rel.z, -spatial_exponent)};
    const F3 sd{ldexpf(d.x, -direction_exponent), ldexpf(d.y, -direction_exponent), ldexpf(d.z, -direction_exponent)};
    const float sr = ldexpf(radius, -spatial_exponent);
    const auto preserved = [](float original, float scaled) { return original == 0.0F || is_normal_float(scaled); };
    if (!isfinite(direction_maximum) || direction_maximum <= 0.0F || !preserved(rel.x, srel.x) ||
        !preserved(rel.y, srel.y) || !preserved(rel.z, srel.z) || !preserved(d.x, sd.x) || !preserved(d.y, sd.y) ||
        !preserved(d.z, sd.z) || !preserved(radius, sr)) {
        return SphereHit{kSphereFailure, 0.0F, F3{0.0F, 0.0F, 0.0F}};
    }
    // Cull: the discriminant |d|^2 r^2 - |rel x d|^2 of the same float inputs in double. Every
    // product of two floats is exact in double, and the rounding of the few sums and products after
    // them stays below 16 u (|d|^2 r^2 + |rel x d|^2), u = 2^-53. A discriminant certainly below
    // zero means the ray misses the sphere, and the exact expansions are skipped. The reference's
    // test has no such cull; like the box cull of the BVH, it only skips spheres the ray does not
    // reach.
    {
        const double dx = sd.x, dy = sd.y, dz = sd.z, rx = srel.x, ry = srel.y, rz = srel.z, r2 = double(sr) * sr;
        const double radial = (dx * dx + dy * dy + dz * dz) * r2;
        const double cx = ry * dz - rz * dy, cy = rz * dx - rx * dz, cz = rx * dy - ry * dx;
        const double perpendicular = cx * cx + cy * cy + cz * cz;
        if (radial - perpendicular < -16.0 * 1.1102230246251565e-16 * (radial + perpendicular)) {
            return out;
        }
    }
    const float a = fused_dot3(sd, sd);
    const float half_b = fused_dot3(srel, sd);
    float c = 0.0F;
    int disc_sign = 0;
    float disc = 0.0F;
    if (!sphere_values_fast(srel, sd, sr, c, disc_sign, disc)) {
        if (!sphere_constant(srel, sr, c)) {
            return SphereHit{kSphereFailure, 0.0F, F3{0.0F, 0.0F, 0.0F}};
        }
        if (!sphere_discriminant(srel, sd, sr, disc_sign, disc)) {
            return SphereHit{kSphereFailure, 0.0F, F3{0.0F, 0.0F, 0.0F}};
        }
    }
    if (!isfinite(a) || !isfinite(half_b) || !isfinite(c) || a <= 0.0F || sr <= 0.0F) {
        return SphereHit{kSphereFailure, 0.0F, F3{0.0F, 0.0F, 0.0F}};
    }
    if (disc_sign < 0) {
        return out;
    }
    float r0, r1;
    if (disc_sign == 0) {
        r0 = -half_b / a;
        r1 = r0;
    } else {
        const float root = sqrtf(disc);
        const float q = -half_b - copysignf(root, half_b);
        if (!isfinite(root) || !isfinite(q) || q == 0.0F) {
            return SphereHit{kSphereFailure, 0.0F, F3{0.0F, 0.0F, 0.0F}};
        }
        r0 = q / a;
        r1 = c / q;
        if (r0 > r1) {
            const float swap = r0;
            r0 = r1;
            r1 = swap;
        }
    }
    const int parameter_exponent = spatial_exponent - direction_exponent;
    const float t0 = ldexpf(r0, parameter_exponent), t1 = ldexpf(r1, parameter_exponent);
    if (!isfinite(t0) || !isfinite(t1) || (r0 != 0.0F && t0 == 0.0F) || (r1 != 0.0F && t1 == 0.0F)) {
        return SphereHit{kSphereFailure, 0.0F, F3{0.0F, 0.0F, 0.0F}};
    }
    float t;
    if (!isnan(t0) && t0 >= t_min && t0 <= t_max) {
        t = t0;
    } else if (!isnan(t1) && t1 >= t_min && t1 <= t_max) {
        t = t1;
    } else {
        return out;
    }
    // Ray::at (Ray.hpp:81-95) and the outward normal at the hit
    const F3 position = o + d * t;
    if (!finite3(position) || !sphere_outward_normal(position - centre, out.normal)) {
        return SphereHit{kSphereFailure, 0.0F, F3{0.0F, 0.0F, 0.0F}};
    }
    out.outcome = kSphereHit;
    out.t = t;
    return out;
}

}  // namespace bf200
