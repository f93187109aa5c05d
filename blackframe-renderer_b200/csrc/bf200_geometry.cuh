// Exact geometry shared by the host scene build and the device kernels.
//
// * triangle_normal / triangle_area: the float floating-expansion construction of the
//   reference's Triangle::create normal (Blackframe/Renderer/Include/Blackframe/Renderer/
//   Triangle.hpp:374-481) and of the mesh-light triangle area (AreaLights.hpp:439-543). Their
//   results are the in-order float sum of the expansion components, so the component layout is
//   reproduced operation for operation.
// * exact_triangle_test: the ray/triangle test of Triangle.hpp:683-822 returning the exact edge
//   signs and the correctly rounded parameter and barycentrics. The device evaluates it in
//   double with a forward error bound and falls back to double-component expansions only when
//   a sign or a rounding is ambiguous.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define BF_HD __host__ __device__ __forceinline__
#define BF_HD_NOINLINE __host__ __device__ __noinline__
#else
#define BF_HD inline
#define BF_HD_NOINLINE
#endif

#include <cmath>
#include <cstring>

namespace bf200 {

struct F3 {
    float x, y, z;
};

BF_HD F3 make_f3(float x, float y, float z) { return F3{x, y, z}; }

BF_HD float bf_abs(float v) { return fabsf(v); }
BF_HD double bf_absd(double v) { return fabs(v); }
// std::max(a, b) returns a unless a < b.
BF_HD float bf_max(float a, float b) { return (a < b) ? b : a; }
BF_HD float bf_min(float a, float b) { return (b < a) ? b : a; }
BF_HD int bf_maxi(int a, int b) { return (a < b) ? b : a; }
BF_HD bool bf_finite(float v) { return isfinite(v); }
BF_HD bool bf_isnormal_f(float v) {
    const float a = fabsf(v);
    return a >= 1.17549435e-38F && a <= 3.40282347e+38F;
}
BF_HD bool bf_isnormal_d(double v) {
    const double a = fabs(v);
    return a >= 2.2250738585072014e-308 && a <= 1.7976931348623157e+308;
}

// ---------------------------------------------------------------------------------------------
// Float expansions (grow-expansion with zero elimination, Triangle.hpp:83-199)
// ---------------------------------------------------------------------------------------------

template <typename S, int N> struct Expansion {
    S c[N];
    int size;
};

template <typename S, int N> BF_HD bool exp_add(Expansion<S, N>& e, S component) {
    if (!isfinite(component)) {
        return false;
    }
    S accumulated = component;
    int out = 0;
    const int input_size = e.size;
    for (int i = 0; i < input_size; ++i) {
        const S existing = e.c[i];
        const S rounded_sum = accumulated + existing;
        const S existing_from_sum = rounded_sum - accumulated;
        const S accumulated_from_sum = rounded_sum - existing_from_sum;
        const S error = (existing - existing_from_sum) + (accumulated - accumulated_from_sum);
        if (!isfinite(rounded_sum) || !isfinite(error)) {
            return false;
        }
        if (error != S(0)) {
            if (out == N) {
                return false;
            }
            e.c[out++] = error;
        }
        accumulated = rounded_sum;
    }
    if (accumulated != S(0) || out == 0) {
        if (out == N) {
            return false;
        }
        e.c[out++] = accumulated;
    }
    e.size = out;
    return true;
}

BF_HD bool product_ok(float l, float r, float p, float err) {
    return isfinite(p) && isfinite(err) && !(l != 0.0F && r != 0.0F && !bf_isnormal_f(p)) &&
           !(err != 0.0F && !bf_isnormal_f(err));
}
BF_HD bool product_ok(double l, double r, double p, double err) {
    return isfinite(p) && isfinite(err) && !(l != 0.0 && r != 0.0 && !bf_isnormal_d(p)) &&
           !(err != 0.0 && !bf_isnormal_d(err));
}

template <int N> BF_HD bool exp_add_product(Expansion<float, N>& e, float l, float r, float sign) {
    const float p = l * r;
    const float err = fmaf(l, r, -p);
    if (!product_ok(l, r, p, err)) {
        return false;
    }
    return exp_add(e, sign * err) && exp_add(e, sign * p);
}

template <int N> BF_HD bool exp_add_product(Expansion<double, N>& e, double l, double r, double sign) {
    const double p = l * r;
    const double err = fma(l, r, -p);
    if (!product_ok(l, r, p, err)) {
        return false;
    }
    return exp_add(e, sign * err) && exp_add(e, sign * p);
}

template <typename S, int O, int L, int R>
BF_HD bool exp_multiply(const Expansion<S, L>& a, const Expansion<S, R>& b, Expansion<S, O>& out) {
    out.size = 0;
    for (int i = 0; i < a.size; ++i) {
        for (int j = 0; j < b.size; ++j) {
            if (!exp_add_product(out, a.c[i], b.c[j], S(1))) {
                return false;
            }
        }
    }
    return true;
}

template <typename S, int N, int M>
BF_HD bool exp_add_expansion(Expansion<S, N>& dst, const Expansion<S, M>& src, S sign) {
    for (int i = 0; i < src.size; ++i) {
        if (!exp_add(dst, sign * src.c[i])) {
            return false;
        }
    }
    return true;
}

template <typename S, int N> BF_HD int exp_sign(const Expansion<S, N>& e) {
    for (int i = e.size; i > 0; --i) {
        if (e.c[i - 1] != S(0)) {
            return e.c[i - 1] > S(0) ? 1 : -1;
        }
    }
    return 0;
}

// resolve_expansion: the in-order float sum of the components (Triangle.hpp:182-199).
template <int N> BF_HD bool exp_resolve(const Expansion<float, N>& e, int& sign, float& value) {
    sign = exp_sign(e);
    value = 0.0F;
    if (sign == 0) {
        return true;
    }
    for (int i = 0; i < e.size; ++i) {
        value += e.c[i];
    }
    return isfinite(value) && value != 0.0F && (value > 0.0F ? 1 : -1) == sign;
}

BF_HD uint32_t float_bits(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
#endif
}

BF_HD int frexp_exponent(float v) {
    int e = 0;
    (void)frexpf(v, &e);
    return e;
}

BF_HD int axis_exponent3(float a, float b, float c) {
    float m = 0.0F;
    m = bf_max(m, bf_abs(a));
    m = bf_max(m, bf_abs(b));
    m = bf_max(m, bf_abs(c));
    return frexp_exponent(m);
}

BF_HD bool scaling_preserves(float original, float scaled) {
    return original == 0.0F || bf_isnormal_f(scaled);
}

// exact difference (left - right) as a 2-component float expansion
BF_HD bool exact_diff_f(float left, float right, Expansion<float, 2>& d) {
    d.size = 0;
    return exp_add(d, left) && exp_add(d, -right);
}

// first_left*first_right - second_left*second_right (Triangle.hpp:279-296)
BF_HD bool diff_of_products(const Expansion<float, 2>& fl, const Expansion<float, 2>& fr,
                            const Expansion<float, 2>& sl, const Expansion<float, 2>& sr,
                            Expansion<float, 32>& out) {
    Expansion<float, 16> first, second;
    out.size = 0;
    return exp_multiply(fl, fr, first) && exp_multiply(sl, sr, second) &&
           exp_add_expansion(out, first, 1.0F) && exp_add_expansion(out, second, -1.0F);
}

struct CrossResolved {
    int sign[3];
    float value[3];
    int exponent[3];  // per-component scale of the cross product
};

// The exact cross product of (v1 - v0) x (v2 - v0) after per-axis power-of-two scaling.
BF_HD bool exact_cross(F3 v0, F3 v1, F3 v2, CrossResolved& out) {
    const int ex = axis_exponent3(v0.x, v1.x, v2.x);
    const int ey = axis_exponent3(v0.y, v1.y, v2.y);
    const int ez = axis_exponent3(v0.z, v1.z, v2.z);
    const F3 s0{ldexpf(v0.x, -ex), ldexpf(v0.y, -ey), ldexpf(v0.z, -ez)};
    const F3 s1{ldexpf(v1.x, -ex), ldexpf(v1.y, -ey), ldexpf(v1.z, -ez)};
    const F3 s2{ldexpf(v2.x, -ex), ldexpf(v2.y, -ey), ldexpf(v2.z, -ez)};
    const F3 originals[3] = {v0, v1, v2};
    const F3 scaled[3] = {s0, s1, s2};
    for (int k = 0; k < 3; ++k) {
        if (!scaling_preserves(originals[k].x, scaled[k].x) ||
            !scaling_preserves(originals[k].y, scaled[k].y) ||
            !scaling_preserves(originals[k].z, scaled[k].z)) {
            return false;
        }
    }
    Expansion<float, 2> e1x, e1y, e1z, e2x, e2y, e2z;
    if (!exact_diff_f(s1.x, s0.x, e1x) || !exact_diff_f(s1.y, s0.y, e1y) ||
        !exact_diff_f(s1.z, s0.z, e1z) || !exact_diff_f(s2.x, s0.x, e2x) ||
        !exact_diff_f(s2.y, s0.y, e2y) || !exact_diff_f(s2.z, s0.z, e2z)) {
        return false;
    }
    Expansion<float, 32> cx, cy, cz;
    if (!diff_of_products(e1y, e2z, e1z, e2y, cx) || !diff_of_products(e1z, e2x, e1x, e2z, cy) ||
        !diff_of_products(e1x, e2y, e1y, e2x, cz)) {
        return false;
    }
    if (!exp_resolve(cx, out.sign[0], out.value[0]) || !exp_resolve(cy, out.sign[1], out.value[1]) ||
        !exp_resolve(cz, out.sign[2], out.value[2])) {
        return false;
    }
    out.exponent[0] = ey + ez;
    out.exponent[1] = ez + ex;
    out.exponent[2] = ex + ey;
    return true;
}

// Triangle.hpp:374-481: the geometric normal of a triangle.
BF_HD bool triangle_normal(F3 v0, F3 v1, F3 v2, F3& normal) {
    CrossResolved c;
    if (!exact_cross(v0, v1, v2, c)) {
        return false;
    }
    if (c.sign[0] == 0 && c.sign[1] == 0 && c.sign[2] == 0) {
        return false;
    }
    int ne = -2147483647 - 1;
    for (int k = 0; k < 3; ++k) {
        if (c.sign[k] != 0) {
            ne = bf_maxi(ne, frexp_exponent(bf_abs(c.value[k])) + c.exponent[k]);
        }
    }
    float adjusted[3];
    for (int k = 0; k < 3; ++k) {
        adjusted[k] = c.sign[k] == 0 ? 0.0F : ldexpf(c.value[k], c.exponent[k] - ne);
        if (!scaling_preserves(c.value[k], adjusted[k])) {
            return false;
        }
    }
    float m = bf_max(bf_max(bf_abs(adjusted[0]), bf_abs(adjusted[1])), bf_abs(adjusted[2]));
    if (!isfinite(m) || m <= 0.0F) {
        return false;
    }
    const float sx = adjusted[0] / m, sy = adjusted[1] / m, sz = adjusted[2] / m;
    const float squared = fmaf(sx, sx, fmaf(sy, sy, sz * sz));
    const float length = sqrtf(squared);
    if (!isfinite(length) || length <= 0.0F) {
        return false;
    }
    normal = F3{sx / length, sy / length, sz / length};
    return true;
}

// libstdc++ std::hypot(float, float, float): scale by the largest magnitude, sqrt of the sum.
BF_HD float hypot3f(float x, float y, float z) {
    x = fabsf(x);
    y = fabsf(y);
    z = fabsf(z);
    const float a = x < y ? (y < z ? z : y) : (x < z ? z : x);
    if (a != 0.0F) {
        const float xa = x / a, ya = y / a, za = z / a;
        return a * sqrtf(xa * xa + ya * ya + za * za);
    }
    return 0.0F;
}

// glibc hypotf: both squares are exact in double; one double rounding of the sum and of the root.
BF_HD float hypot2f(float x, float y) {
    const double dx = static_cast<double>(x), dy = static_cast<double>(y);
    return static_cast<float>(sqrt(dx * dx + dy * dy));
}

// AreaLights.hpp:439-543: the area of a mesh-light triangle.
BF_HD bool triangle_area(F3 v0, F3 v1, F3 v2, float& area) {
    CrossResolved c;
    if (!exact_cross(v0, v1, v2, c)) {
        return false;
    }
    int me = -2147483647 - 1;
    for (int k = 0; k < 3; ++k) {
        if (c.sign[k] != 0) {
            me = bf_maxi(me, frexp_exponent(bf_abs(c.value[k])) + c.exponent[k]);
        }
    }
    if (me == -2147483647 - 1) {
        return false;
    }
    float adjusted[3];
    for (int k = 0; k < 3; ++k) {
        adjusted[k] = c.sign[k] == 0 ? 0.0F : ldexpf(c.value[k], c.exponent[k] - me);
        if ((c.sign[k] != 0 && adjusted[k] == 0.0F) || !isfinite(adjusted[k])) {
            return false;
        }
    }
    const float length = hypot3f(adjusted[0], adjusted[1], adjusted[2]);
    area = scalbnf(length * 0.5F, me);
    return isfinite(length) && length > 0.0F && isfinite(area) && area > 0.0F;
}

// ---------------------------------------------------------------------------------------------
// Ray / triangle test with exact results
// ---------------------------------------------------------------------------------------------

struct TriangleHit {
    float t;
    float b0, b1, b2;
};

enum TriangleOutcome : int { kTriMiss = 0, kTriHit = 1, kTriFailure = 2 };

// Double-component expansion of one determinant of three vectors whose components are single
// doubles (exact float differences). Each triple product x*y*z of doubles is exact as two
// two-products: x*y = p + e, then p*z and e*z.
template <int N> BF_HD bool exp_add_triple(Expansion<double, N>& e, double x, double y, double z,
                                            double sign) {
    const double p = x * y;
    const double pe = fma(x, y, -p);
    return exp_add_product(e, pe, z, sign) && exp_add_product(e, p, z, sign);
}

template <int N>
BF_HD bool exp_det3(Expansion<double, N>& e, const double* a, const double* b, const double* c) {
    e.size = 0;
    return exp_add_triple(e, a[0], b[1], c[2], 1.0) && exp_add_triple(e, a[1], b[2], c[0], 1.0) &&
           exp_add_triple(e, a[2], b[0], c[1], 1.0) && exp_add_triple(e, a[2], b[1], c[0], -1.0) &&
           exp_add_triple(e, a[1], b[0], c[2], -1.0) && exp_add_triple(e, a[0], b[2], c[1], -1.0);
}

// Sign of num - q * den for a float candidate q (exact).
template <int N, int M>
BF_HD bool residual_sign(const Expansion<double, N>& num, const Expansion<double, M>& den, double q,
                         double twice_scale, int& sign) {
    Expansion<double, N + 2 * M + 4> r;
    r.size = 0;
    for (int i = 0; i < num.size; ++i) {
        if (!exp_add_product(r, num.c[i], twice_scale, 1.0)) {
            return false;
        }
    }
    for (int i = 0; i < den.size; ++i) {
        if (!exp_add_product(r, den.c[i], q, -1.0)) {
            return false;
        }
    }
    sign = exp_sign(r);
    return true;
}

// The float nearest to num/den (ties to even), decided exactly. `approx` seeds the search.
template <int N, int M>
BF_HD bool exact_round_quotient(const Expansion<double, N>& num, const Expansion<double, M>& den,
                                float approx, float& out) {
    const int ds = exp_sign(den);
    if (ds == 0) {
        return false;
    }
    if (exp_sign(num) == 0) {
        out = 0.0F;
        return true;
    }
    float candidate = approx;
    if (!isfinite(candidate) || candidate == 0.0F) {
        return false;
    }
    for (int step = 0; step < 28; ++step) {
        int r = 0;
        if (!residual_sign(num, den, static_cast<double>(candidate), 1.0, r)) {
            return false;
        }
        if (r == 0) {
            out = candidate;
            return true;
        }
        const int direction = r * ds;
        const float neighbor = nextafterf(candidate, direction > 0 ? INFINITY : -INFINITY);
        int nr = 0;
        if (!residual_sign(num, den, static_cast<double>(neighbor), 1.0, nr)) {
            return false;
        }
        if (nr == 0) {
            out = neighbor;
            return true;
        }
        if (nr * ds == direction) {
            candidate = neighbor;
            continue;
        }
        const float lower = bf_min(candidate, neighbor);
        const float upper = bf_max(candidate, neighbor);
        // sign of 2*num - (lower + upper)*den: lower + upper is exact in double.
        int mid = 0;
        if (!residual_sign(num, den, static_cast<double>(lower) + static_cast<double>(upper), 2.0,
                           mid)) {
            return false;
        }
        mid *= ds;
        if (mid < 0) {
            out = lower;
        } else if (mid > 0) {
            out = upper;
        } else {
            out = (float_bits(lower) & 1U) == 0U ? lower : upper;
        }
        return true;
    }
    return false;
}

}  // namespace bf200
