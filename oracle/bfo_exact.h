// Oracle (test infrastructure): exact floating-expansion geometry of the reference scalar path.
//
// Restates Blackframe/Renderer/Include/Blackframe/Renderer/Triangle.hpp:78-839 and the mesh-light
// triangle area of AreaLights.hpp:439-543. Only tests and the CPU baselines use it; the product
// has its own device implementation.
//
// Two component types are used:
//   * float components, exactly as the reference does, for the triangle normal and the triangle
//     area. Those results are the float sum of the expansion components (resolve_expansion), so
//     they depend on the expansion's exact component layout and are reproduced bit for bit.
//   * double components for the ray/triangle test. The test's outputs (edge signs, the
//     correctly rounded parameter and barycentrics) are mathematically canonical, so any exact
//     evaluation returns the same values wherever the reference succeeds; double components do
//     not underflow on the tiny error terms that make the float version report "not exactly
//     representable" (Triangle.hpp:262-274).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

namespace bfo {

struct V3 {
    float x, y, z;
};

inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline bool operator==(V3 a, V3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline bool operator!=(V3 a, V3 b) { return !(a == b); }
// GeometryTypes.hpp:202-238: dot is left-to-right x, y, z without contraction.
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline bool finite3(V3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }

// ---------------------------------------------------------------------------------------------
// Floating expansions (Triangle.hpp:78-199)
// ---------------------------------------------------------------------------------------------

template <typename S, int N> struct Expansion {
    S c[N];
    int size = 0;
};

// Triangle.hpp:83-121 (grow-expansion with zero elimination).
template <typename S, int N> bool add_component(Expansion<S, N>& e, S component) {
    if (!std::isfinite(component)) {
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
        const S existing_remainder = existing - existing_from_sum;
        const S accumulated_remainder = accumulated - accumulated_from_sum;
        const S error = existing_remainder + accumulated_remainder;
        if (!std::isfinite(rounded_sum) || !std::isfinite(error)) {
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

// Triangle.hpp:123-135 (two-product with an fma residual; rejects subnormal products).
template <typename S, int N> bool add_product(Expansion<S, N>& e, S left, S right, S sign = S(1)) {
    const S rounded = left * right;
    const S error = std::fma(left, right, -rounded);
    if (!std::isfinite(rounded) || !std::isfinite(error) ||
        (left != S(0) && right != S(0) && !std::isnormal(rounded)) ||
        (error != S(0) && !std::isnormal(error))) {
        return false;
    }
    return add_component(e, sign * error) && add_component(e, sign * rounded);
}

template <typename S, int N, int M>
bool add_expansion(Expansion<S, N>& dst, const Expansion<S, M>& src, S sign = S(1)) {
    for (int i = 0; i < src.size; ++i) {
        if (!add_component(dst, sign * src.c[i])) {
            return false;
        }
    }
    return true;
}

template <typename S, int O, int L, int R>
bool multiply_expansions(const Expansion<S, L>& left, const Expansion<S, R>& right,
                         Expansion<S, O>& product) {
    product.size = 0;
    for (int i = 0; i < left.size; ++i) {
        for (int j = 0; j < right.size; ++j) {
            if (!add_product(product, left.c[i], right.c[j])) {
                return false;
            }
        }
    }
    return true;
}

template <typename S, int N> int expansion_sign(const Expansion<S, N>& e) {
    for (int i = e.size; i > 0; --i) {
        if (e.c[i - 1] != S(0)) {
            return e.c[i - 1] > S(0) ? 1 : -1;
        }
    }
    return 0;
}

template <typename S> struct ExactValue {
    int sign = 0;
    S value = S(0);
};

// Triangle.hpp:182-199: the value is the in-order float sum of the components.
template <typename S, int N> bool resolve_expansion(const Expansion<S, N>& e, ExactValue<S>& out) {
    const int sign = expansion_sign(e);
    if (sign == 0) {
        out = ExactValue<S>{0, S(0)};
        return true;
    }
    S value = S(0);
    for (int i = 0; i < e.size; ++i) {
        value += e.c[i];
    }
    if (!std::isfinite(value) || value == S(0) || (value > S(0) ? 1 : -1) != sign) {
        return false;
    }
    out = ExactValue<S>{sign, value};
    return true;
}

template <typename S> using Coord = Expansion<S, 2>;

template <typename S> struct EV3 {
    Coord<S> x, y, z;
};

template <typename S> bool exact_difference(S left, S right, Coord<S>& d) {
    d.size = 0;
    return add_component(d, left) && add_component(d, -right);
}

template <typename S> bool exact_relative(V3 point, V3 origin, EV3<S>& r) {
    return exact_difference<S>(S(point.x), S(origin.x), r.x) &&
           exact_difference<S>(S(point.y), S(origin.y), r.y) &&
           exact_difference<S>(S(point.z), S(origin.z), r.z);
}

template <typename S> EV3<S> exact_vector(V3 v) {
    EV3<S> r;
    r.x.c[0] = S(v.x);
    r.x.size = 1;
    r.y.c[0] = S(v.y);
    r.y.size = 1;
    r.z.c[0] = S(v.z);
    r.z.size = 1;
    return r;
}

template <typename S> using Pair = Expansion<S, 16>;
template <typename S> using Triple = Expansion<S, 64>;
template <typename S> using Det = Expansion<S, 512>;

template <typename S>
bool add_triple_product(Det<S>& det, const Coord<S>& a, const Coord<S>& b, const Coord<S>& c,
                        S sign) {
    Pair<S> pair;
    Triple<S> triple;
    return multiply_expansions(a, b, pair) && multiply_expansions(pair, c, triple) &&
           add_expansion(det, triple, sign);
}

// Triangle.hpp:260-275.
template <typename S>
bool exact_determinant(const EV3<S>& a, const EV3<S>& b, const EV3<S>& c, Det<S>& det) {
    det.size = 0;
    return add_triple_product(det, a.x, b.y, c.z, S(1)) &&
           add_triple_product(det, a.y, b.z, c.x, S(1)) &&
           add_triple_product(det, a.z, b.x, c.y, S(1)) &&
           add_triple_product(det, a.z, b.y, c.x, S(-1)) &&
           add_triple_product(det, a.y, b.x, c.z, S(-1)) &&
           add_triple_product(det, a.x, b.z, c.y, S(-1));
}

template <typename S> using CrossC = Expansion<S, 32>;

template <typename S>
bool exact_difference_of_products(const Coord<S>& fl, const Coord<S>& fr, const Coord<S>& sl,
                                  const Coord<S>& sr, CrossC<S>& d) {
    Pair<S> first, second;
    d.size = 0;
    return multiply_expansions(fl, fr, first) && multiply_expansions(sl, sr, second) &&
           add_expansion(d, first) && add_expansion(d, second, S(-1));
}

// Triangle.hpp:309-318.
template <int K> int scaling_exponent(const float (&values)[K]) {
    float maximum = 0.0F;
    for (float v : values) {
        maximum = std::max(maximum, std::abs(v));
    }
    int exponent = 0;
    (void)std::frexp(maximum, &exponent);
    return exponent;
}

struct AxisExp {
    int x, y, z;
};

inline V3 scaled_point(V3 p, AxisExp e) {
    return {std::ldexp(p.x, -e.x), std::ldexp(p.y, -e.y), std::ldexp(p.z, -e.z)};
}

inline bool scaling_preserves(float original, float scaled) {
    return original == 0.0F || std::isnormal(scaled);
}
inline bool scaling_preserves(V3 o, V3 s) {
    return scaling_preserves(o.x, s.x) && scaling_preserves(o.y, s.y) &&
           scaling_preserves(o.z, s.z);
}

// Triangle.hpp:374-481: the geometric normal of (v0, v1, v2), float expansions.
inline bool triangle_normal(V3 v0, V3 v1, V3 v2, V3& out) {
    const AxisExp e{scaling_exponent<3>({v0.x, v1.x, v2.x}), scaling_exponent<3>({v0.y, v1.y, v2.y}),
                    scaling_exponent<3>({v0.z, v1.z, v2.z})};
    const V3 s0 = scaled_point(v0, e), s1 = scaled_point(v1, e), s2 = scaled_point(v2, e);
    if (!scaling_preserves(v0, s0) || !scaling_preserves(v1, s1) || !scaling_preserves(v2, s2)) {
        return false;
    }
    EV3<float> e1, e2;
    if (!exact_relative<float>(s1, s0, e1) || !exact_relative<float>(s2, s0, e2)) {
        return false;
    }
    CrossC<float> cx, cy, cz;
    if (!exact_difference_of_products(e1.y, e2.z, e1.z, e2.y, cx) ||
        !exact_difference_of_products(e1.z, e2.x, e1.x, e2.z, cy) ||
        !exact_difference_of_products(e1.x, e2.y, e1.y, e2.x, cz)) {
        return false;
    }
    ExactValue<float> x, y, z;
    if (!resolve_expansion(cx, x) || !resolve_expansion(cy, y) || !resolve_expansion(cz, z)) {
        return false;
    }
    if (x.sign == 0 && y.sign == 0 && z.sign == 0) {
        return false;
    }
    const AxisExp ce{e.y + e.z, e.z + e.x, e.x + e.y};
    int normal_exponent = std::numeric_limits<int>::min();
    auto include = [&](ExactValue<float> c, int ex) {
        if (c.sign == 0) {
            return;
        }
        int ce2 = 0;
        (void)std::frexp(std::abs(c.value), &ce2);
        normal_exponent = std::max(normal_exponent, ce2 + ex);
    };
    include(x, ce.x);
    include(y, ce.y);
    include(z, ce.z);
    const float ax = x.sign == 0 ? 0.0F : std::ldexp(x.value, ce.x - normal_exponent);
    const float ay = y.sign == 0 ? 0.0F : std::ldexp(y.value, ce.y - normal_exponent);
    const float az = z.sign == 0 ? 0.0F : std::ldexp(z.value, ce.z - normal_exponent);
    if (!scaling_preserves(x.value, ax) || !scaling_preserves(y.value, ay) ||
        !scaling_preserves(z.value, az)) {
        return false;
    }
    const float m = std::max({std::abs(ax), std::abs(ay), std::abs(az)});
    if (!std::isfinite(m) || m <= 0.0F) {
        return false;
    }
    const float sx = ax / m, sy = ay / m, sz = az / m;
    const float squared = std::fma(sx, sx, std::fma(sy, sy, sz * sz));
    const float length = std::sqrt(squared);
    if (!std::isfinite(length) || length <= 0.0F) {
        return false;
    }
    out = V3{sx / length, sy / length, sz / length};
    return true;
}

// AreaLights.hpp:439-543: triangle area of a mesh-light triangle, float expansions.
inline bool triangle_area(V3 v0, V3 v1, V3 v2, float& area) {
    const AxisExp e{scaling_exponent<3>({v0.x, v1.x, v2.x}), scaling_exponent<3>({v0.y, v1.y, v2.y}),
                    scaling_exponent<3>({v0.z, v1.z, v2.z})};
    const V3 s0 = scaled_point(v0, e), s1 = scaled_point(v1, e), s2 = scaled_point(v2, e);
    if (!scaling_preserves(v0, s0) || !scaling_preserves(v1, s1) || !scaling_preserves(v2, s2)) {
        return false;
    }
    EV3<float> first, second;
    if (!exact_relative<float>(s1, s0, first) || !exact_relative<float>(s2, s0, second)) {
        return false;
    }
    CrossC<float> cx, cy, cz;
    if (!exact_difference_of_products(first.y, second.z, first.z, second.y, cx) ||
        !exact_difference_of_products(first.z, second.x, first.x, second.z, cy) ||
        !exact_difference_of_products(first.x, second.y, first.y, second.x, cz)) {
        return false;
    }
    ExactValue<float> x, y, z;
    if (!resolve_expansion(cx, x) || !resolve_expansion(cy, y) || !resolve_expansion(cz, z)) {
        return false;
    }
    const AxisExp ce{e.y + e.z, e.z + e.x, e.x + e.y};
    int me = std::numeric_limits<int>::min();
    auto include = [&](ExactValue<float> c, int ex) {
        if (c.sign == 0) {
            return;
        }
        int ve = 0;
        (void)std::frexp(std::abs(c.value), &ve);
        me = std::max(me, ve + ex);
    };
    include(x, ce.x);
    include(y, ce.y);
    include(z, ce.z);
    if (me == std::numeric_limits<int>::min()) {
        return false;
    }
    const float ax = x.sign == 0 ? 0.0F : std::ldexp(x.value, ce.x - me);
    const float ay = y.sign == 0 ? 0.0F : std::ldexp(y.value, ce.y - me);
    const float az = z.sign == 0 ? 0.0F : std::ldexp(z.value, ce.z - me);
    if ((x.sign != 0 && ax == 0.0F) || (y.sign != 0 && ay == 0.0F) || (z.sign != 0 && az == 0.0F) ||
        !std::isfinite(ax) || !std::isfinite(ay) || !std::isfinite(az)) {
        return false;
    }
    const float adjusted_length = std::hypot(ax, ay, az);
    area = std::scalbn(adjusted_length * 0.5F, me);
    return std::isfinite(adjusted_length) && adjusted_length > 0.0F && std::isfinite(area) &&
           area > 0.0F;
}

// ---------------------------------------------------------------------------------------------
// Ray/triangle intersection (Triangle.hpp:517-822) with double components
// ---------------------------------------------------------------------------------------------

template <int N, int M>
int quotient_residual_sign(const Expansion<double, N>& num, const Expansion<double, M>& den,
                           double candidate, bool& ok) {
    Expansion<double, N + 2 * M + 8> residual;
    ok = add_expansion(residual, num);
    for (int i = 0; ok && i < den.size; ++i) {
        ok = add_product(residual, den.c[i], candidate, -1.0);
    }
    return ok ? expansion_sign(residual) : 0;
}

template <int N, int M>
int quotient_midpoint_sign(const Expansion<double, N>& num, const Expansion<double, M>& den,
                           double lower, double upper, bool& ok) {
    Expansion<double, 2 * N + 4 * M + 8> cmp;
    ok = true;
    for (int i = 0; ok && i < num.size; ++i) {
        ok = add_product(cmp, num.c[i], 2.0);
    }
    for (int i = 0; ok && i < den.size; ++i) {
        ok = add_product(cmp, den.c[i], lower, -1.0);
    }
    for (int i = 0; ok && i < den.size; ++i) {
        ok = add_product(cmp, den.c[i], upper, -1.0);
    }
    return ok ? expansion_sign(cmp) : 0;
}

// Triangle.hpp:566-645: the float nearest to num/den (ties to even), refined exactly.
template <int N, int M>
bool correctly_rounded_quotient(const Expansion<double, N>& num, const Expansion<double, M>& den,
                                float& out) {
    const int num_sign = expansion_sign(num);
    const int den_sign = expansion_sign(den);
    if (den_sign == 0) {
        return false;
    }
    if (num_sign == 0) {
        out = 0.0F;
        return true;
    }
    double nv = 0.0, dv = 0.0;
    for (int i = 0; i < num.size; ++i) {
        nv += num.c[i];
    }
    for (int i = 0; i < den.size; ++i) {
        dv += den.c[i];
    }
    float candidate = static_cast<float>(nv / dv);
    if (!std::isfinite(candidate) || candidate == 0.0F || !std::isnormal(candidate)) {
        return false;
    }
    for (int correction = 0; correction < 26; ++correction) {
        bool ok = true;
        const int r = quotient_residual_sign(num, den, candidate, ok);
        if (!ok) {
            return false;
        }
        if (r == 0) {
            out = candidate;
            return true;
        }
        const int direction = r * den_sign;
        const float neighbor = std::nextafter(
            candidate, direction > 0 ? std::numeric_limits<float>::infinity()
                                     : -std::numeric_limits<float>::infinity());
        if (!std::isfinite(neighbor) || neighbor == 0.0F || !std::isnormal(neighbor)) {
            return false;
        }
        const int nr = quotient_residual_sign(num, den, neighbor, ok);
        if (!ok) {
            return false;
        }
        if (nr == 0) {
            out = neighbor;
            return true;
        }
        if (nr * den_sign == direction) {
            candidate = neighbor;
            continue;
        }
        const float lower = std::min(candidate, neighbor);
        const float upper = std::max(candidate, neighbor);
        const int mid = quotient_midpoint_sign(num, den, lower, upper, ok) * den_sign;
        if (!ok) {
            return false;
        }
        if (mid < 0) {
            out = lower;
            return true;
        }
        if (mid > 0) {
            out = upper;
            return true;
        }
        uint32_t bits;
        std::memcpy(&bits, &lower, 4);
        out = (bits & 1U) == 0 ? lower : upper;
        return true;
    }
    return false;
}

enum class TriResult { miss, hit, coplanar, failure };

struct TriHit {
    float t;
    float b0, b1, b2;
};

// Triangle.hpp:683-822 (intersect_classified). Ray parameter interval is closed.
inline TriResult intersect_triangle(V3 v0, V3 v1, V3 v2, V3 o, V3 d, float t_min, float t_max,
                                    TriHit& hit) {
    const AxisExp e{scaling_exponent<4>({v0.x, v1.x, v2.x, o.x}),
                    scaling_exponent<4>({v0.y, v1.y, v2.y, o.y}),
                    scaling_exponent<4>({v0.z, v1.z, v2.z, o.z})};
    int de = std::numeric_limits<int>::min();
    auto include = [&](float c, int se) {
        if (c == 0.0F) {
            return;
        }
        int ce = 0;
        (void)std::frexp(std::abs(c), &ce);
        de = std::max(de, ce - se);
    };
    include(d.x, e.x);
    include(d.y, e.y);
    include(d.z, e.z);
    const V3 s0 = scaled_point(v0, e), s1 = scaled_point(v1, e), s2 = scaled_point(v2, e);
    const V3 so = scaled_point(o, e);
    const V3 sd{std::ldexp(d.x, -e.x - de), std::ldexp(d.y, -e.y - de), std::ldexp(d.z, -e.z - de)};
    if (!scaling_preserves(v0, s0) || !scaling_preserves(v1, s1) || !scaling_preserves(v2, s2) ||
        !scaling_preserves(o, so) || !scaling_preserves(d, sd)) {
        return TriResult::failure;
    }
    EV3<double> p0, p1, p2;
    if (!exact_relative<double>(s0, so, p0) || !exact_relative<double>(s1, so, p1) ||
        !exact_relative<double>(s2, so, p2)) {
        return TriResult::failure;
    }
    const EV3<double> dir = exact_vector<double>(sd);
    static thread_local Det<double> edge0, edge1, edge2, volume, det;
    if (!exact_determinant(p1, p2, dir, edge0) || !exact_determinant(p2, p0, dir, edge1) ||
        !exact_determinant(p0, p1, dir, edge2) || !exact_determinant(p0, p1, p2, volume)) {
        return TriResult::failure;
    }
    det.size = 0;
    if (!add_expansion(det, edge0) || !add_expansion(det, edge1) || !add_expansion(det, edge2)) {
        return TriResult::failure;
    }
    const int ds = expansion_sign(det);
    const int vs = expansion_sign(volume);
    if (ds == 0) {
        return vs == 0 ? TriResult::coplanar : TriResult::miss;
    }
    const int e0 = expansion_sign(edge0), e1 = expansion_sign(edge1), e2 = expansion_sign(edge2);
    const bool nonneg = e0 >= 0 && e1 >= 0 && e2 >= 0;
    const bool nonpos = e0 <= 0 && e1 <= 0 && e2 <= 0;
    if (!nonneg && !nonpos) {
        return TriResult::miss;
    }
    float scaled_t;
    if (!correctly_rounded_quotient(volume, det, scaled_t)) {
        return TriResult::failure;
    }
    const float t = std::ldexp(scaled_t, -de);
    if (!std::isfinite(t) || (scaled_t != 0.0F && t == 0.0F)) {
        return TriResult::failure;
    }
    if (std::isnan(t) || t < t_min || t > t_max) {
        return TriResult::miss;
    }
    float b0, b1, b2;
    if (!correctly_rounded_quotient(edge0, det, b0) || !correctly_rounded_quotient(edge1, det, b1) ||
        !correctly_rounded_quotient(edge2, det, b2)) {
        return TriResult::failure;
    }
    hit = TriHit{t, b0, b1, b2};
    return TriResult::hit;
}

}  // namespace bfo
