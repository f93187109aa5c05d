// bf200 device kernels: scene setup, exact-robust BVH traversal, the persistent wavefront
// (regenerate -> trace -> route -> shade with NEE -> occlusion) and film accumulation.
//
// Hot-path mapping to the reference CUDA backend (Blackframe/XPU/CUDA/Source):
//   k_regenerate : path retirement and regeneration with device camera rays (seed/camera stages,
//                  CudaWavefrontStages.cu:1269-1406)
//   k_trace      : scene_closest_hit_kernel + classify/miss stages (CudaSceneClosestHit.cu:1199,
//                  CudaWavefrontStages.cu:1434, :3962); writes each slot's shading route
//   k_shade<K>   : shade_stage_kernel (CudaWavefrontStages.cu:4107-4727), one instantiation per
//                  closure kind over that route's queue (bf200_compact.cu builds the queues)
//   k_occlude    : scene_occlusion_kernel + process_shadow_kernel (CudaSceneClosestHit.cu:1243,
//                  CudaWavefrontStages.cu:4772-4908) over the compacted shadow queue
//   k_film       : the caller-side CIE XYZ -> linear RGB -> Film::add_sample loop
//                  (Tests/Backends/GPU/CUDA/CudaTransportParityTest.cpp:906-927), on the device.
// Arithmetic follows the reference scalar loop (Blackframe/Engine/Source/SceneMisPathLoop.cpp)
// operation for operation; every translation unit that includes this file is compiled with
// -fmad=false. bf200_kernels.cu (BF200_KERNELS_MAIN_TU) compiles the non-template kernels and the
// launchers; bf200_shade_*.cu each instantiate one shading launcher.
#pragma once

#include <cuda_runtime.h>

#include <climits>

#include "bf200_device.cuh"
#include "bf200_kernels.h"
#include "bf200_sphere.cuh"
#include "bf200_light_tree_device.cuh"

// Resident 256-thread blocks per SM the register allocation must allow, per stage kernel.
#ifndef BF200_INTERSECT_MIN_BLOCKS
#define BF200_INTERSECT_MIN_BLOCKS 2
#endif
#ifndef BF200_SHADE_MIN_BLOCKS
#define BF200_SHADE_MIN_BLOCKS 2
#endif
#ifndef BF200_OCCLUDE_MIN_BLOCKS
#define BF200_OCCLUDE_MIN_BLOCKS 2
#endif

namespace bf200 {

// ------------------------------------------------------------------------------------------------
// Scene setup
// ------------------------------------------------------------------------------------------------

__device__ __forceinline__ F3 xform_point(const float4* m, F3 p) {
    const float4 r0 = m[0], r1 = m[1], r2 = m[2];
    return {r0.x * p.x + r0.y * p.y + r0.z * p.z + r0.w, r1.x * p.x + r1.y * p.y + r1.z * p.z + r1.w,
            r2.x * p.x + r2.y * p.y + r2.z * p.z + r2.w};
}
__device__ __forceinline__ F3 xform_vector(const float4* m, F3 v) {
    const float4 r0 = m[0], r1 = m[1], r2 = m[2];
    return {r0.x * v.x + r0.y * v.y + r0.z * v.z, r1.x * v.x + r1.y * v.y + r1.z * v.z,
            r2.x * v.x + r2.y * v.y + r2.z * v.z};
}

__device__ __forceinline__ F3 load_vertex(const float* p, uint32_t i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }

#ifdef BF200_KERNELS_MAIN_TU
// World-space geometric normal of every instance triangle: the normal the analytic accel
// reports for a hit (AccelBackend.cpp:84-97, Triangle.hpp:374-481).
__global__ void k_world_normals(SceneView s, uint32_t total, float4* out, uint32_t* failures) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        // the instance whose triangle range [inst_normal_offset[inst], next offset) holds i: the
        // last instance starting at or before i (empty ranges start where the next one does)
        uint32_t lo = 0, hi = s.instance_count;
        while (hi - lo > 1U) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s.inst_normal_offset[mid] <= i) {
                lo = mid;
            } else {
                hi = mid;
            }
        }
        const uint32_t inst = lo;
        const uint32_t prim = i - s.inst_normal_offset[inst];
        const uint4 info = s.inst_info[inst];
        const uint4 geom = s.geom_info[info.x];
        const uint32_t* tri = s.triangles + 3ULL * (geom.y + prim);
        const float4* m = s.inst_to_world + 3ULL * inst;
        const F3 w0 = xform_point(m, load_vertex(s.positions, geom.x + tri[0]));
        const F3 w1 = xform_point(m, load_vertex(s.positions, geom.x + tri[1]));
        const F3 w2 = xform_point(m, load_vertex(s.positions, geom.x + tri[2]));
        F3 n{0.0F, 0.0F, 0.0F};
        if (!triangle_normal(w0, w1, w2, n)) {
            atomicAdd(failures, 1U);
        }
        out[i] = make_float4(n.x, n.y, n.z, 0.0F);
    }
}
#endif  // BF200_KERNELS_MAIN_TU

// ------------------------------------------------------------------------------------------------
// Ray / triangle test: exact edge signs, correctly rounded parameter and barycentrics
// ------------------------------------------------------------------------------------------------

constexpr double kU = 1.1102230246251565e-16;  // 2^-53

struct Dets {
    double p[3][3];
    double d[3];
};

// Exact evaluation of the four determinants as double expansions and an exact decision.
// Returns kTriHit with t (and barycentrics if requested), kTriMiss, or kTriFailure when a
// coordinate difference is not exact in double (exponent gap above 29 bits).
__device__ __forceinline__ int slow_triangle_decision(float4 v0, float4 v1, float4 v2, F3 o, F3 d, float t_min,
                                                      float t_max, float approx_t, bool want_bary, TriangleHit& hit) {
    Dets q;
    const double ox = o.x, oy = o.y, oz = o.z;
    q.p[0][0] = double(v0.x) - ox; q.p[0][1] = double(v0.y) - oy; q.p[0][2] = double(v0.z) - oz;
    q.p[1][0] = double(v1.x) - ox; q.p[1][1] = double(v1.y) - oy; q.p[1][2] = double(v1.z) - oz;
    q.p[2][0] = double(v2.x) - ox; q.p[2][1] = double(v2.y) - oy; q.p[2][2] = double(v2.z) - oz;
    q.d[0] = d.x; q.d[1] = d.y; q.d[2] = d.z;
    Expansion<double, 32> e0, e1, e2, vol;
    if (!exp_det3(e0, q.p[1], q.p[2], q.d) || !exp_det3(e1, q.p[2], q.p[0], q.d) ||
        !exp_det3(e2, q.p[0], q.p[1], q.d) || !exp_det3(vol, q.p[0], q.p[1], q.p[2])) {
        return kTriFailure;
    }
    Expansion<double, 96> det;
    det.size = 0;
    if (!exp_add_expansion(det, e0, 1.0) || !exp_add_expansion(det, e1, 1.0) || !exp_add_expansion(det, e2, 1.0)) {
        return kTriFailure;
    }
    const int ds = exp_sign(det);
    if (ds == 0) {
        return kTriMiss;  // coplanar or parallel: the accel skips both
    }
    const int s0 = exp_sign(e0), s1 = exp_sign(e1), s2 = exp_sign(e2);
    const bool nonneg = s0 >= 0 && s1 >= 0 && s2 >= 0;
    const bool nonpos = s0 <= 0 && s1 <= 0 && s2 <= 0;
    if (!nonneg && !nonpos) {
        return kTriMiss;
    }
    double dv = 0.0, vv = 0.0;
    for (int i = 0; i < det.size; ++i) dv += det.c[i];
    for (int i = 0; i < vol.size; ++i) vv += vol.c[i];
    float seed = isfinite(approx_t) && approx_t != 0.0F ? approx_t : static_cast<float>(vv / dv);
    float t = 0.0F;
    if (exp_sign(vol) == 0) {
        t = 0.0F;
    } else {
        if (seed == 0.0F || !isfinite(seed)) {
            return kTriFailure;
        }
        if (!exact_round_quotient(vol, det, seed, t)) {
            return kTriFailure;
        }
    }
    if (isnan(t) || t < t_min || t > t_max) {
        return kTriMiss;
    }
    hit.t = t;
    if (want_bary) {
        const Expansion<double, 32>* es[3] = {&e0, &e1, &e2};
        float out[3];
        for (int k = 0; k < 3; ++k) {
            if (exp_sign(*es[k]) == 0) {
                out[k] = 0.0F;
                continue;
            }
            double ev = 0.0;
            for (int i = 0; i < es[k]->size; ++i) ev += es[k]->c[i];
            if (!exact_round_quotient(*es[k], det, static_cast<float>(ev / dv), out[k])) {
                return kTriFailure;
            }
        }
        hit.b0 = out[0];
        hit.b1 = out[1];
        hit.b2 = out[2];
    }
    return kTriHit;
}

// The out-of-line copy of the exact test. It takes the vertices and the ray by value, rebuilds the
// differences itself and returns its result by value, so the fast path that calls it keeps
// everything in registers.
struct SlowResult {
    int code;
    TriangleHit hit;
};

static __device__ __noinline__ SlowResult exact_triangle_slow(float4 v0, float4 v1, float4 v2, F3 o, F3 d, float t_min,
                                                       float t_max, float approx_t, bool want_bary) {
    SlowResult r;
    r.code = slow_triangle_decision(v0, v1, v2, o, d, t_min, t_max, approx_t, want_bary, r.hit);
    return r;
}

__device__ __forceinline__ int slow_path(float4 v0, float4 v1, float4 v2, F3 o, F3 d, float t_min, float t_max,
                                         float approx_t, bool want_bary, TriangleHit& hit) {
    const SlowResult r = exact_triangle_slow(v0, v1, v2, o, d, t_min, t_max, approx_t, want_bary);
    if (r.code == kTriHit) {
        hit = r.hit;
    }
    return r.code;
}

// The float nearest to num/den when a forward error bound proves it; otherwise NaN.
__device__ __forceinline__ float certain_round(double num, double num_bound, double den, double den_bound) {
    if (!(fabs(num) > 2.0 * num_bound) || !(fabs(den) > 2.0 * den_bound)) {
        return __int_as_float(0x7fc00000);
    }
    const double q = num / den;
    const double rel = num_bound / fabs(num) + den_bound / fabs(den) + 4.0 * kU;
    if (!(rel < 0x1p-27)) {
        return __int_as_float(0x7fc00000);
    }
    const double lo = q - fabs(q) * (2.0 * rel);
    const double hi = q + fabs(q) * (2.0 * rel);
    const float flo = __double2float_rn(lo);
    const float fhi = __double2float_rn(hi);
    return flo == fhi ? flo : __int_as_float(0x7fc00000);
}

// Returns kTriHit (t set), kTriMiss or kTriFailure. Object-space floats in; the decision and
// the parameter equal those of the exact test in Triangle.hpp:683-822.
// d . (p x f) and a bound on its evaluation error: edge differences, products and the two
// subtractions / additions round at most seven times along any term, so the error is below
// 8u * sum |d_i| (|p_j f_k| + |p_k f_j|); 16u of that sum is returned as the bound.
__device__ __forceinline__ double edge_function(const double (&p)[3], double fx, double fy, double fz,
                                                const double (&dd)[3], double& bound) {
    const double cx = p[1] * fz - p[2] * fy, cy = p[2] * fx - p[0] * fz, cz = p[0] * fy - p[1] * fx;
    const double bx = fabs(p[1] * fz) + fabs(p[2] * fy), by = fabs(p[2] * fx) + fabs(p[0] * fz),
                 bz = fabs(p[0] * fy) + fabs(p[1] * fx);
    bound = 16.0 * kU * ((fabs(dd[0]) * bx + fabs(dd[1]) * by) + fabs(dd[2]) * bz);
    return (dd[0] * cx + dd[1] * cy) + dd[2] * cz;
}

__device__ __forceinline__ int triangle_test(float4 v0, float4 v1, float4 v2, F3 o, F3 d, float t_min, float t_max,
                                             bool want_bary, TriangleHit& hit) {
    const double ox = o.x, oy = o.y, oz = o.z;
    const double p0[3] = {double(v0.x) - ox, double(v0.y) - oy, double(v0.z) - oz};
    const double p1[3] = {double(v1.x) - ox, double(v1.y) - oy, double(v1.z) - oz};
    const double p2[3] = {double(v2.x) - ox, double(v2.y) - oy, double(v2.z) - oz};
    const double dd[3] = {d.x, d.y, d.z};
    // Edge functions e0 = det(p1, p2, d), e1 = det(p2, p0, d), e2 = det(p0, p1, d), evaluated as
    // e0 = d . (p1 x (v2 - v1)), e1 = d . (p2 x (v0 - v2)), e2 = d . (p0 x (v1 - v0)): the same
    // exact values (p_j = p_i + v_j - v_i), with terms of the size (distance x edge) instead of
    // distance squared, so their error bounds stay small for small distant triangles.
    double e[3], bound[3];
    e[0] = edge_function(p1, double(v2.x) - double(v1.x), double(v2.y) - double(v1.y),
                         double(v2.z) - double(v1.z), dd, bound[0]);
    e[1] = edge_function(p2, double(v0.x) - double(v2.x), double(v0.y) - double(v2.y),
                         double(v0.z) - double(v2.z), dd, bound[1]);
    e[2] = edge_function(p0, double(v1.x) - double(v0.x), double(v1.y) - double(v0.y),
                         double(v1.z) - double(v0.z), dd, bound[2]);
    int pos = 0, neg = 0;
    bool ambiguous = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (e[k] > bound[k]) {
            ++pos;
        } else if (e[k] < -bound[k]) {
            ++neg;
        } else {
            ambiguous = true;
        }
    }
    if (pos > 0 && neg > 0) {
        return kTriMiss;
    }
    // A coordinate difference that is not exact in double makes the slow path unusable; such
    // inputs (exponent gaps above 29 bits) are reported as a lane failure.
    const auto exact_diffs = [&]() {
        return (p0[0] + ox == double(v0.x)) && (p0[1] + oy == double(v0.y)) && (p0[2] + oz == double(v0.z)) &&
               (p1[0] + ox == double(v1.x)) && (p1[1] + oy == double(v1.y)) && (p1[2] + oz == double(v1.z)) &&
               (p2[0] + ox == double(v2.x)) && (p2[1] + oy == double(v2.y)) && (p2[2] + oz == double(v2.z));
    };
    if (ambiguous) {
        if (!exact_diffs()) {
            return kTriFailure;
        }
        return slow_path(v0, v1, v2, o, d, t_min, t_max, __int_as_float(0x7fc00000), want_bary, hit);
    }
    // vol = det(p0, p1, p2) and det = e0 + e1 + e2 have the exact values p0 . N and d . N with
    // N = (v1 - v0) x (v2 - v0) (the scalar triple product identities). Evaluated in that form
    // their rounding error scales with the triangle's own size instead of its distance from the ray
    // origin, so small distant triangles certify their parameter without the exact fallback; the
    // quotient certified is still the exact one, so t is unchanged. Error bound: each edge
    // difference and product rounds once (u), each cross component and three-term dot product
    // rounds twice and three times more, at most 8u of the magnitudes summed below; 16u is used.
    const double e1x = double(v1.x) - double(v0.x), e1y = double(v1.y) - double(v0.y),
                 e1z = double(v1.z) - double(v0.z);
    const double e2x = double(v2.x) - double(v0.x), e2y = double(v2.y) - double(v0.y),
                 e2z = double(v2.z) - double(v0.z);
    const double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    const double ax = fabs(e1y * e2z) + fabs(e1z * e2y), ay = fabs(e1z * e2x) + fabs(e1x * e2z),
                 az = fabs(e1x * e2y) + fabs(e1y * e2x);
    const double vol = (p0[0] * nx + p0[1] * ny) + p0[2] * nz;
    const double vol_bound = 16.0 * kU * ((fabs(p0[0]) * ax + fabs(p0[1]) * ay) + fabs(p0[2]) * az);
    const double det = (dd[0] * nx + dd[1] * ny) + dd[2] * nz;
    const double det_bound = 16.0 * kU * ((fabs(dd[0]) * ax + fabs(dd[1]) * ay) + fabs(dd[2]) * az);
    float t = certain_round(vol, vol_bound, det, det_bound);
    if (isnan(t)) {
        if (!exact_diffs()) {
            return kTriFailure;
        }
        return slow_path(v0, v1, v2, o, d, t_min, t_max, __double2float_rn(vol / det), want_bary, hit);
    }
    if (t < t_min || t > t_max) {
        return kTriMiss;
    }
    hit.t = t;
    if (want_bary) {
        const float b0 = certain_round(e[0], bound[0], det, det_bound);
        const float b1 = certain_round(e[1], bound[1], det, det_bound);
        const float b2 = certain_round(e[2], bound[2], det, det_bound);
        if (isnan(b0) || isnan(b1) || isnan(b2)) {
            if (!exact_diffs()) {
                return kTriFailure;
            }
            return slow_path(v0, v1, v2, o, d, t_min, t_max, t, true, hit);
        }
        hit.b0 = b0;
        hit.b1 = b1;
        hit.b2 = b2;
    }
    return kTriHit;
}

// ------------------------------------------------------------------------------------------------
// BVH traversal
// ------------------------------------------------------------------------------------------------

constexpr float kGamma3 = 3.0F * 5.96046448e-8F / (1.0F - 3.0F * 5.96046448e-8F);
constexpr float kSlackLo = 1.0F - 2.0F * kGamma3;
constexpr float kSlackHi = 1.0F + 2.0F * kGamma3;

struct RayInv {
    F3 o;
    F3 inv;
    bool px, py, pz;  // axis-parallel components
    bool parallel;    // any of them
};

__device__ __forceinline__ RayInv make_ray_inv(F3 o, F3 d) {
    RayInv r;
    r.o = o;
    r.px = d.x == 0.0F;
    r.py = d.y == 0.0F;
    r.pz = d.z == 0.0F;
    r.inv = F3{r.px ? 0.0F : 1.0F / d.x, r.py ? 0.0F : 1.0F / d.y, r.pz ? 0.0F : 1.0F / d.z};
    r.parallel = r.px || r.py || r.pz;
    return r;
}

// Conservative slab test: never rejects a box that contains a point of the ray with parameter
// in [t_min, t_max] (each computed slab parameter is within a relative gamma(3) of the exact one,
// and its sign is exact). A ray with no axis-parallel component takes the first branch, where the
// slack factors scale the largest entry and smallest exit parameter once: rounding a product with
// a positive factor is monotonic, so that equals scaling each axis's parameter first.
__device__ __forceinline__ bool slab(const RayInv& r, float lox, float hix, float loy, float hiy, float loz, float hiz,
                                     float t_min, float t_max, float& near_out) {
    if (!r.parallel) {
        const float ax = (lox - r.o.x) * r.inv.x, bx = (hix - r.o.x) * r.inv.x;
        const float ay = (loy - r.o.y) * r.inv.y, by = (hiy - r.o.y) * r.inv.y;
        const float az = (loz - r.o.z) * r.inv.z, bz = (hiz - r.o.z) * r.inv.z;
        const float entry = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz));
        const float exit = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz));
        const float near = fmaxf(t_min, entry * kSlackLo);
        near_out = near;
        return near <= fminf(t_max, exit * kSlackHi);
    }
    float near = t_min, far = t_max;
    bool inside = true;
    if (r.px) {
        inside = inside && lox <= r.o.x && r.o.x <= hix;
    } else {
        const float a = (lox - r.o.x) * r.inv.x, b = (hix - r.o.x) * r.inv.x;
        near = fmaxf(near, fminf(a, b) * kSlackLo);
        far = fminf(far, fmaxf(a, b) * kSlackHi);
    }
    if (r.py) {
        inside = inside && loy <= r.o.y && r.o.y <= hiy;
    } else {
        const float a = (loy - r.o.y) * r.inv.y, b = (hiy - r.o.y) * r.inv.y;
        near = fmaxf(near, fminf(a, b) * kSlackLo);
        far = fminf(far, fmaxf(a, b) * kSlackHi);
    }
    if (r.pz) {
        inside = inside && loz <= r.o.z && r.o.z <= hiz;
    } else {
        const float a = (loz - r.o.z) * r.inv.z, b = (hiz - r.o.z) * r.inv.z;
        near = fmaxf(near, fminf(a, b) * kSlackLo);
        far = fminf(far, fmaxf(a, b) * kSlackHi);
    }
    near_out = near;
    return inside && near <= far;
}

// The slack factors only widen positive parameters; a negative lower bound is harmless because
// t_min >= 0 clamps it, and a negative upper bound means the box is entirely behind the origin.

// Traversal stack of one thread. The first kSharedStackEntries entries live in shared memory in
// thread-interleaved columns (entry k of thread t at k * blockDim.x + t: every lane of a warp hits
// its own bank at any depth); deeper entries, which the shallow BVHs of small scenes never reach,
// go to a local array.
constexpr int kSharedStackEntries = 32;

struct TraversalStack {
    int* column;
    uint32_t stride;
    int deep[kTraversalStack - kSharedStackEntries];
    __device__ __forceinline__ void set(int sp, int v) {
        if (sp < kSharedStackEntries) {
            column[sp * stride] = v;
        } else {
            deep[sp - kSharedStackEntries] = v;
        }
    }
    __device__ __forceinline__ int get(int sp) const {
        return sp < kSharedStackEntries ? column[sp * stride] : deep[sp - kSharedStackEntries];
    }
};

__device__ __forceinline__ TraversalStack thread_stack(int* shared) {
    TraversalStack st;
    st.column = shared + threadIdx.x;
    st.stride = blockDim.x;
    return st;
}

struct ClosestResult {
    float t;
    uint32_t instance, primitive;
    uint32_t leaf;  // leaf triangle index of the winner
    bool failed;
};

__device__ __forceinline__ bool precedes(float t, uint32_t inst, uint32_t prim, const ClosestResult& best) {
    if (t != best.t) {
        return t < best.t;
    }
    if (inst != best.instance) {
        return inst < best.instance;
    }
    return prim < best.primitive;
}

// Children of a BVH4 node whose boxes the ray meets within [t_min, limit], ordered near to far
// (a five-comparator sorting network on fixed slots, so everything stays in registers); returns
// how many. Unused slots (k >= info.x) are never tested; missed and unused slots sort last with an
// infinite distance.
__device__ __forceinline__ void order_pair(float& na, int& ca, float& nb, int& cb) {
    if (nb < na) {
        const float tn = na;
        na = nb;
        nb = tn;
        const int tc = ca;
        ca = cb;
        cb = tc;
    }
}

__device__ __forceinline__ int hit_children(const RayInv& r, const BvhNode4& n, float t_min, float limit,
                                            int (&kids)[4]) {
    float near[4];
    int code[4];
    int count = 0;
    const float lox[4] = {n.lo_x.x, n.lo_x.y, n.lo_x.z, n.lo_x.w};
    const float hix[4] = {n.hi_x.x, n.hi_x.y, n.hi_x.z, n.hi_x.w};
    const float loy[4] = {n.lo_y.x, n.lo_y.y, n.lo_y.z, n.lo_y.w};
    const float hiy[4] = {n.hi_y.x, n.hi_y.y, n.hi_y.z, n.hi_y.w};
    const float loz[4] = {n.lo_z.x, n.lo_z.y, n.lo_z.z, n.lo_z.w};
    const float hiz[4] = {n.hi_z.x, n.hi_z.y, n.hi_z.z, n.hi_z.w};
    const int child[4] = {n.child.x, n.child.y, n.child.z, n.child.w};
    const int used = n.info.x;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float t = 0.0F;
        const bool hit = k < used && slab(r, lox[k], hix[k], loy[k], hiy[k], loz[k], hiz[k], t_min, limit, t);
        near[k] = hit ? t : kInf;
        code[k] = child[k];
        count += hit ? 1 : 0;
    }
    order_pair(near[0], code[0], near[1], code[1]);
    order_pair(near[2], code[2], near[3], code[3]);
    order_pair(near[0], code[0], near[2], code[2]);
    order_pair(near[1], code[1], near[3], code[3]);
    order_pair(near[1], code[1], near[2], code[2]);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        kids[k] = code[k];
    }
    return count;
}

// Stack entries of both traversals: a BLAS node index (>= 0), a BLAS leaf (the node's child code,
// in [-2^30, 0): ~child = first_leaf_triangle << 3 | (count - 1)), or an instance-level entry
// below -2^30, kInstanceEntry + code with code < 2^30: a TLAS node (code = kTlasFlag | node) or an
// instance range (code = first << 15 | count: the instances [first, first + count), index order).
constexpr int kInstanceEntry = INT_MIN;
constexpr int kLeafEntryMin = -(1 << 30);
constexpr int kInstanceBits = 15;
constexpr uint32_t kTlasFlag = 1U << 29;

__device__ __forceinline__ int instance_range(uint32_t first, uint32_t count) {
    return kInstanceEntry + static_cast<int>((first << kInstanceBits) | count);
}

__device__ __forceinline__ int tlas_entry(int node) {
    return kInstanceEntry + static_cast<int>(kTlasFlag | static_cast<uint32_t>(node));
}

// Starts a walk's stack. With few instances every visible instance whose world box the ray meets
// within [t_min, t_max] goes on as a one-instance range, the lowest index on top, with the warp in
// step; otherwise the TLAS root goes on and the instance boxes are met through it.
__device__ __forceinline__ void push_instances(const SceneView& s, const RayInv& world, float t_min, float t_max,
                                               uint32_t mask, TraversalStack& stack, int& sp) {
    if (s.tlas_root >= 0) {
        stack.set(sp++, tlas_entry(s.tlas_root));
        return;
    }
    for (int inst = static_cast<int>(s.instance_count) - 1; inst >= 0; --inst) {
        const float4 blo = s.inst_world_box[2 * inst], bhi = s.inst_world_box[2 * inst + 1];
        float near;
        if ((mask & __float_as_uint(blo.w)) == 0U ||
            !slab(world, blo.x, bhi.x, blo.y, bhi.y, blo.z, bhi.z, t_min, t_max, near)) {
            continue;
        }
        stack.set(sp++, instance_range(static_cast<uint32_t>(inst), 1U));
    }
}

// Pushes the children a node visit returned, the farthest first so that the nearest comes next.
// Children of a TLAS node go on as TLAS entries (nodes) and one-instance ranges (instance leaves).
__device__ __forceinline__ void push_children(const int (&kids)[4], int count, bool tlas, TraversalStack& stack,
                                              int& sp, bool& failed) {
#pragma unroll
    for (int k = 3; k >= 0; --k) {
        if (k < count) {
            if (sp < kTraversalStack) {
                const int kid = kids[k];
                stack.set(sp++, !tlas ? kid
                                      : kid >= 0 ? tlas_entry(kid) : instance_range(static_cast<uint32_t>(~kid), 1U));
            } else {
                failed = true;
            }
        }
    }
}

// An instance range (code = first << 15 | count) yields its first instance: false when the ray's
// visibility mask excludes it or its world box is not met within [t_min, limit]; otherwise the ray
// moves into its object space, its BLAS root goes on above the rest of the range, and the call
// returns true.
__device__ __forceinline__ bool enter_instance(const SceneView& s, uint32_t code, const RayInv& world, F3 o, F3 d,
                                               float t_min, float limit, uint32_t mask, TraversalStack& stack,
                                               int& sp, bool& failed, uint32_t& inst_out, F3& ro, F3& rd,
                                               RayInv& r) {
    const uint32_t inst = code >> kInstanceBits, count = code & ((1U << kInstanceBits) - 1U);
    if (count > 1U) {
        stack.set(sp++, instance_range(inst + 1U, count - 1U));
    }
    const float4 blo = s.inst_world_box[2ULL * inst], bhi = s.inst_world_box[2ULL * inst + 1];
    float near;
    if ((mask & __float_as_uint(blo.w)) == 0U ||
        !slab(world, blo.x, bhi.x, blo.y, bhi.y, blo.z, bhi.z, t_min, limit, near)) {
        return false;
    }
    if (sp >= kTraversalStack) {
        failed = true;
        return false;
    }
    inst_out = inst;
    const float4* m = s.inst_to_object + 3ULL * inst;
    ro = xform_point(m, o);
    rd = xform_vector(m, d);
    r = make_ray_inv(ro, rd);
    stack.set(sp++, static_cast<int>(s.geom_info[s.inst_info[inst].x].z));
    return true;
}

// A sphere leaf's outcome codes are the triangle test's, so the walks treat both alike.
static_assert(int(kSphereMiss) == int(kTriMiss) && int(kSphereHit) == int(kTriHit) &&
                  int(kSphereFailure) == int(kTriFailure),
              "outcome codes");

// Per-lane walk state shared by the two traversals.
struct Walk {
    RayInv r;       // current ray (object space of the current instance)
    F3 ro, rd;
    uint32_t inst;  // current instance
    int sp;
    bool failed;
};

// Advances the walk until this lane holds a leaf (returned, in [-2^30, 0)) or its stack is empty
// (returns 0). TLAS and BLAS nodes share one visit (with the world or the object-space ray), so
// lanes at either level run it together; instance ranges are entered by enter_instance. Children
// are pushed far first, so the nearer one comes next.
__device__ __forceinline__ int next_leaf(const SceneView& s, const RayInv& world, F3 o, F3 d, float t_min,
                                         float limit, uint32_t mask, TraversalStack& stack, Walk& w) {
    while (w.sp > 0) {
        const int entry = stack.get(--w.sp);
        const uint32_t code = static_cast<uint32_t>(entry) ^ 0x80000000U;
        const bool instance_level = entry < kLeafEntryMin;
        if (instance_level && (code & kTlasFlag) == 0U) {
            enter_instance(s, code, world, o, d, t_min, limit, mask, stack, w.sp, w.failed, w.inst, w.ro, w.rd, w.r);
            continue;
        }
        if (!instance_level && entry < 0) {
            return entry;
        }
        const int node = instance_level ? static_cast<int>(code & (kTlasFlag - 1U)) : entry;
        int kids[4];
        const int count = hit_children(instance_level ? world : w.r, s.nodes[node], t_min, limit, kids);
        push_children(kids, count, instance_level, stack, w.sp, w.failed);
    }
    return 0;
}

// Closest-hit walk of one ray, in steps. closest_begin pushes the instance entries; each
// closest_step advances the lane through nodes and instance entries to its next leaf ("while-
// while": the warp reconverges before the leaf) and runs the exact triangle tests of that leaf;
// it returns false once the ray's stack is empty. Ties keep the hit that comes first in
// (instance, primitive) order, as the analytic accel's in-order scan does; boxes are culled only
// when they start strictly beyond the current closest t, so neither the order nor the culling
// changes the winner.
struct ClosestWalk {
    F3 o, d;
    float t_min, t_max;
    uint32_t mask;
    RayInv world;
    Walk w;
    ClosestResult best;
    bool found;
};

__device__ __forceinline__ void closest_begin(const SceneView& s, F3 o, F3 d, float t_min, float t_max,
                                              uint32_t mask, TraversalStack& stack, ClosestWalk& c) {
    c.o = o;
    c.d = d;
    c.t_min = t_min;
    c.t_max = t_max;
    c.mask = mask;
    c.world = make_ray_inv(o, d);
    c.w = Walk{c.world, o, d, 0xFFFFFFFFU, 0, false};
    c.best.t = t_max;
    c.best.instance = 0xFFFFFFFFU;
    c.best.primitive = 0xFFFFFFFFU;
    c.best.leaf = 0xFFFFFFFFU;
    c.best.failed = false;
    c.found = false;
    push_instances(s, c.world, t_min, t_max, mask, stack, c.w.sp);
}

// SPH: the scene has analytic spheres (the walks of triangle-only scenes carry no sphere code).
template <bool SPH>
__device__ __forceinline__ bool closest_step(const SceneView& s, TraversalStack& stack, ClosestWalk& c) {
    const int leaf_code =
        next_leaf(s, c.world, c.o, c.d, c.t_min, c.found ? c.best.t : c.t_max, c.mask, stack, c.w);
    if (leaf_code == 0) {
        return false;
    }
    const uint32_t packed = static_cast<uint32_t>(~leaf_code);
    const uint32_t first = packed >> kLeafCountBits;
    const uint32_t n = (packed & (kMaxLeafSize - 1)) + 1U;
    if (SPH && n == kSphereLeafCount) {  // an analytic sphere: one record, tested apart from the triangle loop
        const float4 v0 = s.leaf_tris[3ULL * first];
        const SphereHit h = sphere_intersect(v0, s.leaf_tris[3ULL * first + 1].x, c.w.ro, c.w.rd, c.t_min,
                                             c.found ? c.best.t : c.t_max);
        const uint32_t prim = __float_as_uint(v0.w);
        if (h.outcome == kSphereFailure) {
            c.w.failed = true;
        } else if (h.outcome == kSphereHit && (!c.found || precedes(h.t, c.w.inst, prim, c.best))) {
            c.best.t = h.t;
            c.best.instance = c.w.inst;
            c.best.primitive = prim;
            c.best.leaf = first;
            c.found = true;
        }
        return true;
    }
    for (uint32_t j = 0; j < n; ++j) {
        const uint32_t leaf = first + j;
        const float4 v0 = s.leaf_tris[3ULL * leaf];
        const float4 v1 = s.leaf_tris[3ULL * leaf + 1];
        const float4 v2 = s.leaf_tris[3ULL * leaf + 2];
        TriangleHit th;
        const int res =
            triangle_test(v0, v1, v2, c.w.ro, c.w.rd, c.t_min, c.found ? c.best.t : c.t_max, false, th);
        if (res == kTriFailure) {
            c.w.failed = true;
            continue;
        }
        if (res != kTriHit) {
            continue;
        }
        const uint32_t prim = __float_as_uint(v0.w);
        if (!c.found || precedes(th.t, c.w.inst, prim, c.best)) {
            c.best.t = th.t;
            c.best.instance = c.w.inst;
            c.best.primitive = prim;
            c.best.leaf = leaf;
            c.found = true;
        }
    }
    return true;
}

__device__ __forceinline__ ClosestResult closest_end(ClosestWalk& c) {
    c.best.failed = c.w.failed;
    if (!c.found) {
        c.best.instance = 0xFFFFFFFFU;
    }
    return c.best;
}

// Closest hit of one ray (the standalone query kernel); k_trace runs the same steps with dynamic
// ray fetch.
template <bool SPH>
__device__ ClosestResult closest_hit(const SceneView& s, F3 o, F3 d, float t_min, float t_max, uint32_t mask,
                                     TraversalStack& stack) {
    ClosestWalk c;
    closest_begin(s, o, d, t_min, t_max, mask, stack, c);
    while (closest_step<SPH>(s, stack, c)) {
    }
    return closest_end(c);
}

// Any hit in [t_min, t_max] (AccelBackend.cpp:114-147). One loop serves both levels, with one
// visit for TLAS and BLAS nodes as in next_leaf; leaves go through the stack like nodes (the
// nearest child on top), so every pass of the loop handles one entry per lane -- a node, an
// instance range or one leaf -- and a lane stops at its first hit.
// The set of leaves met does not depend on the order (the interval never shrinks), so neither does
// the answer. Returns 1 occluded, 0 clear, -1 failure.
template <bool SPH>
__device__ int any_hit(const SceneView& s, F3 o, F3 d, float t_min, float t_max, uint32_t mask,
                       TraversalStack& stack) {
    bool failed = false;
    const RayInv world = make_ray_inv(o, d);
    int sp = 0;
    push_instances(s, world, t_min, t_max, mask, stack, sp);
    RayInv r = world;
    F3 ro = o, rd = d;
    while (sp > 0) {
        const int entry = stack.get(--sp);
        const uint32_t code = static_cast<uint32_t>(entry) ^ 0x80000000U;
        const bool instance_level = entry < kLeafEntryMin;
        if (instance_level && (code & kTlasFlag) == 0U) {
            uint32_t inst = 0U;
            enter_instance(s, code, world, o, d, t_min, t_max, mask, stack, sp, failed, inst, ro, rd, r);
            continue;
        }
        if (!instance_level && entry < 0) {
            const uint32_t packed = static_cast<uint32_t>(~entry);
            const uint32_t first = packed >> kLeafCountBits;
            const uint32_t n = (packed & (kMaxLeafSize - 1)) + 1U;
            if (SPH && n == kSphereLeafCount) {
                const int res = sphere_intersect(s.leaf_tris[3ULL * first], s.leaf_tris[3ULL * first + 1].x, ro, rd,
                                                 t_min, t_max)
                                    .outcome;
                if (res == kSphereHit) {
                    return 1;
                }
                failed = failed || res == kSphereFailure;
                continue;
            }
            for (uint32_t j = 0; j < n; ++j) {
                const uint32_t leaf = first + j;
                TriangleHit th;
                const int res = triangle_test(s.leaf_tris[3ULL * leaf], s.leaf_tris[3ULL * leaf + 1],
                                              s.leaf_tris[3ULL * leaf + 2], ro, rd, t_min, t_max, false, th);
                if (res == kTriHit) {
                    return 1;
                }
                if (res == kTriFailure) {
                    failed = true;
                }
            }
            continue;
        }
        const int node = instance_level ? static_cast<int>(code & (kTlasFlag - 1U)) : entry;
        int kids[4];
        const int count = hit_children(instance_level ? world : r, s.nodes[node], t_min, t_max, kids);
        push_children(kids, count, instance_level, stack, sp, failed);
    }
    return failed ? -1 : 0;
}

// Barycentrics of the winning triangle (correctly rounded e_i / det); for a sphere, its outward
// object-space normal at the hit.
template <bool SPH>
__device__ bool hit_barycentrics(const SceneView& s, const ClosestResult& c, F3 o, F3 d, float t_min, float t_max,
                                 TriangleHit& th) {
    const float4* m = s.inst_to_object + 3ULL * c.instance;
    const F3 lo = xform_point(m, o);
    const F3 ld = xform_vector(m, d);
    const float4 v1 = s.leaf_tris[3ULL * c.leaf + 1];
    if (SPH && __float_as_uint(v1.w) == kSphereLeaf) {
        const SphereHit h = sphere_intersect(s.leaf_tris[3ULL * c.leaf], v1.x, lo, ld, t_min, t_max);
        th.t = h.t;
        th.b0 = h.normal.x;
        th.b1 = h.normal.y;
        th.b2 = h.normal.z;
        return h.outcome == kSphereHit && h.t == c.t;
    }
    const int res = triangle_test(s.leaf_tris[3ULL * c.leaf], s.leaf_tris[3ULL * c.leaf + 1],
                                  s.leaf_tris[3ULL * c.leaf + 2], lo, ld, t_min, t_max, true, th);
    return res == kTriHit && th.t == c.t;
}

// ------------------------------------------------------------------------------------------------
// Wavefront helpers
// ------------------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t depth_total(uint32_t packed) {
    return (packed & 0xFFU) + ((packed >> 8) & 0xFFU) + ((packed >> 16) & 0xFFU);
}

__device__ __forceinline__ uint32_t depth_blocked(const TransportParams& p, uint32_t packed, uint32_t lobes) {
    uint32_t blocked = 0;
    if ((lobes & kLobeDiffuse) && (packed & 0xFFU) >= p.limits[0]) blocked |= kLobeDiffuse;
    if ((lobes & kLobeGlossy) && ((packed >> 8) & 0xFFU) >= p.limits[1]) blocked |= kLobeGlossy;
    if ((lobes & kLobeSpecular) && ((packed >> 16) & 0xFFU) >= p.limits[2]) blocked |= kLobeSpecular;
    if ((lobes & kLobeTransmission) && ((packed >> 24) & 0xFFU) >= p.limits[3]) blocked |= kLobeTransmission;
    if ((lobes & kLobeVolume) && 0U >= p.limits[4]) blocked |= kLobeVolume;
    return blocked;
}

__device__ __forceinline__ uint32_t depth_advance(uint32_t packed, uint32_t lobes) {
    if (lobes & kLobeDiffuse) packed += 1U;
    if (lobes & kLobeGlossy) packed += 1U << 8;
    if (lobes & kLobeSpecular) packed += 1U << 16;
    if (lobes & kLobeTransmission) packed += 1U << 24;
    return packed;
}

__device__ __forceinline__ Stream load_stream(const Wavefront& w, const PathSource& src, uint32_t slot) {
    const uint2 v = w.stream[slot];
    Stream r;
    r.state = (static_cast<uint64_t>(v.y) << 32) | v.x;
    r.sobol = src.sobol;
    r.sample = r.seed = r.pixel_hash = 0U;
    if (src.sobol != nullptr) {
        const uint4 q = w.sobol_index[slot];
        const uint2 h = w.pixel_hash[slot];
        r.sample = (static_cast<uint64_t>(q.y) << 32) | q.x;
        r.seed = (static_cast<uint64_t>(q.w) << 32) | q.z;
        r.pixel_hash = (static_cast<uint64_t>(h.y) << 32) | h.x;
    }
    return r;
}

__device__ __forceinline__ void record_failure(const Wavefront& w, uint32_t slot, uint32_t code) {
    atomicAdd(&w.counters[5], 1ULL);
    atomicMin(&w.counters[6], static_cast<unsigned long long>(w.path_id[slot]));
    atomicCAS(&w.counters[7], 0ULL, static_cast<unsigned long long>(code));
}

// PinholeCamera.hpp:194-283: jittered primary ray of (pixel, sample).
static __device__ bool camera_ray(const PathSource& src, uint32_t px, uint32_t py, const Stream& stream, F3& o, F3& d,
                           Lane& lane) {
    float ox = 0.5F, oy = 0.5F;
    if (src.jitter != 0U) {
        ox = stream.sample_1d(kCameraRasterX);
        oy = stream.sample_1d(kCameraRasterY);
    }
    const float rw = static_cast<float>(src.width), rh = static_cast<float>(src.height);
    const float tpx = 2.0F * static_cast<float>(px);
    const float tpy = 2.0F * static_cast<float>(py);
    const float nx = (tpx + 2.0F * ox) / rw - 1.0F;
    const float ny = 1.0F - (tpy + 2.0F * oy) / rh;
    const F3 cd{nx * src.half_width, ny * src.half_height, -1.0F};
    const F3 uc = robust_unit(cd, lane);
    const F3 t{src.cam_t[0], src.cam_t[1], src.cam_t[2]};
    const F3 b{src.cam_b[0], src.cam_b[1], src.cam_b[2]};
    const F3 n{src.cam_n[0], src.cam_n[1], src.cam_n[2]};
    const F3 world{t.x * uc.x + b.x * uc.y + n.x * uc.z, t.y * uc.x + b.y * uc.y + n.y * uc.z,
                   t.z * uc.x + b.z * uc.y + n.z * uc.z};
    d = robust_unit(world, lane);
    o = F3{src.cam_origin[0], src.cam_origin[1], src.cam_origin[2]};
    return lane.err == 0;
}

// Claims the next path of the job into `slot` and writes its primary ray and initial state.
// Returns false when the job has no more paths.
static __device__ bool start_path(const Wavefront& w, const PathSource& src, uint32_t slot, uint64_t id) {
    Lane lane;
    F3 o, d;
    float tmin, tmax;
    Stream stream;
    uint32_t mask;
    if (src.mode == 0U) {
        const uint64_t pixels = static_cast<uint64_t>(src.width) * src.height;
        const uint64_t pixel = id % pixels;
        const uint64_t sample = src.first_sample + id / pixels;
        const uint32_t px = static_cast<uint32_t>(pixel % src.width);
        const uint32_t py = static_cast<uint32_t>(pixel / src.width);
        stream = Stream::make(px, py, sample, src.seed, src.sobol);
        // the jitter uses the independent stream of the same index (PixelJitter.hpp:47-64)
        camera_ray(src, px, py, stream, o, d, lane);
        tmin = src.t_min;
        tmax = src.t_max;
        mask = src.mask;
    } else {
        const bf200_path_input_v1& in = src.inputs[id];
        stream = Stream::make(in.sample.pixel_x, in.sample.pixel_y, in.sample.sample_index, in.sample.seed,
                              src.sobol);
        o = F3{in.primary_ray.origin[0], in.primary_ray.origin[1], in.primary_ray.origin[2]};
        d = F3{in.primary_ray.direction[0], in.primary_ray.direction[1], in.primary_ray.direction[2]};
        tmin = in.primary_ray.t_min;
        tmax = in.primary_ray.t_max;
        mask = in.primary_ray.mask;
        if (src.cones_in != nullptr) {
            // the camera stage's valid_ray_cone check (CudaWavefrontStages.cu:1378-1380)
            const float2 cone = src.cones_in[id];
            w.cone[slot] = cone;
            if (!cone_valid(cone)) {
                lane.fail();
            }
        }
    }
    float4 beta = make_float4(1.0F, 1.0F, 1.0F, 1.0F);
    float4 radiance = make_float4(0.0F, 0.0F, 0.0F, 0.0F);
    float eta = 1.0F;
    if (src.mode == 1U && src.states_in != nullptr) {
        // a depth-zero initial state; the camera stage's valid_path_state check
        // (CudaWavefrontStages.cu:545-560, 1378-1380)
        const bf200_path_state_v1& st = src.states_in[id];
        beta = make_float4(st.beta[0], st.beta[1], st.beta[2], st.beta[3]);
        radiance = make_float4(st.radiance[0], st.radiance[1], st.radiance[2], st.radiance[3]);
        eta = st.eta_scale;
        bool valid = isfinite(eta) && eta > 0.0F;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            valid = valid && isfinite(st.beta[l]) && st.beta[l] >= 0.0F && isfinite(st.radiance[l]) &&
                    st.radiance[l] >= 0.0F;
        }
        if (!valid) {
            lane.fail();
        }
    }
    w.path_id[slot] = id;
    w.ray_o[slot] = make_float4(o.x, o.y, o.z, tmax);
    w.ray_d[slot] = make_float4(d.x, d.y, d.z, tmin);
    w.beta[slot] = beta;
    w.radiance[slot] = radiance;
    w.depth[slot] = 0U;
    w.eta[slot] = eta;
    w.prev[slot] = make_float4(0.0F, 0.0F, 0.0F, 0.0F);
    w.flags[slot] = 0U;
    w.status[slot] = lane.err;
    w.stream[slot] = make_uint2(static_cast<uint32_t>(stream.state), static_cast<uint32_t>(stream.state >> 32));
    if (src.sobol != nullptr) {
        w.sobol_index[slot] = make_uint4(static_cast<uint32_t>(stream.sample), static_cast<uint32_t>(stream.sample >> 32),
                                         static_cast<uint32_t>(stream.seed), static_cast<uint32_t>(stream.seed >> 32));
        w.pixel_hash[slot] = make_uint2(static_cast<uint32_t>(stream.pixel_hash),
                                        static_cast<uint32_t>(stream.pixel_hash >> 32));
    }
    w.mask[slot] = mask;
    w.state[slot] = kSlotActive;
    return true;
}

// Writes a finished path's outputs (film radiance or the full result record).
static __device__ void finish_path(const Wavefront& w, const PathSource& src, uint32_t slot) {
    const uint64_t id = w.path_id[slot];
    const uint32_t status = w.status[slot];
    if ((status & 0xFFU) != 0U) {
        record_failure(w, slot, status & 0xFFU);
    }
    if (src.mode == 0U) {
        src.path_radiance[id] = (status & 0xFFU) != 0U ? make_float4(__int_as_float(0x7fc00000), 0.0F, 0.0F, 0.0F)
                                                        : w.radiance[slot];
        return;
    }
    bf200_path_result_v1 r;
    const float4 beta = w.beta[slot], rad = w.radiance[slot];
    r.beta[0] = beta.x; r.beta[1] = beta.y; r.beta[2] = beta.z; r.beta[3] = beta.w;
    r.radiance[0] = rad.x; r.radiance[1] = rad.y; r.radiance[2] = rad.z; r.radiance[3] = rad.w;
    const uint32_t dp = w.depth[slot];
    r.depth = depth_total(dp);
    r.depth_counters[0] = dp & 0xFFU;
    r.depth_counters[1] = (dp >> 8) & 0xFFU;
    r.depth_counters[2] = (dp >> 16) & 0xFFU;
    r.depth_counters[3] = (dp >> 24) & 0xFFU;
    r.depth_counters[4] = 0U;
    r.eta_scale = w.eta[slot];
    const uint32_t flags = w.flags[slot];
    r.delta_flags = flags & 0xFFU;
    r.termination = (flags >> 8) & 0xFFU;
    r.blocked_depth_limits = (flags >> 16) & 0xFFU;
    r.lane_status = status & 0xFFU;
    r.segments = status >> 8;
    const float4 o = w.ray_o[slot], dd = w.ray_d[slot];
    r.terminal_ray.origin[0] = o.x; r.terminal_ray.origin[1] = o.y; r.terminal_ray.origin[2] = o.z;
    r.terminal_ray.direction[0] = dd.x; r.terminal_ray.direction[1] = dd.y; r.terminal_ray.direction[2] = dd.z;
    r.terminal_ray.t_min = dd.w;
    r.terminal_ray.t_max = o.w;
    r.terminal_ray.time = src.mode == 1U ? src.inputs[id].primary_ray.time : src.time;
    r.terminal_ray.mask = src.mode == 1U ? src.inputs[id].primary_ray.mask : src.mask;
    r.terminal_ray.medium = 0U;
    r.terminal_ray.reserved = 0U;
    src.results[id] = r;
    if (src.cones_out != nullptr) {
        src.cones_out[id] = w.cone[slot];  // defined at the terminal ray's origin
    }
}

#ifdef BF200_KERNELS_MAIN_TU
// ------------------------------------------------------------------------------------------------
// k_camera_rays: primary rays of given (pixel, sample) records, as start_path generates them
// ------------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(128) k_camera_rays(PathSource src, const bf200_sample_index_v1* samples, uint64_t n,
                                                     bf200_ray_v1* rays, uint32_t* status) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const bf200_sample_index_v1 si = samples[i];
        const Stream stream = Stream::make(si.pixel_x, si.pixel_y, si.sample_index, si.seed, src.sobol);
        Lane lane;
        F3 o{}, d{};
        camera_ray(src, si.pixel_x, si.pixel_y, stream, o, d, lane);
        bf200_ray_v1 r{};
        r.origin[0] = o.x;
        r.origin[1] = o.y;
        r.origin[2] = o.z;
        r.direction[0] = d.x;
        r.direction[1] = d.y;
        r.direction[2] = d.z;
        r.t_min = src.t_min;
        r.t_max = src.t_max;
        r.time = src.time;
        r.mask = src.mask;
        rays[i] = r;
        status[i] = lane.err;
    }
}

cudaError_t launch_camera_rays(const PathSource& src, const bf200_sample_index_v1* samples, uint64_t n,
                               bf200_ray_v1* rays, uint32_t* status, cudaStream_t stream) {
    const uint64_t blocks = (n + 127U) / 128U;
    k_camera_rays<<<static_cast<uint32_t>(blocks == 0 ? 1 : (blocks < 65535U ? blocks : 65535U)), 128, 0, stream>>>(
        src, samples, n, rays, status);
    return cudaGetLastError();
}
#endif  // BF200_KERNELS_MAIN_TU

#ifdef BF200_KERNELS_MAIN_TU
// ------------------------------------------------------------------------------------------------
// k_regenerate: retire finished slots and start new paths in empty ones (camera rays or inputs)
// ------------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_regenerate(Wavefront w, PathSource src) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        w.counters[8] = 0ULL;  // k_trace's fetch cursor for this iteration
    }
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t first = blockIdx.x * blockDim.x + threadIdx.x;
    // every thread of a warp runs the same number of iterations so the warp-wide claim below is
    // entered by whole warps
    const uint32_t rounds = (w.capacity + stride - 1U) / stride;
    for (uint32_t round = 0; round < rounds; ++round) {
        const uint32_t slot = first + round * stride;
        const bool in_range = slot < w.capacity;
        uint8_t state = in_range ? w.state[slot] : kSlotActive + 16;
        if (state == kSlotDone) {
            finish_path(w, src, slot);
            state = kSlotEmpty;
            w.state[slot] = kSlotEmpty;
        }
        // claim new paths for empty slots: one atomic per warp (ballot / popc)
        const bool wants = in_range && state == kSlotEmpty;
        const unsigned want_mask = __ballot_sync(0xFFFFFFFFU, wants);
        unsigned long long base = 0;
        if (want_mask != 0U) {
            const int leader = __ffs(want_mask) - 1;
            if (static_cast<int>(threadIdx.x & 31U) == leader) {
                base = atomicAdd(&w.counters[1], static_cast<unsigned long long>(__popc(want_mask)));
            }
            base = __shfl_sync(0xFFFFFFFFU, base, leader);
        }
        if (wants) {
            const unsigned rank = __popc(want_mask & ((1U << (threadIdx.x & 31U)) - 1U));
            const uint64_t id = base + rank;
            if (id < src.total) {
                start_path(w, src, slot, id);
                if ((w.status[slot] & 0xFFU) != 0U) {
                    w.state[slot] = kSlotDone;
                }
            }
        }
    }
}
#endif  // BF200_KERNELS_MAIN_TU

// ------------------------------------------------------------------------------------------------
// k_trace: closest hit of every active slot's ray; writes the hit and the slot's shading route
// ------------------------------------------------------------------------------------------------

// Finishes one slot's trace: writes the hit (t and the barycentrics of the winning triangle) or
// the miss or failure, and the slot's shading route.
template <bool SPH>
__device__ __forceinline__ void trace_finish(const SceneView& s, const Wavefront& w, uint32_t slot,
                                             const ClosestResult& c, F3 o, F3 d, float t_min, float t_max) {
    if (c.failed) {
        w.status[slot] = (w.status[slot] & ~0xFFU) | kLaneTraversal;
        w.state[slot] = kSlotDone;
        w.route[slot] = kRouteNone;
        return;
    }
    if (c.instance == 0xFFFFFFFFU) {
        w.hit_id[slot] = make_uint2(0xFFFFFFFFU, 0U);
        w.route[slot] = static_cast<uint8_t>(kRouteGeneric);
        return;
    }
    TriangleHit th;
    if (!hit_barycentrics<SPH>(s, c, o, d, t_min, t_max, th)) {
        w.status[slot] = (w.status[slot] & ~0xFFU) | kLaneNumerical;
        w.state[slot] = kSlotDone;
        w.route[slot] = kRouteNone;
        return;
    }
    w.hit_tb[slot] = make_float4(c.t, th.b0, th.b1, th.b2);
    // the winner's leaf record (its vertices, and the primitive index in the first record's w):
    // shading reads the triangle from there, where this trace has just read it
    w.hit_id[slot] = make_uint2(c.instance, c.leaf);
    w.route[slot] = s.inst_route[c.instance];
}

// Persistent traversal with dynamic ray fetch: every lane keeps one ray in flight and, when its ray
// is finished, takes the next slot from a cursor over [0, capacity) (one atomic per warp for all
// of the warp's idle lanes), so a warp's lanes stay busy instead of waiting for its slowest ray.
// Slots that are not active are marked unrouted as they are fetched.
template <bool SPH>
__global__ void __launch_bounds__(256, BF200_INTERSECT_MIN_BLOCKS) k_trace(SceneView s, Wavefront w) {
    __shared__ int stack_columns[kSharedStackEntries * 256];
    TraversalStack stack = thread_stack(stack_columns);
    const uint32_t lane = threadIdx.x & 31U;
    const uint32_t below = (1U << lane) - 1U;
    uint32_t slot = 0xFFFFFFFFU;
    bool drained = false;
    ClosestWalk c;
    while (true) {
        const bool idle = slot == 0xFFFFFFFFU;
        const unsigned idle_mask = __ballot_sync(0xFFFFFFFFU, idle);
        if (idle_mask != 0U && !drained) {
            unsigned long long base = 0;
            if (lane == static_cast<uint32_t>(__ffs(idle_mask) - 1)) {
                base = atomicAdd(&w.counters[8], static_cast<unsigned long long>(__popc(idle_mask)));
            }
            base = __shfl_sync(0xFFFFFFFFU, base, __ffs(idle_mask) - 1);
            drained = base + __popc(idle_mask) >= w.capacity;
            if (idle) {
                const unsigned long long index = base + __popc(idle_mask & below);
                if (index < w.capacity) {
                    const uint32_t candidate = static_cast<uint32_t>(index);
                    if (w.state[candidate] == kSlotActive) {
                        slot = candidate;
                        const float4 o4 = w.ray_o[slot], d4 = w.ray_d[slot];
                        closest_begin(s, ld3(o4), ld3(d4), d4.w, o4.w, w.mask[slot], stack, c);
                        w.status[slot] += 1U << 8;  // one extension segment
                    } else {
                        w.route[candidate] = kRouteNone;
                    }
                }
            }
        }
        const bool busy = slot != 0xFFFFFFFFU;
        const unsigned busy_mask = __ballot_sync(0xFFFFFFFFU, busy);
        if (busy_mask == 0U) {
            if (drained) {
                break;
            }
            continue;
        }
        if (lane == static_cast<uint32_t>(__ffs(busy_mask) - 1) && idle_mask != 0U) {
            // extension segments started in this pass (lanes that took an active slot)
            const unsigned started = busy_mask & idle_mask;
            if (started != 0U) {
                atomicAdd(&w.counters[3], static_cast<unsigned long long>(__popc(started)));
            }
        }
        if (busy && !closest_step<SPH>(s, stack, c)) {
            trace_finish<SPH>(s, w, slot, closest_end(c), c.o, c.d, c.t_min, c.t_max);
            slot = 0xFFFFFFFFU;
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Surface reconstruction (SceneSurfaceInteraction.cpp:54-350, 804-937)
// ------------------------------------------------------------------------------------------------

struct Surface {
    F3 position, error, ng, ns;
    Frame frame;
};

// transform_position_with_error (SurfaceInteraction :135-189): an object-space point with its
// per-axis error bound into world space; the bound also covers the point's distance from the
// ray's own hit position.
static __device__ bool transform_position_with_error(const SceneView& s, uint32_t inst, const float (&point)[3],
                                              const float (&perr)[3], F3 hit_position, Surface& out, Lane& lane) {
    const float4* mw = s.inst_to_world + 3ULL * inst;
    const F3 world = xform_point(mw, F3{point[0], point[1], point[2]});
    const float wv[3] = {world.x, world.y, world.z};
    const float hv[3] = {hit_position.x, hit_position.y, hit_position.z};
    const double eps = static_cast<double>(kEps);
    const double g7 = (7.0 * eps) / (1.0 - 7.0 * eps);
    float err[3];
#pragma unroll
    for (int row = 0; row < 3; ++row) {
        const float4 r = mw[row];
        const float rr[4] = {r.x, r.y, r.z, r.w};
        double magnitude = fabs(static_cast<double>(rr[3]));
        double propagated = 0.0;
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            const double coefficient = fabs(static_cast<double>(rr[col]));
            magnitude += coefficient * fabs(static_cast<double>(point[col]));
            propagated += coefficient * static_cast<double>(perr[col]);
        }
        const double discrepancy = fabs(static_cast<double>(wv[row]) - static_cast<double>(hv[row]));
        const double bound = g7 * magnitude + (1.0 + g7) * propagated + discrepancy;
        if (!isfinite(bound) || bound < 0.0 || bound > 3.4028234663852886e38) {
            lane.fail();
            return false;
        }
        err[row] = __double2float_rn(bound);
        if (static_cast<double>(err[row]) < bound) {
            err[row] = nextafterf(err[row], kInf);
        }
    }
    out.position = world;
    out.error = F3{err[0], err[1], err[2]};
    return true;
}

// robust_transformed_normal (:252-295): an object-space normal through the inverse transpose, in
// double, scaled by its largest component and normalised.
static __device__ bool transform_normal(const SceneView& s, uint32_t inst, F3 on, F3& ns, Lane& lane) {
    const float4* mi = s.inst_to_object + 3ULL * inst;
    const float4 i0 = mi[0], i1 = mi[1], i2 = mi[2];
    const double n[3] = {on.x, on.y, on.z};
    const double tr[3] = {fma(double(i0.x), n[0], fma(double(i1.x), n[1], double(i2.x) * n[2])),
                          fma(double(i0.y), n[0], fma(double(i1.y), n[1], double(i2.y) * n[2])),
                          fma(double(i0.z), n[0], fma(double(i1.z), n[1], double(i2.z) * n[2]))};
    double mc = fabs(tr[0]);
    mc = mc < fabs(tr[1]) ? fabs(tr[1]) : mc;
    mc = mc < fabs(tr[2]) ? fabs(tr[2]) : mc;
    if (!isfinite(mc) || mc == 0.0) {
        lane.fail();
        return false;
    }
    const double sc[3] = {tr[0] / mc, tr[1] / mc, tr[2] / mc};
    const double mag = sqrt(fma(sc[0], sc[0], fma(sc[1], sc[1], sc[2] * sc[2])));
    ns = F3{__double2float_rn(sc[0] / mag), __double2float_rn(sc[1] / mag), __double2float_rn(sc[2] / mag)};
    return true;
}

// Surface of an analytic sphere hit (a design of this backend: the reference has no scene-level
// spheres). The outward normal is robust_outward_normal of the object-space hit point minus the
// centre, as in Sphere.hpp. The shading point is moved onto the sphere along that normal
// (centre + r n), so the error of t does not enter the spawn offset; its bound is 7 ulps of
// |centre| + r per axis. The geometric normal is the world normal through the inverse transpose,
// and the shading normal equals it.
static __device__ bool resolve_sphere_surface(const SceneView& s, uint32_t inst, const uint4 geom, F3 hit_position,
                                       uint32_t material, Surface& out, Lane& lane) {
    const float4 c4 = s.leaf_tris[3ULL * geom.x];
    const float radius = s.leaf_tris[3ULL * geom.x + 1].x;
    const float centre[3] = {c4.x, c4.y, c4.z};
    const F3 local = xform_point(s.inst_to_object + 3ULL * inst, hit_position);
    F3 n;
    if (!sphere_outward_normal(local - F3{c4.x, c4.y, c4.z}, n)) {
        lane.fail();
        return false;
    }
    const float nv[3] = {n.x, n.y, n.z};
    const float gamma7 = (7.0F * kEps) / (1.0F - 7.0F * kEps);
    float point[3], perr[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        point[a] = centre[a] + nv[a] * radius;
        perr[a] = gamma7 * (fabsf(centre[a]) + radius);
    }
    if (!transform_position_with_error(s, inst, point, perr, hit_position, out, lane)) {
        return false;
    }
    F3 ng;
    if (!transform_normal(s, inst, n, ng, lane)) {
        return false;
    }
    out.ng = ng;
    out.ns = ng;
    const uint4 minfo = s.material_info[material];
    if (minfo.y != 0U) {
        lane.fail(kLaneUnsupported);
        return false;
    }
    out.frame = rotated_about_normal(frame_from_normal(ng, lane), __uint_as_float(minfo.z), lane);
    return lane.err == 0;
}

static __device__ bool resolve_surface(const SceneView& s, uint32_t inst, uint32_t leaf, const float4 tb, F3 hit_position,
                                uint32_t material, Surface& out, Lane& lane) {
    {
        const uint4 geom = s.geom_info[s.inst_info[inst].x];
        if (geom.w == kGeometrySphere) {
            return resolve_sphere_surface(s, inst, geom, hit_position, material, out, lane);
        }
    }
    const float b0 = tb.y, b1 = tb.z, b2 = tb.w;
    const float tolerance = 32.0F * kEps;
    if (!isfinite(b0) || b0 < -tolerance || b0 > 1.0F + tolerance || !isfinite(b1) || b1 < -tolerance ||
        b1 > 1.0F + tolerance || !isfinite(b2) || b2 < -tolerance || b2 > 1.0F + tolerance) {
        lane.fail();
        return false;
    }
    const float sum = b0 + b1 + b2;
    if (!isfinite(sum) || fabsf(sum - 1.0F) > tolerance) {
        lane.fail();
        return false;
    }
    const uint4 info = s.inst_info[inst];
    const uint4 geom = s.geom_info[info.x];
    // the hit triangle's object-space vertices from its leaf record (copies of the mesh positions)
    const float4 r0 = s.leaf_tris[3ULL * leaf], r1 = s.leaf_tris[3ULL * leaf + 1], r2 = s.leaf_tris[3ULL * leaf + 2];
    const uint32_t prim = __float_as_uint(r0.w);
    const uint32_t* tri = s.triangles + 3ULL * (geom.y + prim);
    const F3 p0{r0.x, r0.y, r0.z};
    const F3 p1{r1.x, r1.y, r1.z};
    const F3 p2{r2.x, r2.y, r2.z};
    const F3 n0 = load_vertex(s.normals, geom.x + tri[0]);
    const F3 n1 = load_vertex(s.normals, geom.x + tri[1]);
    const F3 n2 = load_vertex(s.normals, geom.x + tri[2]);
    // interpolate_position_with_error (:82-133)
    const float gamma7 = (7.0F * kEps) / (1.0F - 7.0F * kEps);
    const float c[3][3] = {{p0.x, p0.y, p0.z}, {p1.x, p1.y, p1.z}, {p2.x, p2.y, p2.z}};
    float scale = 0.0F;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        scale = bf_max(scale, fabsf(c[1][a] - c[0][a]));
        scale = bf_max(scale, fabsf(c[2][a] - c[0][a]));
    }
    const float floor_error = kEps * scale;
    if (!isfinite(scale) || !isfinite(floor_error) || !(floor_error > 0.0F)) {
        lane.fail();
        return false;
    }
    float point[3], perr[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float q0 = b0 * c[0][a], q1 = b1 * c[1][a], q2 = b2 * c[2][a];
        point[a] = fmaf(b0, c[0][a], fmaf(b1, c[1][a], q2));
        const float magnitude = fabsf(q0) + fabsf(q1) + fabsf(q2);
        perr[a] = bf_max(gamma7 * magnitude, floor_error);
    }
    if (!transform_position_with_error(s, inst, point, perr, hit_position, out, lane)) {
        return false;
    }
    const float4 ngw = s.world_normals[s.inst_normal_offset[inst] + prim];
    out.ng = F3{ngw.x, ngw.y, ngw.z};
    // interpolate_shading_normal (:305-349) with robust_transformed_normal (:252-295)
    const F3 on{fmaf(b0, n0.x, fmaf(b1, n1.x, b2 * n2.x)), fmaf(b0, n0.y, fmaf(b1, n1.y, b2 * n2.y)),
                fmaf(b0, n0.z, fmaf(b1, n1.z, b2 * n2.z))};
    F3 ns;
    if (!transform_normal(s, inst, on, ns, lane)) {
        return false;
    }
    if (info.w >> 31) {  // orientation flag precomputed at scene build (transform_orientation)
        ns = -ns;
    }
    if (!(dot(out.ng, ns) > 0.0F)) {
        lane.fail();
        return false;
    }
    out.ns = ns;
    const uint4 minfo = s.material_info[material];
    if (minfo.y != 0U) {
        lane.fail(kLaneUnsupported);
        return false;
    }
    out.frame = rotated_about_normal(frame_from_normal(ns, lane), __uint_as_float(minfo.z), lane);
    return lane.err == 0;
}

// ------------------------------------------------------------------------------------------------
// Mesh-light sampling (AreaLights.hpp:1184-1243, 1296-1309) and uniform light selection
// ------------------------------------------------------------------------------------------------

struct LightSample {
    bool valid;
    F3 position, error, normal, direction;
    float pdf;  // solid angle, or the discrete mass (1) of a punctual light
    float radiance[4];
    uint32_t endpoint;  // 0 surface point, 1 finite point (point, spot), 2 infinite (directional)
};

__device__ __forceinline__ uint32_t upper_bound(const float* a, uint32_t n, float u) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (u < a[mid]) {
            hi = mid;
        } else {
            lo = mid + 1U;
        }
    }
    return lo;
}

static __device__ void sample_mesh_light(const SceneView& s, const LightInfo& light, F3 context, float u, float v,
                                  LightSample& out, Lane& lane) {
    out.valid = false;
    const float* cdf = s.light_tri_cdf + light.tri_offset;
    const uint32_t index = upper_bound(cdf, light.tri_count, u);
    if (index >= light.tri_count) {
        lane.fail();
        return;
    }
    const float previous = index == 0 ? 0.0F : cdf[index - 1];
    const float selection = cdf[index] - previous;
    const float remapped = (u - previous) / selection;
    if (!isfinite(selection) || !(selection > 0.0F) || !isfinite(remapped) || remapped < 0.0F || !(remapped < 1.0F)) {
        lane.fail();
        return;
    }
    const float density = selection / s.light_tri_areas[light.tri_offset + index];
    if (!isfinite(density) || !(density > 0.0F)) {
        lane.fail();
        return;
    }
    const float root = sqrtf(remapped);
    const float bary[3] = {1.0F - root, root * (1.0F - v), root * v};
    const float4* tv = s.light_tri_vertices + 3ULL * (light.tri_offset + index);
    const float4 a = tv[0], b = tv[1], c = tv[2];
    const float cs[3][3] = {{a.x, a.y, a.z}, {b.x, b.y, b.z}, {c.x, c.y, c.z}};
    const float gamma12 = (12.0F * kEps) / (1.0F - 12.0F * kEps);
    const float underflow = 12.0F * kDenormMin;
    const float base[3] = {light.err_x, light.err_y, light.err_z};
    float point[3], error[3];
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const float q0 = bary[0] * cs[0][axis], q1 = bary[1] * cs[1][axis], q2 = bary[2] * cs[2][axis];
        point[axis] = fmaf(bary[0], cs[0][axis], fmaf(bary[1], cs[1][axis], q2));
        const float magnitude = fabsf(q0) + fabsf(q1) + fabsf(q2);
        const float arithmetic = fmaf(gamma12, magnitude, underflow);
        error[axis] = nextafterf(base[axis] + arithmetic, kInf);
    }
    out.position = F3{point[0], point[1], point[2]};
    out.error = F3{error[0], error[1], error[2]};
    const float4 ln = s.light_tri_normals[light.tri_offset + index];
    out.normal = F3{ln.x, ln.y, ln.z};
    if (emission_side(out.normal, context - out.position, lane) <= 0) {
        return;
    }
    out.pdf = area_to_solid_angle(density, context, out.position, out.normal, lane);
    // IncidentLightSample::create_finite (Light.hpp:401-441)
    const F3 disp = out.position - context;
    const float scale = max_abs3(disp);
    if (!(scale > 0.0F) || !isfinite(scale)) {
        lane.fail();
        return;
    }
    const F3 sd = disp / scale;
    const float sq = fmaf(sd.x, sd.x, fmaf(sd.y, sd.y, sd.z * sd.z));
    const float sl = sqrtf(sq);
    const float distance = scale * sl;
    if (!isfinite(sl) || !(sl > 0.0F) || !isfinite(distance) || !(distance > 0.0F)) {
        lane.fail();
        return;
    }
    out.direction = sd / sl;
    if (!unit_length(out.direction) || !isfinite(out.pdf) || !(out.pdf > 0.0F)) {
        lane.fail();
        return;
    }
    bool black = true;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        out.radiance[l] = light.radiance[l];
        black = black && light.radiance[l] == 0.0F;
    }
    out.endpoint = 0U;
    out.valid = !black && lane.err == 0;
}

// scale_radiometric_value (PunctualLights.hpp:131-183) with n numerator and three denominator factors
__device__ __forceinline__ float scale_radiometric(float value, const float* num, int n, const float (&den)[3],
                                                   Lane& lane) {
    if (!isfinite(value) || value < 0.0F) {
        lane.fail();
        return 0.0F;
    }
    for (int i = 0; i < n; ++i) {
        if (!isfinite(num[i]) || !(num[i] > 0.0F)) {
            lane.fail();
            return 0.0F;
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (!isfinite(den[i]) || !(den[i] > 0.0F)) {
            lane.fail();
            return 0.0F;
        }
    }
    if (value == 0.0F) {
        return 0.0F;
    }
    int exponent = 0;
    float fraction = frexpf(value, &exponent);
    int accumulated = exponent;
    for (int i = 0; i < n; ++i) {
        int e = 0;
        fraction *= frexpf(num[i], &e);
        accumulated += e;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        int e = 0;
        fraction /= frexpf(den[i], &e);
        accumulated -= e;
    }
    int ne = 0;
    fraction = frexpf(fraction, &ne);
    const float result = scalbnf(fraction, accumulated + ne);
    if (!isfinite(result) || !(result > 0.0F)) {
        lane.fail();
    }
    return result;
}

// PointLight / DirectionalLight / SpotLight::sample_li (PunctualLights.hpp:390-430, 510-530,
// 654-720) with IncidentLightSample::create_finite / create_infinite (Light.hpp:404-456).
static __device__ void sample_punctual_light(const PunctualLight& light, F3 context, float u, float v,
                                             LightSample& out, Lane& lane) {
    out.valid = false;
    out.pdf = 1.0F;
    if (!isfinite(u) || !isfinite(v) || u < 0.0F || u >= 1.0F || v < 0.0F || v >= 1.0F) {
        lane.fail();
        return;
    }
    const bool black = light.spectrum[0] == 0.0F && light.spectrum[1] == 0.0F && light.spectrum[2] == 0.0F &&
                       light.spectrum[3] == 0.0F;
    if (light.kind == BF200_PUNCTUAL_DIRECTIONAL) {
        if (black) {
            return;
        }
        out.direction = F3{-light.dx, -light.dy, -light.dz};
        if (!unit_length(out.direction)) {
            lane.fail();
            return;
        }
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            out.radiance[l] = light.spectrum[l];
        }
        out.endpoint = 2U;
        out.valid = true;
        return;
    }
    // finite_light_geometry (PunctualLights.hpp:102-129)
    const F3 position{light.px, light.py, light.pz};
    const F3 disp = position - context;
    if (!finite3(disp)) {
        lane.fail();
        return;
    }
    const float scale = max_abs3(disp);
    if (!(scale > 0.0F) || !isfinite(scale)) {
        lane.fail();
        return;
    }
    const F3 scaled = disp / scale;
    const float squared = fmaf(scaled.x, scaled.x, fmaf(scaled.y, scaled.y, scaled.z * scaled.z));
    const float root = sqrtf(squared);
    const float distance = scale * root;
    if (!isfinite(squared) || !(squared > 0.0F) || !isfinite(root) || !(root > 0.0F) || !isfinite(distance) ||
        !(distance > 0.0F)) {
        lane.fail();
        return;
    }
    const F3 to_light = scaled / root;
    if (!unit_length(to_light)) {
        lane.fail();
        return;
    }
    float falloff[3] = {1.0F, 1.0F, 1.0F};
    int falloff_count = 0;
    if (light.kind == BF200_PUNCTUAL_SPOT) {
        const float cone = fmaf(light.dx, -to_light.x, fmaf(light.dy, -to_light.y, light.dz * -to_light.z));
        if (!isfinite(cone)) {
            lane.fail();
            return;
        }
        if (cone <= light.cos_outer) {
            return;
        }
        falloff_count = 3;
        if (light.hard == 0U && cone < light.cos_inner) {
            const float transition = (cone - light.cos_outer) / (light.cos_inner - light.cos_outer);
            const float smooth = 3.0F - 2.0F * transition;
            if (!isfinite(transition) || !(transition > 0.0F) || !(transition < 1.0F) || !isfinite(smooth) ||
                !(smooth > 0.0F)) {
                lane.fail();
                return;
            }
            falloff[0] = transition;
            falloff[1] = transition;
            falloff[2] = smooth;
        }
    }
    const float den[3] = {scale, scale, squared};
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        out.radiance[l] = scale_radiometric(light.spectrum[l], falloff, falloff_count, den, lane);
    }
    if (black) {
        return;
    }
    out.direction = to_light;  // create_finite repeats the same arithmetic
    out.position = position;
    out.error = F3{light.ex, light.ey, light.ez};
    out.endpoint = 1U;
    out.valid = lane.err == 0;
}

// contract_point_endpoint (ShadowRay.hpp:66-113)
__device__ __forceinline__ F3 contract_point_endpoint(F3 point, F3 error, F3 to_light, Lane& lane) {
    float contraction = 0.0F;
    const float d[3] = {to_light.x, to_light.y, to_light.z}, e[3] = {error.x, error.y, error.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float candidate = fmaf(fabsf(d[a]), e[a], contraction);
        if (!isfinite(candidate) || candidate < contraction) {
            lane.fail();
        }
        contraction = (d[a] != 0.0F && e[a] != 0.0F) ? nextafterf(candidate, kInf) : candidate;
    }
    if (!isfinite(contraction)) {
        lane.fail();
    }
    if (contraction == 0.0F) {
        return point;
    }
    float c[3] = {fmaf(-d[0], contraction, point.x), fmaf(-d[1], contraction, point.y),
                  fmaf(-d[2], contraction, point.z)};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (d[a] != 0.0F) {
            c[a] = nextafterf(c[a], d[a] > 0.0F ? -kInf : kInf);
        }
    }
    const F3 out{c[0], c[1], c[2]};
    if (!finite3(out)) {
        lane.fail();
    }
    return out;
}

// DepthFilteredClosureMixture::create (DepthFilteredClosureMixture.hpp:262-364) on the generic
// route: the material's closures filtered by the depth limits into `m`.
static __device__ void mix_filter(const SceneView& s, uint32_t material, const TransportParams& p, uint32_t depth,
                                  Mix& m, Lane& lane) {
    const uint4 minfo = s.material_info[material];
    const MixDistribution& dist = s.mix_dist[material];
    m.closures = s.mix_closures + minfo.w;
    m.count = 0U;
    m.blocked = 0U;
    for (uint32_t i = 0; i < minfo.x; ++i) {
        const ClosureData c = m.closures[i];
        uint32_t allowed = 0U;
        if (c.kind == kClosureDielectric) {
            const uint32_t br = depth_blocked(p, depth, kLobeGlossy | kLobeReflection);
            const uint32_t bt = depth_blocked(p, depth, kLobeGlossy | kLobeTransmission);
            if (br == 0U) allowed |= kLobeReflection; else m.blocked |= br;
            if (bt == 0U) allowed |= kLobeTransmission; else m.blocked |= bt;
        } else {
            if (!cone_surface_event(c.lobes)) {  // is_valid_surface_scattering_event
                lane.fail();
                return;
            }
            const uint32_t bl = depth_blocked(p, depth, c.lobes);
            if (bl == 0U) allowed |= c.lobes & (kLobeReflection | kLobeTransmission); else m.blocked |= bl;
        }
        if (allowed == 0U) {
            continue;
        }
        m.source[m.count] = static_cast<uint8_t>(i);
        m.allowed[m.count] = static_cast<uint8_t>(allowed);
        m.p[m.count] = dist.p[i];
        ++m.count;
    }
    if (m.count == 0U) {
        return;
    }
    if (m.count == minfo.x) {
        for (uint32_t i = 0; i <= m.count; ++i) {
            m.cdf[i] = dist.cdf[i];
        }
        return;
    }
    if (m.count == 1U) {
        m.p[0] = 1.0F;
        m.cdf[0] = 0.0F;
        m.cdf[1] = 1.0F;
        return;
    }
    float sum = 0.0F, correction = 0.0F;
    for (uint32_t i = 0; i < m.count; ++i) {
        if (!add_compensated(m.p[i], sum, correction)) {
            lane.fail();
            return;
        }
    }
    const float total = sum + correction;
    if (!isfinite(total) || !(total > 0.0F)) {
        lane.fail();
        return;
    }
    float normalized[kMaxClosures];
    for (uint32_t i = 0; i < m.count; ++i) {
        normalized[i] = m.p[i] / total;
    }
    if (!component_distribution(normalized, m.count, m.p, m.cdf)) {
        lane.fail();
    }
}

// ------------------------------------------------------------------------------------------------
// k_shade: one bounce of the scalar MIS loop (SceneMisPathLoop.cpp:685-916) per active slot
// ------------------------------------------------------------------------------------------------

struct ShadowRecord {
    bool valid;
    F3 origin, direction;
    float t_max;
    float contribution[4];
};

__device__ __forceinline__ void terminate(const Wavefront& w, uint32_t slot, uint32_t termination, uint32_t blocked) {
    w.flags[slot] = (w.flags[slot] & 0xFFU) | (termination << 8) | (blocked << 16);
    w.state[slot] = kSlotDone;
}

__device__ __forceinline__ void add_product(float4& acc, const float4 a, const float (&b)[4], Lane& lane) {
    const float av[4] = {a.x, a.y, a.z, a.w};
    float r[4] = {acc.x, acc.y, acc.z, acc.w};
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        const float p = av[l] * b[l];
        if (!isfinite(p) || (av[l] != 0.0F && b[l] != 0.0F && p == 0.0F)) {
            lane.fail();
        }
        r[l] = r[l] + p;
        if (!isfinite(r[l])) {
            lane.fail();
        }
    }
    acc = make_float4(r[0], r[1], r[2], r[3]);
}

// SceneMisPathLoop.cpp:481-528
__device__ __forceinline__ void add_weighted_emission(float4& acc, const float4 beta, const float (&le)[4], float wgt,
                                                      Lane& lane) {
    if (!isfinite(wgt) || wgt < 0.0F || wgt > 1.0F) {
        lane.fail();
        return;
    }
    if (wgt == 1.0F) {
        add_product(acc, beta, le, lane);
        return;
    }
    const float bv[4] = {beta.x, beta.y, beta.z, beta.w};
    float r[4] = {acc.x, acc.y, acc.z, acc.w};
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        if (bv[l] == 0.0F || le[l] == 0.0F || wgt == 0.0F) {
            continue;
        }
        int e1 = 0, e2 = 0, e3 = 0, en = 0;
        const float significand = frexpf(bv[l], &e1) * frexpf(le[l], &e2) * frexpf(wgt, &e3);
        const float normalized = frexpf(significand, &en);
        const float contribution = scalbnf(normalized, e1 + e2 + e3 + en);
        if (!isfinite(contribution) || !(contribution > 0.0F)) {
            lane.fail();
        }
        r[l] = r[l] + contribution;
    }
    acc = make_float4(r[0], r[1], r[2], r[3]);
}

__device__ __forceinline__ bool is_black4(const float (&v)[4]) {
    return v[0] == 0.0F && v[1] == 0.0F && v[2] == 0.0F && v[3] == 0.0F;
}

// SceneMisPathLoop.cpp:136-275 (estimate) without the visibility query: the record carries the
// shadow ray and the contribution it adds when unoccluded (transmittance 1). The light is a
// punctual light (registry slots [0, punctual_count), a discrete sample without MIS) or a mesh light.
template <int K, bool TREE>
__device__ void direct_lighting(const SceneView& s, const TransportParams& p, const Surface& surf, const Mix& mix,
                                const float4 beta4, F3 wo_world, uint64_t dims, const Stream& stream, uint32_t mask,
                                ShadowRecord& rec, Lane& lane) {
    rec.valid = false;
    const float beta[4] = {beta4.x, beta4.y, beta4.z, beta4.w};
    if (is_black4(beta)) {
        return;
    }
    bool all_black = true;
    for (uint32_t i = 0; i < (K != 0 ? 1U : mix.count); ++i) {
        all_black = all_black && is_black4(mix_closure<K>(mix, i).w);
    }
    if (all_black) {
        return;
    }
    const float u_sel = stream.sample_1d(dims + 0);
    uint32_t b = 0;
    float selection = 0.0F;
    if constexpr (TREE) {  // LightSampler::sample(context, u) at the shading point
        const float at[3] = {surf.position.x, surf.position.y, surf.position.z};
        if (!d_tree_select(s.tree, s.tree_node_count, s.tree_root, s.light_count, s.tree_log_extent,
                           s.tree_has_extent != 0U, at, u_sel, b, selection)) {
            lane.fail();
            return;
        }
    } else {
        b = upper_bound(s.light_select_cdf + 1, s.light_count, u_sel);
        if (b >= s.light_count) {
            lane.fail();
            return;
        }
        selection = s.light_select_cdf[b + 1] - s.light_select_cdf[b];
    }
    LightSample ls;
    const float lu = stream.sample_1d(dims + 1), lv = stream.sample_1d(dims + 2);
    if (b < s.punctual_count) {
        sample_punctual_light(s.punctual[b], surf.position, lu, lv, ls, lane);
    } else {
        const LightInfo light = s.lights[b - s.punctual_count];
        if ((s.inst_info[light.instance].z & mask) == 0U) {
            return;
        }
        sample_mesh_light(s, light, surf.position, lu, lv, ls, lane);
    }
    if (!ls.valid) {
        return;
    }
    const F3 wo = surf.frame.to_local(wo_world);
    const F3 wi = surf.frame.to_local(ls.direction);
    if (wo.z == 0.0F || wi.z == 0.0F) {
        return;
    }
    const ClosureData first = mix_closure<K>(mix, 0);
    const bool lambert = (K != 0 || mix.count == 1U) && kind_is<K>(first, kClosureLambert);
    float f[4] = {0.0F, 0.0F, 0.0F, 0.0F};
    if (!lambert) {
        mix_eval<K>(mix, wo, wi, f, lane);
        if (is_black4(f)) {
            return;
        }
    }
    // shading_normal_correction in radiance mode (ShadingNormalCorrection.hpp:65-121)
    {
        const float og = dot(surf.ng, wo_world), os = dot(surf.ns, wo_world);
        const float ig = dot(surf.ng, ls.direction), is = dot(surf.ns, ls.direction);
        if (og == 0.0F || os == 0.0F || ig == 0.0F || is == 0.0F || signbit(og) != signbit(os) ||
            signbit(ig) != signbit(is)) {
            return;
        }
    }
    float weight = 1.0F;
    if (ls.endpoint == 0U) {  // a solid-angle density: MIS against the closures' density
        const float bsdf_pdf = mix_pdf<K>(mix, wo, wi, lane);
        const float light_pdf = joint_light_pdf(selection, ls.pdf, lane);
        weight = mis_weight(p.heuristic, light_pdf, bsdf_pdf, lane);
    }
    // make_shadow_ray (ShadowRay.hpp:181-253)
    const F3 origin = offset_surface_point(surf.position, surf.error, surf.ng, ls.direction, lane);
    F3 sd = ls.direction;
    float t_max = kInf;
    if (ls.endpoint != 2U) {
        F3 endpoint;
        if (ls.endpoint == 1U) {
            F3 nominal{0.0F, 0.0F, 1.0F};
            float nominal_length = 1.0F;
            unit_segment(origin, ls.position, ls.direction, nominal, nominal_length, lane);
            endpoint = contract_point_endpoint(ls.position, ls.error, nominal, lane);
        } else {
            endpoint = offset_surface_point(ls.position, ls.error, ls.normal, origin - ls.position, lane);
        }
        float length = 1.0F;
        unit_segment(origin, endpoint, ls.direction, sd, length, lane);
        t_max = nextafterf(length, 0.0F);
        if (!(t_max > 0.0F) || !isfinite(t_max)) {
            lane.fail();
        }
    }
    if (lane.err != 0) {
        return;
    }
    float out[4];
    if (lambert) {
        // evaluate_lambertian_direct_lighting (DirectLighting.hpp:171-236)
        if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
            return;
        }
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const float den[2] = {selection, ls.pdf};
            if (weight == 1.0F) {
                const float num[6] = {beta[l], first.w[l], kInvPi, ls.radiance[l], wi.z, 1.0F};
                out[l] = checked_product_quotient(num, den, lane);
            } else {
                const float num[7] = {beta[l], first.w[l], kInvPi, ls.radiance[l], wi.z, 1.0F, weight};
                out[l] = checked_product_quotient(num, den, lane);
            }
        }
    } else {
        // evaluate_bsdf_direct_lighting (DirectLighting.hpp:66-145)
        const float cosine = fabsf(wi.z);
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const float den[2] = {selection, ls.pdf};
            if (weight == 1.0F) {
                const float num[5] = {beta[l], f[l], ls.radiance[l], cosine, 1.0F};
                out[l] = checked_product_quotient(num, den, lane);
            } else {
                const float num[6] = {beta[l], f[l], ls.radiance[l], cosine, 1.0F, weight};
                out[l] = checked_product_quotient(num, den, lane);
            }
        }
    }
    rec.valid = true;
    rec.origin = origin;
    rec.direction = sd;
    rec.t_max = t_max;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        rec.contribution[l] = out[l];
    }
}

// ------------------------------------------------------------------------------------------------
// Path-replay adjoint. A replay traces every path of the forward pass again (same sample indices,
// so the same vertices) and knows, from the forward pass, the radiance L the path ends with. With
// the sampled directions held fixed, every contribution a path adds after its vertex v is linear in
// v's closure weight, so dL/dw(v) = (L - radiance accumulated through v's emission) / w(v): path
// replay backpropagation (Vicini, Speierer and Jakob, SIGGRAPH 2021) without a reverse pass. The
// roughness enters only through the BSDF value (the sampling density and MIS weights are held
// fixed, "detached"), so a vertex contributes (what follows it) x d log f / d alpha; the score of the
// continuation is applied at the next vertex, once that vertex knows what the shadow ray added. The
// loss derivative per path lane is g = dLoss/d(pixel rgb) x the film's linear sensor map.
// ------------------------------------------------------------------------------------------------

struct AdjointLane {
    bool on;         // false for a path the forward pass failed (it is not in the film)
    float g[4];      // dLoss / d(path radiance lane l)
    float4 forward;  // the path's forward radiance
};

__device__ __forceinline__ AdjointLane adjoint_lane(const AdjointView& a, uint64_t id) {
    AdjointLane al;
    al.forward = a.forward[id];
    al.on = !isnan(al.forward.x);
    const float4 gp = a.pixel_adjoint[id % a.pixels];
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        al.g[l] = gp.x * a.lane_rgb[0][l] + gp.y * a.lane_rgb[1][l] + gp.z * a.lane_rgb[2][l];
    }
    return al;
}

// sum over lanes of g_l (L_l - acc_l): the loss derivative carried by what the path adds after acc
__device__ __forceinline__ double adjoint_rest(const AdjointLane& al, float4 acc) {
    return static_cast<double>(al.g[0]) * (static_cast<double>(al.forward.x) - acc.x) +
           static_cast<double>(al.g[1]) * (static_cast<double>(al.forward.y) - acc.y) +
           static_cast<double>(al.g[2]) * (static_cast<double>(al.forward.z) - acc.z) +
           static_cast<double>(al.g[3]) * (static_cast<double>(al.forward.w) - acc.w);
}

__device__ __forceinline__ double adjoint_dot(const AdjointLane& al, const float (&c)[4]) {
    return static_cast<double>(al.g[0]) * c[0] + static_cast<double>(al.g[1]) * c[1] +
           static_cast<double>(al.g[2]) * c[2] + static_cast<double>(al.g[3]) * c[3];
}

struct D3 {
    double x, y, z;
};

__device__ __forceinline__ D3 unit_d3(double x, double y, double z) {
    const double n = sqrt(x * x + y * y + z * z);
    return {x / n, y / n, z / n};
}

__device__ __forceinline__ double smith_root(double ax, double ay, D3 v) {
    return sqrt(1.0 + (ax * ax * v.x * v.x + ay * ay * v.y * v.y) / (v.z * v.z));
}

// d log f / d(alpha_x, alpha_y) of a GGX lobe with microfacet normal m whose height-correlated
// masking pairs the directions a and b (local frame, z > 0). f depends on the roughness only
// through D(m) = 1 / (pi ax ay A^2), A = mx^2/ax^2 + my^2/ay^2 + mz^2, and G2 = 2 / (q(a) + q(b)),
// q(v) = sqrt(1 + (ax^2 vx^2 + ay^2 vy^2) / vz^2) (the G2 of ggx_g2, written with q = 1 / nor).
static __device__ double2 ggx_log_roughness_gradient(double ax, double ay, D3 m, D3 a, D3 b) {
    const double mx2 = m.x * m.x, my2 = m.y * m.y;
    const double area = mx2 / (ax * ax) + my2 / (ay * ay) + m.z * m.z;
    double dx = -1.0 / ax + 4.0 * mx2 / (ax * ax * ax * area);
    double dy = -1.0 / ay + 4.0 * my2 / (ay * ay * ay * area);
    const double qa = smith_root(ax, ay, a), qb = smith_root(ax, ay, b);
    const double sum = qa + qb;
    dx -= (ax * a.x * a.x / (a.z * a.z * qa) + ax * b.x * b.x / (b.z * b.z * qb)) / sum;
    dy -= (ay * a.y * a.y / (a.z * a.z * qa) + ay * b.y * b.y / (b.z * b.z * qb)) / sum;
    return make_double2(dx, dy);
}

// Roughness score of a closure for the local directions (wo, wi): false for closures without a
// roughness (Lambert) and for direction pairs the closure gives no value.
static __device__ bool closure_roughness_score(const ClosureData& c, F3 wo, F3 wi, double2& out) {
    if (c.kind == kClosureConductor) {
        if (!(wo.z > 0.0F) || !(wi.z > 0.0F)) {
            return false;
        }
        const D3 m = unit_d3(static_cast<double>(wo.x) + wi.x, static_cast<double>(wo.y) + wi.y,
                             static_cast<double>(wo.z) + wi.z);
        out = ggx_log_roughness_gradient(c.p[8], c.p[9], m, D3{wo.x, wo.y, wo.z}, D3{wi.x, wi.y, wi.z});
        return true;
    }
    if (c.kind != kClosureDielectric || wo.z == 0.0F || wi.z == 0.0F) {
        return false;
    }
    // the face-oriented pair of dielectric_eval
    const double sign = wo.z > 0.0F ? 1.0 : -1.0;
    const D3 of{sign * wo.x, sign * wo.y, sign * wo.z};
    const D3 in{sign * wi.x, sign * wi.y, sign * wi.z};
    if (in.z > 0.0) {
        const D3 m = unit_d3(of.x + in.x, of.y + in.y, of.z + in.z);
        out = ggx_log_roughness_gradient(c.p[2], c.p[3], m, of, in);
        return true;
    }
    const double incident = sign > 0.0 ? c.p[0] : c.p[1];
    const double transmitted = sign > 0.0 ? c.p[1] : c.p[0];
    D3 m = unit_d3(incident * of.x + transmitted * in.x, incident * of.y + transmitted * in.y,
                   incident * of.z + transmitted * in.z);
    if (m.z < 0.0) {
        m = D3{-m.x, -m.y, -m.z};
    }
    if (!(m.z > 0.0)) {
        return false;
    }
    out = ggx_log_roughness_gradient(c.p[2], c.p[3], m, of, D3{-in.x, -in.y, -in.z});
    return true;
}

__device__ __forceinline__ void adjoint_zero(double* sum) {
    for (uint32_t i = threadIdx.x; i < kAdjointWords; i += blockDim.x) {
        sum[i] = 0.0;
    }
    __syncthreads();
}

__device__ __forceinline__ void adjoint_flush(double* sum, double* gradients) {
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kAdjointWords; i += blockDim.x) {
        if (sum[i] != 0.0) {
            atomicAdd(&gradients[i], sum[i]);
        }
    }
}

// One launch per route: K is the closure kind the route's slots all share (0: generic route,
// misses and any other material). The route queue lists the route's slots in slot order.
// ADJ: the replay of the path-replay adjoint (`a` is read only then).
// K: closure kind (0 reads it from the record); ADJ: path-replay adjoint; CONE: the slots carry ray
// cones (the cone column is read and written only then); TREE: lights are selected by the scene's
// spatial light tree.
template <int K, bool ADJ, bool CONE, bool TREE>
__global__ void __launch_bounds__(256, BF200_SHADE_MIN_BLOCKS) k_shade(SceneView s, Wavefront w, PathSource src, TransportParams p,
                                               uint32_t route, AdjointView a) {
    __shared__ double adjoint_sum[ADJ ? kAdjointWords : 1];
    if constexpr (ADJ) {
        adjoint_zero(adjoint_sum);
    }
    const uint32_t begin = w.route_offsets[route], end = w.route_offsets[route + 1U];
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t active_here = 0;
    // the reference's stage counts, kept by the cone-carrying instantiations only: closure samples,
    // light samples and misses (CudaWavefrontStages.cu:4348, 4384, 4985-4997)
    uint32_t closures_here = 0, lights_here = 0, misses_here = 0;
    for (uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += stride) {
        const uint32_t slot = w.route_queue[i];
        ShadowRecord rec;
        rec.valid = false;
        {
            Lane lane;
            const uint2 id = w.hit_id[slot];
            const float4 o4 = w.ray_o[slot], d4 = w.ray_d[slot];
            float4 beta = w.beta[slot];
            float4 rad = w.radiance[slot];
            const uint32_t depth = w.depth[slot];
            const float eta = w.eta[slot];
            const float4 prev = w.prev[slot];
            const uint32_t mask = w.mask[slot];
            const Stream stream = load_stream(w, src, slot);
            const F3 ro = ld3(o4), rd = ld3(d4);
            AdjointLane al{};
            uint32_t path_tag = 0U;
            if constexpr (ADJ) {
                const uint64_t path = w.path_id[slot];
                path_tag = static_cast<uint32_t>(path) + 1U;
                al = adjoint_lane(a, path);
                const uint4 pend = a.pending[slot];
                if (al.on && pend.w == path_tag) {
                    // the previous vertex's continuation: everything from here on
                    const double rest = adjoint_rest(al, rad);
                    atomicAdd(&adjoint_sum[pend.z * kAdjointStride + 4U], rest * __uint_as_float(pend.x));
                    atomicAdd(&adjoint_sum[pend.z * kAdjointStride + 5U], rest * __uint_as_float(pend.y));
                    a.pending[slot].w = 0U;
                }
            }
            if (K == 0 && id.x == 0xFFFFFFFFU) {
                if constexpr (CONE) {
                    ++misses_here;
                }
                const float env[4] = {s.environment.x, s.environment.y, s.environment.z, s.environment.w};
                add_product(rad, beta, env, lane);
                w.radiance[slot] = rad;
                if (lane.err) {
                    w.status[slot] |= lane.err;
                }
                terminate(w, slot, 0U /*escaped*/, 0U);
            } else {
                const float4 tb = w.hit_tb[slot];
                const uint4 inst = s.inst_info[id.x];
                const uint32_t material = inst.y;
                // Ray::at (Ray.hpp:81-95)
                const F3 hit_position = ro + rd * tb.x;
                Surface surf;
                bool done = false;
                uint32_t termination = 0U, blocked = 0U;
                if (!resolve_surface(s, id.x, id.y, tb, hit_position, material, surf, lane)) {
                    done = true;
                }
                float4 emission4 = make_float4(0.0F, 0.0F, 0.0F, 0.0F);
                if (!done) {
                    const int side = emission_side(surf.ng, -rd, lane);
                    if (side > 0) {
                        emission4 = s.emission[material];
                    }
                    const float emitted[4] = {emission4.x, emission4.y, emission4.z, emission4.w};
                    float emission_weight = 1.0F;
                    if (!is_black4(emitted) && prev.w > 0.0F) {
                        const uint32_t mesh_index = inst.w & 0x7FFFFFFFU;
                        const uint32_t light_index = s.punctual_count + mesh_index;  // registry slot
                        if (light_index >= s.light_count) {
                            lane.fail();
                        } else {
                            const LightInfo light = s.lights[mesh_index];
                            float selection = 0.0F;
                            if constexpr (TREE) {  // probability(context, i) at the previous vertex
                                const float at[3] = {prev.x, prev.y, prev.z};
                                if (!d_tree_probability(s.tree, s.tree_node_count, s.tree_root, s.tree_light_to_node,
                                                        s.light_count, s.tree_log_extent, s.tree_has_extent != 0U, at,
                                                        light_index, selection)) {
                                    lane.fail();
                                }
                            } else {
                                selection = s.light_select_cdf[light_index + 1] - s.light_select_cdf[light_index];
                            }
                            const F3 pp = ld3(prev);
                            float conditional = 0.0F;
                            if (emission_side(surf.ng, pp - surf.position, lane) > 0) {
                                conditional = area_to_solid_angle(light.inverse_area, pp, surf.position, surf.ng, lane);
                            }
                            const float light_pdf = joint_light_pdf(selection, conditional, lane);
                            emission_weight = mis_weight(p.heuristic, prev.w, light_pdf, lane);
                        }
                    }
                    add_weighted_emission(rad, beta, emitted, emission_weight, lane);
                    if constexpr (ADJ) {
                        if (al.on && lane.err == 0 && !is_black4(emitted)) {
                            const float added[4] = {beta.x * emitted[0] * emission_weight,
                                                    beta.y * emitted[1] * emission_weight,
                                                    beta.z * emitted[2] * emission_weight,
                                                    beta.w * emitted[3] * emission_weight};
                            atomicAdd(&adjoint_sum[kAdjointEmission], adjoint_dot(al, added));
                        }
                    }
                    if (lane.err) {
                        done = true;
                    }
                }
                Mix mix;
                mix.count = 0U;
                if (!done) {
                    if (beta.x == 0.0F && beta.y == 0.0F && beta.z == 0.0F && beta.w == 0.0F) {
                        done = true;
                        termination = 3U;  // zero_throughput
                    }
                }
                if (!done) {
                    const uint4 minfo = s.material_info[material];
                    if (minfo.x == 0U) {
                        done = true;
                        termination = 2U;  // outside_bsdf_support
                    } else if (K == 0) {
                        mix_filter(s, material, p, depth, mix, lane);
                        if (lane.err != 0) {
                            done = true;
                        } else if (mix.count == 0U) {
                            done = true;
                            termination = 1U;  // depth_limit
                            blocked = mix.blocked;
                        }
                    } else {
                        ClosureData& closure = mix.first;
                        uint32_t allowed = 0U;
                        closure = s.closures[material];
                        // depth filter of one closure (DepthFilteredClosureMixture.hpp:262-364)
                        uint32_t block_mask = 0U;
                        if (kind_is<K>(closure, kClosureDielectric)) {
                            const uint32_t br = depth_blocked(p, depth, kLobeGlossy | kLobeReflection);
                            const uint32_t bt = depth_blocked(p, depth, kLobeGlossy | kLobeTransmission);
                            if (br == 0U) allowed |= kLobeReflection; else block_mask |= br;
                            if (bt == 0U) allowed |= kLobeTransmission; else block_mask |= bt;
                        } else {
                            const uint32_t bl = depth_blocked(p, depth, closure.lobes);
                            if (bl == 0U) allowed |= closure.lobes & (kLobeReflection | kLobeTransmission);
                            else block_mask |= bl;
                        }
                        if (allowed == 0U) {
                            done = true;
                            termination = 1U;  // depth_limit
                            blocked = block_mask;
                        }
                        mix.count = 1U;
                        mix.source[0] = 0U;
                        mix.allowed[0] = static_cast<uint8_t>(allowed);
                        mix.p[0] = 1.0F;
                        mix.cdf[0] = 0.0F;
                        mix.cdf[1] = 1.0F;
                    }
                }
                if (!done) {
                    // the single closure of the adjoint's scenes (mixtures are refused there)
                    const ClosureData closure = mix_closure<K>(mix, 0);
                    if constexpr (ADJ) {
                        if (al.on) {  // everything after this vertex scales with its closure weight
                            const float fv[4] = {al.forward.x, al.forward.y, al.forward.z, al.forward.w};
                            const float rv[4] = {rad.x, rad.y, rad.z, rad.w};
#pragma unroll
                            for (int l = 0; l < 4; ++l) {
                                if (closure.w[l] != 0.0F) {
                                    atomicAdd(&adjoint_sum[material * kAdjointStride + l],
                                              static_cast<double>(al.g[l]) *
                                                  (static_cast<double>(fv[l]) - rv[l]) / closure.w[l]);
                                }
                            }
                        }
                    }
                    const F3 wo_world = robust_unit(-rd, lane);
                    const F3 wo = surf.frame.to_local(wo_world);
                    const uint64_t dims = bounce_base(depth_total(depth));
                    BsdfSample bs;
                    mix_sample<K>(mix, wo, stream.sample_1d(dims + 3), stream.sample_1d(dims + 4),
                                  stream.sample_1d(dims + 5), bs, lane);
                    if constexpr (CONE) {
                        ++closures_here;
                        bool all_black = true;
                        for (uint32_t i = 0; i < (K != 0 ? 1U : mix.count); ++i) {
                            all_black = all_black && is_black4(mix_closure<K>(mix, i).w);
                        }
                        if (s.light_count != 0U && !all_black) {
                            ++lights_here;
                        }
                    }
                    uint32_t next_depth = depth;
                    if (bs.valid) {
                        bool finite_value = true;
#pragma unroll
                        for (int l = 0; l < 4; ++l) {
                            finite_value = finite_value && isfinite(bs.value[l]) && bs.value[l] >= 0.0F;
                        }
                        if (!cone_surface_event(bs.lobes) || !finite_value || !isfinite(bs.pdf) || !(bs.pdf > 0.0F) ||
                            bs.wi.z == 0.0F || depth_blocked(p, depth, bs.lobes) != 0U) {
                            lane.fail();
                        }
                        next_depth = depth_advance(depth, bs.lobes);
                    }
                    if (lane.err == 0) {
                        direct_lighting<K, TREE>(s, p, surf, mix, beta, wo_world, dims, stream, mask, rec, lane);
                        if constexpr (ADJ) {
                            if (al.on && rec.valid) {
                                double2 score = make_double2(0.0, 0.0);
                                const bool rough =
                                    closure_roughness_score(closure, wo, surf.frame.to_local(rec.direction), score);
                                a.shadow_score[slot] =
                                    make_uint4(__float_as_uint(static_cast<float>(score.x)),
                                               __float_as_uint(static_cast<float>(score.y)), material, rough ? 1U : 0U);
                            }
                        }
                    }
                    if (lane.err != 0) {
                        rec.valid = false;
                        done = true;
                    } else if (!bs.valid) {
                        done = true;
                        termination = 2U;
                    } else {
                        const F3 wi_world = robust_unit(surf.frame.to_world(bs.wi), lane);
                        const float og = dot(surf.ng, wo_world), os = dot(surf.ns, wo_world);
                        const float ig = dot(surf.ng, wi_world), is = dot(surf.ns, wi_world);
                        const bool corr_zero = og == 0.0F || os == 0.0F || ig == 0.0F || is == 0.0F ||
                                               signbit(og) != signbit(os) || signbit(ig) != signbit(is);
                        if (corr_zero) {
                            done = true;
                            termination = 2U;
                        } else {
                            // update_closure_throughput (BsdfOnlyPathLoop.hpp:64-131), correction 1
                            const bool delta = (bs.lobes & kLobeSpecular) != 0U;
                            if (bs.delta != delta || (delta && bs.pdf > 1.0F)) {
                                lane.fail();
                            }
                            const float bv[4] = {beta.x, beta.y, beta.z, beta.w};
                            float nb[4];
                            if ((K != 0 || mix.count == 1U) && kind_is<K>(closure, kClosureLambert)) {
#pragma unroll
                                for (int l = 0; l < 4; ++l) {
                                    nb[l] = bv[l] * closure.w[l];
                                    if (!isfinite(nb[l]) || (bv[l] != 0.0F && closure.w[l] != 0.0F && nb[l] == 0.0F)) {
                                        lane.fail();
                                    }
                                }
                            } else {
                                const float cosine = fabsf(bs.wi.z);
#pragma unroll
                                for (int l = 0; l < 4; ++l) {
                                    const float num[4] = {bv[l], bs.value[l], cosine, 1.0F};
                                    float significand = 1.0F;
                                    int exponent = 0;
                                    bool zero = false;
#pragma unroll
                                    for (int k = 0; k < 4; ++k) {
                                        if (!isfinite(num[k]) || num[k] < 0.0F) {
                                            lane.fail();
                                        }
                                        if (num[k] == 0.0F) {
                                            zero = true;
                                        }
                                        if (!zero) {
                                            int fe = 0;
                                            significand *= frexpf(num[k], &fe);
                                            exponent += fe;
                                        }
                                    }
                                    if (zero) {
                                        nb[l] = 0.0F;
                                        continue;
                                    }
                                    int pe = 0, ne = 0;
                                    significand /= frexpf(bs.pdf, &pe);
                                    exponent -= pe;
                                    significand = frexpf(significand, &ne);
                                    nb[l] = scalbnf(significand, exponent + ne);
                                    if (!isfinite(nb[l]) || !(nb[l] > 0.0F)) {
                                        lane.fail();
                                    }
                                }
                            }
                            const float next_eta = eta * bs.eta_scale;
                            if (!isfinite(next_eta) || !(next_eta > 0.0F)) {
                                lane.fail();
                            }
                            const F3 origin = offset_ray_origin(surf.position, surf.error, surf.ng, wi_world, lane);
                            if (origin == surf.position) {
                                lane.fail();
                            }
                            // the continuation's ray cone: advanced to this hit, then scattered
                            // (CudaWavefrontStages.cu:4606-4623)
                            float2 next_cone = make_float2(0.0F, 0.0F);
                            if (CONE && lane.err == 0 &&
                                (!cone_advance(w.cone[slot], rd, tb.x, next_cone) ||
                                 !cone_scatter<K>(next_cone, mix_closure<K>(mix, bs.selected), bs.lobes, wo, bs.wi,
                                                  next_cone))) {
                                lane.fail();
                            }
                            if (lane.err == 0) {
                                if constexpr (CONE) {
                                    w.cone[slot] = next_cone;
                                }
                                beta = make_float4(nb[0], nb[1], nb[2], nb[3]);
                                w.beta[slot] = beta;
                                w.depth[slot] = next_depth;
                                w.eta[slot] = next_eta;
                                // record_bsdf_sample: a delta continuation leaves no density (w = 0) for
                                // the next emissive hit's MIS weight; next_delta_flags: bit 0 previous
                                // bounce was delta, bit 1 any non-delta bounce
                                w.prev[slot] = make_float4(surf.position.x, surf.position.y, surf.position.z,
                                                           delta ? 0.0F : bs.pdf);
                                const uint32_t old_flags = w.flags[slot];
                                w.flags[slot] = (old_flags & ~0xFFU) | (old_flags & 2U) | (delta ? 1U : 2U);
                                w.ray_o[slot] = make_float4(origin.x, origin.y, origin.z, kInf);
                                w.ray_d[slot] = make_float4(wi_world.x, wi_world.y, wi_world.z, 0.0F);
                                if (nb[0] == 0.0F && nb[1] == 0.0F && nb[2] == 0.0F && nb[3] == 0.0F) {
                                    done = true;
                                    termination = 3U;
                                } else if (p.roulette != 0U && depth_total(next_depth) >= p.roulette_first) {
                                    // evaluate_russian_roulette (RussianRoulette.cpp)
                                    float mt = 0.0F;
#pragma unroll
                                    for (int l = 0; l < 4; ++l) mt = bf_max(mt, nb[l]);
                                    float survival;
                                    if (mt >= p.roulette_max / next_eta) {
                                        survival = p.roulette_max;
                                    } else if (mt <= p.roulette_min / next_eta) {
                                        survival = p.roulette_min;
                                    } else {
                                        const float v = mt * next_eta;
                                        survival = v < p.roulette_min ? p.roulette_min
                                                                      : (p.roulette_max < v ? p.roulette_max : v);
                                    }
                                    const float u = stream.sample_1d(dims + 9);
                                    if (!(u < survival)) {
                                        done = true;
                                        termination = 4U;  // russian_roulette
                                    } else {
                                        float cb[4];
#pragma unroll
                                        for (int l = 0; l < 4; ++l) {
                                            cb[l] = nb[l] / survival;
                                            if (!isfinite(cb[l]) || (nb[l] != 0.0F && cb[l] == 0.0F)) {
                                                lane.fail();
                                            }
                                        }
                                        w.beta[slot] = make_float4(cb[0], cb[1], cb[2], cb[3]);
                                    }
                                }
                                if constexpr (ADJ) {
                                    double2 score;
                                    if (al.on && !done && closure_roughness_score(closure, wo, bs.wi, score)) {
                                        a.pending[slot] = make_uint4(__float_as_uint(static_cast<float>(score.x)),
                                                                     __float_as_uint(static_cast<float>(score.y)),
                                                                     material, path_tag);
                                    }
                                }
                            } else {
                                done = true;
                            }
                        }
                    }
                }
                w.radiance[slot] = rad;
                if (lane.err != 0) {
                    rec.valid = false;
                    w.status[slot] = (w.status[slot] & ~0xFFU) | lane.err;
                    w.state[slot] = kSlotDone;
                } else if (done) {
                    terminate(w, slot, termination, blocked);
                } else {
                    ++active_here;
                }
            }
        }
        if (rec.valid) {
            w.shadow_o[slot] = make_float4(rec.origin.x, rec.origin.y, rec.origin.z, rec.t_max);
            w.shadow_d[slot] = make_float4(rec.direction.x, rec.direction.y, rec.direction.z, 0.0F);
            w.shadow_c[slot] = make_float4(rec.contribution[0], rec.contribution[1], rec.contribution[2],
                                           rec.contribution[3]);
            w.shadow_key[slot] = 0U;
        }
    }
    // active-slot count for the host's termination test
    for (int off = 16; off > 0; off >>= 1) {
        active_here += __shfl_down_sync(0xFFFFFFFFU, active_here, off);
    }
    if ((threadIdx.x & 31U) == 0U && active_here != 0U) {
        atomicAdd(&w.counters[2], static_cast<unsigned long long>(active_here));
    }
    if constexpr (CONE) {
        for (int off = 16; off > 0; off >>= 1) {
            closures_here += __shfl_down_sync(0xFFFFFFFFU, closures_here, off);
            lights_here += __shfl_down_sync(0xFFFFFFFFU, lights_here, off);
            misses_here += __shfl_down_sync(0xFFFFFFFFU, misses_here, off);
        }
        if ((threadIdx.x & 31U) == 0U) {
            // cumulative over the trace: [11] closure samples, [12] light samples, [13] misses,
            // [14] continuations
            atomicAdd(&w.counters[11], static_cast<unsigned long long>(closures_here));
            atomicAdd(&w.counters[12], static_cast<unsigned long long>(lights_here));
            atomicAdd(&w.counters[13], static_cast<unsigned long long>(misses_here));
            atomicAdd(&w.counters[14], static_cast<unsigned long long>(active_here));
        }
    }
    if constexpr (ADJ) {
        adjoint_flush(adjoint_sum, a.gradients);
    }
}

// ------------------------------------------------------------------------------------------------
// k_occlude: shadow rays of the compacted queue; unoccluded contributions join the path radiance
// ------------------------------------------------------------------------------------------------

template <bool ADJ, bool SPH>
__global__ void __launch_bounds__(256, BF200_OCCLUDE_MIN_BLOCKS) k_occlude(SceneView s, Wavefront w, AdjointView a) {
    __shared__ int stack_columns[kSharedStackEntries * 256];
    __shared__ double adjoint_sum[ADJ ? kAdjointWords : 1];
    if constexpr (ADJ) {
        adjoint_zero(adjoint_sum);
    }
    TraversalStack stack = thread_stack(stack_columns);
    const uint32_t count = w.shadow_offsets[1];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const uint32_t slot = w.shadow_queue[i];
        const float4 o = w.shadow_o[slot], d = w.shadow_d[slot];
        const int occluded = any_hit<SPH>(s, ld3(o), ld3(d), 0.0F, o.w, w.mask[slot], stack);
        if (occluded < 0) {
            w.status[slot] = (w.status[slot] & ~0xFFU) | kLaneTraversal;
            w.state[slot] = kSlotDone;
            continue;
        }
        if (occluded == 0) {
            const float4 c = w.shadow_c[slot];
            float4 r = w.radiance[slot];
            r.x = r.x + c.x;
            r.y = r.y + c.y;
            r.z = r.z + c.z;
            r.w = r.w + c.w;
            w.radiance[slot] = r;
            if constexpr (ADJ) {
                const AdjointLane al = adjoint_lane(a, w.path_id[slot]);
                if (al.on) {  // the light's radiance scales this contribution; so may the roughness
                    const float added[4] = {c.x, c.y, c.z, c.w};
                    const double e = adjoint_dot(al, added);
                    atomicAdd(&adjoint_sum[kAdjointEmission], e);
                    const uint4 score = a.shadow_score[slot];
                    if (score.w != 0U) {
                        atomicAdd(&adjoint_sum[score.z * kAdjointStride + 4U], e * __uint_as_float(score.x));
                        atomicAdd(&adjoint_sum[score.z * kAdjointStride + 5U], e * __uint_as_float(score.y));
                    }
                }
            }
        }
    }
    if constexpr (ADJ) {
        adjoint_flush(adjoint_sum, a.gradients);
    }
}

#ifdef BF200_KERNELS_MAIN_TU
// ------------------------------------------------------------------------------------------------
// k_film: CIE 1931 XYZ -> linear sRGB -> add_sample(x, y, rgb, 1) in sample order per pixel
// ------------------------------------------------------------------------------------------------

struct SensorView {
    float response[4][3];
    float pdf[4];
    float normalization;
};

__device__ __forceinline__ float sensor_term(float c, float r, float n, float p) {
    if (c == 0.0F || r == 0.0F) {
        return 0.0F;
    }
    int ec = 0, er = 0, en = 0, ep = 0;
    const float mc = frexpf(c, &ec), mr = frexpf(r, &er), mn = frexpf(n, &en), mp = frexpf(p, &ep);
    const float mantissa = mc * mr * mn / mp;
    return ldexpf(mantissa, ec + er + en - ep);
}

__global__ void k_film(const float4* path_radiance, uint32_t pixels, uint32_t samples, SensorView sensor,
                       uint32_t precision, float4* film32, double* film64, unsigned long long* counts,
                       unsigned long long* skipped) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pixels) {
        return;
    }
    float4 f = precision == 0U ? film32[p] : make_float4(0.0F, 0.0F, 0.0F, 0.0F);
    double sum[4] = {0, 0, 0, 0}, comp[4] = {0, 0, 0, 0};
    if (precision != 0U) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            sum[k] = film64[8ULL * p + k];
            comp[k] = film64[8ULL * p + 4 + k];
        }
    }
    unsigned long long count = counts[p];
    for (uint32_t s = 0; s < samples; ++s) {
        const float4 L = path_radiance[static_cast<uint64_t>(s) * pixels + p];
        if (isnan(L.x)) {
            atomicAdd(skipped, 1ULL);
            continue;
        }
        const float lv[4] = {L.x, L.y, L.z, L.w};
        float xyz[3] = {0.0F, 0.0F, 0.0F};
#pragma unroll
        for (int l = 0; l < 4; ++l) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                xyz[k] += sensor_term(lv[l], sensor.response[l][k], sensor.normalization, sensor.pdf[l]);
            }
        }
        const float red = 3.2404542F * xyz[0] - 1.5371385F * xyz[1] - 0.4985314F * xyz[2];
        const float green = -0.9692660F * xyz[0] + 1.8760108F * xyz[1] + 0.0415560F * xyz[2];
        const float blue = 0.0556434F * xyz[0] - 0.2040259F * xyz[1] + 1.0572252F * xyz[2];
        if (precision == 0U) {
            f.x += red * 1.0F;
            f.y += green * 1.0F;
            f.z += blue * 1.0F;
            f.w += 1.0F;
        } else {
            const double v[4] = {static_cast<double>(red), static_cast<double>(green), static_cast<double>(blue), 1.0};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double updated = sum[k] + v[k];
                if (fabs(sum[k]) >= fabs(v[k])) {
                    comp[k] += (sum[k] - updated) + v[k];
                } else {
                    comp[k] += (v[k] - updated) + sum[k];
                }
                sum[k] = updated;
            }
        }
        ++count;
    }
    if (precision == 0U) {
        film32[p] = f;
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            film64[8ULL * p + k] = sum[k];
            film64[8ULL * p + 4 + k] = comp[k];
        }
    }
    counts[p] = count;
}

// Per-pixel adjoint of the path-replay adjoint: dLoss/d(image) / weight, the derivative per
// unit-weight sample, where the image is the film's weighted mean rgb / weight (the Neumaier sum
// plus its compensation for a float64 film). With a target, the loss is the sum over pixels and
// channels of (image - target)^2 (added to *loss) and dLoss/d(image) = 2 (image - target);
// without one, dLoss/d(image) is the caller's image_adjoint.
__global__ void __launch_bounds__(256) k_adjoint_image(const float4* film32, const double* film64, const float* target,
                                                       const float* image_adjoint, uint32_t pixels, uint32_t precision,
                                                       float4* pixel_adjoint, double* loss) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    double part = 0.0;
    if (p < pixels) {
        double rgb[3], weight;
        if (precision == 0U) {
            const float4 f = film32[p];
            rgb[0] = f.x;
            rgb[1] = f.y;
            rgb[2] = f.z;
            weight = f.w;
        } else {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                rgb[k] = film64[8ULL * p + k] + film64[8ULL * p + 4 + k];
            }
            weight = film64[8ULL * p + 3] + film64[8ULL * p + 7];
        }
        float adj[3] = {0.0F, 0.0F, 0.0F};
        if (weight > 0.0 && target != nullptr) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double d = rgb[k] / weight - static_cast<double>(target[3ULL * p + k]);
                part += d * d;
                adj[k] = static_cast<float>(2.0 * d / weight);
            }
        } else if (weight > 0.0) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                adj[k] = static_cast<float>(static_cast<double>(image_adjoint[3ULL * p + k]) / weight);
            }
        }
        pixel_adjoint[p] = make_float4(adj[0], adj[1], adj[2], 0.0F);
    }
    for (int off = 16; off > 0; off >>= 1) {
        part += __shfl_down_sync(0xFFFFFFFFU, part, off);
    }
    if ((threadIdx.x & 31U) == 0U && part != 0.0 && loss != nullptr) {
        atomicAdd(loss, part);
    }
}
#endif  // BF200_KERNELS_MAIN_TU

// Standalone closest-hit / occlusion queries (ClosestHit.hpp:21-28, Occlusion.hpp:19-26).
template <bool SPH>
__global__ void __launch_bounds__(128) k_query_closest(SceneView s, const bf200_ray_v1* rays, uint64_t n,
                                                      bf200_hit_v1* hits) {
    __shared__ int stack_columns[kSharedStackEntries * 128];
    TraversalStack stack = thread_stack(stack_columns);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const bf200_ray_v1 r = rays[i];
        const F3 o{r.origin[0], r.origin[1], r.origin[2]}, d{r.direction[0], r.direction[1], r.direction[2]};
        const ClosestResult c = closest_hit<SPH>(s, o, d, r.t_min, r.t_max, r.mask, stack);
        bf200_hit_v1 h;
        h.t = 0.0F;
        h.barycentrics[0] = h.barycentrics[1] = h.barycentrics[2] = 0.0F;
        h.instance_index = 0xFFFFFFFFU;
        h.primitive_index = 0xFFFFFFFFU;
        h.status = c.failed ? kLaneTraversal : 0U;
        h.reserved = 0U;
        if (!c.failed && c.instance != 0xFFFFFFFFU) {
            TriangleHit th;
            if (hit_barycentrics<SPH>(s, c, o, d, r.t_min, r.t_max, th)) {
                h.t = c.t;
                h.barycentrics[0] = th.b0;
                h.barycentrics[1] = th.b1;
                h.barycentrics[2] = th.b2;
                h.instance_index = c.instance;
                h.primitive_index = c.primitive;
            } else {
                h.status = kLaneNumerical;
            }
        }
        hits[i] = h;
    }
}

template <bool SPH>
__global__ void __launch_bounds__(128) k_query_occlusion(SceneView s, const bf200_ray_v1* rays, uint64_t n,
                                                        uint32_t* out) {
    __shared__ int stack_columns[kSharedStackEntries * 128];
    TraversalStack stack = thread_stack(stack_columns);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const bf200_ray_v1 r = rays[i];
        const F3 o{r.origin[0], r.origin[1], r.origin[2]}, d{r.direction[0], r.direction[1], r.direction[2]};
        const int occ = any_hit<SPH>(s, o, d, r.t_min, r.t_max, r.mask, stack);
        out[i] = occ < 0 ? 2U : static_cast<uint32_t>(occ);
    }
}

// The four shading kernels of one wavefront iteration, one per route.
template <bool ADJ, bool CONE, bool TREE>
void launch_shading(const SceneView& s, const Wavefront& w, const PathSource& src, const TransportParams& p,
                    uint32_t grid, const AdjointView& a, cudaStream_t stream) {
    k_shade<0, ADJ, CONE, TREE><<<grid, 256, 0, stream>>>(s, w, src, p, kRouteGeneric, a);
    k_shade<static_cast<int>(kClosureLambert), ADJ, CONE, TREE><<<grid, 256, 0, stream>>>(s, w, src, p,
                                                                                           kRouteLambert, a);
    k_shade<static_cast<int>(kClosureConductor), ADJ, CONE, TREE><<<grid, 256, 0, stream>>>(s, w, src, p,
                                                                                             kRouteConductor, a);
    k_shade<static_cast<int>(kClosureDielectric), ADJ, CONE, TREE><<<grid, 256, 0, stream>>>(s, w, src, p,
                                                                                              kRouteDielectric, a);
}

#ifdef BF200_KERNELS_MAIN_TU
// The shading launchers are instantiated in their own translation units (bf200_shade_*.cu), which
// compile in parallel.
extern template void launch_shading<false, false, false>(const SceneView&, const Wavefront&, const PathSource&,
    const TransportParams&, uint32_t, const AdjointView&, cudaStream_t);
extern template void launch_shading<false, true, false>(const SceneView&, const Wavefront&, const PathSource&,
    const TransportParams&, uint32_t, const AdjointView&, cudaStream_t);
extern template void launch_shading<false, false, true>(const SceneView&, const Wavefront&, const PathSource&,
    const TransportParams&, uint32_t, const AdjointView&, cudaStream_t);
extern template void launch_shading<false, true, true>(const SceneView&, const Wavefront&, const PathSource&,
    const TransportParams&, uint32_t, const AdjointView&, cudaStream_t);
extern template void launch_shading<true, false, false>(const SceneView&, const Wavefront&, const PathSource&,
    const TransportParams&, uint32_t, const AdjointView&, cudaStream_t);

// ------------------------------------------------------------------------------------------------
// k_iteration_gate: the end of one wavefront iteration inside a graph's device-side loop
// ------------------------------------------------------------------------------------------------

// One thread. Accumulates the iteration's shadow segments, counts the iteration, clears the
// per-iteration counters for the next one, and keeps the loop running while paths remain to be
// claimed or traced -- but never past `max_iterations`, when it raises counters[10] instead.
__global__ void k_iteration_gate(Wavefront w, uint64_t total, uint64_t max_iterations,
                                 cudaGraphConditionalHandle loop) {
    unsigned long long* c = w.counters;
    c[4] += c[0];
    const unsigned long long iteration = ++c[9];
    const bool drained = c[2] == 0ULL && c[1] >= total;
    const bool bound = iteration >= max_iterations;
    if (!drained && bound) {
        c[10] = 1ULL;
    }
    c[0] = 0ULL;
    c[2] = 0ULL;
    cudaGraphSetConditional(loop, (!drained && !bound) ? 1U : 0U);
}

// ------------------------------------------------------------------------------------------------
// Host-side launchers
// ------------------------------------------------------------------------------------------------

cudaError_t launch_gate(const Wavefront& w, uint64_t total, uint64_t max_iterations, cudaGraphConditionalHandle loop,
                        cudaStream_t stream) {
    k_iteration_gate<<<1, 1, 0, stream>>>(w, total, max_iterations, loop);
    return cudaGetLastError();
}


cudaError_t launch_world_normals(const SceneView& s, uint32_t total, float4* out, uint32_t* failures,
                                 cudaStream_t stream) {
    if (total == 0U) {
        return cudaSuccess;
    }
    const uint32_t blocks = (total + 127U) / 128U;
    k_world_normals<<<blocks < 4096U ? blocks : 4096U, 128, 0, stream>>>(s, total, out, failures);
    return cudaGetLastError();
}

cudaError_t launch_stage(int stage, const SceneView& s, const Wavefront& w, const PathSource& src,
                         const TransportParams& p, uint32_t grid, cudaStream_t stream, uint32_t* launches,
                         const AdjointView* adjoint) {
    cudaError_t e = cudaSuccess;
    if (stage == 0) {
        k_regenerate<<<grid, 256, 0, stream>>>(w, src);
        *launches += 1U;
        return cudaGetLastError();
    }
    if (stage == 1) {
        if (s.sphere_count != 0U) {
            k_trace<true><<<grid, 256, 0, stream>>>(s, w);
        } else {
            k_trace<false><<<grid, 256, 0, stream>>>(s, w);
        }
        *launches += 1U;
        return cudaGetLastError();
    }
    if (stage == 2) {
        // route the traced slots, shade each route with its own kernel, then queue the shadow rays
        e = launch_compaction(w.route, w.capacity, kRouteCount, w.tile_counts, w.route_queue, w.route_offsets,
                              nullptr, w.shadow_key, stream, launches);
        if (e != cudaSuccess) {
            return e;
        }
        if (adjoint != nullptr) {
            launch_shading<true, false, false>(s, w, src, p, grid, *adjoint, stream);
        } else if (s.tree != nullptr) {
            if (src.cones_in != nullptr) {
                launch_shading<false, true, true>(s, w, src, p, grid, AdjointView{}, stream);
            } else {
                launch_shading<false, false, true>(s, w, src, p, grid, AdjointView{}, stream);
            }
        } else if (src.cones_in != nullptr) {
            launch_shading<false, true, false>(s, w, src, p, grid, AdjointView{}, stream);
        } else {
            launch_shading<false, false, false>(s, w, src, p, grid, AdjointView{}, stream);
        }
        *launches += 4U;
        if ((e = cudaGetLastError()) != cudaSuccess) {
            return e;
        }
        return launch_compaction(w.shadow_key, w.capacity, 1U, w.tile_counts, w.shadow_queue, w.shadow_offsets,
                                 w.counters + 0, nullptr, stream, launches);
    }
    const AdjointView a = adjoint != nullptr ? *adjoint : AdjointView{};
    if (s.sphere_count != 0U) {
        if (adjoint != nullptr) {
            k_occlude<true, true><<<grid, 256, 0, stream>>>(s, w, a);
        } else {
            k_occlude<false, true><<<grid, 256, 0, stream>>>(s, w, a);
        }
    } else if (adjoint != nullptr) {
        k_occlude<true, false><<<grid, 256, 0, stream>>>(s, w, a);
    } else {
        k_occlude<false, false><<<grid, 256, 0, stream>>>(s, w, a);
    }
    *launches += 1U;
    return cudaGetLastError();
}

cudaError_t launch_retire(const Wavefront& w, const PathSource& src, uint32_t grid, cudaStream_t stream) {
    k_regenerate<<<grid, 256, 0, stream>>>(w, src);
    return cudaGetLastError();
}

cudaError_t launch_film(const float4* path_radiance, uint32_t pixels, uint32_t samples, const float* response12,
                        const float* pdf4, float normalization, uint32_t precision, float4* film32, double* film64,
                        unsigned long long* counts, unsigned long long* skipped, cudaStream_t stream) {
    SensorView sv;
    for (int l = 0; l < 4; ++l) {
        for (int k = 0; k < 3; ++k) {
            sv.response[l][k] = response12[3 * l + k];
        }
        sv.pdf[l] = pdf4[l];
    }
    sv.normalization = normalization;
    k_film<<<(pixels + 127U) / 128U, 128, 0, stream>>>(path_radiance, pixels, samples, sv, precision, film32, film64,
                                                      counts, skipped);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_image(const float4* film32, const double* film64, const float* target,
                                 const float* image_adjoint, uint32_t pixels, uint32_t precision, float4* pixel_adjoint,
                                 double* loss, cudaStream_t stream) {
    k_adjoint_image<<<(pixels + 255U) / 256U, 256, 0, stream>>>(film32, film64, target, image_adjoint, pixels,
                                                                precision, pixel_adjoint, loss);
    return cudaGetLastError();
}

cudaError_t launch_queries(const SceneView& s, const bf200_ray_v1* rays, uint64_t n, bf200_hit_v1* hits,
                           uint32_t* occluded, cudaStream_t stream) {
    const uint64_t blocks64 = (n + 127U) / 128U;
    const uint32_t blocks = static_cast<uint32_t>(blocks64 < 65535U ? (blocks64 == 0 ? 1 : blocks64) : 65535U);
    if (hits != nullptr) {
        if (s.sphere_count != 0U) {
            k_query_closest<true><<<blocks, 128, 0, stream>>>(s, rays, n, hits);
        } else {
            k_query_closest<false><<<blocks, 128, 0, stream>>>(s, rays, n, hits);
        }
    } else {
        if (s.sphere_count != 0U) {
            k_query_occlusion<true><<<blocks, 128, 0, stream>>>(s, rays, n, occluded);
        } else {
            k_query_occlusion<false><<<blocks, 128, 0, stream>>>(s, rays, n, occluded);
        }
    }
    return cudaGetLastError();
}

#endif  // BF200_KERNELS_MAIN_TU

}  // namespace bf200
