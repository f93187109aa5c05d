// Environment-map light on the device: batch sample_li, pdf_li and le of EnvironmentMapLightT<float>
// (EnvironmentLights.hpp:750-852, 967-1060) over the tables built on the host (bf200_envmap.cpp).
// Every step is the reference's, in float with its rounding: divisions and square roots are IEEE,
// fma is fmaf, and contraction is off (-fmad=false). Sines, cosines and the arctangent are the
// double-precision values rounded once to float -- the convention of all of the device's trig;
// the reference calls the C library's float functions, which differ by an ulp on a small share of
// angles (the oracle has both conventions).
#include <cuda_runtime.h>

#include <cstdint>

#include "bf200.h"
#include "bf200_envmap.h"
#include "bf200_kernels.h"

namespace bf200 {
namespace {

struct V3 {
    float x, y, z;
};

constexpr uint32_t kEnvMaxInteriorSteps = 24;  // std::numeric_limits<float>::digits

__device__ __forceinline__ float env_midpoint(float a, float b) {
    constexpr float lo = 1.17549435e-38F * 2.0F;  // std::numeric_limits<float>::min() * 2
    constexpr float hi = 3.40282347e+38F / 2.0F;  // std::numeric_limits<float>::max() / 2
    const float abs_a = a < 0.0F ? -a : a, abs_b = b < 0.0F ? -b : b;
    if (abs_a <= hi && abs_b <= hi) {
        return (a + b) / 2.0F;
    }
    if (abs_a < lo) {
        return a + b / 2.0F;
    }
    if (abs_b < lo) {
        return a / 2.0F + b;
    }
    return a / 2.0F + b / 2.0F;
}

__device__ __noinline__ float env_cos(float a) { return static_cast<float>(cos(static_cast<double>(a))); }
__device__ __noinline__ float env_sin(float a) { return static_cast<float>(sin(static_cast<double>(a))); }
__device__ __noinline__ float env_atan2(float y, float x) {
    return static_cast<float>(atan2(static_cast<double>(y), static_cast<double>(x)));
}

// light_detail::unit_direction (Light.hpp:57-64).
__device__ __forceinline__ bool unit_direction(V3 d) {
    const float squared = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
    const float tolerance = 128.0F * 1.1920929e-7F;  // 128 * FLT_EPSILON
    return isfinite(d.x) && isfinite(d.y) && isfinite(d.z) && isfinite(squared) &&
           fabsf(squared - 1.0F) <= tolerance;
}

// robust_unit_direction (:97-121).
__device__ __forceinline__ bool robust_unit(V3 d, V3& out) {
    if (!isfinite(d.x) || !isfinite(d.y) || !isfinite(d.z)) {
        return false;
    }
    const float scale = fmaxf(fmaxf(fabsf(d.x), fabsf(d.y)), fabsf(d.z));
    if (!(scale > 0.0F) || !isfinite(scale)) {
        return false;
    }
    const V3 s{d.x / scale, d.y / scale, d.z / scale};
    const float squared = fmaf(s.x, s.x, fmaf(s.y, s.y, s.z * s.z));
    const float length = sqrtf(squared);
    if (!isfinite(squared) || !(squared > 0.0F) || !isfinite(length) || !(length > 0.0F)) {
        return false;
    }
    out = V3{s.x / length, s.y / length, s.z / length};
    return unit_direction(out);
}

// transform_vector (Transforms.hpp:101-108) with a row-major 3x3.
__device__ __forceinline__ V3 apply3(const float (&m)[9], V3 v) {
    return V3{m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
              m[6] * v.x + m[7] * v.y + m[8] * v.z};
}

// std::upper_bound over an ascending range: the first index whose value is > v.
__device__ __forceinline__ uint32_t upper_ascending(const float* a, uint32_t n, float v) {
    uint32_t lo = 0, count = n;
    while (count > 0) {
        const uint32_t step = count / 2;
        if (!(v < a[lo + step])) {
            lo += step + 1;
            count -= step + 1;
        } else {
            count = step;
        }
    }
    return lo;
}

// std::upper_bound with std::greater over a descending range: the first index whose value is < v.
__device__ __forceinline__ uint32_t upper_descending(const float* a, uint32_t n, float v) {
    uint32_t lo = 0, count = n;
    while (count > 0) {
        const uint32_t step = count / 2;
        if (!(v > a[lo + step])) {
            lo += step + 1;
            count -= step + 1;
        } else {
            count = step;
        }
    }
    return lo;
}

struct Texel {
    uint32_t column, row, index;
};

// direction_texel (:264-314) of a local direction; status on failure.
__device__ uint32_t direction_texel(const EnvironmentView& v, V3 local, Texel& out) {
    V3 d;
    if (!robust_unit(local, d)) {
        return kEnvQueryInvalidDirection;
    }
    const float full = v.azimuth[v.width];
    float azimuth = 0.0F;
    if (d.x != 0.0F || d.z != 0.0F) {  // std::hypot(x, z) != 0
        azimuth = env_atan2(d.z, d.x);
        if (azimuth < 0.0F) {
            azimuth += full;
        }
    }
    if (!isfinite(azimuth) || azimuth < 0.0F) {
        return kEnvQueryNotRepresentable;
    }
    if (!(azimuth < full)) {
        azimuth = 0.0F;
    }
    const uint32_t column_end = upper_ascending(v.azimuth, v.width + 1, azimuth);
    const uint32_t row_end = upper_descending(v.cosine, v.height + 1, d.y);
    if (column_end == 0 || row_end == 0) {
        return kEnvQueryEscaped;
    }
    out.column = min(column_end - 1, v.width - 1);
    out.row = min(row_end - 1, v.height - 1);
    out.index = out.row * v.width + out.column;
    return kEnvQueryOk;
}

// world_direction_texel (:1003-1015).
__device__ __forceinline__ uint32_t world_texel(const EnvironmentView& v, V3 world, Texel& out) {
    V3 n;
    if (!robust_unit(world, n)) {
        return kEnvQueryInvalidDirection;
    }
    return direction_texel(v, apply3(v.inverse, n), out);
}

struct CdfSelection {
    uint32_t index;
    float probability, remapped;
};

// select_cdf_interval (:227-254).
__device__ __forceinline__ bool select_cdf(const float* cdf, uint32_t n, float u, CdfSelection& out) {
    const uint32_t index = upper_ascending(cdf, n, u);
    if (index == n) {
        return false;
    }
    const float previous = index == 0 ? 0.0F : cdf[index - 1];
    const float probability = cdf[index] - previous;
    const float lower = u - previous;
    const float upper = cdf[index] - u;
    const float remapped = lower <= upper ? lower / probability : 1.0F - upper / probability;
    if (!isfinite(probability) || !(probability > 0.0F) || !isfinite(remapped) || !isfinite(lower) || lower < 0.0F ||
        !isfinite(upper) || !(upper > 0.0F) || remapped < 0.0F || !(remapped < 1.0F)) {
        return false;
    }
    out = CdfSelection{index, probability, remapped};
    return true;
}

// sample_local_direction (:1017-1060).
__device__ uint32_t local_direction(const EnvironmentView& v, uint32_t row, uint32_t column, float row_remapped,
                                    float column_remapped, uint32_t row_steps, uint32_t column_steps, V3& out) {
    const float cosine0 = v.cosine[row], cosine1 = v.cosine[row + 1];
    const float cosine_span = cosine0 - cosine1;
    const float cosine_mid = env_midpoint(cosine0, cosine1);
    float cosine = fmaf(-row_remapped, cosine_span, cosine0);
    if (!(cosine < cosine0) || !(cosine > cosine1)) {
        cosine = row_remapped == 0.0F ? cosine_mid
                                      : (cosine >= cosine0 ? nextafterf(cosine0, cosine1) : nextafterf(cosine1, cosine0));
        if (!(cosine < cosine0) || !(cosine > cosine1)) {
            return kEnvQueryNotRepresentable;
        }
    }
    for (uint32_t step = 0; step < row_steps; ++step) {
        const float moved = nextafterf(cosine, cosine_mid);
        if (moved == cosine || !(moved < cosine0) || !(moved > cosine1)) {
            return kEnvQueryNotRepresentable;
        }
        cosine = moved;
    }
    if (!isfinite(cosine) || !(cosine > -1.0F) || !(cosine < 1.0F)) {
        return kEnvQueryNotRepresentable;
    }
    const float radial_squared = (1.0F - cosine) * (1.0F + cosine);
    const float radial = sqrtf(radial_squared);
    if (!isfinite(radial_squared) || !(radial_squared > 0.0F) || !isfinite(radial) || !(radial > 0.0F)) {
        return kEnvQueryNotRepresentable;
    }
    const float azimuth0 = v.azimuth[column], azimuth1 = v.azimuth[column + 1];
    const float azimuth_span = azimuth1 - azimuth0;
    const float azimuth_mid = env_midpoint(azimuth0, azimuth1);
    float azimuth = fmaf(column_remapped, azimuth_span, azimuth0);
    if (!(azimuth > azimuth0) || !(azimuth < azimuth1)) {
        azimuth = column_remapped == 0.0F
                      ? azimuth_mid
                      : (azimuth <= azimuth0 ? nextafterf(azimuth0, azimuth1) : nextafterf(azimuth1, azimuth0));
        if (!(azimuth > azimuth0) || !(azimuth < azimuth1)) {
            return kEnvQueryNotRepresentable;
        }
    }
    for (uint32_t step = 0; step < column_steps; ++step) {
        const float moved = nextafterf(azimuth, azimuth_mid);
        if (moved == azimuth || !(moved > azimuth0) || !(moved < azimuth1)) {
            return kEnvQueryNotRepresentable;
        }
        azimuth = moved;
    }
    if (!isfinite(azimuth) || azimuth < 0.0F || !(azimuth < v.azimuth[v.width])) {
        return kEnvQueryNotRepresentable;
    }
    return robust_unit(V3{radial * env_cos(azimuth), cosine, radial * env_sin(azimuth)}, out)
               ? kEnvQueryOk
               : kEnvQueryNotRepresentable;
}

__global__ void __launch_bounds__(128) k_env_sample(EnvironmentView v, const float2* canonical, uint64_t n,
                                                    bf200_environment_sample_v1* out) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        bf200_environment_sample_v1 r{};
        const float2 u = canonical[i];
        if (!isfinite(u.x) || !isfinite(u.y) || u.x < 0.0F || u.x >= 1.0F || u.y < 0.0F || u.y >= 1.0F) {
            r.status = kEnvQueryInvalidSample;
            out[i] = r;
            continue;
        }
        if (v.black != 0U) {
            out[i] = r;  // no sample
            continue;
        }
        CdfSelection rs, cs;
        if (!select_cdf(v.row_cdf, v.height, u.y, rs) ||
            !select_cdf(v.column_cdfs + static_cast<uint64_t>(rs.index) * v.width, v.width, u.x, cs)) {
            r.status = kEnvQueryEscaped;
            out[i] = r;
            continue;
        }
        const uint32_t index = rs.index * v.width + cs.index;
        uint32_t row_steps = 0, column_steps = 0, status = kEnvQueryUnstable;
        V3 world{};
        for (uint32_t attempt = 0; attempt <= kEnvMaxInteriorSteps * 2; ++attempt) {
            V3 local;
            uint32_t e = local_direction(v, rs.index, cs.index, rs.remapped, cs.remapped, row_steps, column_steps, local);
            if (e != kEnvQueryOk) {
                status = e;
                break;
            }
            if (!robust_unit(apply3(v.matrix, local), world)) {
                status = kEnvQueryNotRepresentable;
                break;
            }
            Texel replayed;
            e = world_texel(v, world, replayed);
            if (e != kEnvQueryOk) {
                status = e;
                break;
            }
            if (replayed.index == index) {
                status = kEnvQueryOk;
                break;
            }
            if (replayed.row != rs.index) {
                if (row_steps == kEnvMaxInteriorSteps) {
                    break;
                }
                ++row_steps;
            }
            if (replayed.column != cs.index) {
                if (column_steps == kEnvMaxInteriorSteps) {
                    break;
                }
                ++column_steps;
            }
        }
        if (status == kEnvQueryOk) {
            const float density = v.density[index];
            const float* t = v.texels + 4ULL * index;
            if (!isfinite(density) || !(density > 0.0F)) {
                status = kEnvQueryNotRepresentable;
            } else {
                r.direction[0] = world.x;
                r.direction[1] = world.y;
                r.direction[2] = world.z;
                for (int lane = 0; lane < 4; ++lane) {
                    r.radiance[lane] = t[lane];
                }
                r.pdf = density;
                r.valid = 1U;
            }
        }
        r.status = status;
        out[i] = r;
    }
}

__global__ void __launch_bounds__(128) k_env_pdf(EnvironmentView v, const float* directions, uint64_t n, float* pdf,
                                                 uint32_t* status) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const V3 d{directions[3 * i], directions[3 * i + 1], directions[3 * i + 2]};
        float value = 0.0F;
        uint32_t e = kEnvQueryOk;
        if (!unit_direction(d)) {
            e = kEnvQueryInvalidDirection;
        } else if (v.black == 0U) {
            Texel t;
            e = world_texel(v, d, t);
            if (e == kEnvQueryOk) {
                value = v.density[t.index];
            }
        }
        pdf[i] = value;
        status[i] = e;
    }
}

__global__ void __launch_bounds__(128) k_env_le(EnvironmentView v, const float* directions, uint64_t n,
                                                float4* radiance, uint32_t* status) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const V3 d{directions[3 * i], directions[3 * i + 1], directions[3 * i + 2]};
        float4 value = make_float4(0.0F, 0.0F, 0.0F, 0.0F);
        Texel t;
        const uint32_t e = world_texel(v, d, t);
        if (e == kEnvQueryOk) {
            const float* p = v.texels + 4ULL * t.index;
            value = make_float4(p[0], p[1], p[2], p[3]);
        }
        radiance[i] = value;
        status[i] = e;
    }
}

uint32_t query_blocks(uint64_t n) {
    const uint64_t blocks = (n + 127U) / 128U;
    return static_cast<uint32_t>(blocks == 0 ? 1 : (blocks < 65535U ? blocks : 65535U));
}

}  // namespace

cudaError_t launch_environment_sample(const EnvironmentView& v, const float2* canonical, uint64_t n,
                                      bf200_environment_sample_v1* out, cudaStream_t stream) {
    k_env_sample<<<query_blocks(n), 128, 0, stream>>>(v, canonical, n, out);
    return cudaGetLastError();
}

cudaError_t launch_environment_pdf(const EnvironmentView& v, const float* directions, uint64_t n, float* pdf,
                                   uint32_t* status, cudaStream_t stream) {
    k_env_pdf<<<query_blocks(n), 128, 0, stream>>>(v, directions, n, pdf, status);
    return cudaGetLastError();
}

cudaError_t launch_environment_le(const EnvironmentView& v, const float* directions, uint64_t n, float4* radiance,
                                  uint32_t* status, cudaStream_t stream) {
    k_env_le<<<query_blocks(n), 128, 0, stream>>>(v, directions, n, radiance, status);
    return cudaGetLastError();
}

}  // namespace bf200
