// Spatial light-tree selection on the device: the traversal of LightSampler::sample(context, u)
// (Blackframe/Renderer/Source/LightSampler.cpp:953-1129) over the node array that
// build_light_tree (bf200_light_tree.cpp) lays out, one query per thread.
//
// The arithmetic and its order are the host restatement's. The logarithms and exponentials are
// the double-precision values rounded once to float; the C library's logf/expf/log1pf are within
// about an ulp of those, so a probability can differ from the host's in its last bits (and a
// selection only when the sample lies on that bit of a branch boundary). The three-argument
// hypotenuse is a * sqrt((x/a)^2 + (y/a)^2 + (z/a)^2) with a = max(|x|, |y|, |z|), the formula the
// host's std::hypot(float, float, float) evaluates (identical on 2,000,000 random inputs).
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "bf200.h"
#include "bf200_light_tree.h"

namespace bf200 {
namespace {

struct DScaled {
    float mantissa;
    int exponent;
};

__device__ __forceinline__ float d_logf(float x) { return static_cast<float>(log(static_cast<double>(x))); }
__device__ __forceinline__ float d_expf(float x) { return static_cast<float>(exp(static_cast<double>(x))); }
__device__ __forceinline__ float d_log1pf(float x) { return static_cast<float>(log1p(static_cast<double>(x))); }

__device__ bool d_unbounded(const LightTreeNode& n) {
    const float inf = __int_as_float(0x7f800000);
    return n.lo[0] == -inf && n.lo[1] == -inf && n.lo[2] == -inf && n.hi[0] == inf && n.hi[1] == inf &&
           n.hi[2] == inf;
}

__device__ bool d_finite(const LightTreeNode& n) {
    return isfinite(n.lo[0]) && isfinite(n.lo[1]) && isfinite(n.lo[2]) && isfinite(n.hi[0]) && isfinite(n.hi[1]) &&
           isfinite(n.hi[2]);
}

// scaled_positive_difference
__device__ bool d_scaled_difference(float upper, float lower, DScaled& out) {
    if (!isfinite(upper) || !isfinite(lower) || upper < lower) {
        return false;
    }
    int ue = 0, le = 0;
    static_cast<void>(frexpf(fabsf(upper), &ue));
    static_cast<void>(frexpf(fabsf(lower), &le));
    const int scale = ue > le ? ue : le;
    const float difference = scalbnf(upper, -scale) - scalbnf(lower, -scale);
    if (!isfinite(difference) || difference < 0.0F) {
        return false;
    }
    if (difference == 0.0F) {
        out = DScaled{0.0F, 0};
        return true;
    }
    int normalized = 0;
    const float mantissa = frexpf(difference, &normalized);
    if (!isfinite(mantissa) || !(mantissa > 0.0F)) {
        return false;
    }
    out = DScaled{mantissa, scale + normalized};
    return true;
}

__device__ bool d_scaled_less(DScaled l, DScaled r) {
    if (l.mantissa == 0.0F) {
        return r.mantissa > 0.0F;
    }
    if (r.mantissa == 0.0F) {
        return false;
    }
    return l.exponent != r.exponent ? l.exponent < r.exponent : l.mantissa < r.mantissa;
}

__device__ float d_hypot3(float x, float y, float z) {
    x = fabsf(x);
    y = fabsf(y);
    z = fabsf(z);
    const float a = x < y ? (y < z ? z : y) : (x < z ? z : x);
    if (a == 0.0F) {
        return 0.0F;
    }
    const float xa = x / a, ya = y / a, za = z / a;
    return a * sqrtf(xa * xa + ya * ya + za * za);
}

__device__ float d_scaled_log(DScaled v) {
    return d_logf(v.mantissa) + static_cast<float>(v.exponent) * d_logf(2.0F);
}

// log_distance_attenuation
__device__ bool d_log_attenuation(const LightTreeNode& n, const float* p, float root_log, bool root_has, float& out) {
    out = 0.0F;
    if (d_unbounded(n) || !root_has) {
        return true;
    }
    if (!d_finite(n) || !isfinite(root_log)) {
        return false;
    }
    DScaled axis[3];
    for (int a = 0; a < 3; ++a) {
        axis[a] = DScaled{0.0F, 0};
        if (p[a] < n.lo[a]) {
            if (!d_scaled_difference(n.lo[a], p[a], axis[a])) {
                return false;
            }
        } else if (p[a] > n.hi[a]) {
            if (!d_scaled_difference(p[a], n.hi[a], axis[a])) {
                return false;
            }
        }
    }
    DScaled maximum = axis[0];
    if (d_scaled_less(maximum, axis[1])) {
        maximum = axis[1];
    }
    if (d_scaled_less(maximum, axis[2])) {
        maximum = axis[2];
    }
    if (maximum.mantissa == 0.0F) {
        return true;
    }
    float c[3];
    for (int a = 0; a < 3; ++a) {
        c[a] = axis[a].mantissa == 0.0F ? 0.0F : scalbnf(axis[a].mantissa, axis[a].exponent - maximum.exponent);
    }
    const float hypotenuse = d_hypot3(c[0], c[1], c[2]);
    if (!isfinite(hypotenuse) || !(hypotenuse > 0.0F)) {
        return false;
    }
    int normalized = 0;
    const float mantissa = frexpf(hypotenuse, &normalized);
    const float log_distance = d_scaled_log(DScaled{mantissa, maximum.exponent + normalized}) - root_log;
    if (!isfinite(log_distance)) {
        return false;
    }
    float attenuation;
    if (log_distance <= 0.0F) {
        const float normalized_distance = d_expf(log_distance);
        attenuation = -d_log1pf(normalized_distance * normalized_distance);
    } else {
        const float inverse_squared = d_expf(-2.0F * log_distance);
        attenuation = -2.0F * log_distance - d_log1pf(inverse_squared);
    }
    if (!isfinite(attenuation) || attenuation > 0.0F) {
        return false;
    }
    out = attenuation;
    return true;
}

// tree_left_probability
__device__ bool d_left_probability(const LightTreeNode* nodes, uint32_t count, const float* p, uint32_t index,
                                   float root_log, bool root_has, float& out) {
    if (index >= count) {
        return false;
    }
    const LightTreeNode node = nodes[index];
    if (node.kind != kLightTreeInternal || node.left >= count || node.right >= count) {
        return false;
    }
    float score[2];
    const uint32_t children[2] = {node.left, node.right};
    for (int c = 0; c < 2; ++c) {
        const LightTreeNode child = nodes[children[c]];
        if (!isfinite(child.power) || !(child.power > 0.0F)) {
            return false;
        }
        float attenuation = 0.0F;
        if (!d_log_attenuation(child, p, root_log, root_has, attenuation)) {
            return false;
        }
        score[c] = d_logf(child.power) + attenuation;
        if (!isfinite(score[c])) {
            return false;
        }
    }
    float left;
    if (score[0] <= score[1]) {
        const float ratio = d_expf(score[0] - score[1]);
        if (!isfinite(ratio) || !(ratio > 0.0F)) {
            return false;
        }
        left = ratio / (1.0F + ratio);
    } else {
        const float ratio = d_expf(score[1] - score[0]);
        if (!isfinite(ratio) || !(ratio > 0.0F)) {
            return false;
        }
        left = 1.0F - ratio / (1.0F + ratio);
    }
    const float right = 1.0F - left;
    if (!isfinite(left) || !(left > 0.0F) || !(left < 1.0F) || !isfinite(right) || !(right > 0.0F) || !(right < 1.0F)) {
        return false;
    }
    out = left;
    return true;
}

// LightSampler::sample(context, u); a refused query writes 0xFFFFFFFF and -1
__global__ void k_light_tree_select(const LightTreeNode* nodes, uint32_t node_count, uint32_t root,
                                    uint32_t light_count, float root_log, int root_has, const float* positions,
                                    const float* samples, uint64_t query_count, uint32_t* lights,
                                    float* probabilities) {
    const uint64_t q = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= query_count) {
        return;
    }
    const float p[3] = {positions[3 * q], positions[3 * q + 1], positions[3 * q + 2]};
    const float u = samples[q];
    lights[q] = kLightTreeInvalid;
    probabilities[q] = -1.0F;
    if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2]) || !isfinite(u) || u < 0.0F || !(u < 1.0F) ||
        root >= node_count) {
        return;
    }
    uint32_t index = root;
    float remapped = u, selection = 1.0F;
    for (uint32_t depth = 0; depth < 64U && nodes[index].kind == kLightTreeInternal; ++depth) {
        float left = 0.0F;
        if (!d_left_probability(nodes, node_count, p, index, root_log, root_has != 0, left)) {
            return;
        }
        const bool go_left = remapped < left;
        const float branch = go_left ? left : 1.0F - left;
        const float product = selection * branch;
        if (!isfinite(product) || !(product > 0.0F) || product > 1.0F) {
            return;
        }
        // remap_canonical_sample
        const float begin = go_left ? 0.0F : left;
        const float end = begin + branch;
        const float from_begin = remapped - begin;
        const float to_end = end - remapped;
        if (!isfinite(end) || from_begin < 0.0F || !(to_end > 0.0F)) {
            return;
        }
        const float next = from_begin <= to_end ? from_begin / branch : 1.0F - to_end / branch;
        if (!isfinite(next) || next < 0.0F || !(next < 1.0F)) {
            return;
        }
        selection = product;
        remapped = next;
        index = go_left ? nodes[index].left : nodes[index].right;
        if (index >= node_count) {
            return;
        }
    }
    const LightTreeNode leaf = nodes[index];
    if (leaf.kind == kLightTreeInternal || leaf.light >= light_count || !(selection > 0.0F) || selection > 1.0F) {
        return;
    }
    lights[q] = leaf.light;
    probabilities[q] = selection;
}

}  // namespace
}  // namespace bf200

extern "C" {

BF200_EXPORT blackframe_status bf200_light_tree_select_device(const bf200_light_tree_input_v1* lights,
                                                              uint32_t light_count, const float* device_positions,
                                                              const float* device_samples, uint64_t query_count,
                                                              uint32_t* device_light_indices,
                                                              float* device_probabilities) noexcept {
    if (lights == nullptr || (query_count != 0 && (device_positions == nullptr || device_samples == nullptr ||
                                                   device_light_indices == nullptr ||
                                                   device_probabilities == nullptr))) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    try {
        bf200::LightTree tree;
        std::string error;
        if (const auto st = bf200::build_light_tree(lights, light_count, tree, error); st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        if (query_count == 0) {
            return BLACKFRAME_STATUS_SUCCESS;
        }
        bf200::LightTreeNode* nodes = nullptr;
        const size_t bytes = tree.nodes.size() * sizeof(bf200::LightTreeNode);
        cudaError_t e = cudaMalloc(&nodes, bytes);
        if (e == cudaSuccess) {
            e = cudaMemcpy(nodes, tree.nodes.data(), bytes, cudaMemcpyHostToDevice);
        }
        const uint64_t blocks = (query_count + 255) / 256;
        if (blocks > 0x7FFFFFFFULL) {
            cudaFree(nodes);
            return BLACKFRAME_STATUS_OUT_OF_RANGE;
        }
        if (e == cudaSuccess) {
            bf200::k_light_tree_select<<<static_cast<unsigned>(blocks), 256>>>(
                nodes, static_cast<uint32_t>(tree.nodes.size()), tree.root, light_count, tree.root_log_extent,
                tree.root_has_extent ? 1 : 0, device_positions, device_samples, query_count, device_light_indices,
                device_probabilities);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) {
            e = cudaDeviceSynchronize();
        }
        if (nodes != nullptr) {
            cudaFree(nodes);
        }
        return e == cudaSuccess ? BLACKFRAME_STATUS_SUCCESS : BLACKFRAME_STATUS_EXTENSION_FAILURE;
    } catch (const std::bad_alloc&) {
        return BLACKFRAME_STATUS_OUT_OF_RANGE;
    }
}

}  // extern "C"
