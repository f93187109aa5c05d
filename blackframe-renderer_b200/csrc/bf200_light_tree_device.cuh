// Spatial light-tree traversal on the device, shared by the query kernel (bf200_light_tree.cu) and
// the transport's tree-selecting shading kernels (bf200_kernels.cu): LightSampler's
// tree_left_probability, sample(context, u) and probability(context, i)
// (Blackframe/Renderer/Source/LightSampler.cpp:953-1225) over the node array build_light_tree lays
// out. The arithmetic and its order are the host restatement's (bf200_light_tree.cpp); logarithms
// and exponentials are the double-precision values rounded once to float, within about an ulp of
// the C library's float functions; the three-argument hypotenuse is the host library's formula.
#pragma once

#include <cstdint>

#include "bf200_light_tree.h"

namespace bf200 {

struct DScaled {
    float mantissa;
    int exponent;
};

__device__ __forceinline__ float d_logf(float x) { return static_cast<float>(log(static_cast<double>(x))); }
__device__ __forceinline__ float d_expf(float x) { return static_cast<float>(exp(static_cast<double>(x))); }
__device__ __forceinline__ float d_log1pf(float x) { return static_cast<float>(log1p(static_cast<double>(x))); }

__device__ __forceinline__ bool d_unbounded(const LightTreeNode& n) {
    const float inf = __int_as_float(0x7f800000);
    return n.lo[0] == -inf && n.lo[1] == -inf && n.lo[2] == -inf && n.hi[0] == inf && n.hi[1] == inf &&
           n.hi[2] == inf;
}

__device__ __forceinline__ bool d_finite(const LightTreeNode& n) {
    return isfinite(n.lo[0]) && isfinite(n.lo[1]) && isfinite(n.lo[2]) && isfinite(n.hi[0]) && isfinite(n.hi[1]) &&
           isfinite(n.hi[2]);
}

// scaled_positive_difference
static __device__ bool d_scaled_difference(float upper, float lower, DScaled& out) {
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

static __device__ bool d_scaled_less(DScaled l, DScaled r) {
    if (l.mantissa == 0.0F) {
        return r.mantissa > 0.0F;
    }
    if (r.mantissa == 0.0F) {
        return false;
    }
    return l.exponent != r.exponent ? l.exponent < r.exponent : l.mantissa < r.mantissa;
}

static __device__ float d_hypot3(float x, float y, float z) {
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

static __device__ float d_scaled_log(DScaled v) {
    return d_logf(v.mantissa) + static_cast<float>(v.exponent) * d_logf(2.0F);
}

// log_distance_attenuation
static __device__ bool d_log_attenuation(const LightTreeNode& n, const float* p, float root_log, bool root_has, float& out) {
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
static __device__ bool d_left_probability(const LightTreeNode* nodes, uint32_t count, const float* p, uint32_t index,
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

// sample(context, u): the selected light slot and its probability; false where the reference
// refuses the query
static __device__ bool d_tree_select(const LightTreeNode* nodes, uint32_t node_count, uint32_t root,
                                     uint32_t light_count, float root_log, bool root_has, const float* p, float u,
                                     uint32_t& light, float& probability) {
    if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2]) || !isfinite(u) || u < 0.0F || !(u < 1.0F) ||
        root >= node_count) {
        return false;
    }
    uint32_t index = root;
    float remapped = u, selection = 1.0F;
    for (uint32_t depth = 0; depth < 64U && nodes[index].kind == kLightTreeInternal; ++depth) {
        float left = 0.0F;
        if (!d_left_probability(nodes, node_count, p, index, root_log, root_has, left)) {
            return false;
        }
        const bool go_left = remapped < left;
        const float branch = go_left ? left : 1.0F - left;
        const float product = selection * branch;
        if (!isfinite(product) || !(product > 0.0F) || product > 1.0F) {
            return false;
        }
        // remap_canonical_sample
        const float begin = go_left ? 0.0F : left;
        const float end = begin + branch;
        const float from_begin = remapped - begin;
        const float to_end = end - remapped;
        if (!isfinite(end) || from_begin < 0.0F || !(to_end > 0.0F)) {
            return false;
        }
        const float next = from_begin <= to_end ? from_begin / branch : 1.0F - to_end / branch;
        if (!isfinite(next) || next < 0.0F || !(next < 1.0F)) {
            return false;
        }
        selection = product;
        remapped = next;
        index = go_left ? nodes[index].left : nodes[index].right;
        if (index >= node_count) {
            return false;
        }
    }
    const LightTreeNode leaf = nodes[index];
    if (leaf.kind == kLightTreeInternal || leaf.light >= light_count || !(selection > 0.0F) || selection > 1.0F) {
        return false;
    }
    light = leaf.light;
    probability = selection;
    return true;
}

// probability(context, i) of a supported light: the product of the branch probabilities on its
// leaf-to-root path, taken from the root down
static __device__ bool d_tree_probability(const LightTreeNode* nodes, uint32_t node_count, uint32_t root,
                                          const uint32_t* light_to_node, uint32_t light_count, float root_log,
                                          bool root_has, const float* p, uint32_t light, float& probability) {
    if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2]) || light >= light_count || root >= node_count) {
        return false;
    }
    uint32_t index = light_to_node[light];
    if (index == kLightTreeInvalid) {  // a zero-power slot: no support (the CDF's zero width)
        probability = 0.0F;
        return true;
    }
    if (index >= node_count || nodes[index].light != light) {
        return false;
    }
    uint32_t parents[64];
    bool chose_left[64];
    uint32_t length = 0;
    while (index != root) {
        if (length == 64U) {
            return false;
        }
        const uint32_t parent = nodes[index].parent;
        if (parent >= node_count || nodes[parent].kind != kLightTreeInternal) {
            return false;
        }
        const bool left = nodes[parent].left == index;
        if (!left && nodes[parent].right != index) {
            return false;
        }
        parents[length] = parent;
        chose_left[length] = left;
        ++length;
        index = parent;
    }
    float selection = 1.0F;
    for (uint32_t k = length; k > 0U; --k) {
        float left = 0.0F;
        if (!d_left_probability(nodes, node_count, p, parents[k - 1U], root_log, root_has, left)) {
            return false;
        }
        const float product = selection * (chose_left[k - 1U] ? left : 1.0F - left);
        if (!isfinite(product) || !(product > 0.0F) || product > 1.0F) {
            return false;
        }
        selection = product;
    }
    probability = selection;
    return true;
}

}  // namespace bf200
