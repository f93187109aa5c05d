// Spatial light tree: LightSampler::create_spatial_tree and its context selection
// (Blackframe/Renderer/Source/LightSampler.cpp:256-535, 626-1226) restated on the host.
//
// The tree is a deterministic median tree over the lights' bound centroids: a node's lights are
// sorted along the axis of largest centroid extent (ties by registry slot) and split at the
// middle; lights with the canonical unbounded box form a second subtree in slot order, and a root
// joins the two when both exist. At a query point a child's score is log(power) plus the log of
// 1 / (1 + (d / s)^2), d the distance to its box and s the finite root's largest extent, and the
// left probability is the normalised exponent of the score difference. Every arithmetic step,
// its order and its failure checks follow the reference (float arithmetic, the C library's
// logf/expf/log1pf/hypot), so selections and probabilities are the reference's bit for bit.
#include "bf200_light_tree.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

namespace bf200 {

// ------------------------------------------------------------------------------------------------
// Power-weighted light selection (LightSampler::create_power_weighted,
// Blackframe/Renderer/Source/LightSampler.cpp:605-625 with power_weights :200-245 and
// build_power_cdf :117-190). The steps and their float order are kept alike: the boundaries must be
// the reference's, bit for bit, or selections and their probabilities would differ.
// ------------------------------------------------------------------------------------------------

// Neumaier step (add_compensated :78-95): false for a negative or non-finite value or sum.
static bool compensated_add(float value, float& sum, float& correction) {
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

// The selection CDF (light_count + 1 boundaries) of four-lane spectral powers in registry order.
static blackframe_status power_cdf(const float* powers, uint32_t count, std::vector<float>& cdf, std::string& error,
                                   std::vector<float>* weights_out) {
    if (count == 0) {
        error = "Light sampling requires at least one registry slot.";
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    float peak = 0.0F;
    for (uint64_t i = 0; i < 4ULL * count; ++i) {
        if (!std::isfinite(powers[i]) || powers[i] < 0.0F) {
            error = "Power-weighted light sampling requires finite non-negative spectral lanes.";
            return BLACKFRAME_STATUS_INVALID_ARGUMENT;
        }
        peak = std::max(peak, powers[i]);
    }
    if (peak == 0.0F) {
        error = "Power-weighted light sampling requires positive spectral power.";
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    std::vector<float> weights(count);
    for (uint32_t i = 0; i < count; ++i) {
        float sum = 0.0F, correction = 0.0F;
        bool positive = false;
        for (int l = 0; l < 4; ++l) {
            const float lane = powers[4ULL * i + l];
            const float ratio = lane / peak;
            if (lane > 0.0F) {
                positive = true;
                if (!(ratio > 0.0F)) {
                    error = "A positive spectral power lane is not representable after scaling.";
                    return BLACKFRAME_STATUS_OUT_OF_RANGE;
                }
            }
            if (!compensated_add(ratio, sum, correction)) {
                error = "A spectral light-selection weight is not representable.";
                return BLACKFRAME_STATUS_OUT_OF_RANGE;
            }
        }
        const float weight = sum + correction;
        if (!std::isfinite(weight) || weight < 0.0F || (positive && !(weight > 0.0F))) {
            error = "A spectral light-selection weight is not representable.";
            return BLACKFRAME_STATUS_OUT_OF_RANGE;
        }
        weights[i] = weight == 0.0F ? 0.0F : weight;
    }
    float total_sum = 0.0F, total_correction = 0.0F;
    for (float w : weights) {
        if (!compensated_add(w, total_sum, total_correction)) {
            error = "Light-selection power accumulation is not representable.";
            return BLACKFRAME_STATUS_OUT_OF_RANGE;
        }
    }
    float total = total_sum + total_correction;
    if (!std::isfinite(total) || total < 0.0F) {
        error = "Light-selection power accumulation is not representable.";
        return BLACKFRAME_STATUS_OUT_OF_RANGE;
    }
    total = total == 0.0F ? 0.0F : total;
    if (total == 0.0F) {
        error = "Power-weighted light sampling requires positive spectral power.";
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    uint32_t last_positive = count;
    for (uint32_t i = count; i > 0; --i) {
        if (weights[i - 1] > 0.0F) {
            last_positive = i - 1;
            break;
        }
    }
    cdf.assign(count + 1ULL, 0.0F);
    float prefix_sum = 0.0F, prefix_correction = 0.0F, previous = 0.0F;
    for (uint32_t i = 0; i < count; ++i) {
        const float weight = weights[i];
        if (weight == 0.0F) {
            cdf[i + 1ULL] = previous;
            continue;
        }
        if (!compensated_add(weight, prefix_sum, prefix_correction)) {
            error = "Light-selection power prefix is not representable.";
            return BLACKFRAME_STATUS_OUT_OF_RANGE;
        }
        const float prefix = prefix_sum + prefix_correction;
        if (!std::isfinite(prefix) || !(prefix > 0.0F)) {
            error = "Light-selection power prefix is not representable.";
            return BLACKFRAME_STATUS_OUT_OF_RANGE;
        }
        float boundary = 1.0F;
        if (i != last_positive) {
            boundary = prefix / total;
            if (!std::isfinite(boundary) || !(boundary > previous) || !(boundary < 1.0F)) {
                error = "A positive light-selection probability is not representable.";
                return BLACKFRAME_STATUS_OUT_OF_RANGE;
            }
        } else {
            const float nominal = weight / total;
            const float candidate = previous + nominal;
            if (!std::isfinite(nominal) || !(nominal > 0.0F) || !std::isfinite(candidate) || !(candidate > previous)) {
                error = "The terminal positive light-selection probability is not representable.";
                return BLACKFRAME_STATUS_OUT_OF_RANGE;
            }
        }
        cdf[i + 1ULL] = boundary;
        previous = boundary;
    }
    if (cdf[count] != 1.0F) {
        error = "Light-selection CDF does not terminate at one.";
        return BLACKFRAME_STATUS_EXTENSION_FAILURE;
    }
    for (uint32_t i = 0; i < count; ++i) {
        const float probability = cdf[i + 1ULL] - cdf[i];
        if (!std::isfinite(probability) || probability < 0.0F || ((weights[i] > 0.0F) != (probability > 0.0F))) {
            error = "Light-selection CDF lost or created probability support.";
            return BLACKFRAME_STATUS_OUT_OF_RANGE;
        }
    }
    if (weights_out != nullptr) {
        *weights_out = std::move(weights);
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

blackframe_status light_power_cdf(const float* powers, uint32_t count, std::vector<float>& cdf, std::string& error) {
    return power_cdf(powers, count, cdf, error, nullptr);
}

blackframe_status light_power_weights(const float* powers, uint32_t count, std::vector<float>& weights,
                                      std::vector<float>& cdf, std::string& error) {
    return power_cdf(powers, count, cdf, error, &weights);
}

namespace {

constexpr float kInfinity = std::numeric_limits<float>::infinity();

struct Box {
    float lo[3];
    float hi[3];
};

struct Scaled {  // mantissa in [0.5, 1) times 2^exponent; mantissa 0 is zero
    float mantissa = 0.0F;
    int exponent = 0;
};

blackframe_status invalid(std::string& error, const char* message) {
    error = message;
    return BLACKFRAME_STATUS_INVALID_ARGUMENT;
}
blackframe_status exhausted(std::string& error, const char* message) {
    error = message;
    return BLACKFRAME_STATUS_OUT_OF_RANGE;
}
blackframe_status inconsistent(std::string& error, const char* message) {
    error = message;
    return BLACKFRAME_STATUS_EXTENSION_FAILURE;
}

bool finite_box(const Box& b) {
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(b.lo[a]) || !std::isfinite(b.hi[a])) {
            return false;
        }
    }
    return true;
}

bool unbounded_box(const Box& b) {
    for (int a = 0; a < 3; ++a) {
        if (b.lo[a] != -kInfinity || b.hi[a] != kInfinity) {
            return false;
        }
    }
    return true;
}

// The correctly rounded midpoint of two floats (the rule std::midpoint specifies).
float midpoint(float a, float b) {
    const float low = std::numeric_limits<float>::min() * 2.0F;
    const float high = std::numeric_limits<float>::max() / 2.0F;
    const float abs_a = a < 0.0F ? -a : a;
    const float abs_b = b < 0.0F ? -b : b;
    if (abs_a <= high && abs_b <= high) {
        return (a + b) / 2.0F;
    }
    if (abs_a < low) {
        return a + b / 2.0F;
    }
    if (abs_b < low) {
        return a / 2.0F + b;
    }
    return a / 2.0F + b / 2.0F;
}

Box merged(const Box& l, const Box& r) {
    if (unbounded_box(l) || unbounded_box(r)) {
        return Box{{-kInfinity, -kInfinity, -kInfinity}, {kInfinity, kInfinity, kInfinity}};
    }
    Box m;
    for (int a = 0; a < 3; ++a) {
        m.lo[a] = std::min(l.lo[a], r.lo[a]);
        m.hi[a] = std::max(l.hi[a], r.hi[a]);
    }
    return m;
}

// scaled_positive_difference (LightSampler.cpp:308-340)
blackframe_status scaled_difference(float upper, float lower, Scaled& out, std::string& error) {
    if (!std::isfinite(upper) || !std::isfinite(lower) || upper < lower) {
        return inconsistent(error, "Light-tree scaled difference requires finite ordered values.");
    }
    int upper_exponent = 0, lower_exponent = 0;
    static_cast<void>(std::frexp(std::abs(upper), &upper_exponent));
    static_cast<void>(std::frexp(std::abs(lower), &lower_exponent));
    const int scale = std::max(upper_exponent, lower_exponent);
    const float difference = std::scalbn(upper, -scale) - std::scalbn(lower, -scale);
    if (!std::isfinite(difference) || difference < 0.0F) {
        return exhausted(error, "Light-tree coordinate difference is not representable after scaling.");
    }
    if (difference == 0.0F) {
        out = Scaled{};
        return BLACKFRAME_STATUS_SUCCESS;
    }
    int normalized = 0;
    const float mantissa = std::frexp(difference, &normalized);
    if (!std::isfinite(mantissa) || !(mantissa > 0.0F)) {
        return exhausted(error, "Light-tree coordinate difference is not representable after scaling.");
    }
    out = Scaled{mantissa, scale + normalized};
    return BLACKFRAME_STATUS_SUCCESS;
}

bool scaled_less(const Scaled& l, const Scaled& r) {
    if (l.mantissa == 0.0F) {
        return r.mantissa > 0.0F;
    }
    if (r.mantissa == 0.0F) {
        return false;
    }
    return l.exponent != r.exponent ? l.exponent < r.exponent : l.mantissa < r.mantissa;
}

// scaled_distance (LightSampler.cpp:355-412): distance from `p` to the box, as a Scaled value
blackframe_status scaled_distance(const Box& b, const float (&p)[3], Scaled& out, std::string& error) {
    Scaled axis[3];
    for (int a = 0; a < 3; ++a) {
        blackframe_status st = BLACKFRAME_STATUS_SUCCESS;
        if (p[a] < b.lo[a]) {
            st = scaled_difference(b.lo[a], p[a], axis[a], error);
        } else if (p[a] > b.hi[a]) {
            st = scaled_difference(p[a], b.hi[a], axis[a], error);
        }
        if (st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
    }
    Scaled maximum = axis[0];
    if (scaled_less(maximum, axis[1])) {
        maximum = axis[1];
    }
    if (scaled_less(maximum, axis[2])) {
        maximum = axis[2];
    }
    if (maximum.mantissa == 0.0F) {
        out = maximum;
        return BLACKFRAME_STATUS_SUCCESS;
    }
    float component[3];
    for (int a = 0; a < 3; ++a) {
        component[a] = axis[a].mantissa == 0.0F ? 0.0F : std::scalbn(axis[a].mantissa, axis[a].exponent - maximum.exponent);
    }
    const float hypotenuse = std::hypot(component[0], component[1], component[2]);
    if (!std::isfinite(hypotenuse) || !(hypotenuse > 0.0F)) {
        return exhausted(error, "Light-tree query distance is not representable after scaling.");
    }
    int normalized = 0;
    const float mantissa = std::frexp(hypotenuse, &normalized);
    out = Scaled{mantissa, maximum.exponent + normalized};
    return BLACKFRAME_STATUS_SUCCESS;
}

float scaled_log(const Scaled& v) {
    return std::log(v.mantissa) + static_cast<float>(v.exponent) * std::log(2.0F);
}

// log_distance_attenuation (LightSampler.cpp:456-493): log of 1 / (1 + (d / s)^2)
blackframe_status log_attenuation(const Box& b, const float (&p)[3], float root_log, bool root_has, float& out,
                                  std::string& error) {
    out = 0.0F;
    if (unbounded_box(b) || !root_has) {
        return BLACKFRAME_STATUS_SUCCESS;
    }
    if (!finite_box(b) || !std::isfinite(root_log)) {
        return inconsistent(error, "Light-tree spatial attenuation received inconsistent finite bounds.");
    }
    Scaled distance;
    if (const auto st = scaled_distance(b, p, distance, error); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    if (distance.mantissa == 0.0F) {
        return BLACKFRAME_STATUS_SUCCESS;
    }
    const float log_distance = scaled_log(distance) - root_log;
    if (!std::isfinite(log_distance)) {
        return exhausted(error, "Light-tree normalized log-distance is not representable.");
    }
    float attenuation = 0.0F;
    if (log_distance <= 0.0F) {
        const float normalized = std::exp(log_distance);
        attenuation = -std::log1p(normalized * normalized);
    } else {
        const float inverse_squared = std::exp(-2.0F * log_distance);
        attenuation = -2.0F * log_distance - std::log1p(inverse_squared);
    }
    if (!std::isfinite(attenuation) || attenuation > 0.0F) {
        return exhausted(error, "Light-tree logarithmic attenuation is not representable.");
    }
    out = attenuation;
    return BLACKFRAME_STATUS_SUCCESS;
}

blackframe_status multiply_probability(float accumulated, float branch, float& out, std::string& error) {
    out = accumulated * branch;
    if (!std::isfinite(out) || !(out > 0.0F) || out > 1.0F) {
        return exhausted(error, "Light-tree traversal lost positive selection probability.");
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

// remap_canonical_sample (LightSampler.cpp:506-531)
blackframe_status remap(float u, float begin, float probability, float& out, std::string& error) {
    const float end = begin + probability;
    const float from_begin = u - begin;
    const float to_end = end - u;
    if (!std::isfinite(end) || from_begin < 0.0F || !(to_end > 0.0F)) {
        return inconsistent(error, "Light-tree traversal could not remap its canonical sample.");
    }
    out = from_begin <= to_end ? from_begin / probability : 1.0F - to_end / probability;
    if (!std::isfinite(out) || out < 0.0F || !(out < 1.0F)) {
        return inconsistent(error, "Light-tree canonical remap is not representable without clamping.");
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

Box node_box(const LightTreeNode& n) {
    return Box{{n.lo[0], n.lo[1], n.lo[2]}, {n.hi[0], n.hi[1], n.hi[2]}};
}

// tree_left_probability (LightSampler.cpp:953-1019)
blackframe_status left_probability(const LightTree& t, const float (&p)[3], uint32_t index, float& out,
                                   std::string& error) {
    if (index >= t.nodes.size()) {
        return inconsistent(error, "Light-tree traversal reached an invalid node index.");
    }
    const LightTreeNode& node = t.nodes[index];
    if (node.kind != kLightTreeInternal || node.left >= t.nodes.size() || node.right >= t.nodes.size()) {
        return inconsistent(error, "Light-tree traversal reached an invalid branch.");
    }
    float score[2];
    const uint32_t children[2] = {node.left, node.right};
    for (int c = 0; c < 2; ++c) {
        const LightTreeNode& child = t.nodes[children[c]];
        if (!std::isfinite(child.power) || !(child.power > 0.0F)) {
            return inconsistent(error, "Light-tree branch contains invalid aggregate power.");
        }
        float attenuation = 0.0F;
        if (const auto st = log_attenuation(node_box(child), p, t.root_log_extent, t.root_has_extent, attenuation,
                                            error);
            st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        score[c] = std::log(child.power) + attenuation;
        if (!std::isfinite(score[c])) {
            return exhausted(error, "Light-tree log-importance is not representable.");
        }
    }
    float left = 0.0F;
    if (score[0] <= score[1]) {
        const float ratio = std::exp(score[0] - score[1]);
        if (!std::isfinite(ratio) || !(ratio > 0.0F)) {
            return exhausted(error, "Light-tree branch normalization lost positive support.");
        }
        left = ratio / (1.0F + ratio);
    } else {
        const float ratio = std::exp(score[1] - score[0]);
        if (!std::isfinite(ratio) || !(ratio > 0.0F)) {
            return exhausted(error, "Light-tree branch normalization lost positive support.");
        }
        left = 1.0F - ratio / (1.0F + ratio);
    }
    const float right = 1.0F - left;
    if (!std::isfinite(left) || !(left > 0.0F) || !(left < 1.0F) || !std::isfinite(right) || !(right > 0.0F) ||
        !(right < 1.0F)) {
        return exhausted(error, "Light-tree branch probability is not representable.");
    }
    out = left;
    return BLACKFRAME_STATUS_SUCCESS;
}

struct Entry {
    Box box;
    float centroid[3];
    float power;
    uint32_t light;
};

struct Builder {
    LightTree& tree;
    std::string& error;

    // build_subtree (LightSampler.cpp:740-861): the node index of entries [begin, end)
    blackframe_status build(std::vector<Entry>& entries, size_t begin, size_t end, bool spatial, uint32_t parent,
                            uint32_t depth, uint32_t& index) {
        if (begin >= end) {
            return inconsistent(error, "Light-tree construction received an empty supported range.");
        }
        if (tree.nodes.size() >= kLightTreeInvalid) {
            return exhausted(error, "Light-tree node indices exceed the stable 32-bit domain.");
        }
        index = static_cast<uint32_t>(tree.nodes.size());
        if (end - begin == 1) {
            const Entry& e = entries[begin];
            LightTreeNode leaf{};
            std::copy(e.box.lo, e.box.lo + 3, leaf.lo);
            std::copy(e.box.hi, e.box.hi + 3, leaf.hi);
            leaf.power = e.power;
            leaf.parent = parent;
            leaf.left = leaf.right = kLightTreeInvalid;
            leaf.light = e.light;
            leaf.kind = spatial ? kLightTreeFiniteLeaf : kLightTreeUnboundedLeaf;
            tree.nodes.push_back(leaf);
            tree.light_to_node[e.light] = index;
            tree.maximum_depth = std::max(tree.maximum_depth, depth);
            return BLACKFRAME_STATUS_SUCCESS;
        }
        if (spatial) {
            float minimum[3], maximum[3];
            for (int a = 0; a < 3; ++a) {
                minimum[a] = maximum[a] = entries[begin].centroid[a];
            }
            for (size_t i = begin + 1; i < end; ++i) {
                for (int a = 0; a < 3; ++a) {
                    minimum[a] = std::min(minimum[a], entries[i].centroid[a]);
                    maximum[a] = std::max(maximum[a], entries[i].centroid[a]);
                }
            }
            Scaled extent[3];
            for (int a = 0; a < 3; ++a) {
                if (const auto st = scaled_difference(maximum[a], minimum[a], extent[a], error);
                    st != BLACKFRAME_STATUS_SUCCESS) {
                    return st;
                }
            }
            int axis = 0;
            if (scaled_less(extent[axis], extent[1])) {
                axis = 1;
            }
            if (scaled_less(extent[axis], extent[2])) {
                axis = 2;
            }
            std::sort(entries.begin() + static_cast<std::ptrdiff_t>(begin),
                      entries.begin() + static_cast<std::ptrdiff_t>(end), [axis](const Entry& l, const Entry& r) {
                          if (l.centroid[axis] != r.centroid[axis]) {
                              return l.centroid[axis] < r.centroid[axis];
                          }
                          return l.light < r.light;
                      });
        }
        LightTreeNode internal{};
        internal.parent = parent;
        internal.left = internal.right = internal.light = kLightTreeInvalid;
        internal.kind = kLightTreeInternal;
        tree.nodes.push_back(internal);
        const size_t middle = begin + (end - begin) / 2;
        uint32_t left = 0, right = 0;
        if (const auto st = build(entries, begin, middle, spatial, index, depth + 1, left);
            st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        if (const auto st = build(entries, middle, end, spatial, index, depth + 1, right);
            st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        const Box box = merged(node_box(tree.nodes[left]), node_box(tree.nodes[right]));
        const float power = tree.nodes[left].power + tree.nodes[right].power;
        if (!std::isfinite(power) || !(power > tree.nodes[left].power) || !(power > tree.nodes[right].power)) {
            return exhausted(error, "Light-tree aggregation lost positive subtree power.");
        }
        LightTreeNode& node = tree.nodes[index];
        std::copy(box.lo, box.lo + 3, node.lo);
        std::copy(box.hi, box.hi + 3, node.hi);
        node.power = power;
        node.left = left;
        node.right = right;
        return BLACKFRAME_STATUS_SUCCESS;
    }
};

}  // namespace

blackframe_status build_light_tree(const bf200_light_tree_input_v1* lights, uint32_t count, LightTree& tree,
                                   std::string& error) {
    tree = LightTree{};
    if (count == 0) {
        return invalid(error, "Light sampling requires at least one registry slot.");
    }
    std::vector<float> powers(4ULL * count);
    std::vector<bool> unbounded(count);
    for (uint32_t i = 0; i < count; ++i) {
        const Box box{{lights[i].bounds_min[0], lights[i].bounds_min[1], lights[i].bounds_min[2]},
                      {lights[i].bounds_max[0], lights[i].bounds_max[1], lights[i].bounds_max[2]}};
        for (int a = 0; a < 3; ++a) {  // Bounds3::from_minimum_maximum: ordered, no NaN
            if (std::isnan(box.lo[a]) || std::isnan(box.hi[a]) || box.lo[a] > box.hi[a]) {
                return invalid(error, "Bounds require ordered coordinates without NaN.");
            }
        }
        const bool is_finite = finite_box(box), is_unbounded = unbounded_box(box);
        if (!is_finite && !is_unbounded) {
            return invalid(error, "Light-tree bounds must be finite and non-empty or canonically unbounded.");
        }
        unbounded[i] = is_unbounded;
        std::copy(lights[i].spectral_power, lights[i].spectral_power + 4, powers.begin() + 4ULL * i);
    }
    std::vector<float> weights;
    if (const auto st = light_power_weights(powers.data(), count, weights, tree.cdf, error);
        st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    std::vector<Entry> finite, infinite;
    size_t supported = 0;
    for (uint32_t i = 0; i < count; ++i) {
        if (weights[i] == 0.0F) {
            continue;
        }
        ++supported;
        Entry e{};
        if (unbounded[i]) {
            e.box = Box{{-kInfinity, -kInfinity, -kInfinity}, {kInfinity, kInfinity, kInfinity}};
        } else {
            e.box = Box{{lights[i].bounds_min[0], lights[i].bounds_min[1], lights[i].bounds_min[2]},
                        {lights[i].bounds_max[0], lights[i].bounds_max[1], lights[i].bounds_max[2]}};
            for (int a = 0; a < 3; ++a) {
                e.centroid[a] = midpoint(e.box.lo[a], e.box.hi[a]);
            }
        }
        e.power = weights[i];
        e.light = i;
        (unbounded[i] ? infinite : finite).push_back(e);
    }
    if (supported == 0) {
        return inconsistent(error, "Positive light-tree power has no supported registry slot.");
    }
    if (supported > (static_cast<uint64_t>(kLightTreeInvalid) + 1ULL) / 2ULL) {
        return exhausted(error, "Light-tree node indices exceed the stable 32-bit domain.");
    }
    tree.light_to_node.assign(count, kLightTreeInvalid);
    tree.nodes.reserve(2 * supported - 1);
    Builder builder{tree, error};
    uint32_t finite_root = kLightTreeInvalid, unbounded_root = kLightTreeInvalid;
    if (!finite.empty() && !infinite.empty()) {
        tree.root = 0;
        LightTreeNode root{};
        root.parent = root.left = root.right = root.light = kLightTreeInvalid;
        root.kind = kLightTreeInternal;
        tree.nodes.push_back(root);
        if (const auto st = builder.build(finite, 0, finite.size(), true, 0, 2, finite_root);
            st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        if (const auto st = builder.build(infinite, 0, infinite.size(), false, 0, 2, unbounded_root);
            st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        const float power = tree.nodes[finite_root].power + tree.nodes[unbounded_root].power;
        if (!std::isfinite(power) || !(power > tree.nodes[finite_root].power) ||
            !(power > tree.nodes[unbounded_root].power)) {
            return exhausted(error, "Light-tree aggregation lost positive finite or unbounded power.");
        }
        LightTreeNode& node = tree.nodes[0];
        for (int a = 0; a < 3; ++a) {
            node.lo[a] = -kInfinity;
            node.hi[a] = kInfinity;
        }
        node.power = power;
        node.left = finite_root;
        node.right = unbounded_root;
    } else if (!finite.empty()) {
        if (const auto st = builder.build(finite, 0, finite.size(), true, kLightTreeInvalid, 1, finite_root);
            st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        tree.root = finite_root;
    } else {
        if (const auto st = builder.build(infinite, 0, infinite.size(), false, kLightTreeInvalid, 1, unbounded_root);
            st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        tree.root = unbounded_root;
    }
    if (finite_root != kLightTreeInvalid) {  // root_extent (LightSampler.cpp:424-454)
        const LightTreeNode& root = tree.nodes[finite_root];
        Scaled extent[3];
        for (int a = 0; a < 3; ++a) {
            if (const auto st = scaled_difference(root.hi[a], root.lo[a], extent[a], error);
                st != BLACKFRAME_STATUS_SUCCESS) {
                return st;
            }
        }
        Scaled maximum = extent[0];
        if (scaled_less(maximum, extent[1])) {
            maximum = extent[1];
        }
        if (scaled_less(maximum, extent[2])) {
            maximum = extent[2];
        }
        if (maximum.mantissa != 0.0F) {
            const float logarithm = scaled_log(maximum);
            if (!std::isfinite(logarithm)) {
                return exhausted(error, "Light-tree root extent logarithm is not representable.");
            }
            tree.root_log_extent = logarithm;
            tree.root_has_extent = true;
        }
    }
    if (tree.nodes.size() != 2 * supported - 1 || tree.root == kLightTreeInvalid || tree.maximum_depth == 0) {
        return inconsistent(error, "Light-tree construction produced invalid storage.");
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

blackframe_status light_tree_sample(const LightTree& t, const float (&p)[3], float u, uint32_t& light,
                                    float& probability, std::string& error) {
    if (t.nodes.empty() || t.root >= t.nodes.size() || t.light_to_node.size() + 1 != t.cdf.size()) {
        return inconsistent(error, "A moved-from or inconsistent light tree cannot classify canonical samples.");
    }
    if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) {  // LightSampleContext::create
        return invalid(error, "A light sample context requires a finite world-space position.");
    }
    if (!std::isfinite(u) || u < 0.0F || !(u < 1.0F)) {
        return invalid(error, "Light-tree sampling requires a finite canonical sample in [0, 1).");
    }
    uint32_t index = t.root;
    float remapped = u, selection = 1.0F;
    while (t.nodes[index].kind == kLightTreeInternal) {
        float left = 0.0F;
        if (const auto st = left_probability(t, p, index, left, error); st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        const LightTreeNode& node = t.nodes[index];
        const bool go_left = remapped < left;
        const float branch = go_left ? left : 1.0F - left;
        float product = 0.0F, next = 0.0F;
        if (const auto st = multiply_probability(selection, branch, product, error); st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        if (const auto st = remap(remapped, go_left ? 0.0F : left, branch, next, error);
            st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        selection = product;
        remapped = next;
        index = go_left ? node.left : node.right;
        if (index >= t.nodes.size()) {
            return inconsistent(error, "Light-tree traversal reached an invalid child index.");
        }
    }
    light = t.nodes[index].light;
    if (light >= t.light_to_node.size() || !(selection > 0.0F) || selection > 1.0F) {
        return inconsistent(error, "Light-tree traversal reached an invalid supported leaf.");
    }
    probability = selection;
    return BLACKFRAME_STATUS_SUCCESS;
}

blackframe_status light_tree_probability(const LightTree& t, const float (&p)[3], uint32_t light, float& probability,
                                         std::string& error) {
    if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) {  // LightSampleContext::create
        return invalid(error, "A light sample context requires a finite world-space position.");
    }
    if (light >= t.light_to_node.size()) {
        return invalid(error, "Light-tree probability index is out of range.");
    }
    if (t.nodes.empty() || t.root >= t.nodes.size()) {
        return inconsistent(error, "A moved-from or inconsistent light tree has no queryable probability.");
    }
    const float baseline = t.cdf[light + 1ULL] - t.cdf[light];
    if (!std::isfinite(baseline) || baseline < 0.0F) {
        return inconsistent(error, "Light-tree support CDF contains an invalid probability.");
    }
    if (baseline == 0.0F) {
        probability = 0.0F;
        return BLACKFRAME_STATUS_SUCCESS;
    }
    uint32_t path[64];
    bool chose_left[64];
    size_t length = 0;
    uint32_t index = t.light_to_node[light];
    if (index >= t.nodes.size() || t.nodes[index].light != light) {
        return inconsistent(error, "Light-tree slot does not map to its supported leaf.");
    }
    while (index != t.root) {
        if (length == 64) {
            return inconsistent(error, "Light-tree path exceeds its validated balanced depth.");
        }
        const uint32_t parent = t.nodes[index].parent;
        if (parent >= t.nodes.size() || t.nodes[parent].kind != kLightTreeInternal) {
            return inconsistent(error, "Light-tree leaf has an invalid parent path.");
        }
        const bool left = t.nodes[parent].left == index;
        if (!left && t.nodes[parent].right != index) {
            return inconsistent(error, "Light-tree parent does not reference its child.");
        }
        path[length] = parent;
        chose_left[length] = left;
        ++length;
        index = parent;
    }
    float selection = 1.0F;
    for (size_t k = length; k > 0; --k) {
        float left = 0.0F;
        if (const auto st = left_probability(t, p, path[k - 1], left, error); st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        float product = 0.0F;
        if (const auto st = multiply_probability(selection, chose_left[k - 1] ? left : 1.0F - left, product, error);
            st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        selection = product;
    }
    probability = selection;
    return BLACKFRAME_STATUS_SUCCESS;
}

}  // namespace bf200

using bf200::LightTree;

extern "C" {

BF200_EXPORT blackframe_status bf200_light_tree_select(const bf200_light_tree_input_v1* lights, uint32_t light_count,
                                                       const float* positions, const float* samples,
                                                       uint64_t query_count, uint32_t* light_indices,
                                                       float* probabilities) noexcept {
    if (lights == nullptr || (query_count != 0 && (positions == nullptr || samples == nullptr ||
                                                   light_indices == nullptr || probabilities == nullptr))) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    try {
        LightTree tree;
        std::string error;
        if (const auto st = bf200::build_light_tree(lights, light_count, tree, error); st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        for (uint64_t q = 0; q < query_count; ++q) {
            const float p[3] = {positions[3 * q], positions[3 * q + 1], positions[3 * q + 2]};
            uint32_t light = 0;
            float probability = 0.0F;
            if (bf200::light_tree_sample(tree, p, samples[q], light, probability, error) == BLACKFRAME_STATUS_SUCCESS) {
                light_indices[q] = light;
                probabilities[q] = probability;
            } else {
                light_indices[q] = bf200::kLightTreeInvalid;
                probabilities[q] = -1.0F;
            }
        }
    } catch (const std::bad_alloc&) {
        return BLACKFRAME_STATUS_OUT_OF_RANGE;
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

BF200_EXPORT blackframe_status bf200_light_tree_probability(const bf200_light_tree_input_v1* lights,
                                                            uint32_t light_count, const float* positions,
                                                            const uint32_t* light_indices, uint64_t query_count,
                                                            float* probabilities) noexcept {
    if (lights == nullptr ||
        (query_count != 0 && (positions == nullptr || light_indices == nullptr || probabilities == nullptr))) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    try {
        LightTree tree;
        std::string error;
        if (const auto st = bf200::build_light_tree(lights, light_count, tree, error); st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        for (uint64_t q = 0; q < query_count; ++q) {
            const float p[3] = {positions[3 * q], positions[3 * q + 1], positions[3 * q + 2]};
            float probability = 0.0F;
            probabilities[q] =
                bf200::light_tree_probability(tree, p, light_indices[q], probability, error) == BLACKFRAME_STATUS_SUCCESS
                    ? probability
                    : -1.0F;
        }
    } catch (const std::bad_alloc&) {
        return BLACKFRAME_STATUS_OUT_OF_RANGE;
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

}  // extern "C"
