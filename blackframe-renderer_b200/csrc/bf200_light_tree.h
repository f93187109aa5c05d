// Power-weighted light selection and the spatial light tree of the reference's LightSampler:
// LightSampler::create_power_weighted and LightSampler::create_spatial_tree
// (Blackframe/Renderer/Source/LightSampler.cpp:626-951), built on the host as a flat node array
// the device can read, and its selection at a shading point (LightSampler.cpp:953-1226).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "bf200.h"

namespace bf200 {

// The selection CDF (count + 1 boundaries) of four-lane spectral powers in registry order, as
// LightSampler::create_power_weighted builds it (LightSampler.cpp:116-249, 605-625), and the
// same with the per-light power weights.
blackframe_status light_power_cdf(const float* powers, uint32_t count, std::vector<float>& cdf, std::string& error);
blackframe_status light_power_weights(const float* powers, uint32_t count, std::vector<float>& weights,
                                      std::vector<float>& cdf, std::string& error);

constexpr uint32_t kLightTreeInvalid = 0xFFFFFFFFU;
constexpr uint32_t kLightTreeInternal = 0U, kLightTreeFiniteLeaf = 1U, kLightTreeUnboundedLeaf = 2U;

// One node: bounds (the canonical unbounded box is +-infinity), aggregate power weight, links,
// the registry slot of a leaf, and the kind. 48 bytes, in build order (a parent before its children).
struct LightTreeNode {
    float lo[3];
    float hi[3];
    float power;
    uint32_t parent;
    uint32_t left;
    uint32_t right;
    uint32_t light;
    uint32_t kind;
};
static_assert(sizeof(LightTreeNode) == 48, "light-tree node layout");

struct LightTree {
    std::vector<LightTreeNode> nodes;
    std::vector<uint32_t> light_to_node;  // per registry slot; kLightTreeInvalid for zero-power slots
    std::vector<float> cdf;               // the power CDF: baseline support of every slot
    uint32_t root = kLightTreeInvalid;
    float root_log_extent = 0.0F;  // log of the finite root's largest extent
    bool root_has_extent = false;
    uint32_t maximum_depth = 0;
};

blackframe_status build_light_tree(const bf200_light_tree_input_v1* lights, uint32_t count, LightTree& tree,
                                   std::string& error);

// Selection of a light for a canonical sample u at `position`: the light slot and its discrete
// probability (LightSampler.cpp:1058-1129).
blackframe_status light_tree_sample(const LightTree& tree, const float (&position)[3], float u, uint32_t& light,
                                    float& probability, std::string& error);

// The probability that `position` selects `light` (LightSampler.cpp:1151-1225).
blackframe_status light_tree_probability(const LightTree& tree, const float (&position)[3], uint32_t light,
                                         float& probability, std::string& error);

}  // namespace bf200
