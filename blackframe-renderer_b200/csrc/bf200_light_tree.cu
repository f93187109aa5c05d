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
#include "bf200_light_tree_device.cuh"

namespace bf200 {
namespace {

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
    uint32_t light = kLightTreeInvalid;
    float probability = -1.0F;
    if (!d_tree_select(nodes, node_count, root, light_count, root_log, root_has != 0, p, samples[q], light,
                       probability)) {
        light = kLightTreeInvalid;
        probability = -1.0F;
    }
    lights[q] = light;
    probabilities[q] = probability;
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
