// Device-side scene layout and wavefront state of the bf200 backend.
#pragma once

#include <cstdint>

#include "bf200.h"
#include "bf200_shading.cuh"
#include "bf200_light_tree.h"

namespace bf200 {

// BVH2 node, 64 bytes, both children's boxes in one node (one 64-byte fetch per step):
//   a = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   b = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   c = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   d = (child0, child1, -, -) as int bits. child >= 0: internal node index (global);
//       child < 0: leaf, ~child = first_leaf_triangle << 3 | (count - 1).
struct alignas(16) BvhNode {
    float4 a, b, c;
    int4 d;
};

// BVH4 node, 128 bytes (one L2 line): the boxes of up to four children in structure-of-arrays
// form, so one node is eight 16-byte loads. child[k] >= 0: internal node index (always greater
// than this node's own index, so a walk cannot revisit a node); child[k] < 0: leaf, the same code
// as BvhNode. The used slots come first and info.x counts them; unused slots are never tested
// (their boxes are not meaningful to the slab test).
struct alignas(128) BvhNode4 {
    float4 lo_x, hi_x, lo_y, hi_y, lo_z, hi_z;
    int4 child;
    int4 info;  // x: used child slots (1..4)
};

constexpr int kLeafCountBits = 3;
// Scenes with at most this many instances test every instance box up front; larger ones walk a
// TLAS over the instances' world boxes.
constexpr uint32_t kEagerInstances = 32;
constexpr int kMaxLeafSize = 1 << kLeafCountBits;
constexpr int kTraversalStack = 128;  // up to 32 instance entries plus one BLAS walk

struct LightInfo {
    uint32_t instance;
    uint32_t tri_offset;  // into light_tri_* arrays
    uint32_t tri_count;
    float area;
    float inverse_area;
    float err_x, err_y, err_z;  // world position error of the emitter mesh
    float radiance[4];
};

// A punctual light of the registry (slots [0, punctual_count)), with the cone cosines a spot light
// samples with (PunctualLights.hpp:593-815).
struct PunctualLight {
    uint32_t kind;  // BF200_PUNCTUAL_*
    uint32_t hard;  // spot: inner == outer
    float px, py, pz;
    float ex, ey, ez;
    float dx, dy, dz;
    float cos_inner, cos_outer;
    float spectrum[4];
};

// Everything a kernel needs about a committed scene; passed by value as a kernel parameter.
struct SceneView {
    uint32_t instance_count;
    uint32_t light_count;
    const float4* inst_world_box;  // padded world box per instance: lo (xyz, w = visibility mask bits), hi
    int32_t tlas_root;             // BVH4 over the instances' world boxes (leaves ~instance), or -1
    const float4* inst_to_object;  // 3 rows (m0..m3) per instance
    const float4* inst_to_world;   // 3 rows per instance
    const uint4* inst_info;        // geometry, material, visibility mask, light index or ~0
    const uint8_t* inst_route;     // shading route of a hit on the instance (kRoute*)
    const uint32_t* inst_normal_offset;
    const uint4* geom_info;        // vertex offset (sphere: leaf record), triangle offset, bvh root node, kind
    const float* positions;        // object space, 3 per vertex
    const float* normals;          // 3 per vertex
    const uint32_t* triangles;     // geometry-local vertex indices, 3 per triangle
    const BvhNode4* nodes;
    const float4* leaf_tris;       // 3 per leaf triangle: v0 (w = primitive index bits), v1, v2
    const float4* world_normals;   // per instance triangle
    const ClosureData* closures;   // per material: its first closure (the single-closure routes)
    const ClosureData* mix_closures;       // every material's closures, material_info.w the first
    const MixDistribution* mix_dist;       // per material: projected component distribution
    const PunctualLight* punctual;         // registry slots [0, punctual_count)
    uint32_t punctual_count;
    const float4* emission;        // per material
    const uint4* material_info;    // closure count, frame mode, rotation bits, first closure
    const float* light_select_cdf; // light_count + 1 boundaries over the registry (punctual, then mesh)
    const LightInfo* lights;       // mesh lights: registry slot punctual_count + index
    const float4* light_tri_vertices;  // 3 per light triangle, world space
    const float4* light_tri_normals;
    const float* light_tri_areas;
    const float* light_tri_cdf;
    float4 environment;
    uint32_t sphere_count;  // analytic sphere geometries (0: the walks run their triangle-only form)
    // spatial light tree (bf200_scene_set_light_tree); null: selection by light_select_cdf
    const LightTreeNode* tree;
    const uint32_t* tree_light_to_node;
    uint32_t tree_node_count;
    uint32_t tree_root;
    float tree_log_extent;
    uint32_t tree_has_extent;
};

// geom_info.w: the geometry's kind. A sphere's geom_info.x is its leaf record (centre, radius).
constexpr uint32_t kGeometryTriangles = 0U, kGeometrySphere = 1U;
// A sphere's leaf record in the leaf-triangle array: v0 = centre (w: primitive index 0),
// v1 = (radius, 0, 0, kSphereLeaf as bits), v2 = 0. Triangle records have 0 in v1.w.
constexpr uint32_t kSphereLeaf = 0x53504845U;
// A sphere's leaf code carries the record count 8, which no triangle leaf has (at most 4), so the
// walks branch to the sphere test once per leaf, outside the triangle loop.
constexpr uint32_t kSphereLeafCount = 8U;

// Transport options resolved for the device.
struct TransportParams {
    uint32_t heuristic;
    uint32_t limits[5];
    uint32_t roulette;
    uint32_t roulette_first;
    float roulette_min;
    float roulette_max;
};

// Shading routes. A hit is shaded by the kernel specialised for its material's single closure
// kind; misses and every other material take the generic kernel.
constexpr uint32_t kRouteGeneric = 0U, kRouteLambert = 1U, kRouteConductor = 2U, kRouteDielectric = 3U;
constexpr uint32_t kRouteCount = 4U;
constexpr uint8_t kRouteNone = 0xFFU;  // slot not shaded this iteration / no shadow ray

// Stable compaction tiles: one 256-thread block per 4096 consecutive slots.
constexpr uint32_t kCompactTile = 4096U;
constexpr uint32_t kCompactMaxRoutes = 4U;

// Slot states of the persistent wavefront.
constexpr uint8_t kSlotEmpty = 0, kSlotActive = 1, kSlotDone = 2;

// Path sources: film (camera rays generated on the device) or an explicit input batch.
struct PathSource {
    uint32_t mode;  // 0 film, 1 batch
    uint64_t total;
    // film
    uint32_t width, height;
    uint64_t first_sample;
    uint64_t seed;
    float cam_origin[3], cam_t[3], cam_b[3], cam_n[3];
    float half_width, half_height, t_min, t_max, time;
    uint32_t mask;
    uint32_t jitter;
    // batch
    const bf200_path_input_v1* inputs;
    bf200_path_result_v1* results;
    float4* path_radiance;  // film mode: radiance per path id of the chunk
    // batch mode with ray cones: the primary cone of every input (width, spread) and the cone at
    // every result's terminal-ray origin; both null when the caller traces without cones
    const float2* cones_in;
    float2* cones_out;
    // batch mode: depth-zero initial states (beta, radiance, eta scale); null = PathState::create_initial
    const bf200_path_state_v1* states_in;
    // sampler: null for the hash SampleStream; otherwise the Owen-scrambled Sobol direction heads
    // (kDeviceSobolDimensions x 64 leading 32-bit direction numbers)
    const uint32_t* sobol;
};

// Sobol dimensions carried on the device: the raster pair, the four primary dimensions and
// 256 bounces of 10 dimensions each.
constexpr uint32_t kDeviceSobolDimensions = 2U + 4U + 10U * 256U;

// Path-replay adjoint of a film render: the replay launches of the wavefront (and only they) carry
// this view. The gradient of an image loss is accumulated per material as kAdjointStride doubles:
// d/d(closure weight lane 0..3), d/d(alpha_x), d/d(alpha_y) and two unused words; the derivative
// with respect to a common factor on every emitter's radiance follows the last material record.
constexpr uint32_t kAdjointMaterials = 64U;
constexpr uint32_t kAdjointStride = 8U;
constexpr uint32_t kAdjointEmission = kAdjointMaterials * kAdjointStride;
constexpr uint32_t kAdjointWords = kAdjointEmission + 1U;
struct AdjointView {
    const float4* pixel_adjoint;  // per pixel: dLoss/d(pixel rgb) divided by the pixel's weight
    const float4* forward;        // per path of the chunk: forward radiance (NaN x: failed path)
    double* gradients;            // kAdjointWords
    uint4* pending;               // per slot: roughness score of the last continuation (x, y float
                                  // bits), its material, and the path tag (path id + 1)
    uint4* shadow_score;          // per slot: roughness score of the queued shadow ray, material, flag
    float lane_rgb[3][4];         // d(sample rgb c)/d(radiance lane l), the film's sensor map
    uint32_t pixels;
};

// Per-slot wavefront state, structure of arrays in HBM.
struct Wavefront {
    uint32_t capacity;
    uint8_t* state;
    uint64_t* path_id;
    float4* ray_o;      // origin, t_max
    float4* ray_d;      // direction, t_min
    float4* beta;
    float4* radiance;
    uint32_t* depth;    // diffuse | glossy << 8 | specular << 16 | transmission << 24
    float* eta;
    float4* prev;       // previous continuous BSDF vertex position, pdf (0 = none)
    uint32_t* flags;    // delta flags | termination << 8 | blocked << 16
    uint32_t* status;   // lane failure code | segments << 8
    uint2* stream;      // sample-stream prefix state (64-bit), split
    uint4* sobol_index; // Owen-Sobol sampler only: sample index, seed (64-bit each, split)
    uint2* pixel_hash;  // Owen-Sobol sampler only: mix_bits of the packed pixel
    uint32_t* mask;     // ray visibility mask of the path
    float2* cone;       // ray cone (width, spread) at the ray origin; null unless cones are traced
    float4* hit_tb;     // t, b0, b1, b2
    uint2* hit_id;      // instance, leaf record of the hit triangle (instance = ~0 on a miss)
    // routing: shading route per slot, and the slots of every route in slot order
    uint8_t* route;
    uint32_t* route_queue;
    uint32_t* route_offsets;  // kRouteCount + 1 queue boundaries
    // shadow rays, stored at their slot; shadow_key 0 marks a slot with a shadow ray
    uint8_t* shadow_key;
    float4* shadow_o;   // origin, t_max
    float4* shadow_d;   // direction
    float4* shadow_c;   // contribution (unoccluded)
    uint32_t* shadow_queue;    // slots with a shadow ray, in slot order
    uint32_t* shadow_offsets;  // 2 queue boundaries
    uint32_t* tile_counts;     // compaction scratch: kCompactMaxRoutes x tiles
    // counters: [0] shadow queue size, [1] next path to claim, [2] active slots,
    //           [3] extension segments, [4] shadow segments, [5] failed lanes,
    //           [6] first failure path (min), [7] first failure code, [8] k_trace fetch cursor,
    //           [9] iterations and [10] iteration-bound flag of a device-side loop
    unsigned long long* counters;
};

}  // namespace bf200
