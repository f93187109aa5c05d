// bf200 host runtime and C ABI: context, scene build, wavefront driver, extension tables.
//
// Replaces, behind the C ABI of include/bf200.h:
//   CudaSceneSoA::upload + CudaSceneBvh::build (Blackframe/Backends/GPU/CUDA/Source/SceneSoA.cpp,
//   SceneBvh.cpp:1109-1146) -> bf200_scene_create: validation, mesh-light registry, per-geometry
//   BLAS build (binned SAH) and the device upload;
//   trace_cuda_wavefront_transport (WavefrontTransport.cpp:1984-2835) -> bf200_trace_paths /
//   bf200_render_film: a persistent wavefront with in-place path regeneration. The host touches
//   the device once per wavefront iteration (an 8-byte counter read), never per stage.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <future>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "bf200.h"
#include "bf200_device.cuh"
#include "bf200_envmap.h"
#include "bf200_kernels.h"
#include "bf200_light_tree.h"
#include "bf200_records.h"
#include "bf200_sobol.h"

using namespace bf200;

static_assert(kClosureCapacity == kMaxClosures, "one closure capacity");

struct bf200_context {
    int device = 0;
    uint32_t build_mode = BF200_BUILD_HOST_SAH;  // bf200_context_set_build_mode
    // measured batch lane counts per job-size class, and the count of the last batch call
    std::map<uint32_t, uint32_t> batch_lanes_by_class;
    uint32_t last_batch_lanes = 0;
    cudaStream_t stream = nullptr;
    uint32_t sm_count = 148;
    uint64_t capacity = 0;
    std::string last_error;
    // wavefront buffers
    void* arena = nullptr;
    Wavefront w{};
    unsigned long long* pinned_counters = nullptr;
    // grow-only workspaces of the film and batch entry points, kept across calls
    void* film_radiance = nullptr;  // per-path radiance of one film chunk, then the skipped counter
    size_t film_radiance_bytes = 0;
    void* film_staging = nullptr;   // device copy of a host film
    size_t film_staging_bytes = 0;
    void* batch_staging = nullptr;  // device copies of host path inputs and results
    size_t batch_staging_bytes = 0;
    // film batches (bf200_render_films_device): one stream, event, arena slice, pinned counter
    // block and radiance buffer per lane, kept across calls
    std::vector<cudaStream_t> lane_streams;
    std::vector<cudaEvent_t> lane_events;
    void* lane_arena = nullptr;
    size_t lane_arena_bytes = 0;
    unsigned long long* lane_counters = nullptr;  // pinned, 8 per lane
    size_t lane_counter_lanes = 0;
    std::vector<void*> lane_radiance;
    std::vector<size_t> lane_radiance_bytes;
    // path-replay adjoint: pixel adjoint, gradient sums, loss, per-slot scores
    void* adjoint_workspace = nullptr;
    size_t adjoint_workspace_bytes = 0;
    // ray cones of the wavefront slots (bf200_trace_paths_with_cones*), capacity x (width, spread)
    void* cone_column = nullptr;
    size_t cone_column_bytes = 0;
};

struct bf200_scene {
    bf200_context* context = nullptr;
    SceneView view{};
    std::vector<void*> allocations;
    uint32_t light_count = 0;
    uint32_t material_count = 0;
    uint64_t triangle_count = 0;
    uint64_t node_count = 0;
    // transform-only refit (bf200_scene_refit): what the instance level is rebuilt from
    uint64_t fingerprint = 0;           // the description without its instance transforms
    std::vector<float> object_boxes;    // per geometry: lo xyz, hi xyz
    uint32_t tlas_first = 0;            // first TLAS node in the node array (when there is a TLAS)
    std::vector<BvhNode4> tlas_nodes;   // host copy of the TLAS nodes
    uint32_t instance_triangles = 0;
    uint32_t* normal_failures = nullptr;     // device counter of k_world_normals
    size_t light_triangles = 0;
    uint32_t punctual_count = 0;        // light registry slots [0, punctual_count) are punctual
    bool plain_materials = true;        // no mixtures and only Lambert / GGX conductor / dielectric
    // the spatial light tree (bf200_scene_set_light_tree): device node array and light-to-node map,
    // owned here (not in `allocations`) so a new tree reuses them and a cleared tree frees them
    void* tree_nodes = nullptr;
    void* tree_map = nullptr;
    size_t tree_node_bytes = 0;
    size_t tree_map_bytes = 0;
    bf200_scene_stats_v1 stats{};       // bf200_scene_stats: sizes and host wall time per build phase
};

namespace {

blackframe_status fail(bf200_context* c, blackframe_status status, const std::string& message) {
    if (c != nullptr) {
        c->last_error = message;
    }
    return status;
}

blackframe_status cuda_fail(bf200_context* c, cudaError_t e, const char* what) {
    return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------------------------
// Host helpers restating the reference's scene-side arithmetic
// ---------------------------------------------------------------------------------------------

F3 transform_point_h(const float* m, F3 p) {  // Transforms.hpp:93-101
    return {m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
            m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]};
}

// SceneSurfaceInteraction.cpp:204-250 (transform_orientation): sign of the upper 3x3
// determinant by partial-pivot elimination in double.
// Grows a context workspace to at least `need` bytes (contents are not kept).
blackframe_status grow_workspace(bf200_context* c, void** buffer, size_t* have, size_t need, const char* what) {
    if (need <= *have && *buffer != nullptr) {
        return BLACKFRAME_STATUS_SUCCESS;
    }
    if (*buffer != nullptr) {
        cudaFree(*buffer);
        *buffer = nullptr;
        *have = 0;
    }
    const cudaError_t e = cudaMalloc(buffer, need);
    if (e != cudaSuccess) {
        *buffer = nullptr;
        return cuda_fail(c, e, what);
    }
    *have = need;
    return BLACKFRAME_STATUS_SUCCESS;
}

bool transform_orientation(const float* m4, int& orientation) {
    double m[9];
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) {
            m[r * 3 + c] = static_cast<double>(m4[r * 4 + c]);
        }
    }
    orientation = 1;
    for (int col = 0; col < 3; ++col) {
        int pr = col;
        double pm = std::abs(m[col * 3 + col]);
        for (int cand = col + 1; cand < 3; ++cand) {
            const double cm = std::abs(m[cand * 3 + col]);
            if (cm > pm) {
                pm = cm;
                pr = cand;
            }
        }
        if (!std::isfinite(pm) || pm == 0.0) {
            return false;
        }
        if (pr != col) {
            for (int k = col; k < 3; ++k) {
                std::swap(m[col * 3 + k], m[pr * 3 + k]);
            }
            orientation = -orientation;
        }
        const double pivot = m[col * 3 + col];
        orientation = pivot < 0.0 ? -orientation : orientation;
        for (int row = col + 1; row < 3; ++row) {
            const double factor = m[row * 3 + col] / pivot;
            for (int k = col + 1; k < 3; ++k) {
                m[row * 3 + k] -= factor * m[col * 3 + k];
            }
        }
    }
    return true;
}

// ---------------------------------------------------------------------------------------------
// BLAS build: binned SAH over triangle boxes, leaves of at most 4 triangles, BVH2 nodes that
// carry both children's boxes.
// ---------------------------------------------------------------------------------------------

struct Box {
    float lo[3] = {std::numeric_limits<float>::infinity(), std::numeric_limits<float>::infinity(),
                   std::numeric_limits<float>::infinity()};
    float hi[3] = {-std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity(),
                   -std::numeric_limits<float>::infinity()};
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    double area() const {
        if (!(lo[0] <= hi[0])) {
            return 0.0;
        }
        const double dx = double(hi[0]) - lo[0], dy = double(hi[1]) - lo[1], dz = double(hi[2]) - lo[2];
        return 2.0 * (dx * dy + dy * dz + dz * dx);
    }
};

struct Prim {
    Box box;
    float c[3];
    uint32_t index;
};

constexpr int kLeafSize = 4;
static_assert(kLeafSize < static_cast<int>(kSphereLeafCount) && kSphereLeafCount == kMaxLeafSize,
              "triangle leaves never carry the sphere leaf count");
constexpr int kBins = 16;

// Subtrees of at least this many primitives are built on their own thread (down to
// Builder::parallel_levels levels), into their own arrays that are then appended: the appended
// result is the sequential build's, node for node and record for record.
constexpr int kParallelPrims = 32768;
constexpr uint32_t kDeviceBuildMinimum = 4096;  // smaller geometries build faster on the host

struct Builder {
    std::vector<Prim>& prims;
    std::vector<BvhNode>& nodes;
    std::vector<float4>& leaf_tris;
    const float* positions;  // geometry-local base
    const uint32_t* tris;
    uint32_t max_depth = 0;
    int leaf_limit = kLeafSize;
    bool instance_leaves = false;  // TLAS: one instance per leaf, encoded as ~instance
    int parallel_levels = 0;       // levels whose large right subtrees go to their own thread

    int make_leaf(int begin, int end) {
        if (instance_leaves) {
            return ~static_cast<int>(prims[begin].index);
        }
        const uint32_t first = static_cast<uint32_t>(leaf_tris.size() / 3);
        for (int i = begin; i < end; ++i) {
            const uint32_t t = prims[i].index;
            for (int k = 0; k < 3; ++k) {
                const float* p = positions + 3ULL * tris[3ULL * t + k];
                float w = 0.0F;
                if (k == 0) {
                    std::memcpy(&w, &t, 4);
                }
                leaf_tris.push_back(make_float4(p[0], p[1], p[2], w));
            }
        }
        const uint32_t packed = (first << kLeafCountBits) | static_cast<uint32_t>(end - begin - 1);
        return ~static_cast<int>(packed);
    }

    Box bounds(int begin, int end) const {
        Box b;
        for (int i = begin; i < end; ++i) {
            b.grow(prims[i].box);
        }
        return b;
    }

    // Returns the child encoding for prims[begin, end).
    int build(int begin, int end, uint32_t depth) {
        max_depth = std::max(max_depth, depth);
        const int n = end - begin;
        if (n <= leaf_limit) {
            return make_leaf(begin, end);
        }
        Box cb;
        for (int i = begin; i < end; ++i) {
            cb.grow(prims[i].c);
        }
        int best_axis = -1, best_bin = -1;
        double best_cost = std::numeric_limits<double>::infinity();
        for (int axis = 0; axis < 3; ++axis) {
            const float extent = cb.hi[axis] - cb.lo[axis];
            if (!(extent > 0.0F)) {
                continue;
            }
            Box bin_box[kBins];
            int bin_count[kBins] = {};
            for (int i = begin; i < end; ++i) {
                int b = static_cast<int>(kBins * ((prims[i].c[axis] - cb.lo[axis]) / extent));
                b = std::min(std::max(b, 0), kBins - 1);
                bin_box[b].grow(prims[i].box);
                ++bin_count[b];
            }
            Box left_box[kBins];
            int left_count[kBins];
            Box acc;
            int cnt = 0;
            for (int b = 0; b < kBins; ++b) {
                acc.grow(bin_box[b]);
                cnt += bin_count[b];
                left_box[b] = acc;
                left_count[b] = cnt;
            }
            acc = Box{};
            cnt = 0;
            for (int b = kBins - 1; b > 0; --b) {
                acc.grow(bin_box[b]);
                cnt += bin_count[b];
                const int lc = left_count[b - 1];
                if (lc == 0 || cnt == 0) {
                    continue;
                }
                const double cost = left_box[b - 1].area() * lc + acc.area() * cnt;
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = axis;
                    best_bin = b;
                }
            }
        }
        int mid;
        if (best_axis < 0) {
            mid = begin + n / 2;  // coincident centroids: split in index order
        } else {
            const float extent = cb.hi[best_axis] - cb.lo[best_axis];
            auto it = std::partition(prims.begin() + begin, prims.begin() + end, [&](const Prim& p) {
                int b = static_cast<int>(kBins * ((p.c[best_axis] - cb.lo[best_axis]) / extent));
                b = std::min(std::max(b, 0), kBins - 1);
                return b < best_bin;
            });
            mid = static_cast<int>(it - prims.begin());
            if (mid == begin || mid == end) {
                mid = begin + n / 2;
            }
        }
        const int node_index = static_cast<int>(nodes.size());
        nodes.push_back(BvhNode{});
        const Box lb = bounds(begin, mid), rb = bounds(mid, end);
        int left = 0, right = 0;
        if (parallel_levels > 0 && !instance_leaves && end - mid >= kParallelPrims) {
            // the right subtree on its own thread into its own arrays, the left one here
            std::vector<BvhNode> right_nodes;
            std::vector<float4> right_leaves;
            Builder sub{prims, right_nodes, right_leaves, positions, tris};
            sub.leaf_limit = leaf_limit;
            sub.parallel_levels = parallel_levels - 1;
            auto pending = std::async(std::launch::async, [&sub, mid, end, depth] { return sub.build(mid, end, depth + 1); });
            --parallel_levels;
            left = build(begin, mid, depth + 1);
            ++parallel_levels;
            const int sub_root = pending.get();
            // append: node codes move by the nodes before them, leaf codes by the records before them
            const int node_offset = static_cast<int>(nodes.size());
            const uint32_t leaf_offset = static_cast<uint32_t>(leaf_tris.size() / 3);
            const auto moved = [&](int code) {
                if (code >= 0) {
                    return code + node_offset;
                }
                const uint32_t packed = ~static_cast<uint32_t>(code);
                return ~static_cast<int>(packed + (leaf_offset << kLeafCountBits));
            };
            for (BvhNode n : right_nodes) {
                n.d.x = moved(n.d.x);
                n.d.y = moved(n.d.y);
                nodes.push_back(n);
            }
            leaf_tris.insert(leaf_tris.end(), right_leaves.begin(), right_leaves.end());
            right = moved(sub_root);
            max_depth = std::max(max_depth, sub.max_depth);
        } else {
            left = build(begin, mid, depth + 1);
            right = build(mid, end, depth + 1);
        }
        BvhNode& node = nodes[node_index];
        node.a = make_float4(lb.lo[0], lb.hi[0], lb.lo[1], lb.hi[1]);
        node.b = make_float4(rb.lo[0], rb.hi[0], rb.lo[1], rb.hi[1]);
        node.c = make_float4(lb.lo[2], lb.hi[2], rb.lo[2], rb.hi[2]);
        node.d = make_int4(left, right, 0, 0);
        return node_index;
    }
};

// Rounds a double down (dir < 0) or up (dir > 0) to a float.
float round_outward(double x, int dir) {
    float f = static_cast<float>(x);
    if (dir < 0 && static_cast<double>(f) > x) {
        f = std::nextafter(f, -std::numeric_limits<float>::infinity());
    }
    if (dir > 0 && static_cast<double>(f) < x) {
        f = std::nextafter(f, std::numeric_limits<float>::infinity());
    }
    return f;
}

// Object box of a sphere: centre -+ radius, rounded outward.
Box sphere_box(const bf200_scene_desc_v1& d, uint32_t g) {
    const float* centre = d.positions + 3ULL * d.geometries[g].vertex_offset;
    const double r = d.geometries[g].radius;
    Box b;
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = round_outward(static_cast<double>(centre[a]) - r, -1);
        b.hi[a] = round_outward(static_cast<double>(centre[a]) + r, 1);
    }
    return b;
}

// Builds the BLAS of one geometry; returns the root node index. A sphere's BLAS is one node whose
// single leaf is the sphere's record (centre, radius; see kSphereLeaf).
uint32_t build_blas(const bf200_scene_desc_v1& d, uint32_t g, std::vector<BvhNode>& nodes,
                    std::vector<float4>& leaf_tris, uint32_t& depth) {
    const auto& geom = d.geometries[g];
    if (geom.kind == BF200_GEOMETRY_SPHERE) {
        const float* centre = d.positions + 3ULL * geom.vertex_offset;
        const uint32_t first = static_cast<uint32_t>(leaf_tris.size() / 3);
        float marker;
        std::memcpy(&marker, &kSphereLeaf, 4);
        leaf_tris.push_back(make_float4(centre[0], centre[1], centre[2], 0.0F));  // primitive 0
        leaf_tris.push_back(make_float4(geom.radius, 0.0F, 0.0F, marker));
        leaf_tris.push_back(make_float4(0.0F, 0.0F, 0.0F, 0.0F));
        const int leaf = ~static_cast<int>((first << kLeafCountBits) | (kSphereLeafCount - 1U));
        const Box lb = sphere_box(d, g);
        const float inf = std::numeric_limits<float>::infinity();
        const uint32_t root = static_cast<uint32_t>(nodes.size());
        BvhNode node{};
        node.a = make_float4(lb.lo[0], lb.hi[0], lb.lo[1], lb.hi[1]);
        node.b = make_float4(inf, -inf, inf, -inf);
        node.c = make_float4(lb.lo[2], lb.hi[2], inf, -inf);
        node.d = make_int4(leaf, leaf, 0, 0);
        nodes.push_back(node);
        depth = 1;
        return root;
    }
    const float* positions = d.positions + 3ULL * geom.vertex_offset;
    const uint32_t* tris = d.triangles + 3ULL * geom.triangle_offset;
    std::vector<Prim> prims(geom.triangle_count);
    for (uint32_t t = 0; t < geom.triangle_count; ++t) {
        Prim& p = prims[t];
        for (int k = 0; k < 3; ++k) {
            p.box.grow(positions + 3ULL * tris[3ULL * t + k]);
        }
        for (int a = 0; a < 3; ++a) {
            p.c[a] = 0.5F * p.box.lo[a] + 0.5F * p.box.hi[a];
        }
        p.index = t;
    }
    Builder b{prims, nodes, leaf_tris, positions, tris};
    const unsigned threads = std::max(1U, std::thread::hardware_concurrency());
    while ((1U << b.parallel_levels) < threads && b.parallel_levels < 5) {
        ++b.parallel_levels;  // up to 2^levels subtrees in flight, at most 32
    }
    const uint32_t root = static_cast<uint32_t>(nodes.size());
    if (static_cast<int>(prims.size()) <= kLeafSize) {
        nodes.push_back(BvhNode{});
        const Box lb = b.bounds(0, static_cast<int>(prims.size()));
        const int leaf = b.make_leaf(0, static_cast<int>(prims.size()));
        const float inf = std::numeric_limits<float>::infinity();
        BvhNode& node = nodes[root];
        node.a = make_float4(lb.lo[0], lb.hi[0], lb.lo[1], lb.hi[1]);
        node.b = make_float4(inf, -inf, inf, -inf);
        node.c = make_float4(lb.lo[2], lb.hi[2], inf, -inf);
        node.d = make_int4(leaf, leaf, 0, 0);
        depth = 1;
        return root;
    }
    const int r = b.build(0, static_cast<int>(prims.size()), 1);
    depth = b.max_depth;
    return static_cast<uint32_t>(r);
}

// World box of an instance: the object box's eight corners through object_to_world in double,
// padded by 1e-4 of the box's largest coordinate magnitude. Triangles are tested against the
// object-space ray, whose transform rounding moves it by a few ulps of those magnitudes; the pad
// is thousands of times larger, so a world-space cull never drops an instance the object-space
// test would hit.
Box instance_world_box(const Box& object, const float* m4) {
    double lo[3] = {std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
                    std::numeric_limits<double>::infinity()};
    double hi[3] = {-lo[0], -lo[1], -lo[2]};
    for (int corner = 0; corner < 8; ++corner) {
        const double p[3] = {(corner & 1) ? object.hi[0] : object.lo[0], (corner & 2) ? object.hi[1] : object.lo[1],
                             (corner & 4) ? object.hi[2] : object.lo[2]};
        for (int r = 0; r < 3; ++r) {
            const double w = double(m4[4 * r]) * p[0] + double(m4[4 * r + 1]) * p[1] + double(m4[4 * r + 2]) * p[2] +
                             double(m4[4 * r + 3]);
            lo[r] = std::min(lo[r], w);
            hi[r] = std::max(hi[r], w);
        }
    }
    double scale = 0.0;
    for (int r = 0; r < 3; ++r) {
        scale = std::max(scale, std::max(std::fabs(lo[r]), std::fabs(hi[r])));
    }
    const double pad = 1e-4 * scale + 1e-30;
    Box b;
    for (int r = 0; r < 3; ++r) {
        b.lo[r] = round_outward(lo[r] - pad, -1);
        b.hi[r] = round_outward(hi[r] + pad, 1);
    }
    return b;
}

// TLAS over the instances' padded world boxes: binned SAH, one instance per leaf (~instance).
// Returns the BVH2 root index in `nodes`.
int build_tlas(const std::vector<Box>& world, std::vector<BvhNode>& nodes) {
    std::vector<Prim> prims(world.size());
    for (size_t i = 0; i < world.size(); ++i) {
        prims[i].box = world[i];
        for (int a = 0; a < 3; ++a) {
            prims[i].c[a] = 0.5F * world[i].lo[a] + 0.5F * world[i].hi[a];
        }
        prims[i].index = static_cast<uint32_t>(i);
    }
    std::vector<float4> unused;
    Builder b{prims, nodes, unused, nullptr, nullptr};
    b.leaf_limit = 1;
    b.instance_leaves = true;
    return b.build(0, static_cast<int>(prims.size()), 1);
}

// ---------------------------------------------------------------------------------------------
// BVH4 collapse: every BVH4 node takes a BVH2 node's two children and repeatedly opens the
// internal child with the largest box surface area until it holds four children (or only
// leaves). Halving the tree depth halves the dependent node fetches of a traversal.
// ---------------------------------------------------------------------------------------------

struct Collapser {
    const std::vector<BvhNode>& bvh2;
    std::vector<BvhNode4>& out;

    struct Slot {
        int code;
        Box box;
    };

    static Box child_box(const BvhNode& n, int k) {
        Box b;
        if (k == 0) {
            b.lo[0] = n.a.x; b.hi[0] = n.a.y; b.lo[1] = n.a.z; b.hi[1] = n.a.w; b.lo[2] = n.c.x; b.hi[2] = n.c.y;
        } else {
            b.lo[0] = n.b.x; b.hi[0] = n.b.y; b.lo[1] = n.b.z; b.hi[1] = n.b.w; b.lo[2] = n.c.z; b.hi[2] = n.c.w;
        }
        return b;
    }

    static bool empty(const Box& b) { return !(b.lo[0] <= b.hi[0] && b.lo[1] <= b.hi[1] && b.lo[2] <= b.hi[2]); }

    // Builds the BVH4 node for BVH2 node `index`; returns its index in `out`.
    int collapse(int index, uint32_t depth, uint32_t& max_depth) {
        max_depth = std::max(max_depth, depth);
        // at most 4 slots at once: an expansion removes one slot and adds two, from at most 3
        Slot slot_store[6];
        struct {
            Slot* data;
            int count;
            int size() const { return count; }
            Slot& operator[](int k) { return data[k]; }
            void push_back(const Slot& v) { data[count++] = v; }
            void erase_at(int k) {
                for (int m = k + 1; m < count; ++m) {
                    data[m - 1] = data[m];
                }
                --count;
            }
        } slots{slot_store, 0};
        for (int k = 0; k < 2; ++k) {
            const Box b = child_box(bvh2[index], k);
            if (!empty(b)) {
                slots.push_back(Slot{k == 0 ? bvh2[index].d.x : bvh2[index].d.y, b});
            }
        }
        while (slots.size() < 4) {
            int open = -1;
            double best = -1.0;
            for (int k = 0; k < slots.size(); ++k) {
                if (slots[k].code >= 0 && slots[k].box.area() > best) {
                    best = slots[k].box.area();
                    open = k;
                }
            }
            if (open < 0) {
                break;
            }
            const BvhNode& n = bvh2[slots[open].code];
            slots.erase_at(open);
            for (int k = 0; k < 2; ++k) {
                const Box b = child_box(n, k);
                if (!empty(b)) {
                    slots.push_back(Slot{k == 0 ? n.d.x : n.d.y, b});
                }
            }
        }
        const int me = static_cast<int>(out.size());
        out.push_back(BvhNode4{});
        int child[4] = {0, 0, 0, 0};
        for (int k = 0; k < slots.size(); ++k) {
            child[k] = slots[k].code >= 0 ? collapse(slots[k].code, depth + 1, max_depth) : slots[k].code;
        }
        const float inf = std::numeric_limits<float>::infinity();
        float lo[3][4], hi[3][4];
        for (int k = 0; k < 4; ++k) {
            for (int a = 0; a < 3; ++a) {
                lo[a][k] = k < slots.size() ? slots[k].box.lo[a] : inf;
                hi[a][k] = k < slots.size() ? slots[k].box.hi[a] : -inf;
            }
        }
        BvhNode4& node = out[me];
        node.lo_x = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
        node.hi_x = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
        node.lo_y = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
        node.hi_y = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
        node.lo_z = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
        node.hi_z = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
        node.child = make_int4(child[0], child[1], child[2], child[3]);
        node.info = make_int4(static_cast<int>(slots.size()), 0, 0, 0);
        return me;
    }
};

// Structural check of a collapsed BVH4 before upload: every node uses 1..4 slots, every internal
// child index lies inside the array and above its parent's (so no walk can cycle), and every node
// is reached exactly once from the roots.
bool valid_bvh4(const std::vector<BvhNode4>& nodes, const std::vector<uint32_t>& roots) {
    std::vector<uint32_t> refs(nodes.size(), 0);
    for (const uint32_t root : roots) {
        if (root >= nodes.size()) {
            return false;
        }
        ++refs[root];
    }
    for (size_t i = 0; i < nodes.size(); ++i) {
        const int used = nodes[i].info.x;
        if (used < 1 || used > 4) {
            return false;
        }
        const int child[4] = {nodes[i].child.x, nodes[i].child.y, nodes[i].child.z, nodes[i].child.w};
        for (int k = 0; k < used; ++k) {
            if (child[k] >= 0) {
                if (static_cast<size_t>(child[k]) >= nodes.size() || static_cast<size_t>(child[k]) <= i) {
                    return false;
                }
                ++refs[static_cast<size_t>(child[k])];
            }
        }
    }
    for (uint32_t r : refs) {
        if (r != 1) {
            return false;
        }
    }
    return true;
}

template <typename T> blackframe_status upload(bf200_scene* s, const std::vector<T>& host, const T*& out) {
    const size_t bytes = std::max<size_t>(host.size() * sizeof(T), 16);
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        return cuda_fail(s->context, e, "device allocation");
    }
    s->allocations.push_back(p);
    if (!host.empty()) {
        e = cudaMemcpy(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            return cuda_fail(s->context, e, "scene upload");
        }
    }
    out = static_cast<const T*>(p);
    return BLACKFRAME_STATUS_SUCCESS;
}

bool is_black4(const float* v) { return v[0] == 0.0F && v[1] == 0.0F && v[2] == 0.0F && v[3] == 0.0F; }

// FrameScene.cpp:138-195 and AreaLights.hpp:1023-1183: one mesh light of an emissive instance.
bool build_light(const bf200_scene_desc_v1& d, uint32_t inst_index, LightInfo& info,
                 std::vector<float4>& tri_vertices, std::vector<float4>& tri_normals, std::vector<float>& areas,
                 std::vector<float>& cdf, std::string& error) {
    const auto& inst = d.instances[inst_index];
    const auto& geom = d.geometries[inst.geometry_index];
    const float* m = inst.object_to_world;
    constexpr double eps = static_cast<double>(std::numeric_limits<float>::epsilon());
    constexpr double gamma7 = (7.0 * eps) / (1.0 - 7.0 * eps);
    constexpr double underflow = 7.0 * static_cast<double>(std::numeric_limits<float>::denorm_min());
    float max_error[3] = {0.0F, 0.0F, 0.0F};
    std::vector<F3> world(geom.vertex_count);
    for (uint32_t v = 0; v < geom.vertex_count; ++v) {
        const float* p = d.positions + 3ULL * (geom.vertex_offset + v);
        const F3 src{p[0], p[1], p[2]};
        world[v] = transform_point_h(m, src);
        const float s[3] = {src.x, src.y, src.z};
        for (int row = 0; row < 3; ++row) {
            double magnitude = std::abs(static_cast<double>(m[row * 4 + 3]));
            for (int col = 0; col < 3; ++col) {
                magnitude += std::abs(static_cast<double>(m[row * 4 + col])) * std::abs(static_cast<double>(s[col]));
            }
            const double bound = std::fma(gamma7, magnitude, underflow);
            float rounded = static_cast<float>(bound);
            if (static_cast<double>(rounded) < bound) {
                rounded = std::nextafter(rounded, std::numeric_limits<float>::infinity());
            }
            max_error[row] = std::max(max_error[row], rounded);
        }
    }
    info.err_x = max_error[0];
    info.err_y = max_error[1];
    info.err_z = max_error[2];
    info.tri_offset = static_cast<uint32_t>(areas.size());
    info.tri_count = geom.triangle_count;
    float sum = 0.0F, comp = 0.0F;
    std::vector<float> local_areas;
    for (uint32_t t = 0; t < geom.triangle_count; ++t) {
        const uint32_t* tri = d.triangles + 3ULL * (geom.triangle_offset + t);
        const F3 a = world[tri[0]], b = world[tri[1]], c = world[tri[2]];
        F3 n;
        float area;
        if (!triangle_normal(a, b, c, n) || !triangle_area(a, b, c, area)) {
            error = "A mesh-light triangle is not representable.";
            return false;
        }
        tri_vertices.push_back(make_float4(a.x, a.y, a.z, 0.0F));
        tri_vertices.push_back(make_float4(b.x, b.y, b.z, 0.0F));
        tri_vertices.push_back(make_float4(c.x, c.y, c.z, 0.0F));
        tri_normals.push_back(make_float4(n.x, n.y, n.z, 0.0F));
        const float next = sum + area;
        if (std::abs(sum) >= std::abs(area)) {
            comp += (sum - next) + area;
        } else {
            comp += (area - next) + sum;
        }
        sum = next;
        local_areas.push_back(area);
        areas.push_back(area);
    }
    const float total = sum + comp;
    if (!std::isfinite(total) || !(total > 0.0F)) {
        error = "Mesh area-light total area is not representable.";
        return false;
    }
    info.area = total;
    info.inverse_area = 1.0F / total;
    float cumulative = 0.0F;
    for (size_t t = 0; t < local_areas.size(); ++t) {
        float next = 1.0F;
        if (t + 1 != local_areas.size()) {
            const float selection = local_areas[t] / info.area;
            next = cumulative + selection;
            if (!(selection > 0.0F) || !(next > cumulative) || !(next < 1.0F)) {
                error = "Mesh area-light selection probabilities are not distinguishable.";
                return false;
            }
        }
        cumulative = next;
        cdf.push_back(cumulative);
    }
    const auto& mat = d.materials[inst.material_index];
    for (int l = 0; l < 4; ++l) {
        info.radiance[l] = mat.emitted_radiance[l];
    }
    info.instance = inst_index;
    return true;
}

// A 64-bit hash (FNV-1a's step over 8-byte words, then the tail bytes) of everything a
// description holds except its instance transforms: a refit must leave all of it unchanged.
uint64_t description_fingerprint(const bf200_scene_desc_v1& d) {
    uint64_t h = 0xcbf29ce484222325ULL;
    auto mix = [&h](const void* p, size_t bytes) {
        const auto* b = static_cast<const unsigned char*>(p);
        size_t i = 0;
        for (; i + 8 <= bytes; i += 8) {
            uint64_t word;
            std::memcpy(&word, b + i, 8);
            h = (h ^ word) * 0x100000001b3ULL;
            h ^= h >> 29;
        }
        for (; i < bytes; ++i) {
            h = (h ^ b[i]) * 0x100000001b3ULL;
        }
    };
    const uint32_t counts[7] = {d.geometry_count, d.vertex_count, d.triangle_count, d.material_count,
                                d.closure_count, d.instance_count, d.punctual_light_count};
    mix(counts, sizeof(counts));
    mix(d.geometries, sizeof(bf200_geometry_v1) * d.geometry_count);
    mix(d.positions, sizeof(float) * 3 * d.vertex_count);
    mix(d.normals, sizeof(float) * 3 * d.vertex_count);
    if (d.texture_coordinates != nullptr) {
        mix(d.texture_coordinates, sizeof(float) * 2 * d.vertex_count);
    }
    mix(d.triangles, sizeof(uint32_t) * 3 * d.triangle_count);
    mix(d.materials, sizeof(bf200_material_v1) * d.material_count);
    if (d.closures != nullptr) {
        mix(d.closures, sizeof(bf200_closure_v1) * d.closure_count);
    }
    if (d.struct_size >= sizeof(bf200_scene_desc_v1) && d.punctual_lights != nullptr) {
        mix(d.punctual_lights, sizeof(bf200_punctual_light_v1) * d.punctual_light_count);
    }
    for (uint32_t i = 0; i < d.instance_count; ++i) {
        const bf200_instance_v1& inst = d.instances[i];
        const uint32_t fields[5] = {inst.instance_id, inst.object_id, inst.geometry_index, inst.material_index,
                                    inst.visibility_mask};
        mix(fields, sizeof(fields));
    }
    mix(d.wavelength_nanometers, sizeof(d.wavelength_nanometers));
    mix(d.wavelength_pdf, sizeof(d.wavelength_pdf));
    mix(d.environment_radiance, sizeof(d.environment_radiance));
    return h;
}

// The device record of a punctual light after the create() checks of PointLight, DirectionalLight
// and SpotLight (punctual_light_checks); false when they refuse it.
bool punctual_record(const bf200_punctual_light_v1& src, bf200::PunctualLight& out) {
    out = bf200::PunctualLight{};
    out.kind = src.kind;
    out.px = src.position[0], out.py = src.position[1], out.pz = src.position[2];
    out.ex = src.position_error[0], out.ey = src.position_error[1], out.ez = src.position_error[2];
    out.dx = src.direction[0], out.dy = src.direction[1], out.dz = src.direction[2];
    for (int l = 0; l < 4; ++l) {
        out.spectrum[l] = src.spectrum[l];
    }
    out.hard = src.kind == BF200_PUNCTUAL_SPOT && src.inner_half_angle == src.outer_half_angle ? 1U : 0U;
    return punctual_light_checks(src, out.cos_inner, out.cos_outer);
}

blackframe_status validate_desc(bf200_context* c, const bf200_scene_desc_v1* d) {
    if (d == nullptr || d->struct_size < BF200_SCENE_DESC_V1_BASE_SIZE) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "scene description missing or too small");
    }
    if (d->punctual_light_count != 0) {
        if (d->struct_size < sizeof(bf200_scene_desc_v1) || d->punctual_lights == nullptr) {
            return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "punctual lights need the punctual_lights array");
        }
        for (uint32_t k = 0; k < d->punctual_light_count; ++k) {
            bf200::PunctualLight record;
            if (!punctual_record(d->punctual_lights[k], record)) {
                return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT,
                            "punctual light " + std::to_string(k) + " is refused by its light model's checks");
            }
        }
    }
    if (d->instance_count == 0 || d->geometry_count == 0 || d->material_count == 0) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "a scene needs geometry, materials and instances");
    }
    for (uint32_t g = 0; g < d->geometry_count; ++g) {
        const auto& geom = d->geometries[g];
        if (geom.reserved != 0U || geom.kind > BF200_GEOMETRY_SPHERE) {
            return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "unknown geometry kind or reserved field set");
        }
        if (geom.kind == BF200_GEOMETRY_SPHERE) {
            // SphereT::create (Sphere.hpp:303-315): finite centre, finite positive radius
            if (geom.vertex_count != 1U || geom.triangle_count != 0U ||
                geom.vertex_offset + 1ULL > d->vertex_count) {
                return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "a sphere is one centre vertex and no triangles");
            }
            const float* centre = d->positions + 3ULL * geom.vertex_offset;
            if (!std::isfinite(centre[0]) || !std::isfinite(centre[1]) || !std::isfinite(centre[2])) {
                return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "A sphere center must be finite.");
            }
            if (!std::isfinite(geom.radius) || geom.radius <= 0.0F) {
                return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "A sphere radius must be finite and positive.");
            }
            continue;
        }
        if (geom.radius != 0.0F) {
            return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "a triangle mesh has no radius");
        }
        if (geom.vertex_offset + static_cast<uint64_t>(geom.vertex_count) > d->vertex_count ||
            geom.triangle_offset + static_cast<uint64_t>(geom.triangle_count) > d->triangle_count ||
            geom.triangle_count == 0) {
            return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "geometry range outside the scene arrays");
        }
        for (uint32_t t = 0; t < geom.triangle_count; ++t) {
            for (int k = 0; k < 3; ++k) {
                if (d->triangles[3ULL * (geom.triangle_offset + t) + k] >= geom.vertex_count) {
                    return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "triangle vertex index out of range");
                }
            }
        }
    }
    for (uint32_t m = 0; m < d->material_count; ++m) {
        const auto& mat = d->materials[m];
        if (mat.closure_count > bf200::kMaxClosures) {
            return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "a closure mixture holds at most 8 closures");
        }
        if (mat.frame_mode != 0) {
            return fail(c, BLACKFRAME_STATUS_INVALID_STATE, "surface-tangent closure frames are not supported");
        }
        if (mat.closure_count != 0 && static_cast<uint64_t>(mat.closure_offset) + mat.closure_count > d->closure_count) {
            return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "closure index out of range");
        }
        for (uint32_t k = 0; k < mat.closure_count; ++k) {
            const uint32_t kind = d->closures[mat.closure_offset + k].kind;
            if (kind < BF200_CLOSURE_LAMBERTIAN_REFLECTION || kind > BF200_CLOSURE_SPECULAR_TRANSMISSION) {
                return fail(c, BLACKFRAME_STATUS_INVALID_STATE, "closure kind not supported by this backend");
            }
            if (!valid_closure_payload(d->closures[mat.closure_offset + k])) {
                return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT,
                            "material " + std::to_string(m) + " has an invalid closure payload");
            }
        }
        float p[bf200::kMaxClosures], cdf[bf200::kMaxClosures + 1];
        if (!project_component_distribution(mat.component_probabilities, mat.closure_count, p, cdf)) {
            return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT,
                        "material " + std::to_string(m) + " has component probabilities that are not a distribution");
        }
    }
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        const auto& inst = d->instances[i];
        if (inst.geometry_index >= d->geometry_count || inst.material_index >= d->material_count) {
            return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "instance references out of range");
        }
        const float* m = inst.object_to_world;
        if (m[12] != 0.0F || m[13] != 0.0F || m[14] != 0.0F || m[15] != 1.0F) {
            return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "an instance transform must be affine");
        }
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

// Carves the wavefront arrays of `capacity` slots out of one arena starting at `base` (16-byte
// aligned pieces). With base == nullptr only the size is computed. Returns the bytes used.
size_t carve_wavefront(char* base, uint32_t capacity, Wavefront* out) {
    const size_t n = capacity;
    const size_t tiles = (n + kCompactTile - 1) / kCompactTile;
    size_t offset = 0;
    auto take = [&](size_t size) {
        offset = (offset + 255) & ~size_t(255);
        char* r = base == nullptr ? nullptr : base + offset;
        offset += size;
        return r;
    };
    Wavefront w{};
    w.capacity = capacity;
    w.ray_o = reinterpret_cast<float4*>(take(16 * n));
    w.ray_d = reinterpret_cast<float4*>(take(16 * n));
    w.beta = reinterpret_cast<float4*>(take(16 * n));
    w.radiance = reinterpret_cast<float4*>(take(16 * n));
    w.prev = reinterpret_cast<float4*>(take(16 * n));
    w.hit_tb = reinterpret_cast<float4*>(take(16 * n));
    w.shadow_o = reinterpret_cast<float4*>(take(16 * n));
    w.shadow_d = reinterpret_cast<float4*>(take(16 * n));
    w.shadow_c = reinterpret_cast<float4*>(take(16 * n));
    w.path_id = reinterpret_cast<uint64_t*>(take(8 * n));
    w.stream = reinterpret_cast<uint2*>(take(8 * n));
    w.hit_id = reinterpret_cast<uint2*>(take(8 * n));
    w.sobol_index = reinterpret_cast<uint4*>(take(16 * n));
    w.pixel_hash = reinterpret_cast<uint2*>(take(8 * n));
    w.depth = reinterpret_cast<uint32_t*>(take(4 * n));
    w.eta = reinterpret_cast<float*>(take(4 * n));
    w.flags = reinterpret_cast<uint32_t*>(take(4 * n));
    w.status = reinterpret_cast<uint32_t*>(take(4 * n));
    w.mask = reinterpret_cast<uint32_t*>(take(4 * n));
    w.route_queue = reinterpret_cast<uint32_t*>(take(4 * n));
    w.shadow_queue = reinterpret_cast<uint32_t*>(take(4 * n));
    w.state = reinterpret_cast<uint8_t*>(take(n));
    w.route = reinterpret_cast<uint8_t*>(take(n));
    w.shadow_key = reinterpret_cast<uint8_t*>(take(n));
    w.tile_counts = reinterpret_cast<uint32_t*>(take(4 * kCompactMaxRoutes * (tiles == 0 ? 1 : tiles)));
    w.route_offsets = reinterpret_cast<uint32_t*>(take(4 * (kRouteCount + 1)));
    w.shadow_offsets = reinterpret_cast<uint32_t*>(take(4 * 2));
    w.counters = reinterpret_cast<unsigned long long*>(take(16 * sizeof(unsigned long long)));
    if (out != nullptr) {
        *out = w;
    }
    return offset;
}

blackframe_status ensure_capacity(bf200_context* c) {
    if (c->arena != nullptr) {
        return BLACKFRAME_STATUS_SUCCESS;
    }
    const uint32_t n = static_cast<uint32_t>(c->capacity);
    const size_t total = carve_wavefront(nullptr, n, nullptr);
    cudaError_t e = cudaMalloc(&c->arena, total);
    if (e != cudaSuccess) {
        return cuda_fail(c, e, "wavefront allocation");
    }
    carve_wavefront(static_cast<char*>(c->arena), n, &c->w);
    e = cudaMallocHost(&c->pinned_counters, 16 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        return cuda_fail(c, e, "pinned counters");
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

TransportParams make_params(const bf200_transport_options_v1& o) {
    TransportParams p{};
    p.heuristic = o.mis_heuristic;
    for (int i = 0; i < 5; ++i) {
        p.limits[i] = o.depth_limits[i];
    }
    p.roulette = o.roulette_enabled;
    p.roulette_first = o.roulette_first_eligible_depth;
    p.roulette_min = o.roulette_minimum_survival;
    p.roulette_max = o.roulette_maximum_survival;
    return p;
}

blackframe_status validate_options(bf200_context* c, const bf200_transport_options_v1* o) {
    if (o == nullptr || o->struct_size < sizeof(bf200_transport_options_v1)) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "transport options missing or too small");
    }
    if (o->mis_heuristic > 1) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "unknown MIS heuristic");
    }
    if (o->sampler > BF200_SAMPLER_OWEN_SOBOL) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "unknown sampler");
    }
    if (o->sampler == BF200_SAMPLER_OWEN_SOBOL &&
        static_cast<uint64_t>(o->depth_limits[0]) + o->depth_limits[1] + o->depth_limits[2] > 255U) {
        return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE,
                    "the Owen-Sobol sampler carries Sobol dimensions for total path depths up to 255");
    }
    for (int i = 0; i < 4; ++i) {
        if (o->depth_limits[i] > 255) {
            return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "depth limits above 255 are not supported");
        }
    }
    if (o->roulette_enabled != 0) {
        // RussianRoulette.hpp:24-55 (create_enabled)
        if (o->roulette_first_eligible_depth == 0 || !std::isfinite(o->roulette_minimum_survival) ||
            !std::isfinite(o->roulette_maximum_survival) || !(o->roulette_minimum_survival > 0.0F) ||
            !(o->roulette_minimum_survival < 1.0F) ||
            o->roulette_maximum_survival < o->roulette_minimum_survival || o->roulette_maximum_survival > 1.0F) {
            return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "invalid Russian roulette policy");
        }
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

// Owen-Sobol direction heads: one static device table per device, filled on the first trace that
// selects the sampler (a synchronous copy, made before that trace's first launch).
static __device__ uint32_t g_sobol_heads[kDeviceSobolDimensions * 64U];
std::mutex g_sobol_mutex;
const uint32_t* g_sobol_address[64] = {};

blackframe_status sobol_table(bf200_context* c, const bf200_transport_options_v1& o, const uint32_t** out) {
    *out = nullptr;
    if (o.sampler != BF200_SAMPLER_OWEN_SOBOL) {
        return BLACKFRAME_STATUS_SUCCESS;
    }
    if (c->device < 0 || c->device >= 64) {
        return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "device ordinal outside the Sobol table registry");
    }
    std::lock_guard<std::mutex> lock(g_sobol_mutex);
    if (g_sobol_address[c->device] == nullptr) {
        const std::vector<uint32_t>& heads = device_sobol_heads();
        cudaError_t e = cudaMemcpyToSymbol(g_sobol_heads, heads.data(), heads.size() * sizeof(uint32_t));
        void* address = nullptr;
        if (e == cudaSuccess) {
            e = cudaGetSymbolAddress(&address, g_sobol_heads);
        }
        if (e != cudaSuccess) {
            return cuda_fail(c, e, "Sobol direction table");
        }
        g_sobol_address[c->device] = static_cast<const uint32_t*>(address);
    }
    *out = g_sobol_address[c->device];
    return BLACKFRAME_STATUS_SUCCESS;
}

// Camera paths of film samples [first, first + chunk) of a request, radiance per path into `radiance`.
PathSource film_source(const bf200_camera_v1* cam, const bf200_film_request_v1* req, uint64_t first, uint64_t chunk,
                       float4* radiance, const uint32_t* sobol) {
    PathSource src{};
    src.mode = 0;
    src.total = chunk * cam->width * cam->height;
    src.width = cam->width;
    src.height = cam->height;
    src.first_sample = req->first_sample + first;
    src.seed = req->seed;
    for (int a = 0; a < 3; ++a) {
        src.cam_origin[a] = cam->origin[a];
        src.cam_t[a] = cam->tangent[a];
        src.cam_b[a] = cam->bitangent[a];
        src.cam_n[a] = cam->normal[a];
    }
    src.half_width = cam->half_width;
    src.half_height = cam->half_height;
    src.t_min = cam->t_min;
    src.t_max = cam->t_max;
    src.time = cam->time;
    src.mask = cam->mask;
    src.jitter = cam->jitter_mode;
    src.path_radiance = radiance;
    src.sobol = sobol;
    return src;
}

// Samples per film chunk: whole sample passes, at most ~64M paths of radiance per chunk.
uint64_t film_samples_per_chunk(uint64_t pixels, uint64_t samples_per_pixel) {
    const uint64_t max_chunk_paths = 1ULL << 26;
    return std::min<uint64_t>(std::max<uint64_t>(1, max_chunk_paths / pixels), samples_per_pixel);
}

// The persistent wavefront as one CUDA graph: a conditional WHILE node whose body is one iteration
// (the stage kernels and k_iteration_gate, which decides on the device whether another iteration
// runs), so the whole trace is one graph launch with no host round trip per iteration. The gate
// stops at the same iteration bound as the host loop.
blackframe_status run_wavefront_graph(bf200_context* c, const bf200_scene* s, PathSource src,
                                      const TransportParams& p, bf200_report_v1* report,
                                      const AdjointView* adjoint = nullptr) {
    Wavefront& w = c->w;
    cudaStream_t st = c->stream;
    cudaError_t e = cudaMemsetAsync(w.state, 0, w.capacity, st);
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(w.counters, 0, 16 * sizeof(unsigned long long), st);
    }
    if (e == cudaSuccess) {  // counters[6], the first failing path, is a minimum
        e = cudaMemsetAsync(w.counters + 6, 0xFF, sizeof(unsigned long long), st);
    }
    if (e != cudaSuccess) {
        return cuda_fail(c, e, "wavefront reset");
    }
    const uint32_t grid =
        std::max<uint32_t>(1, std::min<uint32_t>((w.capacity + 255U) / 256U, c->sm_count * 8U));
    const uint64_t depth_bound = static_cast<uint64_t>(p.limits[0]) + p.limits[1] + p.limits[2] + 2;
    const uint64_t max_iterations = 64 + 2 * (src.total / w.capacity + 2) * depth_bound;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle loop = 0;
    uint32_t per_iteration = 0;
    e = cudaGraphCreate(&graph, 0);
    if (e == cudaSuccess) {
        e = cudaGraphConditionalHandleCreate(&loop, graph, 1U, cudaGraphCondAssignDefault);
    }
    cudaGraphNode_t node = nullptr;
    cudaGraphNodeParams params{};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = loop;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    if (e == cudaSuccess) {
        e = cudaGraphAddNode(&node, graph, nullptr, 0, &params);
    }
    if (e == cudaSuccess) {
        cudaGraph_t body = params.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        for (int stage = 0; stage < 4 && e == cudaSuccess; ++stage) {
            e = launch_stage(stage, s->view, w, src, p, grid, st, &per_iteration, adjoint);
        }
        if (e == cudaSuccess) {
            e = launch_gate(w, src.total, max_iterations, loop, st);
            ++per_iteration;
        }
        cudaGraph_t captured = nullptr;
        const cudaError_t end = cudaStreamEndCapture(st, &captured);
        if (e == cudaSuccess) {
            e = end;
        }
    }
    if (e == cudaSuccess) {
        e = cudaGraphInstantiate(&exec, graph, 0);
    }
    if (e == cudaSuccess) {
        e = cudaGraphLaunch(exec, st);
    }
    if (e == cudaSuccess) {
        e = launch_retire(w, src, grid, st);
    }
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(c->pinned_counters, w.counters, 16 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            st);
    }
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(st);
    }
    if (exec != nullptr) {
        cudaGraphExecDestroy(exec);
    }
    if (graph != nullptr) {
        cudaGraphDestroy(graph);
    }
    if (e != cudaSuccess) {
        return cuda_fail(c, e, "wavefront graph");
    }
    const unsigned long long* k = c->pinned_counters;
    if (k[10] != 0ULL) {
        return fail(c, BLACKFRAME_STATUS_INVALID_STATE, "the wavefront did not drain within its iteration bound");
    }
    if (report != nullptr) {
        report->struct_size = sizeof(bf200_report_v1);
        report->registered_light_count = s->light_count;
        report->path_count += src.total;
        report->extension_segments += k[3];
        report->shadow_segments += k[4];
        report->failed_lanes += k[5];
        report->terminated_paths += src.total - std::min<uint64_t>(src.total, k[5]);
        report->closure_samples += k[11];
        report->light_samples += k[12];
        report->miss_segments += k[13];
        report->continuation_segments += k[14];
        if (k[5] != 0 && report->first_failure_status == 0) {
            report->first_failure_status = static_cast<uint32_t>(k[7]);
            report->first_failure_path = static_cast<uint32_t>(k[6]);
        }
        report->kernel_launches += k[9] * per_iteration + 1U;
        report->iterations += k[9];
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

// Runs the persistent wavefront until every path of `src` has been traced and retired. Without
// instrumentation the loop runs on the device inside one graph; with it, the host drives every
// iteration so each stage can be timed with events (and profilers, which do not see the kernels of
// a device-side loop, see every launch). `adjoint` makes the run a path-replay adjoint replay.
blackframe_status run_wavefront(bf200_context* c, const bf200_scene* s, PathSource src, const TransportParams& p,
                                bool instrument, bf200_report_v1* report, const AdjointView* adjoint = nullptr) {
    if (!instrument) {
        return run_wavefront_graph(c, s, src, p, report, adjoint);
    }
    Wavefront& w = c->w;
    cudaStream_t st = c->stream;
    cudaError_t e = cudaMemsetAsync(w.state, 0, w.capacity, st);
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(w.counters, 0, 16 * sizeof(unsigned long long), st);
    }
    if (e != cudaSuccess) {
        return cuda_fail(c, e, "wavefront reset");
    }
    // counters[6] holds the minimum failing path id
    static const unsigned long long kNone = ~0ULL;
    cudaMemcpyAsync(w.counters + 6, &kNone, sizeof(kNone), cudaMemcpyHostToDevice, st);
    const uint32_t grid =
        std::max<uint32_t>(1, std::min<uint32_t>((w.capacity + 255U) / 256U, c->sm_count * 8U));
    cudaEvent_t ev[5];
    for (auto& x : ev) {
        cudaEventCreate(&x);
    }
    cudaEvent_t start, stop;
    cudaEventCreate(&start);
    cudaEventCreate(&stop);
    cudaEventRecord(start, st);
    uint64_t iterations = 0, launches = 0, shadow_segments = 0;
    double stage_ms[4] = {0.0, 0.0, 0.0, 0.0};
    // every path finishes within (sum of surface depth limits + 1) extension segments, and a
    // slot hosts at most ceil(total / capacity) + 1 paths: bound the host loop accordingly
    const uint64_t depth_bound = static_cast<uint64_t>(p.limits[0]) + p.limits[1] + p.limits[2] + 2;
    const uint64_t max_iterations = 64 + 2 * (src.total / w.capacity + 2) * depth_bound;
    while (iterations < max_iterations) {
        // the shadow queue and the active count are per iteration
        cudaMemsetAsync(w.counters + 0, 0, sizeof(unsigned long long), st);
        cudaMemsetAsync(w.counters + 2, 0, sizeof(unsigned long long), st);
        uint32_t stage_launches = 0;
        for (int stage = 0; stage < 4 && e == cudaSuccess; ++stage) {
            if (instrument) {
                cudaEventRecord(ev[stage], st);
            }
            e = launch_stage(stage, s->view, w, src, p, grid, st, &stage_launches, adjoint);
        }
        if (instrument) {
            cudaEventRecord(ev[4], st);
        }
        launches += stage_launches;
        ++iterations;
        if (e != cudaSuccess) {
            return cuda_fail(c, e, "wavefront launch");
        }
        e = cudaMemcpyAsync(c->pinned_counters, w.counters, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            st);
        if (e == cudaSuccess) {
            e = cudaStreamSynchronize(st);
        }
        if (e != cudaSuccess) {
            return cuda_fail(c, e, "wavefront iteration");
        }
        if (instrument) {
            for (int stage = 0; stage < 4; ++stage) {
                float ms = 0.0F;
                cudaEventElapsedTime(&ms, ev[stage], ev[stage + 1]);
                stage_ms[stage] += ms;
            }
        }
        shadow_segments += c->pinned_counters[0];
        const unsigned long long active = c->pinned_counters[2];
        const unsigned long long claimed = c->pinned_counters[1];
        if (active == 0 && claimed >= src.total) {
            break;
        }
    }
    if (iterations >= max_iterations) {
        return fail(c, BLACKFRAME_STATUS_INVALID_STATE, "the wavefront did not drain within its iteration bound");
    }
    // retire the last finished slots
    e = launch_retire(w, src, grid, st);
    ++launches;
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(c->pinned_counters, w.counters, 16 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            st);
    }
    cudaEventRecord(stop, st);
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) {
        return cuda_fail(c, e, "wavefront retire");
    }
    float ms = 0.0F;
    cudaEventElapsedTime(&ms, start, stop);
    for (auto& x : ev) {
        cudaEventDestroy(x);
    }
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    if (report != nullptr) {
        report->struct_size = sizeof(bf200_report_v1);
        report->registered_light_count = s->light_count;
        report->path_count += src.total;
        report->extension_segments += c->pinned_counters[3];
        report->shadow_segments += shadow_segments;
        report->failed_lanes += c->pinned_counters[5];
        report->terminated_paths += src.total - std::min<uint64_t>(src.total, c->pinned_counters[5]);
        report->closure_samples += c->pinned_counters[11];
        report->light_samples += c->pinned_counters[12];
        report->miss_segments += c->pinned_counters[13];
        report->continuation_segments += c->pinned_counters[14];
        if (c->pinned_counters[5] != 0 && report->first_failure_status == 0) {
            report->first_failure_status = static_cast<uint32_t>(c->pinned_counters[7]);
            report->first_failure_path = static_cast<uint32_t>(c->pinned_counters[6]);
        }
        report->kernel_launches += launches;
        report->gpu_milliseconds += ms;
        report->regenerate_milliseconds += stage_ms[0];
        report->intersect_milliseconds += stage_ms[1];
        report->shade_milliseconds += stage_ms[2];
        report->occlude_milliseconds += stage_ms[3];
        report->iterations += iterations;
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

}  // namespace

// =============================================================================================
// C ABI
// =============================================================================================

extern "C" {

BF200_EXPORT const char* bf200_build_info(void) noexcept {
    return "bf200 wavefront path tracer, sm_100a, render ABI 1.0";
}

namespace {

// LocalFrame.hpp:32-48 (robust_unit_vector) on the host.
bool host_unit(const float* v, float* out) {
    const float m = std::max({std::abs(v[0]), std::abs(v[1]), std::abs(v[2])});
    if (!std::isfinite(v[0]) || !std::isfinite(v[1]) || !std::isfinite(v[2]) || m == 0.0F) {
        return false;
    }
    const float s[3] = {v[0] / m, v[1] / m, v[2] / m};
    const float magnitude = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    out[0] = s[0] / magnitude;
    out[1] = s[1] / magnitude;
    out[2] = s[2] / magnitude;
    return true;
}

void host_cross(const float* a, const float* b, float* out) {
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
}

}  // namespace

BF200_EXPORT blackframe_status bf200_camera_create(const float origin[3], const float normal[3],
                                                    const float tangent_seed[3], uint32_t width, uint32_t height,
                                                    float vfov, float time, uint32_t jitter_mode,
                                                    bf200_camera_v1* out) noexcept {
    if (origin == nullptr || normal == nullptr || tangent_seed == nullptr || out == nullptr || width == 0 ||
        height == 0 || !std::isfinite(vfov) || vfov <= 0.0F || vfov >= 3.14159265358979323846F) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    // from_normal_and_tangent: robust_unit_normal (LocalFrame.hpp:8-30), then
    // from_unit_normal_and_tangent (LocalFrame.hpp:188-219)
    float n[3], td[3], t[3], b[3];
    {
        const float m = std::max({std::abs(normal[0]), std::abs(normal[1]), std::abs(normal[2])});
        if (m == 0.0F) {
            return BLACKFRAME_STATUS_INVALID_ARGUMENT;
        }
        const float s[3] = {normal[0] / m, normal[1] / m, normal[2] / m};
        const float magnitude = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
        n[0] = s[0] / magnitude;
        n[1] = s[1] / magnitude;
        n[2] = s[2] / magnitude;
    }
    if (!host_unit(tangent_seed, td)) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    const float d = td[0] * n[0] + td[1] * n[1] + td[2] * n[2];
    const float projected[3] = {td[0] - n[0] * d, td[1] - n[1] * d, td[2] - n[2] * d};
    float c[3];
    if (!host_unit(projected, t)) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    host_cross(n, t, c);
    if (!host_unit(c, b)) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    host_cross(b, n, c);
    if (!host_unit(c, t)) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    *out = bf200_camera_v1{};
    for (int a = 0; a < 3; ++a) {
        out->origin[a] = origin[a];
        out->tangent[a] = t[a];
        out->bitangent[a] = b[a];
        out->normal[a] = n[a];
    }
    const float half_height = std::tan(vfov / 2.0F);
    out->half_height = half_height;
    out->half_width = half_height * (static_cast<float>(width) / static_cast<float>(height));
    out->t_min = 0.0F;
    out->t_max = std::numeric_limits<float>::infinity();
    out->time = time;
    out->mask = 0xFFFFFFFFU;
    out->width = width;
    out->height = height;
    out->jitter_mode = jitter_mode;
    return BLACKFRAME_STATUS_SUCCESS;
}

BF200_EXPORT blackframe_status bf200_context_create(int32_t device_ordinal, uint64_t path_capacity,
                                                     bf200_context** out_context) noexcept {
    if (out_context == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    *out_context = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device_ordinal < 0 || device_ordinal >= count) {
        return BLACKFRAME_STATUS_OUT_OF_RANGE;
    }
    auto* c = new (std::nothrow) bf200_context{};
    if (c == nullptr) {
        return BLACKFRAME_STATUS_EXTENSION_FAILURE;
    }
    c->device = device_ordinal;
    cudaSetDevice(device_ordinal);
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device_ordinal) != cudaSuccess || prop.major < 10) {
        delete c;
        return BLACKFRAME_STATUS_INVALID_STATE;
    }
    c->sm_count = static_cast<uint32_t>(prop.multiProcessorCount);
    c->capacity = path_capacity != 0 ? path_capacity : (1ULL << 21);
    if (c->capacity > (1ULL << 26)) {
        delete c;
        return BLACKFRAME_STATUS_OUT_OF_RANGE;
    }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return BLACKFRAME_STATUS_EXTENSION_FAILURE;
    }
    *out_context = c;
    return BLACKFRAME_STATUS_SUCCESS;
}

BF200_EXPORT blackframe_status bf200_context_destroy(bf200_context* c) noexcept {
    if (c == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    cudaSetDevice(c->device);
    if (c->stream != nullptr) {
        cudaStreamSynchronize(c->stream);
        cudaStreamDestroy(c->stream);
    }
    if (c->arena != nullptr) {
        cudaFree(c->arena);
    }
    if (c->pinned_counters != nullptr) {
        cudaFreeHost(c->pinned_counters);
    }
    for (void* p : {c->film_radiance, c->film_staging, c->batch_staging, c->lane_arena, c->adjoint_workspace,
                    c->cone_column}) {
        if (p != nullptr) {
            cudaFree(p);
        }
    }
    for (void* p : c->lane_radiance) {
        if (p != nullptr) {
            cudaFree(p);
        }
    }
    for (cudaStream_t st : c->lane_streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    for (cudaEvent_t ev : c->lane_events) {
        cudaEventDestroy(ev);
    }
    if (c->lane_counters != nullptr) {
        cudaFreeHost(c->lane_counters);
    }
    delete c;
    return BLACKFRAME_STATUS_SUCCESS;
}

BF200_EXPORT const char* bf200_context_last_error(const bf200_context* c) noexcept {
    return c == nullptr ? "null context" : c->last_error.c_str();
}

BF200_EXPORT blackframe_status bf200_scene_create(bf200_context* c, const bf200_scene_desc_v1* d,
                                                   bf200_scene** out_scene) noexcept {
    if (c == nullptr || out_scene == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    *out_scene = nullptr;
    if (const auto st = validate_desc(c, d); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    cudaSetDevice(c->device);
    auto scene = std::make_unique<bf200_scene>();
    scene->context = c;
    using Clock = std::chrono::steady_clock;
    const auto ms_since = [](Clock::time_point t0) {
        return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    };
    const auto t_start = Clock::now();
    bf200_scene_stats_v1& stats = scene->stats;
    stats.struct_size = sizeof(bf200_scene_stats_v1);
    try {
        // BLAS per geometry
        std::vector<BvhNode> nodes;
        std::vector<float4> leaf_tris;
        std::vector<uint4> geom_info(d->geometry_count);
        std::vector<Box> object_box(d->geometry_count);
        std::vector<BvhNode4> nodes4;
        uint32_t blas_depth = 0;
        for (uint32_t g = 0; g < d->geometry_count; ++g) {
            uint32_t depth = 0;
            const auto& geom = d->geometries[g];
            const size_t node_mark = nodes.size(), leaf_mark = leaf_tris.size(), node4_mark = nodes4.size();
            const bool on_device = c->build_mode == BF200_BUILD_DEVICE_LBVH && geom.kind == BF200_GEOMETRY_TRIANGLES &&
                                   geom.triangle_count >= kDeviceBuildMinimum;
            auto t0 = Clock::now();
            uint32_t root = 0;
            if (on_device) {
                const cudaError_t e = build_blas_lbvh(
                    d->positions + 3ULL * geom.vertex_offset, geom.vertex_count, d->triangles + 3ULL * geom.triangle_offset,
                    geom.triangle_count, static_cast<uint32_t>(node_mark), static_cast<uint32_t>(leaf_mark / 3), nodes,
                    leaf_tris, c->stream);
                if (e != cudaSuccess) {
                    return cuda_fail(c, e, "device BLAS build");
                }
                root = static_cast<uint32_t>(node_mark);
            } else {
                root = build_blas(*d, g, nodes, leaf_tris, depth);
            }
            stats.blas_build_ms += ms_since(t0);
            t0 = Clock::now();
            uint32_t depth4 = 1;
            Collapser collapser{nodes, nodes4};
            int root4 = collapser.collapse(static_cast<int>(root), 1, depth4);
            if (on_device && 3 * depth4 + 1 + kEagerInstances + 3 >= static_cast<uint32_t>(kTraversalStack)) {
                // too deep for the traversal stack: this geometry takes the host build
                nodes.resize(node_mark);
                leaf_tris.resize(leaf_mark);
                nodes4.resize(node4_mark);
                root = build_blas(*d, g, nodes, leaf_tris, depth);
                depth4 = 1;
                root4 = collapser.collapse(static_cast<int>(root), 1, depth4);
            } else if (on_device) {
                ++stats.device_built_geometries;
            }
            stats.collapse_ms += ms_since(t0);
            stats.blas_depth = std::max(stats.blas_depth, depth4);
            blas_depth = std::max(blas_depth, 3 * depth4 + 1);  // at most 3 net entries per level
            if (geom.kind == BF200_GEOMETRY_SPHERE) {
                // the sphere's leaf record is the last one this BLAS added
                geom_info[g] = make_uint4(static_cast<uint32_t>(leaf_tris.size() / 3 - 1), 0U,
                                          static_cast<uint32_t>(root4), kGeometrySphere);
                object_box[g] = sphere_box(*d, g);
                continue;
            }
            geom_info[g] = make_uint4(d->geometries[g].vertex_offset, d->geometries[g].triangle_offset,
                                      static_cast<uint32_t>(root4), kGeometryTriangles);
            const uint32_t* local = d->triangles + 3ULL * geom.triangle_offset;
            for (uint32_t t = 0; t < 3 * geom.triangle_count; ++t) {
                object_box[g].grow(d->positions + 3ULL * (geom.vertex_offset + local[t]));
            }
        }
        const auto t_instances = Clock::now();
        // instance ranges on the traversal stack carry 14-bit first indices
        if (d->instance_count >= (1U << 14)) {
            return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "more than 16383 instances");
        }
        // instance level: the padded world box of every instance, tested before its ray transform;
        // beyond kEagerInstances instances a BVH4 over those boxes (TLAS) leads to them
        std::vector<Box> world_boxes(d->instance_count);
        for (uint32_t i = 0; i < d->instance_count; ++i) {
            world_boxes[i] = instance_world_box(object_box[d->instances[i].geometry_index],
                                                d->instances[i].object_to_world);
        }
        int tlas_root = -1;
        uint32_t instance_level_depth = kEagerInstances;  // entries an eager instance pass may push
        if (d->instance_count > kEagerInstances) {
            std::vector<BvhNode> tlas2;
            const int root2 = build_tlas(world_boxes, tlas2);
            uint32_t tlas_depth4 = 1;
            scene->tlas_first = static_cast<uint32_t>(nodes4.size());
            Collapser collapser{tlas2, nodes4};
            tlas_root = collapser.collapse(root2, 1, tlas_depth4);
            instance_level_depth = 3 * tlas_depth4 + 1;
            scene->tlas_nodes.assign(nodes4.begin() + scene->tlas_first, nodes4.end());
        }
        for (const Box& b : object_box) {
            scene->object_boxes.insert(scene->object_boxes.end(), {b.lo[0], b.lo[1], b.lo[2], b.hi[0], b.hi[1], b.hi[2]});
        }
        scene->fingerprint = description_fingerprint(*d);
        std::vector<uint32_t> roots;
        for (const uint4& g : geom_info) {
            roots.push_back(g.z);
        }
        if (tlas_root >= 0) {
            roots.push_back(static_cast<uint32_t>(tlas_root));
        }
        if (!valid_bvh4(nodes4, roots)) {
            return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, "internal error: malformed BVH4");
        }
        if (blas_depth + instance_level_depth + 3 >= kTraversalStack) {
            return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "BLAS deeper than the traversal stack allows");
        }
        std::vector<float4> world_box(2ULL * d->instance_count);
        for (uint32_t i = 0; i < d->instance_count; ++i) {
            const Box& b = world_boxes[i];
            world_box[2ULL * i] = make_float4(b.lo[0], b.lo[1], b.lo[2], 0.0F);
            std::memcpy(&world_box[2ULL * i].w, &d->instances[i].visibility_mask, 4);  // mask bits, not a number
            world_box[2ULL * i + 1] = make_float4(b.hi[0], b.hi[1], b.hi[2], 0.0F);
        }
        scene->node_count = nodes4.size();
        scene->triangle_count = leaf_tris.size() / 3;
        // leaf codes and TLAS node indices must stay inside their traversal-stack tag ranges
        // (first leaf triangle < 2^27, node index < 2^29)
        if (scene->triangle_count >= (1ULL << 27) || nodes4.size() >= (1ULL << 29)) {
            return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "scene exceeds 2^27 triangles or 2^29 BVH nodes");
        }
        // instances, mesh lights (FrameScene.cpp:201-261) and the uniform light sampler
        std::vector<float4> to_object(3ULL * d->instance_count), to_world(3ULL * d->instance_count);
        std::vector<uint4> inst_info(d->instance_count);
        std::vector<uint32_t> normal_offset(d->instance_count);
        uint64_t instance_triangles = 0;  // every instance's triangles, in instance order
        std::vector<LightInfo> lights;
        std::vector<float4> light_vertices, light_normals;
        std::vector<float> light_areas, light_cdf;
        for (uint32_t i = 0; i < d->instance_count; ++i) {
            const auto& inst = d->instances[i];
            for (int r = 0; r < 3; ++r) {
                const float* a = inst.world_to_object + 4 * r;
                const float* b = inst.object_to_world + 4 * r;
                to_object[3ULL * i + r] = make_float4(a[0], a[1], a[2], a[3]);
                to_world[3ULL * i + r] = make_float4(b[0], b[1], b[2], b[3]);
            }
            int orientation = 1;
            if (!transform_orientation(inst.object_to_world, orientation)) {
                return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "instance transform orientation is singular");
            }
            uint32_t light_index = 0x7FFFFFFFU;
            if (is_black4(d->materials[inst.material_index].emitted_radiance) == false &&
                d->geometries[inst.geometry_index].kind == BF200_GEOMETRY_SPHERE) {
                return fail(c, BLACKFRAME_STATUS_INVALID_STATE,
                            "emissive analytic spheres are not supported: lights are meshes (no substitution)");
            }
            if (is_black4(d->materials[inst.material_index].emitted_radiance) == false) {
                LightInfo info{};
                std::string error;
                if (!build_light(*d, i, info, light_vertices, light_normals, light_areas, light_cdf, error)) {
                    return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, error);
                }
                light_index = static_cast<uint32_t>(lights.size());
                lights.push_back(info);
            }
            inst_info[i] = make_uint4(inst.geometry_index, inst.material_index, inst.visibility_mask,
                                      light_index | (orientation < 0 ? 0x80000000U : 0U));
            normal_offset[i] = static_cast<uint32_t>(instance_triangles);
            instance_triangles += d->geometries[inst.geometry_index].triangle_count;
        }
        if (instance_triangles >= (1ULL << 32)) {
            return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "more than 2^32 - 1 instanced triangles");
        }
        // the light registry: punctual lights (slots [0, P)), then the mesh lights
        std::vector<bf200::PunctualLight> punctual(d->punctual_light_count);
        for (uint32_t k = 0; k < d->punctual_light_count; ++k) {
            punctual_record(d->punctual_lights[k], punctual[k]);
        }
        const size_t registry = punctual.size() + lights.size();
        if (registry == 0) {
            return fail(c, BLACKFRAME_STATUS_INVALID_STATE,
                        "MIS requires at least one punctual or emissive mesh light in the committed scene");
        }
        // LightSampler::create_uniform (LightSampler.cpp:574-602)
        std::vector<float> select(registry + 1, 0.0F);
        for (size_t k = 1; k < registry; ++k) {
            select[k] = static_cast<float>(k) / static_cast<float>(registry);
        }
        select[registry] = 1.0F;
        scene->light_count = static_cast<uint32_t>(registry);
        scene->punctual_count = static_cast<uint32_t>(punctual.size());
        scene->material_count = d->material_count;
        // materials: the first closure per material (single-closure routes), every closure and the
        // projected component distribution (the generic route's mixtures)
        std::vector<ClosureData> closures(d->material_count);
        std::vector<ClosureData> mix_closures;
        std::vector<bf200::MixDistribution> mix_dist(d->material_count);
        std::vector<float4> emission(d->material_count);
        std::vector<uint4> material_info(d->material_count);
        bool plain_materials = true;  // every material a single Lambert, conductor or dielectric closure
        for (uint32_t m = 0; m < d->material_count; ++m) {
            const auto& mat = d->materials[m];
            bf200::MixDistribution& dist = mix_dist[m];
            dist = bf200::MixDistribution{};
            dist.closure_offset = static_cast<uint32_t>(mix_closures.size());
            project_component_distribution(mat.component_probabilities, mat.closure_count, dist.p, dist.cdf);
            for (uint32_t k = 0; k < mat.closure_count; ++k) {
                const auto& src = d->closures[mat.closure_offset + k];
                ClosureData cd{};
                cd.kind = src.kind;
                cd.lobes = src.lobes;
                std::memcpy(cd.w, src.weight, sizeof(cd.w));
                std::memcpy(cd.p, src.parameters, sizeof(cd.p));
                mix_closures.push_back(cd);
                if (k == 0) {
                    closures[m] = cd;
                }
            }
            if (mat.closure_count > 1 ||
                (mat.closure_count == 1 && closures[m].kind != kClosureLambert &&
                 closures[m].kind != kClosureConductor && closures[m].kind != kClosureDielectric)) {
                plain_materials = false;
            }
            emission[m] = make_float4(mat.emitted_radiance[0], mat.emitted_radiance[1], mat.emitted_radiance[2],
                                      mat.emitted_radiance[3]);
            uint32_t rotation_bits;
            std::memcpy(&rotation_bits, &mat.tangent_rotation_radians, 4);
            material_info[m] = make_uint4(mat.closure_count, mat.frame_mode, rotation_bits, dist.closure_offset);
        }
        if (mix_closures.empty()) {
            mix_closures.push_back(ClosureData{});
        }
        scene->plain_materials = plain_materials;
        // shading route of a hit on each instance: the kernel specialised for its material's single
        // closure kind, or the generic one (several closures, or another kind)
        std::vector<uint8_t> inst_route(d->instance_count, static_cast<uint8_t>(kRouteGeneric));
        for (uint32_t i = 0; i < d->instance_count; ++i) {
            const uint32_t m = d->instances[i].material_index;
            if (d->materials[m].closure_count != 1) {
                continue;
            }
            switch (closures[m].kind) {
                case kClosureLambert: inst_route[i] = static_cast<uint8_t>(kRouteLambert); break;
                case kClosureConductor: inst_route[i] = static_cast<uint8_t>(kRouteConductor); break;
                case kClosureDielectric: inst_route[i] = static_cast<uint8_t>(kRouteDielectric); break;
                default: break;
            }
        }
        stats.instance_ms = ms_since(t_instances);
        const auto t_upload = Clock::now();
        std::vector<float> positions(d->positions, d->positions + 3ULL * d->vertex_count);
        std::vector<float> normals(d->normals, d->normals + 3ULL * d->vertex_count);
        std::vector<uint32_t> triangles(d->triangles, d->triangles + 3ULL * d->triangle_count);
        SceneView& v = scene->view;
        v.instance_count = d->instance_count;
        v.light_count = scene->light_count;
        v.sphere_count = 0U;
        for (uint32_t g = 0; g < d->geometry_count; ++g) {
            v.sphere_count += d->geometries[g].kind == BF200_GEOMETRY_SPHERE ? 1U : 0U;
        }
        v.tlas_root = tlas_root;
        blackframe_status st = BLACKFRAME_STATUS_SUCCESS;
        auto up = [&](auto& host, auto& dst) {
            if (st == BLACKFRAME_STATUS_SUCCESS) {
                st = upload(scene.get(), host, dst);
            }
        };
        up(to_object, v.inst_to_object);
        up(to_world, v.inst_to_world);
        up(inst_info, v.inst_info);
        up(inst_route, v.inst_route);
        up(world_box, v.inst_world_box);
        up(normal_offset, v.inst_normal_offset);
        up(geom_info, v.geom_info);
        up(positions, v.positions);
        up(normals, v.normals);
        up(triangles, v.triangles);
        up(nodes4, v.nodes);
        up(leaf_tris, v.leaf_tris);
        up(closures, v.closures);
        up(mix_closures, v.mix_closures);
        up(mix_dist, v.mix_dist);
        v.punctual_count = static_cast<uint32_t>(punctual.size());
        if (!punctual.empty()) {
            up(punctual, v.punctual);
        }
        up(emission, v.emission);
        up(material_info, v.material_info);
        up(select, v.light_select_cdf);
        up(lights, v.lights);
        up(light_vertices, v.light_tri_vertices);
        up(light_normals, v.light_tri_normals);
        up(light_areas, v.light_tri_areas);
        up(light_cdf, v.light_tri_cdf);
        scene->instance_triangles = static_cast<uint32_t>(instance_triangles);
        scene->light_triangles = light_areas.size();
        if (st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        v.environment = make_float4(d->environment_radiance[0], d->environment_radiance[1],
                                    d->environment_radiance[2], d->environment_radiance[3]);
        // world-space geometric normals of every instance triangle, on the device
        float4* world_normals = nullptr;
        uint32_t* failures = nullptr;
        cudaError_t e = cudaMalloc(&world_normals, std::max<size_t>(16, instance_triangles * sizeof(float4)));
        if (e == cudaSuccess) {
            scene->allocations.push_back(world_normals);
            e = cudaMalloc(&failures, sizeof(uint32_t));
        }
        if (e == cudaSuccess) {
            scene->allocations.push_back(failures);
            e = cudaMemsetAsync(failures, 0, sizeof(uint32_t), c->stream);
        }
        if (e == cudaSuccess) {
            e = launch_world_normals(v, scene->instance_triangles, world_normals, failures, c->stream);
        }
        uint32_t host_failures = 0;
        if (e == cudaSuccess) {
            e = cudaMemcpyAsync(&host_failures, failures, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream);
        }
        if (e == cudaSuccess) {
            e = cudaStreamSynchronize(c->stream);
        }
        if (e != cudaSuccess) {
            return cuda_fail(c, e, "scene build");
        }
        if (host_failures != 0) {
            return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "a world-space triangle normal is not representable");
        }
        v.world_normals = world_normals;
        scene->normal_failures = failures;
        stats.upload_ms = ms_since(t_upload);
        stats.node_count = nodes4.size();
        stats.leaf_triangle_count = leaf_tris.size() / 3;
        stats.total_ms = ms_since(t_start);
    } catch (const std::bad_alloc&) {
        return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, "scene build exhausted host memory");
    }
    *out_scene = scene.release();
    return BLACKFRAME_STATUS_SUCCESS;
}

BF200_EXPORT blackframe_status bf200_context_batch_lanes(const bf200_context* c, uint32_t* lanes) noexcept {
    if (c == nullptr || lanes == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    *lanes = c->last_batch_lanes;
    return BLACKFRAME_STATUS_SUCCESS;
}

BF200_EXPORT blackframe_status bf200_context_set_build_mode(bf200_context* c, uint32_t mode) noexcept {
    if (c == nullptr || (mode != BF200_BUILD_HOST_SAH && mode != BF200_BUILD_DEVICE_LBVH)) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    c->build_mode = mode;
    return BLACKFRAME_STATUS_SUCCESS;
}

BF200_EXPORT blackframe_status bf200_scene_stats(const bf200_scene* s, bf200_scene_stats_v1* out) noexcept {
    if (s == nullptr || out == nullptr || out->struct_size < sizeof(bf200_scene_stats_v1)) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    *out = s->stats;
    return BLACKFRAME_STATUS_SUCCESS;
}

// Transform-only refit: instance matrices, orientation flags, world boxes, the TLAS boxes (same
// topology, each node the union of its children bottom-up; children follow their parents in the
// node array), mesh lights and the world normals of every instance triangle are recomputed in
// place; the BLASes and every buffer size stay as they are.
BF200_EXPORT blackframe_status bf200_scene_refit(bf200_scene* s, const bf200_scene_desc_v1* d) noexcept {
    if (s == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    bf200_context* c = s->context;
    if (d == nullptr || d->struct_size < BF200_SCENE_DESC_V1_BASE_SIZE || d->geometries == nullptr ||
        d->positions == nullptr || d->normals == nullptr || d->triangles == nullptr || d->materials == nullptr ||
        d->instances == nullptr) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "scene description missing or too small");
    }
    // everything but the transforms was validated when the scene was created and must be unchanged
    if (description_fingerprint(*d) != s->fingerprint) {
        return fail(c, BLACKFRAME_STATUS_INVALID_STATE,
                    "a refit accepts only instance transform changes (no rebuild fallback)");
    }
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        const float* m = d->instances[i].object_to_world;
        if (m[12] != 0.0F || m[13] != 0.0F || m[14] != 0.0F || m[15] != 1.0F) {
            return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "an instance transform must be affine");
        }
    }
    cudaSetDevice(c->device);
    try {
        const uint32_t n = d->instance_count;
        std::vector<float4> to_object(3ULL * n), to_world(3ULL * n), world_box(2ULL * n);
        std::vector<uint4> inst_info(n);
        std::vector<Box> boxes(n);
        std::vector<LightInfo> lights;
        std::vector<float4> light_vertices, light_normals;
        std::vector<float> light_areas, light_cdf;
        for (uint32_t i = 0; i < n; ++i) {
            const auto& inst = d->instances[i];
            for (int r = 0; r < 3; ++r) {
                const float* a = inst.world_to_object + 4 * r;
                const float* b = inst.object_to_world + 4 * r;
                to_object[3ULL * i + r] = make_float4(a[0], a[1], a[2], a[3]);
                to_world[3ULL * i + r] = make_float4(b[0], b[1], b[2], b[3]);
            }
            int orientation = 1;
            if (!transform_orientation(inst.object_to_world, orientation)) {
                return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "instance transform orientation is singular");
            }
            uint32_t light_index = 0x7FFFFFFFU;
            if (!is_black4(d->materials[inst.material_index].emitted_radiance)) {
                LightInfo info{};
                std::string error;
                if (!build_light(*d, i, info, light_vertices, light_normals, light_areas, light_cdf, error)) {
                    return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, error);
                }
                light_index = static_cast<uint32_t>(lights.size());
                lights.push_back(info);
            }
            inst_info[i] = make_uint4(inst.geometry_index, inst.material_index, inst.visibility_mask,
                                      light_index | (orientation < 0 ? 0x80000000U : 0U));
            Box object;
            const float* ob = &s->object_boxes[6ULL * inst.geometry_index];
            for (int a = 0; a < 3; ++a) {
                object.lo[a] = ob[a];
                object.hi[a] = ob[3 + a];
            }
            boxes[i] = instance_world_box(object, inst.object_to_world);
            world_box[2ULL * i] = make_float4(boxes[i].lo[0], boxes[i].lo[1], boxes[i].lo[2], 0.0F);
            std::memcpy(&world_box[2ULL * i].w, &inst.visibility_mask, 4);  // mask bits, not a number
            world_box[2ULL * i + 1] = make_float4(boxes[i].hi[0], boxes[i].hi[1], boxes[i].hi[2], 0.0F);
        }
        if (lights.size() != s->light_count || light_areas.size() != s->light_triangles) {
            return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, "internal error: refit changed the light layout");
        }
        // TLAS refit, deepest nodes first
        std::vector<BvhNode4>& tlas = s->tlas_nodes;
        for (size_t k = tlas.size(); k-- > 0;) {
            BvhNode4& node = tlas[k];
            float* lo_x = &node.lo_x.x;
            float* hi_x = &node.hi_x.x;
            float* lo_y = &node.lo_y.x;
            float* hi_y = &node.hi_y.x;
            float* lo_z = &node.lo_z.x;
            float* hi_z = &node.hi_z.x;
            const int* child = &node.child.x;
            for (int slot = 0; slot < node.info.x; ++slot) {
                Box b;
                if (child[slot] < 0) {
                    b = boxes[static_cast<uint32_t>(~child[slot])];
                } else {
                    const BvhNode4& sub = tlas[static_cast<size_t>(child[slot]) - s->tlas_first];
                    for (int q = 0; q < sub.info.x; ++q) {
                        Box cb;
                        cb.lo[0] = (&sub.lo_x.x)[q], cb.hi[0] = (&sub.hi_x.x)[q];
                        cb.lo[1] = (&sub.lo_y.x)[q], cb.hi[1] = (&sub.hi_y.x)[q];
                        cb.lo[2] = (&sub.lo_z.x)[q], cb.hi[2] = (&sub.hi_z.x)[q];
                        b.grow(cb);
                    }
                }
                lo_x[slot] = b.lo[0], hi_x[slot] = b.hi[0];
                lo_y[slot] = b.lo[1], hi_y[slot] = b.hi[1];
                lo_z[slot] = b.lo[2], hi_z[slot] = b.hi[2];
            }
        }
        SceneView& v = s->view;
        cudaStream_t st = c->stream;
        auto put = [&](auto& host, const void* device) {
            return host.empty() ? cudaSuccess
                                : cudaMemcpyAsync(const_cast<void*>(device), host.data(),
                                                  host.size() * sizeof(host[0]), cudaMemcpyHostToDevice, st);
        };
        cudaError_t e = put(to_object, v.inst_to_object);
        if (e == cudaSuccess) e = put(to_world, v.inst_to_world);
        if (e == cudaSuccess) e = put(inst_info, v.inst_info);
        if (e == cudaSuccess) e = put(world_box, v.inst_world_box);
        if (e == cudaSuccess) e = put(lights, v.lights);
        if (e == cudaSuccess) e = put(light_vertices, v.light_tri_vertices);
        if (e == cudaSuccess) e = put(light_normals, v.light_tri_normals);
        if (e == cudaSuccess) e = put(light_areas, v.light_tri_areas);
        if (e == cudaSuccess) e = put(light_cdf, v.light_tri_cdf);
        if (e == cudaSuccess && !tlas.empty()) {
            e = cudaMemcpyAsync(const_cast<BvhNode4*>(v.nodes) + s->tlas_first, tlas.data(),
                                tlas.size() * sizeof(BvhNode4), cudaMemcpyHostToDevice, st);
        }
        if (e == cudaSuccess) e = cudaMemsetAsync(s->normal_failures, 0, sizeof(uint32_t), st);
        if (e == cudaSuccess) {
            e = launch_world_normals(v, s->instance_triangles, const_cast<float4*>(v.world_normals), s->normal_failures,
                                     st);
        }
        uint32_t failures = 0;
        if (e == cudaSuccess) {
            e = cudaMemcpyAsync(&failures, s->normal_failures, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        }
        if (e == cudaSuccess) {
            e = cudaStreamSynchronize(st);
        }
        if (e != cudaSuccess) {
            return cuda_fail(c, e, "scene refit");
        }
        if (failures != 0) {
            return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "a world-space triangle normal is not representable");
        }
    } catch (const std::bad_alloc&) {
        return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, "scene refit exhausted host memory");
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

BF200_EXPORT blackframe_status bf200_light_power_cdf(const float* spectral_powers, uint32_t light_count,
                                                     float* boundaries) noexcept {
    if (spectral_powers == nullptr || boundaries == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    try {
        std::vector<float> cdf;
        std::string error;
        const blackframe_status st = bf200::light_power_cdf(spectral_powers, light_count, cdf, error);
        if (st == BLACKFRAME_STATUS_SUCCESS) {
            std::memcpy(boundaries, cdf.data(), cdf.size() * sizeof(float));
        }
        return st;
    } catch (const std::bad_alloc&) {
        return BLACKFRAME_STATUS_OUT_OF_RANGE;
    }
}

}  // extern "C"

namespace {

// Frees the scene's light-tree buffers (after the stream that may still read them) and returns the
// scene to selection by its CDF.
void release_light_tree(bf200_scene* s) {
    s->view.tree = nullptr;
    s->view.tree_light_to_node = nullptr;
    if (s->tree_nodes == nullptr && s->tree_map == nullptr) {
        return;
    }
    cudaSetDevice(s->context->device);
    cudaStreamSynchronize(s->context->stream);
    cudaFree(s->tree_nodes);
    cudaFree(s->tree_map);
    s->tree_nodes = s->tree_map = nullptr;
    s->tree_node_bytes = s->tree_map_bytes = 0;
}

// Device buffer of at least `bytes` in `slot` (capacity `held`): reused when it fits, else the old
// one is freed after the stream and a new one allocated.
cudaError_t fit_buffer(bf200_context* c, void*& slot, size_t& held, size_t bytes) {
    if (slot != nullptr && held >= bytes) {
        return cudaSuccess;
    }
    if (slot != nullptr) {
        if (const cudaError_t e = cudaStreamSynchronize(c->stream); e != cudaSuccess) {
            return e;
        }
        cudaFree(slot);
        slot = nullptr;
        held = 0;
    }
    const cudaError_t e = cudaMalloc(&slot, bytes);
    if (e == cudaSuccess) {
        held = bytes;
    } else {
        slot = nullptr;
    }
    return e;
}

}  // namespace

extern "C" {

// Selection by the spatial light tree of `lights` (one input per scene light), or back to the
// scene's CDF when `lights` is null. A new tree reuses the previous tree's device buffers when it
// fits in them; a refused call leaves the scene's selection as it was.
BF200_EXPORT blackframe_status bf200_scene_set_light_tree(bf200_scene* s, const bf200_light_tree_input_v1* lights,
                                                          uint32_t light_count) noexcept {
    if (s == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    bf200_context* c = s->context;
    if (lights == nullptr) {
        release_light_tree(s);
        return BLACKFRAME_STATUS_SUCCESS;
    }
    if (light_count != s->light_count) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "one light-tree input per scene light is required");
    }
    try {
        bf200::LightTree tree;
        std::string error;
        if (const auto st = bf200::build_light_tree(lights, light_count, tree, error); st != BLACKFRAME_STATUS_SUCCESS) {
            return fail(c, st, error);
        }
        if (const cudaError_t e = cudaSetDevice(c->device); e != cudaSuccess) {
            return cuda_fail(c, e, "select the scene's device");
        }
        const size_t node_bytes = tree.nodes.size() * sizeof(bf200::LightTreeNode);
        const size_t map_bytes = tree.light_to_node.size() * sizeof(uint32_t);
        // the stream may still read the old tree: it is replaced only after the stream drained
        // (fit_buffer synchronises before it frees; an in-place rewrite is ordered on the stream)
        cudaError_t e = fit_buffer(c, s->tree_nodes, s->tree_node_bytes, node_bytes);
        if (e == cudaSuccess) {
            e = fit_buffer(c, s->tree_map, s->tree_map_bytes, map_bytes);
        }
        if (e == cudaSuccess) {
            e = cudaMemcpyAsync(s->tree_nodes, tree.nodes.data(), node_bytes, cudaMemcpyHostToDevice, c->stream);
        }
        if (e == cudaSuccess) {
            e = cudaMemcpyAsync(s->tree_map, tree.light_to_node.data(), map_bytes, cudaMemcpyHostToDevice, c->stream);
        }
        if (e == cudaSuccess) {
            e = cudaStreamSynchronize(c->stream);
        }
        if (e != cudaSuccess) {
            release_light_tree(s);  // the buffers' contents are unknown: back to the CDF
            return cuda_fail(c, e, "light-tree upload");
        }
        s->view.tree = static_cast<const bf200::LightTreeNode*>(s->tree_nodes);
        s->view.tree_light_to_node = static_cast<const uint32_t*>(s->tree_map);
        s->view.tree_node_count = static_cast<uint32_t>(tree.nodes.size());
        s->view.tree_root = tree.root;
        s->view.tree_log_extent = tree.root_log_extent;
        s->view.tree_has_extent = tree.root_has_extent ? 1U : 0U;
    } catch (const std::bad_alloc&) {
        return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "light-tree construction exhausted host memory");
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

// The scene's light-selection CDF: power-weighted from `spectral_powers` (4 per light), or uniform
// again (LightSampler::create_uniform) when it is null. Selection by a light tree, if one was set,
// ends once the new CDF is in place; a refused call changes nothing.
BF200_EXPORT blackframe_status bf200_scene_set_light_powers(bf200_scene* s, const float* spectral_powers,
                                                            uint32_t light_count) noexcept {
    if (s == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    bf200_context* c = s->context;
    if (light_count != s->light_count) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "one spectral power per scene light is required");
    }
    try {
        std::vector<float> cdf;
        if (spectral_powers == nullptr) {
            cdf.assign(light_count + 1ULL, 0.0F);
            for (uint32_t k = 1; k < light_count; ++k) {
                cdf[k] = static_cast<float>(k) / static_cast<float>(light_count);
            }
            cdf[light_count] = 1.0F;
        } else {
            std::string error;
            if (const auto st = bf200::light_power_cdf(spectral_powers, light_count, cdf, error);
                st != BLACKFRAME_STATUS_SUCCESS) {
                return fail(c, st, error);
            }
        }
        cudaSetDevice(c->device);
        cudaError_t e = cudaMemcpyAsync(const_cast<float*>(s->view.light_select_cdf), cdf.data(),
                                        cdf.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) {
            e = cudaStreamSynchronize(c->stream);
        }
        if (e != cudaSuccess) {
            return cuda_fail(c, e, "light selection upload");
        }
        release_light_tree(s);  // selection by the CDF this call installed
    } catch (const std::bad_alloc&) {
        return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, "light selection exhausted host memory");
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

// Device bytes the context holds: the wavefront arena and every grow-only workspace of the film,
// batch, cone and adjoint entry points (not its scenes, which own their buffers).
BF200_EXPORT blackframe_status bf200_context_device_bytes(const bf200_context* c, uint64_t* out_bytes) noexcept {
    if (c == nullptr || out_bytes == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    uint64_t bytes = 0;
    if (c->arena != nullptr) {
        Wavefront w{};
        bytes += carve_wavefront(nullptr, static_cast<uint32_t>(c->capacity), &w);
    }
    bytes += c->film_radiance_bytes + c->film_staging_bytes + c->batch_staging_bytes + c->lane_arena_bytes +
             c->adjoint_workspace_bytes + c->cone_column_bytes;
    for (size_t b : c->lane_radiance_bytes) {
        bytes += b;
    }
    *out_bytes = bytes;
    return BLACKFRAME_STATUS_SUCCESS;
}

BF200_EXPORT blackframe_status bf200_scene_destroy(bf200_scene* s) noexcept {
    if (s == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    cudaSetDevice(s->context->device);
    cudaStreamSynchronize(s->context->stream);
    for (void* p : s->allocations) {
        cudaFree(p);
    }
    cudaFree(s->tree_nodes);
    cudaFree(s->tree_map);
    delete s;
    return BLACKFRAME_STATUS_SUCCESS;
}

}  // extern "C"

namespace {

// The batch trace from device inputs to device results. cones_in / cones_out (both or neither)
// carry every path's ray cone through the wavefront; states_in (optional) gives every path's
// depth-zero initial state.
blackframe_status trace_batch_device(bf200_context* c, const bf200_scene* s, const bf200_path_input_v1* device_inputs,
                                     const bf200_path_state_v1* states_in, const float2* cones_in,
                                     uint64_t path_count, const bf200_transport_options_v1* o,
                                     bf200_path_result_v1* device_results, float2* cones_out,
                                     bf200_report_v1* report) {
    if (c == nullptr || s == nullptr || (path_count != 0 && (device_inputs == nullptr || device_results == nullptr))) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    if (s->context != c) {
        return fail(c, BLACKFRAME_STATUS_INVALID_STATE, "scene belongs to another context");
    }
    if (const auto st = validate_options(c, o); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    if (report != nullptr) {
        std::memset(report, 0, sizeof(*report));
    }
    if (path_count == 0) {
        return BLACKFRAME_STATUS_SUCCESS;
    }
    cudaSetDevice(c->device);
    if (const auto st = ensure_capacity(c); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    PathSource src{};
    src.mode = 1;
    src.total = path_count;
    src.inputs = device_inputs;
    src.results = device_results;
    src.states_in = states_in;
    if (cones_in != nullptr) {
        if (const auto st = grow_workspace(c, &c->cone_column, &c->cone_column_bytes, c->capacity * sizeof(float2),
                                           "ray-cone column");
            st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        c->w.cone = static_cast<float2*>(c->cone_column);
        src.cones_in = cones_in;
        src.cones_out = cones_out;
    }
    if (const auto st = sobol_table(c, *o, &src.sobol); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    return run_wavefront(c, s, src, make_params(*o), o->instrumentation != 0, report);
}

// Host arrays to host arrays through the context's batch staging (one 256-byte aligned piece per
// array that is present).
blackframe_status trace_batch_host(bf200_context* c, const bf200_scene* s, const bf200_path_input_v1* inputs,
                                   const bf200_path_state_v1* states_in, const bf200_ray_cone_v1* cones_in,
                                   uint64_t path_count, const bf200_transport_options_v1* o,
                                   bf200_path_result_v1* results, bf200_ray_cone_v1* cones_out,
                                   bf200_report_v1* report) {
    if (path_count == 0) {
        return trace_batch_device(c, s, nullptr, nullptr, nullptr, 0, o, nullptr, nullptr, report);
    }
    cudaSetDevice(c->device);
    const auto span = [](size_t bytes) { return (bytes + 255) & ~size_t(255); };
    const size_t in_bytes = path_count * sizeof(bf200_path_input_v1);
    const size_t out_bytes = path_count * sizeof(bf200_path_result_v1);
    const size_t state_bytes = states_in != nullptr ? path_count * sizeof(bf200_path_state_v1) : 0;
    const size_t cone_bytes = cones_in != nullptr ? path_count * sizeof(bf200_ray_cone_v1) : 0;
    if (const auto st = grow_workspace(c, &c->batch_staging, &c->batch_staging_bytes,
                                       span(in_bytes) + span(out_bytes) + span(state_bytes) + 2 * span(cone_bytes),
                                       "batch staging");
        st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    char* cursor = static_cast<char*>(c->batch_staging);
    const auto take = [&](size_t bytes) {
        char* piece = bytes != 0 ? cursor : nullptr;
        cursor += span(bytes);
        return piece;
    };
    auto* d_in = reinterpret_cast<bf200_path_input_v1*>(take(in_bytes));
    auto* d_out = reinterpret_cast<bf200_path_result_v1*>(take(out_bytes));
    auto* d_states = reinterpret_cast<bf200_path_state_v1*>(take(state_bytes));
    auto* d_cone_in = reinterpret_cast<float2*>(take(cone_bytes));
    auto* d_cone_out = reinterpret_cast<float2*>(take(cone_bytes));
    cudaError_t e = cudaMemcpyAsync(d_in, inputs, in_bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && states_in != nullptr) {
        e = cudaMemcpyAsync(d_states, states_in, state_bytes, cudaMemcpyHostToDevice, c->stream);
    }
    if (e == cudaSuccess && cones_in != nullptr) {
        e = cudaMemcpyAsync(d_cone_in, cones_in, cone_bytes, cudaMemcpyHostToDevice, c->stream);
    }
    blackframe_status st = e == cudaSuccess ? BLACKFRAME_STATUS_SUCCESS : cuda_fail(c, e, "batch upload");
    if (st == BLACKFRAME_STATUS_SUCCESS) {
        st = trace_batch_device(c, s, d_in, d_states, d_cone_in, path_count, o, d_out, d_cone_out, report);
    }
    if (st == BLACKFRAME_STATUS_SUCCESS) {
        e = cudaMemcpyAsync(results, d_out, out_bytes, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess && cones_out != nullptr) {
            e = cudaMemcpyAsync(cones_out, d_cone_out, cone_bytes, cudaMemcpyDeviceToHost, c->stream);
        }
        if (e == cudaSuccess) {
            e = cudaStreamSynchronize(c->stream);
        }
        if (e != cudaSuccess) {
            st = cuda_fail(c, e, "batch download");
        }
    }
    return st;
}

}  // namespace

extern "C" {

BF200_EXPORT blackframe_status bf200_trace_paths_device(bf200_context* c, const bf200_scene* s,
                                                         const bf200_path_input_v1* device_inputs,
                                                         uint64_t path_count, const bf200_transport_options_v1* o,
                                                         bf200_path_result_v1* device_results,
                                                         bf200_report_v1* report) noexcept {
    return trace_batch_device(c, s, device_inputs, nullptr, nullptr, path_count, o, device_results, nullptr, report);
}

BF200_EXPORT blackframe_status bf200_trace_paths_with_cones_device(
    bf200_context* c, const bf200_scene* s, const bf200_path_input_v1* device_inputs,
    const bf200_path_state_v1* device_initial_states, const bf200_ray_cone_v1* device_primary_cones,
    uint64_t path_count, const bf200_transport_options_v1* o, bf200_path_result_v1* device_results,
    bf200_ray_cone_v1* device_terminal_cones, bf200_report_v1* report) noexcept {
    if (path_count != 0 && (device_primary_cones == nullptr || device_terminal_cones == nullptr)) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    return trace_batch_device(c, s, device_inputs, device_initial_states,
                              reinterpret_cast<const float2*>(device_primary_cones), path_count, o, device_results,
                              reinterpret_cast<float2*>(device_terminal_cones), report);
}

BF200_EXPORT blackframe_status bf200_trace_paths_with_cones(bf200_context* c, const bf200_scene* s,
                                                             const bf200_path_input_v1* inputs,
                                                             const bf200_path_state_v1* initial_states,
                                                             const bf200_ray_cone_v1* primary_cones,
                                                             uint64_t path_count, const bf200_transport_options_v1* o,
                                                             bf200_path_result_v1* results,
                                                             bf200_ray_cone_v1* terminal_cones,
                                                             bf200_report_v1* report) noexcept {
    if (c == nullptr || s == nullptr ||
        (path_count != 0 && (inputs == nullptr || results == nullptr || primary_cones == nullptr ||
                             terminal_cones == nullptr))) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    // the reference's preflight: finite non-negative cones and path spectra (WavefrontTransport.cpp:524-566)
    for (uint64_t i = 0; i < path_count; ++i) {
        const bf200_ray_cone_v1& cone = primary_cones[i];
        if (!std::isfinite(cone.width) || cone.width < 0.0F || !std::isfinite(cone.spread) || cone.spread < 0.0F) {
            return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT,
                        "path " + std::to_string(i) + " has a primary ray cone that is not finite and non-negative");
        }
        if (initial_states != nullptr) {
            const bf200_path_state_v1& st = initial_states[i];
            bool valid = std::isfinite(st.eta_scale) && st.eta_scale > 0.0F && st.reserved[0] == 0U &&
                         st.reserved[1] == 0U && st.reserved[2] == 0U;
            for (int l = 0; l < 4; ++l) {
                valid = valid && std::isfinite(st.beta[l]) && st.beta[l] >= 0.0F && std::isfinite(st.radiance[l]) &&
                        st.radiance[l] >= 0.0F;
            }
            if (!valid) {
                return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT,
                            "path " + std::to_string(i) +
                                " has an initial state with a non-finite or negative spectrum or eta scale");
            }
        }
    }
    return trace_batch_host(c, s, inputs, initial_states, primary_cones, path_count, o, results, terminal_cones,
                            report);
}

// ---------------------------------------------------------------------------------------------
// Allocation-free trace: the same wavefront over a scratch array compiled into the library
// ---------------------------------------------------------------------------------------------

}  // extern "C"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[BF200_NOALLOC_SCRATCH_BYTES];

constexpr int kScratchDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_address[kScratchDevices] = {};

// Device address of the scratch array on the context's device, looked up once per device.
blackframe_status noalloc_scratch(bf200_context* c, void** out) {
    if (c->device < 0 || c->device >= kScratchDevices) {
        return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "device ordinal outside the scratch address table");
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_scratch_address[c->device] == nullptr) {
        void* address = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&address, g_noalloc_scratch);
        if (e != cudaSuccess) {
            return cuda_fail(c, e, "scratch symbol address");
        }
        g_scratch_address[c->device] = address;
    }
    *out = g_scratch_address[c->device];
    return BLACKFRAME_STATUS_SUCCESS;
}

// The wavefront loop of run_wavefront without its allocations: no events (no stage timing), and
// the per-iteration counters are read into host stack memory instead of pinned memory.
blackframe_status run_wavefront_noalloc(bf200_context* c, const bf200_scene* s, const Wavefront& w, PathSource src,
                                        const TransportParams& p, bf200_report_v1* report) {
    cudaStream_t st = c->stream;
    // what must start at zero: slot states (all empty) and the counters; the first failing path
    // (counters[6], a minimum) starts at all ones
    cudaError_t e = cudaMemsetAsync(w.state, 0, w.capacity, st);
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(w.counters, 0, 8 * sizeof(unsigned long long), st);
    }
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(w.counters + 6, 0xFF, sizeof(unsigned long long), st);
    }
    if (e != cudaSuccess) {
        return cuda_fail(c, e, "scratch reset");
    }
    const uint32_t grid =
        std::max<uint32_t>(1, std::min<uint32_t>((w.capacity + 255U) / 256U, c->sm_count * 8U));
    unsigned long long counters[8] = {};
    uint64_t iterations = 0, launches = 0, shadow_segments = 0;
    const uint64_t depth_bound = static_cast<uint64_t>(p.limits[0]) + p.limits[1] + p.limits[2] + 2;
    const uint64_t max_iterations = 64 + 2 * (src.total / w.capacity + 2) * depth_bound;
    while (iterations < max_iterations) {
        e = cudaMemsetAsync(w.counters + 0, 0, sizeof(unsigned long long), st);
        if (e == cudaSuccess) {
            e = cudaMemsetAsync(w.counters + 2, 0, sizeof(unsigned long long), st);
        }
        uint32_t stage_launches = 0;
        for (int stage = 0; stage < 4 && e == cudaSuccess; ++stage) {
            e = launch_stage(stage, s->view, w, src, p, grid, st, &stage_launches);
        }
        launches += stage_launches;
        ++iterations;
        if (e != cudaSuccess) {
            return cuda_fail(c, e, "wavefront launch");
        }
        e = cudaMemcpyAsync(counters, w.counters, sizeof(counters), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) {
            e = cudaStreamSynchronize(st);
        }
        if (e != cudaSuccess) {
            return cuda_fail(c, e, "wavefront iteration");
        }
        shadow_segments += counters[0];
        if (counters[2] == 0 && counters[1] >= src.total) {
            break;
        }
    }
    if (iterations >= max_iterations) {
        return fail(c, BLACKFRAME_STATUS_INVALID_STATE, "the wavefront did not drain within its iteration bound");
    }
    e = launch_retire(w, src, grid, st);
    ++launches;
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(counters, w.counters, sizeof(counters), cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) {
        return cuda_fail(c, e, "wavefront retire");
    }
    if (report != nullptr) {
        report->struct_size = sizeof(bf200_report_v1);
        report->registered_light_count = s->light_count;
        report->path_count = src.total;
        report->extension_segments = counters[3];
        report->shadow_segments = shadow_segments;
        report->failed_lanes = counters[5];
        if (counters[5] != 0) {
            report->first_failure_status = static_cast<uint32_t>(counters[7]);
            report->first_failure_path = static_cast<uint32_t>(counters[6]);
        }
        report->kernel_launches = launches;
        report->iterations = iterations;
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

}  // namespace

extern "C" {

BF200_EXPORT blackframe_status bf200_trace_paths_device_noalloc(bf200_context* c, const bf200_scene* s,
                                                                 const bf200_path_input_v1* device_inputs,
                                                                 uint64_t path_count,
                                                                 const bf200_transport_options_v1* o,
                                                                 bf200_path_result_v1* device_results,
                                                                 uint32_t path_capacity,
                                                                 bf200_report_v1* report) noexcept {
    if (c == nullptr || s == nullptr || (path_count != 0 && (device_inputs == nullptr || device_results == nullptr))) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    if (s->context != c) {
        return fail(c, BLACKFRAME_STATUS_INVALID_STATE, "scene belongs to another context");
    }
    if (const auto st = validate_options(c, o); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    if (path_capacity > BF200_NOALLOC_MAX_SLOTS) {
        return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE,
                    "path_capacity exceeds the allocation-free scratch limit of 65536 slots (16 MiB of device scratch)");
    }
    const uint32_t capacity = path_capacity == 0 ? BF200_NOALLOC_MAX_SLOTS : path_capacity;
    if (report != nullptr) {
        std::memset(report, 0, sizeof(*report));
    }
    if (path_count == 0) {
        return BLACKFRAME_STATUS_SUCCESS;
    }
    if (const cudaError_t e = cudaSetDevice(c->device); e != cudaSuccess) {
        return cuda_fail(c, e, "select the context's device");
    }
    void* base = nullptr;
    if (const auto st = noalloc_scratch(c, &base); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    Wavefront w{};
    if (carve_wavefront(static_cast<char*>(base), capacity, &w) > BF200_NOALLOC_SCRATCH_BYTES) {
        return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, "scratch layout exceeds the static scratch array");
    }
    PathSource src{};
    src.mode = 1;
    src.total = path_count;
    src.inputs = device_inputs;
    src.results = device_results;
    if (const auto st = sobol_table(c, *o, &src.sobol); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    return run_wavefront_noalloc(c, s, w, src, make_params(*o), report);
}

BF200_EXPORT blackframe_status bf200_trace_paths(bf200_context* c, const bf200_scene* s,
                                                  const bf200_path_input_v1* inputs, uint64_t path_count,
                                                  const bf200_transport_options_v1* o, bf200_path_result_v1* results,
                                                  bf200_report_v1* report) noexcept {
    if (c == nullptr || s == nullptr || (path_count != 0 && (inputs == nullptr || results == nullptr))) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    return trace_batch_host(c, s, inputs, nullptr, nullptr, path_count, o, results, nullptr, report);
}

BF200_EXPORT blackframe_status bf200_render_film_device(bf200_context* c, const bf200_scene* s,
                                                         const bf200_camera_v1* cam, const bf200_sensor_v1* sensor,
                                                         const bf200_film_request_v1* req,
                                                         const bf200_transport_options_v1* o, bf200_film_v1* film,
                                                         bf200_report_v1* report) noexcept {
    if (c == nullptr || s == nullptr || cam == nullptr || sensor == nullptr || req == nullptr || film == nullptr) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    if (req->struct_size < sizeof(bf200_film_request_v1) || req->precision > 1 || film->precision != req->precision ||
        film->width != cam->width || film->height != cam->height || cam->width == 0 || cam->height == 0 ||
        film->sums == nullptr || film->sample_counts == nullptr) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "inconsistent film request");
    }
    if (const auto st = validate_options(c, o); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    if (report != nullptr) {
        std::memset(report, 0, sizeof(*report));
    }
    cudaSetDevice(c->device);
    if (const auto st = ensure_capacity(c); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    const uint64_t pixels = static_cast<uint64_t>(cam->width) * cam->height;
    if (pixels > 0xFFFFFFFFULL) {
        return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "film too large");
    }
    const uint64_t samples_per_chunk = film_samples_per_chunk(pixels, req->samples_per_pixel);
    const size_t radiance_bytes = std::max<uint64_t>(1, samples_per_chunk * pixels) * sizeof(float4);
    if (const auto st = grow_workspace(c, &c->film_radiance, &c->film_radiance_bytes, radiance_bytes + 256,
                                       "film chunk workspace");
        st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    auto* radiance = static_cast<float4*>(c->film_radiance);
    auto* skipped = reinterpret_cast<unsigned long long*>(static_cast<char*>(c->film_radiance) + radiance_bytes);
    cudaError_t e = cudaMemsetAsync(skipped, 0, sizeof(unsigned long long), c->stream);
    if (e != cudaSuccess) {
        return cuda_fail(c, e, "film chunk workspace");
    }
    const TransportParams params = make_params(*o);
    const uint32_t* sobol = nullptr;
    if (const auto sst = sobol_table(c, *o, &sobol); sst != BLACKFRAME_STATUS_SUCCESS) {
        return sst;
    }
    blackframe_status st = BLACKFRAME_STATUS_SUCCESS;
    for (uint64_t first = 0; first < req->samples_per_pixel && st == BLACKFRAME_STATUS_SUCCESS;
         first += samples_per_chunk) {
        const uint64_t chunk = std::min<uint64_t>(samples_per_chunk, req->samples_per_pixel - first);
        const PathSource src = film_source(cam, req, first, chunk, radiance, sobol);
        st = run_wavefront(c, s, src, params, o->instrumentation != 0, report);
        cudaEvent_t film_start = nullptr, film_stop = nullptr;
        if (st == BLACKFRAME_STATUS_SUCCESS && o->instrumentation != 0) {
            cudaEventCreate(&film_start);
            cudaEventCreate(&film_stop);
            cudaEventRecord(film_start, c->stream);
        }
        if (st == BLACKFRAME_STATUS_SUCCESS) {
            e = launch_film(radiance, static_cast<uint32_t>(pixels), static_cast<uint32_t>(chunk),
                            &sensor->response_xyz[0][0], sensor->wavelength_pdf, sensor->normalization,
                            req->precision, req->precision == 0 ? static_cast<float4*>(film->sums) : nullptr,
                            req->precision == 1 ? static_cast<double*>(film->sums) : nullptr,
                            reinterpret_cast<unsigned long long*>(film->sample_counts), skipped, c->stream);
            if (report != nullptr) {
                report->kernel_launches += 1;
            }
            if (e != cudaSuccess) {
                st = cuda_fail(c, e, "film accumulation");
            }
        }
        if (film_start != nullptr) {
            cudaEventRecord(film_stop, c->stream);
            cudaEventSynchronize(film_stop);
            float fms = 0.0F;
            cudaEventElapsedTime(&fms, film_start, film_stop);
            if (report != nullptr) {
                report->film_milliseconds += fms;
                report->gpu_milliseconds += fms;
            }
            cudaEventDestroy(film_start);
            cudaEventDestroy(film_stop);
        }
    }
    if (st == BLACKFRAME_STATUS_SUCCESS) {
        e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) {
            st = cuda_fail(c, e, "film synchronisation");
        }
    }
    return st;
}

}  // extern "C"

namespace {

// The replay half of the path-replay adjoint, shared by the one-call loss entry point and the
// backward entry point. `film` (device) holds the forward render of `req` and gives every pixel's
// weight; `target` (loss mode) or `image_adjoint` (the caller's dLoss/d(image)) gives the loss
// derivative. Each chunk of paths is traced forward again before its replay, to recover every
// path's radiance (vertices are recomputed, not stored), unless `forward_resident`: the chunk
// buffer still holds the radiance of a forward render that was a single chunk.
blackframe_status adjoint_pass(bf200_context* c, const bf200_scene* s, const bf200_camera_v1* cam,
                               const bf200_sensor_v1* sensor, const bf200_film_request_v1* req,
                               const bf200_transport_options_v1* o, const bf200_film_v1* film, const float* target,
                               const float* image_adjoint, bool forward_resident, bf200_material_gradient_v1* gradients,
                               double* emission_gradient, double* loss_out, bf200_report_v1* retrace_report) {
    const uint64_t pixels = static_cast<uint64_t>(film->width) * film->height;
    const uint64_t samples_per_chunk = film_samples_per_chunk(pixels, req->samples_per_pixel);
    const size_t radiance_bytes = std::max<uint64_t>(1, samples_per_chunk * pixels) * sizeof(float4);
    if (const auto st = grow_workspace(c, &c->film_radiance, &c->film_radiance_bytes, radiance_bytes + 256,
                                       "film chunk workspace");
        st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    // workspace: pixel adjoint | gradient sums + loss | pending scores | shadow scores
    const size_t pixel_bytes = ((pixels * sizeof(float4)) + 255) & ~size_t(255);
    const size_t sum_bytes = ((kAdjointWords + 1) * sizeof(double) + 255) & ~size_t(255);
    const size_t slot_bytes = c->capacity * sizeof(uint4);
    if (const auto st = grow_workspace(c, &c->adjoint_workspace, &c->adjoint_workspace_bytes,
                                       pixel_bytes + sum_bytes + 2 * slot_bytes, "adjoint workspace");
        st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    char* base = static_cast<char*>(c->adjoint_workspace);
    AdjointView av{};
    auto* pixel_adjoint = reinterpret_cast<float4*>(base);
    av.pixel_adjoint = pixel_adjoint;
    av.gradients = reinterpret_cast<double*>(base + pixel_bytes);
    double* loss = av.gradients + kAdjointWords;
    av.pending = reinterpret_cast<uint4*>(base + pixel_bytes + sum_bytes);
    av.shadow_score = reinterpret_cast<uint4*>(base + pixel_bytes + sum_bytes + slot_bytes);
    av.pixels = static_cast<uint32_t>(pixels);
    auto* radiance = static_cast<float4*>(c->film_radiance);
    av.forward = radiance;
    // d(sample rgb)/d(radiance lane): the linear map of k_film (sensor term, then XYZ to linear sRGB)
    static const double kXyzToRgb[3][3] = {{3.2404542, -1.5371385, -0.4985314},
                                           {-0.9692660, 1.8760108, 0.0415560},
                                           {0.0556434, -0.2040259, 1.0572252}};
    for (int ch = 0; ch < 3; ++ch) {
        for (int l = 0; l < 4; ++l) {
            double v = 0.0;
            for (int k = 0; k < 3; ++k) {
                v += kXyzToRgb[ch][k] * sensor->response_xyz[l][k];
            }
            av.lane_rgb[ch][l] = static_cast<float>(v * sensor->normalization / sensor->wavelength_pdf[l]);
        }
    }
    cudaError_t e = cudaMemsetAsync(av.gradients, 0, (kAdjointWords + 1) * sizeof(double), c->stream);
    if (e == cudaSuccess) {
        e = launch_adjoint_image(film->precision == 0U ? static_cast<const float4*>(film->sums) : nullptr,
                                 film->precision == 1U ? static_cast<const double*>(film->sums) : nullptr, target,
                                 image_adjoint, static_cast<uint32_t>(pixels), film->precision, pixel_adjoint, loss,
                                 c->stream);
    }
    if (e != cudaSuccess) {
        return cuda_fail(c, e, "adjoint image");
    }
    const TransportParams params = make_params(*o);
    const uint32_t* sobol = nullptr;
    if (const auto sst = sobol_table(c, *o, &sobol); sst != BLACKFRAME_STATUS_SUCCESS) {
        return sst;
    }
    const bool resident = forward_resident && samples_per_chunk >= req->samples_per_pixel;
    blackframe_status st = BLACKFRAME_STATUS_SUCCESS;
    for (uint64_t first = 0; first < req->samples_per_pixel && st == BLACKFRAME_STATUS_SUCCESS;
         first += samples_per_chunk) {
        const uint64_t chunk = std::min<uint64_t>(samples_per_chunk, req->samples_per_pixel - first);
        const PathSource src = film_source(cam, req, first, chunk, radiance, sobol);
        const bool instrument = o->instrumentation != 0U;
        if (!resident) {
            st = run_wavefront(c, s, src, params, instrument, retrace_report);
        }
        if (st == BLACKFRAME_STATUS_SUCCESS) {
            // pending tags of an earlier replay must not match this chunk's paths
            e = cudaMemsetAsync(av.pending, 0, slot_bytes, c->stream);
            st = e == cudaSuccess ? run_wavefront(c, s, src, params, instrument, nullptr, &av)
                                  : cuda_fail(c, e, "adjoint scores reset");
        }
    }
    if (st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    e = cudaMemcpyAsync(gradients, av.gradients, s->material_count * sizeof(bf200_material_gradient_v1),
                        cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(emission_gradient, av.gradients + kAdjointEmission, sizeof(double),
                            cudaMemcpyDeviceToDevice, c->stream);
    }
    double host_loss = 0.0;
    if (e == cudaSuccess && loss_out != nullptr) {
        e = cudaMemcpyAsync(&host_loss, loss, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    }
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(c->stream);
    }
    if (e != cudaSuccess) {
        return cuda_fail(c, e, "adjoint results");
    }
    if (loss_out != nullptr) {
        *loss_out = host_loss;
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

blackframe_status check_adjoint_scene(bf200_context* c, const bf200_scene* s) {
    if (s->context != c) {
        return fail(c, BLACKFRAME_STATUS_INVALID_STATE, "scene belongs to another context");
    }
    if (s->material_count > kAdjointMaterials) {
        return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "the adjoint takes scenes of at most 64 materials");
    }
    if (s->view.tree != nullptr) {
        return fail(c, BLACKFRAME_STATUS_INVALID_STATE, "the adjoint does not replay light-tree selection");
    }
    if (!s->plain_materials || s->punctual_count != 0U) {
        return fail(c, BLACKFRAME_STATUS_INVALID_STATE,
                    "the adjoint replays single Lambert, GGX conductor or GGX dielectric closures and mesh "
                    "lights only (no closure mixtures, rough-diffuse or specular closures, punctual lights)");
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

}  // namespace

extern "C" {

// One-call loss mode: forward render (film cleared first), L2 loss against the target and replay.
// With a single-chunk film the forward render's radiance is reused and not traced again.
BF200_EXPORT blackframe_status bf200_render_adjoint_device(bf200_context* c, const bf200_scene* s,
                                                            const bf200_camera_v1* cam, const bf200_sensor_v1* sensor,
                                                            const bf200_film_request_v1* req,
                                                            const bf200_transport_options_v1* o, bf200_film_v1* film,
                                                            bf200_adjoint_v1* adj, bf200_report_v1* report) noexcept {
    if (c == nullptr || s == nullptr || cam == nullptr || sensor == nullptr || req == nullptr || film == nullptr ||
        adj == nullptr) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    if (adj->struct_size < sizeof(bf200_adjoint_v1) || adj->reserved != 0U || adj->target == nullptr ||
        adj->gradients == nullptr || adj->emission_gradient == nullptr) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "incomplete adjoint request");
    }
    if (const auto st = check_adjoint_scene(c, s); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    if (film->sums == nullptr || film->sample_counts == nullptr || film->precision > 1U) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "inconsistent film request");
    }
    cudaSetDevice(c->device);
    const uint64_t pixels = static_cast<uint64_t>(film->width) * film->height;
    cudaError_t e = cudaMemsetAsync(film->sums, 0, pixels * (film->precision == 0U ? 16U : 64U), c->stream);
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(film->sample_counts, 0, pixels * 8U, c->stream);
    }
    if (e != cudaSuccess) {
        return cuda_fail(c, e, "adjoint film reset");
    }
    if (const auto st = bf200_render_film_device(c, s, cam, sensor, req, o, film, report);
        st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    return adjoint_pass(c, s, cam, sensor, req, o, film, adj->target, nullptr, true, adj->gradients,
                        adj->emission_gradient, &adj->loss, nullptr);
}

// Backward half of the forward/backward pair (the forward is bf200_render_film_device).
BF200_EXPORT blackframe_status bf200_render_backward_device(
    bf200_context* c, const bf200_scene* s, const bf200_camera_v1* cam, const bf200_sensor_v1* sensor,
    const bf200_film_request_v1* req, const bf200_transport_options_v1* o, const bf200_film_v1* film,
    const float* image_adjoint, bf200_material_gradient_v1* gradients, double* emission_gradient,
    bf200_report_v1* report) noexcept {
    if (c == nullptr || s == nullptr || cam == nullptr || sensor == nullptr || req == nullptr || film == nullptr ||
        image_adjoint == nullptr || gradients == nullptr || emission_gradient == nullptr) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    if (const auto st = check_adjoint_scene(c, s); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    if (req->struct_size < sizeof(bf200_film_request_v1) || req->precision > 1 || film->precision != req->precision ||
        film->width != cam->width || film->height != cam->height || cam->width == 0 || cam->height == 0 ||
        film->sums == nullptr || film->sample_counts == nullptr) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "inconsistent film request");
    }
    if (const auto st = validate_options(c, o); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    if (static_cast<uint64_t>(cam->width) * cam->height > 0xFFFFFFFFULL) {
        return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "film too large");
    }
    if (report != nullptr) {
        std::memset(report, 0, sizeof(*report));
    }
    cudaSetDevice(c->device);
    if (const auto st = ensure_capacity(c); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    return adjoint_pass(c, s, cam, sensor, req, o, film, nullptr, image_adjoint, false, gradients, emission_gradient,
                        nullptr, report);
}

BF200_EXPORT blackframe_status bf200_render_film(bf200_context* c, const bf200_scene* s, const bf200_camera_v1* cam,
                                                  const bf200_sensor_v1* sensor, const bf200_film_request_v1* req,
                                                  const bf200_transport_options_v1* o, bf200_film_v1* host_film,
                                                  bf200_report_v1* report) noexcept {
    if (c == nullptr || host_film == nullptr || host_film->sums == nullptr || host_film->sample_counts == nullptr) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    cudaSetDevice(c->device);
    const uint64_t pixels = static_cast<uint64_t>(host_film->width) * host_film->height;
    const size_t sum_bytes = pixels * (host_film->precision == 0 ? 16 : 64);
    const size_t sum_span = (std::max<size_t>(16, sum_bytes) + 255) & ~size_t(255);
    if (const auto st = grow_workspace(c, &c->film_staging, &c->film_staging_bytes,
                                       sum_span + std::max<size_t>(8, pixels * 8), "film staging");
        st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    void* d_sums = c->film_staging;
    auto* d_counts = reinterpret_cast<uint64_t*>(static_cast<char*>(c->film_staging) + sum_span);
    cudaError_t e = cudaMemcpyAsync(d_sums, host_film->sums, sum_bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(d_counts, host_film->sample_counts, pixels * 8, cudaMemcpyHostToDevice, c->stream);
    }
    blackframe_status st = e == cudaSuccess ? BLACKFRAME_STATUS_SUCCESS : cuda_fail(c, e, "film upload");
    if (st == BLACKFRAME_STATUS_SUCCESS) {
        bf200_film_v1 dev = *host_film;
        dev.sums = d_sums;
        dev.sample_counts = d_counts;
        st = bf200_render_film_device(c, s, cam, sensor, req, o, &dev, report);
    }
    if (st == BLACKFRAME_STATUS_SUCCESS) {
        e = cudaMemcpyAsync(host_film->sums, d_sums, sum_bytes, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) {
            e = cudaMemcpyAsync(host_film->sample_counts, d_counts, pixels * 8, cudaMemcpyDeviceToHost, c->stream);
        }
        if (e == cudaSuccess) {
            e = cudaStreamSynchronize(c->stream);
        }
        if (e != cudaSuccess) {
            st = cuda_fail(c, e, "film download");
        }
    }
    return st;
}

// ---------------------------------------------------------------------------------------------
// Film batches: many jobs' wavefronts in concurrent lanes
// ---------------------------------------------------------------------------------------------

}  // extern "C"

namespace {

constexpr uint32_t kMaxLanes = 16;

struct LaneState {
    int job = -1;   // job index, -1 when idle
    int phase = 0;  // 1: iterating a chunk, 2: chunk end (retire + film) queued
    uint64_t pixels = 0, samples_per_chunk = 0, first = 0, chunk = 0;
    uint64_t iterations = 0, max_iterations = 0, shadow_segments = 0, launches = 0;
    PathSource src{};
    TransportParams params{};
    Wavefront w{};
    uint32_t grid = 1;
    float4* radiance = nullptr;
    unsigned long long* skipped = nullptr;
    unsigned long long* counters = nullptr;  // pinned host copy of the lane's counters
};

// Chooses the lane count from the jobs' path counts: twice as many lanes as it takes for the
// median job to fill a slice of the path slots (one lane's kernels run while the other's host
// round trip completes), at least two whenever there are two jobs, at most eight (past that the
// lanes' slices get small and the kernels' grids shrink). On the 64-scene batch (136 M paths, jobs from 32 k to 33 M
// paths) one B200 measured 1.22x, 1.30x, 1.25x, 1.23x and 1.13x the serial throughput with 2,
// 4, 6, 8 and 16 lanes.
uint32_t autotune_lanes(uint64_t capacity, std::vector<uint64_t> job_paths) {
    const uint32_t jobs = static_cast<uint32_t>(job_paths.size());
    if (jobs <= 1) {
        return 1;
    }
    std::nth_element(job_paths.begin(), job_paths.begin() + jobs / 2, job_paths.end());
    const uint64_t median = std::max<uint64_t>(1, job_paths[jobs / 2]);
    const uint64_t want = (2 * capacity + median - 1) / median;
    return static_cast<uint32_t>(std::min<uint64_t>({std::max<uint64_t>(want, 2), 8, jobs}));
}

cudaError_t lane_iterate(const bf200_scene* s, LaneState& lane, cudaStream_t st, cudaEvent_t ev) {
    cudaError_t e = cudaMemsetAsync(lane.w.counters + 0, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(lane.w.counters + 2, 0, sizeof(unsigned long long), st);
    }
    uint32_t launches = 0;
    for (int stage = 0; stage < 4 && e == cudaSuccess; ++stage) {
        e = launch_stage(stage, s->view, lane.w, lane.src, lane.params, lane.grid, st, &launches);
    }
    lane.launches += launches;
    ++lane.iterations;
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(lane.counters, lane.w.counters, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            st);
    }
    if (e == cudaSuccess) {
        e = cudaEventRecord(ev, st);
    }
    return e;
}

// Sets up the lane's next chunk of its job (camera rays of samples [first, first + chunk)) and
// queues the slot reset and the first iteration.
cudaError_t lane_start_chunk(const bf200_film_job_v1& job, LaneState& lane, cudaStream_t st, cudaEvent_t ev) {
    const bf200_camera_v1* cam = job.camera;
    lane.chunk = std::min<uint64_t>(lane.samples_per_chunk, job.request->samples_per_pixel - lane.first);
    PathSource& src = lane.src;
    const uint32_t* sobol = src.sobol;
    src = PathSource{};
    src.mode = 0;
    src.total = lane.chunk * lane.pixels;
    src.width = cam->width;
    src.height = cam->height;
    src.first_sample = job.request->first_sample + lane.first;
    src.seed = job.request->seed;
    for (int a = 0; a < 3; ++a) {
        src.cam_origin[a] = cam->origin[a];
        src.cam_t[a] = cam->tangent[a];
        src.cam_b[a] = cam->bitangent[a];
        src.cam_n[a] = cam->normal[a];
    }
    src.half_width = cam->half_width;
    src.half_height = cam->half_height;
    src.t_min = cam->t_min;
    src.t_max = cam->t_max;
    src.time = cam->time;
    src.mask = cam->mask;
    src.jitter = cam->jitter_mode;
    src.path_radiance = lane.radiance;
    src.sobol = sobol;
    const TransportParams& p = lane.params;
    const uint64_t depth_bound = static_cast<uint64_t>(p.limits[0]) + p.limits[1] + p.limits[2] + 2;
    lane.max_iterations = 64 + 2 * (src.total / lane.w.capacity + 2) * depth_bound;
    lane.iterations = 0;
    lane.phase = 1;
    cudaError_t e = cudaMemsetAsync(lane.w.state, 0, lane.w.capacity, st);
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(lane.w.counters, 0, 8 * sizeof(unsigned long long), st);
    }
    if (e == cudaSuccess) {  // counters[6], the first failing path, is a minimum
        e = cudaMemsetAsync(lane.w.counters + 6, 0xFF, sizeof(unsigned long long), st);
    }
    return e == cudaSuccess ? lane_iterate(job.scene, lane, st, ev) : e;
}

// Queues the chunk's end: retirement of the last slots, the chunk's film accumulation and the
// final counter readback.
cudaError_t lane_finish_chunk(const bf200_film_job_v1& job, LaneState& lane, cudaStream_t st, cudaEvent_t ev) {
    lane.phase = 2;
    cudaError_t e = launch_retire(lane.w, lane.src, lane.grid, st);
    const bf200_film_request_v1* req = job.request;
    const bf200_sensor_v1* sensor = job.sensor;
    if (e == cudaSuccess) {
        e = launch_film(lane.radiance, static_cast<uint32_t>(lane.pixels), static_cast<uint32_t>(lane.chunk),
                        &sensor->response_xyz[0][0], sensor->wavelength_pdf, sensor->normalization, req->precision,
                        req->precision == 0 ? static_cast<float4*>(job.film->sums) : nullptr,
                        req->precision == 1 ? static_cast<double*>(job.film->sums) : nullptr,
                        reinterpret_cast<unsigned long long*>(job.film->sample_counts), lane.skipped, st);
    }
    lane.launches += 2;
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(lane.counters, lane.w.counters, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            st);
    }
    if (e == cudaSuccess) {
        e = cudaEventRecord(ev, st);
    }
    return e;
}

// Adds a finished chunk to its job's report.
void lane_report(const bf200_film_job_v1& job, const LaneState& lane) {
    bf200_report_v1* r = job.report;
    if (r == nullptr) {
        return;
    }
    r->struct_size = sizeof(bf200_report_v1);
    r->registered_light_count = job.scene->light_count;
    r->path_count += lane.src.total;
    r->extension_segments += lane.counters[3];
    r->shadow_segments += lane.shadow_segments;
    r->failed_lanes += lane.counters[5];
    r->terminated_paths += lane.src.total - std::min<uint64_t>(lane.src.total, lane.counters[5]);
    if (lane.counters[5] != 0 && r->first_failure_status == 0) {
        r->first_failure_status = static_cast<uint32_t>(lane.counters[7]);
        r->first_failure_path = static_cast<uint32_t>(lane.counters[6]);
    }
    r->kernel_launches += lane.launches;
    r->iterations += lane.iterations;
}

}  // namespace

namespace {

// Renders jobs[0, job_count) in lane_count concurrent wavefront lanes (the body of
// bf200_render_films_device once its arguments are checked); returns after every lane drained.
blackframe_status run_batch(bf200_context* c, const bf200_film_job_v1* jobs, uint32_t job_count,
                            uint32_t lane_count) {
    cudaSetDevice(c->device);
    const uint32_t slice = static_cast<uint32_t>(std::max<uint64_t>(4096, (c->capacity / lane_count) & ~4095ULL));
    const size_t slice_bytes = (carve_wavefront(nullptr, slice, nullptr) + 255) & ~size_t(255);
    if (const auto st = grow_workspace(c, &c->lane_arena, &c->lane_arena_bytes, slice_bytes * lane_count,
                                       "batch lane arena");
        st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    while (c->lane_streams.size() < lane_count) {
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, "batch lane stream");
        }
        c->lane_streams.push_back(st);
        c->lane_events.push_back(ev);
        c->lane_radiance.push_back(nullptr);
        c->lane_radiance_bytes.push_back(0);
    }
    if (c->lane_counter_lanes < lane_count) {
        if (c->lane_counters != nullptr) {
            cudaFreeHost(c->lane_counters);
            c->lane_counters = nullptr;
        }
        if (cudaMallocHost(&c->lane_counters, 8 * sizeof(unsigned long long) * kMaxLanes) != cudaSuccess) {
            c->lane_counter_lanes = 0;
            return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, "batch lane counters");
        }
        c->lane_counter_lanes = kMaxLanes;
    }
    // each lane's film chunks: whole sample passes of at most this many paths; every lane's
    // radiance buffer is sized once for the largest chunk of the batch, so no lane reallocates
    // (a cudaFree would stall every lane) while others run
    const uint64_t chunk_paths = std::max<uint64_t>(1ULL << 22, (1ULL << 26) / lane_count);
    size_t radiance_bytes = 256;
    for (uint32_t j = 0; j < job_count; ++j) {
        const uint64_t pixels = static_cast<uint64_t>(jobs[j].camera->width) * jobs[j].camera->height;
        const uint64_t per_chunk = std::min<uint64_t>(std::max<uint64_t>(1, chunk_paths / pixels),
                                                      std::max<uint64_t>(1, jobs[j].request->samples_per_pixel));
        radiance_bytes = std::max<size_t>(radiance_bytes, per_chunk * pixels * sizeof(float4) + 256);
    }
    for (uint32_t k = 0; k < lane_count; ++k) {
        if (const auto st = grow_workspace(c, &c->lane_radiance[k], &c->lane_radiance_bytes[k], radiance_bytes,
                                           "batch lane radiance");
            st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
    }
    std::vector<LaneState> lane(lane_count);
    for (uint32_t k = 0; k < lane_count; ++k) {
        carve_wavefront(static_cast<char*>(c->lane_arena) + slice_bytes * k, slice, &lane[k].w);
        lane[k].grid = std::max<uint32_t>(1, std::min<uint32_t>((slice + 255U) / 256U, c->sm_count * 8U));
        lane[k].counters = c->lane_counters + 8ULL * k;
    }
    blackframe_status status = BLACKFRAME_STATUS_SUCCESS;
    uint32_t next_job = 0, active = 0;
    auto drain = [&]() {
        for (uint32_t k = 0; k < lane_count; ++k) {
            cudaStreamSynchronize(c->lane_streams[k]);
        }
    };
    // starts the next job on an idle lane; false when none is left
    auto start_job = [&](uint32_t k) -> bool {
        if (next_job >= job_count) {
            return false;
        }
        const uint32_t j = next_job++;
        const bf200_film_job_v1& job = jobs[j];
        LaneState& L = lane[k];
        L.job = static_cast<int>(j);
        L.pixels = static_cast<uint64_t>(job.camera->width) * job.camera->height;
        L.samples_per_chunk = std::min<uint64_t>(std::max<uint64_t>(1, chunk_paths / L.pixels),
                                                 std::max<uint64_t>(1, job.request->samples_per_pixel));
        L.first = 0;
        L.params = make_params(*job.options);
        L.shadow_segments = 0;
        L.launches = 0;
        L.radiance = static_cast<float4*>(c->lane_radiance[k]);
        L.skipped = reinterpret_cast<unsigned long long*>(static_cast<char*>(c->lane_radiance[k]) +
                                                          c->lane_radiance_bytes[k] - 256);
        const uint32_t* sobol = nullptr;
        if (sobol_table(c, *job.options, &sobol) != BLACKFRAME_STATUS_SUCCESS) {
            status = BLACKFRAME_STATUS_EXTENSION_FAILURE;
            return false;
        }
        L.src.sobol = sobol;
        if (job.request->samples_per_pixel == 0) {  // nothing to render: done at once
            L.job = -1;
            return true;
        }
        cudaError_t e = cudaMemsetAsync(L.skipped, 0, sizeof(unsigned long long), c->lane_streams[k]);
        if (e == cudaSuccess) {
            e = lane_start_chunk(job, L, c->lane_streams[k], c->lane_events[k]);
        }
        if (e != cudaSuccess) {
            status = cuda_fail(c, e, "batch lane launch");
            return false;
        }
        ++active;
        return true;
    };
    for (uint32_t k = 0; k < lane_count && status == BLACKFRAME_STATUS_SUCCESS; ++k) {
        while (lane[k].job < 0 && start_job(k) && lane[k].job < 0) {
        }
    }
    uint32_t cursor = 0;
    while (active > 0 && status == BLACKFRAME_STATUS_SUCCESS) {
        bool progressed = false;
        for (uint32_t n = 0; n < lane_count && status == BLACKFRAME_STATUS_SUCCESS; ++n) {
            const uint32_t k = (cursor + n) % lane_count;
            LaneState& L = lane[k];
            if (L.job < 0) {
                continue;
            }
            const cudaError_t q = cudaEventQuery(c->lane_events[k]);
            if (q == cudaErrorNotReady) {
                continue;
            }
            if (q != cudaSuccess) {
                status = cuda_fail(c, q, "batch lane");
                break;
            }
            progressed = true;
            const bf200_film_job_v1& job = jobs[static_cast<uint32_t>(L.job)];
            cudaError_t e = cudaSuccess;
            if (L.phase == 1) {
                L.shadow_segments += L.counters[0];
                if (L.counters[2] == 0 && L.counters[1] >= L.src.total) {
                    e = lane_finish_chunk(job, L, c->lane_streams[k], c->lane_events[k]);
                } else if (L.iterations >= L.max_iterations) {
                    status = fail(c, BLACKFRAME_STATUS_INVALID_STATE,
                                  "a batch job's wavefront did not drain within its iteration bound");
                    break;
                } else {
                    e = lane_iterate(job.scene, L, c->lane_streams[k], c->lane_events[k]);
                }
            } else {
                lane_report(job, L);
                L.first += L.chunk;
                if (L.first < job.request->samples_per_pixel) {
                    e = lane_start_chunk(job, L, c->lane_streams[k], c->lane_events[k]);
                } else {
                    L.job = -1;
                    --active;
                    while (L.job < 0 && start_job(k) && L.job < 0) {
                    }
                }
            }
            if (e != cudaSuccess) {
                status = cuda_fail(c, e, "batch lane launch");
            }
        }
        cursor = (cursor + 1) % lane_count;
        if (!progressed) {
            // every lane still busy: poll again (a blocking wait on one lane would leave the lanes
            // that finish meanwhile idle)
            std::this_thread::yield();
        }
    }
    drain();
    return status;
}

}  // namespace

extern "C" {

BF200_EXPORT blackframe_status bf200_render_films_device(bf200_context* c, const bf200_film_job_v1* jobs,
                                                         uint32_t job_count, uint32_t lanes) noexcept {
    if (c == nullptr || (job_count != 0 && jobs == nullptr)) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    std::vector<uint64_t> job_paths(job_count);
    for (uint32_t j = 0; j < job_count; ++j) {
        const bf200_film_job_v1& job = jobs[j];
        const bf200_camera_v1* cam = job.camera;
        const bf200_film_request_v1* req = job.request;
        const bf200_film_v1* film = job.film;
        if (job.struct_size < sizeof(bf200_film_job_v1) || job.scene == nullptr || cam == nullptr ||
            job.sensor == nullptr || req == nullptr || job.options == nullptr || film == nullptr) {
            return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "film job with a missing argument");
        }
        if (job.scene->context != c) {
            return fail(c, BLACKFRAME_STATUS_INVALID_STATE, "film job scene belongs to another context");
        }
        if (req->struct_size < sizeof(bf200_film_request_v1) || req->precision > 1 ||
            film->precision != req->precision || film->width != cam->width || film->height != cam->height ||
            cam->width == 0 || cam->height == 0 || film->sums == nullptr || film->sample_counts == nullptr) {
            return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "inconsistent film request in a batch");
        }
        if (const auto st = validate_options(c, job.options); st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        const uint64_t pixels = static_cast<uint64_t>(cam->width) * cam->height;
        if (pixels > 0xFFFFFFFFULL) {
            return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "film too large");
        }
        job_paths[j] = pixels * req->samples_per_pixel;
    }
    for (uint32_t j = 0; j < job_count; ++j) {
        if (jobs[j].report != nullptr) {
            std::memset(jobs[j].report, 0, sizeof(bf200_report_v1));
        }
    }
    if (job_count == 0) {
        return BLACKFRAME_STATUS_SUCCESS;
    }
    if (lanes != 0) {
        c->last_batch_lanes = std::min<uint32_t>(std::min<uint32_t>(lanes, kMaxLanes), job_count);
        return run_batch(c, jobs, job_count, c->last_batch_lanes);
    }
    // The lane count by measurement: the context keeps the fastest count per job-size class (the
    // binary order of magnitude of the median job's paths). A class seen for the first time is
    // measured on this batch's own jobs when there are enough of them: consecutive groups of jobs
    // run with 2, 4 and 8 lanes, each group timed to its drain, and the count with the highest
    // path rate serves the remaining jobs and later batches. Films do not depend on the lane
    // count, so the measured groups are part of the result. Small batches use the closed-form
    // estimate until a larger batch has measured their class.
    std::vector<uint64_t> sorted = job_paths;
    std::nth_element(sorted.begin(), sorted.begin() + job_count / 2, sorted.end());
    uint32_t size_class = 0;
    for (uint64_t m = std::max<uint64_t>(1, sorted[job_count / 2]); m > 1; m >>= 1) {
        ++size_class;
    }
    const auto known = c->batch_lanes_by_class.find(size_class);
    if (known != c->batch_lanes_by_class.end()) {
        c->last_batch_lanes = std::min<uint32_t>(known->second, job_count);
        return run_batch(c, jobs, job_count, c->last_batch_lanes);
    }
    constexpr uint32_t kCandidates[] = {2, 4, 8};
    const uint32_t group = std::max<uint32_t>(8, job_count / 8);
    if (job_count < 4 * group) {
        c->last_batch_lanes = std::min<uint32_t>(autotune_lanes(c->capacity, job_paths), job_count);
        return run_batch(c, jobs, job_count, c->last_batch_lanes);
    }
    // the measured jobs are the first 3 x group, dealt round-robin to the candidates so that each
    // count sees the same mix of job sizes
    constexpr uint32_t kCount = sizeof(kCandidates) / sizeof(kCandidates[0]);
    const uint32_t measured = kCount * group;
    uint32_t best = kCandidates[0];
    double best_rate = -1.0;
    std::vector<bf200_film_job_v1> dealt(group);
    for (uint32_t k = 0; k < kCount; ++k) {
        uint64_t paths = 0;
        for (uint32_t g = 0; g < group; ++g) {
            dealt[g] = jobs[g * kCount + k];
            paths += job_paths[g * kCount + k];
        }
        const auto t0 = std::chrono::steady_clock::now();
        if (const auto st = run_batch(c, dealt.data(), group, kCandidates[k]); st != BLACKFRAME_STATUS_SUCCESS) {
            return st;
        }
        const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        const double rate = static_cast<double>(paths) / std::max(seconds, 1e-9);
        if (rate > best_rate) {
            best_rate = rate;
            best = kCandidates[k];
        }
    }
    c->batch_lanes_by_class[size_class] = best;
    c->last_batch_lanes = best;
    return run_batch(c, jobs + measured, job_count - measured, std::min<uint32_t>(best, job_count - measured));
}

static blackframe_status run_queries(bf200_context* c, const bf200_scene* s, const bf200_ray_v1* rays, uint64_t n,
                                     bf200_hit_v1* hits, uint32_t* occluded) {
    if (c == nullptr || s == nullptr || (n != 0 && rays == nullptr)) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    if (n == 0) {
        return BLACKFRAME_STATUS_SUCCESS;
    }
    cudaSetDevice(c->device);
    bf200_ray_v1* d_rays = nullptr;
    void* d_out = nullptr;
    const size_t out_bytes = n * (hits != nullptr ? sizeof(bf200_hit_v1) : sizeof(uint32_t));
    cudaError_t e = cudaMalloc(&d_rays, n * sizeof(bf200_ray_v1));
    if (e == cudaSuccess) {
        e = cudaMalloc(&d_out, out_bytes);
    }
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(d_rays, rays, n * sizeof(bf200_ray_v1), cudaMemcpyHostToDevice, c->stream);
    }
    if (e == cudaSuccess) {
        e = launch_queries(s->view, d_rays, n, hits != nullptr ? static_cast<bf200_hit_v1*>(d_out) : nullptr,
                           hits != nullptr ? nullptr : static_cast<uint32_t*>(d_out), c->stream);
    }
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(hits != nullptr ? static_cast<void*>(hits) : static_cast<void*>(occluded), d_out, out_bytes,
                            cudaMemcpyDeviceToHost, c->stream);
    }
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(c->stream);
    }
    cudaFree(d_rays);
    cudaFree(d_out);
    return e == cudaSuccess ? BLACKFRAME_STATUS_SUCCESS : cuda_fail(c, e, "query");
}

BF200_EXPORT blackframe_status bf200_closest_hits(bf200_context* c, const bf200_scene* s, const bf200_ray_v1* rays,
                                                   uint64_t n, bf200_hit_v1* hits) noexcept {
    if (hits == nullptr && n != 0) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null hits");
    }
    return run_queries(c, s, rays, n, hits, nullptr);
}

BF200_EXPORT blackframe_status bf200_occlusions(bf200_context* c, const bf200_scene* s, const bf200_ray_v1* rays,
                                                 uint64_t n, uint32_t* occluded) noexcept {
    if (occluded == nullptr && n != 0) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null output");
    }
    return run_queries(c, s, rays, n, nullptr, occluded);
}

BF200_EXPORT blackframe_status bf200_compact_routes_device(bf200_context* c, const uint8_t* keys, uint32_t n,
                                                           uint32_t routes, uint32_t* queue, uint32_t* offsets) noexcept {
    if (c == nullptr || offsets == nullptr || (n != 0 && (keys == nullptr || queue == nullptr))) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    if (routes == 0U || routes > kCompactMaxRoutes) {
        return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "routes must be 1..4");
    }
    if (cudaSetDevice(c->device) != cudaSuccess) {
        return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, "cudaSetDevice failed");
    }
    const uint32_t tiles = n == 0U ? 1U : (n + kCompactTile - 1U) / kCompactTile;
    uint32_t* tile_counts = nullptr;
    cudaError_t e = cudaMalloc(&tile_counts, static_cast<size_t>(routes) * tiles * sizeof(uint32_t));
    uint32_t launches = 0;
    if (e == cudaSuccess) {
        e = launch_compaction(keys, n, routes, tile_counts, queue, offsets, nullptr, nullptr, c->stream, &launches);
    }
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(c->stream);
    }
    cudaFree(tile_counts);
    return e == cudaSuccess ? BLACKFRAME_STATUS_SUCCESS : cuda_fail(c, e, "route compaction");
}

BF200_EXPORT blackframe_status bf200_camera_rays(bf200_context* c, const bf200_camera_v1* cam,
                                                 const bf200_sample_index_v1* samples, uint64_t n, uint32_t sampler,
                                                 bf200_ray_v1* rays, uint32_t* status) noexcept {
    if (c == nullptr || cam == nullptr || (n != 0 && (samples == nullptr || rays == nullptr || status == nullptr))) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    if (sampler != BF200_SAMPLER_HASH && sampler != BF200_SAMPLER_OWEN_SOBOL) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "unknown sampler");
    }
    if (cam->width == 0U || cam->height == 0U) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "camera without pixels");
    }
    if (n == 0) {
        return BLACKFRAME_STATUS_SUCCESS;
    }
    if (cudaSetDevice(c->device) != cudaSuccess) {
        return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, "cudaSetDevice failed");
    }
    bf200_transport_options_v1 o{};
    o.sampler = sampler;
    const uint32_t* sobol = nullptr;
    if (const auto st = sobol_table(c, o, &sobol); st != BLACKFRAME_STATUS_SUCCESS) {
        return st;
    }
    bf200_film_request_v1 req{};
    const PathSource src = film_source(cam, &req, 0, 0, nullptr, sobol);
    void* d_samples = nullptr;
    void* d_rays = nullptr;
    void* d_status = nullptr;
    cudaError_t e = cudaMalloc(&d_samples, n * sizeof(bf200_sample_index_v1));
    if (e == cudaSuccess) {
        e = cudaMalloc(&d_rays, n * sizeof(bf200_ray_v1));
    }
    if (e == cudaSuccess) {
        e = cudaMalloc(&d_status, n * sizeof(uint32_t));
    }
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(d_samples, samples, n * sizeof(bf200_sample_index_v1), cudaMemcpyHostToDevice, c->stream);
    }
    if (e == cudaSuccess) {
        e = launch_camera_rays(src, static_cast<const bf200_sample_index_v1*>(d_samples), n,
                               static_cast<bf200_ray_v1*>(d_rays), static_cast<uint32_t*>(d_status), c->stream);
    }
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(rays, d_rays, n * sizeof(bf200_ray_v1), cudaMemcpyDeviceToHost, c->stream);
    }
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(status, d_status, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream);
    }
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(c->stream);
    }
    cudaFree(d_samples);
    cudaFree(d_rays);
    cudaFree(d_status);
    return e == cudaSuccess ? BLACKFRAME_STATUS_SUCCESS : cuda_fail(c, e, "camera rays");
}

// --------------------------------------------------------------------------------------------
// Environment-map light (EnvironmentLights.hpp:468-1075): host tables, device batch queries
// --------------------------------------------------------------------------------------------

struct bf200_environment_map {
    bf200_context* context = nullptr;
    bf200::EnvironmentTables tables;
    void* device = nullptr;  // texels, azimuth, cosine, row CDF, column CDFs, densities
    bf200::EnvironmentView view{};
};

namespace {

bool same_packet(const bf200_environment_map* m, const float nanometers[4]) {
    for (int lane = 0; lane < 4; ++lane) {
        if (nanometers[lane] != m->tables.nanometers[lane]) {
            return false;
        }
    }
    return true;
}

// Validates a batch call; on success leaves the map's device current.
blackframe_status environment_batch_check(bf200_context* c, const bf200_environment_map* m,
                                          const float nanometers[4], const void* in, uint64_t n, const void* out) {
    if (c == nullptr || m == nullptr || nanometers == nullptr || (n != 0 && (in == nullptr || out == nullptr))) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    if (m->context != c) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "environment map belongs to another context");
    }
    if (!same_packet(m, nanometers)) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT,
                    "A packet-bound environment map cannot be evaluated at different wavelengths.");
    }
    if (cudaSetDevice(c->device) != cudaSuccess) {
        return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, "cudaSetDevice failed");
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

}  // namespace

BF200_EXPORT blackframe_status bf200_environment_map_create(bf200_context* c, const bf200_environment_map_desc_v1* d,
                                                            bf200_environment_map** out) noexcept {
    if (c == nullptr || d == nullptr || out == nullptr) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    *out = nullptr;
    if (d->struct_size < sizeof(bf200_environment_map_desc_v1)) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "environment map descriptor too small");
    }
    std::unique_ptr<bf200_environment_map> m(new (std::nothrow) bf200_environment_map);
    if (!m) {
        return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "out of host memory");
    }
    const char* message = nullptr;
    int code = bf200::kEnvironmentOk;
    try {
        code = bf200::build_environment_tables(d->width, d->height, d->texels, d->nanometers, d->environment_to_world,
                                               m->tables, message);
    } catch (const std::bad_alloc&) {
        return fail(c, BLACKFRAME_STATUS_OUT_OF_RANGE, "Environment-map distribution exhausted host memory.");
    }
    if (code != bf200::kEnvironmentOk) {
        return fail(c,
                    code == bf200::kEnvironmentExhausted ? BLACKFRAME_STATUS_OUT_OF_RANGE
                                                         : BLACKFRAME_STATUS_INVALID_ARGUMENT,
                    message != nullptr ? message : "invalid environment map");
    }
    const bf200::EnvironmentTables& t = m->tables;
    const size_t parts[6] = {t.texels.size(), t.azimuth.size(), t.cosine.size(), t.row_cdf.size(),
                             t.column_cdfs.size(), t.density.size()};
    const std::vector<float>* sources[6] = {&t.texels, &t.azimuth, &t.cosine, &t.row_cdf, &t.column_cdfs, &t.density};
    size_t total = 0;
    for (const size_t p : parts) {
        total += p;
    }
    if (cudaSetDevice(c->device) != cudaSuccess) {
        return fail(c, BLACKFRAME_STATUS_EXTENSION_FAILURE, "cudaSetDevice failed");
    }
    cudaError_t e = cudaMalloc(&m->device, total * sizeof(float));
    float* base = static_cast<float*>(m->device);
    const float* placed[6] = {};
    size_t offset = 0;
    for (int k = 0; k < 6 && e == cudaSuccess; ++k) {
        placed[k] = base + offset;
        e = cudaMemcpy(base + offset, sources[k]->data(), parts[k] * sizeof(float), cudaMemcpyHostToDevice);
        offset += parts[k];
    }
    if (e != cudaSuccess) {
        cudaFree(m->device);
        m->device = nullptr;
        return cuda_fail(c, e, "environment map upload");
    }
    bf200::EnvironmentView& v = m->view;
    v.width = t.width;
    v.height = t.height;
    v.texels = placed[0];
    v.azimuth = placed[1];
    v.cosine = placed[2];
    v.row_cdf = placed[3];
    v.column_cdfs = placed[4];
    v.density = placed[5];
    for (int k = 0; k < 9; ++k) {
        v.matrix[k] = t.matrix[k];
        v.inverse[k] = t.inverse[k];
    }
    v.black = t.black ? 1U : 0U;
    m->context = c;
    *out = m.release();
    return BLACKFRAME_STATUS_SUCCESS;
}

BF200_EXPORT blackframe_status bf200_environment_map_destroy(bf200_environment_map* m) noexcept {
    if (m == nullptr) {
        return BLACKFRAME_STATUS_SUCCESS;
    }
    if (m->device != nullptr && m->context != nullptr) {
        cudaSetDevice(m->context->device);
        cudaFree(m->device);
    }
    delete m;
    return BLACKFRAME_STATUS_SUCCESS;
}

extern "C++" {
namespace {

// One device batch: copy `in_bytes` in, launch, copy the outputs back, synchronize.
template <typename Launch>
blackframe_status environment_batch(bf200_context* c, const void* in, size_t in_bytes, void* out0, size_t out0_bytes,
                                    void* out1, size_t out1_bytes, Launch launch) {
    void* d_in = nullptr;
    void* d_out0 = nullptr;
    void* d_out1 = nullptr;
    cudaError_t e = cudaMalloc(&d_in, in_bytes);
    if (e == cudaSuccess) {
        e = cudaMalloc(&d_out0, out0_bytes);
    }
    if (e == cudaSuccess && out1 != nullptr) {
        e = cudaMalloc(&d_out1, out1_bytes);
    }
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(d_in, in, in_bytes, cudaMemcpyHostToDevice, c->stream);
    }
    if (e == cudaSuccess) {
        e = launch(d_in, d_out0, d_out1);
    }
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(out0, d_out0, out0_bytes, cudaMemcpyDeviceToHost, c->stream);
    }
    if (e == cudaSuccess && out1 != nullptr) {
        e = cudaMemcpyAsync(out1, d_out1, out1_bytes, cudaMemcpyDeviceToHost, c->stream);
    }
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(c->stream);
    }
    cudaFree(d_in);
    cudaFree(d_out0);
    cudaFree(d_out1);
    return e == cudaSuccess ? BLACKFRAME_STATUS_SUCCESS : cuda_fail(c, e, "environment map query");
}

}  // namespace
}  // extern "C++"

BF200_EXPORT blackframe_status bf200_environment_map_sample(bf200_context* c, const bf200_environment_map* m,
                                                            const float nanometers[4], const float* canonical,
                                                            uint64_t n, bf200_environment_sample_v1* samples) noexcept {
    const blackframe_status st = environment_batch_check(c, m, nanometers, canonical, n, samples);
    if (st != BLACKFRAME_STATUS_SUCCESS || n == 0) {
        return st;
    }
    return environment_batch(c, canonical, n * 2 * sizeof(float), samples, n * sizeof(bf200_environment_sample_v1),
                             nullptr, 0, [&](void* in, void* out0, void*) {
                                 return bf200::launch_environment_sample(
                                     m->view, static_cast<const float2*>(in), n,
                                     static_cast<bf200_environment_sample_v1*>(out0), c->stream);
                             });
}

BF200_EXPORT blackframe_status bf200_environment_map_pdf(bf200_context* c, const bf200_environment_map* m,
                                                         const float nanometers[4], const float* directions,
                                                         uint64_t n, float* pdf, uint32_t* status) noexcept {
    blackframe_status st = environment_batch_check(c, m, nanometers, directions, n, pdf);
    if (st == BLACKFRAME_STATUS_SUCCESS && n != 0 && status == nullptr) {
        st = fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null status");
    }
    if (st != BLACKFRAME_STATUS_SUCCESS || n == 0) {
        return st;
    }
    return environment_batch(c, directions, n * 3 * sizeof(float), pdf, n * sizeof(float), status,
                             n * sizeof(uint32_t), [&](void* in, void* out0, void* out1) {
                                 return bf200::launch_environment_pdf(m->view, static_cast<const float*>(in), n,
                                                                      static_cast<float*>(out0),
                                                                      static_cast<uint32_t*>(out1), c->stream);
                             });
}

BF200_EXPORT blackframe_status bf200_environment_map_le(bf200_context* c, const bf200_environment_map* m,
                                                        const float nanometers[4], const float* directions, uint64_t n,
                                                        float* radiance, uint32_t* status) noexcept {
    blackframe_status st = environment_batch_check(c, m, nanometers, directions, n, radiance);
    if (st == BLACKFRAME_STATUS_SUCCESS && n != 0 && status == nullptr) {
        st = fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null status");
    }
    if (st != BLACKFRAME_STATUS_SUCCESS || n == 0) {
        return st;
    }
    return environment_batch(c, directions, n * 3 * sizeof(float), radiance, n * 4 * sizeof(float), status,
                             n * sizeof(uint32_t), [&](void* in, void* out0, void* out1) {
                                 return bf200::launch_environment_le(m->view, static_cast<const float*>(in), n,
                                                                     static_cast<float4*>(out0),
                                                                     static_cast<uint32_t*>(out1), c->stream);
                             });
}

BF200_EXPORT blackframe_status bf200_environment_map_power(bf200_context* c, const bf200_environment_map* m,
                                                           const float nanometers[4], const float bounds_min[3],
                                                           const float bounds_max[3], float power[4]) noexcept {
    if (c == nullptr || m == nullptr || nanometers == nullptr || bounds_min == nullptr || bounds_max == nullptr ||
        power == nullptr) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, "null argument");
    }
    if (!same_packet(m, nanometers)) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT,
                    "A packet-bound environment map cannot be evaluated at different wavelengths.");
    }
    const char* message = nullptr;
    if (bf200::environment_power(m->tables, bounds_min, bounds_max, power, message) != bf200::kEnvironmentOk) {
        return fail(c, BLACKFRAME_STATUS_INVALID_ARGUMENT, message != nullptr ? message : "invalid bounds");
    }
    return BLACKFRAME_STATUS_SUCCESS;
}

// --------------------------------------------------------------------------------------------
// Extension ABI v1 + XPU v1 enumeration + render interface v1
// --------------------------------------------------------------------------------------------

namespace {

constexpr char kBackendName[] = "bf200 B200 wavefront";
constexpr char kVendorName[] = "NVIDIA";

struct DeviceNames {
    char name[256];
};
DeviceNames g_device_names[64];

blackframe_utf8_view view_of(const char* text) {
    return blackframe_utf8_view{text, static_cast<uint32_t>(std::strlen(text)), 0};
}

blackframe_status xpu_device_count(void*, uint32_t* out) noexcept {
    if (out == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        count = 0;
    }
    *out = static_cast<uint32_t>(std::min(count, 64));
    return BLACKFRAME_STATUS_SUCCESS;
}

blackframe_status xpu_device_descriptor(void*, uint32_t index, blackframe_xpu_device_descriptor_v1* out) noexcept {
    if (out == nullptr || out->struct_size < sizeof(blackframe_xpu_device_descriptor_v1)) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    uint32_t count = 0;
    xpu_device_count(nullptr, &count);
    if (index >= count) {
        return BLACKFRAME_STATUS_OUT_OF_RANGE;
    }
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, static_cast<int>(index)) != cudaSuccess) {
        return BLACKFRAME_STATUS_EXTENSION_FAILURE;
    }
    std::snprintf(g_device_names[index].name, sizeof(g_device_names[index].name), "%s", prop.name);
    uint64_t high = 0, low = 0;
    std::memcpy(&high, prop.uuid.bytes, 8);
    std::memcpy(&low, prop.uuid.bytes + 8, 8);
    *out = blackframe_xpu_device_descriptor_v1{};
    out->struct_size = sizeof(blackframe_xpu_device_descriptor_v1);
    out->kind = BLACKFRAME_XPU_DEVICE_KIND_GPU;
    out->identifier_high = high;
    out->identifier_low = low;
    out->name = view_of(g_device_names[index].name);
    out->vendor = view_of(kVendorName);
    return BLACKFRAME_STATUS_SUCCESS;
}

blackframe_status get_interface(void*, blackframe_interface_id id, uint32_t major, uint32_t, void* out,
                                uint32_t out_size) noexcept {
    if (out == nullptr) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    if (id.high == BLACKFRAME_XPU_BACKEND_INTERFACE_ID_HIGH && id.low == BLACKFRAME_XPU_BACKEND_INTERFACE_ID_LOW) {
        if (out_size < sizeof(blackframe_xpu_backend_api_v1)) {
            return BLACKFRAME_STATUS_INVALID_ARGUMENT;
        }
        if (major != BLACKFRAME_XPU_BACKEND_ABI_MAJOR) {
            return BLACKFRAME_STATUS_UNSUPPORTED_ABI;
        }
        auto* api = static_cast<blackframe_xpu_backend_api_v1*>(out);
        *api = blackframe_xpu_backend_api_v1{};
        api->struct_size = sizeof(blackframe_xpu_backend_api_v1);
        api->abi_major = BLACKFRAME_XPU_BACKEND_ABI_MAJOR;
        api->abi_minor = BLACKFRAME_XPU_BACKEND_ABI_MINOR;
        api->backend_name = view_of(kBackendName);
        api->get_device_count = &xpu_device_count;
        api->get_device_descriptor = &xpu_device_descriptor;
        return BLACKFRAME_STATUS_SUCCESS;
    }
    if (id.high == BF200_RENDER_INTERFACE_ID_HIGH && id.low == BF200_RENDER_INTERFACE_ID_LOW) {
        if (out_size < sizeof(bf200_render_api_v1)) {
            return BLACKFRAME_STATUS_INVALID_ARGUMENT;
        }
        if (major != BF200_RENDER_ABI_MAJOR) {
            return BLACKFRAME_STATUS_UNSUPPORTED_ABI;
        }
        auto* api = static_cast<bf200_render_api_v1*>(out);
        *api = bf200_render_api_v1{};
        api->struct_size = sizeof(bf200_render_api_v1);
        api->abi_major = BF200_RENDER_ABI_MAJOR;
        api->abi_minor = BF200_RENDER_ABI_MINOR;
        api->context_create = &bf200_context_create;
        api->context_destroy = &bf200_context_destroy;
        api->context_last_error = &bf200_context_last_error;
        api->scene_create = &bf200_scene_create;
        api->scene_destroy = &bf200_scene_destroy;
        api->trace_paths = &bf200_trace_paths;
        api->render_film = &bf200_render_film;
        api->closest_hits = &bf200_closest_hits;
        api->occlusions = &bf200_occlusions;
        api->scene_create_from_soa = &bf200_scene_create_from_soa;
        api->trace_paths_with_cones = &bf200_trace_paths_with_cones;
        return BLACKFRAME_STATUS_SUCCESS;
    }
    return BLACKFRAME_STATUS_INTERFACE_NOT_FOUND;
}

void shutdown_extension(void*) noexcept {}

}  // namespace

BF200_EXPORT blackframe_status blackframe_query_extension(const blackframe_extension_query_v1* query,
                                                           blackframe_extension_api_v1* out) noexcept {
    if (query == nullptr || out == nullptr || query->struct_size < sizeof(blackframe_extension_query_v1) ||
        out->struct_size < sizeof(blackframe_extension_api_v1)) {
        return BLACKFRAME_STATUS_INVALID_ARGUMENT;
    }
    if (query->abi_major != BLACKFRAME_EXTENSION_ABI_MAJOR) {
        return BLACKFRAME_STATUS_UNSUPPORTED_ABI;
    }
    *out = blackframe_extension_api_v1{};
    out->struct_size = sizeof(blackframe_extension_api_v1);
    out->abi_major = BLACKFRAME_EXTENSION_ABI_MAJOR;
    out->abi_minor = BLACKFRAME_EXTENSION_ABI_MINOR;
    out->extension_context = nullptr;
    out->get_interface = &get_interface;
    out->shutdown = &shutdown_extension;
    return BLACKFRAME_STATUS_SUCCESS;
}

}  // extern "C"

static_assert(sizeof(bf200_closure_v1) == 64, "closure record layout");
static_assert(sizeof(bf200_path_input_v1) == 80, "path input layout");
static_assert(sizeof(bf200_path_result_v1) == 128, "path result layout");
static_assert(sizeof(bf200_ray_v1) == 48, "ray layout");
static_assert(sizeof(bf200_material_gradient_v1) == kAdjointStride * sizeof(double), "gradient record layout");
static_assert(sizeof(bf200_adjoint_v1) == 40, "adjoint request layout");
static_assert(sizeof(bf200_instance_v1) == 160, "instance layout");
static_assert(sizeof(bf200_ray_cone_v1) == sizeof(float2), "ray cone layout (the device cone column is float2)");
static_assert(sizeof(bf200_path_state_v1) == 48, "path state layout");
