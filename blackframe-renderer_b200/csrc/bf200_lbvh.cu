// Device BLAS build: a linear BVH over the triangles of one geometry, built on the GPU, for scenes
// whose build time matters more than the last few percent of traversal speed (the context's
// BF200_BUILD_DEVICE_LBVH mode). The host binned-SAH build stays the default.
//
//   k_lbvh_bounds    per triangle: its box and centroid (the host build's box and 0.5 lo + 0.5 hi),
//                    and the centroid bounds of the geometry (warp min/max, one atomic per warp)
//   k_lbvh_morton    63-bit Morton code of the centroid on a 2^21-per-axis grid over those bounds
//   sort             stable LSD radix sort of (code, triangle) pairs, 2 bits per pass: each pass is
//                    the wavefront's stable route compaction with 4 routes (bf200_compact.cu) and a
//                    gather, so equal codes keep triangle order and the tree is deterministic
//   k_lbvh_hierarchy Karras' construction ("Maximizing parallelism in the construction of BVHs,
//                    octrees, and k-d trees", HPG 2012): internal node i finds its key range and
//                    split from common-prefix lengths of the sorted (code, position) keys alone, one
//                    thread per node. A child range of at most four triangles becomes a leaf (the
//                    host build's leaf bound); nodes inside such a leaf are never referenced
//   k_lbvh_leaves    the leaf triangle records in sorted order (vertex positions, the triangle
//                    index in the first record's w), the layout the host build writes
//   k_lbvh_boxes     bottom-up boxes: every node that owns a leaf child starts by writing that
//                    child's box; a thread that completes a node's second child (atomic arrival
//                    counter) goes on to its parent. Nothing waits on another thread, so every
//                    thread ends after at most one pass to the root.
//
// The result is BVH2 nodes in the host builder's format (child boxes in a, b, c; child codes in d:
// a node index, or ~((first leaf record << kLeafCountBits) | (count - 1))), with node and leaf
// indices offset to the scene's arrays, so the same BVH4 collapse and every traversal consume it.
// Any conservative BVH gives the same closest hit (ties go to the lower instance, then primitive).
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "bf200_device.cuh"
#include "bf200_kernels.h"

namespace bf200 {
namespace {

constexpr int kLbvhLeaf = 4;  // the host build's leaf bound (kLeafSize)
constexpr uint32_t kLbvhThreads = 256;
constexpr int kMortonBits = 63;

__device__ __forceinline__ uint32_t ordered_bits(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000U) ? ~u : (u | 0x80000000U);
}

__device__ __forceinline__ float from_ordered_bits(uint32_t u) {
    return __uint_as_float((u & 0x80000000U) ? (u & 0x7FFFFFFFU) : ~u);
}

__global__ void __launch_bounds__(kLbvhThreads) k_lbvh_bounds(const float* __restrict__ positions,
                                                              const uint32_t* __restrict__ triangles, uint32_t n,
                                                              float4* __restrict__ box_lo, float4* __restrict__ box_hi,
                                                              float4* __restrict__ centroid,
                                                              uint32_t* __restrict__ centroid_bounds) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const float inf = __int_as_float(0x7F800000);
    float cmin[3] = {inf, inf, inf}, cmax[3] = {-inf, -inf, -inf};
    if (t < n) {
        float lo[3] = {inf, inf, inf}, hi[3] = {-inf, -inf, -inf};
        for (int k = 0; k < 3; ++k) {
            const uint32_t v = triangles[3ULL * t + k];
            for (int a = 0; a < 3; ++a) {
                const float x = positions[3ULL * v + a];
                lo[a] = fminf(lo[a], x);
                hi[a] = fmaxf(hi[a], x);
            }
        }
        float c[3];
        for (int a = 0; a < 3; ++a) {
            c[a] = __fadd_rn(__fmul_rn(0.5F, lo[a]), __fmul_rn(0.5F, hi[a]));
            cmin[a] = cmax[a] = c[a];
        }
        box_lo[t] = make_float4(lo[0], lo[1], lo[2], 0.0F);
        box_hi[t] = make_float4(hi[0], hi[1], hi[2], 0.0F);
        centroid[t] = make_float4(c[0], c[1], c[2], 0.0F);
    }
    for (int off = 16; off > 0; off >>= 1) {
        for (int a = 0; a < 3; ++a) {
            cmin[a] = fminf(cmin[a], __shfl_xor_sync(0xFFFFFFFFU, cmin[a], off));
            cmax[a] = fmaxf(cmax[a], __shfl_xor_sync(0xFFFFFFFFU, cmax[a], off));
        }
    }
    if ((threadIdx.x & 31U) == 0U && cmin[0] <= cmax[0]) {
        for (int a = 0; a < 3; ++a) {
            atomicMin(&centroid_bounds[a], ordered_bits(cmin[a]));
            atomicMax(&centroid_bounds[3 + a], ordered_bits(cmax[a]));
        }
    }
}

__device__ __forceinline__ unsigned long long spread_bits(unsigned long long x) {  // 21 bits -> every third bit
    x &= 0x1FFFFFULL;
    x = (x | x << 32) & 0x1F00000000FFFFULL;
    x = (x | x << 16) & 0x1F0000FF0000FFULL;
    x = (x | x << 8) & 0x100F00F00F00F00FULL;
    x = (x | x << 4) & 0x10C30C30C30C30C3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

__global__ void __launch_bounds__(kLbvhThreads) k_lbvh_morton(const float4* __restrict__ centroid, uint32_t n,
                                                              const uint32_t* __restrict__ centroid_bounds,
                                                              unsigned long long* __restrict__ keys,
                                                              uint32_t* __restrict__ ids) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) {
        return;
    }
    const float4 c = centroid[t];
    const float cv[3] = {c.x, c.y, c.z};
    unsigned long long q[3];
    for (int a = 0; a < 3; ++a) {
        const float lo = from_ordered_bits(centroid_bounds[a]);
        const float extent = from_ordered_bits(centroid_bounds[3 + a]) - lo;
        const float u = extent > 0.0F ? (cv[a] - lo) / extent * 2097152.0F : 0.0F;
        q[a] = static_cast<unsigned long long>(fminf(fmaxf(u, 0.0F), 2097151.0F));
    }
    keys[t] = (spread_bits(q[0]) << 2) | (spread_bits(q[1]) << 1) | spread_bits(q[2]);
    ids[t] = t;
}

__global__ void __launch_bounds__(kLbvhThreads) k_lbvh_digits(const unsigned long long* __restrict__ keys, uint32_t n,
                                                              uint32_t shift, uint8_t* __restrict__ digits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        digits[i] = static_cast<uint8_t>((keys[i] >> shift) & 3U);
    }
}

__global__ void __launch_bounds__(kLbvhThreads) k_lbvh_gather(const unsigned long long* __restrict__ keys_in,
                                                              const uint32_t* __restrict__ ids_in,
                                                              const uint32_t* __restrict__ order, uint32_t n,
                                                              unsigned long long* __restrict__ keys_out,
                                                              uint32_t* __restrict__ ids_out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const uint32_t from = order[i];
        keys_out[i] = keys_in[from];
        ids_out[i] = ids_in[from];
    }
}

// Common-prefix length of the sorted keys at positions i and j, each key made unique by its
// position appended below the code (so equal codes continue into the positions' bits); -1 outside
// [0, n).
__device__ __forceinline__ int prefix(const unsigned long long* keys, int n, int i, int j) {
    if (j < 0 || j >= n) {
        return -1;
    }
    const unsigned long long a = keys[i], b = keys[j];
    return a != b ? __clzll(a ^ b) : 64 + __clz(static_cast<uint32_t>(i ^ j));
}

__device__ __forceinline__ int leaf_code(uint32_t first, int count) {
    return ~static_cast<int>((first << kLeafCountBits) | static_cast<uint32_t>(count - 1));
}

__global__ void __launch_bounds__(kLbvhThreads) k_lbvh_hierarchy(const unsigned long long* __restrict__ keys, int n,
                                                                 uint32_t node_base, uint32_t leaf_base,
                                                                 BvhNode* __restrict__ nodes, int* __restrict__ parent,
                                                                 int4* __restrict__ ranges) {
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= n - 1) {
        return;
    }
    const int d = prefix(keys, n, i, i + 1) - prefix(keys, n, i, i - 1) >= 0 ? 1 : -1;
    const int dmin = prefix(keys, n, i, i - d);
    int lmax = 2;
    while (prefix(keys, n, i, i + lmax * d) > dmin) {  // ends once i + lmax d leaves [0, n)
        lmax *= 2;
    }
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2) {
        if (prefix(keys, n, i, i + (l + t) * d) > dmin) {
            l += t;
        }
    }
    const int j = i + l * d;
    const int dnode = prefix(keys, n, i, j);
    int s = 0;
    for (int divisor = 2;; divisor *= 2) {
        const int t = (l + divisor - 1) / divisor;
        if (prefix(keys, n, i, i + (s + t) * d) > dnode) {
            s += t;
        }
        if (t <= 1) {
            break;
        }
    }
    const int split = i + s * d + min(d, 0);
    const int first = min(i, j), last = max(i, j);
    const int left_count = split - first + 1, right_count = last - split;
    const bool left_leaf = left_count <= kLbvhLeaf, right_leaf = right_count <= kLbvhLeaf;
    const int left = left_leaf ? leaf_code(leaf_base + static_cast<uint32_t>(first), left_count)
                               : static_cast<int>(node_base) + split;
    const int right = right_leaf ? leaf_code(leaf_base + static_cast<uint32_t>(split + 1), right_count)
                                 : static_cast<int>(node_base) + split + 1;
    const float inf = __int_as_float(0x7F800000);
    nodes[i].a = make_float4(inf, -inf, inf, -inf);
    nodes[i].b = make_float4(inf, -inf, inf, -inf);
    nodes[i].c = make_float4(inf, -inf, inf, -inf);
    nodes[i].d = make_int4(left, right, 0, 0);
    if (!left_leaf) {
        parent[split] = i;
    }
    if (!right_leaf) {
        parent[split + 1] = i;
    }
    // w: the node is referenced (its range exceeds a leaf); the root always is
    ranges[i] = make_int4(first, split, last, (last - first + 1 > kLbvhLeaf || i == 0) ? 1 : 0);
}

__global__ void __launch_bounds__(kLbvhThreads) k_lbvh_leaves(const float* __restrict__ positions,
                                                              const uint32_t* __restrict__ triangles,
                                                              const uint32_t* __restrict__ ids, uint32_t n,
                                                              float4* __restrict__ leaf_tris) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) {
        return;
    }
    const uint32_t t = ids[k];
    for (int v = 0; v < 3; ++v) {
        const float* p = positions + 3ULL * triangles[3ULL * t + v];
        leaf_tris[3ULL * k + v] = make_float4(p[0], p[1], p[2], v == 0 ? __uint_as_float(t) : 0.0F);
    }
}

__device__ __forceinline__ void write_slot(BvhNode& node, int slot, const float lo[3], const float hi[3]) {
    if (slot == 0) {
        node.a = make_float4(lo[0], hi[0], lo[1], hi[1]);
        node.c.x = lo[2];
        node.c.y = hi[2];
    } else {
        node.b = make_float4(lo[0], hi[0], lo[1], hi[1]);
        node.c.z = lo[2];
        node.c.w = hi[2];
    }
}

// Writes a child box into its slot and reports whether this was the node's second child.
__device__ __forceinline__ bool complete(BvhNode* nodes, uint32_t* arrive, int node, int slot, const float lo[3],
                                         const float hi[3]) {
    write_slot(nodes[node], slot, lo, hi);
    __threadfence();
    const bool second = atomicAdd(&arrive[node], 1U) == 1U;
    __threadfence();
    return second;
}

__global__ void __launch_bounds__(kLbvhThreads) k_lbvh_boxes(BvhNode* __restrict__ nodes,
                                                             const int4* __restrict__ ranges,
                                                             const int* __restrict__ parent,
                                                             uint32_t* __restrict__ arrive,
                                                             const float4* __restrict__ box_lo,
                                                             const float4* __restrict__ box_hi,
                                                             const uint32_t* __restrict__ ids, int n,
                                                             uint32_t node_base) {
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= n - 1) {
        return;
    }
    const int4 r = ranges[i];
    if (r.w == 0) {
        return;
    }
    const float inf = __int_as_float(0x7F800000);
    bool owner = false;
    for (int slot = 0; slot < 2; ++slot) {
        const int first = slot == 0 ? r.x : r.y + 1;
        const int last = slot == 0 ? r.y : r.z;
        if (last - first + 1 > kLbvhLeaf) {
            continue;
        }
        float lo[3] = {inf, inf, inf}, hi[3] = {-inf, -inf, -inf};
        for (int k = first; k <= last; ++k) {
            const uint32_t t = ids[k];
            const float4 l = box_lo[t], h = box_hi[t];
            lo[0] = fminf(lo[0], l.x), lo[1] = fminf(lo[1], l.y), lo[2] = fminf(lo[2], l.z);
            hi[0] = fmaxf(hi[0], h.x), hi[1] = fmaxf(hi[1], h.y), hi[2] = fmaxf(hi[2], h.z);
        }
        owner = complete(nodes, arrive, i, slot, lo, hi);
    }
    int node = i;
    while (owner) {
        // both children of `node` are written: its box is their union (read through L2)
        const float4 a = __ldcg(&nodes[node].a), b = __ldcg(&nodes[node].b), c = __ldcg(&nodes[node].c);
        const float lo[3] = {fminf(a.x, b.x), fminf(a.z, b.z), fminf(c.x, c.z)};
        const float hi[3] = {fmaxf(a.y, b.y), fmaxf(a.w, b.w), fmaxf(c.y, c.w)};
        const int p = parent[node];
        if (p < 0) {
            break;
        }
        const int slot = nodes[p].d.x == static_cast<int>(node_base) + node ? 0 : 1;
        owner = complete(nodes, arrive, p, slot, lo, hi);
        node = p;
    }
}

uint32_t blocks(uint32_t n) {
    return (n + kLbvhThreads - 1) / kLbvhThreads;
}

}  // namespace

cudaError_t build_blas_lbvh(const float* positions, uint32_t vertex_count, const uint32_t* triangles, uint32_t n,
                            uint32_t node_base, uint32_t leaf_base, std::vector<BvhNode>& nodes,
                            std::vector<float4>& leaf_tris, cudaStream_t stream) {
    if (n <= static_cast<uint32_t>(kLbvhLeaf)) {
        return cudaErrorInvalidValue;  // tiny geometries take the host build
    }
    const uint32_t tiles = (n + kCompactTile - 1) / kCompactTile;
    const size_t bytes_positions = 12ULL * vertex_count, bytes_triangles = 12ULL * n;
    // one allocation, carved into 256-byte aligned regions:
    //  0 positions, 1 triangles, 2 box lo, 3 box hi, 4 centroids, 5-6 keys, 7-8 triangle ids,
    //  9 sort order, 10 digits, 11 compaction tile counts, 12 centroid bounds and route offsets,
    //  13 BVH2 nodes, 14 parents + arrival counters + ranges, 15 leaf records
    const size_t sizes[16] = {bytes_positions, bytes_triangles, 16ULL * n, 16ULL * n, 16ULL * n, 8ULL * n, 8ULL * n,
                              4ULL * n, 4ULL * n, 4ULL * n, static_cast<size_t>(n), 4ULL * kCompactMaxRoutes * tiles,
                              64, sizeof(BvhNode) * (n - 1), 8ULL * (n - 1) + 16 + 16ULL * (n - 1), 48ULL * n};
    size_t offsets[16] = {};
    size_t total = 0;
    for (int k = 0; k < 16; ++k) {
        offsets[k] = total;
        total += (sizes[k] + 255) & ~static_cast<size_t>(255);
    }
    char* base = nullptr;
    cudaError_t e = cudaMalloc(&base, total);
    if (e != cudaSuccess) {
        return e;
    }
    float* d_positions = reinterpret_cast<float*>(base + offsets[0]);
    uint32_t* d_triangles = reinterpret_cast<uint32_t*>(base + offsets[1]);
    float4* d_lo = reinterpret_cast<float4*>(base + offsets[2]);
    float4* d_hi = reinterpret_cast<float4*>(base + offsets[3]);
    float4* d_centroid = reinterpret_cast<float4*>(base + offsets[4]);
    unsigned long long* keys[2] = {reinterpret_cast<unsigned long long*>(base + offsets[5]),
                                   reinterpret_cast<unsigned long long*>(base + offsets[6])};
    uint32_t* ids[2] = {reinterpret_cast<uint32_t*>(base + offsets[7]), reinterpret_cast<uint32_t*>(base + offsets[8])};
    uint32_t* order = reinterpret_cast<uint32_t*>(base + offsets[9]);
    uint8_t* digits = reinterpret_cast<uint8_t*>(base + offsets[10]);
    uint32_t* tile_counts = reinterpret_cast<uint32_t*>(base + offsets[11]);
    uint32_t* small = reinterpret_cast<uint32_t*>(base + offsets[12]);  // centroid bounds [0, 6), route offsets [8, 13)
    BvhNode* d_nodes = reinterpret_cast<BvhNode*>(base + offsets[13]);
    int* d_parent = reinterpret_cast<int*>(base + offsets[14]);
    uint32_t* d_arrive = reinterpret_cast<uint32_t*>(d_parent + (n - 1));
    int4* d_ranges = reinterpret_cast<int4*>(base + offsets[14] + ((8ULL * (n - 1) + 15) & ~15ULL));
    float4* d_leaf_tris = reinterpret_cast<float4*>(base + offsets[15]);
    const size_t node_first = nodes.size(), leaf_first = leaf_tris.size();
    int cur = 0;
    uint32_t launches = 0;
    e = cudaMemcpyAsync(d_positions, positions, bytes_positions, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(d_triangles, triangles, bytes_triangles, cudaMemcpyHostToDevice, stream);
    }
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(small, 0xFF, 12, stream);  // centroid minima start at the largest code
    }
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(small + 3, 0, 12, stream);  // maxima at the smallest
    }
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(d_parent, 0xFF, 4ULL * (n - 1), stream);  // -1: the root has no parent
    }
    if (e == cudaSuccess) {
        e = cudaMemsetAsync(d_arrive, 0, 4ULL * (n - 1), stream);
    }
    if (e == cudaSuccess) {
        k_lbvh_bounds<<<blocks(n), kLbvhThreads, 0, stream>>>(d_positions, d_triangles, n, d_lo, d_hi, d_centroid,
                                                               small);
        k_lbvh_morton<<<blocks(n), kLbvhThreads, 0, stream>>>(d_centroid, n, small, keys[0], ids[0]);
        e = cudaGetLastError();
    }
    for (int shift = 0; e == cudaSuccess && shift < kMortonBits; shift += 2) {
        k_lbvh_digits<<<blocks(n), kLbvhThreads, 0, stream>>>(keys[cur], n, static_cast<uint32_t>(shift), digits);
        e = cudaGetLastError();
        if (e == cudaSuccess) {
            e = launch_compaction(digits, n, kCompactMaxRoutes, tile_counts, order, small + 8, nullptr, nullptr,
                                  stream, &launches);
        }
        if (e == cudaSuccess) {
            k_lbvh_gather<<<blocks(n), kLbvhThreads, 0, stream>>>(keys[cur], ids[cur], order, n, keys[1 - cur],
                                                                   ids[1 - cur]);
            e = cudaGetLastError();
            cur = 1 - cur;
        }
    }
    if (e == cudaSuccess) {
        k_lbvh_hierarchy<<<blocks(n - 1), kLbvhThreads, 0, stream>>>(keys[cur], static_cast<int>(n), node_base,
                                                                      leaf_base, d_nodes, d_parent, d_ranges);
        k_lbvh_leaves<<<blocks(n), kLbvhThreads, 0, stream>>>(d_positions, d_triangles, ids[cur], n, d_leaf_tris);
        k_lbvh_boxes<<<blocks(n - 1), kLbvhThreads, 0, stream>>>(d_nodes, d_ranges, d_parent, d_arrive, d_lo, d_hi,
                                                                  ids[cur], static_cast<int>(n), node_base);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        nodes.resize(node_first + (n - 1));
        leaf_tris.resize(leaf_first + 3ULL * n);
        e = cudaMemcpyAsync(nodes.data() + node_first, d_nodes, sizeof(BvhNode) * (n - 1), cudaMemcpyDeviceToHost,
                            stream);
    }
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(leaf_tris.data() + leaf_first, d_leaf_tris, 48ULL * n, cudaMemcpyDeviceToHost, stream);
    }
    if (e == cudaSuccess) {
        e = cudaStreamSynchronize(stream);
    }
    const cudaError_t freed = cudaFree(base);
    if (e != cudaSuccess) {
        nodes.resize(node_first);
        leaf_tris.resize(leaf_first);
        return e;
    }
    return freed;
}

}  // namespace bf200
