// Stable queue compaction of the wavefront (the reference's select + exclusive scan + scatter of
// CudaWavefrontQueueCompaction.cu:253-315, there five launches and a host sync per route).
//
// Here one pass builds every route's queue at once and keeps slot order, with no host round trip:
//   k_compact_count   one block per tile of 4096 slots; each warp owns 512 consecutive slots and
//                     counts them per route with __ballot_sync / __popc; one word per (route, tile)
//   k_compact_scan    one block: exclusive scan of the route-major (route, tile) counts, so the
//                     queue of route r starts where route r - 1 ends and tiles follow slot order
//   k_compact_scatter one block per tile: per-warp counts, a block scan over the 8 warps, then each
//                     lane writes its slot at base + popc(ballot & lanes below it)
// Slots are therefore queued in increasing slot order within each route, which makes the shading
// and occlusion kernels' gathers ascending (coalescing where neighbouring slots share a route).
#include <cuda_runtime.h>

#include <cstdint>

#include "bf200_kernels.h"

namespace bf200 {
namespace {

constexpr uint32_t kCompactWarps = 8U;
constexpr uint32_t kWarpSlots = kCompactTile / kCompactWarps;  // 512
constexpr uint32_t kScanThreads = 1024U;

__device__ __forceinline__ uint32_t key_at(const uint8_t* keys, uint32_t n, uint32_t slot) {
    return slot < n ? static_cast<uint32_t>(keys[slot]) : 0xFFU;
}

__global__ void __launch_bounds__(256) k_compact_count(const uint8_t* __restrict__ keys, uint32_t n, uint32_t routes,
                                                       uint32_t tiles, uint32_t* __restrict__ tile_counts) {
    __shared__ uint32_t partial[kCompactWarps][kCompactMaxRoutes];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31U;
    const uint32_t first = blockIdx.x * kCompactTile + warp * kWarpSlots;
    uint32_t count[kCompactMaxRoutes] = {0U, 0U, 0U, 0U};
    for (uint32_t step = 0; step < kWarpSlots; step += 32U) {
        const uint32_t key = key_at(keys, n, first + step + lane);
#pragma unroll
        for (uint32_t r = 0; r < kCompactMaxRoutes; ++r) {
            count[r] += __popc(__ballot_sync(0xFFFFFFFFU, key == r && r < routes));
        }
    }
    if (lane == 0U) {
#pragma unroll
        for (uint32_t r = 0; r < kCompactMaxRoutes; ++r) {
            partial[warp][r] = count[r];
        }
    }
    __syncthreads();
    if (threadIdx.x < routes) {
        uint32_t total = 0U;
#pragma unroll
        for (uint32_t k = 0; k < kCompactWarps; ++k) {
            total += partial[k][threadIdx.x];
        }
        tile_counts[threadIdx.x * tiles + blockIdx.x] = total;
    }
}

__global__ void __launch_bounds__(kScanThreads) k_compact_scan(uint32_t* __restrict__ tile_counts, uint32_t routes,
                                                               uint32_t tiles, uint32_t* __restrict__ offsets,
                                                               unsigned long long* __restrict__ total) {
    __shared__ uint32_t sums[kScanThreads];
    const uint32_t m = routes * tiles;
    const uint32_t per = (m + kScanThreads - 1U) / kScanThreads;
    const uint32_t begin = threadIdx.x * per;
    const uint32_t end = begin + per < m ? begin + per : m;
    uint32_t local = 0U;
    for (uint32_t i = begin; i < end; ++i) {
        local += tile_counts[i];
    }
    sums[threadIdx.x] = local;
    __syncthreads();
    for (uint32_t off = 1U; off < kScanThreads; off <<= 1U) {
        const uint32_t v = threadIdx.x >= off ? sums[threadIdx.x - off] : 0U;
        __syncthreads();
        sums[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t running = threadIdx.x == 0U ? 0U : sums[threadIdx.x - 1U];
    for (uint32_t i = begin; i < end; ++i) {
        const uint32_t c = tile_counts[i];
        tile_counts[i] = running;
        running += c;
    }
    __syncthreads();
    if (threadIdx.x <= routes) {
        offsets[threadIdx.x] = threadIdx.x < routes ? tile_counts[threadIdx.x * tiles] : sums[kScanThreads - 1U];
    }
    if (threadIdx.x == 0U && total != nullptr) {
        *total = sums[kScanThreads - 1U];
    }
}

__global__ void __launch_bounds__(256) k_compact_scatter(const uint8_t* __restrict__ keys, uint32_t n,
                                                         uint32_t routes, uint32_t tiles,
                                                         const uint32_t* __restrict__ tile_offsets,
                                                         uint32_t* __restrict__ queue, uint8_t* __restrict__ reset_keys) {
    __shared__ uint32_t warp_base[kCompactWarps][kCompactMaxRoutes];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31U;
    const uint32_t first = blockIdx.x * kCompactTile + warp * kWarpSlots;
    uint32_t count[kCompactMaxRoutes] = {0U, 0U, 0U, 0U};
    for (uint32_t step = 0; step < kWarpSlots; step += 32U) {
        const uint32_t key = key_at(keys, n, first + step + lane);
#pragma unroll
        for (uint32_t r = 0; r < kCompactMaxRoutes; ++r) {
            count[r] += __popc(__ballot_sync(0xFFFFFFFFU, key == r && r < routes));
        }
    }
    if (lane == 0U) {
#pragma unroll
        for (uint32_t r = 0; r < kCompactMaxRoutes; ++r) {
            warp_base[warp][r] = count[r];
        }
    }
    __syncthreads();
    if (threadIdx.x < routes) {
        uint32_t running = tile_offsets[threadIdx.x * tiles + blockIdx.x];
#pragma unroll
        for (uint32_t k = 0; k < kCompactWarps; ++k) {
            const uint32_t c = warp_base[k][threadIdx.x];
            warp_base[k][threadIdx.x] = running;
            running += c;
        }
    }
    __syncthreads();
    uint32_t base[kCompactMaxRoutes];
#pragma unroll
    for (uint32_t r = 0; r < kCompactMaxRoutes; ++r) {
        base[r] = r < routes ? warp_base[warp][r] : 0U;
    }
    const uint32_t below = (1U << lane) - 1U;
    for (uint32_t step = 0; step < kWarpSlots; step += 32U) {
        const uint32_t slot = first + step + lane;
        const uint32_t key = key_at(keys, n, slot);
#pragma unroll
        for (uint32_t r = 0; r < kCompactMaxRoutes; ++r) {
            const bool mine = key == r && r < routes;
            const unsigned ballot = __ballot_sync(0xFFFFFFFFU, mine);
            if (mine) {
                queue[base[r] + __popc(ballot & below)] = slot;
            }
            base[r] += __popc(ballot);
        }
        if (reset_keys != nullptr && slot < n) {
            reset_keys[slot] = kRouteNone;
        }
    }
}

}  // namespace

cudaError_t launch_compaction(const uint8_t* keys, uint32_t n, uint32_t routes, uint32_t* tile_counts,
                              uint32_t* queue, uint32_t* offsets, unsigned long long* total, uint8_t* reset_keys,
                              cudaStream_t stream, uint32_t* launches) {
    if (routes == 0U || routes > kCompactMaxRoutes) {
        return cudaErrorInvalidValue;
    }
    const uint32_t tiles = n == 0U ? 1U : (n + kCompactTile - 1U) / kCompactTile;
    k_compact_count<<<tiles, 256, 0, stream>>>(keys, n, routes, tiles, tile_counts);
    k_compact_scan<<<1, kScanThreads, 0, stream>>>(tile_counts, routes, tiles, offsets, total);
    k_compact_scatter<<<tiles, 256, 0, stream>>>(keys, n, routes, tiles, tile_counts, queue, reset_keys);
    *launches += 3U;
    return cudaGetLastError();
}

}  // namespace bf200
