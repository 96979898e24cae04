// Counting sort of small integer keys (at most 2^16 values) into a permutation, shared by the
// ray sort of the ray queries and the spatial sort of radiance-cache queries.
//
// Three passes: every item's key and a count per key value (count_key: global atomics, lanes
// of a warp with equal keys sharing one, so that coherent inputs do not serialise on one
// counter); k_key_offsets turns the counts into each key's first slot within its chunk of 1,024
// keys plus the chunk totals (one block per chunk); scatter_keys gives every item the next slot
// of its key (an atomic on the same counters, plus the slots of the chunks before) and writes
// the item's index there. The order within one key is the atomics' order, so it can differ
// between runs; the callers' results do not depend on it.
#pragma once

#include <cstdint>

namespace rbr {
namespace {

constexpr int kScanThreads = 1024;        // keys per chunk, threads of k_key_offsets
constexpr uint32_t kNoKey = 0xFFFFFFFFu;  // lanes with no item (real keys are below 2^16)

// Adds this lane's key to the counts; every lane of the warp calls it (k = kNoKey: no item).
__device__ __forceinline__ void count_key(uint32_t* counts, uint32_t k) {
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, k);
    if (k != kNoKey && (threadIdx.x & 31u) == static_cast<uint32_t>(__ffs(peers) - 1))
        atomicAdd(counts + k, __popc(peers));
}

// Exclusive prefix sums of the counts within each chunk of 1,024 keys, in place, one block of
// 1,024 threads per chunk; the chunk totals go to `chunk_sum`.
__global__ void __launch_bounds__(kScanThreads) k_key_offsets(uint32_t* counts, uint32_t* chunk_sum) {
    __shared__ uint32_t warp_sum[kScanThreads / 32];
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    uint32_t* c = counts + blockIdx.x * kScanThreads;
    const uint32_t v = c[t];
    uint32_t incl = v;  // inclusive scan over the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= static_cast<uint32_t>(o)) incl += y;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = warp_sum[lane];
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if (lane >= static_cast<uint32_t>(o)) wi += y;
        }
        warp_sum[lane] = wi - w;  // exclusive over the warps
        if (lane == 31) chunk_sum[blockIdx.x] = wi;
    }
    __syncthreads();
    c[t] = warp_sum[warp] + incl - v;
}

// The scatter pass over n items (keys[i] for item i), for kChunks chunks of keys (32 or 64).
// The whole warp walks the grid-stride loop together (its base is a multiple of the block), so
// every lane takes part in the match. Called by every thread of the block.
template <int kChunks>
__device__ __forceinline__ void scatter_keys(const uint16_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ offsets,
                                             const uint32_t* __restrict__ chunk_sum, uint32_t* __restrict__ perm) {
    static_assert(kChunks == 32 || kChunks == 64, "32 or 64 chunks of keys");
    constexpr int kPer = kChunks / 32;
    // first slot of each chunk of keys: exclusive sum of the chunk totals
    __shared__ uint32_t chunk_first[kChunks];
    if (threadIdx.x < 32) {
        const uint32_t l = threadIdx.x;
        uint32_t v[kPer], sum = 0;
#pragma unroll
        for (int q = 0; q < kPer; ++q) sum += (v[q] = chunk_sum[kPer * l + q]);
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (l >= static_cast<uint32_t>(o)) incl += y;
        }
        uint32_t run = incl - sum;
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            chunk_first[kPer * l + q] = run;
            run += v[q];
        }
    }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t k = i < n ? keys[i] : kNoKey;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, k);
        const uint32_t leader = static_cast<uint32_t>(__ffs(peers) - 1);
        uint32_t first = 0;
        if (k != kNoKey && lane == leader) first = chunk_first[k / kScanThreads] + atomicAdd(offsets + k, __popc(peers));
        first = __shfl_sync(0xFFFFFFFFu, first, leader);
        if (k != kNoKey) perm[first + __popc(peers & lt)] = i;
    }
}

}  // namespace
}  // namespace rbr
