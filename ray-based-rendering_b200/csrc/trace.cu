// Ray-query kernels: closest hit and any hit for a batch of rbr_ray records.
//
// One thread per ray. Rays are read as two 16 B words (origin+tmax, direction+pad), answers
// written as one 8 B word (closest) or one byte (any). The traversal itself is in
// rbr_device.cuh.
#include "rbr_context.h"
#include "rbr_device.cuh"

namespace rbr {

namespace {

constexpr int kTraceBlock = 128;

__global__ void __launch_bounds__(kTraceBlock) k_trace_closest(DeviceScene s, const float4* __restrict__ rays,
                                                               uint32_t n, uint2* __restrict__ hits, int* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(rays + 2 * static_cast<size_t>(i));
    const float4 b = __ldg(rays + 2 * static_cast<size_t>(i) + 1);
    float t = 0.0f;
    const uint32_t prim = traverse<false>(s, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, t, err);
    hits[i] = make_uint2(prim, prim == 0xFFFFFFFFu ? 0u : __float_as_uint(t));
}

__global__ void __launch_bounds__(kTraceBlock) k_trace_any(DeviceScene s, const float4* __restrict__ rays, uint32_t n,
                                                           uint8_t* __restrict__ occ, int* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(rays + 2 * static_cast<size_t>(i));
    const float4 b = __ldg(rays + 2 * static_cast<size_t>(i) + 1);
    float t;
    occ[i] = static_cast<uint8_t>(traverse<true>(s, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, t, err));
}

// Same traversal, counting wide nodes fetched and leaf records tested (summed over the batch).
template <bool kAny>
__global__ void __launch_bounds__(kTraceBlock) k_trace_count(DeviceScene s, const float4* __restrict__ rays,
                                                             uint32_t n, unsigned long long* totals, int* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint2 c = make_uint2(0, 0);
    if (i < n) {
        const float4 a = __ldg(rays + 2 * static_cast<size_t>(i));
        const float4 b = __ldg(rays + 2 * static_cast<size_t>(i) + 1);
        float t;
        traverse<kAny, true>(s, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, t, err, &c);
    }
    unsigned long long nodes = c.x, recs = c.y;
    for (int off = 16; off > 0; off >>= 1) {
        nodes += __shfl_down_sync(0xFFFFFFFFu, nodes, off);
        recs += __shfl_down_sync(0xFFFFFFFFu, recs, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(totals, nodes);
        atomicAdd(totals + 1, recs);
    }
}

}  // namespace

cudaError_t launch_trace_counts(const DeviceScene& s, const rbr_ray* rays, uint32_t n, int any_hit,
                                unsigned long long* totals, int* err, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const uint32_t blocks = (n + kTraceBlock - 1) / kTraceBlock;
    if (any_hit)
        k_trace_count<true><<<blocks, kTraceBlock, 0, stream>>>(s, reinterpret_cast<const float4*>(rays), n, totals, err);
    else
        k_trace_count<false><<<blocks, kTraceBlock, 0, stream>>>(s, reinterpret_cast<const float4*>(rays), n, totals, err);
    return cudaGetLastError();
}

cudaError_t launch_trace_closest(const DeviceScene& s, const rbr_ray* rays, uint32_t n, rbr_hit* hits, int* err,
                                 int /*num_sms*/, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const uint32_t blocks = (n + kTraceBlock - 1) / kTraceBlock;
    k_trace_closest<<<blocks, kTraceBlock, 0, stream>>>(s, reinterpret_cast<const float4*>(rays), n,
                                                        reinterpret_cast<uint2*>(hits), err);
    return cudaGetLastError();
}

cudaError_t launch_trace_any(const DeviceScene& s, const rbr_ray* rays, uint32_t n, uint8_t* occ, int* err,
                             int /*num_sms*/, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const uint32_t blocks = (n + kTraceBlock - 1) / kTraceBlock;
    k_trace_any<<<blocks, kTraceBlock, 0, stream>>>(s, reinterpret_cast<const float4*>(rays), n, occ, err);
    return cudaGetLastError();
}

}  // namespace rbr
