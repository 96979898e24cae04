// Ray-query kernels: closest hit and any hit for a batch of rbr_ray records.
//
// One thread per ray. Rays are read as two 16 B words (origin+tmax, direction+pad), answers
// written as one 8 B word (closest) or one byte (any). The traversal itself is in
// rbr_device.cuh.
#include <algorithm>
#include <cmath>

#include <cub/device/device_radix_sort.cuh>

#include "rbr_context.h"
#include "rbr_device.cuh"
#include "rbr_sort.cuh"

namespace rbr {

namespace {

constexpr int kTraceBlock = 128;

// Ray loads and hit stores: with kStream, evict-first (streaming) hints, since every ray and
// hit is touched once and the L2 is better spent on the BVH.
template <bool kStream>
__device__ __forceinline__ float4 ray_word(const float4* p) { return kStream ? __ldcs(p) : __ldg(p); }
template <bool kStream>
__device__ __forceinline__ void put_hit(uint2* p, uint2 h) {
    if (kStream) __stcs(p, h);
    else *p = h;
}

// kMinBlocks: resident blocks per SM the register allocation must allow (8: up to 64
// registers a thread, 10: 48, 12: 40) -- occupancy against register spills, picked by tuning.
template <int kMinBlocks, bool kStream>
__global__ void __launch_bounds__(kTraceBlock, kMinBlocks) k_trace_closest(DeviceScene s, const float4* __restrict__ rays,
                                                                           uint32_t n, uint2* __restrict__ hits, int* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = ray_word<kStream>(rays + 2 * static_cast<size_t>(i));
    const float4 b = ray_word<kStream>(rays + 2 * static_cast<size_t>(i) + 1);
    float t = 0.0f;
    const uint32_t prim = traverse<false>(s, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, t, err);
    put_hit<kStream>(hits + i, make_uint2(prim, prim == 0xFFFFFFFFu ? 0u : __float_as_uint(t)));
}

// The same query on the rays in the order `perm` (a permutation of 0..n-1): rays that start
// close together with directions of the same octant share warps, so they walk the same nodes.
// Answers go to the rays' own positions.
template <int kMinBlocks, bool kStream, bool kLean = false>
__global__ void __launch_bounds__(kTraceBlock, kMinBlocks)
    k_trace_closest_perm(DeviceScene s, const float4* __restrict__ rays, uint32_t n, const uint32_t* __restrict__ perm,
                         uint2* __restrict__ hits, int* err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t i = kStream ? __ldcs(perm + j) : __ldg(perm + j);
    const float4 a = ray_word<kStream>(rays + 2 * static_cast<size_t>(i));
    const float4 b = ray_word<kStream>(rays + 2 * static_cast<size_t>(i) + 1);
    float t = 0.0f;
    const uint32_t prim = traverse<false, false, kLean>(s, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, t, err);
    put_hit<kStream>(hits + i, make_uint2(prim, prim == 0xFFFFFFFFu ? 0u : __float_as_uint(t)));
}

// Launches a ray-query kernel; with trace.l2_persist the BVH's address range (nodes and leaf
// records) is marked persisting in L2 for this launch only (a launch attribute: the caller's
// stream keeps its own attributes).
template <typename... Params, typename... Args>
cudaError_t launch_query(const rbr_ctx* ctx, void (*kernel)(Params...), uint32_t blocks, cudaStream_t stream,
                         Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kTraceBlock);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    if (ctx->trace_l2_persist && ctx->bvh_bytes && ctx->l2_persist_bytes) {
        attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[0].val.accessPolicyWindow.base_ptr = const_cast<void*>(ctx->bvh_base);
        attr[0].val.accessPolicyWindow.num_bytes = ctx->bvh_bytes;
        attr[0].val.accessPolicyWindow.hitRatio =
            static_cast<float>(std::min(1.0, double(ctx->l2_persist_bytes) / double(ctx->bvh_bytes)));
        attr[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attr[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Params>(args)...);
}

__global__ void __launch_bounds__(kTraceBlock) k_trace_any_perm(DeviceScene s, const float4* __restrict__ rays, uint32_t n,
                                                                const uint32_t* __restrict__ perm,
                                                                uint8_t* __restrict__ occ, int* err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t i = __ldg(perm + j);
    const float4 a = __ldg(rays + 2 * static_cast<size_t>(i));
    const float4 b = __ldg(rays + 2 * static_cast<size_t>(i) + 1);
    float t;
    occ[i] = static_cast<uint8_t>(traverse<true>(s, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, t, err));
}

// Sort keys from the direction octant (3 bits) and a Morton code of the origin's cell over the
// scene box. order 1: octant, then 27-bit Morton code of 512^3 cells (30 key bits); order 2:
// octant, then 18-bit code of 64^3 cells (21 bits, one radix pass fewer); order 3: the 64^3
// cell first, octant last (21 bits), so consecutive warps stay in one region of the scene.
// Orders 4 and 5 bin the direction finely and the origin coarsely (16 bits, two radix passes):
// the direction's octahedral map onto the unit square in 16 x 8 cells (7 bits) and a Morton
// code of 8^3 origin cells (9 bits); order 4 direction first, order 5 origin first. Rays of one
// direction cell from nearby origins diverge less than rays of one octant, whose directions
// span 90 degrees.
__device__ __forceinline__ uint32_t spread3(uint32_t x) {  // 9 bits -> every third of 27
    x &= 0x1FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// Sort key of one ray (a = origin and tmax, b = direction). Orders 1-3: direction octant and
// Morton code of the origin cell (64^3 or 512^3 cells); orders 4 and 5: octahedral direction
// cell of 16 x 8 and origin cell of 8^3, 16 bits.
__device__ __forceinline__ uint32_t ray_key(float4 a, float4 b, float3 lo, float3 scale, int order) {
    const uint32_t oct = (signbit(b.x) ? 4u : 0u) | (signbit(b.y) ? 2u : 0u) | (signbit(b.z) ? 1u : 0u);
    auto cell = [](float v, float l, float sc) {
        const float c = (v - l) * sc;  // NaN and out-of-box origins clamp to the box
        return static_cast<uint32_t>(fminf(fmaxf(c, 0.0f), 511.0f));
    };
    const uint32_t m = spread3(cell(a.x, lo.x, scale.x)) << 2 | spread3(cell(a.y, lo.y, scale.y)) << 1 |
                       spread3(cell(a.z, lo.z, scale.z));
    if (order >= 4) {
        // octahedral map: (x, y) / (|x| + |y| + |z|), the lower hemisphere folded outwards
        const float l1 = fabsf(b.x) + fabsf(b.y) + fabsf(b.z);
        float u = l1 > 0.0f ? b.x / l1 : 0.0f, v = l1 > 0.0f ? b.y / l1 : 0.0f;
        if (b.z < 0.0f) {
            const float uu = (1.0f - fabsf(v)) * (u < 0.0f ? -1.0f : 1.0f);
            v = (1.0f - fabsf(u)) * (v < 0.0f ? -1.0f : 1.0f);
            u = uu;
        }
        const uint32_t du = static_cast<uint32_t>(fminf(fmaxf((u + 1.0f) * 8.0f, 0.0f), 15.0f));  // NaN -> 0
        const uint32_t dv = static_cast<uint32_t>(fminf(fmaxf((v + 1.0f) * 4.0f, 0.0f), 7.0f));
        const uint32_t dir = (du << 3) | dv;
        const uint32_t c = m >> 18;  // 8^3 cells: the top 9 bits of the 27-bit code
        return order == 4 ? (dir << 9) | c : (c << 7) | dir;
    }
    return order == 1 ? (oct << 27) | m : order == 2 ? (oct << 18) | (m >> 9) : ((m >> 9) << 3) | oct;
}

__global__ void k_ray_keys(const float4* __restrict__ rays, uint32_t n, float3 lo, float3 scale, int order,
                           uint32_t* keys, uint32_t* idx) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 a = __ldg(rays + 2 * static_cast<size_t>(i));
        const float4 b = __ldg(rays + 2 * static_cast<size_t>(i) + 1);
        keys[i] = ray_key(a, b, lo, scale, order);
        idx[i] = i;
    }
}

// Orders 4 and 5 (16-bit keys) use the counting sort of rbr_sort.cuh: 65,536 key values in 64
// chunks.
constexpr uint32_t kKeyValues = 1u << 16;
constexpr uint32_t kScanChunks = kKeyValues / kScanThreads;

__global__ void k_ray_keys16(const float4* __restrict__ rays, uint32_t n, float3 lo, float3 scale, int order,
                             uint16_t* __restrict__ keys, uint32_t* __restrict__ counts) {
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        uint32_t k = kNoKey;
        if (i < n) {
            const float4 a = __ldg(rays + 2 * static_cast<size_t>(i));
            const float4 b = __ldg(rays + 2 * static_cast<size_t>(i) + 1);
            k = ray_key(a, b, lo, scale, order);
            keys[i] = static_cast<uint16_t>(k);
        }
        count_key(counts, k);
    }
}

__global__ void k_ray_scatter16(const uint16_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ offsets,
                                const uint32_t* __restrict__ chunk_sum, uint32_t* __restrict__ perm) {
    scatter_keys<kScanChunks>(keys, n, offsets, chunk_sum, perm);
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

__device__ __forceinline__ uint32_t lane_mask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Persistent warps: each warp takes chunks of kChunk consecutive rays from a global cursor
// (one atomic per chunk) and hands the next ray of its chunk to any lane whose ray is done,
// so lanes keep working while the warp's other rays are still traversing. Every loop
// iteration each active lane advances its ray by one step (a leaf-record test or a node test).
// With `perm` (sorted rays), position j of the cursor's order is ray perm[j].
constexpr int kPersistBlock = 128;
constexpr uint32_t kChunk = 256;

template <bool kAny>
__global__ void __launch_bounds__(kPersistBlock) k_trace_persist(DeviceScene s, const float4* __restrict__ rays,
                                                                 uint32_t n, const uint32_t* __restrict__ perm,
                                                                 uint2* __restrict__ hits, uint8_t* __restrict__ occ,
                                                                 int* err, uint32_t* cursor, uint32_t refill_min) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t chunk_next = 0, chunk_end = 0;  // warp-uniform
    bool exhausted = false;                  // warp-uniform
    uint32_t idx = 0xFFFFFFFFu;              // this lane's ray
    uint32_t anyhit = 0;
    TraceState st;
    uint2 stack[kStackSize];
    while (true) {
        uint32_t need = __ballot_sync(0xFFFFFFFFu, idx == 0xFFFFFFFFu);
        // refill once at least refill_min lanes are idle (or all of them): a refill costs the
        // whole warp a few ballots and a ray load, so lanes may idle for a few steps first
        while (need != 0 && !exhausted && (static_cast<uint32_t>(__popc(need)) >= refill_min || need == 0xFFFFFFFFu)) {
            if (chunk_next == chunk_end) {
                uint32_t b = 0;
                if (lane == 0) b = atomicAdd(cursor, kChunk);
                b = __shfl_sync(0xFFFFFFFFu, b, 0);
                if (b >= n) {
                    exhausted = true;
                    break;
                }
                chunk_next = b;
                chunk_end = min(b + kChunk, n);
            }
            const uint32_t avail = chunk_end - chunk_next;
            const uint32_t rank = __popc(need & lane_mask_lt());
            if (((need >> lane) & 1u) && rank < avail) {
                idx = perm ? __ldg(perm + chunk_next + rank) : chunk_next + rank;
                const float4 a = __ldg(rays + 2 * static_cast<size_t>(idx));
                const float4 b = __ldg(rays + 2 * static_cast<size_t>(idx) + 1);
                if (trace_begin<kAny>(s, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, st, anyhit)) {
                    if (kAny) occ[idx] = static_cast<uint8_t>(anyhit);
                    else hits[idx] = make_uint2(st.best < 0 ? 0xFFFFFFFFu : static_cast<uint32_t>(st.best),
                                                st.best < 0 ? 0u : __float_as_uint(st.tbest));
                    idx = 0xFFFFFFFFu;  // finished at once: takes another ray in this round
                }
            }
            chunk_next += min(__popc(need), avail);  // each round consumes at least one ray
            need = __ballot_sync(0xFFFFFFFFu, idx == 0xFFFFFFFFu);
        }
        const bool active = idx != 0xFFFFFFFFu;
        if (__ballot_sync(0xFFFFFFFFu, active) == 0) break;  // only when the rays are exhausted
        if (active && trace_step<kAny>(s, st, stack, err, anyhit)) {
            if (kAny) occ[idx] = static_cast<uint8_t>(anyhit);
            else hits[idx] = make_uint2(st.best < 0 ? 0xFFFFFFFFu : static_cast<uint32_t>(st.best),
                                        st.best < 0 ? 0u : __float_as_uint(st.tbest));
            idx = 0xFFFFFFFFu;
        }
    }
}

// ------------------------------------------------------------------------------------------
// Warp-cooperative traversal: a group of 8 lanes traces one ray (4 rays per warp). In a node
// step lane j tests child slot j of the node and the group ORs the slots' bits of the node's
// hit mask (internal children and leaf records) with shuffles; in a leaf step the lanes test up to 8
// of the node's leaf records at once and keep the closest with a shuffle min-reduction
// (key = t bits, then the highest id). Group state is replicated in the 8 lanes, so the group
// never diverges internally; the short stack lives in shared memory (all 8 lanes write the
// same entry and read back their own write, so no cross-lane synchronisation is needed).
// ------------------------------------------------------------------------------------------
constexpr int kCoopBlock = 128;
constexpr int kCoopGroups = kCoopBlock / 8;

__device__ __forceinline__ uint32_t nth_set_bit(uint32_t m, int n) {  // n-th (0-based) set bit, or 32
    for (int k = 0; k < n && m; ++k) m &= m - 1;
    return m ? static_cast<uint32_t>(__ffs(m) - 1) : 32u;
}

template <bool kAny>
__global__ void __launch_bounds__(kCoopBlock) k_trace_coop(DeviceScene s, const float4* __restrict__ rays, uint32_t n,
                                                           uint2* __restrict__ hits, uint8_t* __restrict__ occ,
                                                           int* err, uint32_t* cursor) {
    __shared__ uint2 sstack[kCoopGroups][kStackSize];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t j = lane & 7u;             // slot / record lane within the group
    const uint32_t g = lane >> 3;             // group within the warp
    const uint32_t gmask = 0xFFu << (8 * g);  // the group's lanes
    uint2* stack = sstack[threadIdx.x >> 3];
    uint32_t chunk_next = 0, chunk_end = 0;   // warp-uniform
    bool exhausted = false;                   // warp-uniform
    uint32_t idx = 0xFFFFFFFFu;               // group-uniform
    RayCtx r;
    float tbest = 0.0f;
    int best = -1;
    uint2 ng = make_uint2(0, 0), pg = make_uint2(0, 0);
    int sp = 0;
    while (true) {
        // give idle groups new rays from the warp's chunk
        uint32_t need = __ballot_sync(0xFFFFFFFFu, j == 0 && idx == 0xFFFFFFFFu);
        while (need != 0 && !exhausted) {
            if (chunk_next == chunk_end) {
                uint32_t b = 0;
                if (lane == 0) b = atomicAdd(cursor, kChunk);
                b = __shfl_sync(0xFFFFFFFFu, b, 0);
                if (b >= n) {
                    exhausted = true;
                    break;
                }
                chunk_next = b;
                chunk_end = min(b + kChunk, n);
            }
            const uint32_t avail = chunk_end - chunk_next;
            const uint32_t rank = __popc(need & ((1u << (8 * g)) - 1u));
            if (((need >> (8 * g)) & 1u) && rank < avail) {
                idx = chunk_next + rank;
                const float4 a = __ldg(rays + 2 * static_cast<size_t>(idx));
                const float4 b = __ldg(rays + 2 * static_cast<size_t>(idx) + 1);
                const f3 o = mk(a.x, a.y, a.z), d = mk(b.x, b.y, b.z);
                tbest = a.w;
                best = -1;
                bool done = false;
                for (uint32_t i = 0; i < s.num_planes && !done; ++i) {
                    const float4 pl = __ldg(s.planes + i);
                    const float t = hit_plane(o, d, mk(pl.x, pl.y, pl.z), pl.w, tbest);
                    if (t >= 0.0f) {
                        const uint32_t id = __ldg(s.plane_tags + i) & kIdMask;
                        if (kAny) done = true;
                        else if (accept(t, id, tbest, best)) {
                            tbest = t;
                            best = static_cast<int>(id);
                        }
                    }
                }
                if (kAny && done) {
                    if (j == 0) occ[idx] = 1;
                    idx = 0xFFFFFFFFu;
                } else if (s.num_nodes == 0) {
                    if (j == 0) {
                        if (kAny) occ[idx] = 0;
                        else hits[idx] = make_uint2(best < 0 ? 0xFFFFFFFFu : static_cast<uint32_t>(best),
                                                    best < 0 ? 0u : __float_as_uint(tbest));
                    }
                    idx = 0xFFFFFFFFu;
                } else {
                    r = make_ctx(o, d);
                    sp = 0;
                    pg = make_uint2(0, 0);
                    // a pseudo node group whose only child is the root (slot 0, internal)
                    ng = make_uint2(0u, (1u << (24 + (0u ^ r.oct))) | (1u << 16));
                }
            }
            chunk_next += min(__popc(need), avail);
            need = __ballot_sync(0xFFFFFFFFu, j == 0 && idx == 0xFFFFFFFFu);
        }
        if (__ballot_sync(0xFFFFFFFFu, idx != 0xFFFFFFFFu) == 0) break;  // rays exhausted
        if (idx == 0xFFFFFFFFu) continue;
        bool finished = false;
        uint32_t anyres = 0;
        if (pg.y != 0) {
            // leaf step: up to 8 records at once
            const uint32_t bit = nth_set_bit(pg.y, static_cast<int>(j));
            unsigned long long key = ~0ull;
            if (bit < 32) {
                uint32_t tag;
                const float t = hit_record(s.records, pg.x + bit, r.o, r.d, tbest, tag);
                if (t >= 0.0f) key = (static_cast<unsigned long long>(__float_as_uint(t)) << 32) | (~(tag & kIdMask));
            }
            if (kAny) {
                if (__ballot_sync(gmask, key != ~0ull) != 0) {
                    finished = true;
                    anyres = 1;
                }
            } else {
                for (int off = 1; off < 8; off <<= 1) {
                    const unsigned long long o2 = __shfl_xor_sync(gmask, key, off, 8);
                    key = o2 < key ? o2 : key;
                }
                if (key != ~0ull) {
                    const float t = __uint_as_float(static_cast<uint32_t>(key >> 32));
                    const uint32_t id = ~static_cast<uint32_t>(key) & kIdMask;
                    if (accept(t, id, tbest, best)) {
                        tbest = t;
                        best = static_cast<int>(id);
                    }
                }
            }
            // drop the (up to) 8 records just tested
            pg.y = __popc(pg.y) <= 8 ? 0u : pg.y & ~((2u << nth_set_bit(pg.y, 7)) - 1u);
        } else {
            // node step (after a pop if the current group is exhausted)
            if ((ng.y & 0xFF000000u) == 0) {
                if (sp == 0) {
                    finished = true;
                } else {
                    ng = stack[--sp];
                }
            }
            if (!finished) {
                const int b = 31 - __clz(ng.y);
                ng.y &= ~(1u << b);
                const uint32_t slot = static_cast<uint32_t>(b - 24) ^ r.oct;
                const uint32_t imask_p = (ng.y >> 16) & 0xFFu;
                const uint32_t child = ng.x + __popc(imask_p & ((1u << slot) - 1u));
                if (ng.y & 0xFF000000u) {
                    if (sp < kStackSize) stack[sp++] = ng;
                    else atomicOr(err, kErrStackOverflow);
                }
                // lane j tests slot j; the group ORs the slots' bits of the node's hit mask
                const NodeView v = node_view(s.nodes, child, r);
                const int jj = static_cast<int>(j);
                uint32_t bits = slot_hit(v, jj, tbest) ? slot_bits(v, jj) : 0u;
                bits |= __shfl_xor_sync(gmask, bits, 1, 8);
                bits |= __shfl_xor_sync(gmask, bits, 2, 8);
                bits |= __shfl_xor_sync(gmask, bits, 4, 8);
                split_hits(v, bits, ng, pg);
            }
        }
        if (finished) {
            if (j == 0) {
                if (kAny) occ[idx] = static_cast<uint8_t>(anyres);
                else hits[idx] = make_uint2(best < 0 ? 0xFFFFFFFFu : static_cast<uint32_t>(best),
                                            best < 0 ? 0u : __float_as_uint(tbest));
            }
            idx = 0xFFFFFFFFu;
        }
    }
}

}  // namespace

cudaError_t launch_trace_coop(const DeviceScene& s, const rbr_ray* rays, uint32_t n, int any_hit, void* out, int* err,
                              uint32_t* cursor, int grid, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(cursor, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    const auto* r = reinterpret_cast<const float4*>(rays);
    if (any_hit)
        k_trace_coop<true><<<grid, kCoopBlock, 0, stream>>>(s, r, n, nullptr, static_cast<uint8_t*>(out), err, cursor);
    else
        k_trace_coop<false><<<grid, kCoopBlock, 0, stream>>>(s, r, n, static_cast<uint2*>(out), nullptr, err, cursor);
    return cudaGetLastError();
}

int trace_coop_blocks_per_sm(int any_hit) {
    int b = 0;
    if (any_hit) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_trace_coop<true>, kCoopBlock, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_trace_coop<false>, kCoopBlock, 0);
    return b > 0 ? b : 1;
}

cudaError_t launch_trace_persist(const DeviceScene& s, const rbr_ray* rays, uint32_t n, int any_hit, void* out,
                                 int* err, uint32_t* cursor, int grid, cudaStream_t stream, const uint32_t* perm,
                                 uint32_t refill_min) {
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(cursor, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    const auto* r = reinterpret_cast<const float4*>(rays);
    if (any_hit)
        k_trace_persist<true><<<grid, kPersistBlock, 0, stream>>>(s, r, n, perm, nullptr, static_cast<uint8_t*>(out),
                                                                  err, cursor, refill_min);
    else
        k_trace_persist<false><<<grid, kPersistBlock, 0, stream>>>(s, r, n, perm, static_cast<uint2*>(out), nullptr,
                                                                   err, cursor, refill_min);
    return cudaGetLastError();
}

// The sort buffers of the streams of a chunked rbr_trace_host (slot 0: the context's stream).
static DevBuf& sort_slot(rbr_ctx* ctx, int slot) {
    return slot <= 0 ? ctx->sort_buf : slot == 1 ? ctx->sort_buf2 : ctx->sort_more[slot == 2 ? 0 : 1];
}

// Sorts the rays by their key of order ctx->trace_order on `stream` and returns the permutation:
// orders 4 and 5 by the counting sort above, orders 1-3 (21- and 30-bit keys) by CUB's radix sort.
static cudaError_t sort_rays(rbr_ctx* ctx, DevBuf& sort_buf, const rbr_ray* rays, uint32_t n, const uint32_t** perm,
                             cudaStream_t stream) {
    const int order = ctx->trace_order;
    float3 lo = make_float3(0.0f, 0.0f, 0.0f), sc = make_float3(0.0f, 0.0f, 0.0f);
    const float* blo = ctx->bounds_lo;
    const float* bhi = ctx->bounds_hi;
    float* so[3] = {&sc.x, &sc.y, &sc.z};
    float* lo3[3] = {&lo.x, &lo.y, &lo.z};
    for (int a = 0; a < 3; ++a) {
        const float ext = bhi[a] - blo[a];
        if (std::isfinite(blo[a]) && std::isfinite(ext) && ext > 0.0f) {
            *lo3[a] = blo[a];
            *so[a] = 512.0f / ext;
        }
    }
    const int grid = std::min<int>((n + 255) / 256, ctx->num_sms * 8);
    if (order >= 4) {  // 16-bit keys: the counting sort above
        const size_t perm_bytes = (size_t(n) * 4 + 255) & ~size_t(255);
        const size_t key_bytes = (size_t(n) * 2 + 255) & ~size_t(255);
        if (ensure(ctx, sort_buf, perm_bytes + key_bytes + (kKeyValues + kScanChunks) * 4, "ray sort") != RBR_OK)
            return cudaErrorMemoryAllocation;
        char* base = static_cast<char*>(sort_buf.ptr);
        auto* pm = reinterpret_cast<uint32_t*>(base);
        auto* keys = reinterpret_cast<uint16_t*>(base + perm_bytes);
        auto* counts = reinterpret_cast<uint32_t*>(base + perm_bytes + key_bytes);
        uint32_t* chunk_sum = counts + kKeyValues;
        cudaError_t e = cudaMemsetAsync(counts, 0, kKeyValues * 4, stream);
        if (e != cudaSuccess) return e;
        k_ray_keys16<<<grid, 256, 0, stream>>>(reinterpret_cast<const float4*>(rays), n, lo, sc, order, keys, counts);
        k_key_offsets<<<kScanChunks, kScanThreads, 0, stream>>>(counts, chunk_sum);
        k_ray_scatter16<<<grid, 256, 0, stream>>>(keys, n, counts, chunk_sum, pm);
        *perm = pm;
        return cudaGetLastError();
    }
    const int key_bits = order == 1 ? 30 : 21;
    size_t temp = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, temp, static_cast<const uint32_t*>(nullptr),
                                                    static_cast<uint32_t*>(nullptr), static_cast<const uint32_t*>(nullptr),
                                                    static_cast<uint32_t*>(nullptr), static_cast<int>(n), 0, key_bits, stream);
    if (e != cudaSuccess) return e;
    if (ensure(ctx, sort_buf, size_t(n) * 16 + temp + 256, "ray sort") != RBR_OK) return cudaErrorMemoryAllocation;
    uint32_t* base = static_cast<uint32_t*>(sort_buf.ptr);
    uint32_t *keys = base, *keys2 = base + n, *idx = base + 2 * size_t(n), *idx2 = base + 3 * size_t(n);
    void* tmp = reinterpret_cast<char*>(base + 4 * size_t(n)) + (256 - (reinterpret_cast<uintptr_t>(base + 4 * size_t(n)) & 255));
    k_ray_keys<<<grid, 256, 0, stream>>>(reinterpret_cast<const float4*>(rays), n, lo, sc, order, keys, idx);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cub::DeviceRadixSort::SortPairs(tmp, temp, keys, keys2, idx, idx2, static_cast<int>(n), 0, key_bits, stream);
    *perm = idx2;
    return e;
}

cudaError_t launch_trace(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, int any_hit, void* out, cudaStream_t stream,
                         int slot) {
    if (ctx->trace_kernel == 0 && ctx->trace_order != 0 && n > 0) {
        const uint32_t* perm = nullptr;
        cudaError_t e = sort_rays(ctx, sort_slot(ctx, slot), rays, n, &perm, stream);
        if (e != cudaSuccess) return e;
        const uint32_t blocks = (n + kTraceBlock - 1) / kTraceBlock;
        const auto* r = reinterpret_cast<const float4*>(rays);
        if (any_hit) {
            k_trace_any_perm<<<blocks, kTraceBlock, 0, stream>>>(ctx->scene, r, n, perm, static_cast<uint8_t*>(out),
                                                                ctx->d_error);
        } else {
            auto* h = static_cast<uint2*>(out);
            const bool st = ctx->trace_stream_io != 0;
            const int mb = ctx->trace_min_blocks;
            auto k = ctx->trace_node_test == 1
                         ? (mb >= 12 ? k_trace_closest_perm<12, true, true>
                            : mb >= 10 ? k_trace_closest_perm<10, true, true> : k_trace_closest_perm<8, true, true>)
                     : mb >= 12 ? (st ? k_trace_closest_perm<12, true> : k_trace_closest_perm<12, false>)
                     : mb >= 10 ? (st ? k_trace_closest_perm<10, true> : k_trace_closest_perm<10, false>)
                                : (st ? k_trace_closest_perm<8, true> : k_trace_closest_perm<8, false>);
            return launch_query(ctx, k, blocks, stream, ctx->scene, r, n, perm, h, ctx->d_error);
        }
        return cudaGetLastError();
    }
    if (ctx->trace_kernel == 0) {
        if (any_hit)
            return launch_trace_any(ctx->scene, rays, n, static_cast<uint8_t*>(out), ctx->d_error, ctx->trace_min_blocks,
                                    stream);
        if (n == 0) return cudaSuccess;
        const uint32_t blocks = (n + kTraceBlock - 1) / kTraceBlock;
        const auto* r = reinterpret_cast<const float4*>(rays);
        auto* h = static_cast<uint2*>(out);
        const bool st = ctx->trace_stream_io != 0;
        const int mb = ctx->trace_min_blocks;
        auto k = mb >= 12 ? (st ? k_trace_closest<12, true> : k_trace_closest<12, false>)
               : mb >= 10 ? (st ? k_trace_closest<10, true> : k_trace_closest<10, false>)
                          : (st ? k_trace_closest<8, true> : k_trace_closest<8, false>);
        return launch_query(ctx, k, blocks, stream, ctx->scene, r, n, h, ctx->d_error);
    }
    const bool coop = ctx->trace_kernel == 2;
    const uint32_t* perm = nullptr;  // kernel 1 refills its lanes in sorted order when trace.order is set
    if (!coop && ctx->trace_order != 0 && n > 0) {
        cudaError_t e = sort_rays(ctx, sort_slot(ctx, slot), rays, n, &perm, stream);
        if (e != cudaSuccess) return e;
    }
    const int per_sm = ctx->trace_blocks_per_sm > 0
                           ? ctx->trace_blocks_per_sm
                           : (coop ? trace_coop_blocks_per_sm(any_hit) : trace_persist_blocks_per_sm(any_hit));
    // no more warps than there are chunks of rays
    const int need = static_cast<int>((n + kChunk - 1) / kChunk + (kPersistBlock / 32) - 1) / (kPersistBlock / 32);
    const int grid = std::max(1, std::min(ctx->num_sms * per_sm, need));
    uint32_t* cursor = ctx->d_cursors + (ctx->cursor_next++ % kCursorRing);
    if (coop) return launch_trace_coop(ctx->scene, rays, n, any_hit, out, ctx->d_error, cursor, grid, stream);
    return launch_trace_persist(ctx->scene, rays, n, any_hit, out, ctx->d_error, cursor, grid, stream, perm,
                                static_cast<uint32_t>(ctx->trace_refill_min));
}

// Times every traversal variant on the caller's rays (device pointer) and keeps the fastest.
rbr_status autotune_trace(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, int any_hit, int64_t* chosen_ms_x1000) {
    struct Cand {
        int kernel, min_blocks, per_sm, order, node_test;
    };
    // Unsorted variants, and sorted ones with the 16-bit keys of orders 4 and 5 (the counting
    // sort of this file) and either node test. Orders 1-3 (CUB's radix sort) stay selectable
    // by parameter; measured slower than orders 4 and 5, they are not candidates.
    const Cand cands[] = {{0, 8, 0, 0, 0},  {0, 10, 0, 0, 0}, {0, 12, 0, 0, 0}, {1, 10, 0, 0, 0}, {2, 10, 0, 0, 0},
                          {0, 8, 0, 4, 0},  {0, 10, 0, 4, 0}, {0, 10, 0, 5, 0}, {0, 12, 0, 5, 0}, {0, 8, 0, 5, 1},
                          {0, 10, 0, 4, 1}, {0, 10, 0, 5, 1}, {0, 12, 0, 5, 1}, {1, 10, 0, 5, 0}};
    rbr_status st = ensure(ctx, ctx->stage_out, size_t(n) * (any_hit ? 1 : sizeof(rbr_hit)), "autotune output");
    if (st != RBR_OK) return st;
    const Cand saved{ctx->trace_kernel, ctx->trace_min_blocks, ctx->trace_blocks_per_sm, ctx->trace_order,
                     ctx->trace_node_test};
    float best_ms = 1e30f;
    Cand best = saved;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    for (const Cand& c : cands) {
        ctx->trace_kernel = c.kernel;
        ctx->trace_min_blocks = c.min_blocks;
        ctx->trace_blocks_per_sm = c.per_sm;
        ctx->trace_order = c.order;
        ctx->trace_node_test = c.node_test;
        cudaError_t e = launch_trace(ctx, rays, n, any_hit, ctx->stage_out.ptr, ctx->stream);  // warm-up
        float ms = 0.0f, total = 0.0f;
        for (int k = 0; k < 3 && e == cudaSuccess; ++k) {
            cudaEventRecord(a, ctx->stream);
            e = launch_trace(ctx, rays, n, any_hit, ctx->stage_out.ptr, ctx->stream);
            cudaEventRecord(b, ctx->stream);
            cudaEventSynchronize(b);
            cudaEventElapsedTime(&ms, a, b);
            total += ms;
        }
        if (e != cudaSuccess) {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
            ctx->trace_kernel = saved.kernel;
            ctx->trace_min_blocks = saved.min_blocks;
            ctx->trace_blocks_per_sm = saved.per_sm;
            ctx->trace_order = saved.order;
            ctx->trace_node_test = saved.node_test;
            return cuda_fail(ctx, e, "autotune launch");
        }
        if (total < best_ms) {
            best_ms = total;
            best = c;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    ctx->trace_kernel = best.kernel;
    ctx->trace_min_blocks = best.min_blocks;
    ctx->trace_blocks_per_sm = best.per_sm;
    ctx->trace_order = best.order;
    ctx->trace_node_test = best.node_test;
    if (chosen_ms_x1000) *chosen_ms_x1000 = static_cast<int64_t>(best_ms / 3.0f * 1000.0f);
    return check_device_error(ctx, ctx->stream);
}

int trace_persist_blocks_per_sm(int any_hit) {
    int b = 0;
    if (any_hit) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_trace_persist<true>, kPersistBlock, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_trace_persist<false>, kPersistBlock, 0);
    return b > 0 ? b : 1;
}

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
                                 int min_blocks, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const uint32_t blocks = (n + kTraceBlock - 1) / kTraceBlock;
    const auto* r = reinterpret_cast<const float4*>(rays);
    auto* h = reinterpret_cast<uint2*>(hits);
    if (min_blocks >= 12) k_trace_closest<12, true><<<blocks, kTraceBlock, 0, stream>>>(s, r, n, h, err);
    else if (min_blocks >= 10) k_trace_closest<10, true><<<blocks, kTraceBlock, 0, stream>>>(s, r, n, h, err);
    else k_trace_closest<8, true><<<blocks, kTraceBlock, 0, stream>>>(s, r, n, h, err);
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
