// Radiance cache on the tensor cores: multiresolution hash-grid encoding fused with a 64-wide
// five-matrix MLP (inference), the same forward pass followed by the backward pass, weight
// gradients and hash-grid gradient scatter (training), and Adam.
//
// One CTA of 128 threads owns a tile of 128 samples: thread r encodes sample r and writes its
// 64 BF16 inputs as row r of the A operand in shared memory; one thread issues the
// tcgen05.mma instructions of a layer (M = 128 samples, K = 64, N = 64 or 16), FP32
// accumulators land in tensor memory, every thread reads back its own row (TMEM lane r),
// applies ReLU, rounds to BF16 and writes the next layer's A operand.
//
// Training keeps every activation of the tile (a0..a4, 320 features a row) and every
// back-propagated error (d1..d4 and the output error, 272 features a row) in shared memory:
//   d_l = (d_{l+1} W_l) * [a_l > 0]          M = 128 samples, N = 64, K = 64 (16 for W4),
//   the W operand read transposed (MN-major) from the same shared copy as the forward pass;
//   dW_l^T = a_l^T d_{l+1}                   contraction over the 128 samples: M = features,
//   both operands MN-major views of the activation and error buffers. Two layers share one
//   M = 128, N = 128 product: [a0 a1]^T [d1 d2] holds dW0^T and dW1^T on its diagonal
//   blocks (the off-diagonal blocks are not used), [a2 a3]^T [d3 d4] holds dW2^T and dW3^T,
//   and [a4 -]^T dy (N = 16) holds dW4^T. They accumulate in tensor memory over all tiles
//   a CTA processes and are added to the global FP32 gradients once, at the end.
//   The gradient of the 32 hash features, d1 W0[:, :32] (N = 32), is scattered to the FP32
//   grid gradient with the trilinear weights of the forward pass.
//
// Methods: multiresolution hash encoding (Mueller, Evans, Schied, Keller, SIGGRAPH 2022),
// spatial hash with the primes 1, 2654435761, 805459861; Adam (Kingma & Ba 2015); the
// relative L2 loss and online training of neural radiance caching (Mueller, Rousselle, Novak,
// Keller, SIGGRAPH 2021). None of this has a counterpart in the reference renderer.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "rbr_bsdf.cuh"
#include "rbr_cache.h"
#include "rbr_context.h"
#include "rbr_sort.cuh"
#include "rbr_tc.cuh"

namespace rbr {

namespace {

// --------------------------------------------------------------------------------------------
// Shared-memory layout (bytes)
// --------------------------------------------------------------------------------------------
constexpr uint32_t kWBytes = kRcWeights * 2;          // 34816: W0..W3 at l*8192, W4 at 32768
constexpr uint32_t kActRgTrain = 384 / 8 * 128;       // 6144: one 8-row group of 384 features
constexpr uint32_t kActBytesTrain = 16 * kActRgTrain; // 98304
constexpr uint32_t kDelRg = 272 / 8 * 128;            // 4352: one 8-row group of 272 features
constexpr uint32_t kDelBytes = 16 * kDelRg;           // 69632
constexpr uint32_t kActRgInfer = 64 / 8 * 128;        // 1024
constexpr uint32_t kActBytesInfer = 16 * kActRgInfer; // 16384
constexpr uint32_t kMisc = 64;
constexpr uint32_t kSmemTrain = kWBytes + kActBytesTrain + kDelBytes + kMisc;  // 202816
constexpr uint32_t kSmemInfer = kWBytes + kActBytesInfer + kMisc;              // 51264
constexpr uint32_t kTmemTrain = 512;   // [0,64) layer accumulator, 128/256: weight-gradient pairs, 384: dW4
constexpr uint32_t kTmemInfer = 64;

// Byte offset of element (row, feature) in a buffer of 8x8 core matrices whose 8-row groups
// are `rg` bytes apart (K-major for the row-major reading, MN-major for the transposed one).
__device__ __forceinline__ uint32_t cm_off(uint32_t row, uint32_t feat, uint32_t rg) {
    return (row >> 3) * rg + (feat >> 3) * 128u + (row & 7u) * 16u + (feat & 7u) * 2u;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Writes features [f0, f0 + 8*chunks) of row `row` (BF16, round to nearest even).
__device__ __forceinline__ void store_row(uint8_t* buf, uint32_t rg, uint32_t row, uint32_t f0, const float* v,
                                          int chunks) {
#pragma unroll
    for (int c = 0; c < chunks; ++c) {
        uint4 q;
        q.x = pack_bf16(v[8 * c + 0], v[8 * c + 1]);
        q.y = pack_bf16(v[8 * c + 2], v[8 * c + 3]);
        q.z = pack_bf16(v[8 * c + 4], v[8 * c + 5]);
        q.w = pack_bf16(v[8 * c + 6], v[8 * c + 7]);
        *reinterpret_cast<uint4*>(buf + cm_off(row, f0 + 8 * c, rg)) = q;
    }
}

// Row `row`, features [f0, f0+64) as 64 booleans "value > 0" (ReLU derivative).
__device__ __forceinline__ void load_positive(const uint8_t* buf, uint32_t rg, uint32_t row, uint32_t f0,
                                              uint64_t& mask) {
    mask = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const uint4 q = *reinterpret_cast<const uint4*>(buf + cm_off(row, f0 + 8 * c, rg));
        const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            // BF16 x > 0: sign bit clear and not +0
            const uint32_t lo = w[i] & 0xFFFFu, hi = w[i] >> 16;
            if (lo != 0 && (lo & 0x8000u) == 0) mask |= 1ull << (8 * c + 2 * i);
            if (hi != 0 && (hi & 0x8000u) == 0) mask |= 1ull << (8 * c + 2 * i + 1);
        }
    }
}

// Copies the row-major BF16 weights into the core-matrix layout (row = output neuron).
__device__ __forceinline__ void load_weights(const __nv_bfloat16* w, uint8_t* ws) {
    const uint4* src = reinterpret_cast<const uint4*>(w);
    for (uint32_t q = threadIdx.x; q < kRcWeights / 8; q += blockDim.x) {
        const uint32_t e = q * 8;
        const uint32_t layer = e < 4 * 4096 ? e / 4096 : 4;
        const uint32_t r = (e - layer * 4096) / 64, col = (e - layer * 4096) % 64;
        *reinterpret_cast<uint4*>(ws + layer * 8192 + cm_off(r, col, 1024)) = __ldg(src + q);
    }
}

// --------------------------------------------------------------------------------------------
// Hash-grid encoding
// --------------------------------------------------------------------------------------------
__device__ __forceinline__ float clamp01(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }

__device__ __forceinline__ void unit_position(const CacheDev& c, float4 r0, float p[3]) {
    p[0] = clamp01(fm(fs(r0.x, c.lo[0]), c.inv_ext[0]));
    p[1] = clamp01(fm(fs(r0.y, c.lo[1]), c.inv_ext[1]));
    p[2] = clamp01(fm(fs(r0.z, c.lo[2]), c.inv_ext[2]));
}

// Cell of level l containing p: lower corner i and fractional position w (both per axis).
__device__ __forceinline__ void level_cell(const CacheDev& c, int l, const float p[3], uint32_t i[3], float w[3]) {
    const uint32_t n = c.res[l];
    const float nf = static_cast<float>(n);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float x = fm(p[a], nf);
        uint32_t xi = static_cast<uint32_t>(floorf(x));
        if (xi > n - 1) xi = n - 1;
        i[a] = xi;
        w[a] = fs(x, static_cast<float>(xi));
    }
}

__device__ __forceinline__ uint32_t corner_index(const CacheDev& c, int l, const uint32_t i[3], int k) {
    const uint32_t x = i[0] + (k & 1), y = i[1] + ((k >> 1) & 1), z = i[2] + (k >> 2);
    if ((c.dense_mask >> l) & 1u) {
        const uint32_t n1 = c.res[l] + 1;
        return x + n1 * (y + n1 * z);
    }
    return (x ^ (y * 2654435761u) ^ (z * 805459861u)) & ((1u << c.log2_table) - 1u);
}

__device__ __forceinline__ float corner_weight(const float w[3], int k) {
    const float wx = (k & 1) ? w[0] : fs(1.0f, w[0]);
    const float wy = ((k >> 1) & 1) ? w[1] : fs(1.0f, w[1]);
    const float wz = (k >> 2) ? w[2] : fs(1.0f, w[2]);
    return fm(fm(wx, wy), wz);
}

// The 64 network inputs of a record, FP32 (rounded to BF16 when stored as the A operand):
//   [0,32)  hash features, level l at 2l, 2l+1 (trilinear over the cell's 8 corners)
//   [32,47) direction, per axis five tent functions max(0, 1 - |2(d+1) - k|), k = 0..4
//   [47,50) normal, [50] roughness, [51,54) diffuse albedo, [54,57) specular albedo,
//   [57] 1 (bias), [58,64) 0
__device__ __forceinline__ void encode(const CacheDev& c, const float4* rec, float* in) {
    const float4 r0 = __ldg(rec), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2), r3 = __ldg(rec + 3);
    float p[3];
    unit_position(c, r0, p);
#pragma unroll
    for (int l = 0; l < kRcLevels; ++l) {
        uint32_t i[3];
        float w[3];
        level_cell(c, l, p, i, w);
        const __half2* tab = c.grid + (static_cast<size_t>(l) << c.log2_table);
        float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float wt = corner_weight(w, k);
            const float2 v = __half22float2(__ldg(tab + corner_index(c, l, i, k)));
            f0 = fa(f0, fm(wt, v.x));
            f1 = fa(f1, fm(wt, v.y));
        }
        in[2 * l] = f0;
        in[2 * l + 1] = f1;
    }
    const float d[3] = {r0.w, r1.x, r1.y};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float s = fm(fa(d[a], 1.0f), 2.0f);
#pragma unroll
        for (int k = 0; k < 5; ++k) in[32 + 5 * a + k] = fmaxf(0.0f, fs(1.0f, fabsf(fs(s, static_cast<float>(k)))));
    }
    in[47] = r1.z;
    in[48] = r1.w;
    in[49] = r2.x;
    in[50] = r2.y;
    in[51] = r2.z;
    in[52] = r2.w;
    in[53] = r3.x;
    in[54] = r3.y;
    in[55] = r3.z;
    in[56] = r3.w;
    in[57] = 1.0f;
#pragma unroll
    for (int k = 58; k < 64; ++k) in[k] = 0.0f;
}

// Adds the gradient of the 32 hash features of one sample to the grid gradient.
__device__ __forceinline__ void scatter_grid_grad(const CacheDev& c, float4 r0, const float* g) {
    float p[3];
    unit_position(c, r0, p);
#pragma unroll 1
    for (int l = 0; l < kRcLevels; ++l) {
        const float g0 = g[2 * l], g1 = g[2 * l + 1];
        if (g0 == 0.0f && g1 == 0.0f) continue;
        uint32_t i[3];
        float w[3];
        level_cell(c, l, p, i, w);
        float2* tab = c.grid_grad + (static_cast<size_t>(l) << c.log2_table);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float wt = corner_weight(w, k);
            atomicAdd(tab + corner_index(c, l, i, k), make_float2(fm(wt, g0), fm(wt, g1)));
        }
    }
}

// Waits for the pending tensor-core work (at most `limit` polls); all threads agree on the
// outcome. A wait that ran out sets kErrDeviceTimeout; the kernel then stops issuing work and
// drains the outstanding MMA with the full bound before it frees its tensor memory.
__device__ __forceinline__ bool wait_mma(uint64_t* mbar, uint32_t& phase, int* err, uint32_t limit) {
    const bool done = tc::mbar_wait(mbar, phase, limit);
    phase ^= 1u;
    const int bad = __syncthreads_or(done ? 0 : 1);
    if (bad && threadIdx.x == 0) atomicOr(err, kErrDeviceTimeout);
    return bad == 0;
}

// Makes this thread's shared-memory writes and finished TMEM reads visible before the MMA
// issuer runs (the issuer then calls fence_after_sync).
__device__ __forceinline__ void publish() {
    tc::fence_smem_async();
    tc::fence_before_sync();
    __syncthreads();
}

__device__ __forceinline__ void ld64(uint32_t taddr, float* v) {
#pragma unroll
    for (int q = 0; q < 4; ++q) tc::tmem_ld16(taddr + 16 * q, v + 16 * q);
}

// Records available to a training batch: the first list [0, n0) and, with count2_ptr, a
// second list that starts at `split`; i-th available record -> its index.
__device__ __forceinline__ uint32_t batch_avail(const TrainBatchDev& b, uint32_t& n0) {
    if (!b.count_ptr) {
        n0 = b.count;
        return b.count;
    }
    n0 = min(*b.count_ptr, b.cap);
    return n0 + (b.count2_ptr ? min(*b.count2_ptr, b.cap) : 0u);
}
__device__ __forceinline__ uint32_t batch_record(const TrainBatchDev& b, uint32_t i, uint32_t n0) {
    return i < n0 ? i : b.split + (i - n0);
}

__device__ __forceinline__ uint32_t shuffle_index(uint32_t x, uint32_t n) {
    return static_cast<uint32_t>((static_cast<uint64_t>(x) * 2654435761ull + 0x9E3779B9ull) % n);
}

// --------------------------------------------------------------------------------------------
// Inference: prediction (RGB) per record. Output either to rgb[n x 3], or added, times the
// path throughput, to the radiance of the path that ended into the cache.
// --------------------------------------------------------------------------------------------
struct InferOut {
    float* rgb;
    float4* path_rad;
    const float4* q_info;  // throughput rgb, path index bits
    const uint32_t* perm;  // optional: tile slot j serves query perm[j] (queries sorted by cell)
};

__global__ void __launch_bounds__(128, 4)
    k_rc_infer(CacheDev c, const float4* records, uint32_t n, const uint32_t* n_ptr, InferOut o, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* ws = smem;
    uint8_t* act = smem + kWBytes;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kWBytes + kActBytesInfer);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kWBytes + kActBytesInfer + 8);
    const uint32_t count = n_ptr ? min(*n_ptr, n) : n;
    const uint32_t tiles = (count + kRcTile - 1) / kRcTile;
    if (blockIdx.x >= tiles) return;
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) tc::mbar_init(mbar, 1);
    load_weights(c.w, ws);
    if (warp == 0) {
        tc::tmem_alloc(tslot, kTmemInfer);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = *tslot;
    const uint32_t tl = tm + ((warp * 32u) << 16);
    const uint32_t act_s = tc::smem_addr(act), w_s = tc::smem_addr(ws);
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const uint32_t j = tile * kRcTile + tid;
        const bool valid = j < count;
        const uint32_t src = valid && o.perm ? __ldg(o.perm + j) : j;  // the query this slot serves
        {
            float in[64];
            if (valid) encode(c, records + 4 * static_cast<size_t>(src), in);
            else
#pragma unroll
                for (int k = 0; k < 64; ++k) in[k] = 0.0f;
            store_row(act, kActRgInfer, tid, 0, in, 8);
        }
        float y[16];
        for (int l = 0; l < 5 && ok; ++l) {
            publish();
            if (tid == 0) {
                tc::fence_after_sync();
                const uint32_t id = tc::idesc_bf16(128, l < 4 ? 64 : 16, 0, 0);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    tc::mma_bf16(tm, tc::sdesc(act_s + k * 256, 128, kActRgInfer),
                                 tc::sdesc(w_s + l * 8192 + k * 256, 128, 1024), id, k > 0);
                tc::mma_commit(mbar);
            }
            ok = wait_mma(mbar, phase, err, c.wait_limit);
            if (!ok) break;
            tc::fence_after_sync();
            if (l < 4) {
                float z[64];
                ld64(tl, z);
#pragma unroll
                for (int k = 0; k < 64; ++k) z[k] = fmaxf(z[k], 0.0f);
                store_row(act, kActRgInfer, tid, 0, z, 8);
            } else {
                tc::tmem_ld16(tl, y);
            }
        }
        if (ok && valid) {
            const float r = fmaxf(y[0], 0.0f), g = fmaxf(y[1], 0.0f), b = fmaxf(y[2], 0.0f);
            if (o.rgb) {
                o.rgb[3 * static_cast<size_t>(src)] = r;
                o.rgb[3 * static_cast<size_t>(src) + 1] = g;
                o.rgb[3 * static_cast<size_t>(src) + 2] = b;
            } else {
                const float4 q = o.q_info[src];
                float4* L = o.path_rad + __float_as_uint(q.w);
                float4 v = *L;
                v.x = fa(v.x, fm(q.x, r));
                v.y = fa(v.y, fm(q.y, g));
                v.z = fa(v.z, fm(q.z, b));
                *L = v;
            }
        }
    }
    if (!ok) tc::mbar_wait(mbar, phase ^ 1u);  // let an overdue MMA drain before freeing TMEM
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tm, kTmemInfer);
    }
}

// --------------------------------------------------------------------------------------------
// Inference with eight warps per 128-sample tile: thread t and thread t + 128 share row t & 127.
// The first half encodes hash levels 0-7 (features 0-15), the second levels 8-15 and the other
// 32 features; in the epilogues warp w reads the accumulator lanes of quarter w % 4 and the
// column half w / 4. A thread then holds half the values of the four-warp kernel, so four CTAs
// of 256 threads fit an SM (twice the warps to hide the hash-grid gathers), and each thread
// issues half the gathers. Same arithmetic per feature, so the same results as k_rc_infer.
// --------------------------------------------------------------------------------------------
// Part `part` (0 or 1) of the encoding of `rec`, written into row `row` of the A operand.
__device__ __forceinline__ void encode_part(const CacheDev& c, const float4* rec, uint8_t* act, uint32_t rg,
                                            uint32_t row, uint32_t part) {
    const float4 r0 = __ldg(rec);
    float p[3];
    unit_position(c, r0, p);
#pragma unroll 1
    for (int q = 0; q < 2; ++q) {
        float v[8];
#pragma unroll
        for (int ll = 0; ll < 4; ++ll) {
            const int l = 8 * static_cast<int>(part) + 4 * q + ll;
            uint32_t i[3];
            float w[3];
            level_cell(c, l, p, i, w);
            const __half2* tab = c.grid + (static_cast<size_t>(l) << c.log2_table);
            float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float wt = corner_weight(w, k);
                const float2 g = __half22float2(__ldg(tab + corner_index(c, l, i, k)));
                f0 = fa(f0, fm(wt, g.x));
                f1 = fa(f1, fm(wt, g.y));
            }
            v[2 * ll] = f0;
            v[2 * ll + 1] = f1;
        }
        store_row(act, rg, row, 16 * part + 8 * q, v, 1);
    }
    if (part == 0) return;
    const float4 r1 = __ldg(rec + 1), r2 = __ldg(rec + 2), r3 = __ldg(rec + 3);
    float v[32];
    const float d[3] = {r0.w, r1.x, r1.y};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float t = fm(fa(d[a], 1.0f), 2.0f);
#pragma unroll
        for (int k = 0; k < 5; ++k) v[5 * a + k] = fmaxf(0.0f, fs(1.0f, fabsf(fs(t, static_cast<float>(k)))));
    }
    v[15] = r1.z;
    v[16] = r1.w;
    v[17] = r2.x;
    v[18] = r2.y;
    v[19] = r2.z;
    v[20] = r2.w;
    v[21] = r3.x;
    v[22] = r3.y;
    v[23] = r3.z;
    v[24] = r3.w;
    v[25] = 1.0f;
#pragma unroll
    for (int k = 26; k < 32; ++k) v[k] = 0.0f;
    store_row(act, rg, row, 32, v, 4);
}

__global__ void __launch_bounds__(256, 4)
    k_rc_infer8(CacheDev c, const float4* records, uint32_t n, const uint32_t* n_ptr, InferOut o, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* ws = smem;
    uint8_t* act = smem + kWBytes;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kWBytes + kActBytesInfer);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kWBytes + kActBytesInfer + 8);
    const uint32_t count = n_ptr ? min(*n_ptr, n) : n;
    const uint32_t tiles = (count + kRcTile - 1) / kRcTile;
    if (blockIdx.x >= tiles) return;
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t row = tid & 127u, part = tid >> 7;  // part: encoding half and column half
    if (tid == 0) tc::mbar_init(mbar, 1);
    load_weights(c.w, ws);
    if (warp == 0) {
        tc::tmem_alloc(tslot, kTmemInfer);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = *tslot;
    const uint32_t tl = tm + (((warp & 3u) * 32u) << 16) + 32u * part;  // lane quarter, column half
    const uint32_t act_s = tc::smem_addr(act), w_s = tc::smem_addr(ws);
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const uint32_t j = tile * kRcTile + row;
        const bool valid = j < count;
        const uint32_t src = valid && o.perm ? __ldg(o.perm + j) : j;  // the query this slot serves
        if (valid) {
            encode_part(c, records + 4 * static_cast<size_t>(src), act, kActRgInfer, row, part);
        } else {
            float z[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) z[k] = 0.0f;
            for (uint32_t q = 2 * part; q < (part ? 8u : 2u); ++q) store_row(act, kActRgInfer, row, 8 * q, z, 1);
        }
        float y[16];
        for (int l = 0; l < 5 && ok; ++l) {
            publish();
            if (tid == 0) {
                tc::fence_after_sync();
                const uint32_t id = tc::idesc_bf16(128, l < 4 ? 64 : 16, 0, 0);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    tc::mma_bf16(tm, tc::sdesc(act_s + k * 256, 128, kActRgInfer),
                                 tc::sdesc(w_s + l * 8192 + k * 256, 128, 1024), id, k > 0);
                tc::mma_commit(mbar);
            }
            ok = wait_mma(mbar, phase, err, c.wait_limit);
            if (!ok) break;
            tc::fence_after_sync();
            if (l < 4) {
                float z[32];
                tc::tmem_ld16(tl, z);
                tc::tmem_ld16(tl + 16, z + 16);
#pragma unroll
                for (int k = 0; k < 32; ++k) z[k] = fmaxf(z[k], 0.0f);
                store_row(act, kActRgInfer, row, 32 * part, z, 4);
            } else if (part == 0) {
                tc::tmem_ld16(tl, y);
            }
        }
        if (ok && valid && part == 0) {
            const float r = fmaxf(y[0], 0.0f), g = fmaxf(y[1], 0.0f), b = fmaxf(y[2], 0.0f);
            if (o.rgb) {
                o.rgb[3 * static_cast<size_t>(src)] = r;
                o.rgb[3 * static_cast<size_t>(src) + 1] = g;
                o.rgb[3 * static_cast<size_t>(src) + 2] = b;
            } else {
                const float4 q = o.q_info[src];
                float4* L = o.path_rad + __float_as_uint(q.w);
                float4 v = *L;
                v.x = fa(v.x, fm(q.x, r));
                v.y = fa(v.y, fm(q.y, g));
                v.z = fa(v.z, fm(q.z, b));
                *L = v;
            }
        }
    }
    if (!ok) tc::mbar_wait(mbar, phase ^ 1u);  // let an overdue MMA drain before freeing TMEM
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tm, kTmemInfer);
    }
}

// --------------------------------------------------------------------------------------------
// Inference with several tiles in flight per CTA: G groups of 128 threads (four warps) each own
// a 128-sample tile and run its chain (encode, five layers of MMA, commit, wait, epilogue)
// independently of the other groups, with a named barrier per group instead of the CTA
// barrier; the weights are loaded once per CTA and shared. While one group waits for its MMAs
// or its hash-grid gathers, the others issue. The encoding and the epilogues stream eight or
// sixteen features at a time, so that a thread keeps few values live and two CTAs of four
// groups fit an SM (eight tiles in flight instead of four).
// --------------------------------------------------------------------------------------------
__device__ __forceinline__ void group_sync(uint32_t g) { asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory"); }
// OR of `v` over the group's 128 threads (a barrier of the group).
__device__ __forceinline__ bool group_any(uint32_t g, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %2, 0;\n\t"
        "bar.red.or.pred q, %1, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"(1 + g), "r"(v ? 1u : 0u)
        : "memory");
    return r != 0;
}

// The encoding of `encode`, written as row `row` of the A operand eight features at a time.
__device__ __forceinline__ void encode_row(const CacheDev& c, const float4* rec, uint8_t* act, uint32_t rg,
                                           uint32_t row) {
    const float4 r0 = __ldg(rec), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2), r3 = __ldg(rec + 3);
    float p[3];
    unit_position(c, r0, p);
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
        float v[8];
#pragma unroll
        for (int ll = 0; ll < 4; ++ll) {
            const int l = 4 * q + ll;
            uint32_t i[3];
            float w[3];
            level_cell(c, l, p, i, w);
            const __half2* tab = c.grid + (static_cast<size_t>(l) << c.log2_table);
            float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float wt = corner_weight(w, k);
                const float2 g = __half22float2(__ldg(tab + corner_index(c, l, i, k)));
                f0 = fa(f0, fm(wt, g.x));
                f1 = fa(f1, fm(wt, g.y));
            }
            v[2 * ll] = f0;
            v[2 * ll + 1] = f1;
        }
        store_row(act, rg, row, 8 * q, v, 1);
    }
    float v[32];
    const float d[3] = {r0.w, r1.x, r1.y};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float t = fm(fa(d[a], 1.0f), 2.0f);
#pragma unroll
        for (int k = 0; k < 5; ++k) v[5 * a + k] = fmaxf(0.0f, fs(1.0f, fabsf(fs(t, static_cast<float>(k)))));
    }
    v[15] = r1.z;
    v[16] = r1.w;
    v[17] = r2.x;
    v[18] = r2.y;
    v[19] = r2.z;
    v[20] = r2.w;
    v[21] = r3.x;
    v[22] = r3.y;
    v[23] = r3.z;
    v[24] = r3.w;
    v[25] = 1.0f;
#pragma unroll
    for (int k = 26; k < 32; ++k) v[k] = 0.0f;
    store_row(act, rg, row, 32, v, 4);
}

template <int G>
__global__ void __launch_bounds__(128 * G, 8 / G)
    k_rc_infer_groups(CacheDev c, const float4* records, uint32_t n, const uint32_t* n_ptr, InferOut o, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* ws = smem;
    uint64_t* mbars = reinterpret_cast<uint64_t*>(smem + kWBytes + G * kActBytesInfer);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kWBytes + G * kActBytesInfer + 8 * G);
    const uint32_t count = n_ptr ? min(*n_ptr, n) : n;
    const uint32_t tiles = (count + kRcTile - 1) / kRcTile;
    if (blockIdx.x * G >= tiles) return;
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t g = tid >> 7, lt = tid & 127u;  // tile group, thread within the group
    uint8_t* act = smem + kWBytes + g * kActBytesInfer;
    uint64_t* mbar = mbars + g;
    if (lt == 0) tc::mbar_init(mbar, 1);
    load_weights(c.w, ws);
    if (warp == 0) {
        tc::tmem_alloc(tslot, 64 * G);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = *tslot + 64u * g;                 // the group's 64 accumulator columns
    const uint32_t tl = tm + (((warp & 3u) * 32u) << 16);  // this warp's 32 lanes
    const uint32_t act_s = tc::smem_addr(act), w_s = tc::smem_addr(ws);
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x * G + g; tile < tiles && ok; tile += gridDim.x * G) {
        const uint32_t j = tile * kRcTile + lt;
        const bool valid = j < count;
        const uint32_t src = valid && o.perm ? __ldg(o.perm + j) : j;  // the query this slot serves
        if (valid) {
            encode_row(c, records + 4 * static_cast<size_t>(src), act, kActRgInfer, lt);
        } else {
            float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int q = 0; q < 8; ++q) store_row(act, kActRgInfer, lt, 8 * q, z, 1);
        }
        float y[16];
        for (int l = 0; l < 5 && ok; ++l) {
            tc::fence_smem_async();
            tc::fence_before_sync();
            group_sync(g);
            if (lt == 0) {
                tc::fence_after_sync();
                const uint32_t id = tc::idesc_bf16(128, l < 4 ? 64 : 16, 0, 0);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    tc::mma_bf16(tm, tc::sdesc(act_s + k * 256, 128, kActRgInfer),
                                 tc::sdesc(w_s + l * 8192 + k * 256, 128, 1024), id, k > 0);
                tc::mma_commit(mbar);
            }
            const bool done = tc::mbar_wait(mbar, phase, c.wait_limit);
            phase ^= 1u;
            ok = !group_any(g, !done);
            if (!ok) {
                if (lt == 0) atomicOr(err, kErrDeviceTimeout);
                break;
            }
            tc::fence_after_sync();
            if (l < 4) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    float z[16];
                    tc::tmem_ld16(tl + 16 * q, z);
#pragma unroll
                    for (int k = 0; k < 16; ++k) z[k] = fmaxf(z[k], 0.0f);
                    store_row(act, kActRgInfer, lt, 16 * q, z, 2);
                }
            } else {
                tc::tmem_ld16(tl, y);
            }
        }
        if (ok && valid) {
            const float r = fmaxf(y[0], 0.0f), gg = fmaxf(y[1], 0.0f), b = fmaxf(y[2], 0.0f);
            if (o.rgb) {
                o.rgb[3 * static_cast<size_t>(src)] = r;
                o.rgb[3 * static_cast<size_t>(src) + 1] = gg;
                o.rgb[3 * static_cast<size_t>(src) + 2] = b;
            } else {
                const float4 qi = o.q_info[src];
                float4* L = o.path_rad + __float_as_uint(qi.w);
                float4 v = *L;
                v.x = fa(v.x, fm(qi.x, r));
                v.y = fa(v.y, fm(qi.y, gg));
                v.z = fa(v.z, fm(qi.z, b));
                *L = v;
            }
        }
    }
    if (!ok) tc::mbar_wait(mbar, phase ^ 1u);  // let an overdue MMA drain before freeing TMEM
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(*tslot, 64 * G);
    }
}

constexpr uint32_t smem_infer_groups(int G) { return kWBytes + G * kActBytesInfer + 8 * G + 8; }

// --------------------------------------------------------------------------------------------
// Training: forward + loss gradient + backward + weight and grid gradients for one batch.
// --------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1) k_rc_train(CacheDev c, TrainBatchDev b, float* scalars, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* ws = smem;
    uint8_t* act = smem + kWBytes;
    uint8_t* del = smem + kWBytes + kActBytesTrain;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kWBytes + kActBytesTrain + kDelBytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kWBytes + kActBytesTrain + kDelBytes + 8);
    uint32_t n0 = 0;
    const uint32_t avail = batch_avail(b, n0);
    const uint32_t nsamp = min(b.batch, avail);
    const uint32_t tiles = (nsamp + kRcTile - 1) / kRcTile;
    if (blockIdx.x >= tiles) return;
    const float scale = fd(1.0f, fm(3.0f, static_cast<float>(nsamp)));
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) tc::mbar_init(mbar, 1);
    load_weights(c.w, ws);
    {   // features [320, 384) are read by the dW4 product's unused half: keep them finite
        const uint4 z = make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int q = 0; q < 8; ++q) *reinterpret_cast<uint4*>(act + cm_off(tid, 320 + 8 * q, kActRgTrain)) = z;
    }
    if (warp == 0) {
        tc::tmem_alloc(tslot, kTmemTrain);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = *tslot;
    const uint32_t tl = tm + ((warp * 32u) << 16);
    const uint32_t act_s = tc::smem_addr(act), del_s = tc::smem_addr(del), w_s = tc::smem_addr(ws);
    uint32_t phase = 0;
    bool ok = true, first = true;
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const uint32_t j = tile * kRcTile + tid;
        const bool valid = j < nsamp;
        uint32_t ridx = 0;
        if (valid) ridx = batch_record(b, b.shuffle ? shuffle_index(b.step_index * b.batch + j, avail) : j, n0);
        const float4* rec = b.records + 4 * static_cast<size_t>(ridx);
        float4 tgt = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        {
            float in[64];
            if (valid) {
                encode(c, rec, in);
                tgt = b.targets[ridx];
            } else {
#pragma unroll
                for (int k = 0; k < 64; ++k) in[k] = 0.0f;
            }
            store_row(act, kActRgTrain, tid, 0, in, 8);
        }
        // forward
        float y[16];
        for (int l = 0; l < 5 && ok; ++l) {
            publish();
            if (tid == 0) {
                tc::fence_after_sync();
                const uint32_t id = tc::idesc_bf16(128, l < 4 ? 64 : 16, 0, 0);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    tc::mma_bf16(tm, tc::sdesc(act_s + l * 1024 + k * 256, 128, kActRgTrain),
                                 tc::sdesc(w_s + l * 8192 + k * 256, 128, 1024), id, k > 0);
                tc::mma_commit(mbar);
            }
            ok = wait_mma(mbar, phase, err, c.wait_limit);
            if (!ok) break;
            tc::fence_after_sync();
            if (l < 4) {
                float z[64];
                ld64(tl, z);
#pragma unroll
                for (int k = 0; k < 64; ++k) z[k] = fmaxf(z[k], 0.0f);
                store_row(act, kActRgTrain, tid, 64 * (l + 1), z, 8);
            } else {
                tc::tmem_ld16(tl, y);
            }
        }
        if (!ok) break;
        // relative L2 loss and its gradient (prediction held constant in the denominator)
        {
            float g[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) g[k] = 0.0f;
            float loss = 0.0f;
            if (valid) {
                const uint32_t mask = __float_as_uint(tgt.w);
                const float t[3] = {tgt.x, tgt.y, tgt.z};
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) {
                    if ((mask >> ch) & 1u) {
                        const float d = fs(y[ch], t[ch]);
                        const float den = fa(fm(y[ch], y[ch]), 0.01f);
                        g[ch] = fm(fd(fm(2.0f, d), den), scale);
                        loss = fa(loss, fd(fm(d, d), den));
                    }
                }
            }
            store_row(del, kDelRg, tid, 256, g, 2);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, off);
            if ((tid & 31) == 0 && loss != 0.0f) atomicAdd(scalars + kRcLoss, loss * scale);
        }
        // backward through W4 .. W1
        for (int l = 4; l >= 1 && ok; --l) {
            publish();
            if (tid == 0) {
                tc::fence_after_sync();
                const uint32_t id = tc::idesc_bf16(128, 64, 0, 1);
                const uint32_t a0 = del_s + (l == 4 ? 32u : 8u * l) * 128u;  // error of W_l's output
                const int ks = l == 4 ? 1 : 4;
                for (int k = 0; k < ks; ++k)
                    tc::mma_bf16(tm, tc::sdesc(a0 + k * 256, 128, kDelRg), tc::sdesc(w_s + l * 8192 + k * 2048, 1024, 128),
                                 id, k > 0);
                tc::mma_commit(mbar);
            }
            ok = wait_mma(mbar, phase, err, c.wait_limit);
            if (!ok) break;
            tc::fence_after_sync();
            float z[64];
            ld64(tl, z);
            uint64_t pos;
            load_positive(act, kActRgTrain, tid, 64 * l, pos);
#pragma unroll
            for (int k = 0; k < 64; ++k) z[k] = ((pos >> k) & 1ull) ? z[k] : 0.0f;
            store_row(del, kDelRg, tid, 64 * (l - 1), z, 8);
        }
        if (!ok) break;
        // input gradient of the hash features and the weight gradients
        publish();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t id0 = tc::idesc_bf16(128, 32, 0, 1);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                tc::mma_bf16(tm, tc::sdesc(del_s + k * 256, 128, kDelRg), tc::sdesc(w_s + k * 2048, 1024, 128), id0, k > 0);
            const uint32_t idp = tc::idesc_bf16(128, 128, 1, 1);
            for (int p = 0; p < 2; ++p)
                for (int k = 0; k < 8; ++k)
                    tc::mma_bf16(tm + 128 + 128 * p, tc::sdesc(act_s + p * 2048 + k * 2 * kActRgTrain, kActRgTrain, 128),
                                 tc::sdesc(del_s + p * 2048 + k * 2 * kDelRg, kDelRg, 128), idp, (!first || k > 0) ? 1u : 0u);
            const uint32_t id4 = tc::idesc_bf16(128, 16, 1, 1);
            for (int k = 0; k < 8; ++k)
                tc::mma_bf16(tm + 384, tc::sdesc(act_s + 4096 + k * 2 * kActRgTrain, kActRgTrain, 128),
                             tc::sdesc(del_s + 4096 + k * 2 * kDelRg, kDelRg, 128), id4, (!first || k > 0) ? 1u : 0u);
            tc::mma_commit(mbar);
        }
        ok = wait_mma(mbar, phase, err, c.wait_limit);
        if (!ok) break;
        tc::fence_after_sync();
        first = false;
        {
            float g[32];
            tc::tmem_ld16(tl, g);
            tc::tmem_ld16(tl + 16, g + 16);
            if (valid) scatter_grid_grad(c, __ldg(rec), g);
        }
    }
    if (ok && !first) {
        // weight gradients: lanes 0..63 hold the first matrix of a pair, 64..127 the second
        const uint32_t in = tid & 63u;
        float v[64];
        for (int p = 0; p < 2; ++p) {
            const uint32_t m = 2 * p + (warp >> 1);
            ld64(tl + 128 + 128 * p + 64 * (warp >> 1), v);
            float* gw = c.w_grad + m * 4096 + in;
#pragma unroll 8
            for (int o = 0; o < 64; ++o) atomicAdd(gw + o * 64, v[o]);
        }
        tc::tmem_ld16(tl + 384, v);
        if (warp < 2) {
            float* gw = c.w_grad + 4 * 4096 + in;
#pragma unroll
            for (int o = 0; o < 16; ++o)
                if (v[o] != 0.0f) atomicAdd(gw + o * 64, v[o]);
        }
    }
    if (!ok) tc::mbar_wait(mbar, phase ^ 1u);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tm, kTmemTrain);
    }
}

// --------------------------------------------------------------------------------------------
// Adam
// --------------------------------------------------------------------------------------------
// Starts an optimiser step if the batch had samples: t += 1, bias corrections 1 - beta^t.
__global__ void k_rc_adam_prep(AdamDev a, TrainBatchDev b, float* scalars) {
    uint32_t n0 = 0;
    const uint32_t avail = batch_avail(b, n0);
    uint32_t* step = reinterpret_cast<uint32_t*>(scalars + kRcStep);
    if (avail == 0 || b.batch == 0) {
        scalars[kRcBias] = 0.0f;  // no step: the update kernels do nothing
        return;
    }
    const uint32_t t = *step + 1;
    *step = t;
    scalars[kRcBias] = static_cast<float>(1.0 - pow(static_cast<double>(a.beta1), static_cast<double>(t)));
    scalars[kRcBias + 1] = static_cast<float>(1.0 - pow(static_cast<double>(a.beta2), static_cast<double>(t)));
    scalars[kRcLastLoss] = scalars[kRcLoss];
    scalars[kRcLoss] = 0.0f;
}

__device__ __forceinline__ float adam_update(float p, float& m, float& v, float g, const AdamDev& a, float c1, float c2) {
    m = fa(fm(a.beta1, m), fm(fs(1.0f, a.beta1), g));
    v = fa(fm(a.beta2, v), fm(fm(fs(1.0f, a.beta2), g), g));
    const float mh = fd(m, c1), vh = fd(v, c2);
    return fs(p, fd(fm(a.lr, mh), fa(__fsqrt_rn(vh), a.eps)));
}

// Dense Adam over the MLP weights (FP32 master, BF16 working copy); clears the gradients.
__global__ void k_rc_adam_mlp(AdamDev a, float* master, float* m, float* v, float* grad, __nv_bfloat16* w,
                              const float* scalars) {
    const float c1 = scalars[kRcBias], c2 = scalars[kRcBias + 1];
    if (c1 == 0.0f) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < kRcWeights; i += gridDim.x * blockDim.x) {
        const float g = grad[i];
        grad[i] = 0.0f;
        float mi = m[i], vi = v[i];
        const float p = adam_update(master[i], mi, vi, g, a, c1, c2);
        m[i] = mi;
        v[i] = vi;
        master[i] = p;
        w[i] = __float2bfloat16_rn(p);
    }
}

// Adam over the hash-grid entries that received a gradient (entries with a zero gradient keep
// their parameters and moments); clears the gradients it consumed. The scan reads the dense
// gradient array; a touched entry's master copy and moments are one 32-byte sector
// (interleaved state), so an update reads and writes one sector of state plus its FP16 copy.
__device__ __forceinline__ void adam_entry(const AdamDev& a, float4* state, __half2* h, uint32_t i, float2 g,
                                           float c1, float c2) {
    float4* st = state + 2 * static_cast<size_t>(i);
    float4 pm = st[0];  // master.xy, m.xy
    const float4 vv = st[1];
    float vx = vv.x, vy = vv.y;
    pm.x = adam_update(pm.x, pm.z, vx, g.x, a, c1, c2);
    pm.y = adam_update(pm.y, pm.w, vy, g.y, a, c1, c2);
    st[0] = pm;
    st[1] = make_float4(vx, vy, 0.0f, 0.0f);
    h[i] = __floats2half2_rn(pm.x, pm.y);
}

__global__ void k_rc_adam_grid(AdamDev a, float4* state, float2* grad, __half2* h, uint32_t count, const float* scalars) {
    const float c1 = scalars[kRcBias], c2 = scalars[kRcBias + 1];
    if (c1 == 0.0f) return;
    // Four entries per thread and pass, their gradients loaded together (two 16-byte loads), so
    // that the scan of the (mostly untouched) gradient array keeps several loads in flight.
    const uint32_t quads = count / 4;
    const float4* g4 = reinterpret_cast<const float4*>(grad);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < quads; q += gridDim.x * blockDim.x) {
        const float4 ga = g4[2 * q], gb = g4[2 * q + 1];
        const float2 gs[4] = {make_float2(ga.x, ga.y), make_float2(ga.z, ga.w), make_float2(gb.x, gb.y),
                              make_float2(gb.z, gb.w)};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float2 g = gs[e];
            if (g.x == 0.0f && g.y == 0.0f) continue;
            const uint32_t i = 4 * q + e;
            grad[i] = make_float2(0.0f, 0.0f);
            adam_entry(a, state, h, i, g, c1, c2);
        }
    }
    // entries past the last full group of four
    for (uint32_t i = 4 * quads + blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float2 g = grad[i];
        if (g.x == 0.0f && g.y == 0.0f) continue;
        grad[i] = make_float2(0.0f, 0.0f);
        adam_entry(a, state, h, i, g, c1, c2);
    }
}

// --------------------------------------------------------------------------------------------
// Initialisation and unit kernels
// --------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t mix32(uint32_t x) {  // integer finaliser (splitmix-style)
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return x;
}

// Sets the FP32 master copy of entry i (the first two floats of its Adam state) to its FP16 value.
__device__ __forceinline__ void set_master(float4* state, uint32_t i, __half2 q) {
    const float2 f = __half22float2(q);
    float4 s = state[2 * static_cast<size_t>(i)];
    s.x = f.x;
    s.y = f.y;
    state[2 * static_cast<size_t>(i)] = s;
}

__global__ void k_rc_init_grid(float4* state, __half2* h, uint32_t count, uint32_t seed) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t a = mix32(2 * i + 1 + seed * 0x9E3779B9u), b = mix32(2 * i + 2 + seed * 0x9E3779B9u);
        const float x = (static_cast<float>(a >> 8) * (1.0f / 16777216.0f) * 2.0f - 1.0f) * 1e-4f;
        const float y = (static_cast<float>(b >> 8) * (1.0f / 16777216.0f) * 2.0f - 1.0f) * 1e-4f;
        const __half2 q = __floats2half2_rn(x, y);
        h[i] = q;
        set_master(state, i, q);
    }
}

// Master copies of caller-given FP16 parameters.
__global__ void k_rc_master_from_h(float4* state, const __half2* h, uint32_t count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        set_master(state, i, h[i]);
}

__global__ void k_rc_encode(CacheDev c, const float4* records, uint32_t n, float* out) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        float in[64];
        encode(c, records + 4 * static_cast<size_t>(j), in);
        for (int k = 0; k < 64; ++k) out[64 * static_cast<size_t>(j) + k] = in[k];
    }
}

// Training targets of the vertices gathered in this wave: radiance past the vertex divided
// by the throughput that reached it, per channel; channels with no throughput are masked.
__global__ void k_rc_finalize(const float4* t_aux, float4* t_target, const float4* path_rad, const uint32_t* counters,
                              int base_word, int count_word, uint32_t cap) {
    const uint32_t lo = min(counters[base_word], cap), hi = min(counters[count_word], cap);
    for (uint32_t j = lo + blockIdx.x * blockDim.x + threadIdx.x; j < hi; j += gridDim.x * blockDim.x) {
        const float4 a = t_aux[2 * static_cast<size_t>(j)], rb = t_aux[2 * static_cast<size_t>(j) + 1];
        const float4 L = path_rad[__float_as_uint(a.w)];
        const float T[3] = {a.x, a.y, a.z}, d[3] = {fs(L.x, rb.x), fs(L.y, rb.y), fs(L.z, rb.z)};
        float t[3];
        uint32_t mask = 0;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            if (T[ch] > 1e-8f) {
                t[ch] = fmaxf(fd(d[ch], T[ch]), 0.0f);
                mask |= 1u << ch;
            } else {
                t[ch] = 0.0f;
            }
        }
        t_target[j] = make_float4(t[0], t[1], t[2], __uint_as_float(mask));
    }
}

// --------------------------------------------------------------------------------------------
// Host helpers
// --------------------------------------------------------------------------------------------
uint16_t f32_to_bf16(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x7FFFFFu)) return static_cast<uint16_t>((u >> 16) | 0x40u);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return static_cast<uint16_t>(u >> 16);
}
float bf16_to_f32(uint16_t h) {
    const uint32_t u = static_cast<uint32_t>(h) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

template <typename T>
T* as(void* p) {
    return static_cast<T*>(p);
}

void free_dev(void*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

cudaError_t alloc_dev(void*& p, size_t bytes) {
    free_dev(p);
    return cudaMalloc(&p, bytes);
}

int g_attr_done = -1;

cudaError_t set_kernel_attributes(int device) {
    if (g_attr_done == device) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_rc_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemTrain);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_rc_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemInfer);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_rc_infer8, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemInfer);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_rc_infer_groups<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem_infer_groups(2));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_rc_infer_groups<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem_infer_groups(4));
    if (e == cudaSuccess) g_attr_done = device;
    return e;
}

AdamDev adam_dev(CacheState& cs) {
    AdamDev a;
    a.lr = cs.cfg.learning_rate;
    a.beta1 = cs.cfg.beta1;
    a.beta2 = cs.cfg.beta2;
    a.eps = cs.cfg.epsilon;
    a.step = as<uint32_t>(cs.scalars) + kRcStep;
    a.bias = as<float>(cs.scalars) + kRcBias;
    return a;
}

size_t grid_entries(const CacheState& cs) { return size_t(kRcLevels) * cs.table; }

}  // namespace

// --------------------------------------------------------------------------------------------
// Host side
// --------------------------------------------------------------------------------------------
// The cache's parameters and optimiser state.
static void free_cache_params(CacheState& cs) {
    free_dev(cs.grid_h);
    free_dev(cs.grid_state);
    free_dev(cs.grid_grad);
    free_dev(cs.w_bf16);
    free_dev(cs.w_master);
    free_dev(cs.scalars);
    cs.ready = false;
}

void cache_destroy(rbr_ctx* ctx) {
    CacheState& cs = ctx->cache;
    free_cache_params(cs);
    free_dev(cs.q_rec);  // render buffers (queries, training vertices)
    free_dev(cs.q_sort);
    free_dev(cs.q_info);
    free_dev(cs.t_rec);
    free_dev(cs.t_aux);
    free_dev(cs.t_target);
    cs.q_cap = cs.t_cap = 0;
}

void cache_config_default(rbr_cache_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->log2_table_size = 19;
    c->min_resolution = 16;
    c->max_resolution = 2048;
    c->learning_rate = 1e-2f;
    c->beta1 = 0.9f;
    c->beta2 = 0.99f;
    c->epsilon = 1e-15f;
    c->train_batch = 16384;
    c->train_steps = 4;
    c->train_paths = 65536;
    c->termination_depth = 1;
    c->train_suffix = 2;
    c->seed = 0;
    for (int a = 0; a < 3; ++a) {
        c->bounds_min[a] = 0.0f;
        c->bounds_max[a] = 0.0f;
    }
}

static rbr_status reset_params(rbr_ctx* ctx, const uint16_t* mlp_bf16, const uint16_t* grid_f16) {
    CacheState& cs = ctx->cache;
    const size_t ng = grid_entries(cs);
    std::vector<float> master(kRcWeights);
    std::vector<uint16_t> w16(kRcWeights);
    if (mlp_bf16) {
        for (int i = 0; i < kRcWeights; ++i) {
            w16[i] = mlp_bf16[i];
            master[i] = bf16_to_f32(mlp_bf16[i]);
        }
    } else {
        // Xavier-uniform; W4 rows 3..15 (padding outputs) stay zero
        uint64_t s = cs.cfg.seed * 0x2545F4914F6CDD1Dull + 1;
        for (int l = 0; l < 5; ++l) {
            const int rows = l < 4 ? 64 : 16, real_rows = l < 4 ? 64 : 3;
            const float lim = static_cast<float>(std::sqrt(6.0 / (64.0 + real_rows)));
            for (int r = 0; r < rows; ++r)
                for (int col = 0; col < 64; ++col) {
                    const double u = static_cast<double>(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
                    const float x = r < real_rows ? static_cast<float>((2.0 * u - 1.0) * lim) : 0.0f;
                    const int i = l * 4096 + r * 64 + col;
                    w16[i] = f32_to_bf16(x);
                    master[i] = bf16_to_f32(w16[i]);
                }
        }
    }
    cudaError_t e = cudaMemcpy(cs.w_bf16, w16.data(), kRcWeights * 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(cs.w_master, master.data(), kRcWeights * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(as<float>(cs.w_master) + kRcWeights, 0, size_t(kRcWeights) * 12);  // m, v, grad
    if (e == cudaSuccess) e = cudaMemset(cs.grid_state, 0, ng * 32);  // master (set below), m, v
    if (e == cudaSuccess) e = cudaMemset(cs.grid_grad, 0, ng * 8);
    if (e == cudaSuccess) e = cudaMemset(cs.scalars, 0, kRcScalarWords * 4);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: setting parameters");
    if (grid_f16 || mlp_bf16) {
        // caller-given grid, or the grid left as it is: the master copy restarts from the FP16 values
        if (grid_f16) e = cudaMemcpy(cs.grid_h, grid_f16, ng * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            k_rc_master_from_h<<<ctx->num_sms * 8, 256>>>(as<float4>(cs.grid_state), as<__half2>(cs.grid_h),
                                                          static_cast<uint32_t>(ng));
            e = cudaGetLastError();
        }
    } else {
        k_rc_init_grid<<<ctx->num_sms * 8, 256>>>(as<float4>(cs.grid_state), as<__half2>(cs.grid_h),
                                                  static_cast<uint32_t>(ng), static_cast<uint32_t>(cs.cfg.seed));
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: setting parameters");
    cs.last_loss = 0.0f;
    return RBR_OK;
}

rbr_status cache_create(rbr_ctx* ctx, const rbr_cache_config* cfg_in) {
    rbr_cache_config cfg;
    if (cfg_in) cfg = *cfg_in;
    else cache_config_default(&cfg);
    if (cfg.log2_table_size < 10 || cfg.log2_table_size > 24)
        return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "radiance cache: log2_table_size must lie in [10, 24]");
    if (cfg.min_resolution < 2 || cfg.max_resolution < cfg.min_resolution || cfg.max_resolution > (1 << 20))
        return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "radiance cache: resolutions must satisfy 2 <= min <= max <= 2^20");
    if (!(cfg.learning_rate > 0.0f) || !(cfg.beta1 >= 0.0f && cfg.beta1 < 1.0f) || !(cfg.beta2 >= 0.0f && cfg.beta2 < 1.0f) ||
        !(cfg.epsilon >= 0.0f))
        return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "radiance cache: Adam parameters out of range");
    float lo[3], hi[3];
    bool given = true;
    for (int a = 0; a < 3; ++a) given = given && cfg.bounds_min[a] < cfg.bounds_max[a];
    if (given) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = cfg.bounds_min[a];
            hi[a] = cfg.bounds_max[a];
        }
    } else {
        if (!ctx->has_scene)
            return fail(ctx, RBR_ERR_NO_SCENE, "radiance cache: no bounds given and no scene uploaded");
        for (int a = 0; a < 3; ++a) {
            const float l = ctx->bounds_lo[a], h = ctx->bounds_hi[a];
            if (!(std::isfinite(l) && std::isfinite(h) && l <= h && h - l < 1e30f))
                return fail(ctx, RBR_ERR_INVALID_ARGUMENT,
                            "radiance cache: the scene's bounded geometry has no finite box; give bounds in the config");
            const float pad = std::max(0.01f * (h - l), 1e-3f);
            lo[a] = l - pad;
            hi[a] = h + pad;
        }
    }
    const DeviceScope scope(ctx->device);
    cudaError_t e = scope.status();
    if (e == cudaSuccess) e = set_kernel_attributes(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: device setup");
    // a new cache replaces the parameters; the render buffers stay (they only grow)
    free_cache_params(ctx->cache);
    CacheState& cs = ctx->cache;
    cs.cfg = cfg;
    cs.table = 1u << cfg.log2_table_size;
    for (int a = 0; a < 3; ++a) {
        cs.cfg.bounds_min[a] = lo[a];
        cs.cfg.bounds_max[a] = hi[a];
        cs.dev.lo[a] = lo[a];
        cs.dev.inv_ext[a] = 1.0f / (hi[a] - lo[a]);
    }
    cs.dev.log2_table = static_cast<uint32_t>(cfg.log2_table_size);
    cs.dev.dense_mask = 0;
    const double ratio = std::log2(static_cast<double>(cfg.max_resolution) / cfg.min_resolution);
    for (int l = 0; l < kRcLevels; ++l) {
        const double r = std::floor(cfg.min_resolution * std::exp2(l * ratio / (kRcLevels - 1)));
        cs.dev.res[l] = static_cast<uint32_t>(r);
        const uint64_t n1 = cs.dev.res[l] + 1ull;
        if (n1 * n1 * n1 <= cs.table) cs.dev.dense_mask |= 1u << l;
    }
    const size_t ng = grid_entries(cs);
    if ((e = alloc_dev(cs.grid_h, ng * 4)) != cudaSuccess || (e = alloc_dev(cs.grid_state, ng * 32)) != cudaSuccess ||
        (e = alloc_dev(cs.grid_grad, ng * 8)) != cudaSuccess || (e = alloc_dev(cs.w_bf16, kRcWeights * 2)) != cudaSuccess ||
        (e = alloc_dev(cs.w_master, size_t(kRcWeights) * 16)) != cudaSuccess ||
        (e = alloc_dev(cs.scalars, kRcScalarWords * 4)) != cudaSuccess) {
        cudaGetLastError();
        cache_destroy(ctx);
        return fail(ctx, RBR_ERR_OUT_OF_MEMORY, std::string("radiance cache: cudaMalloc: ") + cudaGetErrorString(e));
    }
    cs.dev.grid = as<__half2>(cs.grid_h);
    cs.dev.grid_grad = as<float2>(cs.grid_grad);
    cs.dev.w = as<__nv_bfloat16>(cs.w_bf16);
    cs.dev.w_grad = as<float>(cs.w_master) + 3 * kRcWeights;
    const rbr_status st = reset_params(ctx, nullptr, nullptr);
    if (st != RBR_OK) {
        cache_destroy(ctx);
        return st;
    }
    cs.ready = true;
    return RBR_OK;
}

rbr_status cache_info(rbr_ctx* ctx, rbr_cache_info* out) {
    CacheState& cs = ctx->cache;
    if (!cs.ready) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "no radiance cache: call rbr_cache_create first");
    std::memset(out, 0, sizeof(*out));
    out->levels = kRcLevels;
    out->table_size = cs.table;
    for (int l = 0; l < kRcLevels; ++l) out->resolution[l] = cs.dev.res[l];
    out->dense_levels = cs.dev.dense_mask;
    uint32_t sc[kRcScalarWords];
    cudaError_t e = cudaMemcpy(sc, cs.scalars, sizeof(sc), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: reading its counters");
    out->optimiser_steps = sc[kRcStep];
    float ll;
    std::memcpy(&ll, &sc[kRcLastLoss], 4);
    out->last_loss = ll;
    out->last_queries = sc[kRcLastQueries];
    out->last_train_records = std::min(sc[kRcTrain], cs.t_cap);
    for (int a = 0; a < 3; ++a) {
        out->bounds_min[a] = cs.cfg.bounds_min[a];
        out->bounds_max[a] = cs.cfg.bounds_max[a];
    }
    return RBR_OK;
}

rbr_status cache_set_params(rbr_ctx* ctx, const uint16_t* mlp, const uint16_t* grid) {
    CacheState& cs = ctx->cache;
    if (!cs.ready) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "no radiance cache: call rbr_cache_create first");
    std::vector<uint16_t> keep;
    if (!mlp) {  // keep the current MLP
        keep.resize(kRcWeights);
        cudaError_t e = cudaMemcpy(keep.data(), cs.w_bf16, kRcWeights * 2, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: reading the MLP");
        mlp = keep.data();
    }
    return reset_params(ctx, mlp, grid);
}

rbr_status cache_get_params(rbr_ctx* ctx, uint16_t* mlp, uint16_t* grid) {
    CacheState& cs = ctx->cache;
    if (!cs.ready) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "no radiance cache: call rbr_cache_create first");
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && mlp) e = cudaMemcpy(mlp, cs.w_bf16, kRcWeights * 2, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && grid) e = cudaMemcpy(grid, cs.grid_h, grid_entries(cs) * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: reading parameters");
    return RBR_OK;
}

rbr_status cache_grads(rbr_ctx* ctx, float* mlp, float* grid) {
    CacheState& cs = ctx->cache;
    if (!cs.ready) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "no radiance cache: call rbr_cache_create first");
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && mlp) e = cudaMemcpy(mlp, cs.dev.w_grad, kRcWeights * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && grid) e = cudaMemcpy(grid, cs.grid_grad, grid_entries(cs) * 8, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: reading gradients");
    return RBR_OK;
}

static rbr_status stage_records(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, const float* targets) {
    const size_t rb = size_t(n) * 64, tb = targets ? size_t(n) * 16 : 0;
    rbr_status st = ensure(ctx, ctx->stage_in, rb + tb, "cache staging");
    if (st != RBR_OK) return st;
    cudaError_t e = cudaMemcpy(ctx->stage_in.ptr, records, rb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && targets) {
        std::vector<float> t4(size_t(n) * 4);
        const uint32_t all = 7u;
        for (uint32_t i = 0; i < n; ++i) {
            t4[4 * i] = targets[3 * i];
            t4[4 * i + 1] = targets[3 * i + 1];
            t4[4 * i + 2] = targets[3 * i + 2];
            std::memcpy(&t4[4 * i + 3], &all, 4);
        }
        e = cudaMemcpy(static_cast<char*>(ctx->stage_in.ptr) + rb, t4.data(), tb, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: copying records");
    return RBR_OK;
}

rbr_status cache_encode_host(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, float* inputs) {
    CacheState& cs = ctx->cache;
    if (!cs.ready) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "no radiance cache: call rbr_cache_create first");
    if (n == 0) return RBR_OK;
    if (!records || !inputs) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "records or inputs is NULL");
    rbr_status st = stage_records(ctx, n, records, nullptr);
    if (st == RBR_OK) st = ensure(ctx, ctx->stage_out, size_t(n) * 256, "cache staging");
    if (st != RBR_OK) return st;
    k_rc_encode<<<std::min<uint32_t>((n + 127) / 128, ctx->num_sms * 8), 128>>>(cs.dev, as<float4>(ctx->stage_in.ptr), n,
                                                                              as<float>(ctx->stage_out.ptr));
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(inputs, ctx->stage_out.ptr, size_t(n) * 256, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: encode");
    return RBR_OK;
}

// Spatial order of the queries (cache.sort_queries): key = Morton code of the query's cell on
// a 32^3 grid over the cache's box (15 bits, 32 chunks of 1,024 keys, the counting sort of
// rbr_sort.cuh); inference then serves the queries cell by cell, so that the samples of a tile
// read nearby hash-grid entries. Scratch: counts and chunk totals, permutation, keys.
constexpr uint32_t kQueryKeys = 1u << 15;
constexpr uint32_t kQueryChunks = kQueryKeys / kScanThreads;

static constexpr size_t round256(size_t b) { return (b + 255) & ~size_t(255); }
size_t query_sort_bytes(uint32_t n) {
    return round256((kQueryKeys + kQueryChunks) * 4) + round256(size_t(n) * 4) + round256(size_t(n) * 2);
}

namespace {
__device__ __forceinline__ uint32_t spread5(uint32_t x) {  // 5 bits -> every third of 15
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < 5; ++i) r |= ((x >> i) & 1u) << (3 * i);
    return r;
}

__global__ void k_rc_query_keys(CacheDev c, const float4* __restrict__ records, uint32_t n, const uint32_t* n_ptr,
                                uint16_t* __restrict__ keys, uint32_t* __restrict__ counts) {
    const uint32_t count = n_ptr ? min(*n_ptr, n) : n;
    for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        uint32_t k = kNoKey;
        if (i < count) {
            float p[3];
            unit_position(c, __ldg(records + 4 * static_cast<size_t>(i)), p);
            k = 0;
#pragma unroll
            for (int a = 0; a < 3; ++a) k |= spread5(min(static_cast<uint32_t>(p[a] * 32.0f), 31u)) << (2 - a);
            keys[i] = static_cast<uint16_t>(k);
        }
        count_key(counts, k);
    }
}

__global__ void k_rc_query_scatter(const uint16_t* __restrict__ keys, uint32_t n, const uint32_t* n_ptr,
                                   uint32_t* __restrict__ offsets, const uint32_t* __restrict__ chunk_sum,
                                   uint32_t* __restrict__ perm) {
    scatter_keys<kQueryChunks>(keys, n_ptr ? min(*n_ptr, n) : n, offsets, chunk_sum, perm);
}
}  // namespace

cudaError_t cache_launch_infer(rbr_ctx* ctx, const float4* records, uint32_t n, const uint32_t* n_ptr, float* rgb,
                               float4* path_rad, const float4* q_info, cudaStream_t stream, void* sort_scratch) {
    CacheState& cs = ctx->cache;
    InferOut o;
    o.rgb = rgb;
    o.path_rad = path_rad;
    o.q_info = q_info;
    o.perm = nullptr;
    const uint32_t tiles = (n + kRcTile - 1) / kRcTile;
    CacheDev dev = cs.dev;
    dev.wait_limit = ctx->cache_wait_limit;
    if (ctx->cache_sort_queries && sort_scratch && n > 0) {
        char* base = static_cast<char*>(sort_scratch);
        auto* counts = reinterpret_cast<uint32_t*>(base);
        uint32_t* chunk_sum = counts + kQueryKeys;
        auto* perm = reinterpret_cast<uint32_t*>(base + round256((kQueryKeys + kQueryChunks) * 4));
        auto* keys = reinterpret_cast<uint16_t*>(base + round256((kQueryKeys + kQueryChunks) * 4) + round256(size_t(n) * 4));
        cudaError_t e = cudaMemsetAsync(counts, 0, kQueryKeys * 4, stream);
        if (e != cudaSuccess) return e;
        const uint32_t sgrid = std::max(1u, std::min<uint32_t>((n + 255) / 256, ctx->num_sms * 8));
        k_rc_query_keys<<<sgrid, 256, 0, stream>>>(dev, records, n, n_ptr, keys, counts);
        k_key_offsets<<<kQueryChunks, kScanThreads, 0, stream>>>(counts, chunk_sum);
        k_rc_query_scatter<<<sgrid, 256, 0, stream>>>(keys, n, n_ptr, counts, chunk_sum, perm);
        o.perm = perm;
    }
    const int G = ctx->cache_infer_groups;
    if (G == 2 || G == 4) {  // G tiles per CTA, 8 / G CTAs per SM
        const uint32_t ctas = (tiles + G - 1) / G;
        const uint32_t grid = std::max(1u, std::min<uint32_t>(ctas, ctx->num_sms * (8 / G)));
        if (G == 2) k_rc_infer_groups<2><<<grid, 256, smem_infer_groups(2), stream>>>(dev, records, n, n_ptr, o, ctx->d_error);
        else k_rc_infer_groups<4><<<grid, 512, smem_infer_groups(4), stream>>>(dev, records, n, n_ptr, o, ctx->d_error);
        return cudaGetLastError();
    }
    const uint32_t grid = std::max(1u, std::min<uint32_t>(tiles, ctx->num_sms * 4));
    if (ctx->cache_infer_warps == 8) k_rc_infer8<<<grid, 256, kSmemInfer, stream>>>(dev, records, n, n_ptr, o, ctx->d_error);
    else k_rc_infer<<<grid, 128, kSmemInfer, stream>>>(dev, records, n, n_ptr, o, ctx->d_error);
    return cudaGetLastError();
}

rbr_status cache_infer_host(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, float* rgb) {
    CacheState& cs = ctx->cache;
    if (!cs.ready) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "no radiance cache: call rbr_cache_create first");
    if (n == 0) return RBR_OK;
    if (!records || !rgb) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "records or rgb is NULL");
    rbr_status st = stage_records(ctx, n, records, nullptr);
    if (st == RBR_OK) st = ensure(ctx, ctx->stage_out, size_t(n) * 12, "cache staging");
    if (st != RBR_OK) return st;
    if ((st = ensure(ctx, ctx->sort_buf, query_sort_bytes(n), "query sort")) != RBR_OK) return st;
    cudaError_t e = cache_launch_infer(ctx, as<float4>(ctx->stage_in.ptr), n, nullptr, as<float>(ctx->stage_out.ptr),
                                       nullptr, nullptr, 0, ctx->sort_buf.ptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: inference");
    st = check_device_error(ctx, 0);
    if (st != RBR_OK) return st;
    e = cudaMemcpy(rgb, ctx->stage_out.ptr, size_t(n) * 12, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: inference");
    return RBR_OK;
}

// One optimiser step (training kernel, then Adam) on `b`.
cudaError_t cache_launch_step(rbr_ctx* ctx, const TrainBatchDev& b, bool apply, cudaStream_t stream) {
    CacheState& cs = ctx->cache;
    const uint32_t tiles = (b.batch + kRcTile - 1) / kRcTile;
    const uint32_t grid = std::max(1u, std::min<uint32_t>(tiles, ctx->num_sms));
    CacheDev dev = cs.dev;
    dev.wait_limit = ctx->cache_wait_limit;
    k_rc_train<<<grid, 128, kSmemTrain, stream>>>(dev, b, as<float>(cs.scalars), ctx->d_error);
    if (!apply) return cudaGetLastError();
    const AdamDev a = adam_dev(cs);
    k_rc_adam_prep<<<1, 1, 0, stream>>>(a, b, as<float>(cs.scalars));
    float* wm = as<float>(cs.w_master);
    k_rc_adam_mlp<<<(kRcWeights + 255) / 256, 256, 0, stream>>>(a, wm, wm + kRcWeights, wm + 2 * kRcWeights,
                                                                 wm + 3 * kRcWeights, as<__nv_bfloat16>(cs.w_bf16),
                                                                 as<float>(cs.scalars));
    k_rc_adam_grid<<<ctx->num_sms * 8, 256, 0, stream>>>(a, as<float4>(cs.grid_state), as<float2>(cs.grid_grad),
                                                        as<__half2>(cs.grid_h), static_cast<uint32_t>(grid_entries(cs)),
                                                        as<float>(cs.scalars));
    return cudaGetLastError();
}

rbr_status cache_train_host(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, const float* targets, int apply,
                            float* loss) {
    CacheState& cs = ctx->cache;
    if (!cs.ready) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "no radiance cache: call rbr_cache_create first");
    if (!records || !targets) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "records or targets is NULL");
    if (n == 0) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "empty training batch");
    rbr_status st = stage_records(ctx, n, records, targets);
    if (st != RBR_OK) return st;
    cudaError_t e = cudaSuccess;
    if (!apply) {  // gradients of this batch alone
        e = cudaMemset(cs.dev.w_grad, 0, kRcWeights * 4);
        if (e == cudaSuccess) e = cudaMemset(cs.grid_grad, 0, grid_entries(cs) * 8);
    }
    if (e == cudaSuccess) e = cudaMemset(as<float>(cs.scalars) + kRcLoss, 0, 4);
    TrainBatchDev b;
    b.records = as<float4>(ctx->stage_in.ptr);
    b.targets = reinterpret_cast<const float4*>(static_cast<char*>(ctx->stage_in.ptr) + size_t(n) * 64);
    b.count_ptr = nullptr;
    b.count = n;
    b.cap = n;
    b.batch = n;
    b.step_index = 0;
    b.shuffle = 0;
    if (e == cudaSuccess) e = cache_launch_step(ctx, b, apply != 0, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: training step");
    st = check_device_error(ctx, 0);
    if (st != RBR_OK) return st;
    float sc[kRcScalarWords];
    e = cudaMemcpy(sc, cs.scalars, sizeof(sc), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "radiance cache: reading the loss");
    if (loss) *loss = apply ? sc[kRcLastLoss] : sc[kRcLoss];
    return RBR_OK;
}

// Buffers for one wave of `paths` paths with queries and training vertices.
rbr_status cache_ensure_render(rbr_ctx* ctx, uint32_t paths, uint32_t train_cap) {
    CacheState& cs = ctx->cache;
    cudaError_t e = cudaSuccess;
    if (cs.q_cap < paths) {
        free_dev(cs.q_rec);
        free_dev(cs.q_info);
        free_dev(cs.q_sort);
        cs.q_cap = 0;
        cs.q_sort_stride = query_sort_bytes(paths);
        if ((e = alloc_dev(cs.q_rec, size_t(paths) * 64)) == cudaSuccess &&
            (e = alloc_dev(cs.q_info, size_t(paths) * 16)) == cudaSuccess &&
            (e = alloc_dev(cs.q_sort, 2 * cs.q_sort_stride)) == cudaSuccess)
            cs.q_cap = paths;
    }
    if (e == cudaSuccess && cs.t_cap < train_cap) {
        free_dev(cs.t_rec);
        free_dev(cs.t_aux);
        free_dev(cs.t_target);
        cs.t_cap = 0;
        if ((e = alloc_dev(cs.t_rec, size_t(train_cap) * 64)) == cudaSuccess &&
            (e = alloc_dev(cs.t_aux, size_t(train_cap) * 32)) == cudaSuccess &&
            (e = alloc_dev(cs.t_target, size_t(train_cap) * 16)) == cudaSuccess)
            cs.t_cap = train_cap;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, RBR_ERR_OUT_OF_MEMORY, std::string("radiance cache: render buffers: ") + cudaGetErrorString(e));
    }
    return RBR_OK;
}

cudaError_t cache_launch_finalize(rbr_ctx* ctx, const float4* path_rad, const float4* t_aux, const uint32_t* counters,
                                  int base_word, int count_word, uint32_t cap, cudaStream_t stream) {
    CacheState& cs = ctx->cache;
    // the targets of a list that starts at t_aux (a wave slot's half) start at the same index
    const size_t first = static_cast<size_t>(t_aux - as<float4>(cs.t_aux)) / 2;
    k_rc_finalize<<<ctx->num_sms * 4, 128, 0, stream>>>(t_aux, as<float4>(cs.t_target) + first, path_rad, counters,
                                                       base_word, count_word, cap);
    return cudaGetLastError();
}

// The frame's optimiser steps on the training vertices gathered (count on the device).
cudaError_t cache_launch_train_frame(rbr_ctx* ctx, const uint32_t* count_ptr, const uint32_t* count2_ptr, uint32_t cap,
                                     uint32_t frame, cudaStream_t stream) {
    CacheState& cs = ctx->cache;
    TrainBatchDev b;
    b.records = as<float4>(cs.t_rec);
    b.targets = as<float4>(cs.t_target);
    b.count_ptr = count_ptr;
    b.count2_ptr = count2_ptr;
    b.split = cap;
    b.count = 0;
    b.cap = cap;
    b.batch = cs.cfg.train_batch;
    b.shuffle = 1;
    cudaError_t e = cudaSuccess;
    for (uint32_t s = 0; s < cs.cfg.train_steps && e == cudaSuccess; ++s) {
        b.step_index = frame * cs.cfg.train_steps + s;
        e = cache_launch_step(ctx, b, true, stream);
    }
    return e;
}

}  // namespace rbr
