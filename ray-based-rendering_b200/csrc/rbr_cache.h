// Radiance cache: device-visible parameter block and the host state a context owns.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "rbr_b200.h"

namespace rbr {

constexpr int kRcLevels = RBR_CACHE_LEVELS;
constexpr int kRcWeights = RBR_CACHE_MLP_WEIGHTS;  // 17408
constexpr uint32_t kRcTile = 128;                   // samples per tensor-core tile (MMA M)

// What the fused kernels read: the hash grid, the MLP and where gradients go.
struct CacheDev {
    const __half2* grid;          // levels x table entries, 2 FP16 features each
    float2* grid_grad;            // same shape, FP32 gradient accumulators
    const __nv_bfloat16* w;       // MLP weights, row-major per matrix (row = output)
    float* w_grad;                // FP32 gradient accumulators, same layout
    uint32_t res[kRcLevels];      // grid resolution per level
    uint32_t dense_mask;          // bit l: level l indexed densely
    uint32_t log2_table;
    float lo[3], inv_ext[3];      // position -> [0,1]^3: (p - lo) * inv_ext, clamped
    uint32_t wait_limit;          // polls of a tensor-core completion wait before it gives up
};

// Adam's per-run constants and device-side step state.
struct AdamDev {
    float lr, beta1, beta2, eps;
    uint32_t* step;               // steps taken (device)
    float* bias;                  // [0] = 1 - beta1^t, [1] = 1 - beta2^t of the current step (device)
};

// A batch of training pairs in device memory. The number of available pairs is `count`, or
// *count_ptr (clamped to cap) when count_ptr is set (counts produced on the device).
struct TrainBatchDev {
    const float4* records;        // 4 float4 per record (rbr_cache_record)
    const float4* targets;        // rgb + channel mask bits (w, as uint32)
    const uint32_t* count_ptr;
    const uint32_t* count2_ptr = nullptr;  // optional second list of *count2_ptr records starting at `split`
    uint32_t split = 0;
    uint32_t count, cap;                   // cap: records per list
    uint32_t batch;               // samples per step; sample j of step s reads pair perm(s*batch + j) % avail
    uint32_t step_index;
    uint32_t shuffle;             // 0: sample j reads pair j
};

struct DevBuf;

// Host-side state of a context's cache.
struct CacheState {
    bool ready = false;
    rbr_cache_config cfg{};
    CacheDev dev{};
    uint32_t table = 0;
    // parameters (device)
    void* grid_h = nullptr;       // __half2 [L*T]
    void* grid_state = nullptr;   // Adam state, 32 B per entry: float4 (master.xy, m.xy), float4 (v.xy, 0, 0)
    void* grid_grad = nullptr;    // float2
    void* w_bf16 = nullptr;       // bf16 [kRcWeights]
    void* w_master = nullptr;     // float [kRcWeights] x4: master, m, v, grad
    void* scalars = nullptr;      // uint32 step, float bias[2], float loss, uint32 counters
    // render-time buffers
    void* q_rec = nullptr;        // float4 x4 per query
    void* q_info = nullptr;       // float4 per query: throughput rgb, path index bits
    void* q_sort = nullptr;       // two query-sort scratch areas (one per wave slot), q_sort_stride apart
    size_t q_sort_stride = 0;
    uint32_t q_cap = 0;
    void* t_rec = nullptr;        // float4 x4 per training vertex
    void* t_aux = nullptr;        // float4 x2 per training vertex: (T, path), (radiance before, -)
    void* t_target = nullptr;     // float4 per training vertex
    uint32_t t_cap = 0;
    // host staging for unit calls
    void* stage = nullptr;
    size_t stage_bytes = 0;
    float last_loss = 0.0f;
    uint32_t last_queries = 0, last_train = 0;
};

// Offsets in CacheState::scalars (32-bit words).
enum : int {
    kRcStep = 0,        // Adam steps taken
    kRcBias = 1,        // 2 floats
    kRcLoss = 3,        // float: loss sum of the current step
    kRcLastLoss = 4,    // float: loss of the last step
    kRcQueries = 5,     // uint32: queries appended in this wave
    kRcTrain = 6,       // uint32: training vertices appended in this frame
    kRcTrainBase = 7,   // uint32: training count at the start of the current wave
    kRcLastQueries = 8, // uint32: queries of the last frame (summed over waves)
    kRcScalarWords = 16
};

}  // namespace rbr
