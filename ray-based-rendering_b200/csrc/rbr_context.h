// Internal definition of rbr_ctx and the host-side helpers shared by the library's files.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "rbr_b200.h"
#include "rbr_cache.h"
#include "rbr_scene_dev.h"
#include "rbr_layout.h"

namespace rbr {

// A device allocation owned by the context.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

// Path-tracer working set (sized for one wave of paths).
struct PathBuffers {
    uint32_t capacity = 0;      // paths per wave
    uint32_t shadow_capacity = 0;
    DevBuf ray;                 // float4 x2 per path: (o, -), (d, -)
    DevBuf thr;                 // float4 per path: throughput rgb, w = specular flag
    DevBuf rad;                 // float4 per path: radiance rgb
    DevBuf hit;                 // uint2 per path
    DevBuf queue[2];            // active path indices (ping-pong)
    DevBuf classq;              // material-class queues: kClasses x capacity
    DevBuf shadow;              // 3 float4 per shadow ray
    DevBuf counters;            // uint32 counters (see pt kernels)
};

}  // namespace rbr

struct rbr_ctx {
    int device = 0;
    int num_sms = 0;
    std::string error;
    cudaStream_t stream = nullptr;  // internal stream for host-buffer calls
    // scene
    bool has_scene = false;
    rbr::DeviceScene scene{};
    std::vector<rbr::DevBuf> scene_bufs;
    const void* bvh_base = nullptr;   // nodes followed by leaf records, one allocation
    size_t bvh_bytes = 0;
    rbr_scene_stats stats{};
    float bounds_lo[3] = {0, 0, 0}, bounds_hi[3] = {0, 0, 0};
    // host-call staging
    rbr::DevBuf stage_in, stage_out;
    // device error word (rbr::kErr*)
    int* d_error = nullptr;
    // work cursors of the persistent trace kernel: one per launch, taken round-robin so that
    // launches overlapping on different streams never share one
    uint32_t* d_cursors = nullptr;
    uint32_t cursor_next = 0;
    // tunables (rbr_param_set / rbr_autotune)
    int trace_kernel = 0;          // 0: one thread per ray, 1: persistent lane refill, 2: warp-cooperative
    int trace_blocks_per_sm = 0;   // persistent grid per SM (0: occupancy limit)
    int trace_min_blocks = 10;     // kernel 0: register budget for 8, 10 or 12 resident blocks per SM
    int trace_order = 0;           // kernel 0: 0 rays in the given order, 1 sorted by direction octant and origin
    int trace_node_test = 0;       // sorted ray queries: 0 packed node test, 1 register-lean one
    int trace_stream_io = 1;       // kernel 0: rays read and hits written with evict-first (streaming) hints
    int trace_l2_persist = 0;      // kernel 0: the BVH's address range marked persisting in L2
    size_t l2_persist_bytes = 0;   // the context's persisting-L2 set-aside while trace_l2_persist is on
    rbr::DevBuf sort_buf;          // keys, permutation and radix-sort scratch of trace_order 1
    rbr::DevBuf sort_buf2;         // the same for the second stream of a chunked rbr_trace_host
    rbr::DevBuf sort_more[2];      // the same for its third and fourth streams
    uint32_t trace_host_chunk = 1u << 19;  // rbr_trace_host: rays per pipelined chunk (0: one piece)
    int trace_host_streams = 4;    // rbr_trace_host: streams the chunks rotate over (2-4)
    int trace_refill_min = 1;      // kernel 1: idle lanes of a warp before it fetches new rays (1-32)
    cudaStream_t host_streams[2] = {nullptr, nullptr};  // rbr_trace_host's third and fourth streams
    cudaEvent_t host_join[2] = {nullptr, nullptr};
    uint32_t pt_wave_paths = 1u << 23;
    int bvh_record_cost_milli = 1000;      // 8-wide collapse: record test cost / node test cost x1000
    uint32_t cache_wait_limit = 1u << 22;  // polls of a tensor-core completion wait (cache kernels)
    int cache_infer_groups = 1;            // tiles in flight per inference CTA: 1, 2 or 4
    int cache_infer_warps = 4;             // warps per tile of the one-tile inference kernel: 4 or 8
    int cache_sort_queries = 0;            // inference serves the queries in spatial order (0 or 1)
    uint32_t fail_alloc_countdown = 0;     // > 0: the n-th next device allocation fails (fault injection)
    // path tracer
    rbr::PathBuffers pt;
    rbr::PathBuffers pt2;                  // second wave in flight (rbr_render, pt_streams 2)
    int pt_streams = 2;                    // waves in flight in rbr_render: 1 or 2
    int pt_shade_split = 0;                // rbr_render: one shading launch per material class
    int pt_fetch = 1;                      // wavefront stages hand out long queues by claims on cursors (0: grid stride)
    bool pt_last_two = false;              // the last rbr_render used pt2
    cudaStream_t side_stream = nullptr;    // stream of the second wave
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    rbr::DevBuf pt_seg_of;  // packed waves: segment of each path
    rbr::DevBuf pt_seg_of2;  // the same for the second wave in flight (pt2)
    uint32_t pt_generation = 0;  // incremented whenever a path buffer set or segment index is reallocated
    rbr_render_stats last_render{};
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    bool render_pending = false;
    // radiance cache
    rbr::CacheState cache;
};

namespace rbr {

// Makes `device` current for the lifetime of the scope and gives the calling thread its
// previous current device back at exit: an entry point never changes the caller's device.
class DeviceScope {
  public:
    explicit DeviceScope(int device) : device_(device) {
        if (cudaGetDevice(&prev_) != cudaSuccess) {
            cudaGetLastError();
            prev_ = -1;
        }
        if (prev_ != device_) status_ = cudaSetDevice(device_);
    }
    ~DeviceScope() {
        if (prev_ >= 0 && prev_ != device_) cudaSetDevice(prev_);
    }
    DeviceScope(const DeviceScope&) = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;
    cudaError_t status() const { return status_; }

  private:
    int device_;
    int prev_ = -1;
    cudaError_t status_ = cudaSuccess;
};

rbr_status fail(rbr_ctx* ctx, rbr_status code, const std::string& msg);
rbr_status cuda_fail(rbr_ctx* ctx, cudaError_t e, const char* what);
rbr_status ensure(rbr_ctx* ctx, DevBuf& b, size_t bytes, const char* what);
void release(DevBuf& b);
rbr_status check_device_error(rbr_ctx* ctx, cudaStream_t stream);

rbr_status upload_scene(rbr_ctx* ctx, const rbr_scene_desc* desc);
rbr_status upload_scene_variant(rbr_ctx* dst, const rbr_ctx* base, const rbr_material* materials, uint32_t num_materials,
                                const rbr_light* lights, uint32_t num_lights, const rbr_medium* medium);
void free_scene(rbr_ctx* ctx);

// kernels (trace.cu)
cudaError_t launch_trace_closest(const DeviceScene& s, const rbr_ray* rays, uint32_t n, rbr_hit* hits, int* err,
                                 int num_sms, cudaStream_t stream);
cudaError_t launch_trace_any(const DeviceScene& s, const rbr_ray* rays, uint32_t n, uint8_t* occ, int* err,
                             int num_sms, cudaStream_t stream);
cudaError_t launch_trace_counts(const DeviceScene& s, const rbr_ray* rays, uint32_t n, int any_hit,
                                unsigned long long* totals, int* err, cudaStream_t stream);
cudaError_t launch_trace_persist(const DeviceScene& s, const rbr_ray* rays, uint32_t n, int any_hit, void* out,
                                 int* err, uint32_t* cursor, int grid, cudaStream_t stream, const uint32_t* perm = nullptr,
                                 uint32_t refill_min = 1);
int trace_persist_blocks_per_sm(int any_hit);
cudaError_t launch_trace_coop(const DeviceScene& s, const rbr_ray* rays, uint32_t n, int any_hit, void* out, int* err,
                              uint32_t* cursor, int grid, cudaStream_t stream);
int trace_coop_blocks_per_sm(int any_hit);
rbr_status autotune_trace(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, int any_hit, int64_t* chosen_us);
constexpr int kCursorRing = 64;
// Launches a ray query with the context's chosen kernel (closest hit into rbr_hit[n] or any
// hit into uint8_t[n]).
// slot 0 or 1: which sort scratch a sorted launch uses (launches in flight on two streams).
cudaError_t launch_trace(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, int any_hit, void* out, cudaStream_t stream,
                         int slot = 0);
// Creates the context's second stream and its fork/join events on first use.
rbr_status ensure_side_stream(rbr_ctx* ctx);

// path tracer (pt.cu)
rbr_status render(rbr_ctx* ctx, const rbr_camera* cam, const rbr_render_params* p, float* film_mean, float* film_m2,
                  cudaStream_t stream);
void free_path_buffers(rbr_ctx* ctx);
rbr_status read_render_counters(rbr_ctx* ctx);
// radiance cache (cache.cu)
void cache_config_default(rbr_cache_config* c);
rbr_status cache_create(rbr_ctx* ctx, const rbr_cache_config* cfg);
void cache_destroy(rbr_ctx* ctx);
rbr_status cache_info(rbr_ctx* ctx, rbr_cache_info* out);
rbr_status cache_set_params(rbr_ctx* ctx, const uint16_t* mlp, const uint16_t* grid);
rbr_status cache_get_params(rbr_ctx* ctx, uint16_t* mlp, uint16_t* grid);
rbr_status cache_grads(rbr_ctx* ctx, float* mlp, float* grid);
rbr_status cache_encode_host(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, float* inputs);
rbr_status cache_infer_host(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, float* rgb);
rbr_status cache_train_host(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, const float* targets, int apply,
                            float* loss);
rbr_status cache_ensure_render(rbr_ctx* ctx, uint32_t paths, uint32_t train_cap);
// sort_scratch (optional, query_sort_bytes(n) bytes): with cache.sort_queries the queries are
// served in spatial order (a counting sort of their cells) instead of the order given.
cudaError_t cache_launch_infer(rbr_ctx* ctx, const float4* records, uint32_t n, const uint32_t* n_ptr, float* rgb,
                               float4* path_rad, const float4* q_info, cudaStream_t stream,
                               void* sort_scratch = nullptr);
size_t query_sort_bytes(uint32_t n);
cudaError_t cache_launch_finalize(rbr_ctx* ctx, const float4* path_rad, const float4* t_aux, const uint32_t* counters,
                                  int base_word, int count_word, uint32_t cap, cudaStream_t stream);
cudaError_t cache_launch_train_frame(rbr_ctx* ctx, const uint32_t* count_ptr, const uint32_t* count2_ptr, uint32_t cap,
                                     uint32_t frame, cudaStream_t stream);
rbr_status render_cached(rbr_ctx* ctx, const rbr_camera* cam, const rbr_render_params* p, uint32_t frames, int train,
                         float* film_mean, float* film_m2, cudaStream_t stream);

// batched request loop (pt.cu, batch.cpp)
CameraDev camera_dev(const rbr_camera* cam);
struct PackedWave {
    int mode = 0;                 // 0 path tracer, 1 path tracer + radiance cache, 2 volumetric
    uint32_t max_depth = 0;       // depth iterations (the largest max depth of its requests)
    int grid = 0;                 // blocks of the wavefront kernels
    const SegDev* segs = nullptr; // device segment table
    const uint32_t* hdr = nullptr;  // device [paths, segments]
    uint32_t capacity = 0;        // path capacity of the wave buffers
    bool train = false;           // mode 1: gather training vertices and train after the wave
    uint32_t train_thresh = 0;
    uint32_t train_steps = 0;
    int slot = 0;                 // path buffers: 0 pt / pt_seg_of, 1 pt2 / pt_seg_of2
};
// Path buffers for packed waves: `slots` (1 or 2) sets of `cap` paths with their segment index.
rbr_status ensure_wave_buffers(rbr_ctx* ctx, uint32_t cap, uint32_t shadow_cap, int slots = 1);
cudaError_t launch_packed_wave(rbr_ctx* eng, rbr_ctx* scn, const PackedWave& pw, cudaStream_t stream);
// One cooperative launch that renders `nwaves` waves (modes 0 and 2) of up to 16 scenes; with
// halves 2 the grid's halves render alternate waves on the context's two path-buffer sets.
// Device-clock stamps: [0] start, [1 + w] end of wave w. bar: kLoopBarrierWords words.
constexpr int kLoopBarrierWords = 6;
cudaError_t launch_wave_loop(rbr_ctx* eng, const std::vector<rbr_ctx*>& scenes, const LoopWave* waves, uint32_t nwaves,
                             const char* tables, unsigned long long* stamps, uint32_t* bar, uint64_t limit_ns,
                             int halves, cudaStream_t stream, int* grid_out);
cudaError_t launch_stamp(unsigned long long* at, cudaStream_t stream);
cudaError_t launch_release(const unsigned long long* start, uint64_t release_ns, cudaStream_t stream);
uint32_t packed_wave_launches(const PackedWave& pw);

rbr_status render_noalloc(rbr_ctx* ctx, const rbr_camera* cam, const rbr_render_params* p, float* film_mean,
                          cudaStream_t stream);

}  // namespace rbr
