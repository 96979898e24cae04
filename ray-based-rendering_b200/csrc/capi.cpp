// The C ABI of include/rbr_b200.h.
#include <algorithm>
#include <cstring>
#include <new>
#include <string>

#include "rbr_context.h"

namespace rbr {

rbr_status fail(rbr_ctx* ctx, rbr_status code, const std::string& msg) {
    if (ctx) ctx->error = msg;
    return code;
}

rbr_status cuda_fail(rbr_ctx* ctx, cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(ctx, RBR_ERR_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
    }
    return fail(ctx, RBR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void release(DevBuf& b) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
}

rbr_status ensure(rbr_ctx* ctx, DevBuf& b, size_t bytes, const char* what) {
    if (b.bytes >= bytes && b.ptr) return RBR_OK;
    release(b);
    if (bytes == 0) return RBR_OK;
    if (ctx->fail_alloc_countdown > 0 && --ctx->fail_alloc_countdown == 0)
        return fail(ctx, RBR_ERR_OUT_OF_MEMORY, std::string("cudaMalloc for ") + what + " (" + std::to_string(bytes) +
                                                    " B): failure injected by debug.fail_alloc");
    cudaError_t e = cudaMalloc(&b.ptr, bytes);
    if (e != cudaSuccess) {
        b.ptr = nullptr;
        cudaGetLastError();
        return fail(ctx, RBR_ERR_OUT_OF_MEMORY, std::string("cudaMalloc for ") + what + " (" + std::to_string(bytes) +
                                                    " B): " + cudaGetErrorString(e));
    }
    b.bytes = bytes;
    return RBR_OK;
}

rbr_status ensure_side_stream(rbr_ctx* ctx) {
    cudaError_t e = cudaSuccess;
    if (!ctx->side_stream) e = cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess && !ctx->ev_fork) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess && !ctx->ev_join) e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
    return e == cudaSuccess ? RBR_OK : cuda_fail(ctx, e, "second stream");
}

// Reads (and clears) the device error word after the work on `stream` has finished.
rbr_status check_device_error(rbr_ctx* ctx, cudaStream_t stream) {
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "reading the device error word");
    if (h == 0) return RBR_OK;
    cudaMemsetAsync(ctx->d_error, 0, sizeof(int), stream);
    cudaStreamSynchronize(stream);
    std::string what;
    if (h & kErrStackOverflow) what += " traversal-stack overflow;";
    if (h & kErrQueueOverflow) what += " queue overflow;";
    if (h & kErrDeviceTimeout) {
        what += " a bounded device wait (tensor-core completion or grid barrier) ran out;";
        return fail(ctx, RBR_ERR_DEVICE_TIMEOUT, "device check failed:" + what);
    }
    return fail(ctx, RBR_ERR_INTERNAL, "device check failed:" + what);
}

}  // namespace rbr

using namespace rbr;

extern "C" {

uint32_t rbr_abi_version(void) { return RBR_ABI_VERSION; }

size_t rbr_struct_size(const char* name) {
    if (!name) return 0;
    const std::string n(name);
    if (n == "rbr_material") return sizeof(rbr_material);
    if (n == "rbr_light") return sizeof(rbr_light);
    if (n == "rbr_scene_desc") return sizeof(rbr_scene_desc);
    if (n == "rbr_scene_stats") return sizeof(rbr_scene_stats);
    if (n == "rbr_ray") return sizeof(rbr_ray);
    if (n == "rbr_hit") return sizeof(rbr_hit);
    if (n == "rbr_camera") return sizeof(rbr_camera);
    if (n == "rbr_render_params") return sizeof(rbr_render_params);
    if (n == "rbr_render_stats") return sizeof(rbr_render_stats);
    if (n == "rbr_cache_record") return sizeof(rbr_cache_record);
    if (n == "rbr_cache_config") return sizeof(rbr_cache_config);
    if (n == "rbr_cache_info") return sizeof(rbr_cache_info);
    if (n == "rbr_medium") return sizeof(rbr_medium);
    if (n == "rbr_batch_config") return sizeof(rbr_batch_config);
    if (n == "rbr_request") return sizeof(rbr_request);
    if (n == "rbr_request_stats") return sizeof(rbr_request_stats);
    if (n == "rbr_batch_stats") return sizeof(rbr_batch_stats);
    return 0;
}

rbr_status rbr_ctx_create(int device, rbr_ctx** out) {
    if (!out) return RBR_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return RBR_ERR_CUDA;  // no usable device: there is no CPU fallback
    }
    if (device < 0 || device >= count) return RBR_ERR_INVALID_ARGUMENT;
    rbr_ctx* ctx = new (std::nothrow) rbr_ctx();
    if (!ctx) return RBR_ERR_OUT_OF_MEMORY;
    ctx->device = device;
    const DeviceScope scope(device);
    if ((e = scope.status()) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMalloc(reinterpret_cast<void**>(&ctx->d_error), sizeof(int))) != cudaSuccess ||
        (e = cudaMemset(ctx->d_error, 0, sizeof(int))) != cudaSuccess ||
        (e = cudaMalloc(reinterpret_cast<void**>(&ctx->d_cursors), kCursorRing * sizeof(uint32_t))) != cudaSuccess ||
        (e = cudaEventCreate(&ctx->ev_start)) != cudaSuccess || (e = cudaEventCreate(&ctx->ev_stop)) != cudaSuccess) {
        cudaGetLastError();
        rbr_ctx_destroy(ctx);
        return RBR_ERR_CUDA;
    }
    *out = ctx;
    return RBR_OK;
}

void rbr_ctx_destroy(rbr_ctx* ctx) {
    if (!ctx) return;
    const DeviceScope scope(ctx->device);
    cudaDeviceSynchronize();
    free_scene(ctx);
    free_path_buffers(ctx);
    cache_destroy(ctx);
    release(ctx->stage_in);
    release(ctx->stage_out);
    release(ctx->sort_buf);
    release(ctx->sort_buf2);
    release(ctx->sort_more[0]);
    release(ctx->sort_more[1]);
    if (ctx->d_error) cudaFree(ctx->d_error);
    if (ctx->d_cursors) cudaFree(ctx->d_cursors);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
    if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
    if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
    for (int i = 0; i < 2; ++i) {
        if (ctx->host_streams[i]) cudaStreamDestroy(ctx->host_streams[i]);
        if (ctx->host_join[i]) cudaEventDestroy(ctx->host_join[i]);
    }
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    delete ctx;
}

const char* rbr_last_error(const rbr_ctx* ctx) { return ctx ? ctx->error.c_str() : "no context"; }

rbr_status rbr_scene_upload(rbr_ctx* ctx, const rbr_scene_desc* desc) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    cudaDeviceSynchronize();  // nothing may still read the scene being replaced
    return upload_scene(ctx, desc);
}

rbr_status rbr_param_set(rbr_ctx* ctx, const char* name, int64_t value) {
    if (!ctx || !name) return RBR_ERR_INVALID_ARGUMENT;
    const std::string n(name);
    if (n == "trace.kernel") {
        if (value < 0 || value > 2) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "trace.kernel is 0, 1 or 2");
        ctx->trace_kernel = static_cast<int>(value);
    } else if (n == "trace.blocks_per_sm") {
        if (value < 0 || value > 32) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "trace.blocks_per_sm is 0..32");
        ctx->trace_blocks_per_sm = static_cast<int>(value);
    } else if (n == "trace.order") {
        if (value < 0 || value > 5) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "trace.order is 0..5");
        ctx->trace_order = static_cast<int>(value);
    } else if (n == "trace.min_blocks") {
        if (value != 8 && value != 10 && value != 12) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "trace.min_blocks is 8, 10 or 12");
        ctx->trace_min_blocks = static_cast<int>(value);
    } else if (n == "trace.host_chunk") {
        if (value < 0 || value > 0xFFFFFFFFll) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "trace.host_chunk is 0..2^32-1");
        ctx->trace_host_chunk = static_cast<uint32_t>(value);
    } else if (n == "trace.refill_min") {
        if (value < 1 || value > 32) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "trace.refill_min is 1..32");
        ctx->trace_refill_min = static_cast<int>(value);
    } else if (n == "trace.host_streams") {
        if (value < 2 || value > 4) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "trace.host_streams is 2, 3 or 4");
        ctx->trace_host_streams = static_cast<int>(value);
    } else if (n == "pt.streams") {
        if (value != 1 && value != 2) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "pt.streams is 1 or 2");
        ctx->pt_streams = static_cast<int>(value);
    } else if (n == "pt.wave_paths") {
        if (value < 1024 || value > (int64_t(1) << 26)) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "pt.wave_paths is 1024..2^26");
        ctx->pt_wave_paths = static_cast<uint32_t>(value);
    } else if (n == "trace.node_test") {
        if (value != 0 && value != 1) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "trace.node_test is 0 or 1");
        ctx->trace_node_test = static_cast<int>(value);
    } else if (n == "trace.stream_io") {
        if (value != 0 && value != 1) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "trace.stream_io is 0 or 1");
        ctx->trace_stream_io = static_cast<int>(value);
    } else if (n == "trace.l2_persist") {
        if (value != 0 && value != 1) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "trace.l2_persist is 0 or 1");
        const DeviceScope scope(ctx->device);
        // the set-aside is a limit of this process's context: it ends with the context
        size_t bytes = 0;
        if (value) {
            int max_persist = 0;
            cudaError_t e = cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, ctx->device);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "persisting L2 size");
            bytes = static_cast<size_t>(max_persist);
        }
        cudaError_t e = cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, bytes);
        if (e == cudaSuccess && !value) e = cudaCtxResetPersistingL2Cache();
        if (e != cudaSuccess) return cuda_fail(ctx, e, "persisting L2 set-aside");
        ctx->l2_persist_bytes = bytes;
        ctx->trace_l2_persist = static_cast<int>(value);
    } else if (n == "pt.shade_split") {
        if (value != 0 && value != 1) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "pt.shade_split is 0 or 1");
        ctx->pt_shade_split = static_cast<int>(value);
    } else if (n == "pt.fetch") {
        if (value != 0 && value != 1) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "pt.fetch is 0 or 1");
        if (ctx->pt_fetch != static_cast<int>(value)) ++ctx->pt_generation;  // captured wave graphs hold the old value
        ctx->pt_fetch = static_cast<int>(value);
    } else if (n == "cache.sort_queries") {
        if (value != 0 && value != 1) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "cache.sort_queries is 0 or 1");
        ctx->cache_sort_queries = static_cast<int>(value);
    } else if (n == "cache.infer_warps") {
        if (value != 4 && value != 8) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "cache.infer_warps is 4 or 8");
        ctx->cache_infer_warps = static_cast<int>(value);
    } else if (n == "cache.infer_groups") {
        if (value != 1 && value != 2 && value != 4) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "cache.infer_groups is 1, 2 or 4");
        ctx->cache_infer_groups = static_cast<int>(value);
    } else if (n == "cache.wait_limit") {
        if (value < 0 || value > (int64_t(1) << 22)) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "cache.wait_limit is 0..2^22");
        ctx->cache_wait_limit = static_cast<uint32_t>(value);
    } else if (n == "debug.fail_alloc") {
        if (value < 0 || value > 1000000) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "debug.fail_alloc is 0..1000000");
        ctx->fail_alloc_countdown = static_cast<uint32_t>(value);
    } else if (n == "bvh.record_cost_milli") {
        if (value < 1 || value > 100000) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "bvh.record_cost_milli is 1..100000");
        ctx->bvh_record_cost_milli = static_cast<int>(value);
    } else {
        return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "unknown parameter " + n);
    }
    return RBR_OK;
}

rbr_status rbr_autotune_trace(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, int any_hit, int64_t* out_us) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    if (!ctx->has_scene) return fail(ctx, RBR_ERR_NO_SCENE, "rbr_autotune_trace before rbr_scene_upload");
    if (!rays || n == 0) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "rbr_autotune_trace needs rays");
    const DeviceScope scope(ctx->device);
    return autotune_trace(ctx, rays, n, any_hit, out_us);
}

rbr_status rbr_param_get(const rbr_ctx* ctx, const char* name, int64_t* value) {
    if (!ctx || !name || !value) return RBR_ERR_INVALID_ARGUMENT;
    const std::string n(name);
    if (n == "trace.kernel") *value = ctx->trace_kernel;
    else if (n == "trace.blocks_per_sm") *value = ctx->trace_blocks_per_sm;
    else if (n == "trace.min_blocks") *value = ctx->trace_min_blocks;
    else if (n == "trace.order") *value = ctx->trace_order;
    else if (n == "pt.wave_paths") *value = ctx->pt_wave_paths;
    else if (n == "pt.streams") *value = ctx->pt_streams;
    else if (n == "trace.host_chunk") *value = ctx->trace_host_chunk;
    else if (n == "trace.host_streams") *value = ctx->trace_host_streams;
    else if (n == "trace.refill_min") *value = ctx->trace_refill_min;
    else if (n == "bvh.record_cost_milli") *value = ctx->bvh_record_cost_milli;
    else if (n == "cache.wait_limit") *value = ctx->cache_wait_limit;
    else if (n == "cache.infer_groups") *value = ctx->cache_infer_groups;
    else if (n == "cache.infer_warps") *value = ctx->cache_infer_warps;
    else if (n == "cache.sort_queries") *value = ctx->cache_sort_queries;
    else if (n == "pt.shade_split") *value = ctx->pt_shade_split;
    else if (n == "pt.fetch") *value = ctx->pt_fetch;
    else if (n == "trace.stream_io") *value = ctx->trace_stream_io;
    else if (n == "trace.node_test") *value = ctx->trace_node_test;
    else if (n == "trace.l2_persist") *value = ctx->trace_l2_persist;
    else if (n == "debug.fail_alloc") *value = ctx->fail_alloc_countdown;
    else return RBR_ERR_INVALID_ARGUMENT;
    return RBR_OK;
}

rbr_status rbr_scene_stats_get(const rbr_ctx* ctx, rbr_scene_stats* out) {
    if (!ctx || !out) return RBR_ERR_INVALID_ARGUMENT;
    if (!ctx->has_scene) return RBR_ERR_NO_SCENE;
    *out = ctx->stats;
    return RBR_OK;
}

rbr_status rbr_world_bounds(const rbr_ctx* ctx, float out_min[3], float out_max[3]) {
    if (!ctx || !out_min || !out_max) return RBR_ERR_INVALID_ARGUMENT;
    if (!ctx->has_scene) return RBR_ERR_NO_SCENE;
    for (int a = 0; a < 3; ++a) {
        out_min[a] = ctx->bounds_lo[a];
        out_max[a] = ctx->bounds_hi[a];
    }
    return RBR_OK;
}

rbr_status rbr_trace_closest(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, rbr_hit* hits, void* stream) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    if (!ctx->has_scene) return fail(ctx, RBR_ERR_NO_SCENE, "rbr_trace_closest before rbr_scene_upload");
    if (n && (!rays || !hits)) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "rays or hits is NULL");
    const DeviceScope scope(ctx->device);
    const cudaError_t e = launch_trace(ctx, rays, n, 0, hits, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? RBR_OK : cuda_fail(ctx, e, "closest-hit launch");
}

rbr_status rbr_trace_any(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, uint8_t* occluded, void* stream) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    if (!ctx->has_scene) return fail(ctx, RBR_ERR_NO_SCENE, "rbr_trace_any before rbr_scene_upload");
    if (n && (!rays || !occluded)) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "rays or occluded is NULL");
    const DeviceScope scope(ctx->device);
    const cudaError_t e = launch_trace(ctx, rays, n, 1, occluded, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? RBR_OK : cuda_fail(ctx, e, "any-hit launch");
}

rbr_status rbr_trace_host(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, int any_hit, void* out) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    if (!ctx->has_scene) return fail(ctx, RBR_ERR_NO_SCENE, "rbr_trace_host before rbr_scene_upload");
    if (n == 0) return RBR_OK;
    if (!rays || !out) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "rays or out is NULL");
    const DeviceScope scope(ctx->device);
    const size_t in_bytes = size_t(n) * sizeof(rbr_ray);
    const size_t out_bytes = size_t(n) * (any_hit ? 1 : sizeof(rbr_hit));
    rbr_status st;
    if ((st = ensure(ctx, ctx->stage_in, in_bytes, "ray staging")) != RBR_OK) return st;
    if ((st = ensure(ctx, ctx->stage_out, out_bytes, "hit staging")) != RBR_OK) return st;
    cudaStream_t s = ctx->stream;
    // Chunks rotate over `trace.host_streams` streams (upload, traversal and download of a
    // chunk in order on its stream), so that the upload of one chunk, the traversal of another
    // and the download of a third overlap: copies in each direction and kernels run on
    // separate engines, and a chunk's upload waits only for the download of the chunk that
    // used its stream before.
    const uint32_t chunk = ctx->trace_host_chunk && n > ctx->trace_host_chunk ? ctx->trace_host_chunk : n;
    const bool two = chunk < n;
    const int ns = two ? std::max(2, std::min(4, ctx->trace_host_streams)) : 1;
    if (two && (st = ensure_side_stream(ctx)) != RBR_OK) return st;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i + 2 < ns && e == cudaSuccess; ++i) {
        if (!ctx->host_streams[i]) e = cudaStreamCreateWithFlags(&ctx->host_streams[i], cudaStreamNonBlocking);
        if (e == cudaSuccess && !ctx->host_join[i]) e = cudaEventCreateWithFlags(&ctx->host_join[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "trace streams");
    const cudaStream_t streams[4] = {s, ctx->side_stream, ctx->host_streams[0], ctx->host_streams[1]};
    const cudaEvent_t joins[4] = {nullptr, ctx->ev_join, ctx->host_join[0], ctx->host_join[1]};
    const size_t osz = any_hit ? 1 : sizeof(rbr_hit);
    if (two) {
        e = cudaEventRecord(ctx->ev_fork, s);
        for (int i = 1; i < ns && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(streams[i], ctx->ev_fork, 0);
    }
    uint32_t k = 0;
    // The last chunk's traversal and download run after the last upload, so the rays of the
    // last full chunk are split into halving pieces (down to a quarter chunk): a shorter tail.
    const uint32_t min_piece = std::max(1u, chunk / 4);
    uint32_t m = 0;
    for (uint32_t off = 0; off < n && e == cudaSuccess; off += m, ++k) {
        const uint32_t rest = n - off;
        m = !two || rest > chunk ? std::min(chunk, rest) : rest > min_piece ? rest - rest / 2 : rest;
        const int slot = static_cast<int>(k % static_cast<uint32_t>(ns));
        const cudaStream_t cs = streams[slot];
        rbr_ray* din = static_cast<rbr_ray*>(ctx->stage_in.ptr) + off;
        char* dout = static_cast<char*>(ctx->stage_out.ptr) + size_t(off) * osz;
        e = cudaMemcpyAsync(din, rays + off, size_t(m) * sizeof(rbr_ray), cudaMemcpyHostToDevice, cs);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "ray upload");
        e = launch_trace(ctx, din, m, any_hit, dout, cs, slot);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "trace launch");
        e = cudaMemcpyAsync(static_cast<char*>(out) + size_t(off) * osz, dout, size_t(m) * osz, cudaMemcpyDeviceToHost, cs);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "hit download");
    }
    for (int i = 1; i < ns && e == cudaSuccess; ++i) {
        e = cudaEventRecord(joins[i], streams[i]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, joins[i], 0);
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "trace pipeline");
    return check_device_error(ctx, s);
}

rbr_status rbr_trace_counts(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, int any_hit, uint64_t out[2]) {
    if (!ctx || !out) return RBR_ERR_INVALID_ARGUMENT;
    if (!ctx->has_scene) return fail(ctx, RBR_ERR_NO_SCENE, "rbr_trace_counts before rbr_scene_upload");
    if (n && !rays) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "rays is NULL");
    const DeviceScope scope(ctx->device);
    rbr_status st = ensure(ctx, ctx->stage_out, 2 * sizeof(unsigned long long), "count totals");
    if (st != RBR_OK) return st;
    auto* d = static_cast<unsigned long long*>(ctx->stage_out.ptr);
    cudaError_t e = cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), ctx->stream);
    if (e == cudaSuccess) e = launch_trace_counts(ctx->scene, rays, n, any_hit, d, ctx->d_error, ctx->stream);
    unsigned long long h[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "counting traversal");
    st = check_device_error(ctx, ctx->stream);
    out[0] = h[0];
    out[1] = h[1];
    return st;
}

rbr_status rbr_render(rbr_ctx* ctx, const rbr_camera* camera, const rbr_render_params* params, float* film_mean,
                      float* film_m2, void* stream) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    return render(ctx, camera, params, film_mean, film_m2, static_cast<cudaStream_t>(stream));
}

rbr_status rbr_render_noalloc(rbr_ctx* ctx, const rbr_camera* camera, const rbr_render_params* params,
                              float* film_mean, void* stream) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    return render_noalloc(ctx, camera, params, film_mean, static_cast<cudaStream_t>(stream));
}

rbr_status rbr_render_host(rbr_ctx* ctx, const rbr_camera* camera, const rbr_render_params* params, float* film_mean,
                           float* film_m2) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    if (!camera || !film_mean) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "camera or film_mean is NULL");
    if (camera->width <= 0 || camera->height <= 0) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "empty image");
    const DeviceScope scope(ctx->device);
    const size_t bytes = size_t(camera->width) * camera->height * 3 * sizeof(float);
    rbr_status st;
    if ((st = ensure(ctx, ctx->stage_out, 2 * bytes, "film staging")) != RBR_OK) return st;
    float* dmean = static_cast<float*>(ctx->stage_out.ptr);
    float* dm2 = film_m2 ? dmean + size_t(camera->width) * camera->height * 3 : nullptr;
    if ((st = render(ctx, camera, params, dmean, dm2, ctx->stream)) != RBR_OK) return st;
    cudaError_t e = cudaMemcpyAsync(film_mean, dmean, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && film_m2) e = cudaMemcpyAsync(film_m2, dm2, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "film download");
    return check_device_error(ctx, ctx->stream);
}

rbr_status rbr_render_stats_get(rbr_ctx* ctx, rbr_render_stats* out) {
    if (!ctx || !out) return RBR_ERR_INVALID_ARGUMENT;
    if (ctx->render_pending) {
        const DeviceScope scope(ctx->device);
        cudaError_t e = cudaEventSynchronize(ctx->ev_stop);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "waiting for the render");
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
        ctx->last_render.milliseconds = ms;
        ctx->render_pending = false;
        const rbr_status st = read_render_counters(ctx);
        if (st != RBR_OK) return st;
    }
    *out = ctx->last_render;
    return RBR_OK;
}

// ---- radiance cache ----------------------------------------------------------------------
void rbr_cache_config_default(rbr_cache_config* out) {
    if (out) cache_config_default(out);
}

rbr_status rbr_cache_create(rbr_ctx* ctx, const rbr_cache_config* config) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    cudaDeviceSynchronize();  // nothing may still use the cache being replaced
    return cache_create(ctx, config);
}

void rbr_cache_destroy(rbr_ctx* ctx) {
    if (!ctx) return;
    const DeviceScope scope(ctx->device);
    cudaDeviceSynchronize();
    cache_destroy(ctx);
}

rbr_status rbr_cache_info_get(rbr_ctx* ctx, rbr_cache_info* out) {
    if (!ctx || !out) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "NULL argument");
    const DeviceScope scope(ctx->device);
    return cache_info(ctx, out);
}

rbr_status rbr_cache_set_params(rbr_ctx* ctx, const uint16_t* mlp_bf16, const uint16_t* grid_f16) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    cudaDeviceSynchronize();
    return cache_set_params(ctx, mlp_bf16, grid_f16);
}

rbr_status rbr_cache_get_params(rbr_ctx* ctx, uint16_t* mlp_bf16, uint16_t* grid_f16) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    return cache_get_params(ctx, mlp_bf16, grid_f16);
}

rbr_status rbr_cache_grads_get(rbr_ctx* ctx, float* mlp, float* grid) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    return cache_grads(ctx, mlp, grid);
}

rbr_status rbr_cache_encode_host(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, float* inputs) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    return cache_encode_host(ctx, n, records, inputs);
}

rbr_status rbr_cache_infer_host(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, float* rgb) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    return cache_infer_host(ctx, n, records, rgb);
}

rbr_status rbr_cache_train_host(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, const float* targets,
                                int apply, float* loss) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    return cache_train_host(ctx, n, records, targets, apply, loss);
}

rbr_status rbr_cache_render(rbr_ctx* ctx, const rbr_camera* camera, const rbr_render_params* params, uint32_t frames,
                            int train, float* film_mean, float* film_m2, void* stream) {
    if (!ctx) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    return render_cached(ctx, camera, params, frames, train, film_mean, film_m2, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
