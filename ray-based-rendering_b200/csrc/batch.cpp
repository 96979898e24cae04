// Batched request loop: packs requests of several scenes, resolutions, sample counts and
// integrators into waves of the wavefront path tracer, replays each wave shape from a captured
// CUDA graph, and records per-request latency. No counterpart in the reference.
//
// A wave holds "segments" (pixel ranges of requests, with all their samples) of one scene
// and one integrator mode; a request larger than the free part of a wave continues in the
// next. Every path finds its request's camera, random-number key and parameters in the
// segment table (SegDev) that is copied to a fixed device address before the wave, so the
// kernels' arguments, and with them the captured graph, are the same for every wave of a
// given (scene, mode, depth, grid).
//
// Requests may carry an arrival time: they are then served in arrival order and no wave
// starts before its last request has arrived (device clock), which makes the latencies those
// of a server under staggered arrivals. With `persistent`, one cooperative launch of
// k_wave_loop renders every wave of the run (all stages, grid barriers between them, bounded
// waits) instead of one graph launch per wave. Either way the device clock stamps the start of
// the run and the end of every wave, and a request's latency runs from its arrival to the end
// of its last wave.
#include <algorithm>
#include <numeric>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "rbr_context.h"

using namespace rbr;

namespace {

constexpr uint32_t kMaxSegs = 512;                       // segments per wave
constexpr size_t kHdrBytes = 64;                         // [paths, segments], padded
constexpr size_t kTableBytes = kHdrBytes + sizeof(SegDev) * kMaxSegs;

constexpr uint64_t kMaxArrivalUs = 600000000ull;        // 10 minutes

struct Req {
    rbr_request r{};
    float* host_film = nullptr;  // rbr_batch_set_host_film: copied there after the last wave
    uint32_t id = 0;
    uint32_t first_wave = 0, last_wave = 0, waves = 0, segments = 0;
    uint64_t paths = 0;
};

struct WavePlan {
    uint32_t scene = 0;
    int mode = 0;
    bool train = false;
    uint32_t max_depth = 0;
    uint32_t paths = 0;
    uint64_t release_ns = 0;  // arrival of its last request
    std::vector<SegDev> segs;
};

using GraphKey = std::tuple<uint32_t, int, uint32_t, int, bool, uint32_t, int>;  // scene, mode, depth, grid, train, capacity, slot

size_t film_bytes(const rbr_request& r) { return size_t(r.camera.width) * size_t(r.camera.height) * 3 * sizeof(float); }

}  // namespace

struct rbr_batch {
    rbr_ctx* eng = nullptr;
    rbr_batch_config cfg{};
    std::string error;
    std::vector<rbr_ctx*> scenes;
    std::vector<Req> pending;
    std::vector<Req> done;                       // requests of the last run
    std::map<uint32_t, size_t> done_index;
    uint32_t next_id = 0;
    void* d_table = nullptr;
    void* h_stage = nullptr;
    size_t h_stage_bytes = 0;
    std::vector<cudaEvent_t> events;            // [0] run start, [w + 1] end of wave w, [waves + 1] run end
    uint32_t run_waves = 0;
    int run_slots = 1;                           // waves in flight in the last run
    cudaStream_t side = nullptr;                 // stream of the odd waves (two in flight)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_cache = nullptr;
    std::map<GraphKey, cudaGraphExec_t> graphs;
    uint32_t graph_generation = 0;               // path-buffer generation the graphs were captured with
    std::map<uint32_t, const void*> cache_buffers;  // per cached scene: its query buffer at capture
    rbr_batch_stats stats{};
    bool ran = false;
    // device clock of the last run: [0] start, [1 + w] end of wave w
    unsigned long long* d_stamps = nullptr;
    size_t d_stamps_n = 0;
    std::vector<unsigned long long> h_stamps;
    bool stamps_read = false;
    std::vector<uint64_t> run_release;           // release time of every wave of the last run (ns)
    bool run_persistent = false;
    // persistent runs: wave list + segment tables of the whole run, and the grid barrier
    void* d_loop = nullptr;
    size_t d_loop_bytes = 0;
    uint32_t* d_bar = nullptr;
};

namespace {

rbr_status bfail(rbr_batch* b, rbr_status code, const std::string& msg) {
    if (b) b->error = msg;
    return code;
}

rbr_status bcuda(rbr_batch* b, cudaError_t e, const char* what) {
    cudaGetLastError();
    return bfail(b, e == cudaErrorMemoryAllocation ? RBR_ERR_OUT_OF_MEMORY : RBR_ERR_CUDA,
                 std::string(what) + ": " + cudaGetErrorString(e));
}

void drop_graphs(rbr_batch* b) {
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
}

int mode_of(const rbr_request& r) {
    if (r.use_cache) return 1;
    return (r.params.flags & RBR_RENDER_VOLUMETRIC) ? 2 : 0;
}

uint32_t max_lights(const rbr_batch* b) {
    uint32_t n = 1;
    for (const rbr_ctx* s : b->scenes) n = std::max(n, s->scene.num_lights);
    return n;
}

// Paths per wave: the configured count, else what the memory budget allows (path state,
// segment index, shadow queue of every light, cache query records), at most 2^23.
uint32_t wave_capacity(const rbr_batch* b, bool any_cache) {
    if (b->cfg.wave_paths) return b->cfg.wave_paths;
    const uint64_t per_path = 96 + 4 + 48ull * max_lights(b) + (any_cache ? 80 : 0);
    const uint64_t cap = b->cfg.path_memory_bytes / per_path;
    return static_cast<uint32_t>(std::max<uint64_t>(1u << 16, std::min<uint64_t>(cap, 1u << 23)));
}

using WaveKey = std::tuple<uint32_t, int, bool>;  // scene, mode, train
WaveKey key_of(const Req& q) { return std::make_tuple(q.r.scene, mode_of(q.r), q.r.use_cache && q.r.train_cache); }

// Packs the requests into waves of `cap` paths, first come first served. Without arrival
// times the requests are grouped by (scene, mode, train) in order of first appearance; with
// them they are taken in arrival order and a wave closes whenever the next request needs
// another scene or mode. A wave's release time is the arrival of its last request.
std::vector<WavePlan> plan(rbr_batch* b, std::vector<Req>& reqs, uint32_t cap) {
    bool arrivals = false;
    for (const Req& q : reqs) arrivals = arrivals || q.r.arrival_us != 0;
    std::vector<std::vector<size_t>> groups;  // request indices, packed group by group
    if (arrivals) {
        std::vector<size_t> order(reqs.size());
        std::iota(order.begin(), order.end(), size_t(0));
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t x, size_t y) { return reqs[x].r.arrival_us < reqs[y].r.arrival_us; });
        for (size_t i : order) {
            if (groups.empty() || key_of(reqs[groups.back().front()]) != key_of(reqs[i])) groups.emplace_back();
            groups.back().push_back(i);
        }
    } else {
        std::vector<WaveKey> keys;
        for (size_t i = 0; i < reqs.size(); ++i) {
            const auto it = std::find(keys.begin(), keys.end(), key_of(reqs[i]));
            if (it == keys.end()) {
                keys.push_back(key_of(reqs[i]));
                groups.emplace_back();
                groups.back().push_back(i);
            } else {
                groups[static_cast<size_t>(it - keys.begin())].push_back(i);
            }
        }
    }
    std::vector<WavePlan> waves;
    for (const auto& group : groups) {
        const WaveKey k = key_of(reqs[group.front()]);
        WavePlan cur;
        cur.scene = std::get<0>(k);
        cur.mode = std::get<1>(k);
        cur.train = std::get<2>(k);
        auto close = [&]() {
            if (!cur.segs.empty()) waves.push_back(cur);
            cur.segs.clear();
            cur.paths = 0;
            cur.max_depth = 0;
            cur.release_ns = 0;
        };
        for (size_t qi : group) {
            Req& q = reqs[qi];
            const rbr_request& r = q.r;
            const uint32_t spp = static_cast<uint32_t>(r.params.samples_per_pixel);
            const uint32_t npix = static_cast<uint32_t>(r.camera.width) * static_cast<uint32_t>(r.camera.height);
            uint32_t next = 0;
            while (next < npix) {
                const uint32_t take = std::min(npix - next, (cap - cur.paths) / spp);
                if (take == 0 || cur.segs.size() == kMaxSegs) {
                    close();
                    continue;
                }
                SegDev g{};
                g.cam = camera_dev(&r.camera);
                g.film = r.film;
                g.seed = r.params.seed;
                g.path0 = cur.paths;
                g.npaths = take * spp;
                g.p0 = next;
                g.spp = spp;
                g.sample_offset = r.params.sample_offset;
                g.width = static_cast<uint32_t>(r.camera.width);
                g.max_depth = static_cast<uint32_t>(r.params.max_depth);
                g.use_nee = r.params.use_nee != 0;
                g.use_mis = r.params.use_mis != 0;
                const uint32_t w = static_cast<uint32_t>(waves.size());
                if (q.waves == 0 || q.last_wave != w) {
                    if (q.waves == 0) q.first_wave = w;
                    q.last_wave = w;
                    ++q.waves;
                }
                ++q.segments;
                q.paths += g.npaths;
                cur.release_ns = std::max(cur.release_ns, uint64_t(r.arrival_us) * 1000u);
                cur.segs.push_back(g);
                cur.paths += g.npaths;
                cur.max_depth = std::max(cur.max_depth, g.max_depth);
                next += take;
            }
        }
        close();
    }
    return waves;
}

rbr_status ensure_events(rbr_batch* b, size_t n) {
    while (b->events.size() < n) {
        cudaEvent_t e;
        const cudaError_t c = cudaEventCreate(&e);
        if (c != cudaSuccess) return bcuda(b, c, "cudaEventCreate");
        b->events.push_back(e);
    }
    return RBR_OK;
}

// Renders `reqs` (the queue is not modified). Fills the requests' wave bookkeeping.
rbr_status run(rbr_batch* b, std::vector<Req>& reqs, cudaStream_t stream) {
    rbr_ctx* eng = b->eng;
    if (b->ran) {  // the staging buffer and events of the previous run are reused
        const cudaError_t e = cudaEventSynchronize(b->events[b->run_waves + 1]);
        if (e != cudaSuccess) return bcuda(b, e, "waiting for the previous run");
    }
    const int slots = b->cfg.waves_in_flight == 1 ? 1 : 2;
    if (slots == 2 && !b->side) {
        cudaError_t e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_cache, cudaEventDisableTiming);
        if (e != cudaSuccess) return bcuda(b, e, "second wave stream");
    }
    bool any_cache = false;
    for (const Req& q : reqs) any_cache = any_cache || q.r.use_cache;
    const uint32_t cap = wave_capacity(b, any_cache);
    for (const Req& q : reqs)
        if (static_cast<uint32_t>(q.r.params.samples_per_pixel) > cap)
            return bfail(b, RBR_ERR_INVALID_ARGUMENT, "request " + std::to_string(q.id) + ": samples per pixel exceed the wave");
    for (const Req& q : reqs)
        if (q.r.arrival_us > kMaxArrivalUs)
            return bfail(b, RBR_ERR_INVALID_ARGUMENT, "request " + std::to_string(q.id) + ": arrival beyond 600 s");
    std::vector<WavePlan> waves = plan(b, reqs, cap);
    const bool persistent = b->cfg.persistent && !any_cache && !waves.empty() && b->scenes.size() <= 16;
    const uint32_t nl = max_lights(b);
    rbr_status st = ensure_wave_buffers(eng, cap, cap * nl, slots);
    if (st != RBR_OK) return bfail(b, st, eng->error);
    for (const WavePlan& w : waves) {
        if (w.mode != 1) continue;
        rbr_ctx* scn = b->scenes[w.scene];
        const uint32_t t_cap = static_cast<uint32_t>(
            std::min<uint64_t>(uint64_t(std::max(1u, scn->cache.cfg.train_paths)) * std::max(1u, w.max_depth), 1u << 23));
        st = cache_ensure_render(scn, cap, t_cap);
        if (st != RBR_OK) return bfail(b, st, scn->error);
        const void* qb = scn->cache.q_rec;
        auto it = b->cache_buffers.find(w.scene);
        if (it != b->cache_buffers.end() && (it->second != qb)) drop_graphs(b);
        b->cache_buffers[w.scene] = qb;
    }
    if (b->graph_generation != eng->pt_generation) {  // path buffers reallocated since the capture
        drop_graphs(b);
        b->graph_generation = eng->pt_generation;
    }
    // persistent runs upload the wave list and every segment table at once
    const size_t list_bytes = (waves.size() * sizeof(LoopWave) + 255) & ~size_t(255);
    const size_t need = (persistent ? list_bytes : 0) + std::max<size_t>(1, waves.size()) * kTableBytes;
    if (b->h_stage_bytes < need) {
        if (b->h_stage) cudaFreeHost(b->h_stage);
        b->h_stage = nullptr;
        b->h_stage_bytes = 0;
        const cudaError_t e = cudaMallocHost(&b->h_stage, need);
        if (e != cudaSuccess) return bcuda(b, e, "pinned segment tables");
        b->h_stage_bytes = need;
    }
    st = ensure_events(b, waves.size() + 2);
    if (st != RBR_OK) return st;
    if (b->d_stamps_n < waves.size() + 1) {
        if (b->d_stamps) cudaFree(b->d_stamps);
        b->d_stamps = nullptr;
        b->d_stamps_n = 0;
        const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->d_stamps), (waves.size() + 1) * 8);
        if (e != cudaSuccess) return bcuda(b, e, "wave time stamps");
        b->d_stamps_n = waves.size() + 1;
    }
    b->run_release.clear();
    for (const WavePlan& w : waves) b->run_release.push_back(w.release_ns);
    b->stamps_read = false;
    const int grid = eng->num_sms * static_cast<int>(b->cfg.blocks_per_sm ? b->cfg.blocks_per_sm : 8);
    rbr_batch_stats s{};
    s.requests = static_cast<uint32_t>(reqs.size());
    s.wave_paths = cap;
    s.blocks_per_sm = b->cfg.blocks_per_sm ? b->cfg.blocks_per_sm : 8;
    if (persistent) {
        // one cooperative launch: the wave list, then every wave's segment table
        char* host = static_cast<char*>(b->h_stage);
        for (size_t wi = 0; wi < waves.size(); ++wi) {
            const WavePlan& w = waves[wi];
            LoopWave lw{};
            lw.scene = w.scene;
            lw.mode = static_cast<uint32_t>(w.mode);
            lw.max_depth = w.max_depth;
            lw.table = static_cast<uint32_t>(wi * kTableBytes);
            lw.release_ns = w.release_ns;
            std::memcpy(host + wi * sizeof(LoopWave), &lw, sizeof(lw));
            char* tab = host + list_bytes + wi * kTableBytes;
            const uint32_t hdr[2] = {w.paths, static_cast<uint32_t>(w.segs.size())};
            std::memcpy(tab, hdr, sizeof(hdr));
            std::memcpy(tab + kHdrBytes, w.segs.data(), w.segs.size() * sizeof(SegDev));
            s.segments += static_cast<uint32_t>(w.segs.size());
            s.paths += w.paths;
        }
        if (b->d_loop_bytes < need) {
            if (b->d_loop) cudaFree(b->d_loop);
            b->d_loop = nullptr;
            b->d_loop_bytes = 0;
            const cudaError_t e = cudaMalloc(&b->d_loop, need);
            if (e != cudaSuccess) return bcuda(b, e, "persistent wave list");
            b->d_loop_bytes = need;
        }
        if (!b->d_bar) {
            const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->d_bar), kLoopBarrierWords * sizeof(uint32_t));
            if (e != cudaSuccess) return bcuda(b, e, "grid barrier");
        }
        const uint64_t limit_ns = uint64_t(b->cfg.barrier_timeout_us ? b->cfg.barrier_timeout_us : 2000000u) * 1000ull;
        int loop_grid = 0;
        cudaError_t e = cudaEventRecord(b->events[0], stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_loop, host, need, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess)
            e = launch_wave_loop(eng, b->scenes, static_cast<const LoopWave*>(b->d_loop), static_cast<uint32_t>(waves.size()),
                                 static_cast<const char*>(b->d_loop) + list_bytes, b->d_stamps, b->d_bar, limit_ns, slots,
                                 stream, &loop_grid);
        for (const Req& q : reqs)
            if (e == cudaSuccess && q.host_film)
                e = cudaMemcpyAsync(q.host_film, q.r.film, film_bytes(q.r), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaEventRecord(b->events[waves.size() + 1], stream);
        if (e != cudaSuccess) return bcuda(b, e, "persistent wave loop");
        s.waves = static_cast<uint32_t>(waves.size());
        s.kernel_launches = 1;
        s.persistent_launches = 1;
        s.blocks_per_sm = static_cast<uint32_t>(loop_grid / std::max(1, eng->num_sms));
        b->stats = s;
        b->run_waves = s.waves;
        b->run_slots = slots;
        b->run_persistent = true;
        b->ran = true;
        return RBR_OK;
    }
    // Waves alternate between two path-buffer sets, segment tables and streams (slot = wave
    // index & 1), so one wave's latency-bound last bounces run beside the next wave. Waves
    // with the radiance cache share the scene's cache buffers and weights: each waits for the
    // previous one.
    cudaError_t e = cudaEventRecord(b->events[0], stream);
    if (e == cudaSuccess) e = launch_stamp(b->d_stamps, stream);
    ++s.kernel_launches;
    if (e == cudaSuccess && slots == 2) e = cudaEventRecord(b->ev_fork, stream);
    if (e == cudaSuccess && slots == 2) e = cudaStreamWaitEvent(b->side, b->ev_fork, 0);
    bool cache_wave = false;
    // requests whose film goes to the host, by their last wave: the copy follows that wave on
    // its stream and overlaps the waves after it
    std::vector<std::vector<const Req*>> to_host(waves.size());
    for (const Req& q : reqs)
        if (q.host_film && q.waves > 0) to_host[q.last_wave].push_back(&q);
    for (size_t wi = 0; wi < waves.size() && e == cudaSuccess; ++wi) {
        const WavePlan& w = waves[wi];
        rbr_ctx* scn = b->scenes[w.scene];
        const int slot = slots == 2 ? static_cast<int>(wi & 1) : 0;
        const cudaStream_t ws = slot ? b->side : stream;
        if (w.mode == 1 && cache_wave && slots == 2) {
            e = cudaStreamWaitEvent(ws, b->ev_cache, 0);
            if (e != cudaSuccess) break;
        }
        if (w.release_ns) {  // admission: not before the arrival of the wave's last request
            e = launch_release(b->d_stamps, w.release_ns, ws);
            ++s.kernel_launches;
            if (e != cudaSuccess) break;
        }
        char* dtab = static_cast<char*>(b->d_table) + slot * kTableBytes;
        char* tab = static_cast<char*>(b->h_stage) + wi * kTableBytes;
        uint32_t hdr[2] = {w.paths, static_cast<uint32_t>(w.segs.size())};
        std::memcpy(tab, hdr, sizeof(hdr));
        std::memcpy(tab + kHdrBytes, w.segs.data(), w.segs.size() * sizeof(SegDev));
        e = cudaMemcpyAsync(dtab, tab, kHdrBytes + w.segs.size() * sizeof(SegDev), cudaMemcpyHostToDevice, ws);
        if (e != cudaSuccess) break;
        PackedWave pw;
        pw.mode = w.mode;
        pw.max_depth = w.max_depth;
        pw.grid = grid;
        pw.hdr = reinterpret_cast<const uint32_t*>(dtab);
        pw.segs = reinterpret_cast<const SegDev*>(dtab + kHdrBytes);
        pw.capacity = eng->pt.capacity;
        pw.train = w.train;
        pw.slot = slot;
        if (w.mode == 1) {
            const double frac = double(scn->cache.cfg.train_paths) / double(cap);
            pw.train_thresh = static_cast<uint32_t>(std::min(4294967295.0, frac * 4294967296.0));
            pw.train_steps = scn->cache.cfg.train_steps;
        }
        s.kernel_launches += packed_wave_launches(pw);
        s.segments += static_cast<uint32_t>(w.segs.size());
        s.paths += w.paths;
        if (b->cfg.use_graphs) {
            const GraphKey key{w.scene, w.mode, w.max_depth, grid, w.train, eng->pt.capacity, slot};
            auto it = b->graphs.find(key);
            if (it == b->graphs.end()) {
                cudaGraph_t g = nullptr;
                e = cudaStreamBeginCapture(eng->stream, cudaStreamCaptureModeThreadLocal);
                if (e != cudaSuccess) break;
                const cudaError_t le = launch_packed_wave(eng, scn, pw, eng->stream);
                e = cudaStreamEndCapture(eng->stream, &g);
                if (le != cudaSuccess) e = le;
                cudaGraphExec_t exec = nullptr;
                if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
                if (g) cudaGraphDestroy(g);
                if (e != cudaSuccess) break;
                it = b->graphs.emplace(key, exec).first;
                ++s.graphs_captured;
            }
            e = cudaGraphLaunch(it->second, ws);
            ++s.graph_launches;
        } else {
            e = launch_packed_wave(eng, scn, pw, ws);
        }
        if (e == cudaSuccess) e = launch_stamp(b->d_stamps + 1 + wi, ws);
        ++s.kernel_launches;
        for (const Req* q : to_host[wi]) {
            // a request spread over several waves also has pixels from waves of the other slot:
            // wait for that stream's last wave before this one (it holds every earlier one)
            if (e == cudaSuccess && slots == 2 && q->first_wave < wi) e = cudaStreamWaitEvent(ws, b->events[wi], 0);
            if (e == cudaSuccess) e = cudaMemcpyAsync(q->host_film, q->r.film, film_bytes(q->r), cudaMemcpyDeviceToHost, ws);
        }
        if (e == cudaSuccess) e = cudaEventRecord(b->events[wi + 1], ws);
        if (e == cudaSuccess && w.mode == 1 && slots == 2) {
            e = cudaEventRecord(b->ev_cache, ws);
            cache_wave = true;
        }
    }
    if (e == cudaSuccess && slots == 2) e = cudaEventRecord(b->ev_join, b->side);
    if (e == cudaSuccess && slots == 2) e = cudaStreamWaitEvent(stream, b->ev_join, 0);
    if (e == cudaSuccess) e = cudaEventRecord(b->events[waves.size() + 1], stream);
    if (e != cudaSuccess) return bcuda(b, e, "batched wave launch");
    s.waves = static_cast<uint32_t>(waves.size());
    b->stats = s;
    b->run_waves = s.waves;
    b->run_slots = slots;
    b->run_persistent = false;
    b->ran = true;
    return RBR_OK;
}

}  // namespace

extern "C" {

void rbr_batch_config_default(rbr_batch_config* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->path_memory_bytes = 2ull << 30;
    out->wave_paths = 0;
    out->blocks_per_sm = 8;
    out->use_graphs = 1;
    out->waves_in_flight = 2;
    out->persistent = 0;
    out->barrier_timeout_us = 2000000;
}

rbr_status rbr_batch_create(rbr_ctx* ctx, const rbr_batch_config* config, rbr_batch** out) {
    if (!ctx || !out) return RBR_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    rbr_batch* b = new (std::nothrow) rbr_batch();
    if (!b) return RBR_ERR_OUT_OF_MEMORY;
    b->eng = ctx;
    if (config) b->cfg = *config;
    else rbr_batch_config_default(&b->cfg);
    if (b->cfg.path_memory_bytes == 0) b->cfg.path_memory_bytes = 2ull << 30;
    const DeviceScope scope(ctx->device);
    const cudaError_t e = cudaMalloc(&b->d_table, 2 * kTableBytes);  // a segment table per wave in flight
    if (e != cudaSuccess) {
        delete b;
        return RBR_ERR_OUT_OF_MEMORY;
    }
    *out = b;
    return RBR_OK;
}

void rbr_batch_destroy(rbr_batch* b) {
    if (!b) return;
    const DeviceScope scope(b->eng->device);
    cudaDeviceSynchronize();
    drop_graphs(b);
    for (cudaEvent_t e : b->events) cudaEventDestroy(e);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->ev_cache) cudaEventDestroy(b->ev_cache);
    for (size_t i = b->scenes.size(); i-- > 0;) rbr_ctx_destroy(b->scenes[i]);  // variants before their bases
    if (b->d_table) cudaFree(b->d_table);
    if (b->d_stamps) cudaFree(b->d_stamps);
    if (b->d_loop) cudaFree(b->d_loop);
    if (b->d_bar) cudaFree(b->d_bar);
    if (b->h_stage) cudaFreeHost(b->h_stage);
    delete b;
}

const char* rbr_batch_last_error(const rbr_batch* b) { return b ? b->error.c_str() : "no batch"; }

rbr_status rbr_batch_add_scene(rbr_batch* b, const rbr_scene_desc* desc, uint32_t* scene_id) {
    if (!b || !desc || !scene_id) return bfail(b, RBR_ERR_INVALID_ARGUMENT, "NULL argument");
    rbr_ctx* s = nullptr;
    rbr_status st = rbr_ctx_create(b->eng->device, &s);
    if (st != RBR_OK) return bfail(b, st, "creating the scene slot");
    st = rbr_scene_upload(s, desc);
    if (st != RBR_OK) {
        b->error = s->error;
        rbr_ctx_destroy(s);
        return st;
    }
    *scene_id = static_cast<uint32_t>(b->scenes.size());
    b->scenes.push_back(s);
    return RBR_OK;
}

rbr_status rbr_batch_add_scene_variant(rbr_batch* b, uint32_t base_scene, const rbr_material* materials,
                                       uint32_t num_materials, const rbr_light* lights, uint32_t num_lights,
                                       const rbr_medium* medium, uint32_t* scene_id) {
    if (!b || !scene_id || base_scene >= b->scenes.size()) return bfail(b, RBR_ERR_INVALID_ARGUMENT, "unknown base scene");
    rbr_ctx* s = nullptr;
    rbr_status st = rbr_ctx_create(b->eng->device, &s);
    if (st != RBR_OK) return bfail(b, st, "creating the scene slot");
    st = upload_scene_variant(s, b->scenes[base_scene], materials, num_materials, lights, num_lights, medium);
    if (st != RBR_OK) {
        b->error = s->error;
        rbr_ctx_destroy(s);
        return st;
    }
    *scene_id = static_cast<uint32_t>(b->scenes.size());
    b->scenes.push_back(s);
    return RBR_OK;
}

rbr_status rbr_batch_cache_create(rbr_batch* b, uint32_t scene_id, const rbr_cache_config* config) {
    if (!b || scene_id >= b->scenes.size()) return bfail(b, RBR_ERR_INVALID_ARGUMENT, "unknown scene");
    drop_graphs(b);  // graphs of this scene's cache mode point at the old cache buffers
    const rbr_status st = rbr_cache_create(b->scenes[scene_id], config);
    if (st != RBR_OK) b->error = b->scenes[scene_id]->error;
    return st;
}

rbr_status rbr_batch_submit(rbr_batch* b, const rbr_request* r, uint32_t* request_id) {
    if (!b || !r) return bfail(b, RBR_ERR_INVALID_ARGUMENT, "NULL argument");
    if (r->scene >= b->scenes.size()) return bfail(b, RBR_ERR_INVALID_ARGUMENT, "unknown scene");
    if (!r->film) return bfail(b, RBR_ERR_INVALID_ARGUMENT, "film is NULL");
    if (r->camera.width <= 0 || r->camera.height <= 0 || r->params.samples_per_pixel <= 0 || r->params.max_depth < 1)
        return bfail(b, RBR_ERR_INVALID_ARGUMENT, "image size, samples per pixel or max depth (>= 1) out of range");
    if (r->camera.model != RBR_CAMERA_PINHOLE && r->camera.model != RBR_CAMERA_THIN_LENS)
        return bfail(b, RBR_ERR_UNSUPPORTED, "camera model " + std::to_string(r->camera.model));
    if (r->params.flags & ~static_cast<uint32_t>(RBR_RENDER_VOLUMETRIC))
        return bfail(b, RBR_ERR_UNSUPPORTED, "batched requests take no flag other than RBR_RENDER_VOLUMETRIC");
    if (r->use_cache && (r->params.flags & RBR_RENDER_VOLUMETRIC))
        return bfail(b, RBR_ERR_UNSUPPORTED, "the radiance cache serves the surface path tracer only");
    if (r->use_cache && !b->scenes[r->scene]->cache.ready)
        return bfail(b, RBR_ERR_INVALID_ARGUMENT, "the scene has no radiance cache (rbr_batch_cache_create)");
    if (uint64_t(r->camera.width) * r->camera.height * r->params.samples_per_pixel > 0xFFFFFFFFull)
        return bfail(b, RBR_ERR_INVALID_ARGUMENT, "more than 2^32 samples in one request");
    if (r->arrival_us > kMaxArrivalUs || r->reserved != 0)
        return bfail(b, RBR_ERR_INVALID_ARGUMENT, "arrival beyond 600 s, or reserved field not 0");
    Req q;
    q.r = *r;
    q.id = b->next_id++;
    b->pending.push_back(q);
    if (request_id) *request_id = q.id;
    return RBR_OK;
}

rbr_status rbr_batch_set_host_film(rbr_batch* b, uint32_t request_id, float* host_film) {
    if (!b) return RBR_ERR_INVALID_ARGUMENT;
    for (Req& q : b->pending)
        if (q.id == request_id) {
            q.host_film = host_film;
            return RBR_OK;
        }
    return bfail(b, RBR_ERR_INVALID_ARGUMENT, "request not queued (rbr_batch_set_host_film before rbr_batch_run)");
}

rbr_status rbr_batch_run(rbr_batch* b, void* stream) {
    if (!b) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(b->eng->device);
    std::vector<Req> reqs = b->pending;
    const rbr_status st = run(b, reqs, static_cast<cudaStream_t>(stream));
    if (st != RBR_OK) return st;
    b->pending.clear();
    b->done = reqs;
    b->done_index.clear();
    for (size_t i = 0; i < b->done.size(); ++i) b->done_index[b->done[i].id] = i;
    return RBR_OK;
}

rbr_status rbr_batch_request_stats(rbr_batch* b, uint32_t id, rbr_request_stats* out) {
    if (!b || !out) return RBR_ERR_INVALID_ARGUMENT;
    auto it = b->done_index.find(id);
    if (it == b->done_index.end()) return bfail(b, RBR_ERR_INVALID_ARGUMENT, "request not in the last run");
    const Req& q = b->done[it->second];
    const DeviceScope scope(b->eng->device);
    cudaError_t e = cudaEventSynchronize(b->events[b->run_waves + 1]);
    if (e == cudaSuccess && !b->stamps_read) {
        b->h_stamps.assign(b->run_waves + 1, 0ull);
        e = cudaMemcpy(b->h_stamps.data(), b->d_stamps, (b->run_waves + 1) * 8, cudaMemcpyDeviceToHost);
        b->stamps_read = e == cudaSuccess;
    }
    if (e != cudaSuccess) return bcuda(b, e, "request timing");
    // device clock, ns: the run's start, the request's arrival, the end of its last wave; its
    // first wave started at its release time, or when the wave before it on the same path
    // buffers ended, whichever was later
    const double t0 = static_cast<double>(b->h_stamps[0]);
    const double arrival = t0 + 1000.0 * q.r.arrival_us;
    const double end = static_cast<double>(b->h_stamps[1 + q.last_wave]);
    const uint32_t fw = q.first_wave, lag = b->run_slots == 2 ? 2u : 1u;
    double start = fw >= lag ? static_cast<double>(b->h_stamps[1 + fw - lag]) : t0;
    start = std::max(start, t0 + static_cast<double>(b->run_release[fw]));
    out->start_ms = static_cast<float>(std::max(0.0, start - arrival) / 1e6);
    out->latency_ms = static_cast<float>(std::max(0.0, end - arrival) / 1e6);
    out->waves = q.waves;
    out->segments = q.segments;
    out->paths = q.paths;
    return RBR_OK;
}

rbr_status rbr_batch_stats_get(rbr_batch* b, rbr_batch_stats* out) {
    if (!b || !out) return RBR_ERR_INVALID_ARGUMENT;
    if (!b->ran) return bfail(b, RBR_ERR_INVALID_ARGUMENT, "no run yet");
    const DeviceScope scope(b->eng->device);
    cudaError_t e = cudaEventSynchronize(b->events[b->run_waves + 1]);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b->events[0], b->events[b->run_waves + 1]);
    if (e != cudaSuccess) return bcuda(b, e, "batch timing");
    *out = b->stats;
    out->milliseconds = ms;
    const rbr_status st = check_device_error(b->eng, 0);
    if (st != RBR_OK) b->error = b->eng->error;
    return st;
}

rbr_status rbr_batch_autotune(rbr_batch* b, void* stream) {
    if (!b) return RBR_ERR_INVALID_ARGUMENT;
    if (b->pending.empty()) return bfail(b, RBR_ERR_INVALID_ARGUMENT, "no queued requests to tune on");
    const DeviceScope scope(b->eng->device);
    const rbr_batch_config saved = b->cfg;
    bool any_cache = false;
    for (const Req& q : b->pending) any_cache = any_cache || q.r.use_cache;
    rbr_batch_config probe = saved;
    probe.wave_paths = 0;
    b->cfg = probe;
    const uint32_t budget_cap = wave_capacity(b, any_cache);
    float best = -1.0f;
    rbr_batch_config best_cfg = saved;
    for (uint32_t wp : {1u << 20, 1u << 21, 1u << 22, 1u << 23}) {
        if (wp > budget_cap) continue;
        for (uint32_t bps : {4u, 8u, 16u}) {
            b->cfg = saved;
            b->cfg.wave_paths = wp;
            b->cfg.blocks_per_sm = bps;
            float ms = 0.0f;
            for (int rep = 0; rep < 2; ++rep) {  // the first run captures the graphs
                std::vector<Req> reqs = b->pending;
                const rbr_status st = run(b, reqs, static_cast<cudaStream_t>(stream));
                if (st != RBR_OK) {
                    b->cfg = saved;
                    return st;
                }
                const cudaError_t e = cudaEventSynchronize(b->events[b->run_waves + 1]);
                if (e == cudaSuccess) cudaEventElapsedTime(&ms, b->events[0], b->events[b->run_waves + 1]);
            }
            if (best < 0.0f || ms < best) {
                best = ms;
                best_cfg = b->cfg;
            }
        }
    }
    b->cfg = best_cfg;
    b->ran = false;  // the tuning runs are not a run of the queue
    return RBR_OK;
}

}  // extern "C"
