// Wavefront path tracer: the GPU form of Integrator::render + PathTracingIntegrator::Li
// (src/renderers/integrator.cpp:7-50, src/renderers/path_tracing_integrator.cpp:5-138).
//
// Paths are processed in waves of up to `capacity` camera samples; all samples of a pixel
// belong to one wave, path k of a wave is sample (k % spp) of pixel (p0 + k / spp). Per wave:
//   raygen                         camera rays for every path (counter-RNG jitter and lens)
//   for depth = 0 .. maxDepth-1:
//     begin    reset the per-depth queue counters and claim cursors
//     extend   closest hit for the active queue; misses add background; hits are appended
//              to one of six material-class queues (match.any + one atomic per class and warp)
//     shade    per class queue: emission, next-event estimation over ALL lights (one shadow
//              ray per light with a non-black BSDF value, appended to the shadow queue with
//              its MIS-weighted contribution), BSDF sampling, Russian roulette after depth 3;
//              surviving paths are appended to the next active queue
//     shadow   any hit for the shadow queue; unoccluded contributions are added to the path
//   (extend, shade and shadow hand out a long queue by claims: see Claim)
//   film     per pixel, the sum of its samples' radiance in sample order / spp (what
//            Film::addSample(x, y, sum / spp) stores), plus the sum of squares on request
// The reference's estimator is reproduced, quirks included: emission only at depth 0 or after
// a delta bounce, MIS weight on light samples without the BSDF-sampled emitter term, NEE over
// every light, Russian roulette always on (q = max(0.05, 1 - max(T)) after depth 3). Its
// BSDF-sampled "MIS" trace whose result is discarded (path_tracing_integrator.cpp:118-134)
// changes nothing and is not traced.
#include <algorithm>

#include "rbr_bsdf.cuh"
#include "rbr_context.h"

namespace rbr {

namespace {

constexpr int kBlock = 128;
constexpr int kLoopScenes = 16;  // scenes one persistent batched run can address
constexpr uint32_t kDefaultCapacity = 1u << 22;  // most samples per pixel in one call (a wave holds a pixel's samples)
constexpr size_t kShadowBytesLimit = size_t(2) << 30;

// counters (uint32 words)
enum : int {
    kCQ0 = 0,       // active queue counts, ping-pong by depth parity
    kCClass = 2,    // kNumClasses class-queue counts
    kCShadow = 8,   // shadow queue count
    kCExt = 10,     // 64-bit: extension rays traced
    kCSh = 12,      // 64-bit: shadow rays traced
    kCQuery = 14,   // radiance cache: paths ended into the cache in this wave
    kCTrain = 15,   // radiance cache: training vertices gathered in this frame
    kCTrainBase = 16,  // radiance cache: kCTrain at the start of this wave
    kCShade = 18,      // 64-bit: hit vertices shaded
    kCTraffic = 20,    // 4 x 64-bit (RBR_RENDER_COUNT_TRAFFIC): extension nodes, records; shadow nodes, records
    kCCursor = 28,     // 3 claim cursors of one depth (Paths::fetch): extension, shading, shadow queue
    kCWords = 32
};
static_assert(kCClass + static_cast<int>(kNumClasses) <= kCShadow, "class-queue counts overlap the shadow count");
static_assert(kCExt % 2 == 0 && kCSh % 2 == 0 && kCShade % 2 == 0 && kCTraffic % 2 == 0, "64-bit counters");
static_assert(kCTraffic + 8 <= kCCursor && kCCursor + 3 <= kCWords, "claim cursors overlap");

// The blocks a stage runs on: the whole grid for the wavefront kernels, one half of it for a
// half of the persistent wave loop. Grid-stride loops start at block `block` of `blocks`.
struct Span {
    uint32_t block, blocks;
};
__device__ __forceinline__ Span grid_span() { return Span{blockIdx.x, gridDim.x}; }

// Work distribution of a stage over the n entries of a queue. A stage's cost per entry varies
// widely (a traversal that leaves the scene at once beside one that walks deep into the mesh),
// so with a fixed grid-stride share per warp the warps that drew the long traversals keep the
// launch alive while the others have exited. With a claim cursor (a queue counter reset at the
// start of each depth), a warp done with its entries instead claims the next ones by one atomic
// on the cursor, so warps that drew short traversals take more. Claims shrink as the queue
// drains (guided self-scheduling): a quarter of the entries left per warp, in multiples of 32
// from 256 down to 32, so that early claims are few and the last ones leave no warp with a
// long run of work behind the others. Atomics on the one cursor are served one after another,
// so a short queue of cheap entries would wait on its claims (claims from four rounds up made
// the foggy Cornell box 12 % slower): queues of fewer than kClaimRounds grid-stride rounds go
// out in the grid-stride order.
// take() returns this thread's entry (entries >= n are lanes without work) and sets `live`
// (warp-uniform) while the warp has entries: `for (j = c.take(); c.live; j = c.take())`.
constexpr uint32_t kClaimRounds = 8;
struct Claim {
    uint32_t* cursor;          // nullptr: grid-stride order
    uint32_t n, next, stride;  // grid-stride order: this block's next base
    uint32_t cb = 0, ce = 0;   // the warp's claimed range (warp-uniform)
    bool live = true;
    __device__ __forceinline__ Claim(uint32_t* cur, uint32_t count, Span g)
        : cursor(nullptr), n(count), next(g.block * blockDim.x), stride(g.blocks * blockDim.x) {
        if (cur && n / stride >= kClaimRounds) cursor = cur;
    }
    __device__ __forceinline__ uint32_t take() {
        const uint32_t lane = threadIdx.x & 31u;
        uint32_t j;
        if (!cursor) {
            j = next + threadIdx.x;
            next += stride;
        } else {
            if (cb >= ce) {
                uint32_t b = 0, r = 0;
                if (lane == 0) {
                    // the cursor as it stands (a plain load: this warp's own last claim can be far
                    // behind it, and sizing by that would hand out long runs near the end)
                    const uint32_t at = *reinterpret_cast<volatile uint32_t*>(cursor);
                    const uint32_t left = at < n ? n - at : 0u;
                    r = min(256u, max(32u, (left / (stride / 8u)) & ~31u));  // left / (4 x warps)
                    b = atomicAdd(cursor, r);
                }
                cb = __shfl_sync(0xFFFFFFFFu, b, 0);
                ce = cb + __shfl_sync(0xFFFFFFFFu, r, 0);
            }
            j = cb + lane;
            cb += 32u;
        }
        live = j - lane < n;
        return j;
    }
};

// Adds this warp's node / record counts to two 64-bit counters (every lane of the warp calls it).
__device__ __forceinline__ void warp_add_counts(uint32_t* counters, int word, uint2 c) {
    unsigned long long nodes = c.x, recs = c.y;
    for (int off = 16; off > 0; off >>= 1) {
        nodes += __shfl_down_sync(0xFFFFFFFFu, nodes, off);
        recs += __shfl_down_sync(0xFFFFFFFFu, recs, off);
    }
    if ((threadIdx.x & 31) == 0 && (nodes | recs) != 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(counters + word), nodes);
        atomicAdd(reinterpret_cast<unsigned long long*>(counters + word + 2), recs);
    }
}

struct Wave {
    uint32_t p0;       // first pixel
    uint32_t npaths;   // paths in this wave
    uint32_t spp;
    uint32_t sample_offset;
    uint32_t width;
    uint32_t max_depth;
    uint32_t use_nee, use_mis;
    uint64_t seed;
    // radiance cache (cache_on = 0: the plain path tracer)
    uint32_t cache_on = 0;
    uint32_t term_depth = 0;    // first depth at which a path may end into the cache
    uint32_t train_suffix = 0;  // > 0: training paths end into the cache at term_depth + this
    uint32_t train_thresh = 0;  // a path is a training path if its hash is below this
    float film_weight = 0.0f;   // > 0: film_mean += weight * mean (frames averaged), else film_mean = mean
};

struct Paths {
    float4* ray;      // 2 per path: (origin, -), (direction, -)
    float4* thr;      // throughput rgb, w: 1 if the last bounce was a delta bounce
    float4* rad;      // radiance rgb
    uint2* hit;       // primitive id, t bits
    uint32_t* q0;
    uint32_t* q1;
    uint32_t* classq; // kNumClasses x cap
    float4* shadow;   // 3 per shadow ray: (origin, tmax), (direction, path index bits), (contribution, -)
    uint32_t* counters;
    uint32_t cap;
    uint32_t shadow_cap;
    uint32_t fetch = 0;  // 1: the extension, shading and shadow stages hand out long queues by claims
    // radiance cache
    float4* q_rec = nullptr;   // 4 per query (rbr_cache_record)
    float4* q_info = nullptr;  // per query: throughput rgb, path index bits
    void* q_sort = nullptr;    // scratch of the queries' spatial sort (host side only)
    float4* t_rec = nullptr;   // 4 per training vertex
    float4* t_aux = nullptr;   // 2 per training vertex: (throughput rgb, path index bits), (radiance before, -)
    uint32_t t_cap = 0;
    // packed waves (several requests in one wave; see SegDev)
    const SegDev* segs = nullptr;
    uint32_t* seg_of = nullptr;        // segment of each path (written by k_raygen<true>)
    const uint32_t* wave_hdr = nullptr;  // [0] paths in the wave, [1] segments
};

// Which request a path belongs to, and its random-number key and integrator parameters.
struct PathKey {
    uint32_t pixel, sample, max_depth;
    uint64_t seed;
    bool nee, mis;
};

template <bool kPacked>
__device__ __forceinline__ PathKey path_key(const Wave& w, const Paths& P, uint32_t k) {
    PathKey r;
    if (kPacked) {
        const SegDev& g = P.segs[P.seg_of[k]];
        const uint32_t local = k - g.path0;
        r.pixel = g.p0 + local / g.spp;
        r.sample = g.sample_offset + local % g.spp;
        r.seed = g.seed;
        r.max_depth = g.max_depth;
        r.nee = g.use_nee != 0;
        r.mis = g.use_mis != 0;
    } else {
        r.pixel = w.p0 + k / w.spp;
        r.sample = w.sample_offset + k % w.spp;
        r.seed = w.seed;
        r.max_depth = w.max_depth;
        r.nee = w.use_nee != 0;
        r.mis = w.use_mis != 0;
    }
    return r;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Warp-aggregated append: every lane with `pred` gets a distinct slot of `queue`; one atomic
// per warp (ballot + prefix count of the lanes below).
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool pred) {
    const uint32_t mask = __ballot_sync(0xFFFFFFFFu, pred);
    if (mask == 0) return 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    return pred ? base + __popc(mask & lanemask_lt()) : 0xFFFFFFFFu;
}

__device__ __forceinline__ f3 ld_f3(float4 v) { return mk(v.x, v.y, v.z); }

// Origin (o.xyz) or direction (d.xyz) not finite, or a zero direction.
__device__ __forceinline__ bool degenerate(float4 o, float4 d) {
    const float big = 3.402823466e38f;
    const bool finite = fabsf(o.x) <= big && fabsf(o.y) <= big && fabsf(o.z) <= big && fabsf(d.x) <= big &&
                        fabsf(d.y) <= big && fabsf(d.z) <= big;
    return !finite || (d.x == 0.0f && d.y == 0.0f && d.z == 0.0f);
}

// ------------------------------------------------------------------------------------------
template <bool kPacked>
__device__ __forceinline__ void raygen_body(const CameraDev& cam, const Wave& w, const Paths& P, Span g) {
    const uint32_t n = kPacked ? P.wave_hdr[0] : w.npaths;
    const uint32_t stride = g.blocks * blockDim.x;
    for (uint32_t k = g.block * blockDim.x + threadIdx.x; k < n; k += stride) {
        uint32_t width = w.width, seg = 0;
        if (kPacked) {  // the segment holding path k (segments are sorted by first path)
            uint32_t hi = P.wave_hdr[1] - 1;
            while (seg < hi) {
                const uint32_t mid = (seg + hi + 1) >> 1;
                if (P.segs[mid].path0 <= k) seg = mid;
                else hi = mid - 1;
            }
            P.seg_of[k] = seg;
            width = P.segs[seg].width;
        }
        const PathKey key = path_key<kPacked>(w, P, k);
        const uint32_t x = key.pixel % width, y = key.pixel / width;
        const float4 u = draw4(key.seed, key.pixel, key.sample, 0u, kRngCamera);
        f3 o, d;
        if (kPacked)
            camera_ray(P.segs[seg].cam, fa(static_cast<float>(x), u.x), fa(static_cast<float>(y), u.y), u.z, u.w, o, d);
        else
            camera_ray(cam, fa(static_cast<float>(x), u.x), fa(static_cast<float>(y), u.y), u.z, u.w, o, d);
        P.ray[2 * k] = make_float4(o.x, o.y, o.z, 0.0f);
        P.ray[2 * k + 1] = make_float4(d.x, d.y, d.z, 0.0f);
        P.thr[k] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);  // specularBounce starts true
        P.rad[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        P.q0[k] = k;
    }
    if (g.block == 0 && threadIdx.x == 0) {
        P.counters[kCQ0] = n;
        if (w.cache_on) {
            P.counters[kCQuery] = 0;
            P.counters[kCTrainBase] = P.counters[kCTrain];
        }
    }
}

template <bool kPacked>
__global__ void __launch_bounds__(kBlock) k_raygen(CameraDev cam, Wave w, Paths P) {
    raygen_body<kPacked>(cam, w, P, grid_span());
}

// Resets the counters depth `d` appends to.
__device__ __forceinline__ void begin_body(const Paths& P, uint32_t d) {
    uint32_t* c = P.counters;
    c[kCQ0 + ((d + 1) & 1)] = 0;
    for (int i = 0; i < kNumClasses; ++i) c[kCClass + i] = 0;
    c[kCShadow] = 0;
    for (int i = 0; i < 3; ++i) c[kCCursor + i] = 0;
}

__global__ void k_begin(Paths P, uint32_t d) {
    begin_body(P, d);
}

// Closest hit for the active queue; misses add the background, hits are appended to their
// material-class queue. kVol (VolumetricPathIntegrator::Li, volumetric_path_integrator.cpp:
// 11-43): a distance is sampled in the scene's medium up to the hit (or infinity) and the
// throughput multiplied by the medium weight; a scattering event is handled here: next-event
// estimation towards point lights (directLightingVolume, :92-118) and a phase-function sample
// that continues the path from the scatter point.
// Register budget for 8 resident blocks per SM (64 registers): the volumetric variant, which
// also samples the medium and traces point-light shadow rays from scatter points, gains 5 % over
// the natural 56-register allocation (foggy Cornell box); the surface variant is unchanged.
// kCount (RBR_RENDER_COUNT_TRAFFIC): also counts the nodes and records the traversals fetch.
template <bool kVol, bool kPacked, bool kCount>
__device__ __forceinline__ void extend_body(const DeviceScene& s, const Wave& w, const Paths& P, uint32_t d, int* err, Span g) {
    const uint32_t n = P.counters[kCQ0 + (d & 1)];
    const uint32_t* q = (d & 1) ? P.q1 : P.q0;
    uint32_t* nextq = (d & 1) ? P.q0 : P.q1;
    uint32_t* nextc = P.counters + kCQ0 + ((d + 1) & 1);
    if (g.block == 0 && threadIdx.x == 0) atomicAdd(reinterpret_cast<unsigned long long*>(P.counters + kCExt), n);
    uint2 traffic = make_uint2(0u, 0u);
    Claim cl(P.fetch ? P.counters + kCCursor : nullptr, n, g);
    for (uint32_t j = cl.take(); cl.live; j = cl.take()) {
        const bool valid = j < n;
        uint32_t k = 0, cls = kNumClasses;
        bool scatter = false, last = true, nee = false;
        f3 T = mk(0.0f, 0.0f, 0.0f), sp = T, rd = T;
        float4 u = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (valid) {
            k = q[j];
            const float4 a = P.ray[2 * k], b = P.ray[2 * k + 1];
            float t = 0.0f;
            // A ray with a zero or non-finite direction or origin: no traversal, no hit.
            const uint32_t prim = degenerate(a, b) ? 0xFFFFFFFFu
                                                   : traverse<false, kCount>(s, ld_f3(a), ld_f3(b), __int_as_float(0x7f800000),
                                                                             t, err, &traffic);
            P.hit[k] = make_uint2(prim, __float_as_uint(t));
            if (kVol && s.has_medium) {
                const float4 T4 = P.thr[k];
                T = ld_f3(T4);
                const PathKey key = path_key<kPacked>(w, P, k);
                last = d + 1 >= key.max_depth;
                nee = key.nee;
                u = draw4(key.seed, key.pixel, key.sample, d, kRngMedium);
                float ts = 0.0f;
                f3 wgt;
                scatter = medium_sample(s, prim == 0xFFFFFFFFu ? __int_as_float(0x7f800000) : t, u.x, ts, wgt);
                T = xmul(T, wgt);
                P.thr[k] = make_float4(T.x, T.y, T.z, T4.w);
                if (scatter) {
                    rd = ld_f3(b);
                    sp = xadd(ld_f3(a), xmuls(rd, ts));  // Ray::at
                }
            }
            if (!scatter) {
                if (prim == 0xFFFFFFFFu) {
                    if (!(kVol && s.has_medium)) T = ld_f3(P.thr[k]);
                    float4 L = P.rad[k];
                    L.x = fa(L.x, fm(T.x, s.background[0]));
                    L.y = fa(L.y, fm(T.y, s.background[1]));
                    L.z = fa(L.z, fm(T.z, s.background[2]));
                    P.rad[k] = L;
                } else {
                    cls = s.materials[s.prim_material[prim]].cls;
                }
            }
        }
        {
            // append to the class queue: lanes of one class share an atomic (match.any), one
            // per class present in the warp; kNumClasses marks a lane with nothing to shade
            const uint32_t peers = __match_any_sync(0xFFFFFFFFu, cls);
            const int leader = __ffs(peers) - 1;
            uint32_t first = 0;
            if (cls < kNumClasses && static_cast<int>(threadIdx.x & 31) == leader)
                first = atomicAdd(P.counters + kCClass + cls, __popc(peers));
            first = __shfl_sync(0xFFFFFFFFu, first, leader);
            if (cls < kNumClasses) P.classq[cls * P.cap + first + __popc(peers & lanemask_lt())] = k;
        }
        if (kVol) {
            // next-event estimation from the scatter point: point lights only, unoccluded
            // segment of length dist, Li * Tr(dist) * phase(wo = ray direction, wi)
            for (uint32_t l = 0; l < s.num_lights; ++l) {
                bool emit = false;
                f3 contrib, sd;
                float dist = 0.0f;
                if (scatter && nee && s.lights[l].type == RBR_LIGHT_POINT) {
                    const LightDev& L = s.lights[l];
                    const f3 toL = xsub(ld3(L.position), sp);
                    dist = xlen(toL);
                    const f3 wi = xdivs(toL, dist);
                    sd = xnorm(wi);  // the shadow Ray's constructor normalises
                    const f3 Li = xdivs(xmuls(ld3(L.color), L.intensity), fm(dist, dist));
                    const float ph = hg_eval(s.hg_g, rd, wi);
                    contrib = xmul(T, xmuls(xmul(Li, transmittance(s, dist)), ph));
                    emit = true;
                }
                const uint32_t slot = warp_append(P.counters + kCShadow, emit);
                if (emit && slot < P.shadow_cap) {
                    float4* e = P.shadow + 3 * static_cast<size_t>(slot);
                    e[0] = make_float4(sp.x, sp.y, sp.z, dist);
                    e[1] = make_float4(sd.x, sd.y, sd.z, __uint_as_float(k));
                    e[2] = make_float4(contrib.x, contrib.y, contrib.z, 0.0f);
                }
            }
            // the path continues from the scatter point in a phase-function direction
            const bool cont = scatter && !last;
            if (cont) {
                const f3 nd = xnorm(hg_sample(s.hg_g, rd, u.y, u.z));
                P.ray[2 * k] = make_float4(sp.x, sp.y, sp.z, 0.0f);
                P.ray[2 * k + 1] = make_float4(nd.x, nd.y, nd.z, 0.0f);
            }
            const uint32_t slot = warp_append(nextc, cont);
            if (cont) nextq[slot] = k;
        }
    }
    if (kCount) warp_add_counts(P.counters, kCTraffic, traffic);
}

template <bool kVol, bool kPacked, bool kCount = false>
__global__ void __launch_bounds__(kBlock, 8) k_extend(DeviceScene s, Wave w, Paths P, uint32_t d, int* err) {
    extend_body<kVol, kPacked, kCount>(s, w, P, d, err, grid_span());
}

// Surface data of a hit, as the primitive's intersect() fills SurfaceInteraction. The normal
// that faces the incoming ray (setFaceNormal) is the outward normal or its negation, kept as a
// flag (face_normal) so that a shading thread holds three floats fewer.
struct Hit {
    f3 point;
    f3 outward;  // outwardNormal()
    bool front;  // the ray arrived on the outward side
};
__device__ __forceinline__ f3 face_normal(const Hit& h) { return h.front ? h.outward : xneg(h.outward); }

__device__ __forceinline__ Hit surface(const DeviceScene& s, uint32_t prim, float t, f3 o, f3 d) {
    Hit h;
    h.point = xadd(o, xmuls(d, t));  // Ray::at
    const uint32_t rec = s.prim_record[prim];
    f3 outward;
    if (rec & 0x80000000u) {  // plane
        const float4 pl = s.planes[rec & 0x7FFFFFFFu];
        outward = mk(pl.x, pl.y, pl.z);
    } else {
        const float4 a = s.records[3 * rec], b = s.records[3 * rec + 1], c = s.records[3 * rec + 2];
        const uint32_t type = __float_as_uint(c.y) >> kTypeShift;
        if (type == kPrimTriangle) {
            const f3 v0 = mk(a.x, a.y, a.z), e1 = mk(a.w, b.x, b.y), e2 = mk(b.z, b.w, c.x);
            const f3 geo = xnorm(xcross(e1, e2));
            outward = geo;
            if (s.tri_normals) {  // interpolated shading normal (triangle.cpp:40-46)
                float u = 0.0f, v = 0.0f;
                hit_triangle(o, d, v0, e1, e2, __int_as_float(0x7f800000), &u, &v);
                const float wb = fs(fs(1.0f, u), v);
                const float4 n0 = s.tri_normals[3 * rec], n1 = s.tri_normals[3 * rec + 1], n2 = s.tri_normals[3 * rec + 2];
                f3 n = xnorm(xadd(xadd(xmuls(ld_f3(n0), wb), xmuls(ld_f3(n1), u)), xmuls(ld_f3(n2), v)));
                if (xdot(n, geo) < 0.0f) n = xneg(n);
                outward = n;
            }
        } else if (type == kPrimSphere) {
            outward = xdivs(xsub(h.point, mk(a.x, a.y, a.z)), a.w);  // (hitPoint - center) / radius
        } else {
            outward = xnorm(xcross(mk(a.w, b.x, b.y), mk(b.z, b.w, c.x)));  // quad normal
        }
    }
    h.front = xdot(d, outward) < 0.0f;
    h.outward = outward;
    return h;
}

// Interaction::spawnRay (interaction.h:22-29); the Ray constructor normalises the direction.
__device__ __forceinline__ void spawn(const Hit& h, f3 dir, f3& o, f3& d) {
    const f3 n = face_normal(h);
    f3 off = xmuls(n, kEpsilon);
    if (xdot(dir, n) < 0.0f) off = xneg(off);
    o = xadd(h.point, off);
    d = xnorm(dir);
}

// Radiance-cache record of a vertex: position, direction towards the viewer, ray-facing
// normal, roughness, diffuse albedo base (1-metallic)(1-transmission), specular albedo
// base*metallic + 0.04 (1-metallic).
__device__ __forceinline__ void cache_record(const Hit& h, f3 rd, const MaterialDev& m, float4* rec) {
    const float met = oclamp(m.metallic, 0.0f, 1.0f), tr = oclamp(m.transmission, 0.0f, 1.0f);
    const float kd = fm(fs(1.0f, met), fs(1.0f, tr));
    const float k4 = fm(0.04f, fs(1.0f, met));
    rec[0] = make_float4(h.point.x, h.point.y, h.point.z, -rd.x);
    const f3 n = face_normal(h);
    rec[1] = make_float4(-rd.y, -rd.z, n.x, n.y);
    rec[2] = make_float4(n.z, m.roughness, fm(m.base[0], kd), fm(m.base[1], kd));
    rec[3] = make_float4(fm(m.base[2], kd), fa(fm(m.base[0], met), k4), fa(fm(m.base[1], met), k4),
                         fa(fm(m.base[2], met), k4));
}

// Training paths of the radiance cache: a hash of (pixel, sample, seed) below the threshold.
__device__ __forceinline__ bool train_path(const Wave& w, uint64_t seed, uint32_t pixel, uint32_t sample) {
    uint32_t x = (pixel * 0x9E3779B1u) ^ ((sample + 0x7F4A7C15u) * 0x85EBCA77u) ^ static_cast<uint32_t>(seed);
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return x < w.train_thresh;
}

// Surface vertices, per material-class queue. kMode 0: PathTracingIntegrator::Li; 1: the same
// with the radiance cache; 2: the surface part of VolumetricPathIntegrator::Li
// (volumetric_path_integrator.cpp:45-88: emission at every hit, NEE without MIS weights).
// Register budget for 8 resident blocks per SM (64 registers, a few spills): the kernel is
// latency-bound on its division and square-root chains, and twice the warps of its natural
// 124-register allocation hide more of it (GGX scene +5 %, Cornell box +3 %; 5, 6, 10 and 12
// blocks were measured slower).
// kCls < 0: one launch over the six class queues; kCls = a material class: that class's
// queue only, with the lobe kinds of the class known at compile time (no microfacet code for
// the diffuse and delta-only classes, no next-event estimation for delta-only and lobeless
// materials, whose light samples always evaluate to zero).
constexpr int kShadeDiffuse = static_cast<int>(kClassDiffuse), kShadeGlossy = static_cast<int>(kClassGlossy),
              kShadeSpecular = static_cast<int>(kClassSpecular), kShadeNone = static_cast<int>(kClassNone),
              kShadeGlossyRefl = static_cast<int>(kClassGlossyRefl),
              kShadeGlossyTrans = static_cast<int>(kClassGlossyTrans);
constexpr uint32_t kGGXReflKinds = (1u << kCondGGX) | (1u << kDielGGX);
template <int kCls>
__host__ __device__ constexpr uint32_t class_kinds() {
    return kCls == kShadeDiffuse       ? kNoGGXKinds
           : kCls == kShadeSpecular    ? kDeltaKinds
           : kCls == kShadeNone        ? 0u
           : kCls == kShadeGlossy      ? kGGXReflKinds | (1u << kLambert)
           : kCls == kShadeGlossyRefl  ? kGGXReflKinds
           : kCls == kShadeGlossyTrans ? kGGXReflKinds | (1u << kTransGGX) | (1u << kLambert)
                                       : kAllKinds;
}

template <int kMode, bool kPacked, int kCls>
__device__ __forceinline__ void shade_body(const DeviceScene& s, const Wave& w, const Paths& P, uint32_t d, Span g) {
    constexpr bool kCache = kMode == 1, kVolSurface = kMode == 2;
    constexpr uint32_t kKinds = class_kinds<kCls>();
    constexpr bool kNoNee = kCls == kShadeSpecular || kCls == kShadeNone;
    uint32_t cnt[kNumClasses + 1];
    cnt[0] = 0;
    if (kCls < 0)
        for (int c = 0; c < kNumClasses; ++c) cnt[c + 1] = cnt[c] + P.counters[kCClass + c];
    const uint32_t n = kCls < 0 ? cnt[kNumClasses] : P.counters[kCClass + (kCls < 0 ? 0 : kCls)];
    uint32_t* nextq = (d & 1) ? P.q0 : P.q1;
    uint32_t* nextc = P.counters + kCQ0 + ((d + 1) & 1);
    if (g.block == 0 && threadIdx.x == 0) atomicAdd(reinterpret_cast<unsigned long long*>(P.counters + kCShade), n);
    // one cursor per depth: the per-class launches keep the grid-stride order
    Claim cl(P.fetch && kCls < 0 ? P.counters + kCCursor + 1 : nullptr, n, g);
    for (uint32_t j = cl.take(); cl.live; j = cl.take()) {
        const bool valid = j < n;
        uint32_t k = 0;
        bool alive = false, nee = false, to_cache = false, to_train = false, last = true, mis = false;
        uint64_t seed = 0;
        float4 rec[4];
        Hit h;
        f3 T = mk(0.0f, 0.0f, 0.0f), wo = mk(0.0f, 0.0f, 0.0f);
        Bsdf bs;
        bs.n = 0;
        Mix mx;
        mx.total = 0.0f;
        uint32_t pixel = 0, sample = 0;
        if (valid) {
            if (kCls < 0) {
                int c = 0;
                while (j >= cnt[c + 1]) ++c;
                k = P.classq[c * P.cap + (j - cnt[c])];
            } else {
                k = P.classq[static_cast<uint32_t>(kCls < 0 ? 0 : kCls) * P.cap + j];
            }
            const PathKey key = path_key<kPacked>(w, P, k);
            pixel = key.pixel;
            sample = key.sample;
            seed = key.seed;
            last = d + 1 >= key.max_depth;
            mis = key.mis;
            const uint2 hv = P.hit[k];
            const f3 ro = ld_f3(P.ray[2 * k]), rd = ld_f3(P.ray[2 * k + 1]);
            const float4 t4 = P.thr[k];
            T = mk(t4.x, t4.y, t4.z);
            const bool specular = t4.w != 0.0f;
            h = surface(s, hv.x, __uint_as_float(hv.y), ro, rd);
            const MaterialDev& m = s.materials[s.prim_material[hv.x]];
            if (m.emissive && (kVolSurface || d == 0 || specular)) {
                float4 L = P.rad[k];
                L.x = fa(L.x, fm(T.x, m.emission[0]));
                L.y = fa(L.y, fm(T.y, m.emission[1]));
                L.z = fa(L.z, fm(T.z, m.emission[2]));
                P.rad[k] = L;
            }
            bs = make_bsdf(m);
            wo = to_local(make_frame(h.outward), xneg(rd));  // isect.wo = -ray.direction
            mx = mixture(bs, wo);
            nee = !kNoNee && key.nee && !bsdf_delta(bs);
            alive = true;
            if (kCache && bs.n > 0 && !bsdf_delta(bs)) {
                if (train_path(w, seed, pixel, sample)) {
                    if (w.train_suffix != 0 && d >= w.term_depth + w.train_suffix && !specular) {
                        to_cache = true;  // self-training: the suffix ends in the cache's prediction
                        nee = false;
                        alive = false;
                    } else {
                        to_train = true;
                    }
                } else if (d >= w.term_depth && !specular) {
                    to_cache = true;  // the cache's prediction replaces NEE and everything further
                    nee = false;
                    alive = false;
                }
                if (to_train || to_cache) cache_record(h, rd, m, rec);
            }
        }
        if (kCache) {
            const uint32_t qs = warp_append(P.counters + kCQuery, to_cache);
            if (to_cache) {
                float4* q = P.q_rec + 4 * static_cast<size_t>(qs);
                q[0] = rec[0];
                q[1] = rec[1];
                q[2] = rec[2];
                q[3] = rec[3];
                P.q_info[qs] = make_float4(T.x, T.y, T.z, __uint_as_float(k));
            }
            const uint32_t ts = warp_append(P.counters + kCTrain, to_train);
            if (to_train && ts < P.t_cap) {
                float4* q = P.t_rec + 4 * static_cast<size_t>(ts);
                q[0] = rec[0];
                q[1] = rec[1];
                q[2] = rec[2];
                q[3] = rec[3];
                P.t_aux[2 * static_cast<size_t>(ts)] = make_float4(T.x, T.y, T.z, __uint_as_float(k));
                P.t_aux[2 * static_cast<size_t>(ts) + 1] = P.rad[k];  // radiance gathered before this vertex's NEE
            }
        }
        // next-event estimation: one shadow ray per light (estimateDirectLighting)
        for (uint32_t l = 0; l < s.num_lights; ++l) {
            bool emit = false;
            f3 contrib, wi;
            float stmax = 0.0f;
            if (!kNoNee && valid && nee) {
                const float4 u = draw4(seed, pixel, sample, d, kRngLights + ((l >> 1) << 8));
                const LightDev& L = s.lights[l];
                const LSample ls = light_sample(L, h.point, (l & 1) ? u.z : u.x, (l & 1) ? u.w : u.y);
                if (ls.pdf > 0.0f && !black(ls.Li)) {
                    // the shading frame is rebuilt from the outward normal where it is needed
                    // (the same bits each time) instead of being held across the loop
                    const f3 wiL = to_local(make_frame(h.outward), ls.wi);
                    f3 f;
                    float bpdf;
                    bsdf_eval_pdf<kKinds>(bs, mx, wo, wiL, f, bpdf);
                    if (!black(f)) {
                        wi = ls.wi;
                        stmax = fs(ls.dist, kEpsilon);
                        // |wi . n| of the face normal: negating n negates every product exactly
                        const float c = fabsf(xdot(ls.wi, h.outward));
                        f3 ld;
                        if (!kVolSurface && mis && !ls.delta) {
                            const float wgt = power_heuristic(ls.pdf, bpdf);
                            ld = xdivs(xmuls(xmuls(xmul(f, ls.Li), c), wgt), ls.pdf);
                        } else {
                            ld = xdivs(xmuls(xmul(f, ls.Li), c), ls.pdf);
                        }
                        contrib = xmul(T, ld);
                        emit = true;
                    }
                }
            }
            const uint32_t slot = warp_append(P.counters + kCShadow, emit);
            if (emit && slot < P.shadow_cap) {
                f3 so, sd;
                spawn(h, wi, so, sd);  // after the append: fewer values live across it
                float4* e = P.shadow + 3 * static_cast<size_t>(slot);
                e[0] = make_float4(so.x, so.y, so.z, stmax);
                e[1] = make_float4(sd.x, sd.y, sd.z, __uint_as_float(k));
                e[2] = make_float4(contrib.x, contrib.y, contrib.z, 0.0f);
            }
        }
        // BSDF sampling, throughput update, Russian roulette, next ray
        bool cont = false;
        if (valid && alive && !last) {
            const float4 u = draw4(seed, pixel, sample, d, kRngBounce);
            const BSample b = bsdf_sample<kKinds>(bs, mx, wo, u.x, u.y);
            if (b.pdf > 0.0f && !black(b.f)) {
                const f3 wiW = to_world(make_frame(h.outward), b.wi);
                const float c = fabsf(xdot(wiW, h.outward));
                T = xmul(T, xmuls(b.f, fd(c, b.pdf)));
                cont = true;
                if (d > 3) {
                    const float q = omax(0.05f, fs(1.0f, maxc(T)));
                    if (u.z < q) cont = false;
                    else T = xdivs(T, fs(1.0f, q));
                }
                if (cont) {
                    f3 no, nd;
                    spawn(h, wiW, no, nd);
                    P.ray[2 * k] = make_float4(no.x, no.y, no.z, 0.0f);
                    P.ray[2 * k + 1] = make_float4(nd.x, nd.y, nd.z, 0.0f);
                    P.thr[k] = make_float4(T.x, T.y, T.z, b.delta ? 1.0f : 0.0f);
                }
            }
        }
        const uint32_t slot = warp_append(nextc, cont);
        if (cont) nextq[slot] = k;
    }
}

// Resident blocks per SM the register budget of a shading kernel allows: the unified kernel and
// the lobeless and delta-only classes 8 (64 registers); the glossy class 6 (80 registers) and
// the diffuse class 7 (72), which keeps their spills small (76 / 68 bytes instead of 232 / 156).
template <int kCls>
__host__ __device__ constexpr int shade_blocks() {
    return kCls == kShadeGlossy || kCls == kShadeGlossyRefl || kCls == kShadeGlossyTrans ? 6 : kCls == kShadeDiffuse ? 7 : 8;
}

template <int kMode, bool kPacked, int kCls = -1>
__global__ void __launch_bounds__(kBlock, shade_blocks<kCls>()) k_shade(DeviceScene s, Wave w, Paths P, uint32_t d) {
    shade_body<kMode, kPacked, kCls>(s, w, P, d, grid_span());
}

template <bool kCount>
__device__ __forceinline__ void shadow_body(const DeviceScene& s, const Paths& P, int* err, Span g) {
    uint32_t n = P.counters[kCShadow];
    if (n > P.shadow_cap) {
        if (g.block == 0 && threadIdx.x == 0) atomicOr(err, kErrQueueOverflow);
        n = P.shadow_cap;
    }
    if (g.block == 0 && threadIdx.x == 0) atomicAdd(reinterpret_cast<unsigned long long*>(P.counters + kCSh), n);
    uint2 traffic = make_uint2(0u, 0u);
    Claim cl(P.fetch ? P.counters + kCCursor + 2 : nullptr, n, g);
    for (uint32_t j = cl.take(); cl.live; j = cl.take()) {
        if (j < n) {  // lanes past the end claim again with their warp
            const float4* e = P.shadow + 3 * static_cast<size_t>(j);
            const float4 a = e[0], b = e[1];
            float t;
            if (!degenerate(a, b) && !traverse<true, kCount>(s, ld_f3(a), ld_f3(b), a.w, t, err, &traffic)) {
                const float4 c = e[2];
                float4* L = P.rad + __float_as_uint(b.w);
                atomicAdd(&L->x, c.x);
                atomicAdd(&L->y, c.y);
                atomicAdd(&L->z, c.z);
            }
        }
    }
    if (kCount) warp_add_counts(P.counters, kCTraffic + 4, traffic);
}

// 8 resident blocks per SM (64 registers), the grid's blocks per SM: with more registers a
// launch would run in two waves of blocks.
template <bool kCount = false>
__global__ void __launch_bounds__(kBlock, 8) k_shadow(DeviceScene s, Paths P, int* err) {
    shadow_body<kCount>(s, P, err, grid_span());
}

__global__ void __launch_bounds__(kBlock) k_film(Wave w, Paths P, float* film_mean, float* film_m2) {
    const uint32_t npix = w.npaths / w.spp;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += stride) {
        f3 sum = mk(0.0f, 0.0f, 0.0f), sq = mk(0.0f, 0.0f, 0.0f);
        for (uint32_t s = 0; s < w.spp; ++s) {
            const f3 L = ld_f3(P.rad[i * w.spp + s]);
            sum = xadd(sum, L);
            sq = xadd(sq, xmul(L, L));
        }
        const f3 mean = xdivs(sum, static_cast<float>(w.spp));  // pixelColor / samplesPerPixel
        float* o = film_mean + 3 * static_cast<size_t>(w.p0 + i);
        float* q = film_m2 ? film_m2 + 3 * static_cast<size_t>(w.p0 + i) : nullptr;
        if (w.film_weight > 0.0f) {  // average over frames
            o[0] = fa(o[0], fm(mean.x, w.film_weight));
            o[1] = fa(o[1], fm(mean.y, w.film_weight));
            o[2] = fa(o[2], fm(mean.z, w.film_weight));
            if (q) {
                q[0] = fa(q[0], sq.x);
                q[1] = fa(q[1], sq.y);
                q[2] = fa(q[2], sq.z);
            }
        } else {
            o[0] = mean.x;
            o[1] = mean.y;
            o[2] = mean.z;
            if (q) {
                q[0] = sq.x;
                q[1] = sq.y;
                q[2] = sq.z;
            }
        }
    }
}

// Film of a packed wave: the first path of each pixel sums the pixel's samples into its
// request's film.
__device__ __forceinline__ void film_packed_body(const Paths& P, Span g) {
    const uint32_t n = P.wave_hdr[0];
    const uint32_t stride = g.blocks * blockDim.x;
    for (uint32_t k = g.block * blockDim.x + threadIdx.x; k < n; k += stride) {
        const SegDev& g = P.segs[P.seg_of[k]];
        const uint32_t local = k - g.path0;
        if (local % g.spp != 0) continue;
        f3 sum = mk(0.0f, 0.0f, 0.0f);
        for (uint32_t s = 0; s < g.spp; ++s) sum = xadd(sum, ld_f3(P.rad[k + s]));
        const f3 mean = xdivs(sum, static_cast<float>(g.spp));
        float* o = g.film + 3 * static_cast<size_t>(g.p0 + local / g.spp);
        o[0] = mean.x;
        o[1] = mean.y;
        o[2] = mean.z;
    }
}

__global__ void __launch_bounds__(kBlock) k_film_packed(Paths P) {
    film_packed_body(P, grid_span());
}

// ------------------------------------------------------------------------------------------
// Persistent wave loop: one cooperative launch renders every wave of a batched run. The
// stages of all waves run in the same resident blocks, separated by grid barriers instead of
// kernel boundaries; a wave starts once its release time (the arrival of its last request)
// has passed, and the device clock stamps its end.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Barrier of `nblocks` blocks of a cooperative launch (every block is resident). bar[0] counts
// arrivals, bar[1] is the generation the last arrival advances. A wait longer than limit_ns of
// device time records kErrDeviceTimeout; after that, or when another block recorded it, the
// barrier reports failure and the caller leaves the kernel, so the blocks still waiting give
// up in turn and nothing waits without bound.
__device__ bool grid_barrier(uint32_t* bar, uint32_t& gen, uint32_t nblocks, uint64_t limit_ns, int* err) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        if (atomicAdd(bar, 1u) + 1u == nblocks) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicExch(bar + 1, gen + 1u);
        } else {
            const uint64_t t0 = global_ns();
            while (ld_acquire(bar + 1) == gen) {
                if (global_ns() - t0 > limit_ns || (*reinterpret_cast<volatile int*>(err) & kErrDeviceTimeout)) {
                    ok = 0;
                    atomicOr(err, kErrDeviceTimeout);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok_s = ok;
    }
    __syncthreads();
    ++gen;
    return ok_s != 0;
}

// The stages as separate (not inlined) functions: each keeps the register allocation of its own
// kernel instead of the loop kernel holding all of them at once.
__device__ __noinline__ void loop_raygen(const Paths& P, Span g) {
    const Wave w{};
    const CameraDev unused{};
    raygen_body<true>(unused, w, P, g);
}
template <bool kVol>
__device__ __noinline__ void loop_extend(const DeviceScene& s, const Paths& P, uint32_t d, int* err, Span g) {
    const Wave w{};
    extend_body<kVol, true, false>(s, w, P, d, err, g);
}
template <int kMode>
__device__ __noinline__ void loop_shade(const DeviceScene& s, const Paths& P, uint32_t d, Span g) {
    const Wave w{};
    shade_body<kMode, true, -1>(s, w, P, d, g);
}
__device__ __noinline__ void loop_shadow(const DeviceScene& s, const Paths& P, int* err, Span g) {
    shadow_body<false>(s, P, err, g);
}
__device__ __noinline__ void loop_film(const Paths& P, Span g) { film_packed_body(P, g); }

struct LoopParams {
    DeviceScene scenes[kLoopScenes];
    const LoopWave* waves;
    uint32_t nwaves;
    uint32_t halves;             // 1, or 2: the grid's halves render alternate waves
    const char* tables;          // segment tables, at LoopWave::table
    Paths P[2];                  // path buffers of each half (segments and header set per wave)
    unsigned long long* stamps;  // [0] start of the run, [1 + w] end of wave w (device ns)
    uint32_t* bar;               // per half [2h] arrivals, [2h + 1] generation; [4], [5] whole grid
    int* err;
    uint64_t limit_ns;           // longest wait at a barrier
};

// With two halves, blocks [0, G/2) render the even waves on the first path-buffer set and
// blocks [G/2, G) the odd waves on the second, each half with its own barrier, so that one
// half's latency-bound last bounces run beside the other half's full stages (what two waves in
// flight on two streams give the graph-replayed path).
__global__ void __launch_bounds__(kBlock, 8) k_wave_loop(const __grid_constant__ LoopParams p) {
    uint32_t gen0 = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) p.stamps[0] = global_ns();
    if (!grid_barrier(p.bar + 4, gen0, gridDim.x, p.limit_ns, p.err)) return;
    const uint64_t t0 = *reinterpret_cast<volatile unsigned long long*>(p.stamps);
    const uint32_t per = gridDim.x / p.halves;
    const uint32_t h = min(blockIdx.x / per, p.halves - 1);
    const Span g{blockIdx.x - h * per, per};
    uint32_t* bar = p.bar + 2 * h;
    uint32_t gen = 0;
    for (uint32_t wi = h; wi < p.nwaves; wi += p.halves) {
        const LoopWave lw = p.waves[wi];
        // admission: the wave's last request arrives release_ns after the run's start (the host
        // bounds release_ns, so this wait ends)
        while (global_ns() - t0 < lw.release_ns) __nanosleep(2048);
        Paths P = p.P[h];
        P.wave_hdr = reinterpret_cast<const uint32_t*>(p.tables + lw.table);
        P.segs = reinterpret_cast<const SegDev*>(p.tables + lw.table + kSegTableHeader);
        const DeviceScene& s = p.scenes[lw.scene];
        if (g.block == 0)
            for (uint32_t i = threadIdx.x; i < kCWords; i += blockDim.x) P.counters[i] = 0;
        if (!grid_barrier(bar, gen, per, p.limit_ns, p.err)) return;
        loop_raygen(P, g);
        if (!grid_barrier(bar, gen, per, p.limit_ns, p.err)) return;
        for (uint32_t d = 0; d < lw.max_depth; ++d) {
            if (g.block == 0 && threadIdx.x == 0) begin_body(P, d);
            if (!grid_barrier(bar, gen, per, p.limit_ns, p.err)) return;
            if (lw.mode == 2) loop_extend<true>(s, P, d, p.err, g);
            else loop_extend<false>(s, P, d, p.err, g);
            if (!grid_barrier(bar, gen, per, p.limit_ns, p.err)) return;
            if (lw.mode == 2) loop_shade<2>(s, P, d, g);
            else loop_shade<0>(s, P, d, g);
            if (!grid_barrier(bar, gen, per, p.limit_ns, p.err)) return;
            loop_shadow(s, P, p.err, g);
            if (!grid_barrier(bar, gen, per, p.limit_ns, p.err)) return;
        }
        loop_film(P, g);
        if (!grid_barrier(bar, gen, per, p.limit_ns, p.err)) return;
        if (g.block == 0 && threadIdx.x == 0) p.stamps[1 + wi] = global_ns();
    }
}

// Device clock stamps and admission for the graph-replayed waves of a batched run.
__global__ void k_stamp(unsigned long long* at) { *at = global_ns(); }
__global__ void k_release(const unsigned long long* start, uint64_t release_ns) {
    const uint64_t t0 = *start;
    while (global_ns() - t0 < release_ns) __nanosleep(2048);
}

}  // namespace

rbr_status read_render_counters(rbr_ctx* ctx) {
    if (!ctx->pt.counters.ptr) return RBR_OK;
    rbr_render_stats& r = ctx->last_render;
    r.extension_rays = r.shadow_rays = r.shaded_vertices = 0;
    r.ext_nodes = r.ext_records = r.shadow_nodes = r.shadow_records = 0;
    for (int b = 0; b < (ctx->pt_last_two ? 2 : 1); ++b) {
        const PathBuffers& pb = b ? ctx->pt2 : ctx->pt;
        uint32_t h[kCWords];
        const cudaError_t e = cudaMemcpy(h, pb.counters.ptr, sizeof(h), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "reading the render counters");
        auto u64 = [&](int word) { return uint64_t(h[word]) | (uint64_t(h[word + 1]) << 32); };
        r.extension_rays += u64(kCExt);
        r.shadow_rays += u64(kCSh);
        r.shaded_vertices += u64(kCShade);
        r.ext_nodes += u64(kCTraffic);
        r.ext_records += u64(kCTraffic + 2);
        r.shadow_nodes += u64(kCTraffic + 4);
        r.shadow_records += u64(kCTraffic + 6);
    }
    return RBR_OK;
}

static void free_paths(PathBuffers& p) {
    release(p.ray);
    release(p.thr);
    release(p.rad);
    release(p.hit);
    release(p.queue[0]);
    release(p.queue[1]);
    release(p.classq);
    release(p.shadow);
    release(p.counters);
    p.capacity = 0;
    p.shadow_capacity = 0;
}

void free_path_buffers(rbr_ctx* ctx) {
    free_paths(ctx->pt);
    free_paths(ctx->pt2);
    release(ctx->pt_seg_of);
    release(ctx->pt_seg_of2);
    ctx->pt_last_two = false;
    ++ctx->pt_generation;
}

static rbr_status ensure_paths(rbr_ctx* ctx, uint32_t cap, uint32_t shadow_cap, PathBuffers* which = nullptr) {
    PathBuffers& p = which ? *which : ctx->pt;
    if (p.capacity >= cap && p.shadow_capacity >= shadow_cap && p.counters.ptr) return RBR_OK;
    free_paths(p);
    ++ctx->pt_generation;
    rbr_status st;
    if ((st = ensure(ctx, p.ray, size_t(cap) * 32, "path rays")) != RBR_OK ||
        (st = ensure(ctx, p.thr, size_t(cap) * 16, "path throughput")) != RBR_OK ||
        (st = ensure(ctx, p.rad, size_t(cap) * 16, "path radiance")) != RBR_OK ||
        (st = ensure(ctx, p.hit, size_t(cap) * 8, "path hits")) != RBR_OK ||
        (st = ensure(ctx, p.queue[0], size_t(cap) * 4, "active queue")) != RBR_OK ||
        (st = ensure(ctx, p.queue[1], size_t(cap) * 4, "active queue")) != RBR_OK ||
        (st = ensure(ctx, p.classq, size_t(cap) * 4 * kNumClasses, "class queues")) != RBR_OK ||
        (st = ensure(ctx, p.shadow, size_t(std::max(1u, shadow_cap)) * 48, "shadow queue")) != RBR_OK ||
        (st = ensure(ctx, p.counters, kCWords * 4, "queue counters")) != RBR_OK) {
        free_paths(p);
        return st;
    }
    p.capacity = cap;
    p.shadow_capacity = shadow_cap;
    return RBR_OK;
}

rbr_status render(rbr_ctx* ctx, const rbr_camera* cam, const rbr_render_params* p, float* film_mean, float* film_m2,
                  cudaStream_t stream) {
    if (!cam || !p || !film_mean) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "camera, params or film_mean is NULL");
    if (!ctx->has_scene) return fail(ctx, RBR_ERR_NO_SCENE, "rbr_render before rbr_scene_upload");
    if (cam->width <= 0 || cam->height <= 0 || p->samples_per_pixel <= 0 || p->max_depth < 0)
        return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "image size, samples per pixel or max depth out of range");
    if (cam->model != RBR_CAMERA_PINHOLE && cam->model != RBR_CAMERA_THIN_LENS)
        return fail(ctx, RBR_ERR_UNSUPPORTED, "camera model " + std::to_string(cam->model));
    if (p->flags & RBR_RENDER_CORRECTED_MIS)
        return fail(ctx, RBR_ERR_UNSUPPORTED, "RBR_RENDER_CORRECTED_MIS is not implemented");
    if ((p->flags & RBR_RENDER_SECOND_MOMENT) == 0) film_m2 = nullptr;
    const bool volumetric = (p->flags & RBR_RENDER_VOLUMETRIC) != 0;
    const bool count = (p->flags & RBR_RENDER_COUNT_TRAFFIC) != 0;
    const uint64_t npix = uint64_t(cam->width) * cam->height;
    const uint32_t spp = static_cast<uint32_t>(p->samples_per_pixel);
    if (npix * spp > 0xFFFFFFFFull || spp > kDefaultCapacity)
        return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "more than 2^32 camera samples in one render call");
    const uint32_t nl = std::max(1u, ctx->scene.num_lights);
    uint32_t cap = static_cast<uint32_t>(std::min<uint64_t>(npix * spp, std::max(ctx->pt_wave_paths, spp)));
    cap = std::min<uint64_t>(cap, kShadowBytesLimit / (48ull * nl));
    cap = std::max(spp, cap / spp * spp);
    // Two waves in flight (a second path-buffer set on a second stream): the latency-bound
    // launches at the end of one wave's bounces, which occupy few SMs, run beside the full
    // launches of the next wave. An image that fits one wave is split into two halves. When
    // the second set cannot be allocated, the waves run one at a time in the first.
    bool two = ctx->pt_streams == 2 && npix >= 2;
    if (two && npix * spp <= cap) cap = static_cast<uint32_t>((npix + 1) / 2) * spp;
    rbr_status st = ensure_paths(ctx, cap, cap * nl);
    if (st != RBR_OK) return st;
    if (two) {
        st = ensure_paths(ctx, cap, cap * nl, &ctx->pt2);  // frees what it allocated on failure
        if (st == RBR_ERR_OUT_OF_MEMORY) {
            two = false;
            st = RBR_OK;
        } else if (st == RBR_OK) {
            st = ensure_side_stream(ctx);
        }
        if (st != RBR_OK) return st;
    }
    ctx->pt_last_two = two;
    Paths PP[2];
    for (int b = 0; b < (two ? 2 : 1); ++b) {
        PathBuffers& pb = b ? ctx->pt2 : ctx->pt;
        Paths& P = PP[b];
        P.ray = static_cast<float4*>(pb.ray.ptr);
        P.thr = static_cast<float4*>(pb.thr.ptr);
        P.rad = static_cast<float4*>(pb.rad.ptr);
        P.hit = static_cast<uint2*>(pb.hit.ptr);
        P.q0 = static_cast<uint32_t*>(pb.queue[0].ptr);
        P.q1 = static_cast<uint32_t*>(pb.queue[1].ptr);
        P.classq = static_cast<uint32_t*>(pb.classq.ptr);
        P.shadow = static_cast<float4*>(pb.shadow.ptr);
        P.counters = static_cast<uint32_t*>(pb.counters.ptr);
        P.cap = pb.capacity;
        P.shadow_cap = pb.shadow_capacity;
        P.fetch = static_cast<uint32_t>(ctx->pt_fetch);
    }
    const cudaStream_t streams[2] = {stream, two ? ctx->side_stream : stream};

    CameraDev cd;
    cd.width = cam->width;
    cd.height = cam->height;
    cd.model = cam->model;
    for (int a = 0; a < 3; ++a) {
        cd.position[a] = cam->position[a];
        cd.forward[a] = cam->forward[a];
        cd.right[a] = cam->right[a];
        cd.up[a] = cam->up[a];
    }
    cd.fx = cam->fx;
    cd.fy = cam->fy;
    cd.cx = cam->cx;
    cd.cy = cam->cy;
    cd.lens_radius = cam->lens_radius;
    cd.focal_distance = cam->focal_distance;

    const int grid = ctx->num_sms * 8;
    const uint32_t pix_per_wave = cap / spp;
    uint32_t launches = 0, waves = 0;
    cudaError_t e = cudaMemsetAsync(PP[0].counters, 0, kCWords * 4, stream);
    if (e == cudaSuccess && two) e = cudaMemsetAsync(PP[1].counters, 0, kCWords * 4, stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_start, stream);
    if (e == cudaSuccess && two) e = cudaEventRecord(ctx->ev_fork, stream);
    if (e == cudaSuccess && two) e = cudaStreamWaitEvent(ctx->side_stream, ctx->ev_fork, 0);
    for (uint64_t p0 = 0; p0 < npix && e == cudaSuccess; p0 += pix_per_wave) {
        const Paths& P = PP[waves & (two ? 1u : 0u)];
        const cudaStream_t ws = streams[waves & 1u];
        Wave w;
        w.p0 = static_cast<uint32_t>(p0);
        w.npaths = static_cast<uint32_t>(std::min<uint64_t>(pix_per_wave, npix - p0)) * spp;
        w.spp = spp;
        w.sample_offset = p->sample_offset;
        w.width = static_cast<uint32_t>(cam->width);
        w.max_depth = static_cast<uint32_t>(p->max_depth);
        w.use_nee = p->use_nee != 0;
        w.use_mis = p->use_mis != 0;
        w.seed = p->seed;
        k_raygen<false><<<grid, kBlock, 0, ws>>>(cd, w, P);
        ++launches;
        for (uint32_t d = 0; d < w.max_depth; ++d) {
            k_begin<<<1, 1, 0, ws>>>(P, d);
            if (volumetric) {
                if (count) k_extend<true, false, true><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d, ctx->d_error);
                else k_extend<true, false><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d, ctx->d_error);
                k_shade<2, false><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d);
            } else {
                if (count) k_extend<false, false, true><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d, ctx->d_error);
                else k_extend<false, false><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d, ctx->d_error);
                if (ctx->pt_shade_split) {
                    k_shade<0, false, kShadeGlossy><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d);
                    k_shade<0, false, kShadeGlossyRefl><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d);
                    k_shade<0, false, kShadeGlossyTrans><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d);
                    k_shade<0, false, kShadeDiffuse><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d);
                    k_shade<0, false, kShadeSpecular><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d);
                    k_shade<0, false, kShadeNone><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d);
                    launches += 3;
                } else {
                    k_shade<0, false><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d);
                }
            }
            if (count) k_shadow<true><<<grid, kBlock, 0, ws>>>(ctx->scene, P, ctx->d_error);
            else k_shadow<<<grid, kBlock, 0, ws>>>(ctx->scene, P, ctx->d_error);
            launches += 4;
        }
        k_film<<<grid, kBlock, 0, ws>>>(w, P, film_mean, film_m2);  // the wave's own pixels
        ++launches;
        ++waves;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && two) e = cudaEventRecord(ctx->ev_join, ctx->side_stream);
    if (e == cudaSuccess && two) e = cudaStreamWaitEvent(stream, ctx->ev_join, 0);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_stop, stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "path tracer launch");
    ctx->last_render.paths = npix * spp;
    ctx->last_render.extension_rays = 0;  // read from the device by rbr_render_stats_get
    ctx->last_render.shadow_rays = 0;
    ctx->last_render.waves = waves;
    ctx->last_render.launches = launches;
    ctx->render_pending = true;
    return RBR_OK;
}

// ------------------------------------------------------------------------------------------
// Rendering with the radiance cache: frames of the wavefront path tracer in which paths end
// into the cache (inference after each wave's bounces), training paths gather targets, and
// the cache trains after each frame.
// ------------------------------------------------------------------------------------------
namespace {

__global__ void k_cache_wave_end(const uint32_t* counters, uint32_t* scalars) {
    atomicAdd(scalars + kRcLastQueries, counters[kCQuery]);
}

// Training vertices of the frame: the sum over the waves in flight of their own lists.
__global__ void k_cache_frame_end(const uint32_t* c0, const uint32_t* c1, uint32_t* scalars, uint32_t cap) {
    scalars[kRcTrain] = min(*c0, cap) + (c1 ? min(*c1, cap) : 0u);
}


}  // namespace

CameraDev camera_dev(const rbr_camera* cam) {
    CameraDev cd;
    cd.width = cam->width;
    cd.height = cam->height;
    cd.model = cam->model;
    for (int a = 0; a < 3; ++a) {
        cd.position[a] = cam->position[a];
        cd.forward[a] = cam->forward[a];
        cd.right[a] = cam->right[a];
        cd.up[a] = cam->up[a];
    }
    cd.fx = cam->fx;
    cd.fy = cam->fy;
    cd.cx = cam->cx;
    cd.cy = cam->cy;
    cd.lens_radius = cam->lens_radius;
    cd.focal_distance = cam->focal_distance;
    return cd;
}

rbr_status render_cached(rbr_ctx* ctx, const rbr_camera* cam, const rbr_render_params* p, uint32_t frames, int train,
                         float* film_mean, float* film_m2, cudaStream_t stream) {
    if (!cam || !p || !film_mean) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "camera, params or film_mean is NULL");
    if (!ctx->has_scene) return fail(ctx, RBR_ERR_NO_SCENE, "rbr_cache_render before rbr_scene_upload");
    CacheState& cs = ctx->cache;
    if (!cs.ready) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "no radiance cache: call rbr_cache_create first");
    if (cam->width <= 0 || cam->height <= 0 || p->samples_per_pixel <= 0 || p->max_depth < 0 || frames == 0)
        return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "image size, samples per pixel, max depth or frames out of range");
    if (cam->model != RBR_CAMERA_PINHOLE && cam->model != RBR_CAMERA_THIN_LENS)
        return fail(ctx, RBR_ERR_UNSUPPORTED, "camera model " + std::to_string(cam->model));
    if (p->flags & RBR_RENDER_CORRECTED_MIS)
        return fail(ctx, RBR_ERR_UNSUPPORTED, "RBR_RENDER_CORRECTED_MIS is not implemented");
    if (p->flags & RBR_RENDER_VOLUMETRIC)
        return fail(ctx, RBR_ERR_UNSUPPORTED, "the radiance cache serves the surface path tracer, not RBR_RENDER_VOLUMETRIC");
    if ((p->flags & RBR_RENDER_SECOND_MOMENT) == 0) film_m2 = nullptr;
    const uint64_t npix = uint64_t(cam->width) * cam->height;
    const uint32_t spp = static_cast<uint32_t>(p->samples_per_pixel);
    if (npix * spp > 0xFFFFFFFFull || spp > kDefaultCapacity ||
        uint64_t(p->sample_offset) + uint64_t(frames) * spp > 0xFFFFFFFFull)
        return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "more than 2^32 camera samples per frame or sample indices");
    const uint32_t nl = std::max(1u, ctx->scene.num_lights);
    uint32_t cap = static_cast<uint32_t>(std::min<uint64_t>(npix * spp, std::max(ctx->pt_wave_paths, spp)));
    cap = std::min<uint64_t>(cap, kShadowBytesLimit / (48ull * nl));
    cap = std::max(spp, cap / spp * spp);
    // Two waves in flight as in render(): each has its own path buffers, query records and
    // half of the training-vertex list with its own counter; the frame's optimiser steps
    // draw from both halves once both waves have ended.
    const bool two = ctx->pt_streams == 2 && npix >= 2;
    if (two && npix * spp <= cap) cap = static_cast<uint32_t>((npix + 1) / 2) * spp;
    rbr_status st = ensure_paths(ctx, cap, cap * nl);
    if (st == RBR_OK && two) st = ensure_paths(ctx, cap, cap * nl, &ctx->pt2);
    if (st == RBR_OK && two) st = ensure_side_stream(ctx);
    if (st != RBR_OK) return st;
    const uint32_t depth = std::max(1, p->max_depth);
    const uint32_t t_cap =
        train ? static_cast<uint32_t>(std::min<uint64_t>(uint64_t(std::max(1u, cs.cfg.train_paths)) * depth, 1u << 23)) : 1;
    st = cache_ensure_render(ctx, two ? 2 * cap : cap, two ? 2 * t_cap : t_cap);
    if (st != RBR_OK) return st;
    const uint32_t t_half = two ? cs.t_cap / 2 : cs.t_cap;  // training vertices per wave slot

    Paths PP[2];
    for (int b = 0; b < (two ? 2 : 1); ++b) {
        PathBuffers& pb = b ? ctx->pt2 : ctx->pt;
        Paths& P = PP[b];
        P.ray = static_cast<float4*>(pb.ray.ptr);
        P.thr = static_cast<float4*>(pb.thr.ptr);
        P.rad = static_cast<float4*>(pb.rad.ptr);
        P.hit = static_cast<uint2*>(pb.hit.ptr);
        P.q0 = static_cast<uint32_t*>(pb.queue[0].ptr);
        P.q1 = static_cast<uint32_t*>(pb.queue[1].ptr);
        P.classq = static_cast<uint32_t*>(pb.classq.ptr);
        P.shadow = static_cast<float4*>(pb.shadow.ptr);
        P.counters = static_cast<uint32_t*>(pb.counters.ptr);
        P.cap = pb.capacity;
        P.shadow_cap = pb.shadow_capacity;
        P.fetch = static_cast<uint32_t>(ctx->pt_fetch);
        P.q_rec = static_cast<float4*>(cs.q_rec) + 4 * size_t(b) * cap;
        P.q_info = static_cast<float4*>(cs.q_info) + size_t(b) * cap;
        P.q_sort = static_cast<char*>(cs.q_sort) + size_t(b) * cs.q_sort_stride;
        P.t_rec = static_cast<float4*>(cs.t_rec) + 4 * size_t(b) * t_half;
        P.t_aux = static_cast<float4*>(cs.t_aux) + 2 * size_t(b) * t_half;
        P.t_cap = train ? t_half : 0;
    }
    const cudaStream_t streams[2] = {stream, two ? ctx->side_stream : stream};
    const CameraDev cd = camera_dev(cam);

    const double frac = train ? double(cs.cfg.train_paths) / double(npix * spp) : 0.0;
    const uint32_t thresh = static_cast<uint32_t>(std::min(4294967295.0, std::floor(frac * 4294967296.0)));
    const float weight = 1.0f / static_cast<float>(frames);
    uint32_t* scalars = static_cast<uint32_t*>(cs.scalars);

    const int grid = ctx->num_sms * 8;
    const uint32_t pix_per_wave = cap / spp;
    uint32_t launches = 0, waves = 0;
    cudaError_t e = cudaMemsetAsync(PP[0].counters, 0, kCWords * 4, stream);
    if (e == cudaSuccess && two) e = cudaMemsetAsync(PP[1].counters, 0, kCWords * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(film_mean, 0, npix * 12, stream);
    if (e == cudaSuccess && film_m2) e = cudaMemsetAsync(film_m2, 0, npix * 12, stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_start, stream);
    for (uint32_t f = 0; f < frames && e == cudaSuccess; ++f) {
        e = cudaMemsetAsync(PP[0].counters + kCTrain, 0, 4, stream);
        if (e == cudaSuccess && two) e = cudaMemsetAsync(PP[1].counters + kCTrain, 0, 4, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(scalars + kRcLastQueries, 0, 4, stream);
        if (e == cudaSuccess && two) e = cudaEventRecord(ctx->ev_fork, stream);
        if (e == cudaSuccess && two) e = cudaStreamWaitEvent(ctx->side_stream, ctx->ev_fork, 0);
        uint32_t wave_in_frame = 0;
        for (uint64_t p0 = 0; p0 < npix && e == cudaSuccess; p0 += pix_per_wave, ++wave_in_frame) {
            const Paths& P = PP[two ? (wave_in_frame & 1u) : 0u];
            const cudaStream_t ws = streams[wave_in_frame & 1u];
            Wave w;
            w.p0 = static_cast<uint32_t>(p0);
            w.npaths = static_cast<uint32_t>(std::min<uint64_t>(pix_per_wave, npix - p0)) * spp;
            w.spp = spp;
            w.sample_offset = p->sample_offset + f * spp;
            w.width = static_cast<uint32_t>(cam->width);
            w.max_depth = static_cast<uint32_t>(p->max_depth);
            w.use_nee = p->use_nee != 0;
            w.use_mis = p->use_mis != 0;
            w.seed = p->seed;
            w.cache_on = 1;
            w.term_depth = cs.cfg.termination_depth;
            w.train_suffix = cs.cfg.train_suffix;
            w.train_thresh = thresh;
            w.film_weight = weight;
            k_raygen<false><<<grid, kBlock, 0, ws>>>(cd, w, P);
            ++launches;
            for (uint32_t d = 0; d < w.max_depth; ++d) {
                k_begin<<<1, 1, 0, ws>>>(P, d);
                k_extend<false, false><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d, ctx->d_error);
                k_shade<1, false><<<grid, kBlock, 0, ws>>>(ctx->scene, w, P, d);
                k_shadow<<<grid, kBlock, 0, ws>>>(ctx->scene, P, ctx->d_error);
                launches += 4;
            }
            e = cache_launch_infer(ctx, P.q_rec, w.npaths, P.counters + kCQuery, nullptr, P.rad, P.q_info, ws, P.q_sort);
            ++launches;
            if (e == cudaSuccess && train) {
                e = cache_launch_finalize(ctx, P.rad, P.t_aux, P.counters, kCTrainBase, kCTrain, t_half, ws);
                ++launches;
            }
            k_film<<<grid, kBlock, 0, ws>>>(w, P, film_mean, film_m2);
            k_cache_wave_end<<<1, 1, 0, ws>>>(P.counters, scalars);
            launches += 2;
            ++waves;
            if (e == cudaSuccess) e = cudaGetLastError();
        }
        if (e == cudaSuccess && two) e = cudaEventRecord(ctx->ev_join, ctx->side_stream);
        if (e == cudaSuccess && two) e = cudaStreamWaitEvent(stream, ctx->ev_join, 0);
        const uint32_t* c1 = two ? PP[1].counters + kCTrain : nullptr;
        if (e == cudaSuccess) {
            k_cache_frame_end<<<1, 1, 0, stream>>>(PP[0].counters + kCTrain, c1, scalars, PP[0].t_cap);
            ++launches;
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && train) {
            e = cache_launch_train_frame(ctx, PP[0].counters + kCTrain, c1, t_half, f, stream);
            launches += 4 * cs.cfg.train_steps;
        }
    }
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_stop, stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cached path tracer launch");
    ctx->last_render.paths = npix * spp * frames;
    ctx->last_render.extension_rays = 0;
    ctx->last_render.shadow_rays = 0;
    ctx->last_render.waves = waves;
    ctx->last_render.launches = launches;
    ctx->pt_last_two = false;
    ctx->render_pending = true;
    return RBR_OK;
}

// ------------------------------------------------------------------------------------------
// Packed waves of the batched request loop (batch.cpp): several requests of one scene in one
// wave; per-path request data come from the segment table in device memory, so the launch
// sequence of a wave depends only on (scene, mode, depth, grid) and is captured once as a
// CUDA graph and replayed for every wave of that shape.
// ------------------------------------------------------------------------------------------
rbr_status ensure_wave_buffers(rbr_ctx* ctx, uint32_t cap, uint32_t shadow_cap, int slots) {
    for (int k = 0; k < slots; ++k) {
        DevBuf& seg = k ? ctx->pt_seg_of2 : ctx->pt_seg_of;
        rbr_status st = ensure_paths(ctx, cap, shadow_cap, k ? &ctx->pt2 : &ctx->pt);
        if (st != RBR_OK) return st;
        if (seg.bytes < size_t(cap) * 4) {
            ++ctx->pt_generation;
            st = ensure(ctx, seg, size_t(cap) * 4, "segment index per path");
            if (st != RBR_OK) return st;
        }
    }
    return RBR_OK;
}

cudaError_t launch_packed_wave(rbr_ctx* eng, rbr_ctx* scn, const PackedWave& pw, cudaStream_t stream) {
    PathBuffers& pb = pw.slot ? eng->pt2 : eng->pt;
    Paths P;
    P.ray = static_cast<float4*>(pb.ray.ptr);
    P.thr = static_cast<float4*>(pb.thr.ptr);
    P.rad = static_cast<float4*>(pb.rad.ptr);
    P.hit = static_cast<uint2*>(pb.hit.ptr);
    P.q0 = static_cast<uint32_t*>(pb.queue[0].ptr);
    P.q1 = static_cast<uint32_t*>(pb.queue[1].ptr);
    P.classq = static_cast<uint32_t*>(pb.classq.ptr);
    P.shadow = static_cast<float4*>(pb.shadow.ptr);
    P.counters = static_cast<uint32_t*>(pb.counters.ptr);
    P.cap = pb.capacity;
    P.shadow_cap = pb.shadow_capacity;
    P.fetch = static_cast<uint32_t>(eng->pt_fetch);
    P.segs = pw.segs;
    P.seg_of = static_cast<uint32_t*>((pw.slot ? eng->pt_seg_of2 : eng->pt_seg_of).ptr);
    P.wave_hdr = pw.hdr;
    Wave w{};
    if (pw.mode == 1) {
        CacheState& cs = scn->cache;
        P.q_rec = static_cast<float4*>(cs.q_rec);
        P.q_info = static_cast<float4*>(cs.q_info);
        P.q_sort = cs.q_sort;
        P.t_rec = static_cast<float4*>(cs.t_rec);
        P.t_aux = static_cast<float4*>(cs.t_aux);
        P.t_cap = pw.train ? cs.t_cap : 0;
        w.cache_on = 1;
        w.term_depth = cs.cfg.termination_depth;
        w.train_suffix = cs.cfg.train_suffix;
        w.train_thresh = pw.train_thresh;
    }
    const CameraDev unused{};
    const int grid = pw.grid;
    cudaError_t e = cudaMemsetAsync(P.counters, 0, kCWords * 4, stream);
    if (e != cudaSuccess) return e;
    k_raygen<true><<<grid, kBlock, 0, stream>>>(unused, w, P);
    for (uint32_t d = 0; d < pw.max_depth; ++d) {
        k_begin<<<1, 1, 0, stream>>>(P, d);
        if (pw.mode == 2) {
            k_extend<true, true><<<grid, kBlock, 0, stream>>>(scn->scene, w, P, d, eng->d_error);
            k_shade<2, true><<<grid, kBlock, 0, stream>>>(scn->scene, w, P, d);
        } else {
            k_extend<false, true><<<grid, kBlock, 0, stream>>>(scn->scene, w, P, d, eng->d_error);
            if (pw.mode == 1) k_shade<1, true><<<grid, kBlock, 0, stream>>>(scn->scene, w, P, d);
            else k_shade<0, true><<<grid, kBlock, 0, stream>>>(scn->scene, w, P, d);
        }
        k_shadow<<<grid, kBlock, 0, stream>>>(scn->scene, P, eng->d_error);
    }
    if (pw.mode == 1) {
        e = cache_launch_infer(scn, P.q_rec, pw.capacity, P.counters + kCQuery, nullptr, P.rad, P.q_info, stream, P.q_sort);
        if (e == cudaSuccess && pw.train)
            e = cache_launch_finalize(scn, P.rad, P.t_aux, P.counters, kCTrainBase, kCTrain, scn->cache.t_cap, stream);
        if (e != cudaSuccess) return e;
    }
    k_film_packed<<<grid, kBlock, 0, stream>>>(P);
    if (pw.mode == 1 && pw.train) {
        e = cache_launch_train_frame(scn, P.counters + kCTrain, nullptr, scn->cache.t_cap, 0, stream);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

cudaError_t launch_wave_loop(rbr_ctx* eng, const std::vector<rbr_ctx*>& scenes, const LoopWave* waves, uint32_t nwaves,
                             const char* tables, unsigned long long* stamps, uint32_t* bar, uint64_t limit_ns,
                             int halves, cudaStream_t stream, int* grid_out) {
    if (scenes.size() > static_cast<size_t>(kLoopScenes) || (halves != 1 && halves != 2)) return cudaErrorInvalidValue;
    LoopParams lp{};
    for (size_t i = 0; i < scenes.size(); ++i) lp.scenes[i] = scenes[i]->scene;
    lp.waves = waves;
    lp.nwaves = nwaves;
    lp.halves = static_cast<uint32_t>(halves);
    lp.tables = tables;
    for (int h = 0; h < halves; ++h) {
        PathBuffers& pb = h ? eng->pt2 : eng->pt;
        Paths& P = lp.P[h];
        P.ray = static_cast<float4*>(pb.ray.ptr);
        P.thr = static_cast<float4*>(pb.thr.ptr);
        P.rad = static_cast<float4*>(pb.rad.ptr);
        P.hit = static_cast<uint2*>(pb.hit.ptr);
        P.q0 = static_cast<uint32_t*>(pb.queue[0].ptr);
        P.q1 = static_cast<uint32_t*>(pb.queue[1].ptr);
        P.classq = static_cast<uint32_t*>(pb.classq.ptr);
        P.shadow = static_cast<float4*>(pb.shadow.ptr);
        P.counters = static_cast<uint32_t*>(pb.counters.ptr);
        P.cap = pb.capacity;
        P.shadow_cap = pb.shadow_capacity;
        P.fetch = static_cast<uint32_t>(eng->pt_fetch);
        P.seg_of = static_cast<uint32_t*>((h ? eng->pt_seg_of2 : eng->pt_seg_of).ptr);
    }
    lp.stamps = stamps;
    lp.bar = bar;
    lp.err = eng->d_error;
    lp.limit_ns = limit_ns;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wave_loop, kBlock, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    int grid = eng->num_sms * per_sm;  // every block resident: the barriers depend on it
    grid -= grid % halves;
    if (grid_out) *grid_out = grid;
    e = cudaMemsetAsync(bar, 0, kLoopBarrierWords * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    void* args[] = {&lp};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_wave_loop), dim3(grid), dim3(kBlock), args, 0,
                                       stream);
}

cudaError_t launch_stamp(unsigned long long* at, cudaStream_t stream) {
    k_stamp<<<1, 1, 0, stream>>>(at);
    return cudaGetLastError();
}

cudaError_t launch_release(const unsigned long long* start, uint64_t release_ns, cudaStream_t stream) {
    if (release_ns == 0) return cudaSuccess;
    k_release<<<1, 1, 0, stream>>>(start, release_ns);
    return cudaGetLastError();
}

uint32_t packed_wave_launches(const PackedWave& pw) {
    uint32_t n = 2 + 4 * pw.max_depth;  // raygen, film, depth loop
    if (pw.mode == 1) n += 1 + (pw.train ? 1 + 4 * pw.train_steps : 0);
    return n;
}

// ------------------------------------------------------------------------------------------
// Rendering without allocating: the wave state lives in a fixed array compiled into the
// library instead of buffers the context allocates on demand.
// ------------------------------------------------------------------------------------------
namespace {

// Every GPU that loads this library holds this array until the process exits.
__device__ __align__(256) unsigned char g_render_scratch[RBR_NOALLOC_SCRATCH_BYTES];

// Device address of g_render_scratch on the current device, looked up on every call: the
// lookup allocates nothing, and a cached address would go stale if the application reset the
// device or its primary context between calls. In host code the array's name only stands in
// for the symbol; kernels must be given this address, never the host-side name.
cudaError_t scratch_address(unsigned char** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_render_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<unsigned char*>(p);
    return cudaSuccess;
}

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

rbr_status render_noalloc(rbr_ctx* ctx, const rbr_camera* cam, const rbr_render_params* p, float* film_mean,
                          cudaStream_t stream) {
    if (!cam || !p || !film_mean) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "camera, params or film_mean is NULL");
    if (!ctx->has_scene) return fail(ctx, RBR_ERR_NO_SCENE, "rbr_render_noalloc before rbr_scene_upload");
    if (cam->width <= 0 || cam->height <= 0 || p->samples_per_pixel <= 0 || p->max_depth < 0)
        return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "image size, samples per pixel or max depth out of range");
    if (cam->model != RBR_CAMERA_PINHOLE && cam->model != RBR_CAMERA_THIN_LENS)
        return fail(ctx, RBR_ERR_UNSUPPORTED, "camera model " + std::to_string(cam->model));
    if (p->flags != 0)
        return fail(ctx, RBR_ERR_UNSUPPORTED, "rbr_render_noalloc takes no flags (it writes the mean film only)");
    const uint64_t npix = uint64_t(cam->width) * cam->height;
    const uint32_t spp = static_cast<uint32_t>(p->samples_per_pixel);
    if (npix * spp > 0xFFFFFFFFull)
        return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "more than 2^32 camera samples in one render call");
    // wave capacity that fits the fixed array: 88 B of path state, 4 B per class queue and 48 B
    // per light and path
    const uint32_t nl = std::max(1u, ctx->scene.num_lights);
    const size_t per_path = 88 + 4 * size_t(kNumClasses) + 48 * size_t(nl);
    const size_t fixed = 9 * 256;  // counters + alignment of the eight arrays
    uint64_t cap = (RBR_NOALLOC_SCRATCH_BYTES - fixed) / per_path;
    cap = std::min<uint64_t>(cap, npix * spp);
    cap = cap / spp * spp;
    if (cap < spp)
        return fail(ctx, RBR_ERR_INVALID_ARGUMENT,
                    "rbr_render_noalloc: " + std::to_string(spp) + " samples per pixel with " + std::to_string(nl) +
                        " lights do not fit its " + std::to_string(RBR_NOALLOC_SCRATCH_BYTES) +
                        "-byte scratch array (at most " +
                        std::to_string((RBR_NOALLOC_SCRATCH_BYTES - fixed) / per_path) + " samples per pixel)");
    unsigned char* base = nullptr;
    cudaError_t e = scratch_address(&base);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "looking up the render scratch array");

    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* q = base + off;
        off += align256(bytes);
        return q;
    };
    Paths P;
    P.counters = reinterpret_cast<uint32_t*>(take(kCWords * 4));
    P.ray = reinterpret_cast<float4*>(take(cap * 32));
    P.thr = reinterpret_cast<float4*>(take(cap * 16));
    P.rad = reinterpret_cast<float4*>(take(cap * 16));
    P.hit = reinterpret_cast<uint2*>(take(cap * 8));
    P.q0 = reinterpret_cast<uint32_t*>(take(cap * 4));
    P.q1 = reinterpret_cast<uint32_t*>(take(cap * 4));
    P.classq = reinterpret_cast<uint32_t*>(take(cap * 4 * kNumClasses));
    P.shadow = reinterpret_cast<float4*>(take(cap * nl * 48));
    if (off > RBR_NOALLOC_SCRATCH_BYTES) return fail(ctx, RBR_ERR_INTERNAL, "scratch layout exceeds the array");
    P.cap = static_cast<uint32_t>(cap);
    P.shadow_cap = static_cast<uint32_t>(cap * nl);
    P.fetch = static_cast<uint32_t>(ctx->pt_fetch);

    CameraDev cd;
    cd.width = cam->width;
    cd.height = cam->height;
    cd.model = cam->model;
    for (int a = 0; a < 3; ++a) {
        cd.position[a] = cam->position[a];
        cd.forward[a] = cam->forward[a];
        cd.right[a] = cam->right[a];
        cd.up[a] = cam->up[a];
    }
    cd.fx = cam->fx;
    cd.fy = cam->fy;
    cd.cx = cam->cx;
    cd.cy = cam->cy;
    cd.lens_radius = cam->lens_radius;
    cd.focal_distance = cam->focal_distance;

    // The array keeps the previous call's contents: only the counters must start at zero,
    // every other array is written before it is read within a wave.
    e = cudaMemsetAsync(P.counters, 0, kCWords * 4, stream);
    const int grid = ctx->num_sms * 8;
    const uint32_t pix_per_wave = static_cast<uint32_t>(cap / spp);
    for (uint64_t p0 = 0; p0 < npix && e == cudaSuccess; p0 += pix_per_wave) {
        Wave w;
        w.p0 = static_cast<uint32_t>(p0);
        w.npaths = static_cast<uint32_t>(std::min<uint64_t>(pix_per_wave, npix - p0)) * spp;
        w.spp = spp;
        w.sample_offset = p->sample_offset;
        w.width = static_cast<uint32_t>(cam->width);
        w.max_depth = static_cast<uint32_t>(p->max_depth);
        w.use_nee = p->use_nee != 0;
        w.use_mis = p->use_mis != 0;
        w.seed = p->seed;
        k_raygen<false><<<grid, kBlock, 0, stream>>>(cd, w, P);
        for (uint32_t d = 0; d < w.max_depth; ++d) {
            k_begin<<<1, 1, 0, stream>>>(P, d);
            k_extend<false, false><<<grid, kBlock, 0, stream>>>(ctx->scene, w, P, d, ctx->d_error);
            k_shade<0, false><<<grid, kBlock, 0, stream>>>(ctx->scene, w, P, d);
            k_shadow<<<grid, kBlock, 0, stream>>>(ctx->scene, P, ctx->d_error);
        }
        k_film<<<grid, kBlock, 0, stream>>>(w, P, film_mean, nullptr);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "path tracer launch (no-alloc)");
    return RBR_OK;
}

}  // namespace rbr
