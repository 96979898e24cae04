/*
 * rbr_b200.h — C ABI of the B200 path-tracing library (librbr_b200.so).
 *
 * The library is the GPU side of two drop-ins for the Ray-Based-Rendering C++17 API:
 *   - an Accelerator   (include/render/acceleration/accelerator.h:19-34) selected with `-a gpubvh`,
 *   - an Integrator    (include/render/renderers/integrator.h:37-73)     selected with `-i gpupt`.
 * The C++ adapters that derive from those classes (adapters/gpu_accelerator.h,
 * adapters/gpu_integrator.h) flatten a render::Scene into the plain arrays below and call
 * these entry points. Nothing here uses C++ or CUDA types: streams are passed as `void*`
 * (a cudaStream_t, NULL = the legacy default stream) and every buffer is a plain pointer.
 *
 * Conventions
 *   - Every entry point returns an rbr_status; on failure rbr_last_error() holds a message.
 *   - A context owns all of its device memory (scene, BVH, queues, film, cache). Calls on one
 *     context are not re-entrant: callers that share a context across threads serialise them.
 *   - "device pointer" arguments must point to memory of the context's device;
 *     "host pointer" arguments may be pageable or pinned host memory.
 *   - There is no CPU fallback: without a usable CUDA device rbr_ctx_create fails.
 */
#ifndef RBR_B200_H
#define RBR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RBR_ABI_VERSION 1u

typedef enum rbr_status {
    RBR_OK = 0,
    RBR_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size, index or NaN in a descriptor */
    RBR_ERR_CUDA = 2,             /* a CUDA runtime call failed (message has the CUDA error) */
    RBR_ERR_OUT_OF_MEMORY = 3,    /* device or pinned-host allocation failed */
    RBR_ERR_NO_SCENE = 4,         /* a trace/render call before rbr_scene_upload */
    RBR_ERR_UNSUPPORTED = 5,      /* input the GPU path does not implement (reported, never emulated) */
    RBR_ERR_DEVICE_TIMEOUT = 6,   /* a bounded device-side wait ran out; the context stays usable */
    RBR_ERR_INTERNAL = 7          /* a device-side consistency check failed (e.g. stack overflow) */
} rbr_status;

/* Marks "no primitive" in rbr_hit.prim. */
#define RBR_MISS 0xFFFFFFFFu

typedef struct rbr_ctx rbr_ctx;

/* ------------------------------------------------------------------------------------------
 * Scene description. Mirrors what render::Scene holds (include/render/scene/scene.h:92-95):
 * primitives with a material each, the six-parameter materials, lights and a background.
 * Primitive ids: the index of the primitive in Scene::primitives(); the per-type `*_ids`
 * arrays give it. When an ids array is NULL the ids of that type follow one another in the
 * order triangles, spheres, quads, planes (so an all-NULL scene numbers them in that order).
 * ids must be a permutation of 0..N-1 over all primitives of the scene.
 * ------------------------------------------------------------------------------------------ */

/* render::Material's six public parameters (include/render/materials/material.h:28-36). */
typedef struct rbr_material {
    float base_color[3];
    float metallic;
    float roughness;
    float ior;
    float transmission;
    float emission[3];
} rbr_material;

enum { RBR_LIGHT_AREA = 0, RBR_LIGHT_POINT = 1 };

/* render::AreaLight (include/render/lighting/area_light.h:16-27: centre `position`, edges u, v)
 * or render::PointLight (include/render/lighting/point_light.h:13-20; u, v unused). */
typedef struct rbr_light {
    uint32_t type;        /* RBR_LIGHT_AREA or RBR_LIGHT_POINT */
    float position[3];
    float u[3];
    float v[3];
    float color[3];
    float intensity;
} rbr_light;

/* render::HomogeneousMedium (include/render/materials/medium.h:54-70): absorption and
 * scattering coefficients and the Henyey-Greenstein asymmetry g of its phase function. The
 * medium fills all space (Scene::medium(), include/render/scene/scene.h:95). */
typedef struct rbr_medium {
    float sigma_a[3];
    float sigma_s[3];
    float g;
} rbr_medium;

typedef struct rbr_scene_desc {
    /* render::Triangle (include/render/geometry/triangle.h:13-52): v0, v1, v2 per triangle. */
    uint32_t num_triangles;
    const float* triangle_vertices;     /* [num_triangles][9] */
    const float* triangle_normals;      /* optional [num_triangles][9] unit n0, n1, n2, or NULL */
    const uint32_t* triangle_materials; /* [num_triangles] */
    const uint32_t* triangle_ids;       /* optional */
    /* render::Sphere (include/render/geometry/sphere.h:13-19): centre, radius. */
    uint32_t num_spheres;
    const float* spheres;               /* [num_spheres][4] */
    const uint32_t* sphere_materials;
    const uint32_t* sphere_ids;
    /* render::Quad (include/render/geometry/quad.h:13-19): corner `origin`, edges u, v. */
    uint32_t num_quads;
    const float* quads;                 /* [num_quads][9] */
    const uint32_t* quad_materials;
    const uint32_t* quad_ids;
    /* render::Plane (include/render/geometry/plane.h:13-19): unit normal and d (n.p + d = 0). */
    uint32_t num_planes;
    const float* planes;                /* [num_planes][4] */
    const uint32_t* plane_materials;
    const uint32_t* plane_ids;
    uint32_t num_materials;
    const rbr_material* materials;
    uint32_t num_lights;                /* in Scene::lights() order */
    const rbr_light* lights;
    float background[3];                /* Scene::backgroundColor */
    const rbr_medium* medium;           /* Scene::medium(), or NULL for none */
} rbr_scene_desc;

/* Sizes of what rbr_scene_upload built. */
typedef struct rbr_scene_stats {
    uint32_t num_primitives;      /* all primitives */
    uint32_t num_bounded;         /* primitives inside the BVH */
    uint32_t num_unbounded;       /* planes, tested outside the BVH */
    uint32_t num_wide_nodes;      /* 8-wide nodes (80 B each) */
    uint32_t num_leaf_records;    /* leaf primitive records (48 B each) */
    uint32_t max_depth;           /* depth of the wide tree */
    uint32_t wrapped_leaves;      /* leaves given a wide node of their own: a node beside internal
                                     children holds at most 24 leaf records */
    uint32_t record_cost_milli;   /* "bvh.record_cost_milli" the tree was built with */
    uint64_t device_bytes;        /* device memory held by the scene */
    double build_seconds;         /* host SAH build + collapse + quantisation */
} rbr_scene_stats;

/* ------------------------------------------------------------------------------------------
 * Ray queries. render::Ray (include/render/core/ray.h:10-35): origin, unit direction, tMax;
 * the implicit tMin is the primitives' EPSILON = 1e-4 (include/render/core/common.h:22).
 * Directions are used exactly as given (render::Ray normalises in its constructor, so a
 * caller passes the already-normalised direction of its Ray).
 * ------------------------------------------------------------------------------------------ */
typedef struct rbr_ray {
    float origin[3];
    float tmax;
    float direction[3];
    float pad;
} rbr_ray; /* 32 B, two 16 B loads */

typedef struct rbr_hit {
    uint32_t prim; /* primitive id, RBR_MISS if nothing was hit */
    float t;       /* SurfaceInteraction::t of the closest hit */
} rbr_hit;

/* ------------------------------------------------------------------------------------------
 * Camera and integrator parameters.
 * ------------------------------------------------------------------------------------------ */

enum { RBR_CAMERA_PINHOLE = 0, RBR_CAMERA_THIN_LENS = 1 };

/* A PinholeCamera or a ThinLensCamera: CameraExtrinsics
 * (include/render/camera/camera_extrinsics.h:16-21) + PerspectiveIntrinsics
 * (include/render/camera/perspective_intrinsics.h:21-24) + thin-lens parameters
 * (include/render/camera/thin_lens_camera.h:15-16). */
typedef struct rbr_camera {
    int32_t width, height;
    uint32_t model;          /* RBR_CAMERA_PINHOLE or RBR_CAMERA_THIN_LENS */
    float position[3];
    float forward[3];
    float right[3];
    float up[3];
    float fx, fy, cx, cy;
    float lens_radius;
    float focal_distance;
} rbr_camera;

/* Flags of rbr_render_params.flags. */
enum {
    /* Adds the BSDF-sampled hit of emissive geometry with the matching MIS weight instead of
     * discarding it (the reference's estimator drops it: path_tracing_integrator.cpp:130-133).
     * Off by default so that images converge to what the reference converges to. */
    RBR_RENDER_CORRECTED_MIS = 1u << 0,
    /* Also return per-pixel sums of squared sample values (for Monte-Carlo error bars). */
    RBR_RENDER_SECOND_MOMENT = 1u << 1,
    /* VolumetricPathIntegrator's estimator (src/renderers/volumetric_path_integrator.cpp:6-143)
     * instead of PathTracingIntegrator's: distance sampling in the scene's medium, next-event
     * estimation from scatter points towards point lights with transmittance and the phase
     * function, emission added at every surface hit, surface next-event estimation without MIS
     * weights, Russian roulette at surface vertices after depth 3. */
    RBR_RENDER_VOLUMETRIC = 1u << 2,
    /* Diagnostic (rbr_render only): also count the 8-wide nodes fetched and leaf records tested
     * by every extension and shadow ray (rbr_render_stats), for the path tracer's algorithmic
     * traffic. Same images; the counting kernels run slower. */
    RBR_RENDER_COUNT_TRAFFIC = 1u << 3
};

/* IntegratorConfig (include/render/renderers/integrator.h:22-28). */
typedef struct rbr_render_params {
    int32_t samples_per_pixel;
    int32_t max_depth;
    int32_t use_nee;
    int32_t use_mis;
    uint64_t seed;            /* key of the counter-based RNG */
    uint32_t sample_offset;   /* index of the first sample (independent batches use disjoint ranges) */
    uint32_t flags;           /* RBR_RENDER_* */
} rbr_render_params;

/* Timings and counters of the last rbr_render call. */
typedef struct rbr_render_stats {
    uint64_t paths;           /* camera samples traced */
    uint64_t extension_rays;  /* closest-hit rays */
    uint64_t shadow_rays;     /* any-hit rays */
    uint32_t waves;           /* path chunks processed */
    uint32_t launches;        /* kernels launched */
    float milliseconds;       /* device time of the whole render (CUDA events) */
    uint64_t shaded_vertices; /* extension rays that hit a surface and were shaded */
    uint64_t ext_nodes;       /* with RBR_RENDER_COUNT_TRAFFIC: wide nodes fetched by extension rays */
    uint64_t ext_records;     /*   leaf records tested by extension rays */
    uint64_t shadow_nodes;    /*   wide nodes fetched by shadow rays */
    uint64_t shadow_records;  /*   leaf records tested by shadow rays (0 without the flag) */
} rbr_render_stats;

/* ------------------------------------------------------------------------------------------
 * Entry points.
 * ------------------------------------------------------------------------------------------ */

uint32_t rbr_abi_version(void);
/* sizeof() of a struct of this header by name ("rbr_ray", ...), 0 for an unknown name; lets
 * bindings check their struct mirrors against the compiled library. */
size_t rbr_struct_size(const char* name);

/* Creates a context on CUDA device `device`. */
rbr_status rbr_ctx_create(int device, rbr_ctx** out);
void rbr_ctx_destroy(rbr_ctx* ctx);
const char* rbr_last_error(const rbr_ctx* ctx);

/* Replaces the context's scene: validates the description, builds the SAH BVH on the host,
 * collapses it into the 8-wide quantised layout and uploads everything.
 * Replaces: Scene::buildAccelerator / Accelerator::build (src/scene/scene.cpp:22-28,
 * include/render/acceleration/accelerator.h:25). A rebuild drops the previous contents. */
rbr_status rbr_scene_upload(rbr_ctx* ctx, const rbr_scene_desc* desc);
rbr_status rbr_scene_stats_get(const rbr_ctx* ctx, rbr_scene_stats* out);

/* Tunables of a context (no reference counterpart). Names:
 *   "trace.kernel"         0: one thread per ray (default); 1: persistent warps that hand a
 *                          finished lane the next ray of the warp's chunk; 2: warp-cooperative,
 *                          8 lanes per ray, one child box per lane
 *   "trace.blocks_per_sm"  resident blocks per SM of kernels 1 and 2 (0: occupancy limit)
 *   "trace.refill_min"     kernel 1: idle lanes a warp waits for before it fetches new rays,
 *                          1..32 (default 1: refill after every step with an idle lane)
 *   "trace.min_blocks"     kernel 0's register budget: 8, 10 or 12 resident blocks per SM
 *   "trace.order"          kernels 0 and 1: 0 traces the rays in the order given; 1..5 first sort
 *                          them on the device so that warps hold rays that walk the same nodes:
 *                          1 by direction octant, then origin cell of 512^3; 2 octant, then cell
 *                          of 64^3; 3 cell of 64^3, then octant; 4 direction cell (octahedral
 *                          16 x 8), then origin cell of 8^3; 5 origin cell of 8^3, then direction
 *                          cell. Orders 4 and 5 (16-bit keys) use the library's counting sort;
 *                          1-3 (21- and 30-bit keys) CUB's radix sort
 *   "trace.host_chunk"     rbr_trace_host: rays per chunk of its upload / trace / download
 *                          pipeline (default 2^19; 0: one piece)
 *   "trace.host_streams"   rbr_trace_host: streams the chunks rotate over, 2, 3 or 4 (default 4);
 *                          the last full chunk is split into halving pieces (shorter tail)
 *   "pt.wave_paths"        camera samples per path-tracer wave (default 2^23)
 *   "pt.streams"           rbr_render: waves in flight, 1 or 2 (default 2: waves alternate
 *                          between two sets of path buffers on two streams; an image that
 *                          fits one wave is rendered as two half-image waves; when the second
 *                          set cannot be allocated, the waves run one at a time in the first)
 *   "trace.node_test"      sorted queries of kernel 0: 0 the packed node test (f32x2 FMAs), 1 a
 *                          register-lean one (scalar FMAs, fewer live registers)
 *   "trace.stream_io"      kernel 0: rays read and hits written with evict-first hints (default 1)
 *   "trace.l2_persist"     kernel 0: 1 reserves the largest persisting-L2 set-aside this process's
 *                          context allows and marks the BVH (nodes and leaf records) persisting for
 *                          each ray-query launch; 0 (default) releases it
 *   "pt.shade_split"       rbr_render: 1 shades each material class (Lambertian, GGX with a
 *                          Lambertian lobe, GGX reflection only, GGX transmission, delta-only,
 *                          none) in a launch of its own, compiled for that class's lobes; 0 one
 *                          launch for all classes (default)
 *   "pt.fetch"             path tracer: 1 (default) the extension, shading and shadow launches
 *                          hand out a queue of eight grid rounds or more in claims of 32 to 256
 *                          entries to whichever warp is free (one atomic per claim), so warps
 *                          that drew short traversals take more; 0 a fixed grid-stride share
 *                          per warp
 *   "cache.infer_groups"   radiance-cache inference: 128-sample tiles in flight per CTA, 1, 2 or 4
 *                          (groups of four warps sharing one copy of the weights; default 1)
 *   "cache.infer_warps"    one-tile inference: 4 or 8 warps per 128-sample tile (default 4)
 *   "cache.sort_queries"   1: inference serves the queries in spatial order (a counting sort of
 *                          their cells on a 32^3 grid); 0: in the order given (default 0)
 *   "cache.wait_limit"     polls of a tensor-core completion wait in the radiance-cache kernels
 *                          before it gives up with RBR_ERR_DEVICE_TIMEOUT (default 2^22; 0
 *                          makes every such wait give up at once, which tests the error path:
 *                          the kernel still drains its work before it frees tensor memory)
 *   "debug.fail_alloc"     n > 0: the n-th next device allocation of the context fails with
 *                          RBR_ERR_OUT_OF_MEMORY (fault injection for callers' error paths)
 *   "bvh.record_cost_milli" cost of testing one leaf record relative to one wide-node test,
 *                          x1000, in the 8-wide collapse's surface-area cost (default 1000);
 *                          applies to the next rbr_scene_upload
 * Results do not depend on them; only speed and memory do. rbr_autotune picks them. */
rbr_status rbr_param_set(rbr_ctx* ctx, const char* name, int64_t value);
rbr_status rbr_param_get(const rbr_ctx* ctx, const char* name, int64_t* value);
/* Autotuner (no reference counterpart): times the traversal variants ("trace.kernel",
 * "trace.min_blocks", "trace.order" 0, 4 and 5, "trace.node_test") on n rays of the caller's own
 * workload (device pointer) against the uploaded scene, keeps the fastest in the context and
 * returns its time per launch in microseconds (out_us may be NULL). Waits for the timings. */
rbr_status rbr_autotune_trace(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, int any_hit, int64_t* out_us);
/* World bounds of the bounded primitives (Accelerator::worldBounds, accelerator.h:33).
 * An empty scene gives min = +FLT_MAX, max = -FLT_MAX (an empty BoundingBox). */
rbr_status rbr_world_bounds(const rbr_ctx* ctx, float out_min[3], float out_max[3]);

/* Closest hit for n rays (device pointers), asynchronous on `stream`.
 * Replaces: Accelerator::intersect / BVH::intersect (accelerator.h:28, src/acceleration/bvh.cpp:33-36). */
rbr_status rbr_trace_closest(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, rbr_hit* hits, void* stream);
/* Any hit (occluded[i] = 1 if something lies in [EPSILON, tmax]), device pointers, asynchronous.
 * Replaces: Accelerator::intersectP / BVH::intersectP (accelerator.h:31, bvh.cpp:38-41). */
rbr_status rbr_trace_any(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, uint8_t* occluded, void* stream);
/* The same two queries on host buffers: copies the rays in, traces, copies the answers out and
 * waits. `out` is rbr_hit[n] when any_hit == 0, uint8_t[n] otherwise. */
rbr_status rbr_trace_host(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, int any_hit, void* out);

/* Diagnostic: replays the traversal of n rays (device pointer) and returns the total number of
 * 8-wide nodes fetched (out[0]) and leaf records tested (out[1]); waits for the result.
 * The traversal order of a ray is deterministic, so these are its algorithmic node and leaf
 * traffic (80 B per node, 48 B per record) for roofline accounting. No reference counterpart. */
rbr_status rbr_trace_counts(rbr_ctx* ctx, const rbr_ray* rays, uint32_t n, int any_hit, uint64_t out[2]);

/* Renders the scene with the wavefront path tracer.
 * film_mean: device pointer, width*height*3 floats, receives the per-pixel mean over the
 * samples, as Film::addSample(x, y, sum / spp) stores it (src/renderers/integrator.cpp:36).
 * film_m2: device pointer or NULL; with RBR_RENDER_SECOND_MOMENT it receives per-pixel sums
 * of squared sample values (width*height*3 floats). Asynchronous on `stream`: with
 * "pt.streams" 2 every other wave runs on a second stream of the context that forks from
 * `stream` at the start and joins it at the end, so work queued on `stream` afterwards sees
 * the whole film.
 * Replaces: Integrator::render with PathTracingIntegrator::Li (src/renderers/integrator.cpp:7-50,
 * src/renderers/path_tracing_integrator.cpp:5-138). */
rbr_status rbr_render(rbr_ctx* ctx, const rbr_camera* camera, const rbr_render_params* params,
                      float* film_mean, float* film_m2, void* stream);
/* The same on host buffers (film_mean required, film_m2 optional); waits for the result. */
rbr_status rbr_render_host(rbr_ctx* ctx, const rbr_camera* camera, const rbr_render_params* params,
                           float* film_mean, float* film_m2);
/* Counters and device time of the last render (waits for it). */
rbr_status rbr_render_stats_get(rbr_ctx* ctx, rbr_render_stats* out);

/* ------------------------------------------------------------------------------------------
 * Unit entry points: the path tracer's own device functions applied to caller-given inputs
 * (host buffers, each call waits), for one-to-one comparison with the reference's CPU code.
 * ------------------------------------------------------------------------------------------ */

/* Material::createBSDF + BSDF::evaluate / pdf (src/materials/material.cpp:69-108,
 * mixture_bsdf.cpp:48-67) for n (wo, wi) pairs in the shading frame (normal = +z).
 * out: 6 floats per pair: f[3], pdf, isDelta (0/1), BSDFType bits. */
rbr_status rbr_bsdf_eval_host(rbr_ctx* ctx, const rbr_material* material, uint32_t n, const float* wo,
                              const float* wi, float* out);
/* Material::createBSDF + BSDF::sample (mixture_bsdf.cpp:69-105) for n (wo, u1, u2).
 * out: 8 floats per sample: wi[3], f[3], pdf, isDelta. */
rbr_status rbr_bsdf_sample_host(rbr_ctx* ctx, const rbr_material* material, uint32_t n, const float* wo,
                                const float* u, float* out);
/* Light::sample at n surface points (area_light.cpp:13-39, point_light.cpp:5-19).
 * out: 9 floats per sample: wi[3], Li[3], pdf, distance, isDelta. */
rbr_status rbr_light_sample_host(rbr_ctx* ctx, const rbr_light* light, uint32_t n, const float* points,
                                 const float* u, float* out);
/* Camera::generateRay for n CameraSamples (filmX, filmY, lensU, lensV)
 * (camera.cpp:5-9, pinhole_camera.cpp:5-7, thin_lens_camera.cpp:6-23). out: origin[3], dir[3]. */
rbr_status rbr_camera_rays_host(rbr_ctx* ctx, const rbr_camera* camera, uint32_t n, const float* samples,
                                float* out);
/* sampling::powerHeuristic(1, pdf_pairs[2i], 1, pdf_pairs[2i+1]) (sampler.h:137-149). */
rbr_status rbr_mis_weights_host(rbr_ctx* ctx, uint32_t n, const float* pdf_pairs, float* out);

/* ------------------------------------------------------------------------------------------
 * Learned radiance cache (no reference counterpart): a multiresolution hash-grid encoding
 * (16 levels x 2^log2_table_size entries x 2 FP16 features) of the surface position, plus
 * the outgoing direction, shading normal, roughness and diffuse/specular albedo, feeding a
 * 64-wide MLP of five BF16 weight matrices (64x64 x4, then 64->3 padded to 16 outputs, ReLU
 * between them, no biases; a constant-1 input stands in for the first layer's bias) that
 * predicts the outgoing radiance at a path vertex. Inference, the backward pass and Adam run
 * in the library's own kernels, the matrix products on the tensor cores (tcgen05, FP32
 * accumulation in tensor memory). Trained online, with the relative L2 loss
 * mean((y - t)^2 / (y^2 + 0.01)) (y held constant in the denominator), on the radiance that
 * training paths of the path tracer gather past each vertex.
 * ------------------------------------------------------------------------------------------ */
#define RBR_CACHE_LEVELS 16
#define RBR_CACHE_FEATURES 2
#define RBR_CACHE_INPUTS 64
#define RBR_CACHE_MLP_WEIGHTS (4 * 64 * 64 + 16 * 64) /* W0..W3 (64x64), W4 (16x64), row = output */
#define RBR_CACHE_RECORD_FLOATS 16

/* One cache query / training vertex (16 floats): world position[3], direction[3] (towards
 * the viewer, -ray.direction), ray-facing shading normal[3], roughness, diffuse albedo[3],
 * specular albedo[3]. */
typedef struct rbr_cache_record {
    float position[3];
    float direction[3];
    float normal[3];
    float roughness;
    float diffuse[3];
    float specular[3];
} rbr_cache_record;

typedef struct rbr_cache_config {
    int32_t log2_table_size;    /* hash-table entries per level = 2^this (default 19) */
    int32_t min_resolution;     /* grid resolution of level 0 (default 16) */
    int32_t max_resolution;     /* grid resolution of level 15 (default 2048) */
    float learning_rate;        /* Adam (default 1e-2) */
    float beta1, beta2, epsilon;/* Adam (0.9, 0.99, 1e-15) */
    uint32_t train_batch;       /* samples per optimiser step (default 16384) */
    uint32_t train_steps;       /* optimiser steps per rendered frame (default 4) */
    uint32_t train_paths;       /* training paths per rendered frame (default 65536) */
    uint32_t termination_depth; /* first vertex depth a path may end into the cache (default 1) */
    uint64_t seed;              /* initial weights */
    float bounds_min[3];        /* box the hash grid covers; min >= max on any axis: the */
    float bounds_max[3];        /* scene's bounded geometry, enlarged by 1% */
    uint32_t train_suffix;      /* k > 0 (default 2): training paths end into the cache k bounces
                                   after termination_depth, so their targets include the cache's
                                   own prediction (self-training); 0: they run to max_depth */
} rbr_cache_config;

typedef struct rbr_cache_info {
    uint32_t levels, table_size;
    uint32_t resolution[RBR_CACHE_LEVELS];
    uint32_t dense_levels;       /* bit l: level l is indexed densely ((res+1)^3 <= table_size) */
    uint32_t optimiser_steps;    /* Adam steps taken */
    float bounds_min[3], bounds_max[3];
    float last_loss;             /* training loss of the last optimiser step (rbr_cache_render) */
    uint32_t last_queries;       /* paths ended into the cache by the last frame */
    uint32_t last_train_records; /* training vertices gathered by the last frame */
} rbr_cache_info;

void rbr_cache_config_default(rbr_cache_config* out);
/* Creates (or re-creates) the context's cache with seeded initial parameters: Xavier-uniform
 * MLP weights, hash features uniform in [-1e-4, 1e-4]. Needs a scene unless the config gives
 * bounds. */
rbr_status rbr_cache_create(rbr_ctx* ctx, const rbr_cache_config* config);
void rbr_cache_destroy(rbr_ctx* ctx);
rbr_status rbr_cache_info_get(rbr_ctx* ctx, rbr_cache_info* out);
/* Parameters as 16-bit words: mlp = RBR_CACHE_MLP_WEIGHTS BF16 values, grid = levels x
 * table_size x 2 FP16 values (NULL to leave / skip). Setting also resets Adam's state. */
rbr_status rbr_cache_set_params(rbr_ctx* ctx, const uint16_t* mlp_bf16, const uint16_t* grid_f16);
rbr_status rbr_cache_get_params(rbr_ctx* ctx, uint16_t* mlp_bf16, uint16_t* grid_f16);
/* The FP32 gradient accumulators left by the last rbr_cache_train_host(apply = 0) call:
 * mlp = RBR_CACHE_MLP_WEIGHTS floats, grid = levels x table_size x 2 floats (NULL to skip). */
rbr_status rbr_cache_grads_get(rbr_ctx* ctx, float* mlp, float* grid);
/* Unit entry points on host buffers (each waits): the 64 network inputs of n records before
 * their BF16 rounding; the cache's prediction (RGB) for n records; one optimiser step on n
 * (record, target RGB) pairs (apply = 0: gradients only, kept for rbr_cache_grads_get).
 * loss (may be NULL) receives the mean relative L2 loss of the batch. */
rbr_status rbr_cache_encode_host(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, float* inputs);
rbr_status rbr_cache_infer_host(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, float* rgb);
rbr_status rbr_cache_train_host(rbr_ctx* ctx, uint32_t n, const rbr_cache_record* records, const float* targets,
                                int apply, float* loss);
/* Renders `frames` frames of params->samples_per_pixel samples each with the radiance cache:
 * a path ends into the cache at its first vertex of depth >= termination_depth reached by a
 * non-delta bounce on a non-delta material (its emission there is still added, then the
 * throughput times the cache's prediction replaces everything further), except about
 * train_paths paths per frame, which continue as the plain path tracer does (for train_suffix
 * more bounces, then they end into the cache as well; train_suffix 0: to the maximum depth) and
 * whose vertices, with the radiance gathered past each of them, train the cache for
 * train_steps Adam steps after the frame. A frame runs as two half-image waves in flight
 * ("pt.streams" 2) on a second stream that forks from and joins `stream`.
 * Frame f uses samples sample_offset + f*spp ... ; film_mean
 * (device) receives the mean over all frames, film_m2 (device or NULL, with
 * RBR_RENDER_SECOND_MOMENT) the sum of squared sample values. Asynchronous on `stream`. */
rbr_status rbr_cache_render(rbr_ctx* ctx, const rbr_camera* camera, const rbr_render_params* params,
                            uint32_t frames, int train, float* film_mean, float* film_m2, void* stream);

/* ------------------------------------------------------------------------------------------
 * Batched request loop (no reference counterpart). Requests of uneven resolution, samples
 * per pixel, scene and integrator are packed into waves of the wavefront path tracer: a wave
 * holds pixel ranges ("segments") of several requests of one scene, each path reading its
 * request's camera, random-number key and parameters from a segment table in device memory.
 * The launch sequence of a wave therefore depends only on (scene, integrator, depth, grid)
 * and is captured once as a CUDA graph and replayed. Scenes, BVHs, films and caches stay
 * resident; requests are admitted into a wave while its path-state memory budget allows (a
 * request larger than a wave is split over several). rbr_batch_autotune picks the wave size
 * and the grid by timing the pending requests.
 * ------------------------------------------------------------------------------------------ */
typedef struct rbr_batch rbr_batch;

typedef struct rbr_batch_config {
    uint64_t path_memory_bytes; /* budget for one wave's path state (default 2 GiB) */
    uint32_t wave_paths;        /* paths per wave; 0: the budget decides (at most 2^23) */
    uint32_t blocks_per_sm;     /* grid of the wavefront kernels = this x SMs (default 8) */
    int32_t use_graphs;         /* replay each wave shape from a captured CUDA graph (default 1) */
    uint32_t waves_in_flight;   /* 1, or 2 (default; 0 means 2): waves alternate between two
                                   path-buffer sets and streams, each set within the budget */
    uint32_t persistent;        /* 1: one cooperative launch renders every wave of a run (all
                                   its stages, grid barriers between them; with two waves in
                                   flight the grid's halves take alternate waves) when no request
                                   uses the radiance cache and the run has at most 16 scenes; 0
                                   (default): one captured graph per wave shape */
    uint32_t barrier_timeout_us; /* persistent run: longest wait of a block at a grid barrier, in
                                   microseconds, before the run gives up with RBR_ERR_DEVICE_TIMEOUT
                                   (default 2,000,000; 0 means the default) */
} rbr_batch_config;

typedef struct rbr_request {
    uint32_t scene;             /* id from rbr_batch_add_scene */
    rbr_camera camera;
    rbr_render_params params;   /* spp, max_depth (>= 1), use_nee, use_mis, seed, sample_offset;
                                   flags: 0 or RBR_RENDER_VOLUMETRIC */
    int32_t use_cache;          /* end paths into the scene's radiance cache (rbr_batch_cache_create) */
    int32_t train_cache;        /* with use_cache: also train it on this request's paths */
    float* film;                /* device pointer, width*height*3 floats: per-pixel mean */
    uint32_t arrival_us;        /* arrival after the start of rbr_batch_run, in microseconds (at
                                   most 600 s): no wave holding the request starts before it, and
                                   its latency counts from it. 0: present at the start */
    uint32_t reserved;          /* 0 */
} rbr_request;

typedef struct rbr_request_stats {
    float start_ms;             /* from its arrival to the start of its first wave (queueing) */
    float latency_ms;           /* from its arrival to the end of its last wave (device clock) */
    uint32_t waves;             /* waves it was spread over */
    uint32_t segments;
    uint64_t paths;
} rbr_request_stats;

typedef struct rbr_batch_stats {
    float milliseconds;         /* device time of the last rbr_batch_run */
    uint32_t requests, waves, segments;
    uint32_t graphs_captured, graph_launches, kernel_launches;
    uint32_t wave_paths, blocks_per_sm;
    uint32_t persistent_launches; /* cooperative launches that rendered the run (0 or 1) */
    uint64_t paths;
} rbr_batch_stats;

void rbr_batch_config_default(rbr_batch_config* out);
/* The batch uses `ctx` (device, path-state buffers) and owns its scenes. */
rbr_status rbr_batch_create(rbr_ctx* ctx, const rbr_batch_config* config, rbr_batch** out);
void rbr_batch_destroy(rbr_batch* batch);
const char* rbr_batch_last_error(const rbr_batch* batch);
rbr_status rbr_batch_add_scene(rbr_batch* batch, const rbr_scene_desc* desc, uint32_t* scene_id);
/* A scene sharing `base_scene`'s geometry and BVH on the device (no rebuild, no copy) with its
 * own materials (as many as the base has), lights and medium (NULL for none). */
rbr_status rbr_batch_add_scene_variant(rbr_batch* batch, uint32_t base_scene, const rbr_material* materials,
                                       uint32_t num_materials, const rbr_light* lights, uint32_t num_lights,
                                       const rbr_medium* medium, uint32_t* scene_id);
rbr_status rbr_batch_cache_create(rbr_batch* batch, uint32_t scene_id, const rbr_cache_config* config);
/* Queues a request; it is rendered by the next rbr_batch_run. */
rbr_status rbr_batch_submit(rbr_batch* batch, const rbr_request* request, uint32_t* request_id);
/* Optional, for a queued request: the next rbr_batch_run also copies its film to `host_film`
 * (width*height*3 floats; page-locked memory for the copy to run asynchronously) on the stream
 * of its last wave, right after that wave, so the copy overlaps the waves after it. The copy is
 * complete when the stream given to rbr_batch_run is. */
rbr_status rbr_batch_set_host_film(rbr_batch* batch, uint32_t request_id, float* host_film);
/* Renders every queued request (asynchronous on `stream`); the queue is then empty. */
rbr_status rbr_batch_run(rbr_batch* batch, void* stream);
/* Per-request and whole-run timings of the last run (wait for it). */
rbr_status rbr_batch_request_stats(rbr_batch* batch, uint32_t request_id, rbr_request_stats* out);
rbr_status rbr_batch_stats_get(rbr_batch* batch, rbr_batch_stats* out);
/* Renders the queued requests once per candidate (wave size x blocks per SM), keeps the
 * fastest in the batch's configuration and leaves the requests queued. Waits. */
rbr_status rbr_batch_autotune(rbr_batch* batch, void* stream);

/* HenyeyGreensteinPhase::evaluate (src/materials/phase_function.cpp:17-21) for n (wo, wi). */
rbr_status rbr_phase_eval_host(rbr_ctx* ctx, float g, uint32_t n, const float* wo, const float* wi, float* out);
/* HenyeyGreensteinPhase::sample (phase_function.cpp:23-41) for n (wo, u1, u2); out: wi[3]. */
rbr_status rbr_phase_sample_host(rbr_ctx* ctx, float g, uint32_t n, const float* wo, const float* u, float* out);
/* HomogeneousMedium::sampleDistance (src/materials/medium.cpp:9-32) for n (maxDist, u);
 * out: 5 floats each: t (0 without scattering), weight[3], scattered (0/1). */
rbr_status rbr_medium_sample_host(rbr_ctx* ctx, const rbr_medium* medium, uint32_t n, const float* max_dist,
                                  const float* u, float* out);
/* Measurement (no reference counterpart): read bandwidth of an L2-resident buffer of `bytes`
 * (4 KiB..1 GiB), read `passes` times per launch (1..1000) with L2-only loads; the best of 5
 * launches in GB/s. The denominator of the traversal kernels' L2 roofline. */
rbr_status rbr_l2_read_bandwidth(rbr_ctx* ctx, uint64_t bytes, uint32_t passes, double* gb_per_s);

/* ------------------------------------------------------------------------------------------
 * Meshes and film export.
 * ------------------------------------------------------------------------------------------ */
typedef struct rbr_mesh rbr_mesh;

/* ObjImporter::load / ::parse (src/io/obj_importer.cpp) followed by TriangleMesh::toPrimitives
 * (src/geometry/mesh.cpp:14-38): the mesh as rbr_scene_desc triangle arrays. On failure the
 * message is written to `error` (may be NULL). */
rbr_status rbr_mesh_load_obj(const char* path, rbr_mesh** out, char* error, size_t error_len);
rbr_status rbr_mesh_parse_obj(const char* text, size_t length, rbr_mesh** out, char* error, size_t error_len);
uint32_t rbr_mesh_triangles(const rbr_mesh* mesh);
/* 9 floats per triangle (v0, v1, v2) */
const float* rbr_mesh_triangle_vertices(const rbr_mesh* mesh);
/* 9 floats per triangle of unit vertex normals when the file gives a normal for every corner
 * (as Triangle's normal constructor normalises them), else NULL */
const float* rbr_mesh_triangle_normals(const rbr_mesh* mesh);
void rbr_mesh_destroy(rbr_mesh* mesh);

/* Film::toRGB8 (tonemap = 0) and Film::toRGB8ToneMapped (tonemap != 0; exposure, then Reinhard)
 * (src/core/film.cpp:34-62) of a film of per-pixel means (width*height*3 floats) into
 * width*height*3 bytes: device pointers, asynchronous on `stream`. */
rbr_status rbr_film_to_rgb8(rbr_ctx* ctx, const float* film, int32_t width, int32_t height, float exposure, float gamma,
                            int tonemap, uint8_t* out, void* stream);
/* The same on host buffers; waits. */
rbr_status rbr_film_to_rgb8_host(rbr_ctx* ctx, const float* film, int32_t width, int32_t height, float exposure,
                                 float gamma, int tonemap, uint8_t* out);

/* Size of the fixed scratch array used by rbr_render_noalloc (16 MiB). */
#define RBR_NOALLOC_SCRATCH_BYTES (16u << 20)

/* rbr_render without any device allocation (no counterpart in the reference).
 *
 * rbr_render allocates its per-path working memory on first use and whenever a larger image
 * needs more. Some callers can't let it: an application that reserves the GPU's memory for
 * its own pool up front and allows no other allocation, or a frame loop that must never
 * stall on cudaMalloc/cudaFree (they can synchronise the whole device). This entry point
 * keeps the path state in a fixed RBR_NOALLOC_SCRATCH_BYTES array compiled into the library
 * (every GPU that loads the library holds it until the process exits) and renders in as many
 * waves as that array requires, so it calls no cudaMalloc, cudaFree or allocating routine.
 *
 * Arguments as rbr_render; film_mean is a device pointer (width*height*3 floats, the
 * per-pixel mean) and params->flags must be 0 (no second moment, no corrected MIS). The
 * result equals rbr_render's for the same parameters. A sample count per pixel whose wave
 * state does not fit the array (about 116,000 samples per pixel with one light, fewer with
 * more lights) is rejected with RBR_ERR_INVALID_ARGUMENT and a message giving the limit.
 * The scene must have been uploaded with rbr_scene_upload beforehand; render statistics
 * (rbr_render_stats_get) are not updated.
 *
 * Every call looks up the array's device address on the context's device (the first lookup
 * on a device loads the library's device code there if nothing has yet, so make the first
 * call on a device before any stream capture); a device reset between calls is therefore
 * harmless. All calls in the process share the one array per device and it keeps the
 * previous call's contents, so calls whose work overlaps on the GPU (different streams or
 * contexts on the same device) race and corrupt each other: serialise them. */
rbr_status rbr_render_noalloc(rbr_ctx* ctx, const rbr_camera* camera, const rbr_render_params* params,
                              float* film_mean, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RBR_B200_H */
