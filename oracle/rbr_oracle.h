/*
 * rbr_oracle.h — CPU restatement of the reference's path-tracing hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the GPU library is compared with; nothing in
 * the product links, loads or calls it. It restates, operation for operation and in the same
 * floating-point order, the reference's C++ code for:
 *   ray/primitive intersection     src/geometry/{triangle,quad,sphere,plane}.cpp
 *   brute-force closest / any hit  tests/test_accelerators.cpp:58-74
 *   materials and BSDF lobes       src/materials/{material,mixture_bsdf,lambertian_bsdf,
 *                                  specular_bsdf,microfacet_bsdf}.cpp, include/render/materials/fresnel.h
 *   light sampling                 src/lighting/{area_light,point_light}.cpp
 *   camera rays                    src/camera/{camera,thin_lens_camera}.cpp, perspective_intrinsics.h
 *   the path integrator            src/renderers/path_tracing_integrator.cpp, integrator.cpp
 *   the volumetric path integrator src/renderers/volumetric_path_integrator.cpp,
 *                                  src/materials/{medium,phase_function}.cpp
 * with one deliberate difference: random numbers come from the counter-based generator that
 * the GPU library uses (Philox-4x32-10 keyed by the seed, counters = pixel, sample, bounce,
 * purpose), so GPU and oracle draw identical numbers for identical (pixel, sample, bounce).
 * Its pinning against the reference itself (oracle/_ref) is in tests/test_oracle_pin.py.
 * Scene descriptions use the rbr_scene_desc layout of include/rbr_b200.h.
 */
#ifndef RBR_ORACLE_H
#define RBR_ORACLE_H

#include <stdint.h>

#include "rbr_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_scene orc_scene;

orc_scene* orc_scene_create(const rbr_scene_desc* desc);
void orc_scene_destroy(orc_scene* s);

/* Brute-force closest hit / any hit over the primitives in id order. */
void orc_trace_closest(const orc_scene* s, const rbr_ray* rays, int64_t n, rbr_hit* hits, int nthreads);
void orc_trace_any(const orc_scene* s, const rbr_ray* rays, int64_t n, uint8_t* occluded, int nthreads);

/* Material::createBSDF + evaluate/pdf and sample, batched (local shading frame). */
void orc_bsdf_eval(const rbr_material* m, int64_t n, const float* wo, const float* wi, float* f, float* pdf,
                   uint32_t* info);
void orc_bsdf_sample(const rbr_material* m, int64_t n, const float* wo, const float* u, float* out);

/* Light::sample: out = wi[3], Li[3], pdf, distance, isDelta per sample. */
void orc_light_sample(const rbr_light* l, int64_t n, const float* points, const float* u, float* out);

/* Camera::generateRay: samples = filmX, filmY, lensU, lensV; out = origin[3], direction[3]. */
void orc_camera_rays(const rbr_camera* c, int64_t n, const float* samples, float* out);

float orc_power_heuristic(int nf, float fpdf, int ng, float gpdf);

/* HenyeyGreensteinPhase::evaluate / sample (phase_function.cpp:17-41). */
float orc_hg_eval(float g, const float wo[3], const float wi[3]);
void orc_hg_sample(float g, int64_t n, const float* wo, const float* u, float* out);

/* Philox-4x32-10 block: counters c[4], key k[2] -> out[4]. */
void orc_philox(const uint32_t c[4], const uint32_t k[2], uint32_t out[4]);

/* Path tracer with the GPU library's random-number streams. For every pixel:
 * sum[3] += L and sumsq[3] += L*L over samples sample_offset .. sample_offset+spp-1, and
 * mean[3] = (float sum over the samples) / spp as Film::addSample receives it.
 * mean may be NULL; sum and sumsq may be NULL. */
void orc_render(const orc_scene* s, const rbr_camera* c, const rbr_render_params* p, float* mean, double* sum,
                double* sumsq, int nthreads);

/* Radiance of one path (pixel, sample) for debugging (returns L[3]). */
void orc_path(const orc_scene* s, const rbr_camera* c, const rbr_render_params* p, int x, int y, uint32_t sample,
              float* L);

#ifdef __cplusplus
}
#endif

#endif
