// Test infrastructure: a C interface over the UNMODIFIED Ray-Based-Rendering library.
//
// oracle/Makefile compiles this file together with the reference's own sources into
// oracle/_ref/librbr_ref.so. Only the tests, the golden-fixture script and the CPU-baseline
// arm of bench.py load it; the product never does. Every function builds reference objects
// through the reference's public API and calls the reference's code for the answer:
//   scenes       render::Scene + Triangle/Sphere/Quad/Plane + Material + AreaLight/PointLight
//   ray queries  Scene::intersect / intersectP (src/scene/scene.cpp:30-36) through the BVH
//                (src/acceleration/bvh.cpp), and the brute-force loop of
//                tests/test_accelerators.cpp:58-74
//   materials    Material::createBSDF (src/materials/material.cpp:69-108) + BSDF::evaluate/pdf/sample
//   lights       AreaLight::sample (src/lighting/area_light.cpp:13-39), PointLight::sample
//   cameras      PinholeCamera / ThinLensCamera::generateRay (src/camera/*.cpp)
//   rendering    Integrator::render (src/renderers/integrator.cpp:7-50) and Li of the
//                path tracer (src/renderers/path_tracing_integrator.cpp:5-138)
// Scene descriptions use the rbr_scene_desc layout of include/rbr_b200.h, so the same arrays
// feed the GPU library and the reference.

#include "rbr_b200.h"

#include "render/acceleration/accelerator_factory.h"
#include "render/camera/camera_extrinsics.h"
#include "render/camera/perspective_intrinsics.h"
#include "render/camera/pinhole_camera.h"
#include "render/camera/thin_lens_camera.h"
#include "render/core/film.h"
#include "render/core/sampler.h"
#include "render/geometry/plane.h"
#include "render/geometry/quad.h"
#include "render/geometry/sphere.h"
#include "render/geometry/triangle.h"
#include "render/lighting/area_light.h"
#include "render/lighting/point_light.h"
#include "render/materials/material.h"
#include "render/materials/medium.h"
#include "render/renderers/path_tracing_integrator.h"
#include "render/renderers/volumetric_path_integrator.h"
#include "render/scene/scene.h"

#include <omp.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <unordered_map>
#include <vector>

using namespace render;

namespace {

struct RefScene {
    Scene scene;
    std::unordered_map<const Primitive*, uint32_t> index;  // primitive -> position in primitives()
    std::vector<const Primitive*> ordered;                   // primitives() as raw pointers
};

Vec3 v3(const float* p) { return Vec3(p[0], p[1], p[2]); }

void put3(float* out, const Vec3& v) {
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
}

Material toMaterial(const rbr_material& m) {
    Material r;
    r.baseColor = v3(m.base_color);
    r.metallic = m.metallic;
    r.roughness = m.roughness;
    r.ior = m.ior;
    r.transmission = m.transmission;
    r.emission = v3(m.emission);
    return r;
}

Ray toRay(const rbr_ray& r) {
    Ray ray;  // set the members directly: the direction is used exactly as given
    ray.origin = v3(r.origin);
    ray.direction = v3(r.direction);
    ray.tMax = r.tmax;
    return ray;
}

int threads(int n) { return n > 0 ? n : omp_get_max_threads(); }

}  // namespace

extern "C" {

int ref_max_threads(void) { return omp_get_max_threads(); }

// Builds a render::Scene whose primitives() follow the ids of the description and whose
// accelerator is `accel_type` (0 BVH, 1 grid, 2 kd-tree, 3 octree; AcceleratorType order).
void* ref_scene_create(const rbr_scene_desc* d, int accel_type) {
    auto rs = std::make_unique<RefScene>();
    Scene& scene = rs->scene;
    std::vector<Material*> mats;
    for (uint32_t i = 0; i < d->num_materials; ++i) {
        mats.push_back(scene.addMaterial(std::make_unique<Material>(toMaterial(d->materials[i]))));
    }
    const uint32_t total = d->num_triangles + d->num_spheres + d->num_quads + d->num_planes;
    std::vector<std::unique_ptr<Primitive>> slots(total);
    uint32_t next = 0;
    auto idOf = [&](const uint32_t* ids, uint32_t i) { return ids ? ids[i] : next + i; };
    for (uint32_t i = 0; i < d->num_triangles; ++i) {
        const float* v = d->triangle_vertices + 9 * i;
        std::unique_ptr<Triangle> t;
        if (d->triangle_normals) {
            const float* n = d->triangle_normals + 9 * i;
            t = std::make_unique<Triangle>(v3(v), v3(v + 3), v3(v + 6), v3(n), v3(n + 3), v3(n + 6),
                                           mats[d->triangle_materials[i]]);
            t->n0 = v3(n);  // keep the caller's unit normals bit for bit
            t->n1 = v3(n + 3);
            t->n2 = v3(n + 6);
        } else {
            t = std::make_unique<Triangle>(v3(v), v3(v + 3), v3(v + 6), mats[d->triangle_materials[i]]);
        }
        slots[idOf(d->triangle_ids, i)] = std::move(t);
    }
    next += d->num_triangles;
    for (uint32_t i = 0; i < d->num_spheres; ++i) {
        const float* s = d->spheres + 4 * i;
        slots[idOf(d->sphere_ids, i)] = std::make_unique<Sphere>(v3(s), s[3], mats[d->sphere_materials[i]]);
    }
    next += d->num_spheres;
    for (uint32_t i = 0; i < d->num_quads; ++i) {
        const float* q = d->quads + 9 * i;
        slots[idOf(d->quad_ids, i)] =
            std::make_unique<Quad>(v3(q), v3(q + 3), v3(q + 6), mats[d->quad_materials[i]]);
    }
    next += d->num_quads;
    for (uint32_t i = 0; i < d->num_planes; ++i) {
        const float* p = d->planes + 4 * i;
        auto pl = std::make_unique<Plane>(v3(p), p[3], mats[d->plane_materials[i]]);
        pl->normal = v3(p);  // the caller's unit normal, bit for bit
        slots[idOf(d->plane_ids, i)] = std::move(pl);
    }
    for (auto& s : slots) {
        if (!s) return nullptr;  // ids were not a permutation
        scene.addPrimitive(std::move(s));
    }
    for (uint32_t i = 0; i < d->num_lights; ++i) {
        const rbr_light& l = d->lights[i];
        if (l.type == RBR_LIGHT_AREA) {
            scene.addLight(std::make_unique<AreaLight>(v3(l.position), v3(l.u), v3(l.v), v3(l.color), l.intensity));
        } else {
            scene.addLight(std::make_unique<PointLight>(v3(l.position), v3(l.color), l.intensity));
        }
    }
    scene.backgroundColor = v3(d->background);
    if (d->medium) {
        scene.setMedium(std::make_unique<HomogeneousMedium>(v3(d->medium->sigma_a), v3(d->medium->sigma_s), d->medium->g));
    }
    scene.setAcceleratorType(static_cast<AcceleratorType>(accel_type));
    scene.buildAccelerator();
    for (uint32_t i = 0; i < scene.primitives().size(); ++i) {
        rs->index[scene.primitives()[i].get()] = i;
        rs->ordered.push_back(scene.primitives()[i].get());
    }
    return rs.release();
}

void ref_scene_destroy(void* s) { delete static_cast<RefScene*>(s); }

// Adds a homogeneous medium (SceneBuilder::medium, src/scene/scene_builder.cpp:97-100).
void ref_scene_set_medium(void* s, const float sigma_a[3], const float sigma_s[3], float g) {
    static_cast<RefScene*>(s)->scene.setMedium(
        std::make_unique<HomogeneousMedium>(v3(sigma_a), v3(sigma_s), g));
}

// HenyeyGreensteinPhase::evaluate for n (wo, wi) pairs.
void ref_hg_eval(float g, int64_t n, const float* wo, const float* wi, float* out) {
    const HenyeyGreensteinPhase ph(g);
    for (int64_t i = 0; i < n; ++i) out[i] = ph.evaluate(v3(wo + 3 * i), v3(wi + 3 * i));
}

// HenyeyGreensteinPhase::sample for n (wo, u1, u2).
void ref_hg_sample(float g, int64_t n, const float* wo, const float* u, float* out) {
    const HenyeyGreensteinPhase ph(g);
    for (int64_t i = 0; i < n; ++i) put3(out + 3 * i, ph.sample(v3(wo + 3 * i), u[2 * i], u[2 * i + 1]));
}

// HomogeneousMedium::sampleDistance for n (maxDist, u): out = t, weight[3], scattered.
void ref_medium_sample(const rbr_medium* m, int64_t n, const float* max_dist, const float* u, float* out) {
    const HomogeneousMedium med(v3(m->sigma_a), v3(m->sigma_s), m->g);
    const Ray ray(Vec3(0.0f), Vec3(0.0f, 0.0f, 1.0f));
    for (int64_t i = 0; i < n; ++i) {
        float t = 0.0f;
        Color w;
        const bool sc = med.sampleDistance(ray, max_dist[i], u[i], t, w);
        out[5 * i] = sc ? t : 0.0f;
        put3(out + 5 * i + 1, w);
        out[5 * i + 4] = sc ? 1.0f : 0.0f;
    }
}

// Film::toRGB8 / toRGB8ToneMapped of a film whose pixels hold `film` (one sample each).
void ref_film_rgb8(const float* film, int w, int h, float exposure, float gamma, int tonemap, uint8_t* out) {
    Film f(w, h);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) f.addSample(x, y, v3(film + 3 * (static_cast<size_t>(y) * w + x)));
    const std::vector<unsigned char> d = tonemap ? f.toRGB8ToneMapped(exposure, gamma) : f.toRGB8(gamma);
    std::memcpy(out, d.data(), d.size());
}

// Closest hit through the scene's accelerator (Scene::intersect).
void ref_trace_closest(void* s, const rbr_ray* rays, int64_t n, rbr_hit* hits, int nthreads) {
    const RefScene& rs = *static_cast<RefScene*>(s);
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads(nthreads))
    for (int64_t i = 0; i < n; ++i) {
        Ray ray = toRay(rays[i]);
        SurfaceInteraction isect;
        if (rs.scene.intersect(ray, isect)) {
            hits[i].prim = rs.index.at(isect.primitive);
            hits[i].t = isect.t;
        } else {
            hits[i].prim = RBR_MISS;
            hits[i].t = 0.0f;
        }
    }
}

// Any hit through the scene's accelerator (Scene::intersectP).
void ref_trace_any(void* s, const rbr_ray* rays, int64_t n, uint8_t* occluded, int nthreads) {
    const RefScene& rs = *static_cast<RefScene*>(s);
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads(nthreads))
    for (int64_t i = 0; i < n; ++i) {
        occluded[i] = rs.scene.intersectP(toRay(rays[i])) ? 1 : 0;
    }
}

// Brute force over primitives() in order, as tests/test_accelerators.cpp:58-67 does.
void ref_brute_closest(void* s, const rbr_ray* rays, int64_t n, rbr_hit* hits, int nthreads) {
    const RefScene& rs = *static_cast<RefScene*>(s);
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads(nthreads))
    for (int64_t i = 0; i < n; ++i) {
        Ray ray = toRay(rays[i]);
        SurfaceInteraction isect;
        bool hit = false;
        for (const Primitive* p : rs.ordered) {
            if (p->intersect(ray, isect)) hit = true;
        }
        hits[i].prim = hit ? rs.index.at(isect.primitive) : RBR_MISS;
        hits[i].t = hit ? isect.t : 0.0f;
    }
}

// Brute-force any hit (tests/test_accelerators.cpp:69-74).
void ref_brute_any(void* s, const rbr_ray* rays, int64_t n, uint8_t* occluded, int nthreads) {
    const RefScene& rs = *static_cast<RefScene*>(s);
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads(nthreads))
    for (int64_t i = 0; i < n; ++i) {
        const Ray ray = toRay(rays[i]);
        uint8_t hit = 0;
        for (const Primitive* p : rs.ordered) {
            if (p->intersectP(ray)) {
                hit = 1;
                break;
            }
        }
        occluded[i] = hit;
    }
}

// Surface data of the closest hit: point, ray-facing normal, outward normal, frontFace.
// out[i*10 + 0..2] point, 3..5 normal, 6..8 outwardNormal, 9 frontFace (1/0).
void ref_hit_details(void* s, const rbr_ray* rays, int64_t n, float* out) {
    const RefScene& rs = *static_cast<RefScene*>(s);
    for (int64_t i = 0; i < n; ++i) {
        Ray ray = toRay(rays[i]);
        SurfaceInteraction isect;
        float* o = out + 10 * i;
        if (rs.scene.intersect(ray, isect)) {
            put3(o, isect.point);
            put3(o + 3, isect.normal);
            put3(o + 6, isect.outwardNormal());
            o[9] = isect.frontFace ? 1.0f : 0.0f;
        } else {
            std::memset(o, 0, 10 * sizeof(float));
        }
    }
}

// World bounds of the accelerator (Accelerator::worldBounds).
void ref_world_bounds(void* s, float out_min[3], float out_max[3]) {
    const BoundingBox b = static_cast<RefScene*>(s)->scene.worldBounds();
    put3(out_min, b.pMin);
    put3(out_max, b.pMax);
}

// Material::createBSDF then evaluate + pdf for n (wo, wi) pairs in the local frame.
// info[0] = isDelta, info[1] = BSDFType bits, info[2] = lobe count is not exposed (0).
void ref_bsdf_eval(const rbr_material* m, int64_t n, const float* wo, const float* wi, float* f,
                   float* pdf, uint32_t* info) {
    const Material mat = toMaterial(*m);
    auto bsdf = mat.createBSDF();
    for (int64_t i = 0; i < n; ++i) {
        const Color c = bsdf->evaluate(v3(wo + 3 * i), v3(wi + 3 * i));
        put3(f + 3 * i, c);
        pdf[i] = bsdf->pdf(v3(wo + 3 * i), v3(wi + 3 * i));
    }
    if (info) {
        info[0] = bsdf->isDelta() ? 1u : 0u;
        info[1] = static_cast<uint32_t>(bsdf->type());
    }
}

// Material::createBSDF then sample for n (wo, u1, u2).
// out: wi[3], f[3], pdf, isDelta per sample (8 floats).
void ref_bsdf_sample(const rbr_material* m, int64_t n, const float* wo, const float* u, float* out) {
    const Material mat = toMaterial(*m);
    auto bsdf = mat.createBSDF();
    for (int64_t i = 0; i < n; ++i) {
        const BSDFSample s = bsdf->sample(v3(wo + 3 * i), u[2 * i], u[2 * i + 1]);
        float* o = out + 8 * i;
        put3(o, s.wi);
        put3(o + 3, s.f);
        o[6] = s.pdf;
        o[7] = s.isDelta ? 1.0f : 0.0f;
    }
}

// Light::sample at surface points (only isect.point is read by Area/Point lights).
// out: wi[3], Li[3], pdf, distance, isDelta per sample (9 floats).
void ref_light_sample(const rbr_light* l, int64_t n, const float* points, const float* u, float* out) {
    std::unique_ptr<Light> light;
    if (l->type == RBR_LIGHT_AREA) {
        light = std::make_unique<AreaLight>(v3(l->position), v3(l->u), v3(l->v), v3(l->color), l->intensity);
    } else {
        light = std::make_unique<PointLight>(v3(l->position), v3(l->color), l->intensity);
    }
    for (int64_t i = 0; i < n; ++i) {
        SurfaceInteraction isect;
        isect.point = v3(points + 3 * i);
        const LightSample s = light->sample(isect, u[2 * i], u[2 * i + 1]);
        float* o = out + 9 * i;
        put3(o, s.wi);
        put3(o + 3, s.Li);
        o[6] = s.pdf;
        o[7] = s.distance;
        o[8] = s.isDelta ? 1.0f : 0.0f;
    }
}

// The camera the reference factory builds (src/config/render_factory.cpp:16-43):
// PerspectiveCamera(width, height, position, lookAt, up, fov) with lookAt extrinsics and
// fromVerticalFov intrinsics, as an rbr_camera.
void ref_camera_setup(int width, int height, const float position[3], const float look_at[3],
                      const float up[3], float fov, float lens_radius, float focal_distance,
                      rbr_camera* out) {
    const CameraExtrinsics e = CameraExtrinsics::lookAt(v3(position), v3(look_at), v3(up));
    const PerspectiveIntrinsics k = PerspectiveIntrinsics::fromVerticalFov(width, height, fov);
    out->width = width;
    out->height = height;
    out->model = lens_radius > 0.0f ? RBR_CAMERA_THIN_LENS : RBR_CAMERA_PINHOLE;
    put3(out->position, e.position);
    put3(out->forward, e.forward);
    put3(out->right, e.right);
    put3(out->up, e.up);
    out->fx = k.fx;
    out->fy = k.fy;
    out->cx = k.cx;
    out->cy = k.cy;
    out->lens_radius = lens_radius;
    out->focal_distance = focal_distance;
}

namespace {
std::unique_ptr<Camera> makeCamera(const rbr_camera& c) {
    CameraExtrinsics e;
    e.position = v3(c.position);
    e.forward = v3(c.forward);
    e.right = v3(c.right);
    e.up = v3(c.up);
    const PerspectiveIntrinsics k(c.fx, c.fy, c.cx, c.cy);
    if (c.model == RBR_CAMERA_THIN_LENS) {
        return std::make_unique<ThinLensCamera>(c.width, c.height, e, k, c.lens_radius, c.focal_distance);
    }
    return std::make_unique<PinholeCamera>(c.width, c.height, e, k);
}

IntegratorConfig toConfig(const rbr_render_params& p) {
    IntegratorConfig cfg;
    cfg.maxDepth = p.max_depth;
    cfg.samplesPerPixel = p.samples_per_pixel;
    cfg.useNEE = p.use_nee != 0;
    cfg.useMIS = p.use_mis != 0;
    return cfg;
}
}  // namespace

// Camera::generateRay for n CameraSamples (filmX, filmY, lensU, lensV per sample).
// out: origin[3], direction[3] per ray.
void ref_camera_rays(const rbr_camera* c, int64_t n, const float* samples, float* out) {
    auto cam = makeCamera(*c);
    for (int64_t i = 0; i < n; ++i) {
        const float* s = samples + 4 * i;
        const Ray r = cam->generateRay(CameraSample{s[0], s[1], s[2], s[3], 0.0f});
        put3(out + 6 * i, r.origin);
        put3(out + 6 * i + 3, r.direction);
    }
}

// The reference's own render loop: Integrator::render with the path tracer (OpenMP over rows,
// per-row reseeding y*width). film_out receives W*H*3 floats of Film::getPixel.
// volumetric != 0 selects VolumetricPathIntegrator (needs a medium on the scene).
void ref_render(void* s, const rbr_camera* c, const rbr_render_params* p, int volumetric, float* film_out,
                int nthreads) {
    const RefScene& rs = *static_cast<RefScene*>(s);
    auto cam = makeCamera(*c);
    Film film(c->width, c->height);
    omp_set_num_threads(threads(nthreads));
    if (volumetric) {
        VolumetricPathIntegrator integrator(toConfig(*p), VolumeConfig());
        integrator.render(rs.scene, *cam, film);
    } else {
        PathTracingIntegrator integrator(toConfig(*p));
        integrator.render(rs.scene, *cam, film);
    }
    for (int y = 0; y < c->height; ++y) {
        for (int x = 0; x < c->width; ++x) {
            put3(film_out + 3 * (static_cast<size_t>(y) * c->width + x), film.getPixel(x, y));
        }
    }
}

// Per-pixel sample statistics from the reference integrator's public Li, with independent
// seeds: the same per-sample work as Integrator::render (src/renderers/integrator.cpp:20-33),
// but each row of batch `batch` is seeded with (batch + 1) * 0x9E3779B97F4A7C15 + y*width so
// that batches are independent. sum / sumsq: W*H*3 floats, accumulated in double.
void ref_render_moments(void* s, const rbr_camera* c, const rbr_render_params* p, int volumetric,
                        uint64_t batch, double* sum, double* sumsq, int nthreads) {
    const RefScene& rs = *static_cast<RefScene*>(s);
    auto cam = makeCamera(*c);
    std::unique_ptr<Integrator> integrator;
    if (volumetric) {
        integrator = std::make_unique<VolumetricPathIntegrator>(toConfig(*p), VolumeConfig());
    } else {
        integrator = std::make_unique<PathTracingIntegrator>(toConfig(*p));
    }
    const int W = c->width, H = c->height, spp = p->samples_per_pixel;
#pragma omp parallel num_threads(threads(nthreads))
    {
        UniformSampler sampler;
#pragma omp for schedule(dynamic, 4)
        for (int y = 0; y < H; ++y) {
            sampler.setSeed((batch + 1) * 0x9E3779B97F4A7C15ull + static_cast<uint64_t>(y) * W);
            for (int x = 0; x < W; ++x) {
                double* ps = sum + 3 * (static_cast<size_t>(y) * W + x);
                double* pq = sumsq + 3 * (static_cast<size_t>(y) * W + x);
                for (int k = 0; k < spp; ++k) {
                    auto [jx, jy] = sampler.get2D();
                    const float lu = sampler.get1D();
                    const float lv = sampler.get1D();
                    const CameraSample cs{x + jx, y + jy, lu, lv, 0.0f};
                    const Ray ray = cam->generateRay(cs);
                    const Color L = integrator->Li(ray, rs.scene, sampler);
                    ps[0] += L.x;
                    ps[1] += L.y;
                    ps[2] += L.z;
                    pq[0] += static_cast<double>(L.x) * L.x;
                    pq[1] += static_cast<double>(L.y) * L.y;
                    pq[2] += static_cast<double>(L.z) * L.z;
                }
            }
        }
    }
}

// sampling::powerHeuristic (include/render/core/sampler.h:137-149).
float ref_power_heuristic(int nf, float fpdf, int ng, float gpdf) {
    return sampling::powerHeuristic(nf, fpdf, ng, gpdf);
}

// sampling::Frame(n): tangent, bitangent (include/render/core/sampler.h:104-118).
void ref_frame(const float n[3], float tangent[3], float bitangent[3]) {
    const sampling::Frame f(v3(n));
    put3(tangent, f.tangent);
    put3(bitangent, f.bitangent);
}

}  // extern "C"
