/*
 * rbr_oracle.c — CPU restatement of the reference's path-tracing hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see rbr_oracle.h). Compiled by oracle/Makefile with
 * -std=c11 -ffp-contract=off so that every float operation rounds on its own, as the
 * reference's ISO C++17 build does; expressions keep the reference's evaluation order.
 * std::min / std::max semantics (NaN handling included) are restated as omin / omax.
 */
#include "rbr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* include/render/core/common.h:20-26 */
#define ORC_PI 3.14159265358979323846f
static const float TWO_PI = 2.0f * ORC_PI;
static const float INV_PI = 1.0f / ORC_PI;
#define ORC_EPS 1e-4f

/* std::min / std::max / render::clamp (common.h:38-40) */
static inline float omin(float a, float b) { return (b < a) ? b : a; }
static inline float omax(float a, float b) { return (a < b) ? b : a; }
static inline float oclamp(float v, float lo, float hi) { return omax(lo, omin(hi, v)); }

/* ---------------------------------------------------------------------------------------
 * Vec3 (include/render/core/vector.h:112-289)
 * --------------------------------------------------------------------------------------- */
typedef struct { float x, y, z; } v3;

static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 vload(const float* p) { return V(p[0], p[1], p[2]); }
static inline void vstore(float* p, v3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
static inline v3 vneg(v3 a) { return V(-a.x, -a.y, -a.z); }
static inline v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vmuls(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 vmul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 vdivs(v3 a, float s) { float inv = 1.0f / s; return V(a.x * inv, a.y * inv, a.z * inv); }
static inline float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b) {
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float vlen(v3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline v3 vnorm(v3 a) {
    float len = vlen(a);
    if (len > 0.0f) return vdivs(a, len);
    return V(0.0f, 0.0f, 0.0f);
}
static inline int vblack(v3 a) { return a.x <= 0.0f && a.y <= 0.0f && a.z <= 0.0f; }
/* std::max({x, y, z}): the first largest element */
static inline float vmaxc(v3 a) {
    float m = a.x;
    if (m < a.y) m = a.y;
    if (m < a.z) m = a.z;
    return m;
}

/* coordinateSystem (vector.h:282-289) and sampling::Frame (sampler.h:104-118) */
typedef struct { v3 t, b, n; } frame;
static frame make_frame(v3 n) {
    frame f;
    f.n = n;
    if (fabsf(n.x) > fabsf(n.y)) f.t = vnorm(V(-n.z, 0.0f, n.x));
    else f.t = vnorm(V(0.0f, n.z, -n.y));
    f.b = vcross(n, f.t);
    return f;
}
static inline v3 to_world(const frame* f, v3 l) {
    return vadd(vadd(vmuls(f->t, l.x), vmuls(f->b, l.y)), vmuls(f->n, l.z));
}
static inline v3 to_local(const frame* f, v3 w) { return V(vdot(w, f->t), vdot(w, f->b), vdot(w, f->n)); }

/* ---------------------------------------------------------------------------------------
 * Counter-based RNG: Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
 * as easy as 1, 2, 3", SC'11). Shared definition with the GPU library.
 * --------------------------------------------------------------------------------------- */
void orc_philox(const uint32_t c[4], const uint32_t k[2], uint32_t out[4]) {
    uint32_t x0 = c[0], x1 = c[1], x2 = c[2], x3 = c[3];
    uint32_t k0 = k[0], k1 = k[1];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * x0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * x2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        x0 = hi1 ^ x1 ^ k0;
        x1 = lo1;
        x2 = hi0 ^ x3 ^ k1;
        x3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = x0; out[1] = x1; out[2] = x2; out[3] = x3;
}

/* 24 high bits -> [0, 1 - 2^-24] */
static inline float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

/* Purposes of the fourth counter word (must match the GPU library). */
enum { RNG_CAMERA = 0, RNG_BOUNCE = 1, RNG_LIGHTS = 2, RNG_MEDIUM = 3 };

static void draw4(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t depth, uint32_t purpose, float u[4]) {
    const uint32_t c[4] = {pixel, sample, depth, purpose};
    const uint32_t k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    orc_philox(c, k, o);
    for (int i = 0; i < 4; ++i) u[i] = u01(o[i]);
}

/* ---------------------------------------------------------------------------------------
 * Scene
 * --------------------------------------------------------------------------------------- */
enum { P_TRI = 0, P_SPHERE = 1, P_QUAD = 2, P_PLANE = 3 };

typedef struct {
    int type;
    uint32_t material;
    v3 a, b, c;        /* tri: v0 v1 v2; sphere: centre (a), radius (r); quad: origin u v; plane: normal (a), d (r) */
    v3 n0, n1, n2;     /* triangle vertex normals */
    int has_normals;
    v3 qn;             /* quad normal */
    float r;
} prim;

typedef struct {
    int type;
    v3 position, u, v, normal, color;
    float intensity;
} light;

struct orc_scene {
    uint32_t nprims;
    prim* prims; /* in id order */
    uint32_t nmats;
    rbr_material* mats;
    uint32_t nlights;
    light* lights;
    v3 background;
    int has_medium;          /* HomogeneousMedium (medium.h:54-70) */
    v3 sigma_s, sigma_t;
    float avg_sigma_t, g;
};

orc_scene* orc_scene_create(const rbr_scene_desc* d) {
    orc_scene* s = (orc_scene*)calloc(1, sizeof(orc_scene));
    const uint32_t n = d->num_triangles + d->num_spheres + d->num_quads + d->num_planes;
    s->nprims = n;
    s->prims = (prim*)calloc(n ? n : 1, sizeof(prim));
    char* used = (char*)calloc(n ? n : 1, 1);
    uint32_t next = 0;
#define ID_OF(ids, i) ((ids) ? (ids)[i] : next + (i))
#define CLAIM(id)                                                  \
    do {                                                           \
        if ((id) >= n || used[id]) { free(used); orc_scene_destroy(s); return NULL; } \
        used[id] = 1;                                              \
    } while (0)
    for (uint32_t i = 0; i < d->num_triangles; ++i) {
        const uint32_t id = ID_OF(d->triangle_ids, i);
        CLAIM(id);
        prim* p = &s->prims[id];
        const float* v = d->triangle_vertices + 9 * i;
        p->type = P_TRI;
        p->material = d->triangle_materials[i];
        p->a = vload(v); p->b = vload(v + 3); p->c = vload(v + 6);
        if (d->triangle_normals) {
            const float* nn = d->triangle_normals + 9 * i;
            p->has_normals = 1;
            p->n0 = vload(nn); p->n1 = vload(nn + 3); p->n2 = vload(nn + 6);
        }
    }
    next += d->num_triangles;
    for (uint32_t i = 0; i < d->num_spheres; ++i) {
        const uint32_t id = ID_OF(d->sphere_ids, i);
        CLAIM(id);
        prim* p = &s->prims[id];
        p->type = P_SPHERE;
        p->material = d->sphere_materials[i];
        p->a = vload(d->spheres + 4 * i);
        p->r = d->spheres[4 * i + 3];
    }
    next += d->num_spheres;
    for (uint32_t i = 0; i < d->num_quads; ++i) {
        const uint32_t id = ID_OF(d->quad_ids, i);
        CLAIM(id);
        prim* p = &s->prims[id];
        const float* q = d->quads + 9 * i;
        p->type = P_QUAD;
        p->material = d->quad_materials[i];
        p->a = vload(q); p->b = vload(q + 3); p->c = vload(q + 6);
        p->qn = vnorm(vcross(p->b, p->c)); /* Quad::Quad, quad.cpp:6-10 */
    }
    next += d->num_quads;
    for (uint32_t i = 0; i < d->num_planes; ++i) {
        const uint32_t id = ID_OF(d->plane_ids, i);
        CLAIM(id);
        prim* p = &s->prims[id];
        p->type = P_PLANE;
        p->material = d->plane_materials[i];
        p->a = vload(d->planes + 4 * i);
        p->r = d->planes[4 * i + 3];
    }
#undef ID_OF
#undef CLAIM
    free(used);
    s->nmats = d->num_materials;
    s->mats = (rbr_material*)calloc(d->num_materials ? d->num_materials : 1, sizeof(rbr_material));
    if (d->num_materials) memcpy(s->mats, d->materials, d->num_materials * sizeof(rbr_material));
    s->nlights = d->num_lights;
    s->lights = (light*)calloc(d->num_lights ? d->num_lights : 1, sizeof(light));
    for (uint32_t i = 0; i < d->num_lights; ++i) {
        const rbr_light* l = &d->lights[i];
        light* o = &s->lights[i];
        o->type = (int)l->type;
        o->position = vload(l->position);
        o->u = vload(l->u);
        o->v = vload(l->v);
        o->color = vload(l->color);
        o->intensity = l->intensity;
        o->normal = vnorm(vcross(o->u, o->v)); /* AreaLight::AreaLight, area_light.cpp:5-11 */
    }
    s->background = vload(d->background);
    if (d->medium) {
        s->has_medium = 1;
        s->sigma_s = vload(d->medium->sigma_s);
        s->sigma_t = vadd(vload(d->medium->sigma_a), s->sigma_s); /* Medium::getSigmaT */
        s->avg_sigma_t = (s->sigma_t.x + s->sigma_t.y + s->sigma_t.z) / 3.0f;
        s->g = d->medium->g;
    }
    return s;
}

void orc_scene_destroy(orc_scene* s) {
    if (!s) return;
    free(s->prims);
    free(s->mats);
    free(s->lights);
    free(s);
}

/* ---------------------------------------------------------------------------------------
 * Intersection (the isect fields the integrator reads)
 * --------------------------------------------------------------------------------------- */
typedef struct {
    v3 point, normal, wo;
    float t;
    int front;
    uint32_t prim;
} isect_t;

typedef struct { v3 o, d; float tmax; } ray_t;

/* SurfaceInteraction::setFaceNormal (interaction.h:74-78) */
static inline void set_face_normal(isect_t* is, v3 dir, v3 outward) {
    is->front = vdot(dir, outward) < 0.0f;
    is->normal = is->front ? outward : vneg(outward);
}

/* Triangle::intersect (triangle.cpp:6-65) */
static int hit_triangle(const prim* p, ray_t* r, isect_t* is, uint32_t id) {
    v3 e1 = vsub(p->b, p->a);
    v3 e2 = vsub(p->c, p->a);
    v3 h = vcross(r->d, e2);
    float a = vdot(e1, h);
    if (fabsf(a) < ORC_EPS) return 0;
    float f = 1.0f / a;
    v3 s = vsub(r->o, p->a);
    float u = f * vdot(s, h);
    if (u < 0.0f || u > 1.0f) return 0;
    v3 q = vcross(s, e1);
    float v = f * vdot(r->d, q);
    if (v < 0.0f || u + v > 1.0f) return 0;
    float t = f * vdot(e2, q);
    if (t < ORC_EPS || t > r->tmax) return 0;
    if (is) {
        float w = 1.0f - u - v;
        is->point = vadd(r->o, vmuls(r->d, t));
        is->t = t;
        is->wo = vneg(r->d);
        is->prim = id;
        v3 geo = vnorm(vcross(e1, e2));
        v3 nrm = geo;
        if (p->has_normals) {
            nrm = vnorm(vadd(vadd(vmuls(p->n0, w), vmuls(p->n1, u)), vmuls(p->n2, v)));
            if (vdot(nrm, geo) < 0.0f) nrm = vneg(nrm);
        }
        set_face_normal(is, r->d, nrm);
    }
    r->tmax = t;
    return 1;
}

/* Sphere::intersect (sphere.cpp:6-43) */
static int hit_sphere(const prim* p, ray_t* r, isect_t* is, uint32_t id) {
    v3 oc = vsub(r->o, p->a);
    float a = vdot(r->d, r->d);
    float halfB = vdot(oc, r->d);
    float c = vdot(oc, oc) - p->r * p->r;
    float disc = halfB * halfB - a * c;
    if (disc < 0.0f) return 0;
    float sq = sqrtf(disc);
    float t = (-halfB - sq) / a;
    if (t < ORC_EPS || t > r->tmax) {
        t = (-halfB + sq) / a;
        if (t < ORC_EPS || t > r->tmax) return 0;
    }
    if (is) {
        v3 hp = vadd(r->o, vmuls(r->d, t));
        v3 n = vdivs(vsub(hp, p->a), p->r);
        is->point = hp;
        is->t = t;
        is->wo = vneg(r->d);
        is->prim = id;
        set_face_normal(is, r->d, n);
    }
    r->tmax = t;
    return 1;
}

/* Quad::intersect (quad.cpp:12-42) */
static int hit_quad(const prim* p, ray_t* r, isect_t* is, uint32_t id) {
    float denom = vdot(p->qn, r->d);
    if (fabsf(denom) < ORC_EPS) return 0;
    float t = vdot(vsub(p->a, r->o), p->qn) / denom;
    if (t < ORC_EPS || t > r->tmax) return 0;
    v3 hp = vadd(r->o, vmuls(r->d, t));
    v3 lp = vsub(hp, p->a);
    float uLen2 = vdot(p->b, p->b);
    float vLen2 = vdot(p->c, p->c);
    float uc = vdot(lp, p->b) / uLen2;
    float vc = vdot(lp, p->c) / vLen2;
    if (uc < 0.0f || uc > 1.0f || vc < 0.0f || vc > 1.0f) return 0;
    if (is) {
        is->point = hp;
        is->t = t;
        is->wo = vneg(r->d);
        is->prim = id;
        set_face_normal(is, r->d, p->qn);
    }
    r->tmax = t;
    return 1;
}

/* Plane::intersect (plane.cpp:12-35) */
static int hit_plane(const prim* p, ray_t* r, isect_t* is, uint32_t id) {
    float denom = vdot(p->a, r->d);
    if (fabsf(denom) < ORC_EPS) return 0;
    float t = -(vdot(p->a, r->o) + p->r) / denom;
    if (t < ORC_EPS || t > r->tmax) return 0;
    if (is) {
        is->point = vadd(r->o, vmuls(r->d, t));
        is->t = t;
        is->wo = vneg(r->d);
        is->prim = id;
        set_face_normal(is, r->d, p->a);
    }
    r->tmax = t;
    return 1;
}

static int hit_prim(const prim* p, ray_t* r, isect_t* is, uint32_t id) {
    switch (p->type) {
        case P_TRI: return hit_triangle(p, r, is, id);
        case P_SPHERE: return hit_sphere(p, r, is, id);
        case P_QUAD: return hit_quad(p, r, is, id);
        default: return hit_plane(p, r, is, id);
    }
}

/* Brute-force closest hit over all primitives in order (test_accelerators.cpp:58-67):
 * a later primitive at the same t replaces an earlier one (t > tMax rejects, t == tMax accepts). */
static int closest(const orc_scene* s, ray_t r, isect_t* is) {
    int hit = 0;
    for (uint32_t i = 0; i < s->nprims; ++i) {
        if (hit_prim(&s->prims[i], &r, is, i)) hit = 1;
    }
    return hit;
}

/* Brute-force any hit (test_accelerators.cpp:69-74; Primitive::intersectP = intersect). */
static int occluded(const orc_scene* s, ray_t r) {
    for (uint32_t i = 0; i < s->nprims; ++i) {
        ray_t rr = r;
        if (hit_prim(&s->prims[i], &rr, NULL, i)) return 1;
    }
    return 0;
}

static int nthr(int n);

void orc_trace_closest(const orc_scene* s, const rbr_ray* rays, int64_t n, rbr_hit* hits, int nthreads) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthr(nthreads))
    for (int64_t i = 0; i < n; ++i) {
        ray_t r = {vload(rays[i].origin), vload(rays[i].direction), rays[i].tmax};
        isect_t is;
        if (closest(s, r, &is)) {
            hits[i].prim = is.prim;
            hits[i].t = is.t;
        } else {
            hits[i].prim = RBR_MISS;
            hits[i].t = 0.0f;
        }
    }
}

void orc_trace_any(const orc_scene* s, const rbr_ray* rays, int64_t n, uint8_t* occ, int nthreads) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthr(nthreads))
    for (int64_t i = 0; i < n; ++i) {
        ray_t r = {vload(rays[i].origin), vload(rays[i].direction), rays[i].tmax};
        occ[i] = (uint8_t)occluded(s, r);
    }
}

/* ---------------------------------------------------------------------------------------
 * Sampling helpers (include/render/core/sampler.h:58-149)
 * --------------------------------------------------------------------------------------- */
static v3 cosine_hemisphere(float u1, float u2) {
    float r = sqrtf(u1);
    float theta = TWO_PI * u2;
    float x = r * cosf(theta);
    float y = r * sinf(theta);
    float z = sqrtf(omax(0.0f, 1.0f - u1));
    return V(x, y, z);
}

static void concentric_disk(float u1, float u2, float* ox, float* oy) {
    float sx = 2.0f * u1 - 1.0f;
    float sy = 2.0f * u2 - 1.0f;
    if (sx == 0.0f && sy == 0.0f) { *ox = 0.0f; *oy = 0.0f; return; }
    float r, theta;
    if (fabsf(sx) > fabsf(sy)) {
        r = sx;
        theta = (ORC_PI / 4.0f) * (sy / sx);
    } else {
        r = sy;
        theta = (ORC_PI / 2.0f) - (ORC_PI / 4.0f) * (sx / sy);
    }
    *ox = r * cosf(theta);
    *oy = r * sinf(theta);
}

float orc_power_heuristic(int nf, float fPdf, int ng, float gPdf) {
    float f = (float)nf * fPdf;
    float g = (float)ng * gPdf;
    if (isinf(f)) return 1.0f;
    if (isinf(g)) return 0.0f;
    const float m = omax(f, g);
    if (m <= 0.0f) return 0.0f;
    f /= m;
    g /= m;
    return (f * f) / (f * f + g * g);
}

/* ---------------------------------------------------------------------------------------
 * Fresnel (include/render/materials/fresnel.h:16-80)
 * --------------------------------------------------------------------------------------- */
static float fresnel_dielectric(float cosThetaI, float etaI, float etaT) {
    cosThetaI = oclamp(cosThetaI, -1.0f, 1.0f);
    if (cosThetaI < 0.0f) {
        float tmp = etaI; etaI = etaT; etaT = tmp;
        cosThetaI = -cosThetaI;
    }
    const float sinThetaI = sqrtf(omax(0.0f, 1.0f - cosThetaI * cosThetaI));
    const float sinThetaT = etaI / etaT * sinThetaI;
    if (sinThetaT >= 1.0f) return 1.0f;
    const float cosThetaT = sqrtf(omax(0.0f, 1.0f - sinThetaT * sinThetaT));
    const float rParl = (etaT * cosThetaI - etaI * cosThetaT) / (etaT * cosThetaI + etaI * cosThetaT);
    const float rPerp = (etaI * cosThetaI - etaT * cosThetaT) / (etaI * cosThetaI + etaT * cosThetaT);
    return 0.5f * (rParl * rParl + rPerp * rPerp);
}

static v3 fresnel_schlick(float cosTheta, v3 f0) {
    const float m = 1.0f - oclamp(fabsf(cosTheta), 0.0f, 1.0f);
    const float m2 = m * m;
    return vadd(f0, vmuls(vsub(V(1.0f, 1.0f, 1.0f), f0), m2 * m2 * m));
}

enum { FR_NONE = 0, FR_DIELECTRIC = 1, FR_SCHLICK = 2 };
typedef struct { int kind; float etaI, etaT; v3 f0; } fresnel;

static v3 fresnel_eval(const fresnel* f, float c) {
    switch (f->kind) {
        case FR_DIELECTRIC: { float v = fresnel_dielectric(c, f->etaI, f->etaT); return V(v, v, v); }
        case FR_SCHLICK: return fresnel_schlick(c, f->f0);
        default: return V(1.0f, 1.0f, 1.0f);
    }
}

/* ---------------------------------------------------------------------------------------
 * Lobes
 * --------------------------------------------------------------------------------------- */
enum { L_LAMBERT = 0, L_SPEC_REFL = 1, L_SPEC_TRANS = 2, L_GGX_REFL = 3, L_GGX_TRANS = 4 };
/* BSDFType bits (bsdf.h:10-24) */
enum { T_REFL = 1, T_TRANS = 2, T_DIFFUSE = 4, T_GLOSSY = 8, T_SPECULAR = 16 };

typedef struct {
    int kind;
    float weight;
    int substrate;
    v3 color;       /* albedo / reflectance / transmittance */
    fresnel fr;
    float etaO, etaI;
    float alpha;    /* GGXDistribution::alpha, already clamped to >= 1e-3 */
} lobe;

typedef struct {
    int n;
    lobe l[6];
    fresnel sub;
} mixture;

typedef struct { v3 wi, f; float pdf; int type; int delta; } bsample;

static bsample no_sample(void) { bsample s; memset(&s, 0, sizeof(s)); return s; }

static inline int same_hemi(v3 a, v3 b) { return a.z * b.z > 0.0f; }

/* GGXDistribution (microfacet_bsdf.cpp:9-58) */
static float ggx_D(float alpha, v3 wh) {
    const float cos2 = wh.z * wh.z;
    if (cos2 <= 0.0f) return 0.0f;
    const float a2 = alpha * alpha;
    const float d = cos2 * (a2 - 1.0f) + 1.0f;
    return a2 / (ORC_PI * d * d);
}
static float ggx_lambda(float alpha, v3 w) {
    const float cos2 = w.z * w.z;
    if (cos2 <= 0.0f) return 0.0f;
    const float tan2 = omax(0.0f, 1.0f - cos2) / cos2;
    return 0.5f * (sqrtf(1.0f + alpha * alpha * tan2) - 1.0f);
}
static float ggx_G1(float alpha, v3 w) { return 1.0f / (1.0f + ggx_lambda(alpha, w)); }
static float ggx_G(float alpha, v3 wo, v3 wi) { return 1.0f / (1.0f + ggx_lambda(alpha, wo) + ggx_lambda(alpha, wi)); }
static float ggx_pdf(float alpha, v3 wo, v3 wh) {
    const float cosO = fabsf(wo.z);
    if (cosO == 0.0f) return 0.0f;
    return ggx_D(alpha, wh) * ggx_G1(alpha, wo) * fabsf(vdot(wo, wh)) / cosO;
}
static v3 ggx_sample_wh(float alpha, v3 wo, float u1, float u2) {
    const int flip = wo.z < 0.0f;
    const v3 v = flip ? vneg(wo) : wo;
    const v3 vh = vnorm(V(alpha * v.x, alpha * v.y, v.z));
    const v3 t1 = vh.z < 0.9999f ? vnorm(vcross(V(0.0f, 0.0f, 1.0f), vh)) : V(1.0f, 0.0f, 0.0f);
    const v3 t2 = vcross(vh, t1);
    const float r = sqrtf(u1);
    const float phi = TWO_PI * u2;
    const float p1 = r * cosf(phi);
    float p2 = r * sinf(phi);
    const float s = 0.5f * (1.0f + vh.z);
    p2 = (1.0f - s) * sqrtf(omax(0.0f, 1.0f - p1 * p1)) + s * p2;
    const v3 nh = vadd(vadd(vmuls(t1, p1), vmuls(t2, p2)), vmuls(vh, sqrtf(omax(0.0f, 1.0f - p1 * p1 - p2 * p2))));
    const v3 wh = vnorm(V(alpha * nh.x, alpha * nh.y, omax(1e-6f, nh.z)));
    return flip ? vneg(wh) : wh;
}

/* MicrofacetReflectionBSDF (microfacet_bsdf.cpp:64-104) */
static v3 ggxr_eval(const lobe* L, v3 wo, v3 wi) {
    if (!same_hemi(wo, wi)) return V(0, 0, 0);
    const float cosO = fabsf(wo.z), cosI = fabsf(wi.z);
    if (cosO == 0.0f || cosI == 0.0f) return V(0, 0, 0);
    v3 wh = vadd(wo, wi);
    if (wh.x == 0.0f && wh.y == 0.0f && wh.z == 0.0f) return V(0, 0, 0);
    wh = vnorm(wh);
    if (wh.z < 0.0f) wh = vneg(wh);
    const v3 F = fresnel_eval(&L->fr, vdot(wo, wh));
    return vmuls(vmul(L->color, F), ggx_D(L->alpha, wh) * ggx_G(L->alpha, wo, wi) / (4.0f * cosO * cosI));
}
static float ggxr_pdf(const lobe* L, v3 wo, v3 wi) {
    if (!same_hemi(wo, wi)) return 0.0f;
    v3 wh = vadd(wo, wi);
    if (wh.x == 0.0f && wh.y == 0.0f && wh.z == 0.0f) return 0.0f;
    wh = vnorm(wh);
    if (wh.z < 0.0f) wh = vneg(wh);
    const float dotOH = vdot(wo, wh);
    if (dotOH == 0.0f) return 0.0f;
    return ggx_pdf(L->alpha, wo, wh) / (4.0f * fabsf(dotOH));
}
static bsample ggxr_sample(const lobe* L, v3 wo, float u1, float u2) {
    bsample r = no_sample();
    if (wo.z == 0.0f) return r;
    const v3 wh = ggx_sample_wh(L->alpha, wo, u1, u2);
    const v3 wi = vsub(vmuls(wh, 2.0f * vdot(wo, wh)), wo);
    if (!same_hemi(wo, wi)) return r;
    const float p = ggxr_pdf(L, wo, wi);
    if (p <= 0.0f) return r;
    r.wi = wi;
    r.pdf = p;
    r.f = ggxr_eval(L, wo, wi);
    r.type = T_GLOSSY | T_REFL;
    return r;
}

/* MicrofacetTransmissionBSDF (microfacet_bsdf.cpp:110-179) */
static int ggxt_half(const lobe* L, v3 wo, v3 wi, v3* wh, float* eta) {
    if (same_hemi(wo, wi)) return 0;
    if (wo.z == 0.0f || wi.z == 0.0f) return 0;
    *eta = wo.z > 0.0f ? L->etaI / L->etaO : L->etaO / L->etaI;
    v3 h = vadd(wo, vmuls(wi, *eta));
    if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return 0;
    h = vnorm(h);
    if (vdot(wo, h) < 0.0f) h = vneg(h);
    *wh = h;
    return h.z * wo.z > 0.0f && vdot(wi, h) <= 0.0f;
}
static v3 ggxt_eval(const lobe* L, v3 wo, v3 wi) {
    v3 wh;
    float eta;
    if (!ggxt_half(L, wo, wi, &wh, &eta)) return V(0, 0, 0);
    const float cosO = wo.z, cosI = wi.z;
    const float dotOH = vdot(wo, wh), dotIH = vdot(wi, wh);
    const float F = fresnel_dielectric(wo.z > 0.0f ? dotOH : -dotOH, L->etaO, L->etaI);
    const float denom = dotOH + eta * dotIH;
    if (denom == 0.0f) return V(0, 0, 0);
    const float value = ggx_D(L->alpha, wh) * ggx_G(L->alpha, wo, wi) * fabsf(dotIH * dotOH) /
                        fabsf(cosI * cosO * denom * denom);
    return vmuls(L->color, (1.0f - F) * value);
}
static float ggxt_pdf(const lobe* L, v3 wo, v3 wi) {
    v3 wh;
    float eta;
    if (!ggxt_half(L, wo, wi, &wh, &eta)) return 0.0f;
    const float dotOH = vdot(wo, wh), dotIH = vdot(wi, wh);
    const float denom = dotOH + eta * dotIH;
    if (denom == 0.0f) return 0.0f;
    const float dwhDwi = fabsf(eta * eta * dotIH) / (denom * denom);
    return ggx_pdf(L->alpha, wo, wh) * dwhDwi;
}
static bsample ggxt_sample(const lobe* L, v3 wo, float u1, float u2) {
    bsample r = no_sample();
    if (wo.z == 0.0f) return r;
    const v3 wh = ggx_sample_wh(L->alpha, wo, u1, u2);
    const float dotOH = vdot(wo, wh);
    if (dotOH <= 0.0f) return r;
    const int entering = wo.z > 0.0f;
    const float etaRatio = entering ? L->etaO / L->etaI : L->etaI / L->etaO;
    const float sin2T = etaRatio * etaRatio * omax(0.0f, 1.0f - dotOH * dotOH);
    if (sin2T >= 1.0f) return r;
    const float cosT = sqrtf(1.0f - sin2T);
    const v3 wi = vsub(vmuls(wh, etaRatio * dotOH - cosT), vmuls(wo, etaRatio));
    if (same_hemi(wo, wi) || wi.z == 0.0f) return r;
    const float p = ggxt_pdf(L, wo, wi);
    if (p <= 0.0f) return r;
    r.wi = wi;
    r.pdf = p;
    r.f = ggxt_eval(L, wo, wi);
    r.type = T_GLOSSY | T_TRANS;
    return r;
}

/* LambertianBSDF (lambertian_bsdf.cpp:5-28) */
static v3 lam_eval(const lobe* L, v3 wo, v3 wi) {
    if (!same_hemi(wo, wi)) return V(0, 0, 0);
    return vmuls(L->color, INV_PI);
}
static float lam_pdf(v3 wo, v3 wi) {
    if (!same_hemi(wo, wi)) return 0.0f;
    return fabsf(wi.z) * INV_PI;
}
static bsample lam_sample(const lobe* L, v3 wo, float u1, float u2) {
    bsample r = no_sample();
    r.wi = cosine_hemisphere(u1, u2);
    if (wo.z < 0.0f) r.wi.z = -r.wi.z;
    r.f = vmuls(L->color, INV_PI);
    r.pdf = fabsf(r.wi.z) * INV_PI;
    r.type = T_DIFFUSE | T_REFL;
    return r;
}

/* SpecularReflection/TransmissionBSDF (specular_bsdf.cpp:5-57) */
static bsample sr_sample(const lobe* L, v3 wo) {
    bsample r = no_sample();
    const float cosO = fabsf(wo.z);
    if (cosO == 0.0f) return r;
    r.wi = V(-wo.x, -wo.y, wo.z);
    r.f = vdivs(vmul(L->color, fresnel_eval(&L->fr, wo.z)), cosO);
    r.pdf = 1.0f;
    r.type = T_SPECULAR | T_REFL;
    r.delta = 1;
    return r;
}
static bsample st_sample(const lobe* L, v3 wo) {
    bsample r = no_sample();
    if (wo.z == 0.0f) return r;
    const int entering = wo.z > 0.0f;
    const float etaI = entering ? L->etaO : L->etaI;
    const float etaT = entering ? L->etaI : L->etaO;
    const float eta = etaI / etaT;
    const float cosI = fabsf(wo.z);
    const float sin2T = eta * eta * omax(0.0f, 1.0f - cosI * cosI);
    if (sin2T >= 1.0f) return r;
    const float cosT = sqrtf(1.0f - sin2T);
    r.wi = V(-eta * wo.x, -eta * wo.y, entering ? -cosT : cosT);
    const float fr = fresnel_dielectric(wo.z, L->etaO, L->etaI);
    r.f = vmuls(L->color, (1.0f - fr) * eta * eta / cosT);
    r.pdf = 1.0f;
    r.type = T_SPECULAR | T_TRANS;
    r.delta = 1;
    return r;
}

static int lobe_delta(const lobe* L) { return L->kind == L_SPEC_REFL || L->kind == L_SPEC_TRANS; }

static int lobe_type(const lobe* L) {
    switch (L->kind) {
        case L_LAMBERT: return T_DIFFUSE | T_REFL;
        case L_SPEC_REFL: return T_SPECULAR | T_REFL;
        case L_SPEC_TRANS: return T_SPECULAR | T_TRANS;
        case L_GGX_REFL: return T_GLOSSY | T_REFL;
        default: return T_GLOSSY | T_TRANS;
    }
}

static v3 lobe_rho(const lobe* L, v3 wo) {
    switch (L->kind) {
        case L_LAMBERT: return L->color;
        case L_SPEC_REFL:
        case L_GGX_REFL: return vmul(L->color, fresnel_eval(&L->fr, wo.z));
        default: return vmuls(L->color, 1.0f - fresnel_dielectric(wo.z, L->etaO, L->etaI));
    }
}

static v3 lobe_eval(const lobe* L, v3 wo, v3 wi) {
    switch (L->kind) {
        case L_LAMBERT: return lam_eval(L, wo, wi);
        case L_GGX_REFL: return ggxr_eval(L, wo, wi);
        case L_GGX_TRANS: return ggxt_eval(L, wo, wi);
        default: return V(0, 0, 0);
    }
}

static float lobe_pdf(const lobe* L, v3 wo, v3 wi) {
    switch (L->kind) {
        case L_LAMBERT: return lam_pdf(wo, wi);
        case L_GGX_REFL: return ggxr_pdf(L, wo, wi);
        case L_GGX_TRANS: return ggxt_pdf(L, wo, wi);
        default: return 0.0f;
    }
}

static bsample lobe_sample(const lobe* L, v3 wo, float u1, float u2) {
    switch (L->kind) {
        case L_LAMBERT: return lam_sample(L, wo, u1, u2);
        case L_SPEC_REFL: return sr_sample(L, wo);
        case L_SPEC_TRANS: return st_sample(L, wo);
        case L_GGX_REFL: return ggxr_sample(L, wo, u1, u2);
        default: return ggxt_sample(L, wo, u1, u2);
    }
}

/* MixtureBSDF (mixture_bsdf.cpp:5-82) */
static void mix_add(mixture* m, lobe L, float weight, int substrate) {
    if (weight <= 0.0f || m->n >= 6) return;
    L.weight = weight;
    L.substrate = substrate;
    m->l[m->n++] = L;
}

static float eff_weight(const mixture* m, const lobe* L, v3 wo) {
    if (!L->substrate) return L->weight;
    return L->weight * omax(0.0f, 1.0f - fresnel_eval(&m->sub, wo.z).x);
}

static float mix_selection(const mixture* m, v3 wo, float* w, float* sc) {
    float total = 0.0f;
    for (int i = 0; i < m->n; ++i) {
        w[i] = eff_weight(m, &m->l[i], wo);
        sc[i] = w[i] * vmaxc(lobe_rho(&m->l[i], wo));
        total += sc[i];
    }
    return total;
}

static v3 mix_eval(const mixture* m, v3 wo, v3 wi) {
    v3 f = V(0, 0, 0);
    for (int i = 0; i < m->n; ++i) {
        if (lobe_delta(&m->l[i])) continue;
        f = vadd(f, vmuls(lobe_eval(&m->l[i], wo, wi), eff_weight(m, &m->l[i], wo)));
    }
    return f;
}

static float mix_pdf(const mixture* m, v3 wo, v3 wi) {
    float w[6], sc[6];
    const float total = mix_selection(m, wo, w, sc);
    if (total <= 0.0f) return 0.0f;
    float p = 0.0f;
    for (int i = 0; i < m->n; ++i) {
        if (lobe_delta(&m->l[i])) continue;
        p += sc[i] * lobe_pdf(&m->l[i], wo, wi);
    }
    return p / total;
}

static bsample mix_sample(const mixture* m, v3 wo, float u1, float u2) {
    bsample none = no_sample();
    float w[6], sc[6];
    const float total = mix_selection(m, wo, w, sc);
    if (total <= 0.0f) return none;
    float u = u1 * total;
    int chosen = m->n - 1;
    for (int i = 0; i < m->n; ++i) {
        if (sc[i] <= 0.0f) continue;
        if (u < sc[i] || i + 1 == m->n) {
            chosen = i;
            break;
        }
        u -= sc[i];
    }
    if (sc[chosen] <= 0.0f) return none;
    const float v1 = omin(u / sc[chosen], 0.99999994f);
    const lobe* L = &m->l[chosen];
    bsample s = lobe_sample(L, wo, v1, u2);
    if (s.pdf <= 0.0f || vblack(s.f)) return none;
    const float pChosen = sc[chosen] / total;
    if (lobe_delta(L)) {
        s.f = vmuls(s.f, w[chosen]);
        s.pdf *= pChosen;
        return s;
    }
    s.f = mix_eval(m, wo, s.wi);
    s.pdf = mix_pdf(m, wo, s.wi);
    if (s.pdf <= 0.0f) return none;
    return s;
}

static int mix_delta(const mixture* m) {
    if (m->n == 0) return 0;
    for (int i = 0; i < m->n; ++i)
        if (!lobe_delta(&m->l[i])) return 0;
    return 1;
}

static int mix_type(const mixture* m) {
    int t = 0;
    for (int i = 0; i < m->n; ++i) t |= lobe_type(&m->l[i]);
    return t;
}

/* Material::createBSDF (material.cpp:69-108) */
static void create_bsdf(const rbr_material* mat, mixture* mix) {
    memset(mix, 0, sizeof(*mix));
    const v3 base = vload(mat->base_color);
    const float m = oclamp(mat->metallic, 0.0f, 1.0f);
    const float t = oclamp(mat->transmission, 0.0f, 1.0f);
    const float dielectric = 1.0f - m;
    const int smooth = mat->roughness < 0.03f;
    const int hasInterface = fabsf(mat->ior - 1.0f) > 1e-3f;
    const int tinted = !vblack(base);
    const float alpha = omax(mat->roughness * mat->roughness, 1e-3f);
    lobe L;
    if (m > 0.0f && tinted) {
        memset(&L, 0, sizeof(L));
        L.kind = smooth ? L_SPEC_REFL : L_GGX_REFL;
        L.color = V(1, 1, 1);
        L.fr.kind = FR_SCHLICK;
        L.fr.f0 = base;
        L.alpha = alpha;
        mix_add(mix, L, m, 0);
    }
    if (dielectric > 0.0f) {
        if (hasInterface) {
            fresnel fr;
            memset(&fr, 0, sizeof(fr));
            fr.kind = FR_DIELECTRIC;
            fr.etaI = 1.0f;
            fr.etaT = mat->ior;
            fr.f0 = V(1, 1, 1);
            memset(&L, 0, sizeof(L));
            L.kind = smooth ? L_SPEC_REFL : L_GGX_REFL;
            L.color = V(1, 1, 1);
            L.fr = fr;
            L.alpha = alpha;
            mix_add(mix, L, dielectric, 0);
            mix->sub = fr;
            if (t > 0.0f && tinted) {
                memset(&L, 0, sizeof(L));
                L.kind = smooth ? L_SPEC_TRANS : L_GGX_TRANS;
                L.color = base;
                L.etaO = 1.0f;
                L.etaI = mat->ior;
                L.alpha = alpha;
                mix_add(mix, L, dielectric * t, 0);
            }
            if (t < 1.0f && tinted) {
                memset(&L, 0, sizeof(L));
                L.kind = L_LAMBERT;
                L.color = base;
                mix_add(mix, L, dielectric * (1.0f - t), 1);
            }
        } else {
            if (t > 0.0f && tinted) {
                memset(&L, 0, sizeof(L));
                L.kind = L_SPEC_TRANS;
                L.color = base;
                L.etaO = 1.0f;
                L.etaI = 1.0f;
                mix_add(mix, L, dielectric * t, 0);
            }
            if (t < 1.0f && tinted) {
                memset(&L, 0, sizeof(L));
                L.kind = L_LAMBERT;
                L.color = base;
                mix_add(mix, L, dielectric * (1.0f - t), 0);
            }
        }
    }
}

void orc_bsdf_eval(const rbr_material* m, int64_t n, const float* wo, const float* wi, float* f, float* pdf,
                   uint32_t* info) {
    mixture mix;
    create_bsdf(m, &mix);
    for (int64_t i = 0; i < n; ++i) {
        const v3 a = vload(wo + 3 * i), b = vload(wi + 3 * i);
        vstore(f + 3 * i, mix_eval(&mix, a, b));
        pdf[i] = mix_pdf(&mix, a, b);
    }
    if (info) {
        info[0] = (uint32_t)mix_delta(&mix);
        info[1] = (uint32_t)mix_type(&mix);
    }
}

void orc_bsdf_sample(const rbr_material* m, int64_t n, const float* wo, const float* u, float* out) {
    mixture mix;
    create_bsdf(m, &mix);
    for (int64_t i = 0; i < n; ++i) {
        const bsample s = mix_sample(&mix, vload(wo + 3 * i), u[2 * i], u[2 * i + 1]);
        float* o = out + 8 * i;
        vstore(o, s.wi);
        vstore(o + 3, s.f);
        o[6] = s.pdf;
        o[7] = s.delta ? 1.0f : 0.0f;
    }
}

/* ---------------------------------------------------------------------------------------
 * Lights (area_light.cpp:13-39, point_light.cpp:5-19)
 * --------------------------------------------------------------------------------------- */
typedef struct { v3 wi, Li; float pdf, dist; int delta; } lsample;

static lsample light_sample(const light* l, v3 p, float u1, float u2) {
    lsample s;
    memset(&s, 0, sizeof(s));
    if (l->type == RBR_LIGHT_AREA) {
        v3 lp = vadd(vadd(l->position, vmuls(l->u, u1 - 0.5f)), vmuls(l->v, u2 - 0.5f));
        v3 toL = vsub(lp, p);
        float d2 = vdot(toL, toL);
        s.dist = sqrtf(d2);
        s.wi = vdivs(toL, s.dist);
        float c = -vdot(l->normal, s.wi);
        if (c <= 0.0f) {
            s.Li = V(0, 0, 0);
            s.pdf = 0.0f;
            return s;
        }
        float area = vlen(vcross(l->u, l->v));
        s.pdf = d2 / (c * area);
        s.Li = vmuls(l->color, l->intensity);
        s.delta = 0;
    } else {
        v3 toL = vsub(l->position, p);
        float d2 = vdot(toL, toL);
        s.dist = sqrtf(d2);
        s.wi = vdivs(toL, s.dist);
        s.Li = vdivs(vmuls(l->color, l->intensity), d2);
        s.pdf = 1.0f;
        s.delta = 1;
    }
    return s;
}

void orc_light_sample(const rbr_light* rl, int64_t n, const float* points, const float* u, float* out) {
    light l;
    l.type = (int)rl->type;
    l.position = vload(rl->position);
    l.u = vload(rl->u);
    l.v = vload(rl->v);
    l.color = vload(rl->color);
    l.intensity = rl->intensity;
    l.normal = vnorm(vcross(l.u, l.v));
    for (int64_t i = 0; i < n; ++i) {
        lsample s = light_sample(&l, vload(points + 3 * i), u[2 * i], u[2 * i + 1]);
        float* o = out + 9 * i;
        vstore(o, s.wi);
        vstore(o + 3, s.Li);
        o[6] = s.pdf;
        o[7] = s.dist;
        o[8] = s.delta ? 1.0f : 0.0f;
    }
}

/* ---------------------------------------------------------------------------------------
 * Camera (camera.cpp:5-9, pinhole_camera.cpp:5-7, thin_lens_camera.cpp:6-23,
 * perspective_intrinsics.h:43-45, camera_extrinsics.h:52-54)
 * --------------------------------------------------------------------------------------- */
static v3 cam_to_world(const rbr_camera* c, v3 d) {
    return vadd(vadd(vmuls(vload(c->right), d.x), vmuls(vload(c->up), d.y)), vmuls(vload(c->forward), d.z));
}

static ray_t camera_ray(const rbr_camera* c, float px, float py, float lu, float lv) {
    const v3 local = V((px - c->cx) / c->fx, (c->cy - py) / c->fy, 1.0f);
    const v3 pos = vload(c->position);
    /* generateIntrinsicRay: Ray(position + cameraToWorldDir(0), cameraToWorldDir(dir).normalized()),
     * and the Ray constructor normalises once more. */
    const v3 org = vadd(pos, cam_to_world(c, V(0.0f, 0.0f, 0.0f)));
    const v3 dir = vnorm(vnorm(cam_to_world(c, local)));
    ray_t r;
    r.tmax = INFINITY;
    if (c->model != RBR_CAMERA_THIN_LENS) { /* PinholeCamera::generateRay */
        r.o = org;
        r.d = dir;
        return r;
    }
    if (c->lens_radius > 0.0f) {
        float lx, ly;
        concentric_disk(lu, lv, &lx, &ly);
        const v3 lens = vadd(pos, vmuls(vadd(vmuls(vload(c->right), lx), vmuls(vload(c->up), ly)), c->lens_radius));
        const float ft = c->focal_distance / fabsf(vdot(dir, vload(c->forward)));
        const v3 focus = vadd(pos, vmuls(dir, ft));
        r.o = lens;
        r.d = vnorm(vnorm(vsub(focus, lens)));
        return r;
    }
    r.o = pos; /* Ray(extrinsics.position, rayDir): normalised again */
    r.d = vnorm(dir);
    return r;
}

void orc_camera_rays(const rbr_camera* c, int64_t n, const float* samples, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        const float* s = samples + 4 * i;
        ray_t r = camera_ray(c, s[0], s[1], s[2], s[3]);
        vstore(out + 6 * i, r.o);
        vstore(out + 6 * i + 3, r.d);
    }
}

/* ---------------------------------------------------------------------------------------
 * Path tracer (path_tracing_integrator.cpp:5-138) with the counter RNG
 * --------------------------------------------------------------------------------------- */
/* Interaction::spawnRay (interaction.h:22-29); the Ray constructor normalises. */
static ray_t spawn_ray(const isect_t* is, v3 dir) {
    v3 off = vmuls(is->normal, ORC_EPS);
    if (vdot(dir, is->normal) < 0.0f) off = vneg(off);
    ray_t r;
    r.o = vadd(is->point, off);
    r.d = vnorm(dir);
    r.tmax = INFINITY;
    return r;
}

static v3 path_li(const orc_scene* s, const rbr_render_params* p, ray_t ray, uint32_t pixel, uint32_t sample) {
    v3 L = V(0, 0, 0);
    v3 T = V(1, 1, 1);
    int specular = 1;
    for (int depth = 0; depth < p->max_depth; ++depth) {
        isect_t is;
        if (!closest(s, ray, &is)) {
            L = vadd(L, vmul(T, s->background));
            break;
        }
        const rbr_material* mat = &s->mats[s->prims[is.prim].material];
        const v3 emission = vload(mat->emission);
        const int emissive = emission.x > 0.0f || emission.y > 0.0f || emission.z > 0.0f;
        if (emissive && (depth == 0 || specular)) L = vadd(L, vmul(T, emission));
        mixture bsdf;
        create_bsdf(mat, &bsdf);
        const v3 outward = is.front ? is.normal : vneg(is.normal);
        const frame fr = make_frame(outward);
        const v3 woL = to_local(&fr, is.wo);
        if (p->use_nee && !mix_delta(&bsdf)) {
            v3 Ld = V(0, 0, 0);
            for (uint32_t li = 0; li < s->nlights; ++li) {
                float u[4];
                draw4(p->seed, pixel, sample, (uint32_t)depth, RNG_LIGHTS + ((li / 2) << 8), u);
                const light* l = &s->lights[li];
                const lsample ls = light_sample(l, is.point, u[(li & 1) * 2], u[(li & 1) * 2 + 1]);
                v3 contrib = V(0, 0, 0);
                if (ls.pdf > 0.0f && !vblack(ls.Li)) {
                    const v3 wiL = to_local(&fr, ls.wi);
                    const v3 f = mix_eval(&bsdf, woL, wiL);
                    const float bpdf = mix_pdf(&bsdf, woL, wiL);
                    if (!vblack(f)) {
                        ray_t sh = spawn_ray(&is, ls.wi);
                        sh.tmax = ls.dist - ORC_EPS;
                        if (!occluded(s, sh)) {
                            const float c = fabsf(vdot(ls.wi, is.normal));
                            if (p->use_mis && !ls.delta) {
                                const float w = orc_power_heuristic(1, ls.pdf, 1, bpdf);
                                contrib = vdivs(vmuls(vmuls(vmul(f, ls.Li), c), w), ls.pdf);
                            } else {
                                contrib = vdivs(vmuls(vmul(f, ls.Li), c), ls.pdf);
                            }
                        }
                    }
                }
                Ld = vadd(Ld, contrib);
            }
            L = vadd(L, vmul(T, Ld));
        }
        float u[4];
        draw4(p->seed, pixel, sample, (uint32_t)depth, RNG_BOUNCE, u);
        const bsample bs = mix_sample(&bsdf, woL, u[0], u[1]);
        if (bs.pdf <= 0.0f || vblack(bs.f)) break;
        const v3 wiW = to_world(&fr, bs.wi);
        const float c = fabsf(vdot(wiW, is.normal));
        T = vmul(T, vmuls(bs.f, c / bs.pdf));
        if (depth > 3) {
            const float q = omax(0.05f, 1.0f - vmaxc(T));
            if (u[2] < q) break;
            T = vdivs(T, 1.0f - q);
        }
        ray = spawn_ray(&is, wiW);
        specular = bs.delta;
    }
    return L;
}

/* ---------------------------------------------------------------------------------------
 * Participating medium and the volumetric path integrator (medium.cpp:9-44,
 * phase_function.cpp:17-47, volumetric_path_integrator.cpp:6-143) with the counter RNG:
 * per depth, the distance and the phase direction use purpose RNG_MEDIUM (u0; u1, u2), the
 * surface lights and the BSDF the same streams as the path tracer.
 * --------------------------------------------------------------------------------------- */
float orc_hg_eval(float g, const float wo[3], const float wi[3]) {
    const float c = vdot(vload(wo), vload(wi));
    const float denom = 1.0f + g * g + 2.0f * g * c;
    return (1.0f - g * g) / (4.0f * ORC_PI * denom * sqrtf(denom));
}

static v3 hg_sample(float g, v3 wo, float u1, float u2) {
    float c;
    if (fabsf(g) < 1e-3f) {
        c = 1.0f - 2.0f * u1;
    } else {
        const float sq = (1.0f - g * g) / (1.0f + g - 2.0f * g * u1);
        c = -(1.0f + g * g - sq * sq) / (2.0f * g);
    }
    const float st = sqrtf(omax(0.0f, 1.0f - c * c));
    const float phi = TWO_PI * u2;
    const frame f = make_frame(wo); /* coordinateSystem(wo, tangent, bitangent) */
    return vadd(vadd(vmuls(f.t, st * cosf(phi)), vmuls(f.b, st * sinf(phi))), vmuls(wo, c));
}

static v3 transmittance(const orc_scene* s, float dist) {
    return V(expf(-s->sigma_t.x * dist), expf(-s->sigma_t.y * dist), expf(-s->sigma_t.z * dist));
}

static int medium_sample(const orc_scene* s, float max_dist, float u, float* t, v3* weight) {
    if (s->avg_sigma_t < 1e-6f) {
        *weight = V(1, 1, 1);
        return 0;
    }
    *t = -logf(1.0f - u) / s->avg_sigma_t;
    if (*t < max_dist) {
        const v3 tr = transmittance(s, *t);
        *weight = vdivs(vmul(s->sigma_s, tr), s->avg_sigma_t * s->avg_sigma_t);
        return 1;
    }
    *weight = transmittance(s, max_dist);
    return 0;
}

void orc_hg_sample(float g, int64_t n, const float* wo, const float* u, float* out) {
    for (int64_t i = 0; i < n; ++i) vstore(out + 3 * i, hg_sample(g, vload(wo + 3 * i), u[2 * i], u[2 * i + 1]));
}

static v3 vol_li(const orc_scene* s, const rbr_render_params* p, ray_t ray, uint32_t pixel, uint32_t sample) {
    v3 L = V(0, 0, 0);
    v3 T = V(1, 1, 1);
    for (int depth = 0; depth < p->max_depth; ++depth) {
        isect_t is;
        const int hit = closest(s, ray, &is);
        if (s->has_medium) {
            float u[4];
            draw4(p->seed, pixel, sample, (uint32_t)depth, RNG_MEDIUM, u);
            float t = 0.0f;
            v3 w;
            const int scattered = medium_sample(s, hit ? is.t : INFINITY, u[0], &t, &w);
            T = vmul(T, w);
            if (scattered) {
                const v3 sp = vadd(ray.o, vmuls(ray.d, t));
                if (p->use_nee) {
                    v3 Ld = V(0, 0, 0);
                    for (uint32_t li = 0; li < s->nlights; ++li) {
                        const light* l = &s->lights[li];
                        if (l->type != RBR_LIGHT_POINT) continue;
                        const v3 toL = vsub(l->position, sp);
                        const float dist = vlen(toL);
                        const v3 wi = vdivs(toL, dist);
                        ray_t sh;
                        sh.o = sp;
                        sh.d = vnorm(wi);
                        sh.tmax = dist;
                        if (occluded(s, sh)) continue;
                        const v3 tr = transmittance(s, dist);
                        const v3 Li = vdivs(vmuls(l->color, l->intensity), dist * dist);
                        const float wo3[3] = {ray.d.x, ray.d.y, ray.d.z}, wi3[3] = {wi.x, wi.y, wi.z};
                        Ld = vadd(Ld, vmuls(vmul(Li, tr), orc_hg_eval(s->g, wo3, wi3)));
                    }
                    L = vadd(L, vmul(T, Ld));
                }
                ray.o = sp;
                ray.d = vnorm(hg_sample(s->g, ray.d, u[1], u[2]));
                ray.tmax = INFINITY;
                continue;
            }
        }
        if (!hit) {
            L = vadd(L, vmul(T, s->background));
            break;
        }
        const rbr_material* mat = &s->mats[s->prims[is.prim].material];
        const v3 emission = vload(mat->emission);
        if (emission.x > 0.0f || emission.y > 0.0f || emission.z > 0.0f) L = vadd(L, vmul(T, emission));
        mixture bsdf;
        create_bsdf(mat, &bsdf);
        const v3 outward = is.front ? is.normal : vneg(is.normal);
        const frame fr = make_frame(outward);
        const v3 woL = to_local(&fr, is.wo);
        if (p->use_nee && !mix_delta(&bsdf)) {
            v3 Ld = V(0, 0, 0);
            for (uint32_t li = 0; li < s->nlights; ++li) {
                float u[4];
                draw4(p->seed, pixel, sample, (uint32_t)depth, RNG_LIGHTS + ((li / 2) << 8), u);
                const lsample ls = light_sample(&s->lights[li], is.point, u[(li & 1) * 2], u[(li & 1) * 2 + 1]);
                if (ls.pdf <= 0.0f || vblack(ls.Li)) continue;
                ray_t sh = spawn_ray(&is, ls.wi);
                sh.tmax = ls.dist - ORC_EPS;
                if (occluded(s, sh)) continue;
                const v3 f = mix_eval(&bsdf, woL, to_local(&fr, ls.wi));
                const float c = fabsf(vdot(ls.wi, is.normal));
                Ld = vadd(Ld, vdivs(vmuls(vmul(f, ls.Li), c), ls.pdf));
            }
            L = vadd(L, vmul(T, Ld));
        }
        float u[4];
        draw4(p->seed, pixel, sample, (uint32_t)depth, RNG_BOUNCE, u);
        const bsample bs = mix_sample(&bsdf, woL, u[0], u[1]);
        if (bs.pdf <= 0.0f || vblack(bs.f)) break;
        const v3 wiW = to_world(&fr, bs.wi);
        const float c = fabsf(vdot(wiW, is.normal));
        T = vmul(T, vmuls(bs.f, c / bs.pdf));
        if (depth > 3) {
            const float q = omax(0.05f, 1.0f - vmaxc(T));
            if (u[2] < q) break;
            T = vdivs(T, 1.0f - q);
        }
        ray = spawn_ray(&is, wiW);
    }
    return L;
}

static int nthr(int n) {
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return n > 0 ? n : omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* Integrator::render's per-sample work (integrator.cpp:20-36) with counter-RNG camera samples. */
void orc_render(const orc_scene* s, const rbr_camera* c, const rbr_render_params* p, float* mean, double* sum,
                double* sumsq, int nthreads) {
    const int W = c->width, H = c->height;
    const int spp = p->samples_per_pixel;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthr(nthreads))
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const uint32_t pixel = (uint32_t)(y * W + x);
            v3 acc = V(0, 0, 0);
            double s0 = 0, s1 = 0, s2 = 0, q0 = 0, q1 = 0, q2 = 0;
            for (int k = 0; k < spp; ++k) {
                const uint32_t sample = p->sample_offset + (uint32_t)k;
                float u[4];
                draw4(p->seed, pixel, sample, 0u, RNG_CAMERA, u);
                const float px = (float)x + u[0];
                const float py = (float)y + u[1];
                const ray_t r = camera_ray(c, px, py, u[2], u[3]);
                const v3 L = (p->flags & RBR_RENDER_VOLUMETRIC) ? vol_li(s, p, r, pixel, sample)
                                                                : path_li(s, p, r, pixel, sample);
                acc = vadd(acc, L);
                s0 += L.x; s1 += L.y; s2 += L.z;
                q0 += (double)L.x * L.x; q1 += (double)L.y * L.y; q2 += (double)L.z * L.z;
            }
            const size_t o = 3 * (size_t)pixel;
            if (mean) vstore(mean + o, vdivs(acc, (float)spp));
            if (sum) { sum[o] += s0; sum[o + 1] += s1; sum[o + 2] += s2; }
            if (sumsq) { sumsq[o] += q0; sumsq[o + 1] += q1; sumsq[o + 2] += q2; }
        }
    }
}

void orc_path(const orc_scene* s, const rbr_camera* c, const rbr_render_params* p, int x, int y, uint32_t sample,
              float* Lout) {
    const uint32_t pixel = (uint32_t)(y * c->width + x);
    float u[4];
    draw4(p->seed, pixel, sample, 0u, RNG_CAMERA, u);
    const ray_t r = camera_ray(c, (float)x + u[0], (float)y + u[1], u[2], u[3]);
    vstore(Lout, (p->flags & RBR_RENDER_VOLUMETRIC) ? vol_li(s, p, r, pixel, sample) : path_li(s, p, r, pixel, sample));
}
