// rbr_scene_upload: validation, host BVH build and upload of a scene description.
//
// Host arithmetic that must match the reference bit for bit (edge vectors, r*r, |u|^2,
// light normals) is compiled without FMA contraction (-ffp-contract=off), as the reference is.
#include <algorithm>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>

#include "bvh_build.h"
#include "rbr_context.h"

namespace rbr {

namespace {

struct V3 {
    float x, y, z;
};
inline V3 ld(const float* p) { return V3{p[0], p[1], p[2]}; }
inline V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V3 normalized(V3 a) {  // Vec3::normalized
    const float len = std::sqrt(dot(a, a));
    if (len > 0.0f) {
        const float inv = 1.0f / len;
        return V3{a.x * inv, a.y * inv, a.z * inv};
    }
    return V3{0.0f, 0.0f, 0.0f};
}
inline bool finite3(const float* p, int n) {
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}
inline void box_point(Box& b, V3 p) {
    b.lo[0] = std::min(b.lo[0], p.x);
    b.lo[1] = std::min(b.lo[1], p.y);
    b.lo[2] = std::min(b.lo[2], p.z);
    b.hi[0] = std::max(b.hi[0], p.x);
    b.hi[1] = std::max(b.hi[1], p.y);
    b.hi[2] = std::max(b.hi[2], p.z);
}
inline Box empty_box() { return Box{{FLT_MAX, FLT_MAX, FLT_MAX}, {-FLT_MAX, -FLT_MAX, -FLT_MAX}}; }

// The lobes Material::createBSDF (src/materials/material.cpp:69-108) adds for `m`, reduced to
// the shading class of the material.
uint32_t material_class(const rbr_material& m) {
    const float met = std::max(0.0f, std::min(1.0f, m.metallic));
    const float t = std::max(0.0f, std::min(1.0f, m.transmission));
    const float diel = 1.0f - met;
    const bool smooth = m.roughness < 0.03f;
    const bool iface = std::fabs(m.ior - 1.0f) > 1e-3f;
    const bool tinted = !(m.base_color[0] <= 0.0f && m.base_color[1] <= 0.0f && m.base_color[2] <= 0.0f);
    bool ggx = false, ggx_trans = false, lambert = false, delta = false;
    auto lobe = [&](bool is_delta) { (is_delta ? delta : ggx) = true; };
    if (met > 0.0f && tinted) lobe(smooth);
    if (diel > 0.0f) {
        if (iface) {
            lobe(smooth);
            if (t > 0.0f && tinted) {
                lobe(smooth);
                ggx_trans = !smooth;
            }
            if (t < 1.0f && tinted) lambert = true;
        } else {
            if (t > 0.0f && tinted) delta = true;
            if (t < 1.0f && tinted) lambert = true;
        }
    }
    if (ggx_trans) return kClassGlossyTrans;
    if (ggx) return lambert ? kClassGlossy : kClassGlossyRefl;
    if (lambert) return kClassDiffuse;
    if (delta) return kClassSpecular;
    return kClassNone;
}

// A box containing every point at which a primitive's reference test can report a hit, for a
// leaf record `w` whose getBounds() box is `gb`. Two effects make it larger than `gb`:
//  1. Quad::intersect accepts plane points with 0 <= (p-O).u <= |u|^2 and 0 <= (p-O).v <= |v|^2
//     (src/geometry/quad.cpp:30-37). For non-orthogonal u, v that is the parallelogram with
//     corners O + x u + y v, (x, y) = A^-1 (a, b), A = [[u.u, u.v], [u.v, v.v]],
//     (a, b) in {0, |u|^2} x {0, |v|^2} -- not the parallelogram (O, u, v) that
//     Quad::getBounds (quad.cpp:44-51) boxes. (The reference's own BVH misses hits there.)
//  2. Near grazing incidence a test's distance t carries a large rounding error: the tests
//     reject only |e1.(d x e2)| < 1e-4 or |n.d| < 1e-4 (an absolute EPSILON), so t may be off
//     by about 2^-24 * L / 1e-4 times the primitive's size factor, L bounding the distances
//     involved (4x the largest coordinate). Boxes grow by 4x that bound; a sphere's tangent
//     point moves along the tangent by ~2^-12 L, leaving its box by at most (2^-12 L)^2 / 2r.
std::vector<MaterialDev> device_materials(const rbr_material* src, uint32_t n) {
    std::vector<MaterialDev> mats(n);
    for (uint32_t i = 0; i < n; ++i) {
        const rbr_material& m = src[i];
        MaterialDev& o = mats[i];
        std::memcpy(o.base, m.base_color, 12);
        o.metallic = m.metallic;
        o.roughness = m.roughness;
        o.ior = m.ior;
        o.transmission = m.transmission;
        std::memcpy(o.emission, m.emission, 12);
        o.cls = material_class(m);
        o.emissive = (m.emission[0] > 0.0f || m.emission[1] > 0.0f || m.emission[2] > 0.0f) ? 1u : 0u;
    }
    return mats;
}

std::vector<LightDev> device_lights(const rbr_light* src, uint32_t n) {
    std::vector<LightDev> lights(n);
    for (uint32_t i = 0; i < n; ++i) {
        const rbr_light& l = src[i];
        LightDev& o = lights[i];
        o.type = l.type;
        std::memcpy(o.position, l.position, 12);
        std::memcpy(o.u, l.u, 12);
        std::memcpy(o.v, l.v, 12);
        std::memcpy(o.color, l.color, 12);
        o.intensity = l.intensity;
        const V3 c = cross(ld(l.u), ld(l.v));
        const V3 nn = normalized(c);  // AreaLight::AreaLight (area_light.cpp:5-11)
        o.normal[0] = nn.x;
        o.normal[1] = nn.y;
        o.normal[2] = nn.z;
        o.area = std::sqrt(dot(c, c));  // cross(u, v).length() (area_light.cpp:33)
    }
    return lights;
}

void set_medium(DeviceScene& s, const rbr_medium* m) {
    s.has_medium = m ? 1u : 0u;
    if (!m) return;
    // Color sigma_t = sigma_a + sigma_s; avgSigmaT = (x + y + z) / 3 (medium.cpp:13-14)
    for (int a = 0; a < 3; ++a) {
        s.sigma_s[a] = m->sigma_s[a];
        s.sigma_t[a] = m->sigma_a[a] + m->sigma_s[a];
    }
    s.avg_sigma_t = (s.sigma_t[0] + s.sigma_t[1] + s.sigma_t[2]) / 3.0f;
    s.hg_g = m->g;
}

Box hit_region_box(const uint32_t* w, const Box& gb, float maxabs) {
    float f[12];
    std::memcpy(f, w, sizeof(f));
    const uint32_t type = w[9] >> kTypeShift;
    const double eps = 1.0 / 16777216.0, L = 4.0 * maxabs, K = 4.0;
    double lo[3] = {gb.lo[0], gb.lo[1], gb.lo[2]}, hi[3] = {gb.hi[0], gb.hi[1], gb.hi[2]};
    double pad = 0.0;
    if (type == kPrimTriangle) {
        const double l1 = std::sqrt(double(f[3]) * f[3] + double(f[4]) * f[4] + double(f[5]) * f[5]);
        const double l2 = std::sqrt(double(f[6]) * f[6] + double(f[7]) * f[7] + double(f[8]) * f[8]);
        pad = K * eps * L * std::max(1.0, l1 * l2 / 1e-4);
    } else if (type == kPrimSphere) {
        const double r = f[3], s = L / 4096.0;
        pad = K * std::max(r > 0.0 ? s * s / (2.0 * r) : 0.0, 4.0 * eps * L);
    } else {  // quad
        const double O[3] = {f[0], f[1], f[2]}, u[3] = {f[3], f[4], f[5]}, v[3] = {f[6], f[7], f[8]};
        const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        const double vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        const double uv = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
        const double det = uu * vv - uv * uv;
        if (det > 1e-12 * uu * vv) {
            const double ab[4][2] = {{0, 0}, {uu, 0}, {0, vv}, {uu, vv}};
            for (const auto& c : ab) {
                const double x = (c[0] * vv - c[1] * uv) / det, y = (c[1] * uu - c[0] * uv) / det;
                for (int a = 0; a < 3; ++a) {
                    const double p = O[a] + x * u[a] + y * v[a];
                    lo[a] = std::min(lo[a], p);
                    hi[a] = std::max(hi[a], p);
                }
            }
        }
        pad = K * eps * L * 3.0 / 1e-4;
    }
    pad = std::min(pad, L);
    Box out;
    for (int a = 0; a < 3; ++a) {
        out.lo[a] = static_cast<float>(lo[a] - pad);
        out.hi[a] = static_cast<float>(hi[a] + pad);
        if (out.lo[a] > lo[a] - pad) out.lo[a] = std::nextafter(out.lo[a], -FLT_MAX);
        if (out.hi[a] < hi[a] + pad) out.hi[a] = std::nextafter(out.hi[a], FLT_MAX);
    }
    return out;
}

template <class T>
rbr_status upload(rbr_ctx* ctx, const std::vector<T>& host, const char* what, void** out) {
    *out = nullptr;
    if (host.empty()) return RBR_OK;
    DevBuf b;
    b.bytes = host.size() * sizeof(T);
    cudaError_t e = cudaMalloc(&b.ptr, b.bytes);
    if (e != cudaSuccess) return fail(ctx, RBR_ERR_OUT_OF_MEMORY, std::string("cudaMalloc for ") + what + ": " + cudaGetErrorString(e));
    ctx->scene_bufs.push_back(b);
    e = cudaMemcpy(b.ptr, host.data(), b.bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(ctx, e, what);
    ctx->stats.device_bytes += b.bytes;
    *out = b.ptr;
    return RBR_OK;
}

}  // namespace

void free_scene(rbr_ctx* ctx) {
    for (auto& b : ctx->scene_bufs) release(b);
    ctx->scene_bufs.clear();
    ctx->scene = DeviceScene{};
    ctx->bvh_base = nullptr;
    ctx->bvh_bytes = 0;
    ctx->has_scene = false;
    ctx->stats = rbr_scene_stats{};
}

rbr_status upload_scene(rbr_ctx* ctx, const rbr_scene_desc* d) {
    if (!d) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "scene description is NULL");
    const auto t0 = std::chrono::steady_clock::now();
    const uint64_t total64 = uint64_t(d->num_triangles) + d->num_spheres + d->num_quads + d->num_planes;
    if (total64 > kIdMask) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "too many primitives (limit 2^30 - 1)");
    const uint32_t total = static_cast<uint32_t>(total64);
    struct TypeIn {
        uint32_t n;
        const float* data;
        int stride;
        const uint32_t* mats;
        const uint32_t* ids;
        const char* name;
    } types[4] = {
        {d->num_triangles, d->triangle_vertices, 9, d->triangle_materials, d->triangle_ids, "triangle"},
        {d->num_spheres, d->spheres, 4, d->sphere_materials, d->sphere_ids, "sphere"},
        {d->num_quads, d->quads, 9, d->quad_materials, d->quad_ids, "quad"},
        {d->num_planes, d->planes, 4, d->plane_materials, d->plane_ids, "plane"},
    };
    if (d->num_materials > 0 && !d->materials) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "materials is NULL");
    if (d->num_lights > 0 && !d->lights) return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "lights is NULL");
    // ids and materials
    std::vector<uint32_t> prim_material(total), prim_record(total, 0xFFFFFFFFu);
    std::vector<uint32_t> first_id_of_type(4);
    {
        std::vector<uint8_t> used(total, 0);
        uint32_t next = 0;
        for (int ty = 0; ty < 4; ++ty) {
            const TypeIn& T = types[ty];
            if (T.n && (!T.data || !T.mats))
                return fail(ctx, RBR_ERR_INVALID_ARGUMENT, std::string(T.name) + " data or materials is NULL");
            for (uint32_t i = 0; i < T.n; ++i) {
                const uint32_t id = T.ids ? T.ids[i] : next + i;
                if (id >= total || used[id])
                    return fail(ctx, RBR_ERR_INVALID_ARGUMENT,
                                std::string(T.name) + " ids are not a permutation of 0..N-1 (id " + std::to_string(id) + ")");
                used[id] = 1;
                if (T.mats[i] >= d->num_materials)
                    return fail(ctx, RBR_ERR_INVALID_ARGUMENT,
                                std::string(T.name) + " " + std::to_string(i) + " uses material " +
                                    std::to_string(T.mats[i]) + " of " + std::to_string(d->num_materials));
                if (!finite3(T.data + size_t(T.stride) * i, T.stride))
                    return fail(ctx, RBR_ERR_INVALID_ARGUMENT,
                                std::string(T.name) + " " + std::to_string(i) + " has a non-finite coordinate");
                prim_material[id] = T.mats[i];
            }
            next += T.n;
        }
    }
    for (uint32_t i = 0; i < d->num_materials; ++i) {
        const rbr_material& m = d->materials[i];
        if (!finite3(m.base_color, 3) || !finite3(m.emission, 3) || !std::isfinite(m.metallic) ||
            !std::isfinite(m.roughness) || !std::isfinite(m.ior) || !std::isfinite(m.transmission))
            return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "material " + std::to_string(i) + " has a non-finite parameter");
    }
    if (d->medium && (!finite3(d->medium->sigma_a, 3) || !finite3(d->medium->sigma_s, 3) ||
                      !std::isfinite(d->medium->g) || std::fabs(d->medium->g) >= 1.0f))
        return fail(ctx, RBR_ERR_INVALID_ARGUMENT, "medium has a non-finite coefficient or |g| >= 1");
    for (uint32_t i = 0; i < d->num_lights; ++i) {
        const rbr_light& l = d->lights[i];
        if (l.type != RBR_LIGHT_AREA && l.type != RBR_LIGHT_POINT)
            return fail(ctx, RBR_ERR_UNSUPPORTED, "light " + std::to_string(i) + " has unknown type " + std::to_string(l.type));
    }

    // bounded primitives: boxes (as getBounds() computes them) and record words
    std::vector<Box> boxes;
    std::vector<uint32_t> words;  // kRecordWords per bounded primitive
    std::vector<uint32_t> bounded_id;
    boxes.reserve(total);
    words.reserve(size_t(total) * kRecordWords);
    Box world = empty_box();
    auto put = [&](std::initializer_list<float> f, uint32_t tag, float w10, float w11) {
        uint32_t w[kRecordWords] = {};
        int k = 0;
        for (float x : f) std::memcpy(&w[k++], &x, 4);
        w[9] = tag;
        std::memcpy(&w[10], &w10, 4);
        std::memcpy(&w[11], &w11, 4);
        words.insert(words.end(), w, w + kRecordWords);
    };
    uint32_t next = 0;
    for (uint32_t i = 0; i < d->num_triangles; ++i) {
        const uint32_t id = d->triangle_ids ? d->triangle_ids[i] : next + i;
        const float* p = d->triangle_vertices + 9 * size_t(i);
        const V3 v0 = ld(p), v1 = ld(p + 3), v2 = ld(p + 6);
        const V3 e1 = sub(v1, v0), e2 = sub(v2, v0);
        Box b = empty_box();
        box_point(b, v0);
        box_point(b, v1);
        box_point(b, v2);
        boxes.push_back(b);
        bounded_id.push_back(id);
        put({v0.x, v0.y, v0.z, e1.x, e1.y, e1.z, e2.x, e2.y, e2.z}, id | (kPrimTriangle << kTypeShift), 0.0f, 0.0f);
    }
    next += d->num_triangles;
    for (uint32_t i = 0; i < d->num_spheres; ++i) {
        const uint32_t id = d->sphere_ids ? d->sphere_ids[i] : next + i;
        const float* p = d->spheres + 4 * size_t(i);
        const float r = p[3];
        Box b = empty_box();
        box_point(b, V3{p[0] - r, p[1] - r, p[2] - r});  // BoundingBox(center - r, center + r)
        box_point(b, V3{p[0] + r, p[1] + r, p[2] + r});
        boxes.push_back(b);
        bounded_id.push_back(id);
        put({p[0], p[1], p[2], r, r * r, 0.0f, 0.0f, 0.0f, 0.0f}, id | (kPrimSphere << kTypeShift), 0.0f, 0.0f);
    }
    next += d->num_spheres;
    for (uint32_t i = 0; i < d->num_quads; ++i) {
        const uint32_t id = d->quad_ids ? d->quad_ids[i] : next + i;
        const float* p = d->quads + 9 * size_t(i);
        const V3 o = ld(p), u = ld(p + 3), v = ld(p + 6);
        Box b = empty_box();  // Quad::getBounds (quad.cpp:44-51)
        box_point(b, o);
        box_point(b, add(o, u));
        box_point(b, add(o, v));
        box_point(b, add(add(o, u), v));
        boxes.push_back(b);
        bounded_id.push_back(id);
        put({o.x, o.y, o.z, u.x, u.y, u.z, v.x, v.y, v.z}, id | (kPrimQuad << kTypeShift), dot(u, u), dot(v, v));
    }
    next += d->num_quads;
    std::vector<float4> planes(d->num_planes);
    std::vector<uint32_t> plane_tags(d->num_planes);
    for (uint32_t i = 0; i < d->num_planes; ++i) {
        const uint32_t id = d->plane_ids ? d->plane_ids[i] : next + i;
        const float* p = d->planes + 4 * size_t(i);
        planes[i] = make_float4(p[0], p[1], p[2], p[3]);
        plane_tags[i] = id | (kPrimPlane << kTypeShift);
        prim_record[id] = 0x80000000u | i;
    }
    float maxabs = 1.0f;
    for (const Box& b : boxes) {
        for (int a = 0; a < 3; ++a) {
            world.lo[a] = std::min(world.lo[a], b.lo[a]);
            world.hi[a] = std::max(world.hi[a], b.hi[a]);
            maxabs = std::max(maxabs, std::max(std::fabs(b.lo[a]), std::fabs(b.hi[a])));
        }
    }
    if (d->num_planes) {  // BVH::worldBounds includes the planes' +-FLT_MAX boxes
        for (int a = 0; a < 3; ++a) {
            world.lo[a] = -FLT_MAX;
            world.hi[a] = FLT_MAX;
        }
    }

    // BVH boxes bound where each primitive's test can report a hit, not just its getBounds()
    std::vector<Box> hit_boxes(boxes.size());
    for (size_t b = 0; b < boxes.size(); ++b) hit_boxes[b] = hit_region_box(&words[b * kRecordWords], boxes[b], maxabs);
    const int threads = std::max(1u, std::thread::hardware_concurrency());
    WideBVH bvh = build_wide_bvh(hit_boxes, maxabs * (1.0f / 1048576.0f), threads, ctx->bvh_record_cost_milli / 1000.0);

    std::vector<uint32_t> records(bvh.leaf_order.size() * kRecordWords);
    for (size_t r = 0; r < bvh.leaf_order.size(); ++r) {
        const uint32_t b = bvh.leaf_order[r];
        std::memcpy(&records[r * kRecordWords], &words[size_t(b) * kRecordWords], kRecordWords * 4);
        prim_record[bounded_id[b]] = static_cast<uint32_t>(r);
    }
    std::vector<float4> tri_normals;
    if (d->triangle_normals && d->num_triangles) {
        tri_normals.assign(bvh.leaf_order.size() * 3, make_float4(0, 0, 0, 0));
        for (size_t r = 0; r < bvh.leaf_order.size(); ++r) {
            const uint32_t b = bvh.leaf_order[r];
            if (b >= d->num_triangles) continue;  // triangles come first in the bounded list
            const float* n = d->triangle_normals + 9 * size_t(b);
            for (int k = 0; k < 3; ++k) tri_normals[3 * r + k] = make_float4(n[3 * k], n[3 * k + 1], n[3 * k + 2], 0.0f);
        }
    }
    std::vector<MaterialDev> mats = device_materials(d->materials, d->num_materials);
    std::vector<LightDev> lights = device_lights(d->lights, d->num_lights);

    free_scene(ctx);
    ctx->stats.device_bytes = 0;
    DeviceScene s{};
    void* p = nullptr;
    rbr_status st;
    // nodes and leaf records in one allocation (records right after the nodes, 16-byte aligned
    // since a node is 80 bytes): the traversal's whole read set is one address range, which an
    // L2 access-policy window can cover ("trace.l2_persist")
    {
        std::vector<uint32_t> bvh_words(bvh.nodes.size() + records.size());
        std::copy(bvh.nodes.begin(), bvh.nodes.end(), bvh_words.begin());
        std::copy(records.begin(), records.end(), bvh_words.begin() + static_cast<std::ptrdiff_t>(bvh.nodes.size()));
        if ((st = upload(ctx, bvh_words, "BVH nodes and leaf records", &p)) != RBR_OK) return free_scene(ctx), st;
        s.nodes = bvh.nodes.empty() ? nullptr : static_cast<const uint4*>(p);
        s.records = records.empty() ? nullptr : reinterpret_cast<const float4*>(static_cast<const uint32_t*>(p) + bvh.nodes.size());
        ctx->bvh_base = p;
        ctx->bvh_bytes = bvh_words.size() * 4;
    }
    if ((st = upload(ctx, planes, "planes", &p)) != RBR_OK) return free_scene(ctx), st;
    s.planes = static_cast<const float4*>(p);
    if ((st = upload(ctx, plane_tags, "plane tags", &p)) != RBR_OK) return free_scene(ctx), st;
    s.plane_tags = static_cast<const uint32_t*>(p);
    if ((st = upload(ctx, prim_record, "primitive records", &p)) != RBR_OK) return free_scene(ctx), st;
    s.prim_record = static_cast<const uint32_t*>(p);
    if ((st = upload(ctx, prim_material, "primitive materials", &p)) != RBR_OK) return free_scene(ctx), st;
    s.prim_material = static_cast<const uint32_t*>(p);
    if ((st = upload(ctx, tri_normals, "triangle normals", &p)) != RBR_OK) return free_scene(ctx), st;
    s.tri_normals = static_cast<const float4*>(p);
    if ((st = upload(ctx, mats, "materials", &p)) != RBR_OK) return free_scene(ctx), st;
    s.materials = static_cast<const MaterialDev*>(p);
    if ((st = upload(ctx, lights, "lights", &p)) != RBR_OK) return free_scene(ctx), st;
    s.lights = static_cast<const LightDev*>(p);
    s.num_nodes = static_cast<uint32_t>(bvh.nodes.size() / kNodeWords);
    s.num_planes = d->num_planes;
    s.num_materials = d->num_materials;
    s.num_lights = d->num_lights;
    std::memcpy(s.background, d->background, 12);
    set_medium(s, d->medium);
    ctx->scene = s;
    ctx->has_scene = true;
    for (int a = 0; a < 3; ++a) {
        ctx->bounds_lo[a] = world.lo[a];
        ctx->bounds_hi[a] = world.hi[a];
    }
    ctx->stats.num_primitives = total;
    ctx->stats.num_bounded = static_cast<uint32_t>(boxes.size());
    ctx->stats.num_unbounded = d->num_planes;
    ctx->stats.num_wide_nodes = s.num_nodes;
    ctx->stats.num_leaf_records = static_cast<uint32_t>(bvh.leaf_order.size());
    ctx->stats.max_depth = bvh.max_depth;
    ctx->stats.wrapped_leaves = bvh.wrapped_leaves;
    ctx->stats.record_cost_milli = static_cast<uint32_t>(ctx->bvh_record_cost_milli);
    ctx->stats.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (bvh.max_depth >= static_cast<uint32_t>(kStackSize))
        return fail(ctx, RBR_ERR_INTERNAL, "BVH deeper than the traversal stack");
    return RBR_OK;
}

// A scene that shares `base`'s geometry and BVH (device buffers owned by `base`) with its
// own materials, lights and medium. `dst` owns only the new arrays.
rbr_status upload_scene_variant(rbr_ctx* dst, const rbr_ctx* base, const rbr_material* materials, uint32_t num_materials,
                                const rbr_light* lights, uint32_t num_lights, const rbr_medium* medium) {
    if (!base->has_scene) return fail(dst, RBR_ERR_NO_SCENE, "the base scene is empty");
    if (num_materials != base->scene.num_materials || (num_materials && !materials) || (num_lights && !lights))
        return fail(dst, RBR_ERR_INVALID_ARGUMENT, "a variant needs as many materials as its base scene (" +
                                                       std::to_string(base->scene.num_materials) + ")");
    for (uint32_t i = 0; i < num_materials; ++i) {
        const rbr_material& m = materials[i];
        if (!finite3(m.base_color, 3) || !finite3(m.emission, 3) || !std::isfinite(m.metallic) ||
            !std::isfinite(m.roughness) || !std::isfinite(m.ior) || !std::isfinite(m.transmission))
            return fail(dst, RBR_ERR_INVALID_ARGUMENT, "material " + std::to_string(i) + " has a non-finite parameter");
    }
    for (uint32_t i = 0; i < num_lights; ++i)
        if (lights[i].type != RBR_LIGHT_AREA && lights[i].type != RBR_LIGHT_POINT)
            return fail(dst, RBR_ERR_UNSUPPORTED, "light " + std::to_string(i) + " has unknown type");
    free_scene(dst);
    dst->stats.device_bytes = 0;
    DeviceScene s = base->scene;
    void* p = nullptr;
    rbr_status st;
    if ((st = upload(dst, device_materials(materials, num_materials), "materials", &p)) != RBR_OK) return free_scene(dst), st;
    s.materials = static_cast<const MaterialDev*>(p);
    if ((st = upload(dst, device_lights(lights, num_lights), "lights", &p)) != RBR_OK) return free_scene(dst), st;
    s.lights = static_cast<const LightDev*>(p);
    s.num_lights = num_lights;
    set_medium(s, medium);
    dst->scene = s;
    dst->bvh_base = base->bvh_base;
    dst->bvh_bytes = base->bvh_bytes;
    dst->has_scene = true;
    for (int a = 0; a < 3; ++a) {
        dst->bounds_lo[a] = base->bounds_lo[a];
        dst->bounds_hi[a] = base->bounds_hi[a];
    }
    const uint64_t own = dst->stats.device_bytes;
    dst->stats = base->stats;
    dst->stats.device_bytes = own;
    return RBR_OK;
}

}  // namespace rbr
