#include "scene_flatten.h"

#include <typeinfo>

#include "render/geometry/plane.h"
#include "render/geometry/quad.h"
#include "render/geometry/sphere.h"
#include "render/geometry/triangle.h"
#include "render/lighting/area_light.h"
#include "render/lighting/point_light.h"

namespace render {

namespace {
void put(std::vector<float>& v, const Vec3& a) {
    v.push_back(a.x);
    v.push_back(a.y);
    v.push_back(a.z);
}
void put3(float* o, const Vec3& a) {
    o[0] = a.x;
    o[1] = a.y;
    o[2] = a.z;
}
}  // namespace

bool flatten_primitives(const std::vector<const Primitive*>& prims, bool material_check, FlatScene& out,
                        std::string& error) {
    std::unordered_map<const Material*, uint32_t> mat_index;
    auto material_of = [&](const Material* m, uint32_t& idx) -> bool {
        auto it = mat_index.find(m);
        if (it != mat_index.end()) {
            idx = it->second;
            return true;
        }
        rbr_material r{};
        if (m) {
            if (material_check && typeid(*m) != typeid(Material)) {
                error = std::string("material of type ") + typeid(*m).name() +
                        " derives from Material; its createBSDF() is not reproduced on the GPU";
                return false;
            }
            put3(r.base_color, m->baseColor);
            r.metallic = m->metallic;
            r.roughness = m->roughness;
            r.ior = m->ior;
            r.transmission = m->transmission;
            put3(r.emission, m->emission);
        } else {  // no material: nothing is scattered or emitted
            r.roughness = 1.0f;
            r.ior = 1.0f;
        }
        idx = static_cast<uint32_t>(out.materials.size());
        out.materials.push_back(r);
        mat_index[m] = idx;
        return true;
    };
    // two passes: normals are all-or-nothing per scene in the C ABI
    for (const Primitive* p : prims) {
        if (auto t = dynamic_cast<const Triangle*>(p)) out.any_normals |= t->hasNormals;
    }
    for (uint32_t id = 0; id < prims.size(); ++id) {
        const Primitive* p = prims[id];
        uint32_t m = 0;
        if (!p) {
            error = "null primitive at index " + std::to_string(id);
            return false;
        }
        if (!material_of(p->material, m)) return false;
        if (auto t = dynamic_cast<const Triangle*>(p)) {
            put(out.tri, t->v0);
            put(out.tri, t->v1);
            put(out.tri, t->v2);
            if (out.any_normals) {
                // without vertex normals the geometric normal is used; give all three the face normal
                const Vec3 fn = t->hasNormals ? Vec3(0.0f) : t->faceNormal();
                put(out.tri_normals, t->hasNormals ? t->n0 : fn);
                put(out.tri_normals, t->hasNormals ? t->n1 : fn);
                put(out.tri_normals, t->hasNormals ? t->n2 : fn);
            }
            out.tri_mat.push_back(m);
            out.tri_id.push_back(id);
        } else if (auto s = dynamic_cast<const Sphere*>(p)) {
            put(out.sph, s->center);
            out.sph.push_back(s->radius);
            out.sph_mat.push_back(m);
            out.sph_id.push_back(id);
        } else if (auto q = dynamic_cast<const Quad*>(p)) {
            put(out.quad, q->origin);
            put(out.quad, q->u);
            put(out.quad, q->v);
            out.quad_mat.push_back(m);
            out.quad_id.push_back(id);
        } else if (auto pl = dynamic_cast<const Plane*>(p)) {
            put(out.plane, pl->normal);
            out.plane.push_back(pl->d);
            out.plane_mat.push_back(m);
            out.plane_id.push_back(id);
        } else {
            error = std::string("unsupported primitive type ") + typeid(*p).name() + " at index " + std::to_string(id);
            return false;
        }
    }
    return true;
}

bool flatten_lights(const std::vector<const Light*>& lights, FlatScene& out, std::string& error) {
    for (const Light* l : lights) {
        rbr_light r{};
        if (auto a = dynamic_cast<const AreaLight*>(l)) {
            r.type = RBR_LIGHT_AREA;
            put3(r.position, a->position);
            put3(r.u, a->u);
            put3(r.v, a->v);
        } else if (auto pt = dynamic_cast<const PointLight*>(l)) {
            r.type = RBR_LIGHT_POINT;
            put3(r.position, pt->position);
        } else {
            error = std::string("unsupported light type ") + typeid(*l).name();
            return false;
        }
        put3(r.color, l->color);
        r.intensity = l->intensity;
        out.lights.push_back(r);
    }
    return true;
}

bool flatten_medium(const Medium* medium, FlatScene& out, std::string& error) {
    const auto* h = dynamic_cast<const HomogeneousMedium*>(medium);
    const auto* hg = h ? dynamic_cast<const HenyeyGreensteinPhase*>(h->getPhaseFunction()) : nullptr;
    if (!h || !hg) {
        error = std::string("unsupported medium ") + (medium ? typeid(*medium).name() : "(null)") +
                " (the GPU path implements HomogeneousMedium with a Henyey-Greenstein phase function)";
        return false;
    }
    put3(out.medium.sigma_a, h->sigma_a);
    put3(out.medium.sigma_s, h->sigma_s);
    out.medium.g = hg->g;
    out.has_medium = true;
    return true;
}

void FlatScene::finalize(const float background[3]) {
    desc = rbr_scene_desc{};
    desc.num_triangles = static_cast<uint32_t>(tri_mat.size());
    desc.triangle_vertices = tri.data();
    desc.triangle_normals = any_normals ? tri_normals.data() : nullptr;
    desc.triangle_materials = tri_mat.data();
    desc.triangle_ids = tri_id.data();
    desc.num_spheres = static_cast<uint32_t>(sph_mat.size());
    desc.spheres = sph.data();
    desc.sphere_materials = sph_mat.data();
    desc.sphere_ids = sph_id.data();
    desc.num_quads = static_cast<uint32_t>(quad_mat.size());
    desc.quads = quad.data();
    desc.quad_materials = quad_mat.data();
    desc.quad_ids = quad_id.data();
    desc.num_planes = static_cast<uint32_t>(plane_mat.size());
    desc.planes = plane.data();
    desc.plane_materials = plane_mat.data();
    desc.plane_ids = plane_id.data();
    desc.num_materials = static_cast<uint32_t>(materials.size());
    desc.materials = materials.data();
    desc.num_lights = static_cast<uint32_t>(lights.size());
    desc.lights = lights.data();
    for (int a = 0; a < 3; ++a) desc.background[a] = background[a];
    desc.medium = has_medium ? &medium : nullptr;
}

}  // namespace render
