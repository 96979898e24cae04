// Flattens reference scene objects into the plain arrays of rbr_scene_desc.
#pragma once

#include <string>
#include <unordered_map>
#include <vector>

#include "rbr_b200.h"
#include "render/geometry/primitive.h"
#include "render/lighting/light.h"
#include "render/materials/material.h"
#include "render/materials/medium.h"

namespace render {

// Owns the arrays an rbr_scene_desc points to.
struct FlatScene {
    std::vector<float> tri, tri_normals, sph, quad, plane;
    std::vector<uint32_t> tri_mat, tri_id, sph_mat, sph_id, quad_mat, quad_id, plane_mat, plane_id;
    std::vector<rbr_material> materials;
    std::vector<rbr_light> lights;
    rbr_medium medium{};
    bool has_medium = false;
    bool any_normals = false;
    rbr_scene_desc desc{};

    // Builds `desc` from the vectors (call after filling them).
    void finalize(const float background[3]);
};

// Adds `prims` (ids = their position in the vector). Materials are deduplicated by pointer;
// a primitive without material gets a black diffuse one. `material_check` rejects Material
// subclasses (their createBSDF may differ from the six-parameter model the GPU reproduces).
// Returns false with `error` set for an unsupported primitive or material.
bool flatten_primitives(const std::vector<const Primitive*>& prims, bool material_check, FlatScene& out,
                        std::string& error);

// Adds AreaLight / PointLight lights; false with `error` for any other light type.
bool flatten_lights(const std::vector<const Light*>& lights, FlatScene& out, std::string& error);

// Sets the scene's HomogeneousMedium with its Henyey-Greenstein phase function; false with
// `error` for any other medium or phase function.
bool flatten_medium(const Medium* medium, FlatScene& out, std::string& error);

}  // namespace render
