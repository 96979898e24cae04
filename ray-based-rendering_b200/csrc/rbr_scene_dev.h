// Plain structs describing a scene in device memory (usable from host C++ and from kernels).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rbr {

// Shading classes: paths are bucketed by the class of the material they hit so that one
// warp shades one kind of BSDF.
// Shading classes of a material, by the lobes Material::createBSDF gives it: Lambertian (and
// delta) lobes only; GGX reflection with a Lambertian lobe (plastics); delta lobes only; no
// lobes; GGX reflection only (metals); GGX with GGX transmission (rough glass). The path tracer
// queues hits per class, so that a warp of the shading kernel runs one lobe combination.
enum : uint32_t {
    kClassDiffuse = 0,
    kClassGlossy = 1,
    kClassSpecular = 2,
    kClassNone = 3,
    kClassGlossyRefl = 4,
    kClassGlossyTrans = 5,
    kNumClasses = 6
};

struct MaterialDev {
    float base[3];
    float metallic, roughness, ior, transmission;
    float emission[3];
    uint32_t cls;     // kClass*: any GGX lobe -> glossy; else Lambertian -> diffuse; else delta-only
                      // -> specular; no lobe at all (lights, black) -> none
    uint32_t emissive;
};

struct LightDev {
    uint32_t type;
    float position[3], u[3], v[3], color[3];
    float intensity;
    float normal[3];  // normalize(u x v), AreaLight::AreaLight
    float area;       // |u x v|
};

// Everything a kernel needs to read a scene. Passed by value.
struct DeviceScene {
    const uint4* nodes;      // kNodeWords/4 uint4 per node
    const float4* records;   // 3 float4 per leaf record
    const float4* planes;    // per plane: (unit normal, d)
    const uint32_t* plane_tags;
    uint32_t num_nodes;
    uint32_t num_planes;
    // shading data, indexed by primitive id
    const uint32_t* prim_record;   // leaf record index, or (plane index | 0x80000000)
    const uint32_t* prim_material;
    const float4* tri_normals;     // 3 float4 per leaf record of a triangle with normals, or null
    const MaterialDev* materials;
    const LightDev* lights;
    uint32_t num_materials;
    uint32_t num_lights;
    float background[3];
    // homogeneous medium (HomogeneousMedium, src/materials/medium.cpp:9-44)
    uint32_t has_medium;
    float sigma_s[3];
    float sigma_t[3];   // sigma_a + sigma_s
    float avg_sigma_t;  // (sigma_t.x + sigma_t.y + sigma_t.z) / 3
    float hg_g;         // Henyey-Greenstein asymmetry
};

// A PinholeCamera or ThinLensCamera (rbr_camera) as the kernels read it.
struct CameraDev {
    int32_t width, height;
    uint32_t model;
    float position[3], forward[3], right[3], up[3];
    float fx, fy, cx, cy;
    float lens_radius, focal_distance;
};

// One request's share of a packed wave of the batched request loop: a range of its pixels
// with all their samples.
struct SegDev {
    CameraDev cam;
    float* film;             // the request's film (per-pixel mean, width*height*3)
    uint64_t seed;
    uint32_t path0, npaths;  // its paths in the wave
    uint32_t p0;             // its first pixel in the request's image
    uint32_t spp, sample_offset, width, max_depth, use_nee, use_mis;
};

// Device segment tables of the batched loop: a 64-byte header ([0] paths of the wave, [1]
// segments) followed by the wave's SegDev entries.
constexpr uint32_t kSegTableHeader = 64;

// One wave of a persistent batched run (k_wave_loop): its scene, integrator mode (0 path
// tracer, 2 volumetric), depth iterations, the byte offset of its segment table in the run's
// table array, and the earliest device time (ns after the run's start) at which it may start:
// the arrival of its last request.
struct LoopWave {
    uint32_t scene, mode, max_depth, table;
    uint64_t release_ns;
};

}  // namespace rbr
