// GpuPathIntegrator: a render::Integrator (include/render/renderers/integrator.h:37-73) whose
// render() runs the wavefront path tracer of librbr_b200 on the GPU.
//
// render(scene, camera, film) flattens the scene (primitives, six-parameter materials, area
// and point lights, background), uploads it once per scene contents, renders
// config.samplesPerPixel samples per pixel with config.maxDepth, useNEE and useMIS, and adds
// one averaged sample per pixel to the film, as Integrator::render does
// (src/renderers/integrator.cpp:36). The estimator is the reference's
// PathTracingIntegrator::Li, quirks included: emission only at depth 0 or after a delta
// bounce, MIS weights on light samples without the BSDF-sampled emitter term, next-event
// estimation over every light, Russian roulette always on after depth 3.
//
// With volumetric = true it is the drop-in for VolumetricPathIntegrator
// (src/renderers/volumetric_path_integrator.cpp): the scene's HomogeneousMedium is uploaded and
// the GPU runs that integrator's estimator (RBR_RENDER_VOLUMETRIC). Without it, as
// PathTracingIntegrator does, the medium is ignored.
//
// Unsupported input — a Material subclass with its own createBSDF(), a camera other than
// PinholeCamera/ThinLensCamera, a light other than AreaLight/PointLight, in volumetric mode a
// medium other than HomogeneousMedium with a Henyey-Greenstein phase function — leaves the
// film untouched and is reported by status()/error(). There is no CPU fallback; Li() for
// single rays is not provided on the GPU and returns black with status RBR_ERR_UNSUPPORTED.
#pragma once

#include <cstdint>
#include <mutex>
#include <string>

#include "rbr_b200.h"
#include "render/renderers/integrator.h"

namespace render {

class GpuPathIntegrator : public Integrator {
public:
    explicit GpuPathIntegrator(const IntegratorConfig& config = IntegratorConfig(), int device = 0,
                               uint64_t seed = 0, bool volumetric = false);
    ~GpuPathIntegrator() override;
    GpuPathIntegrator(const GpuPathIntegrator&) = delete;
    GpuPathIntegrator& operator=(const GpuPathIntegrator&) = delete;

    std::string name() const override { return volumetric_ ? "GPU Volumetric Path Tracing" : "GPU Path Tracing"; }
    Color Li(const Ray& ray, const Scene& scene, Sampler& sampler) const override;
    void render(const Scene& scene, const Camera& camera, Film& film,
                std::function<void(float)> progress = nullptr) const override;

    rbr_status status() const { return status_; }
    const std::string& error() const { return error_; }
    // Device milliseconds of the last render.
    float lastMilliseconds() const { return last_ms_; }

private:
    bool upload(const Scene& scene) const;

    rbr_ctx* ctx_ = nullptr;
    uint64_t seed_;
    bool volumetric_;
    mutable std::mutex mu_;
    mutable const Scene* uploaded_ = nullptr;
    mutable size_t uploaded_count_ = 0;
    mutable rbr_status status_ = RBR_OK;
    mutable std::string error_;
    mutable float last_ms_ = 0.0f;
};

}  // namespace render
