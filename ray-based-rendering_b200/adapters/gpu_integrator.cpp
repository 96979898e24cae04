#include "gpu_integrator.h"

#include <vector>

#include "render/camera/pinhole_camera.h"
#include "render/camera/thin_lens_camera.h"
#include "scene_flatten.h"

namespace render {

GpuPathIntegrator::GpuPathIntegrator(const IntegratorConfig& config, int device, uint64_t seed, bool volumetric)
    : Integrator(config), seed_(seed), volumetric_(volumetric) {
    status_ = rbr_ctx_create(device, &ctx_);
    if (status_ != RBR_OK) error_ = "rbr_ctx_create failed (no usable CUDA device)";
}

GpuPathIntegrator::~GpuPathIntegrator() { rbr_ctx_destroy(ctx_); }

Color GpuPathIntegrator::Li(const Ray&, const Scene&, Sampler&) const {
    std::lock_guard<std::mutex> lock(mu_);
    status_ = RBR_ERR_UNSUPPORTED;
    error_ = "GpuPathIntegrator traces whole images (render()); single-ray Li is not provided";
    return Color(0.0f);
}

bool GpuPathIntegrator::upload(const Scene& scene) const {
    if (uploaded_ == &scene && uploaded_count_ == scene.primitives().size()) return true;
    FlatScene flat;
    std::vector<const Primitive*> prims;
    for (const auto& p : scene.primitives()) prims.push_back(p.get());
    std::vector<const Light*> lights;
    for (const auto& l : scene.lights()) lights.push_back(l.get());
    std::string err;
    if (!flatten_primitives(prims, /*material_check=*/true, flat, err) || !flatten_lights(lights, flat, err) ||
        (volumetric_ && scene.hasMedium() && !flatten_medium(scene.medium(), flat, err))) {
        status_ = RBR_ERR_UNSUPPORTED;
        error_ = err;
        return false;
    }
    const float bg[3] = {scene.backgroundColor.x, scene.backgroundColor.y, scene.backgroundColor.z};
    flat.finalize(bg);
    status_ = rbr_scene_upload(ctx_, &flat.desc);
    if (status_ != RBR_OK) {
        error_ = rbr_last_error(ctx_);
        return false;
    }
    uploaded_ = &scene;
    uploaded_count_ = scene.primitives().size();
    return true;
}

void GpuPathIntegrator::render(const Scene& scene, const Camera& camera, Film& film,
                               std::function<void(float)> progress) const {
    std::lock_guard<std::mutex> lock(mu_);
    if (!ctx_) return;
    rbr_camera cam{};
    cam.width = film.width;
    cam.height = film.height;
    const auto* thin = dynamic_cast<const ThinLensCamera*>(&camera);
    const auto* persp = dynamic_cast<const PerspectiveCamera*>(&camera);
    if (!persp || (!thin && !dynamic_cast<const PinholeCamera*>(&camera))) {
        status_ = RBR_ERR_UNSUPPORTED;
        error_ = "only PinholeCamera and ThinLensCamera are supported on the GPU";
        return;
    }
    cam.model = thin ? RBR_CAMERA_THIN_LENS : RBR_CAMERA_PINHOLE;
    const CameraExtrinsics& e = camera.extrinsics;
    float* dst[4] = {cam.position, cam.forward, cam.right, cam.up};
    const Vec3* src[4] = {&e.position, &e.forward, &e.right, &e.up};
    for (int i = 0; i < 4; ++i) {
        dst[i][0] = src[i]->x;
        dst[i][1] = src[i]->y;
        dst[i][2] = src[i]->z;
    }
    const PerspectiveIntrinsics& k = persp->perspectiveIntrinsics();
    cam.fx = k.fx;
    cam.fy = k.fy;
    cam.cx = k.cx;
    cam.cy = k.cy;
    cam.lens_radius = thin ? thin->lensRadius : 0.0f;
    cam.focal_distance = thin ? thin->focalDistance : 1.0f;
    if (!upload(scene)) return;
    rbr_render_params p{};
    p.samples_per_pixel = config.samplesPerPixel;
    p.max_depth = config.maxDepth;
    p.use_nee = config.useNEE ? 1 : 0;
    p.use_mis = config.useMIS ? 1 : 0;
    p.seed = seed_;
    p.flags = volumetric_ ? static_cast<uint32_t>(RBR_RENDER_VOLUMETRIC) : 0u;
    std::vector<float> mean(static_cast<size_t>(film.width) * film.height * 3);
    status_ = rbr_render_host(ctx_, &cam, &p, mean.data(), nullptr);
    if (status_ != RBR_OK) {
        error_ = rbr_last_error(ctx_);
        return;
    }
    rbr_render_stats st{};
    if (rbr_render_stats_get(ctx_, &st) == RBR_OK) last_ms_ = st.milliseconds;
    for (int y = 0; y < film.height; ++y) {
        for (int x = 0; x < film.width; ++x) {
            const float* c = &mean[3 * (static_cast<size_t>(y) * film.width + x)];
            film.addSample(x, y, Color(c[0], c[1], c[2]));
        }
    }
    if (progress) progress(1.0f);
}

}  // namespace render
