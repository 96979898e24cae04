// The reference's own non-path-tracing integrators (Whitted, simple, normals, depth, ambient
// occlusion) rendering the reference's Cornell box with GpuBVHAccelerator as the scene's
// accelerator, selected through Scene::setAcceleratorType the way a registration of
// GpuBVHAccelerator in the reference's accelerator factory selects it: every image equals the one rendered through the reference's BVH
// (the GPU answers each per-ray query with the same primitive and the same t). This is the
// per-ray path of the accelerator drop-in, one launch per query and micro-batched (queries of
// the integrators' OpenMP threads gathered into one launch); the render times of the three are
// printed. Exit code 0 = all checks passed. Needs a CUDA device.

#include <chrono>
#include <cmath>
#include <iostream>
#include <memory>
#include <string>
#include <thread>

#include "cornell_box/cornell_box.h"
#include "gpu_accelerator.h"
#include "render/acceleration/accelerator_factory.h"
#include "render/acceleration/bvh.h"
#include "render/renderers/debug_integrators.h"
#include "render/renderers/simple_integrator.h"
#include "render/renderers/whitted_integrator.h"

namespace render {

// The factory entry a maintainer adds (src/acceleration/accelerator_factory.cpp:13-25 with a
// new AcceleratorType value). This test binary is linked with -rdynamic, so this definition
// stands in for the library's: the stock BVH for every existing type, the GPU accelerator for
// the new value.
constexpr AcceleratorType kGpuBVH = static_cast<AcceleratorType>(100);
// and one more for the micro-batched per-ray path
constexpr AcceleratorType kGpuBVHBatched = static_cast<AcceleratorType>(101);
GpuBVHAccelerator* g_batched = nullptr;  // the micro-batched instance, for its launch counts

std::unique_ptr<Accelerator> createAccelerator(AcceleratorType type) {
    if (type == kGpuBVH) return std::make_unique<GpuBVHAccelerator>(0);
    if (type == kGpuBVHBatched) {
        auto a = std::make_unique<GpuBVHAccelerator>(0);
        const size_t threads = std::max(1u, std::thread::hardware_concurrency());
        a->setMicroBatching(threads, 100);
        g_batched = a.get();
        return a;
    }
    return std::make_unique<BVH>();
}

}  // namespace render

using namespace render;

namespace {

int failures = 0;

void check(bool ok, const std::string& what) {
    if (!ok) {
        std::cerr << "FAIL: " << what << "\n";
        ++failures;
    }
}

double render_ms(const Integrator& integ, const Scene& scene, const Camera& cam, Film& film) {
    const auto t0 = std::chrono::steady_clock::now();
    integ.render(scene, cam, film);
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

int count_differ(const Film& a, const Film& b, int w, int h, double* maxd, double* sum) {
    int differ = 0;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const Color p = a.getPixel(x, y), q = b.getPixel(x, y);
            const double d = std::fabs(p.x - q.x) + std::fabs(p.y - q.y) + std::fabs(p.z - q.z);
            if (d > 0.0) ++differ;
            *maxd = std::max(*maxd, d);
            *sum += p.x + p.y + p.z;
        }
    return differ;
}

void compare(const char* name, const Integrator& integ, const Scene& cpu, const Scene& gpu, const Scene& gpub,
             const Camera& cam, int w, int h) {
    Film a(w, h), b(w, h), c(w, h);
    const double ta = render_ms(integ, cpu, cam, a);
    const double tb = render_ms(integ, gpu, cam, b);
    const uint64_t l0 = g_batched->perRayLaunches(), r0 = g_batched->perRayRays();
    const double tc = render_ms(integ, gpub, cam, c);
    const uint64_t launches = g_batched->perRayLaunches() - l0, rays = g_batched->perRayRays() - r0;
    double maxd = 0.0, sum = 0.0, maxc = 0.0, sumc = 0.0;
    const int differ = count_differ(a, b, w, h, &maxd, &sum);
    const int differc = count_differ(a, c, w, h, &maxc, &sumc);
    std::cout << name << ": " << differ << " of " << w * h << " pixels differ (max " << maxd << "), micro-batched "
              << differc << "; image sum " << sum << "; ms: BVH " << ta << ", GPU per ray " << tb << ", GPU micro-batched "
              << tc << " (" << rays << " queries in " << launches << " launches)\n";
    check(differ == 0, std::string(name) + ": GPU-accelerated image equals the BVH image");
    check(differc == 0, std::string(name) + ": micro-batched GPU image equals the BVH image");
    check(sum > 0.0, std::string(name) + ": image is not black");
}

}  // namespace

int main() {
    const int W = 40, H = 40;
    Scene cpu = cornell_box::createScene(false);
    Scene gpu = cornell_box::createScene(false);
    gpu.setAcceleratorType(kGpuBVH);
    gpu.buildAccelerator();
    cpu.setAcceleratorType(AcceleratorType::BVH);
    cpu.buildAccelerator();
    Scene gpub = cornell_box::createScene(false);
    gpub.setAcceleratorType(kGpuBVHBatched);
    gpub.buildAccelerator();
    auto cam = cornell_box::createCamera(W, H);
    {
        // the accelerator in place is the GPU one and it is healthy
        UniformSampler s(1);
        SurfaceInteraction is;
        const bool hit = gpu.intersect(Ray(Vec3(0.0f, 1.0f, 3.0f), Vec3(0.0f, 0.0f, -1.0f)), is);
        check(hit, "a ray through the box hits the back wall on the GPU");
    }
    IntegratorConfig cfg;
    cfg.maxDepth = 5;
    cfg.samplesPerPixel = 2;
    compare("Whitted", WhittedIntegrator(cfg), cpu, gpu, gpub, *cam, W, H);
    compare("Simple", SimpleIntegrator(cfg), cpu, gpu, gpub, *cam, W, H);
    compare("Normals", NormalIntegrator(), cpu, gpu, gpub, *cam, W, H);
    compare("Depth", DepthIntegrator(0.1f, 10.0f), cpu, gpu, gpub, *cam, W, H);
    compare("AmbientOcclusion", AOIntegrator(4, 2.0f), cpu, gpu, gpub, *cam, W, H);
    if (failures == 0) std::cout << "All GPU-accelerator integrator tests passed\n";
    return failures == 0 ? 0 : 1;
}
