// GpuBVHAccelerator through the reference's own Accelerator interface: every query must return
// exactly what a brute-force loop over the primitives returns (same primitive, same t bits,
// same surface data), in the style of the reference's tests/test_accelerators.cpp.
// Exit code 0 = all checks passed. Needs a CUDA device.

#include <cmath>
#include <typeinfo>
#include <cstring>
#include <iostream>
#include <memory>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "gpu_accelerator.h"
#include "render/geometry/plane.h"
#include "render/geometry/quad.h"
#include "render/geometry/sphere.h"
#include "render/geometry/triangle.h"

using namespace render;

namespace {

int failures = 0;

void check(bool ok, const std::string& what) {
    if (!ok) {
        std::cerr << "FAIL: " << what << "\n";
        ++failures;
    }
}

struct World {
    std::vector<std::unique_ptr<Primitive>> owned;
    std::vector<Primitive*> prims;
    void add(std::unique_ptr<Primitive> p) {
        prims.push_back(p.get());
        owned.push_back(std::move(p));
    }
};

World randomWorld(std::mt19937& rng, int spheres, int triangles, int quads, bool plane) {
    std::uniform_real_distribution<float> pos(-10.0f, 10.0f), size(0.1f, 1.5f);
    World w;
    for (int i = 0; i < spheres; ++i) w.add(std::make_unique<Sphere>(Vec3(pos(rng), pos(rng), pos(rng)), size(rng)));
    for (int i = 0; i < triangles; ++i) {
        const Vec3 c(pos(rng), pos(rng), pos(rng));
        auto j = [&]() { return Vec3(size(rng), size(rng), size(rng)) - Vec3(0.8f); };
        w.add(std::make_unique<Triangle>(c + j(), c + j(), c + j()));
    }
    for (int i = 0; i < quads; ++i) {
        const Vec3 o(pos(rng), pos(rng), pos(rng));
        w.add(std::make_unique<Quad>(o, Vec3(size(rng), 0.0f, 0.3f), Vec3(0.0f, size(rng), size(rng))));
    }
    for (int i = 0; i < 10; ++i) {  // axis-aligned flat triangles: zero-thickness bounds
        const float x = pos(rng), y = pos(rng), z = pos(rng);
        w.add(std::make_unique<Triangle>(Vec3(x, y, z), Vec3(x + 2, y, z), Vec3(x, y + 2, z)));
    }
    if (plane) w.add(std::make_unique<Plane>(Vec3(0, 1, 0), 12.0f));
    return w;
}

bool bruteForce(const std::vector<Primitive*>& prims, const Ray& ray, SurfaceInteraction& isect) {
    Ray r = ray;
    bool hit = false;
    for (const Primitive* p : prims)
        if (p->intersect(r, isect)) hit = true;
    return hit;
}

bool bits_equal(float a, float b) { return std::memcmp(&a, &b, sizeof(float)) == 0; }
bool same(const Vec3& a, const Vec3& b) { return bits_equal(a.x, b.x) && bits_equal(a.y, b.y) && bits_equal(a.z, b.z); }

void compare(GpuBVHAccelerator& accel, const World& w, std::mt19937& rng, int nRays, const std::string& label) {
    accel.build(w.prims);
    check(accel.status() == RBR_OK, label + ": build status " + accel.error());
    std::uniform_real_distribution<float> pos(-14.0f, 14.0f), dir(-1.0f, 1.0f), len(0.5f, 40.0f);
    int bad = 0, badP = 0, badSurface = 0, hits = 0;
    std::vector<Ray> rays;
    for (int i = 0; i < nRays; ++i) {
        Vec3 d(dir(rng), dir(rng), dir(rng));
        if (i % 3 == 0) d = Vec3(0.0f, 0.0f, (i % 2) ? 1.0f : -1.0f);
        else if (i % 7 == 0) d = Vec3(dir(rng), 0.0f, dir(rng));
        if (d.length() < 1e-3f) continue;
        Ray ray(Vec3(pos(rng), pos(rng), pos(rng)), d);
        if (i % 4 == 0) ray.tMax = len(rng);
        rays.push_back(ray);
    }
    std::vector<rbr_hit> batch(rays.size());
    check(accel.intersectBatch(rays.data(), rays.size(), batch.data()), label + ": batch query");
    for (size_t i = 0; i < rays.size(); ++i) {
        SurfaceInteraction ref, got;
        const bool refHit = bruteForce(w.prims, rays[i], ref);
        hits += refHit;
        Ray r = rays[i];
        const bool hit = accel.intersect(r, got);
        if (hit != refHit || (hit && (got.primitive != ref.primitive || !bits_equal(got.t, ref.t) || !bits_equal(r.tMax, ref.t)))) {
            if (bad < 5) {
                const Primitive* p = refHit ? ref.primitive : got.primitive;
                std::cerr << "  mismatch " << label << " ray " << i << ": ref " << (refHit ? "hit" : "miss") << " t=" << ref.t
                          << " gpu " << (hit ? "hit" : "miss") << " t=" << got.t << " tMax=" << rays[i].tMax << " prim "
                          << (p ? typeid(*p).name() : "-") << " |cos|="
                          << (refHit ? std::fabs(dot(ref.normal, rays[i].direction)) : -1.0f) << "\n";
            }
            ++bad;
        }
        else if (hit && (!same(got.point, ref.point) || !same(got.normal, ref.normal) || got.frontFace != ref.frontFace))
            ++badSurface;
        const bool bh = batch[i].prim != RBR_MISS;
        if (bh != refHit || (bh && (w.prims[batch[i].prim] != ref.primitive || !bits_equal(batch[i].t, ref.t)))) ++bad;
        bool refP = false;
        for (const Primitive* p : w.prims)
            if (p->intersectP(rays[i])) {
                refP = true;
                break;
            }
        if (accel.intersectP(rays[i]) != refP) ++badP;
    }
    check(bad == 0, label + ": closest hit, " + std::to_string(bad) + " mismatches");
    check(badSurface == 0, label + ": surface interaction, " + std::to_string(badSurface) + " mismatches");
    check(badP == 0, label + ": any hit, " + std::to_string(badP) + " mismatches");
    check(hits > nRays / 20, label + ": test rays hit nothing");
}

// A primitive type the GPU does not know.
class Disk : public Primitive {
public:
    bool intersect(const Ray&, SurfaceInteraction&) const override { return false; }
    BoundingBox getBounds() const override { return BoundingBox(Vec3(-1.0f), Vec3(1.0f)); }
};

}  // namespace

int main() {
    std::mt19937 rng(2024);
    GpuBVHAccelerator accel(0);
    if (accel.status() != RBR_OK) {
        std::cerr << "no CUDA device: " << accel.error() << "\n";
        return 2;
    }
    {  // empty and single-primitive structures
        accel.build({});
        Ray ray(Vec3(0, 0, 5), Vec3(0, 0, -1));
        SurfaceInteraction isect;
        check(!accel.intersect(ray, isect), "empty hit");
        check(!accel.intersectP(ray), "empty hitP");
        check(accel.worldBounds().isEmpty(), "empty bounds");
        World one;
        one.add(std::make_unique<Sphere>(Vec3(0, 0, 0), 1.0f));
        accel.build(one.prims);
        Ray r2(Vec3(0, 0, 5), Vec3(0, 0, -1));
        check(accel.intersect(r2, isect) && std::fabs(isect.t - 4.0f) < 1e-3f && r2.tMax == isect.t, "single sphere");
        const BoundingBox b = accel.worldBounds();
        check(b.pMin.x == -1.0f && b.pMax.z == 1.0f, "single sphere bounds");
    }
    World small = randomWorld(rng, 30, 30, 10, false);
    compare(accel, small, rng, 3000, "small");
    World big = randomWorld(rng, 400, 1500, 100, false);
    compare(accel, big, rng, 6000, "large");
    World withPlane = randomWorld(rng, 60, 200, 20, true);
    compare(accel, withPlane, rng, 3000, "with infinite plane");
    {  // a rebuild replaces the previous contents
        accel.build(big.prims);
        accel.build(small.prims);
        Ray probe(Vec3(0, 0, 50), Vec3(0, 0, -1));
        SurfaceInteraction a, b;
        const bool refHit = bruteForce(small.prims, probe, b);
        const bool hit = accel.intersect(probe, a);
        check(hit == refHit && (!hit || a.primitive == b.primitive), "rebuild");
    }
    {  // micro-batched per-ray queries from concurrent threads: the answers of single queries
        World w = randomWorld(rng, 200, 800, 50, true);
        accel.build(w.prims);
        std::uniform_real_distribution<float> pos(-14.0f, 14.0f), dir(-1.0f, 1.0f);
        std::vector<Ray> rays;
        while (rays.size() < 4000) {
            const Vec3 d(dir(rng), dir(rng), dir(rng));
            if (d.length() > 1e-3f) rays.push_back(Ray(Vec3(pos(rng), pos(rng), pos(rng)), d));
        }
        std::vector<int> refHit(rays.size()), refP(rays.size());
        std::vector<const Primitive*> refPrim(rays.size(), nullptr);
        std::vector<float> refT(rays.size(), 0.0f);
        for (size_t i = 0; i < rays.size(); ++i) {
            SurfaceInteraction is;
            refHit[i] = bruteForce(w.prims, rays[i], is);
            if (refHit[i]) refPrim[i] = is.primitive, refT[i] = is.t;
            for (const Primitive* q : w.prims)
                if (q->intersectP(rays[i])) {
                    refP[i] = 1;
                    break;
                }
        }
        accel.setMicroBatching(8, 200);
        const int kThreads = 8;
        std::vector<int> bad(kThreads, 0);
        std::vector<std::thread> pool;
        for (int t = 0; t < kThreads; ++t)
            pool.emplace_back([&, t] {
                for (size_t i = t; i < rays.size(); i += kThreads) {
                    Ray r = rays[i];
                    SurfaceInteraction is;
                    const bool hit = accel.intersect(r, is);
                    if (hit != static_cast<bool>(refHit[i]) || (hit && (is.primitive != refPrim[i] || !bits_equal(is.t, refT[i]))))
                        ++bad[t];
                    if (accel.intersectP(rays[i]) != static_cast<bool>(refP[i])) ++bad[t];
                }
            });
        for (auto& th : pool) th.join();
        int total = 0;
        for (int b : bad) total += b;
        const double per_launch = static_cast<double>(accel.perRayRays()) / std::max<uint64_t>(1, accel.perRayLaunches());
        std::cout << "micro-batched queries: " << accel.perRayRays() << " rays in " << accel.perRayLaunches()
                  << " launches (" << per_launch << " per launch), " << total << " mismatches\n";
        check(total == 0, "micro-batched per-ray queries equal brute force");
        check(accel.perRayRays() == 2 * rays.size(), "every micro-batched query was traced once");
        check(per_launch > 1.0, "micro-batching gathers queries of several threads");
        accel.setMicroBatching(1, 0);
    }
    {  // unsupported primitive: reported, no CPU fallback
        World odd;
        odd.add(std::make_unique<Disk>());
        accel.build(odd.prims);
        check(accel.status() == RBR_ERR_UNSUPPORTED && !accel.error().empty(), "unknown primitive type is reported");
        Ray ray(Vec3(0, 0, 5), Vec3(0, 0, -1));
        SurfaceInteraction isect;
        check(!accel.intersect(ray, isect), "no answer after an unsupported build");
    }
    if (failures == 0) std::cout << "All GPU accelerator tests passed\n";
    return failures == 0 ? 0 : 1;
}
