// GpuBVHAccelerator: a render::Accelerator (include/render/acceleration/accelerator.h:19-34)
// whose queries run on the GPU through librbr_b200 (include/rbr_b200.h).
//
// Semantics of the reference interface are kept: primitives are not owned and must outlive
// the accelerator; build() replaces the previous contents; intersect() returns the closest hit
// with ray.tMax set to its distance and `isect` filled by the hit primitive's own intersect()
// (the GPU distance is bit-identical to what that primitive computes, so the primitive accepts
// it); intersectP() answers the shadow query. Queries are thread-safe (serialised internally).
// Batched queries (intersectBatch / intersectPBatch) are the fast path: one launch per batch.
//
// Micro-batching (setMicroBatching(max_rays, max_wait_us), off by default): per-ray queries
// from concurrent threads (the reference integrators render rows on OpenMP threads, one query
// at a time each) are gathered into one launch. A query joins the pending batch of its kind
// (closest or any hit) and waits; the batch is traced when it holds max_rays rays, or by the
// first waiter whose max_wait_us ran out. Results are the same as one query per launch.
//
// Unsupported input (a primitive that is not a Triangle, Sphere, Quad or Plane) is reported
// through status()/error(); the accelerator then answers every query with "no hit" — there is
// no CPU traversal fallback.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "rbr_b200.h"
#include "render/acceleration/accelerator.h"

namespace render {

class GpuBVHAccelerator : public Accelerator {
public:
    explicit GpuBVHAccelerator(int device = 0);
    ~GpuBVHAccelerator() override;
    GpuBVHAccelerator(const GpuBVHAccelerator&) = delete;
    GpuBVHAccelerator& operator=(const GpuBVHAccelerator&) = delete;

    void build(std::vector<Primitive*> primitives) override;
    bool intersect(const Ray& ray, SurfaceInteraction& isect) const override;
    bool intersectP(const Ray& ray) const override;
    BoundingBox worldBounds() const override;

    // Batched queries: hits[i] = index into the built primitive list (RBR_MISS if none) and t.
    bool intersectBatch(const Ray* rays, size_t n, rbr_hit* hits) const;
    bool intersectPBatch(const Ray* rays, size_t n, uint8_t* occluded) const;

    // Per-ray queries gathered into launches of up to max_rays rays (1: one launch per query);
    // a waiting query traces the pending batch after max_wait_us microseconds. Call it while
    // no queries run.
    void setMicroBatching(size_t max_rays, int max_wait_us);
    // Launches made for per-ray queries and the rays they carried (for measurements).
    uint64_t perRayLaunches() const;
    uint64_t perRayRays() const;

    rbr_status status() const { return status_; }
    const std::string& error() const { return error_; }
    const std::vector<Primitive*>& primitives() const { return prims_; }

private:
    rbr_ctx* ctx_ = nullptr;
    std::vector<Primitive*> prims_;
    BoundingBox bounds_;
    rbr_status status_ = RBR_OK;
    std::string error_;
    mutable std::mutex mu_;

    // micro-batching of per-ray queries
    struct Waiter {
        rbr_ray ray;
        rbr_hit hit;
        uint8_t occluded;
        bool done;
    };
    struct PendingBatch {
        std::vector<Waiter*> waiters;
        uint64_t generation = 0;
    };
    bool query(const Ray& ray, bool any_hit, rbr_hit* hit, uint8_t* occluded) const;
    void flushLocked(int kind, std::unique_lock<std::mutex>& lock) const;
    size_t batch_max_ = 1;
    int batch_wait_us_ = 0;
    mutable std::mutex bmu_;
    mutable std::condition_variable bcv_;
    mutable PendingBatch pending_[2];  // [0] closest hit, [1] any hit
    mutable uint64_t launches_ = 0, rays_ = 0;
};

}  // namespace render
