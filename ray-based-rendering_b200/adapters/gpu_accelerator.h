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
// Unsupported input (a primitive that is not a Triangle, Sphere, Quad or Plane) is reported
// through status()/error(); the accelerator then answers every query with "no hit" — there is
// no CPU traversal fallback.
#pragma once

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
};

}  // namespace render
