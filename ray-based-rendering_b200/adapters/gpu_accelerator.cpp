#include "gpu_accelerator.h"

#include <cfloat>

#include "scene_flatten.h"

namespace render {

namespace {
rbr_ray to_rbr(const Ray& r) {
    rbr_ray o{};
    o.origin[0] = r.origin.x;
    o.origin[1] = r.origin.y;
    o.origin[2] = r.origin.z;
    o.direction[0] = r.direction.x;
    o.direction[1] = r.direction.y;
    o.direction[2] = r.direction.z;
    o.tmax = r.tMax;
    return o;
}
}  // namespace

GpuBVHAccelerator::GpuBVHAccelerator(int device) {
    status_ = rbr_ctx_create(device, &ctx_);
    if (status_ != RBR_OK) error_ = "rbr_ctx_create failed (no usable CUDA device)";
}

GpuBVHAccelerator::~GpuBVHAccelerator() { rbr_ctx_destroy(ctx_); }

void GpuBVHAccelerator::build(std::vector<Primitive*> primitives) {
    std::lock_guard<std::mutex> lock(mu_);
    prims_ = std::move(primitives);
    bounds_ = BoundingBox();
    if (!ctx_) return;
    FlatScene flat;
    std::vector<const Primitive*> cp(prims_.begin(), prims_.end());
    std::string err;
    if (!flatten_primitives(cp, /*material_check=*/false, flat, err)) {
        status_ = RBR_ERR_UNSUPPORTED;
        error_ = err;
        prims_.clear();
        return;
    }
    const float bg[3] = {0.0f, 0.0f, 0.0f};
    flat.finalize(bg);
    status_ = rbr_scene_upload(ctx_, &flat.desc);
    if (status_ != RBR_OK) {
        error_ = rbr_last_error(ctx_);
        prims_.clear();
        return;
    }
    error_.clear();
    float lo[3], hi[3];
    rbr_world_bounds(ctx_, lo, hi);
    bounds_.pMin = Vec3(lo[0], lo[1], lo[2]);
    bounds_.pMax = Vec3(hi[0], hi[1], hi[2]);
}

bool GpuBVHAccelerator::intersectBatch(const Ray* rays, size_t n, rbr_hit* hits) const {
    std::lock_guard<std::mutex> lock(mu_);
    if (status_ != RBR_OK || prims_.empty()) {
        for (size_t i = 0; i < n; ++i) hits[i] = rbr_hit{RBR_MISS, 0.0f};
        return status_ == RBR_OK;
    }
    std::vector<rbr_ray> rr(n);
    for (size_t i = 0; i < n; ++i) rr[i] = to_rbr(rays[i]);
    return rbr_trace_host(ctx_, rr.data(), static_cast<uint32_t>(n), 0, hits) == RBR_OK;
}

bool GpuBVHAccelerator::intersectPBatch(const Ray* rays, size_t n, uint8_t* occluded) const {
    std::lock_guard<std::mutex> lock(mu_);
    if (status_ != RBR_OK || prims_.empty()) {
        for (size_t i = 0; i < n; ++i) occluded[i] = 0;
        return status_ == RBR_OK;
    }
    std::vector<rbr_ray> rr(n);
    for (size_t i = 0; i < n; ++i) rr[i] = to_rbr(rays[i]);
    return rbr_trace_host(ctx_, rr.data(), static_cast<uint32_t>(n), 1, occluded) == RBR_OK;
}

bool GpuBVHAccelerator::intersect(const Ray& ray, SurfaceInteraction& isect) const {
    rbr_hit h{RBR_MISS, 0.0f};
    if (!intersectBatch(&ray, 1, &h) || h.prim == RBR_MISS) return false;
    // Let the primitive fill the interaction: with tMax = t it computes the same t and accepts.
    ray.tMax = h.t;
    return prims_[h.prim]->intersect(ray, isect);
}

bool GpuBVHAccelerator::intersectP(const Ray& ray) const {
    uint8_t occ = 0;
    return intersectPBatch(&ray, 1, &occ) && occ != 0;
}

BoundingBox GpuBVHAccelerator::worldBounds() const {
    std::lock_guard<std::mutex> lock(mu_);
    return bounds_;
}

}  // namespace render
