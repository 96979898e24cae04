#include "gpu_accelerator.h"

#include <cfloat>
#include <chrono>

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

void GpuBVHAccelerator::setMicroBatching(size_t max_rays, int max_wait_us) {
    std::lock_guard<std::mutex> lock(bmu_);
    batch_max_ = max_rays < 1 ? 1 : max_rays;
    batch_wait_us_ = max_wait_us < 0 ? 0 : max_wait_us;
}

uint64_t GpuBVHAccelerator::perRayLaunches() const {
    std::lock_guard<std::mutex> lock(bmu_);
    return launches_;
}

uint64_t GpuBVHAccelerator::perRayRays() const {
    std::lock_guard<std::mutex> lock(bmu_);
    return rays_;
}

// Traces the pending batch of `kind` (0 closest, 1 any hit). Called with `lock` held on bmu_;
// releases it for the trace, so that other threads can start the next batch meanwhile, and
// returns with it held and the batch's waiters marked done.
void GpuBVHAccelerator::flushLocked(int kind, std::unique_lock<std::mutex>& lock) const {
    std::vector<Waiter*> batch;
    batch.swap(pending_[kind].waiters);
    ++pending_[kind].generation;
    ++launches_;
    rays_ += batch.size();
    lock.unlock();
    std::vector<rbr_ray> rr(batch.size());
    for (size_t i = 0; i < batch.size(); ++i) rr[i] = batch[i]->ray;
    bool ok = false;
    {
        std::lock_guard<std::mutex> g(mu_);
        if (status_ == RBR_OK && !prims_.empty()) {
            if (kind == 0) {
                std::vector<rbr_hit> hits(batch.size());
                ok = rbr_trace_host(ctx_, rr.data(), static_cast<uint32_t>(rr.size()), 0, hits.data()) == RBR_OK;
                for (size_t i = 0; i < batch.size(); ++i) batch[i]->hit = ok ? hits[i] : rbr_hit{RBR_MISS, 0.0f};
            } else {
                std::vector<uint8_t> occ(batch.size());
                ok = rbr_trace_host(ctx_, rr.data(), static_cast<uint32_t>(rr.size()), 1, occ.data()) == RBR_OK;
                for (size_t i = 0; i < batch.size(); ++i) batch[i]->occluded = ok ? occ[i] : 0;
            }
        } else {
            for (Waiter* w : batch) {
                w->hit = rbr_hit{RBR_MISS, 0.0f};
                w->occluded = 0;
            }
        }
    }
    lock.lock();
    for (Waiter* w : batch) w->done = true;
    bcv_.notify_all();
}

// One per-ray query through the micro-batch of its kind.
bool GpuBVHAccelerator::query(const Ray& ray, bool any_hit, rbr_hit* hit, uint8_t* occluded) const {
    const int kind = any_hit ? 1 : 0;
    Waiter me{to_rbr(ray), rbr_hit{RBR_MISS, 0.0f}, 0, false};
    std::unique_lock<std::mutex> lock(bmu_);
    PendingBatch& b = pending_[kind];
    b.waiters.push_back(&me);
    const uint64_t gen = b.generation;
    if (b.waiters.size() >= batch_max_) {
        flushLocked(kind, lock);
    } else {
        const auto deadline = std::chrono::steady_clock::now() + std::chrono::microseconds(batch_wait_us_);
        while (!me.done) {
            if (bcv_.wait_until(lock, deadline) == std::cv_status::timeout && !me.done) {
                // still pending (not taken by a flush in progress): trace it now
                if (pending_[kind].generation == gen) flushLocked(kind, lock);
                else bcv_.wait(lock, [&] { return me.done; });
            }
        }
    }
    if (hit) *hit = me.hit;
    if (occluded) *occluded = me.occluded;
    return true;
}

bool GpuBVHAccelerator::intersect(const Ray& ray, SurfaceInteraction& isect) const {
    rbr_hit h{RBR_MISS, 0.0f};
    if (batch_max_ > 1) query(ray, false, &h, nullptr);
    else if (!intersectBatch(&ray, 1, &h)) return false;
    if (h.prim == RBR_MISS) return false;
    // Let the primitive fill the interaction: with tMax = t it computes the same t and accepts.
    ray.tMax = h.t;
    return prims_[h.prim]->intersect(ray, isect);
}

bool GpuBVHAccelerator::intersectP(const Ray& ray) const {
    uint8_t occ = 0;
    if (batch_max_ > 1) {
        query(ray, true, nullptr, &occ);
        return occ != 0;
    }
    return intersectPBatch(&ray, 1, &occ) && occ != 0;
}

BoundingBox GpuBVHAccelerator::worldBounds() const {
    std::lock_guard<std::mutex> lock(mu_);
    return bounds_;
}

}  // namespace render
