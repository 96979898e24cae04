// Wavefront path tracer (placeholder until the kernels land).
#include "rbr_context.h"

namespace rbr {

rbr_status render(rbr_ctx* ctx, const rbr_camera*, const rbr_render_params*, float*, float*, cudaStream_t) {
    return fail(ctx, RBR_ERR_UNSUPPORTED, "rbr_render is not built yet");
}

void free_path_buffers(rbr_ctx* ctx) {
    PathBuffers& p = ctx->pt;
    release(p.ray);
    release(p.thr);
    release(p.rad);
    release(p.hit);
    release(p.queue[0]);
    release(p.queue[1]);
    release(p.classq);
    release(p.shadow);
    release(p.counters);
    p.capacity = 0;
}

}  // namespace rbr
