// Film export on the device: Film::toRGB8 and Film::toRGB8ToneMapped (src/core/film.cpp:34-62)
// over a film of per-pixel means (what Film::getPixel returns after one averaged sample).
#include "rbr_bsdf.cuh"
#include <algorithm>
#include "rbr_context.h"

namespace rbr {
namespace {

// encode(): gamma, clamp to [0, 1] as std::max(0, std::min(1, v)), * 255 + 0.5, truncated.
__device__ __forceinline__ uint8_t encode8(float v, float inv_gamma) {
    const float p = static_cast<float>(pow(static_cast<double>(v), static_cast<double>(inv_gamma)));
    // std::max(0, std::min(1, p)) sends NaN (a negative value's power) to 1; a saturating
    // clamp would send it to 0, so NaN is handled before clamping.
    const float c = (p != p) ? 1.0f : fminf(fmaxf(p, 0.0f), 1.0f);
    return static_cast<uint8_t>(__float2uint_rz(fa(fm(c, 255.0f), 0.5f)));
}

__global__ void k_film_rgb8(const float* film, uint32_t npix, float exposure, float inv_gamma, int tonemap,
                            uint8_t* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        f3 c = mk(film[3 * i], film[3 * i + 1], film[3 * i + 2]);
        if (tonemap) {  // Reinhard: c = c * exposure; c = c / (c + 1)
            c = xmuls(c, exposure);
            c = mk(fd(c.x, fa(c.x, 1.0f)), fd(c.y, fa(c.y, 1.0f)), fd(c.z, fa(c.z, 1.0f)));
        }
        out[3 * i] = encode8(c.x, inv_gamma);
        out[3 * i + 1] = encode8(c.y, inv_gamma);
        out[3 * i + 2] = encode8(c.z, inv_gamma);
    }
}

}  // namespace
}  // namespace rbr

using namespace rbr;

extern "C" {

rbr_status rbr_film_to_rgb8(rbr_ctx* ctx, const float* film, int32_t width, int32_t height, float exposure, float gamma,
                            int tonemap, uint8_t* out, void* stream) {
    if (!ctx || !film || !out || width <= 0 || height <= 0 || !(gamma > 0.0f)) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    const uint32_t npix = static_cast<uint32_t>(width) * static_cast<uint32_t>(height);
    const float inv_gamma = 1.0f / gamma;
    const int grid = std::min<int>((npix + 255) / 256, ctx->num_sms * 16);
    k_film_rgb8<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(film, npix, exposure, inv_gamma, tonemap, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "film export");
    return RBR_OK;
}

rbr_status rbr_film_to_rgb8_host(rbr_ctx* ctx, const float* film, int32_t width, int32_t height, float exposure,
                                 float gamma, int tonemap, uint8_t* out) {
    if (!ctx || !film || !out || width <= 0 || height <= 0) return RBR_ERR_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    const size_t npix = size_t(width) * size_t(height);
    rbr_status st = ensure(ctx, ctx->stage_in, npix * 12, "film staging");
    if (st == RBR_OK) st = ensure(ctx, ctx->stage_out, npix * 3, "film staging");
    if (st != RBR_OK) return st;
    cudaError_t e = cudaMemcpyAsync(ctx->stage_in.ptr, film, npix * 12, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "film export");
    st = rbr_film_to_rgb8(ctx, static_cast<const float*>(ctx->stage_in.ptr), width, height, exposure, gamma, tonemap,
                          static_cast<uint8_t*>(ctx->stage_out.ptr), ctx->stream);
    if (st != RBR_OK) return st;
    e = cudaMemcpyAsync(out, ctx->stage_out.ptr, npix * 3, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "film export");
    return RBR_OK;
}

}  // extern "C"
