// Device materials, BSDF lobes, lights, camera rays and the counter-based RNG.
//
// Restates the reference operation for operation with exactly rounded intrinsics, so BSDF
// values and densities equal the reference's bit for bit; only the sampling routines need sin
// and cos, taken correctly rounded here (glibc's sinf/cosf, which the reference calls, are
// within an ulp but not always correctly rounded, so a sampled direction may differ in its
// last bits).
//   Material::createBSDF      src/materials/material.cpp:69-108
//   MixtureBSDF               src/materials/mixture_bsdf.cpp:5-82
//   LambertianBSDF            src/materials/lambertian_bsdf.cpp:5-28
//   Specular{Reflection,Transmission}BSDF  src/materials/specular_bsdf.cpp:5-57
//   GGXDistribution, Microfacet{Reflection,Transmission}BSDF  src/materials/microfacet_bsdf.cpp:9-179
//   fresnelDielectric / fresnelSchlick     include/render/materials/fresnel.h:16-48
//   AreaLight::sample / PointLight::sample src/lighting/area_light.cpp:13-39, point_light.cpp:5-19
//   Camera rays               src/camera/camera.cpp:5-9, thin_lens_camera.cpp:6-23
//   sampling::*               include/render/core/sampler.h:58-149
#pragma once

#include "rbr_b200.h"
#include "rbr_device.cuh"
#include "rbr_trig.h"

namespace rbr {

// ----------------------------------------------------------------------------------------
// scalar helpers: exactly rounded arithmetic and std::min/max/clamp semantics
// ----------------------------------------------------------------------------------------
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fq(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ float omax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float omin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float oclamp(float v, float lo, float hi) { return omax(lo, omin(hi, v)); }
__device__ __forceinline__ bool black(f3 a) { return a.x <= 0.0f && a.y <= 0.0f && a.z <= 0.0f; }
__device__ __forceinline__ float maxc(f3 a) {  // std::max({x, y, z})
    float m = a.x;
    if (m < a.y) m = a.y;
    if (m < a.z) m = a.z;
    return m;
}

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 2.0f * kPi;
constexpr float kInvPi = 1.0f / kPi;

// ----------------------------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11). Counter = (pixel, sample, depth,
// purpose), key = seed. The same streams as the CPU restatement in oracle/rbr_oracle.c.
// ----------------------------------------------------------------------------------------
enum : uint32_t { kRngCamera = 0, kRngBounce = 1, kRngLights = 2, kRngMedium = 3 };

__device__ __forceinline__ uint4 philox(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}
__device__ __forceinline__ float u01(uint32_t x) { return static_cast<float>(x >> 8) * (1.0f / 16777216.0f); }
__device__ __forceinline__ float4 draw4(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t depth,
                                        uint32_t purpose) {
    const uint4 o = philox(make_uint4(pixel, sample, depth, purpose),
                           make_uint2(static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32)));
    return make_float4(u01(o.x), u01(o.y), u01(o.z), u01(o.w));
}

// ----------------------------------------------------------------------------------------
// Frame (coordinateSystem, vector.h:282-289; sampling::Frame, sampler.h:104-118)
// ----------------------------------------------------------------------------------------
struct Frame {
    f3 t, b, n;
};
__device__ __forceinline__ Frame make_frame(f3 n) {
    Frame f;
    f.n = n;
    if (fabsf(n.x) > fabsf(n.y)) f.t = xnorm(mk(-n.z, 0.0f, n.x));
    else f.t = xnorm(mk(0.0f, n.z, -n.y));
    f.b = xcross(n, f.t);
    return f;
}
__device__ __forceinline__ f3 to_world(const Frame& f, f3 l) {
    return xadd(xadd(xmuls(f.t, l.x), xmuls(f.b, l.y)), xmuls(f.n, l.z));
}
__device__ __forceinline__ f3 to_local(const Frame& f, f3 w) { return mk(xdot(w, f.t), xdot(w, f.b), xdot(w, f.n)); }

// ----------------------------------------------------------------------------------------
// Fresnel
// ----------------------------------------------------------------------------------------
__device__ __forceinline__ float fresnel_dielectric(float c, float etaI, float etaT) {
    c = oclamp(c, -1.0f, 1.0f);
    if (c < 0.0f) {
        const float tmp = etaI;
        etaI = etaT;
        etaT = tmp;
        c = -c;
    }
    const float sinI = fq(omax(0.0f, fs(1.0f, fm(c, c))));
    const float sinT = fm(fd(etaI, etaT), sinI);
    if (sinT >= 1.0f) return 1.0f;
    const float cosT = fq(omax(0.0f, fs(1.0f, fm(sinT, sinT))));
    const float rParl = fd(fs(fm(etaT, c), fm(etaI, cosT)), fa(fm(etaT, c), fm(etaI, cosT)));
    const float rPerp = fd(fs(fm(etaI, c), fm(etaT, cosT)), fa(fm(etaI, c), fm(etaT, cosT)));
    return fm(0.5f, fa(fm(rParl, rParl), fm(rPerp, rPerp)));
}
__device__ __forceinline__ f3 fresnel_schlick(float c, f3 f0) {
    const float m = fs(1.0f, oclamp(fabsf(c), 0.0f, 1.0f));
    const float m2 = fm(m, m);
    return xadd(f0, xmuls(xsub(mk(1.0f, 1.0f, 1.0f), f0), fm(fm(m2, m2), m)));
}

// ----------------------------------------------------------------------------------------
// Lobes. A mixture is built from the six material parameters exactly as createBSDF does;
// each lobe stores its kind and weight, everything else derives from the material.
// ----------------------------------------------------------------------------------------
enum : uint32_t {
    kLambert = 0,
    kCondSpec = 1,   // SpecularReflection, Schlick(baseColor)
    kCondGGX = 2,    // MicrofacetReflection, Schlick(baseColor)
    kDielSpec = 3,   // SpecularReflection, Dielectric(1, ior)
    kDielGGX = 4,    // MicrofacetReflection, Dielectric(1, ior)
    kTransSpec = 5,  // SpecularTransmission(baseColor, 1, ior)
    kTransGGX = 6,   // MicrofacetTransmission(baseColor, 1, ior)
    kPassSpec = 7    // SpecularTransmission(baseColor, 1, 1)
};
// BSDFType bits (include/render/materials/bsdf.h:10-24)
enum : uint32_t { kTRefl = 1, kTTrans = 2, kTDiffuse = 4, kTGlossy = 8, kTSpecular = 16 };

struct Bsdf {
    f3 base;
    float ior;
    float alpha;       // GGXDistribution alpha: max(roughness^2, 1e-3)
    bool has_sub;      // substrate Fresnel set (dielectric interface)
    int n;
    // Lobe i (i < n): kind in bits 4i..4i+3 of `kinds`, substrate flag in bit i of `subs`,
    // weight wt[i]. Packed in scalars so that no lobe list is indexed in local memory.
    uint32_t kinds, subs;
    float wt0, wt1, wt2, wt3;
};

// element i (0..3) of four scalars, without an indexed array
__device__ __forceinline__ float pick4(float a0, float a1, float a2, float a3, int i) {
    return i == 0 ? a0 : i == 1 ? a1 : i == 2 ? a2 : a3;
}
__device__ __forceinline__ uint32_t kind_of(const Bsdf& b, int i) { return (b.kinds >> (4 * i)) & 0xFu; }
__device__ __forceinline__ float weight_of(const Bsdf& b, int i) { return pick4(b.wt0, b.wt1, b.wt2, b.wt3, i); }

__device__ __forceinline__ bool lobe_delta(uint32_t k) { return k == kCondSpec || k == kDielSpec || k == kTransSpec || k == kPassSpec; }

__device__ __forceinline__ uint32_t lobe_type(uint32_t k) {
    switch (k) {
        case kLambert: return kTDiffuse | kTRefl;
        case kCondSpec:
        case kDielSpec: return kTSpecular | kTRefl;
        case kCondGGX:
        case kDielGGX: return kTGlossy | kTRefl;
        case kTransGGX: return kTGlossy | kTTrans;
        default: return kTSpecular | kTTrans;
    }
}

__device__ __forceinline__ void add_lobe(Bsdf& b, uint32_t kind, float w, bool substrate) {
    if (w <= 0.0f || b.n >= 4) return;
    b.kinds |= kind << (4 * b.n);
    b.subs |= (substrate ? 1u : 0u) << b.n;
    b.wt0 = b.n == 0 ? w : b.wt0;
    b.wt1 = b.n == 1 ? w : b.wt1;
    b.wt2 = b.n == 2 ? w : b.wt2;
    b.wt3 = b.n == 3 ? w : b.wt3;
    ++b.n;
}

// Material::createBSDF (material.cpp:69-108)
__device__ __forceinline__ Bsdf make_bsdf(const MaterialDev& m) {
    Bsdf b;
    b.base = mk(m.base[0], m.base[1], m.base[2]);
    b.ior = m.ior;
    b.alpha = omax(fm(m.roughness, m.roughness), 1e-3f);
    b.has_sub = false;
    b.n = 0;
    b.kinds = b.subs = 0;
    b.wt0 = b.wt1 = b.wt2 = b.wt3 = 0.0f;
    const float met = oclamp(m.metallic, 0.0f, 1.0f);
    const float t = oclamp(m.transmission, 0.0f, 1.0f);
    const float diel = fs(1.0f, met);
    const bool smooth = m.roughness < 0.03f;
    const bool iface = fabsf(fs(m.ior, 1.0f)) > 1e-3f;
    const bool tinted = !black(b.base);
    if (met > 0.0f && tinted) add_lobe(b, smooth ? kCondSpec : kCondGGX, met, false);
    if (diel > 0.0f) {
        if (iface) {
            add_lobe(b, smooth ? kDielSpec : kDielGGX, diel, false);
            b.has_sub = true;
            if (t > 0.0f && tinted) add_lobe(b, smooth ? kTransSpec : kTransGGX, fm(diel, t), false);
            if (t < 1.0f && tinted) add_lobe(b, kLambert, fm(diel, fs(1.0f, t)), true);
        } else {
            if (t > 0.0f && tinted) add_lobe(b, kPassSpec, fm(diel, t), false);
            if (t < 1.0f && tinted) add_lobe(b, kLambert, fm(diel, fs(1.0f, t)), false);
        }
    }
    return b;
}

__device__ __forceinline__ bool bsdf_delta(const Bsdf& b) {
    if (b.n == 0) return false;
    for (int i = 0; i < b.n; ++i)
        if (!lobe_delta(kind_of(b, i))) return false;
    return true;
}

// Fresnel term of a reflection lobe (Schlick for conductors, dielectric for dielectrics)
__device__ __forceinline__ f3 lobe_fresnel(const Bsdf& b, uint32_t k, float c) {
    if (k == kCondSpec || k == kCondGGX) return fresnel_schlick(c, b.base);
    const float v = fresnel_dielectric(c, 1.0f, b.ior);
    return mk(v, v, v);
}
__device__ __forceinline__ float trans_eta_inside(const Bsdf& b, uint32_t k) { return k == kPassSpec ? 1.0f : b.ior; }

// rho (BSDF::rho overrides)
__device__ __forceinline__ f3 lobe_rho(const Bsdf& b, uint32_t k, f3 wo) {
    switch (k) {
        case kLambert: return b.base;
        case kCondSpec:
        case kCondGGX:
        case kDielSpec:
        case kDielGGX: return xmul(mk(1.0f, 1.0f, 1.0f), lobe_fresnel(b, k, wo.z));
        default: return xmuls(b.base, fs(1.0f, fresnel_dielectric(wo.z, 1.0f, trans_eta_inside(b, k))));
    }
}

// GGX distribution
__device__ __forceinline__ float ggx_D(float alpha, f3 wh) {
    const float cos2 = fm(wh.z, wh.z);
    if (cos2 <= 0.0f) return 0.0f;
    const float a2 = fm(alpha, alpha);
    const float d = fa(fm(cos2, fs(a2, 1.0f)), 1.0f);
    return fd(a2, fm(fm(kPi, d), d));
}
__device__ __forceinline__ float ggx_lambda(float alpha, f3 w) {
    const float cos2 = fm(w.z, w.z);
    if (cos2 <= 0.0f) return 0.0f;
    const float tan2 = fd(omax(0.0f, fs(1.0f, cos2)), cos2);
    return fm(0.5f, fs(fq(fa(1.0f, fm(fm(alpha, alpha), tan2))), 1.0f));
}
// GGXDistribution::pdf(wo, wh) = D(wh) G1(wo) |wo.wh| / |cos wo|, given D(wh), lambda(wo) and
// wo.wh; G(wo, wi) = 1 / (1 + lambda(wo) + lambda(wi)).
__device__ __forceinline__ float ggx_pdf(float D, float lambda_o, float dotOH, f3 wo) {
    const float cosO = fabsf(wo.z);
    if (cosO == 0.0f) return 0.0f;
    return fd(fm(fm(D, fd(1.0f, fa(1.0f, lambda_o))), fabsf(dotOH)), cosO);
}
__device__ __forceinline__ float ggx_G(float lambda_o, float lambda_i) {
    return fd(1.0f, fa(fa(1.0f, lambda_o), lambda_i));
}
__device__ __forceinline__ f3 ggx_sample_wh(float alpha, f3 wo, float u1, float u2) {
    const bool flip = wo.z < 0.0f;
    const f3 v = flip ? xneg(wo) : wo;
    const f3 vh = xnorm(mk(fm(alpha, v.x), fm(alpha, v.y), v.z));
    const f3 t1 = vh.z < 0.9999f ? xnorm(xcross(mk(0.0f, 0.0f, 1.0f), vh)) : mk(1.0f, 0.0f, 0.0f);
    const f3 t2 = xcross(vh, t1);
    const float r = fq(u1);
    const float phi = fm(kTwoPi, u2);
    float sp, cp;
    sincos_f(phi, sp, cp);
    const float p1 = fm(r, cp);
    float p2 = fm(r, sp);
    const float s = fm(0.5f, fa(1.0f, vh.z));
    p2 = fa(fm(fs(1.0f, s), fq(omax(0.0f, fs(1.0f, fm(p1, p1))))), fm(s, p2));
    const f3 nh = xadd(xadd(xmuls(t1, p1), xmuls(t2, p2)), xmuls(vh, fq(omax(0.0f, fs(fs(1.0f, fm(p1, p1)), fm(p2, p2))))));
    const f3 wh = xnorm(mk(fm(alpha, nh.x), fm(alpha, nh.y), omax(1e-6f, nh.z)));
    return flip ? xneg(wh) : wh;
}

struct BSample {
    f3 wi, f;
    float pdf;
    bool delta;
};
__device__ __forceinline__ BSample none() {
    BSample s;
    s.wi = mk(0.0f, 0.0f, 0.0f);
    s.f = mk(0.0f, 0.0f, 0.0f);
    s.pdf = 0.0f;
    s.delta = false;
    return s;
}
__device__ __forceinline__ bool same_hemi(f3 a, f3 b) { return fm(a.z, b.z) > 0.0f; }

// MicrofacetReflectionBSDF: evaluate() and pdf() for one (wo, wi) together. Both take the same
// half vector; D(wh) and lambda(wo) are computed once for both, with the operations and the
// zero checks of each of the two (microfacet_bsdf.cpp), so the results are the same as two
// separate calls.
__device__ __forceinline__ void ggxr_eval_pdf(const Bsdf& b, uint32_t k, f3 wo, f3 wi, f3& f, float& pdf) {
    f = mk(0.0f, 0.0f, 0.0f);
    pdf = 0.0f;
    if (!same_hemi(wo, wi)) return;
    f3 wh = xadd(wo, wi);
    if (wh.x == 0.0f && wh.y == 0.0f && wh.z == 0.0f) return;
    wh = xnorm(wh);
    if (wh.z < 0.0f) wh = xneg(wh);
    const float cosO = fabsf(wo.z), cosI = fabsf(wi.z);
    const float D = ggx_D(b.alpha, wh);
    const float lo = ggx_lambda(b.alpha, wo);
    const float dotOH = xdot(wo, wh);
    if (dotOH != 0.0f) pdf = fd(ggx_pdf(D, lo, dotOH, wo), fm(4.0f, fabsf(dotOH)));
    if (cosO == 0.0f || cosI == 0.0f) return;
    const f3 F = lobe_fresnel(b, k, dotOH);
    f = xmuls(xmul(mk(1.0f, 1.0f, 1.0f), F), fd(fm(D, ggx_G(lo, ggx_lambda(b.alpha, wi))), fm(fm(4.0f, cosO), cosI)));
}
__device__ __forceinline__ BSample ggxr_sample(const Bsdf& b, uint32_t k, f3 wo, float u1, float u2) {
    BSample r = none();
    if (wo.z == 0.0f) return r;
    const f3 wh = ggx_sample_wh(b.alpha, wo, u1, u2);
    const f3 wi = xsub(xmuls(wh, fm(2.0f, xdot(wo, wh))), wo);
    if (!same_hemi(wo, wi)) return r;
    f3 f;
    float p;
    ggxr_eval_pdf(b, k, wo, wi, f, p);
    if (p <= 0.0f) return r;
    r.wi = wi;
    r.pdf = p;
    r.f = f;
    return r;
}

// MicrofacetTransmissionBSDF (etaOutside = 1, etaInside = ior)
__device__ __forceinline__ bool ggxt_half(const Bsdf& b, f3 wo, f3 wi, f3& wh, float& eta) {
    if (same_hemi(wo, wi)) return false;
    if (wo.z == 0.0f || wi.z == 0.0f) return false;
    eta = wo.z > 0.0f ? fd(b.ior, 1.0f) : fd(1.0f, b.ior);
    f3 h = xadd(wo, xmuls(wi, eta));
    if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return false;
    h = xnorm(h);
    if (xdot(wo, h) < 0.0f) h = xneg(h);
    wh = h;
    return fm(h.z, wo.z) > 0.0f && xdot(wi, h) <= 0.0f;
}
// MicrofacetTransmissionBSDF: evaluate() and pdf() together, as for reflection.
__device__ __forceinline__ void ggxt_eval_pdf(const Bsdf& b, f3 wo, f3 wi, f3& f, float& pdf) {
    f = mk(0.0f, 0.0f, 0.0f);
    pdf = 0.0f;
    f3 wh;
    float eta;
    if (!ggxt_half(b, wo, wi, wh, eta)) return;
    const float cosO = wo.z, cosI = wi.z;
    const float dotOH = xdot(wo, wh), dotIH = xdot(wi, wh);
    const float denom = fa(dotOH, fm(eta, dotIH));
    if (denom == 0.0f) return;
    const float D = ggx_D(b.alpha, wh);
    const float lo = ggx_lambda(b.alpha, wo);
    const float dwh = fd(fabsf(fm(fm(eta, eta), dotIH)), fm(denom, denom));
    pdf = fm(ggx_pdf(D, lo, dotOH, wo), dwh);
    const float F = fresnel_dielectric(wo.z > 0.0f ? dotOH : -dotOH, 1.0f, b.ior);
    const float value = fd(fm(fm(D, ggx_G(lo, ggx_lambda(b.alpha, wi))), fabsf(fm(dotIH, dotOH))),
                           fabsf(fm(fm(fm(cosI, cosO), denom), denom)));
    f = xmuls(b.base, fm(fs(1.0f, F), value));
}
__device__ __forceinline__ BSample ggxt_sample(const Bsdf& b, f3 wo, float u1, float u2) {
    BSample r = none();
    if (wo.z == 0.0f) return r;
    const f3 wh = ggx_sample_wh(b.alpha, wo, u1, u2);
    const float dotOH = xdot(wo, wh);
    if (dotOH <= 0.0f) return r;
    const bool entering = wo.z > 0.0f;
    const float etaRatio = entering ? fd(1.0f, b.ior) : fd(b.ior, 1.0f);
    const float sin2T = fm(fm(etaRatio, etaRatio), omax(0.0f, fs(1.0f, fm(dotOH, dotOH))));
    if (sin2T >= 1.0f) return r;
    const float cosT = fq(fs(1.0f, sin2T));
    const f3 wi = xsub(xmuls(wh, fs(fm(etaRatio, dotOH), cosT)), xmuls(wo, etaRatio));
    if (same_hemi(wo, wi) || wi.z == 0.0f) return r;
    f3 f;
    float p;
    ggxt_eval_pdf(b, wo, wi, f, p);
    if (p <= 0.0f) return r;
    r.wi = wi;
    r.pdf = p;
    r.f = f;
    return r;
}

// Lambertian
__device__ __forceinline__ f3 cosine_hemisphere(float u1, float u2) {
    const float r = fq(u1);
    const float theta = fm(kTwoPi, u2);
    float st, ct;
    sincos_f(theta, st, ct);
    return mk(fm(r, ct), fm(r, st), fq(omax(0.0f, fs(1.0f, u1))));
}

// Specular lobes
__device__ __forceinline__ BSample sr_sample(const Bsdf& b, uint32_t k, f3 wo) {
    BSample r = none();
    const float cosO = fabsf(wo.z);
    if (cosO == 0.0f) return r;
    r.wi = mk(-wo.x, -wo.y, wo.z);
    r.f = xdivs(xmul(mk(1.0f, 1.0f, 1.0f), lobe_fresnel(b, k, wo.z)), cosO);
    r.pdf = 1.0f;
    r.delta = true;
    return r;
}
__device__ __forceinline__ BSample st_sample(const Bsdf& b, uint32_t k, f3 wo) {
    BSample r = none();
    if (wo.z == 0.0f) return r;
    const float etaIn = trans_eta_inside(b, k);
    const bool entering = wo.z > 0.0f;
    const float etaI = entering ? 1.0f : etaIn;
    const float etaT = entering ? etaIn : 1.0f;
    const float eta = fd(etaI, etaT);
    const float cosI = fabsf(wo.z);
    const float sin2T = fm(fm(eta, eta), omax(0.0f, fs(1.0f, fm(cosI, cosI))));
    if (sin2T >= 1.0f) return r;
    const float cosT = fq(fs(1.0f, sin2T));
    r.wi = mk(fm(-eta, wo.x), fm(-eta, wo.y), entering ? -cosT : cosT);
    const float fr = fresnel_dielectric(wo.z, 1.0f, etaIn);
    r.f = xmuls(b.base, fd(fm(fm(fs(1.0f, fr), eta), eta), cosT));
    r.pdf = 1.0f;
    r.delta = true;
    return r;
}

// Lobe kinds a BSDF may hold, as a bit set over the kinds above. Code templated on a set
// compiles only the lobes in it: the path tracer shades each material class (material_class:
// any GGX lobe -> glossy; else a Lambertian lobe -> diffuse; else delta lobes only) with the
// set of that class, so the diffuse and delta-only kernels carry no microfacet code.
constexpr uint32_t kAllKinds = 0xFFu;
constexpr uint32_t kDeltaKinds = (1u << kCondSpec) | (1u << kDielSpec) | (1u << kTransSpec) | (1u << kPassSpec);
constexpr uint32_t kNoGGXKinds = kDeltaKinds | (1u << kLambert);
__host__ __device__ constexpr bool has_kind(uint32_t set, uint32_t k) { return ((set >> k) & 1u) != 0; }

// evaluate() and pdf() of a non-delta lobe (delta lobes give 0 and 0)
template <uint32_t kKinds = kAllKinds>
__device__ __forceinline__ void lobe_eval_pdf(const Bsdf& b, uint32_t k, f3 wo, f3 wi, f3& f, float& pdf) {
    // a switch over the kind with each case compiled in only if the set holds it
    switch (k) {
        case kLambert:
            if (has_kind(kKinds, kLambert)) {
                const bool same = same_hemi(wo, wi);
                f = same ? xmuls(b.base, kInvPi) : mk(0.0f, 0.0f, 0.0f);
                pdf = same ? fm(fabsf(wi.z), kInvPi) : 0.0f;
                return;
            }
            break;
        case kCondGGX:
        case kDielGGX:
            if (has_kind(kKinds, kCondGGX) || has_kind(kKinds, kDielGGX)) {
                ggxr_eval_pdf(b, k, wo, wi, f, pdf);
                return;
            }
            break;
        case kTransGGX:
            if (has_kind(kKinds, kTransGGX)) {
                ggxt_eval_pdf(b, wo, wi, f, pdf);
                return;
            }
            break;
        default: break;
    }
    f = mk(0.0f, 0.0f, 0.0f);
    pdf = 0.0f;
}
template <uint32_t kKinds = kAllKinds>
__device__ __forceinline__ BSample lobe_sample(const Bsdf& b, uint32_t k, f3 wo, float u1, float u2) {
    switch (k) {
        case kLambert:
            if (has_kind(kKinds, kLambert)) {
                BSample r = none();
                r.wi = cosine_hemisphere(u1, u2);
                if (wo.z < 0.0f) r.wi.z = -r.wi.z;
                r.f = xmuls(b.base, kInvPi);
                r.pdf = fm(fabsf(r.wi.z), kInvPi);
                return r;
            }
            break;
        case kCondSpec:
        case kDielSpec:
            if (has_kind(kKinds, kCondSpec) || has_kind(kKinds, kDielSpec)) return sr_sample(b, k, wo);
            break;
        case kTransSpec:
        case kPassSpec:
            if (has_kind(kKinds, kTransSpec) || has_kind(kKinds, kPassSpec)) return st_sample(b, k, wo);
            break;
        case kCondGGX:
        case kDielGGX:
            if (has_kind(kKinds, kCondGGX) || has_kind(kKinds, kDielGGX)) return ggxr_sample(b, k, wo, u1, u2);
            break;
        default:
            if (has_kind(kKinds, kTransGGX)) return ggxt_sample(b, wo, u1, u2);
            break;
    }
    return none();
}

// MixtureBSDF
__device__ __forceinline__ float eff_weight(const Bsdf& b, int i, f3 wo) {
    if (!((b.subs >> i) & 1u)) return weight_of(b, i);
    return fm(weight_of(b, i), omax(0.0f, fs(1.0f, fresnel_dielectric(wo.z, 1.0f, b.ior))));
}
// MixtureBSDF::selection: per-lobe effective weights and sampling scores. They depend on wo
// only, so a vertex computes them once (mixture) and every evaluation, pdf and sample of that
// vertex reuses them; the values are the ones each reference call recomputes.
struct Mix {
    float w0, w1, w2, w3;      // effective weights
    float sc0, sc1, sc2, sc3;  // sampling scores
    float total;
};
__device__ __forceinline__ float mix_w(const Mix& m, int i) { return pick4(m.w0, m.w1, m.w2, m.w3, i); }
__device__ __forceinline__ float mix_sc(const Mix& m, int i) { return pick4(m.sc0, m.sc1, m.sc2, m.sc3, i); }
__device__ __forceinline__ Mix mixture(const Bsdf& b, f3 wo) {
    Mix m;
    m.w0 = m.w1 = m.w2 = m.w3 = 0.0f;
    m.sc0 = m.sc1 = m.sc2 = m.sc3 = 0.0f;
    m.total = 0.0f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i >= b.n) break;
        const float w = eff_weight(b, i, wo);
        const float sc = fm(w, maxc(lobe_rho(b, kind_of(b, i), wo)));
        if (i == 0) m.w0 = w, m.sc0 = sc;
        if (i == 1) m.w1 = w, m.sc1 = sc;
        if (i == 2) m.w2 = w, m.sc2 = sc;
        if (i == 3) m.w3 = w, m.sc3 = sc;
        m.total = fa(m.total, sc);
    }
    return m;
}
// MixtureBSDF::evaluate and MixtureBSDF::pdf for one (wo, wi), in one pass over the lobes:
// f = sum of w_i f_i, pdf = (sum of score_i pdf_i) / total over the non-delta lobes.
template <uint32_t kKinds = kAllKinds>
__device__ __forceinline__ void bsdf_eval_pdf(const Bsdf& b, const Mix& m, f3 wo, f3 wi, f3& f, float& pdf) {
    f = mk(0.0f, 0.0f, 0.0f);
    float p = 0.0f;
    for (int i = 0; i < b.n; ++i) {
        const uint32_t k = kind_of(b, i);
        if (lobe_delta(k)) continue;
        f3 fl;
        float pl;
        lobe_eval_pdf<kKinds>(b, k, wo, wi, fl, pl);
        f = xadd(f, xmuls(fl, mix_w(m, i)));
        p = fa(p, fm(mix_sc(m, i), pl));
    }
    pdf = m.total <= 0.0f ? 0.0f : fd(p, m.total);
}
template <uint32_t kKinds = kAllKinds>
__device__ __forceinline__ BSample bsdf_sample(const Bsdf& b, const Mix& m, f3 wo, float u1, float u2) {
    if (m.total <= 0.0f) return none();
    float u = fm(u1, m.total);
    int chosen = b.n - 1;
    for (int i = 0; i < b.n; ++i) {
        const float sc = mix_sc(m, i);
        if (sc <= 0.0f) continue;
        if (u < sc || i + 1 == b.n) {
            chosen = i;
            break;
        }
        u = fs(u, sc);
    }
    const float sc = mix_sc(m, chosen);
    if (sc <= 0.0f) return none();
    const float v1 = omin(fd(u, sc), 0.99999994f);
    const uint32_t k = kind_of(b, chosen);
    BSample s = lobe_sample<kKinds>(b, k, wo, v1, u2);
    if (s.pdf <= 0.0f || black(s.f)) return none();
    const float pChosen = fd(sc, m.total);
    if (lobe_delta(k)) {
        s.f = xmuls(s.f, mix_w(m, chosen));
        s.pdf = fm(s.pdf, pChosen);
        return s;
    }
    bsdf_eval_pdf<kKinds>(b, m, wo, s.wi, s.f, s.pdf);
    if (s.pdf <= 0.0f) return none();
    return s;
}
__device__ __forceinline__ uint32_t bsdf_type(const Bsdf& b) {
    uint32_t t = 0;
    for (int i = 0; i < b.n; ++i) t |= lobe_type(kind_of(b, i));
    return t;
}

// sampling::powerHeuristic (sampler.h:137-149)
__device__ __forceinline__ float power_heuristic(float fPdf, float gPdf) {
    float f = fPdf, g = gPdf;  // nf = ng = 1
    if (isinf(f)) return 1.0f;
    if (isinf(g)) return 0.0f;
    const float m = omax(f, g);
    if (m <= 0.0f) return 0.0f;
    f = fd(f, m);
    g = fd(g, m);
    return fd(fm(f, f), fa(fm(f, f), fm(g, g)));
}

// ----------------------------------------------------------------------------------------
// Lights
// ----------------------------------------------------------------------------------------
struct LSample {
    f3 wi, Li;
    float pdf, dist;
    bool delta;
};
__device__ __forceinline__ LSample light_sample(const LightDev& l, f3 p, float u1, float u2) {
    LSample s;
    s.delta = false;
    if (l.type == RBR_LIGHT_AREA) {
        const f3 lp = xadd(xadd(ld3(l.position), xmuls(ld3(l.u), fs(u1, 0.5f))), xmuls(ld3(l.v), fs(u2, 0.5f)));
        const f3 toL = xsub(lp, p);
        const float d2 = xdot(toL, toL);
        s.dist = fq(d2);
        s.wi = xdivs(toL, s.dist);
        const float c = -xdot(ld3(l.normal), s.wi);
        if (c <= 0.0f) {
            s.Li = mk(0.0f, 0.0f, 0.0f);
            s.pdf = 0.0f;
            return s;
        }
        s.pdf = fd(d2, fm(c, l.area));
        s.Li = xmuls(ld3(l.color), l.intensity);
    } else {
        const f3 toL = xsub(ld3(l.position), p);
        const float d2 = xdot(toL, toL);
        s.dist = fq(d2);
        s.wi = xdivs(toL, s.dist);
        s.Li = xdivs(xmuls(ld3(l.color), l.intensity), d2);
        s.pdf = 1.0f;
        s.delta = true;
    }
    return s;
}

// ----------------------------------------------------------------------------------------
// Participating medium (src/materials/medium.cpp:9-44, src/materials/phase_function.cpp:17-47)
// ----------------------------------------------------------------------------------------
// HenyeyGreensteinPhase::evaluate: (1 - g^2) / (4 pi denom sqrt(denom)),
// denom = 1 + g^2 + 2 g cos(wo, wi), with wo the propagation direction (the reference's sign).
__device__ __forceinline__ float hg_eval(float g, f3 wo, f3 wi) {
    const float c = xdot(wo, wi);
    const float denom = fa(fa(1.0f, fm(g, g)), fm(fm(2.0f, g), c));
    return fd(fs(1.0f, fm(g, g)), fm(fm(fm(4.0f, kPi), denom), fq(denom)));
}

// HenyeyGreensteinPhase::sample: cos(theta) by inversion, phi = 2 pi u2, around wo.
__device__ __forceinline__ f3 hg_sample(float g, f3 wo, float u1, float u2) {
    float c;
    if (fabsf(g) < 1e-3f) {
        c = fs(1.0f, fm(2.0f, u1));
    } else {
        const float sq = fd(fs(1.0f, fm(g, g)), fs(fa(1.0f, g), fm(fm(2.0f, g), u1)));
        c = fd(-fs(fa(1.0f, fm(g, g)), fm(sq, sq)), fm(2.0f, g));
    }
    const float st = fq(omax(0.0f, fs(1.0f, fm(c, c))));
    const float phi = fm(kTwoPi, u2);
    float sp, cp;
    sincos_f(phi, sp, cp);
    const Frame f = make_frame(wo);  // coordinateSystem(wo, tangent, bitangent)
    return xadd(xadd(xmuls(f.t, fm(st, cp)), xmuls(f.b, fm(st, sp))), xmuls(wo, c));
}

// HomogeneousMedium::transmittance: exp(-sigma_t * distance) per channel.
__device__ __forceinline__ f3 transmittance(const DeviceScene& s, float dist) {
    return mk(expf(fm(-s.sigma_t[0], dist)), expf(fm(-s.sigma_t[1], dist)), expf(fm(-s.sigma_t[2], dist)));
}

// HomogeneousMedium::sampleDistance: exponential distance with the mean extinction; returns
// true and the distance t for a scattering event before maxDist (weight sigma_s * Tr / avg^2),
// else false with weight Tr(maxDist).
__device__ __forceinline__ bool medium_sample(const DeviceScene& s, float max_dist, float u, float& t, f3& weight) {
    if (s.avg_sigma_t < 1e-6f) {
        weight = mk(1.0f, 1.0f, 1.0f);
        return false;
    }
    t = fd(-logf(fs(1.0f, u)), s.avg_sigma_t);
    if (t < max_dist) {
        const f3 tr = transmittance(s, t);
        weight = xdivs(xmul(ld3(s.sigma_s), tr), fm(s.avg_sigma_t, s.avg_sigma_t));
        return true;
    }
    weight = transmittance(s, max_dist);
    return false;
}

// ----------------------------------------------------------------------------------------
// Camera rays
// ----------------------------------------------------------------------------------------

__device__ __forceinline__ void concentric_disk(float u1, float u2, float& ox, float& oy) {
    const float sx = fs(fm(2.0f, u1), 1.0f);
    const float sy = fs(fm(2.0f, u2), 1.0f);
    if (sx == 0.0f && sy == 0.0f) {
        ox = oy = 0.0f;
        return;
    }
    float r, theta;
    if (fabsf(sx) > fabsf(sy)) {
        r = sx;
        theta = fm(kPi / 4.0f, fd(sy, sx));
    } else {
        r = sy;
        theta = fs(kPi / 2.0f, fm(kPi / 4.0f, fd(sx, sy)));
    }
    float st, ct;
    sincos_f(theta, st, ct);
    ox = fm(r, ct);
    oy = fm(r, st);
}

__device__ __forceinline__ f3 cam_to_world(const CameraDev& c, f3 d) {
    return xadd(xadd(xmuls(ld3(c.right), d.x), xmuls(ld3(c.up), d.y)), xmuls(ld3(c.forward), d.z));
}

// PinholeCamera / ThinLensCamera::generateRay
__device__ __forceinline__ void camera_ray(const CameraDev& c, float px, float py, float lu, float lv, f3& o, f3& d) {
    const f3 local = mk(fd(fs(px, c.cx), c.fx), fd(fs(c.cy, py), c.fy), 1.0f);
    const f3 pos = ld3(c.position);
    const f3 dir = xnorm(xnorm(cam_to_world(c, local)));
    if (c.model != RBR_CAMERA_THIN_LENS) {
        o = xadd(pos, cam_to_world(c, mk(0.0f, 0.0f, 0.0f)));
        d = dir;
        return;
    }
    if (c.lens_radius > 0.0f) {
        float lx, ly;
        concentric_disk(lu, lv, lx, ly);
        const f3 lens = xadd(pos, xmuls(xadd(xmuls(ld3(c.right), lx), xmuls(ld3(c.up), ly)), c.lens_radius));
        const float ft = fd(c.focal_distance, fabsf(xdot(dir, ld3(c.forward))));
        const f3 focus = xadd(pos, xmuls(dir, ft));
        o = lens;
        d = xnorm(xnorm(xsub(focus, lens)));
        return;
    }
    o = pos;
    d = xnorm(dir);
}

}  // namespace rbr
