// Float sine and cosine of one angle for the path tracer's sampling routines.
//
// Every call site passes an angle in [-pi, 2 pi] (2 pi u for a uniform u, and the concentric
// disk's pi/4 ratios). On |x| <= 8 both results are within 1 ulp of the exact values (faithful:
// one of the two floats that bracket sin x and cos x), which the CPU test
// tests/test_trig.py checks on every float of [-2 pi, 2 pi] at and above 2^-12 in magnitude and
// on a sample of the rest.
//
// Method (Cody and Waite, "Software Manual for the Elementary Functions", 1980): k = the
// integer nearest x / (pi/2); r = x - k pi/2 with pi/2 split into three floats, each product
// subtracted by one fused multiply-add, so |r| <= pi/4 carries about 70 bits of pi/2; then the
// Taylor polynomials sin r = r - r^3/3! + ... + r^9/9! and cos r = 1 - r^2/2! + ... - r^10/10!
// (truncation below 3e-9 relative on |r| <= pi/4), evaluated by Horner's rule with fused
// multiply-adds; the quadrant k mod 4 picks and signs the pair.
//
// All arithmetic is written as explicit fused multiply-adds and correctly rounded products, so
// the host build (the CPU test) and the device build give the same bits.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define RBR_TRIG_HD __host__ __device__ __forceinline__
#else
#define RBR_TRIG_HD inline
#endif

namespace rbr {

namespace trig_detail {
// pi/2 = kPio2A + kPio2B + kPio2C: each the float nearest what the previous parts leave.
constexpr float kPio2A = 1.57079637050628662109375f;
constexpr float kPio2B = -4.371138828673792886547e-8f;
constexpr float kPio2C = -1.715124510005881872797e-15f;
constexpr float kTwoOverPi = 0.636619772367581343f;

// Correctly rounded operations that the device compiler may not fuse into multiply-adds (the
// host build compiles without contraction, -ffp-contract=off).
#if defined(__CUDA_ARCH__)
RBR_TRIG_HD float mul(float a, float b) { return __fmul_rn(a, b); }
RBR_TRIG_HD float add(float a, float b) { return __fadd_rn(a, b); }
RBR_TRIG_HD float sub(float a, float b) { return __fsub_rn(a, b); }
#else
RBR_TRIG_HD float mul(float a, float b) { return a * b; }
RBR_TRIG_HD float add(float a, float b) { return a + b; }
RBR_TRIG_HD float sub(float a, float b) { return a - b; }
#endif
}  // namespace trig_detail

// sin x and cos x for |x| <= 8, each within 1 ulp.
RBR_TRIG_HD void sincos_f(float x, float& s, float& c) {
    using namespace trig_detail;
    const float k = rintf(mul(x, kTwoOverPi));
    // r = rh + rl = x - k pi/2. x - k A is exact (x and k A agree in their leading bits); -k B
    // is split into a float and its exact rounding error (one fused multiply-add), and the sum
    // t - k B into rh and its exact error (Knuth's two-sum); -k C only enters rl.
    const float t = fmaf(-k, kPio2A, x);
    const float pb = mul(-k, kPio2B);
    const float pbl = fmaf(-k, kPio2B, -pb);
    const float rh = add(t, pb);
    const float bv = sub(rh, t);
    const float err = add(sub(t, sub(rh, bv)), sub(pb, bv));
    const float rl = fmaf(-k, kPio2C, add(err, pbl));
    const float r2 = mul(rh, rh);
    const float r2l = fmaf(rh, rh, -r2);  // r2 + r2l = rh^2 exactly
    // sin r = r + r^3 p(r^2), p = -1/3! + r^2 (1/5! + r^2 (-1/7! + r^2 / 9!)); the terms below
    // rh are summed first and added to rh once.
    float ps = fmaf(r2, 2.75573192239858907e-6f, -1.98412698412698413e-4f);
    ps = fmaf(ps, r2, 8.33333333333333333e-3f);
    ps = fmaf(ps, r2, -1.66666666666666667e-1f);
    const float ts = fmaf(mul(r2, rh), ps, fmaf(mul(-0.5f, r2), rl, rl));
    const float sr = add(rh, ts);
    // cos r = 1 - r^2/2 + r^4 q(r^2), q = 1/4! + r^2 (-1/6! + r^2 (1/8! - r^2 / 10!)); 1 - r^2/2
    // is kept as a float plus its exact rounding error.
    float pc = fmaf(r2, -2.75573192239858907e-7f, 2.48015873015873016e-5f);
    pc = fmaf(pc, r2, -1.38888888888888889e-3f);
    pc = fmaf(pc, r2, 4.16666666666666667e-2f);
    const float h = fmaf(-0.5f, r2, 1.0f);
    const float hl = fmaf(-0.5f, r2, sub(1.0f, h));  // 1 - r2/2 - h, exact
    const float tc = fmaf(mul(pc, r2), r2, fmaf(-0.5f, r2l, fmaf(-rh, rl, hl)));
    const float cr = add(h, tc);
    const int q = static_cast<int>(k) & 3;
    s = q == 0 ? sr : q == 1 ? cr : q == 2 ? -sr : -cr;
    c = q == 0 ? cr : q == 1 ? -sr : q == 2 ? -cr : sr;
}

}  // namespace rbr
