// Accuracy of rbr::sincos_f (ray-based-rendering_b200/csrc/rbr_trig.h), the float sine and
// cosine of the path tracer's sampling routines, compiled for the host: the same source and the
// same operation sequence (explicit fused multiply-adds, no contraction) as the device build.
// Checked against double-precision sin/cos on
//   - every float of [2^-12, 8] and of [-8, -2^-12] whose bit pattern is a multiple of `stride`
//     (stride 1 = all of them),
//   - every float within 2^16 representable steps of k pi/2, k = -5..5 (where the reduction
//     cancels most digits),
//   - zero, subnormals and a sample of the floats below 2^-12.
// Prints the largest error of each function in ulps of the exact result and the fraction of
// results that are the correctly rounded float.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "rbr_trig.h"

namespace {
double ulp_error(float got, double exact) {
    const float e = static_cast<float>(exact);
    double ulp = std::ldexp(1.0, -149);
    if (std::fabs(e) >= 1.17549435e-38f) {
        int ex = 0;
        std::frexp(static_cast<double>(e), &ex);
        ulp = std::ldexp(1.0, ex - 24);
    }
    return std::fabs(static_cast<double>(got) - exact) / ulp;
}
float from_bits(uint32_t u) {
    float x;
    std::memcpy(&x, &u, 4);
    return x;
}
uint32_t to_bits(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    return u;
}
struct Acc {
    double max_s = 0, max_c = 0;
    float at_s = 0, at_c = 0;
    uint64_t n = 0, cr = 0;
    void add(float x) {
        float s, c;
        rbr::sincos_f(x, s, c);
        const double ds = std::sin(static_cast<double>(x)), dc = std::cos(static_cast<double>(x));
        const double es = ulp_error(s, ds), ec = ulp_error(c, dc);
        if (es > max_s) max_s = es, at_s = x;
        if (ec > max_c) max_c = ec, at_c = x;
        cr += (s == static_cast<float>(ds)) + (c == static_cast<float>(dc));
        ++n;
    }
};
}  // namespace

int main(int argc, char** argv) {
    const uint32_t stride = argc > 1 ? static_cast<uint32_t>(std::strtoul(argv[1], nullptr, 10)) : 1u;
    Acc a;
    const uint32_t lo = to_bits(std::ldexp(1.0f, -12)), hi = to_bits(8.0f);
    for (uint32_t u = lo; u <= hi; u += stride) {
        a.add(from_bits(u));
        a.add(-from_bits(u));
    }
    for (int k = -5; k <= 5; ++k) {
        const float c = static_cast<float>(k * 1.57079632679489661923);
        const uint32_t b = to_bits(std::fabs(c));
        for (int32_t i = -65536; i <= 65536; ++i) {
            if (k == 0) break;
            const float x = from_bits(b + static_cast<uint32_t>(i));
            a.add(c < 0 ? -x : x);
        }
    }
    for (uint32_t u = 0; u < lo; u += 4099u) {
        a.add(from_bits(u));
        a.add(-from_bits(u));
    }
    std::printf("%llu %.6f %.9g %.6f %.9g %.6f\n", static_cast<unsigned long long>(a.n), a.max_s, a.at_s, a.max_c,
                a.at_c, static_cast<double>(a.cr) / (2.0 * static_cast<double>(a.n)));
    return 0;
}
