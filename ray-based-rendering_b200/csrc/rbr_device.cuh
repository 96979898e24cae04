// Device-side scene view, exact float helpers and the 8-wide BVH traversal.
//
// Primitive tests restate the reference operation for operation with explicitly rounded
// intrinsics (__fmul_rn/__fadd_rn/__fsub_rn/__fdiv_rn/__fsqrt_rn never fuse into an FMA), so
// a GPU hit distance equals the reference's bit for bit:
//   Triangle::intersect  src/geometry/triangle.cpp:6-24   (Moller-Trumbore, |a| < EPSILON cull)
//   Sphere::intersect    src/geometry/sphere.cpp:6-19
//   Quad::intersect      src/geometry/quad.cpp:12-28
//   Plane::intersect     src/geometry/plane.cpp:12-20
// Closest hit keeps the smallest t and, at equal t, the highest primitive id: exactly what a
// loop over Scene::primitives() in order returns (a later primitive at t == tMax replaces an
// earlier one because only t > tMax is rejected).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rbr_layout.h"
#include "rbr_scene_dev.h"

namespace rbr {

// ----------------------------------------------------------------------------------------
// Exactly rounded float3 arithmetic (the reference's Vec3, include/render/core/vector.h)
// ----------------------------------------------------------------------------------------
struct f3 {
    float x, y, z;
};

__device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 xsub(f3 a, f3 b) { return mk(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
__device__ __forceinline__ f3 xadd(f3 a, f3 b) { return mk(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)); }
__device__ __forceinline__ f3 xmuls(f3 a, float s) { return mk(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)); }
__device__ __forceinline__ f3 xmul(f3 a, f3 b) { return mk(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z)); }
__device__ __forceinline__ f3 xneg(f3 a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float xdot(f3 a, f3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ f3 xcross(f3 a, f3 b) {
    return mk(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
              __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
// Vec3::operator/(float): multiply by the rounded reciprocal
__device__ __forceinline__ f3 xdivs(f3 a, float s) { return xmuls(a, __fdiv_rn(1.0f, s)); }
__device__ __forceinline__ float xlen(f3 a) { return __fsqrt_rn(xdot(a, a)); }
__device__ __forceinline__ f3 xnorm(f3 a) {
    const float l = xlen(a);
    return l > 0.0f ? xdivs(a, l) : mk(0.0f, 0.0f, 0.0f);
}
__device__ __forceinline__ f3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }

// ----------------------------------------------------------------------------------------
// Primitive tests. `tbest`/`best` hold the current closest hit (best = -1: none yet).
// Each returns the candidate t (or a negative value for no hit); acceptance with the tie rule
// happens in accept().
// ----------------------------------------------------------------------------------------
__device__ __forceinline__ bool accept(float t, uint32_t id, float tbest, int best) {
    return t < tbest || (t == tbest && static_cast<int>(id) > best);
}

// Triangle::intersect (triangle.cpp:6-24). v0, e1 = v1 - v0, e2 = v2 - v0.
__device__ __forceinline__ float hit_triangle(f3 o, f3 d, f3 v0, f3 e1, f3 e2, float tmax, float* pu = nullptr,
                                              float* pv = nullptr) {
    const f3 h = xcross(d, e2);
    const float a = xdot(e1, h);
    if (fabsf(a) < kEpsilon) return -1.0f;
    const float f = __fdiv_rn(1.0f, a);
    const f3 s = xsub(o, v0);
    const float u = __fmul_rn(f, xdot(s, h));
    if (u < 0.0f || u > 1.0f) return -1.0f;
    const f3 q = xcross(s, e1);
    const float v = __fmul_rn(f, xdot(d, q));
    if (v < 0.0f || __fadd_rn(u, v) > 1.0f) return -1.0f;
    const float t = __fmul_rn(f, xdot(e2, q));
    if (t < kEpsilon || t > tmax) return -1.0f;
    if (pu) {
        *pu = u;
        *pv = v;
    }
    return t;
}

// Sphere::intersect (sphere.cpp:6-19): near root, else far root, both within [EPSILON, tmax].
__device__ __forceinline__ float hit_sphere(f3 o, f3 d, f3 c, float r2, float tmax) {
    const f3 oc = xsub(o, c);
    const float a = xdot(d, d);
    const float halfB = xdot(oc, d);
    const float cc = __fsub_rn(xdot(oc, oc), r2);
    const float disc = __fsub_rn(__fmul_rn(halfB, halfB), __fmul_rn(a, cc));
    if (disc < 0.0f) return -1.0f;
    const float sq = __fsqrt_rn(disc);
    float t = __fdiv_rn(__fsub_rn(-halfB, sq), a);
    if (t < kEpsilon || t > tmax) {
        t = __fdiv_rn(__fadd_rn(-halfB, sq), a);
        if (t < kEpsilon || t > tmax) return -1.0f;
    }
    return t;
}

// Quad::intersect (quad.cpp:12-28); the normal is recomputed as the constructor computes it.
__device__ __forceinline__ float hit_quad(f3 o, f3 d, f3 org, f3 u, f3 v, float ulen2, float vlen2, float tmax) {
    const f3 n = xnorm(xcross(u, v));
    const float denom = xdot(n, d);
    if (fabsf(denom) < kEpsilon) return -1.0f;
    const float t = __fdiv_rn(xdot(xsub(org, o), n), denom);
    if (t < kEpsilon || t > tmax) return -1.0f;
    const f3 hp = xadd(o, xmuls(d, t));
    const f3 lp = xsub(hp, org);
    const float uc = __fdiv_rn(xdot(lp, u), ulen2);
    const float vc = __fdiv_rn(xdot(lp, v), vlen2);
    if (uc < 0.0f || uc > 1.0f || vc < 0.0f || vc > 1.0f) return -1.0f;
    return t;
}

// Plane::intersect (plane.cpp:12-20).
__device__ __forceinline__ float hit_plane(f3 o, f3 d, f3 n, float pd, float tmax) {
    const float denom = xdot(n, d);
    if (fabsf(denom) < kEpsilon) return -1.0f;
    const float t = __fdiv_rn(-__fadd_rn(xdot(n, o), pd), denom);
    if (t < kEpsilon || t > tmax) return -1.0f;
    return t;
}

// Tests leaf record `rec`; returns t or negative. `tag` receives the record's tag word.
__device__ __forceinline__ float hit_record(const float4* __restrict__ records, uint32_t rec, f3 o, f3 d, float tmax,
                                            uint32_t& tag) {
    const float4 a = __ldg(records + 3 * rec);
    const float4 b = __ldg(records + 3 * rec + 1);
    const float4 c = __ldg(records + 3 * rec + 2);
    tag = __float_as_uint(c.y);
    const uint32_t type = tag >> kTypeShift;
    if (type == kPrimTriangle) {
        return hit_triangle(o, d, mk(a.x, a.y, a.z), mk(a.w, b.x, b.y), mk(b.z, b.w, c.x), tmax);
    } else if (type == kPrimSphere) {
        return hit_sphere(o, d, mk(a.x, a.y, a.z), b.x, tmax);
    } else {
        return hit_quad(o, d, mk(a.x, a.y, a.z), mk(a.w, b.x, b.y), mk(b.z, b.w, c.x), c.z, c.w, tmax);
    }
}

// ----------------------------------------------------------------------------------------
// 8-wide node test
// ----------------------------------------------------------------------------------------
struct RayCtx {
    f3 o, d;
    float ix, iy, iz;   // 1 / d
    uint32_t oct;       // bit k set: d_k negative (visiting order)
    bool nx, ny, nz;    // sign of 1/d per axis (near/far plane choice)
};

// 1 / x with |x| raised to at least 2^-100 (sign kept). With an exact zero component the
// slab distances of that axis would be q*inf + (-inf) = NaN, which fminf/fmaxf ignore: every
// box the ray crosses in the other two axes would pass, a traversal of much of the tree. With
// 2^100 the distances stay finite and the axis is tested by containment, as the reference's
// BoundingBox::intersect does for a zero component (include/render/acceleration/bbox.h:92-120).
// Boxes stay conservative: a component below 2^-100 moves the ray by less than 2^-100 * t.
__device__ __forceinline__ float safe_inv(float x) {
    return __fdiv_rn(1.0f, copysignf(fmaxf(fabsf(x), 7.888609052e-31f), x));
}

__device__ __forceinline__ RayCtx make_ctx(f3 o, f3 d) {
    RayCtx r;
    r.o = o;
    r.d = d;
    r.ix = safe_inv(d.x);
    r.iy = safe_inv(d.y);
    r.iz = safe_inv(d.z);
    r.nx = signbit(r.ix);
    r.ny = signbit(r.iy);
    r.nz = signbit(r.iz);
    r.oct = (r.nx ? 1u : 0u) | (r.ny ? 2u : 0u) | (r.nz ? 4u : 0u);
    return r;
}

// kGridBias + (byte k of word), exactly: one byte permute of the byte into bits 8-15 of the
// mantissa of 32768.0f (bits 0x47000000).
__device__ __forceinline__ float qplane(uint32_t word, uint32_t k) {
    return __uint_as_float(__byte_perm(word, kGridBiasBits, 0x7404u | (k << 4)));
}

// Three-input minimum / maximum (sm_100); a NaN input is ignored unless all three are NaN.
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Mask of (width mod 32) bits starting at bit (pos mod 32); bits above 31 are dropped. PTX's
// bmsk.wrap uses the low five bits of both operands, so a word whose low byte holds a slot's
// field (and whose other bits hold anything) can be passed as it is.
__device__ __forceinline__ uint32_t bitmask_at(uint32_t pos, uint32_t width) {
    uint32_t d;
    asm("bmsk.wrap.b32 %0, %1, %2;" : "=r"(d) : "r"(pos), "r"(width));
    return d;
}

// Byte j of the result = oct if slot j of the four slots in imask4 is internal, else 0.
__device__ __forceinline__ uint32_t inner_oct4(uint32_t imask4, uint32_t oct) {
    return ((imask4 * 0x00204081u) & 0x01010101u) * oct;
}

// Relative widening of box intervals in t (2^-16): covers the rounding of the slab
// arithmetic and of the primitive tests near a box face.
constexpr float kTLo = 1.0f - 1.0f / 65536.0f;
constexpr float kTHi = 1.0f + 1.0f / 65536.0f;

// Per node and ray: the slab arithmetic of the node's grid and its slot bookkeeping.
// Plane byte q of axis k is hit at t = (kGridBias + q) a_k + b_k with a_k = s_k / d_k and
// b_k = (p_k - o_k) / d_k; near planes are scaled by kTLo and far planes by kTHi (the
// widening), so a (near, far) pair is one packed FMA.
struct NodeView {
    float2 ax, bx, ay, by, az, bz;   // (near, far) factors per axis
    uint2 nx, fx, ny, fy, nz, fz;    // near / far plane bytes per axis (8 slots)
    uint32_t pos_lo, pos_hi;         // per slot byte: first bit in bits 0-4 (internal: 24 + (slot ^ octant))
    uint32_t wid_lo, wid_hi;         // per slot byte: number of bits
    uint32_t imask, child_base, prim_base;
};

__device__ __forceinline__ NodeView node_view(const uint4* __restrict__ nodes, uint32_t idx, const RayCtx& r) {
    const uint4* np = nodes + 5 * static_cast<size_t>(idx);
    const uint4 w0 = __ldg(np);
    const uint4 w1 = __ldg(np + 1);
    const uint4 w2 = __ldg(np + 2);
    const uint4 w3 = __ldg(np + 3);
    const uint4 w4 = __ldg(np + 4);
    NodeView v;
    const float sx = __uint_as_float((w0.w & 0xFFu) << 23);
    const float sy = __uint_as_float(((w0.w >> 8) & 0xFFu) << 23);
    const float sz = __uint_as_float(((w0.w >> 16) & 0xFFu) << 23);
    const float2 kw = make_float2(kTLo, kTHi);
    const float ax = sx * r.ix, ay = sy * r.iy, az = sz * r.iz;
    const float bx = (__uint_as_float(w0.x) - r.o.x) * r.ix;
    const float by = (__uint_as_float(w0.y) - r.o.y) * r.iy;
    const float bz = (__uint_as_float(w0.z) - r.o.z) * r.iz;
    v.ax = __fmul2_rn(make_float2(ax, ax), kw);
    v.bx = __fmul2_rn(make_float2(bx, bx), kw);
    v.ay = __fmul2_rn(make_float2(ay, ay), kw);
    v.by = __fmul2_rn(make_float2(by, by), kw);
    v.az = __fmul2_rn(make_float2(az, az), kw);
    v.bz = __fmul2_rn(make_float2(bz, bz), kw);
    const uint2 qlox = make_uint2(w2.x, w2.y), qloy = make_uint2(w2.z, w2.w), qloz = make_uint2(w3.x, w3.y);
    const uint2 qhix = make_uint2(w3.z, w3.w), qhiy = make_uint2(w4.x, w4.y), qhiz = make_uint2(w4.z, w4.w);
    v.nx = r.nx ? qhix : qlox;
    v.fx = r.nx ? qlox : qhix;
    v.ny = r.ny ? qhiy : qloy;
    v.fy = r.ny ? qloy : qhiy;
    v.nz = r.nz ? qhiz : qloz;
    v.fz = r.nz ? qloz : qhiz;
    v.imask = w0.w >> 24;
    v.pos_lo = w1.z ^ inner_oct4(v.imask & 0xFu, r.oct);  // bits 5-7 of each byte (the width) are
    v.pos_hi = w1.w ^ inner_oct4(v.imask >> 4, r.oct);    // dropped by bmsk.wrap
    v.wid_lo = (w1.z >> 5) & 0x07070707u;
    v.wid_hi = (w1.w >> 5) & 0x07070707u;
    v.child_base = w1.x;
    v.prim_base = w1.y;
    return v;
}

// Slab test of slot i (0..7) against [0, tbest].
__device__ __forceinline__ bool slot_hit(const NodeView& v, int i, float tbest) {
    const uint32_t k = static_cast<uint32_t>(i & 3);
    const bool h = i >= 4;
    const float2 tx = __ffma2_rn(make_float2(qplane(h ? v.nx.y : v.nx.x, k), qplane(h ? v.fx.y : v.fx.x, k)), v.ax, v.bx);
    const float2 ty = __ffma2_rn(make_float2(qplane(h ? v.ny.y : v.ny.x, k), qplane(h ? v.fy.y : v.fy.x, k)), v.ay, v.by);
    const float2 tz = __ffma2_rn(make_float2(qplane(h ? v.nz.y : v.nz.x, k), qplane(h ? v.fz.y : v.fz.x, k)), v.az, v.bz);
    const float tn = fmax3(tx.x, ty.x, tz.x);
    const float tf = fmin3(tx.y, ty.y, tz.y);
    return fmaxf(tn, 0.0f) <= fminf(tf, tbest);
}

// Bits of slot i in the node's hit mask: its leaf records, or bit 24 + (slot ^ octant). The
// slot's position and width bytes are shifted to the bottom; bmsk.wrap ignores the rest (the
// widths are at most 7, so the next byte's bits start above bit 4).
__device__ __forceinline__ uint32_t slot_bits(const NodeView& v, int i) {
    const uint32_t sh = 8u * static_cast<uint32_t>(i & 3);
    return bitmask_at((i >= 4 ? v.pos_hi : v.pos_lo) >> sh, (i >= 4 ? v.wid_hi : v.wid_lo) >> sh);
}

// Splits a node's hit mask into ngroup = (child_base, internal hit bits << 24 | imask << 16)
// and pgroup = (prim_base, mask of the leaf records to test).
__device__ __forceinline__ void split_hits(const NodeView& v, uint32_t bits, uint2& ngroup, uint2& pgroup) {
    const uint32_t inner = v.imask ? 0xFF000000u : 0u;
    ngroup = make_uint2(v.child_base, (bits & inner) | (v.imask << 16));
    pgroup = make_uint2(v.prim_base, bits & ~inner);
}

// Tests the 8 children of node `idx`.
__device__ __forceinline__ void intersect_node(const uint4* __restrict__ nodes, uint32_t idx, const RayCtx& r,
                                               float tbest, uint2& ngroup, uint2& pgroup) {
    const NodeView v = node_view(nodes, idx, r);
    uint32_t bits = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
        if (slot_hit(v, i, tbest)) bits |= slot_bits(v, i);
    split_hits(v, bits, ngroup, pgroup);
}

// The same node test with fewer live registers: one (a, b) pair per axis instead of a
// (near, far) pair of pairs, scalar FMAs, and the widening applied after the min / max
// (c max(x) = max(c x) for c > 0). More issued instructions per slot, fewer registers.
__device__ __forceinline__ void intersect_node_lean(const uint4* __restrict__ nodes, uint32_t idx, const RayCtx& r,
                                                    float tbest, uint2& ngroup, uint2& pgroup) {
    const uint4* np = nodes + 5 * static_cast<size_t>(idx);
    const uint4 w0 = __ldg(np);
    const uint4 w1 = __ldg(np + 1);
    const uint4 w2 = __ldg(np + 2);
    const uint4 w3 = __ldg(np + 3);
    const uint4 w4 = __ldg(np + 4);
    const float ax = __uint_as_float((w0.w & 0xFFu) << 23) * r.ix;
    const float ay = __uint_as_float(((w0.w >> 8) & 0xFFu) << 23) * r.iy;
    const float az = __uint_as_float(((w0.w >> 16) & 0xFFu) << 23) * r.iz;
    const float bx = (__uint_as_float(w0.x) - r.o.x) * r.ix;
    const float by = (__uint_as_float(w0.y) - r.o.y) * r.iy;
    const float bz = (__uint_as_float(w0.z) - r.o.z) * r.iz;
    const uint2 qlox = make_uint2(w2.x, w2.y), qloy = make_uint2(w2.z, w2.w), qloz = make_uint2(w3.x, w3.y);
    const uint2 qhix = make_uint2(w3.z, w3.w), qhiy = make_uint2(w4.x, w4.y), qhiz = make_uint2(w4.z, w4.w);
    const uint2 nx = r.nx ? qhix : qlox, fx = r.nx ? qlox : qhix;
    const uint2 ny = r.ny ? qhiy : qloy, fy = r.ny ? qloy : qhiy;
    const uint2 nz = r.nz ? qhiz : qloz, fz = r.nz ? qloz : qhiz;
    const uint32_t imask = w0.w >> 24;
    const uint32_t pos_lo = w1.z ^ inner_oct4(imask & 0xFu, r.oct);
    const uint32_t pos_hi = w1.w ^ inner_oct4(imask >> 4, r.oct);
    const uint32_t wid_lo = (w1.z >> 5) & 0x07070707u, wid_hi = (w1.w >> 5) & 0x07070707u;
    uint32_t bits = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t k = static_cast<uint32_t>(i & 3), sh = 8u * k;
        const bool h = i >= 4;
        const float tnx = fmaf(qplane(h ? nx.y : nx.x, k), ax, bx), tfx = fmaf(qplane(h ? fx.y : fx.x, k), ax, bx);
        const float tny = fmaf(qplane(h ? ny.y : ny.x, k), ay, by), tfy = fmaf(qplane(h ? fy.y : fy.x, k), ay, by);
        const float tnz = fmaf(qplane(h ? nz.y : nz.x, k), az, bz), tfz = fmaf(qplane(h ? fz.y : fz.x, k), az, bz);
        const float tn = fmax3(tnx, tny, fmaxf(tnz, 0.0f)) * kTLo;
        const float tf = fmin3(tfx, tfy, tfz) * kTHi;
        if (tn <= fminf(tf, tbest))
            bits |= bitmask_at((h ? pos_hi : pos_lo) >> sh, (h ? wid_hi : wid_lo) >> sh);
    }
    const uint32_t inner = imask ? 0xFF000000u : 0u;
    ngroup = make_uint2(w1.x, (bits & inner) | (imask << 16));
    pgroup = make_uint2(w1.y, bits & ~inner);
}

// ----------------------------------------------------------------------------------------
// Traversal. Closest hit: returns the primitive id (or RBR_MISS) and its t.
// Any hit: returns 1 as soon as a primitive lies in [EPSILON, tmax].
// ----------------------------------------------------------------------------------------
// With kCount, `counts` receives the number of wide nodes fetched (x) and leaf records
// tested (y) by this ray: the traversal is deterministic per ray, so these are the ray's
// algorithmic node and record traffic.
// kLean: the node test with fewer live registers (intersect_node_lean).
template <bool kAny, bool kCount = false, bool kLean = false>
__device__ __forceinline__ uint32_t traverse(const DeviceScene& s, f3 o, f3 d, float tmax, float& thit, int* err,
                                             uint2* counts = nullptr) {
    float tbest = tmax;
    int best = -1;
    for (uint32_t i = 0; i < s.num_planes; ++i) {
        const float4 pl = __ldg(s.planes + i);
        const float t = hit_plane(o, d, mk(pl.x, pl.y, pl.z), pl.w, tbest);
        if (t >= 0.0f) {
            const uint32_t id = __ldg(s.plane_tags + i) & kIdMask;
            if (kAny) return 1u;
            if (accept(t, id, tbest, best)) {
                tbest = t;
                best = static_cast<int>(id);
            }
        }
    }
    if (s.num_nodes != 0) {
        const RayCtx r = make_ctx(o, d);
        uint2 stack[kStackSize];
        int sp = 0;
        uint2 ng, pg;
        if (kLean) intersect_node_lean(s.nodes, 0, r, tbest, ng, pg);
        else intersect_node(s.nodes, 0, r, tbest, ng, pg);
        if (kCount) counts->x += 1;
        while (true) {
            while (pg.y != 0) {
                const int i = __ffs(pg.y) - 1;
                pg.y &= pg.y - 1;
                if (kCount) counts->y += 1;
                uint32_t tag;
                const float t = hit_record(s.records, pg.x + i, o, d, tbest, tag);
                if (t >= 0.0f) {
                    if (kAny) return 1u;
                    const uint32_t id = tag & kIdMask;
                    if (accept(t, id, tbest, best)) {
                        tbest = t;
                        best = static_cast<int>(id);
                    }
                }
            }
            if (ng.y & 0xFF000000u) {
                const int b = 31 - __clz(ng.y);
                ng.y &= ~(1u << b);
                const uint32_t slot = static_cast<uint32_t>(b - 24) ^ r.oct;
                const uint32_t imask = (ng.y >> 16) & 0xFFu;
                const uint32_t child = ng.x + __popc(imask & ((1u << slot) - 1u));
                if (ng.y & 0xFF000000u) {
                    if (sp < kStackSize) {
                        stack[sp++] = ng;
                    } else {
                        atomicOr(err, kErrStackOverflow);
                        break;
                    }
                }
                if (kLean) intersect_node_lean(s.nodes, child, r, tbest, ng, pg);
                else intersect_node(s.nodes, child, r, tbest, ng, pg);
                if (kCount) counts->x += 1;
                continue;
            }
            if (sp == 0) break;
            ng = stack[--sp];
        }
    }
    if (kAny) return 0u;
    thit = tbest;
    return best < 0 ? 0xFFFFFFFFu : static_cast<uint32_t>(best);
}

// ----------------------------------------------------------------------------------------
// The same traversal as resumable steps, for persistent kernels that give a lane a new ray as
// soon as its current one is done (so a warp does not idle behind its longest ray).
// A step is one leaf-record test or one node test (after an optional stack pop).
// ----------------------------------------------------------------------------------------
struct TraceState {
    RayCtx r;
    float tbest;
    int best;
    uint2 ng, pg;
    int sp;
};

// Starts a ray: planes, then the root node. Returns true if the ray is already complete
// (any hit on a plane, or no BVH).
template <bool kAny>
__device__ __forceinline__ bool trace_begin(const DeviceScene& s, f3 o, f3 d, float tmax, TraceState& st,
                                            uint32_t& anyhit) {
    st.tbest = tmax;
    st.best = -1;
    anyhit = 0;
    for (uint32_t i = 0; i < s.num_planes; ++i) {
        const float4 pl = __ldg(s.planes + i);
        const float t = hit_plane(o, d, mk(pl.x, pl.y, pl.z), pl.w, st.tbest);
        if (t >= 0.0f) {
            const uint32_t id = __ldg(s.plane_tags + i) & kIdMask;
            if (kAny) {
                anyhit = 1;
                return true;
            }
            if (accept(t, id, st.tbest, st.best)) {
                st.tbest = t;
                st.best = static_cast<int>(id);
            }
        }
    }
    if (s.num_nodes == 0) return true;
    st.r = make_ctx(o, d);
    st.sp = 0;
    intersect_node(s.nodes, 0, st.r, st.tbest, st.ng, st.pg);
    return false;
}

// One step: the pending leaf records, then one node; returns true when the ray is complete.
template <bool kAny>
__device__ __forceinline__ bool trace_step(const DeviceScene& s, TraceState& st, uint2* stack, int* err,
                                           uint32_t& anyhit) {
    while (st.pg.y != 0) {
        const int i = __ffs(st.pg.y) - 1;
        st.pg.y &= st.pg.y - 1;
        uint32_t tag;
        const float t = hit_record(s.records, st.pg.x + i, st.r.o, st.r.d, st.tbest, tag);
        if (t >= 0.0f) {
            if (kAny) {
                anyhit = 1;
                return true;
            }
            const uint32_t id = tag & kIdMask;
            if (accept(t, id, st.tbest, st.best)) {
                st.tbest = t;
                st.best = static_cast<int>(id);
            }
        }
    }
    if ((st.ng.y & 0xFF000000u) == 0) {
        if (st.sp == 0) return true;
        st.ng = stack[--st.sp];  // only non-empty groups are pushed
    }
    const int b = 31 - __clz(st.ng.y);
    st.ng.y &= ~(1u << b);
    const uint32_t slot = static_cast<uint32_t>(b - 24) ^ st.r.oct;
    const uint32_t imask = (st.ng.y >> 16) & 0xFFu;
    const uint32_t child = st.ng.x + __popc(imask & ((1u << slot) - 1u));
    if (st.ng.y & 0xFF000000u) {
        if (st.sp < kStackSize) {
            stack[st.sp++] = st.ng;
        } else {
            atomicOr(err, kErrStackOverflow);
            return true;
        }
    }
    intersect_node(s.nodes, child, st.r, st.tbest, st.ng, st.pg);
    return false;
}

}  // namespace rbr
