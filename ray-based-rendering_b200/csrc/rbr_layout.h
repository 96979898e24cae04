// Device memory layout of a scene (shared by the host builder and the kernels).
//
// Wide BVH node (80 B, five 16 B words, 16 B aligned):
//   word0  px, py, pz (f32)      origin of the node's quantisation grid
//          ex|ey|ez|imask (u8)   biased exponents of the per-axis grid step 2^(e-127),
//                                imask bit s = slot s holds an internal node
//   word1  child_base (u32)      index of the first internal child (children are stored
//                                consecutively in slot order)
//          prim_base (u32)       index of the first leaf record of this node's leaves
//          meta[8] (u8)          per slot: leaf -> (count << 5) | offset (count 1..3,
//                                offset from prim_base); internal or empty -> 0
//   word2  qlo_x[8], qlo_y[8]    child boxes, 8-bit grid coordinates, rounded outwards
//   word3  qlo_z[8], qhi_x[8]
//   word4  qhi_y[8], qhi_z[8]
// Slot s holds the child whose centre lies furthest towards the octant whose axis k is
// negative when bit k of s is set, so a ray with direction-sign bits D visits children in
// decreasing order of (s ^ D): roughly front to back, without sorting.
//
// Leaf record (48 B, three 16 B words) in leaf order:
//   triangle  v0.xyz, e1.xyz, e2.xyz, tag      (e1 = v1 - v0, e2 = v2 - v0, rounded as
//                                               Triangle::intersect computes them)
//   sphere    centre.xyz, radius, r*r, -, -, -, -, -, tag
//   quad      origin.xyz, u.xyz, v.xyz, tag, dot(u,u), dot(v,v)
//   tag = primitive id | (type << 30)
// Planes (unbounded) live outside the tree: float4 (unit normal, d) + id.
#pragma once

#include <stdint.h>

namespace rbr {

constexpr uint32_t kPrimTriangle = 0;
constexpr uint32_t kPrimSphere = 1;
constexpr uint32_t kPrimQuad = 2;
constexpr uint32_t kPrimPlane = 3;
constexpr uint32_t kTypeShift = 30;
constexpr uint32_t kIdMask = (1u << kTypeShift) - 1;

constexpr int kNodeWords = 20;   // u32 words per wide node
constexpr int kRecordWords = 12; // u32 words per leaf record
constexpr int kMaxLeafPrims = 4;
constexpr int kStackSize = 64;   // traversal stack entries; the builder keeps the tree shallower
constexpr int kMaxTreeDepth = 62;

// Geometry constant of the reference (include/render/core/common.h:22).
constexpr float kEpsilon = 1e-4f;

// Device-side error bits (rbr_ctx::d_error).
constexpr int kErrStackOverflow = 1;
constexpr int kErrQueueOverflow = 2;
constexpr int kErrDeviceTimeout = 4;  // a bounded wait (tensor-core completion) ran out

}  // namespace rbr
