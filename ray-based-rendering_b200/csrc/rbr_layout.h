// Device memory layout of a scene (shared by the host builder and the kernels).
//
// Wide BVH node (80 B, five 16 B words, 16 B aligned):
//   word0  px, py, pz (f32)      biased origin of the node's quantisation grid: plane byte q of
//                                axis k lies at p_k + (kGridBias + q) * 2^(e_k - 127), so one
//                                byte permute of q into the mantissa of 32768.0f gives the
//                                factor (kGridBias + q) as an exact float
//          ex|ey|ez|imask (u8)   biased exponents of the per-axis grid step 2^(e-127),
//                                imask bit s = slot s holds an internal node
//   word1  child_base (u32)      index of the first internal child (children are stored
//                                consecutively in slot order)
//          prim_base (u32)       index of the first leaf record of this node's leaves
//          meta[8] (u8)          per slot: (width << 5) | position of the slot's bits in the
//                                node's 32-bit hit mask -- leaf: width = record count (1..4),
//                                position = first record offset from prim_base; internal:
//                                width 1, position 24 + slot; empty: 0
//   word2  qlo_x[8], qlo_y[8]    child boxes, 8-bit grid coordinates, rounded outwards with a
//   word3  qlo_z[8], qhi_x[8]    margin of at least kQuantMargin grid steps
//   word4  qhi_y[8], qhi_z[8]
// Slot s holds the child whose centre lies furthest towards the octant whose axis k is
// negative when bit k of s is set, so a ray with direction-sign bits D visits children in
// decreasing order of (s ^ D): roughly front to back, without sorting. A ray XORs the
// position of an internal slot with D, so bits 24-31 of its hit mask are in visiting order.
// A node with internal children keeps its leaf records at offsets below 24 (bits 24-31 are
// the internal slots'); a node without internal children may use all 32 record bits.
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
constexpr double kGridBias = 32768.0;        // plane byte q sits at grid coordinate kGridBias + q
constexpr uint32_t kGridBiasBits = 0x47000000u;  // 32768.0f
constexpr double kQuantMargin = 1.0 / 64.0;  // least outward rounding of a child plane, in grid steps
constexpr uint32_t kInnerRecordLimit = 24;   // records of a node that also has internal children

// Geometry constant of the reference (include/render/core/common.h:22).
constexpr float kEpsilon = 1e-4f;

// Device-side error bits (rbr_ctx::d_error).
constexpr int kErrStackOverflow = 1;
constexpr int kErrQueueOverflow = 2;
constexpr int kErrDeviceTimeout = 4;  // a bounded wait (tensor-core completion) ran out

}  // namespace rbr
