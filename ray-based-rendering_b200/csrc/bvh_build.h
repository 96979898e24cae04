// Host BVH construction: binned SAH binary tree -> 8-wide tree -> quantised node words.
#pragma once

#include <stdint.h>

#include <vector>

namespace rbr {

struct Box {
    float lo[3];
    float hi[3];
};

struct WideBVH {
    std::vector<uint32_t> nodes;      // kNodeWords words per node; node 0 is the root
    std::vector<uint32_t> leaf_order; // input primitive index of every leaf record, in record order
    uint32_t max_depth = 0;           // depth of the wide tree (root = 1)
    uint32_t binary_nodes = 0;
    uint32_t wrapped_leaves = 0;      // leaves moved into a wide node of their own (rbr_layout.h:
                                      // at most kInnerRecordLimit records beside internal children)
};

// Builds the wide BVH over `boxes` (one per bounded primitive). Each box is grown by `pad`
// (absolute, world units) before quantisation so that box tests stay conservative with
// respect to the rounding of the primitive tests. Uses up to `threads` host threads.
// record_cost: cost of one leaf-record test relative to one wide-node test in the collapse's
// surface-area cost.
WideBVH build_wide_bvh(const std::vector<Box>& boxes, float pad, int threads, double record_cost = 1.0);

}  // namespace rbr
