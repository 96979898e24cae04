// Host BVH construction for the GPU traversal kernels.
//
// 1. Binary tree, binned SAH (32 bins on each of the three axes, centroid binning), leaves of
//    at most 4 primitives (a wide node's leaf records then fit one 32-bit mask). The reference's own builder (src/acceleration/bvh.cpp:47-209) bins
//    12 buckets on the single axis of largest centroid extent and stops at 4 primitives; its
//    tree shape does not enter any result here: closest-hit answers are defined by the
//    primitives alone (smallest t, ties to the highest primitive id, as a brute-force loop in
//    primitive order gives), so the GPU tree is free to be a better one.
// 2. Collapse into 8-wide nodes by dynamic programming over the binary tree: for every binary
//    node and every slot budget i = 1..8, the least SAH cost of representing its subtree with
//    at most i children of the parent wide node, where a child is a leaf (a subtree of at most
//    kMaxLeafPrims primitives, cost area x primitives) or a wide node of its own (cost area +
//    the best spread of its subtree over 8 slots); the tree is then read off top-down.
// 3. Quantise each node's child boxes to 8-bit coordinates on a per-axis power-of-two grid,
//    rounded outwards with a margin of kQuantMargin steps, after growing every box by `pad`.
//    The stored grid origin is biased by kGridBias steps (rbr_layout.h).
#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>

#include "rbr_layout.h"

namespace rbr {
namespace {

constexpr int kBins = 32;
constexpr int kForceMedianDepth = 40;     // below this depth splits become plain median splits
constexpr uint32_t kParallelMin = 32768;  // subtrees at least this large may get their own thread
constexpr float kTraversalCost = 1.0f;
constexpr float kIntersectCost = 1.0f;

struct BNode {
    Box box;
    uint32_t left = 0, right = 0;
    uint32_t begin = 0, count = 0;  // count > 0: leaf over refs[begin, begin + count)
};

inline Box empty_box() {
    Box b;
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = FLT_MAX;
        b.hi[a] = -FLT_MAX;
    }
    return b;
}

inline void grow(Box& b, const Box& o) {
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = std::min(b.lo[a], o.lo[a]);
        b.hi[a] = std::max(b.hi[a], o.hi[a]);
    }
}

inline float half_area(const Box& b) {
    const float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    if (dx < 0.0f || dy < 0.0f || dz < 0.0f) return 0.0f;
    return dx * dy + dy * dz + dz * dx;
}

struct Builder {
    const std::vector<Box>& boxes;
    std::vector<float> cen;
    std::vector<uint32_t> refs;
    std::vector<BNode> nodes;
    std::atomic<uint32_t> next_node{1};
    std::atomic<int> threads_left{0};
    std::atomic<uint32_t> depth_seen{0};

    explicit Builder(const std::vector<Box>& b) : boxes(b) {}

    int bin_of(float c, float cmin, float scale) const {
        int k = static_cast<int>((c - cmin) * scale);
        return std::min(kBins - 1, std::max(0, k));
    }

    void build(uint32_t ni, uint32_t begin, uint32_t end, uint32_t depth) {
        uint32_t seen = depth_seen.load(std::memory_order_relaxed);
        while (depth > seen && !depth_seen.compare_exchange_weak(seen, depth)) {
        }
        Box b = empty_box(), cb = empty_box();
        for (uint32_t i = begin; i < end; ++i) {
            const uint32_t r = refs[i];
            grow(b, boxes[r]);
            for (int a = 0; a < 3; ++a) {
                cb.lo[a] = std::min(cb.lo[a], cen[3 * r + a]);
                cb.hi[a] = std::max(cb.hi[a], cen[3 * r + a]);
            }
        }
        BNode& node = nodes[ni];
        node.box = b;
        const uint32_t n = end - begin;
        if (n <= 1) {
            node.begin = begin;
            node.count = n;
            return;
        }
        uint32_t mid = begin;
        bool split = false;
        if (depth < kForceMedianDepth) {
            // binned SAH over the three axes
            float best = FLT_MAX;
            int best_axis = -1, best_bin = -1;
            float scale[3];
            struct Bin {
                Box box;
                uint32_t count;
            } bins[3][kBins];
            for (int a = 0; a < 3; ++a) {
                const float ext = cb.hi[a] - cb.lo[a];
                scale[a] = ext > 0.0f ? (kBins * (1.0f - 1e-6f)) / ext : 0.0f;
                for (int k = 0; k < kBins; ++k) {
                    bins[a][k].box = empty_box();
                    bins[a][k].count = 0;
                }
            }
            for (uint32_t i = begin; i < end; ++i) {
                const uint32_t r = refs[i];
                for (int a = 0; a < 3; ++a) {
                    if (scale[a] == 0.0f) continue;
                    Bin& bin = bins[a][bin_of(cen[3 * r + a], cb.lo[a], scale[a])];
                    grow(bin.box, boxes[r]);
                    bin.count++;
                }
            }
            for (int a = 0; a < 3; ++a) {
                if (scale[a] == 0.0f) continue;
                float rarea[kBins];
                uint32_t rcount[kBins];
                Box acc = empty_box();
                uint32_t cnt = 0;
                for (int k = kBins - 1; k >= 0; --k) {
                    grow(acc, bins[a][k].box);
                    cnt += bins[a][k].count;
                    rarea[k] = half_area(acc);
                    rcount[k] = cnt;
                }
                acc = empty_box();
                cnt = 0;
                for (int k = 0; k < kBins - 1; ++k) {
                    grow(acc, bins[a][k].box);
                    cnt += bins[a][k].count;
                    if (cnt == 0 || rcount[k + 1] == 0) continue;
                    const float cost = half_area(acc) * cnt + rarea[k + 1] * rcount[k + 1];
                    if (cost < best) {
                        best = cost;
                        best_axis = a;
                        best_bin = k;
                    }
                }
            }
            const float area = half_area(b);
            const float leaf_cost = kIntersectCost * n * area;
            const float split_cost = kTraversalCost * area + kIntersectCost * best;
            if (n <= static_cast<uint32_t>(kMaxLeafPrims) && (best_axis < 0 || leaf_cost <= split_cost)) {
                node.begin = begin;
                node.count = n;
                return;
            }
            if (best_axis >= 0) {
                const int a = best_axis;
                const float cmin = cb.lo[a], sc = scale[a];
                uint32_t* m = std::partition(refs.data() + begin, refs.data() + end, [&](uint32_t r) {
                    return bin_of(cen[3 * r + a], cmin, sc) <= best_bin;
                });
                mid = static_cast<uint32_t>(m - refs.data());
                split = mid > begin && mid < end;
            }
        }
        if (!split) {
            if (n <= static_cast<uint32_t>(kMaxLeafPrims)) {
                node.begin = begin;
                node.count = n;
                return;
            }
            int a = 0;
            float ext = -1.0f;
            for (int k = 0; k < 3; ++k) {
                const float e = cb.hi[k] - cb.lo[k];
                if (e > ext) {
                    ext = e;
                    a = k;
                }
            }
            mid = begin + n / 2;
            std::nth_element(refs.data() + begin, refs.data() + mid, refs.data() + end,
                             [&](uint32_t x, uint32_t y) { return cen[3 * x + a] < cen[3 * y + a]; });
        }
        const uint32_t c = next_node.fetch_add(2);
        nodes[ni].left = c;
        nodes[ni].right = c + 1;
        if (n >= kParallelMin && threads_left.fetch_sub(1) > 0) {
            std::thread t([=] { build(c, begin, mid, depth + 1); });
            build(c + 1, mid, end, depth + 1);
            t.join();
        } else {
            build(c, begin, mid, depth + 1);
            build(c + 1, mid, end, depth + 1);
        }
    }
};

inline float nudge_down(double x) {
    float f = static_cast<float>(x);
    if (static_cast<double>(f) > x) f = std::nextafter(f, -FLT_MAX);
    return f;
}

struct ChildRef {
    uint32_t bnode;
    bool leaf;
};

// The collapse's cost tables. Children have larger indices than their parent, so one pass from
// the last binary node to the root fills them.
// Costs are kept in double throughout, so that equal-cost choices resolve the same way in
// the table fill and in the read-off.
struct Collapse {
    static constexpr double kNodeCost = 1.0;  // per unit of half area: a wide-node test
    const double kPrimCost;                   // per unit of half area and primitive: a record test
    const Builder& B;
    std::vector<double> cost;    // cost[8 n + i - 1]: subtree n in at most i slots
    std::vector<double> single;  // subtree n in one slot: a leaf or a wide node
    std::vector<uint8_t> as_leaf;
    std::vector<uint32_t> rbeg, rcnt;  // the subtree's primitives: refs[rbeg, rbeg + rcnt)

    Collapse(const Builder& b, uint32_t used, double record_cost) : kPrimCost(record_cost), B(b) {
        cost.assign(size_t(used) * 8, 0.0);
        single.assign(used, 0.0);
        as_leaf.assign(used, 0);
        rbeg.assign(used, 0);
        rcnt.assign(used, 0);
        for (uint32_t ni = used; ni-- > 0;) {
            const BNode& nd = B.nodes[ni];
            const double area = half_area(nd.box);
            double* c = &cost[size_t(ni) * 8];
            if (nd.count > 0) {
                rbeg[ni] = nd.begin;
                rcnt[ni] = nd.count;
                single[ni] = area * nd.count * kPrimCost;
                as_leaf[ni] = 1;
                for (int i = 0; i < 8; ++i) c[i] = single[ni];
                continue;
            }
            rbeg[ni] = rbeg[nd.left];  // the left subtree's primitives precede the right's
            rcnt[ni] = rcnt[nd.left] + rcnt[nd.right];
            const double leafc = rcnt[ni] <= static_cast<uint32_t>(kMaxLeafPrims) ? area * rcnt[ni] * kPrimCost : 1e30;
            const double nodec = area * kNodeCost + spread(ni, 8);
            single[ni] = std::min(leafc, nodec);
            as_leaf[ni] = leafc <= nodec;
            c[0] = single[ni];
            for (int i = 2; i <= 8; ++i) c[i - 1] = std::min(c[i - 2], spread(ni, i));
        }
    }
    // least cost of spreading internal node ni's two subtrees over j slots, and the left's share
    double spread(uint32_t ni, int j, int* left_slots = nullptr) const {
        const BNode& nd = B.nodes[ni];
        double best = 1e30;
        for (int k = 1; k < j; ++k) {
            const double v = cost[size_t(nd.left) * 8 + k - 1] + cost[size_t(nd.right) * 8 + j - k - 1];
            if (v < best) {
                best = v;
                if (left_slots) *left_slots = k;
            }
        }
        return best;
    }
    // the children of the wide node made from internal node ni
    void children(uint32_t ni, int j, std::vector<uint32_t>& out) const {
        int k = 1;
        spread(ni, j, &k);
        place(B.nodes[ni].left, k, out);
        place(B.nodes[ni].right, j - k, out);
    }
    void place(uint32_t m, int i, std::vector<uint32_t>& out) const {
        if (i == 1 || B.nodes[m].count > 0) {
            out.push_back(m);
            return;
        }
        double best = single[m];
        int bj = 1;
        for (int j = 2; j <= i; ++j) {
            const double v = spread(m, j);
            if (v < best) {
                best = v;
                bj = j;
            }
        }
        if (bj == 1) out.push_back(m);
        else children(m, bj, out);
    }
};

}  // namespace

WideBVH build_wide_bvh(const std::vector<Box>& boxes, float pad, int threads, double record_cost) {
    WideBVH out;
    const uint32_t n = static_cast<uint32_t>(boxes.size());
    if (n == 0) return out;

    Builder B(boxes);
    B.cen.resize(3 * static_cast<size_t>(n));
    B.refs.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        B.refs[i] = i;
        for (int a = 0; a < 3; ++a) B.cen[3 * i + a] = 0.5f * (boxes[i].lo[a] + boxes[i].hi[a]);
    }
    B.nodes.resize(2 * static_cast<size_t>(n));
    B.threads_left = std::max(0, threads - 1);
    B.build(0, 0, n, 1);
    out.binary_nodes = B.next_node.load();
    const Collapse CP(B, out.binary_nodes, record_cost);

    // Collapse to 8-wide nodes, breadth first.
    struct Item {
        uint32_t wide;
        uint32_t bnode;
        uint32_t depth;
    };
    std::vector<Item> queue;
    queue.push_back({0, 0, 1});
    out.nodes.assign(kNodeWords, 0u);
    out.leaf_order.reserve(n);
    for (size_t head = 0; head < queue.size(); ++head) {
        const Item item = queue[head];
        out.max_depth = std::max(out.max_depth, item.depth);
        ChildRef ch[8];
        int k = 0;
        const BNode& root = B.nodes[item.bnode];
        if (root.count > 0) {
            ch[k++] = {item.bnode, true};
        } else {
            std::vector<uint32_t> lst;
            CP.children(item.bnode, 8, lst);
            for (uint32_t m : lst) ch[k++] = {m, CP.as_leaf[m] != 0};
        }
        // A node with internal children keeps its leaf records below bit kInnerRecordLimit of
        // the hit mask; over that, its largest leaves become internal children of their own
        // (a wide node holding just that leaf).
        {
            bool has_inner = false;
            uint32_t records = 0;
            for (int i = 0; i < k; ++i) {
                if (ch[i].leaf) records += CP.rcnt[ch[i].bnode];
                else has_inner = true;
            }
            while (has_inner && records > kInnerRecordLimit) {
                int big = -1;
                for (int i = 0; i < k; ++i)
                    if (ch[i].leaf && (big < 0 || CP.rcnt[ch[i].bnode] > CP.rcnt[ch[big].bnode])) big = i;
                ch[big].leaf = false;
                records -= CP.rcnt[ch[big].bnode];
                ++out.wrapped_leaves;
            }
        }
        // padded child boxes in double precision
        double clo[8][3], chi[8][3], nlo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, nhi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
        for (int i = 0; i < k; ++i) {
            const Box& bx = B.nodes[ch[i].bnode].box;
            for (int a = 0; a < 3; ++a) {
                clo[i][a] = static_cast<double>(bx.lo[a]) - pad;
                chi[i][a] = static_cast<double>(bx.hi[a]) + pad;
                nlo[a] = std::min(nlo[a], clo[i][a]);
                nhi[a] = std::max(nhi[a], chi[i][a]);
            }
        }
        // slots: child i goes to the slot whose octant direction its centre points to most
        int slot_child[8];
        for (int s = 0; s < 8; ++s) slot_child[s] = -1;
        {
            double score[8][8];
            for (int i = 0; i < k; ++i) {
                for (int s = 0; s < 8; ++s) {
                    double v = 0.0;
                    for (int a = 0; a < 3; ++a) {
                        const double d = 0.5 * (clo[i][a] + chi[i][a]) - 0.5 * (nlo[a] + nhi[a]);
                        v += ((s >> a) & 1) ? -d : d;
                    }
                    score[i][s] = v;
                }
            }
            bool child_used[8] = {}, slot_used[8] = {};
            for (int it = 0; it < k; ++it) {
                double best = -DBL_MAX;
                int bi = -1, bs = -1;
                for (int i = 0; i < k; ++i) {
                    if (child_used[i]) continue;
                    for (int s = 0; s < 8; ++s) {
                        if (slot_used[s]) continue;
                        if (score[i][s] > best) {
                            best = score[i][s];
                            bi = i;
                            bs = s;
                        }
                    }
                }
                child_used[bi] = slot_used[bs] = true;
                slot_child[bs] = bi;
            }
        }
        // Quantisation grid per axis: step s = 2^e, stored origin p (a float), grid coordinate 0
        // at g = p + kGridBias * s (exact in double). Every child plane must land on 0..255
        // with kQuantMargin steps to spare: g <= lo - margin and hi + margin <= g + 255 s.
        uint32_t* w = &out.nodes[static_cast<size_t>(item.wide) * kNodeWords];
        float p[3];
        double scale[3], gorg[3];
        uint32_t ebits = 0;
        for (int a = 0; a < 3; ++a) {
            const double ext = nhi[a] - nlo[a];
            int e = -126;
            if (ext > 0.0) {
                e = static_cast<int>(std::ceil(std::log2(ext / 254.0)));
                e = std::max(-126, std::min(127, e));
                while (e > -126 && std::ldexp(254.0, e - 1) >= ext) --e;
            }
            for (;; ++e) {
                scale[a] = std::ldexp(1.0, e);
                p[a] = nudge_down(nlo[a] - (kGridBias + 2.0 * kQuantMargin) * scale[a]);
                gorg[a] = static_cast<double>(p[a]) + kGridBias * scale[a];
                if ((nlo[a] - gorg[a] >= kQuantMargin * scale[a] &&
                     nhi[a] - gorg[a] <= (255.0 - kQuantMargin) * scale[a]) || e >= 127)
                    break;
            }
            ebits |= static_cast<uint32_t>(e + 127) << (8 * a);
            std::memcpy(&w[a], &p[a], 4);
        }
        uint8_t meta[8] = {}, qlo[3][8], qhi[3][8];
        uint32_t imask = 0;
        const uint32_t child_base = static_cast<uint32_t>(out.nodes.size() / kNodeWords);
        const uint32_t prim_base = static_cast<uint32_t>(out.leaf_order.size());
        uint32_t internal_rank = 0, prim_offset = 0;
        for (int s = 0; s < 8; ++s) {
            const int i = slot_child[s];
            if (i < 0) {
                for (int a = 0; a < 3; ++a) {
                    qlo[a][s] = 255;  // inverted box: never hit
                    qhi[a][s] = 0;
                }
                continue;
            }
            for (int a = 0; a < 3; ++a) {
                const double lo = std::floor((clo[i][a] - gorg[a]) / scale[a] - kQuantMargin);
                const double hi = std::ceil((chi[i][a] - gorg[a]) / scale[a] + kQuantMargin);
                qlo[a][s] = static_cast<uint8_t>(std::max(0.0, std::min(255.0, lo)));
                qhi[a][s] = static_cast<uint8_t>(std::max(0.0, std::min(255.0, hi)));
            }
            if (ch[i].leaf) {
                const uint32_t cb = CP.rbeg[ch[i].bnode], cc = CP.rcnt[ch[i].bnode];
                meta[s] = static_cast<uint8_t>((cc << 5) | prim_offset);
                for (uint32_t j = 0; j < cc; ++j) out.leaf_order.push_back(B.refs[cb + j]);
                prim_offset += cc;
            } else {
                meta[s] = static_cast<uint8_t>((1u << 5) | (24u + static_cast<uint32_t>(s)));
                imask |= 1u << s;
                queue.push_back({child_base + internal_rank, ch[i].bnode, item.depth + 1});
                ++internal_rank;
            }
        }
        out.nodes.resize(out.nodes.size() + static_cast<size_t>(internal_rank) * kNodeWords, 0u);
        w = &out.nodes[static_cast<size_t>(item.wide) * kNodeWords];  // may have moved
        for (int a = 0; a < 3; ++a) std::memcpy(&w[a], &p[a], 4);
        w[3] = ebits | (imask << 24);
        w[4] = internal_rank ? child_base : 0u;
        w[5] = prim_base;
        std::memcpy(&w[6], meta, 8);
        std::memcpy(&w[8], qlo[0], 8);
        std::memcpy(&w[10], qlo[1], 8);
        std::memcpy(&w[12], qlo[2], 8);
        std::memcpy(&w[14], qhi[0], 8);
        std::memcpy(&w[16], qhi[1], 8);
        std::memcpy(&w[18], qhi[2], 8);
    }
    return out;
}

}  // namespace rbr
