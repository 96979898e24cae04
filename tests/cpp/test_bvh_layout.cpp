// CPU check of the wide-BVH builder (ray-based-rendering_b200/csrc/bvh_build.cpp) without a GPU:
// builds trees over seeded triangle soups, checks the node layout the traversal kernels rely on
// (every primitive in exactly one leaf record, leaves of at most kMaxLeafPrims records, at most
// 32 records per node, child indices inside the node array, quantised child boxes that contain
// every primitive below them), then replays the kernels' traversal order on the host (the same
// quantised slab test and nearest-first slot order as traverse() in rbr_device.cuh) and
// compares its closest hits with a brute-force loop over the same triangles.
// Usage: test_bvh_layout  (exit status 0 on success; one line per case on stdout)
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <utility>
#include <vector>

#include "bvh_build.h"
#include "rbr_layout.h"

using namespace rbr;

namespace {

struct V {
    float x, y, z;
};
V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V cross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Moller-Trumbore with the reference's absolute epsilon; the same function on both sides.
float hit_tri(const float* t, V o, V d, float tmax) {
    const V v0{t[0], t[1], t[2]}, e1 = sub(V{t[3], t[4], t[5]}, v0), e2 = sub(V{t[6], t[7], t[8]}, v0);
    const V h = cross(d, e2);
    const float a = dot(e1, h);
    if (std::fabs(a) < 1e-4f) return -1.0f;
    const float f = 1.0f / a;
    const V s = sub(o, v0);
    const float u = f * dot(s, h);
    if (u < 0.0f || u > 1.0f) return -1.0f;
    const V q = cross(s, e1);
    const float v = f * dot(d, q);
    if (v < 0.0f || u + v > 1.0f) return -1.0f;
    const float t2 = f * dot(e2, q);
    return (t2 < 1e-4f || t2 > tmax) ? -1.0f : t2;
}

float qbyte(uint64_t w, int i) { return static_cast<float>((w >> (8 * i)) & 0xFFu); }

struct Tree {
    const WideBVH& b;
    size_t nodes() const { return b.nodes.size() / kNodeWords; }
    const uint32_t* node(size_t i) const { return &b.nodes[i * kNodeWords]; }
};

// World-space box of slot s of node w (quantised planes).
void slot_box(const uint32_t* w, int s, double lo[3], double hi[3]) {
    for (int a = 0; a < 3; ++a) {
        float p;
        std::memcpy(&p, &w[a], 4);
        const int e = static_cast<int>((w[3] >> (8 * a)) & 0xFFu) - 127;
        uint64_t ql, qh;
        std::memcpy(&ql, &w[8 + 2 * a], 8);
        std::memcpy(&qh, &w[14 + 2 * a], 8);
        lo[a] = p + std::ldexp(kGridBias + static_cast<double>((ql >> (8 * s)) & 0xFFu), e);
        hi[a] = p + std::ldexp(kGridBias + static_cast<double>((qh >> (8 * s)) & 0xFFu), e);
    }
}

int fail(const char* what, size_t a = 0, size_t b = 0) {
    std::printf("FAIL: %s (%zu, %zu)\n", what, a, b);
    return 1;
}

// Layout checks, walking the tree from the root with the (node, slot) path to every leaf.
int check_layout(const Tree& t, const std::vector<Box>& boxes) {
    const size_t n = boxes.size(), nn = t.nodes();
    std::vector<int> seen(n, 0);
    struct Item {
        uint32_t node;
        std::vector<std::pair<uint32_t, int>> path;
    };
    std::vector<Item> todo{{0, {}}};
    size_t visited = 0;
    while (!todo.empty()) {
        Item it = todo.back();
        todo.pop_back();
        if (it.node >= nn) return fail("child index outside the node array", it.node, nn);
        if (++visited > nn) return fail("node reached twice (not a tree)", visited, nn);
        const uint32_t* w = t.node(it.node);
        const uint32_t imask = w[3] >> 24;
        uint64_t meta;
        std::memcpy(&meta, &w[6], 8);
        uint32_t rank = 0, records = 0;
        for (int s = 0; s < 8; ++s) {
            const uint32_t m = static_cast<uint32_t>((meta >> (8 * s)) & 0xFFu);
            if ((imask >> s) & 1u) {
                if (m != ((1u << 5) | (24u + static_cast<uint32_t>(s)))) return fail("internal slot meta", it.node, s);
                Item c{w[4] + rank++, it.path};
                c.path.push_back({it.node, s});
                todo.push_back(c);
                continue;
            }
            const uint32_t cnt = m >> 5, off = m & 31u;
            if (cnt > static_cast<uint32_t>(kMaxLeafPrims)) return fail("leaf larger than kMaxLeafPrims", cnt);
            if (off + cnt > 32) return fail("leaf records beyond the node's 32-bit mask", off, cnt);
            records += cnt;
            for (uint32_t r = 0; r < cnt; ++r) {
                const size_t rec = size_t(w[5]) + off + r;
                if (rec >= t.b.leaf_order.size()) return fail("record index outside the record array", rec);
                const uint32_t prim = t.b.leaf_order[rec];
                if (prim >= n) return fail("primitive index out of range", prim, n);
                ++seen[prim];
                // the primitive's box lies inside this slot's box and every slot box above it
                auto inside = [&](const uint32_t* ww, int ss) {
                    double lo[3], hi[3];
                    slot_box(ww, ss, lo, hi);
                    for (int a = 0; a < 3; ++a)
                        if (boxes[prim].lo[a] < lo[a] || boxes[prim].hi[a] > hi[a]) return false;
                    return true;
                };
                if (!inside(w, s)) return fail("leaf slot box does not contain its primitive", prim);
                for (auto& ps : it.path)
                    if (!inside(t.node(ps.first), ps.second)) return fail("ancestor slot box misses a primitive", prim);
            }
        }
        if (records > 32) return fail("more than 32 records in one node", records);
        if (imask != 0 && records > kInnerRecordLimit)
            return fail("records beside internal children beyond the limit", it.node, records);
    }
    for (size_t i = 0; i < n; ++i)
        if (seen[i] != 1) return fail("primitive not in exactly one leaf", i, static_cast<size_t>(seen[i]));
    return 0;
}

// Host replay of traverse<false>() (rbr_device.cuh): returns the closest primitive or -1.
int replay(const Tree& t, const std::vector<float>& tris, V o, V d, float tmax) {
    float inv[3];
    bool neg[3];
    const float dd[3] = {d.x, d.y, d.z}, oo[3] = {o.x, o.y, o.z};
    for (int a = 0; a < 3; ++a) {
        inv[a] = 1.0f / std::copysign(std::max(std::fabs(dd[a]), 7.888609052e-31f), dd[a]);
        neg[a] = std::signbit(inv[a]);
    }
    const uint32_t oct = (neg[0] ? 1u : 0u) | (neg[1] ? 2u : 0u) | (neg[2] ? 4u : 0u);
    float tbest = tmax;
    int best = -1;
    struct G {
        uint32_t x, y;
    };
    auto visit = [&](uint32_t idx, G& ng, G& pg) {
        const uint32_t* w = t.node(idx);
        float p[3], A[3][2], B[3][2];
        std::memcpy(p, w, 12);
        const float kw[2] = {1.0f - 1.0f / 65536.0f, 1.0f + 1.0f / 65536.0f};
        for (int a = 0; a < 3; ++a) {
            const uint32_t bits = ((w[3] >> (8 * a)) & 0xFFu) << 23;
            float sc;
            std::memcpy(&sc, &bits, 4);
            for (int j = 0; j < 2; ++j) {
                A[a][j] = (sc * inv[a]) * kw[j];
                B[a][j] = ((p[a] - oo[a]) * inv[a]) * kw[j];
            }
        }
        const uint32_t imask = w[3] >> 24;
        uint64_t ql[3], qh[3], meta;
        for (int a = 0; a < 3; ++a) {
            std::memcpy(&ql[a], &w[8 + 2 * a], 8);
            std::memcpy(&qh[a], &w[14 + 2 * a], 8);
        }
        std::memcpy(&meta, &w[6], 8);
        uint32_t bits = 0;
        for (int i = 0; i < 8; ++i) {
            float tn[3], tf[3];
            for (int a = 0; a < 3; ++a) {
                tn[a] = std::fma(static_cast<float>(kGridBias) + qbyte(neg[a] ? qh[a] : ql[a], i), A[a][0], B[a][0]);
                tf[a] = std::fma(static_cast<float>(kGridBias) + qbyte(neg[a] ? ql[a] : qh[a], i), A[a][1], B[a][1]);
            }
            const float n_ = std::max({tn[0], tn[1], tn[2], 0.0f});
            const float f_ = std::min({tf[0], tf[1], tf[2], tbest});
            if (n_ <= f_) {
                uint32_t m = static_cast<uint32_t>((meta >> (8 * i)) & 0xFFu);
                if ((imask >> i) & 1u) m ^= oct;  // internal: bit 24 + (slot ^ octant)
                const uint32_t pos = m & 31u, width = m >> 5;
                const uint64_t mask = ((uint64_t(1) << width) - 1u) << pos;
                bits |= static_cast<uint32_t>(mask);
            }
        }
        const uint32_t inner = imask ? 0xFF000000u : 0u;
        ng = {w[4], (bits & inner) | (imask << 16)};
        pg = {w[5], bits & ~inner};
    };
    G stack[kStackSize];
    int sp = 0;
    G ng, pg;
    visit(0, ng, pg);
    while (true) {
        while (pg.y != 0) {
            const int i = __builtin_ctz(pg.y);
            pg.y &= pg.y - 1;
            const uint32_t prim = t.b.leaf_order[pg.x + i];
            const float h = hit_tri(&tris[9 * size_t(prim)], o, d, tbest);
            if (h >= 0.0f && (h < tbest || (h == tbest && static_cast<int>(prim) > best))) {
                tbest = h;
                best = static_cast<int>(prim);
            }
        }
        if (ng.y & 0xFF000000u) {
            const int b = 31 - __builtin_clz(ng.y);
            ng.y &= ~(1u << b);
            const uint32_t slot = static_cast<uint32_t>(b - 24) ^ oct, imask = (ng.y >> 16) & 0xFFu;
            const uint32_t child = ng.x + static_cast<uint32_t>(__builtin_popcount(imask & ((1u << slot) - 1u)));
            if (ng.y & 0xFF000000u) {
                if (sp == kStackSize) return -2;
                stack[sp++] = ng;
            }
            visit(child, ng, pg);
            continue;
        }
        if (sp == 0) break;
        ng = stack[--sp];
    }
    return best;
}

int brute(const std::vector<float>& tris, V o, V d, float tmax) {
    float tbest = tmax;
    int best = -1;
    for (size_t p = 0; p < tris.size() / 9; ++p) {
        const float h = hit_tri(&tris[9 * p], o, d, tbest);
        if (h >= 0.0f && (h < tbest || (h == tbest && static_cast<int>(p) > best))) {
            tbest = h;
            best = static_cast<int>(p);
        }
    }
    return best;
}

// kind 0: uniform soup in a cube; 1: all triangles in one plane; 2: each triangle twice;
// 3: a few large triangles among many tiny ones
std::vector<float> soup(int kind, size_t n, uint32_t seed) {
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> U(-10.0f, 10.0f), S(-1.0f, 1.0f);
    std::vector<float> t;
    for (size_t i = 0; i < n; ++i) {
        const float c[3] = {U(rng), U(rng), kind == 1 ? 0.0f : U(rng)};
        const float sz = kind == 3 ? (i % 50 == 0 ? 8.0f : 0.05f) : 1.0f;
        float tri[9];
        for (int k = 0; k < 3; ++k)
            for (int a = 0; a < 3; ++a) tri[3 * k + a] = c[a] + ((kind == 1 && a == 2) ? 0.0f : sz * S(rng));
        t.insert(t.end(), tri, tri + 9);
        if (kind == 2) t.insert(t.end(), tri, tri + 9);
    }
    return t;
}

}  // namespace

int main() {
    int failures = 0;
    const struct {
        int kind;
        size_t n;
    } cases[] = {{0, 1}, {0, 7}, {0, 100}, {0, 5000}, {0, 60000}, {1, 3000}, {2, 2000}, {3, 20000}};
    uint32_t seed = 1;
    for (const auto& c : cases) {
        const std::vector<float> tris = soup(c.kind, c.n, seed++);
        const size_t nt = tris.size() / 9;
        std::vector<Box> boxes(nt);
        float maxabs = 0.0f;
        for (size_t i = 0; i < nt; ++i)
            for (int a = 0; a < 3; ++a) {
                const float v0 = tris[9 * i + a], v1 = tris[9 * i + 3 + a], v2 = tris[9 * i + 6 + a];
                boxes[i].lo[a] = std::min({v0, v1, v2}) - 1e-3f;
                boxes[i].hi[a] = std::max({v0, v1, v2}) + 1e-3f;
                maxabs = std::max({maxabs, std::fabs(boxes[i].lo[a]), std::fabs(boxes[i].hi[a])});
            }
        const WideBVH bvh = build_wide_bvh(boxes, maxabs * (1.0f / 1048576.0f), 4);
        const Tree t{bvh};
        if (check_layout(t, boxes)) {
            ++failures;
            continue;
        }
        std::mt19937 rng(seed * 7919u);
        std::uniform_real_distribution<float> U(-12.0f, 12.0f);
        std::normal_distribution<float> N(0.0f, 1.0f);
        int mismatches = 0, hits = 0;
        const int rays = 2000;
        std::uniform_int_distribution<size_t> T(0, nt - 1);
        for (int r = 0; r < rays; ++r) {
            V o{U(rng), U(rng), U(rng)}, d{N(rng), N(rng), N(rng)};
            if (r % 2 == 1) {  // aimed at a random triangle's centroid: hits in every case
                const float* tr = &tris[9 * T(rng)];
                const V c{(tr[0] + tr[3] + tr[6]) / 3.0f, (tr[1] + tr[4] + tr[7]) / 3.0f, (tr[2] + tr[5] + tr[8]) / 3.0f};
                d = sub(c, o);
            } else if (r % 5 == 0) {
                d = {0.0f, 0.0f, (r % 10 == 0) ? 1.0f : -1.0f};  // axis-aligned: zero components
            }
            const float l = std::sqrt(dot(d, d));
            d = {d.x / l, d.y / l, d.z / l};
            const int a = replay(t, tris, o, d, 1e30f), b = brute(tris, o, d, 1e30f);
            hits += b >= 0;
            if (a != b) ++mismatches;
        }
        std::printf("kind %d, %zu triangles: %zu wide nodes, depth %u, %u wrapped leaves, %d of %d rays hit, "
                    "%d mismatches\n", c.kind, nt, t.nodes(), bvh.max_depth, bvh.wrapped_leaves, hits, rays, mismatches);
        if (mismatches) ++failures;
    }
    return failures ? 1 : 0;
}
