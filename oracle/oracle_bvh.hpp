// ORACLE -- test infrastructure only. Not part of the product library.
//
// CPU restatement of the reference's binned-SAH BVH2 builder
// (reference core/src/accel/Bvh.cpp:41-156, Bvh.hpp:15-38) and its AABB type
// (core/include/mrt/MathTypes.hpp:18-46). The node layout is the reference's
// 32-byte BvhNode: lo.xyz + leftOrPrim, hi.xyz + packed = (count << 2) | axis;
// internal nodes have count 0 and children (left, left + 1).
//
// The floating-point operations and the std::partition / std::nth_element
// calls follow the reference order, so the tree is bit-identical to the
// reference build compiled with the same compiler (pinned by
// tests/test_oracle_pins.py against oracle/_ref).
#pragma once

#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <vector>

#include "oracle_math.hpp"

namespace orc {

using V3f = V3<float>;

struct Aabb {  // MathTypes.hpp:18-46
    V3f lo{FLT_MAX, FLT_MAX, FLT_MAX};
    V3f hi{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void expand(const V3f& p) { lo = vmin(lo, p); hi = vmax(hi, p); }
    void expand(const Aabb& b) { lo = vmin(lo, b.lo); hi = vmax(hi, b.hi); }
    V3f extent() const { return hi - lo; }
    V3f center() const { return 0.5f * (lo + hi); }
    bool valid() const { return lo.x <= hi.x; }
    float surfaceArea() const {
        if (!valid()) return 0.0f;
        const V3f e = extent();
        return 2.0f * (e.x * e.y + e.y * e.z + e.z * e.x);
    }
    // 8-corner transform (MathTypes.hpp:35-45)
    Aabb transformed(const M4<float>& m) const {
        Aabb out;
        for (int i = 0; i < 8; ++i) {
            const V3f c((i & 1) ? hi.x : lo.x, (i & 2) ? hi.y : lo.y, (i & 4) ? hi.z : lo.z);
            out.expand(m.mulPoint(c));
        }
        return out;
    }
};

struct BvhNode {  // Bvh.hpp:15-26
    float lo[3];
    uint32_t leftOrPrim;
    float hi[3];
    uint32_t packed;
};
static_assert(sizeof(BvhNode) == 32, "BvhNode is 32 bytes");

struct BvhBuild {
    std::vector<BvhNode> nodes;
    std::vector<uint32_t> primOrder;
    Aabb rootBounds;
};

namespace detail {

constexpr uint32_t kBins = 32;          // Bvh.cpp:13
constexpr float kTravCost = 1.0f;       // Bvh.cpp:14
constexpr float kIsectCost = 1.5f;      // Bvh.cpp:15

struct Ref {
    Aabb box;
    V3f c;
    uint32_t id;
};

inline void setBox(BvhNode& n, const Aabb& b) {
    n.lo[0] = b.lo.x; n.lo[1] = b.lo.y; n.lo[2] = b.lo.z;
    n.hi[0] = b.hi.x; n.hi[1] = b.hi.y; n.hi[2] = b.hi.z;
}

// Bvh.cpp:41-133 (recursive range build)
inline void build(std::vector<Ref>& refs, std::vector<BvhNode>& nodes, uint32_t maxLeaf,
                  uint32_t node, uint32_t begin, uint32_t end) {
    const uint32_t n = end - begin;
    Aabb box;
    for (uint32_t i = begin; i < end; ++i) box.expand(refs[i].box);
    setBox(nodes[node], box);

    Aabb cbox;
    for (uint32_t i = begin; i < end; ++i) cbox.expand(refs[i].c);
    const V3f ce = cbox.extent();
    uint32_t axis = 0;  // widest centroid axis only (Bvh.cpp:52-55)
    if (ce.y > ce.x) axis = 1;
    if (ce.z > ce[axis]) axis = 2;

    auto leaf = [&](uint32_t first, uint32_t cnt) {
        nodes[node].leftOrPrim = first;
        nodes[node].packed = (cnt << 2) | axis;
    };
    if (n <= maxLeaf || ce[axis] < 1e-8f) {
        leaf(begin, n);
        return;
    }

    Aabb binBox[kBins];
    uint32_t binCnt[kBins] = {};
    const float k = kBins * (1.0f - 1e-6f) / ce[axis];
    const float origin = cbox.lo[axis];
    for (uint32_t i = begin; i < end; ++i) {
        const uint32_t b = static_cast<uint32_t>(k * (refs[i].c[axis] - origin));
        binBox[b].expand(refs[i].box);
        binCnt[b]++;
    }
    float rArea[kBins];
    uint32_t rCnt[kBins];
    {
        Aabb acc;
        uint32_t cnt = 0;
        for (int i = int(kBins) - 1; i > 0; --i) {
            acc.expand(binBox[i]);
            cnt += binCnt[i];
            rArea[i] = acc.surfaceArea();
            rCnt[i] = cnt;
        }
    }
    float bestCost = kIsectCost * n;
    int best = -1;
    {
        Aabb acc;
        uint32_t cnt = 0;
        const float invArea = 1.0f / mmax(box.surfaceArea(), 1e-12f);
        for (uint32_t i = 0; i < kBins - 1; ++i) {
            acc.expand(binBox[i]);
            cnt += binCnt[i];
            if (cnt == 0 || rCnt[i + 1] == 0) continue;
            const float cost =
                kTravCost + kIsectCost * invArea * (acc.surfaceArea() * cnt + rArea[i + 1] * rCnt[i + 1]);
            if (cost < bestCost) {
                bestCost = cost;
                best = int(i);
            }
        }
    }
    uint32_t mid;
    if (best < 0) {
        if (n <= maxLeaf * 2) {
            leaf(begin, n);
            return;
        }
        mid = begin + n / 2;  // forced median split (Bvh.cpp:148-153)
        std::nth_element(refs.begin() + begin, refs.begin() + mid, refs.begin() + end,
                         [axis](const Ref& a, const Ref& b) { return a.c[axis] < b.c[axis]; });
    } else {
        auto it = std::partition(refs.begin() + begin, refs.begin() + end, [&](const Ref& r) {
            const uint32_t b = static_cast<uint32_t>(k * (r.c[axis] - origin));
            return b <= static_cast<uint32_t>(best);
        });
        mid = static_cast<uint32_t>(it - refs.begin());
        if (mid == begin || mid == end) mid = begin + n / 2;
    }
    const uint32_t left = static_cast<uint32_t>(nodes.size());
    nodes.emplace_back();
    nodes.emplace_back();
    nodes[node].leftOrPrim = left;
    nodes[node].packed = axis;
    build(refs, nodes, maxLeaf, left, begin, mid);
    build(refs, nodes, maxLeaf, left + 1, mid, end);
}

}  // namespace detail

// Bvh.cpp:137-156
inline BvhBuild buildBvh(const std::vector<Aabb>& bounds, uint32_t maxLeaf) {
    BvhBuild out;
    const uint32_t n = static_cast<uint32_t>(bounds.size());
    if (n == 0) return out;
    std::vector<detail::Ref> refs(n);
    for (uint32_t i = 0; i < n; ++i) refs[i] = {bounds[i], bounds[i].center(), i};
    out.nodes.reserve(2 * size_t(n));
    out.nodes.emplace_back();
    detail::build(refs, out.nodes, std::max(1u, maxLeaf), 0, 0, n);
    out.primOrder.resize(n);
    for (uint32_t i = 0; i < n; ++i) out.primOrder[i] = refs[i].id;
    for (uint32_t i = 0; i < n; ++i) out.rootBounds.expand(refs[i].box);
    return out;
}

}  // namespace orc
