#include "lbvh.h"

#include <algorithm>
#include <cfloat>
#include <numeric>

#include "../common/lbvh_common.h"

namespace mrt {

MortonFrame mortonFrame(const std::vector<Box3>& boxes) {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (const Box3& b : boxes)
        for (int a = 0; a < 3; ++a) {
            const float c = (b.lo[a] + b.hi[a]) * 0.5f;
            lo[a] = std::min(lo[a], c);
            hi[a] = std::max(hi[a], c);
        }
    // one scale for all axes (the largest extent): cells stay cubes, so a
    // thin axis gets fewer significant code bits and is split late
    MortonFrame f;
    float ext = 0.0f;
    for (int a = 0; a < 3; ++a) {
        f.lo[a] = lo[a];
        ext = std::max(ext, hi[a] - lo[a]);
    }
    const float scale = ext > 0.0f ? 1024.0f / ext : 0.0f;
    for (int a = 0; a < 3; ++a) f.scale[a] = scale;
    return f;
}

BvhResult buildLbvh(const std::vector<Box3>& boxes) {
    BvhResult r;
    for (int k = 0; k < 3; ++k) {
        r.bounds.lo[k] = FLT_MAX;
        r.bounds.hi[k] = -FLT_MAX;
    }
    const uint32_t n = uint32_t(boxes.size());
    if (n == 0) return r;
    const MortonFrame f = mortonFrame(boxes);
    std::vector<uint32_t> code(n), order(n);
    for (uint32_t i = 0; i < n; ++i) code[i] = mortonCode(boxes[i].lo, boxes[i].hi, f.lo, f.scale);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return code[a] < code[b]; });
    std::vector<uint32_t> sorted(n);
    for (uint32_t i = 0; i < n; ++i) sorted[i] = code[order[i]];
    r.primOrder = order;

    // radix tree: internal nodes 0..n-2, children as MRT_LBVH_LEAF | position
    std::vector<uint32_t> left(n > 1 ? n - 1 : 0), right(n > 1 ? n - 1 : 0);
    for (int i = 0; i + 1 < int(n); ++i) {
        int first, last;
        lbvhNode(sorted.data(), int(n), i, left[size_t(i)], right[size_t(i)], first, last);
    }
    // flatten depth first with adjacent child pairs; boxes bottom-up afterwards
    r.nodes.resize(size_t(2) * n - 1);
    std::vector<uint32_t> src(r.nodes.size());  // radix-tree reference of each flattened node
    src[0] = n == 1 ? (MRT_LBVH_LEAF | 0u) : 0u;
    uint32_t next = 1;
    struct Item {
        uint32_t slot, depth;
    };
    std::vector<Item> stack{{0, 1}};
    while (!stack.empty()) {
        const Item it = stack.back();
        stack.pop_back();
        r.maxDepth = std::max(r.maxDepth, it.depth);
        MrtNode& o = r.nodes[it.slot];
        const uint32_t s = src[it.slot];
        if (s & MRT_LBVH_LEAF) {
            o.leftOrPrim = s & ~MRT_LBVH_LEAF;
            o.packed = 1u << 2;
            continue;
        }
        o.leftOrPrim = next;
        o.packed = 0;
        src[next] = left[s];
        src[next + 1] = right[s];
        stack.push_back({next + 1, it.depth + 1});
        stack.push_back({next, it.depth + 1});
        next += 2;
    }
    // children follow their parent, so a reverse sweep sees children first
    for (size_t i = r.nodes.size(); i-- > 0;) {
        MrtNode& o = r.nodes[i];
        if (o.packed >> 2) {
            const Box3& b = boxes[order[o.leftOrPrim]];
            for (int a = 0; a < 3; ++a) {
                o.lo[a] = b.lo[a];
                o.hi[a] = b.hi[a];
            }
        } else {
            const MrtNode& c0 = r.nodes[o.leftOrPrim];
            const MrtNode& c1 = r.nodes[o.leftOrPrim + 1];
            for (int a = 0; a < 3; ++a) {
                o.lo[a] = std::min(c0.lo[a], c1.lo[a]);
                o.hi[a] = std::max(c0.hi[a], c1.hi[a]);
            }
        }
    }
    for (int a = 0; a < 3; ++a) {
        r.bounds.lo[a] = r.nodes[0].lo[a];
        r.bounds.hi[a] = r.nodes[0].hi[a];
    }
    return r;
}

}  // namespace mrt
