#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <future>
#include <thread>

namespace mrt {

namespace {

constexpr int kBins = 32;
constexpr float kTraversal = 1.0f;
constexpr float kIntersect = 1.5f;
constexpr uint32_t kParallelThreshold = 1u << 15;

struct Bounds {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(const float* l, const float* h) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], l[k]);
            hi[k] = std::max(hi[k], h[k]);
        }
    }
    void growPoint(const float* p) { grow(p, p); }
    void grow(const Bounds& b) { grow(b.lo, b.hi); }
    float area() const {
        if (lo[0] > hi[0]) return 0.0f;
        const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.0f * (dx * dy + dy * dz + dz * dx);
    }
};

struct TmpNode {
    Bounds box;
    uint32_t child[2];
    uint32_t first, count;
    uint32_t axis;
};

struct Ctx {
    const std::vector<Box3>& boxes;
    std::vector<float> cent;  // 3 per prim
    std::vector<uint32_t> idx;
    std::vector<TmpNode> nodes;
    std::atomic<uint32_t> next{0};
    uint32_t maxLeaf;
    std::atomic<int> freeThreads;
};

void buildRange(Ctx& c, uint32_t nodeId, uint32_t b, uint32_t e) {
    TmpNode& node = c.nodes[nodeId];
    Bounds box, cb;
    for (uint32_t i = b; i < e; ++i) {
        const Box3& p = c.boxes[c.idx[i]];
        box.grow(p.lo, p.hi);
        cb.growPoint(&c.cent[3 * c.idx[i]]);
    }
    node.box = box;
    const uint32_t n = e - b;
    auto makeLeaf = [&](uint32_t axis) {
        node.child[0] = node.child[1] = ~0u;
        node.first = b;
        node.count = n;
        node.axis = axis;
    };
    if (n <= c.maxLeaf) {
        makeLeaf(0);
        return;
    }
    // binned SAH on each axis with a non-degenerate centroid extent
    float bestCost = FLT_MAX;
    int bestAxis = -1, bestSplit = -1;
    float scale[3];
    for (int a = 0; a < 3; ++a) {
        const float ext = cb.hi[a] - cb.lo[a];
        scale[a] = ext > 1e-20f ? kBins * (1.0f - 1e-6f) / ext : 0.0f;
    }
    // all three axes binned in one pass over the range
    Bounds bins[3][kBins];
    uint32_t cnt[3][kBins] = {};
    for (uint32_t i = b; i < e; ++i) {
        const uint32_t p = c.idx[i];
        for (int a = 0; a < 3; ++a) {
            if (scale[a] == 0.0f) continue;
            int k = int(scale[a] * (c.cent[3 * p + a] - cb.lo[a]));
            k = std::min(std::max(k, 0), kBins - 1);
            bins[a][k].grow(c.boxes[p].lo, c.boxes[p].hi);
            cnt[a][k]++;
        }
    }
    for (int a = 0; a < 3; ++a) {
        if (scale[a] == 0.0f) continue;
        // An empty bin changes neither bound nor count: the right-hand
        // areas carry over it, and a split after it costs exactly what the
        // split before it costs, which the strict comparison below keeps.
        float rArea[kBins];
        uint32_t rCnt[kBins];
        Bounds acc;
        uint32_t s = 0;
        float area = 0.0f;
        for (int k = kBins - 1; k > 0; --k) {
            if (cnt[a][k]) {
                acc.grow(bins[a][k]);
                s += cnt[a][k];
                area = acc.area();
            }
            rArea[k] = area;
            rCnt[k] = s;
        }
        Bounds lacc;
        uint32_t ls = 0;
        for (int k = 0; k < kBins - 1; ++k) {
            if (!cnt[a][k]) continue;
            lacc.grow(bins[a][k]);
            ls += cnt[a][k];
            if (rCnt[k + 1] == 0) continue;
            const float cost = lacc.area() * ls + rArea[k + 1] * rCnt[k + 1];
            if (cost < bestCost) {
                bestCost = cost;
                bestAxis = a;
                bestSplit = k;
            }
        }
    }
    const float invArea = 1.0f / std::max(box.area(), 1e-30f);
    const float splitCost = kTraversal + kIntersect * invArea * bestCost;
    const float leafCost = kIntersect * float(n);
    if (bestAxis < 0 || (splitCost >= leafCost && n <= c.maxLeaf)) {
        if (bestAxis < 0 && n > c.maxLeaf) {
            // all centroids coincide: split the range in the middle
            bestAxis = 0;
            bestSplit = -2;
        } else {
            makeLeaf(0);
            return;
        }
    }
    uint32_t mid;
    if (bestSplit == -2) {
        mid = b + n / 2;
    } else {
        const int a = bestAxis;
        const float sc = scale[a], lo = cb.lo[a];
        auto it = std::partition(c.idx.begin() + b, c.idx.begin() + e, [&](uint32_t p) {
            int k = int(sc * (c.cent[3 * p + a] - lo));
            k = std::min(std::max(k, 0), kBins - 1);
            return k <= bestSplit;
        });
        mid = uint32_t(it - c.idx.begin());
        if (mid == b || mid == e) mid = b + n / 2;
    }
    const uint32_t l = c.next.fetch_add(2);
    node.child[0] = l;
    node.child[1] = l + 1;
    node.first = 0;
    node.count = 0;
    node.axis = uint32_t(bestAxis < 0 ? 0 : bestAxis);
    if (n >= kParallelThreshold && c.freeThreads.fetch_sub(1) > 0) {
        auto fut = std::async(std::launch::async, [&c, l, b, mid] { buildRange(c, l, b, mid); });
        buildRange(c, l + 1, mid, e);
        fut.get();
        c.freeThreads.fetch_add(1);
    } else {
        if (n >= kParallelThreshold) c.freeThreads.fetch_add(1);
        buildRange(c, l, b, mid);
        buildRange(c, l + 1, mid, e);
    }
}

}  // namespace

BvhResult buildBvh(const std::vector<Box3>& boxes, uint32_t maxLeaf, unsigned threads) {
    BvhResult r;
    for (int k = 0; k < 3; ++k) {
        r.bounds.lo[k] = FLT_MAX;
        r.bounds.hi[k] = -FLT_MAX;
    }
    const uint32_t n = uint32_t(boxes.size());
    if (n == 0) return r;
    Ctx c{boxes, {}, {}, {}, {}, std::max(1u, maxLeaf), {}};
    c.freeThreads = int(threads > 1 ? threads - 1 : 0);
    c.cent.resize(size_t(n) * 3);
    c.idx.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        c.idx[i] = i;
        for (int k = 0; k < 3; ++k) {
            c.cent[3 * i + k] = 0.5f * (boxes[i].lo[k] + boxes[i].hi[k]);
            r.bounds.lo[k] = std::min(r.bounds.lo[k], boxes[i].lo[k]);
            r.bounds.hi[k] = std::max(r.bounds.hi[k], boxes[i].hi[k]);
        }
    }
    c.nodes.resize(size_t(2) * n);
    c.next = 1;
    buildRange(c, 0, 0, n);
    // flatten depth-first; children of a node get two adjacent slots
    const uint32_t used = c.next.load();
    r.nodes.resize(used);
    uint32_t out = 1;
    struct Item {
        uint32_t tmp, slot, depth;
    };
    std::vector<Item> stack{{0, 0, 1}};
    while (!stack.empty()) {
        const Item it = stack.back();
        stack.pop_back();
        const TmpNode& t = c.nodes[it.tmp];
        MrtNode& o = r.nodes[it.slot];
        for (int k = 0; k < 3; ++k) {
            o.lo[k] = t.box.lo[k];
            o.hi[k] = t.box.hi[k];
        }
        r.maxDepth = std::max(r.maxDepth, it.depth);
        if (t.count > 0) {
            o.leftOrPrim = t.first;
            o.packed = (t.count << 2) | t.axis;
        } else {
            const uint32_t l = out;
            out += 2;
            o.leftOrPrim = l;
            o.packed = t.axis;
            stack.push_back({t.child[1], l + 1, it.depth + 1});
            stack.push_back({t.child[0], l, it.depth + 1});
        }
    }
    r.nodes.resize(out);
    r.primOrder = std::move(c.idx);
    return r;
}

std::vector<Box3> triangleBoxes(const float* positions, size_t stride, const uint32_t* indices, size_t nt) {
    std::vector<Box3> boxes(nt);
    for (size_t t = 0; t < nt; ++t) {
        Box3& b = boxes[t];
        for (int k = 0; k < 3; ++k) {
            b.lo[k] = 3.402823466e38f;
            b.hi[k] = -3.402823466e38f;
        }
        for (int c = 0; c < 3; ++c) {
            const float* v = positions + size_t(indices[t * 3 + c]) * stride;
            for (int k = 0; k < 3; ++k) {
                b.lo[k] = std::min(b.lo[k], v[k]);
                b.hi[k] = std::max(b.hi[k], v[k]);
            }
        }
    }
    return boxes;
}

}  // namespace mrt
