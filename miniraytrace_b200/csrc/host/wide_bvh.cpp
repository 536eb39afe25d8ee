#include "wide_bvh.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace mrt {

namespace {

struct BinInfo {
    uint32_t begin = 0, count = 0;  // subtree range in bin.primOrder
};

float area(const float lo[3], const float hi[3]) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

// Smallest power-of-two scale 2^(e-127) with 255 * scale >= extent.
uint8_t exponentFor(float extent) {
    if (!(extent > 0.0f)) return 1;  // flat axis: every plane sits at the node origin
    int e = int(std::ceil(std::log2(double(extent) / 255.0)));
    e = std::max(-126, std::min(127, e));
    while (std::ldexp(255.0, e) < double(extent) && e < 127) ++e;
    return uint8_t(e + 127);
}

double scaleOf(uint8_t e) { return std::ldexp(1.0, int(e) - 127); }

// Grid index of the first plane at or below x (lo) / at or above x (hi):
// x / s is exact in double for a float x and a power-of-two s.
double gridBelow(float x, double s) { return std::floor(double(x) / s); }
double gridAbove(float x, double s) { return std::ceil(double(x) / s); }

// SAH costs of the collapse (Ylitie et al. 2017, section 3.1): a wide node
// costs its surface area times kNodeCost, a leaf its area times kPrimCost
// per primitive.
constexpr float kNodeCost = 1.0f;
constexpr float kPrimCost = 0.3f;

struct Collapser {
    const BvhResult& bin;
    uint32_t maxLeaf;
    std::vector<BinInfo> info;
    // Per binary node n and i = 1..8: cost[8n + i-1] = least SAH cost of the
    // subtree at n represented as a forest of at most i roots. split[8n + i-1]
    // = k when that forest takes k roots from the left child and i-k from the
    // right (0: the forest of i-1 roots is as good; for i = 1 see asLeaf).
    std::vector<float> cost;
    std::vector<uint8_t> split;
    std::vector<uint8_t> asLeaf;  // the single root of subtree n is a leaf
    WideBvh out;

    Collapser(const BvhResult& b, uint32_t ml) : bin(b), maxLeaf(ml) {}

    bool isLeaf(uint32_t n) const { return (bin.nodes[n].packed >> 2) != 0; }
    uint32_t left(uint32_t n) const { return bin.nodes[n].leftOrPrim; }

    void computeInfo() {
        info.resize(bin.nodes.size());
        // children always follow their parent in the flattened order
        for (size_t i = bin.nodes.size(); i-- > 0;) {
            const MrtNode& n = bin.nodes[i];
            if ((n.packed >> 2) != 0) {
                info[i] = {n.leftOrPrim, n.packed >> 2};
            } else {
                const BinInfo& a = info[n.leftOrPrim];
                const BinInfo& b = info[n.leftOrPrim + 1];
                info[i] = {std::min(a.begin, b.begin), a.count + b.count};
            }
        }
    }

    // Bottom-up dynamic programme over the binary tree.
    void plan() {
        const size_t n = bin.nodes.size();
        cost.assign(n * 8, 0.0f);
        split.assign(n * 8, 0);
        asLeaf.assign(n, 0);
        for (size_t i = n; i-- > 0;) {
            float* c = &cost[i * 8];
            const float a = area(bin.nodes[i].lo, bin.nodes[i].hi);
            const uint32_t cnt = info[i].count;
            const float leafCost = cnt <= maxLeaf ? a * kPrimCost * float(cnt) : FLT_MAX;
            if (isLeaf(uint32_t(i))) {
                if (cnt > maxLeaf) throw std::invalid_argument("binary leaf larger than the wide leaf limit");
                for (int j = 0; j < 8; ++j) c[j] = leafCost;
                asLeaf[i] = 1;
                continue;
            }
            const float* cl = &cost[size_t(left(uint32_t(i))) * 8];
            const float* cr = &cost[size_t(left(uint32_t(i)) + 1) * 8];
            float dist[9];
            uint8_t distK[9] = {};
            for (int j = 2; j <= 8; ++j) {
                dist[j] = FLT_MAX;
                for (int k = 1; k < j; ++k) {
                    const float v = cl[k - 1] + cr[j - k - 1];
                    if (v < dist[j]) {
                        dist[j] = v;
                        distK[j] = uint8_t(k);
                    }
                }
            }
            const float internalCost = a * kNodeCost + dist[8];
            asLeaf[i] = leafCost <= internalCost ? 1 : 0;
            c[0] = std::min(leafCost, internalCost);
            split[i * 8] = distK[8];  // the wide node made from n takes this split
            for (int j = 2; j <= 8; ++j) {
                if (dist[j] < c[j - 2]) {
                    c[j - 1] = dist[j];
                    split[i * 8 + size_t(j) - 1] = distK[j];
                } else {
                    c[j - 1] = c[j - 2];
                    split[i * 8 + size_t(j) - 1] = 0;
                }
            }
        }
    }

    // Roots of the best forest of at most j roots for subtree n.
    void gather(uint32_t n, uint32_t j, std::vector<uint32_t>& kids) const {
        while (j > 1 && split[size_t(n) * 8 + j - 1] == 0) --j;
        if (j == 1) {
            kids.push_back(n);
            return;
        }
        const uint32_t k = split[size_t(n) * 8 + j - 1];
        gather(left(n), k, kids);
        gather(left(n) + 1, j - k, kids);
    }

    bool leafChild(uint32_t k) const { return asLeaf[k] != 0; }

    // Fills wide node `w` from the binary subtree rooted at `b`.
    void build(uint32_t w, uint32_t b, uint32_t depth) {
        out.maxDepth = std::max(out.maxDepth, depth);
        std::vector<uint32_t> kids;
        if (leafChild(b)) {
            kids.push_back(b);
        } else {
            const uint32_t k = split[size_t(b) * 8];
            gather(left(b), k, kids);
            gather(left(b) + 1, 8 - k, kids);
        }
        // node box and quantisation frame
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (uint32_t k : kids)
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::min(lo[a], bin.nodes[k].lo[a]);
                hi[a] = std::max(hi[a], bin.nodes[k].hi[a]);
            }
        MrtWideNode node;
        std::memset(&node, 0, sizeof(node));
        // Quantisation grid per axis: planes at (k + q) * s, q = 0..255, s a
        // power of two and the origin p = k * s a multiple of it. Every plane
        // is then an exact real the kernel's error bound is taken against,
        // and the integer grid indices below are exact in double.
        double scale[3], base[3];
        for (int a = 0; a < 3; ++a) {
            uint8_t e = exponentFor(hi[a] - lo[a]);
            while (gridAbove(hi[a], scaleOf(e)) - gridBelow(lo[a], scaleOf(e)) > 255.0 && e < 254) ++e;
            node.e[a] = e;
            scale[a] = scaleOf(e);
            base[a] = gridBelow(lo[a], scale[a]);
            // k * s is a float: for s below lo's ulp, lo itself is a multiple of s;
            // otherwise multiples of s are multiples of the ulp within lo's binade
            node.p[a] = float(base[a] * scale[a]);
            if (double(node.p[a]) != base[a] * scale[a]) throw std::logic_error("wide BVH grid origin not representable");
        }
        // slot assignment by direction from the node centre (greedy on the
        // largest projection of child centre offset onto slot diagonals)
        const size_t nk = kids.size();
        int slotOf[8];
        for (int i = 0; i < 8; ++i) slotOf[i] = -1;
        if (nk == 1) {
            slotOf[0] = 0;
        } else {
            float cost[8][8];
            for (size_t i = 0; i < nk; ++i) {
                float c[3];
                for (int a = 0; a < 3; ++a)
                    c[a] = 0.5f * (bin.nodes[kids[i]].lo[a] + bin.nodes[kids[i]].hi[a]) - 0.5f * (lo[a] + hi[a]);
                for (int s = 0; s < 8; ++s)
                    cost[i][s] = ((s & 1) ? c[0] : -c[0]) + ((s & 2) ? c[1] : -c[1]) + ((s & 4) ? c[2] : -c[2]);
            }
            bool slotUsed[8] = {};
            for (size_t round = 0; round < nk; ++round) {
                float bestC = -FLT_MAX;
                int bi = -1, bs = -1;
                for (size_t i = 0; i < nk; ++i) {
                    if (slotOf[i] >= 0) continue;
                    for (int s = 0; s < 8; ++s)
                        if (!slotUsed[s] && cost[i][s] > bestC) {
                            bestC = cost[i][s];
                            bi = int(i);
                            bs = s;
                        }
                }
                slotOf[bi] = bs;
                slotUsed[bs] = true;
            }
        }
        // children by slot
        int bySlot[8];
        for (int s = 0; s < 8; ++s) bySlot[s] = -1;
        for (size_t i = 0; i < nk; ++i) bySlot[slotOf[i]] = int(i);
        // internal children get consecutive wide nodes in slot order
        std::vector<std::pair<uint32_t, uint32_t>> recurse;  // (wide index, binary node)
        node.childBase = uint32_t(out.nodes.size());
        node.primBase = uint32_t(out.primOrder.size());
        uint32_t primOffset = 0;
        for (int s = 0; s < 8; ++s) {
            if (bySlot[s] < 0) continue;
            const uint32_t k = kids[size_t(bySlot[s])];
            const MrtNode& kb = bin.nodes[k];
            for (int a = 0; a < 3; ++a) {
                // conservative: plane ql at or below the child's lo, qh at or above its hi
                const double ql = gridBelow(kb.lo[a], scale[a]) - base[a];
                const double qh = gridAbove(kb.hi[a], scale[a]) - base[a];
                if (!(ql >= 0.0 && qh <= 255.0 && ql <= qh)) throw std::logic_error("wide BVH child outside its node grid");
                node.qlo[a][s] = uint8_t(ql);
                node.qhi[a][s] = uint8_t(qh);
            }
            if (leafChild(k)) {
                const uint32_t n = info[k].count;
                node.meta[s] = uint8_t((((1u << n) - 1u) << 5) | primOffset);
                for (uint32_t i = 0; i < n; ++i) out.primOrder.push_back(bin.primOrder[info[k].begin + i]);
                primOffset += n;
            } else {
                node.meta[s] = uint8_t((1u << 5) | (24u + uint32_t(s)));
                node.imask |= uint8_t(1u << s);
                recurse.push_back({0u, k});
            }
        }
        // allocate the internal children now so they are consecutive
        const uint32_t first = uint32_t(out.nodes.size());
        out.nodes.resize(out.nodes.size() + recurse.size());
        node.childBase = first;
        out.nodes[w] = node;
        for (size_t i = 0; i < recurse.size(); ++i) build(first + uint32_t(i), recurse[i].second, depth + 1);
    }
};

}  // namespace

WideBvh collapseToWide(const BvhResult& bin, uint32_t maxLeafPrims) {
    Collapser c(bin, std::max(1u, std::min(3u, maxLeafPrims)));
    c.out.bounds = bin.bounds;
    if (bin.nodes.empty()) return std::move(c.out);
    c.computeInfo();
    c.plan();
    c.out.primOrder.reserve(bin.primOrder.size());
    c.out.nodes.resize(1);
    c.build(0, 0, 1);
    return std::move(c.out);
}

}  // namespace mrt
