#include "wide_bvh.h"

#include <algorithm>
#include <cstring>
#include <stdexcept>

#include "../common/wide_collapse.h"

namespace mrt {

namespace {

struct BinInfo {
    uint32_t begin = 0, count = 0;  // subtree range in bin.primOrder
};

struct Collapser {
    const BvhResult& bin;
    uint32_t maxLeaf;
    std::vector<BinInfo> info;
    // Per binary node n: cost[8n .. 8n+7] and split[8n .. 8n+7] as
    // widePlanInternal defines them; asLeaf[n]: n's single root is a leaf.
    std::vector<float> cost;
    std::vector<uint8_t> split;
    std::vector<uint8_t> asLeaf;
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
            const float a = wideArea(bin.nodes[i].lo, bin.nodes[i].hi);
            if (isLeaf(uint32_t(i))) {
                if (info[i].count > maxLeaf) throw std::invalid_argument("binary leaf larger than the wide leaf limit");
                widePlanLeaf(a, info[i].count, maxLeaf, &cost[i * 8]);
                asLeaf[i] = 1;
                continue;
            }
            const uint32_t l = left(uint32_t(i));
            asLeaf[i] = widePlanInternal(&cost[size_t(l) * 8], &cost[size_t(l + 1) * 8], a, info[i].count, maxLeaf,
                                         &cost[i * 8], &split[i * 8]);
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

    // Fills wide node `w` from the binary subtree rooted at `b`. Layout: the
    // node's internal children are allocated consecutively in slot order,
    // then each child's subtree follows in that order (depth first); the
    // node's leaf primitives come before those of its descendants.
    void build(uint32_t w, uint32_t b, uint32_t depth) {
        out.maxDepth = std::max(out.maxDepth, depth);
        std::vector<uint32_t> kids;
        if (asLeaf[b]) {
            kids.push_back(b);
        } else {
            const uint32_t k = split[size_t(b) * 8];
            gather(left(b), k, kids);
            gather(left(b) + 1, 8 - k, kids);
        }
        WideKid wk[8];
        for (size_t i = 0; i < kids.size(); ++i) {
            const MrtNode& kb = bin.nodes[kids[i]];
            for (int a = 0; a < 3; ++a) {
                wk[i].lo[a] = kb.lo[a];
                wk[i].hi[a] = kb.hi[a];
            }
            wk[i].count = info[kids[i]].count;
            wk[i].leaf = asLeaf[kids[i]];
        }
        MrtWideNode node;
        int bySlot[8];
        if (!wideEmitNode(wk, int(kids.size()), node, bySlot)) throw std::logic_error("wide BVH quantisation failed");
        node.primBase = uint32_t(out.primOrder.size());
        std::vector<uint32_t> recurse;
        for (int s = 0; s < 8; ++s) {
            if (bySlot[s] < 0) continue;
            const uint32_t k = kids[size_t(bySlot[s])];
            if (wk[bySlot[s]].leaf) {
                for (uint32_t i = 0; i < info[k].count; ++i) out.primOrder.push_back(bin.primOrder[info[k].begin + i]);
            } else {
                recurse.push_back(k);
            }
        }
        // allocate the internal children now so they are consecutive
        node.childBase = uint32_t(out.nodes.size());
        out.nodes.resize(out.nodes.size() + recurse.size());
        out.nodes[w] = node;
        for (size_t i = 0; i < recurse.size(); ++i) build(node.childBase + uint32_t(i), recurse[i], depth + 1);
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
