#include "wide_bvh.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

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
    if (!(extent > 0.0f)) return 1;  // flat axis: tiny scale, all boxes decode to p
    int e = int(std::ceil(std::log2(double(extent) / 255.0)));
    e = std::max(-126, std::min(127, e));
    while (std::ldexp(255.0, e) < double(extent) && e < 127) ++e;
    return uint8_t(e + 127);
}

float scaleOf(uint8_t e) {
    uint32_t bits = uint32_t(e) << 23;
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// Decoding as the kernel does it: p + q * scale in single precision.
float decode(float p, uint32_t q, float s) { return p + float(q) * s; }

struct Collapser {
    const BvhResult& bin;
    uint32_t maxLeaf;
    std::vector<BinInfo> info;
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

    // Fills wide node `w` from the binary subtree rooted at `b`.
    void build(uint32_t w, uint32_t b, uint32_t depth) {
        out.maxDepth = std::max(out.maxDepth, depth);
        std::vector<uint32_t> kids;
        if (isLeaf(b) || info[b].count <= maxLeaf) {
            kids.push_back(b);
        } else {
            kids.push_back(left(b));
            kids.push_back(left(b) + 1);
            // open the largest child that cannot be a leaf until 8 slots are used
            while (kids.size() < 8) {
                int best = -1;
                float bestArea = -1.0f;
                for (size_t i = 0; i < kids.size(); ++i) {
                    const uint32_t k = kids[i];
                    if (isLeaf(k) || info[k].count <= maxLeaf) continue;
                    const float a = area(bin.nodes[k].lo, bin.nodes[k].hi);
                    if (a > bestArea) {
                        bestArea = a;
                        best = int(i);
                    }
                }
                if (best < 0) break;
                const uint32_t k = kids[size_t(best)];
                kids[size_t(best)] = left(k);
                kids.push_back(left(k) + 1);
            }
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
        float scale[3];
        for (int a = 0; a < 3; ++a) {
            node.p[a] = lo[a];
            node.e[a] = exponentFor(hi[a] - lo[a]);
            // the decoded top of the grid must reach the node's hi in float arithmetic
            while (decode(node.p[a], 255u, scaleOf(node.e[a])) < hi[a] && node.e[a] < 254) node.e[a]++;
            scale[a] = scaleOf(node.e[a]);
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
                // conservative quantisation under the kernel's decode arithmetic
                int ql = int(std::floor((kb.lo[a] - node.p[a]) / scale[a]));
                int qh = int(std::ceil((kb.hi[a] - node.p[a]) / scale[a]));
                ql = std::max(0, std::min(255, ql));
                qh = std::max(0, std::min(255, qh));
                while (ql > 0 && decode(node.p[a], uint32_t(ql), scale[a]) > kb.lo[a]) --ql;
                while (qh < 255 && decode(node.p[a], uint32_t(qh), scale[a]) < kb.hi[a]) ++qh;
                node.qlo[a][s] = uint8_t(ql);
                node.qhi[a][s] = uint8_t(qh);
            }
            const bool leaf = isLeaf(k) || info[k].count <= maxLeaf;
            if (leaf) {
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
    c.out.primOrder.reserve(bin.primOrder.size());
    c.out.nodes.resize(1);
    c.build(0, 0, 1);
    return std::move(c.out);
}

}  // namespace mrt
