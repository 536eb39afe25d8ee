// Collapse of a binary BVH into 8-wide compressed nodes, shared by the host
// collapse (csrc/host/wide_bvh.cpp) and the device builder (csrc/cuda/
// bvh_build.cu). Both compile it without floating-point contraction, and the
// quantisation uses only exact double arithmetic, so a binary tree gives the
// same wide nodes on either side.
//
// Plan (Ylitie, Karras and Laine 2017, section 3.1): for each binary node n
// and i = 1..8, cost[i-1] = least SAH cost of the subtree at n represented
// as a forest of at most i roots; a root is a wide leaf (at most maxLeaf
// primitives) or a wide node whose children are the best forest of at most
// eight roots of n's two subtrees.
#pragma once

#include <math.h>
#include <stdint.h>

#include "device_types.h"

#define MRT_WIDE_NODE_COST 1.0f
#define MRT_WIDE_PRIM_COST 0.3f
#define MRT_WIDE_INF 3.402823466e38f

MRT_HD inline float wideArea(const float lo[3], const float hi[3]) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

// Cost table of a binary leaf (its primitives as one wide leaf; infinite
// when it holds more than maxLeaf).
MRT_HD inline void widePlanLeaf(float area, uint32_t count, uint32_t maxLeaf, float cost[8]) {
    const float c = count <= maxLeaf ? area * MRT_WIDE_PRIM_COST * float(count) : MRT_WIDE_INF;
    for (int j = 0; j < 8; ++j) cost[j] = c;
}

// Cost table of an internal binary node from its children's tables.
// split[0] = roots taken from the left child when n becomes a wide node (the
// right child gives 8 - split[0]); split[j-1] (j >= 2) = left roots of the
// best forest of at most j roots, 0 when the forest of j-1 roots is as good.
// Returns 1 when n's single root is a wide leaf.
MRT_HD inline uint8_t widePlanInternal(const float cl[8], const float cr[8], float area, uint32_t count,
                                       uint32_t maxLeaf, float cost[8], uint8_t split[8]) {
    const float leafCost = count <= maxLeaf ? area * MRT_WIDE_PRIM_COST * float(count) : MRT_WIDE_INF;
    float dist[9];
    uint8_t distK[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = 2; j <= 8; ++j) {
        dist[j] = MRT_WIDE_INF;
        for (int k = 1; k < j; ++k) {
            const float v = cl[k - 1] + cr[j - k - 1];
            if (v < dist[j]) {
                dist[j] = v;
                distK[j] = uint8_t(k);
            }
        }
    }
    const float internalCost = area * MRT_WIDE_NODE_COST + dist[8];
    const uint8_t asLeaf = leafCost <= internalCost ? 1 : 0;
    cost[0] = leafCost < internalCost ? leafCost : internalCost;
    split[0] = distK[8];
    for (int j = 2; j <= 8; ++j) {
        if (dist[j] < cost[j - 2]) {
            cost[j - 1] = dist[j];
            split[j - 1] = distK[j];
        } else {
            cost[j - 1] = cost[j - 2];
            split[j - 1] = 0;
        }
    }
    return asLeaf;
}

// One child of a wide node being emitted.
struct WideKid {
    float lo[3], hi[3];
    uint32_t count;  // primitives in the child's subtree
    uint32_t leaf;   // 1: a wide leaf holding those primitives
};

// Smallest e (biased, >= 1) with 255 * 2^(e-127) >= extent, exactly.
MRT_HD inline uint8_t wideExponentFor(float extent) {
    if (!(extent > 0.0f)) return 1;  // flat axis: every plane sits at the node origin
    int e = ilogb(double(extent)) - 8;
    while (ldexp(255.0, e) < double(extent) && e < 127) ++e;
    e = e < -126 ? -126 : (e > 127 ? 127 : e);
    return uint8_t(e + 127);
}

MRT_HD inline double wideScaleOf(uint32_t e) { return ldexp(1.0, int(e) - 127); }

// Grid index of the first plane at or below (lo) / at or above (hi) x:
// x / s is exact in double for a float x and a power-of-two s.
MRT_HD inline double wideGridBelow(float x, double s) { return floor(double(x) / s); }
MRT_HD inline double wideGridAbove(float x, double s) { return ceil(double(x) / s); }

// Fills node.p, e, imask, meta and the quantised boxes for nk (1..8) kids and
// returns the slot of each kid in slotOf[] (bySlot[s] = kid or -1). Leaf
// meta offsets count primitives in slot order from 0. childBase/primBase
// are left to the caller. Returns false if a kid does not fit the node's
// grid (impossible when every kid box lies inside the union of all kids).
//
// Quantisation grid per axis: planes at (k + q) * s, q = 0..255, s a power
// of two and the origin p = k * s a multiple of it. Every plane is then an
// exact real, and the integer grid indices are exact in double. p is a float:
// for s below lo's ulp, lo itself is a multiple of s; otherwise multiples of
// s are multiples of the ulp within lo's binade.
//
// Slots: children go to slots by direction from the node centre (greedy on
// the largest projection of the child centre offset onto the slot
// diagonals), so a ray visiting slots in (slot XOR ray octant) order meets
// them roughly front to back.
MRT_HD inline bool wideEmitNode(const WideKid* kids, int nk, MrtWideNode& node, int bySlot[8]) {
    float lo[3] = {MRT_WIDE_INF, MRT_WIDE_INF, MRT_WIDE_INF}, hi[3] = {-MRT_WIDE_INF, -MRT_WIDE_INF, -MRT_WIDE_INF};
    for (int i = 0; i < nk; ++i)
        for (int a = 0; a < 3; ++a) {
            lo[a] = kids[i].lo[a] < lo[a] ? kids[i].lo[a] : lo[a];
            hi[a] = kids[i].hi[a] > hi[a] ? kids[i].hi[a] : hi[a];
        }
    uint8_t* raw = reinterpret_cast<uint8_t*>(&node);
    for (size_t i = 0; i < sizeof(MrtWideNode); ++i) raw[i] = 0;
    double scale[3], base[3];
    for (int a = 0; a < 3; ++a) {
        uint32_t e = wideExponentFor(hi[a] - lo[a]);
        while (wideGridAbove(hi[a], wideScaleOf(e)) - wideGridBelow(lo[a], wideScaleOf(e)) > 255.0 && e < 254) ++e;
        node.e[a] = uint8_t(e);
        scale[a] = wideScaleOf(e);
        base[a] = wideGridBelow(lo[a], scale[a]);
        node.p[a] = float(base[a] * scale[a]);
        if (double(node.p[a]) != base[a] * scale[a]) return false;
    }
    int slotOf[8];
    for (int s = 0; s < 8; ++s) {
        slotOf[s] = -1;
        bySlot[s] = -1;
    }
    if (nk == 1) {
        slotOf[0] = 0;
    } else {
        float cost[8][8];
        for (int i = 0; i < nk; ++i) {
            float c[3];
            for (int a = 0; a < 3; ++a) c[a] = 0.5f * (kids[i].lo[a] + kids[i].hi[a]) - 0.5f * (lo[a] + hi[a]);
            for (int s = 0; s < 8; ++s)
                cost[i][s] = ((s & 1) ? c[0] : -c[0]) + ((s & 2) ? c[1] : -c[1]) + ((s & 4) ? c[2] : -c[2]);
        }
        bool used[8] = {false, false, false, false, false, false, false, false};
        for (int round = 0; round < nk; ++round) {
            float best = -MRT_WIDE_INF;
            int bi = -1, bs = -1;
            for (int i = 0; i < nk; ++i) {
                if (slotOf[i] >= 0) continue;
                for (int s = 0; s < 8; ++s)
                    if (!used[s] && cost[i][s] > best) {
                        best = cost[i][s];
                        bi = i;
                        bs = s;
                    }
            }
            if (bi < 0) {  // NaN costs: first free kid into first free slot
                for (int i = 0; i < nk && bi < 0; ++i)
                    if (slotOf[i] < 0) bi = i;
                for (int s = 0; s < 8 && bs < 0; ++s)
                    if (!used[s]) bs = s;
            }
            slotOf[bi] = bs;
            used[bs] = true;
        }
    }
    for (int i = 0; i < nk; ++i) bySlot[slotOf[i]] = i;
    uint32_t primOffset = 0;
    for (int s = 0; s < 8; ++s) {
        if (bySlot[s] < 0) continue;
        const WideKid& k = kids[bySlot[s]];
        for (int a = 0; a < 3; ++a) {
            const double ql = wideGridBelow(k.lo[a], scale[a]) - base[a];
            const double qh = wideGridAbove(k.hi[a], scale[a]) - base[a];
            if (!(ql >= 0.0 && qh <= 255.0 && ql <= qh)) return false;
            node.qlo[a][s] = uint8_t(ql);
            node.qhi[a][s] = uint8_t(qh);
        }
        if (k.leaf) {
            node.meta[s] = uint8_t((((1u << k.count) - 1u) << 5) | primOffset);
            primOffset += k.count;
        } else {
            node.meta[s] = uint8_t((1u << 5) | (24u + uint32_t(s)));
            node.imask |= uint8_t(1u << s);
        }
    }
    return true;
}
