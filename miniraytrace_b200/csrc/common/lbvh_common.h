// Morton codes and radix-tree topology shared by the host LBVH reference
// (csrc/host/lbvh.cpp) and the device builder (csrc/cuda/bvh_build.cu).
// Both sides compile these with no floating-point contraction, so every
// code and every split is the same on both.
#pragma once

#include <stdint.h>

#include "device_types.h"

MRT_HD inline int mrtClz(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __clz(int(x));
#else
    return x == 0u ? 32 : __builtin_clz(x);
#endif
}

// Top bit of a child reference: set for a leaf (sorted primitive position),
// clear for an internal node index.
#define MRT_LBVH_LEAF 0x80000000u

// Spreads the low 10 bits of v to every third bit (bit k -> bit 3k).
MRT_HD inline uint32_t mortonSpread10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// 30-bit code of a box centroid in a frame (lo, scale = 1024 / extent).
MRT_HD inline uint32_t mortonCode(const float boxLo[3], const float boxHi[3], const float lo[3],
                                  const float scale[3]) {
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
        const float c = (boxLo[a] + boxHi[a]) * 0.5f;
        float f = (c - lo[a]) * scale[a];
        f = f > 0.0f ? f : 0.0f;  // also maps NaN to 0
        f = f < 1023.0f ? f : 1023.0f;
        q[a] = uint32_t(f);
    }
    return (mortonSpread10(q[0]) << 2) | (mortonSpread10(q[1]) << 1) | mortonSpread10(q[2]);
}

// Length of the common prefix of sorted keys i and j, extended by the
// positions when the codes are equal; -1 outside [0, n).
MRT_HD inline int lbvhDelta(const uint32_t* codes, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = codes[i], b = codes[j];
    if (a == b) return 32 + mrtClz(uint32_t(i) ^ uint32_t(j));
    return mrtClz(a ^ b);
}

// Internal node i (0 <= i < n-1) of the radix tree over n sorted codes:
// its children (MRT_LBVH_LEAF | position, or an internal index) and the
// range [first, last] of sorted positions it covers (Karras 2012, section 4).
MRT_HD inline void lbvhNode(const uint32_t* codes, int n, int i, uint32_t& left, uint32_t& right, int& first,
                            int& last) {
    const int d = lbvhDelta(codes, n, i, i + 1) - lbvhDelta(codes, n, i, i - 1) > 0 ? 1 : -1;
    const int dMin = lbvhDelta(codes, n, i, i - d);
    int lMax = 2;
    while (lbvhDelta(codes, n, i, i + lMax * d) > dMin) lMax *= 2;
    int l = 0;
    for (int t = lMax / 2; t >= 1; t /= 2)
        if (lbvhDelta(codes, n, i, i + (l + t) * d) > dMin) l += t;
    const int j = i + l * d;
    const int dNode = lbvhDelta(codes, n, i, j);
    int s = 0;
    for (int t = (l + 1) / 2;; t = (t + 1) / 2) {
        if (lbvhDelta(codes, n, i, i + (s + t) * d) > dNode) s += t;
        if (t == 1) break;
    }
    const int gamma = i + s * d + (d < 0 ? -1 : 0);
    first = i < j ? i : j;
    last = i < j ? j : i;
    left = first == gamma ? (MRT_LBVH_LEAF | uint32_t(gamma)) : uint32_t(gamma);
    right = last == gamma + 1 ? (MRT_LBVH_LEAF | uint32_t(gamma + 1)) : uint32_t(gamma + 1);
}
