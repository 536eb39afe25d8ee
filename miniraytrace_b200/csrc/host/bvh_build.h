// Host BVH2 builder used by the commit: binned SAH over all three axes
// (the reference tries only the widest centroid axis, Bvh.cpp:52-55),
// 32 bins per axis, maximum leaf size 4 for triangle BLASes and 1 for the
// instance TLAS (as the reference), subtrees above a size threshold built on
// worker threads. Output uses the reference node encoding (Bvh.hpp:15-26):
// internal nodes hold the index of an adjacent child pair.
#pragma once

#include <cstdint>
#include <vector>

#include "../common/device_types.h"

namespace mrt {

struct Box3 {
    float lo[3], hi[3];
};

struct BvhResult {
    std::vector<MrtNode> nodes;      // node 0 = root; empty when no primitives
    std::vector<uint32_t> primOrder; // leaf ranges index this permutation
    Box3 bounds;                     // root bounds (inverted when empty)
    uint32_t maxDepth = 0;
};

BvhResult buildBvh(const std::vector<Box3>& boxes, uint32_t maxLeaf, unsigned threads);

// Boxes of nt triangles (indices 3 per triangle into positions with
// `stride` floats per vertex, xyz first): min/max over the three vertices
// in order, the arithmetic the device builder repeats.
std::vector<Box3> triangleBoxes(const float* positions, size_t stride, const uint32_t* indices, size_t nt);

}  // namespace mrt
