// Linear BVH over triangle boxes (Lauterbach et al. 2009; topology by
// Karras, "Maximizing Parallelism in the Construction of BVHs, Octrees, and
// k-d Trees", HPG 2012): primitives sorted by the 30-bit Morton code of
// their box centroid (ties by primitive index), internal node i of the
// radix tree split where the common code prefix of its range ends.
//
// This host version is the reference the device builder (csrc/cuda/
// bvh_build.cu) is checked against: both evaluate the same float
// expressions in the same order, so the trees are identical node for node.
#pragma once

#include <cstdint>
#include <vector>

#include "bvh_build.h"

namespace mrt {

// Morton quantisation frame shared with the device builder: centroid bounds
// lo and per-axis scale 1024 / extent (0 for a flat axis).
struct MortonFrame {
    float lo[3];
    float scale[3];
};

MortonFrame mortonFrame(const std::vector<Box3>& boxes);

// The binary LBVH in BvhResult form (adjacent child pairs, depth-first,
// leaves of one primitive), ready for collapseToWide.
BvhResult buildLbvh(const std::vector<Box3>& boxes);

}  // namespace mrt
