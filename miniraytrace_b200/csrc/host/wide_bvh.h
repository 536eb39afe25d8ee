// 8-wide compressed BVH (after Ylitie, Karras and Laine, "Efficient Incoherent
// Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017), built by
// collapsing a binary BVH on the host.
//
// Node record (MrtWideNode, 80 bytes = five 16-byte loads): the node's grid
// origin p and per-axis power-of-two scales s = 2^(e-127); per child slot an
// 8-bit quantised box (lo, hi); a mask of slots holding internal children;
// the index of the first internal child (internal children are stored
// consecutively in slot order) and of the first leaf primitive; and one meta
// byte per slot:
//   0                       empty slot
//   0b001xxxxx, x = 24+slot internal child
//   (2^n - 1) << 5 | offset leaf with n <= 3 primitives starting at
//                           primBase + offset (offset < 24)
// A quantised plane q stands for the exact real p + q * s. p is a multiple of
// s, so every plane lies on the grid k * s and the quantisation is checked
// with exact integer grid indices: the child's real box lies inside its
// planes.
// Children are placed in slots by direction from the parent centre, so a ray
// visiting slots in the order (slot XOR ray-sign-octant) descending meets
// them roughly front to back.
#pragma once

#include <cstdint>
#include <vector>

#include "../common/device_types.h"
#include "bvh_build.h"

namespace mrt {

struct WideBvh {
    std::vector<MrtWideNode> nodes;   // node 0 = root; empty when no primitives
    std::vector<uint32_t> primOrder;  // leaf primitives, in wide-leaf order
    Box3 bounds;
    uint32_t maxDepth = 0;
};

// Collapses `bin` (a binary BVH over prims 0..n-1 whose leaves hold at most
// `maxLeafPrims` primitives; std::invalid_argument otherwise) into an 8-wide
// BVH whose leaves hold at most `maxLeafPrims` (1..3) primitives each. The
// collapse is the SAH-optimal one over the binary tree's nodes (Ylitie et
// al., section 3.1: a dynamic programme over "subtree as a forest of at most
// i roots", i <= 8), so nodes are full wherever the tree allows.
WideBvh collapseToWide(const BvhResult& bin, uint32_t maxLeafPrims);

}  // namespace mrt
