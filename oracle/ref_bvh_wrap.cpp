// ORACLE -- test infrastructure only.
//
// extern "C" wrapper around the reference's own BVH builder
// (core/src/accel/Bvh.cpp, compiled from the reference checkout by
// oracle/build_oracle.py into oracle/_ref/). It exposes the reference's
// BvhBuilder::build (Bvh.hpp:34-38) with the same signature as
// orc_bvh_build in oracle_capi.cpp, so tests can compare the two trees.
#include <cstring>
#include <vector>

#include "Bvh.hpp"

extern "C" uint32_t ref_bvh_build(const float* aabbs, uint32_t n, uint32_t maxLeaf, void* nodesOut,
                                  uint32_t* primOrderOut) {
    std::vector<mrt::Aabb> b(n);
    for (uint32_t i = 0; i < n; ++i) {
        b[i].lo = mrt::vec3(aabbs[i * 6], aabbs[i * 6 + 1], aabbs[i * 6 + 2]);
        b[i].hi = mrt::vec3(aabbs[i * 6 + 3], aabbs[i * 6 + 4], aabbs[i * 6 + 5]);
    }
    const mrt::BvhBuildResult r = mrt::BvhBuilder::build(b, maxLeaf);
    std::memcpy(nodesOut, r.nodes.data(), r.nodes.size() * sizeof(mrt::BvhNode));
    if (!r.primOrder.empty()) std::memcpy(primOrderOut, r.primOrder.data(), r.primOrder.size() * 4);
    return uint32_t(r.nodes.size());
}
