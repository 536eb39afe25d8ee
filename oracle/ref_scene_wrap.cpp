// ORACLE -- test infrastructure only.
//
// extern "C" wrapper around the reference's own scene store
// (core/src/scene/Scene.cpp, compiled from the reference checkout by
// oracle/build_oracle.py into oracle/_ref/). It adds one mesh through
// mrt::Scene::addMesh (Scene.hpp:51) and returns the attributes the
// reference derives for it: area-weighted vertex normals when none are
// given and UV-gradient tangents when uvs are given (Scene.cpp:13-60), so
// tests can compare the oracle's restatement and the engine with them.
#include <cstring>

#include "mrt/Scene.hpp"

extern "C" int ref_mesh_attributes(const float* positions, uint32_t vertexCount, const uint32_t* indices,
                                   uint32_t indexCount, const float* uvs, float* normalsOut, float* tangentsOut) {
    mrt::Scene scene;
    mrt::MeshDesc d;
    d.vertexCount = vertexCount;
    d.indexCount = indexCount;
    d.positions = positions;
    d.normals = nullptr;
    d.uvs = uvs;
    d.indices = indices;
    const mrt::MeshId id = scene.addMesh(d);
    if (id == mrt::kInvalidId) return -1;
    const mrt::MeshData& m = scene.meshes().at(id);
    std::memcpy(normalsOut, m.normals.data(), m.normals.size() * sizeof(mrt::vec4));
    if (tangentsOut && !m.tangents.empty()) std::memcpy(tangentsOut, m.tangents.data(), m.tangents.size() * sizeof(mrt::vec4));
    return int(m.tangents.size());
}
