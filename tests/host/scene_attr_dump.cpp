// Host harness (compiled and run by tests/test_oracle_pins.py, no GPU
// needed): reads one mesh from a binary file, stores it through the
// engine's scene store (miniraytrace_b200/csrc/host/scene.cpp) without
// normals, computes its tangents when it has uvs, and writes the derived
// normals and tangents (4 floats per vertex each) to a second file.
// Input: u32 vertexCount, u32 indexCount, u32 hasUvs, then positions
// (3 floats per vertex), indices, and uvs (2 floats per vertex) if any.
#include <cstdio>
#include <cstdint>
#include <vector>

#include "scene.h"

using namespace mrt;

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 2;
    uint32_t hdr[3];
    if (std::fread(hdr, 4, 3, in) != 3) return 2;
    std::vector<float> pos(size_t(hdr[0]) * 3), uv(hdr[2] ? size_t(hdr[0]) * 2 : 0);
    std::vector<uint32_t> idx(hdr[1]);
    if (std::fread(pos.data(), 4, pos.size(), in) != pos.size() || std::fread(idx.data(), 4, idx.size(), in) != idx.size())
        return 2;
    if (!uv.empty() && std::fread(uv.data(), 4, uv.size(), in) != uv.size()) return 2;
    std::fclose(in);
    mrtMeshDesc d{};
    d.structSize = sizeof(d);
    d.vertexCount = hdr[0];
    d.indexCount = hdr[1];
    d.positions = pos.data();
    d.uvs = uv.empty() ? nullptr : uv.data();
    d.indices = idx.data();
    Scene s;
    const uint32_t id = s.addMesh(d);
    if (id == MRT_INVALID_ID) return 3;
    MeshData& m = s.meshes()[id];
    if (!uv.empty()) Scene::computeTangents(m);
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    std::fwrite(m.normals.data(), sizeof(V4f), m.normals.size(), out);
    if (!m.tangents.empty()) std::fwrite(m.tangents.data(), sizeof(V4f), m.tangents.size(), out);
    std::fclose(out);
    return 0;
}
