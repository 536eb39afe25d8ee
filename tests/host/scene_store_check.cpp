// Host-side checks of the scene store (compiled and run by
// tests/test_host_cpu.py, no GPU needed): a mesh large enough for the
// threaded copy and index check is stored element for element; an index
// past the vertex count anywhere in the array rejects the mesh; tangents are
// not computed when the mesh is stored, and computing them twice gives the
// same bits.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "scene.h"

using namespace mrt;

static int failures = 0;
#define CHECK(c)                                                   \
    do {                                                           \
        if (!(c)) {                                                \
            std::printf("FAILED line %d: %s\n", __LINE__, #c);     \
            ++failures;                                            \
        }                                                          \
    } while (0)

int main() {
    const uint32_t G = 1200;  // 1.44 M vertices, 2.87 M triangles: several threads' ranges
    std::vector<float> pos, nrm, uv;
    std::vector<uint32_t> idx;
    for (uint32_t y = 0; y < G; ++y)
        for (uint32_t x = 0; x < G; ++x) {
            const float h = 0.05f * std::sin(0.013f * x) * std::cos(0.017f * y);
            pos.insert(pos.end(), {x / float(G), h, y / float(G)});
            nrm.insert(nrm.end(), {0.1f * std::sin(0.01f * x), 1.0f, 0.0f});
            uv.insert(uv.end(), {x / float(G - 1), 1.0f - y / float(G - 1)});
        }
    for (uint32_t y = 0; y + 1 < G; ++y)
        for (uint32_t x = 0; x + 1 < G; ++x) {
            const uint32_t a = y * G + x, b = a + 1, c = a + G, d = c + 1;
            idx.insert(idx.end(), {a, c, b, b, c, d});
        }
    mrtMeshDesc desc{};
    desc.structSize = sizeof(mrtMeshDesc);
    desc.vertexCount = G * G;
    desc.indexCount = uint32_t(idx.size());
    desc.positions = pos.data();
    desc.normals = nrm.data();
    desc.uvs = uv.data();
    desc.indices = idx.data();

    Scene s;
    const uint32_t id = s.addMesh(desc);
    CHECK(id != MRT_INVALID_ID);
    MeshData& m = s.meshes()[id];
    CHECK(m.positions.size() == desc.vertexCount && m.indices.size() == idx.size());
    bool same = true;
    for (uint32_t i = 0; i < desc.vertexCount && same; ++i) {
        same = m.positions[i].x == pos[3 * i] && m.positions[i].y == pos[3 * i + 1] &&
               m.positions[i].z == pos[3 * i + 2] && m.positions[i].w == 0.0f && m.normals[i].x == nrm[3 * i] &&
               m.normals[i].y == nrm[3 * i + 1] && m.normals[i].z == nrm[3 * i + 2] && m.uvs[i].x == uv[2 * i] &&
               m.uvs[i].y == uv[2 * i + 1];
    }
    CHECK(same);
    CHECK(std::memcmp(m.indices.data(), idx.data(), idx.size() * 4) == 0);
    CHECK(m.tangents.empty() && !m.tangentsDone);

    // tangents on request, deterministic
    Scene::computeTangents(m);
    CHECK(m.tangents.size() == desc.vertexCount);
    const std::vector<V4f> t1 = m.tangents;
    Scene::computeTangents(m);
    CHECK(std::memcmp(t1.data(), m.tangents.data(), t1.size() * sizeof(V4f)) == 0);
    bool unit = true;
    for (const V4f& t : t1) unit &= std::fabs(t.x * t.x + t.y * t.y + t.z * t.z - 1.0f) < 1e-4f && std::fabs(t.w) == 1.0f;
    CHECK(unit);

    // an out-of-range index in the first, a middle or the last range is rejected
    for (size_t at : {size_t(0), idx.size() / 2 + 1, idx.size() - 1}) {
        std::vector<uint32_t> bad = idx;
        bad[at] = desc.vertexCount;
        mrtMeshDesc b = desc;
        b.indices = bad.data();
        CHECK(s.addMesh(b) == MRT_INVALID_ID);
        s.updateMesh(id, b);  // ignored: the stored mesh stays as it was
        CHECK(std::memcmp(s.meshes()[id].indices.data(), idx.data(), idx.size() * 4) == 0);
    }
    // an update replaces the data and drops computed tangents
    std::vector<float> pos2 = pos;
    for (size_t i = 1; i < pos2.size(); i += 3) pos2[i] += 0.25f;
    mrtMeshDesc d2 = desc;
    d2.positions = pos2.data();
    s.updateMesh(id, d2);
    CHECK(s.meshes()[id].positions[desc.vertexCount - 1].y == pos2[3 * (desc.vertexCount - 1) + 1]);
    CHECK(s.meshes()[id].tangents.empty() && !s.meshes()[id].tangentsDone);

    if (failures == 0) std::printf("ok\n");
    return failures == 0 ? 0 : 1;
}
