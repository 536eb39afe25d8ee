// ORACLE -- test infrastructure only. Not part of the product library.
//
// CPU restatement of the reference scene store and of the renderer's packing
// step, producing the same flat arrays the reference shaders read:
//   - mesh deep copy + area-weighted normals + tangents
//     (reference core/src/scene/Scene.cpp:13-92)
//   - material packing with clamps, default material at index 0
//     (core/src/render/Renderer.cpp:510-550)
//   - global geometry repack in BLAS leaf order, nodes rebased, TLAS after the
//     BLAS nodes, instances in TLAS leaf order (Renderer.cpp:333-508)
//   - light packing with the environment at slot 0 (Renderer.cpp:552-603)
//   - environment CDF (Renderer.cpp:605-662)
//   - per-frame globals / camera basis (Renderer.cpp:711-764)
#pragma once

#include <cmath>
#include <cstdint>
#include <map>
#include <vector>

#include "../include/mini_raytrace.h"
#include "oracle_bvh.hpp"

namespace orc {

struct MeshData {
    std::vector<V4<float>> positions, normals, tangents;
    std::vector<V2<float>> uvs;
    std::vector<uint32_t> indices;
};

struct InstanceData {
    uint32_t mesh = 0, material = 0;
    M4<float> objectToWorld = M4<float>::identity();
};

struct TextureData {
    uint32_t w = 0, h = 0;
    int format = 0;  // mrtTextureFormat
    std::vector<uint8_t> data;
};

// Scene.cpp:13-27
inline void computeNormals(MeshData& m) {
    m.normals.assign(m.positions.size(), V4<float>(0, 0, 0, 0));
    for (size_t t = 0; t + 2 < m.indices.size(); t += 3) {
        const V3f p0 = m.positions[m.indices[t]].xyz();
        const V3f p1 = m.positions[m.indices[t + 1]].xyz();
        const V3f p2 = m.positions[m.indices[t + 2]].xyz();
        const V3f n = cross(p1 - p0, p2 - p0);
        for (int k = 0; k < 3; ++k) {
            V4<float>& d = m.normals[m.indices[t + k]];
            d = V4<float>(d.x + n.x, d.y + n.y, d.z + n.z, d.w + 0.0f);
        }
    }
    for (auto& n : m.normals) {
        const V3f v = n.xyz();
        n = V4<float>(length(v) > 1e-12f ? normalize(v) : V3f(0, 1, 0), 0.0f);
    }
}

// Scene.cpp:31-60
inline void computeTangents(MeshData& m) {
    if (m.uvs.empty()) return;
    std::vector<V3f> tan(m.positions.size(), V3f(0.0f)), bit(m.positions.size(), V3f(0.0f));
    for (size_t t = 0; t + 2 < m.indices.size(); t += 3) {
        const uint32_t i0 = m.indices[t], i1 = m.indices[t + 1], i2 = m.indices[t + 2];
        const V3f e1 = m.positions[i1].xyz() - m.positions[i0].xyz();
        const V3f e2 = m.positions[i2].xyz() - m.positions[i0].xyz();
        const V2<float> d1 = m.uvs[i1] - m.uvs[i0];
        const V2<float> d2 = m.uvs[i2] - m.uvs[i0];
        const float det = d1.x * d2.y - d2.x * d1.y;
        if (std::fabs(det) < 1e-12f) continue;
        const float r = 1.0f / det;
        const V3f T = (e1 * d2.y - e2 * d1.y) * r;
        const V3f B = (e2 * d1.x - e1 * d2.x) * r;
        for (uint32_t i : {i0, i1, i2}) {
            tan[i] += T;
            bit[i] += B;
        }
    }
    m.tangents.resize(m.positions.size());
    for (size_t i = 0; i < m.positions.size(); ++i) {
        const V3f n = m.normals[i].xyz();
        V3f t = tan[i] - n * dot(n, tan[i]);
        if (length(t) < 1e-9f)
            t = std::fabs(n.x) < 0.9f ? cross(n, V3f(1, 0, 0)) : cross(n, V3f(0, 1, 0));
        t = normalize(t);
        const float handed = dot(cross(n, t), bit[i]) < 0.0f ? -1.0f : 1.0f;
        m.tangents[i] = V4<float>(t, handed);
    }
}

// Scene.cpp:64-92
inline MeshData copyMesh(const mrtMeshDesc& d) {
    MeshData m;
    m.positions.resize(d.vertexCount);
    for (uint32_t i = 0; i < d.vertexCount; ++i)
        m.positions[i] = V4<float>(d.positions[i * 3], d.positions[i * 3 + 1], d.positions[i * 3 + 2], 0.0f);
    m.indices.assign(d.indices, d.indices + d.indexCount);
    if (d.normals) {
        m.normals.resize(d.vertexCount);
        for (uint32_t i = 0; i < d.vertexCount; ++i)
            m.normals[i] = V4<float>(d.normals[i * 3], d.normals[i * 3 + 1], d.normals[i * 3 + 2], 0.0f);
    } else {
        computeNormals(m);
    }
    if (d.uvs) {
        m.uvs.resize(d.vertexCount);
        for (uint32_t i = 0; i < d.vertexCount; ++i) m.uvs[i] = V2<float>(d.uvs[i * 2], d.uvs[i * 2 + 1]);
        computeTangents(m);
    }
    return m;
}

// MathTypes.hpp:49-56: row-major 3x4 -> column-major 4x4
inline M4<float> fromRows3x4(const float* r) {
    M4<float> m = M4<float>::identity();
    for (int row = 0; row < 3; ++row)
        for (int col = 0; col < 4; ++col) m.m[col][row] = r[row * 4 + col];
    return m;
}

// ---- packed (device-layout) scene -----------------------------------------

struct GpuInstance {  // GpuTypes.hpp:46-52
    M4<float> objectToWorld, worldToObject;
    uint32_t blasRoot, materialIndex;
    uint32_t userId;  // oracle bookkeeping: the instance id
    uint32_t meshId;
};
struct GpuMaterial {  // GpuTypes.hpp:55-61
    V4<float> baseColorOpacity, emissionRoughness, params;
    int32_t tex[5];  // baseColor, roughness, metallic, normal, emission
};
enum { kLightEnv = 0, kLightSun = 1, kLightPoint = 2, kLightRect = 3 };
struct GpuLight {  // GpuTypes.hpp:69-75
    V4<float> p0, p1, p2, p3;
    int32_t type;
};

struct Globals {  // GpuTypes.hpp:33-43
    V3f camPos, camRight, camUp, camForward;
    float fl, fr, fb, ft;  // camFrustum
    uint32_t width, height, maxBounces, lightCount, envW, envH;
    bool hasEnv, ortho;
    float envRotation, envIntensity, envIntegral, exposure, fireflyClamp;
    uint32_t tonemap, tlasRoot;
};

struct Settings {  // SceneTypes.hpp:142-152 defaults
    uint32_t width = 1280, height = 720, maxBounces = 8, sppLimit = 1024;
    float exposureEV = 0.0f, fireflyClamp = 50.0f;
    uint32_t tonemap = 1;
};

struct Packed {
    std::vector<BvhNode> nodes;
    std::vector<uint32_t> tris;  // 4 per triangle: i0, i1, i2, original index
    std::vector<uint32_t> triMesh;  // mesh id per packed triangle
    std::vector<V4<float>> positions, normals, tangents;
    std::vector<V2<float>> uvs;
    std::vector<GpuInstance> instances;
    std::vector<GpuMaterial> materials;
    std::vector<GpuLight> lights;
    std::vector<float> envCdf;
    TextureData env;  // RGBA32F, 1x1 black when absent
    std::vector<TextureData> textures;  // 64 slots; empty = 1x1 white dummy
    uint32_t tlasRoot = 0;
    uint32_t envW = 0, envH = 0;
    float envIntegral = 1.0f;
    bool hasEnv = false;
};

// Renderer.cpp:49-58: inverted box, unreachable leaf
inline BvhNode sentinelNode() {
    BvhNode n{};
    n.lo[0] = n.lo[1] = n.lo[2] = FLT_MAX;
    n.hi[0] = n.hi[1] = n.hi[2] = -FLT_MAX;
    n.leftOrPrim = 0;
    n.packed = 1u << 2;
    return n;
}

// Renderer.cpp:620-655. Layout [conditional h*w][marginal h]; returns the
// float integral (>= 1e-8).
inline float buildEnvCdf(const float* px, uint32_t w, uint32_t h, std::vector<float>& cdf) {
    cdf.assign(size_t(w) * h + h, 0.0f);
    float* cond = cdf.data();
    float* marg = cdf.data() + size_t(w) * h;
    const float pi = 3.14159265358979323846f;
    const float dTheta = pi / h;
    const float dPhi = 2.0f * pi / w;
    double integral = 0.0;
    std::vector<double> rowSums(h, 0.0);
    for (uint32_t y = 0; y < h; ++y) {
        const float sinTheta = std::sin((y + 0.5f) * dTheta);
        double acc = 0.0;
        for (uint32_t x = 0; x < w; ++x) {
            const float* p = px + (size_t(y) * w + x) * 4;
            const float lum = 0.2126f * p[0] + 0.7152f * p[1] + 0.0722f * p[2];
            acc += double(lum) * sinTheta;
            cond[size_t(y) * w + x] = static_cast<float>(acc);
        }
        rowSums[y] = acc;
        integral += acc * dTheta * dPhi;
        const float inv = acc > 0.0 ? float(1.0 / acc) : 0.0f;
        for (uint32_t x = 0; x < w; ++x) cond[size_t(y) * w + x] *= inv;
    }
    double run = 0.0, total = 0.0;
    for (uint32_t y = 0; y < h; ++y) total += rowSums[y];
    for (uint32_t y = 0; y < h; ++y) {
        run += rowSums[y];
        marg[y] = total > 0.0 ? float(run / total) : 0.0f;
    }
    return mmax(static_cast<float>(integral), 1e-8f);
}

struct Scene {
    uint32_t nextId = 1;
    std::map<uint32_t, MeshData> meshes;
    std::map<uint32_t, InstanceData> instances;
    std::map<uint32_t, mrtMaterialDesc> materials;
    std::map<uint32_t, mrtLightDesc> lights;
    std::map<uint32_t, uint32_t> textureSlots;  // id -> slot
    std::vector<TextureData> textures;          // slot-indexed
    std::vector<uint32_t> freeSlots;
    bool hasEnv = false;
    TextureData env;
    float envRotation = 0.0f, envIntensity = 1.0f;
    bool useCameraEx = false;
    mrtCameraDesc cam{sizeof(mrtCameraDesc), {0, 0, 5}, {0, 0, 0}, {0, 1, 0}, 45.0f};
    mrtCameraDescEx camEx{sizeof(mrtCameraDescEx), 0, {0, 0, 5}, {0, 0, -1}, {0, 1, 0}, -1, 1, -1, 1};
    Settings settings;

    uint32_t addMesh(const mrtMeshDesc& d) {  // Scene.cpp:94-100
        if (!d.positions || !d.indices || d.indexCount % 3 != 0) return 0;
        const uint32_t id = nextId++;
        meshes[id] = copyMesh(d);
        return id;
    }
    uint32_t addInstance(uint32_t mesh, const float* xf, uint32_t mat) {  // Scene.cpp:117-126
        if (!meshes.count(mesh)) return 0;
        const uint32_t id = nextId++;
        InstanceData& in = instances[id];
        in.mesh = mesh;
        in.material = mat;
        in.objectToWorld = xf ? fromRows3x4(xf) : M4<float>::identity();
        return id;
    }
    uint32_t addMaterial(const mrtMaterialDesc& d) {
        const uint32_t id = nextId++;
        materials[id] = d;
        return id;
    }
    uint32_t addLight(const mrtLightDesc& d) {
        const uint32_t id = nextId++;
        lights[id] = d;
        return id;
    }
    uint32_t addTexture(const mrtTextureDesc& d) {  // Scene.cpp:159-188
        if (!d.pixels || d.width == 0 || d.height == 0) return 0;
        const uint32_t id = nextId++;
        TextureData t;
        t.w = d.width;
        t.h = d.height;
        t.format = d.format;
        const size_t bytes = size_t(d.width) * d.height * (d.format == MRT_TEX_RGBA32F ? 16 : 4);
        t.data.assign(static_cast<const uint8_t*>(d.pixels), static_cast<const uint8_t*>(d.pixels) + bytes);
        uint32_t slot;
        if (!freeSlots.empty()) {
            slot = freeSlots.back();
            freeSlots.pop_back();
            textures[slot] = std::move(t);
        } else {
            slot = uint32_t(textures.size());
            textures.push_back(std::move(t));
        }
        textureSlots[id] = slot;
        return id;
    }
    void removeTexture(uint32_t id) {
        auto it = textureSlots.find(id);
        if (it == textureSlots.end()) return;
        textures[it->second] = TextureData{};
        freeSlots.push_back(it->second);
        textureSlots.erase(it);
    }
    void setEnvironment(const mrtTextureDesc* d, float rot, float inten) {  // Scene.cpp:230-253
        if (!d) {
            hasEnv = false;
            env = TextureData{};
            return;
        }
        if (!d->pixels || d->format != MRT_TEX_RGBA32F) return;
        env.w = d->width;
        env.h = d->height;
        env.format = MRT_TEX_RGBA32F;
        const size_t bytes = size_t(d->width) * d->height * 16;
        env.data.assign(static_cast<const uint8_t*>(d->pixels), static_cast<const uint8_t*>(d->pixels) + bytes);
        hasEnv = true;
        envRotation = rot;
        envIntensity = inten;
    }
};

inline int32_t texSlotOf(const Scene& s, uint32_t id) {  // Renderer.cpp:514-517
    auto it = s.textureSlots.find(id);
    const uint32_t slot = it == s.textureSlots.end() ? ~0u : it->second;
    return (slot == ~0u || slot >= 64) ? -1 : int32_t(slot);
}

inline Packed pack(const Scene& s) {
    Packed P;
    // -- materials (Renderer.cpp:510-550)
    std::map<uint32_t, uint32_t> matIndex;
    {
        GpuMaterial def{};
        def.baseColorOpacity = V4<float>(0.8f, 0.8f, 0.8f, 1.0f);
        def.emissionRoughness = V4<float>(0, 0, 0, 0.5f);
        def.params = V4<float>(0, 0, 1.45f, 0);
        for (int i = 0; i < 5; ++i) def.tex[i] = -1;
        P.materials.push_back(def);
        for (auto& [id, m] : s.materials) {
            GpuMaterial g{};
            g.baseColorOpacity = V4<float>(m.baseColor[0], m.baseColor[1], m.baseColor[2], m.opacity);
            g.emissionRoughness =
                V4<float>(m.emission[0], m.emission[1], m.emission[2], clampv(m.roughness, 0.0f, 1.0f));
            g.params = V4<float>(clampv(m.metallic, 0.0f, 1.0f), clampv(m.transmission, 0.0f, 1.0f),
                                 mmax(m.ior, 1.0f), 0.0f);
            g.tex[0] = texSlotOf(s, m.baseColorTex);
            g.tex[1] = texSlotOf(s, m.roughnessTex);
            g.tex[2] = texSlotOf(s, m.metallicTex);
            g.tex[3] = texSlotOf(s, m.normalTex);
            g.tex[4] = texSlotOf(s, m.emissionTex);
            matIndex[id] = uint32_t(P.materials.size());
            P.materials.push_back(g);
        }
    }
    // -- geometry (Renderer.cpp:333-446)
    struct Blas {
        BvhBuild bvh;
        uint32_t root = 0;
    };
    std::map<uint32_t, Blas> blas;
    for (auto& [id, m] : s.meshes) {
        const size_t nt = m.indices.size() / 3;
        std::vector<Aabb> bounds(nt);
        for (size_t t = 0; t < nt; ++t) {
            Aabb b;
            b.expand(m.positions[m.indices[t * 3 + 0]].xyz());
            b.expand(m.positions[m.indices[t * 3 + 1]].xyz());
            b.expand(m.positions[m.indices[t * 3 + 2]].xyz());
            bounds[t] = b;
        }
        blas[id].bvh = buildBvh(bounds, 4);
    }
    for (auto& [id, m] : s.meshes) {
        Blas& b = blas[id];
        const uint32_t vbase = uint32_t(P.positions.size());
        const uint32_t tbase = uint32_t(P.tris.size() / 4);
        const uint32_t nbase = uint32_t(P.nodes.size());
        b.root = nbase;
        P.positions.insert(P.positions.end(), m.positions.begin(), m.positions.end());
        P.normals.insert(P.normals.end(), m.normals.begin(), m.normals.end());
        if (m.uvs.empty()) P.uvs.insert(P.uvs.end(), m.positions.size(), V2<float>(0, 0));
        else P.uvs.insert(P.uvs.end(), m.uvs.begin(), m.uvs.end());
        if (m.tangents.empty()) P.tangents.insert(P.tangents.end(), m.positions.size(), V4<float>(1, 0, 0, 1));
        else P.tangents.insert(P.tangents.end(), m.tangents.begin(), m.tangents.end());
        for (uint32_t lt : b.bvh.primOrder) {
            P.tris.push_back(m.indices[lt * 3 + 0] + vbase);
            P.tris.push_back(m.indices[lt * 3 + 1] + vbase);
            P.tris.push_back(m.indices[lt * 3 + 2] + vbase);
            P.tris.push_back(lt);
            P.triMesh.push_back(id);
        }
        for (BvhNode n : b.bvh.nodes) {
            const uint32_t cnt = n.packed >> 2;
            n.leftOrPrim += (cnt == 0) ? nbase : tbase;
            P.nodes.push_back(n);
        }
    }
    // -- instances / TLAS (Renderer.cpp:448-508)
    P.tlasRoot = uint32_t(P.nodes.size());
    {
        std::vector<std::pair<uint32_t, const InstanceData*>> flat;
        std::vector<Aabb> bounds;
        for (auto& [id, in] : s.instances) {
            auto it = blas.find(in.mesh);
            if (it == blas.end() || !it->second.bvh.rootBounds.valid()) continue;
            flat.push_back({id, &in});
            bounds.push_back(it->second.bvh.rootBounds.transformed(in.objectToWorld));
        }
        BvhBuild tlas = buildBvh(bounds, 1);
        if (tlas.nodes.empty()) tlas.nodes.push_back(sentinelNode());
        for (uint32_t oi : tlas.primOrder) {
            const InstanceData* in = flat[oi].second;
            GpuInstance g{};
            g.objectToWorld = in->objectToWorld;
            g.worldToObject = inverse(in->objectToWorld);
            g.blasRoot = blas[in->mesh].root;
            auto mi = matIndex.find(in->material);
            g.materialIndex = mi != matIndex.end() ? mi->second : 0;
            g.userId = flat[oi].first;
            g.meshId = in->mesh;
            P.instances.push_back(g);
        }
        for (BvhNode& n : tlas.nodes)
            if ((n.packed >> 2) == 0) n.leftOrPrim += P.tlasRoot;
        P.nodes.insert(P.nodes.end(), tlas.nodes.begin(), tlas.nodes.end());
    }
    // -- lights (Renderer.cpp:552-603)
    if (s.hasEnv) {
        GpuLight g{};
        g.type = kLightEnv;
        P.lights.push_back(g);
    }
    for (auto& [id, l] : s.lights) {
        GpuLight g{};
        if (l.type == MRT_LIGHT_SUN) {
            g.type = kLightSun;
            const V3f d = normalize(V3f(l.direction[0], l.direction[1], l.direction[2]));
            g.p0 = V4<float>(d, std::cos(mmax(l.angularRadius, 1e-4f)));
            g.p1 = V4<float>(l.radiance[0], l.radiance[1], l.radiance[2], 0);
        } else if (l.type == MRT_LIGHT_POINT) {
            g.type = kLightPoint;
            g.p0 = V4<float>(l.position[0], l.position[1], l.position[2], 0);
            g.p1 = V4<float>(l.radiance[0], l.radiance[1], l.radiance[2], 0);
        } else {
            g.type = kLightRect;
            const V3f e0(l.edge0[0], l.edge0[1], l.edge0[2]);
            const V3f e1(l.edge1[0], l.edge1[1], l.edge1[2]);
            const float area = length(cross(e0, e1));
            g.p0 = V4<float>(l.corner[0], l.corner[1], l.corner[2], area);
            g.p1 = V4<float>(e0, 0);
            g.p2 = V4<float>(e1, 0);
            g.p3 = V4<float>(l.radiance[0], l.radiance[1], l.radiance[2], l.twoSided ? 1.0f : 0.0f);
        }
        P.lights.push_back(g);
    }
    // -- environment (Renderer.cpp:605-662)
    P.hasEnv = s.hasEnv;
    if (s.hasEnv) {
        P.env = s.env;
        P.envW = s.env.w;
        P.envH = s.env.h;
        P.envIntegral =
            buildEnvCdf(reinterpret_cast<const float*>(s.env.data.data()), s.env.w, s.env.h, P.envCdf);
    } else {
        P.env.w = P.env.h = 1;
        P.env.format = MRT_TEX_RGBA32F;
        const float black[4] = {0, 0, 0, 1};
        P.env.data.assign(reinterpret_cast<const uint8_t*>(black), reinterpret_cast<const uint8_t*>(black) + 16);
    }
    P.textures.resize(64);
    for (size_t i = 0; i < s.textures.size() && i < 64; ++i) P.textures[i] = s.textures[i];
    return P;
}

// Renderer.cpp:711-764
inline Globals makeGlobals(const Scene& s, const Packed& P) {
    Globals g{};
    V3f pos, fwd, upHint;
    float l, r, b, t;
    bool ortho = false;
    if (s.useCameraEx) {
        const mrtCameraDescEx& c = s.camEx;
        pos = V3f(c.position[0], c.position[1], c.position[2]);
        fwd = normalize(V3f(c.forward[0], c.forward[1], c.forward[2]));
        upHint = V3f(c.up[0], c.up[1], c.up[2]);
        l = c.left; r = c.right; b = c.bottom; t = c.top;
        ortho = c.projection == MRT_CAMERA_ORTHOGRAPHIC;
    } else {
        const mrtCameraDesc& c = s.cam;
        pos = V3f(c.position[0], c.position[1], c.position[2]);
        const V3f target(c.target[0], c.target[1], c.target[2]);
        fwd = normalize(target - pos);
        upHint = V3f(c.up[0], c.up[1], c.up[2]);
        const float aspect = float(s.settings.width) / float(s.settings.height);
        const float radians = c.fovYDeg * 0.01745329251994329576923690768489f;  // degrees -> radians
        const float tanHalf = std::tan(radians * 0.5f);
        r = tanHalf * aspect;
        l = -r;
        t = tanHalf;
        b = -t;
    }
    V3f right = cross(fwd, upHint);
    right = (length(right) < 1e-6f) ? V3f(1, 0, 0) : normalize(right);
    const V3f up = cross(right, fwd);
    g.camPos = pos; g.camRight = right; g.camUp = up; g.camForward = fwd;
    g.fl = l; g.fr = r; g.fb = b; g.ft = t;
    g.width = s.settings.width;
    g.height = s.settings.height;
    g.maxBounces = std::min<uint32_t>(s.settings.maxBounces, 16u);
    g.lightCount = uint32_t(P.lights.size());
    g.envW = P.envW;
    g.envH = P.envH;
    g.hasEnv = P.hasEnv;
    g.ortho = ortho;
    g.envRotation = s.envRotation;
    g.envIntensity = s.envIntensity;
    g.envIntegral = P.envIntegral;
    g.exposure = std::exp2(s.settings.exposureEV);
    g.fireflyClamp = s.settings.fireflyClamp;
    g.tonemap = s.settings.tonemap;
    g.tlasRoot = P.tlasRoot;
    return g;
}

}  // namespace orc
