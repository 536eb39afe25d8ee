// Scene store implementation (semantics: reference core/src/scene/Scene.cpp).
#include "scene.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace mrt {

namespace {

// fn(begin, end) over [0, n): on up to 8 threads when n is large (the work
// items are independent), else on the calling thread.
template <class Fn>
void parallelRanges(size_t n, Fn&& fn) {
    const size_t kMinPerThread = size_t(1) << 18;
    const size_t threads = std::min<size_t>({8, std::max(1u, std::thread::hardware_concurrency()),
                                             (n + kMinPerThread - 1) / kMinPerThread});
    if (threads <= 1) {
        fn(size_t(0), n);
        return;
    }
    std::vector<std::thread> pool;
    const size_t step = (n + threads - 1) / threads;
    for (size_t t = 1; t < threads; ++t)
        pool.emplace_back([&, t] { fn(std::min(n, t * step), std::min(n, (t + 1) * step)); });
    fn(size_t(0), std::min(n, step));
    for (auto& th : pool) th.join();
}

inline void sub3(const V4f& a, const V4f& b, float r[3]) {
    r[0] = a.x - b.x;
    r[1] = a.y - b.y;
    r[2] = a.z - b.z;
}
inline void cross3(const float a[3], const float b[3], float r[3]) {
    r[0] = a[1] * b[2] - b[1] * a[2];
    r[1] = a[2] * b[0] - b[2] * a[0];
    r[2] = a[0] * b[1] - b[0] * a[1];
}
inline float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Area-weighted vertex normals: the un-normalised face normal (length =
// twice the area) is summed into each corner (reference Scene.cpp:13-27).
void computeNormals(MeshData& m) {
    m.normals.assign(m.positions.size(), V4f{0, 0, 0, 0});
    for (size_t t = 0; t + 2 < m.indices.size(); t += 3) {
        const uint32_t i0 = m.indices[t], i1 = m.indices[t + 1], i2 = m.indices[t + 2];
        float e1[3], e2[3], n[3];
        sub3(m.positions[i1], m.positions[i0], e1);
        sub3(m.positions[i2], m.positions[i0], e2);
        cross3(e1, e2, n);
        for (uint32_t i : {i0, i1, i2}) {
            m.normals[i].x += n[0];
            m.normals[i].y += n[1];
            m.normals[i].z += n[2];
        }
    }
    for (V4f& n : m.normals) {
        const float v[3] = {n.x, n.y, n.z};
        const float len = std::sqrt(dot3(v, v));
        if (len > 1e-12f) {
            const float inv = 1.0f / std::sqrt(dot3(v, v));
            n = V4f{v[0] * inv, v[1] * inv, v[2] * inv, 0.0f};
        } else {
            n = V4f{0, 1, 0, 0};
        }
    }
}

}  // namespace

// Per-vertex tangents from UV gradients, Gram-Schmidt against the normal,
// handedness in w (reference Scene.cpp:31-60).
void Scene::computeTangents(MeshData& m) {
    if (m.uvs.empty()) return;
    const size_t nv = m.positions.size();
    std::vector<float> tan(nv * 3, 0.0f), bit(nv * 3, 0.0f);
    for (size_t t = 0; t + 2 < m.indices.size(); t += 3) {
        const uint32_t i0 = m.indices[t], i1 = m.indices[t + 1], i2 = m.indices[t + 2];
        float e1[3], e2[3];
        sub3(m.positions[i1], m.positions[i0], e1);
        sub3(m.positions[i2], m.positions[i0], e2);
        const float d1x = m.uvs[i1].x - m.uvs[i0].x, d1y = m.uvs[i1].y - m.uvs[i0].y;
        const float d2x = m.uvs[i2].x - m.uvs[i0].x, d2y = m.uvs[i2].y - m.uvs[i0].y;
        const float det = d1x * d2y - d2x * d1y;
        if (std::fabs(det) < 1e-12f) continue;
        const float r = 1.0f / det;
        float T[3], B[3];
        for (int k = 0; k < 3; ++k) {
            T[k] = (e1[k] * d2y - e2[k] * d1y) * r;
            B[k] = (e2[k] * d1x - e1[k] * d2x) * r;
        }
        for (uint32_t i : {i0, i1, i2})
            for (int k = 0; k < 3; ++k) {
                tan[i * 3 + k] += T[k];
                bit[i * 3 + k] += B[k];
            }
    }
    m.tangents.resize(nv);
    for (size_t i = 0; i < nv; ++i) {
        const float n[3] = {m.normals[i].x, m.normals[i].y, m.normals[i].z};
        const float* ti = &tan[i * 3];
        const float nd = dot3(n, ti);
        float t[3] = {ti[0] - n[0] * nd, ti[1] - n[1] * nd, ti[2] - n[2] * nd};
        if (std::sqrt(dot3(t, t)) < 1e-9f) {
            const float ax[3] = {1, 0, 0}, ay[3] = {0, 1, 0};
            cross3(n, std::fabs(n[0]) < 0.9f ? ax : ay, t);
        }
        const float inv = 1.0f / std::sqrt(dot3(t, t));
        t[0] *= inv;
        t[1] *= inv;
        t[2] *= inv;
        float nt[3];
        cross3(n, t, nt);
        const float handed = dot3(nt, &bit[i * 3]) < 0.0f ? -1.0f : 1.0f;
        m.tangents[i] = V4f{t[0], t[1], t[2], handed};
    }
}

namespace {

void rowsToXf(const float* r, float out[12]) { std::memcpy(out, r, 12 * sizeof(float)); }

MaterialData toMaterial(const mrtMaterialDesc& d) {
    MaterialData m;
    std::memcpy(m.baseColor, d.baseColor, sizeof(m.baseColor));
    m.opacity = d.opacity;
    m.roughness = d.roughness;
    m.metallic = d.metallic;
    m.transmission = d.transmission;
    m.ior = d.ior;
    std::memcpy(m.emission, d.emission, sizeof(m.emission));
    m.tex[0] = d.baseColorTex;
    m.tex[1] = d.roughnessTex;
    m.tex[2] = d.metallicTex;
    m.tex[3] = d.normalTex;
    m.tex[4] = d.emissionTex;
    return m;
}

LightData toLight(const mrtLightDesc& d) {
    LightData l;
    l.type = d.type;
    std::memcpy(l.direction, d.direction, sizeof(l.direction));
    std::memcpy(l.position, d.position, sizeof(l.position));
    std::memcpy(l.radiance, d.radiance, sizeof(l.radiance));
    l.angularRadius = d.angularRadius;
    std::memcpy(l.corner, d.corner, sizeof(l.corner));
    std::memcpy(l.edge0, d.edge0, sizeof(l.edge0));
    std::memcpy(l.edge1, d.edge1, sizeof(l.edge1));
    l.twoSided = d.twoSided != 0;
    return l;
}

}  // namespace

void Scene::copyMesh(const mrtMeshDesc& d, MeshData& out) {
    const size_t nv = d.vertexCount;
    out.positions.resize(nv);
    out.indices.resize(d.indexCount);
    if (d.normals) out.normals.resize(nv);
    if (d.uvs) out.uvs.resize(nv);
    else out.uvs.clear();
    // element-wise copies: independent of the order, split over threads
    parallelRanges(nv, [&](size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) {
            out.positions[i] = V4f{d.positions[i * 3], d.positions[i * 3 + 1], d.positions[i * 3 + 2], 0.0f};
            if (d.normals) out.normals[i] = V4f{d.normals[i * 3], d.normals[i * 3 + 1], d.normals[i * 3 + 2], 0.0f};
            if (d.uvs) out.uvs[i] = V2f{d.uvs[i * 2], d.uvs[i * 2 + 1]};
        }
    });
    parallelRanges(d.indexCount, [&](size_t b, size_t e) {
        std::memcpy(out.indices.data() + b, d.indices + b, (e - b) * sizeof(uint32_t));
    });
    if (!d.normals) computeNormals(out);  // ordered sums: sequential
    out.tangents.clear();  // computed at commit when a normal map needs them
    out.tangentsDone = false;
    out.tangentsPending = false;
    out.blasDirty = true;
}

namespace {
// A descriptor the store can hold: positions and indices present, whole
// triangles, every index inside the vertex array. The reference does not
// check the last condition (an out-of-range index reads outside the vertex
// buffer there); here such a mesh is rejected instead.
bool meshDescUsable(const mrtMeshDesc& d) {
    if (!d.positions || !d.indices || d.indexCount % 3 != 0) return false;
    std::atomic<bool> ok{true};
    parallelRanges(d.indexCount, [&](size_t b, size_t e) {
        uint32_t mx = 0;
        for (size_t i = b; i < e; ++i) mx = std::max(mx, d.indices[i]);
        if (e > b && mx >= d.vertexCount) ok = false;
    });
    return ok;
}
}  // namespace

uint32_t Scene::addMesh(const mrtMeshDesc& d) {
    if (!meshDescUsable(d)) return MRT_INVALID_ID;
    const uint32_t id = m_nextId++;
    copyMesh(d, m_meshes[id]);
    markDirty(DirtyGeometry);
    return id;
}

void Scene::updateMesh(uint32_t id, const mrtMeshDesc& d) {
    auto it = m_meshes.find(id);
    if (it == m_meshes.end()) return;
    // A descriptor that could not be added is ignored, so the store never
    // holds a mesh the packer cannot read.
    if (!meshDescUsable(d)) return;
    copyMesh(d, it->second);
    markDirty(DirtyGeometry);
}

void Scene::removeMesh(uint32_t id) {
    if (m_meshes.erase(id) == 0) return;
    for (auto it = m_instances.begin(); it != m_instances.end();)
        it = (it->second.mesh == id) ? m_instances.erase(it) : std::next(it);
    markDirty(DirtyGeometry | DirtyInstances);
}

uint32_t Scene::addInstance(uint32_t mesh, const float* xform3x4, uint32_t material) {
    if (!m_meshes.count(mesh)) return MRT_INVALID_ID;
    const uint32_t id = m_nextId++;
    InstanceData& in = m_instances[id];
    in.mesh = mesh;
    in.material = material;
    if (xform3x4) rowsToXf(xform3x4, in.o2w);
    markDirty(DirtyInstances);
    return id;
}

void Scene::setInstanceTransform(uint32_t id, const float* xform3x4) {
    auto it = m_instances.find(id);
    if (it == m_instances.end() || !xform3x4) return;
    rowsToXf(xform3x4, it->second.o2w);
    markDirty(DirtyInstances);
}

void Scene::removeInstance(uint32_t id) {
    if (m_instances.erase(id)) markDirty(DirtyInstances);
}

uint32_t Scene::addMaterial(const mrtMaterialDesc& d) {
    const uint32_t id = m_nextId++;
    m_materials[id] = toMaterial(d);
    markDirty(DirtyMaterials);
    return id;
}

void Scene::updateMaterial(uint32_t id, const mrtMaterialDesc& d) {
    auto it = m_materials.find(id);
    if (it == m_materials.end()) return;
    it->second = toMaterial(d);
    markDirty(DirtyMaterials);
}

void Scene::removeMaterial(uint32_t id) {
    if (m_materials.erase(id)) markDirty(DirtyMaterials | DirtyInstances);
}

uint32_t Scene::addTexture(const mrtTextureDesc& d) {
    if (!d.pixels || d.width == 0 || d.height == 0) return MRT_INVALID_ID;
    if (d.format > MRT_TEX_RGBA32F) return MRT_INVALID_ID;
    const uint32_t id = m_nextId++;
    TextureData t;
    t.width = d.width;
    t.height = d.height;
    t.format = d.format;
    const size_t bytes = size_t(d.width) * d.height * (d.format == MRT_TEX_RGBA32F ? 16 : 4);
    t.data.assign(static_cast<const uint8_t*>(d.pixels), static_cast<const uint8_t*>(d.pixels) + bytes);
    uint32_t slot;
    if (!m_freeSlots.empty()) {  // recycle (reference Scene.cpp:170-183)
        slot = m_freeSlots.back();
        m_freeSlots.pop_back();
        t.generation = m_textures[slot].generation + 1;
        m_textures[slot] = std::move(t);
    } else {
        slot = uint32_t(m_textures.size());
        t.generation = 1;
        m_textures.push_back(std::move(t));
    }
    m_textureSlots[id] = slot;
    markDirty(DirtyTextures);
    return id;
}

void Scene::removeTexture(uint32_t id) {
    auto it = m_textureSlots.find(id);
    if (it == m_textureSlots.end()) return;
    TextureData& t = m_textures[it->second];
    t.width = t.height = 0;
    t.data.clear();
    t.data.shrink_to_fit();
    ++t.generation;
    m_freeSlots.push_back(it->second);
    m_textureSlots.erase(it);
    markDirty(DirtyTextures);
}

uint32_t Scene::textureSlot(uint32_t id) const {
    auto it = m_textureSlots.find(id);
    return it != m_textureSlots.end() ? it->second : ~0u;
}

uint32_t Scene::addLight(const mrtLightDesc& d) {
    const uint32_t id = m_nextId++;
    m_lights[id] = toLight(d);
    markDirty(DirtyLights);
    return id;
}

void Scene::updateLight(uint32_t id, const mrtLightDesc& d) {
    auto it = m_lights.find(id);
    if (it == m_lights.end()) return;
    it->second = toLight(d);
    markDirty(DirtyLights);
}

void Scene::removeLight(uint32_t id) {
    if (m_lights.erase(id)) markDirty(DirtyLights);
}

void Scene::setEnvironment(const mrtTextureDesc& d, float rotation, float intensity) {
    if (!d.pixels || d.format != MRT_TEX_RGBA32F || d.width == 0 || d.height == 0) return;
    m_env.width = d.width;
    m_env.height = d.height;
    m_env.format = MRT_TEX_RGBA32F;
    const size_t bytes = size_t(d.width) * d.height * 16;
    m_env.data.resize(bytes);
    const uint8_t* src = static_cast<const uint8_t*>(d.pixels);
    parallelRanges(bytes / 16, [&](size_t b, size_t e) { std::memcpy(m_env.data.data() + 16 * b, src + 16 * b, 16 * (e - b)); });
    m_envValid = true;
    m_envRotation = rotation;
    m_envIntensity = intensity;
    markDirty(DirtyEnv | DirtyLights);
}

void Scene::clearEnvironment() {
    m_envValid = false;
    m_env.data.clear();
    markDirty(DirtyEnv | DirtyLights);
}

void Scene::setCamera(const mrtCameraDesc& d) {
    std::memcpy(m_camera.position, d.position, sizeof(m_camera.position));
    std::memcpy(m_camera.target, d.target, sizeof(m_camera.target));
    std::memcpy(m_camera.up, d.up, sizeof(m_camera.up));
    m_camera.fovYDeg = d.fovYDeg;
    m_useCameraEx = false;
    markDirty(DirtyCamera);
}

void Scene::setCameraEx(const mrtCameraDescEx& d) {
    m_cameraEx.projection = uint32_t(d.projection);
    std::memcpy(m_cameraEx.position, d.position, sizeof(m_cameraEx.position));
    std::memcpy(m_cameraEx.forward, d.forward, sizeof(m_cameraEx.forward));
    std::memcpy(m_cameraEx.up, d.up, sizeof(m_cameraEx.up));
    m_cameraEx.left = d.left;
    m_cameraEx.right = d.right;
    m_cameraEx.bottom = d.bottom;
    m_cameraEx.top = d.top;
    m_useCameraEx = true;
    markDirty(DirtyCamera);
}

}  // namespace mrt
