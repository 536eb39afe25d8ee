// Incremental scene store behind the C ABI. Same semantics as the reference
// store (core/include/mrt/Scene.hpp:39-125, core/src/scene/Scene.cpp):
//   - every add deep-copies the caller's arrays; ids are monotone, shared by
//     all object kinds, and 0 is never valid;
//   - meshes get area-weighted normals when none are supplied; tangents
//     (for meshes with UVs) are computed by the engine's commit for meshes
//     an instance draws with a normal-mapped material (computeTangents);
//   - textures live in slots that are recycled after removal, with a
//     generation counter that tells the engine to re-upload a slot;
//   - every mutation sets dirty bits that the engine's commit consumes.
// Vertex data is stored padded to 16 bytes per vertex so a commit can copy
// it to HBM without a repack.
#pragma once

#include <cstdint>
#include <map>
#include <vector>

#include "../../../include/mini_raytrace.h"

namespace mrt {

struct V4f {
    float x, y, z, w;
};
struct V2f {
    float x, y;
};

enum DirtyBits : uint32_t {
    DirtyNone = 0,
    DirtyGeometry = 1u << 0,
    DirtyInstances = 1u << 1,
    DirtyMaterials = 1u << 2,
    DirtyLights = 1u << 3,
    DirtyEnv = 1u << 4,
    DirtyCamera = 1u << 5,
    DirtyTextures = 1u << 6,
    DirtyEnvParams = 1u << 7,
};

struct MeshData {
    std::vector<V4f> positions;  // w = 0
    std::vector<V4f> normals;    // w = 0
    std::vector<V2f> uvs;        // empty when none
    std::vector<V4f> tangents;   // w = handedness; empty until computed (needs uvs)
    std::vector<uint32_t> indices;
    bool blasDirty = true;
    bool tangentsDone = false;     // tangents computed for the current vertex data
    bool tangentsPending = false;  // computed, not yet on the device
};

struct InstanceData {
    uint32_t mesh = 0;
    uint32_t material = 0;
    float o2w[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};  // row-major 3x4
};

struct TextureData {
    uint32_t width = 0, height = 0;
    uint32_t format = 0;  // mrtTextureFormat
    std::vector<uint8_t> data;  // empty = removed slot
    uint32_t generation = 0;
};

struct MaterialData {
    float baseColor[3] = {0.8f, 0.8f, 0.8f};
    float opacity = 1.0f, roughness = 0.5f, metallic = 0.0f, transmission = 0.0f, ior = 1.45f;
    float emission[3] = {0, 0, 0};
    uint32_t tex[5] = {0, 0, 0, 0, 0};  // baseColor, roughness, metallic, normal, emission ids
};

struct LightData {
    uint32_t type = MRT_LIGHT_SUN;
    float direction[3] = {0, 1, 0};
    float position[3] = {0, 0, 0};
    float radiance[3] = {1, 1, 1};
    float angularRadius = 0.00465f;
    float corner[3] = {0, 0, 0}, edge0[3] = {1, 0, 0}, edge1[3] = {0, 0, 1};
    bool twoSided = false;
};

struct CameraData {  // legacy look-at (SceneTypes.hpp:113-118 defaults)
    float position[3] = {0, 0, 5};
    float target[3] = {0, 0, 0};
    float up[3] = {0, 1, 0};
    float fovYDeg = 45.0f;
};

struct CameraExData {  // explicit frustum (SceneTypes.hpp:129-135 defaults)
    uint32_t projection = MRT_CAMERA_PERSPECTIVE;
    float position[3] = {0, 0, 5};
    float forward[3] = {0, 0, -1};
    float up[3] = {0, 1, 0};
    float left = -1, right = 1, bottom = -1, top = 1;
};

class Scene {
public:
    uint32_t addMesh(const mrtMeshDesc& d);
    // Per-vertex tangents from UV gradients (reference Scene.cpp:31-60). The
    // reference computes them whenever a mesh with uvs is stored; they are
    // read only by normal mapping, so here the commit computes them, once per
    // vertex data, for meshes drawn with a normal-mapped material.
    static void computeTangents(MeshData& m);
    void updateMesh(uint32_t id, const mrtMeshDesc& d);
    void removeMesh(uint32_t id);

    uint32_t addInstance(uint32_t mesh, const float* xform3x4, uint32_t material);
    void setInstanceTransform(uint32_t id, const float* xform3x4);
    void removeInstance(uint32_t id);

    uint32_t addMaterial(const mrtMaterialDesc& d);
    void updateMaterial(uint32_t id, const mrtMaterialDesc& d);
    void removeMaterial(uint32_t id);

    uint32_t addTexture(const mrtTextureDesc& d);
    void removeTexture(uint32_t id);
    uint32_t textureSlot(uint32_t id) const;  // ~0u if unknown

    uint32_t addLight(const mrtLightDesc& d);
    void updateLight(uint32_t id, const mrtLightDesc& d);
    void removeLight(uint32_t id);

    void setEnvironment(const mrtTextureDesc& d, float rotation, float intensity);
    void clearEnvironment();
    void setCamera(const mrtCameraDesc& d);
    void setCameraEx(const mrtCameraDescEx& d);

    uint32_t dirty() const { return m_dirty; }
    void clearDirty() { m_dirty = DirtyNone; }
    void markDirty(uint32_t bits) { m_dirty |= bits; }

    std::map<uint32_t, MeshData>& meshes() { return m_meshes; }
    const std::map<uint32_t, InstanceData>& instances() const { return m_instances; }
    const std::map<uint32_t, MaterialData>& materials() const { return m_materials; }
    const std::map<uint32_t, LightData>& lights() const { return m_lights; }
    const std::vector<TextureData>& textures() const { return m_textures; }
    const CameraData& camera() const { return m_camera; }
    const CameraExData& cameraEx() const { return m_cameraEx; }
    bool usesCameraEx() const { return m_useCameraEx; }
    bool hasEnvironment() const { return m_envValid; }
    const TextureData& environment() const { return m_env; }
    float envRotation() const { return m_envRotation; }
    float envIntensity() const { return m_envIntensity; }

private:
    static void copyMesh(const mrtMeshDesc& d, MeshData& out);

    uint32_t m_nextId = 1;
    uint32_t m_dirty = DirtyNone;
    std::map<uint32_t, MeshData> m_meshes;
    std::map<uint32_t, InstanceData> m_instances;
    std::map<uint32_t, MaterialData> m_materials;
    std::map<uint32_t, LightData> m_lights;
    std::vector<TextureData> m_textures;
    std::map<uint32_t, uint32_t> m_textureSlots;
    std::vector<uint32_t> m_freeSlots;
    CameraData m_camera;
    CameraExData m_cameraEx;
    bool m_useCameraEx = false;
    TextureData m_env;
    bool m_envValid = false;
    float m_envRotation = 0.0f;
    float m_envIntensity = 1.0f;
};

}  // namespace mrt
