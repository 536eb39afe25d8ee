/*
 * mini_raytrace.h -- the C ABI of the B200 progressive path tracer.
 *
 * This header is the drop-in boundary: every type, enum value, struct layout
 * and function below is binary compatible with the MiniRaytrace C ABI
 * (reference: capi/include/mini_raytrace.h:1-242), so an existing caller
 * (the Rhino P/Invoke layer, a C/C++ host) links against libmrt.so from this
 * project without a change.
 *
 * Contract (unchanged from the reference):
 *   - opaque engine handle, result codes; no C++ exception crosses the ABI
 *     (reference capi/src/capi.cpp:116-120);
 *   - every pointer argument is borrowed for the call and deep-copied
 *     (reference Scene.cpp:64-92, 159-188, 230-240);
 *   - calls come from one thread at a time;
 *   - every descriptor starts with `structSize`; a struct smaller than the
 *     version compiled here is rejected (reference capi.cpp:23-24). New
 *     options therefore arrive as new functions (see mrt_ext.h), never as new
 *     struct fields.
 *
 * Differences in the implementation behind the ABI (not in the ABI):
 *   - the device is a CUDA GPU (sm_100a) instead of a Vulkan device; device
 *     initialisation failures still return MRT_ERROR_VULKAN_INIT (value 2),
 *     with a CUDA-specific message in mrtGetLastErrorMessage();
 *   - gpuIndex1 counts CUDA devices (cudaGetDeviceCount order).
 */
#ifndef MINI_RAYTRACE_H
#define MINI_RAYTRACE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define MRT_API __declspec(dllexport)
#else
#define MRT_API __attribute__((visibility("default")))
#endif

typedef struct mrtEngine mrtEngine;

/* reference mini_raytrace.h:28-37 */
typedef enum mrtResult {
    MRT_SUCCESS = 0,
    MRT_ERROR_UNKNOWN = 1,
    MRT_ERROR_VULKAN_INIT = 2, /* device initialisation failed (CUDA here) */
    MRT_ERROR_OUT_OF_MEMORY = 3,
    MRT_ERROR_INVALID_ARGUMENT = 4,
    MRT_ERROR_INVALID_HANDLE = 5,
    MRT_ERROR_SHADER_LOAD = 6, /* kernel image missing for this GPU */
    MRT_ERROR_DEVICE_LOST = 7, /* sticky CUDA error; engine must be destroyed */
} mrtResult;

typedef uint32_t mrtMeshId;
typedef uint32_t mrtInstanceId;
typedef uint32_t mrtMaterialId;
typedef uint32_t mrtTextureId;
typedef uint32_t mrtLightId;
#define MRT_INVALID_ID 0u

/* Readback formats (reference mini_raytrace.h:46-52). Row-major, row 0 is the
 * top of the image, alpha is always exactly 1.0. */
typedef enum mrtPixelFormat {
    MRT_PIXEL_RGBA8_SRGB = 0,     /* exposure + tonemap + sRGB, 4 B/pixel */
    MRT_PIXEL_RGBA32F_LINEAR = 1, /* mean radiance, 16 B/pixel           */
} mrtPixelFormat;

/* reference mini_raytrace.h:54-58 */
typedef enum mrtTextureFormat {
    MRT_TEX_RGBA8_SRGB = 0,
    MRT_TEX_RGBA8_UNORM = 1,
    MRT_TEX_RGBA32F = 2,
} mrtTextureFormat;

/* reference mini_raytrace.h:60-64 */
typedef enum mrtLightType {
    MRT_LIGHT_SUN = 0,
    MRT_LIGHT_POINT = 1,
    MRT_LIGHT_RECT = 2,
} mrtLightType;

/* reference mini_raytrace.h:66-69 */
typedef enum mrtTonemap {
    MRT_TONEMAP_LINEAR = 0,
    MRT_TONEMAP_ACES = 1,
} mrtTonemap;

/* reference mini_raytrace.h:73-83. gpuIndex1: 0 = automatic choice, N > 0 =
 * CUDA device N-1; an index past the device count fails with
 * MRT_ERROR_VULKAN_INIT and a message containing "out of range". */
typedef struct mrtEngineDesc {
    size_t structSize;
    int32_t enableValidation; /* enables extra device-side bounds checks */
    uint32_t width, height;   /* 0 keeps the default 1280 x 720 */
    uint32_t gpuIndex1;
} mrtEngineDesc;

/* reference mini_raytrace.h:85-93 */
typedef struct mrtMeshDesc {
    size_t structSize;
    uint32_t vertexCount;
    uint32_t indexCount;     /* multiple of 3 */
    const float* positions;  /* xyz per vertex (required) */
    const float* normals;    /* xyz per vertex (optional: area-weighted if NULL) */
    const float* uvs;        /* uv per vertex (optional) */
    const uint32_t* indices; /* required */
} mrtMeshDesc;

/* reference mini_raytrace.h:95-109 */
typedef struct mrtMaterialDesc {
    size_t structSize;
    float baseColor[3];
    float opacity;
    float roughness;
    float metallic;
    float transmission;
    float ior;
    float emission[3];
    mrtTextureId baseColorTex; /* MRT_INVALID_ID = constant value */
    mrtTextureId roughnessTex;
    mrtTextureId metallicTex;
    mrtTextureId normalTex;
    mrtTextureId emissionTex;
} mrtMaterialDesc;

/* reference mini_raytrace.h:111-117 */
typedef struct mrtTextureDesc {
    size_t structSize;
    uint32_t width, height;
    mrtTextureFormat format;
    const void* pixels; /* tightly packed RGBA */
    int32_t generateMips;
} mrtTextureDesc;

/* reference mini_raytrace.h:119-128 */
typedef struct mrtLightDesc {
    size_t structSize;
    mrtLightType type;
    float direction[3]; /* sun: unit-ish vector towards the light */
    float position[3];  /* point light */
    float radiance[3];  /* sun/rect: radiance; point: intensity (W/sr) */
    float angularRadius; /* sun cone half-angle, radians */
    float corner[3], edge0[3], edge1[3]; /* rect light */
    int32_t twoSided;                   /* rect light */
} mrtLightDesc;

/* reference mini_raytrace.h:130-136 */
typedef struct mrtCameraDesc {
    size_t structSize;
    float position[3];
    float target[3];
    float up[3];
    float fovYDeg;
} mrtCameraDesc;

/* reference mini_raytrace.h:138-141 */
typedef enum mrtCameraProjection {
    MRT_CAMERA_PERSPECTIVE = 0,
    MRT_CAMERA_ORTHOGRAPHIC = 1,
} mrtCameraProjection;

/* reference mini_raytrace.h:148-155: explicit (possibly asymmetric) frustum.
 * Perspective: left/right/bottom/top of the slice at distance 1 along
 * forward. Orthographic: absolute half-extents. */
typedef struct mrtCameraDescEx {
    size_t structSize;
    int32_t projection; /* mrtCameraProjection */
    float position[3];
    float forward[3];
    float up[3];
    float left, right, bottom, top;
} mrtCameraDescEx;

/* reference mini_raytrace.h:157-166 */
typedef struct mrtRenderSettings {
    size_t structSize;
    uint32_t width, height;
    uint32_t maxBounces;  /* default 8, capped at 16 */
    uint32_t sppLimit;    /* default 1024 */
    float exposureEV;     /* default 0 */
    float fireflyClamp;   /* 0 = off, default 50 */
    mrtTonemap tonemap;   /* default ACES */
    int32_t denoise;      /* accepted and ignored (no denoiser in this build) */
} mrtRenderSettings;

/* reference mini_raytrace.h:168-174 */
typedef struct mrtFrameInfo {
    size_t structSize;
    uint32_t spp;
    int32_t converged;
    int32_t denoised;
    float frameMs;
} mrtFrameInfo;

/* reference mini_raytrace.h:176-181 */
typedef struct mrtCommitStats {
    size_t structSize;
    uint32_t blasRebuilt;
    int32_t tlasRebuilt;
    float commitMs;
} mrtCommitStats;

/* ---- lifecycle (reference mini_raytrace.h:184-185; capi.cpp:95-125) ------ */
MRT_API mrtResult mrtCreateEngine(const mrtEngineDesc* desc, mrtEngine** outEngine);
MRT_API void mrtDestroyEngine(mrtEngine* engine);

/* ---- incremental scene (reference mini_raytrace.h:188-214; Scene.cpp) ---- */
MRT_API mrtMeshId mrtAddMesh(mrtEngine*, const mrtMeshDesc*);
MRT_API void mrtUpdateMesh(mrtEngine*, mrtMeshId, const mrtMeshDesc*);
MRT_API void mrtRemoveMesh(mrtEngine*, mrtMeshId);

/* xform3x4: row-major rows of [R|t]; NULL = identity */
MRT_API mrtInstanceId mrtAddInstance(mrtEngine*, mrtMeshId, const float* xform3x4, mrtMaterialId);
MRT_API void mrtSetInstanceTransform(mrtEngine*, mrtInstanceId, const float* xform3x4);
MRT_API void mrtRemoveInstance(mrtEngine*, mrtInstanceId);

MRT_API mrtMaterialId mrtAddMaterial(mrtEngine*, const mrtMaterialDesc*);
MRT_API void mrtUpdateMaterial(mrtEngine*, mrtMaterialId, const mrtMaterialDesc*);
MRT_API void mrtRemoveMaterial(mrtEngine*, mrtMaterialId);
MRT_API mrtTextureId mrtAddTexture(mrtEngine*, const mrtTextureDesc*);
MRT_API void mrtRemoveTexture(mrtEngine*, mrtTextureId);

MRT_API mrtLightId mrtAddLight(mrtEngine*, const mrtLightDesc*);
MRT_API void mrtUpdateLight(mrtEngine*, mrtLightId, const mrtLightDesc*);
MRT_API void mrtRemoveLight(mrtEngine*, mrtLightId);

/* hdri must be MRT_TEX_RGBA32F (equirectangular); NULL clears the environment */
MRT_API void mrtSetEnvironment(mrtEngine*, const mrtTextureDesc* hdri, float rotationRad,
                               float intensity);
MRT_API void mrtSetCamera(mrtEngine*, const mrtCameraDesc*);
MRT_API void mrtSetCameraEx(mrtEngine*, const mrtCameraDescEx*);

/* Apply pending changes now. Idempotent; outStats may be NULL.
 * (reference mini_raytrace.h:216-219; Engine.cpp:44-55) */
MRT_API mrtResult mrtCommitScene(mrtEngine*, mrtCommitStats* outStats);

/* ---- render (reference mini_raytrace.h:222-228) --------------------------- */
MRT_API mrtResult mrtSetRenderSettings(mrtEngine*, const mrtRenderSettings*);
/* Blocking; adds exactly one sample per pixel until sppLimit is reached. */
MRT_API mrtResult mrtRenderFrame(mrtEngine*, mrtFrameInfo* outInfo);
/* dst holds width*height*4 (RGBA8) or width*height*16 (RGBA32F) bytes. */
MRT_API mrtResult mrtReadFramebuffer(mrtEngine*, mrtPixelFormat, void* dst, size_t dstSize);
MRT_API void mrtResetAccumulation(mrtEngine*);

/* ---- misc (reference mini_raytrace.h:231-237) ----------------------------- */
typedef void (*mrtLogFn)(int level /* 0=debug .. 3=error */, const char* message, void* user);
MRT_API void mrtSetLogCallback(mrtLogFn fn, void* user);
MRT_API const char* mrtResultToString(mrtResult r);
/* Detail of the most recent failure on this thread; "" if none; never NULL. */
MRT_API const char* mrtGetLastErrorMessage(void);

#ifdef __cplusplus
} /* extern "C" */
#endif
#endif /* MINI_RAYTRACE_H */
