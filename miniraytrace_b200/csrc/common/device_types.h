// Plain-old-data layouts shared by the host engine (C++) and the sm_100a
// kernels (CUDA). Nothing here is a C++ class: these cross the seam between
// the host translation units and the .cu translation units as raw bytes.
//
// HBM layout of one committed scene (all arrays 16-byte aligned, read-only
// during a frame, fetched with 128-bit non-coherent loads):
//
//   nodes      MrtNode[]     BVH2 nodes, 32 B each. Per mesh a BLAS, then the
//                            TLAS. Children of an internal node are adjacent
//                            (left, left + 1), so one 64-byte fetch yields
//                            both child boxes.
//   triVerts   float4[3*T]   the three vertex positions of every triangle,
//                            in BLAS leaf order (48 B per triangle test;
//                            w of vertex 0 holds the original triangle index
//                            as bits, w of vertex 1 the global triangle slot).
//   triIndex   uint4[T]      global vertex indices (i0, i1, i2, original
//                            index) in the same order, read once per hit.
//   normals    float4[V]     shading normals (xyz), per global vertex.
//   uvs        float2[V]
//   tangents   float4[V]     xyz + handedness.
//   instances  MrtInstance[] 112 B each, in TLAS leaf order.
//   materials  MrtMaterial[] 80 B each, index 0 = default material.
//   lights     MrtLight[]    80 B each, environment at slot 0 when present.
//   envTexels  float4[w*h]   RGBA32F equirect map.
//   envCdf     float[w*h+h]  conditional rows, then the marginal.
//   textures   MrtTexture[64]
//
//   accum      double4[W*H]  FP64 running sums (r, g, b, sample count).
#pragma once

#include <stdint.h>
#include <vector_types.h>

#ifdef __CUDACC__
#define MRT_HD __host__ __device__
#else
#define MRT_HD
#endif

#define MRT_MAX_TEXTURES 64
#define MRT_MAX_BOUNCES_CAP 16

// Reference BVH node semantics (core/src/accel/Bvh.hpp:15-26): count == 0
// marks an internal node whose children are (leftOrPrim, leftOrPrim + 1);
// otherwise leftOrPrim is the first triangle (or instance, in the TLAS).
typedef struct MrtNode {
    float lo[3];
    uint32_t leftOrPrim;
    float hi[3];
    uint32_t packed;  // (count << 2) | split axis
} MrtNode;

// 8-wide compressed BVH node, 80 bytes (five 16-byte loads); see
// csrc/host/wide_bvh.h for the encoding. Bytes 0-15: origin + exponents +
// internal mask; 16-31: child/primitive bases + meta bytes; 32-79: the eight
// quantised child boxes, axis-major (lo x, lo y, lo z, hi x, hi y, hi z).
typedef struct MrtWideNode {
    float p[3];
    uint8_t e[3];
    uint8_t imask;
    uint32_t childBase;
    uint32_t primBase;
    uint8_t meta[8];
    uint8_t qlo[3][8];
    uint8_t qhi[3][8];
} MrtWideNode;

// Instance: row-major 3x4 transforms (rows of [R | t]).
typedef struct MrtInstance {
    float w2o[12];
    float o2w[12];
    uint32_t blasRoot;
    uint32_t materialIndex;
    uint32_t userId;  // mrtInstanceId
    uint32_t meshId;
} MrtInstance;

// Reference GpuMaterial (core/src/render/GpuTypes.hpp:55-61), 80 bytes.
typedef struct MrtMaterial {
    float baseColorOpacity[4];
    float emissionRoughness[4];
    float params[4];  // metallic, transmission, ior, unused
    int32_t tex[8];   // baseColor, roughness, metallic, normal, emission, -, -, -
} MrtMaterial;

// Reference GpuLight (GpuTypes.hpp:69-75), 80 bytes.
enum { MRT_DLIGHT_ENV = 0, MRT_DLIGHT_SUN = 1, MRT_DLIGHT_POINT = 2, MRT_DLIGHT_RECT = 3 };
typedef struct MrtLight {
    float p0[4];  // sun: dir + cos(angular radius) | point: pos | rect: corner + area
    float p1[4];  // sun: radiance | point: intensity | rect: edge0
    float p2[4];  // rect: edge1
    float p3[4];  // rect: radiance + twoSided
    int32_t type;
    int32_t pad[3];
} MrtLight;

enum { MRT_DTEX_RGBA8_SRGB = 0, MRT_DTEX_RGBA8_UNORM = 1, MRT_DTEX_RGBA32F = 2 };
typedef struct MrtTexture {
    const void* texels;  // NULL = white 1x1 placeholder
    uint32_t width, height;
    uint32_t format;
    uint32_t pad;
} MrtTexture;

enum { MRT_FLAG_HAS_ENV = 1u, MRT_FLAG_ORTHO = 4u };

#define MRT_DEFAULT_MAX_VISITS (1u << 22)

// Radiance-cache mode of one wave (shade kernel's cache instantiation):
// paths other than training paths stop at their second surface vertex and
// append a query there (16 features; beta and the slot); training paths
// continue and append a record at every vertex from the second on
// (features; radiance gathered before the vertex and the slot; beta). A path
// is a training path when hash(pixel, frame index) % trainStride == 0.
typedef struct MrtCacheArgs {
    float* qFeat;
    float4* qBeta;     // beta xyz, slot bits in w
    uint32_t* qCount;
    uint32_t qCap;
    float* rFeat;
    float4* rPrefix;   // radiance before the vertex xyz, slot bits in w
    float4* rBeta;     // beta xyz
    uint32_t* rCount;
    uint32_t rCap;
    uint32_t trainStride;
    uint32_t recordBounces;  // training paths record their vertices 1..recordBounces
    float spreadC;           // path-spread threshold c of the query vertex (a_n > c a_0)
} MrtCacheArgs;

// Everything one path-tracing launch reads; passed by value as the kernel
// parameter block (no constant-memory update, so launches stay
// graph-capturable with new parameters).
typedef struct MrtFrameParams {
    // camera (reference Renderer.cpp:711-764 fillGlobals)
    float camPos[3], camRight[3], camUp[3], camForward[3];
    float frustum[4];  // left, right, bottom, top
    uint32_t width, height;
    uint32_t maxBounces, lightCount;
    uint32_t envW, envH, flags, tlasRoot;
    float envRotation, envIntensity, envIntegral, fireflyClamp;
    // Sample streams: the n-th sample since the last reset uses the pcg4d
    // frame index streamOffset + n * streamStride (reference stream:
    // offset 0, stride 1, pathtrace.comp:105).
    uint32_t streamOffset, streamStride;
    uint32_t nodeCount, instanceCount, triCount, materialCount;
    // Node visits one traversal may make before it gives up and sets bit 0
    // of errorFlags. A well-formed BVH never gets near the default
    // (MRT_DEFAULT_MAX_VISITS); the bound only turns a malformed tree into
    // an error instead of an endless loop.
    uint32_t maxVisits, pad0;
    // sRGB decode of an 8-bit channel value k, (k / 255) -> linear, 256
    // entries built on the host (the decode is a double-precision power;
    // the table keeps it off the GPU and gives the same bits).
    const float* srgbLut;
    // scene arrays (device pointers)
    const MrtWideNode* nodes;  // 8-wide BVH: every BLAS, then the TLAS
    const float4* triVerts;
    const uint4* triIndex;
    const float4* normals;
    const float2* uvs;
    const float4* tangents;
    const MrtInstance* instances;
    const MrtMaterial* materials;
    const MrtLight* lights;
    const float4* envTexels;
    const float* envCdf;
    const MrtTexture* textures;
    // frame buffers
    double* accum;           // 4 doubles per pixel
    uint32_t* errorFlags;    // bit 0: traversal stack overflow, bit 1: bad index
    unsigned long long* rayCounters;  // [closest, shadow], NULL = not counted
} MrtFrameParams;

// Wavefront path state (structure of arrays, one slot per path in flight).
// A wave renders `spp` samples of every pixel: slot = pixel * spp + s, so
// the samples of a pixel sit in neighbouring lanes (their paths start at one
// surface point and traverse similar nodes: 8.7% faster on the 1080p terrain
// than slot = s * pixels + pixel; ordering the pixels in 8x8 tiles instead
// of rows changed nothing).
// Each bounce runs extend (closest hit of the queued rays), shade (surface,
// NEE sample, BSDF sample, Russian roulette; appends the continuing paths to
// the other queue and the shadow rays to the shadow queue) and shadow
// (any-hit; adds the NEE contribution of unoccluded rays).
typedef struct MrtWaveState {
    float4* rayO;       // origin.xyz, w = pdf of the BSDF sample that made the ray
    float4* rayD;       // direction.xyz, w = bits(bounce)
    float4* beta;       // throughput.xyz, w = bits(RNG counter)
    float4* L;          // radiance.xyz
    float4* hit;        // t, u, v, bits(triangle slot; 0xffffffff = miss)
    uint32_t* hitInst;  // instance slot of the hit
    uint32_t* queue[2]; // active slot lists, alternating per bounce
    float4* shO;        // shadow ray origin.xyz, w = tMax
    float4* shD;        // shadow ray direction.xyz, w = bits(slot)
    float4* shC;        // contribution added when the shadow ray is unoccluded
    uint32_t* counts;   // [0..1] path queue lengths, [2..3] shadow queue lengths, [4..7] fetch heads
    uint32_t capacity;  // slots
    uint32_t pad;
} MrtWaveState;

// One job of a one-launch batch (several engines' waves rendered by the
// same kernel launches): the job's frame parameters, its wave (pixels,
// slots = pixels x samples, the first sample's index, samples per pixel),
// and where its slots and pixels start in the batch's concatenated slot and
// pixel ranges. A batch wave's slot s belongs to the last job whose
// slotBase <= s; its local slot is s - slotBase.
typedef struct MrtBatchJob {
    MrtFrameParams params;
    uint32_t pixels, slots, sampleBase, samples;
    uint32_t slotBase, pixelBase;
    uint32_t pad[2];
} MrtBatchJob;

typedef struct MrtBatchJobs {
    const MrtBatchJob* jobs;  // device memory, `count` entries, slotBase ascending
    uint32_t count;
    uint32_t totalSlots, totalPixels;
    uint32_t pad;
} MrtBatchJobs;

// One query ray of mrtxTraceRays (same layout as mrtxRay) and its hit.
typedef struct MrtQueryRay {
    float origin[3];
    float tMax;
    float dir[3];
    float pad;
} MrtQueryRay;

typedef struct MrtQueryHit {
    float t;
    uint32_t instance;
    uint32_t prim;
    uint32_t hit;
    float u, v;
    uint32_t pad[2];
} MrtQueryHit;
