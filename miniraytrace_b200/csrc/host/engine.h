// The engine behind one mrtEngine handle: scene store, device-resident scene
// arrays, accumulation buffers and the per-frame launch logic. It combines
// the roles of the reference's Engine facade (core/src/Engine.cpp) and
// Renderer (core/src/render/Renderer.cpp) on a CUDA device.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <vector>

#include "../../../include/mrt_ext.h"
#include "../common/device_types.h"
#include "../cuda/device_api.h"
#include "bvh_build.h"
#include "lbvh.h"
#include "wide_bvh.h"
#include "common.h"
#include "copy_pool.h"
#include "scene.h"

namespace mrt {

// Grow-only device allocation.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    mrtResult ensure(size_t n);
    mrtResult upload(const void* src, size_t n, cudaStream_t s);
    void release();
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};

struct Settings {  // reference SceneTypes.hpp:142-152 defaults
    uint32_t width = 1280, height = 720, maxBounces = 8, sppLimit = 1024;
    float exposureEV = 0.0f, fireflyClamp = 50.0f;
    uint32_t tonemap = MRT_TONEMAP_ACES;
    bool denoise = true;
};

class Engine {
public:
    static mrtResult create(const mrtEngineDesc& desc, Engine** out);
    ~Engine();

    Scene& scene() { return m_scene; }

    mrtResult setSettings(const Settings& s);
    void resetAccumulation();
    mrtResult commit(mrtCommitStats* stats);
    mrtResult renderFrames(uint32_t count, mrtFrameInfo* info, bool defer = false);
    mrtResult flushPending();  // renders queued samples
    // Several engines' samples issued together (one stream each), then waited for.
    static mrtResult renderBatch(Engine* const* engines, const uint32_t* spp, uint32_t count, mrtFrameInfo* infos);
    mrtResult readFramebuffer(mrtPixelFormat fmt, void* dst, size_t dstSize);

    mrtResult traceRays(const mrtxRay* rays, uint32_t n, mrtxHit* hits);
    mrtResult traceRaysWavefront(const mrtxRay* rays, uint32_t n, mrtxHit* hits);
    mrtResult traceShadowRays(const mrtxRay* rays, uint32_t n, uint32_t* occluded);
    mrtResult readAccumulation(double* dst, size_t dstSize, uint32_t* spp);
    mrtResult getStats(mrtxStats* out) const;
    mrtResult measureL2Bandwidth(float* gbs);
    mrtResult buildEnvCdf(const float* rgba, uint32_t w, uint32_t h, float* cdf, float* integral);
    mrtResult setSampleStream(uint32_t offset, uint32_t stride);
    mrtResult setTraversalBudget(uint32_t maxVisits);
    mrtResult setBvhBuildThresholds(uint32_t minTriangles, uint32_t minInstances);
    mrtResult copyAccumulationDevice(void* dev, size_t bytes, bool accumulate);
    // 8-wide BVH of one triangle mesh built on this engine's GPU (LBVH
    // topology, SAH-optimal collapse), read back into `out`.
    mrtResult setRadianceCache(const mrtxRadianceCacheDesc& d);
    mrtResult cacheQuery(const float* features, uint32_t n, float* rgb);
    mrtResult cacheTrain(const float* features, const float* targets, uint32_t n, uint32_t steps, float* loss);
    mrtResult cacheParams(float* gridOut, float* mlpOut, const float* gridIn, const float* mlpIn);
    mrtResult cacheGradients(const float* features, const float* targets, uint32_t n, float* gridOut, float* mlpOut,
                             float* loss);
    mrtResult setCacheAveraging(float decay);
    mrtResult setCacheSchedule(float lrMin, float halfLifeSteps);
    mrtResult setDenoiser(const mrtxDenoiserDesc& d);
    mrtResult readDenoised(float* rgba, size_t bytes);
    mrtResult readDenoiserGuides(float* albedo, float* normalDepth, size_t bytes);
    mrtResult buildMeshBvhDevice(const V4f* pos, size_t nv, const uint32_t* idx, size_t nt, uint32_t maxLeaf,
                                 WideBvh& out);
    // Device build from device positions/indices into the builder's own
    // output buffers (m_bvhNodes, m_bvhPrims).
    mrtResult buildBvhOnDevice(const float4* pos, const uint32_t* idx, size_t nt, uint32_t maxLeaf, uint32_t& count,
                               Box3& bounds);

private:
    Engine() = default;
    mrtResult init(const mrtEngineDesc& desc);
    mrtResult checkAlive();
    mrtResult guard(mrtResult r);  // records a device loss
    mrtResult allocateFrame();
    mrtResult ensureWave(uint32_t samples);
    mrtResult carveWave(uint64_t slots, MrtWaveState& w);
    mrtResult ensureEvents(size_t stage);
    // mrtxRenderBatch with every engine's waves in one set of launches
    static mrtResult renderBatchOneLaunch(Engine* const* engines, const uint32_t* n, uint32_t count);
    uint32_t waveCapacitySamples() const;
    mrtResult launchPending();    // issues the queued samples' waves, no wait
    mrtResult completePending();  // waits for them, statistics, error flags
    mrtResult up(DeviceBuffer& b, const void* src, size_t n);
    mrtResult sync(mrtCommitStats* stats);  // reference Renderer::syncScene
    mrtResult packMaterials();
    mrtResult packGeometry(uint32_t& rebuilt);
    mrtResult packInstances();
    mrtResult buildTlasOnDevice(const std::vector<Box3>& boxes, std::vector<uint32_t>& order, uint32_t& count);
    mrtResult packLights();
    mrtResult packEnvironment();
    mrtResult uploadTextures();
    mrtResult runEnvCdf(const float* rgba, uint32_t w, uint32_t h, float& integral);
    void fillParams(MrtFrameParams& p) const;
    mrtResult checkErrorFlags();
    mrtResult download(void* dst, const void* src, size_t bytes);

    int m_device = 0;
    cudaStream_t m_stream = nullptr;
    cudaStream_t m_side = nullptr;  // shadow kernels beside the next bounce's extend
    std::vector<cudaEvent_t> m_syncEvents;  // 2 per bounce of a render call, without timing
    cudaEvent_t m_ev0 = nullptr, m_ev1 = nullptr;
    std::vector<cudaEvent_t> m_copyEvents;
    std::vector<cudaEvent_t> m_stageEvents;  // 6 per bounce per wave of one render call
    std::vector<cudaEvent_t> m_cacheEvents;  // cache mode: 3 per wave (inference, training)
    uint64_t m_cacheQueries = 0, m_cacheRecords = 0;  // of the render call in flight
    uint32_t m_cacheSteps = 0;
    bool m_lost = false;
    bool m_validation = false;
    unsigned m_hostThreads = 1;

    Scene m_scene;
    Settings m_settings;

    // device scene
    DeviceBuffer m_nodes, m_triVerts, m_triIndex, m_normals, m_uvs, m_tangents;
    DeviceBuffer m_instances, m_materials, m_lights;
    DeviceBuffer m_envTexels, m_envCdf, m_envSin, m_envRowSums, m_envIntegral;
    DeviceBuffer m_texTable;
    DeviceBuffer m_srgbLut;  // 256 floats: sRGB decode of k / 255
    uint32_t m_maxVisits = 0;  // traversal visit budget (0: the kernels' default)
    // smallest mesh (triangles) and instance set whose BVH is built on the GPU
    uint32_t m_deviceMinTriangles = 0, m_deviceMinInstances = 0;
    DeviceBuffer m_texData[MRT_MAX_TEXTURES];
    std::vector<uint32_t> m_texGeneration;
    // device frame state
    DeviceBuffer m_accum, m_out32, m_out8, m_flags, m_rayCounters, m_queryRays, m_queryOut;
    DeviceBuffer m_wave;  // wavefront path state (one allocation, carved into MrtWaveState arrays)
    DeviceBuffer m_batchJobs;  // job tables of a one-launch batch this engine leads
    DeviceBuffer m_bvhPos, m_bvhIdx, m_bvhScratch, m_bvhNodes, m_bvhPrims;  // device BVH builder
    DeviceBuffer m_packError;  // error word of the commit-time assembly kernels

    // radiance cache: parameters, gradients, Adam moments, query scratch
    struct RadianceCache {
        DeviceBuffer grid, mlp, gGrid, gMlp, mGrid, vGrid, mMlp, vMlp, in, out, loss, partial;
        DeviceBuffer emaGrid, emaMlp;  // moving averages of the parameters, read by inference
        DeviceBuffer qFeat, qBeta, rFeat, rPrefix, rBeta, rTarget, counts, scratch;  // per-wave queries/records
        DeviceBuffer sortScratch;  // Morton keys and order of a wave's queries
        MrtCacheArgs args{};
        McacheParams params{};
        bool allocated = false, enabled = false;
        // Set once a tensor-core wait of a cache kernel gave up: that MMA may
        // still have been writing tensor memory when its CTA freed it, so no
        // cache output of the launch is trusted and no cache kernel runs again
        // in this engine.
        bool failed = false;
        uint32_t trainingPaths = 0, stepsPerSample = 1, seed = 1, samplesPerUpdate = 4, trainingVertices = 0;
        float lr = 1e-2f;
        float emaDecay = 0.99f;  // 0: inference reads the live parameters
        // learning-rate decay: halves every lrHalfLife steps down to lrMin (0: constant)
        float lrMin = 3e-4f, lrHalfLife = 96.0f;
        float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        void release();
    } m_cache;
    // Opt-in denoiser (mrtxSetDenoiser): guides once per accumulation, the
    // filtered image re-made on the reference's doubling schedule.
    struct DenoiserState {
        bool enabled = false;
        MrtDenoiseParams params{0, 0, 5, 0, 1.0f, 64.0f, 0.1f, 0.1f, 0.01f};
        uint32_t guideSamples = 4, minSpp = 8;
        DeviceBuffer albedo, normalDepth, work, out;
        bool guidesValid = false, useDenoised = false;
        uint32_t nextAt = 8, denoisedSpp = 0;
        void release();
    } m_denoiser;
    bool denoiserActive() const { return m_denoiser.enabled && m_settings.denoise; }
    mrtResult ensureGuides();
    mrtResult runDenoise();
    mrtResult ensureCache();
    void cacheBounds();
    mrtResult cacheWaveBuffers(uint32_t samples, uint32_t maxBounces);
    mrtResult cacheStatus(uint32_t status);
    McacheParams inferenceParams() const;  // the parameters queries read (averaged or live)
    mrtResult resetAverage();              // average := live parameters
    mrtResult cacheWave(const MrtFrameParams& p, uint32_t sampleBase, uint32_t samples, const cudaEvent_t* ev);
    MrtWaveState m_waveState{};
    uint32_t m_waveSamples = 0;  // samples per pixel one wave holds
    uint64_t m_maxWaveSlots = uint64_t(1) << 25;  // paths per wave, set from the GPU's memory
    void* m_pinned = nullptr;
    size_t m_pinnedBytes = 0;
    // upload staging: kStageSlots pinned slots of kStageChunk bytes, each
    // with the event of its last DMA
    static constexpr size_t kStageChunk = size_t(4) << 20, kStageSlots = 4;
    void* m_stage = nullptr;
    cudaEvent_t m_stageCopyEvents[kStageSlots] = {};
    bool m_stageUsed[kStageSlots] = {};
    mrtResult uploadStaged(void* dst, const void* src, size_t n);
    std::unique_ptr<CopyPool> m_copyPool;  // copies out of m_pinned on several threads

    // host-side packing state
    // One mesh on the device: its own copies of the vertex data, indices and
    // 8-wide BVH (object space, mesh-relative indices), uploaded or built when
    // the mesh changes; commits assemble the global arrays from these.
    struct Blas {
        DeviceBuffer pos, idx, normals, uvs, tangents, nodes, prims;
        uint32_t vertexCount = 0, triCount = 0, nodeCount = 0;
        Box3 bounds{{3.402823466e38f, 3.402823466e38f, 3.402823466e38f},
                    {-3.402823466e38f, -3.402823466e38f, -3.402823466e38f}};
        uint32_t nodeBase = 0;
        void release();
        size_t deviceBytes() const;
    };
    mrtResult uploadMesh(const MeshData& m, Blas& b);
    bool ensureTangents();
    mrtResult buildBlasOnDevice(Blas& b);
    std::map<uint32_t, Blas> m_blas;
    std::map<uint32_t, uint32_t> m_materialIndex;
    uint32_t m_nodeCount = 0, m_blasNodeCount = 0, m_triCount = 0, m_materialCount = 1;
    uint32_t m_tlasRoot = 0, m_instanceCount = 0, m_lightCount = 0;
    uint32_t m_envW = 0, m_envH = 0;
    float m_sceneLo[3] = {0, 0, 0}, m_sceneHi[3] = {0, 0, 0};  // world bounds of the instances
    float m_envIntegralHost = 1.0f;
    bool m_hasEnv = false;

    // accumulation
    uint32_t m_frameIndex = 0;  // samples per pixel accumulated since reset
    uint32_t m_pending = 0;     // samples queued by mrtRenderFrame, not yet rendered
    uint32_t m_inFlight = 0;    // samples issued by launchPending, not yet completed
    uint32_t m_inFlightWaves = 0, m_inFlightBounces = 0, m_inFlightLaunches = 0;
    bool m_inFlightCache = false;  // the render call in flight uses the radiance cache
    MrtFrameParams m_pendingParams{};
    uint32_t m_streamOffset = 0, m_streamStride = 1;
    float m_resolveExposure = 1.0f;
    uint32_t m_resolveTonemap = MRT_TONEMAP_ACES;

    // statistics
    mrtxStats m_stats{};
};

}  // namespace mrt
