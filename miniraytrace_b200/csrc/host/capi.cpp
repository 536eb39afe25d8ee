// The exported C ABI (include/mini_raytrace.h, include/mrt_ext.h).
//
// Argument handling mirrors the reference translation layer
// (capi/src/capi.cpp:10-316): structs shorter than the version compiled
// here are rejected, a NULL engine yields MRT_ERROR_INVALID_HANDLE for
// commit/render and MRT_ERROR_INVALID_ARGUMENT for readback/settings, void
// scene calls ignore bad handles, add-calls return MRT_INVALID_ID, and no C++
// exception crosses the boundary (std::bad_alloc -> MRT_ERROR_OUT_OF_MEMORY,
// anything else -> MRT_ERROR_UNKNOWN).
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../../include/mrt_ext.h"
#include "../cuda/device_api.h"
#include "engine.h"
#include "lbvh.h"
#include "wide_bvh.h"

namespace {

mrt::Engine* unwrap(mrtEngine* e) { return reinterpret_cast<mrt::Engine*>(e); }

template <class T> bool validStruct(const T* s) { return s && s->structSize >= sizeof(T); }

template <class Fn> mrtResult guarded(Fn fn) {
    try {
        return fn();
    } catch (const std::bad_alloc&) {
        return mrt::fail(MRT_ERROR_OUT_OF_MEMORY, "host allocation failed");
    } catch (...) {
        return mrt::fail(MRT_ERROR_UNKNOWN, "unexpected exception in libmrt");
    }
}

template <class Fn> uint32_t guardedId(Fn fn) {
    try {
        return fn();
    } catch (...) {
        mrt::setLastError("allocation failed while copying scene data");
        return MRT_INVALID_ID;
    }
}

template <class Fn> void guardedVoid(Fn fn) {
    try {
        fn();
    } catch (...) {
        mrt::setLastError("allocation failed while copying scene data");
    }
}

}  // namespace

extern "C" {

MRT_API mrtResult mrtCreateEngine(const mrtEngineDesc* desc, mrtEngine** outEngine) {
    if (!validStruct(desc) || !outEngine) return MRT_ERROR_INVALID_ARGUMENT;
    return guarded([&] {
        mrt::Engine* e = nullptr;
        const mrtResult r = mrt::Engine::create(*desc, &e);
        if (r == MRT_SUCCESS) *outEngine = reinterpret_cast<mrtEngine*>(e);
        return r;
    });
}

MRT_API void mrtDestroyEngine(mrtEngine* engine) { delete unwrap(engine); }

MRT_API mrtMeshId mrtAddMesh(mrtEngine* e, const mrtMeshDesc* d) {
    mrt::Engine* eng = unwrap(e);
    if (!eng || !validStruct(d)) return MRT_INVALID_ID;
    return guardedId([&] { return eng->scene().addMesh(*d); });
}

MRT_API void mrtUpdateMesh(mrtEngine* e, mrtMeshId id, const mrtMeshDesc* d) {
    mrt::Engine* eng = unwrap(e);
    if (eng && validStruct(d)) guardedVoid([&] { eng->scene().updateMesh(id, *d); });
}

MRT_API void mrtRemoveMesh(mrtEngine* e, mrtMeshId id) {
    if (mrt::Engine* eng = unwrap(e)) eng->scene().removeMesh(id);
}

MRT_API mrtInstanceId mrtAddInstance(mrtEngine* e, mrtMeshId mesh, const float* xform3x4, mrtMaterialId mat) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_INVALID_ID;
    return guardedId([&] { return eng->scene().addInstance(mesh, xform3x4, mat); });
}

MRT_API void mrtSetInstanceTransform(mrtEngine* e, mrtInstanceId id, const float* xform3x4) {
    if (mrt::Engine* eng = unwrap(e)) eng->scene().setInstanceTransform(id, xform3x4);
}

MRT_API void mrtRemoveInstance(mrtEngine* e, mrtInstanceId id) {
    if (mrt::Engine* eng = unwrap(e)) eng->scene().removeInstance(id);
}

MRT_API mrtMaterialId mrtAddMaterial(mrtEngine* e, const mrtMaterialDesc* d) {
    mrt::Engine* eng = unwrap(e);
    if (!eng || !validStruct(d)) return MRT_INVALID_ID;
    return guardedId([&] { return eng->scene().addMaterial(*d); });
}

MRT_API void mrtUpdateMaterial(mrtEngine* e, mrtMaterialId id, const mrtMaterialDesc* d) {
    mrt::Engine* eng = unwrap(e);
    if (eng && validStruct(d)) eng->scene().updateMaterial(id, *d);
}

MRT_API void mrtRemoveMaterial(mrtEngine* e, mrtMaterialId id) {
    if (mrt::Engine* eng = unwrap(e)) eng->scene().removeMaterial(id);
}

MRT_API mrtTextureId mrtAddTexture(mrtEngine* e, const mrtTextureDesc* d) {
    mrt::Engine* eng = unwrap(e);
    if (!eng || !validStruct(d)) return MRT_INVALID_ID;
    return guardedId([&] { return eng->scene().addTexture(*d); });
}

MRT_API void mrtRemoveTexture(mrtEngine* e, mrtTextureId id) {
    if (mrt::Engine* eng = unwrap(e)) eng->scene().removeTexture(id);
}

MRT_API mrtLightId mrtAddLight(mrtEngine* e, const mrtLightDesc* d) {
    mrt::Engine* eng = unwrap(e);
    if (!eng || !validStruct(d)) return MRT_INVALID_ID;
    return guardedId([&] { return eng->scene().addLight(*d); });
}

MRT_API void mrtUpdateLight(mrtEngine* e, mrtLightId id, const mrtLightDesc* d) {
    mrt::Engine* eng = unwrap(e);
    if (eng && validStruct(d)) eng->scene().updateLight(id, *d);
}

MRT_API void mrtRemoveLight(mrtEngine* e, mrtLightId id) {
    if (mrt::Engine* eng = unwrap(e)) eng->scene().removeLight(id);
}

MRT_API void mrtSetEnvironment(mrtEngine* e, const mrtTextureDesc* hdri, float rotationRad, float intensity) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return;
    if (!hdri) {
        eng->scene().clearEnvironment();
        return;
    }
    if (validStruct(hdri)) guardedVoid([&] { eng->scene().setEnvironment(*hdri, rotationRad, intensity); });
}

MRT_API void mrtSetCamera(mrtEngine* e, const mrtCameraDesc* d) {
    mrt::Engine* eng = unwrap(e);
    if (!eng || !validStruct(d)) return;
    eng->scene().setCamera(*d);
}

MRT_API void mrtSetCameraEx(mrtEngine* e, const mrtCameraDescEx* d) {
    mrt::Engine* eng = unwrap(e);
    if (!eng || !validStruct(d)) return;
    eng->scene().setCameraEx(*d);
}

MRT_API mrtResult mrtCommitScene(mrtEngine* e, mrtCommitStats* outStats) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] {
        mrtCommitStats s{};
        s.structSize = sizeof(s);
        const mrtResult r = eng->commit(&s);
        if (outStats && outStats->structSize >= sizeof(mrtCommitStats)) {
            outStats->blasRebuilt = s.blasRebuilt;
            outStats->tlasRebuilt = s.tlasRebuilt;
            outStats->commitMs = s.commitMs;
        }
        return r;
    });
}

MRT_API mrtResult mrtSetRenderSettings(mrtEngine* e, const mrtRenderSettings* d) {
    mrt::Engine* eng = unwrap(e);
    if (!eng || !validStruct(d)) return MRT_ERROR_INVALID_ARGUMENT;
    return guarded([&] {
        mrt::Settings s;
        s.width = d->width;
        s.height = d->height;
        s.maxBounces = d->maxBounces;
        s.sppLimit = d->sppLimit;
        s.exposureEV = d->exposureEV;
        s.fireflyClamp = d->fireflyClamp;
        s.tonemap = uint32_t(d->tonemap);
        s.denoise = d->denoise != 0;
        return eng->setSettings(s);
    });
}

MRT_API mrtResult mrtRenderFrame(mrtEngine* e, mrtFrameInfo* outInfo) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] { return eng->renderFrames(1, outInfo, true); });
}

MRT_API mrtResult mrtReadFramebuffer(mrtEngine* e, mrtPixelFormat fmt, void* dst, size_t dstSize) {
    mrt::Engine* eng = unwrap(e);
    if (!eng || !dst) return MRT_ERROR_INVALID_ARGUMENT;
    return guarded([&] { return eng->readFramebuffer(fmt, dst, dstSize); });
}

MRT_API void mrtResetAccumulation(mrtEngine* e) {
    if (mrt::Engine* eng = unwrap(e)) eng->resetAccumulation();
}

MRT_API void mrtSetLogCallback(mrtLogFn fn, void* user) { mrt::setLogCallback(fn, user); }

MRT_API const char* mrtResultToString(mrtResult r) { return mrt::resultName(r); }

MRT_API const char* mrtGetLastErrorMessage(void) { return mrt::lastError().c_str(); }

// ---- extensions (include/mrt_ext.h) --------------------------------------------

MRT_API mrtResult mrtxRenderFrames(mrtEngine* e, uint32_t count, mrtFrameInfo* outInfo) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] { return eng->renderFrames(count, outInfo); });
}

MRT_API mrtResult mrtxTraceRays(mrtEngine* e, const mrtxRay* rays, uint32_t count, mrtxHit* hits) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    if (count && (!rays || !hits)) return MRT_ERROR_INVALID_ARGUMENT;
    return guarded([&] { return eng->traceRays(rays, count, hits); });
}

MRT_API mrtResult mrtxTraceRaysWavefront(mrtEngine* e, const mrtxRay* rays, uint32_t count, mrtxHit* hits) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    if (count && (!rays || !hits)) return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxTraceRaysWavefront: null pointer");
    return guarded([&] { return eng->traceRaysWavefront(rays, count, hits); });
}

MRT_API mrtResult mrtxTraceShadowRays(mrtEngine* e, const mrtxRay* rays, uint32_t count, uint32_t* occluded) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    if (count && (!rays || !occluded)) return MRT_ERROR_INVALID_ARGUMENT;
    return guarded([&] { return eng->traceShadowRays(rays, count, occluded); });
}

MRT_API mrtResult mrtxReadAccumulation(mrtEngine* e, double* dst, size_t dstSize, uint32_t* outSpp) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    if (!dst) return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxReadAccumulation: null destination");
    return guarded([&] { return eng->readAccumulation(dst, dstSize, outSpp); });
}

MRT_API mrtResult mrtxMeasureL2Bandwidth(mrtEngine* e, float* outGBs) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    if (!outGBs) return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxMeasureL2Bandwidth: null output");
    return guarded([&] { return eng->measureL2Bandwidth(outGBs); });
}

MRT_API mrtResult mrtxGetStats(mrtEngine* e, mrtxStats* out) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    // an older, shorter mrtxStats (fields are only ever appended) gets the
    // fields it has
    if (!out || out->structSize < offsetof(mrtxStats, batchJobs))
        return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxGetStats: bad mrtxStats");
    return guarded([&] {
        mrtResult r = eng->flushPending();
        if (r != MRT_SUCCESS) return r;
        mrtxStats full{};
        r = eng->getStats(&full);
        if (r != MRT_SUCCESS) return r;
        const size_t size = std::min(out->structSize, sizeof(mrtxStats));
        std::memcpy(reinterpret_cast<char*>(out) + sizeof(size_t), reinterpret_cast<const char*>(&full) + sizeof(size_t),
                    size - sizeof(size_t));
        return MRT_SUCCESS;
    });
}

MRT_API mrtResult mrtxBuildEnvCdf(mrtEngine* e, const float* rgba, uint32_t w, uint32_t h, float* cdfOut,
                                  float* integralOut) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] { return eng->buildEnvCdf(rgba, w, h, cdfOut, integralOut); });
}

MRT_API mrtResult mrtxSetSampleStream(mrtEngine* e, uint32_t offset, uint32_t stride) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] { return eng->setSampleStream(offset, stride); });
}

MRT_API mrtResult mrtxSetTraversalBudget(mrtEngine* e, uint32_t maxVisits) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] { return eng->setTraversalBudget(maxVisits); });
}

MRT_API mrtResult mrtxSetBvhBuildThresholds(mrtEngine* e, uint32_t minTriangles, uint32_t minInstances) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] { return eng->setBvhBuildThresholds(minTriangles, minInstances); });
}

MRT_API mrtResult mrtxInjectAllocationFailure(int32_t succeedFirst) {
    mrt::setAllocationFailureInjection(succeedFirst);
    return MRT_SUCCESS;
}

MRT_API mrtResult mrtxCopyAccumulationDevice(mrtEngine* e, void* devPtr, size_t bytes, int32_t accumulate) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] { return eng->copyAccumulationDevice(devPtr, bytes, accumulate != 0); });
}

MRT_API mrtResult mrtxBuildWideBvh(const float* aabbs, uint32_t count, uint32_t maxLeafPrims, void* nodesOut,
                                   uint32_t nodeCapacity, uint32_t* primOrderOut, uint32_t* nodeCountOut) {
    if ((count && (!aabbs || !primOrderOut)) || !nodeCountOut || (nodeCapacity && !nodesOut))
        return MRT_ERROR_INVALID_ARGUMENT;
    return guarded([&] {
        std::vector<mrt::Box3> boxes(count);
        for (uint32_t i = 0; i < count; ++i)
            for (int k = 0; k < 3; ++k) {
                boxes[i].lo[k] = aabbs[i * 6 + k];
                boxes[i].hi[k] = aabbs[i * 6 + 3 + k];
            }
        const mrt::WideBvh w = mrt::collapseToWide(mrt::buildBvh(boxes, 1, 4), maxLeafPrims);
        *nodeCountOut = uint32_t(w.nodes.size());
        if (w.nodes.size() > nodeCapacity)
            return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxBuildWideBvh: node capacity too small");
        if (!w.nodes.empty()) std::memcpy(nodesOut, w.nodes.data(), w.nodes.size() * sizeof(MrtWideNode));
        if (count) std::memcpy(primOrderOut, w.primOrder.data(), size_t(count) * 4);
        return MRT_SUCCESS;
    });
}

MRT_API mrtResult mrtxSetRadianceCache(mrtEngine* e, const mrtxRadianceCacheDesc* desc) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    if (!validStruct(desc)) return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxSetRadianceCache: bad descriptor");
    return guarded([&] { return eng->setRadianceCache(*desc); });
}

MRT_API mrtResult mrtxRadianceCacheQuery(mrtEngine* e, const float* features, uint32_t count, float* rgbOut) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    if (count && (!features || !rgbOut)) return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxRadianceCacheQuery: null");
    return guarded([&] { return eng->cacheQuery(features, count, rgbOut); });
}

MRT_API mrtResult mrtxRadianceCacheTrain(mrtEngine* e, const float* features, const float* targets, uint32_t count,
                                         uint32_t steps, float* lossOut) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    if (count && (!features || !targets)) return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxRadianceCacheTrain: null");
    return guarded([&] { return eng->cacheTrain(features, targets, count, steps, lossOut); });
}

MRT_API mrtResult mrtxRadianceCacheGradients(mrtEngine* e, const float* features, const float* targets,
                                             uint32_t count, float* gridGradOut, float* mlpGradOut, float* lossOut) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    if (count && (!features || !targets))
        return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxRadianceCacheGradients: null samples");
    return guarded([&] { return eng->cacheGradients(features, targets, count, gridGradOut, mlpGradOut, lossOut); });
}

MRT_API mrtResult mrtxSetRadianceCacheSchedule(mrtEngine* e, float lrMin, float halfLifeSteps) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] { return eng->setCacheSchedule(lrMin, halfLifeSteps); });
}

MRT_API mrtResult mrtxSetDenoiser(mrtEngine* e, const mrtxDenoiserDesc* d) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    if (!validStruct(d)) return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxSetDenoiser: bad mrtxDenoiserDesc");
    return guarded([&] { return eng->setDenoiser(*d); });
}

MRT_API mrtResult mrtxReadDenoised(mrtEngine* e, float* rgba, size_t bytes) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] { return eng->readDenoised(rgba, bytes); });
}

MRT_API mrtResult mrtxReadDenoiserGuides(mrtEngine* e, float* albedo, float* normalDepth, size_t bytes) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] { return eng->readDenoiserGuides(albedo, normalDepth, bytes); });
}

MRT_API mrtResult mrtxSetRadianceCacheAveraging(mrtEngine* e, float decay) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] { return eng->setCacheAveraging(decay); });
}

MRT_API mrtResult mrtxRadianceCacheParams(mrtEngine* e, float* gridOut, float* mlpOut, const float* gridIn,
                                          const float* mlpIn) {
    mrt::Engine* eng = unwrap(e);
    if (!eng) return MRT_ERROR_INVALID_HANDLE;
    return guarded([&] { return eng->cacheParams(gridOut, mlpOut, gridIn, mlpIn); });
}

MRT_API mrtResult mrtxRenderBatch(mrtEngine* const* engines, const uint32_t* spp, uint32_t count,
                                  mrtFrameInfo* outInfos) {
    if (count && (!engines || !spp)) return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxRenderBatch: null array");
    std::vector<mrt::Engine*> list(count);
    for (uint32_t i = 0; i < count; ++i) {
        list[i] = unwrap(engines[i]);
        if (!list[i]) return mrt::fail(MRT_ERROR_INVALID_HANDLE, "mrtxRenderBatch: null engine");
    }
    return guarded([&] { return mrt::Engine::renderBatch(list.data(), spp, count, outInfos); });
}

MRT_API mrtResult mrtxBuildMeshBvh(mrtEngine* engine, const float* positions, uint32_t vertexCount,
                                   const uint32_t* indices, uint32_t triangleCount, uint32_t builder,
                                   uint32_t maxLeafPrims, void* nodesOut, uint32_t nodeCapacity,
                                   uint32_t* primOrderOut, uint32_t* nodeCountOut) {
    if ((triangleCount && (!positions || !indices || !primOrderOut)) || !nodeCountOut || (nodeCapacity && !nodesOut))
        return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxBuildMeshBvh: null pointer");
    if (builder > MRTX_BVH_DEVICE_LBVH || maxLeafPrims < 1 || maxLeafPrims > 3)
        return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxBuildMeshBvh: unknown builder or leaf size");
    if (builder == MRTX_BVH_DEVICE_LBVH && !engine)
        return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxBuildMeshBvh: the device builder needs an engine");
    for (size_t i = 0; i < size_t(triangleCount) * 3; ++i)
        if (indices[i] >= vertexCount) return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxBuildMeshBvh: index out of range");
    return guarded([&] {
        mrt::WideBvh w;
        if (builder == MRTX_BVH_DEVICE_LBVH) {
            std::vector<mrt::V4f> pos(vertexCount);
            for (uint32_t v = 0; v < vertexCount; ++v)
                pos[v] = mrt::V4f{positions[3 * v], positions[3 * v + 1], positions[3 * v + 2], 1.0f};
            const mrtResult r = unwrap(engine)->buildMeshBvhDevice(pos.data(), pos.size(), indices, triangleCount,
                                                                maxLeafPrims, w);
            if (r != MRT_SUCCESS) return r;
        } else {
            const std::vector<mrt::Box3> boxes = mrt::triangleBoxes(positions, 3, indices, triangleCount);
            w = mrt::collapseToWide(builder == MRTX_BVH_HOST_SAH ? mrt::buildBvh(boxes, 1, 4) : mrt::buildLbvh(boxes),
                                    maxLeafPrims);
        }
        *nodeCountOut = uint32_t(w.nodes.size());
        if (w.nodes.size() > nodeCapacity)
            return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxBuildMeshBvh: node capacity too small");
        if (!w.nodes.empty()) std::memcpy(nodesOut, w.nodes.data(), w.nodes.size() * sizeof(MrtWideNode));
        if (triangleCount) std::memcpy(primOrderOut, w.primOrder.data(), size_t(triangleCount) * 4);
        return MRT_SUCCESS;
    });
}

// Allocation-free CDF: device pointers in and out, scratch in the static
// device array of csrc/cuda/frame.cu. The sin(theta) table is the one
// Engine::runEnvCdf builds (same float expression), held on this thread's
// stack and handed to the device as kernel parameters.
MRT_API mrtResult mrtxBuildEnvCdfNoAlloc(const float* devTexels, uint32_t w, uint32_t h, float* devCdfOut,
                                         float* devIntegralOut, void* stream) {
    if (!devTexels || !devCdfOut || !devIntegralOut || w == 0 || h == 0)
        return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxBuildEnvCdfNoAlloc: null pointer or empty image");
    if (h > MRTX_ENV_CDF_NOALLOC_MAX_HEIGHT)
        return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxBuildEnvCdfNoAlloc: height " + std::to_string(h) +
                                                         " exceeds the maximum of " +
                                                         std::to_string(MRTX_ENV_CDF_NOALLOC_MAX_HEIGHT) + " rows");
    // The row kernel reads texels as 16-byte vectors and the outputs are
    // written as floats: a pointer carved out of a caller's pool at a finer
    // offset would fault on the device (a sticky error that ends the
    // caller's context), so it is refused here, before anything launches.
    if (reinterpret_cast<uintptr_t>(devTexels) % 16 != 0 || reinterpret_cast<uintptr_t>(devCdfOut) % 4 != 0 ||
        reinterpret_cast<uintptr_t>(devIntegralOut) % 4 != 0)
        return mrt::fail(MRT_ERROR_INVALID_ARGUMENT,
                         "mrtxBuildEnvCdfNoAlloc: devTexels must be 16-byte aligned and the outputs 4-byte aligned");
    int device = -1;
    for (const void* ptr : {static_cast<const void*>(devTexels), static_cast<const void*>(devCdfOut),
                            static_cast<const void*>(devIntegralOut)}) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess ||
            (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)) {
            cudaGetLastError();
            return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxBuildEnvCdfNoAlloc: a pointer is not device memory");
        }
        if (device >= 0 && at.device != device)
            return mrt::fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxBuildEnvCdfNoAlloc: pointers on different GPUs");
        device = at.device;
    }
    int previous = -1;
    MRT_CUDA(cudaGetDevice(&previous));
    if (previous != device) MRT_CUDA(cudaSetDevice(device));
    float sinTheta[MRTX_ENV_CDF_NOALLOC_MAX_HEIGHT];
    const float pi = 3.14159265358979323846f;
    const float dTheta = pi / float(h);
    for (uint32_t y = 0; y < h; ++y) sinTheta[y] = std::sin((float(y) + 0.5f) * dTheta);
    unsigned char* scratch = nullptr;
    cudaError_t e = mrtcu_env_cdf_noalloc_setup(device, &scratch);
    if (e == cudaSuccess)
        e = mrtcu_env_cdf_noalloc(scratch, reinterpret_cast<const float4*>(devTexels), sinTheta, w, h, devCdfOut,
                                  devIntegralOut, static_cast<cudaStream_t>(stream));
    if (previous != device) cudaSetDevice(previous);
    if (e != cudaSuccess) return mrt::fromCuda(e, "mrtxBuildEnvCdfNoAlloc");
    return MRT_SUCCESS;
}

}  // extern "C"
