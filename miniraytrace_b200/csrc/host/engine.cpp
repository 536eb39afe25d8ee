// Engine implementation: commit (packing, BVH builds, environment CDF),
// rendering, readback. Reference behaviour is cited per function.
#include "engine.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <atomic>
#include <future>
#include <thread>

#include "../cuda/device_api.h"

namespace mrt {

// ---------------------------------------------------------------- buffers --

namespace {
std::atomic<int64_t> g_allocBudget{-1};  // -1: no injected failures
}

void setAllocationFailureInjection(int64_t succeedFirst) { g_allocBudget.store(succeedFirst < 0 ? -1 : succeedFirst); }

bool allocationFailureInjected() {
    int64_t v = g_allocBudget.load();
    while (v >= 0) {
        if (v == 0) return true;
        if (g_allocBudget.compare_exchange_weak(v, v - 1)) return false;
    }
    return false;
}

mrtResult DeviceBuffer::ensure(size_t n) {
    n = std::max<size_t>(n, 16);
    if (ptr && bytes >= n) return MRT_SUCCESS;
    // grow by 1.5x like the reference's scene buffers (Renderer.cpp:323-330)
    const size_t cap = std::max(n, bytes + bytes / 2);
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    if (allocationFailureInjected()) return fromCuda(cudaErrorMemoryAllocation, "cudaMalloc (injected failure)");
    MRT_CUDA(cudaMalloc(&ptr, cap));
    bytes = cap;
    return MRT_SUCCESS;
}

mrtResult DeviceBuffer::upload(const void* src, size_t n, cudaStream_t s) {
    MRT_TRY(ensure(n));
    if (n) MRT_CUDA(cudaMemcpyAsync(ptr, src, n, cudaMemcpyHostToDevice, s));
    return MRT_SUCCESS;
}

void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

namespace {

// Jobs of one mrtxRenderBatch running on the GPU at once.
#ifndef MRT_BATCH_WINDOW
#define MRT_BATCH_WINDOW 4
#endif
constexpr uint32_t kBatchWindow = MRT_BATCH_WINDOW;

// Largest batch of one radiance-cache training step.
constexpr uint32_t kCacheMaxBatch = 65536;

// Path state per wave slot: rayO, rayD, beta, L, hit (5 x 16 B), hitInst +
// two queues (3 x 4 B), shadow origin/dir/contribution (3 x 16 B).
constexpr size_t kWaveBytesPerSlot = 5 * 16 + 3 * 4 + 3 * 16;

// Default build sites (mrtxSetBvhBuildThresholds changes them per engine).
// Meshes with at least this many triangles get their BLAS built on the GPU
// (LBVH topology, about 4% above the binned-SAH tree's cost on a terrain
// heightfield); smaller meshes keep the host's binned-SAH build, on host
// threads beside the device builds. Instance sets of at least this many
// instances get their TLAS built on the GPU by the same builder. Measured on
// a B200 host: a 44,402-triangle heightfield under 2,501 instances builds in
// 2.6 ms on the device against 34.5 ms on the host, its instance tree alone
// in 0.8 against 3.6 ms. Smaller meshes and instance sets keep the host's
// SAH trees, which are slightly cheaper to trace.
constexpr uint32_t kDeviceBuildMinTriangles = 16384;
constexpr uint32_t kDeviceBuildMinInstances = 2048;

// A wide node with no children: the TLAS root of an empty scene (the
// reference parks an inverted-box sentinel there, Renderer.cpp:49-58).
MrtWideNode emptyNode() {
    MrtWideNode n;
    std::memset(&n, 0, sizeof(n));
    return n;
}

inline float clamp01(float x) { return std::min(std::max(x, 0.0f), 1.0f); }

void normalize3(float v[3]) {
    const float inv = 1.0f / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] *= inv;
    v[1] *= inv;
    v[2] *= inv;
}
void cross3(const float a[3], const float b[3], float r[3]) {
    r[0] = a[1] * b[2] - b[1] * a[2];
    r[1] = a[2] * b[0] - b[2] * a[0];
    r[2] = a[0] * b[1] - b[0] * a[1];
}

// Inverse of a row-major affine 3x4 [R | t] in single precision: with the
// columns c0, c1, c2 of R, the rows of R^-1 are (c1 x c2, c2 x c0, c0 x c1) /
// det, det = c0 . (c1 x c2), and the translation becomes -R^-1 t. (The
// reference inverts with glm::inverse, Renderer.cpp:475; both are exact for
// identity and translate/scale-by-power-of-two transforms.)
void invertAffine(const float m[12], float out[12]) {
    const float c0[3] = {m[0], m[4], m[8]}, c1[3] = {m[1], m[5], m[9]}, c2[3] = {m[2], m[6], m[10]};
    float r0[3], r1[3], r2[3];
    cross3(c1, c2, r0);
    cross3(c2, c0, r1);
    cross3(c0, c1, r2);
    const float invDet = 1.0f / (c0[0] * r0[0] + c0[1] * r0[1] + c0[2] * r0[2]);
    const float* rows[3] = {r0, r1, r2};
    const float t[3] = {m[3], m[7], m[11]};
    for (int row = 0; row < 3; ++row) {
        const float i0 = rows[row][0] * invDet, i1 = rows[row][1] * invDet, i2 = rows[row][2] * invDet;
        out[row * 4 + 0] = i0;
        out[row * 4 + 1] = i1;
        out[row * 4 + 2] = i2;
        out[row * 4 + 3] = -(i0 * t[0] + i1 * t[1] + i2 * t[2]);
    }
}

// World bounds of a box under a row-major 3x4 transform (8 corners, as
// reference MathTypes.hpp:35-45).
Box3 transformBox(const Box3& b, const float m[12]) {
    Box3 o;
    for (int k = 0; k < 3; ++k) {
        o.lo[k] = 3.402823466e38f;
        o.hi[k] = -3.402823466e38f;
    }
    for (int i = 0; i < 8; ++i) {
        const float c[3] = {(i & 1) ? b.hi[0] : b.lo[0], (i & 2) ? b.hi[1] : b.lo[1], (i & 4) ? b.hi[2] : b.lo[2]};
        for (int r = 0; r < 3; ++r) {
            const float v = m[r * 4] * c[0] + m[r * 4 + 1] * c[1] + m[r * 4 + 2] * c[2] + m[r * 4 + 3];
            o.lo[r] = std::min(o.lo[r], v);
            o.hi[r] = std::max(o.hi[r], v);
        }
    }
    return o;
}

}  // namespace

// Upload that counts the bytes a commit moves host-to-device.
mrtResult Engine::up(DeviceBuffer& b, const void* src, size_t n) {
    m_stats.commitH2DBytes += n;
    if (n < kStageChunk) return b.upload(src, n, m_stream);
    MRT_TRY(b.ensure(n));
    return uploadStaged(b.ptr, src, n);
}

// Host -> pinned staging -> device for large uploads: the copy pool's
// threads fill one 4 MB pinned slot while the DMA out of the previous slots
// runs (a copy straight from pageable memory moves ~10 GB/s; this one is
// bound by the host threads' copy).
mrtResult Engine::uploadStaged(void* dst, const void* src, size_t n) {
    if (!m_stage) {
        if (allocationFailureInjected()) return fromCuda(cudaErrorMemoryAllocation, "cudaMallocHost (injected failure)");
        MRT_CUDA(cudaMallocHost(&m_stage, kStageChunk * kStageSlots));
        for (auto& ev : m_stageCopyEvents) MRT_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    for (size_t c = 0, off = 0; off < n; ++c, off += kStageChunk) {
        const size_t len = std::min(kStageChunk, n - off), slot = c % kStageSlots;
        char* stage = static_cast<char*>(m_stage) + slot * kStageChunk;
        if (m_stageUsed[slot]) MRT_CUDA(cudaEventSynchronize(m_stageCopyEvents[slot]));
        m_copyPool->copy(stage, static_cast<const char*>(src) + off, len);
        MRT_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + off, stage, len, cudaMemcpyHostToDevice, m_stream));
        MRT_CUDA(cudaEventRecord(m_stageCopyEvents[slot], m_stream));
        m_stageUsed[slot] = true;
    }
    return MRT_SUCCESS;
}

// ------------------------------------------------------------- lifecycle --

mrtResult Engine::create(const mrtEngineDesc& desc, Engine** out) {
    Engine* e = new Engine();
    const mrtResult r = e->init(desc);
    if (r != MRT_SUCCESS) {
        delete e;
        return r;
    }
    *out = e;
    return MRT_SUCCESS;
}

mrtResult Engine::init(const mrtEngineDesc& desc) {
    if (desc.width > 0 && desc.height > 0) {
        m_settings.width = desc.width;
        m_settings.height = desc.height;
    }
    m_validation = desc.enableValidation != 0;
    m_hostThreads = std::max(1u, std::thread::hardware_concurrency());
    m_copyPool = std::make_unique<CopyPool>(std::min(5u, m_hostThreads - 1));
    int count = 0;
    const cudaError_t ce = cudaGetDeviceCount(&count);
    if (ce != cudaSuccess || count == 0)
        return fail(MRT_ERROR_VULKAN_INIT,
                    std::string("No CUDA device available (") + (ce != cudaSuccess ? cudaGetErrorString(ce) : "0 devices") +
                        "). This build needs an NVIDIA B200-class GPU (sm_100a) and driver.");
    for (int i = 0; i < count; ++i) {
        cudaDeviceProp p{};
        if (cudaGetDeviceProperties(&p, i) == cudaSuccess)
            log(LogLevel::Info, "CUDA device [" + std::to_string(i) + "]: " + p.name + " (sm_" +
                                    std::to_string(p.major) + std::to_string(p.minor) + ", " +
                                    std::to_string(p.multiProcessorCount) + " SMs)");
    }
    if (desc.gpuIndex1 > 0) {
        const uint32_t idx = desc.gpuIndex1 - 1;
        if (idx >= uint32_t(count))
            return fail(MRT_ERROR_VULKAN_INIT, "Requested GPU index " + std::to_string(idx) + " is out of range (" +
                                                   std::to_string(count) + " device(s) found).");
        m_device = int(idx);
    } else {
        m_device = 0;
    }
    const cudaError_t se = cudaSetDevice(m_device);
    if (se != cudaSuccess)
        return fail(MRT_ERROR_VULKAN_INIT, std::string("cudaSetDevice failed: ") + cudaGetErrorString(se));
    cudaDeviceProp prop{};
    MRT_CUDA(cudaGetDeviceProperties(&prop, m_device));
    // paths in flight per wave: 2^27 (64 spp of a 1080p frame, 18.8 GB of
    // path state; one wave per 64-spp step leaves one set of short
    // late-bounce launches instead of one per wave), at most a quarter of
    // the GPU's memory
    m_maxWaveSlots = std::max<uint64_t>(1u << 20, std::min<uint64_t>(uint64_t(1) << 27,
                                                                      prop.totalGlobalMem / 4 / kWaveBytesPerSlot));
    if (prop.major != 10)
        return fail(MRT_ERROR_SHADER_LOAD, std::string("GPU ") + prop.name + " (sm_" + std::to_string(prop.major) +
                                               std::to_string(prop.minor) +
                                               ") cannot run this library's kernels, which are compiled for sm_100a only.");
    MRT_CUDA(cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking));
    MRT_CUDA(cudaStreamCreateWithFlags(&m_side, cudaStreamNonBlocking));
    MRT_CUDA(cudaEventCreate(&m_ev0));
    MRT_CUDA(cudaEventCreate(&m_ev1));
    m_copyEvents.resize(16);
    for (auto& ev : m_copyEvents) MRT_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    log(LogLevel::Info, std::string("GPU: ") + prop.name);

    // pre-commit frames traverse an empty scene safely
    const MrtWideNode s = emptyNode();
    MRT_TRY(m_nodes.upload(&s, sizeof(s), m_stream));
    m_nodeCount = 1;
    m_tlasRoot = 0;
    const MrtMaterial defMat{{0.8f, 0.8f, 0.8f, 1.0f}, {0, 0, 0, 0.5f}, {0, 0, 1.45f, 0}, {-1, -1, -1, -1, -1, -1, -1, -1}};
    MRT_TRY(m_materials.upload(&defMat, sizeof(defMat), m_stream));
    std::vector<MrtTexture> table(MRT_MAX_TEXTURES);
    std::memset(table.data(), 0, table.size() * sizeof(MrtTexture));
    MRT_TRY(m_texTable.upload(table.data(), table.size() * sizeof(MrtTexture), m_stream));
    // sRGB decode of the 256 channel values, with the same expression as the
    // sampler's format conversion in the CPU evaluation of the shaders
    // (power in double, rounded to float); the kernels look it up
    float lut[256];
    for (int k = 0; k < 256; ++k) {
        const float c = float(k) / 255.0f;
        lut[k] = c <= 0.04045f ? c / 12.92f : float(std::pow(double((c + 0.055f) / 1.055f), 2.4));
    }
    MRT_TRY(m_srgbLut.upload(lut, sizeof(lut), m_stream));
    m_texGeneration.assign(MRT_MAX_TEXTURES, 0);
    const float black[4] = {0, 0, 0, 1};
    MRT_TRY(m_envTexels.upload(black, sizeof(black), m_stream));
    MRT_TRY(m_envCdf.ensure(16));
    // 1-vertex placeholders so every pointer in the parameter block is valid
    MRT_TRY(m_triVerts.ensure(48));
    MRT_TRY(m_triIndex.ensure(16));
    MRT_TRY(m_normals.ensure(16));
    MRT_TRY(m_uvs.ensure(16));
    MRT_TRY(m_tangents.ensure(16));
    MRT_TRY(m_instances.ensure(sizeof(MrtInstance)));
    MRT_TRY(m_lights.ensure(sizeof(MrtLight)));
    MRT_TRY(m_flags.ensure(16));
    MRT_CUDA(cudaMemsetAsync(m_flags.ptr, 0, 16, m_stream));
    MRT_TRY(m_rayCounters.ensure(128));
    MRT_CUDA(cudaMemsetAsync(m_rayCounters.ptr, 0, 128, m_stream));
    MRT_TRY(allocateFrame());
    MRT_CUDA(cudaStreamSynchronize(m_stream));
    m_stats.structSize = sizeof(mrtxStats);
    return MRT_SUCCESS;
}

Engine::~Engine() {
    if (m_stream) {
        cudaSetDevice(m_device);
        cudaStreamSynchronize(m_stream);
        if (m_side) cudaStreamSynchronize(m_side);
    }
    DeviceBuffer* bufs[] = {&m_nodes,     &m_triVerts, &m_triIndex,   &m_normals,      &m_uvs,        &m_tangents,
                            &m_instances, &m_materials, &m_lights,     &m_envTexels,    &m_envCdf,     &m_envSin,
                            &m_envRowSums, &m_envIntegral, &m_texTable, &m_accum,       &m_out32,      &m_out8,
                            &m_flags,     &m_rayCounters, &m_queryRays, &m_queryOut, &m_wave,
                            &m_bvhPos,    &m_bvhIdx,    &m_bvhScratch, &m_bvhNodes,    &m_bvhPrims,
                            &m_packError, &m_srgbLut, &m_batchJobs};
    for (DeviceBuffer* b : bufs) b->release();
    for (auto& [id, b] : m_blas) b.release();
    m_cache.release();
    m_denoiser.release();
    for (auto& t : m_texData) t.release();
    if (m_pinned) cudaFreeHost(m_pinned);
    if (m_stage) cudaFreeHost(m_stage);
    for (auto& ev : m_stageCopyEvents)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : m_copyEvents)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : m_stageEvents)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : m_syncEvents)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : m_cacheEvents)
        if (ev) cudaEventDestroy(ev);
    if (m_ev0) cudaEventDestroy(m_ev0);
    if (m_ev1) cudaEventDestroy(m_ev1);
    if (m_side) cudaStreamDestroy(m_side);
    if (m_stream) cudaStreamDestroy(m_stream);
}

mrtResult Engine::checkAlive() {
    if (m_lost)
        return fail(MRT_ERROR_DEVICE_LOST, "The CUDA context of this engine hit an unrecoverable error; destroy it.");
    const cudaError_t e = cudaSetDevice(m_device);
    if (e != cudaSuccess) return guard(fromCuda(e, "cudaSetDevice"));
    return MRT_SUCCESS;
}

mrtResult Engine::guard(mrtResult r) {
    if (r == MRT_ERROR_DEVICE_LOST) m_lost = true;
    return r;
}

mrtResult Engine::allocateFrame() {
    const size_t pixels = size_t(m_settings.width) * m_settings.height;
    m_waveSamples = 0;  // wave slots depend on the frame size
    MRT_TRY(m_accum.ensure(pixels * 32));
    MRT_CUDA(cudaMemsetAsync(m_accum.ptr, 0, pixels * 32, m_stream));
    MRT_TRY(m_out32.ensure(pixels * 16));
    MRT_TRY(m_out8.ensure(pixels * 4));
    return MRT_SUCCESS;
}

// Wavefront state for waves of up to `samples` samples per pixel, capped so
// a wave holds at most 2^25 paths (~4.7 GB of state at 140 bytes a path):
// large waves amortise the last bounces, whose few long rays run at the
// latency of one traversal.
mrtResult Engine::ensureWave(uint32_t samples) {
    const uint64_t pixels = uint64_t(m_settings.width) * m_settings.height;
    // at most half of the device memory free now (other engines may share
    // the GPU), counting this engine's current wave allocation as free
    size_t freeBytes = 0, totalBytes = 0;
    MRT_CUDA(cudaMemGetInfo(&freeBytes, &totalBytes));
    const uint64_t budget = (uint64_t(freeBytes) + m_wave.bytes) / 2 / kWaveBytesPerSlot;
    const uint64_t maxSlots = std::max<uint64_t>(pixels, std::min<uint64_t>(m_maxWaveSlots, budget));
    uint32_t k = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(samples, maxSlots / std::max<uint64_t>(pixels, 1))));
    k = std::min<uint32_t>(k, 64);
    if (m_waveSamples >= k) return MRT_SUCCESS;
    const uint64_t slots = pixels * k;
    if (slots > 0xffffffffull) return fail(MRT_ERROR_INVALID_ARGUMENT, "frame too large for one wave");
    // growing frees the old allocation first: forget the carved pointers
    // before, so a failed allocation leaves no wave state that points into
    // freed memory (the next call allocates again)
    m_waveSamples = 0;
    m_waveState = MrtWaveState{};
    MRT_TRY(carveWave(slots, m_waveState));
    m_waveSamples = k;
    return MRT_SUCCESS;
}

// A wave state of `slots` paths carved out of m_wave, grown as needed (when
// it grows, this engine's own carved state is forgotten first; its next
// ensureWave carves it again).
mrtResult Engine::carveWave(uint64_t slots, MrtWaveState& w) {
    const size_t bytes = size_t(slots) * kWaveBytesPerSlot + 64;
    if (m_wave.bytes < bytes) {
        m_waveSamples = 0;
        m_waveState = MrtWaveState{};
    }
    MRT_TRY(m_wave.ensure(bytes));
    char* base = static_cast<char*>(m_wave.ptr);
    auto carve = [&](size_t n) {
        char* p = base;
        base += n;
        return p;
    };
    w.rayO = reinterpret_cast<float4*>(carve(slots * 16));
    w.rayD = reinterpret_cast<float4*>(carve(slots * 16));
    w.beta = reinterpret_cast<float4*>(carve(slots * 16));
    w.L = reinterpret_cast<float4*>(carve(slots * 16));
    w.hit = reinterpret_cast<float4*>(carve(slots * 16));
    w.shO = reinterpret_cast<float4*>(carve(slots * 16));
    w.shD = reinterpret_cast<float4*>(carve(slots * 16));
    w.shC = reinterpret_cast<float4*>(carve(slots * 16));
    w.hitInst = reinterpret_cast<uint32_t*>(carve(slots * 4));
    w.queue[0] = reinterpret_cast<uint32_t*>(carve(slots * 4));
    w.queue[1] = reinterpret_cast<uint32_t*>(carve(slots * 4));
    w.counts = reinterpret_cast<uint32_t*>(carve(64));
    w.capacity = uint32_t(slots);
    return MRT_SUCCESS;
}

// ---------------------------------------------------------------- settings --

// reference Renderer.cpp:115-127: a resize reallocates; resize, maxBounces or
// fireflyClamp changes restart accumulation.
mrtResult Engine::setSettings(const Settings& s) {
    MRT_TRY(checkAlive());
    if (s.width == 0 || s.height == 0) return fail(MRT_ERROR_INVALID_ARGUMENT, "render size must be non-zero");
    const bool resize = s.width != m_settings.width || s.height != m_settings.height;
    const bool reset = resize || s.maxBounces != m_settings.maxBounces || s.fireflyClamp != m_settings.fireflyClamp;
    if (reset) m_pending = 0;  // dropped before any frame buffer is replaced
    m_settings = s;
    if (resize) MRT_TRY(guard(allocateFrame()));
    if (reset) resetAccumulation();
    return MRT_SUCCESS;
}

void Engine::resetAccumulation() {
    m_frameIndex = 0;
    m_pending = 0;  // queued samples would be discarded by the reset anyway
    // the reference's reset of its denoiser state (Renderer.cpp:766-769)
    m_denoiser.guidesValid = false;
    m_denoiser.useDenoised = false;
    m_denoiser.nextAt = m_denoiser.minSpp;
    m_denoiser.denoisedSpp = 0;
}

mrtResult Engine::setSampleStream(uint32_t offset, uint32_t stride) {
    if (stride == 0) return fail(MRT_ERROR_INVALID_ARGUMENT, "sample stream stride must be >= 1");
    m_streamOffset = offset;
    m_streamStride = stride;
    resetAccumulation();
    return MRT_SUCCESS;
}

// ------------------------------------------------------------------ commit --

// reference Engine.cpp:44-55: camera/env-parameter-only changes restart
// accumulation without touching device scene data.
mrtResult Engine::commit(mrtCommitStats* stats) {
    MRT_TRY(checkAlive());
    const uint32_t light = DirtyCamera | DirtyEnvParams;
    const uint32_t d = m_scene.dirty();
    // every commit that changes something resets the accumulation: queued
    // samples are dropped before any device array is replaced
    if (d != DirtyNone) m_pending = 0;
    if (d != DirtyNone && (d & ~light) == 0) {
        m_scene.clearDirty();
        resetAccumulation();
        if (stats) {
            stats->blasRebuilt = 0;
            stats->tlasRebuilt = 0;
            stats->commitMs = 0.0f;
        }
        return MRT_SUCCESS;
    }
    return guard(sync(stats));
}

// reference Renderer.cpp:290-320
mrtResult Engine::sync(mrtCommitStats* stats) {
    const TraceRange range("mrt commit");
    const auto t0 = std::chrono::steady_clock::now();
    const uint32_t dirty = m_scene.dirty();
    if (dirty == DirtyNone) {
        if (stats) {
            stats->blasRebuilt = 0;
            stats->tlasRebuilt = 0;
            stats->commitMs = 0.0f;
        }
        return MRT_SUCCESS;
    }
    MRT_CUDA(cudaStreamSynchronize(m_stream));
    uint32_t rebuilt = 0;
    m_stats.commitBvhMs = 0.0f;
    m_stats.commitDeviceBlas = 0;
    m_stats.commitDeviceTlas = 0;
    m_stats.commitEnvCdfMs = 0.0f;
    m_stats.commitUploadMs = 0.0f;
    m_stats.commitH2DBytes = 0;
    if (dirty & DirtyTextures) MRT_TRY(uploadTextures());
    if (dirty & DirtyMaterials) MRT_TRY(packMaterials());
    const bool tangents = (dirty & (DirtyGeometry | DirtyInstances | DirtyMaterials)) && ensureTangents();
    if ((dirty & DirtyGeometry) || tangents) MRT_TRY(packGeometry(rebuilt));
    const bool tlas = (dirty & (DirtyGeometry | DirtyInstances | DirtyMaterials)) != 0;
    if (tlas) MRT_TRY(packInstances());
    if (dirty & DirtyEnv) MRT_TRY(packEnvironment());
    if (dirty & (DirtyLights | DirtyEnv)) MRT_TRY(packLights());
    MRT_CUDA(cudaStreamSynchronize(m_stream));
    m_scene.clearDirty();
    resetAccumulation();
    const float ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    m_stats.commitTotalMs = ms;
    if (stats) {
        stats->blasRebuilt = rebuilt;
        stats->tlasRebuilt = tlas ? 1 : 0;
        stats->commitMs = ms;
    }
    return MRT_SUCCESS;
}

// Tangents for every mesh with uvs that an instance draws with a material
// naming a normal texture, computed once per vertex data (on host threads,
// a mesh at a time). Returns whether any were computed (their meshes' device
// tangents and the global attribute arrays need refreshing).
bool Engine::ensureTangents() {
    auto& meshes = m_scene.meshes();
    std::vector<MeshData*> todo;
    for (const auto& [iid, in] : m_scene.instances()) {
        const auto mt = m_scene.materials().find(in.material);
        if (mt == m_scene.materials().end() || mt->second.tex[3] == MRT_INVALID_ID) continue;
        auto it = meshes.find(in.mesh);
        if (it == meshes.end() || it->second.uvs.empty() || it->second.tangentsDone) continue;
        it->second.tangentsDone = true;  // (an instance list may name a mesh twice)
        todo.push_back(&it->second);
    }
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (size_t k; (k = next.fetch_add(1)) < todo.size();) {
            Scene::computeTangents(*todo[k]);
            todo[k]->tangentsPending = true;
        }
    };
    std::vector<std::thread> pool;
    for (size_t t = 1; t < std::min<size_t>(todo.size(), m_hostThreads); ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    return !todo.empty();
}

// reference Renderer.cpp:510-550 (clamps, default material at index 0, texture
// ids resolved to slots, -1 for none)
mrtResult Engine::packMaterials() {
    std::vector<MrtMaterial> mats;
    mats.reserve(m_scene.materials().size() + 1);
    MrtMaterial def{{0.8f, 0.8f, 0.8f, 1.0f}, {0, 0, 0, 0.5f}, {0, 0, 1.45f, 0}, {-1, -1, -1, -1, -1, -1, -1, -1}};
    mats.push_back(def);
    m_materialIndex.clear();
    for (const auto& [id, m] : m_scene.materials()) {
        MrtMaterial g{};
        g.baseColorOpacity[0] = m.baseColor[0];
        g.baseColorOpacity[1] = m.baseColor[1];
        g.baseColorOpacity[2] = m.baseColor[2];
        g.baseColorOpacity[3] = m.opacity;
        g.emissionRoughness[0] = m.emission[0];
        g.emissionRoughness[1] = m.emission[1];
        g.emissionRoughness[2] = m.emission[2];
        g.emissionRoughness[3] = clamp01(m.roughness);
        g.params[0] = clamp01(m.metallic);
        g.params[1] = clamp01(m.transmission);
        g.params[2] = std::max(m.ior, 1.0f);
        g.params[3] = 0.0f;
        for (int k = 0; k < 8; ++k) g.tex[k] = -1;
        for (int k = 0; k < 5; ++k) {
            const uint32_t slot = m_scene.textureSlot(m.tex[k]);
            g.tex[k] = (slot == ~0u || slot >= MRT_MAX_TEXTURES) ? -1 : int32_t(slot);
        }
        m_materialIndex[id] = uint32_t(mats.size());
        mats.push_back(g);
    }
    m_materialCount = uint32_t(mats.size());
    return up(m_materials, mats.data(), mats.size() * sizeof(MrtMaterial));
}

void Engine::Blas::release() {
    for (DeviceBuffer* d : {&pos, &idx, &normals, &uvs, &tangents, &nodes, &prims}) d->release();
}

size_t Engine::Blas::deviceBytes() const {
    size_t n = 0;
    for (const DeviceBuffer* d : {&pos, &idx, &normals, &uvs, &tangents, &nodes, &prims}) n += d->bytes;
    return n;
}

// A changed mesh's vertex data and indices into its own device buffers
// (missing uvs become zeros, missing tangents (1, 0, 0, 1), as the reference
// packs them).
mrtResult Engine::uploadMesh(const MeshData& m, Blas& b) {
    const size_t nv = m.positions.size(), nt = m.indices.size() / 3;
    b.vertexCount = uint32_t(nv);
    b.triCount = uint32_t(nt);
    MRT_TRY(up(b.pos, m.positions.data(), nv * sizeof(V4f)));
    MRT_TRY(up(b.idx, m.indices.data(), nt * 3 * sizeof(uint32_t)));
    MRT_TRY(up(b.normals, m.normals.data(), nv * sizeof(V4f)));
    if (m.uvs.empty()) {
        MRT_TRY(b.uvs.ensure(nv * sizeof(V2f)));
        MRT_CUDA(cudaMemsetAsync(b.uvs.ptr, 0, nv * sizeof(V2f), m_stream));
    } else {
        MRT_TRY(up(b.uvs, m.uvs.data(), nv * sizeof(V2f)));
    }
    if (m.tangents.empty()) {
        MRT_TRY(b.tangents.ensure(nv * sizeof(V4f)));
        MRT_CUDA(mrtcu_fill_f4(b.tangents.as<float4>(), nv, make_float4(1.0f, 0.0f, 0.0f, 1.0f), m_stream));
    } else {
        MRT_TRY(up(b.tangents, m.tangents.data(), nv * sizeof(V4f)));
    }
    return MRT_SUCCESS;
}

// BVH of a mesh whose arrays are on the device, built there and copied into
// the mesh's own node / order buffers (exactly sized).
mrtResult Engine::buildBlasOnDevice(Blas& b) {
    uint32_t count = 0;
    MRT_TRY(buildBvhOnDevice(b.pos.as<float4>(), b.idx.as<uint32_t>(), b.triCount, 3, count, b.bounds));
    b.nodeCount = count;
    MRT_TRY(b.nodes.ensure(size_t(count) * sizeof(MrtWideNode)));
    MRT_TRY(b.prims.ensure(size_t(b.triCount) * sizeof(uint32_t)));
    MRT_CUDA(cudaMemcpyAsync(b.nodes.ptr, m_bvhNodes.ptr, size_t(count) * sizeof(MrtWideNode),
                             cudaMemcpyDeviceToDevice, m_stream));
    MRT_CUDA(cudaMemcpyAsync(b.prims.ptr, m_bvhPrims.ptr, size_t(b.triCount) * sizeof(uint32_t),
                             cudaMemcpyDeviceToDevice, m_stream));
    return MRT_SUCCESS;
}

// reference Renderer.cpp:333-446: rebuild dirty BLASes, then repack every
// mesh into the global arrays in id order with triangles in BLAS leaf order
// and node indices rebased. Here a changed mesh is uploaded once to its own
// device buffers; large meshes get their BVH built on the GPU from those,
// small ones on host threads (concurrently); the global arrays are then
// assembled on the device (node rebase, triangle gather, attribute copies).
mrtResult Engine::packGeometry(uint32_t& rebuilt) {
    const TraceRange range("mrt commit: meshes");
    auto& meshes = m_scene.meshes();
    for (auto it = m_blas.begin(); it != m_blas.end();) {
        if (meshes.count(it->first)) {
            ++it;
            continue;
        }
        it->second.release();
        it = m_blas.erase(it);
    }
    std::vector<uint32_t> changed;
    for (auto& [id, mesh] : meshes)
        if (mesh.blasDirty || !m_blas.count(id)) changed.push_back(id);

    const auto tu = std::chrono::steady_clock::now();
    for (uint32_t id : changed) {
        MRT_TRY(uploadMesh(meshes[id], m_blas[id]));
        meshes[id].tangentsPending = false;
    }
    for (auto& [id, mesh] : meshes) {  // tangents computed since the mesh's upload
        if (!mesh.tangentsPending) continue;
        mesh.tangentsPending = false;
        MRT_TRY(up(m_blas[id].tangents, mesh.tangents.data(), mesh.tangents.size() * sizeof(V4f)));
    }
    m_stats.commitUploadMs += std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - tu).count();

    const auto tb = std::chrono::steady_clock::now();
    std::vector<std::pair<uint32_t, std::future<WideBvh>>> jobs;
    const unsigned threads = m_hostThreads;
    const size_t minDevice = m_deviceMinTriangles ? m_deviceMinTriangles : kDeviceBuildMinTriangles;
    for (uint32_t id : changed) {
        MeshData* m = &meshes[id];
        if (m->indices.size() / 3 >= minDevice) continue;
        jobs.emplace_back(id, std::async(std::launch::async, [m, threads] {
                              const std::vector<Box3> boxes = triangleBoxes(
                                  &m->positions[0].x, 4, m->indices.data(), m->indices.size() / 3);
                              // binary SAH tree down to single triangles, collapsed to
                              // 8-wide nodes with leaves of up to 3 triangles
                              return collapseToWide(buildBvh(boxes, 1, threads), 3);
                          }));
    }
    // large meshes on the GPU, while the host builds the small ones
    for (uint32_t id : changed)
        if (meshes[id].indices.size() / 3 >= minDevice) {
            MRT_TRY(buildBlasOnDevice(m_blas[id]));
            ++m_stats.commitDeviceBlas;
        }
    for (auto& [id, fut] : jobs) {
        const WideBvh w = fut.get();
        Blas& b = m_blas[id];
        b.nodeCount = uint32_t(w.nodes.size());
        b.bounds = w.bounds;
        if (!w.nodes.empty()) MRT_TRY(up(b.nodes, w.nodes.data(), w.nodes.size() * sizeof(MrtWideNode)));
        if (!w.primOrder.empty()) MRT_TRY(up(b.prims, w.primOrder.data(), w.primOrder.size() * sizeof(uint32_t)));
    }
    for (uint32_t id : changed) meshes[id].blasDirty = false;
    rebuilt = uint32_t(changed.size());
    m_stats.commitBvhMs += std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - tb).count();

    // global layout in mesh id order
    const auto ta = std::chrono::steady_clock::now();
    size_t nv = 0, nt = 0, nn = 0;
    for (auto& [id, b] : m_blas) {
        b.nodeBase = uint32_t(nn);
        nv += b.vertexCount;
        nt += b.triCount;
        nn += b.nodeCount;
    }
    if (nt > 0x7fffffffu / 3 || nv > 0xffffffffu || nn > 0xffffffffu)
        return fail(MRT_ERROR_INVALID_ARGUMENT, "scene too large");
    // node buffer keeps room for the TLAS (at most one wide node per instance) behind the BLAS region
    const size_t tlasCap = std::max<size_t>(m_scene.instances().size() + 1, 4);
    MRT_TRY(m_nodes.ensure((nn + tlasCap) * sizeof(MrtWideNode)));
    MRT_TRY(m_triVerts.ensure(nt * 3 * sizeof(float4)));
    MRT_TRY(m_triIndex.ensure(nt * sizeof(uint4)));
    MRT_TRY(m_normals.ensure(nv * sizeof(V4f)));
    MRT_TRY(m_uvs.ensure(nv * sizeof(V2f)));
    MRT_TRY(m_tangents.ensure(nv * sizeof(V4f)));
    MRT_TRY(m_packError.ensure(16));
    MRT_CUDA(cudaMemsetAsync(m_packError.ptr, 0, 4, m_stream));
    uint32_t vbase = 0, tbase = 0;
    for (auto& [id, b] : m_blas) {
        MRT_CUDA(mrtcu_rebase_nodes(b.nodes.as<MrtWideNode>(), b.nodeCount, b.nodeBase, tbase,
                                    m_nodes.as<MrtWideNode>(), m_stream));
        MRT_CUDA(mrtcu_pack_triangles(b.pos.as<float4>(), b.vertexCount, b.idx.as<uint32_t>(), b.prims.as<uint32_t>(),
                                      b.triCount, vbase, tbase, m_triVerts.as<float4>(), m_triIndex.as<uint4>(),
                                      m_packError.as<uint32_t>(), m_stream));
        if (b.vertexCount) {
            MRT_CUDA(cudaMemcpyAsync(m_normals.as<V4f>() + vbase, b.normals.ptr, b.vertexCount * sizeof(V4f),
                                     cudaMemcpyDeviceToDevice, m_stream));
            MRT_CUDA(cudaMemcpyAsync(m_uvs.as<V2f>() + vbase, b.uvs.ptr, b.vertexCount * sizeof(V2f),
                                     cudaMemcpyDeviceToDevice, m_stream));
            MRT_CUDA(cudaMemcpyAsync(m_tangents.as<V4f>() + vbase, b.tangents.ptr, b.vertexCount * sizeof(V4f),
                                     cudaMemcpyDeviceToDevice, m_stream));
        }
        vbase += b.vertexCount;
        tbase += b.triCount;
    }
    uint32_t packError = 0;
    MRT_CUDA(cudaMemcpyAsync(&packError, m_packError.ptr, 4, cudaMemcpyDeviceToHost, m_stream));
    MRT_CUDA(cudaStreamSynchronize(m_stream));
    if (packError) return fail(MRT_ERROR_UNKNOWN, "scene packing met an out-of-range index");
    m_blasNodeCount = uint32_t(nn);
    m_triCount = uint32_t(nt);
    m_stats.commitUploadMs += std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - ta).count();
    return MRT_SUCCESS;
}

// reference Renderer.cpp:448-508: TLAS over instance world bounds (leaf size
// 1), instances stored in TLAS leaf order, TLAS nodes after the BLAS nodes.
mrtResult Engine::packInstances() {
    const TraceRange range("mrt commit: instances");
    std::vector<const InstanceData*> flat;
    std::vector<uint32_t> ids;
    std::vector<Box3> boxes;
    for (const auto& [id, in] : m_scene.instances()) {
        auto it = m_blas.find(in.mesh);
        if (it == m_blas.end() || it->second.nodeCount == 0) continue;
        flat.push_back(&in);
        ids.push_back(id);
        boxes.push_back(transformBox(it->second.bounds, in.o2w));
    }
    for (int a = 0; a < 3; ++a) {
        m_sceneLo[a] = 3.402823466e38f;
        m_sceneHi[a] = -3.402823466e38f;
    }
    for (const Box3& b : boxes)
        for (int a = 0; a < 3; ++a) {
            m_sceneLo[a] = std::min(m_sceneLo[a], b.lo[a]);
            m_sceneHi[a] = std::max(m_sceneHi[a], b.hi[a]);
        }
    const auto tb = std::chrono::steady_clock::now();
    WideBvh tlas;
    uint32_t tlasCount = 0;
    const bool onDevice =
        !boxes.empty() && boxes.size() >= (m_deviceMinInstances ? m_deviceMinInstances : kDeviceBuildMinInstances);
    if (onDevice) {
        // nodes stay in the builder's output buffer until they are rebased below
        MRT_TRY(buildTlasOnDevice(boxes, tlas.primOrder, tlasCount));
    } else {
        tlas = collapseToWide(buildBvh(boxes, 1, 1), 1);
        if (tlas.nodes.empty()) tlas.nodes.push_back(emptyNode());
        tlasCount = uint32_t(tlas.nodes.size());
    }
    m_stats.commitDeviceTlas = onDevice ? 1u : 0u;
    m_stats.commitBvhMs += std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - tb).count();
    std::vector<MrtInstance> gi;
    gi.reserve(flat.size());
    for (uint32_t oi : tlas.primOrder) {
        const InstanceData* in = flat[oi];
        MrtInstance g{};
        std::memcpy(g.o2w, in->o2w, sizeof(g.o2w));
        invertAffine(in->o2w, g.w2o);
        g.blasRoot = m_blas[in->mesh].nodeBase;
        auto mi = m_materialIndex.find(in->material);
        g.materialIndex = mi != m_materialIndex.end() ? mi->second : 0;
        g.userId = ids[oi];
        g.meshId = in->mesh;
        gi.push_back(g);
    }
    m_tlasRoot = m_blasNodeCount;
    for (MrtWideNode& n : tlas.nodes) n.childBase += m_tlasRoot;
    m_instanceCount = uint32_t(gi.size());
    const size_t need = (size_t(m_tlasRoot) + tlasCount) * sizeof(MrtWideNode);
    if (m_nodes.bytes < need) {
        // instance count outgrew the reserved TLAS room: grow, keeping the BLAS part
        DeviceBuffer bigger;
        MRT_TRY(bigger.ensure(need + need / 2));
        cudaError_t e = cudaMemcpyAsync(bigger.ptr, m_nodes.ptr, size_t(m_tlasRoot) * sizeof(MrtWideNode),
                                        cudaMemcpyDeviceToDevice, m_stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(m_stream);
        if (e != cudaSuccess) {
            bigger.release();
            return fromCuda(e, "growing the node buffer for the TLAS");
        }
        m_nodes.release();
        m_nodes = bigger;
    }
    if (onDevice) {
        // child indices rebased behind the BLAS region; leaves index the
        // instance records, which are laid out in the builder's leaf order
        MRT_CUDA(mrtcu_rebase_nodes(m_bvhNodes.as<MrtWideNode>(), tlasCount, m_tlasRoot, 0u, m_nodes.as<MrtWideNode>(),
                                    m_stream));
    } else {
        MRT_CUDA(cudaMemcpyAsync(static_cast<MrtWideNode*>(m_nodes.ptr) + m_tlasRoot, tlas.nodes.data(),
                                 tlas.nodes.size() * sizeof(MrtWideNode), cudaMemcpyHostToDevice, m_stream));
        m_stats.commitH2DBytes += tlas.nodes.size() * sizeof(MrtWideNode);
    }
    m_nodeCount = m_tlasRoot + tlasCount;
    MRT_TRY(up(m_instances, gi.data(), gi.size() * sizeof(MrtInstance)));
    MRT_CUDA(cudaStreamSynchronize(m_stream));
    return MRT_SUCCESS;
}

// The instance tree on the GPU. Each instance's world box becomes a
// degenerate triangle (lo, hi, lo) whose bounding box is exactly that box, so
// the mesh builder (Morton codes, radix sort, LBVH topology, SAH-optimal
// collapse) builds the tree over the instance boxes unchanged, with leaves of
// one instance as the host build makes them. The nodes stay in the builder's
// output buffer; the leaf order comes back to the host, which writes the
// instance records in that order (reference Renderer.cpp:448-508 builds this
// tree on the CPU).
mrtResult Engine::buildTlasOnDevice(const std::vector<Box3>& boxes, std::vector<uint32_t>& order, uint32_t& count) {
    const size_t n = boxes.size();
    if (n > 0x7fffffffu / 3) return fail(MRT_ERROR_INVALID_ARGUMENT, "too many instances for the device BVH builder");
    std::vector<V4f> corners(2 * n);
    std::vector<uint32_t> tris(3 * n);
    for (size_t i = 0; i < n; ++i) {
        const Box3& b = boxes[i];
        corners[2 * i] = V4f{b.lo[0], b.lo[1], b.lo[2], 0.0f};
        corners[2 * i + 1] = V4f{b.hi[0], b.hi[1], b.hi[2], 0.0f};
        tris[3 * i] = uint32_t(2 * i);
        tris[3 * i + 1] = uint32_t(2 * i + 1);
        tris[3 * i + 2] = uint32_t(2 * i);
    }
    MRT_TRY(up(m_bvhPos, corners.data(), corners.size() * sizeof(V4f)));
    MRT_TRY(up(m_bvhIdx, tris.data(), tris.size() * sizeof(uint32_t)));
    Box3 bounds;
    MRT_TRY(buildBvhOnDevice(m_bvhPos.as<float4>(), m_bvhIdx.as<uint32_t>(), n, 1, count, bounds));
    order.resize(n);
    MRT_CUDA(cudaMemcpyAsync(order.data(), m_bvhPrims.ptr, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, m_stream));
    const cudaError_t e = cudaStreamSynchronize(m_stream);
    if (e != cudaSuccess) return guard(fromCuda(e, "device TLAS build"));
    return MRT_SUCCESS;
}

// reference Renderer.cpp:552-603
mrtResult Engine::packLights() {
    std::vector<MrtLight> lights;
    if (m_scene.hasEnvironment()) {
        MrtLight g{};
        g.type = MRT_DLIGHT_ENV;
        lights.push_back(g);
    }
    for (const auto& [id, l] : m_scene.lights()) {
        MrtLight g{};
        if (l.type == MRT_LIGHT_SUN) {
            g.type = MRT_DLIGHT_SUN;
            float d[3] = {l.direction[0], l.direction[1], l.direction[2]};
            normalize3(d);
            g.p0[0] = d[0];
            g.p0[1] = d[1];
            g.p0[2] = d[2];
            g.p0[3] = std::cos(std::max(l.angularRadius, 1e-4f));
            std::memcpy(g.p1, l.radiance, 12);
        } else if (l.type == MRT_LIGHT_POINT) {
            g.type = MRT_DLIGHT_POINT;
            std::memcpy(g.p0, l.position, 12);
            std::memcpy(g.p1, l.radiance, 12);
        } else {
            g.type = MRT_DLIGHT_RECT;
            float c[3];
            cross3(l.edge0, l.edge1, c);
            std::memcpy(g.p0, l.corner, 12);
            g.p0[3] = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
            std::memcpy(g.p1, l.edge0, 12);
            std::memcpy(g.p2, l.edge1, 12);
            std::memcpy(g.p3, l.radiance, 12);
            g.p3[3] = l.twoSided ? 1.0f : 0.0f;
        }
        lights.push_back(g);
    }
    m_lightCount = uint32_t(lights.size());
    if (lights.empty()) return MRT_SUCCESS;
    return up(m_lights, lights.data(), lights.size() * sizeof(MrtLight));
}

// Environment map upload + CDF on the device (reference Renderer.cpp:605-662
// builds it on the CPU).
mrtResult Engine::packEnvironment() {
    const TraceRange range("mrt commit: environment");
    m_hasEnv = m_scene.hasEnvironment();
    if (!m_hasEnv) {
        m_envW = m_envH = 0;
        return MRT_SUCCESS;
    }
    const TextureData& env = m_scene.environment();
    const auto tu = std::chrono::steady_clock::now();
    MRT_TRY(up(m_envTexels, env.data.data(), env.data.size()));
    m_stats.commitUploadMs += std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - tu).count();
    float integral = 1.0f;
    MRT_TRY(runEnvCdf(nullptr, env.width, env.height, integral));
    m_envW = env.width;
    m_envH = env.height;
    m_envIntegralHost = integral;
    return MRT_SUCCESS;
}

// Runs the CDF kernel over the texels already in m_envTexels (rgba == NULL)
// or over `rgba` uploaded first. Leaves the CDF in m_envCdf.
mrtResult Engine::runEnvCdf(const float* rgba, uint32_t w, uint32_t h, float& integral) {
    if (rgba) MRT_TRY(up(m_envTexels, rgba, size_t(w) * h * 16));
    std::vector<float> sinTheta(h);
    const float pi = 3.14159265358979323846f;
    const float dTheta = pi / float(h);
    for (uint32_t y = 0; y < h; ++y) sinTheta[y] = std::sin((float(y) + 0.5f) * dTheta);
    MRT_TRY(up(m_envSin, sinTheta.data(), h * sizeof(float)));
    MRT_TRY(m_envCdf.ensure((size_t(w) * h + h) * sizeof(float)));
    MRT_TRY(m_envRowSums.ensure(size_t(h) * (sizeof(double) + sizeof(float))));
    MRT_TRY(m_envIntegral.ensure(16));
    MRT_CUDA(cudaEventRecord(m_ev0, m_stream));
    MRT_CUDA(mrtcu_env_cdf(m_envTexels.as<float4>(), m_envSin.as<float>(), w, h, m_envCdf.as<float>(),
                           m_envRowSums.as<double>(), reinterpret_cast<float*>(m_envRowSums.as<double>() + h),
                           m_envIntegral.as<float>(), m_stream));
    MRT_CUDA(cudaEventRecord(m_ev1, m_stream));
    MRT_CUDA(cudaMemcpyAsync(&integral, m_envIntegral.ptr, sizeof(float), cudaMemcpyDeviceToHost, m_stream));
    MRT_CUDA(cudaStreamSynchronize(m_stream));
    float ms = 0.0f;
    MRT_CUDA(cudaEventElapsedTime(&ms, m_ev0, m_ev1));
    m_stats.commitEnvCdfMs = ms;
    return MRT_SUCCESS;
}

// reference Renderer.cpp:664-708: per-slot upload when the slot's generation
// changed; removed slots revert to the white placeholder.
mrtResult Engine::uploadTextures() {
    const auto& tex = m_scene.textures();
    const size_t slots = std::min<size_t>(tex.size(), MRT_MAX_TEXTURES);
    std::vector<MrtTexture> table(MRT_MAX_TEXTURES);
    std::memset(table.data(), 0, table.size() * sizeof(MrtTexture));
    for (size_t s = 0; s < slots; ++s) {
        const TextureData& t = tex[s];
        if (m_texGeneration[s] != t.generation) {
            if (t.data.empty()) m_texData[s].release();
            else MRT_TRY(m_texData[s].upload(t.data.data(), t.data.size(), m_stream));
            m_texGeneration[s] = t.generation;
        }
        if (!t.data.empty() && m_texData[s].ptr) {
            table[s].texels = m_texData[s].ptr;
            table[s].width = t.width;
            table[s].height = t.height;
            table[s].format = t.format;
        }
    }
    if (tex.size() > MRT_MAX_TEXTURES) log(LogLevel::Warn, "Texture count exceeds 64 slots; extra textures ignored");
    return up(m_texTable, table.data(), table.size() * sizeof(MrtTexture));
}

// ----------------------------------------------------------------- render --

// reference Renderer.cpp:711-764 fillGlobals (camera basis, frustum)
void Engine::fillParams(MrtFrameParams& p) const {
    std::memset(&p, 0, sizeof(p));
    float pos[3], fwd[3], upHint[3], l, r, b, t;
    bool ortho = false;
    if (m_scene.usesCameraEx()) {
        const CameraExData& c = m_scene.cameraEx();
        std::memcpy(pos, c.position, 12);
        std::memcpy(fwd, c.forward, 12);
        normalize3(fwd);
        std::memcpy(upHint, c.up, 12);
        l = c.left;
        r = c.right;
        b = c.bottom;
        t = c.top;
        ortho = c.projection == MRT_CAMERA_ORTHOGRAPHIC;
    } else {
        const CameraData& c = m_scene.camera();
        std::memcpy(pos, c.position, 12);
        fwd[0] = c.target[0] - pos[0];
        fwd[1] = c.target[1] - pos[1];
        fwd[2] = c.target[2] - pos[2];
        normalize3(fwd);
        std::memcpy(upHint, c.up, 12);
        const float aspect = float(m_settings.width) / float(m_settings.height);
        const float tanHalf = std::tan(c.fovYDeg * 0.01745329251994329576923690768489f * 0.5f);
        r = tanHalf * aspect;
        l = -r;
        t = tanHalf;
        b = -t;
    }
    float right[3];
    cross3(fwd, upHint, right);
    if (std::sqrt(right[0] * right[0] + right[1] * right[1] + right[2] * right[2]) < 1e-6f) {
        right[0] = 1.0f;
        right[1] = right[2] = 0.0f;
    } else {
        normalize3(right);
    }
    float up[3];
    cross3(right, fwd, up);
    std::memcpy(p.camPos, pos, 12);
    std::memcpy(p.camRight, right, 12);
    std::memcpy(p.camUp, up, 12);
    std::memcpy(p.camForward, fwd, 12);
    p.frustum[0] = l;
    p.frustum[1] = r;
    p.frustum[2] = b;
    p.frustum[3] = t;
    p.width = m_settings.width;
    p.height = m_settings.height;
    p.maxBounces = std::min<uint32_t>(m_settings.maxBounces, MRT_MAX_BOUNCES_CAP);
    p.lightCount = m_lightCount;
    p.envW = m_hasEnv ? m_envW : 0;
    p.envH = m_hasEnv ? m_envH : 0;
    p.flags = (m_hasEnv ? uint32_t(MRT_FLAG_HAS_ENV) : 0u) | (ortho ? uint32_t(MRT_FLAG_ORTHO) : 0u);
    p.tlasRoot = m_tlasRoot;
    p.envRotation = m_scene.envRotation();
    p.envIntensity = m_scene.envIntensity();
    p.envIntegral = m_envIntegralHost;
    p.fireflyClamp = m_settings.fireflyClamp;
    p.streamOffset = m_streamOffset;
    p.streamStride = m_streamStride;
    p.nodeCount = m_nodeCount;
    p.instanceCount = m_instanceCount;
    p.triCount = m_triCount;
    p.materialCount = m_materialCount;
    p.maxVisits = m_maxVisits ? m_maxVisits : MRT_DEFAULT_MAX_VISITS;
    p.srgbLut = m_srgbLut.as<float>();
    p.nodes = m_nodes.as<MrtWideNode>();
    p.triVerts = m_triVerts.as<float4>();
    p.triIndex = m_triIndex.as<uint4>();
    p.normals = m_normals.as<float4>();
    p.uvs = m_uvs.as<float2>();
    p.tangents = m_tangents.as<float4>();
    p.instances = m_instances.as<MrtInstance>();
    p.materials = m_materials.as<MrtMaterial>();
    p.lights = m_lights.as<MrtLight>();
    p.envTexels = m_envTexels.as<float4>();
    p.envCdf = m_envCdf.as<float>();
    p.textures = m_texTable.as<MrtTexture>();
    p.accum = m_accum.as<double>();
    p.errorFlags = m_flags.as<uint32_t>();
    p.rayCounters = m_rayCounters.as<unsigned long long>();
}

// A traversal that gave up (stack overflow, visit budget spent) or met an
// out-of-range scene index leaves a bit in the error word. Its rays may have
// missed geometry, so the call that launched them fails; for a render the
// caller's accumulation is reset (the samples are not kept), and the engine
// stays usable.
mrtResult Engine::checkErrorFlags() {
    uint32_t flags = 0;
    MRT_CUDA(cudaMemcpyAsync(&flags, m_flags.ptr, sizeof(flags), cudaMemcpyDeviceToHost, m_stream));
    MRT_CUDA(cudaStreamSynchronize(m_stream));
    if (flags) {
        MRT_CUDA(cudaMemsetAsync(m_flags.ptr, 0, sizeof(uint32_t), m_stream));
        MRT_CUDA(cudaStreamSynchronize(m_stream));
        return fail(MRT_ERROR_UNKNOWN, std::string("traversal problem in at least one ray (flags ") +
                                           std::to_string(flags) + "): " +
                                           ((flags & 1u) ? "stack or node-visit budget exhausted " : "") +
                                           ((flags & 2u) ? "out-of-range scene index " : "") +
                                           "- affected rays may have missed geometry");
    }
    return MRT_SUCCESS;
}

mrtResult Engine::setTraversalBudget(uint32_t maxVisits) {
    MRT_TRY(checkAlive());
    MRT_TRY(flushPending());
    m_maxVisits = maxVisits;
    return MRT_SUCCESS;
}

mrtResult Engine::setBvhBuildThresholds(uint32_t minTriangles, uint32_t minInstances) {
    MRT_TRY(checkAlive());
    m_deviceMinTriangles = minTriangles;
    m_deviceMinInstances = minInstances;
    return MRT_SUCCESS;
}

// reference Engine.cpp:57-60 + Renderer.cpp:773-843: implicit commit, one
// sample per pixel per frame, no-op once sppLimit is reached. With `defer`
// (mrtRenderFrame) the samples are queued and rendered as one wave when a
// full wave has accumulated or when anything reads or replaces the results
// (flushPending); the reported spp counts queued samples, as the reference
// counts rendered ones.
mrtResult Engine::renderFrames(uint32_t count, mrtFrameInfo* info, bool defer) {
    const auto t0 = std::chrono::steady_clock::now();
    MRT_TRY(commit(nullptr));
    const uint32_t queued = m_frameIndex + m_pending;
    uint32_t n = 0;
    if (queued < m_settings.sppLimit) n = std::min(count, m_settings.sppLimit - queued);
    if (n > 0) {
        if (m_pending == 0) fillParams(m_pendingParams);
        m_pending += n;
        m_resolveExposure = std::exp2(m_settings.exposureEV);
        m_resolveTonemap = m_settings.tonemap;
    }
    const bool flush = m_pending > 0 && (!defer || m_pending >= waveCapacitySamples());
    if (flush) MRT_TRY(flushPending());
    if (info && info->structSize >= sizeof(mrtFrameInfo)) {
        info->spp = m_frameIndex + m_pending;
        info->converged = m_frameIndex + m_pending >= m_settings.sppLimit ? 1 : 0;
        info->denoised = denoiserActive() && m_denoiser.useDenoised ? 1 : 0;
        // A call that rendered reports its wall time, as the reference times
        // its render call (Renderer.cpp:774, 837-841). A queued frame has not
        // been rendered yet: it reports the device time of one sample of the
        // last rendered wave, what the frame will cost (0 before any wave).
        const float wall = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        info->frameMs = (flush || n == 0 || m_stats.lastRenderSpp == 0)
                            ? wall
                            : m_stats.lastRenderMs / float(m_stats.lastRenderSpp);
    }
    return MRT_SUCCESS;
}

// Samples per pixel of one full wave at the current resolution (the wave
// state holds at most m_maxWaveSlots paths and 64 samples).
uint32_t Engine::waveCapacitySamples() const {
    const uint64_t pixels = std::max<uint64_t>(uint64_t(m_settings.width) * m_settings.height, 1);
    return uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(64, m_maxWaveSlots / pixels)));
}

// Renders the queued samples with the frame parameters captured when the
// first of them was queued (the device scene cannot change meanwhile: every
// commit that changes it resets the accumulation and drops the queue).
mrtResult Engine::flushPending() {
    MRT_TRY(launchPending());
    return completePending();
}

// Issues the queued samples' waves on this engine's stream and returns
// without waiting (completePending waits and collects the statistics).
mrtResult Engine::launchPending() {
    if (m_pending == 0 || m_inFlight != 0) return MRT_SUCCESS;
    const TraceRange range("mrt render");
    const uint32_t n = m_pending;
    m_pending = 0;
    m_stats.kernelLaunches = 0;
    m_stats.extendLaunches = 0;
    MRT_TRY(guard(ensureWave(n)));
    const MrtFrameParams p = m_pendingParams;
    MRT_CUDA(cudaMemsetAsync(m_rayCounters.ptr, 0, 128, m_stream));
    uint32_t launches = 0;
    // the cache mode renders waves of a few samples and trains after each
    const uint32_t waveCap = m_cache.enabled ? std::min(m_waveSamples, m_cache.samplesPerUpdate) : m_waveSamples;
    if (m_cache.enabled) MRT_TRY(guard(cacheWaveBuffers(waveCap, p.maxBounces)));
    const uint32_t waves = (n + waveCap - 1) / waveCap;
    const size_t perWave = size_t(6) * (p.maxBounces + 1);
    MRT_TRY(ensureEvents(waves * perWave));
    while (m_cache.enabled && m_cacheEvents.size() < size_t(3) * waves) {
        cudaEvent_t ev;
        MRT_CUDA(cudaEventCreate(&ev));
        m_cacheEvents.push_back(ev);
    }
    m_cacheQueries = m_cacheRecords = 0;
    m_cacheSteps = 0;
    MRT_CUDA(cudaEventRecord(m_ev0, m_stream));
    uint32_t wave = 0;
    for (uint32_t done = 0; done < n; ++wave) {
        const uint32_t k = std::min(n - done, waveCap);
        if (m_cache.enabled) MRT_CUDA(cudaMemsetAsync(m_cache.counts.ptr, 0, 8, m_stream));
        const cudaError_t le = mrtcu_wave(&p, &m_waveState, m_frameIndex + done, k, &launches,
                                          m_stageEvents.data() + wave * perWave,
                                          m_syncEvents.data() + wave * perWave / 3,
                                          m_cache.enabled ? &m_cache.args : nullptr, m_stream, m_side);
        if (le != cudaSuccess) return guard(fromCuda(le, "path tracing launch"));
        if (m_cache.enabled) MRT_TRY(guard(cacheWave(p, m_frameIndex + done, k, m_cacheEvents.data() + 3 * wave)));
        done += k;
    }
    MRT_CUDA(cudaEventRecord(m_ev1, m_stream));
    m_inFlight = n;
    m_inFlightWaves = waves;
    m_inFlightBounces = p.maxBounces + 1;
    m_inFlightLaunches = launches;
    m_inFlightCache = m_cache.enabled;
    return MRT_SUCCESS;
}

// At least `stage` timing events (6 per bounce of a render call) and a
// third as many sync events without timing (2 per bounce).
mrtResult Engine::ensureEvents(size_t stage) {
    while (m_stageEvents.size() < stage) {
        cudaEvent_t ev;
        MRT_CUDA(cudaEventCreate(&ev));
        m_stageEvents.push_back(ev);
    }
    while (m_syncEvents.size() < stage / 3) {
        cudaEvent_t ev;
        MRT_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        m_syncEvents.push_back(ev);
    }
    return MRT_SUCCESS;
}

// Device time per wavefront stage of one wave from its stage events (the
// launch order of mrtcu_wave): extend and shade are their kernels' spans on
// the main stream. The shadow stage is the time the shadow kernels add to
// the wave: where they run beside the next bounce's extend kernel, the wait
// of the main stream for them once extend is done, plus the last bounce's
// shadow kernel; in serial order, their spans.
static mrtResult addStageTimes(const cudaEvent_t* ev, uint32_t bounces, float& ext, float& sha, float& shw) {
    const bool overlap = mrtcu_shadow_overlap() != 0;
    for (uint32_t b = 0; b < bounces; ++b) {
        const cudaEvent_t* e = ev + 6 * size_t(b);
        float x = 0.0f, y = 0.0f, z = 0.0f, wait = 0.0f;
        MRT_CUDA(cudaEventElapsedTime(&x, e[0], e[1]));
        MRT_CUDA(cudaEventElapsedTime(&wait, e[1], e[4]));
        MRT_CUDA(cudaEventElapsedTime(&y, e[4], e[2]));
        if (!overlap || b + 1 == bounces) MRT_CUDA(cudaEventElapsedTime(&z, e[2], e[3]));
        ext += x;
        sha += y;
        shw += z + wait;
    }
    return MRT_SUCCESS;
}

mrtResult Engine::completePending() {
    if (m_inFlight == 0) return MRT_SUCCESS;
    const TraceRange range("mrt render: wait");
    const uint32_t n = m_inFlight, waves = m_inFlightWaves, bounces = m_inFlightBounces;
    m_inFlight = 0;
    const cudaError_t se = cudaStreamSynchronize(m_stream);
    if (se != cudaSuccess) return guard(fromCuda(se, "path tracing kernel"));
    float ms = 0.0f;
    MRT_CUDA(cudaEventElapsedTime(&ms, m_ev0, m_ev1));
    m_stats.lastRenderMs = ms;
    const size_t perWave = size_t(6) * bounces;
    float ext = 0.0f, sha = 0.0f, shw = 0.0f;
    for (uint32_t w = 0; w < waves; ++w)
        MRT_TRY(addStageTimes(m_stageEvents.data() + w * perWave, bounces, ext, sha, shw));
    m_stats.extendMs = ext;
    m_stats.shadeMs = sha;
    m_stats.shadowMs = shw;
    m_stats.otherMs = ms - ext - sha - shw;
    m_stats.lastRenderSpp = n;
    m_stats.kernelLaunches = m_inFlightLaunches;
    m_stats.extendLaunches = waves * bounces;
    m_stats.cacheQueryMs = m_stats.cacheTrainMs = 0.0f;
    if (m_inFlightCache)
        for (uint32_t w = 0; w < waves; ++w) {
            const cudaEvent_t* ev = m_cacheEvents.data() + 3 * w;
            float q = 0.0f, t = 0.0f;
            MRT_CUDA(cudaEventElapsedTime(&q, ev[0], ev[1]));
            MRT_CUDA(cudaEventElapsedTime(&t, ev[1], ev[2]));
            m_stats.cacheQueryMs += q;
            m_stats.cacheTrainMs += t;
        }
    m_stats.cacheQueries = m_inFlightCache ? m_cacheQueries : 0;
    m_stats.cacheRecords = m_inFlightCache ? m_cacheRecords : 0;
    m_stats.cacheSteps = m_inFlightCache ? m_cacheSteps : 0;
    m_stats.batchJobs = 1;
    if (const mrtResult fr = checkErrorFlags(); fr != MRT_SUCCESS) {
        resetAccumulation();
        return guard(fr);
    }
    unsigned long long ctr[16];
    MRT_CUDA(cudaMemcpy(ctr, m_rayCounters.ptr, sizeof(ctr), cudaMemcpyDeviceToHost));
    // A build of the kernels with MRT_TRAV_PROFILE defined fills slots 8..14
    // with the extend kernel's warp-step statistics; they are logged.
    if (ctr[8])
        log(LogLevel::Info, "extend warp steps " + std::to_string(ctr[8]) + " active lanes " + std::to_string(ctr[9]) +
                                " triangle steps " + std::to_string(ctr[10]) + " pairs " + std::to_string(ctr[11]) +
                                " rounds " + std::to_string(ctr[12]) + " node steps " + std::to_string(ctr[13]) +
                                " node lanes " + std::to_string(ctr[14]));
    m_stats.raysClosest = ctr[0];
    m_stats.raysShadow = ctr[1];
    m_stats.nodeFetches = ctr[2];
    m_stats.triTests = ctr[3];
    m_stats.surfaceHits = ctr[4];
    m_stats.shadowNodeFetches = ctr[5];
    m_stats.shadowTriTests = ctr[6];
    m_stats.nodeBytes = sizeof(MrtWideNode);
    m_stats.triBytes = 48;
    m_frameIndex += n;
    if (m_inFlightCache) {  // the last wave's cache kernels (earlier waves were checked between waves)
        uint32_t status = 0;
        MRT_CUDA(cudaMemcpy(&status, m_cache.params.status, sizeof(status), cudaMemcpyDeviceToHost));
        MRT_TRY(cacheStatus(status));
    }
    return MRT_SUCCESS;
}

// mrtxRenderBatch: every engine commits and fixes its frame parameters
// first. When all engines are on one GPU and none renders with the radiance
// cache, their waves are rendered by one set of kernel launches
// (renderBatchOneLaunch); otherwise every engine's waves are issued on its
// own stream before any is waited for, so jobs of uneven size overlap.
mrtResult Engine::renderBatch(Engine* const* engines, const uint32_t* spp, uint32_t count, mrtFrameInfo* infos) {
    const TraceRange range("mrt render batch");
    const auto t0 = std::chrono::steady_clock::now();
    // one set of launches when every engine is distinct, on one GPU and
    // without the radiance cache (an engine listed twice keeps the stream
    // path, where its earlier share is rendered before its later one)
    bool oneLaunch = count >= 2;
    for (uint32_t i = 0; i < count && oneLaunch; ++i) {
        const Engine& e = *engines[i];
        oneLaunch = !e.m_cache.enabled && e.m_device == engines[0]->m_device;
        for (uint32_t j = 0; j < i && oneLaunch; ++j) oneLaunch = engines[j] != engines[i];
    }
    std::vector<uint32_t> n(count, 0u);
    for (uint32_t i = 0; i < count; ++i) {
        Engine& e = *engines[i];
        MRT_TRY(e.checkAlive());
        MRT_TRY(e.flushPending());  // samples queued earlier render first, in order
        MRT_TRY(e.commit(nullptr));
        const uint32_t done = e.m_frameIndex;
        n[i] = done < e.m_settings.sppLimit ? std::min(spp[i], e.m_settings.sppLimit - done) : 0u;
        if (n[i] > 0) {
            e.fillParams(e.m_pendingParams);
            e.m_resolveExposure = std::exp2(e.m_settings.exposureEV);
            e.m_resolveTonemap = e.m_settings.tonemap;
            if (!oneLaunch) {
                e.m_pending = n[i];
                MRT_TRY(e.guard(e.ensureWave(n[i])));
            }
        }
    }
    mrtResult result = MRT_SUCCESS;
    if (oneLaunch) {
        result = renderBatchOneLaunch(engines, n.data(), count);
    } else {
        mrtResult launchError = MRT_SUCCESS;
        uint32_t launched = 0;
        for (; launched < count && launchError == MRT_SUCCESS; ++launched) {
            Engine& e = *engines[launched];
            launchError = e.checkAlive();
            // at most kBatchWindow jobs run at once: job i waits on the GPU for
            // job i - kBatchWindow, so a job fills its predecessor's last, short
            // bounces without all jobs contending for SMs and L2
            if (launchError == MRT_SUCCESS && launched >= kBatchWindow) {
                Engine& prev = *engines[launched - kBatchWindow];
                if (prev.m_inFlight) {
                    const cudaError_t we = cudaStreamWaitEvent(e.m_stream, prev.m_ev1, 0);
                    if (we != cudaSuccess) launchError = e.guard(fromCuda(we, "mrtxRenderBatch ordering"));
                }
            }
            if (launchError == MRT_SUCCESS) launchError = e.launchPending();
        }
        result = launchError;
        for (uint32_t i = 0; i < launched; ++i) {  // every launched engine is completed, even after an error
            Engine& e = *engines[i];
            mrtResult r = e.checkAlive();
            if (r == MRT_SUCCESS) r = e.completePending();
            if (result == MRT_SUCCESS) result = r;
        }
    }
    for (uint32_t i = 0; i < count; ++i) {
        Engine& e = *engines[i];
        if (infos && infos[i].structSize >= sizeof(mrtFrameInfo)) {
            infos[i].spp = e.m_frameIndex + e.m_pending;
            infos[i].converged = e.m_frameIndex + e.m_pending >= e.m_settings.sppLimit ? 1 : 0;
            infos[i].denoised = e.denoiserActive() && e.m_denoiser.useDenoised ? 1 : 0;
            infos[i].frameMs = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
    }
    return result;
}

// One-launch batch: every engine's samples are split into the waves the
// engine would render on its own (so each accumulation is bit for bit the
// one it would get alone), and round r gathers every engine's r-th wave
// into one batch wave, split further where it would exceed 2^28 paths. Each
// batch runs as one set of per-bounce kernel launches over the
// concatenated slots (mrtcu_wave_batch) on the first engine's stream, in
// its wave buffer, with its ray counters and error word; the other engines
// contribute their scenes and accumulation buffers. Statistics of every
// engine are those of the whole batch (device time, stage times, rays).
mrtResult Engine::renderBatchOneLaunch(Engine* const* engines, const uint32_t* n, uint32_t count) {
    Engine& lead = *engines[0];
    struct WaveJob {
        uint32_t engine, sampleBase, samples;
        uint64_t slots;
    };
    std::vector<std::vector<WaveJob>> waves(count);
    size_t rounds = 0;
    uint64_t largest = 0;
    int active = -1;
    for (uint32_t i = 0; i < count; ++i) {
        if (n[i] == 0) continue;
        Engine& e = *engines[i];
        if (active < 0) active = int(i);
        const uint64_t pixels = std::max<uint64_t>(1, uint64_t(e.m_settings.width) * e.m_settings.height);
        const uint32_t k = uint32_t(std::max<uint64_t>(
            1, std::min<uint64_t>(n[i], std::min<uint64_t>(64, e.m_maxWaveSlots / pixels))));
        for (uint32_t done = 0; done < n[i]; done += k) {
            const uint32_t s = std::min(k, n[i] - done);
            waves[i].push_back(WaveJob{i, e.m_frameIndex + done, s, pixels * s});
            largest = std::max<uint64_t>(largest, pixels * s);
        }
        rounds = std::max(rounds, waves[i].size());
    }
    if (active < 0) return MRT_SUCCESS;
    // at most 2^28 paths a batch and half the device memory free now (the
    // lead's wave buffer counted as free), but always room for the largest
    // single wave
    size_t freeBytes = 0, totalBytes = 0;
    MRT_CUDA(cudaMemGetInfo(&freeBytes, &totalBytes));
    const uint64_t budget = (uint64_t(freeBytes) + lead.m_wave.bytes) / 2 / kWaveBytesPerSlot;
    const uint64_t cap = std::max<uint64_t>(largest, std::min<uint64_t>(uint64_t(1) << 28, budget));
    if (largest > 0xffffffffull) return fail(MRT_ERROR_INVALID_ARGUMENT, "frame too large for one wave");
    std::vector<std::vector<WaveJob>> batches;
    uint64_t used = 0;
    for (size_t r = 0; r < rounds; ++r) {
        std::vector<WaveJob> cur;
        uint64_t slots = 0;
        for (uint32_t i = 0; i < count; ++i) {
            if (r >= waves[i].size()) continue;
            const WaveJob& w = waves[i][r];
            if (!cur.empty() && slots + w.slots > cap) {
                batches.push_back(cur);
                used = std::max(used, slots);
                cur.clear();
                slots = 0;
            }
            cur.push_back(w);
            slots += w.slots;
        }
        if (!cur.empty()) {
            batches.push_back(cur);
            used = std::max(used, slots);
        }
    }
    MrtWaveState W{};
    MRT_TRY(lead.guard(lead.carveWave(used, W)));
    std::vector<MrtBatchJob> table;
    std::vector<size_t> first;
    std::vector<uint32_t> bounces;
    for (const auto& batch : batches) {
        first.push_back(table.size());
        uint32_t slotBase = 0, pixelBase = 0, maxB = 0;
        for (const WaveJob& w : batch) {
            const Engine& e = *engines[w.engine];
            MrtBatchJob j{};
            j.params = e.m_pendingParams;
            j.pixels = e.m_settings.width * e.m_settings.height;
            j.samples = w.samples;
            j.slots = uint32_t(w.slots);
            j.sampleBase = w.sampleBase;
            j.slotBase = slotBase;
            j.pixelBase = pixelBase;
            slotBase += j.slots;
            pixelBase += j.pixels;
            maxB = std::max(maxB, j.params.maxBounces);
            table.push_back(j);
        }
        bounces.push_back(maxB);
    }
    MRT_TRY(lead.guard(lead.m_batchJobs.ensure(table.size() * sizeof(MrtBatchJob))));
    MRT_CUDA(cudaMemcpyAsync(lead.m_batchJobs.ptr, table.data(), table.size() * sizeof(MrtBatchJob),
                             cudaMemcpyHostToDevice, lead.m_stream));
    MRT_CUDA(cudaMemsetAsync(lead.m_rayCounters.ptr, 0, 128, lead.m_stream));
    MrtFrameParams bp = engines[active]->m_pendingParams;  // the batch's counters and error word
    bp.rayCounters = lead.m_rayCounters.as<unsigned long long>();
    bp.errorFlags = lead.m_flags.as<uint32_t>();
    size_t events = 0;
    for (uint32_t b : bounces) events += size_t(6) * (b + 1);
    MRT_TRY(lead.ensureEvents(events));
    uint32_t launches = 0;
    MRT_CUDA(cudaEventRecord(lead.m_ev0, lead.m_stream));
    size_t ev = 0;
    for (size_t b = 0; b < batches.size(); ++b) {
        const cudaError_t le = mrtcu_wave_batch(&bp, &W, lead.m_batchJobs.as<MrtBatchJob>() + first[b],
                                                table.data() + first[b], uint32_t(batches[b].size()), bounces[b],
                                                &launches, lead.m_stageEvents.data() + ev,
                                                lead.m_syncEvents.data() + ev / 3, lead.m_stream, lead.m_side);
        if (le != cudaSuccess) return lead.guard(fromCuda(le, "one-launch batch"));
        ev += size_t(6) * (bounces[b] + 1);
    }
    MRT_CUDA(cudaEventRecord(lead.m_ev1, lead.m_stream));
    const cudaError_t se = cudaStreamSynchronize(lead.m_stream);
    if (se != cudaSuccess) return lead.guard(fromCuda(se, "one-launch batch kernel"));
    if (const mrtResult fr = lead.checkErrorFlags(); fr != MRT_SUCCESS) {
        for (uint32_t i = 0; i < count; ++i) engines[i]->resetAccumulation();
        return fr;
    }
    float ms = 0.0f, ext = 0.0f, sha = 0.0f, shw = 0.0f;
    MRT_CUDA(cudaEventElapsedTime(&ms, lead.m_ev0, lead.m_ev1));
    ev = 0;
    for (uint32_t nb : bounces) {
        MRT_TRY(addStageTimes(lead.m_stageEvents.data() + ev, nb + 1, ext, sha, shw));
        ev += size_t(6) * (nb + 1);
    }
    unsigned long long ctr[16];
    MRT_CUDA(cudaMemcpy(ctr, lead.m_rayCounters.ptr, sizeof(ctr), cudaMemcpyDeviceToHost));
    uint32_t jobs = 0;
    for (uint32_t i = 0; i < count; ++i) jobs += n[i] > 0 ? 1u : 0u;
    for (uint32_t i = 0; i < count; ++i) {
        if (n[i] == 0) continue;
        Engine& e = *engines[i];
        e.m_frameIndex += n[i];
        mrtxStats& st = e.m_stats;
        st.lastRenderMs = ms;
        st.lastRenderSpp = n[i];
        st.kernelLaunches = launches;
        st.extendLaunches = 0;
        for (uint32_t nb : bounces) st.extendLaunches += nb + 1;
        st.extendMs = ext;
        st.shadeMs = sha;
        st.shadowMs = shw;
        st.otherMs = ms - ext - sha - shw;
        st.raysClosest = ctr[0];
        st.raysShadow = ctr[1];
        st.nodeFetches = ctr[2];
        st.triTests = ctr[3];
        st.surfaceHits = ctr[4];
        st.shadowNodeFetches = ctr[5];
        st.shadowTriTests = ctr[6];
        st.nodeBytes = sizeof(MrtWideNode);
        st.triBytes = 48;
        st.cacheQueryMs = st.cacheTrainMs = 0.0f;
        st.cacheQueries = st.cacheRecords = 0;
        st.cacheSteps = 0;
        st.batchJobs = jobs;
    }
    return MRT_SUCCESS;
}

// Device -> pinned staging -> caller memory, in chunks so the host copy of
// one chunk overlaps the PCIe transfer of the next.
mrtResult Engine::download(void* dst, const void* src, size_t bytes) {
    if (m_pinnedBytes < bytes) {
        if (m_pinned) cudaFreeHost(m_pinned);
        m_pinned = nullptr;
        m_pinnedBytes = 0;
        if (allocationFailureInjected()) return fromCuda(cudaErrorMemoryAllocation, "cudaMallocHost (injected failure)");
        MRT_CUDA(cudaMallocHost(&m_pinned, bytes));
        m_pinnedBytes = bytes;
    }
    const size_t chunk = size_t(4) << 20;
    const size_t nChunks = (bytes + chunk - 1) / chunk;
    size_t issued = 0;
    auto issue = [&](size_t c) -> mrtResult {
        const size_t off = c * chunk, len = std::min(chunk, bytes - off);
        MRT_CUDA(cudaMemcpyAsync(static_cast<char*>(m_pinned) + off, static_cast<const char*>(src) + off, len,
                                 cudaMemcpyDeviceToHost, m_stream));
        MRT_CUDA(cudaEventRecord(m_copyEvents[c % m_copyEvents.size()], m_stream));
        return MRT_SUCCESS;
    };
    const size_t window = m_copyEvents.size();
    for (; issued < std::min(nChunks, window); ++issued) MRT_TRY(issue(issued));
    for (size_t c = 0; c < nChunks; ++c) {
        MRT_CUDA(cudaEventSynchronize(m_copyEvents[c % window]));
        const size_t off = c * chunk, len = std::min(chunk, bytes - off);
        if (issued < nChunks) MRT_TRY(issue(issued++));
        m_copyPool->copy(static_cast<char*>(dst) + off, static_cast<const char*>(m_pinned) + off, len);
    }
    return MRT_SUCCESS;
}

// reference Renderer.cpp:892-909
mrtResult Engine::readFramebuffer(mrtPixelFormat fmt, void* dst, size_t dstSize) {
    MRT_TRY(checkAlive());
    MRT_TRY(flushPending());
    const TraceRange range("mrt readback");
    const size_t pixels = size_t(m_settings.width) * m_settings.height;
    if (fmt == MRT_PIXEL_RGBA8_SRGB) {
        if (dstSize < pixels * 4) return fail(MRT_ERROR_INVALID_ARGUMENT, "dst too small for RGBA8 readback");
        // the denoised display image (reference Renderer.cpp:845-884 with
        // resolve.comp:44-46): first at minSpp samples, then again once the
        // count has doubled
        if (denoiserActive() && m_frameIndex >= m_denoiser.nextAt && m_frameIndex != m_denoiser.denoisedSpp) {
            MRT_TRY(runDenoise());
            m_denoiser.useDenoised = true;
            m_denoiser.nextAt = std::min(m_frameIndex * 2, m_settings.sppLimit);
        }
        if (denoiserActive() && m_denoiser.useDenoised)
            MRT_CUDA(mrtcu_resolve_rgba8_linear(m_denoiser.out.as<float4>(), pixels, m_resolveExposure,
                                                m_resolveTonemap, m_out8.as<uchar4>(), m_stream));
        else
            MRT_CUDA(mrtcu_resolve_rgba8(m_accum.as<double>(), pixels, m_resolveExposure, m_resolveTonemap,
                                         m_out8.as<uchar4>(), m_stream));
        return guard(download(dst, m_out8.ptr, pixels * 4));
    }
    if (fmt != MRT_PIXEL_RGBA32F_LINEAR) return fail(MRT_ERROR_INVALID_ARGUMENT, "unknown pixel format");
    if (dstSize < pixels * 16) return fail(MRT_ERROR_INVALID_ARGUMENT, "dst too small for RGBA32F readback");
    MRT_CUDA(mrtcu_readback_rgba32f(m_accum.as<double>(), pixels, m_frameIndex, m_out32.as<float4>(), m_stream));
    return guard(download(dst, m_out32.ptr, pixels * 16));
}

// ---------------------------------------------------------------- denoiser --

void Engine::DenoiserState::release() {
    albedo.release();
    normalDepth.release();
    work.release();
    out.release();
}

mrtResult Engine::setDenoiser(const mrtxDenoiserDesc& d) {
    MRT_TRY(checkAlive());
    MRT_TRY(flushPending());
    if (d.iterations > 10) return fail(MRT_ERROR_INVALID_ARGUMENT, "denoiser iterations must be at most 10");
    const float weights[4] = {d.sigmaColor, d.normalPower, d.sigmaAlbedo, d.sigmaDepth};
    for (float v : weights)
        if (!(v >= 0.0f) || !std::isfinite(v)) return fail(MRT_ERROR_INVALID_ARGUMENT, "denoiser weights must be >= 0");
    DenoiserState& D = m_denoiser;
    D.enabled = d.enabled != 0;
    D.params.iterations = d.iterations ? d.iterations : 5u;
    D.params.sigmaColor = d.sigmaColor > 0.0f ? d.sigmaColor : 1.0f;
    D.params.normalPower = d.normalPower > 0.0f ? d.normalPower : 64.0f;
    D.params.sigmaAlbedo = d.sigmaAlbedo > 0.0f ? d.sigmaAlbedo : 0.1f;
    D.params.sigmaDepth = d.sigmaDepth > 0.0f ? d.sigmaDepth : 0.1f;
    const uint32_t samples = d.guideSamples ? d.guideSamples : 4u;
    if (samples != D.guideSamples) D.guidesValid = false;
    D.guideSamples = samples;
    D.minSpp = d.minSpp ? d.minSpp : 8u;
    // new parameters apply from the next display read
    D.useDenoised = false;
    D.nextAt = D.minSpp;
    D.denoisedSpp = 0;
    if (!D.enabled) {
        D.release();
        D.guidesValid = false;
    }
    return MRT_SUCCESS;
}

// The guides of the samples rendered so far: computed with the frame
// parameters those samples were rendered with (after the first render; the
// current ones before), on a sample stream of their own.
mrtResult Engine::ensureGuides() {
    DenoiserState& D = m_denoiser;
    const size_t pixels = size_t(m_settings.width) * m_settings.height;
    MRT_TRY(guard(D.albedo.ensure(pixels * 16)));
    MRT_TRY(guard(D.normalDepth.ensure(pixels * 16)));
    if (D.guidesValid) return MRT_SUCCESS;
    MrtFrameParams p;
    if (m_frameIndex > 0) {
        p = m_pendingParams;
    } else {
        MRT_TRY(commit(nullptr));
        fillParams(p);
    }
    MRT_CUDA(mrtcu_denoise_guides(&p, D.guideSamples, 0xC0000000u, D.albedo.as<float4>(),
                                  D.normalDepth.as<float4>(), m_stream));
    const cudaError_t se = cudaStreamSynchronize(m_stream);
    if (se != cudaSuccess) return guard(fromCuda(se, "denoiser guide kernel"));
    MRT_TRY(guard(checkErrorFlags()));
    D.guidesValid = true;
    return MRT_SUCCESS;
}

mrtResult Engine::runDenoise() {
    DenoiserState& D = m_denoiser;
    const size_t pixels = size_t(m_settings.width) * m_settings.height;
    MRT_TRY(ensureGuides());
    MRT_TRY(guard(D.work.ensure(pixels * 48)));
    MRT_TRY(guard(D.out.ensure(pixels * 16)));
    D.params.width = m_settings.width;
    D.params.height = m_settings.height;
    D.params.samples = m_frameIndex;
    MRT_CUDA(mrtcu_denoise(m_accum.as<double>(), D.albedo.as<float4>(), D.normalDepth.as<float4>(), &D.params,
                           D.work.as<float4>(), D.out.as<float4>(), m_stream));
    D.denoisedSpp = m_frameIndex;
    return MRT_SUCCESS;
}

mrtResult Engine::readDenoised(float* rgba, size_t bytes) {
    MRT_TRY(checkAlive());
    MRT_TRY(flushPending());
    if (!m_denoiser.enabled) return fail(MRT_ERROR_INVALID_ARGUMENT, "the denoiser is off (mrtxSetDenoiser)");
    const size_t pixels = size_t(m_settings.width) * m_settings.height;
    if (!rgba || bytes < pixels * 16) return fail(MRT_ERROR_INVALID_ARGUMENT, "dst too small for the denoised image");
    MRT_TRY(runDenoise());
    return guard(download(rgba, m_denoiser.out.ptr, pixels * 16));
}

mrtResult Engine::readDenoiserGuides(float* albedo, float* normalDepth, size_t bytes) {
    MRT_TRY(checkAlive());
    MRT_TRY(flushPending());
    const size_t pixels = size_t(m_settings.width) * m_settings.height;
    if (bytes < pixels * 16) return fail(MRT_ERROR_INVALID_ARGUMENT, "dst too small for the denoiser guides");
    MRT_TRY(ensureGuides());
    if (albedo) MRT_TRY(guard(download(albedo, m_denoiser.albedo.ptr, pixels * 16)));
    if (normalDepth) MRT_TRY(guard(download(normalDepth, m_denoiser.normalDepth.ptr, pixels * 16)));
    return MRT_SUCCESS;
}

// ---------------------------------------------------------------- queries --

mrtResult Engine::traceRays(const mrtxRay* rays, uint32_t n, mrtxHit* hits) {
    MRT_TRY(flushPending());
    MRT_TRY(commit(nullptr));
    if (n == 0) return MRT_SUCCESS;
    MrtFrameParams p;
    fillParams(p);
    MRT_TRY(m_queryRays.upload(rays, size_t(n) * sizeof(mrtxRay), m_stream));
    MRT_TRY(m_queryOut.ensure(size_t(n) * sizeof(mrtxHit)));
    MRT_CUDA(mrtcu_trace_closest(&p, m_queryRays.as<MrtQueryRay>(), n, m_queryOut.as<MrtQueryHit>(), m_stream));
    MRT_CUDA(cudaMemcpyAsync(hits, m_queryOut.ptr, size_t(n) * sizeof(mrtxHit), cudaMemcpyDeviceToHost, m_stream));
    const cudaError_t se = cudaStreamSynchronize(m_stream);
    if (se != cudaSuccess) return guard(fromCuda(se, "trace query kernel"));
    return guard(checkErrorFlags());
}

// Closest hits through the renderer's own extend kernel, in chunks of the
// wave state's capacity (the rays take the place of a wave's paths; no
// render is in flight, and the next render initialises its wave anew). Ray
// counters are off, so render statistics stay those of the last render.
mrtResult Engine::traceRaysWavefront(const mrtxRay* rays, uint32_t n, mrtxHit* hits) {
    MRT_TRY(flushPending());
    MRT_TRY(commit(nullptr));
    if (n == 0) return MRT_SUCCESS;
    MRT_TRY(guard(ensureWave(64)));
    MrtFrameParams p;
    fillParams(p);
    p.rayCounters = nullptr;
    const uint32_t chunk = m_waveState.capacity;
    if (chunk == 0) return fail(MRT_ERROR_UNKNOWN, "no wave state for wavefront trace queries");
    MRT_TRY(m_queryRays.upload(rays, size_t(n) * sizeof(mrtxRay), m_stream));
    MRT_TRY(m_queryOut.ensure(size_t(n) * sizeof(mrtxHit)));
    for (uint32_t first = 0; first < n; first += chunk) {
        const uint32_t k = std::min(chunk, n - first);
        MRT_CUDA(mrtcu_trace_closest_wave(&p, &m_waveState, m_queryRays.as<MrtQueryRay>() + first, k,
                                          m_queryOut.as<MrtQueryHit>() + first, m_stream));
    }
    MRT_CUDA(cudaMemcpyAsync(hits, m_queryOut.ptr, size_t(n) * sizeof(mrtxHit), cudaMemcpyDeviceToHost, m_stream));
    const cudaError_t se = cudaStreamSynchronize(m_stream);
    if (se != cudaSuccess) return guard(fromCuda(se, "wavefront trace query kernel"));
    return guard(checkErrorFlags());
}

mrtResult Engine::traceShadowRays(const mrtxRay* rays, uint32_t n, uint32_t* occluded) {
    MRT_TRY(flushPending());
    MRT_TRY(commit(nullptr));
    if (n == 0) return MRT_SUCCESS;
    MrtFrameParams p;
    fillParams(p);
    MRT_TRY(m_queryRays.upload(rays, size_t(n) * sizeof(mrtxRay), m_stream));
    MRT_TRY(m_queryOut.ensure(size_t(n) * sizeof(uint32_t)));
    MRT_CUDA(mrtcu_trace_any(&p, m_queryRays.as<MrtQueryRay>(), n, m_queryOut.as<uint32_t>(), m_stream));
    MRT_CUDA(cudaMemcpyAsync(occluded, m_queryOut.ptr, size_t(n) * 4, cudaMemcpyDeviceToHost, m_stream));
    const cudaError_t se = cudaStreamSynchronize(m_stream);
    if (se != cudaSuccess) return guard(fromCuda(se, "shadow query kernel"));
    return guard(checkErrorFlags());
}

mrtResult Engine::readAccumulation(double* dst, size_t dstSize, uint32_t* spp) {
    MRT_TRY(checkAlive());
    MRT_TRY(flushPending());
    const size_t bytes = size_t(m_settings.width) * m_settings.height * 32;
    if (dstSize < bytes) return fail(MRT_ERROR_INVALID_ARGUMENT, "dst too small for the accumulation buffer");
    MRT_TRY(guard(download(dst, m_accum.ptr, bytes)));
    if (spp) *spp = m_frameIndex;
    return MRT_SUCCESS;
}

// L2 read bandwidth of this engine's GPU: a 32 MiB zero-filled buffer (well
// inside the 126 MB L2) read 32 times by every SM with L2-only loads, timed
// with events on the engine's stream after one warm-up pass. The buffer is
// released before returning.
mrtResult Engine::measureL2Bandwidth(float* gbs) {
    MRT_TRY(checkAlive());
    MRT_TRY(flushPending());
    const size_t bytes = size_t(32) << 20;
    const uint32_t reps = 32;
    DeviceBuffer buf, sink;
    struct ReleaseOnExit {  // DeviceBuffer frees nothing by itself
        DeviceBuffer &a, &b;
        ~ReleaseOnExit() {
            a.release();
            b.release();
        }
    } releaseOnExit{buf, sink};
    MRT_TRY(buf.ensure(bytes));
    MRT_TRY(sink.ensure(16));
    MRT_CUDA(cudaMemsetAsync(buf.ptr, 0, bytes, m_stream));
    MRT_CUDA(mrtcu_l2_read_probe(buf.ptr, bytes / 16, 2, sink.as<uint32_t>(), m_stream));
    MRT_CUDA(cudaEventRecord(m_ev0, m_stream));
    MRT_CUDA(mrtcu_l2_read_probe(buf.ptr, bytes / 16, reps, sink.as<uint32_t>(), m_stream));
    MRT_CUDA(cudaEventRecord(m_ev1, m_stream));
    const cudaError_t e = cudaStreamSynchronize(m_stream);
    if (e != cudaSuccess) return guard(fromCuda(e, "L2 bandwidth probe"));
    float ms = 0.0f;
    MRT_CUDA(cudaEventElapsedTime(&ms, m_ev0, m_ev1));
    *gbs = float(double(bytes) * reps / (double(ms) * 1e-3) / 1e9);
    return MRT_SUCCESS;
}

mrtResult Engine::getStats(mrtxStats* out) const {
    mrtxStats s = m_stats;
    s.structSize = sizeof(mrtxStats);
    s.bvhNodes = m_nodeCount;
    s.triangles = m_triCount;
    s.instances = m_instanceCount;
    uint64_t bytes = 0;
    const DeviceBuffer* bufs[] = {&m_nodes,     &m_triVerts,  &m_triIndex,   &m_normals,     &m_uvs,
                                  &m_tangents,  &m_instances, &m_materials,  &m_lights,      &m_envTexels,
                                  &m_envCdf,    &m_envSin,    &m_envRowSums, &m_envIntegral, &m_texTable,
                                  &m_accum,     &m_out32,     &m_out8,       &m_flags,       &m_rayCounters,
                                  &m_queryRays, &m_queryOut,    &m_wave,       &m_bvhPos,      &m_bvhIdx,
                                  &m_bvhScratch, &m_bvhNodes,  &m_bvhPrims,  &m_packError};
    for (const DeviceBuffer* b : bufs) bytes += b->bytes;
    for (const auto& [id, b] : m_blas) bytes += b.deviceBytes();
    for (const auto& t : m_texData) bytes += t.bytes;
    s.deviceBytes = bytes;
    *out = s;
    return MRT_SUCCESS;
}

mrtResult Engine::buildEnvCdf(const float* rgba, uint32_t w, uint32_t h, float* cdf, float* integral) {
    MRT_TRY(checkAlive());
    MRT_TRY(flushPending());
    if (!rgba || !cdf || !integral || w == 0 || h == 0)
        return fail(MRT_ERROR_INVALID_ARGUMENT, "mrtxBuildEnvCdf: null pointer or empty image");
    float integ = 1.0f;
    MRT_TRY(guard(runEnvCdf(rgba, w, h, integ)));
    MRT_CUDA(cudaMemcpy(cdf, m_envCdf.ptr, (size_t(w) * h + h) * sizeof(float), cudaMemcpyDeviceToHost));
    *integral = integ;
    // the scratch buffers now hold this image, not the scene's: rebuild on next commit
    if (m_hasEnv) m_scene.markDirty(DirtyEnv | DirtyLights);
    return MRT_SUCCESS;
}

mrtResult Engine::copyAccumulationDevice(void* dev, size_t bytes, bool accumulate) {
    MRT_TRY(checkAlive());
    MRT_TRY(flushPending());
    const size_t need = size_t(m_settings.width) * m_settings.height * 32;
    if (!dev || bytes < need) return fail(MRT_ERROR_INVALID_ARGUMENT, "device buffer missing or too small");
    if (accumulate) MRT_CUDA(mrtcu_add_f64(m_accum.as<double>(), static_cast<const double*>(dev), need / 8, m_stream));
    else MRT_CUDA(cudaMemcpyAsync(dev, m_accum.ptr, need, cudaMemcpyDeviceToDevice, m_stream));
    const cudaError_t se = cudaStreamSynchronize(m_stream);
    if (se != cudaSuccess) return guard(fromCuda(se, "accumulation copy"));
    return MRT_SUCCESS;
}

mrtResult Engine::buildBvhOnDevice(const float4* pos, const uint32_t* idx, size_t nt, uint32_t maxLeaf,
                                   uint32_t& count, Box3& bounds) {
    count = 0;
    if (nt == 0) return MRT_SUCCESS;
    if (nt > 0x7fffffffu / 3) return fail(MRT_ERROR_INVALID_ARGUMENT, "mesh too large for the device BVH builder");
    MRT_TRY(m_bvhScratch.ensure(mrtcu_wide_bvh_scratch_bytes(uint32_t(nt))));
    MRT_TRY(m_bvhNodes.ensure(nt * sizeof(MrtWideNode)));
    MRT_TRY(m_bvhPrims.ensure(nt * sizeof(uint32_t)));
    float box[6];
    const cudaError_t e = mrtcu_build_wide_bvh(pos, idx, uint32_t(nt), maxLeaf, m_bvhScratch.ptr, m_bvhScratch.bytes,
                                               m_bvhNodes.as<MrtWideNode>(), uint32_t(nt), m_bvhPrims.as<uint32_t>(),
                                               &count, box, nullptr, m_stream);
    if (e != cudaSuccess) return guard(fromCuda(e, "device BVH build"));
    for (int k = 0; k < 3; ++k) {
        bounds.lo[k] = box[k];
        bounds.hi[k] = box[3 + k];
    }
    return MRT_SUCCESS;
}

mrtResult Engine::buildMeshBvhDevice(const V4f* pos, size_t nv, const uint32_t* idx, size_t nt, uint32_t maxLeaf,
                                     WideBvh& out) {
    MRT_TRY(checkAlive());
    out = WideBvh{};
    for (int k = 0; k < 3; ++k) {
        out.bounds.lo[k] = 3.402823466e38f;
        out.bounds.hi[k] = -3.402823466e38f;
    }
    if (nt == 0) return MRT_SUCCESS;
    if (nt > 0x7fffffffu / 3 || nv > 0xffffffffu)
        return fail(MRT_ERROR_INVALID_ARGUMENT, "mesh too large for the device BVH builder");
    MRT_TRY(up(m_bvhPos, pos, nv * sizeof(V4f)));
    MRT_TRY(up(m_bvhIdx, idx, nt * 3 * sizeof(uint32_t)));
    uint32_t count = 0;
    MRT_TRY(buildBvhOnDevice(m_bvhPos.as<float4>(), m_bvhIdx.as<uint32_t>(), nt, maxLeaf, count, out.bounds));
    out.nodes.resize(count);
    out.primOrder.resize(nt);
    MRT_CUDA(cudaMemcpyAsync(out.nodes.data(), m_bvhNodes.ptr, count * sizeof(MrtWideNode), cudaMemcpyDeviceToHost,
                             m_stream));
    MRT_CUDA(cudaMemcpyAsync(out.primOrder.data(), m_bvhPrims.ptr, nt * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                             m_stream));
    MRT_CUDA(cudaStreamSynchronize(m_stream));
    return MRT_SUCCESS;
}

// ------------------------------------------------------------ radiance cache --

void Engine::RadianceCache::release() {
    for (DeviceBuffer* d : {&grid, &mlp, &gGrid, &gMlp, &mGrid, &vGrid, &mMlp, &vMlp, &in, &out, &loss, &partial, &qFeat,
                            &qBeta, &rFeat, &rPrefix, &rBeta, &rTarget, &counts, &scratch, &sortScratch, &emaGrid, &emaMlp})
        d->release();
    allocated = false;
}

// Position normalisation: the given box, else the committed scene's bounds,
// else the unit cube.
void Engine::cacheBounds() {
    float lo[3], hi[3];
    bool given = true, scene = true;
    for (int a = 0; a < 3; ++a) {
        given &= m_cache.hi[a] > m_cache.lo[a];
        scene &= m_sceneHi[a] > m_sceneLo[a];
    }
    for (int a = 0; a < 3; ++a) {
        lo[a] = given ? m_cache.lo[a] : scene ? m_sceneLo[a] : 0.0f;
        hi[a] = given ? m_cache.hi[a] : scene ? m_sceneHi[a] : 1.0f;
        m_cache.params.lo[a] = lo[a];
        m_cache.params.invExtent[a] = hi[a] > lo[a] ? 1.0f / (hi[a] - lo[a]) : 1.0f;
    }
}

mrtResult Engine::ensureCache() {
    if (m_cache.allocated) return MRT_SUCCESS;
    const size_t g = mrtcu_rc_grid_floats() * sizeof(float), w = mrtcu_rc_mlp_floats() * sizeof(float);
    for (DeviceBuffer* d : {&m_cache.grid, &m_cache.gGrid, &m_cache.mGrid, &m_cache.vGrid, &m_cache.emaGrid})
        MRT_TRY(d->ensure(g));
    for (DeviceBuffer* d : {&m_cache.mlp, &m_cache.gMlp, &m_cache.mMlp, &m_cache.vMlp, &m_cache.emaMlp})
        MRT_TRY(d->ensure(w));
    MRT_TRY(m_cache.loss.ensure(16));
    MRT_TRY(m_cache.partial.ensure(mrtcu_rc_partial_floats(kCacheMaxBatch) * sizeof(float)));
    McacheParams& c = m_cache.params;
    c.partial = m_cache.partial.as<float>();
    c.status = m_cache.loss.as<uint32_t>() + 1;  // the loss buffer's second word
    c.partialBlocks = mrtcu_rc_partial_blocks(kCacheMaxBatch);
    c.grid = m_cache.grid.as<float>();
    c.mlp = m_cache.mlp.as<float>();
    c.gGrid = m_cache.gGrid.as<float>();
    c.gMlp = m_cache.gMlp.as<float>();
    c.mGrid = m_cache.mGrid.as<float>();
    c.vGrid = m_cache.vGrid.as<float>();
    c.mMlp = m_cache.mMlp.as<float>();
    c.vMlp = m_cache.vMlp.as<float>();
    c.emaGrid = m_cache.emaDecay > 0.0f ? m_cache.emaGrid.as<float>() : nullptr;
    c.emaMlp = m_cache.emaDecay > 0.0f ? m_cache.emaMlp.as<float>() : nullptr;
    c.emaDecay = m_cache.emaDecay;
    c.step = 0;
    c.lr = m_cache.lr;
    c.lrMin = m_cache.lrMin;
    c.lrHalfLife = m_cache.lrHalfLife;
    c.lrStart = 0;
    cacheBounds();
    MRT_CUDA(mrtcu_rc_init(c, m_cache.seed, m_stream));
    MRT_CUDA(cudaStreamSynchronize(m_stream));
    m_cache.allocated = true;
    return MRT_SUCCESS;
}

mrtResult Engine::setRadianceCache(const mrtxRadianceCacheDesc& d) {
    MRT_TRY(checkAlive());
    MRT_TRY(flushPending());
    if (m_cache.failed && d.enabled) return cacheStatus(0);
    const bool reinit = m_cache.allocated && d.seed != m_cache.seed;
    m_cache.trainingPaths = d.trainingPaths;  // 0: a 32nd of the pixels (cacheWaveBuffers)
    m_cache.stepsPerSample = d.stepsPerSample ? d.stepsPerSample : 1u;
    m_cache.samplesPerUpdate = d.samplesPerUpdate ? std::min(d.samplesPerUpdate, 64u) : 4u;
    m_cache.trainingVertices = d.trainingVertices;
    const float lr = d.learningRate > 0.0f ? d.learningRate : 1e-2f;
    const bool newRate = lr != m_cache.lr;
    m_cache.lr = lr;
    m_cache.seed = d.seed;
    for (int a = 0; a < 3; ++a) {
        m_cache.lo[a] = d.boundsLo[a];
        m_cache.hi[a] = d.boundsHi[a];
    }
    if (reinit) m_cache.release();
    MRT_TRY(guard(ensureCache()));
    m_cache.params.lr = m_cache.lr;
    if (newRate) m_cache.params.lrStart = m_cache.params.step;  // the decay restarts from the new rate
    cacheBounds();
    if (bool(d.enabled) != m_cache.enabled) resetAccumulation();  // a different estimator
    m_cache.enabled = d.enabled != 0;
    return MRT_SUCCESS;
}

mrtResult Engine::cacheQuery(const float* features, uint32_t n, float* rgb) {
    MRT_TRY(checkAlive());
    MRT_TRY(cacheStatus(0));
    MRT_TRY(guard(ensureCache()));
    if (n == 0) return MRT_SUCCESS;
    MRT_TRY(up(m_cache.in, features, size_t(n) * 16 * sizeof(float)));
    MRT_TRY(m_cache.out.ensure(size_t(n) * 3 * sizeof(float)));
    MRT_CUDA(mrtcu_rc_query(inferenceParams(), m_cache.in.as<float>(), n, m_cache.out.as<float>(), m_stream));
    MRT_CUDA(cudaMemcpyAsync(rgb, m_cache.out.ptr, size_t(n) * 3 * sizeof(float), cudaMemcpyDeviceToHost, m_stream));
    uint32_t status = 0;
    MRT_CUDA(cudaMemcpyAsync(&status, m_cache.params.status, sizeof(status), cudaMemcpyDeviceToHost, m_stream));
    const cudaError_t e = cudaStreamSynchronize(m_stream);
    if (e != cudaSuccess) return guard(fromCuda(e, "radiance cache query"));
    return cacheStatus(status);
}

mrtResult Engine::cacheTrain(const float* features, const float* targets, uint32_t n, uint32_t steps, float* loss) {
    MRT_TRY(checkAlive());
    MRT_TRY(cacheStatus(0));
    MRT_TRY(guard(ensureCache()));
    if (n == 0 || steps == 0) return MRT_SUCCESS;
    MRT_TRY(m_cache.in.ensure(size_t(n) * 19 * sizeof(float)));
    float* din = m_cache.in.as<float>();
    MRT_CUDA(cudaMemcpyAsync(din, features, size_t(n) * 16 * sizeof(float), cudaMemcpyHostToDevice, m_stream));
    MRT_CUDA(cudaMemcpyAsync(din + size_t(n) * 16, targets, size_t(n) * 3 * sizeof(float), cudaMemcpyHostToDevice,
                             m_stream));
    MRT_CUDA(cudaMemsetAsync(m_cache.loss.ptr, 0, sizeof(float), m_stream));
    MRT_CUDA(mrtcu_rc_train(&m_cache.params, din, din + size_t(n) * 16, n, steps, 65536u, m_cache.loss.as<float>(),
                            m_stream));
    float l = 0.0f;
    MRT_CUDA(cudaMemcpyAsync(&l, m_cache.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost, m_stream));
    const cudaError_t e = cudaStreamSynchronize(m_stream);
    if (e != cudaSuccess) return guard(fromCuda(e, "radiance cache training"));
    if (loss) *loss = l;
    return MRT_SUCCESS;
}

// Learning-rate decay of the online training: the rate halves every
// halfLifeSteps Adam steps down to lrMin (halfLifeSteps 0: constant rate),
// restarting from the full rate now.
mrtResult Engine::setCacheSchedule(float lrMin, float halfLifeSteps) {
    MRT_TRY(checkAlive());
    MRT_TRY(flushPending());
    MRT_TRY(cacheStatus(0));
    if (!(lrMin >= 0.0f) || !(halfLifeSteps >= 0.0f))
        return fail(MRT_ERROR_INVALID_ARGUMENT, "radiance cache schedule: lrMin and halfLifeSteps must be >= 0");
    MRT_TRY(guard(ensureCache()));
    m_cache.lrMin = lrMin;
    m_cache.lrHalfLife = halfLifeSteps;
    m_cache.params.lrMin = lrMin;
    m_cache.params.lrHalfLife = halfLifeSteps;
    m_cache.params.lrStart = m_cache.params.step;
    return MRT_SUCCESS;
}

// Queries read the moving average of the parameters while averaging is on,
// the live parameters otherwise.
McacheParams Engine::inferenceParams() const {
    McacheParams q = m_cache.params;
    if (m_cache.emaDecay > 0.0f) {
        q.grid = m_cache.emaGrid.as<float>();
        q.mlp = m_cache.emaMlp.as<float>();
    }
    return q;
}

mrtResult Engine::resetAverage() {
    MRT_CUDA(cudaMemcpyAsync(m_cache.emaGrid.ptr, m_cache.grid.ptr, mrtcu_rc_grid_floats() * sizeof(float),
                             cudaMemcpyDeviceToDevice, m_stream));
    MRT_CUDA(cudaMemcpyAsync(m_cache.emaMlp.ptr, m_cache.mlp.ptr, mrtcu_rc_mlp_floats() * sizeof(float),
                             cudaMemcpyDeviceToDevice, m_stream));
    return MRT_SUCCESS;
}

// Averaging of the weights queries read: decay in [0, 1); 0 switches it off
// (queries read the live parameters). Switching it on starts the average at
// the live parameters.
mrtResult Engine::setCacheAveraging(float decay) {
    MRT_TRY(checkAlive());
    MRT_TRY(flushPending());
    MRT_TRY(cacheStatus(0));
    if (!(decay >= 0.0f && decay < 1.0f))
        return fail(MRT_ERROR_INVALID_ARGUMENT, "radiance cache averaging: decay must be in [0, 1)");
    MRT_TRY(guard(ensureCache()));
    const bool wasOn = m_cache.emaDecay > 0.0f;
    m_cache.emaDecay = decay;
    m_cache.params.emaDecay = decay;
    m_cache.params.emaGrid = decay > 0.0f ? m_cache.emaGrid.as<float>() : nullptr;
    m_cache.params.emaMlp = decay > 0.0f ? m_cache.emaMlp.as<float>() : nullptr;
    if (decay > 0.0f && !wasOn) MRT_TRY(resetAverage());
    const cudaError_t e = cudaStreamSynchronize(m_stream);
    if (e != cudaSuccess) return guard(fromCuda(e, "radiance cache averaging"));
    return MRT_SUCCESS;
}

// One forward and backward pass of the training kernel over all n samples,
// without the Adam step: the raw gradients of the mean loss, read back. The
// grid gradient is cleared afterwards (the lazy Adam step treats nonzero
// entries as touched), so later training is unaffected.
mrtResult Engine::cacheGradients(const float* features, const float* targets, uint32_t n, float* gridOut,
                                 float* mlpOut, float* loss) {
    MRT_TRY(checkAlive());
    MRT_TRY(cacheStatus(0));
    MRT_TRY(guard(ensureCache()));
    const size_t g = mrtcu_rc_grid_floats() * sizeof(float), w = mrtcu_rc_mlp_floats() * sizeof(float);
    MRT_TRY(m_cache.in.ensure(std::max<size_t>(1, n) * 19 * sizeof(float)));
    float* din = m_cache.in.as<float>();
    MRT_CUDA(cudaMemsetAsync(m_cache.loss.ptr, 0, sizeof(float), m_stream));
    MRT_CUDA(cudaMemsetAsync(m_cache.gMlp.ptr, 0, w, m_stream));
    MRT_CUDA(cudaMemsetAsync(m_cache.gGrid.ptr, 0, g, m_stream));
    if (n) {
        MRT_CUDA(cudaMemcpyAsync(din, features, size_t(n) * 16 * sizeof(float), cudaMemcpyHostToDevice, m_stream));
        MRT_CUDA(cudaMemcpyAsync(din + size_t(n) * 16, targets, size_t(n) * 3 * sizeof(float),
                                 cudaMemcpyHostToDevice, m_stream));
        MRT_CUDA(mrtcu_rc_gradients(&m_cache.params, din, din + size_t(n) * 16, n, m_cache.loss.as<float>(),
                                    m_stream));
    }
    if (mlpOut) MRT_CUDA(cudaMemcpyAsync(mlpOut, m_cache.gMlp.ptr, w, cudaMemcpyDeviceToHost, m_stream));
    if (gridOut) MRT_CUDA(cudaMemcpyAsync(gridOut, m_cache.gGrid.ptr, g, cudaMemcpyDeviceToHost, m_stream));
    float l = 0.0f;
    uint32_t status = 0;
    MRT_CUDA(cudaMemcpyAsync(&l, m_cache.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost, m_stream));
    MRT_CUDA(cudaMemcpyAsync(&status, m_cache.params.status, sizeof(status), cudaMemcpyDeviceToHost, m_stream));
    MRT_CUDA(cudaMemsetAsync(m_cache.gGrid.ptr, 0, g, m_stream));
    const cudaError_t e = cudaStreamSynchronize(m_stream);
    if (e != cudaSuccess) return guard(fromCuda(e, "radiance cache gradients"));
    MRT_TRY(cacheStatus(status));
    if (loss) *loss = l;
    return MRT_SUCCESS;
}

mrtResult Engine::cacheParams(float* gridOut, float* mlpOut, const float* gridIn, const float* mlpIn) {
    MRT_TRY(checkAlive());
    MRT_TRY(guard(ensureCache()));
    const size_t g = mrtcu_rc_grid_floats() * sizeof(float), w = mrtcu_rc_mlp_floats() * sizeof(float);
    if (gridOut) MRT_CUDA(cudaMemcpyAsync(gridOut, m_cache.grid.ptr, g, cudaMemcpyDeviceToHost, m_stream));
    if (mlpOut) MRT_CUDA(cudaMemcpyAsync(mlpOut, m_cache.mlp.ptr, w, cudaMemcpyDeviceToHost, m_stream));
    if (gridIn) MRT_CUDA(cudaMemcpyAsync(m_cache.grid.ptr, gridIn, g, cudaMemcpyHostToDevice, m_stream));
    if (mlpIn) MRT_CUDA(cudaMemcpyAsync(m_cache.mlp.ptr, mlpIn, w, cudaMemcpyHostToDevice, m_stream));
    if (gridIn || mlpIn) {
        for (DeviceBuffer* d : {&m_cache.gGrid, &m_cache.mGrid, &m_cache.vGrid})
            MRT_CUDA(cudaMemsetAsync(d->ptr, 0, g, m_stream));
        for (DeviceBuffer* d : {&m_cache.gMlp, &m_cache.mMlp, &m_cache.vMlp})
            MRT_CUDA(cudaMemsetAsync(d->ptr, 0, w, m_stream));
        m_cache.params.step = 0;
        m_cache.params.lrStart = 0;
        MRT_TRY(resetAverage());
    }
    const cudaError_t e = cudaStreamSynchronize(m_stream);
    if (e != cudaSuccess) return guard(fromCuda(e, "radiance cache parameters"));
    return MRT_SUCCESS;
}

// A cache kernel whose tensor-core wait gave up leaves bit 0 of the status
// word set. That is fatal for the cache: the MMA it waited for may still
// have been writing tensor memory when the CTA freed it, so every output of
// the launch is suspect. The accumulation (which may hold its predictions)
// is discarded, the cache mode is switched off, and every later cache call
// of this engine fails.
mrtResult Engine::cacheStatus(uint32_t status) {
    if (status & 1u) {
        m_cache.failed = true;
        m_cache.enabled = false;
        resetAccumulation();
    }
    if (m_cache.failed)
        return fail(MRT_ERROR_UNKNOWN, "radiance cache: a tensor-core wait timed out; the cache is disabled and "
                                       "the accumulation was discarded");
    return MRT_SUCCESS;
}

// Query and record buffers of one cache-mode wave of `samples` samples.
mrtResult Engine::cacheWaveBuffers(uint32_t samples, uint32_t maxBounces) {
    MRT_TRY(ensureCache());
    const uint64_t pixels = uint64_t(m_settings.width) * m_settings.height;
    const uint64_t q = pixels * samples;
    const uint64_t training = m_cache.trainingPaths ? m_cache.trainingPaths : std::max<uint64_t>(1024, pixels / 32);
    const uint32_t stride = uint32_t(std::max<uint64_t>(1, pixels / training));
    // A vertex k bounces in sees maxBounces - k more bounces; the queried
    // vertex (k = 1) sees maxBounces - 1. Deeper vertices' targets miss the
    // energy of the bounces cut off at the budget, so only the first few
    // vertices train the cache.
    const uint32_t vertices = m_cache.trainingVertices ? m_cache.trainingVertices
                                                       : std::max(1u, maxBounces / 4u);
    const uint64_t r = std::min<uint64_t>(q, (pixels / stride + 1024) * samples * std::min(vertices, std::max(1u, maxBounces)));
    MRT_TRY(m_cache.qFeat.ensure(q * 16 * sizeof(float)));
    MRT_TRY(m_cache.qBeta.ensure(q * sizeof(float4)));
    MRT_TRY(m_cache.scratch.ensure(q * 3 * sizeof(float)));
    MRT_TRY(m_cache.sortScratch.ensure(mrtcu_rc_sort_scratch_words(uint32_t(q)) * sizeof(uint32_t)));
    MRT_TRY(m_cache.rFeat.ensure(r * 16 * sizeof(float)));
    MRT_TRY(m_cache.rPrefix.ensure(r * sizeof(float4)));
    MRT_TRY(m_cache.rBeta.ensure(r * sizeof(float4)));
    MRT_TRY(m_cache.rTarget.ensure(r * 3 * sizeof(float)));
    MRT_TRY(m_cache.counts.ensure(16));
    MrtCacheArgs& K = m_cache.args;
    K.qFeat = m_cache.qFeat.as<float>();
    K.qBeta = m_cache.qBeta.as<float4>();
    K.qCount = m_cache.counts.as<uint32_t>();
    K.qCap = uint32_t(q);
    K.rFeat = m_cache.rFeat.as<float>();
    K.rPrefix = m_cache.rPrefix.as<float4>();
    K.rBeta = m_cache.rBeta.as<float4>();
    K.rCount = m_cache.counts.as<uint32_t>() + 1;
    K.rCap = uint32_t(r);
    K.trainStride = stride;
    K.recordBounces = vertices;
    K.spreadC = 0.01f;  // the neural radiance caching paper's c
    cacheBounds();
    return MRT_SUCCESS;
}

// After a cache-mode wave's bounces: the cache's predictions join the
// stopped paths, the training paths' vertices become training samples, the
// cache trains on them, and the wave is accumulated.
mrtResult Engine::cacheWave(const MrtFrameParams& p, uint32_t sampleBase, uint32_t samples, const cudaEvent_t* ev) {
    uint32_t counts[2] = {0, 0}, status = 0;
    MRT_CUDA(cudaMemcpyAsync(counts, m_cache.counts.ptr, sizeof(counts), cudaMemcpyDeviceToHost, m_stream));
    MRT_CUDA(cudaMemcpyAsync(&status, m_cache.params.status, sizeof(status), cudaMemcpyDeviceToHost, m_stream));
    MRT_CUDA(cudaStreamSynchronize(m_stream));
    MRT_TRY(cacheStatus(status));  // the previous wave's queries
    const MrtCacheArgs& K = m_cache.args;
    const uint32_t nq = std::min(counts[0], K.qCap), nr = std::min(counts[1], K.rCap);
    const uint32_t slots = p.width * p.height * samples;
    MRT_CUDA(cudaEventRecord(ev[0], m_stream));
    MRT_CUDA(mrtcu_rc_apply_queries(inferenceParams(), K.qFeat, K.qBeta, nq, slots, m_cache.scratch.as<float>(),
                                    m_waveState.L, m_cache.sortScratch.as<uint32_t>(), m_stream));
    MRT_CUDA(cudaEventRecord(ev[1], m_stream));
    MRT_CUDA(mrtcu_rc_record_targets(K.rPrefix, K.rBeta, nr, slots, m_waveState.L, m_cache.rTarget.as<float>(),
                                     m_stream));
    // Batches of up to 16,384 records, smaller when the wave has fewer than
    // steps x 16,384: the steps then take disjoint batches, so no record
    // trains the cache twice (re-used noisy targets get memorised).
    const uint32_t steps = m_cache.stepsPerSample * samples;
    const uint32_t batch = std::max(64u, std::min(16384u, nr / std::max(1u, steps)));
    MRT_CUDA(mrtcu_rc_train(&m_cache.params, K.rFeat, m_cache.rTarget.as<float>(), nr, steps, batch, nullptr,
                            m_stream));
    MRT_CUDA(cudaEventRecord(ev[2], m_stream));
    m_cacheQueries += nq;
    m_cacheRecords += nr;
    m_cacheSteps += nr ? steps : 0;
    MRT_CUDA(mrtcu_wave_finalize(&p, &m_waveState, sampleBase, samples, m_stream));
    return MRT_SUCCESS;
}

}  // namespace mrt
