/*
 * mrt_ext.h -- extensions of the MiniRaytrace C ABI exported by libmrt.so.
 *
 * The reference ABI versions its structs by `structSize >= sizeof(T)`
 * (reference capi/src/capi.cpp:23-24), so appending a field to any v1 struct
 * would make every existing caller fail with MRT_ERROR_INVALID_ARGUMENT. Every
 * new capability is therefore a new exported function with its own structs.
 * None of these functions has a counterpart in the reference ABI; each one
 * names the reference behaviour it builds on.
 */
#ifndef MRT_EXT_H
#define MRT_EXT_H

#include "mini_raytrace.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Equivalent to `count` consecutive mrtRenderFrame calls (reference
 * Renderer.cpp:773-843: one sample per pixel per frame, stop at sppLimit),
 * issued as one device submission. outInfo reports the state after the last
 * sample. */
MRT_API mrtResult mrtxRenderFrames(mrtEngine*, uint32_t count, mrtFrameInfo* outInfo);

/* One ray of a trace query: world space, t in (1e-4, tMax). */
typedef struct mrtxRay {
    float origin[3];
    float tMax;
    float dir[3];
    float pad;
} mrtxRay;

/* Closest hit of one ray. instance = the mrtInstanceId that was hit (0 on a
 * miss); prim = triangle index in the mesh's own index buffer order (the
 * reference's "original" triangle order before the BVH leaf reordering,
 * reference Renderer.cpp:403-411); u, v = barycentrics of vertices 1 and 2. */
typedef struct mrtxHit {
    float t;
    uint32_t instance;
    uint32_t prim;
    uint32_t hit;
    float u, v;
    uint32_t pad[2];
} mrtxHit;

/* Closest-hit traversal of the committed scene (reference intersect.glsl:
 * 88-125 `traceRay`) for `count` rays; commits pending scene changes first. */
MRT_API mrtResult mrtxTraceRays(mrtEngine*, const mrtxRay* rays, uint32_t count, mrtxHit* hits);

/* mrtxTraceRays through the renderer's own closest-hit stage: the rays
 * take the place of a wave's paths and one launch of the wavefront's extend
 * kernel (persistent warps that refill finished lanes, warp-batched
 * triangle tests) traces them, exactly as it traces path segments. Each
 * ray's tMax is ignored (path rays are traced to 1e30). Same output as
 * mrtxTraceRays; for checking the kernel a render uses. */
MRT_API mrtResult mrtxTraceRaysWavefront(mrtEngine*, const mrtxRay* rays, uint32_t count, mrtxHit* hits);

/* Any-hit traversal (reference intersect.glsl:128-178 `traceShadowRay`):
 * occluded[i] = 1 when ray i hits anything in (1e-4, tMax), else 0. */
MRT_API mrtResult mrtxTraceShadowRays(mrtEngine*, const mrtxRay* rays, uint32_t count,
                                      uint32_t* occluded);

/* The FP64 accumulation buffer: 4 doubles per pixel (sum r, g, b, and the
 * sample count), row-major, top row first. dstSize >= width*height*32. */
MRT_API mrtResult mrtxReadAccumulation(mrtEngine*, double* dst, size_t dstSize,
                                       uint32_t* outSpp);

/* Device timings and counters. All times are CUDA-event times in ms. */
typedef struct mrtxStats {
    size_t structSize;
    float lastRenderMs;    /* device time of the last render call's kernels */
    uint32_t lastRenderSpp; /* samples per pixel rendered by that call */
    float commitBvhMs;     /* last commit: acceleration structure build */
    float commitEnvCdfMs;  /* last commit: environment CDF kernel */
    float commitUploadMs;  /* last commit: host-to-device copies */
    float commitTotalMs;   /* last commit: host wall time */
    uint32_t bvhNodes;     /* total nodes (all BLAS + TLAS) */
    uint32_t triangles;    /* total triangles */
    uint32_t instances;    /* total instances */
    uint32_t kernelLaunches; /* kernels launched by the last render call */
    uint64_t deviceBytes;  /* device memory held by the engine */
    /* counters of the last render call (all samples of all pixels) */
    uint64_t raysClosest;  /* closest-hit rays traced */
    uint64_t raysShadow;   /* shadow (any-hit) rays traced */
    uint64_t nodeFetches;  /* BVH node records read by closest-hit rays */
    uint64_t triTests;     /* ray/triangle tests of closest-hit rays */
    uint64_t surfaceHits;  /* hits shaded (one surface gather each) */
    uint64_t commitH2DBytes; /* bytes copied host-to-device by the last commit */
    uint64_t shadowNodeFetches; /* BVH node records read by shadow rays */
    uint64_t shadowTriTests;    /* ray/triangle tests of shadow rays */
    uint32_t nodeBytes;    /* bytes of one BVH node record */
    uint32_t triBytes;     /* bytes read by one ray/triangle test */
    /* device time of the last render call per wavefront stage (CUDA events);
     * the shadow rays of a bounce are traced beside the next bounce's extend
     * kernel, so shadowMs is the time they add past it (and the last
     * bounce's shadow kernel); the four sum to lastRenderMs */
    float extendMs, shadeMs, shadowMs, otherMs;
    uint32_t extendLaunches; /* closest-hit (extend) kernel launches of the last render call */
    /* radiance-cache mode, last render call: device time of the cache's
     * inference (queries and their application to the paths) and of its
     * training (targets, steps, Adam), with their counts */
    float cacheQueryMs, cacheTrainMs;
    uint64_t cacheQueries, cacheRecords;
    uint32_t cacheSteps;
    /* engines whose samples the last render call's launches rendered
     * together: 1, or the job count of a one-launch mrtxRenderBatch (whose
     * engines all report the batch's launches, times and counters) */
    uint32_t batchJobs;
    /* last commit that rebuilt geometry or instances: mesh BVHs built on the
     * GPU, and 1 if the instance tree (TLAS) was built there
     * (mrtxSetBvhBuildThresholds) */
    uint32_t commitDeviceBlas;
    uint32_t commitDeviceTlas;
} mrtxStats;
/* out->structSize may be that of an earlier, shorter mrtxStats (fields are
 * only appended; at least up to cacheSteps): the fields it covers are written. */
MRT_API mrtResult mrtxGetStats(mrtEngine*, mrtxStats* out);

/* Measured L2 read bandwidth (GB/s) of the engine's GPU: every SM re-reads a
 * 32 MiB buffer with loads cached in L2 only, timed with CUDA events; a
 * temporary 32 MiB device buffer is allocated and freed. A denominator for
 * L2-bound rooflines (no counterpart in the reference). */
MRT_API mrtResult mrtxMeasureL2Bandwidth(mrtEngine*, float* outGBs);

/* The environment CDF exactly as the commit builds it (reference
 * Renderer.cpp:620-655), computed by the device kernel on this engine's GPU:
 * rgba = w*h RGBA32F texels; cdfOut receives w*h + h floats (conditional rows,
 * then the marginal); *integralOut receives the float integral. */
MRT_API mrtResult mrtxBuildEnvCdf(mrtEngine*, const float* rgba, uint32_t w, uint32_t h,
                                  float* cdfOut, float* integralOut);

/* Sample-stream striping for replicas: sample s of this engine uses the
 * random stream of frame index (s * stride + offset). stride = 1, offset = 0
 * is the reference stream (reference pathtrace.comp:105). Resets accumulation. */
MRT_API mrtResult mrtxSetSampleStream(mrtEngine*, uint32_t offset, uint32_t stride);

/* Node visits one ray's traversal may make before it gives up (0 restores
 * the default, 2^22, which a well-formed BVH never approaches). A ray that
 * gives up, overflows its traversal stack or meets an out-of-range scene
 * index makes the call that traced it fail with MRT_ERROR_UNKNOWN instead of
 * hanging or returning a silently wrong image; a render call then resets
 * the accumulation (its samples are not kept) and the engine stays usable.
 * The reference has no counterpart: its shader loops until its stack
 * empties (intersect.glsl:48-125) and every device error aborts the process
 * (core/src/gpu/GpuContext.hpp:22-31). */
MRT_API mrtResult mrtxSetTraversalBudget(mrtEngine*, uint32_t maxVisits);

/* Where the acceleration structures are built. A mesh of at least
 * minTriangles triangles gets its BVH built on the engine's GPU (Morton
 * codes, radix sort, LBVH topology, SAH-optimal collapse to 8-wide nodes),
 * smaller meshes on host threads (binned SAH, the same collapse); an instance
 * set of at least minInstances instances gets its TLAS built on the GPU by the
 * same builder, a smaller one on the host. 0 selects the default (16384
 * triangles, 2048 instances); 1 builds everything on the GPU and 0xFFFFFFFF
 * everything on the host. Either site gives a valid tree over the same
 * primitives, so closest hits and images do not depend on the choice; the
 * host's SAH tree is slightly cheaper to trace, the GPU's is built in
 * milliseconds. Takes effect at the next commit that rebuilds a mesh or the
 * instances. The reference builds every BVH on the CPU
 * (core/src/render/Renderer.cpp:342-368, 448-508). */
MRT_API mrtResult mrtxSetBvhBuildThresholds(mrtEngine*, uint32_t minTriangles, uint32_t minInstances);

/* Test hook for allocation failures: after this call the next
 * `succeedFirst` device or pinned-host allocations of the library succeed
 * and every later one fails as MRT_ERROR_OUT_OF_MEMORY, in every engine of
 * the process; succeedFirst < 0 turns the injection off. A call that meets
 * the failure returns MRT_ERROR_OUT_OF_MEMORY and leaves the engine usable:
 * the scene stays dirty, so the next commit redoes the work. Nothing is
 * done to the GPU. The reference maps std::bad_alloc the same way
 * (capi/src/capi.cpp:116-120) but has no injection. */
MRT_API mrtResult mrtxInjectAllocationFailure(int32_t succeedFirst);

/* Copy the FP64 accumulation buffer (layout as mrtxReadAccumulation) to a
 * device pointer on this engine's GPU, or add a device buffer of the same
 * layout into it (accumulate != 0). Used to reduce replicas' samples. */
MRT_API mrtResult mrtxCopyAccumulationDevice(mrtEngine*, void* devPtr, size_t bytes,
                                             int32_t accumulate);

/* Renders several engines' frames in one submission: engines[i] gets spp[i]
 * more samples per pixel, as mrtxRenderFrames(engines[i], spp[i], ...) would
 * give it (the same samples, bit for bit). Every engine commits and prepares
 * first; then all engines' waves are issued, each on its own CUDA stream,
 * before any is waited for, so jobs of uneven size overlap on the GPU. The
 * engines may share a GPU. outInfos (optional, count entries with structSize
 * set) receive each engine's state; frameMs is the time from the call's
 * start to that engine's completion. An error stops further launches; engines
 * already launched are still completed. Builds on the reference's per-frame
 * submission (Renderer.cpp:773-843), which renders one engine at a time. */
MRT_API mrtResult mrtxRenderBatch(mrtEngine* const* engines, const uint32_t* spp, uint32_t count,
                                  mrtFrameInfo* outInfos);

/* Radiance cache (no counterpart in the reference): a neural cache of
 * outgoing radiance (multiresolution hash grid of position + spherical
 * harmonics of the direction + surface features into a 5 x 64 ReLU MLP),
 * trained online from full-length training paths. With `enabled`, rendered
 * paths other than the training paths stop at their second surface vertex
 * and take the cache's prediction there (biased, lower variance, fewer
 * bounces). Bounds: the box the position encoding spans; a box with
 * boundsHi <= boundsLo on any axis means the committed scene's bounds. */
typedef struct mrtxRadianceCacheDesc {
    size_t structSize;
    int32_t enabled;
    uint32_t trainingPaths;  /* full-length training paths per rendered sample (0: a 32nd of the pixels) */
    uint32_t stepsPerSample; /* Adam steps per rendered sample (0: 1) */
    float learningRate;      /* 0: 1e-2 */
    uint32_t seed;           /* parameter initialisation */
    float boundsLo[3], boundsHi[3];
    uint32_t samplesPerUpdate; /* samples rendered between training rounds (0: 4) */
    uint32_t trainingVertices; /* vertices of a training path that become training
                                  samples, from the second surface vertex on (0: a
                                  quarter of the bounce budget, at least 1) */
} mrtxRadianceCacheDesc;
MRT_API mrtResult mrtxSetRadianceCache(mrtEngine*, const mrtxRadianceCacheDesc* desc);

/* The cache's prediction for `count` queries of 16 floats each (position
 * xyz, outgoing direction xyz, normal xyz, roughness, albedo rgb, unused),
 * host memory in and out (rgbOut: 3 floats per query). */
MRT_API mrtResult mrtxRadianceCacheQuery(mrtEngine*, const float* features, uint32_t count, float* rgbOut);

/* `steps` Adam steps on host-supplied samples (features as above, targets
 * rgb); *lossOut (optional) receives the summed mean loss of the steps. */
MRT_API mrtResult mrtxRadianceCacheTrain(mrtEngine*, const float* features, const float* targets, uint32_t count,
                                         uint32_t steps, float* lossOut);

/* Reads (gridOut, mlpOut) and then writes (gridIn, mlpIn) the cache's
 * parameters; any pointer may be NULL. Grid: 16 x 2^19 x 2 floats; MLP:
 * 6 x 64 x 64 floats (W0..W4 64 x 64, then the output rows). Writing resets
 * the Adam state. */
MRT_API mrtResult mrtxRadianceCacheParams(mrtEngine*, float* gridOut, float* mlpOut, const float* gridIn,
                                          const float* mlpIn);

/* Averaging of the cache's weights for inference (Polyak averaging): every
 * training step blends the new parameters into a moving average with
 * weight 1 - d, d = min(decay, (1 + k) / (10 + k)) at step k, and every
 * query (rendering and mrtxRadianceCacheQuery) reads the average. The
 * online training's constant learning rate makes the live weights wander
 * from one step to the next; the average does not. decay in [0, 1); 0
 * switches averaging off (queries read the live weights). Default 0.99.
 * Writing parameters (mrtxRadianceCacheParams) restarts the average at
 * them. */
MRT_API mrtResult mrtxSetRadianceCacheAveraging(mrtEngine*, float decay);

/* Learning-rate decay of the cache's online training: Adam step k after
 * the schedule (re)started uses max(min(lrMin, lr), lr * 2^-(k / halfLife))
 * (lr = mrtxRadianceCacheDesc.learningRate; halfLifeSteps 0 keeps lr
 * constant). A constant rate keeps the weights wandering, and the cached
 * image's mean with them; decaying it settles the cache (measured on the
 * config-4 room: mean within 3% of the converged image, against 14% with
 * a constant rate). The schedule restarts from lr at this call, when the
 * learning rate changes, and when parameters are written. Defaults:
 * lrMin 3e-4, halfLifeSteps 96 (of 48, 96 and 192, the shortest time to
 * relMSE 1e-3 on config 4 at 1080p). */
MRT_API mrtResult mrtxSetRadianceCacheSchedule(mrtEngine*, float lrMin, float halfLifeSteps);

/* The gradients the cache's training step computes for one batch, read
 * back without taking the step: the tensor-core forward and backward pass
 * over all `count` samples (features and targets as in
 * mrtxRadianceCacheTrain) gives the gradient of the mean loss over samples
 * and channels with respect to the hash grid (gridGradOut, layout as the
 * grid in mrtxRadianceCacheParams; entries no sample touches are exactly 0)
 * and the MLP (mlpGradOut, layout as the weights); *lossOut receives the
 * mean loss. Any output may be NULL. The parameters and the optimizer's
 * state are unchanged. For checking the training kernels against a CPU
 * evaluation of the same network. */
MRT_API mrtResult mrtxRadianceCacheGradients(mrtEngine*, const float* features, const float* targets, uint32_t count,
                                             float* gridGradOut, float* mlpGradOut, float* lossOut);

/* Host-side build of the acceleration structure the engine uses for a mesh,
 * for inspection and tests (no device needed): an 8-wide compressed BVH over
 * `count` boxes (6 floats each: lo xyz, hi xyz) with leaves of at most
 * maxLeafPrims (1..3) primitives. nodesOut receives up to nodeCapacity
 * 80-byte node records (layout: miniraytrace_b200/csrc/common/device_types.h
 * MrtWideNode), primOrderOut `count` primitive indices in leaf order.
 * Builds on the binned-SAH binary builder (the reference builds a binary
 * tree on the CPU, core/src/accel/Bvh.cpp:137-156). */
MRT_API mrtResult mrtxBuildWideBvh(const float* aabbs, uint32_t count, uint32_t maxLeafPrims, void* nodesOut,
                                   uint32_t nodeCapacity, uint32_t* primOrderOut, uint32_t* nodeCountOut);

/* Builders of mrtxBuildMeshBvh. */
#define MRTX_BVH_HOST_SAH 0u     /* binned-SAH binary tree on the host (by default meshes below 16384 triangles) */
#define MRTX_BVH_HOST_LBVH 1u    /* Morton-code LBVH on the host: the device builder's reference */
#define MRTX_BVH_DEVICE_LBVH 2u  /* the same LBVH built on the engine's GPU (by default meshes of 16384+ triangles) */

/* The 8-wide BVH the engine builds for a triangle mesh (positions: 3 floats
 * per vertex; indices: 3 per triangle, each < vertexCount), from the chosen
 * builder; every builder ends in the same SAH-optimal collapse to 8-wide
 * nodes with leaves of at most maxLeafPrims (1..3) triangles. Output as
 * mrtxBuildWideBvh. MRTX_BVH_DEVICE_LBVH needs an engine (its GPU); the
 * host builders accept engine == NULL. The device and host LBVH builders
 * return identical nodes and orders. Builds on the reference's per-mesh
 * BLAS build (Renderer.cpp:333-446). */
MRT_API mrtResult mrtxBuildMeshBvh(mrtEngine* engine, const float* positions, uint32_t vertexCount,
                                   const uint32_t* indices, uint32_t triangleCount, uint32_t builder,
                                   uint32_t maxLeafPrims, void* nodesOut, uint32_t nodeCapacity,
                                   uint32_t* primOrderOut, uint32_t* nodeCountOut);

/* Opt-in denoiser of the display image, in place of the reference's
 * optional OIDN filter (core/src/post/Denoiser.cpp:10-112, scheduled by
 * Renderer.cpp:845-884; the reference built without OIDN never denoises,
 * and neither does this library until a call enables it): an edge-avoiding
 * a-trous wavelet filter (Dammertz et al. 2010) on the GPU, guided by the
 * first-hit albedo, shading normal and distance (the reference's AOVs),
 * computed by a pass of `guideSamples` jittered camera rays per pixel once
 * per accumulation. With `enabled` and the render setting `denoise` on, the
 * RGBA8_SRGB read shows the denoised image from `minSpp` samples on,
 * re-denoised when the sample count has doubled since (the reference's
 * schedule: 8, 16, 32, ... up to sppLimit), and frame infos report
 * denoised = 1; RGBA32F_LINEAR reads stay the raw mean, as in the
 * reference. Fields of zero take the defaults in brackets. */
typedef struct mrtxDenoiserDesc {
    size_t structSize;
    int32_t enabled;        /* 0: off (the default) */
    uint32_t iterations;    /* filter passes, tap spacing 1, 2, 4, ... [5], at most 10 */
    uint32_t guideSamples;  /* camera rays per pixel of the guide pass [4] */
    uint32_t minSpp;        /* first denoised display at this many samples [8] */
    float sigmaColor;       /* colour weight at 1 sample per pixel [1.0], on log(1 + colour);
                               divided by sqrt(samples) as the noise falls */
    float normalPower;      /* normal weight exponent [64] */
    float sigmaAlbedo;      /* albedo weight [0.1] */
    float sigmaDepth;       /* distance weight, relative to distance and spacing [0.1] */
} mrtxDenoiserDesc;
MRT_API mrtResult mrtxSetDenoiser(mrtEngine*, const mrtxDenoiserDesc*);
/* The denoised linear image of the samples rendered so far (RGBA32F, alpha
 * 1, rows top down; bytes >= width * height * 16), filtered now with the
 * current parameters. MRT_ERROR_INVALID_ARGUMENT while the denoiser is off. */
MRT_API mrtResult mrtxReadDenoised(mrtEngine*, float* rgba, size_t bytes);
/* The denoiser's guides (each width * height RGBA32F; bytes of each buffer
 * >= width * height * 16): mean first-hit albedo (alpha 1), and mean shading
 * normal (not renormalised) with the mean distance to the first hit in
 * alpha (0 where every guide ray missed). Computed if stale. Either pointer
 * may be NULL. */
MRT_API mrtResult mrtxReadDenoiserGuides(mrtEngine*, float* albedo, float* normalDepth, size_t bytes);

/* Largest map height mrtxBuildEnvCdfNoAlloc accepts. */
#define MRTX_ENV_CDF_NOALLOC_MAX_HEIGHT 8192u

/* The environment importance-sampling CDF of mrtxBuildEnvCdf, computed from
 * and into memory the caller already owns on the GPU, without allocating
 * any device memory. No counterpart in the reference (its CDF is built on
 * the host inside scene upload, Renderer.cpp:620-655).
 *
 * Who needs it: a caller whose device memory is all handed out by its own
 * pool or budget (a host application that has reserved the GPU's memory,
 * or a framework whose allocator owns it) cannot let a library call
 * cudaMalloc behind its back, and a caller with latency-critical work on
 * other streams cannot afford cudaFree, which synchronises the whole
 * device. mrtxBuildEnvCdf grows engine-owned buffers as needed; this entry
 * point takes no engine and keeps its scratch (row sums, the sin(theta)
 * table, row reciprocals) in a fixed 128 KiB array compiled into the
 * library, so maps are limited to MRTX_ENV_CDF_NOALLOC_MAX_HEIGHT rows
 * (any width); a taller map fails with MRT_ERROR_INVALID_ARGUMENT.
 *
 *   devTexels       w*h RGBA32F texels (16 bytes each), device memory,
 *                   16-byte aligned (read as 16-byte vectors)
 *   devCdfOut       w*h + h floats, device memory, 4-byte aligned: the
 *                   same layout and values mrtxBuildEnvCdf returns in cdfOut
 *   devIntegralOut  one float, device memory, 4-byte aligned
 *   stream          a cudaStream_t on the GPU that owns devTexels, or NULL
 *                   for that GPU's legacy default stream
 *
 * All three pointers must be device (or managed) memory of one GPU; the
 * work runs on that GPU and is asynchronous: results are complete when
 * `stream` reaches the point of this call. The first call on each GPU does
 * a one-time set-up (it loads the kernels), so make that first call before
 * any stream capture. Every call looks up the scratch array's device
 * address with cudaGetSymbolAddress (no allocation), so a device reset
 * between calls leaves no stale address behind. A call then only launches
 * kernels on `stream`: the sin(theta) table travels in their parameters,
 * so the call does not wait for `stream` and keeps no reference to host
 * memory once it returns. The scratch is shared by every call on a GPU:
 * calls that overlap in time (other threads, other streams) race and
 * corrupt each other's results, so serialise them. Nothing in the scratch
 * has to be cleared between calls. */
MRT_API mrtResult mrtxBuildEnvCdfNoAlloc(const float* devTexels, uint32_t w, uint32_t h, float* devCdfOut,
                                         float* devIntegralOut, void* stream);

#ifdef __cplusplus
} /* extern "C" */
#endif
#endif /* MRT_EXT_H */
