// The seam between the host engine (C++, g++) and the sm_100a kernels
// (CUDA, nvcc): extern "C" launch functions taking plain pointers, sizes and
// a stream, returning cudaError_t. No C++ type crosses this boundary.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../common/device_types.h"

// Radiance-cache parameters and training state on the device
// (radiance_cache.cu): hash grid (16 x 2^19 x 2 floats) and MLP (6 x 64 x 64
// floats), their gradients and Adam moments; position normalisation.
typedef struct McacheParams {
    float *grid, *mlp, *gGrid, *gMlp, *mGrid, *vGrid, *mMlp, *vMlp;
    // Exponential moving average of the parameters (Polyak averaging),
    // updated by every Adam step where the parameter changed; NULL = none.
    // Step k blends with weight 1 - d, d = min(emaDecay, (1 + k) / (10 + k)),
    // so early on the average follows the fast-changing weights closely.
    float *emaGrid, *emaMlp;
    float emaDecay;
    float* partial;          // per-block weight gradients of one step
    uint32_t partialBlocks;  // training CTAs' partial gradients `partial` holds
    float lo[3], invExtent[3];
    uint32_t step;
    float lr;
    // Learning-rate schedule: step k (1-based) uses
    // max(min(lrMin, lr), lr * 2^-((k - lrStart - 1) / lrHalfLife)), so the
    // first step after a (re)start uses lr; lrHalfLife 0 keeps lr constant.
    float lrMin, lrHalfLife;
    uint32_t lrStart;
    uint32_t* status;        // device word: bit 0 set when a tensor-core wait gave up
} McacheParams;

#ifdef __cplusplus
extern "C" {
#endif

// One wave of the wavefront path tracer: samples [sampleBase, sampleBase +
// samples) of every pixel (width * height * samples <= s->capacity slots);
// sampleBase == 0 overwrites the accumulation, otherwise it adds. Adds the
// number of kernels launched to *launches. stageEvents (may be NULL) holds 6
// timing events per bounce: event 6b+0 before extend of bounce b, 6b+1 after
// it, 6b+4 before shade (once bounce b-1's shadow rays are done), 6b+2 after
// shade, 6b+3 after shadow. With a `side` stream and syncEvents (2 per
// bounce, created with cudaEventDisableTiming) the shadow kernel of bounce b
// runs on `side`, in parallel with the extend kernel of bounce b+1; all work
// has joined `stream` again on return.
cudaError_t mrtcu_wave(const MrtFrameParams* p, const MrtWaveState* s, uint32_t sampleBase, uint32_t samples,
                       uint32_t* launches, const cudaEvent_t* stageEvents, const cudaEvent_t* syncEvents,
                       const MrtCacheArgs* cache, cudaStream_t stream, cudaStream_t side);
// Whether mrtcu_wave runs the shadow kernels beside the next bounce's extend
// when given a side stream (the build's MRT_SHADOW_OVERLAP, default 1).
int mrtcu_shadow_overlap(void);
// One-launch batch: the waves of `count` jobs (every job's scene and wave in
// its MrtBatchJob; devJobs is the device copy of hostJobs, slot and pixel
// bases ascending) rendered by one set of per-bounce kernel launches over
// their concatenated slots (sum of slots <= s->capacity). `batch` carries
// the ray counters and the error word of the whole batch; maxBounces is the
// largest of the jobs' (each path stops at its own job's bound). Events and
// the side stream as in mrtcu_wave.
cudaError_t mrtcu_wave_batch(const MrtFrameParams* batch, const MrtWaveState* s, const MrtBatchJob* devJobs,
                             const MrtBatchJob* hostJobs, uint32_t count, uint32_t maxBounces, uint32_t* launches,
                             const cudaEvent_t* stageEvents, const cudaEvent_t* syncEvents, cudaStream_t stream,
                             cudaStream_t side);
// With a cache, mrtcu_wave leaves the wave unfinalised: the cache's
// predictions are added to the paths, then this accumulates the wave.
cudaError_t mrtcu_wave_finalize(const MrtFrameParams* p, const MrtWaveState* s, uint32_t sampleBase,
                                uint32_t samples, cudaStream_t stream);

// Trace queries (closest hit / any hit) for n device-resident rays.
cudaError_t mrtcu_trace_closest(const MrtFrameParams* p, const MrtQueryRay* rays, uint32_t n, MrtQueryHit* hits,
                                cudaStream_t stream);
// The same closest-hit queries through the wavefront's extend kernel (the
// rays occupy wave slots 0..n-1; n <= s->capacity; tMax of the rays ignored:
// the extend stage traces to 1e30).
cudaError_t mrtcu_trace_closest_wave(const MrtFrameParams* p, const MrtWaveState* s, const MrtQueryRay* rays,
                                     uint32_t n, MrtQueryHit* hits, cudaStream_t stream);
cudaError_t mrtcu_trace_any(const MrtFrameParams* p, const MrtQueryRay* rays, uint32_t n, uint32_t* occluded,
                            cudaStream_t stream);

// Environment CDF (reference Renderer.cpp:620-655), bit-exact with the
// reference's sequential sums: texels = w*h float4, sinTheta = h floats
// (sin((y + 0.5) * pi / h) as evaluated on the host), cdf = w*h + h floats
// out, rowSums = h doubles and rowInv = h floats of scratch, integral = one
// float out (device memory).
cudaError_t mrtcu_env_cdf(const float4* texels, const float* sinTheta, uint32_t w, uint32_t h, float* cdf,
                          double* rowSums, float* rowInv, float* integral, cudaStream_t stream);

// Allocation-free variant over a static device scratch array (max
// MRTX_ENV_CDF_NOALLOC_MAX_HEIGHT rows). _setup runs once per device with
// that device current: it takes the scratch address (cudaGetSymbolAddress)
// and loads the kernels. hostSinTheta (h floats) is copied into the scratch.
cudaError_t mrtcu_env_cdf_noalloc_setup(int device, unsigned char** scratch);
cudaError_t mrtcu_env_cdf_noalloc(unsigned char* scratch, const float4* texels, const float* hostSinTheta, uint32_t w,
                                  uint32_t h, float* cdf, float* integral, cudaStream_t stream);

// RGBA32F readback conversion: out[i] = (sum / count, 1) with the pixel's
// own sample count; spp == 0 (nothing accumulated since the last reset)
// gives (0, 0, 0, 1) as the reference does (Renderer.cpp:904).
// Reads `count` 16-byte words at buf `reps` times with loads cached in L2
// only, from every SM (a bandwidth probe); *sink is written only for a value
// a zero-filled buffer never yields.
cudaError_t mrtcu_l2_read_probe(const void* buf, size_t count, uint32_t reps, uint32_t* sink, cudaStream_t stream);
cudaError_t mrtcu_readback_rgba32f(const double* accum, size_t npix, uint32_t spp, float4* out,
                                   cudaStream_t stream);

// Opt-in denoiser (denoise.cu): parameters of the a-trous filter.
typedef struct MrtDenoiseParams {
    uint32_t width, height, iterations, samples;  // samples: per pixel in the accumulation
    float sigmaColor, normalPower, sigmaAlbedo, sigmaDepth, albedoFloor;
} MrtDenoiseParams;
// Denoiser guides of every pixel: mean first-hit albedo (a = 1) and shading
// normal with the mean distance to that hit (w; 0 when no ray hit), over
// `samples` jittered camera rays drawing from frame indices streamBase...
cudaError_t mrtcu_denoise_guides(const MrtFrameParams* p, uint32_t samples, uint32_t streamBase, float4* albedo,
                                 float4* normalDepth, cudaStream_t stream);
// The denoised linear image of the FP64 accumulation (RGBA32F, a = 1);
// work holds 3 x width x height float4.
cudaError_t mrtcu_denoise(const double* accum, const float4* albedo, const float4* normalDepth,
                          const MrtDenoiseParams* d, float4* work, float4* out, cudaStream_t stream);
// RGBA8 resolve of a linear image (the denoised one), as mrtcu_resolve_rgba8.
cudaError_t mrtcu_resolve_rgba8_linear(const float4* color, size_t npix, float exposure, uint32_t tonemap,
                                       uchar4* out, cudaStream_t stream);
// RGBA8 resolve (reference resolve.comp:24-56): mean = sum / count,
// exposure, optional ACES, sRGB encode, UNORM8 store, alpha 255.
cudaError_t mrtcu_resolve_rgba8(const double* accum, size_t npix, float exposure, uint32_t tonemap,
                                uchar4* out, cudaStream_t stream);

// dst[i] += src[i] for n doubles (combining replicas' accumulations).
cudaError_t mrtcu_add_f64(double* dst, const double* src, size_t n, cudaStream_t stream);

// Device build of one mesh's 8-wide BVH (bvh_build.cu): positions as
// float4 (xyz used), indices 3 per triangle. Writes up to nodeCapacity
// (>= triCount) nodes with mesh-relative childBase/primBase, primOrderOut
// (triCount original triangle indices in leaf order), *nodeCountOut and the
// root box (lo xyz, hi xyz). Synchronises `stream` (it reads the per-level
// task counts). scratch: mrtcu_wide_bvh_scratch_bytes(triCount) bytes.
size_t mrtcu_wide_bvh_scratch_bytes(uint32_t triCount);
cudaError_t mrtcu_build_wide_bvh(const float4* positions, const uint32_t* indices, uint32_t triCount,
                                 uint32_t maxLeaf, void* scratch, size_t scratchBytes, MrtWideNode* nodesOut,
                                 uint32_t nodeCapacity, uint32_t* primOrderOut, uint32_t* nodeCountOut,
                                 float boundsOut[6], uint32_t* launchesOut, cudaStream_t stream);

// Commit-time assembly (pack.cu). pack_triangles writes triangles k = 0..nt-1
// of one mesh (leaf order prims[k]) to slot tbase + k of triVerts/triIndex
// with vertex ids offset by vbase; error |= 1 on an out-of-range index.
// rebase_nodes copies n mesh-relative wide nodes to dst + nodeBase with
// childBase += nodeBase and primBase += triBase.
cudaError_t mrtcu_pack_triangles(const float4* pos, uint32_t nv, const uint32_t* idx, const uint32_t* prims,
                                 uint32_t nt, uint32_t vbase, uint32_t tbase, float4* triVerts, uint4* triIndex,
                                 uint32_t* error, cudaStream_t stream);
cudaError_t mrtcu_rebase_nodes(const MrtWideNode* src, uint32_t n, uint32_t nodeBase, uint32_t triBase,
                               MrtWideNode* dst, cudaStream_t stream);
cudaError_t mrtcu_fill_f4(float4* dst, size_t n, float4 value, cudaStream_t stream);

// Radiance cache (radiance_cache.cu). Features: 16 floats per query
// (position, outgoing direction, normal, roughness, albedo, unused).
size_t mrtcu_rc_grid_floats(void);
size_t mrtcu_rc_mlp_floats(void);
uint32_t mrtcu_rc_partial_blocks(uint32_t maxBatch);
size_t mrtcu_rc_partial_floats(uint32_t maxBatch);
cudaError_t mrtcu_rc_init(McacheParams C, uint32_t seed, cudaStream_t stream);
cudaError_t mrtcu_rc_query(McacheParams C, const float* features, uint32_t n, float* out3, cudaStream_t stream);
// Cache mode of a wave: predictions for n queries added to the paths'
// radiance (scratch3: 3 floats per query), and training targets of n
// records (3 floats each). With sortScratch (mrtcu_rc_sort_scratch_words(n)
// words) the queries are evaluated in Morton order of their positions.
size_t mrtcu_rc_sort_scratch_words(uint32_t n);
cudaError_t mrtcu_rc_apply_queries(McacheParams C, const float* qFeat, const float4* qBeta, uint32_t n,
                                   uint32_t slots, float* scratch3, float4* L, uint32_t* sortScratch,
                                   cudaStream_t stream);
// The BVH builder's stable LSD radix sort of (key, value) pairs: `passes`
// 8-bit passes (even; sorted pairs end in keysA / valsA), n at most
// mrtcu_sort_pairs_max(), scratch of mrtcu_sort_pairs_scratch_words(n) words.
uint32_t mrtcu_sort_pairs_max(void);
size_t mrtcu_sort_pairs_scratch_words(uint32_t n);
cudaError_t mrtcu_sort_pairs(uint32_t* keysA, uint32_t* valsA, uint32_t* keysB, uint32_t* valsB, uint32_t n,
                             uint32_t passes, uint32_t* scratch, cudaStream_t stream);
cudaError_t mrtcu_rc_record_targets(const float4* prefix, const float4* beta, uint32_t n, uint32_t slots,
                                    const float4* L, float* targets, cudaStream_t stream);
cudaError_t mrtcu_rc_train(McacheParams* C, const float* features, const float* targets, uint32_t n, uint32_t steps,
                           uint32_t batch, float* lossOut, cudaStream_t stream);
// Gradients of the mean loss over n samples (no optimizer step): the MLP's
// into C->gMlp, the hash grid's into C->gGrid.
cudaError_t mrtcu_rc_gradients(McacheParams* C, const float* features, const float* targets, uint32_t n,
                               float* lossOut, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
