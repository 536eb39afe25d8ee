// Progressive path tracing on sm_100a, plus the trace-query kernels.
//
// The path tracer restates reference core/shaders/pathtrace.comp:100-233 (one
// path per pixel per sample, NEE + MIS against the environment, Russian
// roulette from bounce 3, firefly clamp, NaN guard) as a wavefront: a wave
// holds `samples` paths of every pixel in slot arrays in HBM, and each bounce
// runs three kernels over compacted queues (extend: closest hit; shade:
// surface, NEE, BSDF, roulette; shadow: any hit), so a warp always works on
// 32 live paths of one stage instead of idling on finished ones. Per path the
// arithmetic and the order of random draws are exactly the reference's.
// Other B200 choices:
//   - accumulation is FP64 (double4 per pixel: r, g, b, count), the wave's
//     samples summed per pixel in sample order;
//   - traversal is the watertight two-level walk of trace.cuh;
//   - the first-hit AOV buffers of the reference (which only feed its
//     optional OIDN denoiser) are not accumulated by the path tracer; the
//     opt-in denoiser computes its guides in a pass of its own (aovKernel).
#include <cooperative_groups.h>
#include <map>
#include <mutex>
#include <cuda_runtime.h>

#include "device_api.h"
#include "shade.cuh"
#include "trace.cuh"

namespace cg = cooperative_groups;

namespace {

struct Surface {
    float3 pos, nGeom, nShade;
    float2 uv;
    bool frontFace;
    uint32_t mat;
};

// pathtrace.comp:39-80
MRT_DEV Surface makeSurface(const MrtFrameParams& P, float3 rayDir, const HitRecord& hit) {
    Surface s;
    const MrtInstance* in = P.instances + hit.inst;
    const uint4 tri = ldg4u(P.triIndex + hit.tri);
    const float b1 = hit.u, b2 = hit.v, b0 = 1.0f - b1 - b2;
    const float3 p0 = f3(ldg4(P.triVerts + 3 * hit.tri));
    const float3 p1 = f3(ldg4(P.triVerts + 3 * hit.tri + 1));
    const float3 p2 = f3(ldg4(P.triVerts + 3 * hit.tri + 2));
    const float3 posObj = b0 * p0 + b1 * p1 + b2 * p2;
    s.pos = xformPoint(in->o2w, posObj);
    const float3 ngObj = cross(p1 - p0, p2 - p0);
    float3 nGeom = normalize(xformTransposed(in->w2o, ngObj));
    const float3 nObj = b0 * f3(ldg4(P.normals + tri.x)) + b1 * f3(ldg4(P.normals + tri.y)) + b2 * f3(ldg4(P.normals + tri.z));
    float3 nShade = normalize(xformTransposed(in->w2o, nObj));
    const float2 uv0 = __ldg(P.uvs + tri.x), uv1 = __ldg(P.uvs + tri.y), uv2 = __ldg(P.uvs + tri.z);
    s.uv = make_float2(b0 * uv0.x + b1 * uv1.x + b2 * uv2.x, b0 * uv0.y + b1 * uv1.y + b2 * uv2.y);
    s.frontFace = dot(rayDir, nGeom) < 0.0f;
    if (!s.frontFace) {
        nGeom = -nGeom;
        nShade = -nShade;
    }
    s.mat = in->materialIndex < P.materialCount ? in->materialIndex : 0u;
    const MrtMaterial& m = P.materials[s.mat];
    if (m.tex[3] >= 0) {  // tangent-space normal map
        const float4 ta = ldg4(P.tangents + tri.x), tb = ldg4(P.tangents + tri.y), tc = ldg4(P.tangents + tri.z);
        const float3 tanH = b0 * f3(ta) + b1 * f3(tb) + b2 * f3(tc);
        const float tanW = b0 * ta.w + b1 * tb.w + b2 * tc.w;
        const float3 tangent = normalize(xformDir(in->o2w, tanH));
        const float4 tx = sampleBilinear(P.textures[m.tex[3]], P.srgbLut, s.uv.x, s.uv.y);
        const float3 tn = f3(tx.x, tx.y, tx.z) * 2.0f - f3(1.0f);
        const float3 bitan = cross(nShade, tangent) * tanW;
        nShade = normalize(tangent * tn.x + bitan * tn.y + nShade * tn.z);
        if (dot(nShade, nGeom) < 0.0f) nShade = nGeom;
    }
    s.nGeom = nGeom;
    s.nShade = nShade;
    return s;
}

MRT_DEV float3 texRgb(const MrtFrameParams& P, int slot, float2 uv) {
    const float4 c = sampleBilinear(P.textures[slot], P.srgbLut, uv.x, uv.y);
    return f3(c.x, c.y, c.z);
}

// pathtrace.comp:82-94
MRT_DEV Bsdf makeBsdf(const MrtFrameParams& P, const Surface& s) {
    const MrtMaterial& m = P.materials[s.mat];
    Bsdf b;
    b.baseColor = f3p(m.baseColorOpacity);
    if (m.tex[0] >= 0) b.baseColor = b.baseColor * texRgb(P, m.tex[0], s.uv);
    b.roughness = m.emissionRoughness[3];
    if (m.tex[1] >= 0) b.roughness = b.roughness * texRgb(P, m.tex[1], s.uv).x;
    b.metallic = m.params[0];
    if (m.tex[2] >= 0) b.metallic = b.metallic * texRgb(P, m.tex[2], s.uv).x;
    b.transmission = m.params[1];
    b.ior = m.params[2];
    b.entering = s.frontFace;
    return b;
}

// Counter slots: closest rays, shadow rays, closest-hit node records fetched,
// closest-hit triangle tests, surface hits, shadow node records, shadow
// triangle tests. Added to ctr with one atomic per warp and counter.
#ifdef MRT_TRAV_PROFILE
// Slots 8..14 (a build with MRT_TRAV_PROFILE only): the extend kernel's
// warp-step statistics (TraversalCounters).
enum { kCtrClosest, kCtrShadow, kCtrExtNodes, kCtrExtTris, kCtrHits, kCtrShNodes, kCtrShTris, kCtrPad,
       kCtrSteps, kCtrActive, kCtrTriSteps, kCtrTriPairs, kCtrTriRounds, kCtrNodeSteps, kCtrNodeLanes, kCtrCount };
#else
enum { kCtrClosest, kCtrShadow, kCtrExtNodes, kCtrExtTris, kCtrHits, kCtrShNodes, kCtrShTris, kCtrCount };
#endif
MRT_DEV void warpAddCounters(unsigned long long* ctr, const uint32_t (&c)[kCtrCount]) {
    if (ctr == nullptr) return;
#pragma unroll
    for (int k = 0; k < kCtrCount; ++k) {
        unsigned long long v = c[k];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(ctr + k, v);
    }
}

// Index of this thread's entry in a list that every thread of the current
// coalesced group appends one entry to (one atomic per group).
MRT_DEV uint32_t coalescedAppend(uint32_t* count) {
    const cg::coalesced_group g = cg::coalesced_threads();
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(count, g.size());
    return g.shfl(base, 0) + g.thread_rank();
}

// The wave's counts[] block: [0..1] path queue lengths and [2..3] shadow
// queue lengths, [4..5] and [6..7] the fetch heads of the extend and shadow
// kernels, all indexed by bounce parity `cur`. The shadow rays of bounce b
// are traced while the extend kernel of bounce b+1 runs (on another stream),
// so the two never share a counter: extend(b) resets only counters that no
// kernel of bounces b-1 and b still reads.
enum { kShadowCount = 2, kExtendHead = 4, kShadowHead = 6 };

// Slot layout of a wave: slot = pixel * samples + sample (sample-minor).
struct WaveArgs {
    uint32_t pixels;      // W * H
    uint32_t slots;       // pixels * samples of this wave
    uint32_t sampleBase;  // sample index (since reset) of the wave's first sample
    uint32_t samples;     // samples per pixel in this wave
};

MRT_DEV uint32_t frameOf(const MrtFrameParams& P, const WaveArgs& A, uint32_t slot) {
    return P.streamOffset + (A.sampleBase + slot % A.samples) * P.streamStride;
}

// One-launch batch (kMulti kernels): the job a batch slot (or, with
// `pixels`, a batch pixel) belongs to -- the last job whose base is at most
// v (a binary search over at most a few dozen bases, L1-resident) -- and
// that job's wave.
MRT_DEV uint32_t batchJobOf(const MrtBatchJobs& B, uint32_t v, bool pixels) {
    uint32_t lo = 0, hi = B.count;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((pixels ? B.jobs[mid].pixelBase : B.jobs[mid].slotBase) <= v) lo = mid;
        else hi = mid;
    }
    return lo;
}
MRT_DEV WaveArgs jobWave(const MrtBatchJob& J) { return WaveArgs{J.pixels, J.slots, J.sampleBase, J.samples}; }

// The camera ray through pixel (px, py) at sub-pixel offset `jitter`
// (pathtrace.comp:101-123: perspective or orthographic, asymmetric frustum).
MRT_DEV void cameraRay(const MrtFrameParams& P, uint32_t px, uint32_t py, float2 jitter, float3& ro, float3& rd) {
    const float u = (float(px) + jitter.x) / float(P.width);
    const float v = (float(py) + jitter.y) / float(P.height);
    const float sx = mixf(P.frustum[0], P.frustum[1], u);
    const float sy = mixf(P.frustum[3], P.frustum[2], v);  // top..bottom: rows go down
    if (P.flags & MRT_FLAG_ORTHO) {
        ro = f3p(P.camPos) + sx * f3p(P.camRight) + sy * f3p(P.camUp);
        rd = f3p(P.camForward);
    } else {
        ro = f3p(P.camPos);
        rd = normalize(f3p(P.camForward) + sx * f3p(P.camRight) + sy * f3p(P.camUp));
    }
}

// Camera rays of every slot of the wave (pathtrace.comp:101-130). In a
// one-launch batch every job's slots, each with its job's camera.
template <bool kMulti>
__global__ void __launch_bounds__(256) waveInitKernel(MrtFrameParams Pk, MrtWaveState S, WaveArgs Ak, MrtBatchJobs B) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t total = kMulti ? B.totalSlots : Ak.slots;
    if (slot == 0) {
        S.counts[0] = total;
        S.counts[1] = 0;
        S.counts[kExtendHead] = 0;  // extend fetch counter of bounce 0
    }
    if (slot >= total) return;
    const MrtBatchJob* J = kMulti ? B.jobs + batchJobOf(B, slot, false) : nullptr;
    const MrtFrameParams& P = kMulti ? J->params : Pk;
    const WaveArgs A = kMulti ? jobWave(*J) : Ak;
    const uint32_t lslot = kMulti ? slot - J->slotBase : slot;
    const uint32_t pixel = lslot / A.samples;
    const uint32_t px = pixel % P.width, py = pixel / P.width;
    Rng rng{px, py, frameOf(P, A, lslot), 0u};
    float3 ro, rd;
    cameraRay(P, px, py, rng2(rng), ro, rd);
    S.rayO[slot] = make_float4(ro.x, ro.y, ro.z, 0.0f);
    S.rayD[slot] = make_float4(rd.x, rd.y, rd.z, __uint_as_float(0u));
    S.beta[slot] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(rng.w));
    S.L[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    S.queue[0][slot] = slot;
}


// Lanes of a persistent traversal warp whose ray has finished take new rays
// from the queue (one warp-aggregated atomic) once at least this many lanes
// are idle, so warps do not idle on their longest ray (Aila and Laine 2009).
#ifndef MRT_REFILL_IDLE
#define MRT_REFILL_IDLE 8
#endif
// Threads per block of the traversal kernels and, when non-zero, the
// minimum resident blocks per SM they are compiled for (which bounds their
// registers; 0 leaves the register count to the compiler).
#ifndef MRT_TRAV_MIN_BLOCKS
#define MRT_TRAV_MIN_BLOCKS 7
#endif
#if MRT_TRAV_MIN_BLOCKS > 0
#define MRT_TRAV_BOUNDS __launch_bounds__(MRT_TRAV_THREADS, MRT_TRAV_MIN_BLOCKS)
#else
#define MRT_TRAV_BOUNDS __launch_bounds__(MRT_TRAV_THREADS)
#endif

// Refill step shared by the traversal kernels: idle lanes get consecutive
// queue positions; `drained` becomes true (warp-uniformly) once the whole
// queue is handed out. Returns the lane's position, or 0xffffffff. (One
// atomic per refill of at least MRT_REFILL_IDLE lanes; reserving runs of 32
// to 128 positions per atomic instead measured no faster.)
MRT_DEV uint32_t refillLane(uint32_t* head, uint32_t n, bool active, bool& drained) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t idle = __ballot_sync(0xffffffffu, !active);
    if (__popc(idle) < MRT_REFILL_IDLE) return 0xffffffffu;
    const int leader = __ffs(idle) - 1;
    uint32_t base = 0;
    if (int(lane) == leader) base = atomicAdd(head, uint32_t(__popc(idle)));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (base + uint32_t(__popc(idle)) >= n) drained = true;
    if (active) return 0xffffffffu;
    const uint32_t i = base + uint32_t(__popc(idle & ((1u << lane) - 1u)));
    return i < n ? i : 0xffffffffu;
}

// Closest hit of every queued ray (intersect.glsl:88-125 traceRay).
// Persistent warps with lane refill; every lane of a warp stays in the loop
// until the warp has no ray left.
template <bool kMulti>
__global__ void MRT_TRAV_BOUNDS waveExtendKernel(MrtFrameParams Pk, MrtWaveState S, uint32_t cur, MrtBatchJobs B) {
    const uint32_t* __restrict__ q = S.queue[cur];
    const uint32_t n = S.counts[cur];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S.counts[cur ^ 1u] = 0;  // next queue and this bounce's shadow queue fill during shade
        S.counts[kShadowCount + cur] = 0;
        S.counts[kShadowHead + cur] = 0;
        S.counts[kExtendHead + (cur ^ 1u)] = 0;  // for the next bounce's extend
    }
    uint32_t c[kCtrCount] = {};
    TraversalCounters tc;
    bool ok = true, active = false, drained = false;
    uint32_t slot = 0, job = 0;  // job: the lane's ray's batch job (kMulti)
    WideTrav T;
    SplitStack stack;
    for (;;) {
        if (!drained) {
            const uint32_t i = refillLane(S.counts + kExtendHead + cur, n, active, drained);
            if (i != 0xffffffffu) {
                slot = q[i];
                if (kMulti) job = batchJobOf(B, slot, false);
                const float4 o = S.rayO[slot], d = S.rayD[slot];
                travBegin(kMulti ? B.jobs[job].params : Pk, T, f3(o), f3(d), 1e30f);
                active = true;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        const MrtFrameParams& P = kMulti ? B.jobs[job].params : Pk;
        const int r = travWarpStep<false, kMulti>(P, T, stack, tc, active, B.jobs, job);
        if (active && r != kTravRunning) {
            HitRecord h = T.hit;
            if (h.tri != 0xffffffffu) refineHit(P, T.wo, T.wd, h);
            S.hit[slot] = make_float4(h.t, h.u, h.v, __uint_as_float(h.tri));
            S.hitInst[slot] = h.inst;
            ok &= T.ok;
            c[kCtrClosest]++;
            active = false;
        }
    }
    if (!ok) atomicOr(Pk.errorFlags, 1u);
    if (tc.bad) atomicOr(Pk.errorFlags, 2u);
    c[kCtrExtNodes] = tc.nodes;
    c[kCtrExtTris] = tc.tris;
#ifdef MRT_TRAV_PROFILE
    c[kCtrSteps] = tc.steps;
    c[kCtrActive] = tc.activeLanes;
    c[kCtrTriSteps] = tc.triSteps;
    c[kCtrTriPairs] = tc.triPairs;
    c[kCtrTriRounds] = tc.triRounds;
    c[kCtrNodeSteps] = tc.nodeSteps;
    c[kCtrNodeLanes] = tc.nodeLanes;
#endif
    warpAddCounters(Pk.rayCounters, c);
}

// Shading of every queued path at its hit (pathtrace.comp:133-216): miss ->
// environment with MIS; hit -> alpha pass-through, emission, one-light NEE
// (a shadow ray with its contribution is queued), BSDF sample, Russian
// roulette, next ray queued. The draws from the path's pcg4d stream happen in
// the reference's order; the counter lives in beta.w between bounces.
// Training-path selection of the cache mode: whether the path of (pixel,
// frame index) is a training path, a hash of both, so training paths spread
// over the image and every sample (of every sample stream) picks its own.
MRT_DEV bool cacheTrainingPath(const MrtCacheArgs& K, uint32_t pixel, uint32_t frame) {
    uint32_t x = pixel * 0x9e3779b1u ^ (frame + 1u) * 0x85ebca77u;
    x ^= x >> 15;
    x *= 0x2c1b3c6du;
    x ^= x >> 12;
    return x % K.trainStride == 0u;
}

// The 16 cache input features of a surface vertex: position, outgoing
// direction, shading normal, roughness, base colour, zero padding.
MRT_DEV void writeCacheFeatures(float* out, const Surface& s, float3 wo, const Bsdf& bsdf) {
    float4* f = reinterpret_cast<float4*>(out);
    f[0] = make_float4(s.pos.x, s.pos.y, s.pos.z, wo.x);
    f[1] = make_float4(wo.y, wo.z, s.nShade.x, s.nShade.y);
    f[2] = make_float4(s.nShade.z, bsdf.roughness, bsdf.baseColor.x, bsdf.baseColor.y);
    f[3] = make_float4(bsdf.baseColor.z, 0.0f, 0.0f, 0.0f);
}

// Threads per block of the shade kernel and, when non-zero, the minimum
// resident blocks per SM it is compiled for (a register bound; 0 leaves the
// register count, about 100, to the compiler).
#ifndef MRT_SHADE_THREADS
#define MRT_SHADE_THREADS 256
#endif
#ifndef MRT_SHADE_MIN_BLOCKS
#define MRT_SHADE_MIN_BLOCKS 0
#endif
constexpr uint32_t kShadeBlock = MRT_SHADE_THREADS;
#if MRT_SHADE_MIN_BLOCKS > 0
#define MRT_SHADE_BOUNDS __launch_bounds__(kShadeBlock, MRT_SHADE_MIN_BLOCKS)
#else
#define MRT_SHADE_BOUNDS __launch_bounds__(kShadeBlock)
#endif

// Appends to two lists at once, one atomic per list per block (a per-warp
// atomic on the same counter serialised in L2: 4.2 M a bounce at 1080p x 64
// spp): every thread of the block calls it; *ia / *ib receive the thread's
// entry (valid where pa / pb).
MRT_DEV void blockAppend2(uint32_t* ca, bool pa, uint32_t& ia, uint32_t* cb, bool pb, uint32_t& ib,
                          uint32_t (&s)[2][kShadeBlock / 32 + 1]) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, below = (1u << lane) - 1u;
    const uint32_t ba = __ballot_sync(0xffffffffu, pa), bb = __ballot_sync(0xffffffffu, pb);
    if (lane == 0) {
        s[0][warp] = __popc(ba);
        s[1][warp] = __popc(bb);
    }
    __syncthreads();
    if (threadIdx.x < 2) {  // exclusive prefix over the warps, then the block's base
        uint32_t run = 0;
        for (uint32_t w = 0; w < kShadeBlock / 32; ++w) {
            const uint32_t v = s[threadIdx.x][w];
            s[threadIdx.x][w] = run;
            run += v;
        }
        s[threadIdx.x][kShadeBlock / 32] = run ? atomicAdd(threadIdx.x ? cb : ca, run) : 0u;
    }
    __syncthreads();
    ia = s[0][kShadeBlock / 32] + s[0][warp] + __popc(ba & below);
    ib = s[1][kShadeBlock / 32] + s[1][warp] + __popc(bb & below);
    __syncthreads();  // s is reused by the next call
}

template <bool kCache, bool kMulti>
__global__ void MRT_SHADE_BOUNDS waveShadeKernel(MrtFrameParams Pk, MrtWaveState S, WaveArgs Ak,
                                                               uint32_t cur, MrtCacheArgs K, MrtBatchJobs B) {
    const uint32_t* __restrict__ q = S.queue[cur];
    uint32_t* __restrict__ qn = S.queue[cur ^ 1u];
    const uint32_t n = S.counts[cur];
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t c[kCtrCount] = {};
    __shared__ uint32_t sAppend[2][kShadeBlock / 32 + 1];
    // block-uniform trip count: the queue appends below are block-wide
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i - threadIdx.x < n; i += stride) {
        const bool valid = i < n;
        bool cont = false, shadow = false;
        uint32_t slot = 0;
        float3 shOrig = f3(0.0f), shDir = f3(0.0f), shContrib = f3(0.0f);
        float shTMax = 0.0f;
        bool cacheQuery = false;  // cache mode: the path stops here and takes the cache's prediction
        if (valid) {
            slot = q[i];
            const MrtBatchJob* J = kMulti ? B.jobs + batchJobOf(B, slot, false) : nullptr;
            const MrtFrameParams& P = kMulti ? J->params : Pk;
            const WaveArgs A = kMulti ? jobWave(*J) : Ak;
            const uint32_t lslot = kMulti ? slot - J->slotBase : slot;  // the slot within its job's wave
            const float4 o4 = S.rayO[slot], d4 = S.rayD[slot], b4 = S.beta[slot], L4 = S.L[slot];
            const float4 h4 = S.hit[slot];
            const uint32_t pixel = lslot / A.samples;
            Rng rng{pixel % P.width, pixel / P.width, frameOf(P, A, lslot), __float_as_uint(b4.w)};
            const uint32_t bounce = __float_as_uint(d4.w);
            float3 ro = f3(o4), rd = f3(d4), beta = f3(b4), L = f3(L4);
            float prevBsdfPdf = o4.w;
            float spread = L4.w;  // cache mode: what is left of the path's spread budget
            const uint32_t tri = __float_as_uint(h4.w);
            if (tri == 0xffffffffu) {
                const float3 env = envRadiance(P, rd);
                if (maxComp(env) > 0.0f) {
                    float w = 1.0f;
                    if (bounce > 0u) w = balanceHeuristic(prevBsdfPdf, envPdf(P, rd) * envPickPdf(P));
                    L += beta * env * w;
                }
            } else {
                c[kCtrHits]++;
                HitRecord hit;
                hit.t = h4.x;
                hit.u = h4.y;
                hit.v = h4.z;
                hit.tri = tri;
                hit.inst = S.hitInst[slot];
                const Surface s = makeSurface(P, rd, hit);
                const MrtMaterial& mat = P.materials[s.mat];
                const float opacity = mat.baseColorOpacity[3];
                if (opacity < 1.0f && rng1(rng) >= opacity) {  // stochastic alpha pass-through
                    ro = s.pos + rd * MRT_EPS_RAY;
                    cont = bounce + 1u <= P.maxBounces;
                } else {
                    float3 emission = f3p(mat.emissionRoughness);
                    if (mat.tex[4] >= 0) emission = emission * texRgb(P, mat.tex[4], s.uv);
                    if (maxComp(emission) > 0.0f && s.frontFace) L += beta * emission;
                    const Bsdf bsdf = makeBsdf(P, s);
                    if (kCache) {
                        // Path spread (Mueller et al. 2021, "Real-time Neural
                        // Radiance Caching", section 3.4): the camera vertex
                        // sets the budget sqrt(c a0), a0 = t^2 / (4 pi cos);
                        // every later vertex spends t / sqrt(p cos) of it, p
                        // the solid-angle pdf of the bounce that reached it.
                        // A path is queried at the first vertex past bounce 0
                        // with the budget spent, so sharp reflections and
                        // refractions carry on to the surfaces they show
                        // instead of showing the cache's smooth prediction.
                        const float cosHit = fmaxf(fabsf(dot(rd, s.nGeom)), 1e-4f);
                        if (bounce == 0u) spread = h4.x * sqrtf(K.spreadC * 0.0795774715f / cosHit);  // 1 / (4 pi)
                        else spread -= h4.x * rsqrtf(fmaxf(prevBsdfPdf * cosHit, 1e-30f));
                    }
                    if (kCache && bounce >= 1u) {
                        // A query (the cache stands for everything scattered
                        // from here on) or, on a training path's first
                        // vertices, a training record; its features are
                        // written out here.
                        // (Queries and records append in separate branches: a
                        // coalesced group then shares one list.)
                        const bool training = cacheTrainingPath(K, pixel, frameOf(P, A, lslot));
                        cacheQuery = !training && spread <= 0.0f;
                        const float4 b4 = make_float4(beta.x, beta.y, beta.z, __uint_as_float(slot));
                        if (cacheQuery) {
                            const uint32_t idx = coalescedAppend(K.qCount);
                            if (idx < K.qCap) {
                                writeCacheFeatures(K.qFeat + size_t(idx) * 16, s, -rd, bsdf);
                                K.qBeta[idx] = b4;
                            }
                        } else if (training && bounce <= K.recordBounces) {
                            const uint32_t idx = coalescedAppend(K.rCount);
                            if (idx < K.rCap) {
                                writeCacheFeatures(K.rFeat + size_t(idx) * 16, s, -rd, bsdf);
                                K.rPrefix[idx] = make_float4(L.x, L.y, L.z, __uint_as_float(slot));
                                K.rBeta[idx] = b4;
                            }
                        }
                    }
                    float3 Tn, Bn;
                    buildOnb(s.nShade, Tn, Bn);
                    const float3 nd = -rd;
                    float3 wo = f3(dot(nd, Tn), dot(nd, Bn), dot(nd, s.nShade));
                    if (wo.z < 1e-6f) wo.z = 1e-6f;
                    wo = normalize(wo);
                    const LightSample ls = cacheQuery ? LightSample{} : sampleOneLight(P, s.pos, rng);
                    if (!cacheQuery && ls.valid && ls.pdf > 1e-9f) {
                        const float3 wi = f3(dot(ls.wi, Tn), dot(ls.wi, Bn), dot(ls.wi, s.nShade));
                        float3 f;
                        float bsdfPdf;
                        bsdfEval(bsdf, wo, wi, f, bsdfPdf);
                        if (maxComp(f) > 0.0f) {
                            const float w = ls.delta ? 1.0f : balanceHeuristic(ls.pdf, bsdfPdf);
                            shadow = true;
                            shOrig = s.pos + s.nGeom * (wi.z > 0.0f ? MRT_EPS_RAY : -MRT_EPS_RAY);
                            shDir = ls.wi;
                            shTMax = ls.dist - 2.0f * MRT_EPS_RAY;
                            shContrib = beta * f * fabsf(wi.z) * ls.radiance * w / ls.pdf;
                        }
                    }
                    const BsdfSample bs = cacheQuery ? BsdfSample{} : bsdfSample(bsdf, wo, rng);
                    if (!cacheQuery && bs.valid) {
                        const float3 wiWorld = normalize(Tn * bs.wi.x + Bn * bs.wi.y + s.nShade * bs.wi.z);
                        beta *= bs.f * fabsf(bs.wi.z) / bs.pdf;
                        prevBsdfPdf = bs.pdf;
                        bool alive = true;
                        if (bounce >= 3u) {
                            const float p = clampf(maxComp(beta), 0.05f, 0.95f);
                            if (rng1(rng) >= p) alive = false;
                            else beta /= p;
                        }
                        if (alive) {
                            ro = s.pos + s.nGeom * (bs.wi.z > 0.0f ? MRT_EPS_RAY : -MRT_EPS_RAY);
                            rd = wiWorld;
                            cont = bounce + 1u <= P.maxBounces;
                        }
                    }
                }
            }
            S.L[slot] = make_float4(L.x, L.y, L.z, kCache ? spread : 0.0f);
            if (cont) {
                S.rayO[slot] = make_float4(ro.x, ro.y, ro.z, prevBsdfPdf);
                S.rayD[slot] = make_float4(rd.x, rd.y, rd.z, __uint_as_float(bounce + 1u));
                S.beta[slot] = make_float4(beta.x, beta.y, beta.z, __uint_as_float(rng.w));
            }
        }
        uint32_t qi, si;
        blockAppend2(&S.counts[cur ^ 1u], cont, qi, &S.counts[kShadowCount + cur], shadow, si, sAppend);
        if (cont) qn[qi] = slot;
        if (shadow) {
            S.shO[si] = make_float4(shOrig.x, shOrig.y, shOrig.z, shTMax);
            S.shD[si] = make_float4(shDir.x, shDir.y, shDir.z, __uint_as_float(slot));
            S.shC[si] = make_float4(shContrib.x, shContrib.y, shContrib.z, 0.0f);
        }
    }
    warpAddCounters(Pk.rayCounters, c);
}

// Any-hit test of every queued shadow ray; unoccluded rays add their NEE
// contribution to their path (pathtrace.comp:192-195). A path has at most
// one shadow ray per bounce, so the update needs no atomics. Persistent
// warps with lane refill, as the extend kernel.
template <bool kMulti>
__global__ void MRT_TRAV_BOUNDS waveShadowKernel(MrtFrameParams Pk, MrtWaveState S, uint32_t cur, MrtBatchJobs B) {
    const uint32_t n = S.counts[kShadowCount + cur];
    uint32_t c[kCtrCount] = {};
    TraversalCounters tc;
    bool ok = true, active = false, drained = false;
    uint32_t idx = 0, job = 0;  // job: the lane's ray's batch job (kMulti)
    WideTrav T;
    SplitStack stack;
    for (;;) {
        if (!drained) {
            const uint32_t i = refillLane(S.counts + kShadowHead + cur, n, active, drained);
            if (i != 0xffffffffu) {
                idx = i;
                const float4 o = S.shO[i], d = S.shD[i];
                if (kMulti) job = batchJobOf(B, __float_as_uint(d.w), false);
                travBegin(kMulti ? B.jobs[job].params : Pk, T, f3(o), f3(d), o.w);
                active = true;
                c[kCtrShadow]++;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        const MrtFrameParams& P = kMulti ? B.jobs[job].params : Pk;
        const int r = travWarpStep<true, kMulti>(P, T, stack, tc, active, B.jobs, job);
        if (active) {
            if (r != kTravRunning) {
                ok &= T.ok;
                if (r != kTravOccluded) {
                    const uint32_t slot = __float_as_uint(S.shD[idx].w);
                    const float4 cc = S.shC[idx];
                    float4 L = S.L[slot];
                    L.x = L.x + cc.x;
                    L.y = L.y + cc.y;
                    L.z = L.z + cc.z;
                    S.L[slot] = L;
                }
                active = false;
            }
        }
    }
    if (!ok) atomicOr(Pk.errorFlags, 1u);
    if (tc.bad) atomicOr(Pk.errorFlags, 2u);
    c[kCtrShNodes] = tc.nodes;
    c[kCtrShTris] = tc.tris;
    warpAddCounters(Pk.rayCounters, c);
}

// Firefly clamp and NaN guard of every finished path (pathtrace.comp:219-225),
// then the FP64 accumulation: per pixel, the wave's samples are added in
// sample order (pathtrace.comp:227-228).
// In a one-launch batch every job's pixels, each into its job's
// accumulation.
template <bool kMulti>
__global__ void __launch_bounds__(256) waveFinalizeKernel(MrtFrameParams Pk, MrtWaveState S, WaveArgs Ak,
                                                          MrtBatchJobs B) {
    const uint32_t gp = blockIdx.x * blockDim.x + threadIdx.x;
    if (gp >= (kMulti ? B.totalPixels : Ak.pixels)) return;
    const MrtBatchJob* J = kMulti ? B.jobs + batchJobOf(B, gp, true) : nullptr;
    const MrtFrameParams& P = kMulti ? J->params : Pk;
    const WaveArgs A = kMulti ? jobWave(*J) : Ak;
    const uint32_t pixel = kMulti ? gp - J->pixelBase : gp;
    const size_t slotBase = kMulti ? J->slotBase : 0u;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (uint32_t s = 0; s < A.samples; ++s) {
        const float4 l4 = S.L[slotBase + size_t(pixel) * A.samples + s];
        float3 L = f3(l4);
        if (P.fireflyClamp > 0.0f) {
            const float m = maxComp(L);
            if (m > P.fireflyClamp) L *= P.fireflyClamp / m;
        }
        if (isnan(L.x) || isnan(L.y) || isnan(L.z) || isinf(L.x) || isinf(L.y) || isinf(L.z)) L = f3(0.0f);
        sx += double(L.x);
        sy += double(L.y);
        sz += double(L.z);
    }
    double2* acc = reinterpret_cast<double2*>(P.accum + 4 * size_t(pixel));
    if (A.sampleBase == 0) {
        acc[0] = make_double2(sx, sy);
        acc[1] = make_double2(sz, double(A.samples));
    } else {
        const double2 a0 = acc[0], a1 = acc[1];
        acc[0] = make_double2(a0.x + sx, a0.y + sy);
        acc[1] = make_double2(a1.x + sz, a1.y + double(A.samples));
    }
}

// Query rays through the wavefront's own closest-hit stage: the rays become
// wave slots 0..n-1 on queue 0 (bounce 0, tMax 1e30 as every path ray), the
// extend kernel runs as in a render, and its hit records are converted to
// query hits. This checks the persistent, refilling, warp-batched kernel the
// renderer times, not a one-ray-per-thread twin of it.
__global__ void queryToWaveKernel(const MrtQueryRay* __restrict__ rays, uint32_t n, MrtWaveState S) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        S.counts[0] = n;
        S.counts[kExtendHead] = 0;
    }
    if (i >= n) return;
    const MrtQueryRay r = rays[i];
    S.rayO[i] = make_float4(r.origin[0], r.origin[1], r.origin[2], 0.0f);
    S.rayD[i] = make_float4(r.dir[0], r.dir[1], r.dir[2], __uint_as_float(0u));
    S.queue[0][i] = i;
}

__global__ void waveToQueryKernel(MrtFrameParams P, MrtWaveState S, uint32_t n, MrtQueryHit* __restrict__ hits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 h = S.hit[i];
    const uint32_t tri = __float_as_uint(h.w);
    MrtQueryHit out;
    out.pad[0] = out.pad[1] = 0;
    if (tri != 0xffffffffu && tri < P.triCount) {
        out.t = h.x;
        out.instance = P.instances[S.hitInst[i]].userId;
        out.prim = ldg4u(P.triIndex + tri).w;
        out.hit = 1;
        out.u = h.y;
        out.v = h.z;
    } else {
        out.t = 1e30f;
        out.instance = 0;
        out.prim = 0;
        out.hit = 0;
        out.u = out.v = 0.0f;
    }
    hits[i] = out;
}

__global__ void traceClosestKernel(MrtFrameParams P, const MrtQueryRay* __restrict__ rays, uint32_t n,
                                   MrtQueryHit* __restrict__ hits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const MrtQueryRay r = rays[i];
    HitRecord h;
    TraversalCounters tc;
    const bool ok = traceClosest(P, f3p(r.origin), f3p(r.dir), r.tMax, h, tc);
    if (!ok) atomicOr(P.errorFlags, 1u);
    if (tc.bad) atomicOr(P.errorFlags, 2u);
    MrtQueryHit out;
    out.pad[0] = out.pad[1] = 0;
    if (h.tri != 0xffffffffu) {
        out.t = h.t;
        out.instance = P.instances[h.inst].userId;
        out.prim = ldg4u(P.triIndex + h.tri).w;
        out.hit = 1;
        out.u = h.u;
        out.v = h.v;
    } else {
        out.t = r.tMax;
        out.instance = 0;
        out.prim = 0;
        out.hit = 0;
        out.u = out.v = 0.0f;
    }
    hits[i] = out;
}

__global__ void traceAnyKernel(MrtFrameParams P, const MrtQueryRay* __restrict__ rays, uint32_t n,
                               uint32_t* __restrict__ occluded) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const MrtQueryRay r = rays[i];
    bool ok = true;
    TraversalCounters tc;
    occluded[i] = traceAny(P, f3p(r.origin), f3p(r.dir), r.tMax, ok, tc) ? 1u : 0u;
    if (!ok) atomicOr(P.errorFlags, 1u);
    if (tc.bad) atomicOr(P.errorFlags, 2u);
}

// Denoiser guides: the reference's first-hit AOVs (pathtrace.comp:130-167,
// 230-233) -- at the first surface a camera ray does not pass through
// (stochastic alpha as in the path tracer), the albedo (base colour times
// its texture) and the shading normal -- averaged over `samples` jittered
// camera rays per pixel (a miss adds zero, as in the reference), plus the
// mean distance travelled to that surface over the rays that found one (0
// when none did) in normalDepth.w. The rays draw from frame indices
// streamBase, streamBase + 1, ..., a stream apart from the renders'.
__global__ void __launch_bounds__(128) aovKernel(MrtFrameParams P, uint32_t samples, uint32_t streamBase,
                                                 float4* __restrict__ albedo, float4* __restrict__ normalDepth) {
    const uint32_t pixel = blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= P.width * P.height) return;
    const uint32_t px = pixel % P.width, py = pixel / P.width;
    float3 alb = f3(0.0f), nrm = f3(0.0f);
    float depth = 0.0f;
    uint32_t found = 0;
    TraversalCounters tc;
    bool ok = true;
    for (uint32_t k = 0; k < samples; ++k) {
        Rng rng{px, py, streamBase + k, 0u};
        float3 ro, rd;
        cameraRay(P, px, py, rng2(rng), ro, rd);
        float travelled = 0.0f;
        for (uint32_t layer = 0; layer <= P.maxBounces; ++layer) {  // the path tracer's bound on pass-throughs
            HitRecord hit;
            ok &= traceClosest(P, ro, rd, 1e30f, hit, tc);
            if (hit.tri == 0xffffffffu) break;
            const Surface s = makeSurface(P, rd, hit);
            const MrtMaterial& m = P.materials[s.mat];
            travelled += hit.t;
            const float opacity = m.baseColorOpacity[3];
            if (opacity < 1.0f && rng1(rng) >= opacity) {
                ro = s.pos + rd * MRT_EPS_RAY;
                continue;
            }
            float3 a = f3p(m.baseColorOpacity);
            if (m.tex[0] >= 0) a = a * texRgb(P, m.tex[0], s.uv);
            alb += a;
            nrm += s.nShade;
            depth += travelled;
            ++found;
            break;
        }
    }
    if (!ok) atomicOr(P.errorFlags, 1u);
    if (tc.bad) atomicOr(P.errorFlags, 2u);
    const float inv = 1.0f / float(samples);
    albedo[pixel] = make_float4(alb.x * inv, alb.y * inv, alb.z * inv, 1.0f);
    normalDepth[pixel] = make_float4(nrm.x * inv, nrm.y * inv, nrm.z * inv, found ? depth / float(found) : 0.0f);
}

}  // namespace

namespace {
// Persistent grid for the queue kernels: enough resident blocks to fill every
// SM, each block striding over the queue.
int persistentBlocks(const void* kernel, int threads) {
    int dev = 0, sms = 0, perSm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, threads, 0);
    return sms * (perSm > 0 ? perSm : 1);
}
// Grids of exactly the resident blocks of each wavefront kernel on a device
// (the cache-mode shade kernel uses more registers, so fewer of its blocks
// fit an SM; a grid sized for the other variant would leave a second, serial
// wave of blocks). Computed once per device, on first use with it current.
struct WaveGrids {
    int extend, shade, shadeCache, shadow;
    int extendMulti, shadeMulti, shadowMulti;  // one-launch batch variants
};

const WaveGrids& waveGrids() {
    static std::mutex mutex;
    static std::map<int, WaveGrids> grids;  // nodes never move: references stay valid
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mutex);
    auto it = grids.find(dev);
    if (it == grids.end())
        it = grids.emplace(dev, WaveGrids{persistentBlocks(reinterpret_cast<const void*>(waveExtendKernel<false>),
                                                           MRT_TRAV_THREADS),
                                          persistentBlocks(reinterpret_cast<const void*>(waveShadeKernel<false, false>),
                                                           kShadeBlock),
                                          persistentBlocks(reinterpret_cast<const void*>(waveShadeKernel<true, false>),
                                                           kShadeBlock),
                                          persistentBlocks(reinterpret_cast<const void*>(waveShadowKernel<false>),
                                                           MRT_TRAV_THREADS),
                                          persistentBlocks(reinterpret_cast<const void*>(waveExtendKernel<true>),
                                                           MRT_TRAV_THREADS),
                                          persistentBlocks(reinterpret_cast<const void*>(waveShadeKernel<false, true>),
                                                           kShadeBlock),
                                          persistentBlocks(reinterpret_cast<const void*>(waveShadowKernel<true>),
                                                           MRT_TRAV_THREADS)})
                 .first;
    return it->second;
}
}  // namespace

// Stream order of a wave's bounces. Without a side stream (or without its
// sync events) every kernel runs on `main` in order. With one, the shadow
// kernel of bounce b runs on `side` after shade(b), in parallel with
// extend(b+1) on `main`: the two persistent kernels fill each other's
// draining tails, and shade(b+1) waits for both (the shadow kernel adds to
// the paths' radiance, which shade(b+1) rewrites). The cross-stream waits
// use `sync` (2 events per bounce, created without timing, the cheap kind
// to wait on); the timing events `ev` (may be NULL; 6 per bounce) are only
// recorded: [0] before extend, [1] after extend, [4] once the previous
// bounce's shadow rays are done (before shade), [2] after shade, [3] after
// shadow (on the stream that ran it), [5] unused.
#ifndef MRT_SHADOW_OVERLAP
#define MRT_SHADOW_OVERLAP 1
#endif
struct BounceStreams {
    cudaStream_t main, side;
    const cudaEvent_t* ev;
    const cudaEvent_t* sync;
    bool overlap() const { return MRT_SHADOW_OVERLAP && side != nullptr && sync != nullptr; }
    void record(uint32_t b, int i, cudaStream_t s) const {
        if (ev) cudaEventRecord(ev[6 * size_t(b) + i], s);
    }
    void beforeExtend(uint32_t b) const { record(b, 0, main); }
    void beforeShade(uint32_t b) const {
        record(b, 1, main);
        if (overlap() && b > 0) cudaStreamWaitEvent(main, sync[2 * size_t(b - 1) + 1], 0);
        record(b, 4, main);
    }
    cudaStream_t beforeShadow(uint32_t b) const {
        record(b, 2, main);
        if (!overlap()) return main;
        cudaEventRecord(sync[2 * size_t(b)], main);
        cudaStreamWaitEvent(side, sync[2 * size_t(b)], 0);
        return side;
    }
    void afterShadow(uint32_t b) const {
        record(b, 3, overlap() ? side : main);
        if (overlap()) cudaEventRecord(sync[2 * size_t(b) + 1], side);
    }
    void join(uint32_t last) const {
        if (overlap()) cudaStreamWaitEvent(main, sync[2 * size_t(last) + 1], 0);
    }
};

extern "C" int mrtcu_shadow_overlap(void) { return MRT_SHADOW_OVERLAP; }

extern "C" cudaError_t mrtcu_wave_finalize(const MrtFrameParams* p, const MrtWaveState* s, uint32_t sampleBase,
                                           uint32_t samples, cudaStream_t stream) {
    const uint32_t pixels = p->width * p->height;
    if (pixels == 0 || samples == 0) return cudaSuccess;
    WaveArgs A{pixels, pixels * samples, sampleBase, samples};
    waveFinalizeKernel<false><<<(pixels + 255) / 256, 256, 0, stream>>>(*p, *s, A, MrtBatchJobs{});
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_wave(const MrtFrameParams* p, const MrtWaveState* s, uint32_t sampleBase,
                                  uint32_t samples, uint32_t* launches, const cudaEvent_t* stageEvents,
                                  const cudaEvent_t* syncEvents, const MrtCacheArgs* cache, cudaStream_t stream,
                                  cudaStream_t side) {
    const uint32_t pixels = p->width * p->height;
    if (pixels == 0 || samples == 0) return cudaSuccess;
    if (uint64_t(pixels) * samples > s->capacity) return cudaErrorInvalidValue;
    const WaveGrids& g = waveGrids();
    const int gExtend = g.extend, gShade = g.shade, gShadeCache = g.shadeCache, gShadow = g.shadow;
    WaveArgs A{pixels, pixels * samples, sampleBase, samples};
    uint32_t n = 0;
    waveInitKernel<false><<<(A.slots + 255) / 256, 256, 0, stream>>>(*p, *s, A, MrtBatchJobs{});
    ++n;
    const BounceStreams bs{stream, side, stageEvents, syncEvents};
    for (uint32_t b = 0; b <= p->maxBounces; ++b) {
        const uint32_t cur = b & 1u;
        bs.beforeExtend(b);
        waveExtendKernel<false><<<gExtend, MRT_TRAV_THREADS, 0, stream>>>(*p, *s, cur, MrtBatchJobs{});
        bs.beforeShade(b);
        if (cache)
            waveShadeKernel<true, false><<<gShadeCache, kShadeBlock, 0, stream>>>(*p, *s, A, cur, *cache,
                                                                                   MrtBatchJobs{});
        else
            waveShadeKernel<false, false><<<gShade, kShadeBlock, 0, stream>>>(*p, *s, A, cur, MrtCacheArgs{},
                                                                              MrtBatchJobs{});
        waveShadowKernel<false><<<gShadow, MRT_TRAV_THREADS, 0, bs.beforeShadow(b)>>>(*p, *s, cur, MrtBatchJobs{});
        bs.afterShadow(b);
        n += 3;
    }
    bs.join(p->maxBounces);
    if (!cache) {  // the cache mode finalises after applying the cache (mrtcu_wave_finalize)
        waveFinalizeKernel<false><<<(pixels + 255) / 256, 256, 0, stream>>>(*p, *s, A, MrtBatchJobs{});
        ++n;
    }
    if (launches) *launches += n;
    return cudaGetLastError();
}

// One-launch batch: the waves of `count` jobs (devJobs: device copy of the
// job table; the host copy gives the totals) rendered by one set of
// per-bounce launches over the concatenated slots. `batch` carries the
// batch's ray counters and error word (every job's own parameters carry
// its scene). stageEvents as in mrtcu_wave.
extern "C" cudaError_t mrtcu_wave_batch(const MrtFrameParams* batch, const MrtWaveState* s, const MrtBatchJob* devJobs,
                                        const MrtBatchJob* hostJobs, uint32_t count, uint32_t maxBounces,
                                        uint32_t* launches, const cudaEvent_t* stageEvents,
                                        const cudaEvent_t* syncEvents, cudaStream_t stream, cudaStream_t side) {
    if (count == 0) return cudaSuccess;
    const MrtBatchJob& last = hostJobs[count - 1];
    const uint32_t totalSlots = last.slotBase + last.slots, totalPixels = last.pixelBase + last.pixels;
    if (totalSlots == 0) return cudaSuccess;
    if (totalSlots > s->capacity) return cudaErrorInvalidValue;
    const MrtBatchJobs B{devJobs, count, totalSlots, totalPixels, 0u};
    const WaveGrids& g = waveGrids();
    const WaveArgs none{0u, 0u, 0u, 1u};
    uint32_t n = 0;
    waveInitKernel<true><<<(totalSlots + 255) / 256, 256, 0, stream>>>(*batch, *s, none, B);
    ++n;
    const BounceStreams bs{stream, side, stageEvents, syncEvents};
    for (uint32_t b = 0; b <= maxBounces; ++b) {
        const uint32_t cur = b & 1u;
        bs.beforeExtend(b);
        waveExtendKernel<true><<<g.extendMulti, MRT_TRAV_THREADS, 0, stream>>>(*batch, *s, cur, B);
        bs.beforeShade(b);
        waveShadeKernel<false, true><<<g.shadeMulti, kShadeBlock, 0, stream>>>(*batch, *s, none, cur, MrtCacheArgs{}, B);
        waveShadowKernel<true><<<g.shadowMulti, MRT_TRAV_THREADS, 0, bs.beforeShadow(b)>>>(*batch, *s, cur, B);
        bs.afterShadow(b);
        n += 3;
    }
    bs.join(maxBounces);
    waveFinalizeKernel<true><<<(totalPixels + 255) / 256, 256, 0, stream>>>(*batch, *s, none, B);
    ++n;
    if (launches) *launches += n;
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_trace_closest(const MrtFrameParams* p, const MrtQueryRay* rays, uint32_t n,
                                           MrtQueryHit* hits, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    traceClosestKernel<<<(n + 127) / 128, 128, 0, stream>>>(*p, rays, n, hits);
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_trace_closest_wave(const MrtFrameParams* p, const MrtWaveState* s,
                                                const MrtQueryRay* rays, uint32_t n, MrtQueryHit* hits,
                                                cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    if (n > s->capacity) return cudaErrorInvalidValue;
    const WaveGrids& g = waveGrids();
    queryToWaveKernel<<<(n + 255) / 256, 256, 0, stream>>>(rays, n, *s);
    waveExtendKernel<false><<<g.extend, MRT_TRAV_THREADS, 0, stream>>>(*p, *s, 0u, MrtBatchJobs{});
    waveToQueryKernel<<<(n + 255) / 256, 256, 0, stream>>>(*p, *s, n, hits);
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_trace_any(const MrtFrameParams* p, const MrtQueryRay* rays, uint32_t n,
                                       uint32_t* occluded, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    traceAnyKernel<<<(n + 127) / 128, 128, 0, stream>>>(*p, rays, n, occluded);
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_denoise_guides(const MrtFrameParams* p, uint32_t samples, uint32_t streamBase,
                                            float4* albedo, float4* normalDepth, cudaStream_t stream) {
    const uint32_t pixels = p->width * p->height;
    if (pixels == 0 || samples == 0) return cudaSuccess;
    aovKernel<<<(pixels + 127) / 128, 128, 0, stream>>>(*p, samples, streamBase, albedo, normalDepth);
    return cudaGetLastError();
}
