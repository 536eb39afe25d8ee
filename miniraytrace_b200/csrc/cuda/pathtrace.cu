// Progressive path tracing on sm_100a, plus the trace-query kernels.
//
// pathtraceKernel restates reference core/shaders/pathtrace.comp:100-233 (one
// path per pixel per sample, NEE + MIS against the environment, Russian
// roulette from bounce 3, firefly clamp, NaN guard), with these B200 choices:
//   - a launch renders `sampleCount` consecutive samples per pixel and keeps
//     the running sum in registers, so the FP64 accumulation buffer is read
//     and written once per launch, not once per sample;
//   - accumulation is FP64 (double4 per pixel: r, g, b, count);
//   - traversal is the watertight two-level walk of trace.cuh;
//   - the first-hit AOV buffers of the reference are not produced (they only
//     feed an optional OIDN denoiser and are not readable through the ABI).
#include <cuda_runtime.h>

#include "device_api.h"
#include "shade.cuh"
#include "trace.cuh"

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
        const float4 tx = sampleBilinear(P.textures[m.tex[3]], s.uv.x, s.uv.y);
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
    const float4 c = sampleBilinear(P.textures[slot], uv.x, uv.y);
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

struct PathCounters {
    uint32_t closest, shadow, hits;
    TraversalCounters tc;
    bool ok;
};

// One path (pathtrace.comp:100-225): returns the clamped, NaN-guarded radiance.
MRT_DEV float3 tracePath(const MrtFrameParams& P, uint32_t px, uint32_t py, uint32_t frame, PathCounters& pc) {
    Rng rng{px, py, frame, 0u};
    const float2 jitter = rng2(rng);
    const float u = (float(px) + jitter.x) / float(P.width);
    const float v = (float(py) + jitter.y) / float(P.height);
    const float sx = mixf(P.frustum[0], P.frustum[1], u);
    const float sy = mixf(P.frustum[3], P.frustum[2], v);  // top..bottom: rows go down
    float3 ro, rd;
    if (P.flags & MRT_FLAG_ORTHO) {
        ro = f3p(P.camPos) + sx * f3p(P.camRight) + sy * f3p(P.camUp);
        rd = f3p(P.camForward);
    } else {
        ro = f3p(P.camPos);
        rd = normalize(f3p(P.camForward) + sx * f3p(P.camRight) + sy * f3p(P.camUp));
    }
    float3 L = f3(0.0f), beta = f3(1.0f);
    float prevBsdfPdf = 0.0f;
    for (uint32_t bounce = 0; bounce <= P.maxBounces; ++bounce) {
        HitRecord hit;
        pc.closest++;
        pc.ok &= traceClosest(P, ro, rd, 1e30f, hit, pc.tc);
        if (hit.tri == 0xffffffffu) {
            const float3 env = envRadiance(P, rd);
            if (maxComp(env) > 0.0f) {
                float w = 1.0f;
                if (bounce > 0u) w = balanceHeuristic(prevBsdfPdf, envPdf(P, rd) * envPickPdf(P));
                L += beta * env * w;
            }
            break;
        }
        pc.hits++;
        const Surface s = makeSurface(P, rd, hit);
        const MrtMaterial& mat = P.materials[s.mat];
        const float opacity = mat.baseColorOpacity[3];
        if (opacity < 1.0f && rng1(rng) >= opacity) {  // stochastic alpha pass-through
            ro = s.pos + rd * MRT_EPS_RAY;
            continue;
        }
        float3 emission = f3p(mat.emissionRoughness);
        if (mat.tex[4] >= 0) emission = emission * texRgb(P, mat.tex[4], s.uv);
        if (maxComp(emission) > 0.0f && s.frontFace) L += beta * emission;
        const Bsdf bsdf = makeBsdf(P, s);
        float3 Tn, Bn;
        buildOnb(s.nShade, Tn, Bn);
        const float3 nd = -rd;
        float3 wo = f3(dot(nd, Tn), dot(nd, Bn), dot(nd, s.nShade));
        if (wo.z < 1e-6f) wo.z = 1e-6f;
        wo = normalize(wo);
        // next-event estimation (pathtrace.comp:180-197)
        const LightSample ls = sampleOneLight(P, s.pos, rng);
        if (ls.valid && ls.pdf > 1e-9f) {
            const float3 wi = f3(dot(ls.wi, Tn), dot(ls.wi, Bn), dot(ls.wi, s.nShade));
            float3 f;
            float bsdfPdf;
            bsdfEval(bsdf, wo, wi, f, bsdfPdf);
            if (maxComp(f) > 0.0f) {
                const float3 so = s.pos + s.nGeom * (wi.z > 0.0f ? MRT_EPS_RAY : -MRT_EPS_RAY);
                pc.shadow++;
                if (!traceAny(P, so, ls.wi, ls.dist - 2.0f * MRT_EPS_RAY, pc.ok, pc.tc)) {
                    const float w = ls.delta ? 1.0f : balanceHeuristic(ls.pdf, bsdfPdf);
                    L += beta * f * fabsf(wi.z) * ls.radiance * w / ls.pdf;
                }
            }
        }
        // BSDF bounce (pathtrace.comp:200-216)
        const BsdfSample bs = bsdfSample(bsdf, wo, rng);
        if (!bs.valid) break;
        const float3 wiWorld = normalize(Tn * bs.wi.x + Bn * bs.wi.y + s.nShade * bs.wi.z);
        beta *= bs.f * fabsf(bs.wi.z) / bs.pdf;
        prevBsdfPdf = bs.pdf;
        if (bounce >= 3u) {
            const float p = clampf(maxComp(beta), 0.05f, 0.95f);
            if (rng1(rng) >= p) break;
            beta /= p;
        }
        ro = s.pos + s.nGeom * (bs.wi.z > 0.0f ? MRT_EPS_RAY : -MRT_EPS_RAY);
        rd = wiWorld;
    }
    if (P.fireflyClamp > 0.0f) {
        const float m = maxComp(L);
        if (m > P.fireflyClamp) L *= P.fireflyClamp / m;
    }
    if (isnan(L.x) || isnan(L.y) || isnan(L.z) || isinf(L.x) || isinf(L.y) || isinf(L.z)) L = f3(0.0f);
    return L;
}

// Adds the warp's counters to ctr[0..4] = closest rays, shadow rays, node
// records fetched, triangle tests, surface hits (one atomic per warp).
MRT_DEV void warpAddCounters(unsigned long long* ctr, const PathCounters& pc) {
    if (ctr == nullptr) return;
    unsigned long long v[5] = {pc.closest, pc.shadow, pc.tc.nodes, pc.tc.tris, pc.hits};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
        if ((threadIdx.x & 31) == 0 && v[k]) atomicAdd(ctr + k, v[k]);
    }
}

// 128 threads = a 16 x 8 pixel tile; each warp covers 8 x 4 pixels.
__global__ void __launch_bounds__(128) pathtraceKernel(MrtFrameParams P, uint32_t sampleBase, uint32_t sampleCount) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t px = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const uint32_t py = blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
    const bool active = px < P.width && py < P.height;
    PathCounters pc{0, 0, 0, TraversalCounters{}, true};
    if (active) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (uint32_t s = 0; s < sampleCount; ++s) {
            const uint32_t frame = P.streamOffset + (sampleBase + s) * P.streamStride;
            const float3 L = tracePath(P, px, py, frame, pc);
            sx += double(L.x);
            sy += double(L.y);
            sz += double(L.z);
        }
        double2* a = reinterpret_cast<double2*>(P.accum + 4 * (size_t(py) * P.width + px));
        if (sampleBase == 0) {
            a[0] = make_double2(sx, sy);
            a[1] = make_double2(sz, double(sampleCount));
        } else {
            const double2 a0 = a[0], a1 = a[1];
            a[0] = make_double2(a0.x + sx, a0.y + sy);
            a[1] = make_double2(a1.x + sz, a1.y + double(sampleCount));
        }
        if (!pc.ok) atomicOr(P.errorFlags, 1u);
        if (pc.tc.bad) atomicOr(P.errorFlags, 2u);
    }
    warpAddCounters(P.rayCounters, pc);
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

}  // namespace

extern "C" cudaError_t mrtcu_pathtrace(const MrtFrameParams* p, uint32_t sampleBase, uint32_t sampleCount,
                                       cudaStream_t stream) {
    if (p->width == 0 || p->height == 0 || sampleCount == 0) return cudaSuccess;
    const dim3 grid((p->width + 15) / 16, (p->height + 7) / 8);
    pathtraceKernel<<<grid, 128, 0, stream>>>(*p, sampleBase, sampleCount);
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_trace_closest(const MrtFrameParams* p, const MrtQueryRay* rays, uint32_t n,
                                           MrtQueryHit* hits, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    traceClosestKernel<<<(n + 127) / 128, 128, 0, stream>>>(*p, rays, n, hits);
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_trace_any(const MrtFrameParams* p, const MrtQueryRay* rays, uint32_t n,
                                       uint32_t* occluded, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    traceAnyKernel<<<(n + 127) / 128, 128, 0, stream>>>(*p, rays, n, occluded);
    return cudaGetLastError();
}
