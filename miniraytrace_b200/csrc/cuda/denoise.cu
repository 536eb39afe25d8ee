// Opt-in denoiser of the display image: an edge-avoiding a-trous wavelet
// filter (Dammertz, Sewtz, Hanika and Lensch, "Edge-Avoiding A-Trous Wavelet
// Transform for fast Global Illumination Filtering", HPG 2010) guided by the
// first-hit albedo, shading normal and distance of aovKernel (pathtrace.cu).
// It stands in for the reference's optional OIDN filter (core/src/post/
// Denoiser.cpp:10-112, fed by Renderer.cpp:845-884 with the same three
// images); OIDN's network is not restated, so the outputs differ.
//
// The filter runs on demodulated colour (mean colour / albedo, the albedo
// floored), so texture detail is not blurred, then multiplies the albedo
// back. Pass i (i = 0 .. iterations-1) takes the 5 x 5 B3-spline taps
// (1/16, 1/4, 3/8, 1/4, 1/16) at spacing 2^i, each weighted by
//   colour:  exp(-|c_p - c_q|^2 / (s^2 2^-i)),  c = log(1 + colour) per channel,
//            s = sigmaColor / sqrt(samples) (the noise falls as 1/sqrt(samples))
//   normal:  max(0, n_p . n_q)^normalPower
//   albedo:  exp(-|a_p - a_q|^2 / sigmaAlbedo^2)
//   depth:   exp(-|z_p - z_q| / (sigmaDepth z_p 2^i))
// where a pixel whose rays all missed (distance 0) weighs only other such
// pixels (by colour). A pass reads three float4 images (colour, albedo,
// normal and distance: 100 MB at 1920x1080, within the 126 MB L2) and
// writes one, so its 25 taps are plain loads served by L1 and L2.
#include <cuda_runtime.h>

#include "device_api.h"

namespace {

constexpr int kTile = 16;

__device__ float3 f3of(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ float dist2(float3 a, float3 b) {
    const float x = a.x - b.x, y = a.y - b.y, z = a.z - b.z;
    return x * x + y * y + z * z;
}
// The colour the weights compare: log(1 + colour), the demodulated value
// times the floored albedo (a log keeps bright and dim pixels apart at any
// exposure).
__device__ float3 logColour(float3 irr, float3 al, float floorA) {
    return make_float3(__logf(1.0f + fmaxf(irr.x * fmaxf(al.x, floorA), 0.0f)),
                       __logf(1.0f + fmaxf(irr.y * fmaxf(al.y, floorA), 0.0f)),
                       __logf(1.0f + fmaxf(irr.z * fmaxf(al.z, floorA), 0.0f)));
}

// Mean colour of the FP64 accumulation divided by the albedo guide, and the
// unit shading normal with the distance.
__global__ void demodulateKernel(const double2* __restrict__ accum, const float4* __restrict__ albedo,
                                 const float4* __restrict__ normalDepth, size_t npix, float floorA,
                                 float4* __restrict__ irr, float4* __restrict__ unitNormal) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const double2 a = accum[2 * i], b = accum[2 * i + 1];
    const double inv = b.y > 0.0 ? 1.0 / b.y : 0.0;
    const float4 al = albedo[i];
    irr[i] = make_float4(float(a.x * inv) / fmaxf(al.x, floorA), float(a.y * inv) / fmaxf(al.y, floorA),
                         float(b.x * inv) / fmaxf(al.z, floorA), 1.0f);
    const float4 nd = normalDepth[i];
    const float len2 = nd.x * nd.x + nd.y * nd.y + nd.z * nd.z;
    const float s = len2 > 0.0f ? rsqrtf(len2) : 0.0f;
    unitNormal[i] = make_float4(nd.x * s, nd.y * s, nd.z * s, nd.w);
}

__global__ void __launch_bounds__(kTile * kTile) atrousKernel(const float4* __restrict__ in, float4* __restrict__ out,
                                                              const float4* __restrict__ albedo,
                                                              const float4* __restrict__ unitNormal, MrtDenoiseParams d,
                                                              int step, float invColor2) {
    const int x = blockIdx.x * kTile + threadIdx.x, y = blockIdx.y * kTile + threadIdx.y;
    const int w = int(d.width), h = int(d.height);
    if (x >= w || y >= h) return;
    const float kB3[3] = {0.375f, 0.25f, 0.0625f};
    const size_t p = size_t(y) * w + x;
    const float3 ap = f3of(albedo[p]), ccp = logColour(f3of(in[p]), ap, d.albedoFloor);
    const float4 np = unitNormal[p];
    const bool hitP = np.w > 0.0f;
    const float invAlbedo2 = 1.0f / (d.sigmaAlbedo * d.sigmaAlbedo);
    const float invDepth = hitP ? 1.0f / (d.sigmaDepth * np.w * float(step)) : 0.0f;
    float3 sum = make_float3(0.0f, 0.0f, 0.0f);
    float wsum = 0.0f;
    for (int dy = -2; dy <= 2; ++dy) {
        const int yy = y + dy * step;
        if (yy < 0 || yy >= h) continue;
        for (int dx = -2; dx <= 2; ++dx) {
            const int xx = x + dx * step;
            if (xx < 0 || xx >= w) continue;
            const size_t q = size_t(yy) * w + xx;
            const float4 nq = unitNormal[q];
            if ((nq.w > 0.0f) != hitP) continue;
            const float3 cq = f3of(in[q]), aq = f3of(albedo[q]);
            float wgt = kB3[dx < 0 ? -dx : dx] * kB3[dy < 0 ? -dy : dy] *
                        __expf(-dist2(ccp, logColour(cq, aq, d.albedoFloor)) * invColor2);
            if (hitP) {
                const float nd = fmaxf(np.x * nq.x + np.y * nq.y + np.z * nq.z, 0.0f);
                wgt *= __powf(nd, d.normalPower) * __expf(-dist2(ap, aq) * invAlbedo2) *
                       __expf(-fabsf(np.w - nq.w) * invDepth);
            }
            sum.x += wgt * cq.x;
            sum.y += wgt * cq.y;
            sum.z += wgt * cq.z;
            wsum += wgt;
        }
    }
    // the centre tap always weighs 0.140625 > 0
    const float inv = 1.0f / wsum;
    out[p] = make_float4(sum.x * inv, sum.y * inv, sum.z * inv, 1.0f);
}

__global__ void remodulateKernel(const float4* __restrict__ irr, const float4* __restrict__ albedo, size_t npix,
                                 float floorA, float4* __restrict__ out) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const float4 c = irr[i], al = albedo[i];
    out[i] = make_float4(c.x * fmaxf(al.x, floorA), c.y * fmaxf(al.y, floorA), c.z * fmaxf(al.z, floorA), 1.0f);
}

}  // namespace

extern "C" cudaError_t mrtcu_denoise(const double* accum, const float4* albedo, const float4* normalDepth,
                                     const MrtDenoiseParams* d, float4* work, float4* out, cudaStream_t stream) {
    const size_t npix = size_t(d->width) * d->height;
    if (npix == 0) return cudaSuccess;
    float4* src = work;
    float4* dst = work + npix;
    float4* unitNormal = work + 2 * npix;
    const unsigned blocks = unsigned((npix + 255) / 256);
    demodulateKernel<<<blocks, 256, 0, stream>>>(reinterpret_cast<const double2*>(accum), albedo, normalDepth, npix,
                                                 d->albedoFloor, src, unitNormal);
    const dim3 grid((d->width + kTile - 1) / kTile, (d->height + kTile - 1) / kTile), block(kTile, kTile);
    for (uint32_t i = 0; i < d->iterations; ++i) {
        const float noise2 = d->sigmaColor * d->sigmaColor / float(d->samples > 0 ? d->samples : 1);
        const float sigma2 = noise2 * ldexpf(1.0f, -int(i));
        atrousKernel<<<grid, block, 0, stream>>>(src, dst, albedo, unitNormal, *d, 1 << i, 1.0f / sigma2);
        float4* t = src;
        src = dst;
        dst = t;
    }
    remodulateKernel<<<blocks, 256, 0, stream>>>(src, albedo, npix, d->albedoFloor, out);
    return cudaGetLastError();
}
