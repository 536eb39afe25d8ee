// Per-frame device passes that are bound by HBM bandwidth: the environment
// CDF scan (FP64), the RGBA32F readback conversion, the RGBA8 resolve and
// the FP64 add used to combine replicas.
#include <cuda_runtime.h>

#include "device_api.h"

namespace {

constexpr int kCdfThreads = 512;

// Block-wide scan of one double per thread: `exclusive` receives the sum of
// the values of all lower threads, `total` the sum over the block.
__device__ void blockScan(double v, double* warpSums, double& exclusive, double& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    double incl = v;
    for (int off = 1; off < 32; off <<= 1) {
        const double n = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += n;
    }
    double excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = 0.0;
    if (lane == 31) warpSums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const double s = lane < nw ? warpSums[lane] : 0.0;
        double si = s;
        for (int off = 1; off < 32; off <<= 1) {
            const double n = __shfl_up_sync(0xffffffffu, si, off);
            if (lane >= off) si += n;
        }
        if (lane < nw) warpSums[lane] = si;  // inclusive sums of warp totals
    }
    __syncthreads();
    const double before = warp > 0 ? warpSums[warp - 1] : 0.0;
    exclusive = warp > 0 ? before + excl : excl;
    total = warpSums[nw - 1];
    __syncthreads();
}

// One block per row: lum * sin(theta) in double (the product of two floats is
// exact in double), inclusive prefix along the row, stored as
// float(prefix) * float(1 / rowSum) exactly as the reference's two-pass
// normalisation (Renderer.cpp:632-646). Each thread owns a contiguous run of
// the row; the row is staged through shared memory so global loads and
// stores stay coalesced.
__global__ void __launch_bounds__(kCdfThreads) envCdfRowsKernel(const float4* __restrict__ texels,
                                                                const float* __restrict__ sinTheta, uint32_t w,
                                                                float* __restrict__ cdf, double* __restrict__ rowSums) {
    extern __shared__ float rowLum[];  // w floats
    __shared__ double warpSums[32];
    const uint32_t y = blockIdx.x;
    const float4* row = texels + size_t(y) * w;
    for (uint32_t x = threadIdx.x; x < w; x += blockDim.x) {
        const float4 p = __ldg(row + x);
        // float luminance with the reference's operation order, no contraction
        rowLum[x] = __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, p.x), __fmul_rn(0.7152f, p.y)), __fmul_rn(0.0722f, p.z));
    }
    __syncthreads();
    const double s = double(sinTheta[y]);
    const uint32_t per = (w + blockDim.x - 1) / blockDim.x;
    const uint32_t b = threadIdx.x * per, e = min(w, b + per);
    double local = 0.0;
    for (uint32_t x = b; x < e; ++x) local += double(rowLum[x]) * s;
    double run, rowSum;
    blockScan(local, warpSums, run, rowSum);
    // second pass: per-element prefix, written back into shared memory
    for (uint32_t x = b; x < e; ++x) {
        run += double(rowLum[x]) * s;
        rowLum[x] = float(run);
    }
    __syncthreads();
    const float inv = rowSum > 0.0 ? float(1.0 / rowSum) : 0.0f;
    float* out = cdf + size_t(y) * w;
    for (uint32_t x = threadIdx.x; x < w; x += blockDim.x) out[x] = __fmul_rn(rowLum[x], inv);
    if (threadIdx.x == 0) rowSums[y] = rowSum;
}

// One block: marginal CDF over rows and the integral (Renderer.cpp:642-655).
__global__ void __launch_bounds__(1024) envCdfMarginalKernel(const double* __restrict__ rowSums, uint32_t w, uint32_t h,
                                                             float* __restrict__ marginal, float* __restrict__ integral) {
    __shared__ double warpSums[32];
    const uint32_t per = (h + blockDim.x - 1) / blockDim.x;
    const uint32_t b = threadIdx.x * per, e = min(h, b + per);
    double local = 0.0;
    for (uint32_t y = b; y < e; ++y) local += rowSums[y];
    double run, tot;
    blockScan(local, warpSums, run, tot);
    for (uint32_t y = b; y < e; ++y) {
        run += rowSums[y];
        marginal[y] = tot > 0.0 ? float(run / tot) : 0.0f;
    }
    if (threadIdx.x == 0) {
        const float pi = 3.14159265358979323846f;
        const float dTheta = pi / float(h);
        const float dPhi = __fdiv_rn(__fmul_rn(2.0f, pi), float(w));
        // integral = sum_y rowSum_y * dTheta * dPhi, evaluated as the total
        // times the (exactly representable as double) float step product
        const double integ = tot * double(dTheta) * double(dPhi);
        const float f = float(integ);
        *integral = f > 1e-8f ? f : 1e-8f;
    }
}

// Mean radiance per pixel. The reference divides by the host frame count
// (Renderer.cpp:904); the per-pixel count equals it, and also stays right
// after another replica's samples were added into this buffer.
__global__ void readbackKernel(const double2* __restrict__ accum, size_t npix, bool any, float4* __restrict__ out) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const double2 a = accum[2 * i], b = accum[2 * i + 1];
    const double inv = (any && b.y > 0.0) ? 1.0 / b.y : 0.0;
    out[i] = make_float4(float(a.x * inv), float(a.y * inv), float(b.x * inv), 1.0f);
}

__device__ float acesTonemap(float x) {  // resolve.comp:13-16 (Narkowicz 2015)
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    return fminf(fmaxf((x * (a * x + b)) / (x * (c * x + d) + e), 0.0f), 1.0f);
}
__device__ float linearToSrgb(float c) {  // resolve.comp:18-22
    return c <= 0.0031308f ? c * 12.92f : 1.055f * powf(c, 1.0f / 2.4f) - 0.055f;
}
__device__ unsigned char toUnorm8(float c) { return (unsigned char)floorf(fminf(fmaxf(c, 0.0f), 1.0f) * 255.0f + 0.5f); }

__global__ void resolveKernel(const double2* __restrict__ accum, size_t npix, float exposure, uint32_t tonemap,
                              uchar4* __restrict__ out) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const double2 a = accum[2 * i], b = accum[2 * i + 1];
    float c[3] = {0.0f, 0.0f, 0.0f};
    if (b.y > 0.0) {
        c[0] = float(a.x / b.y);
        c[1] = float(a.y / b.y);
        c[2] = float(b.x / b.y);
    }
    unsigned char o[3];
    for (int k = 0; k < 3; ++k) {
        float v = c[k] * exposure;
        if (tonemap == 1u) v = acesTonemap(v);
        v = linearToSrgb(fminf(fmaxf(v, 0.0f), 1e4f));
        o[k] = toUnorm8(v);
    }
    out[i] = make_uchar4(o[0], o[1], o[2], 255);
}

__global__ void addKernel(double* __restrict__ dst, const double* __restrict__ src, size_t n) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        dst[i] += src[i];
}

}  // namespace

extern "C" cudaError_t mrtcu_env_cdf(const float4* texels, const float* sinTheta, uint32_t w, uint32_t h, float* cdf,
                                     double* rowSums, float* integral, cudaStream_t stream) {
    if (w == 0 || h == 0) return cudaSuccess;
    const size_t smem = size_t(w) * sizeof(float);
    if (smem > 48 * 1024) {
        const cudaError_t e =
            cudaFuncSetAttribute(envCdfRowsKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    envCdfRowsKernel<<<h, kCdfThreads, smem, stream>>>(texels, sinTheta, w, cdf, rowSums);
    envCdfMarginalKernel<<<1, 1024, 0, stream>>>(rowSums, w, h, cdf + size_t(w) * h, integral);
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_readback_rgba32f(const double* accum, size_t npix, uint32_t spp, float4* out,
                                              cudaStream_t stream) {
    if (npix == 0) return cudaSuccess;
    readbackKernel<<<unsigned((npix + 255) / 256), 256, 0, stream>>>(reinterpret_cast<const double2*>(accum), npix,
                                                                       spp > 0, out);
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_resolve_rgba8(const double* accum, size_t npix, float exposure, uint32_t tonemap,
                                           uchar4* out, cudaStream_t stream) {
    if (npix == 0) return cudaSuccess;
    resolveKernel<<<unsigned((npix + 255) / 256), 256, 0, stream>>>(reinterpret_cast<const double2*>(accum), npix,
                                                                      exposure, tonemap, out);
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_add_f64(double* dst, const double* src, size_t n, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    addKernel<<<148 * 8, 256, 0, stream>>>(dst, src, n);
    return cudaGetLastError();
}
