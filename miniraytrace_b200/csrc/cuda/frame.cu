// Per-frame device passes that are bound by HBM bandwidth: the environment
// CDF scan (FP64), the RGBA32F readback conversion, the RGBA8 resolve and
// the FP64 add used to combine replicas.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../../include/mrt_ext.h"
#include "device_api.h"

namespace {

// Environment CDF (reference Renderer.cpp:620-655), bit-exact with the
// reference's sequential double-precision sums. The conditional CDF of a row
// is a prefix sum that must be taken left to right (its rounding is the
// reference's), so each row's sum is one thread's dependent chain of double
// adds; rows run in parallel, 8 to a block so that every SM holds a few
// (a 1024-row map gives 128 blocks). A block's 128 threads stream the map
// through shared memory in 8-row x 128-column tiles with coalesced 16-byte
// loads, and each tile's loads are issued before the previous tile's sums
// are taken, so HBM reads overlap the chains. The marginal CDF and the
// integral are sequential over rows too (Renderer.cpp:642-655); the row
// sums are staged through shared memory so that chain waits on no DRAM
// load.
constexpr int kCdfRows = 8;
constexpr int kCdfCols = 128;

__device__ __forceinline__ float texelLuminance(float4 p) {  // the reference's float expression
    return __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, p.x), __fmul_rn(0.7152f, p.y)), __fmul_rn(0.0722f, p.z));
}

__global__ void __launch_bounds__(kCdfCols) envCdfRowsKernel(const float4* __restrict__ texels,
                                                             const float* __restrict__ sinTheta, uint32_t w,
                                                             uint32_t h, float* __restrict__ cdf,
                                                             double* __restrict__ rowSums,
                                                             float* __restrict__ rowInv) {
    __shared__ float tile[2][kCdfRows][kCdfCols + 1];
    const uint32_t y0 = blockIdx.x * kCdfRows;
    const uint32_t rows = min(uint32_t(kCdfRows), h - y0);
    const uint32_t tid = threadIdx.x;
    double acc = 0.0;  // running row sum, owned by thread tid < rows
    const double s = tid < rows ? double(sinTheta[y0 + tid]) : 0.0;
    float next[kCdfRows];  // this thread's column of the next tile
    auto fetch = [&](uint32_t c0) {
#pragma unroll
        for (int r = 0; r < kCdfRows; ++r)
            if (uint32_t(r) < rows && c0 + tid < w) next[r] = texelLuminance(__ldg(texels + size_t(y0 + r) * w + c0 + tid));
    };
    fetch(0);
    uint32_t buf = 0;
    for (uint32_t c0 = 0; c0 < w; c0 += kCdfCols, buf ^= 1u) {
        const uint32_t cols = min(uint32_t(kCdfCols), w - c0);
#pragma unroll
        for (int r = 0; r < kCdfRows; ++r)
            if (uint32_t(r) < rows && tid < cols) tile[buf][r][tid] = next[r];
        __syncthreads();
        if (c0 + kCdfCols < w) fetch(c0 + kCdfCols);  // in flight while the rows are summed
        if (tid < rows) {
            float* row = tile[buf][tid];
#pragma unroll 8
            for (uint32_t c = 0; c < cols; ++c) {
                acc = __dadd_rn(acc, __dmul_rn(double(row[c]), s));
                row[c] = float(acc);
            }
        }
        __syncthreads();
        for (uint32_t r = 0; r < rows; ++r)
            if (tid < cols) cdf[size_t(y0 + r) * w + c0 + tid] = tile[buf][r][tid];
    }
    if (tid < rows) {
        rowSums[y0 + tid] = acc;
        rowInv[y0 + tid] = acc > 0.0 ? float(1.0 / acc) : 0.0f;
    }
}

// conditional[x] *= float(1 / rowSum), as the reference's second row pass
__global__ void envCdfNormalizeKernel(float* __restrict__ cdf, const float* __restrict__ rowInv, uint32_t w,
                                      uint32_t h) {
    const size_t n = size_t(w) * h;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        cdf[i] = __fmul_rn(cdf[i], rowInv[i / w]);
}

// Marginal CDF and integral, sequential over rows (Renderer.cpp:642-655):
// the block stages 4,096 row sums at a time in shared memory, then thread 0
// runs the chains over them.
constexpr uint32_t kMarginalChunk = 4096;
__global__ void __launch_bounds__(1024) envCdfMarginalKernel(const double* __restrict__ rowSums, uint32_t w,
                                                             uint32_t h, float* __restrict__ marginal,
                                                             float* __restrict__ integral) {
    __shared__ double sRow[kMarginalChunk];
    const float pi = 3.14159265358979323846f;
    const float dTheta = __fdiv_rn(pi, float(h));
    const float dPhi = __fdiv_rn(__fmul_rn(2.0f, pi), float(w));
    double integ = 0.0, total = 0.0, run = 0.0;
    for (int pass = 0; pass < 2; ++pass) {
        for (uint32_t y0 = 0; y0 < h; y0 += kMarginalChunk) {
            const uint32_t n = min(kMarginalChunk, h - y0);
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sRow[i] = rowSums[y0 + i];
            __syncthreads();
            if (threadIdx.x != 0) continue;
            if (pass == 0) {
#pragma unroll 8
                for (uint32_t i = 0; i < n; ++i) {
                    integ = __dadd_rn(integ, __dmul_rn(__dmul_rn(sRow[i], double(dTheta)), double(dPhi)));
                    total = __dadd_rn(total, sRow[i]);
                }
            } else {
#pragma unroll 8
                for (uint32_t i = 0; i < n; ++i) {
                    run = __dadd_rn(run, sRow[i]);
                    marginal[y0 + i] = total > 0.0 ? float(__ddiv_rn(run, total)) : 0.0f;
                }
            }
        }
    }
    if (threadIdx.x == 0) {
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

// The same resolve of a linear image (resolve.comp:44-46, the denoised branch).
__global__ void resolveLinearKernel(const float4* __restrict__ color, size_t npix, float exposure, uint32_t tonemap,
                                    uchar4* __restrict__ out) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const float4 c4 = color[i];
    const float c[3] = {c4.x, c4.y, c4.z};
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
                                     double* rowSums, float* rowInv, float* integral, cudaStream_t stream) {
    if (w == 0 || h == 0) return cudaSuccess;
    envCdfRowsKernel<<<(h + kCdfRows - 1) / kCdfRows, kCdfCols, 0, stream>>>(texels, sinTheta, w, h, cdf, rowSums,
                                                                              rowInv);
    envCdfNormalizeKernel<<<148 * 4, 256, 0, stream>>>(cdf, rowInv, w, h);
    envCdfMarginalKernel<<<1, 1024, 0, stream>>>(rowSums, w, h, cdf + size_t(w) * h, integral);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Allocation-free environment CDF (mrtxBuildEnvCdfNoAlloc). The scratch of
// one call lives in this fixed device array instead of allocated buffers:
// row sums (double) at byte 0, the sin(theta) table (float) at 8 * kMax, the
// row reciprocals (float) at 12 * kMax, for maps of up to kMax rows
// (128 KiB). Nothing in it has to start at zero: every element a kernel
// reads was written earlier in the same call, in stream order. All calls on
// one device share it, so calls that overlap in time race.
namespace {
constexpr uint32_t kNoAllocMaxRows = MRTX_ENV_CDF_NOALLOC_MAX_HEIGHT;
constexpr int kNoAllocMaxDevices = 64;
__device__ __align__(256) unsigned char g_envCdfScratch[size_t(kNoAllocMaxRows) * 16];
std::mutex g_loadMutex;
bool g_kernelsLoaded[kNoAllocMaxDevices] = {};

// The sin(theta) table reaches the scratch as kernel parameters, 1,000 rows
// a launch (4,016 bytes with the destination pointer: within the 4 KiB
// parameter limit), so a call neither waits for its stream, as a copy from
// pageable host memory would, nor refers to the caller's memory once it
// returns.
constexpr uint32_t kSinChunk = 1000;
struct SinChunk {
    uint32_t first, count;
    float v[kSinChunk];
};
static_assert(sizeof(SinChunk) + sizeof(float*) <= 4096, "kernel parameters above 4 KiB");
__global__ void sinChunkKernel(float* dst, SinChunk c) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < c.count) dst[c.first + i] = c.v[i];
}
}  // namespace

// The scratch array's device address on the current device. It is looked up
// on every call (the lookup allocates nothing once the module is loaded), so
// a context that was torn down and created again (cudaDeviceReset) never
// sees a stale address. The kernels are loaded once per device, so later
// calls load no code.
extern "C" cudaError_t mrtcu_env_cdf_noalloc_setup(int device, unsigned char** scratch) {
    if (device < 0 || device >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
    void* addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_envCdfScratch);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_loadMutex);
    if (!g_kernelsLoaded[device]) {
        cudaFuncAttributes fa;
        if ((e = cudaFuncGetAttributes(&fa, envCdfRowsKernel)) != cudaSuccess) return e;
        if ((e = cudaFuncGetAttributes(&fa, envCdfNormalizeKernel)) != cudaSuccess) return e;
        if ((e = cudaFuncGetAttributes(&fa, envCdfMarginalKernel)) != cudaSuccess) return e;
        if ((e = cudaFuncGetAttributes(&fa, sinChunkKernel)) != cudaSuccess) return e;
        g_kernelsLoaded[device] = true;
    }
    *scratch = static_cast<unsigned char*>(addr);
    return cudaSuccess;
}

extern "C" cudaError_t mrtcu_env_cdf_noalloc(unsigned char* scratch, const float4* texels, const float* hostSinTheta,
                                             uint32_t w, uint32_t h, float* cdf, float* integral, cudaStream_t stream) {
    if (w == 0 || h == 0 || h > kNoAllocMaxRows) return cudaErrorInvalidValue;
    double* rowSums = reinterpret_cast<double*>(scratch);
    float* sinTheta = reinterpret_cast<float*>(scratch + size_t(kNoAllocMaxRows) * 8);
    float* rowInv = reinterpret_cast<float*>(scratch + size_t(kNoAllocMaxRows) * 12);
    for (uint32_t first = 0; first < h; first += kSinChunk) {
        SinChunk c{};
        c.first = first;
        c.count = std::min(kSinChunk, h - first);
        std::memcpy(c.v, hostSinTheta + first, c.count * sizeof(float));
        sinChunkKernel<<<(c.count + 255) / 256, 256, 0, stream>>>(sinTheta, c);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return mrtcu_env_cdf(texels, sinTheta, w, h, cdf, rowSums, rowInv, integral, stream);
}

namespace {
// Every block strides over the whole buffer, `reps` times; loads bypass L1
// (ld.global.cg), so a buffer smaller than L2 is served by L2.
__global__ void l2ReadProbeKernel(const uint4* __restrict__ buf, size_t count, uint32_t reps, uint32_t* sink) {
    const size_t stride = size_t(gridDim.x) * blockDim.x;
    uint32_t acc = 0;
    for (uint32_t r = 0; r < reps; ++r)
        for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
            const uint4 v = __ldcg(buf + i);
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    if (acc == 0x9e3779b9u) *sink = acc;
}
}  // namespace

extern "C" cudaError_t mrtcu_l2_read_probe(const void* buf, size_t count, uint32_t reps, uint32_t* sink,
                                           cudaStream_t stream) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    l2ReadProbeKernel<<<sms * 8, 256, 0, stream>>>(static_cast<const uint4*>(buf), count, reps, sink);
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

extern "C" cudaError_t mrtcu_resolve_rgba8_linear(const float4* color, size_t npix, float exposure, uint32_t tonemap,
                                                  uchar4* out, cudaStream_t stream) {
    if (npix == 0) return cudaSuccess;
    resolveLinearKernel<<<unsigned((npix + 255) / 256), 256, 0, stream>>>(color, npix, exposure, tonemap, out);
    return cudaGetLastError();
}
