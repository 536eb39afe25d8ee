// Neural radiance cache (after Mueller, Rousselle, Novak and Keller, "Real-time
// Neural Radiance Caching for Path Tracing", SIGGRAPH 2021): a multiresolution
// hash-grid encoding of position (Mueller et al., "Instant Neural Graphics
// Primitives", 2022), spherical harmonics of the outgoing direction and raw
// surface features, fed to a 5 x 64 ReLU MLP predicting outgoing radiance.
// Trained online with a relative L2 loss and Adam.
//
// Query features, 16 floats: position xyz (world), direction xyz (unit,
// outgoing, world), normal xyz (unit), roughness, albedo rgb, unused.
// Encoding, 64 floats: 16 levels x 2 hash-grid features, 16 SH coefficients
// of the direction (degree 4), normal mapped to [0, 1]^3, roughness, albedo,
// a constant 1 (the network's only bias), zero padding.
// Network: 5 hidden layers of 64 (W0..W4, 64 x 64, ReLU), output W5 (3 x 64
// stored as 16 x 64, rows 3..15 unused). No other biases.
//
// All arithmetic is FP32 on the CUDA cores: at 64 queries per block the
// 5 x 64 x 64 layers cost ~21k FMA per query, about a millisecond for the
// two million queries of a 1080p frame; the weights are read from shared
// memory as broadcasts and the activations from padded shared rows.
#include <cuda_runtime.h>

#include "device_api.h"

namespace {

constexpr int kLevels = 16;
constexpr uint32_t kTableSize = 1u << 19;
constexpr int kWidth = 64;
constexpr int kPad = kWidth + 1;  // shared-memory row stride (no bank conflicts)
constexpr int kLayers = 5;        // hidden layers
constexpr int kOutRows = 16;
constexpr int kBlock = 64;        // queries per block = threads per block
// Grid scale of level l: 16 * 2^(7 l / 15), 16 -> 2048 in 16 geometric
// steps, as float literals so any other implementation can use the same values.
__constant__ float kLevelScale[kLevels] = {16.0f, 22.110605239868164f, 30.554931640625f, 42.2242546081543f, 58.35023880004883f, 80.63494873046875f, 111.43047332763672f, 153.98719787597656f, 212.79690551757812f, 294.0667724609375f, 406.3746643066406f, 561.5744018554688f, 776.046875f, 1072.42919921875f, 1482.003662109375f, 2048.0f};

__device__ float levelScale(int l) { return kLevelScale[l]; }

__device__ uint32_t gridIndex(uint32_t x, uint32_t y, uint32_t z, uint32_t res) {
    const uint64_t dense = uint64_t(res + 1) * (res + 1) * (res + 1);
    if (dense <= kTableSize) return x + (res + 1) * (y + (res + 1) * z);
    return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & (kTableSize - 1u);
}

// Real spherical harmonics up to degree 4 (16 values) of a unit vector.
__device__ void shDeg4(float x, float y, float z, float* o) {
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    o[0] = 0.28209479177387814f;
    o[1] = -0.48860251190291987f * y;
    o[2] = 0.48860251190291987f * z;
    o[3] = -0.48860251190291987f * x;
    o[4] = 1.0925484305920792f * xy;
    o[5] = -1.0925484305920792f * yz;
    o[6] = 0.94617469575755997f * zz - 0.31539156525251999f;
    o[7] = -1.0925484305920792f * xz;
    o[8] = 0.54627421529603959f * (xx - yy);
    o[9] = 0.59004358992664352f * y * (-3.0f * xx + yy);
    o[10] = 2.8906114426405538f * xy * z;
    o[11] = 0.45704579946446572f * y * (1.0f - 5.0f * zz);
    o[12] = 0.3731763325901154f * z * (5.0f * zz - 3.0f);
    o[13] = 0.45704579946446572f * x * (1.0f - 5.0f * zz);
    o[14] = 1.4453057213202769f * z * (xx - yy);
    o[15] = 0.59004358992664352f * x * (-xx + 3.0f * yy);
}

struct Corners {
    uint32_t idx[kLevels][8];
    float w[kLevels][8];
};

// Encoding of one query into enc[0..63]; corner indices and weights kept
// for the backward pass when `corners` is given.
__device__ void encode(const McacheParams& C, const float* f, float* enc, Corners* corners) {
    float p[3];
    for (int a = 0; a < 3; ++a) {
        const float u = (f[a] - C.lo[a]) * C.invExtent[a];
        p[a] = fminf(fmaxf(u, 0.0f), 1.0f);
    }
    for (int l = 0; l < kLevels; ++l) {
        const float s = levelScale(l);
        const uint32_t res = uint32_t(ceilf(s));
        float fr[3];
        uint32_t b[3];
        for (int a = 0; a < 3; ++a) {
            const float x = p[a] * s;
            const float fl = fminf(floorf(x), float(res - 1));
            b[a] = uint32_t(fl);
            fr[a] = x - fl;
        }
        float e0 = 0.0f, e1 = 0.0f;
        for (int c = 0; c < 8; ++c) {
            const uint32_t cx = b[0] + (c & 1), cy = b[1] + ((c >> 1) & 1), cz = b[2] + ((c >> 2) & 1);
            const float w = ((c & 1) ? fr[0] : 1.0f - fr[0]) * ((c & 2) ? fr[1] : 1.0f - fr[1]) *
                            ((c & 4) ? fr[2] : 1.0f - fr[2]);
            const uint32_t i = uint32_t(l) * kTableSize + gridIndex(cx, cy, cz, res);
            const float2 g = reinterpret_cast<const float2*>(C.grid)[i];
            e0 += w * g.x;
            e1 += w * g.y;
            if (corners) {
                corners->idx[l][c] = i;
                corners->w[l][c] = w;
            }
        }
        enc[2 * l] = e0;
        enc[2 * l + 1] = e1;
    }
    float d[3] = {f[3], f[4], f[5]};
    const float dl = rsqrtf(fmaxf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2], 1e-20f));
    shDeg4(d[0] * dl, d[1] * dl, d[2] * dl, enc + 32);
    enc[48] = 0.5f * f[6] + 0.5f;
    enc[49] = 0.5f * f[7] + 0.5f;
    enc[50] = 0.5f * f[8] + 0.5f;
    enc[51] = f[9];
    enc[52] = f[10];
    enc[53] = f[11];
    enc[54] = f[12];
    enc[55] = 1.0f;
    for (int k = 56; k < kWidth; ++k) enc[k] = 0.0f;
}

// Weight matrix `layer` (rows x 64, row-major) into shared memory.
__device__ void loadWeights(const float* __restrict__ mlp, int layer, int rows, float* sW) {
    const float* W = mlp + size_t(layer) * kWidth * kWidth;
    for (int i = threadIdx.x; i < rows * kWidth; i += blockDim.x) sW[(i / kWidth) * kPad + (i % kWidth)] = W[i];
}

// out[t][j] = sum_k W[j][k] * in[t][k] for this thread's row t, j < rows;
// ReLU when `relu`.
__device__ void layerForward(const float* sW, const float* in, float* out, int rows, bool relu) {
    const int t = threadIdx.x;
    for (int j = 0; j < rows; ++j) {
        float acc = 0.0f;
#pragma unroll 16
        for (int k = 0; k < kWidth; ++k) acc = fmaf(sW[j * kPad + k], in[t * kPad + k], acc);
        out[t * kPad + j] = relu ? fmaxf(acc, 0.0f) : acc;
    }
}

// Inference: one query per thread, 64 per block. out3 (n x 3) = max(net, 0).
__global__ void __launch_bounds__(kBlock) queryKernel(McacheParams C, const float* __restrict__ features, uint32_t n,
                                                      float* __restrict__ out3) {
    extern __shared__ float smem[];
    float* sW = smem;                     // kWidth x kPad
    float* a0 = sW + kWidth * kPad;       // kBlock x kPad
    float* a1 = a0 + kBlock * kPad;
    const uint32_t q = blockIdx.x * kBlock + threadIdx.x;
    const bool valid = q < n;
    float f[16];
    for (int k = 0; k < 16; ++k) f[k] = valid ? features[size_t(q) * 16 + k] : 0.0f;
    encode(C, f, a0 + threadIdx.x * kPad, nullptr);
    float* in = a0;
    float* out = a1;
    for (int l = 0; l <= kLayers; ++l) {
        __syncthreads();
        loadWeights(C.mlp, l, l < kLayers ? kWidth : kOutRows, sW);
        __syncthreads();
        layerForward(sW, in, out, l < kLayers ? kWidth : 3, l < kLayers);
        float* t = in;
        in = out;
        out = t;
    }
    if (valid)
        for (int c = 0; c < 3; ++c) out3[size_t(q) * 3 + c] = fmaxf(in[threadIdx.x * kPad + c], 0.0f);
}

// One training step's forward + backward for 64 samples per block: loss =
// mean over samples and channels of (y - t)^2 / (y^2 + 0.01), y held fixed in
// the denominator. Weight gradients are reduced over the block's samples and
// added to gMlp; grid gradients are scattered to the 8 corners of each level.
__global__ void __launch_bounds__(kBlock) trainKernel(McacheParams C, const float* __restrict__ features,
                                                      const float* __restrict__ targets, uint32_t n, float invBatch,
                                                      float* __restrict__ lossOut) {
    extern __shared__ float smem[];
    float* sW = smem;                            // kWidth x kPad
    float* act = sW + kWidth * kPad;             // (kLayers + 1) x kBlock x kPad: enc, h1..h5
    float* dA = act + (kLayers + 1) * kBlock * kPad;  // kBlock x kPad: gradient of the current layer's output
    float* dB = dA + kBlock * kPad;
    const int t = threadIdx.x;
    const uint32_t s = blockIdx.x * kBlock + t;
    const bool valid = s < n;
    float f[16];
    for (int k = 0; k < 16; ++k) f[k] = valid ? features[size_t(s) * 16 + k] : 0.0f;
    Corners corners;
    encode(C, f, act + t * kPad, &corners);
    for (int l = 0; l <= kLayers; ++l) {
        __syncthreads();
        loadWeights(C.mlp, l, l < kLayers ? kWidth : kOutRows, sW);
        __syncthreads();
        float* out = l < kLayers ? act + (l + 1) * kBlock * kPad : dA;  // the output goes to dA first
        layerForward(sW, act + l * kBlock * kPad, out, l < kLayers ? kWidth : 3, l < kLayers);
    }
    // output gradient (3 channels), zero for padding samples
    float loss = 0.0f;
    for (int c = 0; c < kWidth; ++c) {
        float g = 0.0f;
        if (c < 3 && valid) {
            const float y = dA[t * kPad + c], tg = targets[size_t(s) * 3 + c];
            const float den = y * y + 0.01f;
            loss += (y - tg) * (y - tg) / den;
            g = 2.0f * (y - tg) / den * invBatch;
        }
        dA[t * kPad + c] = g;
    }
    if (lossOut && valid) atomicAdd(lossOut, loss * invBatch);
    // backward through W5 .. W0
    for (int l = kLayers; l >= 0; --l) {
        const int rows = l < kLayers ? kWidth : 3;
        __syncthreads();
        loadWeights(C.mlp, l, l < kLayers ? kWidth : kOutRows, sW);
        __syncthreads();
        // weight gradient: gW[j][k] = sum_t dA[t][j] * in[t][k]
        const float* in = act + l * kBlock * kPad;
        float* gW = C.gMlp + size_t(l) * kWidth * kWidth;
        for (int e = t; e < rows * kWidth; e += kBlock) {
            const int j = e / kWidth, k = e % kWidth;
            float acc = 0.0f;
            for (int r = 0; r < kBlock; ++r) acc = fmaf(dA[r * kPad + j], in[r * kPad + k], acc);
            atomicAdd(gW + e, acc);
        }
        // input gradient: dB[t][k] = sum_j W[j][k] * dA[t][j], through the ReLU of `in` (hidden inputs)
        for (int k = 0; k < kWidth; ++k) {
            float acc = 0.0f;
            for (int j = 0; j < rows; ++j) acc = fmaf(sW[j * kPad + k], dA[t * kPad + j], acc);
            if (l > 0 && in[t * kPad + k] <= 0.0f) acc = 0.0f;
            dB[t * kPad + k] = acc;
        }
        __syncthreads();
        float* x = dA;
        dA = dB;
        dB = x;
    }
    // dA holds the encoding gradient: scatter the grid part
    if (valid) {
        for (int l = 0; l < kLevels; ++l) {
            const float g0 = dA[t * kPad + 2 * l], g1 = dA[t * kPad + 2 * l + 1];
            if (g0 == 0.0f && g1 == 0.0f) continue;
            for (int c = 0; c < 8; ++c) {
                const uint32_t i = corners.idx[l][c];
                const float w = corners.w[l][c];
                atomicAdd(C.gGrid + 2 * size_t(i), w * g0);
                atomicAdd(C.gGrid + 2 * size_t(i) + 1, w * g1);
            }
        }
    }
}

// Adam on every parameter; gradients are cleared for the next step.
__global__ void adamKernel(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                           size_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        g[i] = 0.0f;
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

// Deterministic initial values: grid uniform in [-1e-4, 1e-4], weights
// uniform in +-sqrt(6 / (fan_in + fan_out)).
__device__ float hashUniform(uint32_t i, uint32_t seed) {
    uint32_t x = i * 747796405u + seed * 2891336453u + 1u;
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return float(x >> 8) * (1.0f / 16777216.0f) * 2.0f - 1.0f;
}

__global__ void initKernel(float* __restrict__ grid, size_t gridN, float* __restrict__ mlp, uint32_t seed) {
    const size_t total = gridN + size_t(kLayers + 1) * kWidth * kWidth;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        if (i < gridN) {
            grid[i] = 1e-4f * hashUniform(uint32_t(i), seed);
        } else {
            const size_t w = i - gridN;
            const int layer = int(w / (kWidth * kWidth));
            const int row = int((w % (kWidth * kWidth)) / kWidth);
            const float bound = layer < kLayers ? sqrtf(6.0f / (kWidth + kWidth)) : sqrtf(6.0f / (kWidth + 3));
            mlp[w] = (layer == kLayers && row >= 3) ? 0.0f : bound * hashUniform(uint32_t(w), seed ^ 0x9e3779b9u);
        }
    }
}

size_t smemQuery() { return sizeof(float) * (kWidth * kPad + 2 * kBlock * kPad); }
size_t smemTrain() { return sizeof(float) * (kWidth * kPad + (kLayers + 1 + 2) * kBlock * kPad); }

unsigned gridFor(size_t n) {
    const size_t b = (n + 255) / 256;
    return unsigned(b < 148u * 32u ? (b > 0 ? b : 1) : 148u * 32u);
}

}  // namespace

extern "C" size_t mrtcu_rc_grid_floats() { return size_t(kLevels) * kTableSize * 2; }
extern "C" size_t mrtcu_rc_mlp_floats() { return size_t(kLayers + 1) * kWidth * kWidth; }

extern "C" cudaError_t mrtcu_rc_init(McacheParams C, uint32_t seed, cudaStream_t stream) {
    const size_t gridN = mrtcu_rc_grid_floats(), mlpN = mrtcu_rc_mlp_floats();
    initKernel<<<gridFor(gridN + mlpN), 256, 0, stream>>>(C.grid, gridN, C.mlp, seed);
    cudaError_t e;
    for (float* p : {C.gGrid, C.mGrid, C.vGrid})
        if ((e = cudaMemsetAsync(p, 0, gridN * sizeof(float), stream)) != cudaSuccess) return e;
    for (float* p : {C.gMlp, C.mMlp, C.vMlp})
        if ((e = cudaMemsetAsync(p, 0, mlpN * sizeof(float), stream)) != cudaSuccess) return e;
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_rc_query(McacheParams C, const float* features, uint32_t n, float* out3,
                                      cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(queryKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smemQuery()));
    if (e != cudaSuccess) return e;
    queryKernel<<<(n + kBlock - 1) / kBlock, kBlock, smemQuery(), stream>>>(C, features, n, out3);
    return cudaGetLastError();
}

// `steps` Adam steps; step k trains on samples [k*batch, (k+1)*batch) modulo n.
extern "C" cudaError_t mrtcu_rc_train(McacheParams* C, const float* features, const float* targets, uint32_t n,
                                      uint32_t steps, uint32_t batch, float* lossOut, cudaStream_t stream) {
    if (n == 0 || steps == 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(trainKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smemTrain()));
    if (e != cudaSuccess) return e;
    batch = batch < n ? batch : n;
    const size_t gridN = mrtcu_rc_grid_floats(), mlpN = mrtcu_rc_mlp_floats();
    for (uint32_t k = 0; k < steps; ++k) {
        const uint32_t first = uint32_t((uint64_t(k) * batch) % n);
        const uint32_t count = first + batch <= n ? batch : n - first;
        trainKernel<<<(count + kBlock - 1) / kBlock, kBlock, smemTrain(), stream>>>(
            *C, features + size_t(first) * 16, targets + size_t(first) * 3, count, 1.0f / (3.0f * float(count)),
            lossOut);
        ++C->step;
        const float b1 = 0.9f, b2 = 0.99f;
        const float c1 = 1.0f / (1.0f - powf(b1, float(C->step))), c2 = 1.0f / (1.0f - powf(b2, float(C->step)));
        adamKernel<<<gridFor(gridN), 256, 0, stream>>>(C->grid, C->gGrid, C->mGrid, C->vGrid, gridN, C->lr, b1, b2,
                                                       1e-10f, c1, c2);
        adamKernel<<<gridFor(mlpN), 256, 0, stream>>>(C->mlp, C->gMlp, C->mMlp, C->vMlp, mlpN, C->lr, b1, b2,
                                                      1e-10f, c1, c2);
    }
    return cudaGetLastError();
}
