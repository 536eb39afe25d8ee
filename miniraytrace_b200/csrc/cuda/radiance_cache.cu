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
// Inference runs on the tensor cores (tcgen05 MMAs with BF16 operands and
// FP32 accumulators in tensor memory, below). Training keeps FP32 on the CUDA
// cores: 64 samples per block, weights read from shared memory as broadcasts
// and activations from padded shared rows.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "device_api.h"

namespace {

constexpr int kLevels = 16;
constexpr uint32_t kTableSize = 1u << 19;
constexpr int kWidth = 64;
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
// for the backward pass when `corners` is given. Levels are visited kGroup at
// a time (their 8 kGroup gathers can be in flight together).
template <int kGroup = 1>
__device__ __forceinline__ void encode(const McacheParams& C, const float* f, float* enc, Corners* corners) {
    float p[3];
    for (int a = 0; a < 3; ++a) {
        const float u = (f[a] - C.lo[a]) * C.invExtent[a];
        p[a] = fminf(fmaxf(u, 0.0f), 1.0f);
    }
    for (int l0 = 0; l0 < kLevels; l0 += kGroup) {
#pragma unroll
        for (int g = 0; g < kGroup; ++g) {
            const int l = l0 + g;
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
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const uint32_t cx = b[0] + (c & 1), cy = b[1] + ((c >> 1) & 1), cz = b[2] + ((c >> 2) & 1);
                const float w = ((c & 1) ? fr[0] : 1.0f - fr[0]) * ((c & 2) ? fr[1] : 1.0f - fr[1]) *
                                ((c & 4) ? fr[2] : 1.0f - fr[2]);
                const uint32_t i = uint32_t(l) * kTableSize + gridIndex(cx, cy, cz, res);
                const float2 gv = reinterpret_cast<const float2*>(C.grid)[i];
                e0 += w * gv.x;
                e1 += w * gv.y;
                if (corners) {
                    corners->idx[l][c] = i;
                    corners->w[l][c] = w;
                }
            }
            enc[2 * l] = e0;
            enc[2 * l + 1] = e1;
        }
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

constexpr int kAct = 68;  // activation row stride in shared memory (float4 aligned, conflict-free)
constexpr int kMlpFloats = (kLayers + 1) * kWidth * kWidth;

// Weight matrix `layer` (rows x 64, row-major) into shared memory (stride 64).
__device__ void loadWeights(const float* __restrict__ mlp, int layer, int rows, float* sW) {
    const float4* W = reinterpret_cast<const float4*>(mlp + size_t(layer) * kWidth * kWidth);
    float4* d = reinterpret_cast<float4*>(sW);
    for (int i = threadIdx.x; i < rows * kWidth / 4; i += blockDim.x) d[i] = W[i];
}

// A 64-float row of shared memory into registers.
__device__ __forceinline__ void loadRow(const float* row, float (&x)[kWidth]) {
#pragma unroll
    for (int m = 0; m < kWidth / 4; ++m) {
        const float4 v = reinterpret_cast<const float4*>(row)[m];
        x[4 * m] = v.x;
        x[4 * m + 1] = v.y;
        x[4 * m + 2] = v.z;
        x[4 * m + 3] = v.w;
    }
}

// out[j] = sum_k W[j][k] x[k] for j < rows (ReLU when `relu`): x in
// registers, each weight row read as 16 broadcast 128-bit loads.
__device__ __forceinline__ void denseForward(const float* sW, const float (&x)[kWidth], float* out, int rows,
                                             bool relu) {
    for (int j = 0; j < rows; ++j) {
        const float4* w = reinterpret_cast<const float4*>(sW + j * kWidth);
        float acc0 = 0.0f, acc1 = 0.0f;
#pragma unroll
        for (int m = 0; m < kWidth / 4; m += 2) {
            const float4 v = w[m], u = w[m + 1];
            acc0 = fmaf(v.x, x[4 * m], acc0);
            acc1 = fmaf(v.y, x[4 * m + 1], acc1);
            acc0 = fmaf(v.z, x[4 * m + 2], acc0);
            acc1 = fmaf(v.w, x[4 * m + 3], acc1);
            acc0 = fmaf(u.x, x[4 * m + 4], acc0);
            acc1 = fmaf(u.y, x[4 * m + 5], acc1);
            acc0 = fmaf(u.z, x[4 * m + 6], acc0);
            acc1 = fmaf(u.w, x[4 * m + 7], acc1);
        }
        const float acc = acc0 + acc1;
        out[j] = relu ? fmaxf(acc, 0.0f) : acc;
    }
}

// ---------------------------------------------------------------- inference --
// Inference on the tensor cores (tcgen05, kind::f16, BF16 operands, FP32
// accumulation in tensor memory). A CTA of 128 threads takes tiles of 128
// queries: thread r encodes query r into row r of the activation tile A
// (128 x 64 BF16 in shared memory); per layer one thread issues four
// 128 x N x 16 MMAs (N = 64, or 16 for the output layer whose rows 3..15
// are zero) reading A and the layer's weights W (N x 64 BF16, shared memory)
// into a 128 x N FP32 accumulator in tensor memory, commits them to an
// mbarrier, and every thread reads its own row back (tensor-memory lane r),
// applies the ReLU and writes it, as BF16, over its row of A for the next
// layer. Weights are converted once per CTA; the CTA then loops over tiles.
//
// Shared-memory operand layout (no swizzle, K-major): the tile is a grid of
// 8-row x 16-byte core matrices stored as 128 contiguous bytes; element
// (row r, k) of an R x 64 operand sits at (r / 8) * 1024 + (k / 8) * 128 +
// (r % 8) * 16 + (k % 8) * 2. In the matrix descriptor the leading byte
// offset (between the two core matrices along K of one 16-wide K step) is
// 128 and the stride byte offset (between 8-row groups) is 1024; K step s
// starts 256 * s bytes in.

constexpr int kTile = 128;                      // queries per tile = MMA M
constexpr uint32_t kWBytes = kWidth * kWidth * 2;   // one hidden layer, BF16
constexpr uint32_t kWOutBytes = kOutRows * kWidth * 2;
constexpr uint32_t kWAllBytes = kLayers * kWBytes + kWOutBytes;
constexpr uint32_t kABytes = kTile * kWidth * 2;
constexpr uint32_t kTmemCols = 64;              // one accumulator: 128 lanes x 64 FP32 columns
// Tiles a query CTA works on at once. One: the kernel is bound by the
// encoding's hash-grid gathers, and on 2M random queries two groups per CTA
// (twice the warps in flight) took 1.67 ms against 0.92 ms for one, as did
// gathering four levels at a time (1.09 ms): more gathers in flight evict
// each other from L1.
constexpr uint32_t kQueryGroups = 1;
constexpr uint32_t kWaitLimit = 1u << 20;       // mbarrier polls before a tile gives up
constexpr bool kRenderClamp = true;             // rendering takes max(prediction, 0)

__device__ __forceinline__ uint32_t coreOffset(uint32_t r, uint32_t k) {
    return (r >> 3) * 1024u + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

__device__ __forceinline__ uint32_t smemAddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address, leading and stride byte
// offsets (all >> 4), descriptor version 1 (bits 46-47), no swizzle.
__device__ __forceinline__ uint64_t smemDesc(uint32_t addr) {
    return uint64_t((addr & 0x3FFFFu) >> 4) | (uint64_t(128u >> 4) << 16) | (uint64_t(1024u >> 4) << 32) |
           (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1),
// A and B BF16 (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17,
// M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t instrDesc(uint32_t m, uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ void fenceAsyncShared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tcFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tcFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tcMma(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(uint32_t(accumulate))
        : "memory");
}

__device__ __forceinline__ void tcCommit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// Polls the mbarrier for the given phase parity at most kWaitLimit times.
__device__ __forceinline__ bool waitParity(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmemLoad16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmemWaitLoad() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t packBf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // a in the low half
    return *reinterpret_cast<const uint32_t*>(&h);
}

// 64 values (ReLU'd when `relu`) as row r of an operand tile.
__device__ __forceinline__ void storeRow(uint8_t* tile, uint32_t r, const float* v, bool relu) {
#pragma unroll
    for (int c = 0; c < kWidth / 8; ++c) {
        float x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = relu ? fmaxf(v[8 * c + i], 0.0f) : v[8 * c + i];
        const uint4 w = make_uint4(packBf16(x[0], x[1]), packBf16(x[2], x[3]), packBf16(x[4], x[5]),
                                   packBf16(x[6], x[7]));
        *reinterpret_cast<uint4*>(tile + coreOffset(r, 8 * c)) = w;
    }
}

// AND of `v` over the 128 threads of named barrier `id` (a barrier too).
__device__ __forceinline__ bool groupAnd(bool v, uint32_t id) {
    uint32_t out;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.and.pred p, %2, 128, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(out)
        : "r"(uint32_t(v)), "r"(id)
        : "memory");
    return out != 0;
}

__device__ __forceinline__ void groupSync(uint32_t id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

// kGroups independent groups of 128 threads share the CTA's weights; group h
// owns activation tile h, mbarrier h, named barrier 1 + h and tensor-memory
// columns [64 h, 64 h + 64), and walks tiles blockIdx.x * kGroups + h,
// stepping by gridDim.x * kGroups. (Warp w of the CTA reaches tensor-memory
// lanes 32 (w % 4) .. 32 (w % 4) + 31, so every group covers all 128 lanes.)
__global__ void __launch_bounds__(kTile* kQueryGroups, 3) tcQueryKernel(McacheParams C, const float* __restrict__ features,
                                                                     uint32_t n, float* __restrict__ out3,
                                                                     bool clampOut) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sW = smem;  // W0..W4 (8 KiB each), W5 (2 KiB)
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kWAllBytes + kQueryGroups * kABytes);
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(bars + kQueryGroups);
    const uint32_t t = threadIdx.x, warp = t >> 5;
    const uint32_t h = t / kTile, r = t % kTile;  // group, row of its tile
    uint8_t* sA = smem + kWAllBytes + h * kABytes;

    // weights, FP32 row-major in global memory, to BF16 operand tiles
    for (uint32_t i = t; i < uint32_t(kLayers * kWidth * kWidth + kOutRows * kWidth) / 2; i += blockDim.x) {
        const uint32_t e = 2 * i, layer = e / (kWidth * kWidth), rem = e % (kWidth * kWidth);
        const uint32_t j = rem / kWidth, k = rem % kWidth;
        const float2 w = reinterpret_cast<const float2*>(C.mlp)[i];
        *reinterpret_cast<uint32_t*>(sW + layer * kWBytes + coreOffset(j, k)) = packBf16(w.x, w.y);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(tmemSlot)),
                     "r"(kTmemCols * kQueryGroups)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (r == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(bars + h)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fenceAsyncShared();
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tmem = *tmemSlot + kTmemCols * h;                 // this group's columns
    const uint32_t barAddr = smemAddr(bars + h), aAddr = smemAddr(sA), wAddr = smemAddr(sW);
    const uint32_t laneBase = tmem + (((warp % 4u) * 32u) << 16);     // this warp's 32 lanes
    const uint32_t barId = 1u + h;
    uint32_t parity = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x * kQueryGroups + h; ok && size_t(tile) * kTile < n;
         tile += gridDim.x * kQueryGroups) {
        const uint32_t q = tile * kTile + r;
        const bool valid = q < n;
        float f[16];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float4 v = valid ? reinterpret_cast<const float4*>(features)[size_t(q) * 4 + k]
                                   : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            f[4 * k] = v.x;
            f[4 * k + 1] = v.y;
            f[4 * k + 2] = v.z;
            f[4 * k + 3] = v.w;
        }
        float v[kWidth];
        encode<1>(C, f, v, nullptr);
        storeRow(sA, r, v, false);
        fenceAsyncShared();
        tcFenceBefore();
        groupSync(barId);
        for (int l = 0; l <= kLayers; ++l) {
            const uint32_t rows = l < kLayers ? kWidth : kOutRows;
            if (r == 0) {
                tcFenceAfter();
                const uint32_t idesc = instrDesc(kTile, rows);
#pragma unroll
                for (uint32_t s = 0; s < kWidth / 16; ++s)
                    tcMma(tmem, smemDesc(aAddr + 256u * s), smemDesc(wAddr + uint32_t(l) * kWBytes + 256u * s), idesc,
                          s > 0);
                tcCommit(barAddr);
            }
            const bool done = waitParity(barAddr, parity);
            parity ^= 1u;
            if (!groupAnd(done, barId)) {
                ok = false;
                break;
            }
            tcFenceAfter();
            if (l < kLayers) {
#pragma unroll
                for (int c = 0; c < kWidth / 16; ++c) tmemLoad16(laneBase + 16u * c, v + 16 * c);
                tmemWaitLoad();
                storeRow(sA, r, v, true);
                fenceAsyncShared();
                tcFenceBefore();
                groupSync(barId);
            } else {
                tmemLoad16(laneBase, v);
                tmemWaitLoad();
                tcFenceBefore();
                if (valid)
                    for (int c = 0; c < 3; ++c) out3[size_t(q) * 3 + c] = clampOut ? fmaxf(v[c], 0.0f) : v[c];
            }
        }
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmemSlot),
                     "r"(kTmemCols * kQueryGroups)
                     : "memory");
    if (!ok && r == 0) atomicOr(C.status, 1u);
}

// One training step's forward + backward for 64 samples per block: loss =
// mean over samples and channels of (y - t)^2 / (y^2 + 0.01), y held fixed in
// the denominator. Each block writes its weight gradients (summed over its
// samples, 8 x 8 register tiles per thread) to partial[block]; the grid
// gradients are scattered to the 8 corners of each level.
__global__ void __launch_bounds__(kBlock) trainKernel(McacheParams C, const float* __restrict__ features,
                                                      const float* __restrict__ targets, uint32_t n, uint32_t first,
                                                      uint32_t every, float invBatch, float* __restrict__ partial,
                                                      float* __restrict__ lossOut) {
    extern __shared__ float4 smem4[];
    float* sW = reinterpret_cast<float*>(smem4);       // kWidth x kWidth
    float* act = sW + kWidth * kWidth;                 // (kLayers + 1) x kBlock x kAct: enc, h1..h5
    float* dA = act + (kLayers + 1) * kBlock * kAct;   // kBlock x kAct: gradient of the layer's output
    float* dB = dA + kBlock * kAct;
    const int t = threadIdx.x;
    const uint32_t j = blockIdx.x * kBlock + t;  // the step's j-th sample is record first + j * every
    const bool valid = j < n;
    const size_t s = size_t(first) + size_t(j) * every;
    float f[16];
    for (int k = 0; k < 16; ++k) f[k] = valid ? features[s * 16 + k] : 0.0f;
    Corners corners;
    encode(C, f, act + t * kAct, &corners);
    float x[kWidth];
    for (int l = 0; l <= kLayers; ++l) {
        __syncthreads();
        loadWeights(C.mlp, l, l < kLayers ? kWidth : kOutRows, sW);
        __syncthreads();
        loadRow(act + (l * kBlock + t) * kAct, x);
        float* out = l < kLayers ? act + ((l + 1) * kBlock + t) * kAct : dA + t * kAct;
        denseForward(sW, x, out, l < kLayers ? kWidth : 3, l < kLayers);
    }
    // output gradient (3 channels; zero for padding samples and channels)
    float loss = 0.0f;
    for (int c = 0; c < kWidth; ++c) {
        float g = 0.0f;
        if (c < 3 && valid) {
            const float y = dA[t * kAct + c], tg = targets[s * 3 + c];
            const float den = y * y + 0.01f;
            loss += (y - tg) * (y - tg) / den;
            g = 2.0f * (y - tg) / den * invBatch;
        }
        dA[t * kAct + c] = g;
    }
    if (lossOut && valid) atomicAdd(lossOut, loss * invBatch);
    float* myPartial = partial + size_t(blockIdx.x) * kMlpFloats;
    const int jt = t / 8, kt = t % 8;  // this thread's 8 x 8 tile of a weight gradient
    for (int l = kLayers; l >= 0; --l) {
        const int rows = l < kLayers ? kWidth : 3;
        __syncthreads();
        loadWeights(C.mlp, l, l < kLayers ? kWidth : kOutRows, sW);
        __syncthreads();
        const float* in = act + l * kBlock * kAct;
        // weight gradient tile: g[j][k] = sum_r dA[r][j] in[r][k]
        float g[8][8];
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) g[a][b] = 0.0f;
        if (8 * jt < rows) {
            for (int r = 0; r < kBlock; ++r) {
                const float4 d0 = reinterpret_cast<const float4*>(dA + r * kAct + 8 * jt)[0];
                const float4 d1 = reinterpret_cast<const float4*>(dA + r * kAct + 8 * jt)[1];
                const float4 i0 = reinterpret_cast<const float4*>(in + r * kAct + 8 * kt)[0];
                const float4 i1 = reinterpret_cast<const float4*>(in + r * kAct + 8 * kt)[1];
                const float dv[8] = {d0.x, d0.y, d0.z, d0.w, d1.x, d1.y, d1.z, d1.w};
                const float iv[8] = {i0.x, i0.y, i0.z, i0.w, i1.x, i1.y, i1.z, i1.w};
#pragma unroll
                for (int a = 0; a < 8; ++a)
#pragma unroll
                    for (int b = 0; b < 8; ++b) g[a][b] = fmaf(dv[a], iv[b], g[a][b]);
            }
        }
        float* gOut = myPartial + size_t(l) * kWidth * kWidth;
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            float4* o = reinterpret_cast<float4*>(gOut + (8 * jt + a) * kWidth + 8 * kt);
            o[0] = make_float4(g[a][0], g[a][1], g[a][2], g[a][3]);
            o[1] = make_float4(g[a][4], g[a][5], g[a][6], g[a][7]);
        }
        // input gradient of this thread's sample: dB[t][k] = sum_j W[j][k] dA[t][j],
        // through the ReLU of the layer input (hidden layers only)
        float acc[kWidth];
#pragma unroll
        for (int k = 0; k < kWidth; ++k) acc[k] = 0.0f;
        for (int j = 0; j < rows; ++j) {
            const float dj = dA[t * kAct + j];
            const float4* w = reinterpret_cast<const float4*>(sW + j * kWidth);
#pragma unroll
            for (int m = 0; m < kWidth / 4; ++m) {
                const float4 v = w[m];
                acc[4 * m] = fmaf(v.x, dj, acc[4 * m]);
                acc[4 * m + 1] = fmaf(v.y, dj, acc[4 * m + 1]);
                acc[4 * m + 2] = fmaf(v.z, dj, acc[4 * m + 2]);
                acc[4 * m + 3] = fmaf(v.w, dj, acc[4 * m + 3]);
            }
        }
        float xin[kWidth];
        loadRow(in + t * kAct, xin);
#pragma unroll
        for (int k = 0; k < kWidth; ++k)
            dB[t * kAct + k] = (l > 0 && xin[k] <= 0.0f) ? 0.0f : acc[k];
        __syncthreads();
        float* sw = dA;
        dA = dB;
        dB = sw;
    }
    // dA holds the encoding gradient: scatter the grid part
    if (valid) {
        for (int l = 0; l < kLevels; ++l) {
            const float g0 = dA[t * kAct + 2 * l], g1 = dA[t * kAct + 2 * l + 1];
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

// gMlp[i] = sum over blocks of partial[b][i] (rows the output layer leaves
// unwritten are zero in every partial).
__global__ void reducePartialsKernel(const float* __restrict__ partial, uint32_t blocks, float* __restrict__ gMlp) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpFloats; i += gridDim.x * blockDim.x) {
        float acc = 0.0f;
        for (uint32_t b = 0; b < blocks; ++b) acc += partial[size_t(b) * kMlpFloats + i];
        gMlp[i] = acc;
    }
}

// Adam; gradients are cleared for the next step. With `lazy`, entries that
// got no gradient this step are left as they are (their moments and values
// do not decay), which the hash grid needs: a step touches a few of its
// 16.8 M entries.
__global__ void adamKernel(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                           size_t n, float lr, float b1, float b2, float eps, float c1, float c2, bool lazy) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        if (lazy && gi == 0.0f) continue;
        g[i] = 0.0f;
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

// Deterministic initial values: grid uniform in [-1e-4, 1e-4], weights
// uniform in +-sqrt(6 / (fan_in + fan_out)), unused output rows zero.
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
    const size_t total = gridN + size_t(kMlpFloats);
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

// L[slot] += beta * prediction for every query of the wave.
__global__ void applyQueriesKernel(const float* __restrict__ out3, const float4* __restrict__ qBeta, uint32_t n,
                                   uint32_t slots, float4* __restrict__ L) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 b = qBeta[i];
        const uint32_t slot = __float_as_uint(b.w);
        if (slot >= slots) continue;
        float4 l = L[slot];
        l.x += b.x * out3[3 * size_t(i)];
        l.y += b.y * out3[3 * size_t(i) + 1];
        l.z += b.z * out3[3 * size_t(i) + 2];
        L[slot] = l;
    }
}

// Training target of a recorded vertex: the radiance its path gathered from
// the vertex on, divided by the throughput that reached the vertex.
__global__ void recordTargetsKernel(const float4* __restrict__ prefix, const float4* __restrict__ beta, uint32_t n,
                                    uint32_t slots, const float4* __restrict__ L, float* __restrict__ targets) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 pre = prefix[i], b = beta[i];
        const uint32_t slot = __float_as_uint(pre.w);
        const float4 l = slot < slots ? L[slot] : pre;
        const float d[3] = {l.x - pre.x, l.y - pre.y, l.z - pre.z};
        const float bb[3] = {b.x, b.y, b.z};
        for (int c = 0; c < 3; ++c) {
            const float t = bb[c] > 1e-6f ? d[c] / bb[c] : 0.0f;
            targets[3 * size_t(i) + c] = fminf(fmaxf(t, 0.0f), 1e3f);
        }
    }
}

size_t smemQuery() { return kWAllBytes + kQueryGroups * kABytes + 8 * kQueryGroups + 16; }
size_t smemTrain() { return sizeof(float) * (kWidth * kWidth + (kLayers + 1 + 2) * kBlock * kAct); }

unsigned gridFor(size_t n) {
    const size_t b = (n + 255) / 256;
    return unsigned(b < 148u * 32u ? (b > 0 ? b : 1) : 148u * 32u);
}

}  // namespace

extern "C" size_t mrtcu_rc_grid_floats() { return size_t(kLevels) * kTableSize * 2; }
extern "C" size_t mrtcu_rc_mlp_floats() { return size_t(kMlpFloats); }
extern "C" size_t mrtcu_rc_partial_floats(uint32_t maxBatch) {
    return size_t((maxBatch + kBlock - 1) / kBlock) * kMlpFloats;
}

extern "C" cudaError_t mrtcu_rc_init(McacheParams C, uint32_t seed, cudaStream_t stream) {
    const size_t gridN = mrtcu_rc_grid_floats(), mlpN = mrtcu_rc_mlp_floats();
    initKernel<<<gridFor(gridN + mlpN), 256, 0, stream>>>(C.grid, gridN, C.mlp, seed);
    cudaError_t e = cudaMemsetAsync(C.status, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    for (float* p : {C.gGrid, C.mGrid, C.vGrid})
        if ((e = cudaMemsetAsync(p, 0, gridN * sizeof(float), stream)) != cudaSuccess) return e;
    for (float* p : {C.gMlp, C.mMlp, C.vMlp})
        if ((e = cudaMemsetAsync(p, 0, mlpN * sizeof(float), stream)) != cudaSuccess) return e;
    return cudaGetLastError();
}

static cudaError_t launchQuery(const McacheParams& C, const float* features, uint32_t n, float* out3, bool clampOut,
                               cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(tcQueryKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smemQuery()));
    if (e != cudaSuccess) return e;
    // Persistent CTAs: at most 3 fit an SM by shared memory (58 KiB each with
    // one group, 74 KiB with two), so their tensor memory (64 columns a
    // group) never exceeds the SM's 512.
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t groups = (n + kTile - 1) / kTile;
    const uint32_t want = (groups + kQueryGroups - 1) / kQueryGroups;
    const uint32_t ctas = want < uint32_t(sms) * 3u ? want : uint32_t(sms) * 3u;
    tcQueryKernel<<<ctas, kTile * kQueryGroups, smemQuery(), stream>>>(C, features, n, out3, clampOut);
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_rc_query(McacheParams C, const float* features, uint32_t n, float* out3,
                                      cudaStream_t stream) {
    return launchQuery(C, features, n, out3, true, stream);
}

// `steps` Adam steps on batches of up to `batch` of the n samples.
extern "C" cudaError_t mrtcu_rc_train(McacheParams* C, const float* features, const float* targets, uint32_t n,
                                      uint32_t steps, uint32_t batch, float* lossOut, cudaStream_t stream) {
    if (n == 0 || steps == 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(trainKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smemTrain()));
    if (e != cudaSuccess) return e;
    batch = batch < n ? batch : n;
    batch = batch < C->partialBlocks * kBlock ? batch : C->partialBlocks * kBlock;
    const size_t gridN = mrtcu_rc_grid_floats(), mlpN = mrtcu_rc_mlp_floats();
    // Step k trains on every `every`-th sample from sample k mod every: each
    // batch spreads over all of the samples (they arrive ordered by bounce
    // and by pixel), and consecutive steps take disjoint batches.
    const uint32_t every = (n + batch - 1) / batch;
    for (uint32_t k = 0; k < steps; ++k) {
        const uint32_t first = k % every;
        const uint32_t count = (n - first + every - 1) / every;  // <= batch
        const uint32_t blocks = (count + kBlock - 1) / kBlock;
        trainKernel<<<blocks, kBlock, smemTrain(), stream>>>(*C, features, targets, count, first, every,
                                                              1.0f / (3.0f * float(count)), C->partial, lossOut);
        reducePartialsKernel<<<gridFor(kMlpFloats), 256, 0, stream>>>(C->partial, blocks, C->gMlp);
        ++C->step;
        const float b1 = 0.9f, b2 = 0.99f;
        const float c1 = 1.0f / (1.0f - powf(b1, float(C->step))), c2 = 1.0f / (1.0f - powf(b2, float(C->step)));
        adamKernel<<<gridFor(gridN), 256, 0, stream>>>(C->grid, C->gGrid, C->mGrid, C->vGrid, gridN, C->lr, b1, b2,
                                                       1e-10f, c1, c2, true);
        adamKernel<<<gridFor(mlpN), 256, 0, stream>>>(C->mlp, C->gMlp, C->mMlp, C->vMlp, mlpN, C->lr, b1, b2,
                                                      1e-10f, c1, c2, false);
    }
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_rc_apply_queries(McacheParams C, const float* qFeat, const float4* qBeta, uint32_t n,
                                              uint32_t slots, float* scratch3, float4* L, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const cudaError_t e = launchQuery(C, qFeat, n, scratch3, kRenderClamp, stream);
    if (e != cudaSuccess) return e;
    applyQueriesKernel<<<gridFor(n), 256, 0, stream>>>(scratch3, qBeta, n, slots, L);
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_rc_record_targets(const float4* prefix, const float4* beta, uint32_t n, uint32_t slots,
                                               const float4* L, float* targets, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    recordTargetsKernel<<<gridFor(n), 256, 0, stream>>>(prefix, beta, n, slots, L, targets);
    return cudaGetLastError();
}
