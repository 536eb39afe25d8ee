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
// Inference and training run on the tensor cores (tcgen05 MMAs with BF16
// operands and FP32 accumulators in tensor memory, below); the hash-grid
// encoding, the ReLU masks, the loss gradient and Adam run on the CUDA cores
// in FP32, and the parameters are kept in FP32.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "device_api.h"

namespace {

constexpr int kLevels = 16;
constexpr uint32_t kTableSize = 1u << 19;
constexpr int kWidth = 64;
constexpr int kLayers = 5;        // hidden layers
constexpr int kOutRows = 16;
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

constexpr int kMlpFloats = (kLayers + 1) * kWidth * kWidth;

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

// Shared-memory matrix descriptor: start address, leading byte offset (the
// stride between core matrices along K), stride byte offset (between core
// matrices along M or N), all >> 4; descriptor version 1 (bits 46-47); no
// swizzle.
__device__ __forceinline__ uint64_t smemDesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr & 0x3FFFFu) >> 4) | (uint64_t(lbo >> 4) << 16) | (uint64_t(sbo >> 4) << 32) |
           (uint64_t(1) << 46);
}

// An operand tile of the layout above read K-major: K runs along a row (the
// activations of a record, the inputs of a weight row).
__device__ __forceinline__ uint64_t descK(uint32_t addr) { return smemDesc(addr, 128u, 1024u); }

// The same tile read MN-major, i.e. transposed: its rows become the K
// dimension. Element (row r, column c) sits at (r / 8) * 1024 + (r % 8) * 16
// + (c / 8) * 128 + (c % 8) * 2, which is the MN-major canonical layout with
// M/N index c (8-element core-matrix rows, blocks 128 bytes apart) and K
// index r (blocks of 8 rows 1024 bytes apart).
__device__ __forceinline__ uint64_t descMN(uint32_t addr) { return smemDesc(addr, 1024u, 128u); }

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1),
// A and B BF16 (bits 7-9, 10-12 = 1), A and B major-ness (bits 15, 16: 0 K,
// 1 MN), N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t instrDesc(uint32_t m, uint32_t n, bool aMN = false, bool bMN = false) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(aMN) << 15) | (uint32_t(bMN) << 16) | ((n >> 3) << 17) |
           ((m >> 4) << 24);
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

// The weights, FP32 row-major in global memory, as BF16 operand tiles:
// W0..W4 (64 x 64, 8 KiB each), then W5 (16 x 64, 2 KiB).
__device__ void loadWeightTiles(const float* __restrict__ mlp, uint8_t* sW) {
    for (uint32_t i = threadIdx.x; i < uint32_t(kLayers * kWidth * kWidth + kOutRows * kWidth) / 2; i += blockDim.x) {
        const uint32_t e = 2 * i, layer = e / (kWidth * kWidth), rem = e % (kWidth * kWidth);
        const uint32_t j = rem / kWidth, k = rem % kWidth;
        const float2 w = reinterpret_cast<const float2*>(mlp)[i];
        *reinterpret_cast<uint32_t*>(sW + layer * kWBytes + coreOffset(j, k)) = packBf16(w.x, w.y);
    }
}

// Row r of an operand tile as 64 floats.
__device__ __forceinline__ void loadRowBf16(const uint8_t* tile, uint32_t r, float* v) {
#pragma unroll
    for (int c = 0; c < kWidth / 8; ++c) {
        const uint4 w = *reinterpret_cast<const uint4*>(tile + coreOffset(r, 8 * c));
        const uint32_t u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            v[8 * c + 2 * i] = __uint_as_float(u[i] << 16);
            v[8 * c + 2 * i + 1] = __uint_as_float(u[i] & 0xFFFF0000u);
        }
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
// With `order`, row i of the walk is query order[i] (its features read and
// its prediction written there): queries sorted by position share the hash
// grid's cells, so a warp's corner gathers hit the same lines.
__global__ void __launch_bounds__(kTile* kQueryGroups, 3) tcQueryKernel(McacheParams C, const float* __restrict__ features,
                                                                     uint32_t n, float* __restrict__ out3,
                                                                     bool clampOut,
                                                                     const uint32_t* __restrict__ order) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sW = smem;  // W0..W4 (8 KiB each), W5 (2 KiB)
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kWAllBytes + kQueryGroups * kABytes);
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(bars + kQueryGroups);
    const uint32_t t = threadIdx.x, warp = t >> 5;
    const uint32_t h = t / kTile, r = t % kTile;  // group, row of its tile
    uint8_t* sA = smem + kWAllBytes + h * kABytes;

    loadWeightTiles(C.mlp, sW);
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
        const uint32_t row = tile * kTile + r;
        const bool valid = row < n;
        const uint32_t q = valid && order ? order[row] : row;
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
                    tcMma(tmem, descK(aAddr + 256u * s), descK(wAddr + uint32_t(l) * kWBytes + 256u * s), idesc, s > 0);
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
    // A wait that gave up is fatal for the cache, not a retryable error: the
    // MMA it waited for may still be writing the tensor-memory columns freed
    // above, and a later CTA on this SM may be given them. The engine
    // therefore discards every output of the launch (and the accumulation
    // holding them) and never launches the cache kernels again.
    if (!ok && r == 0) atomicOr(C.status, 1u);
}

// ----------------------------------------------------------------- training --
// One training step on the tensor cores. A CTA of 128 threads takes tiles of
// 128 records (the step's j-th record is record first + j * every): thread r
// encodes record r into row r of A0 and the forward pass keeps every layer's
// input A0..A5 (BF16 tiles); the loss gradient of the mean relative L2 loss
// (y - t)^2 / (y^2 + 0.01) over records and channels (y held fixed in the
// denominator) becomes dZ5, and per layer l = 5..0 one thread issues
//   dW_l (64 x 64, rows beyond the layer's outputs zero) = dZ_l^T A_l:
//       M = 128 (rows 64..127 are unused), N = 64, K = 128 records, A = the
//       dZ tile read MN-major, B = the A_l tile read MN-major;
//   dA_l (128 x 64) = dZ_l W_l: M = 128, N = 64, K = the layer's outputs,
//       A = the dZ tile K-major, B = the W_l tile read MN-major;
// then every thread reads its dA row, masks it with the ReLU of A_l into
// dZ_{l-1} (BF16) or, for l = 0, scatters the encoding gradient into the
// hash-grid gradient at the 8 corners of each level. Threads 0..63 read dW_l
// rows from tensor memory into this CTA's partial weight gradient (FP32).
// Operands are BF16 with FP32 accumulation, as in inference.
constexpr uint32_t kDzSlack = 2048;  // read by the dW MMA's unused rows 64..127, kept zero

size_t smemTrain() { return kWAllBytes + (kLayers + 1) * kABytes + kABytes + kDzSlack + 16; }

__global__ void __launch_bounds__(kTile, 1) tcTrainKernel(McacheParams C, const float* __restrict__ features,
                                                          const float* __restrict__ targets, uint32_t n,
                                                          uint32_t first, uint32_t every, float invBatch,
                                                          float* __restrict__ partial, float* __restrict__ lossOut) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sW = smem;                                  // W0..W5
    uint8_t* sAct = smem + kWAllBytes;                   // A0 (encoding) .. A5, kABytes each
    uint8_t* sDz = sAct + (kLayers + 1) * kABytes;       // dZ tile, then kDzSlack zero bytes
    uint64_t* bar = reinterpret_cast<uint64_t*>(sDz + kABytes + kDzSlack);
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(bar + 1);
    const uint32_t t = threadIdx.x, warp = t >> 5;

    loadWeightTiles(C.mlp, sW);
    for (uint32_t i = t; i < kDzSlack / 16; i += kTile)
        reinterpret_cast<uint4*>(sDz + kABytes)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(tmemSlot)),
                     "r"(2u * kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fenceAsyncShared();
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tmem = *tmemSlot;
    const uint32_t accA = tmem, accW = tmem + kTmemCols;   // forward / input gradient, weight gradient
    const uint32_t lane = (warp * 32u) << 16;             // this warp's 32 tensor-memory lanes
    const uint32_t barAddr = smemAddr(bar), wAddr = smemAddr(sW), actAddr = smemAddr(sAct), dzAddr = smemAddr(sDz);
    float* myPartial = partial + size_t(blockIdx.x) * kMlpFloats;
    uint32_t parity = 0;
    bool ok = true, firstTile = true;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    for (uint32_t tile = blockIdx.x; ok && tile < tiles; tile += gridDim.x) {
        const uint32_t j = tile * kTile + t;
        const bool valid = j < n;
        const size_t rec = size_t(first) + size_t(j) * every;
        float f[16];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float4 v = valid ? reinterpret_cast<const float4*>(features)[rec * 4 + k]
                                   : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            f[4 * k] = v.x;
            f[4 * k + 1] = v.y;
            f[4 * k + 2] = v.z;
            f[4 * k + 3] = v.w;
        }
        Corners corners;
        float v[kWidth];
        encode(C, f, v, &corners);
        storeRow(sAct, t, v, false);
        fenceAsyncShared();
        tcFenceBefore();
        __syncthreads();
        // forward
        for (int l = 0; ok && l <= kLayers; ++l) {
            if (t == 0) {
                tcFenceAfter();
                const uint32_t idesc = instrDesc(kTile, l < kLayers ? kWidth : kOutRows);
#pragma unroll
                for (uint32_t s = 0; s < kWidth / 16; ++s)
                    tcMma(accA, descK(actAddr + uint32_t(l) * kABytes + 256u * s),
                          descK(wAddr + uint32_t(l) * kWBytes + 256u * s), idesc, s > 0);
                tcCommit(barAddr);
            }
            const bool done = waitParity(barAddr, parity);
            parity ^= 1u;
            ok = __syncthreads_and(done) != 0;
            if (!ok) break;
            tcFenceAfter();
            if (l < kLayers) {
#pragma unroll
                for (int c = 0; c < kWidth / 16; ++c) tmemLoad16(accA + lane + 16u * c, v + 16 * c);
                tmemWaitLoad();
                storeRow(sAct + uint32_t(l + 1) * kABytes, t, v, true);
                fenceAsyncShared();
            } else {
                tmemLoad16(accA + lane, v);
                tmemWaitLoad();
            }
            tcFenceBefore();
            __syncthreads();
        }
        if (!ok) break;
        // output gradient: dZ5 (channels 0..2; the rest and padding records zero)
        float g[kWidth];
        float loss = 0.0f;
#pragma unroll
        for (int c = 0; c < kWidth; ++c) g[c] = 0.0f;
        if (valid)
            for (int c = 0; c < 3; ++c) {
                const float y = v[c], tg = targets[rec * 3 + c];
                const float den = y * y + 0.01f;
                loss += (y - tg) * (y - tg) / den;
                g[c] = 2.0f * (y - tg) / den * invBatch;
            }
        if (lossOut && valid) atomicAdd(lossOut, loss * invBatch);
        storeRow(sDz, t, g, false);
        fenceAsyncShared();
        tcFenceBefore();
        __syncthreads();
        // backward
        for (int l = kLayers; ok && l >= 0; --l) {
            const uint32_t outs = l < kLayers ? kWidth : kOutRows;  // K of the input-gradient MMA
            if (t == 0) {
                tcFenceAfter();
                const uint32_t idescW = instrDesc(kTile, kWidth, true, true);
#pragma unroll
                for (uint32_t s = 0; s < kTile / 16; ++s)
                    tcMma(accW, descMN(dzAddr + 2048u * s), descMN(actAddr + uint32_t(l) * kABytes + 2048u * s),
                          idescW, s > 0);
                const uint32_t idescA = instrDesc(kTile, kWidth, false, true);
                for (uint32_t s = 0; s < outs / 16; ++s)
                    tcMma(accA, descK(dzAddr + 256u * s), descMN(wAddr + uint32_t(l) * kWBytes + 2048u * s), idescA,
                          s > 0);
                tcCommit(barAddr);
            }
            const bool done = waitParity(barAddr, parity);
            parity ^= 1u;
            ok = __syncthreads_and(done) != 0;
            if (!ok) break;
            tcFenceAfter();
            if (warp < 2) {  // dW rows 0..63: lanes 0..63
                float w[kWidth];
#pragma unroll
                for (int c = 0; c < kWidth / 16; ++c) tmemLoad16(accW + lane + 16u * c, w + 16 * c);
                tmemWaitLoad();
                float4* o = reinterpret_cast<float4*>(myPartial + size_t(l) * kWidth * kWidth + size_t(t) * kWidth);
#pragma unroll
                for (int c = 0; c < kWidth / 4; ++c) {
                    float4 a = make_float4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
                    if (!firstTile) {
                        const float4 b = o[c];
                        a.x += b.x;
                        a.y += b.y;
                        a.z += b.z;
                        a.w += b.w;
                    }
                    o[c] = a;
                }
            }
#pragma unroll
            for (int c = 0; c < kWidth / 16; ++c) tmemLoad16(accA + lane + 16u * c, g + 16 * c);
            tmemWaitLoad();
            if (l > 0) {
                loadRowBf16(sAct + uint32_t(l) * kABytes, t, v);  // A_l = ReLU(Z_{l-1})
#pragma unroll
                for (int c = 0; c < kWidth; ++c) g[c] = v[c] > 0.0f ? g[c] : 0.0f;
                storeRow(sDz, t, g, false);
                fenceAsyncShared();
            } else if (valid) {
                for (int lv = 0; lv < kLevels; ++lv) {
                    const float g0 = g[2 * lv], g1 = g[2 * lv + 1];
                    if (g0 == 0.0f && g1 == 0.0f) continue;
                    for (int c = 0; c < 8; ++c) {
                        const uint32_t i = corners.idx[lv][c];
                        const float w = corners.w[lv][c];
                        atomicAdd(C.gGrid + 2 * size_t(i), w * g0);
                        atomicAdd(C.gGrid + 2 * size_t(i) + 1, w * g1);
                    }
                }
            }
            tcFenceBefore();
            __syncthreads();
        }
        firstTile = false;
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2u * kTmemCols)
                     : "memory");
    // Fatal for the cache, as in the query kernel: the engine discards the
    // launch's results and runs no cache kernel again.
    if (!ok && t == 0) atomicOr(C.status, 1u);
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
// One Adam step (lazy: entries with a zero gradient, untouched by the
// batch, keep their parameter and moments); with `ema`, the moving average
// of each changed parameter takes the new value with weight 1 - emaDecay.
__global__ void adamKernel(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                           size_t n, float lr, float b1, float b2, float eps, float c1, float c2, bool lazy,
                           float* __restrict__ ema, float emaDecay) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        if (lazy && gi == 0.0f) continue;
        g[i] = 0.0f;
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        p[i] = pi;
        if (ema) ema[i] = emaDecay * ema[i] + (1.0f - emaDecay) * pi;
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

// 30-bit Morton code of each query's position in the cache's bounds (10
// bits an axis) and its index: the keys that order a wave's queries.
__device__ uint32_t spread3(uint32_t v) {  // 10 bits to every third of 30
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__global__ void queryKeysKernel(McacheParams C, const float* __restrict__ features, uint32_t n,
                                uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 f = reinterpret_cast<const float4*>(features)[size_t(i) * 4];
        const float pos[3] = {f.x, f.y, f.z};
        uint32_t q[3];
        for (int a = 0; a < 3; ++a) {
            const float u = fminf(fmaxf((pos[a] - C.lo[a]) * C.invExtent[a], 0.0f), 1.0f);
            q[a] = uint32_t(u * 1023.0f);
        }
        keys[i] = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
        vals[i] = i;
    }
}

size_t smemQuery() { return kWAllBytes + kQueryGroups * kABytes + 8 * kQueryGroups + 16; }

unsigned gridFor(size_t n) {
    const size_t b = (n + 255) / 256;
    return unsigned(b < 148u * 32u ? (b > 0 ? b : 1) : 148u * 32u);
}

}  // namespace

extern "C" size_t mrtcu_rc_grid_floats() { return size_t(kLevels) * kTableSize * 2; }
extern "C" size_t mrtcu_rc_mlp_floats() { return size_t(kMlpFloats); }
// Training CTAs (one per SM at most, each writing its own partial weight
// gradient) for batches of up to maxBatch records.
extern "C" uint32_t mrtcu_rc_partial_blocks(uint32_t maxBatch) {
    const uint32_t tiles = (maxBatch + kTile - 1) / kTile;
    return tiles < 512u ? tiles : 512u;
}
extern "C" size_t mrtcu_rc_partial_floats(uint32_t maxBatch) {
    return size_t(mrtcu_rc_partial_blocks(maxBatch)) * kMlpFloats;
}

extern "C" cudaError_t mrtcu_rc_init(McacheParams C, uint32_t seed, cudaStream_t stream) {
    const size_t gridN = mrtcu_rc_grid_floats(), mlpN = mrtcu_rc_mlp_floats();
    initKernel<<<gridFor(gridN + mlpN), 256, 0, stream>>>(C.grid, gridN, C.mlp, seed);
    cudaError_t e = cudaMemsetAsync(C.status, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    if (C.emaGrid && (e = cudaMemcpyAsync(C.emaGrid, C.grid, gridN * sizeof(float), cudaMemcpyDeviceToDevice,
                                          stream)) != cudaSuccess)
        return e;
    if (C.emaMlp && (e = cudaMemcpyAsync(C.emaMlp, C.mlp, mlpN * sizeof(float), cudaMemcpyDeviceToDevice,
                                         stream)) != cudaSuccess)
        return e;
    for (float* p : {C.gGrid, C.mGrid, C.vGrid})
        if ((e = cudaMemsetAsync(p, 0, gridN * sizeof(float), stream)) != cudaSuccess) return e;
    for (float* p : {C.gMlp, C.mMlp, C.vMlp})
        if ((e = cudaMemsetAsync(p, 0, mlpN * sizeof(float), stream)) != cudaSuccess) return e;
    return cudaGetLastError();
}

static cudaError_t launchQuery(const McacheParams& C, const float* features, uint32_t n, float* out3, bool clampOut,
                               cudaStream_t stream, const uint32_t* order = nullptr) {
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
    tcQueryKernel<<<ctas, kTile * kQueryGroups, smemQuery(), stream>>>(C, features, n, out3, clampOut, order);
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
    cudaError_t e = cudaFuncSetAttribute(tcTrainKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smemTrain()));
    if (e != cudaSuccess) return e;
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // one CTA per SM at most (shared memory), each with its own partial
    const uint32_t maxCtas = uint32_t(sms) < C->partialBlocks ? uint32_t(sms) : C->partialBlocks;
    batch = batch < n ? batch : n;
    const size_t gridN = mrtcu_rc_grid_floats(), mlpN = mrtcu_rc_mlp_floats();
    // Step k trains on every `every`-th sample from sample k mod every: each
    // batch spreads over all of the samples (they arrive ordered by bounce
    // and by pixel), and consecutive steps take disjoint batches.
    const uint32_t every = (n + batch - 1) / batch;
    for (uint32_t k = 0; k < steps; ++k) {
        const uint32_t first = k % every;
        const uint32_t count = (n - first + every - 1) / every;  // <= batch
        const uint32_t tiles = (count + kTile - 1) / kTile;
        const uint32_t blocks = tiles < maxCtas ? tiles : maxCtas;
        tcTrainKernel<<<blocks, kTile, smemTrain(), stream>>>(*C, features, targets, count, first, every,
                                                              1.0f / (3.0f * float(count)), C->partial, lossOut);
        reducePartialsKernel<<<gridFor(kMlpFloats), 256, 0, stream>>>(C->partial, blocks, C->gMlp);
        ++C->step;
        const float b1 = 0.9f, b2 = 0.99f;
        const float c1 = 1.0f / (1.0f - powf(b1, float(C->step))), c2 = 1.0f / (1.0f - powf(b2, float(C->step)));
        const float st = float(C->step);
        const float d = fminf(C->emaDecay, (1.0f + st) / (10.0f + st));
        float lr = C->lr;
        if (C->lrHalfLife > 0.0f)
            lr = fmaxf(fminf(C->lrMin, C->lr),
                       C->lr * exp2f(-float(C->step - C->lrStart - 1u) / C->lrHalfLife));
        adamKernel<<<gridFor(gridN), 256, 0, stream>>>(C->grid, C->gGrid, C->mGrid, C->vGrid, gridN, lr, b1, b2,
                                                       1e-10f, c1, c2, true, C->emaGrid, d);
        adamKernel<<<gridFor(mlpN), 256, 0, stream>>>(C->mlp, C->gMlp, C->mMlp, C->vMlp, mlpN, lr, b1, b2,
                                                      1e-10f, c1, c2, false, C->emaMlp, d);
    }
    return cudaGetLastError();
}

// The gradients of one batch without an optimizer step: the training
// kernel's forward and backward pass over all n samples (the mean loss over
// samples and channels), the per-CTA weight gradients summed into C->gMlp,
// the hash-grid gradient scattered into C->gGrid (cleared first). The
// parameters and the Adam moments are not touched; the caller clears gGrid
// afterwards so no later Adam step consumes it.
extern "C" cudaError_t mrtcu_rc_gradients(McacheParams* C, const float* features, const float* targets, uint32_t n,
                                          float* lossOut, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(tcTrainKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smemTrain()));
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(C->gGrid, 0, mrtcu_rc_grid_floats() * sizeof(float), stream)) != cudaSuccess) return e;
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t maxCtas = uint32_t(sms) < C->partialBlocks ? uint32_t(sms) : C->partialBlocks;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    const uint32_t blocks = tiles < maxCtas ? tiles : maxCtas;
    tcTrainKernel<<<blocks, kTile, smemTrain(), stream>>>(*C, features, targets, n, 0u, 1u, 1.0f / (3.0f * float(n)),
                                                          C->partial, lossOut);
    reducePartialsKernel<<<gridFor(kMlpFloats), 256, 0, stream>>>(C->partial, blocks, C->gMlp);
    return cudaGetLastError();
}

extern "C" size_t mrtcu_rc_sort_scratch_words(uint32_t n) { return size_t(4) * n + mrtcu_sort_pairs_scratch_words(n); }

extern "C" cudaError_t mrtcu_rc_apply_queries(McacheParams C, const float* qFeat, const float4* qBeta, uint32_t n,
                                              uint32_t slots, float* scratch3, float4* L, uint32_t* sortScratch,
                                              cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    // queries in Morton order of their positions (when a sort scratch is
    // given and n is within the sort's limit); predictions land at each
    // query's own index either way
    const uint32_t* order = nullptr;
    if (sortScratch && n <= mrtcu_sort_pairs_max()) {
        uint32_t* keysA = sortScratch;
        uint32_t* valsA = keysA + n;
        uint32_t* keysB = valsA + n;
        uint32_t* valsB = keysB + n;
        queryKeysKernel<<<gridFor(n), 256, 0, stream>>>(C, qFeat, n, keysA, valsA);
        const cudaError_t se = mrtcu_sort_pairs(keysA, valsA, keysB, valsB, n, 4u, valsB + n, stream);
        if (se != cudaSuccess) return se;
        order = valsA;
    }
    const cudaError_t e = launchQuery(C, qFeat, n, scratch3, kRenderClamp, stream, order);
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
