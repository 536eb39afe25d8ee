// Device build of one mesh's 8-wide BVH: triangle boxes -> Morton codes ->
// stable radix sort -> radix-tree topology (Karras 2012) -> one bottom-up
// pass for boxes and the SAH-optimal collapse plan -> level-by-level
// emission of the wide nodes. Every step evaluates the same expressions as
// the host reference (csrc/host/lbvh.cpp + csrc/host/wide_bvh.cpp, through
// csrc/common/lbvh_common.h and wide_collapse.h) and the output layout is
// derived from subtree sizes rather than from atomics, so the result is
// identical to the host's, node for node. Compiled with -fmad=false.
//
// Work and memory: every stage streams the triangle arrays once or a few
// times (HBM-bound integer/byte work); the radix sort is four 8-bit LSD
// passes over (code, index) pairs; the bottom-up pass runs one thread per
// leaf up the tree, the second thread to reach a node continues (no waits).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "../common/lbvh_common.h"
#include "../common/wide_collapse.h"
#include "device_api.h"

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 8;
constexpr int kSortTile = kSortThreads * kSortRounds;
constexpr int kScanThreads = 1024;

// ---- float <-> order-preserving unsigned, for atomic min/max of bounds ----
__device__ uint32_t orderedBits(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ float orderedFloat(uint32_t v) {
    return __uint_as_float((v & 0x80000000u) ? (v & 0x7fffffffu) : ~v);
}

// Counters block (uint32 words): [0..2] centroid lo (ordered), [3..5] hi,
// [6..8] frame lo (float bits), [9..11] frame scale, [12] next task count,
// [13] error flag, [14] total wide nodes, [16..21] root box (float bits).
enum { kCtrLo = 0, kCtrHi = 3, kCtrFrameLo = 6, kCtrFrameScale = 9, kCtrNext = 12, kCtrError = 13, kCtrTotal = 14,
       kCtrBounds = 16, kCtrWords = 24 };

__global__ void initCountersKernel(uint32_t* ctr) {
    const int i = threadIdx.x;
    if (i < kCtrWords) ctr[i] = (i < kCtrHi) ? 0xffffffffu : 0u;
}

// Triangle boxes (min/max over the three vertices in order, as the host)
// and the bounds of their centroids.
__global__ void triBoxKernel(const float4* __restrict__ pos, const uint32_t* __restrict__ idx, uint32_t n,
                             float4* __restrict__ boxLo, float4* __restrict__ boxHi, uint32_t* ctr) {
    float cLo[3] = {MRT_WIDE_INF, MRT_WIDE_INF, MRT_WIDE_INF}, cHi[3] = {-MRT_WIDE_INF, -MRT_WIDE_INF, -MRT_WIDE_INF};
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        float lo[3] = {MRT_WIDE_INF, MRT_WIDE_INF, MRT_WIDE_INF}, hi[3] = {-MRT_WIDE_INF, -MRT_WIDE_INF, -MRT_WIDE_INF};
        for (int c = 0; c < 3; ++c) {
            const float4 p = __ldg(pos + __ldg(idx + 3 * size_t(t) + c));
            const float v[3] = {p.x, p.y, p.z};
            for (int a = 0; a < 3; ++a) {
                lo[a] = v[a] < lo[a] ? v[a] : lo[a];
                hi[a] = hi[a] < v[a] ? v[a] : hi[a];
            }
        }
        boxLo[t] = make_float4(lo[0], lo[1], lo[2], 0.0f);
        boxHi[t] = make_float4(hi[0], hi[1], hi[2], 0.0f);
        for (int a = 0; a < 3; ++a) {
            const float c = (lo[a] + hi[a]) * 0.5f;
            cLo[a] = fminf(cLo[a], c);
            cHi[a] = fmaxf(cHi[a], c);
        }
    }
    for (int a = 0; a < 3; ++a) {
        uint32_t l = orderedBits(cLo[a]), h = orderedBits(cHi[a]);
        for (int o = 16; o > 0; o >>= 1) {
            l = min(l, __shfl_xor_sync(0xffffffffu, l, o));
            h = max(h, __shfl_xor_sync(0xffffffffu, h, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(ctr + kCtrLo + a, l);
            atomicMax(ctr + kCtrHi + a, h);
        }
    }
}

// Morton frame: one scale (1024 / largest centroid extent) for all axes.
__global__ void frameKernel(uint32_t* ctr) {
    if (threadIdx.x != 0) return;
    float lo[3], ext = 0.0f;
    for (int a = 0; a < 3; ++a) {
        lo[a] = orderedFloat(ctr[kCtrLo + a]);
        const float e = orderedFloat(ctr[kCtrHi + a]) - lo[a];
        ext = ext < e ? e : ext;
    }
    const float scale = ext > 0.0f ? 1024.0f / ext : 0.0f;
    for (int a = 0; a < 3; ++a) {
        ctr[kCtrFrameLo + a] = __float_as_uint(lo[a]);
        ctr[kCtrFrameScale + a] = __float_as_uint(scale);
    }
}

__global__ void mortonKernel(const float4* __restrict__ boxLo, const float4* __restrict__ boxHi, uint32_t n,
                             const uint32_t* __restrict__ ctr, uint32_t* __restrict__ keys,
                             uint32_t* __restrict__ vals) {
    float lo[3], scale[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = __uint_as_float(ctr[kCtrFrameLo + a]);
        scale[a] = __uint_as_float(ctr[kCtrFrameScale + a]);
    }
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const float4 l = boxLo[t], h = boxHi[t];
        const float bl[3] = {l.x, l.y, l.z}, bh[3] = {h.x, h.y, h.z};
        keys[t] = mortonCode(bl, bh, lo, scale);
        vals[t] = t;
    }
}

// ---- stable LSD radix sort of (key, value) pairs, 8 bits per pass ---------
// Tile = 2048 pairs per block (8 rounds of 256). hist[d * tiles + tile] =
// count of digit d in the tile; its exclusive scan (digit-major) is the
// first output position of each (digit, tile); the scatter ranks equal
// digits by input position within the tile, so the sort is stable.
__global__ void __launch_bounds__(kSortThreads) sortHistKernel(const uint32_t* __restrict__ keys, uint32_t n,
                                                               int shift, uint32_t* __restrict__ hist,
                                                               uint32_t tiles) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * kSortTile;
    for (int k = 0; k < kSortRounds; ++k) {
        const uint32_t i = base + k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of `len` words in place: each block scans a segment of
// kScanSegment words (four per thread) and writes its total; the totals are
// scanned by one block (a single segment) and added back to every segment.
constexpr uint32_t kScanSegment = 4 * kScanThreads;

// Block-wide exclusive scan of one value per thread; *total gets the sum.
__device__ uint32_t blockExclusiveScan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warpSums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warpSums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? warpSums[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kScanThreads / 32) warpSums[lane] = w;
    }
    __syncthreads();
    const uint32_t excl = x - v + (warp > 0 ? warpSums[warp - 1] : 0u);
    if (total) *total = warpSums[kScanThreads / 32 - 1];
    __syncthreads();
    return excl;
}

// Scans segment blockIdx.x of data in place; its total goes to sums[blockIdx.x].
__global__ void __launch_bounds__(kScanThreads) scanSegmentsKernel(uint32_t* __restrict__ data, uint32_t len,
                                                                   uint32_t* __restrict__ sums) {
    const uint32_t b = blockIdx.x * kScanSegment + threadIdx.x * 4;
    uint32_t v[4];
    for (int k = 0; k < 4; ++k) v[k] = b + k < len ? data[b + k] : 0u;
    const uint32_t t = v[0] + v[1] + v[2] + v[3];
    uint32_t total = 0;
    uint32_t run = blockExclusiveScan(t, &total);
    for (int k = 0; k < 4; ++k) {
        if (b + k < len) data[b + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0 && sums) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) addSegmentOffsetsKernel(uint32_t* __restrict__ data, uint32_t len,
                                                                        const uint32_t* __restrict__ offsets) {
    const uint32_t add = offsets[blockIdx.x];
    const uint32_t b = blockIdx.x * kScanSegment + threadIdx.x * 4;
    for (int k = 0; k < 4; ++k)
        if (b + k < len) data[b + k] += add;
}

__global__ void __launch_bounds__(kSortThreads)
    sortScatterKernel(const uint32_t* __restrict__ keysIn, const uint32_t* __restrict__ valsIn,
                      uint32_t* __restrict__ keysOut, uint32_t* __restrict__ valsOut, uint32_t n, int shift,
                      const uint32_t* __restrict__ offsets, uint32_t tiles) {
    __shared__ uint32_t base[256];
    __shared__ uint32_t warpCnt[kSortThreads / 32][256];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    base[tid] = offsets[tid * tiles + blockIdx.x];
    const uint32_t tileBase = blockIdx.x * kSortTile;
    const uint32_t lanesBelow = (1u << lane) - 1u;
    for (int k = 0; k < kSortRounds; ++k) {
        for (int w = 0; w < kSortThreads / 32; ++w) warpCnt[w][tid] = 0;
        __syncthreads();
        const uint32_t i = tileBase + k * kSortThreads + tid;
        const bool valid = i < n;
        const uint32_t key = valid ? keysIn[i] : 0u;
        const uint32_t digit = valid ? ((key >> shift) & 255u) : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, digit);
        const uint32_t rank = __popc(peers & lanesBelow);
        if (valid && rank == 0) warpCnt[warp][digit] = __popc(peers);
        __syncthreads();
        // thread tid owns digit tid: exclusive prefix of its count over warps
        uint32_t running = 0;
        for (int w = 0; w < kSortThreads / 32; ++w) {
            const uint32_t c = warpCnt[w][tid];
            warpCnt[w][tid] = running;
            running += c;
        }
        __syncthreads();
        if (valid) {
            const uint32_t dst = base[digit] + warpCnt[warp][digit] + rank;
            if (dst < n) {  // always: the counts come from the same keys
                keysOut[dst] = key;
                valsOut[dst] = valsIn[i];
            }
        }
        __syncthreads();
        base[tid] += running;
        __syncthreads();
    }
}

// ---- radix tree -----------------------------------------------------------
// Internal node i: children (MRT_LBVH_LEAF | position or internal index),
// first sorted position and primitive count; parent links for both.
struct Tree {
    uint32_t n;                    // primitives
    const uint32_t* codes;         // sorted codes
    const uint32_t* prims;         // sorted primitive indices
    const float4 *triLo, *triHi;   // boxes by primitive index
    uint32_t *left, *right, *first, *count;
    uint32_t* parent;              // [0, n-1): internal; [n-1, 2n-1): leaves by position
    float4 *lo, *hi;               // internal boxes
    float4* cost;                  // 2 per internal node
    uint2* split;                  // 8 bytes per internal node
    uint8_t* asLeaf;
    uint32_t* wideBelow;           // wide nodes below n when n becomes a wide node
    uint32_t* flags;
};

__global__ void karrasKernel(Tree T) {
    const int n = int(T.n);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        uint32_t l, r;
        int f, last;
        lbvhNode(T.codes, n, i, l, r, f, last);
        T.left[i] = l;
        T.right[i] = r;
        T.first[i] = uint32_t(f);
        T.count[i] = uint32_t(last - f + 1);
        T.parent[(l & MRT_LBVH_LEAF) ? (n - 1 + (l & ~MRT_LBVH_LEAF)) : l] = uint32_t(i);
        T.parent[(r & MRT_LBVH_LEAF) ? (n - 1 + (r & ~MRT_LBVH_LEAF)) : r] = uint32_t(i);
        if (i == 0) T.parent[0] = 0xffffffffu;
    }
}

// Reads of data another thread of the running bottom-up pass wrote go
// through L2 (ld.global.cg), never a possibly stale L1 line.
__device__ float4 ldcg4(const float4* p) { return __ldcg(p); }

struct NodeView {
    float lo[3], hi[3];
    float cost[8];
    uint32_t count;
    uint32_t leaf;  // single root is a wide leaf
};

__device__ void loadBox(const Tree& T, uint32_t ref, float lo[3], float hi[3], bool coherent) {
    float4 l, h;
    if (ref & MRT_LBVH_LEAF) {
        const uint32_t p = T.prims[ref & ~MRT_LBVH_LEAF];
        l = T.triLo[p];
        h = T.triHi[p];
    } else if (coherent) {
        l = ldcg4(T.lo + ref);
        h = ldcg4(T.hi + ref);
    } else {
        l = T.lo[ref];
        h = T.hi[ref];
    }
    lo[0] = l.x;
    lo[1] = l.y;
    lo[2] = l.z;
    hi[0] = h.x;
    hi[1] = h.y;
    hi[2] = h.z;
}

__device__ NodeView viewChild(const Tree& T, uint32_t ref, uint32_t maxLeaf) {
    NodeView v;
    loadBox(T, ref, v.lo, v.hi, true);
    if (ref & MRT_LBVH_LEAF) {
        v.count = 1;
        v.leaf = 1;
        widePlanLeaf(wideArea(v.lo, v.hi), 1, maxLeaf, v.cost);
    } else {
        v.count = T.count[ref];
        v.leaf = __ldcg(T.asLeaf + ref);
        const float4 c0 = ldcg4(T.cost + 2 * ref), c1 = ldcg4(T.cost + 2 * ref + 1);
        v.cost[0] = c0.x;
        v.cost[1] = c0.y;
        v.cost[2] = c0.z;
        v.cost[3] = c0.w;
        v.cost[4] = c1.x;
        v.cost[5] = c1.y;
        v.cost[6] = c1.z;
        v.cost[7] = c1.w;
    }
    return v;
}

__device__ uint32_t splitByte(uint2 s, uint32_t j) { return ((j < 4 ? s.x : s.y) >> (8 * (j & 3))) & 0xffu; }

// Kids of internal node n as a wide node, in the host's gather order.
// Binary leaves have all-zero split tables. `coherent` selects L2 loads
// (inside the bottom-up pass).
__device__ int gatherKids(const Tree& T, uint32_t n, uint32_t kids[8], bool coherent) {
    uint2 st[8];  // (ref, j); the pending j's sum to at most 8
    int sp = 0, nk = 0;
    const uint2 s0 = coherent ? __ldcg(T.split + n) : T.split[n];
    const uint32_t k0 = splitByte(s0, 0);
    st[sp++] = make_uint2(T.right[n], 8u - k0);
    st[sp++] = make_uint2(T.left[n], k0);
    while (sp > 0 && nk < 8) {
        const uint2 e = st[--sp];
        const uint32_t ref = e.x;
        uint32_t j = e.y;
        if (ref & MRT_LBVH_LEAF) {
            kids[nk++] = ref;
            continue;
        }
        const uint2 s = coherent ? __ldcg(T.split + ref) : T.split[ref];
        while (j > 1 && splitByte(s, j - 1) == 0) --j;
        if (j == 1) {
            kids[nk++] = ref;
            continue;
        }
        const uint32_t k = splitByte(s, j - 1);
        if (sp + 2 > 8) break;  // unreachable for j <= 8
        st[sp++] = make_uint2(T.right[ref], j - k);
        st[sp++] = make_uint2(T.left[ref], k);
    }
    return nk;
}

__global__ void bottomUpKernel(Tree T, uint32_t maxLeaf) {
    const uint32_t n = T.n;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        uint32_t node = T.parent[n - 1 + p];
        while (node != 0xffffffffu) {
            __threadfence();
            if (atomicAdd(T.flags + node, 1u) == 0u) break;  // the sibling subtree is not done yet
            __threadfence();
            const NodeView a = viewChild(T, T.left[node], maxLeaf);
            const NodeView b = viewChild(T, T.right[node], maxLeaf);
            float lo[3], hi[3];
            for (int k = 0; k < 3; ++k) {  // std::min / std::max of (left, right)
                lo[k] = b.lo[k] < a.lo[k] ? b.lo[k] : a.lo[k];
                hi[k] = a.hi[k] < b.hi[k] ? b.hi[k] : a.hi[k];
            }
            float cost[8];
            uint8_t split[8];
            const uint8_t leaf =
                widePlanInternal(a.cost, b.cost, wideArea(lo, hi), a.count + b.count, maxLeaf, cost, split);
            T.lo[node] = make_float4(lo[0], lo[1], lo[2], 0.0f);
            T.hi[node] = make_float4(hi[0], hi[1], hi[2], 0.0f);
            T.cost[2 * node] = make_float4(cost[0], cost[1], cost[2], cost[3]);
            T.cost[2 * node + 1] = make_float4(cost[4], cost[5], cost[6], cost[7]);
            T.split[node] = make_uint2(uint32_t(split[0]) | uint32_t(split[1]) << 8 | uint32_t(split[2]) << 16 |
                                           uint32_t(split[3]) << 24,
                                       uint32_t(split[4]) | uint32_t(split[5]) << 8 | uint32_t(split[6]) << 16 |
                                           uint32_t(split[7]) << 24);
            T.asLeaf[node] = leaf;
            __threadfence();
            // wide nodes below `node` when it becomes a wide node
            uint32_t kids[8];
            const int nk = gatherKids(T, node, kids, true);
            uint32_t below = 0;
            for (int i = 0; i < nk; ++i) {
                const uint32_t r = kids[i];
                if (!(r & MRT_LBVH_LEAF) && !__ldcg(T.asLeaf + r)) below += 1u + __ldcg(T.wideBelow + r);
            }
            T.wideBelow[node] = below;
            node = T.parent[node];
        }
    }
}

// Root task, the total node count (1 when the whole mesh is one leaf) and
// the root box.
__global__ void rootTaskKernel(Tree T, uint4* tasks, uint32_t* ctr) {
    if (threadIdx.x != 0) return;
    const uint32_t root = T.n == 1 ? MRT_LBVH_LEAF : 0u;
    tasks[0] = make_uint4(0u, root, 1u, 0u);
    ctr[kCtrTotal] = (root & MRT_LBVH_LEAF) || T.asLeaf[0] ? 1u : 1u + T.wideBelow[0];
    float lo[3], hi[3];
    loadBox(T, root, lo, hi, false);
    for (int a = 0; a < 3; ++a) {
        ctr[kCtrBounds + a] = __float_as_uint(lo[a]);
        ctr[kCtrBounds + 3 + a] = __float_as_uint(hi[a]);
    }
}

// One wide node per task (wide index, binary ref, first child slot, first
// primitive slot); its internal children become the next level's tasks.
__global__ void emitKernel(Tree T, uint32_t maxLeaf, const uint4* __restrict__ tasks, uint32_t nTasks,
                           uint4* __restrict__ next, uint32_t* ctr, MrtWideNode* __restrict__ nodes,
                           uint32_t* __restrict__ primOrder, uint32_t nodeCap) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nTasks; t += gridDim.x * blockDim.x) {
        const uint4 task = tasks[t];
        const uint32_t w = task.x, ref = task.y, childBase = task.z, primBase = task.w;
        uint32_t kids[8];
        int nk;
        if ((ref & MRT_LBVH_LEAF) || T.asLeaf[ref]) {
            kids[0] = ref;
            nk = 1;
        } else {
            nk = gatherKids(T, ref, kids, false);
        }
        WideKid wk[8];
        uint32_t firstPos[8];
        for (int i = 0; i < nk; ++i) {
            const uint32_t r = kids[i];
            loadBox(T, r, wk[i].lo, wk[i].hi, false);
            if (r & MRT_LBVH_LEAF) {
                wk[i].count = 1;
                wk[i].leaf = 1;
                firstPos[i] = r & ~MRT_LBVH_LEAF;
            } else {
                wk[i].count = T.count[r];
                wk[i].leaf = T.asLeaf[r];
                firstPos[i] = T.first[r];
            }
        }
        MrtWideNode node;
        int bySlot[8];
        if (!wideEmitNode(wk, nk, node, bySlot) || w >= nodeCap) {
            atomicOr(ctr + kCtrError, 1u);
            continue;
        }
        node.childBase = childBase;
        node.primBase = primBase;
        const uint4* src = reinterpret_cast<const uint4*>(&node);
        uint4* dst = reinterpret_cast<uint4*>(nodes + w);
        for (int q = 0; q < 5; ++q) dst[q] = src[q];
        // leaf primitives in slot order, then the internal children's tasks
        uint32_t off = 0, internal = 0;
        for (int s = 0; s < 8; ++s) {
            const int i = bySlot[s];
            if (i < 0) continue;
            if (wk[i].leaf) {
                if (primBase + off + wk[i].count > T.n || firstPos[i] + wk[i].count > T.n) {
                    atomicOr(ctr + kCtrError, 2u);
                    break;
                }
                for (uint32_t k = 0; k < wk[i].count; ++k) primOrder[primBase + off + k] = T.prims[firstPos[i] + k];
                off += wk[i].count;
            } else {
                ++internal;
            }
        }
        uint32_t nextChild = childBase + internal, nextPrim = primBase + off, rank = 0;
        for (int s = 0; s < 8; ++s) {
            const int i = bySlot[s];
            if (i < 0 || wk[i].leaf) continue;
            const uint32_t r = kids[i];
            const uint32_t slot = atomicAdd(ctr + kCtrNext, 1u);
            if (slot < T.n) next[slot] = make_uint4(childBase + rank, r, nextChild, nextPrim);
            else atomicOr(ctr + kCtrError, 4u);
            nextChild += T.wideBelow[r];
            nextPrim += wk[i].count;
            ++rank;
        }
    }
}

size_t alignUp(size_t x) { return (x + 255) & ~size_t(255); }

struct Carve {
    char* base;
    size_t off = 0;
    template <class T> T* take(size_t count) {
        T* p = reinterpret_cast<T*>(base + off);
        off += alignUp(count * sizeof(T));
        return p;
    }
};

}  // namespace

// The builder's stable LSD radix sort for other callers: `passes` 8-bit
// passes (even, so the sorted pairs end in keysA / valsA) over n pairs.
// scratch holds mrtcu_sort_pairs_scratch_words(n) words. n is limited so the
// digit histogram (256 words a 2,048-pair tile) scans in two levels.
extern "C" uint32_t mrtcu_sort_pairs_max(void) { return uint32_t(kScanSegment) * kScanSegment / 256u * kSortTile; }

extern "C" size_t mrtcu_sort_pairs_scratch_words(uint32_t n) {
    const size_t tiles = (size_t(n) + kSortTile - 1) / kSortTile, len = 256 * tiles;
    return len + (len + kScanSegment - 1) / kScanSegment;
}

extern "C" cudaError_t mrtcu_sort_pairs(uint32_t* keysA, uint32_t* valsA, uint32_t* keysB, uint32_t* valsB,
                                        uint32_t n, uint32_t passes, uint32_t* scratch, cudaStream_t stream) {
    if (n <= 1) return cudaSuccess;
    if ((passes & 1u) || passes > 4u || n > mrtcu_sort_pairs_max()) return cudaErrorInvalidValue;
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    uint32_t* hist = scratch;
    uint32_t* segSums = scratch + size_t(256) * tiles;
    for (uint32_t pass = 0; pass < passes; ++pass) {
        const int shift = 8 * int(pass);
        uint32_t* kIn = pass & 1 ? keysB : keysA;
        uint32_t* vIn = pass & 1 ? valsB : valsA;
        uint32_t* kOut = pass & 1 ? keysA : keysB;
        uint32_t* vOut = pass & 1 ? valsA : valsB;
        sortHistKernel<<<tiles, kSortThreads, 0, stream>>>(kIn, n, shift, hist, tiles);
        const uint32_t len = 256u * tiles, segments = (len + kScanSegment - 1) / kScanSegment;
        if (segments == 1) {
            scanSegmentsKernel<<<1, kScanThreads, 0, stream>>>(hist, len, nullptr);
        } else {
            scanSegmentsKernel<<<segments, kScanThreads, 0, stream>>>(hist, len, segSums);
            scanSegmentsKernel<<<1, kScanThreads, 0, stream>>>(segSums, segments, nullptr);
            addSegmentOffsetsKernel<<<segments, kScanThreads, 0, stream>>>(hist, len, segSums);
        }
        sortScatterKernel<<<tiles, kSortThreads, 0, stream>>>(kIn, vIn, kOut, vOut, n, shift, hist, tiles);
    }
    return cudaGetLastError();
}

extern "C" size_t mrtcu_wide_bvh_scratch_bytes(uint32_t triCount) {
    const size_t n = triCount > 0 ? triCount : 1;
    const size_t tiles = (n + kSortTile - 1) / kSortTile;
    size_t b = 0;
    b += alignUp(kCtrWords * 4);
    b += 2 * alignUp(n * 16);              // triangle boxes
    b += 4 * alignUp(n * 4);               // keys / values, two buffers each
    b += alignUp(256 * tiles * 4);         // histogram
    b += alignUp(kScanSegment * 4);        // scan segment totals
    b += 4 * alignUp(n * 4);               // left, right, first, count
    b += alignUp(2 * n * 4);               // parent
    b += 2 * alignUp(n * 16);              // internal boxes
    b += alignUp(2 * n * 16);              // cost
    b += alignUp(n * 8);                   // split
    b += alignUp(n);                       // asLeaf
    b += 2 * alignUp(n * 4);               // wideBelow, flags
    b += 2 * alignUp(n * 16);              // task queues
    return b;
}

extern "C" cudaError_t mrtcu_build_wide_bvh(const float4* positions, const uint32_t* indices, uint32_t triCount,
                                            uint32_t maxLeaf, void* scratch, size_t scratchBytes,
                                            MrtWideNode* nodesOut, uint32_t nodeCapacity, uint32_t* primOrderOut,
                                            uint32_t* nodeCountOut, float boundsOut[6], uint32_t* launchesOut,
                                            cudaStream_t stream) {
    *nodeCountOut = 0;
    if (triCount == 0) return cudaSuccess;
    if (scratchBytes < mrtcu_wide_bvh_scratch_bytes(triCount) || nodeCapacity < triCount || maxLeaf < 1 ||
        maxLeaf > 3)
        return cudaErrorInvalidValue;
    const uint32_t n = triCount;
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    // the scan of the sort histogram takes at most kScanSegment segments
    // (meshes of up to 134 M triangles)
    if ((256u * uint64_t(tiles) + kScanSegment - 1) / kScanSegment > kScanSegment) return cudaErrorInvalidValue;
    Carve c{static_cast<char*>(scratch)};
    uint32_t* ctr = c.take<uint32_t>(kCtrWords);
    float4* triLo = c.take<float4>(n);
    float4* triHi = c.take<float4>(n);
    uint32_t* keysA = c.take<uint32_t>(n);
    uint32_t* keysB = c.take<uint32_t>(n);
    uint32_t* valsA = c.take<uint32_t>(n);
    uint32_t* valsB = c.take<uint32_t>(n);
    uint32_t* hist = c.take<uint32_t>(size_t(256) * tiles);
    uint32_t* segSums = c.take<uint32_t>(kScanSegment);
    Tree T;
    T.n = n;
    T.left = c.take<uint32_t>(n);
    T.right = c.take<uint32_t>(n);
    T.first = c.take<uint32_t>(n);
    T.count = c.take<uint32_t>(n);
    T.parent = c.take<uint32_t>(2 * size_t(n));
    T.lo = c.take<float4>(n);
    T.hi = c.take<float4>(n);
    T.cost = c.take<float4>(2 * size_t(n));
    T.split = c.take<uint2>(n);
    T.asLeaf = c.take<uint8_t>(n);
    T.wideBelow = c.take<uint32_t>(n);
    T.flags = c.take<uint32_t>(n);
    uint4* tasksA = c.take<uint4>(n);
    uint4* tasksB = c.take<uint4>(n);
    T.triLo = triLo;
    T.triHi = triHi;

    uint32_t launches = 0;
    const int grid = int(std::min<uint32_t>((n + 255) / 256, 148u * 8u));
    initCountersKernel<<<1, 32, 0, stream>>>(ctr);
    triBoxKernel<<<grid, 256, 0, stream>>>(positions, indices, n, triLo, triHi, ctr);
    frameKernel<<<1, 32, 0, stream>>>(ctr);
    mortonKernel<<<grid, 256, 0, stream>>>(triLo, triHi, n, ctr, keysA, valsA);
    launches += 4;
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 8 * pass;
        uint32_t* kIn = pass & 1 ? keysB : keysA;
        uint32_t* vIn = pass & 1 ? valsB : valsA;
        uint32_t* kOut = pass & 1 ? keysA : keysB;
        uint32_t* vOut = pass & 1 ? valsA : valsB;
        sortHistKernel<<<tiles, kSortThreads, 0, stream>>>(kIn, n, shift, hist, tiles);
        const uint32_t len = 256u * tiles, segments = (len + kScanSegment - 1) / kScanSegment;
        if (segments == 1) {
            scanSegmentsKernel<<<1, kScanThreads, 0, stream>>>(hist, len, nullptr);
        } else {
            scanSegmentsKernel<<<segments, kScanThreads, 0, stream>>>(hist, len, segSums);
            scanSegmentsKernel<<<1, kScanThreads, 0, stream>>>(segSums, segments, nullptr);
            addSegmentOffsetsKernel<<<segments, kScanThreads, 0, stream>>>(hist, len, segSums);
            launches += 2;
        }
        sortScatterKernel<<<tiles, kSortThreads, 0, stream>>>(kIn, vIn, kOut, vOut, n, shift, hist, tiles);
        launches += 3;
    }
    T.codes = keysA;  // four passes: the sorted pairs are back in A
    T.prims = valsA;
    if (n > 1) {
        cudaError_t e = cudaMemsetAsync(T.flags, 0, size_t(n) * 4, stream);
        if (e != cudaSuccess) return e;
        karrasKernel<<<grid, 256, 0, stream>>>(T);
        bottomUpKernel<<<grid, 256, 0, stream>>>(T, maxLeaf);
        launches += 2;
    }
    rootTaskKernel<<<1, 32, 0, stream>>>(T, tasksA, ctr);
    ++launches;
    uint32_t host[kCtrWords];  // counters: total nodes, root box
    cudaError_t e = cudaMemcpyAsync(host, ctr, sizeof(host), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    const uint32_t total = host[kCtrTotal];
    if (total > nodeCapacity) return cudaErrorInvalidValue;
    for (int a = 0; a < 6; ++a) {
        const uint32_t bits = host[kCtrBounds + a];
        float f;
        memcpy(&f, &bits, 4);
        boundsOut[a] = f;
    }
    // level by level; the host reads each level's task count
    uint32_t nTasks = 1, levels = 0;
    uint4* in = tasksA;
    uint4* out = tasksB;
    while (nTasks > 0) {
        // a wide tree over n primitives has at most n nodes per level and is
        // no deeper than the radix tree (at most 63 levels: 30 code bits
        // extended by 32 position bits)
        if (nTasks > n || ++levels > 128) return cudaErrorInvalidValue;
        e = cudaMemsetAsync(ctr + kCtrNext, 0, 4, stream);
        if (e != cudaSuccess) return e;
        const int g = int(std::min<uint32_t>((nTasks + 127) / 128, 148u * 16u));
        emitKernel<<<g, 128, 0, stream>>>(T, maxLeaf, in, nTasks, out, ctr, nodesOut, primOrderOut, nodeCapacity);
        ++launches;
        e = cudaMemcpyAsync(&nTasks, ctr + kCtrNext, 4, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
        uint4* t = in;
        in = out;
        out = t;
    }
    uint32_t error = 0;
    e = cudaMemcpyAsync(&error, ctr + kCtrError, 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    if (error) return cudaErrorInvalidValue;
    *nodeCountOut = total;
    if (launchesOut) *launchesOut += launches;
    return cudaGetLastError();
}
