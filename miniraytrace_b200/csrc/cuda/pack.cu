// Commit-time assembly of the global scene arrays on the device (reference
// Renderer.cpp:333-446 repacks every mesh on the host). Each mesh keeps its
// vertex data, indices and 8-wide BVH in its own device buffers; a geometry
// commit uploads only the meshes that changed and rebuilds the global arrays
// from those buffers with the kernels below: HBM-bound copies and gathers.
#include <cuda_runtime.h>

#include "device_api.h"

namespace {

// Triangles in BLAS leaf order: the three positions (w = original triangle
// index bits, slot bits, 0) and the global vertex ids + original index, the
// layout the traversal and shading kernels read. Out-of-range primitive or
// vertex indices (never produced by the builders) skip the write and raise
// the error word.
__global__ void packTrianglesKernel(const float4* __restrict__ pos, uint32_t nv, const uint32_t* __restrict__ idx,
                                    const uint32_t* __restrict__ prims, uint32_t nt, uint32_t vbase, uint32_t tbase,
                                    float4* __restrict__ triVerts, uint4* __restrict__ triIndex,
                                    uint32_t* __restrict__ error) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nt; k += gridDim.x * blockDim.x) {
        const uint32_t lt = prims[k];
        if (lt >= nt) {
            atomicOr(error, 1u);
            continue;
        }
        const uint32_t i0 = idx[3 * size_t(lt)], i1 = idx[3 * size_t(lt) + 1], i2 = idx[3 * size_t(lt) + 2];
        if (i0 >= nv || i1 >= nv || i2 >= nv) {
            atomicOr(error, 1u);
            continue;
        }
        const float4 p0 = pos[i0], p1 = pos[i1], p2 = pos[i2];
        const uint32_t slot = tbase + k;
        triVerts[3 * size_t(slot)] = make_float4(p0.x, p0.y, p0.z, __uint_as_float(lt));
        triVerts[3 * size_t(slot) + 1] = make_float4(p1.x, p1.y, p1.z, __uint_as_float(slot));
        triVerts[3 * size_t(slot) + 2] = make_float4(p2.x, p2.y, p2.z, 0.0f);
        triIndex[slot] = make_uint4(i0 + vbase, i1 + vbase, i2 + vbase, lt);
    }
}

// Mesh-relative wide nodes into the global node array: child and primitive
// bases shifted by the mesh's node and triangle offsets.
__global__ void rebaseNodesKernel(const MrtWideNode* __restrict__ src, uint32_t n, uint32_t nodeBase,
                                  uint32_t triBase, MrtWideNode* __restrict__ dst) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint4* s = reinterpret_cast<const uint4*>(src + i);
        uint4 q[5];
        for (int k = 0; k < 5; ++k) q[k] = s[k];
        q[1].x += nodeBase;  // childBase
        q[1].y += triBase;   // primBase
        uint4* d = reinterpret_cast<uint4*>(dst + nodeBase + i);
        for (int k = 0; k < 5; ++k) d[k] = q[k];
    }
}

__global__ void fillKernel(float4* __restrict__ dst, size_t n, float4 v) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        dst[i] = v;
}

unsigned gridFor(size_t n, unsigned threads) {
    const size_t b = (n + threads - 1) / threads;
    return unsigned(b < 148u * 16u ? (b > 0 ? b : 1) : 148u * 16u);
}

}  // namespace

extern "C" cudaError_t mrtcu_pack_triangles(const float4* pos, uint32_t nv, const uint32_t* idx, const uint32_t* prims,
                                            uint32_t nt, uint32_t vbase, uint32_t tbase, float4* triVerts,
                                            uint4* triIndex, uint32_t* error, cudaStream_t stream) {
    if (nt == 0) return cudaSuccess;
    packTrianglesKernel<<<gridFor(nt, 256), 256, 0, stream>>>(pos, nv, idx, prims, nt, vbase, tbase, triVerts,
                                                              triIndex, error);
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_rebase_nodes(const MrtWideNode* src, uint32_t n, uint32_t nodeBase, uint32_t triBase,
                                          MrtWideNode* dst, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    rebaseNodesKernel<<<gridFor(n, 256), 256, 0, stream>>>(src, n, nodeBase, triBase, dst);
    return cudaGetLastError();
}

extern "C" cudaError_t mrtcu_fill_f4(float4* dst, size_t n, float4 value, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    fillKernel<<<gridFor(n, 256), 256, 0, stream>>>(dst, n, value);
    return cudaGetLastError();
}
