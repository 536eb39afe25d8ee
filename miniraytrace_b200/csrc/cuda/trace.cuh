// Two-level BVH traversal for sm_100a: closest hit and any hit.
//
// Semantics follow the reference (core/shaders/intersect.glsl:48-178): a TLAS
// whose leaves are instances, a per-mesh BLAS in object space, the ray
// transformed into object space with its *unnormalised* direction so t is
// shared between spaces, hits accepted for t in (1e-4, tMax).
//
// Differences from the reference, by design:
//   - watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013) instead of
//     Moeller-Trumbore: no ray slips through a shared edge or vertex;
//   - 8-wide compressed BVH nodes (five 128-bit loads test eight child
//     boxes), traversed by groups: a stack entry is a node's remaining
//     child-hit mask, children are taken in ray-octant order, leaf
//     triangles of a node are tested before descending;
//   - box exits are widened by 1 + 2*gamma(3) = 1 + 3 * 2^-23 (Ize 2013) so a
//     rounding error in the slab test can never cull a real hit (the
//     reference's exact-comparison slab test occasionally drops a hit or an
//     occluder whose point lies on its leaf box's face);
//   - stacks are bounded and an overflow sets an error flag instead of
//     writing out of bounds; node, triangle and instance indices are checked.
#pragma once

#include "../common/device_types.h"
#include "vec.cuh"

#define MRT_EPS_RAY 1e-4f
// Upper bound on node visits of one traversal. A well-formed BVH never gets
// near it; it only turns a malformed tree into an error flag instead of an
// endless loop.
#define MRT_MAX_VISITS (1u << 22)

struct TraceRay {
    float3 o, d;
};

struct HitRecord {
    float t;
    float u, v;            // barycentrics of vertex 1 and 2
    uint32_t tri;          // packed triangle slot (leaf order)
    uint32_t inst;         // instance slot (TLAS leaf order)
};

// Per-ray constants of the watertight test.
struct Shear {
    int kx, ky, kz;
    float sx, sy, sz;
};

MRT_DEV Shear makeShear(float3 d) {
    Shear s;
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    s.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    s.kx = s.kz == 2 ? 0 : s.kz + 1;
    s.ky = s.kx == 2 ? 0 : s.kx + 1;
    if (comp(d, s.kz) < 0.0f) {
        const int t = s.kx;
        s.kx = s.ky;
        s.ky = t;
    }
    const float dz = comp(d, s.kz);
    s.sx = comp(d, s.kx) / dz;
    s.sy = comp(d, s.ky) / dz;
    s.sz = 1.0f / dz;
    return s;
}

MRT_DEV float3 safeInv(float3 d) {
    // 1/0 would give inf and (lo - o) * inf can produce NaN for points on the
    // slab; a huge finite reciprocal keeps the slab test ordered.
    const float big = 1e30f;
    return f3(d.x != 0.0f ? 1.0f / d.x : copysignf(big, d.x), d.y != 0.0f ? 1.0f / d.y : copysignf(big, d.y),
              d.z != 0.0f ? 1.0f / d.z : copysignf(big, d.z));
}

// Watertight test (Woop et al. 2013). Accepts t in (1e-4, tMax); both faces.
// The edge functions use explicit round-to-nearest products with no fused
// multiply-add, so an edge shared by two triangles evaluates to exactly
// opposite values from both sides.
MRT_DEV bool hitTriangle(const float4* __restrict__ tv, uint32_t tri, float3 o, const Shear& s, float tMax, float& tOut,
                         float& uOut, float& vOut) {
    const float4 p0 = ldg4(tv + 3 * tri), p1 = ldg4(tv + 3 * tri + 1), p2 = ldg4(tv + 3 * tri + 2);
    const float3 A = f3(p0) - o, B = f3(p1) - o, C = f3(p2) - o;
    const float Akz = comp(A, s.kz), Bkz = comp(B, s.kz), Ckz = comp(C, s.kz);
    const float Ax = __fsub_rn(comp(A, s.kx), __fmul_rn(s.sx, Akz));
    const float Ay = __fsub_rn(comp(A, s.ky), __fmul_rn(s.sy, Akz));
    const float Bx = __fsub_rn(comp(B, s.kx), __fmul_rn(s.sx, Bkz));
    const float By = __fsub_rn(comp(B, s.ky), __fmul_rn(s.sy, Bkz));
    const float Cx = __fsub_rn(comp(C, s.kx), __fmul_rn(s.sx, Ckz));
    const float Cy = __fsub_rn(comp(C, s.ky), __fmul_rn(s.sy, Ckz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {  // exact fallback on an edge
        U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
        V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
        W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = U + V + W;
    if (det == 0.0f) return false;
    const float T = U * (s.sz * Akz) + V * (s.sz * Bkz) + W * (s.sz * Ckz);
    const float rcp = 1.0f / det;
    const float t = T * rcp;
    if (!(t > MRT_EPS_RAY && t < tMax)) return false;
    tOut = t;
    uOut = V * rcp;
    vOut = W * rcp;
    return true;
}

// Round-to-nearest vector helpers with no fused multiply-add: they evaluate
// exactly the IEEE single-precision operation sequence of the reference
// shader expressions they restate.
MRT_DEV float3 sub_rn(float3 a, float3 b) { return f3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
MRT_DEV float dot_rn(float3 a, float3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
MRT_DEV float3 cross_rn(float3 a, float3 b) {
    return f3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(b.y, a.z)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(b.z, a.x)),
              __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(b.x, a.y)));
}
// Row-major 3x4 transform with the column-by-column sum order of a GLSL
// mat4 * vec4 product.
MRT_DEV float3 xformPoint_rn(const float* m, float3 p) {
    return f3(__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], p.x), __fmul_rn(m[1], p.y)), __fmul_rn(m[2], p.z)), m[3]),
              __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[4], p.x), __fmul_rn(m[5], p.y)), __fmul_rn(m[6], p.z)), m[7]),
              __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[8], p.x), __fmul_rn(m[9], p.y)), __fmul_rn(m[10], p.z)), m[11]));
}
MRT_DEV float3 xformDir_rn(const float* m, float3 d) {
    return f3(__fadd_rn(__fadd_rn(__fmul_rn(m[0], d.x), __fmul_rn(m[1], d.y)), __fmul_rn(m[2], d.z)),
              __fadd_rn(__fadd_rn(__fmul_rn(m[4], d.x), __fmul_rn(m[5], d.y)), __fmul_rn(m[6], d.z)),
              __fadd_rn(__fadd_rn(__fmul_rn(m[8], d.x), __fmul_rn(m[9], d.y)), __fmul_rn(m[10], d.z)));
}

// Re-evaluates the winning triangle with the reference's Moeller-Trumbore
// arithmetic (intersect.glsl:21-45) to report its t and barycentrics: the
// watertight test decides *which* triangle is hit, the reference formula
// gives the hit parameters, so hit points match the reference's to the ulp.
// Keeps the watertight values when the reference formula is degenerate for
// this ray (|det| < 1e-12 or t outside (1e-4, tMax]).
MRT_DEV void refineHit(const MrtFrameParams& P, float3 o, float3 d, HitRecord& hit) {
    const MrtInstance* in = P.instances + hit.inst;
    const float3 oo = xformPoint_rn(in->w2o, o), dd = xformDir_rn(in->w2o, d);
    const float3 v0 = f3(ldg4(P.triVerts + 3 * hit.tri));
    const float3 e1 = sub_rn(f3(ldg4(P.triVerts + 3 * hit.tri + 1)), v0);
    const float3 e2 = sub_rn(f3(ldg4(P.triVerts + 3 * hit.tri + 2)), v0);
    const float3 pv = cross_rn(dd, e2);
    const float det = dot_rn(e1, pv);
    if (!(fabsf(det) >= 1e-12f)) return;
    const float invDet = __fdiv_rn(1.0f, det);
    const float3 sv = sub_rn(oo, v0);
    const float u = __fmul_rn(dot_rn(sv, pv), invDet);
    const float3 q = cross_rn(sv, e1);
    const float v = __fmul_rn(dot_rn(dd, q), invDet);
    const float t = __fmul_rn(dot_rn(e2, q), invDet);
    if (!(t > MRT_EPS_RAY) || !(t <= hit.t * 1.0001f)) return;
    hit.t = t;
    hit.u = u;
    hit.v = v;
}

// Per-thread traffic counters for the roofline's algorithmic bytes: wide node
// records fetched (80 B each) and triangle tests (48 B each). `bad` records an
// out-of-range index met during traversal: the access is redirected to a
// valid element and the ray is reported through the error flag instead of
// reading outside the scene arrays.
struct TraversalCounters {
    uint32_t nodes = 0, tris = 0;
    bool bad = false;
};

// Decoded hits of one wide node.
struct WideHits {
    uint32_t childBase;  // first internal child node
    uint32_t primBase;   // first leaf primitive
    uint32_t nodeBits;   // bits 24-31: internal children hit (ray-ordered), bits 0-7: internal slot mask
    uint32_t primBits;   // bits 0-23: leaf primitives hit, relative to primBase
};

// Exact float of a byte: 2^23 + b - 2^23.
MRT_DEV float byteToFloat(uint32_t b) { return __uint_as_float(0x4B000000u | b) - 8388608.0f; }

// Tests the ray against the eight quantised child boxes of node `idx`.
// Child boxes decode as p + q * 2^(e-127) (the host quantised them
// conservatively for exactly this arithmetic); internal-child hits land on
// bit 24 + (slot XOR oct), so taking bits from the top visits the slots the
// ray reaches first first.
MRT_DEV WideHits intersectWide(const MrtFrameParams& P, uint32_t idx, float3 o, float3 inv, uint32_t oct, float tMax,
                               TraversalCounters& tc) {
    if (idx >= P.nodeCount) {
        tc.bad = true;
        idx = 0;
    }
    const float4* q = reinterpret_cast<const float4*>(P.nodes + idx);
    const float4 q0 = ldg4(q), q1 = ldg4(q + 1), q2 = ldg4(q + 2), q3 = ldg4(q + 3), q4 = ldg4(q + 4);
    tc.nodes++;
    const uint32_t eb = __float_as_uint(q0.w);
    const float sx = __uint_as_float((eb & 0xffu) << 23), sy = __uint_as_float(((eb >> 8) & 0xffu) << 23),
                sz = __uint_as_float(((eb >> 16) & 0xffu) << 23);
    const uint32_t imask = eb >> 24;
    WideHits h;
    h.childBase = __float_as_uint(q1.x);
    h.primBase = __float_as_uint(q1.y);
    h.nodeBits = imask;
    h.primBits = 0;
    const uint32_t meta[2] = {__float_as_uint(q1.z), __float_as_uint(q1.w)};
    const uint32_t lx[2] = {__float_as_uint(q2.x), __float_as_uint(q2.y)};
    const uint32_t ly[2] = {__float_as_uint(q2.z), __float_as_uint(q2.w)};
    const uint32_t lz[2] = {__float_as_uint(q3.x), __float_as_uint(q3.y)};
    const uint32_t hx[2] = {__float_as_uint(q3.z), __float_as_uint(q3.w)};
    const uint32_t hy[2] = {__float_as_uint(q4.x), __float_as_uint(q4.y)};
    const uint32_t hz[2] = {__float_as_uint(q4.z), __float_as_uint(q4.w)};
#pragma unroll
    for (int half = 0; half < 2; ++half) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t sh = 8u * uint32_t(j);
            const uint32_t m = (meta[half] >> sh) & 0xffu;
            if (m == 0u) continue;
            const float bx0 = q0.x + byteToFloat((lx[half] >> sh) & 0xffu) * sx;
            const float by0 = q0.y + byteToFloat((ly[half] >> sh) & 0xffu) * sy;
            const float bz0 = q0.z + byteToFloat((lz[half] >> sh) & 0xffu) * sz;
            const float bx1 = q0.x + byteToFloat((hx[half] >> sh) & 0xffu) * sx;
            const float by1 = q0.y + byteToFloat((hy[half] >> sh) & 0xffu) * sy;
            const float bz1 = q0.z + byteToFloat((hz[half] >> sh) & 0xffu) * sz;
            const float tx0 = (bx0 - o.x) * inv.x, tx1 = (bx1 - o.x) * inv.x;
            const float ty0 = (by0 - o.y) * inv.y, ty1 = (by1 - o.y) * inv.y;
            const float tz0 = (bz0 - o.z) * inv.z, tz1 = (bz1 - o.z) * inv.z;
            const float tEnter = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
            const float tExit =
                fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tMax)) * 1.00000036f;
            if (tEnter <= tExit) {
                const uint32_t slot = uint32_t(half * 4 + j);
                if ((imask >> slot) & 1u) h.nodeBits |= 1u << ((m & 31u) ^ oct);
                else h.primBits |= (m >> 5) << (m & 31u);
            }
        }
    }
    return h;
}

// Ray octant for child ordering: bit k set when direction component k > 0.
MRT_DEV uint32_t rayOctant(float3 d) { return (d.x > 0.0f ? 1u : 0u) | (d.y > 0.0f ? 2u : 0u) | (d.z > 0.0f ? 4u : 0u); }

// Node index of the internal child on hit bit b (24..31) of a group.
MRT_DEV uint32_t childIndex(uint32_t childBase, uint32_t imask, uint32_t b, uint32_t oct) {
    const uint32_t slot = (b - 24u) ^ oct;
    return childBase + uint32_t(__popc(imask & ((1u << slot) - 1u)));
}

#define MRT_WIDE_STACK 32
#define MRT_WIDE_TLAS_STACK 16

// Closest hit within one BLAS (object-space ray). Updates tMax and hit.
// Returns false on a stack overflow or an exhausted visit budget.
MRT_DEV bool closestBlas(const MrtFrameParams& P, uint32_t root, uint32_t inst, float3 o, float3 d, float& tMax,
                         HitRecord& hit, TraversalCounters& tc) {
    const float3 inv = safeInv(d);
    const Shear sh = makeShear(d);
    const uint32_t oct = rayOctant(d);
    uint2 stack[MRT_WIDE_STACK];
    int sp = 0;
    bool ok = true;
    WideHits g = intersectWide(P, root, o, inv, oct, tMax, tc);
    uint32_t visits = 0;
    for (;;) {
        if (++visits > MRT_MAX_VISITS) return false;
        while (g.primBits) {
            const uint32_t b = uint32_t(__ffs(g.primBits) - 1);
            g.primBits &= g.primBits - 1u;
            const uint32_t tri = g.primBase + b;
            ++tc.tris;
            if (tri >= P.triCount) {
                tc.bad = true;
                continue;
            }
            float t, u, v;
            if (hitTriangle(P.triVerts, tri, o, sh, tMax, t, u, v)) {
                tMax = t;
                hit.t = t;
                hit.u = u;
                hit.v = v;
                hit.tri = tri;
                hit.inst = inst;
            }
        }
        if (g.nodeBits & 0xff000000u) {
            const uint32_t b = 31u - uint32_t(__clz(g.nodeBits & 0xff000000u));
            const uint32_t rest = g.nodeBits & ~(1u << b);
            const uint32_t child = childIndex(g.childBase, g.nodeBits & 0xffu, b, oct);
            if (rest & 0xff000000u) {
                if (sp < MRT_WIDE_STACK) stack[sp++] = make_uint2(g.childBase, rest);
                else ok = false;
            }
            g = intersectWide(P, child, o, inv, oct, tMax, tc);
            continue;
        }
        if (sp == 0) return ok;
        const uint2 e = stack[--sp];
        g.childBase = e.x;
        g.nodeBits = e.y;
        g.primBits = 0;
    }
}

// Closest hit over the scene (reference intersect.glsl:88-125): the TLAS's
// leaf primitives are instances; each hit instance's BLAS is walked with the
// ray in its object space.
MRT_DEV bool traceClosest(const MrtFrameParams& P, float3 o, float3 d, float tMax, HitRecord& hit, TraversalCounters& tc) {
    hit.t = tMax;
    hit.tri = 0xffffffffu;
    hit.inst = 0;
    hit.u = hit.v = 0.0f;
    if (P.instanceCount == 0) return true;  // empty scene (the TLAS root is a placeholder)
    const float3 inv = safeInv(d);
    const uint32_t oct = rayOctant(d);
    uint2 stack[MRT_WIDE_TLAS_STACK];
    int sp = 0;
    bool ok = true;
    WideHits g = intersectWide(P, P.tlasRoot, o, inv, oct, tMax, tc);
    uint32_t visits = 0;
    for (;;) {
        if (++visits > MRT_MAX_VISITS) return false;
        while (g.primBits) {
            const uint32_t b = uint32_t(__ffs(g.primBits) - 1);
            g.primBits &= g.primBits - 1u;
            const uint32_t instIdx = g.primBase + b;
            if (instIdx >= P.instanceCount) {
                tc.bad = true;
                continue;
            }
            const MrtInstance* in = P.instances + instIdx;
            const float3 oo = xformPoint(in->w2o, o), dd = xformDir(in->w2o, d);
            ok &= closestBlas(P, in->blasRoot, instIdx, oo, dd, tMax, hit, tc);
        }
        if (g.nodeBits & 0xff000000u) {
            const uint32_t b = 31u - uint32_t(__clz(g.nodeBits & 0xff000000u));
            const uint32_t rest = g.nodeBits & ~(1u << b);
            const uint32_t child = childIndex(g.childBase, g.nodeBits & 0xffu, b, oct);
            if (rest & 0xff000000u) {
                if (sp < MRT_WIDE_TLAS_STACK) stack[sp++] = make_uint2(g.childBase, rest);
                else ok = false;
            }
            g = intersectWide(P, child, o, inv, oct, tMax, tc);
            continue;
        }
        if (sp == 0) break;
        const uint2 e = stack[--sp];
        g.childBase = e.x;
        g.nodeBits = e.y;
        g.primBits = 0;
    }
    if (hit.tri != 0xffffffffu) refineHit(P, o, d, hit);
    return ok;
}

// Any hit in (1e-4, tMax) within one BLAS (reference intersect.glsl:128-178).
MRT_DEV bool anyBlas(const MrtFrameParams& P, uint32_t root, float3 o, float3 d, float tMax, bool& ok,
                     TraversalCounters& tc) {
    const float3 inv = safeInv(d);
    const Shear sh = makeShear(d);
    const uint32_t oct = rayOctant(d);
    uint2 stack[MRT_WIDE_STACK];
    int sp = 0;
    WideHits g = intersectWide(P, root, o, inv, oct, tMax, tc);
    uint32_t visits = 0;
    for (;;) {
        if (++visits > MRT_MAX_VISITS) {
            ok = false;
            return false;
        }
        while (g.primBits) {
            const uint32_t b = uint32_t(__ffs(g.primBits) - 1);
            g.primBits &= g.primBits - 1u;
            const uint32_t tri = g.primBase + b;
            ++tc.tris;
            if (tri >= P.triCount) {
                tc.bad = true;
                continue;
            }
            float t, u, v;
            if (hitTriangle(P.triVerts, tri, o, sh, tMax, t, u, v)) return true;
        }
        if (g.nodeBits & 0xff000000u) {
            const uint32_t b = 31u - uint32_t(__clz(g.nodeBits & 0xff000000u));
            const uint32_t rest = g.nodeBits & ~(1u << b);
            const uint32_t child = childIndex(g.childBase, g.nodeBits & 0xffu, b, oct);
            if (rest & 0xff000000u) {
                if (sp < MRT_WIDE_STACK) stack[sp++] = make_uint2(g.childBase, rest);
                else ok = false;
            }
            g = intersectWide(P, child, o, inv, oct, tMax, tc);
            continue;
        }
        if (sp == 0) return false;
        const uint2 e = stack[--sp];
        g.childBase = e.x;
        g.nodeBits = e.y;
        g.primBits = 0;
    }
}

MRT_DEV bool traceAny(const MrtFrameParams& P, float3 o, float3 d, float tMax, bool& ok, TraversalCounters& tc) {
    if (P.instanceCount == 0) return false;  // empty scene
    const float3 inv = safeInv(d);
    const uint32_t oct = rayOctant(d);
    uint2 stack[MRT_WIDE_TLAS_STACK];
    int sp = 0;
    WideHits g = intersectWide(P, P.tlasRoot, o, inv, oct, tMax, tc);
    uint32_t visits = 0;
    for (;;) {
        if (++visits > MRT_MAX_VISITS) {
            ok = false;
            return false;
        }
        while (g.primBits) {
            const uint32_t b = uint32_t(__ffs(g.primBits) - 1);
            g.primBits &= g.primBits - 1u;
            const uint32_t instIdx = g.primBase + b;
            if (instIdx >= P.instanceCount) {
                tc.bad = true;
                continue;
            }
            const MrtInstance* in = P.instances + instIdx;
            const float3 oo = xformPoint(in->w2o, o), dd = xformDir(in->w2o, d);
            if (anyBlas(P, in->blasRoot, oo, dd, tMax, ok, tc)) return true;
        }
        if (g.nodeBits & 0xff000000u) {
            const uint32_t b = 31u - uint32_t(__clz(g.nodeBits & 0xff000000u));
            const uint32_t rest = g.nodeBits & ~(1u << b);
            const uint32_t child = childIndex(g.childBase, g.nodeBits & 0xffu, b, oct);
            if (rest & 0xff000000u) {
                if (sp < MRT_WIDE_TLAS_STACK) stack[sp++] = make_uint2(g.childBase, rest);
                else ok = false;
            }
            g = intersectWide(P, child, o, inv, oct, tMax, tc);
            continue;
        }
        if (sp == 0) return false;
        const uint2 e = stack[--sp];
        g.childBase = e.x;
        g.nodeBits = e.y;
        g.primBits = 0;
    }
}
