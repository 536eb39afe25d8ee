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
//   - a visited internal node tests both children's boxes (one 64-byte
//     fetch, the pair is adjacent), descends into the nearer and pushes the
//     farther, so culling uses the current closest t;
//   - box exits are widened by 1 + 2*gamma(3) = 1 + 3 * 2^-23 (Ize 2013) so a
//     rounding error in the slab test can never cull a real hit (the
//     reference's exact-comparison slab test occasionally drops a hit or an
//     occluder whose point lies on its leaf box's face);
//   - stacks are bounded and an overflow sets an error flag instead of
//     writing out of bounds.
#pragma once

#include "../common/device_types.h"
#include "vec.cuh"

#define MRT_EPS_RAY 1e-4f
#define MRT_TLAS_STACK 32
#define MRT_BLAS_STACK 48
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

// Slab test; returns the entry distance, or +inf when the box is missed or
// starts beyond tMax.
MRT_DEV float slab(const float* lo, const float* hi, float3 o, float3 inv, float tMax) {
    const float tx0 = (lo[0] - o.x) * inv.x, tx1 = (hi[0] - o.x) * inv.x;
    const float ty0 = (lo[1] - o.y) * inv.y, ty1 = (hi[1] - o.y) * inv.y;
    const float tz0 = (lo[2] - o.z) * inv.z, tz1 = (hi[2] - o.z) * inv.z;
    const float tEnter = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
    const float tExit = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tMax)) * 1.00000036f;
    return tEnter <= tExit ? tEnter : __int_as_float(0x7f800000);
}

MRT_DEV float slabNode(const float4& a, const float4& b, float3 o, float3 inv, float tMax) {
    const float lo[3] = {a.x, a.y, a.z};
    const float hi[3] = {b.x, b.y, b.z};
    return slab(lo, hi, o, inv, tMax);
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

// Per-thread traffic counters for the roofline's algorithmic bytes: node
// records fetched (32 B each) and triangle tests (48 B each).
// `bad` records an out-of-range index met during traversal: the access is
// redirected to a valid element and the ray is reported through the error
// flag instead of reading outside the scene arrays.
struct TraversalCounters {
    uint32_t nodes = 0, tris = 0;
    bool bad = false;
};

MRT_DEV void loadNode(const MrtFrameParams& P, uint32_t i, float4& a, float4& b, TraversalCounters& c) {
    if (i >= P.nodeCount) {
        c.bad = true;
        i = 0;
    }
    const float4* p = reinterpret_cast<const float4*>(P.nodes + i);
    a = ldg4(p);
    b = ldg4(p + 1);
    c.nodes++;
}

// Closest hit within one BLAS (object-space ray). Updates tMax and hit.
// Stack entries carry the far child's entry distance, so a popped subtree
// that starts beyond the current closest hit is skipped without fetching it.
// Returns false on a stack overflow or an exhausted visit budget.
MRT_DEV bool closestBlas(const MrtFrameParams& P, uint32_t root, uint32_t inst, float3 o, float3 d, float& tMax,
                         HitRecord& hit, TraversalCounters& tc) {
    const float3 inv = safeInv(d);
    const Shear sh = makeShear(d);
    uint2 stack[MRT_BLAS_STACK];
    int sp = 0;
    float4 na, nb;
    loadNode(P, root, na, nb, tc);
    if (!(slabNode(na, nb, o, inv, tMax) < __int_as_float(0x7f800000))) return true;
    bool ok = true;
    uint32_t visits = 0;
    for (;;) {
        if (++visits > MRT_MAX_VISITS) { ok = false; return false; }
        const uint32_t packed = __float_as_uint(nb.w);
        const uint32_t first = __float_as_uint(na.w);
        const uint32_t count = packed >> 2;
        if (count == 0) {
            float4 a0, b0, a1, b1;
            loadNode(P, first, a0, b0, tc);
            loadNode(P, first + 1, a1, b1, tc);
            const float t0 = slabNode(a0, b0, o, inv, tMax);
            const float t1 = slabNode(a1, b1, o, inv, tMax);
            const bool h0 = t0 < __int_as_float(0x7f800000), h1 = t1 < __int_as_float(0x7f800000);
            if (h0 && h1) {
                const bool firstNear = t0 <= t1;
                if (sp < MRT_BLAS_STACK) stack[sp++] = make_uint2(firstNear ? first + 1 : first, __float_as_uint(firstNear ? t1 : t0));
                else ok = false;
                na = firstNear ? a0 : a1;
                nb = firstNear ? b0 : b1;
                continue;
            }
            if (h0 || h1) {
                na = h0 ? a0 : a1;
                nb = h0 ? b0 : b1;
                continue;
            }
        } else {
            for (uint32_t i = 0; i < count; ++i) {
                float t, u, v;
                ++tc.tris;
                if (first + i >= P.triCount) {
                    tc.bad = true;
                    break;
                }
                if (hitTriangle(P.triVerts, first + i, o, sh, tMax, t, u, v)) {
                    tMax = t;
                    hit.t = t;
                    hit.u = u;
                    hit.v = v;
                    hit.tri = first + i;
                    hit.inst = inst;
                }
            }
        }
        // pop the nearest pending subtree that can still hold a closer hit
        for (;;) {
            if (sp == 0) return ok;
            const uint2 e = stack[--sp];
            if (__uint_as_float(e.y) <= tMax * 1.00000036f) {
                loadNode(P, e.x, na, nb, tc);
                break;
            }
        }
    }
}

// Closest hit over the scene (reference intersect.glsl:88-125).
MRT_DEV bool traceClosest(const MrtFrameParams& P, float3 o, float3 d, float tMax, HitRecord& hit, TraversalCounters& tc) {
    hit.t = tMax;
    hit.tri = 0xffffffffu;
    hit.inst = 0;
    hit.u = hit.v = 0.0f;
    if (P.instanceCount == 0) return true;  // empty scene (the TLAS root is a placeholder)
    const float3 inv = safeInv(d);
    uint2 stack[MRT_TLAS_STACK];
    int sp = 0;
    float4 na, nb;
    loadNode(P, P.tlasRoot, na, nb, tc);
    if (!(slabNode(na, nb, o, inv, tMax) < __int_as_float(0x7f800000))) return true;
    bool ok = true;
    uint32_t visits = 0;
    for (;;) {
        if (++visits > MRT_MAX_VISITS) { ok = false; return false; }
        const uint32_t packed = __float_as_uint(nb.w);
        const uint32_t first = __float_as_uint(na.w);
        const uint32_t count = packed >> 2;
        if (count == 0) {
            float4 a0, b0, a1, b1;
            loadNode(P, first, a0, b0, tc);
            loadNode(P, first + 1, a1, b1, tc);
            const float t0 = slabNode(a0, b0, o, inv, tMax);
            const float t1 = slabNode(a1, b1, o, inv, tMax);
            const bool h0 = t0 < __int_as_float(0x7f800000), h1 = t1 < __int_as_float(0x7f800000);
            if (h0 && h1) {
                const bool firstNear = t0 <= t1;
                if (sp < MRT_TLAS_STACK) stack[sp++] = make_uint2(firstNear ? first + 1 : first, __float_as_uint(firstNear ? t1 : t0));
                else ok = false;
                na = firstNear ? a0 : a1;
                nb = firstNear ? b0 : b1;
                continue;
            }
            if (h0 || h1) {
                na = h0 ? a0 : a1;
                nb = h0 ? b0 : b1;
                continue;
            }
        } else {
            for (uint32_t i = 0; i < count; ++i) {
                const uint32_t instIdx = first + i;
                if (instIdx >= P.instanceCount) {
                    tc.bad = true;
                    break;
                }
                const MrtInstance* in = P.instances + instIdx;
                const float3 oo = xformPoint(in->w2o, o), dd = xformDir(in->w2o, d);
                ok &= closestBlas(P, in->blasRoot, instIdx, oo, dd, tMax, hit, tc);
            }
        }
        for (;;) {
            if (sp == 0) {
                if (hit.tri != 0xffffffffu) refineHit(P, o, d, hit);
                return ok;
            }
            const uint2 e = stack[--sp];
            if (__uint_as_float(e.y) <= tMax * 1.00000036f) {
                loadNode(P, e.x, na, nb, tc);
                break;
            }
        }
    }
}

// Any hit in (1e-4, tMax) (reference intersect.glsl:128-178).
MRT_DEV bool anyBlas(const MrtFrameParams& P, uint32_t root, float3 o, float3 d, float tMax, bool& ok,
                     TraversalCounters& tc) {
    const float3 inv = safeInv(d);
    const Shear sh = makeShear(d);
    uint32_t stack[MRT_BLAS_STACK];
    int sp = 0;
    float4 na, nb;
    loadNode(P, root, na, nb, tc);
    if (!(slabNode(na, nb, o, inv, tMax) < __int_as_float(0x7f800000))) return false;
    uint32_t visits = 0;
    for (;;) {
        if (++visits > MRT_MAX_VISITS) { ok = false; return false; }
        const uint32_t packed = __float_as_uint(nb.w);
        const uint32_t first = __float_as_uint(na.w);
        const uint32_t count = packed >> 2;
        if (count == 0) {
            float4 a0, b0, a1, b1;
            loadNode(P, first, a0, b0, tc);
            loadNode(P, first + 1, a1, b1, tc);
            const bool h0 = slabNode(a0, b0, o, inv, tMax) < __int_as_float(0x7f800000);
            const bool h1 = slabNode(a1, b1, o, inv, tMax) < __int_as_float(0x7f800000);
            if (h0 && h1) {
                if (sp < MRT_BLAS_STACK) stack[sp++] = first + 1;
                else ok = false;
            }
            if (h0 || h1) {
                na = h0 ? a0 : a1;
                nb = h0 ? b0 : b1;
                continue;
            }
        } else {
            for (uint32_t i = 0; i < count; ++i) {
                float t, u, v;
                ++tc.tris;
                if (first + i >= P.triCount) {
                    tc.bad = true;
                    break;
                }
                if (hitTriangle(P.triVerts, first + i, o, sh, tMax, t, u, v)) return true;
            }
        }
        if (sp == 0) return false;
        loadNode(P, stack[--sp], na, nb, tc);
    }
}

MRT_DEV bool traceAny(const MrtFrameParams& P, float3 o, float3 d, float tMax, bool& ok, TraversalCounters& tc) {
    if (P.instanceCount == 0) return false;  // empty scene
    const float3 inv = safeInv(d);
    uint32_t stack[MRT_TLAS_STACK];
    int sp = 0;
    float4 na, nb;
    loadNode(P, P.tlasRoot, na, nb, tc);
    if (!(slabNode(na, nb, o, inv, tMax) < __int_as_float(0x7f800000))) return false;
    uint32_t visits = 0;
    for (;;) {
        if (++visits > MRT_MAX_VISITS) { ok = false; return false; }
        const uint32_t packed = __float_as_uint(nb.w);
        const uint32_t first = __float_as_uint(na.w);
        const uint32_t count = packed >> 2;
        if (count == 0) {
            float4 a0, b0, a1, b1;
            loadNode(P, first, a0, b0, tc);
            loadNode(P, first + 1, a1, b1, tc);
            const bool h0 = slabNode(a0, b0, o, inv, tMax) < __int_as_float(0x7f800000);
            const bool h1 = slabNode(a1, b1, o, inv, tMax) < __int_as_float(0x7f800000);
            if (h0 && h1) {
                if (sp < MRT_TLAS_STACK) stack[sp++] = first + 1;
                else ok = false;
            }
            if (h0 || h1) {
                na = h0 ? a0 : a1;
                nb = h0 ? b0 : b1;
                continue;
            }
        } else {
            for (uint32_t i = 0; i < count; ++i) {
                if (first + i >= P.instanceCount) {
                    tc.bad = true;
                    break;
                }
                const MrtInstance* in = P.instances + first + i;
                const float3 oo = xformPoint(in->w2o, o), dd = xformDir(in->w2o, d);
                if (anyBlas(P, in->blasRoot, oo, dd, tMax, ok, tc)) return true;
            }
        }
        if (sp == 0) return false;
        loadNode(P, stack[--sp], na, nb, tc);
    }
}
