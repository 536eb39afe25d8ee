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
//     triangles of a node are tested before descending; TLAS and BLAS share
//     one loop and one stack;
//   - a conservative slab test: box planes are exact reals on a power-of-two
//     grid and every rounding of the slab arithmetic is covered by a margin
//     derived per node (see slabAxis), so no child box the ray really
//     enters is culled (the reference's exact-comparison slab test,
//     intersect.glsl:10-18, has no such margin);
//   - every instance is traced: TLAS leaves hold one instance each (the
//     reference can build a 2-instance TLAS leaf, Bvh.cpp:104, and then
//     enters only its first instance, intersect.glsl:116-121, 150-152);
//   - stacks are bounded and an overflow sets an error flag instead of
//     writing out of bounds; node, triangle and instance indices are checked.
#pragma once

#include "../common/device_types.h"
#include "vec.cuh"

#define MRT_EPS_RAY 1e-4f

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

// a * b - c * d by Kahan's algorithm: w = c d rounded, e = w - c d exactly
// (one FMA), result = (a b - w) + e. Its error is at most 2 ulp (Jeannerod,
// Louvet and Muller, Math. Comp. 2013), so the sign is exact and the result
// is zero exactly when a b = c d. Single precision throughout.
MRT_DEV float diffOfProducts(float a, float b, float c, float d) {
    const float w = __fmul_rn(c, d);
    const float e = __fmaf_rn(-c, d, w);
    const float f = __fmaf_rn(a, b, -w);
    return __fadd_rn(f, e);
}

// Watertight test (Woop et al. 2013). Accepts t in (1e-4, tMax); both faces.
// The edge functions use explicit round-to-nearest products with no fused
// multiply-add, so an edge shared by two triangles evaluates to exactly
// opposite values from both sides. When one of them rounds to zero they are
// re-evaluated with correctly signed differences of products, so a ray on
// an edge is decided by the exact sign of every edge function.
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
    if (U == 0.0f || V == 0.0f || W == 0.0f) {  // exactly signed fallback on an edge
        U = diffOfProducts(Cx, By, Cy, Bx);
        V = diffOfProducts(Ax, Cy, Ay, Cx);
        W = diffOfProducts(Bx, Ay, By, Ax);
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
#ifdef MRT_TRAV_PROFILE
    // Warp-step statistics, counted by lane 0 of each warp (a build with
    // MRT_TRAV_PROFILE defined only): steps, lanes with a ray, triangle-phase
    // steps, pairs and rounds, node-phase steps and lanes testing a node.
    uint32_t steps = 0, activeLanes = 0, triSteps = 0, triPairs = 0, triRounds = 0, nodeSteps = 0, nodeLanes = 0;
#endif
};

// Child-hit masks of one wide node.
struct WideGroup {
    uint32_t childBase;  // first internal child node
    uint32_t primBase;   // first leaf primitive
    uint32_t nodeBits;   // bits 24-31: internal children hit (ray-ordered), bits 0-7: internal slot mask
    uint32_t primBits;   // bits 0-23: leaf primitives hit, relative to primBase
};

// Slab offsets of one node axis for one ray. The planes of the axis are the
// exact reals P_q = p + q*s (s = 2^(e-127), q = 0..255); the ray meets P_q at
//   t_q = (P_q - o) * inv = F_q * a + c,  F_q = 2^23 + 256 q,
//   a = s * inv / 256 (exact),  c = (p - o) * inv - 2^23 * a,
// one byte permute and one FMA per plane in the child loop. The float
// evaluation of t_q differs from the real value by less than
//   2 eps |(p-o) inv| + eps |c| (offsets)  +  2 eps (2^24 |a| + |c|)
// (final rounding and the rounding of inv itself), eps = 2^-24; `err` is 5 eps
// times the sum of the three magnitudes, plus 1e-37 for subnormal a. Near
// planes take c - err and far planes c + err, so the computed entry never
// exceeds the real entry and the computed exit never falls below the real
// exit: no child the ray really enters is culled. Overflow (|inv| = 1e30 on
// a huge node) yields inf or NaN, and the NaN-ignoring min/max treat those
// planes as unbounded, which is again conservative.
MRT_DEV void slabAxis(float p, uint32_t e, float o, float inv, float& a, float& cNear, float& cFar) {
    a = __fmul_rn(__uint_as_float(e << 23), __fmul_rn(inv, 0.00390625f));
    const float b = __fmul_rn(__fsub_rn(p, o), inv);
    const float c = __fmaf_rn(-8388608.0f, a, b);
    const float mag = __fmaf_rn(16777216.0f, fabsf(a), __fadd_rn(fabsf(b), fabsf(c)));
    const float err = __fmaf_rn(mag, 2.9802322e-7f, 1e-37f);
    cNear = __fsub_rn(c, err);
    cFar = __fadd_rn(c, err);
}

// Three-input min / max (PTX ISA 8.8, sm_100+): one instruction each; like
// fminf/fmaxf they return the non-NaN operands' extreme.
MRT_DEV float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
MRT_DEV float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// F_q of byte j of a quantised-plane word: 0x4B0000 | q << 8 = 2^23 + 256 q.
template <int j>
MRT_DEV float planeF(uint32_t w) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7404u | (uint32_t(j) << 4)));
}

// Tests the ray against the eight quantised child boxes of node `idx`
// (record layout in MrtWideNode). Per child: six planes (a byte permute and
// an FMA each), two max, two min, one compare. A hit adds the child's meta bits at its bit index:
// internal children at 24 + (slot XOR oct), so taking bits from the top
// visits the slots the ray reaches first first; leaves at their primitive
// offset. Empty slots have meta 0 and add nothing.
MRT_DEV WideGroup intersectWide(const MrtFrameParams& P, uint32_t idx, float3 o, float3 inv, uint32_t oct, float tMax,
                                TraversalCounters& tc) {
    if (idx >= P.nodeCount) {
        tc.bad = true;
        idx = 0;
    }
    const float4* q = reinterpret_cast<const float4*>(P.nodes + idx);
    const float4 q0 = ldg4(q), q1 = ldg4(q + 1), q2 = ldg4(q + 2), q3 = ldg4(q + 3), q4 = ldg4(q + 4);
    tc.nodes++;
    const uint32_t eb = __float_as_uint(q0.w);
    float ax, nx, fx, ay, ny, fy, az, nz, fz;
    slabAxis(q0.x, eb & 0xffu, o.x, inv.x, ax, nx, fx);
    slabAxis(q0.y, (eb >> 8) & 0xffu, o.y, inv.y, ay, ny, fy);
    slabAxis(q0.z, (eb >> 16) & 0xffu, o.z, inv.z, az, nz, fz);
    // a negative reciprocal makes the hi plane the near one
    const bool swx = inv.x < 0.0f, swy = inv.y < 0.0f, swz = inv.z < 0.0f;
    // tolerance of the triangle test's t against the box exit (the reference
    // accepts hits by its own t, so a box must not be culled at the margin)
    const float tMaxF = __fmul_rn(tMax, 1.000001f);
    const uint32_t oct4 = oct * 0x01010101u;
    uint32_t hits = 0;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const uint32_t lx = __float_as_uint(half ? q2.y : q2.x), ly = __float_as_uint(half ? q2.w : q2.z);
        const uint32_t lz = __float_as_uint(half ? q3.y : q3.x), hx = __float_as_uint(half ? q3.w : q3.z);
        const uint32_t hy = __float_as_uint(half ? q4.y : q4.x), hz = __float_as_uint(half ? q4.w : q4.z);
        const uint32_t wnx = swx ? hx : lx, wfx = swx ? lx : hx;
        const uint32_t wny = swy ? hy : ly, wfy = swy ? ly : hy;
        const uint32_t wnz = swz ? hz : lz, wfz = swz ? lz : hz;
        // meta of four slots: internal children (low five bits 24..31) get
        // their bit index XORed with the octant; leaves keep their offset
        const uint32_t m4 = __float_as_uint(half ? q1.w : q1.z);
        const uint32_t inner4 = (m4 & (m4 << 1)) & 0x10101010u;
        const uint32_t bitIndex4 = (m4 ^ (oct4 & ((inner4 >> 4) * 0xffu))) & 0x1f1f1f1fu;
        const uint32_t childBits4 = (m4 >> 5) & 0x07070707u;
#define MRT_WIDE_CHILD(j)                                                                                   \
        {                                                                                                   \
            const float tnx = __fmaf_rn(planeF<j>(wnx), ax, nx), tfx = __fmaf_rn(planeF<j>(wfx), ax, fx);  \
            const float tny = __fmaf_rn(planeF<j>(wny), ay, ny), tfy = __fmaf_rn(planeF<j>(wfy), ay, fy);  \
            const float tnz = __fmaf_rn(planeF<j>(wnz), az, nz), tfz = __fmaf_rn(planeF<j>(wfz), az, fz);  \
            const float tEnter = fmaxf(max3f(tnx, tny, tnz), 0.0f);                                        \
            const float tExit = fminf(min3f(tfx, tfy, tfz), tMaxF);                                        \
            if (tEnter <= tExit)                                                                           \
                hits |= __byte_perm(childBits4, 0u, 0x4440u | (j)) << __byte_perm(bitIndex4, 0u, 0x4440u | (j)); \
        }
        MRT_WIDE_CHILD(0)
        MRT_WIDE_CHILD(1)
        MRT_WIDE_CHILD(2)
        MRT_WIDE_CHILD(3)
#undef MRT_WIDE_CHILD
    }
    WideGroup g;
    g.childBase = __float_as_uint(q1.x);
    g.primBase = __float_as_uint(q1.y);
    g.nodeBits = (hits & 0xff000000u) | (eb >> 24);
    g.primBits = hits & 0x00ffffffu;
    return g;
}

// Ray octant for child ordering: bit k set when direction component k > 0.
MRT_DEV uint32_t rayOctant(float3 d) { return (d.x > 0.0f ? 1u : 0u) | (d.y > 0.0f ? 2u : 0u) | (d.z > 0.0f ? 4u : 0u); }

// Node index of the internal child on hit bit b (24..31) of a group.
MRT_DEV uint32_t childIndex(uint32_t childBase, uint32_t imask, uint32_t b, uint32_t oct) {
    const uint32_t slot = (b - 24u) ^ oct;
    return childBase + uint32_t(__popc(imask & ((1u << slot) - 1u)));
}

// Traversal stack entries (node groups), shared by the TLAS and the BLAS
// being walked.
#define MRT_WIDE_STACK 48
// Threads per block of the traversal kernels (a multiple of 32).
#ifndef MRT_TRAV_THREADS
#define MRT_TRAV_THREADS 128
#endif
// Stack entries of a traversal-kernel thread held in shared memory: the
// bottom ones, which hold nearly every walk (the TLAS and one BLAS of an
// 8-wide tree seldom need more); deeper entries go to local memory. Off by
// default: on the 1080p terrain 8 entries (10 KB of shared memory a block)
// measured 1.9% slower per step and 16 entries 2.6% slower than a stack
// wholly in local memory, whose lines L1 caches (the shared-memory carve-out
// takes L1 capacity from the node fetches).
#ifndef MRT_SHARED_STACK
#define MRT_SHARED_STACK 0
#endif

// Traversal state of one ray, advanced one step at a time (travWarpStep), so a
// persistent warp can start a new ray in a lane whose ray has finished while
// the other lanes keep walking. Two-level walk in one loop (reference
// intersect.glsl:88-178): the TLAS's leaf primitives are instances; on an
// instance the TLAS group is parked, the ray is taken into object space and
// the instance's BLAS is walked on top of the same stack; the TLAS group
// resumes when the stack is back at the depth it had on entry.
struct WideTrav {
    float3 wo, wd;      // world-space ray
    float3 o, inv;      // ray of the level being walked
    Shear sh;           // watertight-test constants (BLAS level)
    uint32_t oct;
    WideGroup g, parked;
    uint32_t inst;
    int blasBase;       // stack depth at BLAS entry; -1 while in the TLAS
    int sp;
    uint32_t visits;
    float tMax;
    HitRecord hit;
    uint32_t pendBase, pendBits;  // BLAS leaf hits of the last node, awaiting their triangle tests
    bool ok;            // cleared on a stack overflow or an exhausted visit budget
};
// The stack of node groups lives apart from WideTrav (an array the walk
// indexes dynamically cannot live in registers; kept separate, the scalar
// state stays in registers). Two forms with the same get/set:
// A one-ray-per-thread walk (trace queries): all entries in local memory.
struct LocalStack {
    uint2 e[MRT_WIDE_STACK];
    MRT_DEV uint2 get(int i) const { return e[i]; }
    MRT_DEV void set(int i, uint2 v) { e[i] = v; }
};
// A persistent traversal kernel's thread (blocks of MRT_TRAV_THREADS):
// entries below MRT_SHARED_STACK in the block's shared array, entry i of
// thread t at [i][t] (a warp's 8-byte entries at one depth fill two
// conflict-free wavefronts; at mixed depths the bank is still that of t),
// the rest in local memory. MRT_SHARED_STACK 0 keeps all in local memory.
#if MRT_SHARED_STACK > 0
MRT_DEV uint2 (&travSharedStack())[MRT_SHARED_STACK][MRT_TRAV_THREADS] {
    __shared__ uint2 s[MRT_SHARED_STACK][MRT_TRAV_THREADS];
    return s;
}
struct SplitStack {
    uint2 deep[MRT_WIDE_STACK - MRT_SHARED_STACK];
    MRT_DEV uint2 get(int i) const {
        return i < MRT_SHARED_STACK ? travSharedStack()[i][threadIdx.x] : deep[i - MRT_SHARED_STACK];
    }
    MRT_DEV void set(int i, uint2 v) {
        if (i < MRT_SHARED_STACK) travSharedStack()[i][threadIdx.x] = v;
        else deep[i - MRT_SHARED_STACK] = v;
    }
};
#else
typedef LocalStack SplitStack;
#endif

MRT_DEV void travBegin(const MrtFrameParams& P, WideTrav& T, float3 o, float3 d, float tMax) {
    T.wo = o;
    T.wd = d;
    T.o = o;
    T.inv = safeInv(d);
    T.oct = rayOctant(d);
    T.sh = Shear{0, 1, 2, 0.0f, 0.0f, 0.0f};
    // a group whose only hit is the root; none in an empty scene (the TLAS
    // root is then a placeholder)
    T.g = WideGroup{P.tlasRoot, 0u, P.instanceCount ? 0x80000000u : 0u, 0u};
    T.parked = WideGroup{0u, 0u, 0u, 0u};
    T.inst = 0;
    T.blasBase = -1;
    T.sp = 0;
    T.visits = 0;
    T.tMax = tMax;
    T.hit.t = tMax;
    T.hit.u = T.hit.v = 0.0f;
    T.hit.tri = 0xffffffffu;
    T.hit.inst = 0;
    T.pendBase = T.pendBits = 0;
    T.ok = true;
}

enum { kTravRunning = 0, kTravDone = 1, kTravOccluded = 2 };

// Node step of one lane with no triangles pending: bookkeeping (instance
// entry, return to the TLAS, stack pops) until the lane has a node to test,
// then one node test. The BLAS leaf hits of that node become the lane's
// pending triangles; TLAS leaf hits (instances) stay in the group and are
// entered on the next step. Returns kTravDone when the walk is over.
// The node test sits after the bookkeeping loop, not inside it: lanes that
// pop first and lanes whose group still holds a child meet before the test,
// so a warp runs it once per step rather than once per loop trip.
template <class Stack>
MRT_DEV int travNodeStep(const MrtFrameParams& P, WideTrav& T, Stack& stack, TraversalCounters& tc) {
    for (;;) {
        if (T.g.primBits) {  // instances (BLAS leaf hits never stay in the group)
            const uint32_t b = uint32_t(__ffs(T.g.primBits) - 1);
            T.g.primBits &= T.g.primBits - 1u;
            const uint32_t instIdx = T.g.primBase + b;
            if (instIdx >= P.instanceCount) {
                tc.bad = true;
                continue;
            }
            const MrtInstance* in = P.instances + instIdx;
            T.parked = T.g;
            T.blasBase = T.sp;
            T.inst = instIdx;
            T.o = xformPoint(in->w2o, T.wo);
            const float3 d = xformDir(in->w2o, T.wd);
            T.inv = safeInv(d);
            T.oct = rayOctant(d);
            T.sh = makeShear(d);
            T.g = WideGroup{in->blasRoot, 0u, 0x80000000u, 0u};
            continue;
        }
        if (T.g.nodeBits & 0xff000000u) break;
        if (T.sp == T.blasBase) {  // BLAS finished: resume the parked TLAS group
            T.g = T.parked;
            T.blasBase = -1;
            T.o = T.wo;
            T.inv = safeInv(T.wd);
            T.oct = rayOctant(T.wd);
            continue;
        }
        if (T.sp == 0) return kTravDone;
        const uint2 e = stack.get(--T.sp);
        T.g.childBase = e.x;
        T.g.nodeBits = e.y;
        T.g.primBits = 0;
    }
    if (++T.visits > P.maxVisits) {
        T.ok = false;
        return kTravDone;
    }
    const uint32_t b = 31u - uint32_t(__clz(T.g.nodeBits & 0xff000000u));
    const uint32_t rest = T.g.nodeBits & ~(1u << b);
    const uint32_t child = childIndex(T.g.childBase, T.g.nodeBits & 0xffu, b, T.oct);
    if (rest & 0xff000000u) {
        if (T.sp < MRT_WIDE_STACK) stack.set(T.sp++, make_uint2(T.g.childBase, rest));
        else T.ok = false;
    }
    T.g = intersectWide(P, child, T.o, T.inv, T.oct, T.tMax, tc);
    if (T.blasBase >= 0 && T.g.primBits) {
        T.pendBase = T.g.primBase;
        T.pendBits = T.g.primBits;
        T.g.primBits = 0;
    }
    return kTravRunning;
}

// Triangle step: the lane's pending triangles. kAny: kTravOccluded at the
// first triangle with t in (1e-4, tMax). Otherwise closest hit: T.tMax and
// T.hit updated.
template <bool kAny>
MRT_DEV int travTriStep(const MrtFrameParams& P, WideTrav& T, TraversalCounters& tc) {
    while (T.pendBits) {
        const uint32_t b = uint32_t(__ffs(T.pendBits) - 1);
        T.pendBits &= T.pendBits - 1u;
        const uint32_t tri = T.pendBase + b;
        ++tc.tris;
        if (tri >= P.triCount) {
            tc.bad = true;
            continue;
        }
        float t, u, v;
        if (hitTriangle(P.triVerts, tri, T.o, T.sh, T.tMax, t, u, v)) {
            if (kAny) {
                T.pendBits = 0;
                return kTravOccluded;
            }
            T.tMax = t;
            T.hit.t = t;
            T.hit.u = u;
            T.hit.v = v;
            T.hit.tri = tri;
            T.hit.inst = T.inst;
        }
    }
    return kTravRunning;
}

// Warp-wide triangle phase: every pending (ray, triangle) pair of the warp
// is tested, 32 pairs a round, one per lane, whichever lane owns the ray, so
// lanes without triangles of their own (or without a ray) work too. Pairs
// are numbered owner by owner in lane order and, within an owner, in
// ascending triangle order; a lane finds the owner of its pair by a binary
// search over the lanes' inclusive pair counts and takes the owner's ray
// constants by shuffles. Closest hit: each hit is folded into its owner's
// slot with a 64-bit shared-memory minimum of (t bits << 32 | triangle);
// t > 0, so the bits order as the values, and the minimum is the nearest
// hit with the lowest triangle index among equal t -- exactly the hit the
// owner's own ascending scan with a shrinking tMax would keep, so results
// are bit-identical to it. The winner's barycentrics follow through a
// second slot written by the lane whose key equals the minimum. Any hit
// (kAny): a warp-wide OR of the owners with a hit. Returns the lane's
// kTrav* state; every pending lane ends with no triangles pending. In a
// one-launch batch (kMulti) lanes may walk different jobs' scenes: a
// lane's `P` is its own job's parameters, and a pair's triangles are read
// from its owner's job (jobs[owner's job]).
template <bool kAny, bool kMulti = false>
MRT_DEV int travTriPhaseWarp(const MrtFrameParams& P, WideTrav& T, TraversalCounters& tc, bool pending,
                             const MrtBatchJob* jobs = nullptr, uint32_t job = 0u) {
    __shared__ unsigned long long sKey[MRT_TRAV_THREADS / 32][32];
    __shared__ float2 sUV[MRT_TRAV_THREADS / 32][32];
    const uint32_t full = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t bits = pending ? T.pendBits : 0u;
    uint32_t incl = uint32_t(__popc(bits));
#pragma unroll
    for (uint32_t off = 1; off < 32; off <<= 1) {
        const uint32_t v = __shfl_up_sync(full, incl, off);
        if (lane >= off) incl += v;
    }
    const uint32_t total = __shfl_sync(full, incl, 31);
    if (!kAny) sKey[warp][lane] = ~0ull;
    __syncwarp();
    const uint32_t kpack = uint32_t(T.sh.kx) | (uint32_t(T.sh.ky) << 2) | (uint32_t(T.sh.kz) << 4);
    uint32_t occ = 0;  // kAny: bit o set when a pair of owner o hit
    for (uint32_t first = 0; first < total; first += 32) {
        const uint32_t k = first + lane;
        // owner o: the first lane whose inclusive count exceeds k
        uint32_t o = 0;
#pragma unroll
        for (uint32_t step = 16; step > 0; step >>= 1)
            if (__shfl_sync(full, incl, o + step - 1) <= k) o += step;
        const uint32_t ob = __shfl_sync(full, bits, o);
        const uint32_t oi = __shfl_sync(full, incl, o);
        const uint32_t obase = __shfl_sync(full, T.pendBase, o);
        const uint32_t okp = __shfl_sync(full, kpack, o);
        const float3 oo = f3(__shfl_sync(full, T.o.x, o), __shfl_sync(full, T.o.y, o), __shfl_sync(full, T.o.z, o));
        Shear sh;
        sh.kx = int(okp & 3u);
        sh.ky = int((okp >> 2) & 3u);
        sh.kz = int((okp >> 4) & 3u);
        sh.sx = __shfl_sync(full, T.sh.sx, o);
        sh.sy = __shfl_sync(full, T.sh.sy, o);
        sh.sz = __shfl_sync(full, T.sh.sz, o);
        const float otMax = __shfl_sync(full, T.tMax, o);
        const float4* triVerts = P.triVerts;
        uint32_t triCount = P.triCount;
        if (kMulti) {
            const MrtFrameParams& Po = jobs[__shfl_sync(full, job, o)].params;
            triVerts = Po.triVerts;
            triCount = Po.triCount;
        }
        bool hit = false;
        unsigned long long key = 0;
        float u = 0.0f, v = 0.0f;
        if (k < total) {
            // the pair is bit number (k - first pair of o) among o's pending bits
            const uint32_t nth = k - (oi - uint32_t(__popc(ob)));
            const uint32_t tri = obase + __fns(ob, 0u, int(nth) + 1);
            ++tc.tris;
            if (tri >= triCount) {
                tc.bad = true;
            } else {
                float t;
                hit = hitTriangle(triVerts, tri, oo, sh, otMax, t, u, v);
                if (hit) {
                    if (kAny) {
                        occ |= 1u << o;
                    } else {
                        key = (uint64_t(__float_as_uint(t)) << 32) | tri;
                        atomicMin(&sKey[warp][o], key);
                    }
                }
            }
        }
        if (!kAny) {
            __syncwarp();
            if (hit && sKey[warp][o] == key) sUV[warp][o] = make_float2(u, v);
        }
    }
    __syncwarp();
    // every lane takes part in the reduction (a full-mask warp operation)
    // before any lane leaves
    const uint32_t occAll = kAny ? __reduce_or_sync(full, occ) : 0u;
    if (!pending) return kTravRunning;
    T.pendBits = 0;
    if (kAny) return (occAll >> lane) & 1u ? kTravOccluded : kTravRunning;
    const unsigned long long best = sKey[warp][lane];
    if (best != ~0ull) {
        const float t = __uint_as_float(uint32_t(best >> 32));
        const float2 uv = sUV[warp][lane];
        T.tMax = t;
        T.hit.t = t;
        T.hit.u = uv.x;
        T.hit.v = uv.y;
        T.hit.tri = uint32_t(best);
        T.hit.inst = T.inst;
    }
    return kTravRunning;
}

// One warp-wide traversal step; every lane of the warp calls it, `active`
// lanes advance their ray. Triangle tests are batched across the warp
// (after Ylitie et al. 2017, section 4): a lane whose node test found leaf
// triangles waits with them pending, and the warp runs a triangle phase
// (travTriPhaseWarp) once at least MRT_TRI_PHASE_PCT percent of its active
// lanes have triangles pending, or no lane has node work left; otherwise
// lanes without pending triangles test one node each. Returns the lane's
// kTrav* state.
#ifndef MRT_TRI_PHASE_PCT
#define MRT_TRI_PHASE_PCT 25
#endif
// The same threshold for any-hit (shadow) walks, which end at their first
// hit and so may prefer another balance of node and triangle work.
#ifndef MRT_TRI_PHASE_PCT_ANY
#define MRT_TRI_PHASE_PCT_ANY MRT_TRI_PHASE_PCT
#endif
template <bool kAny, bool kMulti = false, class Stack>
MRT_DEV int travWarpStep(const MrtFrameParams& P, WideTrav& T, Stack& stack, TraversalCounters& tc,
                         bool active, const MrtBatchJob* jobs = nullptr, uint32_t job = 0u) {
    const bool pending = active && T.pendBits != 0;
    const uint32_t pendLanes = __popc(__ballot_sync(0xffffffffu, pending));
    const uint32_t activeLanes = __popc(__ballot_sync(0xffffffffu, active));
    const uint32_t pct = kAny ? MRT_TRI_PHASE_PCT_ANY : MRT_TRI_PHASE_PCT;
    const bool triPhase = pendLanes * 100u >= activeLanes * pct || pendLanes == activeLanes;
#ifdef MRT_TRAV_PROFILE
    {
        const uint32_t pairs = __reduce_add_sync(0xffffffffu, pending ? uint32_t(__popc(T.pendBits)) : 0u);
        if ((threadIdx.x & 31u) == 0) {
            ++tc.steps;
            tc.activeLanes += activeLanes;
            if (triPhase) {
                ++tc.triSteps;
                tc.triPairs += pairs;
                tc.triRounds += (pairs + 31u) / 32u;
            } else {
                ++tc.nodeSteps;
                tc.nodeLanes += activeLanes - pendLanes;
            }
        }
    }
#endif
    if (triPhase) return travTriPhaseWarp<kAny, kMulti>(P, T, tc, pending, jobs, job);
    return active && !pending ? travNodeStep(P, T, stack, tc) : kTravRunning;
}

// The same walk for one ray on its own (trace queries).
template <bool kAny>
MRT_DEV int travRun(const MrtFrameParams& P, WideTrav& T, LocalStack& stack, TraversalCounters& tc) {
    for (;;) {
        const int r = T.pendBits ? travTriStep<kAny>(P, T, tc) : travNodeStep(P, T, stack, tc);
        if (r != kTravRunning) return r;
    }
}

// Closest hit over the scene; t and barycentrics of the winner re-evaluated
// with the reference's arithmetic. Returns false on a traversal error.
MRT_DEV bool traceClosest(const MrtFrameParams& P, float3 o, float3 d, float tMax, HitRecord& hit, TraversalCounters& tc) {
    WideTrav T;
    LocalStack stack;
    travBegin(P, T, o, d, tMax);
    travRun<false>(P, T, stack, tc);
    hit = T.hit;
    if (hit.tri != 0xffffffffu) refineHit(P, o, d, hit);
    return T.ok;
}

// Any hit in (1e-4, tMax) (reference intersect.glsl:128-178).
MRT_DEV bool traceAny(const MrtFrameParams& P, float3 o, float3 d, float tMax, bool& ok, TraversalCounters& tc) {
    WideTrav T;
    LocalStack stack;
    travBegin(P, T, o, d, tMax);
    const int r = travRun<true>(P, T, stack, tc);
    ok &= T.ok;
    return r == kTravOccluded;
}
