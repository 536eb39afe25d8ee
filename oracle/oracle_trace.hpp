// ORACLE -- test infrastructure only. Not part of the product library.
//
// CPU restatement of the reference path-tracing shaders, line by line:
//   random.glsl:6-31     pcg4d counter RNG, rngInit / rng1 / rng2
//   common.glsl:90-100   luminance, maxComp, Duff et al. 2017 ONB
//   intersect.glsl:10-178 slab test, Moeller-Trumbore, two-level BVH2 walk,
//                         shadow any-hit walk
//   bsdf.glsl:29-192     "Disney-lite" Lambert + GGX (VNDF) + Walter transmission
//   lights.glsl:11-140   equirect mapping, env pdf / CDF sampling, one-light NEE
//   pathtrace.comp:39-233 surface reconstruction, bounce loop, MIS, RR,
//                         firefly clamp, NaN guard, accumulation
//   resolve.comp:13-56   exposure, ACES (Narkowicz), sRGB encode
// T = float reproduces the shader's FP32 arithmetic (parity mode); T = double
// evaluates the same sampling decisions in FP64 (converged-image oracle).
// Texture lookups are bilinear at LOD 0 with REPEAT addressing
// (reference GpuContext.cpp:190-198 sampler; compute shaders sample LOD 0).
#pragma once

#include <cmath>
#include <cstdint>

#include "../miniraytrace_b200/csrc/common/detmath.h"
#include "oracle_scene.hpp"

namespace orc {

// GLSL sin/cos/atan/acos. FP32 mode uses the deterministic implementations
// of detmath.h (the GLSL builtins' precision is implementation-defined; these
// are within 1-3 ulp and evaluate identically on CPU and GPU); FP64 mode uses
// libm.
inline void msincos(float x, float& s, float& c) { detm::sincos(x, &s, &c); }
inline void msincos(double x, double& s, double& c) {
    s = std::sin(x);
    c = std::cos(x);
}
inline float matan2(float y, float x) { return detm::atan2(y, x); }
inline double matan2(double y, double x) { return std::atan2(y, x); }
inline float macos(float x) { return detm::acos(x); }
inline double macos(double x) { return std::acos(x); }

// ---- random.glsl:6-31 -------------------------------------------------------
struct U4 {
    uint32_t x, y, z, w;
};
inline U4 pcg4d(U4 v) {
    v.x = v.x * 1664525u + 1013904223u;
    v.y = v.y * 1664525u + 1013904223u;
    v.z = v.z * 1664525u + 1013904223u;
    v.w = v.w * 1664525u + 1013904223u;
    v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
    v.x ^= v.x >> 16u; v.y ^= v.y >> 16u; v.z ^= v.z >> 16u; v.w ^= v.w >> 16u;
    v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
    return v;
}
struct Rng {
    U4 s;
};
inline Rng rngInit(uint32_t px, uint32_t py, uint32_t frame) { return Rng{{px, py, frame, 0u}}; }
// float(u) rounds to nearest, so a draw can be exactly 1.0 in FP32.
template <class T> inline T u32ToUnit(uint32_t u) {
    return T(u) * T(1.0 / 4294967296.0);
}
template <class T> inline T rng1(Rng& r) {
    r.s.w++;
    return u32ToUnit<T>(pcg4d(r.s).x);
}
template <class T> inline V2<T> rng2(Rng& r) {
    r.s.w++;
    const U4 v = pcg4d(r.s);
    return V2<T>(u32ToUnit<T>(v.x), u32ToUnit<T>(v.y));
}

template <class T> struct C {
    static constexpr T PI = T(3.14159265358979323846);
    static constexpr T TWO_PI = T(6.28318530717958647692);
    static constexpr T INV_PI = T(0.31830988618379067154);
    static constexpr T EPS_RAY = T(1e-4);
};

template <class T> inline V3<T> cv(const V3<float>& v) { return V3<T>(T(v.x), T(v.y), T(v.z)); }
template <class T> inline V3<T> cv(const V4<float>& v) { return V3<T>(T(v.x), T(v.y), T(v.z)); }

// common.glsl:94-100
template <class T> inline void buildOnb(V3<T> n, V3<T>& t, V3<T>& b) {
    const T s = n.z >= T(0) ? T(1) : T(-1);
    const T a = T(-1) / (s + n.z);
    const T c = n.x * n.y * a;
    t = V3<T>(T(1) + s * n.x * n.x * a, s * c, -s * n.x);
    b = V3<T>(c, s + n.y * n.y * a, -n.y);
}

// ---- textures -----------------------------------------------------------------
// sRGB decode of an 8-bit channel (the sampler's SRGB format conversion):
// c <= 0.04045 ? c / 12.92 : ((c + 0.055) / 1.055)^2.4, power in double.
inline float srgbToLinear(float c) {
    return c <= 0.04045f ? c / 12.92f : float(std::pow(double((c + 0.055f) / 1.055f), 2.4));
}
inline V4<float> texel(const TextureData& t, int64_t x, int64_t y) {
    const size_t i = size_t(y) * t.w + size_t(x);
    if (t.format == MRT_TEX_RGBA32F) {
        const float* p = reinterpret_cast<const float*>(t.data.data()) + i * 4;
        return V4<float>(p[0], p[1], p[2], p[3]);
    }
    const uint8_t* p = t.data.data() + i * 4;
    V4<float> c(p[0] / 255.0f, p[1] / 255.0f, p[2] / 255.0f, p[3] / 255.0f);
    if (t.format == MRT_TEX_RGBA8_SRGB) {
        c.x = srgbToLinear(c.x);
        c.y = srgbToLinear(c.y);
        c.z = srgbToLinear(c.z);
    }
    return c;
}
// Bilinear, LOD 0, REPEAT in u and v. Returns RGBA in T.
template <class T> inline V4<T> sampleBilinear(const TextureData& tex, T u, T v) {
    if (tex.data.empty()) return V4<T>(T(1), T(1), T(1), T(1));  // white dummy slot
    const T fx = u * T(tex.w) - T(0.5), fy = v * T(tex.h) - T(0.5);
    const T x0f = std::floor(fx), y0f = std::floor(fy);
    const T ax = fx - x0f, ay = fy - y0f;
    auto wrap = [](int64_t i, int64_t n) { return ((i % n) + n) % n; };
    const int64_t x0 = wrap(int64_t(x0f), tex.w), x1 = wrap(int64_t(x0f) + 1, tex.w);
    const int64_t y0 = wrap(int64_t(y0f), tex.h), y1 = wrap(int64_t(y0f) + 1, tex.h);
    const V4<float> t00 = texel(tex, x0, y0), t10 = texel(tex, x1, y0);
    const V4<float> t01 = texel(tex, x0, y1), t11 = texel(tex, x1, y1);
    auto lerp2 = [&](float a, float b, float c, float d) {
        return (T(1) - ax) * (T(1) - ay) * T(a) + ax * (T(1) - ay) * T(b) + (T(1) - ax) * ay * T(c) +
               ax * ay * T(d);
    };
    return V4<T>(lerp2(t00.x, t10.x, t01.x, t11.x), lerp2(t00.y, t10.y, t01.y, t11.y),
                 lerp2(t00.z, t10.z, t01.z, t11.z), lerp2(t00.w, t10.w, t01.w, t11.w));
}

// ---- ray / hit (common.glsl:80-88) -----------------------------------------------
template <class T> struct Ray {
    V3<T> origin, dir;
    T tMax;
};
template <class T> struct Hit {
    T t;
    uint32_t tri = 0, inst = 0;
    V2<T> bary;
    bool hit = false;
};

template <class T> struct Tracer {
    const Packed& P;
    const Globals& g;
    bool bruteForce = false;  // diagnostic: closest hit by testing every triangle
    bool watertight = false;  // diagnostic: brute force decides with the watertight test
    // Off (the reference): a TLAS leaf enters only instances[leftOrPrim]
    // (intersect.glsl:116-121, 150-152), although Bvh.cpp:104 makes a
    // 2-instance TLAS leaf when SAH prefers it (count <= 2 * maxLeafSize 1);
    // the second instance of such a leaf is never traversed. On: every
    // instance of the leaf is entered, which is what the 1-instance TLAS
    // leaves the reference intends (Bvh.hpp:36) would give.
    bool allLeafInstances = false;

    // intersect.glsl:10-18
    T intersectAabb(const BvhNode& n, V3<T> o, V3<T> invDir, T tMax) const {
        const V3<T> lo(T(n.lo[0]), T(n.lo[1]), T(n.lo[2])), hi(T(n.hi[0]), T(n.hi[1]), T(n.hi[2]));
        const V3<T> t0 = (lo - o) * invDir, t1 = (hi - o) * invDir;
        const V3<T> tminv = vmin(t0, t1), tmaxv = vmax(t0, t1);
        const T tEnter = mmax(mmax(tminv.x, tminv.y), mmax(tminv.z, T(0)));
        const T tExit = mmin(mmin(tmaxv.x, tmaxv.y), mmin(tmaxv.z, tMax));
        return tEnter <= tExit ? tEnter : tMax;
    }
    // intersect.glsl:21-45 (Moeller-Trumbore)
    T intersectTriangle(uint32_t tri, V3<T> o, V3<T> d, T tMax, V2<T>& bary) const {
        const uint32_t* t = &P.tris[size_t(tri) * 4];
        const V3<T> v0 = cv<T>(P.positions[t[0]]);
        const V3<T> e1 = cv<T>(P.positions[t[1]]) - v0;
        const V3<T> e2 = cv<T>(P.positions[t[2]]) - v0;
        const V3<T> p = cross(d, e2);
        const T det = dot(e1, p);
        if (std::fabs(det) < T(1e-12)) return T(-1);
        const T invDet = T(1) / det;
        const V3<T> s = o - v0;
        const T u = dot(s, p) * invDet;
        if (u < T(0) || u > T(1)) return T(-1);
        const V3<T> q = cross(s, e1);
        const T v = dot(d, q) * invDet;
        if (v < T(0) || u + v > T(1)) return T(-1);
        const T tt = dot(e2, q) * invDet;
        if (tt <= C<T>::EPS_RAY || tt >= tMax) return T(-1);
        bary = V2<T>(u, v);
        return tt;
    }
    // intersect.glsl:48-86
    void traverseBlas(uint32_t root, uint32_t inst, V3<T> o, V3<T> d, T& tMax, Hit<T>& hit) const {
        const V3<T> invDir = V3<T>(T(1)) / d;
        uint32_t stack[64];
        int sp = 0;
        stack[sp++] = root;
        while (sp > 0) {
            const BvhNode& n = P.nodes[stack[--sp]];
            if (intersectAabb(n, o, invDir, tMax) >= tMax) continue;
            const uint32_t count = n.packed >> 2;
            if (count == 0) {
                const uint32_t axis = n.packed & 3u;
                uint32_t nearC = n.leftOrPrim, farC = n.leftOrPrim + 1;
                if (d[int(axis)] < T(0)) std::swap(nearC, farC);
                stack[sp++] = farC;
                stack[sp++] = nearC;
            } else {
                for (uint32_t i = 0; i < count; ++i) {
                    V2<T> b;
                    const T t = intersectTriangle(n.leftOrPrim + i, o, d, tMax, b);
                    if (t > T(0)) {
                        tMax = t;
                        hit.t = t;
                        hit.tri = n.leftOrPrim + i;
                        hit.inst = inst;
                        hit.bary = b;
                        hit.hit = true;
                    }
                }
            }
        }
    }
    // intersect.glsl:88-125
    Hit<T> traceRay(const Ray<T>& ray) const {
        if (bruteForce) return traceBrute(ray);
        Hit<T> hit;
        hit.hit = false;
        hit.t = ray.tMax;
        T tMax = ray.tMax;
        const V3<T> invDir = V3<T>(T(1)) / ray.dir;
        uint32_t stack[64];
        int sp = 0;
        stack[sp++] = g.tlasRoot;
        while (sp > 0) {
            const BvhNode& n = P.nodes[stack[--sp]];
            if (intersectAabb(n, ray.origin, invDir, tMax) >= tMax) continue;
            const uint32_t count = n.packed >> 2;
            if (count == 0) {
                const uint32_t axis = n.packed & 3u;
                uint32_t nearC = n.leftOrPrim, farC = n.leftOrPrim + 1;
                if (ray.dir[int(axis)] < T(0)) std::swap(nearC, farC);
                stack[sp++] = farC;
                stack[sp++] = nearC;
            } else {
                const uint32_t walked = allLeafInstances ? count : 1u;
                for (uint32_t k = 0; k < walked; ++k) {
                    const GpuInstance& in = P.instances[n.leftOrPrim + k];
                    const V3<T> oObj = wToO(in, ray.origin, true), dObj = wToO(in, ray.dir, false);
                    traverseBlas(in.blasRoot, n.leftOrPrim + k, oObj, dObj, tMax, hit);
                }
            }
        }
        return hit;
    }
    // Every triangle of every instance, instances and triangles in packed
    // order, keeping the first strictly closest hit.
    Hit<T> traceBrute(const Ray<T>& ray) const {
        Hit<T> hit;
        hit.hit = false;
        hit.t = ray.tMax;
        T tMax = ray.tMax;
        for (uint32_t ii = 0; ii < P.instances.size(); ++ii) {
            const GpuInstance& in = P.instances[ii];
            const V3<T> oObj = wToO(in, ray.origin, true), dObj = wToO(in, ray.dir, false);
            // the BLAS covers a contiguous triangle range: walk its leaves
            uint32_t stack[64];
            int sp = 0;
            stack[sp++] = in.blasRoot;
            while (sp > 0) {
                const BvhNode& n = P.nodes[stack[--sp]];
                const uint32_t count = n.packed >> 2;
                if (count == 0) {
                    stack[sp++] = n.leftOrPrim;
                    stack[sp++] = n.leftOrPrim + 1;
                    continue;
                }
                for (uint32_t i = 0; i < count; ++i) {
                    V2<T> b;
                    const T t = watertight ? intersectWatertight(n.leftOrPrim + i, oObj, dObj, tMax, b)
                                           : intersectTriangle(n.leftOrPrim + i, oObj, dObj, tMax, b);
                    if (t > T(0)) {
                        tMax = t;
                        hit.t = t;
                        hit.tri = n.leftOrPrim + i;
                        hit.inst = ii;
                        hit.bary = b;
                        hit.hit = true;
                    }
                }
            }
        }
        if (watertight && hit.hit) {  // report t/bary with the reference formula
            const GpuInstance& in = P.instances[hit.inst];
            V2<T> b;
            const T t = intersectTriangle(hit.tri, wToO(in, ray.origin, true), wToO(in, ray.dir, false),
                                          hit.t * T(1.0001), b);
            if (t > T(0)) {
                hit.t = t;
                hit.bary = b;
            }
        }
        return hit;
    }
    // a * b - c * d by Kahan's algorithm (rounded product, its exact error by
    // one fused multiply-add, then the sum): within 2 ulp (Jeannerod, Louvet
    // and Muller 2013), so its sign is exact.
    static T diffOfProducts(T a, T b, T c, T d) {
        const T w = c * d;
        const T e = std::fma(-c, d, w);
        const T f = std::fma(a, b, -w);
        return f + e;
    }
    // Woop, Benthin and Wald 2013 watertight test (diagnostic twin of the
    // GPU kernel's decision), t in (1e-4, tMax).
    T intersectWatertight(uint32_t tri, V3<T> o, V3<T> d, T tMax, V2<T>& bary) const {
        const uint32_t* tr = &P.tris[size_t(tri) * 4];
        const V3<T> A = cv<T>(P.positions[tr[0]]) - o, B = cv<T>(P.positions[tr[1]]) - o,
                    Cc = cv<T>(P.positions[tr[2]]) - o;
        const T ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
        int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
        int kx = kz == 2 ? 0 : kz + 1, ky = kx == 2 ? 0 : kx + 1;
        if (d[kz] < T(0)) std::swap(kx, ky);
        const T sx = d[kx] / d[kz], sy = d[ky] / d[kz], sz = T(1) / d[kz];
        const T Ax = A[kx] - sx * A[kz], Ay = A[ky] - sy * A[kz];
        const T Bx = B[kx] - sx * B[kz], By = B[ky] - sy * B[kz];
        const T Cx = Cc[kx] - sx * Cc[kz], Cy = Cc[ky] - sy * Cc[kz];
        T U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
        if (U == T(0) || V == T(0) || W == T(0)) {  // exactly signed edge functions
            U = diffOfProducts(Cx, By, Cy, Bx);
            V = diffOfProducts(Ax, Cy, Ay, Cx);
            W = diffOfProducts(Bx, Ay, By, Ax);
        }
        if ((U < T(0) || V < T(0) || W < T(0)) && (U > T(0) || V > T(0) || W > T(0))) return T(-1);
        const T det = U + V + W;
        if (det == T(0)) return T(-1);
        const T Tt = U * (sz * A[kz]) + V * (sz * B[kz]) + W * (sz * Cc[kz]);
        const T rcp = T(1) / det;
        const T t = Tt * rcp;
        if (!(t > C<T>::EPS_RAY && t < tMax)) return T(-1);
        bary = V2<T>(V * rcp, W * rcp);
        return t;
    }
    V3<T> wToO(const GpuInstance& in, V3<T> v, bool point) const {
        const auto& m = in.worldToObject.m;
        V3<T> r(T(m[0][0]) * v.x + T(m[1][0]) * v.y + T(m[2][0]) * v.z,
                T(m[0][1]) * v.x + T(m[1][1]) * v.y + T(m[2][1]) * v.z,
                T(m[0][2]) * v.x + T(m[1][2]) * v.y + T(m[2][2]) * v.z);
        if (point) r = V3<T>(r.x + T(m[3][0]), r.y + T(m[3][1]), r.z + T(m[3][2]));
        return r;
    }
    // intersect.glsl:128-178
    bool traceShadowRay(const Ray<T>& ray) const {
        if (bruteForce) return traceBrute(ray).hit;
        const T tMax = ray.tMax;
        const V3<T> invDir = V3<T>(T(1)) / ray.dir;
        uint32_t stack[64];
        int sp = 0;
        stack[sp++] = g.tlasRoot;
        while (sp > 0) {
            const BvhNode& n = P.nodes[stack[--sp]];
            if (intersectAabb(n, ray.origin, invDir, tMax) >= tMax) continue;
            const uint32_t count = n.packed >> 2;
            if (count == 0) {
                stack[sp++] = n.leftOrPrim;
                stack[sp++] = n.leftOrPrim + 1;
            } else {
                const uint32_t walked = allLeafInstances ? count : 1u;
                for (uint32_t k = 0; k < walked; ++k) {
                    const GpuInstance& in = P.instances[n.leftOrPrim + k];
                    const V3<T> oObj = wToO(in, ray.origin, true), dObj = wToO(in, ray.dir, false);
                    const V3<T> invObj = V3<T>(T(1)) / dObj;
                    uint32_t bstack[64];
                    int bsp = 0;
                    bstack[bsp++] = in.blasRoot;
                    while (bsp > 0) {
                        const BvhNode& bn = P.nodes[bstack[--bsp]];
                        if (intersectAabb(bn, oObj, invObj, tMax) >= tMax) continue;
                        const uint32_t bcnt = bn.packed >> 2;
                        if (bcnt == 0) {
                            bstack[bsp++] = bn.leftOrPrim;
                            bstack[bsp++] = bn.leftOrPrim + 1;
                        } else {
                            for (uint32_t i = 0; i < bcnt; ++i) {
                                V2<T> b;
                                if (intersectTriangle(bn.leftOrPrim + i, oObj, dObj, tMax, b) > T(0)) return true;
                            }
                        }
                    }
                }
            }
        }
        return false;
    }

    // ---- bsdf.glsl -----------------------------------------------------------
    struct Bsdf {
        V3<T> baseColor;
        T roughness, metallic, transmission, ior;
        bool entering;
    };
    static T ggxD(V3<T> h, T alpha) {  // bsdf.glsl:29-34
        const T a2 = alpha * alpha;
        const T c2 = h.z * h.z;
        const T d = c2 * (a2 - T(1)) + T(1);
        return a2 / mmax(C<T>::PI * d * d, T(1e-12));
    }
    static T ggxLambda(V3<T> w, T alpha) {  // bsdf.glsl:36-40
        const T c2 = w.z * w.z;
        const T t2 = mmax(T(1) - c2, T(0)) / mmax(c2, T(1e-12));
        return T(0.5) * (std::sqrt(T(1) + alpha * alpha * t2) - T(1));
    }
    static T ggxG1(V3<T> w, T alpha) { return T(1) / (T(1) + ggxLambda(w, alpha)); }
    static T ggxG2(V3<T> wo, V3<T> wi, T alpha) {
        return T(1) / (T(1) + ggxLambda(wo, alpha) + ggxLambda(wi, alpha));
    }
    static V3<T> sampleGgxVndf(V3<T> wo, T alpha, V2<T> u) {  // bsdf.glsl:48-61
        const V3<T> vh = normalize(V3<T>(alpha * wo.x, alpha * wo.y, wo.z));
        const T lensq = vh.x * vh.x + vh.y * vh.y;
        const V3<T> T1 = lensq > T(0) ? V3<T>(-vh.y, vh.x, T(0)) * inversesqrt(lensq) : V3<T>(T(1), T(0), T(0));
        const V3<T> T2 = cross(vh, T1);
        const T r = std::sqrt(u.x);
        const T phi = C<T>::TWO_PI * u.y;
        T sphi, cphi;
        msincos(phi, sphi, cphi);
        const T t1 = r * cphi;
        T t2 = r * sphi;
        const T s = T(0.5) * (T(1) + vh.z);
        t2 = (T(1) - s) * std::sqrt(mmax(T(1) - t1 * t1, T(0))) + s * t2;
        const V3<T> nh = t1 * T1 + t2 * T2 + std::sqrt(mmax(T(1) - t1 * t1 - t2 * t2, T(0))) * vh;
        return normalize(V3<T>(alpha * nh.x, alpha * nh.y, mmax(nh.z, T(1e-6))));
    }
    static V3<T> fresnelSchlick(V3<T> f0, T cosTheta) {  // bsdf.glsl:63-67
        const T m = clampv(T(1) - cosTheta, T(0), T(1));
        const T m2 = m * m;
        return f0 + (V3<T>(T(1)) - f0) * (m2 * m2 * m);
    }
    static T fresnelDielectric(T cosI, T eta) {  // bsdf.glsl:69-77
        cosI = clampv(cosI, T(0), T(1));
        const T sin2T = (T(1) - cosI * cosI) / (eta * eta);
        if (sin2T >= T(1)) return T(1);
        const T cosT = std::sqrt(T(1) - sin2T);
        const T rs = (cosI - eta * cosT) / (cosI + eta * cosT);
        const T rp = (eta * cosI - cosT) / (eta * cosI + cosT);
        return T(0.5) * (rs * rs + rp * rp);
    }
    static V2<T> sampleCosineHemispherePdf(V2<T> u, V3<T>& wi) {  // bsdf.glsl:79-84
        const T r = std::sqrt(u.x);
        const T phi = C<T>::TWO_PI * u.y;
        T sphi, cphi;
        msincos(phi, sphi, cphi);
        wi = V3<T>(r * cphi, r * sphi, std::sqrt(mmax(T(1) - u.x, T(0))));
        return V2<T>(wi.z, wi.z * C<T>::INV_PI);
    }
    static void lobeWeights(const Bsdf& m, V3<T> wo, T& wDiff, T& wSpec, T& wTrans) {  // bsdf.glsl:87-95
        const V3<T> f0 = mix(V3<T>(T(0.04)), m.baseColor, m.metallic);
        wSpec = luminance(fresnelSchlick(f0, std::fabs(wo.z)));
        wDiff = (T(1) - m.metallic) * (T(1) - m.transmission) * luminance(m.baseColor);
        wTrans = (T(1) - m.metallic) * m.transmission;
        T total = wDiff + wSpec + wTrans;
        if (total < T(1e-7)) {
            wDiff = T(1);
            wSpec = T(0);
            wTrans = T(0);
            total = T(1);
        }
        wDiff /= total;
        wSpec /= total;
        wTrans /= total;
    }
    static void bsdfEval(const Bsdf& m, V3<T> wo, V3<T> wi, V3<T>& f, T& pdf) {  // bsdf.glsl:100-144
        f = V3<T>(T(0));
        pdf = T(0);
        const T alpha = mmax(m.roughness * m.roughness, T(1e-3));
        T wDiff, wSpec, wTrans;
        lobeWeights(m, wo, wDiff, wSpec, wTrans);
        const T eta = m.entering ? m.ior : T(1) / m.ior;
        if (wi.z > T(0)) {
            if (wDiff > T(0)) {
                const V3<T> fd = (T(1) - m.metallic) * (T(1) - m.transmission) * m.baseColor * C<T>::INV_PI;
                f += fd * T(1);
                pdf += wDiff * wi.z * C<T>::INV_PI;
            }
            const V3<T> h = normalize(wo + wi);
            const T d = ggxD(h, alpha);
            const T g2 = ggxG2(wo, wi, alpha);
            const V3<T> f0 = mix(V3<T>(T(0.04)), m.baseColor, m.metallic);
            const V3<T> F = fresnelSchlick(f0, dot(wo, h));
            f += d * g2 * F / mmax(T(4) * wo.z * wi.z, T(1e-7));
            pdf += wSpec * ggxG1(wo, alpha) * d / mmax(T(4) * wo.z, T(1e-7));
        } else if (wTrans > T(0)) {
            V3<T> h = normalize(wo + wi * eta);
            if (h.z < T(0)) h = -h;
            const T woH = dot(wo, h);
            const T wiH = dot(wi, h);
            if (woH * wiH < T(0)) {
                const T F = fresnelDielectric(std::fabs(woH), eta);
                const T d = ggxD(h, alpha);
                const T g2 = ggxG2(wo, V3<T>(wi.x, wi.y, -wi.z), alpha);
                T denom = woH + eta * wiH;
                denom = mmax(denom * denom, T(1e-7));
                const T jac = eta * eta * std::fabs(wiH) / denom;
                f += m.baseColor * (T(1) - F) * d * g2 * std::fabs(woH) * jac /
                     mmax(std::fabs(wo.z * wi.z), T(1e-7)) * (T(1) - m.metallic) * m.transmission;
                pdf += wTrans * (T(1) - F) * ggxG1(wo, alpha) * d * std::fabs(woH) / mmax(wo.z, T(1e-7)) * jac;
            }
        }
    }
    struct BsdfSample {
        V3<T> wi, f;
        T pdf;
        bool valid;
    };
    static BsdfSample bsdfSample(const Bsdf& m, V3<T> wo, Rng& rng) {  // bsdf.glsl:147-192
        BsdfSample s{};
        s.valid = false;
        const T alpha = mmax(m.roughness * m.roughness, T(1e-3));
        T wDiff, wSpec, wTrans;
        lobeWeights(m, wo, wDiff, wSpec, wTrans);
        const T eta = m.entering ? m.ior : T(1) / m.ior;
        const T pick = rng1<T>(rng);
        V3<T> wi;
        if (pick < wDiff) {
            V3<T> d;
            sampleCosineHemispherePdf(rng2<T>(rng), d);
            wi = d;
        } else if (pick < wDiff + wSpec) {
            const V3<T> h = sampleGgxVndf(wo, alpha, rng2<T>(rng));
            wi = reflect(-wo, h);
            if (wi.z <= T(0)) return s;
        } else {
            const V3<T> h = sampleGgxVndf(wo, alpha, rng2<T>(rng));
            const T woH = dot(wo, h);
            const T F = fresnelDielectric(std::fabs(woH), eta);
            if (rng1<T>(rng) < F) {
                wi = reflect(-wo, h);
                if (wi.z <= T(0)) return s;
            } else {
                wi = refract(-wo, h, T(1) / eta);
                if (wi.z >= T(0) || length(wi) < T(1e-6)) return s;
                wi = normalize(wi);
            }
        }
        V3<T> f;
        T pdf;
        bsdfEval(m, wo, wi, f, pdf);
        if (pdf < T(1e-9)) return s;
        s.wi = wi;
        s.f = f;
        s.pdf = pdf;
        s.valid = true;
        return s;
    }

    // ---- lights.glsl -------------------------------------------------------------
    V2<T> dirToEquirect(V3<T> d) const {  // lights.glsl:11-15
        const T phi = matan2(d.z, d.x) - T(g.envRotation);
        const T theta = macos(clampv(d.y, T(-1), T(1)));
        return V2<T>(fract(phi / C<T>::TWO_PI + T(1)), theta / C<T>::PI);
    }
    V3<T> equirectToDir(V2<T> uv) const {  // lights.glsl:17-22
        const T phi = uv.x * C<T>::TWO_PI + T(g.envRotation);
        const T theta = uv.y * C<T>::PI;
        T st, ct, sp, cp;
        msincos(theta, st, ct);
        msincos(phi, sp, cp);
        return V3<T>(st * cp, ct, st * sp);
    }
    V3<T> envLookup(V2<T> uv) const {
        const V4<T> c = sampleBilinear<T>(P.env, uv.x, uv.y);
        return V3<T>(c.x, c.y, c.z);
    }
    V3<T> envRadiance(V3<T> dir) const {  // lights.glsl:24-27
        if (!g.hasEnv) return V3<T>(T(0));
        return envLookup(dirToEquirect(dir)) * T(g.envIntensity);
    }
    T envPdf(V3<T> dir) const {  // lights.glsl:30-34
        if (!g.hasEnv) return T(0);
        return luminance(envLookup(dirToEquirect(dir))) / T(g.envIntegral);
    }
    uint32_t searchCdf(uint32_t base, uint32_t count, T u) const {  // lights.glsl:37-45
        uint32_t lo = 0, hi = count - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (T(P.envCdf[base + mid]) < u) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    }
    bool sampleEnv(Rng& rng, V3<T>& dir, V3<T>& rad, T& pdf) const {  // lights.glsl:48-58
        const uint32_t w = g.envW, h = g.envH;
        if (w == 0 || h == 0) return false;
        const uint32_t row = searchCdf(w * h, h, rng1<T>(rng));
        const uint32_t col = searchCdf(row * w, w, rng1<T>(rng));
        const V2<T> uv((T(col) + T(0.5)) / T(w), (T(row) + T(0.5)) / T(h));
        dir = equirectToDir(uv);
        rad = envLookup(uv) * T(g.envIntensity);
        pdf = envPdf(dir);
        return pdf > T(1e-9);
    }
    struct LightSample {
        V3<T> wiWorld, radiance;
        T pdf, dist;
        bool delta, valid;
    };
    LightSample sampleOneLight(V3<T> p, Rng& rng) const {  // lights.glsl:70-134
        LightSample ls{};
        ls.valid = false;
        if (g.lightCount == 0) return ls;
        const uint32_t idx = std::min(uint32_t(rng1<T>(rng) * T(g.lightCount)), g.lightCount - 1);
        const T pickPdf = T(1) / T(g.lightCount);
        const GpuLight& l = P.lights[idx];
        if (l.type == kLightEnv) {
            V3<T> dir, rad;
            T pdf;
            if (!sampleEnv(rng, dir, rad, pdf)) return ls;
            ls.wiWorld = dir;
            ls.radiance = rad;
            ls.pdf = pdf * pickPdf;
            ls.dist = T(1e30);
            ls.delta = false;
            ls.valid = true;
        } else if (l.type == kLightSun) {
            const T cosMax = T(l.p0.w);
            const V2<T> u = rng2<T>(rng);
            const T cosT = mix(T(1), cosMax, u.x);
            const T sinT = std::sqrt(mmax(T(1) - cosT * cosT, T(0)));
            const T phi = C<T>::TWO_PI * u.y;
            V3<T> t, b;
            const V3<T> n = cv<T>(l.p0);
            buildOnb(n, t, b);
            T sphi, cphi;
            msincos(phi, sphi, cphi);
            ls.wiWorld = normalize(t * (sinT * cphi) + b * (sinT * sphi) + n * cosT);
            ls.radiance = cv<T>(l.p1);
            const T conePdf = T(1) / (C<T>::TWO_PI * mmax(T(1) - cosMax, T(1e-7)));
            ls.pdf = conePdf * pickPdf;
            ls.dist = T(1e30);
            ls.delta = true;
            ls.valid = true;
        } else if (l.type == kLightPoint) {
            const V3<T> d = cv<T>(l.p0) - p;
            const T d2 = mmax(dot(d, d), T(1e-8));
            ls.dist = std::sqrt(d2);
            ls.wiWorld = d / ls.dist;
            ls.radiance = cv<T>(l.p1) / d2;
            ls.pdf = pickPdf;
            ls.delta = true;
            ls.valid = true;
        } else {
            const V2<T> u = rng2<T>(rng);
            const V3<T> q = cv<T>(l.p0) + cv<T>(l.p1) * u.x + cv<T>(l.p2) * u.y;
            const V3<T> d = q - p;
            const T d2 = mmax(dot(d, d), T(1e-8));
            ls.dist = std::sqrt(d2);
            ls.wiWorld = d / ls.dist;
            const V3<T> n = normalize(cross(cv<T>(l.p1), cv<T>(l.p2)));
            T cosL = dot(n, -ls.wiWorld);
            if (l.p3.w > 0.5f) cosL = std::fabs(cosL);
            if (cosL < T(1e-6)) return ls;
            const T area = mmax(T(l.p0.w), T(1e-8));
            ls.radiance = cv<T>(l.p3);
            ls.pdf = (d2 / (cosL * area)) * pickPdf;
            ls.delta = true;
            ls.valid = true;
        }
        return ls;
    }
    T envPickPdf() const {  // lights.glsl:137-140
        return (g.hasEnv && g.lightCount > 0) ? T(1) / T(g.lightCount) : T(0);
    }

    // ---- pathtrace.comp ----------------------------------------------------------
    struct Surface {
        V3<T> pos, nGeom, nShade, tangent;
        V2<T> uv;
        bool frontFace;
        const GpuMaterial* mat;
    };
    V3<T> texRgb(int slot, V2<T> uv) const {
        const V4<T> c = sampleBilinear<T>(P.textures[slot], uv.x, uv.y);
        return V3<T>(c.x, c.y, c.z);
    }
    Surface makeSurface(const Ray<T>& ray, const Hit<T>& hit) const {  // pathtrace.comp:39-80
        Surface s;
        const GpuInstance& in = P.instances[hit.inst];
        const uint32_t* tri = &P.tris[size_t(hit.tri) * 4];
        const T b1 = hit.bary.x, b2 = hit.bary.y, b0 = T(1) - b1 - b2;
        const V3<T> p0 = cv<T>(P.positions[tri[0]]), p1 = cv<T>(P.positions[tri[1]]), p2 = cv<T>(P.positions[tri[2]]);
        const V3<T> posObj = b0 * p0 + b1 * p1 + b2 * p2;
        const auto& o2w = in.objectToWorld.m;
        s.pos = V3<T>(T(o2w[0][0]) * posObj.x + T(o2w[1][0]) * posObj.y + T(o2w[2][0]) * posObj.z + T(o2w[3][0]),
                      T(o2w[0][1]) * posObj.x + T(o2w[1][1]) * posObj.y + T(o2w[2][1]) * posObj.z + T(o2w[3][1]),
                      T(o2w[0][2]) * posObj.x + T(o2w[1][2]) * posObj.y + T(o2w[2][2]) * posObj.z + T(o2w[3][2]));
        const auto& w2o = in.worldToObject.m;
        auto nrmMat = [&](V3<T> v) {  // transpose(mat3(worldToObject)) * v
            return V3<T>(T(w2o[0][0]) * v.x + T(w2o[0][1]) * v.y + T(w2o[0][2]) * v.z,
                         T(w2o[1][0]) * v.x + T(w2o[1][1]) * v.y + T(w2o[1][2]) * v.z,
                         T(w2o[2][0]) * v.x + T(w2o[2][1]) * v.y + T(w2o[2][2]) * v.z);
        };
        const V3<T> ngObj = cross(p1 - p0, p2 - p0);
        V3<T> nGeom = normalize(nrmMat(ngObj));
        const V3<T> nObj =
            b0 * cv<T>(P.normals[tri[0]]) + b1 * cv<T>(P.normals[tri[1]]) + b2 * cv<T>(P.normals[tri[2]]);
        V3<T> nShade = normalize(nrmMat(nObj));
        const V2<float>& u0 = P.uvs[tri[0]];
        const V2<float>& u1 = P.uvs[tri[1]];
        const V2<float>& u2 = P.uvs[tri[2]];
        s.uv = V2<T>(b0 * T(u0.x) + b1 * T(u1.x) + b2 * T(u2.x), b0 * T(u0.y) + b1 * T(u1.y) + b2 * T(u2.y));
        const V4<float>& ta = P.tangents[tri[0]];
        const V4<float>& tb = P.tangents[tri[1]];
        const V4<float>& tc = P.tangents[tri[2]];
        const V3<T> tanH = b0 * cv<T>(ta) + b1 * cv<T>(tb) + b2 * cv<T>(tc);
        const T tanW = b0 * T(ta.w) + b1 * T(tb.w) + b2 * T(tc.w);
        const V3<T> tangent = normalize(V3<T>(T(o2w[0][0]) * tanH.x + T(o2w[1][0]) * tanH.y + T(o2w[2][0]) * tanH.z,
                                              T(o2w[0][1]) * tanH.x + T(o2w[1][1]) * tanH.y + T(o2w[2][1]) * tanH.z,
                                              T(o2w[0][2]) * tanH.x + T(o2w[1][2]) * tanH.y + T(o2w[2][2]) * tanH.z));
        s.frontFace = dot(ray.dir, nGeom) < T(0);
        if (!s.frontFace) {
            nGeom = -nGeom;
            nShade = -nShade;
        }
        s.mat = &P.materials[in.materialIndex];
        if (s.mat->tex[3] >= 0) {
            const V3<T> tn = texRgb(s.mat->tex[3], s.uv) * T(2) - V3<T>(T(1));
            const V3<T> bitan = cross(nShade, tangent) * tanW;
            nShade = normalize(tangent * tn.x + bitan * tn.y + nShade * tn.z);
            if (dot(nShade, nGeom) < T(0)) nShade = nGeom;
        }
        s.nGeom = nGeom;
        s.nShade = nShade;
        s.tangent = tangent;
        return s;
    }
    Bsdf makeBsdf(const Surface& s) const {  // pathtrace.comp:82-94
        Bsdf b;
        b.baseColor = cv<T>(s.mat->baseColorOpacity);
        if (s.mat->tex[0] >= 0) b.baseColor = b.baseColor * texRgb(s.mat->tex[0], s.uv);
        b.roughness = T(s.mat->emissionRoughness.w);
        if (s.mat->tex[1] >= 0) b.roughness = b.roughness * texRgb(s.mat->tex[1], s.uv).x;
        b.metallic = T(s.mat->params.x);
        if (s.mat->tex[2] >= 0) b.metallic = b.metallic * texRgb(s.mat->tex[2], s.uv).x;
        b.transmission = T(s.mat->params.y);
        b.ior = T(s.mat->params.z);
        b.entering = s.frontFace;
        return b;
    }
    static T balanceHeuristic(T a, T b) { return a / mmax(a + b, T(1e-12)); }  // pathtrace.comp:96-98

    // One path; returns L after clamp and NaN guard (pathtrace.comp:100-225).
    V3<T> tracePath(uint32_t px, uint32_t py, uint32_t frame) const {
        Rng rng = rngInit(px, py, frame);
        const V2<T> jitter = rng2<T>(rng);
        const V2<T> uv((T(px) + jitter.x) / T(g.width), (T(py) + jitter.y) / T(g.height));
        const T sx = mix(T(g.fl), T(g.fr), uv.x);
        const T sy = mix(T(g.ft), T(g.fb), uv.y);
        Ray<T> ray;
        if (g.ortho) {
            ray.origin = cv<T>(g.camPos) + sx * cv<T>(g.camRight) + sy * cv<T>(g.camUp);
            ray.dir = cv<T>(g.camForward);
        } else {
            ray.origin = cv<T>(g.camPos);
            ray.dir = normalize(cv<T>(g.camForward) + sx * cv<T>(g.camRight) + sy * cv<T>(g.camUp));
        }
        ray.tMax = T(1e30);
        V3<T> L(T(0)), beta(T(1));
        T prevBsdfPdf = T(0);
        for (uint32_t bounce = 0; bounce <= g.maxBounces; ++bounce) {
            const Hit<T> hit = traceRay(ray);
            if (!hit.hit) {
                const V3<T> env = envRadiance(ray.dir);
                if (maxComp(env) > T(0)) {
                    T w = T(1);
                    if (bounce > 0) {
                        const T pdfLight = envPdf(ray.dir) * envPickPdf();
                        w = balanceHeuristic(prevBsdfPdf, pdfLight);
                    }
                    L += beta * env * w;
                }
                break;
            }
            const Surface s = makeSurface(ray, hit);
            const T opacity = T(s.mat->baseColorOpacity.w);
            if (opacity < T(1) && rng1<T>(rng) >= opacity) {
                ray.origin = s.pos + ray.dir * C<T>::EPS_RAY;
                continue;
            }
            V3<T> emission = cv<T>(s.mat->emissionRoughness);
            if (s.mat->tex[4] >= 0) emission = emission * texRgb(s.mat->tex[4], s.uv);
            if (maxComp(emission) > T(0) && s.frontFace) L += beta * emission;
            const Bsdf bsdf = makeBsdf(s);
            V3<T> Tn, Bn;
            buildOnb(s.nShade, Tn, Bn);
            const V3<T> nd = -ray.dir;
            V3<T> wo(dot(nd, Tn), dot(nd, Bn), dot(nd, s.nShade));
            if (wo.z < T(1e-6)) wo.z = T(1e-6);
            wo = normalize(wo);
            const LightSample ls = sampleOneLight(s.pos, rng);
            if (ls.valid && ls.pdf > T(1e-9)) {
                const V3<T> wi(dot(ls.wiWorld, Tn), dot(ls.wiWorld, Bn), dot(ls.wiWorld, s.nShade));
                V3<T> f;
                T bsdfPdf;
                bsdfEval(bsdf, wo, wi, f, bsdfPdf);
                if (maxComp(f) > T(0)) {
                    Ray<T> sh;
                    sh.origin = s.pos + s.nGeom * (wi.z > T(0) ? C<T>::EPS_RAY : -C<T>::EPS_RAY);
                    sh.dir = ls.wiWorld;
                    sh.tMax = ls.dist - T(2) * C<T>::EPS_RAY;
                    if (!traceShadowRay(sh)) {
                        const T w = ls.delta ? T(1) : balanceHeuristic(ls.pdf, bsdfPdf);
                        L += beta * f * std::fabs(wi.z) * ls.radiance * w / ls.pdf;
                    }
                }
            }
            const BsdfSample bs = bsdfSample(bsdf, wo, rng);
            if (!bs.valid) break;
            const V3<T> wiWorld = normalize(Tn * bs.wi.x + Bn * bs.wi.y + s.nShade * bs.wi.z);
            beta *= bs.f * std::fabs(bs.wi.z) / bs.pdf;
            prevBsdfPdf = bs.pdf;
            if (bounce >= 3) {
                const T p = clampv(maxComp(beta), T(0.05), T(0.95));
                if (rng1<T>(rng) >= p) break;
                beta /= p;
            }
            ray.origin = s.pos + s.nGeom * (bs.wi.z > T(0) ? C<T>::EPS_RAY : -C<T>::EPS_RAY);
            ray.dir = wiWorld;
            ray.tMax = T(1e30);
        }
        if (g.fireflyClamp > 0.0f) {
            const T m = maxComp(L);
            if (m > T(g.fireflyClamp)) L *= T(g.fireflyClamp) / m;
        }
        if (std::isnan(L.x) || std::isnan(L.y) || std::isnan(L.z) || std::isinf(L.x) || std::isinf(L.y) ||
            std::isinf(L.z))
            L = V3<T>(T(0));
        return L;
    }
};

// resolve.comp:13-22, 47-56: one pixel of the RGBA8 path.
inline float acesTonemap1(float x) {
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    return clampv((x * (a * x + b)) / (x * (c * x + d) + e), 0.0f, 1.0f);
}
inline float linearToSrgb1(float c) {
    return c <= 0.0031308f ? c * 12.92f : 1.055f * std::pow(c, 1.0f / 2.4f) - 0.055f;
}
inline uint8_t toUnorm8(float c) {
    const float v = clampv(c, 0.0f, 1.0f) * 255.0f;
    return static_cast<uint8_t>(std::floor(v + 0.5f));
}

}  // namespace orc
