// Deterministic single-precision transcendentals for the path tracer.
//
// The reference evaluates sin/cos/atan/acos with the GLSL builtins of
// whatever Vulkan driver runs it; their precision is implementation-defined.
// This build evaluates them with the functions below, which use only IEEE
// single-precision add/multiply, correctly rounded fused multiply-add and
// division, so the host (C99 fmaf, no contraction) and the device
// (__fmaf_rn etc.) produce bit-identical results. That makes a path traced
// on the GPU follow exactly the path the CPU evaluation of the same shader
// math follows, even where refraction chains amplify one-ulp differences.
//
// Methods (accuracy within a few ulp for the argument ranges used:
// |x| < 2^10 for sin/cos, any finite input for atan2/acos):
//   sin/cos: Cody-Waite reduction by pi/2 (pi/2 split into 8 + 12 + 24
//            significant bits, so k * part is exact for |k| < 2^12) and the
//            Taylor series of sin (to r^11) and cos (to r^12) on
//            [-pi/4, pi/4];
//   atan2:   reduction to a = min/max in [0, 1], then to |z| <= tan(pi/8)
//            by atan(a) = pi/4 + atan((a - 1) / (a + 1)), and the Taylor
//            series of atan (to z^21); octant fix-up;
//   acos:    atan2(sqrt((1 - x)(1 + x)), x).
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define MRT_DM __host__ __device__ __forceinline__
#else
#define MRT_DM inline
#endif

namespace detm {

MRT_DM float fma_(float a, float b, float c) {
#ifdef __CUDA_ARCH__
    return __fmaf_rn(a, b, c);
#else
    return fmaf(a, b, c);
#endif
}
MRT_DM float mul_(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
MRT_DM float add_(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
MRT_DM float div_(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
MRT_DM float sqrt_(float a) {
#ifdef __CUDA_ARCH__
    return __fsqrt_rn(a);
#else
    return sqrtf(a);
#endif
}
MRT_DM float rint_(float a) { return rintf(a); }  // round half to even on both sides

constexpr float kTwoOverPi = 0.6366197466850281f;
constexpr float kPio2Hi = 1.5703125f;                  // 8 significant bits
constexpr float kPio2Mid = 0.0004838705062866211f;     // 12 significant bits
constexpr float kPio2Lo = -4.371138828673793e-08f;     // remainder
constexpr float kPi = 3.1415927410125732f;
constexpr float kPio2 = 1.5707963705062866f;
constexpr float kPio4 = 0.7853981852531433f;
constexpr float kTanPio8 = 0.4142135679721832f;

MRT_DM void sincos(float x, float* s, float* c) {
    const float k = rint_(mul_(x, kTwoOverPi));
    float r = fma_(-k, kPio2Hi, x);
    r = fma_(-k, kPio2Mid, r);
    r = fma_(-k, kPio2Lo, r);
    const float r2 = mul_(r, r);
    // sin r = r + r^3 (-1/3! + r^2 (1/5! + r^2 (-1/7! + r^2 (1/9! - r^2/11!))))
    float ps = fma_(r2, -2.5052108385441720e-08f, 2.7557319223985893e-06f);
    ps = fma_(r2, ps, -1.9841269841269841e-04f);
    ps = fma_(r2, ps, 8.3333333333333333e-03f);
    ps = fma_(r2, ps, -1.6666666666666667e-01f);
    const float sr = fma_(mul_(r, r2), ps, r);
    // cos r = 1 + r^2 (-1/2! + r^2 (1/4! + r^2 (-1/6! + r^2 (1/8! + r^2 (-1/10! + r^2/12!)))))
    float pc = fma_(r2, 2.0876756987868099e-09f, -2.7557319223985893e-07f);
    pc = fma_(r2, pc, 2.4801587301587302e-05f);
    pc = fma_(r2, pc, -1.3888888888888889e-03f);
    pc = fma_(r2, pc, 4.1666666666666667e-02f);
    pc = fma_(r2, pc, -0.5f);
    const float cr = fma_(r2, pc, 1.0f);
    const int q = int(k) & 3;
    if (q == 0) {
        *s = sr;
        *c = cr;
    } else if (q == 1) {
        *s = cr;
        *c = -sr;
    } else if (q == 2) {
        *s = -sr;
        *c = -cr;
    } else {
        *s = -cr;
        *c = sr;
    }
}

MRT_DM float sin(float x) {
    float s, c;
    sincos(x, &s, &c);
    return s;
}
MRT_DM float cos(float x) {
    float s, c;
    sincos(x, &s, &c);
    return c;
}

// atan(z) for |z| <= tan(pi/8): Taylor series z - z^3/3 + z^5/5 - ... - z^19/19 + z^21/21
MRT_DM float atanSmall(float z) {
    const float z2 = mul_(z, z);
    float p = fma_(z2, 1.0f / 21.0f, -1.0f / 19.0f);
    p = fma_(z2, p, 1.0f / 17.0f);
    p = fma_(z2, p, -1.0f / 15.0f);
    p = fma_(z2, p, 1.0f / 13.0f);
    p = fma_(z2, p, -1.0f / 11.0f);
    p = fma_(z2, p, 1.0f / 9.0f);
    p = fma_(z2, p, -1.0f / 7.0f);
    p = fma_(z2, p, 1.0f / 5.0f);
    p = fma_(z2, p, -1.0f / 3.0f);
    return fma_(mul_(z, z2), p, z);
}

MRT_DM float atan2(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = ax > ay ? ax : ay, mn = ax > ay ? ay : ax;
    if (mx == 0.0f) {  // atan2(+-0, +0) = +-0, atan2(+-0, -0) = +-pi
        const float r = signbit(x) ? kPi : 0.0f;
        return signbit(y) ? -r : r;
    }
    const float a = div_(mn, mx);
    float t;
    if (a > kTanPio8) t = add_(kPio4, atanSmall(div_(add_(a, -1.0f), add_(a, 1.0f))));
    else t = atanSmall(a);
    if (ay > ax) t = add_(kPio2, -t);
    if (signbit(x)) t = add_(kPi, -t);
    return signbit(y) ? -t : t;
}

MRT_DM float acos(float x) {
    const float s = sqrt_(mul_(add_(1.0f, -x), add_(1.0f, x)));
    return atan2(s, x);
}

}  // namespace detm
