// float3 arithmetic for the sm_100a kernels. Operations mirror the GLSL
// builtins the reference shaders use (dot, cross, normalize, mix, reflect,
// refract, clamp, fract) so the kernel code reads like the math it restates.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define MRT_DEV __device__ __forceinline__

MRT_DEV float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
MRT_DEV float3 f3(float s) { return make_float3(s, s, s); }
MRT_DEV float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
MRT_DEV float3 f3p(const float* p) { return make_float3(p[0], p[1], p[2]); }

MRT_DEV float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
MRT_DEV float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
MRT_DEV float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
MRT_DEV float3 operator/(float3 a, float3 b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
MRT_DEV float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
MRT_DEV float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
MRT_DEV float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
MRT_DEV float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
MRT_DEV float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
MRT_DEV float3& operator*=(float3& a, float3 b) { a = a * b; return a; }
MRT_DEV float3& operator*=(float3& a, float s) { a = a * s; return a; }
MRT_DEV float3& operator/=(float3& a, float s) { a = a / s; return a; }

MRT_DEV float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
MRT_DEV float3 cross(float3 a, float3 b) {
    return f3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
MRT_DEV float length(float3 v) { return sqrtf(dot(v, v)); }
MRT_DEV float3 normalize(float3 v) { return v * (1.0f / sqrtf(dot(v, v))); }
// GLSL max/min as the shaders' CPU evaluation computes them: max(a, b) =
// a < b ? b : a and min(a, b) = b < a ? b : a, so signed zeros and NaNs
// resolve identically on both sides.
MRT_DEV float mmax(float a, float b) { return a < b ? b : a; }
MRT_DEV float mmin(float a, float b) { return b < a ? b : a; }
MRT_DEV float maxComp(float3 v) { return mmax(v.x, mmax(v.y, v.z)); }
MRT_DEV float clampf(float x, float lo, float hi) { return mmin(mmax(x, lo), hi); }
MRT_DEV float mixf(float x, float y, float a) { return x * (1.0f - a) + y * a; }
MRT_DEV float3 mix3(float3 x, float3 y, float a) { return x * (1.0f - a) + y * a; }
MRT_DEV float fractf(float x) { return x - floorf(x); }
MRT_DEV float3 reflect(float3 i, float3 n) { return i - 2.0f * dot(n, i) * n; }
MRT_DEV float3 refract(float3 i, float3 n, float eta) {
    const float d = dot(n, i);
    const float k = 1.0f - eta * eta * (1.0f - d * d);
    if (k < 0.0f) return f3(0.0f);
    return eta * i - (eta * d + sqrtf(k)) * n;
}
// Rec. 709 luminance (reference common.glsl:90)
MRT_DEV float luminance(float3 c) { return dot(c, f3(0.2126f, 0.7152f, 0.0722f)); }
MRT_DEV float comp(float3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

// Row-major 3x4 affine transform (rows of [R | t]).
MRT_DEV float3 xformPoint(const float* m, float3 p) {
    return f3(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
              m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]);
}
MRT_DEV float3 xformDir(const float* m, float3 d) {
    return f3(m[0] * d.x + m[1] * d.y + m[2] * d.z, m[4] * d.x + m[5] * d.y + m[6] * d.z,
              m[8] * d.x + m[9] * d.y + m[10] * d.z);
}
// transpose(R) * v: the normal transform with R = the world-to-object
// rotation part (the inverse-transpose of object-to-world).
MRT_DEV float3 xformTransposed(const float* m, float3 v) {
    return f3(m[0] * v.x + m[4] * v.y + m[8] * v.z, m[1] * v.x + m[5] * v.y + m[9] * v.z,
              m[2] * v.x + m[6] * v.y + m[10] * v.z);
}

// 128-bit read-only loads
MRT_DEV float4 ldg4(const float4* p) { return __ldg(p); }
MRT_DEV uint4 ldg4u(const uint4* p) { return __ldg(p); }
