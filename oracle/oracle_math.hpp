// ORACLE -- test infrastructure only. Not part of the product library.
//
// Small vector toolkit for the CPU restatement of the MiniRaytrace shader
// math. Every operation follows the GLSL 4.60 definition of the builtin it
// stands for (dot, cross, normalize = v * inversesqrt(dot(v, v)), mix =
// x*(1-a) + y*a, reflect, refract, fract, clamp), evaluated in T = float
// (parity mode, IEEE single, no contraction) or T = double (converged mode).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace orc {

template <class T>
struct V2 {
    T x = 0, y = 0;
    V2() = default;
    V2(T a, T b) : x(a), y(b) {}
};

template <class T>
struct V3 {
    T x = 0, y = 0, z = 0;
    V3() = default;
    V3(T a, T b, T c) : x(a), y(b), z(c) {}
    explicit V3(T s) : x(s), y(s), z(s) {}
    T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

template <class T>
struct V4 {
    T x = 0, y = 0, z = 0, w = 0;
    V4() = default;
    V4(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    V4(const V3<T>& v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
    V3<T> xyz() const { return V3<T>(x, y, z); }
};

template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline V3<T> operator/(V3<T> a, V3<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> inline V3<T>& operator+=(V3<T>& a, V3<T> b) { a = a + b; return a; }
template <class T> inline V3<T>& operator*=(V3<T>& a, V3<T> b) { a = a * b; return a; }
template <class T> inline V3<T>& operator*=(V3<T>& a, T s) { a = a * s; return a; }
template <class T> inline V3<T>& operator/=(V3<T>& a, T s) { a = a / s; return a; }

template <class T> inline V2<T> operator+(V2<T> a, V2<T> b) { return {a.x + b.x, a.y + b.y}; }
template <class T> inline V2<T> operator-(V2<T> a, V2<T> b) { return {a.x - b.x, a.y - b.y}; }
template <class T> inline V2<T> operator*(T s, V2<T> a) { return {s * a.x, s * a.y}; }

template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
template <class T> inline T msqrt(T x) { return std::sqrt(x); }
template <class T> inline T inversesqrt(T x) { return T(1) / std::sqrt(x); }
template <class T> inline T length(V3<T> v) { return std::sqrt(dot(v, v)); }
template <class T> inline V3<T> normalize(V3<T> v) { return v * inversesqrt(dot(v, v)); }
template <class T> inline T mmax(T a, T b) { return a < b ? b : a; }
template <class T> inline T mmin(T a, T b) { return b < a ? b : a; }
template <class T> inline T clampv(T x, T lo, T hi) { return mmin(mmax(x, lo), hi); }
template <class T> inline V3<T> vmin(V3<T> a, V3<T> b) { return {mmin(a.x, b.x), mmin(a.y, b.y), mmin(a.z, b.z)}; }
template <class T> inline V3<T> vmax(V3<T> a, V3<T> b) { return {mmax(a.x, b.x), mmax(a.y, b.y), mmax(a.z, b.z)}; }
template <class T> inline T maxComp(V3<T> v) { return mmax(v.x, mmax(v.y, v.z)); }
template <class T> inline T mix(T x, T y, T a) { return x * (T(1) - a) + y * a; }
template <class T> inline V3<T> mix(V3<T> x, V3<T> y, T a) { return x * (T(1) - a) + y * a; }
template <class T> inline V3<T> mix(V3<T> x, V3<T> y, V3<T> a) {
    return {mix(x.x, y.x, a.x), mix(x.y, y.y, a.y), mix(x.z, y.z, a.z)};
}
template <class T> inline T fract(T x) { return x - std::floor(x); }
// GLSL reflect(I, N) = I - 2 * dot(N, I) * N
template <class T> inline V3<T> reflect(V3<T> i, V3<T> n) { return i - T(2) * dot(n, i) * n; }
// GLSL refract(I, N, eta)
template <class T> inline V3<T> refract(V3<T> i, V3<T> n, T eta) {
    const T d = dot(n, i);
    const T k = T(1) - eta * eta * (T(1) - d * d);
    if (k < T(0)) return V3<T>(T(0));
    return eta * i - (eta * d + std::sqrt(k)) * n;
}
// common.glsl:90 (Rec. 709 luma weights)
template <class T> inline T luminance(V3<T> c) {
    return dot(c, V3<T>(T(0.2126), T(0.7152), T(0.0722)));
}

// Column-major 4x4 matrix (glm convention): m[col][row].
template <class T>
struct M4 {
    T m[4][4];
    static M4 identity() {
        M4 r{};
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) r.m[i][j] = (i == j) ? T(1) : T(0);
        return r;
    }
    // M * (x, y, z, w)
    V3<T> mulPoint(V3<T> p) const {
        return {m[0][0] * p.x + m[1][0] * p.y + m[2][0] * p.z + m[3][0],
                m[0][1] * p.x + m[1][1] * p.y + m[2][1] * p.z + m[3][1],
                m[0][2] * p.x + m[1][2] * p.y + m[2][2] * p.z + m[3][2]};
    }
    V3<T> mulDir(V3<T> d) const {
        return {m[0][0] * d.x + m[1][0] * d.y + m[2][0] * d.z,
                m[0][1] * d.x + m[1][1] * d.y + m[2][1] * d.z,
                m[0][2] * d.x + m[1][2] * d.y + m[2][2] * d.z};
    }
    // transpose(mat3(M)) * v: rows of the upper 3x3 dotted with v.
    V3<T> mulTransposed3(V3<T> v) const {
        return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z,
                m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
                m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
    }
};

// Inverse of an affine transform [R | t] (the only kind the API produces:
// reference MathTypes.hpp:49-56 builds it from a row-major 3x4). With the
// columns c0, c1, c2 of R, the rows of R^-1 are (c1 x c2, c2 x c0, c0 x c1)
// divided by det = c0 . (c1 x c2); the translation becomes -R^-1 t. The
// reference uses glm::inverse (Renderer.cpp:475), whose rounding is not
// restated here; both are exact for identity, translations and
// power-of-two scales. For other scales s this formula's entries
// s^2 * (1 / s^3) are within 2 ulp of 1/s, and glm's may round differently:
// parity with the reference's inverse is unpinned there.
template <class T>
M4<T> inverse(const M4<T>& a) {
    const V3<T> c0(a.m[0][0], a.m[0][1], a.m[0][2]);
    const V3<T> c1(a.m[1][0], a.m[1][1], a.m[1][2]);
    const V3<T> c2(a.m[2][0], a.m[2][1], a.m[2][2]);
    const V3<T> t(a.m[3][0], a.m[3][1], a.m[3][2]);
    const V3<T> r0 = cross(c1, c2), r1 = cross(c2, c0), r2 = cross(c0, c1);
    const T invDet = T(1) / dot(c0, r0);
    const V3<T> i0 = r0 * invDet, i1 = r1 * invDet, i2 = r2 * invDet;  // rows of R^-1
    M4<T> r = M4<T>::identity();
    r.m[0][0] = i0.x; r.m[1][0] = i0.y; r.m[2][0] = i0.z;
    r.m[0][1] = i1.x; r.m[1][1] = i1.y; r.m[2][1] = i1.z;
    r.m[0][2] = i2.x; r.m[1][2] = i2.y; r.m[2][2] = i2.z;
    r.m[3][0] = -dot(i0, t);
    r.m[3][1] = -dot(i1, t);
    r.m[3][2] = -dot(i2, t);
    return r;
}

inline float bitsToFloat(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline uint32_t floatToBits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

}  // namespace orc
