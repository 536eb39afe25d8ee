// ORACLE -- test infrastructure only.
//
// A minimal stand-in for the subset of the GLM API that the reference's
// core/include/mrt/MathTypes.hpp, core/src/accel/Bvh.cpp,
// core/src/scene/Scene.cpp and its environment-CDF loop use, so that those
// reference sources compile here (glm itself is not vendored in the
// reference checkout). Written from the GLSL/GLM public API: component-wise
// vec2/vec3/vec4 arithmetic, scalar splats, operator[], min/max as
// (b < a ? b : a) / (a < b ? b : a), and a column-major mat4. Only
// component-wise operations reach the BVH build. The geometric functions
// follow the GLSL definitions with glm's evaluation: dot sums the products
// left to right, cross is (y1 z2 - y2 z1, z1 x2 - z2 x1, x1 y2 - x2 y1),
// length = sqrt(dot(v, v)) and normalize(v) = v * (1 / sqrt(dot(v, v)))
// (glm's inversesqrt is 1 / sqrt); these are the only assumptions about
// glm 1.0.1's arithmetic the scene-attribute pin rests on. mat4 * vec4 is
// only compiled, never called by the code the pins run.
#pragma once

#include <cmath>
#include <cstdint>

namespace glm {

template <int N, class T> struct vec;

template <class T> struct vec<2, T> {
    T x, y;
    vec() : x(0), y(0) {}
    explicit vec(T s) : x(s), y(s) {}
    vec(T a, T b) : x(a), y(b) {}
    T& operator[](uint32_t i) { return i == 0 ? x : y; }
    T operator[](uint32_t i) const { return i == 0 ? x : y; }
};

template <class T> struct vec<3, T> {
    T x, y, z;
    vec() : x(0), y(0), z(0) {}
    explicit vec(T s) : x(s), y(s), z(s) {}
    vec(T a, T b, T c) : x(a), y(b), z(c) {}
    explicit vec(const vec<4, T>& v);
    T& operator[](uint32_t i) { return i == 0 ? x : (i == 1 ? y : z); }
    T operator[](uint32_t i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

template <class T> struct vec<4, T> {
    T x, y, z, w;
    vec() : x(0), y(0), z(0), w(0) {}
    explicit vec(T s) : x(s), y(s), z(s), w(s) {}
    vec(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    vec(const vec<3, T>& v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
    T& operator[](uint32_t i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    T operator[](uint32_t i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};

template <class T> vec<3, T>::vec(const vec<4, T>& v) : x(v.x), y(v.y), z(v.z) {}

using vec2 = vec<2, float>;
using vec3 = vec<3, float>;
using vec4 = vec<4, float>;
using uvec2 = vec<2, uint32_t>;

template <int N, class T> vec<N, T> operator+(const vec<N, T>& a, const vec<N, T>& b) {
    vec<N, T> r; for (uint32_t i = 0; i < N; ++i) r[i] = a[i] + b[i]; return r;
}
template <int N, class T> vec<N, T> operator-(const vec<N, T>& a, const vec<N, T>& b) {
    vec<N, T> r; for (uint32_t i = 0; i < N; ++i) r[i] = a[i] - b[i]; return r;
}
template <int N, class T> vec<N, T> operator*(const vec<N, T>& a, const vec<N, T>& b) {
    vec<N, T> r; for (uint32_t i = 0; i < N; ++i) r[i] = a[i] * b[i]; return r;
}
template <int N, class T> vec<N, T> operator*(T s, const vec<N, T>& a) {
    vec<N, T> r; for (uint32_t i = 0; i < N; ++i) r[i] = s * a[i]; return r;
}
template <int N, class T> vec<N, T> operator*(const vec<N, T>& a, T s) {
    vec<N, T> r; for (uint32_t i = 0; i < N; ++i) r[i] = a[i] * s; return r;
}
template <int N, class T> vec<N, T>& operator+=(vec<N, T>& a, const vec<N, T>& b) { a = a + b; return a; }
template <int N, class T> vec<N, T> operator/(const vec<N, T>& a, T s) {
    vec<N, T> r; for (uint32_t i = 0; i < N; ++i) r[i] = a[i] / s; return r;
}
template <int N, class T> vec<N, T> operator-(const vec<N, T>& a) {
    vec<N, T> r; for (uint32_t i = 0; i < N; ++i) r[i] = -a[i]; return r;
}

template <int N, class T> T dot(const vec<N, T>& a, const vec<N, T>& b) {
    T s = a[0] * b[0];
    for (uint32_t i = 1; i < N; ++i) s = s + a[i] * b[i];
    return s;
}
template <class T> vec<3, T> cross(const vec<3, T>& a, const vec<3, T>& b) {
    return vec<3, T>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
template <int N, class T> T length(const vec<N, T>& v) { return std::sqrt(dot(v, v)); }
template <int N, class T> vec<N, T> normalize(const vec<N, T>& v) { return v * (T(1) / std::sqrt(dot(v, v))); }
template <class T> constexpr T pi() { return T(3.14159265358979323846264338327950288); }

template <int N, class T> vec<N, T> min(const vec<N, T>& a, const vec<N, T>& b) {
    vec<N, T> r; for (uint32_t i = 0; i < N; ++i) r[i] = (b[i] < a[i]) ? b[i] : a[i]; return r;
}
template <int N, class T> vec<N, T> max(const vec<N, T>& a, const vec<N, T>& b) {
    vec<N, T> r; for (uint32_t i = 0; i < N; ++i) r[i] = (a[i] < b[i]) ? b[i] : a[i]; return r;
}

struct mat4 {
    vec4 c[4];
    mat4() {}
    explicit mat4(float s) {
        for (int i = 0; i < 4; ++i) c[i] = vec4(0.0f);
        c[0].x = c[1].y = c[2].z = c[3].w = s;
    }
    vec4& operator[](int i) { return c[i]; }
    const vec4& operator[](int i) const { return c[i]; }
};
inline vec4 operator*(const mat4& m, const vec4& v) {
    vec4 r;
    for (uint32_t row = 0; row < 4; ++row)
        r[row] = m[0][row] * v.x + m[1][row] * v.y + m[2][row] * v.z + m[3][row] * v.w;
    return r;
}

}  // namespace glm
