// Stand-in for the glm vector library (https://github.com/g-truc/glm), which
// the reference takes from vcpkg without pinning a version and which is not
// installed here.  It provides only what the reference's fluid-step sources
// use (src/core/FsiCoupling2D.cu, FsiCoupling3D.cu, include/FSI_Simulator/
// core/SolidGeometryProxy_Device.cuh, utils/CudaArray.cuh): 2- and
// 3-component vectors with component-wise arithmetic, conversions between
// component types, and the
// geometric functions below, written from glm's documented definitions:
//   dot(a, b)       sum of the component-wise product a * b
//   cross(a, b)     (a.y b.z - b.y a.z, a.z b.x - b.z a.x, a.x b.y - b.x a.y)
//   length(v)       sqrt(dot(v, v))
//   normalize(v)    v * inversesqrt(dot(v, v)), inversesqrt(x) = 1 / sqrt(x)
//   distance(a, b)  length(b - a)
//   min(a, b)       b < a ? b : a;   max(a, b)  a < b ? b : a
// Test infrastructure: it exists only to compile the reference's own step
// into oracle/_ref, the checker of the product.
#pragma once
#include <cfloat>
#include <cmath>
#include <limits>

#if defined(__CUDACC__)
#define GLMS_FN __host__ __device__ inline
#else
#define GLMS_FN inline
#endif

namespace glm {

template <int L, typename T> struct vec;

template <typename T> struct vec<2, T> {
    T x, y;
    GLMS_FN vec() : x(0), y(0) {}
    GLMS_FN explicit vec(T s) : x(s), y(s) {}
    template <typename A, typename B> GLMS_FN vec(A a, B b) : x(static_cast<T>(a)), y(static_cast<T>(b)) {}
    template <typename U> GLMS_FN vec(const vec<2, U> &o) : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)) {}
    GLMS_FN T &operator[](int i) { return i == 0 ? x : y; }
    GLMS_FN const T &operator[](int i) const { return i == 0 ? x : y; }
    GLMS_FN vec &operator*=(T s) { x *= s; y *= s; return *this; }
    GLMS_FN vec &operator/=(T s) { x /= s; y /= s; return *this; }
    GLMS_FN vec &operator+=(const vec &o) { x += o.x; y += o.y; return *this; }
    GLMS_FN vec &operator-=(const vec &o) { x -= o.x; y -= o.y; return *this; }
};

template <typename T> struct vec<3, T> {
    T x, y, z;
    GLMS_FN vec() : x(0), y(0), z(0) {}
    GLMS_FN explicit vec(T s) : x(s), y(s), z(s) {}
    template <typename A, typename B, typename C>
    GLMS_FN vec(A a, B b, C c) : x(static_cast<T>(a)), y(static_cast<T>(b)), z(static_cast<T>(c)) {}
    template <typename U>
    GLMS_FN vec(const vec<3, U> &o) : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)), z(static_cast<T>(o.z)) {}
    GLMS_FN T &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    GLMS_FN const T &operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    GLMS_FN vec &operator*=(T s) { x *= s; y *= s; z *= s; return *this; }
    GLMS_FN vec &operator/=(T s) { x /= s; y /= s; z /= s; return *this; }
    GLMS_FN vec &operator+=(const vec &o) { x += o.x; y += o.y; z += o.z; return *this; }
    GLMS_FN vec &operator-=(const vec &o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
};

using vec2 = vec<2, float>;
using vec3 = vec<3, float>;
using dvec2 = vec<2, double>;
using dvec3 = vec<3, double>;
using ivec2 = vec<2, int>;
using ivec3 = vec<3, int>;

template <typename T> GLMS_FN vec<2, T> operator+(const vec<2, T> &a, const vec<2, T> &b) { return vec<2, T>(a.x + b.x, a.y + b.y); }
template <typename T> GLMS_FN vec<2, T> operator-(const vec<2, T> &a, const vec<2, T> &b) { return vec<2, T>(a.x - b.x, a.y - b.y); }
template <typename T> GLMS_FN vec<2, T> operator*(const vec<2, T> &a, const vec<2, T> &b) { return vec<2, T>(a.x * b.x, a.y * b.y); }
template <typename T> GLMS_FN vec<2, T> operator*(const vec<2, T> &a, T s) { return vec<2, T>(a.x * s, a.y * s); }
template <typename T> GLMS_FN vec<2, T> operator*(T s, const vec<2, T> &a) { return vec<2, T>(s * a.x, s * a.y); }
template <typename T> GLMS_FN vec<2, T> operator/(const vec<2, T> &a, T s) { return vec<2, T>(a.x / s, a.y / s); }
template <typename T> GLMS_FN vec<2, T> operator-(const vec<2, T> &a) { return vec<2, T>(-a.x, -a.y); }

template <typename T> GLMS_FN vec<3, T> operator+(const vec<3, T> &a, const vec<3, T> &b) { return vec<3, T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename T> GLMS_FN vec<3, T> operator-(const vec<3, T> &a, const vec<3, T> &b) { return vec<3, T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T> GLMS_FN vec<3, T> operator*(const vec<3, T> &a, const vec<3, T> &b) { return vec<3, T>(a.x * b.x, a.y * b.y, a.z * b.z); }
template <typename T> GLMS_FN vec<3, T> operator*(const vec<3, T> &a, T s) { return vec<3, T>(a.x * s, a.y * s, a.z * s); }
template <typename T> GLMS_FN vec<3, T> operator*(T s, const vec<3, T> &a) { return vec<3, T>(s * a.x, s * a.y, s * a.z); }
template <typename T> GLMS_FN vec<3, T> operator/(const vec<3, T> &a, T s) { return vec<3, T>(a.x / s, a.y / s, a.z / s); }
template <typename T> GLMS_FN vec<3, T> operator-(const vec<3, T> &a) { return vec<3, T>(-a.x, -a.y, -a.z); }

template <typename T> GLMS_FN T dot(const vec<2, T> &a, const vec<2, T> &b)
{
    vec<2, T> t = a * b;
    return t.x + t.y;
}
template <typename T> GLMS_FN T dot(const vec<3, T> &a, const vec<3, T> &b)
{
    vec<3, T> t = a * b;
    return t.x + t.y + t.z;
}
template <typename T> GLMS_FN vec<3, T> cross(const vec<3, T> &a, const vec<3, T> &b)
{
    return vec<3, T>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
template <typename T> GLMS_FN T inversesqrt(T v) { return static_cast<T>(1) / sqrt(v); }
template <int L, typename T> GLMS_FN T length(const vec<L, T> &v) { return sqrt(dot(v, v)); }
template <int L, typename T> GLMS_FN vec<L, T> normalize(const vec<L, T> &v) { return v * inversesqrt(dot(v, v)); }
template <int L, typename T> GLMS_FN T distance(const vec<L, T> &a, const vec<L, T> &b) { return length(b - a); }
template <typename T> GLMS_FN T min(T a, T b) { return b < a ? b : a; }
template <typename T> GLMS_FN T max(T a, T b) { return a < b ? b : a; }

} // namespace glm
