// Minimal stand-in for the `owl::common` vector types (OWL v1.1.6,
// owl/common/math/vec.h) so that the reference's header-only kernel library
// (include/colvillea/libkernel/base/*.h, libkernel/bsdfs/*.h) compiles on the
// host with g++.  Test infrastructure only: this shim is used to build
// oracle/_ref, the compiled reference that pins the oracle.
//
// Semantics restated from OWL's published vector math:
//   * component-wise + - * / between vectors and with scalars (both sides);
//   * dot(a,b) = a.x*b.x + a.y*b.y (+ a.z*b.z (+ a.w*b.w)), left to right;
//   * cross(a,b) = (a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x);
//   * normalize(v) = v * (1 / sqrt(dot(v,v)));  length(v) = sqrt(dot(v,v)).
// The scalar broadcast constructor is implicit, as the reference relies on
// returning a float where a vec3f is expected (roughdielectric.h:91, bsdf.h:94).
#pragma once

#include <vector_types.h> // CUDA's host_defines: __host__/__device__/__forceinline__
#include <cmath>
#include <math.h>
#include <cstdint>
#include <cstdlib>
#include <cassert>
#include <type_traits>

using std::abs;

namespace owl
{
namespace common
{
template <typename T, int N> struct vec_t;

template <typename T> struct vec_t<T, 2>
{
    T x{}, y{};
    vec_t() = default;
    __host__ __device__ vec_t(const T& t) : x(t), y(t) {}
    __host__ __device__ vec_t(const T& a, const T& b) : x(a), y(b) {}
    template <typename U>
    __host__ __device__ explicit vec_t(const vec_t<U, 2>& o) : x(T(o.x)), y(T(o.y)) {}
    T&       operator[](int i) { return (&x)[i]; }
    const T& operator[](int i) const { return (&x)[i]; }
};

template <typename T> struct vec_t<T, 3>
{
    T x{}, y{}, z{};
    vec_t() = default;
    __host__ __device__ vec_t(const T& t) : x(t), y(t), z(t) {}
    __host__ __device__ vec_t(const T& a, const T& b, const T& c) : x(a), y(b), z(c) {}
    template <typename U>
    __host__ __device__ explicit vec_t(const vec_t<U, 3>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
    __host__ __device__ explicit vec_t(const vec_t<T, 4>& o) : x(o.x), y(o.y), z(o.z) {}
    T&       operator[](int i) { return (&x)[i]; }
    const T& operator[](int i) const { return (&x)[i]; }
};

template <typename T> struct vec_t<T, 4>
{
    T x{}, y{}, z{}, w{};
    vec_t() = default;
    __host__ __device__ vec_t(const T& t) : x(t), y(t), z(t), w(t) {}
    __host__ __device__ vec_t(const T& a, const T& b, const T& c, const T& d) : x(a), y(b), z(c), w(d) {}
    template <typename U>
    __host__ __device__ explicit vec_t(const vec_t<U, 4>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)), w(T(o.w)) {}
    __host__ __device__ vec_t(const vec_t<T, 3>& v, const T& d) : x(v.x), y(v.y), z(v.z), w(d) {}
    T&       operator[](int i) { return (&x)[i]; }
    const T& operator[](int i) const { return (&x)[i]; }
};

#define SHIM_BINOP(OP)                                                                            \
    template <typename T, int N> inline vec_t<T, N> operator OP(const vec_t<T, N>& a, const vec_t<T, N>& b) \
    {                                                                                             \
        vec_t<T, N> r;                                                                            \
        for (int i = 0; i < N; ++i) r[i] = a[i] OP b[i];                                          \
        return r;                                                                                 \
    }                                                                                             \
    template <typename T, int N, typename S, typename = std::enable_if_t<std::is_arithmetic_v<S>>>  \
    inline vec_t<T, N> operator OP(const vec_t<T, N>& a, const S& s)                              \
    {                                                                                             \
        vec_t<T, N> r;                                                                            \
        for (int i = 0; i < N; ++i) r[i] = a[i] OP T(s);                                          \
        return r;                                                                                 \
    }                                                                                             \
    template <typename T, int N, typename S, typename = std::enable_if_t<std::is_arithmetic_v<S>>>  \
    inline vec_t<T, N> operator OP(const S& s, const vec_t<T, N>& a)                              \
    {                                                                                             \
        vec_t<T, N> r;                                                                            \
        for (int i = 0; i < N; ++i) r[i] = T(s) OP a[i];                                          \
        return r;                                                                                 \
    }                                                                                             \
    template <typename T, int N> inline vec_t<T, N>& operator OP##=(vec_t<T, N>& a, const vec_t<T, N>& b) \
    {                                                                                             \
        for (int i = 0; i < N; ++i) a[i] = a[i] OP b[i];                                          \
        return a;                                                                                 \
    }                                                                                             \
    template <typename T, int N, typename S, typename = std::enable_if_t<std::is_arithmetic_v<S>>>  \
    inline vec_t<T, N>& operator OP##=(vec_t<T, N>& a, const S& s)                                \
    {                                                                                             \
        for (int i = 0; i < N; ++i) a[i] = a[i] OP T(s);                                          \
        return a;                                                                                 \
    }

SHIM_BINOP(+)
SHIM_BINOP(-)
SHIM_BINOP(*)
SHIM_BINOP(/)
#undef SHIM_BINOP

template <typename T, int N> inline vec_t<T, N> operator-(const vec_t<T, N>& a)
{
    vec_t<T, N> r;
    for (int i = 0; i < N; ++i) r[i] = -a[i];
    return r;
}

template <typename T, int N> inline bool operator==(const vec_t<T, N>& a, const vec_t<T, N>& b)
{
    for (int i = 0; i < N; ++i)
        if (!(a[i] == b[i])) return false;
    return true;
}

template <typename T> inline T dot(const vec_t<T, 2>& a, const vec_t<T, 2>& b) { return a.x * b.x + a.y * b.y; }
template <typename T> inline T dot(const vec_t<T, 3>& a, const vec_t<T, 3>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> inline T dot(const vec_t<T, 4>& a, const vec_t<T, 4>& b)
{
    return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}

template <typename T> inline vec_t<T, 3> cross(const vec_t<T, 3>& a, const vec_t<T, 3>& b)
{
    return vec_t<T, 3>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

namespace polymorphic
{
inline float  sqrt(float f) { return ::sqrtf(f); }
inline double sqrt(double f) { return ::sqrt(f); }
} // namespace polymorphic

inline float  sqrt(float f) { return ::sqrtf(f); }
inline double sqrt(double f) { return ::sqrt(f); }
inline float  abs(float f) { return ::fabsf(f); }
inline double abs(double f) { return ::fabs(f); }

template <typename T, int N> inline vec_t<T, N> sqrt(const vec_t<T, N>& a)
{
    vec_t<T, N> r;
    for (int i = 0; i < N; ++i) r[i] = polymorphic::sqrt(a[i]);
    return r;
}

template <typename T, int N> inline T length(const vec_t<T, N>& a) { return polymorphic::sqrt(dot(a, a)); }

template <typename T, int N> inline vec_t<T, N> normalize(const vec_t<T, N>& a)
{
    return a * (T(1) / polymorphic::sqrt(dot(a, a)));
}

template <typename T> inline T clamp(const T& v, const T& lo, const T& hi) { return v < lo ? lo : (v > hi ? hi : v); }

using vec2f  = vec_t<float, 2>;
using vec2ui = vec_t<uint32_t, 2>;
using vec2i  = vec_t<int32_t, 2>;
using vec3f  = vec_t<float, 3>;
using vec3ui = vec_t<uint32_t, 3>;
using vec3i  = vec_t<int32_t, 3>;
using vec4f  = vec_t<float, 4>;
using vec4ui = vec_t<uint32_t, 4>;
using vec4i  = vec_t<int32_t, 4>;
} // namespace common

using common::cross;
using common::dot;
using common::normalize;
} // namespace owl
