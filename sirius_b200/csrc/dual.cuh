// dual.cuh — register-resident forward-mode automatic differentiation.
//
// D3<T> carries a value and its gradient with respect to the three spatial
// coordinates of the integration chart. Metric potentials written with D3
// yield d_l g_{mu nu} without a tape or memory traffic: everything stays in
// registers and the compiler drops the zero tangents of constants. The
// reference's Dual<T> (src/Sirius.Core/Autodiff/MTDL001A.h:19-370) is a
// container whose tangent is never propagated; this type is the working form.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

// The metric templates compile for the device under nvcc and, in host-only
// translation units (the operation counter), as plain host code.
#ifndef SIRIUS_HD
#ifdef __CUDACC__
#define SIRIUS_HD __host__ __device__
#else
#define SIRIUS_HD
#endif
#endif

namespace sirius {

#ifdef __CUDACC__
// Reciprocal and square root used by the metric code. FP32 uses the
// fast single-instruction forms (the FP32 path is an approximation by design:
// its error budget is set by the FP64 state accumulation and FP64 projection);
// FP64 uses IEEE-rounded division and square root.
__device__ __forceinline__ float rcp_(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ double rcp_(double x) { return 1.0 / x; }
__device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
__device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
// Square root of a positive argument. FP32: x * rsqrt(x), two instructions with
// single-precision relative accuracy (the correctly rounded sqrtf is a longer
// sequence with a special-case branch); FP64: sqrt.
__device__ __forceinline__ float sqrtp_(float x) { return x * rsqrtf(x); }
__device__ __forceinline__ double sqrtp_(double x) { return sqrt(x); }
__device__ __forceinline__ double rsqrt_(double x) { return 1.0 / sqrt(x); }
__device__ __forceinline__ float exp_(float x) { return __expf(x); }
__device__ __forceinline__ double exp_(double x) { return exp(x); }
__device__ __forceinline__ float tanh_(float x) { return tanhf(x); }
__device__ __forceinline__ double tanh_(double x) { return tanh(x); }
#else
inline float rcp_(float x) { return 1.0f / x; }
inline double rcp_(double x) { return 1.0 / x; }
inline float sqrt_(float x) { return std::sqrt(x); }
inline double sqrt_(double x) { return std::sqrt(x); }
inline float rsqrt_(float x) { return 1.0f / std::sqrt(x); }
inline float sqrtp_(float x) { return std::sqrt(x); }
inline double sqrtp_(double x) { return std::sqrt(x); }
inline double rsqrt_(double x) { return 1.0 / std::sqrt(x); }
inline float exp_(float x) { return std::exp(x); }
inline double exp_(double x) { return std::exp(x); }
inline float tanh_(float x) { return std::tanh(x); }
inline double tanh_(double x) { return std::tanh(x); }
#endif

template <class T>
struct D3 {
    T v;
    T d[3];
};

template <class T>
SIRIUS_HD __forceinline__ D3<T> dconst(T v) {
    return D3<T>{v, {T(0), T(0), T(0)}};
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> dvar(T v, int axis) {
    D3<T> r{v, {T(0), T(0), T(0)}};
    r.d[axis] = T(1);
    return r;
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> operator+(const D3<T>& a, const D3<T>& b) {
    return D3<T>{a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]}};
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> operator-(const D3<T>& a, const D3<T>& b) {
    return D3<T>{a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2]}};
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> operator-(const D3<T>& a) {
    return D3<T>{-a.v, {-a.d[0], -a.d[1], -a.d[2]}};
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> operator+(const D3<T>& a, T s) {
    return D3<T>{a.v + s, {a.d[0], a.d[1], a.d[2]}};
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> operator-(const D3<T>& a, T s) {
    return D3<T>{a.v - s, {a.d[0], a.d[1], a.d[2]}};
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> operator*(const D3<T>& a, T s) {
    return D3<T>{a.v * s, {a.d[0] * s, a.d[1] * s, a.d[2] * s}};
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> operator*(T s, const D3<T>& a) {
    return a * s;
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> operator*(const D3<T>& a, const D3<T>& b) {
    return D3<T>{a.v * b.v,
                 {a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1], a.d[2] * b.v + a.v * b.d[2]}};
}
// 1/a
template <class T>
SIRIUS_HD __forceinline__ D3<T> inv(const D3<T>& a) {
    const T r = rcp_(a.v);
    const T r2 = -r * r;
    return D3<T>{r, {a.d[0] * r2, a.d[1] * r2, a.d[2] * r2}};
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> operator/(const D3<T>& a, const D3<T>& b) {
    return a * inv(b);
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> dsqrt(const D3<T>& a) {
    const T s = sqrt_(a.v);
    const T h = T(0.5) * rcp_(s);
    return D3<T>{s, {a.d[0] * h, a.d[1] * h, a.d[2] * h}};
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> dexp(const D3<T>& a) {
    const T e = exp_(a.v);
    return D3<T>{e, {a.d[0] * e, a.d[1] * e, a.d[2] * e}};
}
template <class T>
SIRIUS_HD __forceinline__ D3<T> dtanh(const D3<T>& a) {
    const T t = tanh_(a.v);
    const T s = T(1) - t * t;
    return D3<T>{t, {a.d[0] * s, a.d[1] * s, a.d[2] * s}};
}
// a with its gradient replaced by g (the chain-rule seed of an implicit function)
template <class T>
SIRIUS_HD __forceinline__ D3<T> dwith(T v, T g0, T g1, T g2) {
    return D3<T>{v, {g0, g1, g2}};
}

}  // namespace sirius
