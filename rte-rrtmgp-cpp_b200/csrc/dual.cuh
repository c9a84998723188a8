// Forward-mode dual numbers with N tangents, for the local (per layer) derivatives inside
// the adjoint kernels: the two-stream coefficients of one layer as functions of
// (tau, ssa, g), and the cloud optics of one (layer, band) as functions of
// (lwp, iwp, re_liq, re_ice).  Each operation carries the value and its N partial
// derivatives; the value arithmetic is the forward kernels' own.
#pragma once

#include <cfloat>

namespace rrtmgp_b200 {
namespace fused {

template <int N>
struct Dual {
    float v;
    float d[N];
};

template <int N>
__device__ __forceinline__ Dual<N> dconst(float v)
{
    Dual<N> r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = 0.f;
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> dvar(float v, int i)
{
    Dual<N> r = dconst<N>(v);
    r.d[i] = 1.f;
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b)
{
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b)
{
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b)
{
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(float s, const Dual<N>& a)
{
    Dual<N> r;
    r.v = s * a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(float s, const Dual<N>& a)
{
    Dual<N> r = a;
    r.v = s + a.v;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(float s, const Dual<N>& a)
{
    Dual<N> r;
    r.v = s - a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a)
{
    return 0.f - a;
}
// Quotient; fast = the __fdividef value (as the fused forward), else IEEE division.
template <int N>
__device__ __forceinline__ Dual<N> ddiv(const Dual<N>& a, const Dual<N>& b, bool fast)
{
    Dual<N> r;
    const float ib = fast ? __fdividef(1.f, b.v) : 1.f / b.v;
    r.v = fast ? __fdividef(a.v, b.v) : a.v / b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> dselect(bool c, const Dual<N>& a, const Dual<N>& b)
{
    return c ? a : b;
}
template <int N>
__device__ __forceinline__ Dual<N> dmax(const Dual<N>& a, const Dual<N>& b)
{
    return a.v >= b.v ? a : b;
}
template <int N>
__device__ __forceinline__ Dual<N> dmin(const Dual<N>& a, const Dual<N>& b)
{
    return a.v <= b.v ? a : b;
}
}  // namespace fused
}  // namespace rrtmgp_b200
