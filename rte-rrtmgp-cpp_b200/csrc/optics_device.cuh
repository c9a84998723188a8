// Device building blocks for cloud optics and optical-property arithmetic, shared by the
// per-stage kernels and the fused forward kernels.
#pragma once

#include <cfloat>

#include "gas_optics_device.cuh"

namespace rrtmgp_b200 {

template <typename T> __device__ __forceinline__ T eps_value();
template <> __device__ __forceinline__ float eps_value<float>() { return FLT_EPSILON; }
template <> __device__ __forceinline__ double eps_value<double>() { return DBL_EPSILON; }

// LUT layout: [ext, ssa, asy] liquid (nband, nsl) then [ext, ssa, asy] ice (nband, nsi).
template <typename T>
struct CloudLut {
    int nband, nsl, nsi;
    T liq_lwr, liq_step, ice_lwr, ice_step;
    const T* lut;
};

template <typename T>
struct CloudPoint {
    T lwp, iwp, fl, fi;  // water paths and LUT weights
    int il, ii;          // 0-based LUT index
};

// LUT index and weight (compute_from_table_kernel, src_cuda/Cloud_optics.cu:48-52):
// index = min(int((re - offset) / step) + 1, nsteps - 1); mask cwp > 0.  The reference has
// no lower clamp and reads before the table for re < offset - step; here the index is
// clamped to the first interval (same result for every re inside the LUT range).
template <typename T>
__device__ __forceinline__ CloudPoint<T> cloud_point(const CloudLut<T>& L, T lwp, T iwp, T rel, T rei)
{
    CloudPoint<T> c;
    c.lwp = lwp > T(0) ? lwp : T(0);
    c.iwp = iwp > T(0) ? iwp : T(0);
    c.il = max(0, min(int((rel - L.liq_lwr) / L.liq_step) + 1, L.nsl - 1) - 1);
    c.fl = (rel - L.liq_lwr) / L.liq_step - T(c.il);
    c.ii = max(0, min(int((rei - L.ice_lwr) / L.ice_step) + 1, L.nsi - 1) - 1);
    c.fi = (rei - L.ice_lwr) / L.ice_step - T(c.ii);
    if (!(lwp > T(0))) { c.il = 0; c.fl = T(0); }
    if (!(iwp > T(0))) { c.ii = 0; c.fi = T(0); }
    return c;
}

template <typename T>
__device__ __forceinline__ T lut_lerp(const T* tab, int idx, T f)
{
    return tab[idx] + f * (tab[idx + 1] - tab[idx]);
}

// Band b of the combined liquid + ice optics: TwoStream -> tau, ssa, g
// (combine_and_store_kernel 2str, Cloud_optics.cu:83-104, eps = epsilon); else absorption
// tau = (tau - tau*ssa) summed over phases (1scl, :61-80).
template <typename T, bool TwoStream>
__device__ __forceinline__ void cloud_band(const CloudLut<T>& L, const CloudPoint<T>& c, int b, T& tau, T& ssa, T& g)
{
    const size_t nl = size_t(L.nband) * L.nsl, ni = size_t(L.nband) * L.nsi;
    const T* le = L.lut + size_t(b) * L.nsl;
    const T* ie = L.lut + 3 * nl + size_t(b) * L.nsi;
    T lt = T(0), lts = T(0), ltg = T(0), it = T(0), its = T(0), itg = T(0);
    if (c.lwp > T(0)) {
        lt = c.lwp * lut_lerp(le, c.il, c.fl);
        lts = lt * lut_lerp(le + nl, c.il, c.fl);
        ltg = lts * lut_lerp(le + 2 * nl, c.il, c.fl);
    }
    if (c.iwp > T(0)) {
        it = c.iwp * lut_lerp(ie, c.ii, c.fi);
        its = it * lut_lerp(ie + ni, c.ii, c.fi);
        itg = its * lut_lerp(ie + 2 * ni, c.ii, c.fi);
    }
    if (TwoStream) {
        const T eps = eps_value<T>();
        tau = lt + it;
        const T ts = lts + its;
        ssa = ts / max(tau, eps);
        g = (ltg + itg) / max(ts, eps);
    } else {
        tau = (lt - lts) + (it - its);
        ssa = T(0);
        g = T(0);
    }
}

// delta_scale_2str_k_kernel (optical_props_kernels.cu:150-158), eps = 3 * numeric_limits::min.
template <typename T>
__device__ __forceinline__ void delta_scale_point(T& tau, T& ssa, T& g)
{
    const T eps = T(3) * tiny_value<T>();
    const T f = g * g;
    const T wf = ssa * f;
    tau *= (T(1) - wf);
    ssa = (ssa - wf) / max(eps, T(1) - wf);
    g = (g - f) / max(eps, T(1) - f);
}

// increment_2stream_by_2stream_kernel (optical_props_kernels.cu:56-66), eps = 3 * min.
template <typename T>
__device__ __forceinline__ void add_2str_point(T& t1, T& s1, T& g1, T t2, T s2, T g2)
{
    const T eps = T(3) * tiny_value<T>();
    const T t12 = t1 + t2;
    const T ts12 = (t1 * s1) + (t2 * s2);
    g1 = ((t1 * s1 * g1) + (t2 * s2 * g2)) / max(ts12, eps);
    s1 = ts12 / max(eps, t12);
    t1 = t12;
}

}  // namespace rrtmgp_b200
