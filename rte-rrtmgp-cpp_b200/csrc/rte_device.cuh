// Device building blocks of the RTE solvers shared by the per-stage and fused kernels.
#pragma once

#include <cfloat>

#include "optics_device.cuh"

namespace rrtmgp_b200 {

// Gauss-Jacobi secants and weights of Rte_lw::rte_lw (src/Rte_lw.cpp:101-113), row n-1 for
// n quadrature angles.
__device__ __constant__ static const double kGaussDs[4][4] = {
    {1.66, 0., 0., 0.},
    {1.18350343, 2.81649655, 0., 0.},
    {1.09719858, 1.69338507, 4.70941630, 0.},
    {1.06056257, 1.38282560, 2.40148179, 7.15513024}};
__device__ __constant__ static const double kGaussWts[4][4] = {
    {0.5, 0., 0., 0.},
    {0.3180413817, 0.1819586183, 0., 0.},
    {0.2009319137, 0.2292411064, 0.0698269799, 0.},
    {0.1355069134, 0.2034645680, 0.1298475476, 0.0311809710}};

template <typename T> __device__ __forceinline__ T pi_value() { return T(3.14159265358979323846); }

// Transmissivity and linear-in-tau level sources of one layer for one angle
// (lw_solver_noscat_step_1_kernel, rte_solver_kernels.cu:116-125; Clough et al. 1992).
// FP64 uses the reference expressions.  In FP32, (1 - T)/tau - T cancels to a relative error
// of eps/tau for thin layers, so the FP32 path (lw_thin_terms / lw_thick_terms, shared with the
// fused kernels) forms 1 - T itself: below tau = 0.1 the Taylor series of 1 - e^-x and of
// fact = sum_n (-1)^(n+1) n/(n+1)! tau^n (truncation < 2e-11 relative; the fact series equals
// the reference's 2-term series where that one is used); above, 1 - e^-x from the hardware
// exponential (__expf), whose error, scaled by e^-x / (1 - e^-x) <= 10, stays near 2e-6
// relative.
template <typename T>
__device__ __forceinline__ void lw_layer(T tau, T D, T lay, T lev_dn, T lev_up, T& trans, T& src_dn, T& src_up);

template <>
__device__ __forceinline__ void lw_layer<double>(double tau, double D, double lay, double lev_dn, double lev_up,
                                                 double& trans, double& src_dn, double& src_up)
{
    const double eps = DBL_EPSILON;
    const double tl = tau * D;
    trans = exp(-tl);
    const double fact = (tl > 0. && (tl * tl) > eps) ? (1. - trans) / tl - trans : tl * (0.5 - 1. / 3. * tl);
    src_dn = (1. - trans) * lev_dn + 2. * fact * (lay - lev_dn);
    src_up = (1. - trans) * lev_up + 2. * fact * (lay - lev_up);
}

// FP32 1 - T and fact = (1 - T)/tl - T of one layer (tl = tau D): the Taylor series of both
// (7 and 6 terms, truncation < 2e-11 relative), used below tl = 0.1, and the exp/divide
// intrinsics, used above, where no cancellation occurs.  Same physics as
// lw_solver_noscat_step_1_kernel (rte_solver_kernels.cu:116-125).
__device__ __forceinline__ void lw_thin_terms(float tl, float& omt, float& fact)
{
    omt = tl * (1.f + tl * (-0.5f + tl * (1.f / 6.f + tl * (-1.f / 24.f + tl * (1.f / 120.f +
          tl * (-1.f / 720.f + tl * (1.f / 5040.f)))))));
    fact = tl * (0.5f + tl * (-1.f / 3.f + tl * (0.125f + tl * (-1.f / 30.f + tl * (1.f / 144.f -
           tl * (1.f / 840.f))))));
}
__device__ __forceinline__ void lw_thick_terms(float tl, float& omt, float& fact)
{
    const float trans = __expf(-tl);
    omt = 1.f - trans;
    fact = __fdividef(omt, tl) - trans;
}

// Layer transmissivity complement and sources in FP32 for the fused kernels, whose lanes are
// g-points of one layer (thin and thick layers mix within a warp): both forms are evaluated
// and one is selected, so the warp does not diverge.
__device__ __forceinline__ void lw_layer_fast(float tau, float D, float lay, float ldn, float lup, float& omt,
                                              float& sdn, float& sup)
{
    const float tl = tau * D;
    float s_omt, s_fact, e_omt, e_fact;
    lw_thin_terms(tl, s_omt, s_fact);
    lw_thick_terms(tl, e_omt, e_fact);
    const bool thin = tl < 0.1f;
    omt = thin ? s_omt : e_omt;
    const float fact = thin ? s_fact : e_fact;
    sdn = omt * ldn + 2.f * fact * (lay - ldn);
    sup = omt * lup + 2.f * fact * (lay - lup);
}

// The per-stage solvers, whose lanes are neighbouring columns at one g-point and layer (mostly
// alike in tau), branch instead: 4% faster than the select at 8192 x 128.
template <>
__device__ __forceinline__ void lw_layer<float>(float tau, float D, float lay, float lev_dn, float lev_up,
                                               float& trans, float& src_dn, float& src_up)
{
    const float tl = tau * D;
    float omt, fact;
    if (tl < 0.1f)
        lw_thin_terms(tl, omt, fact);
    else
        lw_thick_terms(tl, omt, fact);
    trans = 1.f - omt;
    src_dn = omt * lev_dn + 2.f * fact * (lay - lev_dn);
    src_up = omt * lev_up + 2.f * fact * (lay - lev_up);
}

template <typename T> __device__ __forceinline__ T k_min_value();
template <> __device__ __forceinline__ float k_min_value<float>() { return 1.e-4f; }
template <> __device__ __forceinline__ double k_min_value<double>() { return 1.e-12; }

// Two-stream layer coefficients, Zdunkowski PIFM (sw_2stream_function,
// rte_solver_kernels.cu:535-584; F90 sw_dif_and_source :1032-1110) including the Rdir/Tdir
// clamps of the CUDA build (:581-583).  Evaluated in precision C.
template <typename C>
__device__ __forceinline__ void sw_two_stream(C tau, C w0, C g, C mu0, C& Rdif, C& Tdif, C& Rdir, C& Tdir, C& Tnoscat)
{
    const C tmin = eps_value<C>();
    const C mu0_inv = C(1) / mu0;
    const C gamma1 = (C(8) - w0 * (C(5) + C(3) * g)) * C(.25);
    const C gamma2 = C(3) * (w0 * (C(1) - g)) * C(.25);
    const C gamma3 = (C(2) - C(3) * mu0 * g) * C(.25);
    const C gamma4 = C(1) - gamma3;
    const C alpha1 = gamma1 * gamma4 + gamma2 * gamma3;
    const C alpha2 = gamma1 * gamma3 + gamma2 * gamma4;
    const C k = sqrt(max((gamma1 - gamma2) * (gamma1 + gamma2), k_min_value<C>()));
    const C e1 = exp(-tau * k);
    const C e2 = e1 * e1;
    const C rt = C(1) / (k * (C(1) + e2) + gamma1 * (C(1) - e2));
    Rdif = rt * gamma2 * (C(1) - e2);
    Tdif = rt * C(2) * k * e1;
    Tnoscat = exp(-tau * mu0_inv);
    const C k_mu = k * mu0;
    const C k_gamma3 = k * gamma3;
    const C k_gamma4 = k * gamma4;
    const C fact = (fabs(C(1) - k_mu * k_mu) > tmin) ? C(1) - k_mu * k_mu : tmin;
    const C rt2 = w0 * rt / fact;
    Rdir = rt2 * ((C(1) - k_mu) * (alpha2 + k_gamma3) - (C(1) + k_mu) * (alpha2 - k_gamma3) * e2 -
                  C(2) * (k_gamma3 - alpha2 * k_mu) * e1 * Tnoscat);
    Tdir = -rt2 * ((C(1) + k_mu) * (alpha1 + k_gamma4) * Tnoscat - (C(1) - k_mu) * (alpha1 - k_gamma4) * e2 * Tnoscat -
                   C(2) * (k_gamma4 + alpha1 * k_mu) * e1);
    Rdir = max(tmin, min(Rdir, C(1) - Tnoscat));
    Tdir = max(tmin, min(Tdir, C(1) - Tnoscat - Rdir));
}

}  // namespace rrtmgp_b200
