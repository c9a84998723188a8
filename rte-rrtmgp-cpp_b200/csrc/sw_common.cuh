// Shortwave building blocks shared by the fused forward kernel (forward_sw.cu) and its
// adjoint (adjoint_sw.cu): cloud arguments, 1 - exp(-x), the FP32 two-stream layer
// coefficients and the per-(layer, band) record.
#pragma once

#include "aerosol_device.cuh"
#include "fused_common.cuh"
#include "optics_device.cuh"

namespace rrtmgp_b200 {
namespace fused {

struct SwCloudArgs {
    CloudLut<float> L;
    const float* lwp;
    const float* iwp;
    const float* rel;
    const float* rei;
    int present;
    int delta;
};

// Aerosol optics of the fused shortwave kernels (the reference's switch_aerosol_optics step,
// src_test/Radiation_solver.cu:794-807: aerosol optics, optionally delta-scaled, added by band
// after the clouds).  present == 0: no aerosols.
struct SwAerosolArgs {
    AerosolLut<float> L;
    AerosolSet<float> s;
    const float* rh;     // (ncol, nlay)
    int present;
    int delta;
};

// Aerosol (tau, tau*ssa, tau*ssa*g, tau*(1 - ssa)) of band b at reference-layout layer l of
// column icol, delta-scaled when a.delta (Optical_props_2str_gpu::delta_scale,
// optical_props_kernels.cu:139-160); dp = |p_bottom - p_top| of the layer.  ssa and g are
// formed with the epsilon clamps of combine_and_store_kernel (src_cuda/Aerosol_optics.cu:
// 170-186) at the FP64 build's epsilon, as the other clamps of the FP32 kernels: with the
// FP32 epsilon (1.2e-7) g of the thin upper-layer aerosol would collapse to ~0 and its delta
// scaling differ from the FP64 result.
__device__ __forceinline__ float4 aerosol_point(const SwAerosolArgs& a, int ncol, int icol, int l, float dp, int b)
{
    const size_t cl = icol + size_t(l) * ncol;
    const int ihum = aerosol_rh_class(a.L, a.rh[cl]);
    float mmr[kNAerosol];
#pragma unroll
    for (int s = 0; s < kNAerosol; ++s) mmr[s] = aerosol_mmr(a.s, s, ncol, icol, l);
    float t, ts, tsg, tabs;
    aerosol_band_abs(a.L, mmr, ihum, dp / 9.81f, b, t, ts, tsg, tabs);
    if (a.delta) {
        const float eps = 2.220446049250313e-16f;   // DBL_EPSILON
        float ssa = ts / fmaxf(t, eps), g = tsg / fmaxf(ts, eps);
        delta_scale_point(t, ssa, g);
        ts = t * ssa;
        tsg = ts * g;
    }
    return make_float4(t, ts, tsg, tabs);
}

// 1 - exp(-x) and exp(-x) for x >= 0, each with a small relative error: Taylor series of
// 1 - exp(-x) through x^8 below 0.5 (truncation < 1.4e-8 relative), the exp intrinsic above.
// Both are evaluated and selected (no divergence between the lanes of a warp).
__device__ __forceinline__ void one_minus_exp(float x, float& E, float& e)
{
    const float Es = x * (1.f - x * (1.f / 2.f - x * (1.f / 6.f - x * (1.f / 24.f - x * (1.f / 120.f - x * (1.f / 720.f -
                     x * (1.f / 5040.f - x * (1.f / 40320.f))))))));
    const float ex = __expf(-x);
    const bool small = x < 0.5f;
    E = small ? Es : 1.f - ex;
    e = small ? 1.f - Es : ex;
}

// Layer coefficients of the PIFM two-stream (sw_2stream_function, rte_solver_kernels.cu:
// 535-584) in FP32.  The reference expressions lose all relative accuracy in FP32 for thin and
// for conservatively scattering layers (O(1) terms cancelling to O(tau)); here they are
// rearranged with E1 = 1 - exp(-k tau), E2 = 1 - exp(-2 k tau), En = 1 - exp(-tau/mu0) so
// that the constant parts cancel analytically (same values in exact arithmetic):
//   gamma1 - gamma2 = 2 (1 - w0),  1 - Rdif - Tdif = rt (k E1^2 + 2 (1 - w0) E2),
//   Rdir bracket = E2 (alpha2 - k^2 mu0 gamma3) + k (gamma3 - mu0 alpha2) (E1^2 + 2 e1 En),
//   Tdir bracket = Tn E2 (alpha1 + k^2 mu0 gamma4) + k (gamma4 + mu0 alpha1) (E1^2 - (1 + e2) En),
// the Tdir bracket taking the reference form when both exponentials are small (thick layers).
// omw = 1 - w0 is passed separately, formed from absorption optical depths, so it keeps its
// accuracy for w0 -> 1.  Clamps and k_min are those of the FP64 reference (DBL_EPSILON,
// 1e-12).  Divisions and the square root use the approximate intrinsics (a few ulp; the
// operands are normal numbers).
//
// Near the removable singularity k mu0 = 1 (|1 - (k mu0)^2| < 0.02) both brackets vanish with
// 1 - (k mu0)^2.  With d = 1 - k mu0 and x = tau d / mu0 they factor exactly as
//   Rdir bracket = d [ (alpha2 + k gamma3) Z - 2 X e1^2 (tau/mu0) phi(x) ],
//   Tdir bracket = -d [ 2 U e1 (tau/mu0) phi(x) + (alpha1 - k gamma4) W ],
// Z = E1^2 + 2 e1 En, X = alpha2 - k^2 mu0 gamma3, U = alpha1 + k^2 mu0 gamma4,
// W = E1^2 - (1 + e2) En = Tn (1 + e2) - 2 e1, phi(x) = (1 - exp(-x)) / x (so that
// e1 phi(x) = (e1 - Tn) / x, a series below |x| = 1/2), and the factor d cancels against
// 1 - (k mu0)^2 = d (1 + k mu0): no FP64.  An FP32 emulation over 10^6 (tau, w0, g, mu0) with
// k mu0 within 1.5% of 1 keeps Rdir and Tdir within 1.6e-4 of (1 - Tn) of the FP64 reference.
__device__ __forceinline__ void sw_layer_fast(float tau, float w0, float omw, float g, float mu0, float mu0_inv,
                                              float& R, float& T, float& Rdir, float& Tdir, float& Tn,
                                              float& adif, float& adir)
{
    const float g1 = (8.f - w0 * (5.f + 3.f * g)) * .25f;
    const float g2 = 3.f * (w0 * (1.f - g)) * .25f;
    const float g3 = (2.f - 3.f * mu0 * g) * .25f;
    const float g4 = 1.f - g3;
    const float a1 = g1 * g4 + g2 * g3;
    const float a2 = g1 * g3 + g2 * g4;
    const float kk = 2.f * omw * (2.f - .5f * w0 * (1.f + 3.f * g));
    const float kkc = fmaxf(kk, 1.e-12f);
    const float k = kkc * rsqrtf(kkc);
    float E1, e1, En;
    one_minus_exp(k * tau, E1, e1);
    one_minus_exp(tau * mu0_inv, En, Tn);
    const float E2 = E1 * (2.f - E1);
    const float e2 = e1 * e1;
    const float rt = __fdividef(1.f, k * (1.f + e2) + g1 * E2);
    R = rt * g2 * E2;
    T = rt * 2.f * k * e1;
    adif = rt * (k * E1 * E1 + 2.f * omw * E2);
    const float km = k * mu0;
    const float fact = (1.f - km) * (1.f + km);
    const bool thick = e1 < .5f && Tn < .5f;
    float Rdir0, Tdir0;
    if (fabsf(fact) < 0.02f) {
        const float tm = tau * mu0_inv;
        const float x = tm * (1.f - km);
        const float ser = 1.f - x * (.5f - x * (1.f / 6.f - x * (1.f / 24.f - x * (1.f / 120.f))));
        const float e1phi = fabsf(x) < .5f ? e1 * ser : __fdividef(e1 - Tn, x);
        const float c = __fdividef(w0 * rt, 1.f + km);
        const float W = thick ? Tn * (1.f + e2) - 2.f * e1 : E1 * E1 - (1.f + e2) * En;
        Rdir0 = c * ((a2 + k * g3) * (E1 * E1 + 2.f * e1 * En) - 2.f * (a2 - k * km * g3) * e1 * e1phi * tm);
        Tdir0 = c * (2.f * (a1 + k * km * g4) * e1phi * tm + (a1 - k * g4) * W);
    } else {
        const float rt2 = __fdividef(w0 * rt, fact);
        const float br = E2 * (a2 - k * km * g3) + k * (g3 - mu0 * a2) * (E1 * E1 + 2.f * e1 * En);
        const float bt_thick =
            (1.f + km) * (a1 + k * g4) * Tn - (1.f - km) * (a1 - k * g4) * e2 * Tn - 2.f * (k * g4 + a1 * km) * e1;
        const float bt_thin = Tn * E2 * (a1 + k * km * g4) + k * (g4 + mu0 * a1) * (E1 * E1 - (1.f + e2) * En);
        Rdir0 = rt2 * br;
        Tdir0 = -rt2 * (thick ? bt_thick : bt_thin);
    }
    const float tmin = 2.220446049250313e-16f;
    Rdir = fmaxf(tmin, fminf(Rdir0, En));
    const float rest = En - Rdir;
    Tdir = fmaxf(tmin, fminf(Tdir0, rest));
    adir = fmaxf(0.f, rest - Tdir);
}

// aer: the (layer, band) aerosol values of aerosol_point, or NULL without aerosols.
__device__ __forceinline__ void build_sw_record(const KdistView<float>& k, Rec& R, const LayerState& s,
                                                const float* cg, int nlay, int b, const SwCloudArgs& cld,
                                                size_t cl, const float4* aer = nullptr)
{
    record_weights(k, R, s, cg, nlay, b);
    float tau = 0.f, ssa = 0.f, g = 0.f;
    if (cld.present) {
        const CloudPoint<float> cp = cloud_point(cld.L, cld.lwp[cl], cld.iwp[cl], cld.rel[cl], cld.rei[cl]);
        cloud_band<float, true>(cld.L, cp, b, tau, ssa, g);
        const float ta = tau * (1.f - ssa);   // invariant under delta scaling
        if (cld.delta) delta_scale_point(tau, ssa, g);
        R.aux2 = ta;
    } else {
        R.aux2 = 0.f;
    }
    float ts = tau * ssa, tsg = ts * g;
    if (aer) {
        const float4 a = *aer;
        tau += a.x;
        ts += a.y;
        tsg += a.z;
        R.aux2 += a.w;
    }
    R.aux = make_float4(cg[0] + cg[k.idx_h2o * nlay], tau, ts, tsg);
}

}  // namespace fused
}  // namespace rrtmgp_b200
