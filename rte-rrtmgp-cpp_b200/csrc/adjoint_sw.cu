// Hand-written adjoint of the fused shortwave column forward (forward_sw.cu): gradients of
//   L = sum_l (a_l F_up,l + b_l F_dn,l + c_l F_dir,l) + sum_i e_i HR_i
// (F_dn includes the direct beam) with respect to the layer temperatures, the h2o and o3
// volume mixing ratios, the cloud water paths and effective radii, and the surface albedos.
// No reference counterpart exists.
//
// Layout: one thread-block cluster per column, CS = ceil(nlay / 64) CTAs of 8 warps; warp
// w of CTA r owns the 8-layer chunk W = 8 r + w.  With 8 warps per CTA every thread has up to
// 255 registers, enough to keep the ~16 per-layer values of the reverse sweeps of a chunk in
// registers; chunk composites are exchanged through distributed shared memory with cluster
// barriers.  Per group of 32 g-points the forward is recomputed (records, optical properties,
// two-stream, direct beam, adding: as forward_sw.cu) and then reversed:
//   F_i   (adjoint of the diffuse downward flux fd_i, bottom up)
//         Fraw_i = T_i den_i Fc_(i+1) + b_i + h_i adif_i + a_i ubar_i^0,
//         Fc_(i+1) = Fraw_(i+1) + h_i adif_i a_(i+1)
//   (Abar, Sbar)_i (adjoints of the albedo a_i and upward source s_i, top down)
//         Abar_(i+1) = (T den)^2 Abar_i + T den^2 (sdn + R s_(i+1)) Sbar_i + fd_(i+1) (R den Fc_(i+1) + ubar_(i+1))
//         Sbar_(i+1) = T den Sbar_i + R den Fc_(i+1) + ubar_(i+1),  ubar_l = a_l + h_(l-1) adif_(l-1)
//   Dbar_i (adjoint of the direct flux, bottom up)
//         Dbar_i = b_i + c_i + h_i adir_i + sup_bar_i Rdir_i + sdn_bar_i Tdir_i + Tn_i Dbar_(i+1)
// (den_i = 1 / (1 - R_i a_(i+1)), h_i = g/cp 86400 e_i / dp_i; HR is the per-layer absorbed
// flux A_i = F_dir,i adir_i + (fd_i + fu_(i+1)) adif_i as in the forward).  Each recurrence is
// affine in its adjoint (the albedo/source pair is 2x2 upper triangular), so chunks compose
// exactly like the forward.  Per layer the adjoints of (R, T, Rdir, Tdir, Tn, adif, adir)
// go through the two-stream (reverse mode of the forward's FP32 formulas with its branch
// selections, the k mu0 = 1 form of sw_common.cuh included), the
// gas/Rayleigh/cloud combination, and the gas-optics interpolation (adjoint_common.cuh).
#include <cooperative_groups.h>

#include "adjoint_common.cuh"
#include "dual.cuh"
#include "sw_common.cuh"

namespace cg = cooperative_groups;

namespace rrtmgp_b200 {
namespace {

using namespace fused;

constexpr int kLPC = 64;           // layers per CTA: 8 warps of 8 layers, or 16 warps of 4
// Layers per warp of the launched kernel.  CL = 4 (16 warps per SM at 128 registers, 456 bytes
// of spills) measured the same as CL = 8 (8 warps at 255 registers) at 8192 x 128: 33.9 vs
// 33.4 ms; the occupancy it gains goes into spills and twice the chunk compositions.
constexpr int kSwAdjointChunk = 8;

struct SwAdjOut {
    float* tlay;
    float* h2o;
    float* o3;
    float* lwp;
    float* iwp;
    float* rel;
    float* rei;
    float* alb_dir;
    float* alb_dif;
    // forward fluxes, written when the kernel is instantiated with FLUX (else unused)
    float* flux_up;
    float* flux_dn;
    float* flux_dir;
    float* flux_net;
    float* heating_rate;
};

using D4 = Dual<4>;

// Minor-interval code n < 3 (contributor << kScalBits | scaling kind) of a g-point's list
// (minor_entry); codes 4, 5, ... come from gx = minor_gx[a] + g * minor_gx_stride.
__device__ __forceinline__ int minor_code(const int4& mg, int n)
{
    return n == 0 ? mg.y : (n == 1 ? mg.z : mg.w);
}

// Adjoint of one (layer, g-point) from the adjoints of its two-stream outputs (R, T, Rdir,
// Tdir, Tn, adif, adir) to the optical inputs of the layer: gas absorption tau (x), Rayleigh
// tau (y), cloud tau (z), cloud tau*ssa (w) and cloud tau*ssa*g (v).  The combination is
// tau = ta + tr + tc, w0 = (tr + tsc) / tau, g = tsgc / (tr + tsc).  Reverse mode of
// sw_layer_fast: the forward is recomputed with the same expressions and branch selections
// (clamps: the selected argument carries the derivative, as min/max of dual numbers would),
// then the adjoints run back through it, in the k mu0 = 1 region through its factored form.
struct LocalAdj {
    float ta, tr, tc, tsc, tsg;
};

__device__ __forceinline__ LocalAdj sw_local_adjoint(float tau, float w0, float omw, float g, float mu0, float mu0_inv,
                                                     float Rb, float Tb, float Rdb, float Tdb, float Tnb, float Afb,
                                                     float Arb)
{
    // ---- forward, as sw_layer_fast (same expressions, same branch selections) ----
    const float g1 = (8.f - w0 * (5.f + 3.f * g)) * .25f;
    const float g2 = 3.f * (w0 * (1.f - g)) * .25f;
    const float g3 = (2.f - 3.f * mu0 * g) * .25f;
    const float g4 = 1.f - g3;
    const float a1 = g1 * g4 + g2 * g3;
    const float a2 = g1 * g3 + g2 * g4;
    const float kq = 2.f - .5f * w0 * (1.f + 3.f * g);
    const float kk = 2.f * omw * kq;
    const bool kk_on = kk > 1.e-12f;
    const float kkc = fmaxf(kk, 1.e-12f);
    const float rk = rsqrtf(kkc);   // 1 / k
    const float k = kkc * rk;
    float E1, e1, En, Tn;
    one_minus_exp(k * tau, E1, e1);
    one_minus_exp(tau * mu0_inv, En, Tn);
    const float E2 = E1 * (2.f - E1);
    const float e2 = e1 * e1;
    const float den = k * (1.f + e2) + g1 * E2;
    const float rt = __fdividef(1.f, den);
    const float km = k * mu0;
    const float fact = (1.f - km) * (1.f + km);
    const bool near1 = fabsf(fact) < 0.02f;   // k mu0 = 1 form (sw_layer_fast)
    float Rdir0, Tdir0, rt2 = 0.f, br = 0.f, bt = 0.f;
    const bool thick = e1 < .5f && Tn < .5f;
    // k mu0 = 1 form (sw_layer_fast): d = 1 - k mu0 factored out of both brackets
    const float tmu = tau * mu0_inv, xi = tmu * (1.f - km);
    const bool xs = fabsf(xi) < .5f;
    const float ser = 1.f - xi * (.5f - xi * (1.f / 6.f - xi * (1.f / 24.f - xi * (1.f / 120.f))));
    float e1phi = 0.f, cI = 0.f, WI = 0.f, BR = 0.f, BT = 0.f;
    const float XI = a2 - k * km * g3, UI = a1 + k * km * g4, ZI = E1 * E1 + 2.f * e1 * En;
    if (near1) {
        e1phi = xs ? e1 * ser : __fdividef(e1 - Tn, xi);
        cI = __fdividef(w0 * rt, 1.f + km);
        WI = thick ? Tn * (1.f + e2) - 2.f * e1 : E1 * E1 - (1.f + e2) * En;
        BR = (a2 + k * g3) * ZI - 2.f * XI * e1 * e1phi * tmu;
        BT = 2.f * UI * e1phi * tmu + (a1 - k * g4) * WI;
        Rdir0 = cI * BR;
        Tdir0 = cI * BT;
    } else {
        rt2 = __fdividef(w0 * rt, fact);
        br = E2 * (a2 - k * km * g3) + k * (g3 - mu0 * a2) * (E1 * E1 + 2.f * (e1 * En));
        if (thick)
            bt = (1.f + km) * (a1 + k * g4) * Tn - (1.f - km) * (a1 - k * g4) * e2 * Tn - 2.f * ((k * g4 + a1 * km) * e1);
        else
            bt = Tn * E2 * (a1 + k * km * g4) + k * (g4 + mu0 * a1) * (E1 * E1 - (1.f + e2) * En);
        Rdir0 = rt2 * br;
        Tdir0 = -(rt2 * bt);
    }
    const float tmin = 2.220446049250313e-16f;
    const bool r_lo = Rdir0 <= En;                 // min(Rdir0, En) takes Rdir0
    const float rm = r_lo ? Rdir0 : En;
    const bool r_on = !(tmin >= rm);               // max(tmin, .) takes the value
    const float Rdir = r_on ? rm : tmin;
    const float rest = En - Rdir;
    const bool t_lo = Tdir0 <= rest;
    const float tm = t_lo ? Tdir0 : rest;
    const bool t_on = !(tmin >= tm);
    const float Tdir = t_on ? tm : tmin;
    const bool a_on = !(0.f >= rest - Tdir);

    // ---- reverse ----
    float rest_b = 0.f, Tdir_b = Tdb, Rdir_b = Rdb, En_b = 0.f, Tn_b = Tnb;
    if (a_on) { rest_b += Arb; Tdir_b -= Arb; }
    float Tdir0_b = 0.f;
    if (t_on) {
        if (t_lo) Tdir0_b = Tdir_b; else rest_b += Tdir_b;
    }
    En_b += rest_b;
    Rdir_b -= rest_b;
    float Rdir0_b = 0.f;
    if (r_on) {
        if (r_lo) Rdir0_b = Rdir_b; else En_b += Rdir_b;
    }
    float tau_b = 0.f, w0_b = 0.f, g_b = 0.f, omw_b = 0.f;
    float k_b = 0.f, km_b = 0.f, rt_b = 0.f, E1_b = 0.f, e1_b = 0.f, E2_b = 0.f, e2_b = 0.f;
    float g1_b = 0.f, g2_b = 0.f, g3_b = 0.f, g4_b = 0.f, a1_b = 0.f, a2_b = 0.f;
    if (near1) {
        // reverse of Rdir0 = c BR, Tdir0 = c BT (the k mu0 = 1 form above)
        const float c_b = Rdir0_b * BR + Tdir0_b * BT;
        const float BR_b = Rdir0_b * cI, BT_b = Tdir0_b * cI;
        a2_b += BR_b * ZI;
        k_b += BR_b * g3 * ZI;
        g3_b += BR_b * k * ZI;
        const float Z_b = BR_b * (a2 + k * g3);
        const float P_b = -2.f * BR_b;                 // P = X e1 e1phi tm
        const float X_b = P_b * e1 * e1phi * tmu;
        e1_b += P_b * XI * e1phi * tmu;
        float e1phi_b = P_b * XI * e1 * tmu;
        float tm_b = P_b * XI * e1 * e1phi;
        const float Q_b = 2.f * BT_b;                  // Q = U e1phi tm
        const float U_b = Q_b * e1phi * tmu;
        e1phi_b += Q_b * UI * tmu;
        tm_b += Q_b * UI * e1phi;
        a1_b += BT_b * WI;
        k_b -= BT_b * g4 * WI;
        g4_b -= BT_b * k * WI;
        const float W_b = BT_b * (a1 - k * g4);
        E1_b += Z_b * 2.f * E1;
        e1_b += Z_b * 2.f * En;
        En_b += Z_b * 2.f * e1;
        a2_b += X_b;
        k_b -= X_b * km * g3;
        km_b -= X_b * k * g3;
        g3_b -= X_b * k * km;
        a1_b += U_b;
        k_b += U_b * km * g4;
        km_b += U_b * k * g4;
        g4_b += U_b * k * km;
        if (thick) {
            Tn_b += W_b * (1.f + e2);
            e2_b += W_b * Tn;
            e1_b -= 2.f * W_b;
        } else {
            E1_b += W_b * 2.f * E1;
            e2_b -= W_b * En;
            En_b -= W_b * (1.f + e2);
        }
        // divisions of the reverse mode as products with approximate reciprocals, like the
        // forward's __fdividef (an IEEE division is a multi-instruction sequence)
        const float i1km = __fdividef(1.f, 1.f + km);
        w0_b += c_b * rt * i1km;
        rt_b += c_b * w0 * i1km;
        km_b -= c_b * cI * i1km;
        float x_b;
        if (xs) {
            const float dser = -.5f + xi * (1.f / 3.f - xi * (1.f / 8.f - xi * (1.f / 30.f)));
            e1_b += e1phi_b * ser;
            x_b = e1phi_b * e1 * dser;
        } else {
            const float ixi = __fdividef(1.f, xi);
            e1_b += e1phi_b * ixi;
            Tn_b -= e1phi_b * ixi;
            x_b = -e1phi_b * e1phi * ixi;
        }
        tm_b += x_b * (1.f - km);
        km_b -= x_b * tmu;
        tau_b += tm_b * mu0_inv;
    } else {
        const float rt2_b = Rdir0_b * br - Tdir0_b * bt;
        const float br_b = Rdir0_b * rt2;
        const float bt_b = -Tdir0_b * rt2;
        // br = E2 X + k Y Z
        const float X = a2 - k * km * g3, Y = g3 - mu0 * a2, Z = E1 * E1 + 2.f * (e1 * En);
        E2_b += br_b * X;
        const float X_b = br_b * E2;
        a2_b += X_b;
        k_b -= X_b * km * g3;
        km_b -= X_b * k * g3;
        g3_b -= X_b * k * km;
        k_b += br_b * Y * Z;
        const float Y_b = br_b * k * Z, Z_b = br_b * k * Y;
        g3_b += Y_b;
        a2_b -= Y_b * mu0;
        E1_b += Z_b * 2.f * E1;
        e1_b += Z_b * 2.f * En;
        En_b += Z_b * 2.f * e1;
        if (thick) {
            const float P = a1 + k * g4, Q = a1 - k * g4, S = k * g4 + a1 * km;
            const float P_b = bt_b * (1.f + km) * Tn, Q_b = -bt_b * (1.f - km) * e2 * Tn, S_b = -2.f * bt_b * e1;
            km_b += bt_b * (P * Tn + Q * e2 * Tn);
            Tn_b += bt_b * ((1.f + km) * P - (1.f - km) * Q * e2);
            e2_b -= bt_b * (1.f - km) * Q * Tn;
            e1_b -= 2.f * bt_b * S;
            a1_b += P_b + Q_b + S_b * km;
            k_b += (P_b - Q_b) * g4 + S_b * g4;
            g4_b += (P_b - Q_b) * k + S_b * k;
            km_b += S_b * a1;
        } else {
            const float U = a1 + k * km * g4, V = g4 + mu0 * a1, W2 = E1 * E1 - (1.f + e2) * En;
            Tn_b += bt_b * E2 * U;
            E2_b += bt_b * Tn * U;
            const float U_b = bt_b * Tn * E2;
            a1_b += U_b;
            k_b += U_b * km * g4;
            km_b += U_b * k * g4;
            g4_b += U_b * k * km;
            k_b += bt_b * V * W2;
            const float V_b = bt_b * k * W2, W2_b = bt_b * k * V;
            g4_b += V_b;
            a1_b += V_b * mu0;
            E1_b += W2_b * 2.f * E1;
            e2_b -= W2_b * En;
            En_b -= W2_b * (1.f + e2);
        }
        // rt2 = w0 rt / fact, fact = 1 - km^2
        const float ifact = __fdividef(1.f, fact);
        w0_b += rt2_b * rt * ifact;
        rt_b += rt2_b * w0 * ifact;
        const float fact_b = -rt2_b * rt2 * ifact;
        km_b -= fact_b * 2.f * km;
    }
    k_b += km_b * mu0;
    // R, T, adif
    const float Aq = k * E1 * E1 + 2.f * omw * E2;
    rt_b += Rb * g2 * E2 + Tb * 2.f * k * e1 + Afb * Aq;
    g2_b += Rb * rt * E2;
    E2_b += Rb * rt * g2 + Afb * rt * 2.f * omw;
    k_b += Tb * 2.f * rt * e1 + Afb * rt * E1 * E1;
    e1_b += Tb * 2.f * rt * k;
    E1_b += Afb * rt * 2.f * k * E1;
    omw_b += Afb * rt * 2.f * E2;
    // rt = 1 / den, den = k (1 + e2) + g1 E2
    const float den_b = -rt_b * rt * rt;
    k_b += den_b * (1.f + e2);
    e2_b += den_b * k;
    g1_b += den_b * E2;
    E2_b += den_b * g1;
    // E2 = E1 (2 - E1), e2 = e1^2
    E1_b += E2_b * (2.f - 2.f * E1);
    e1_b += e2_b * 2.f * e1;
    // (E1, e1) = one_minus_exp(k tau): dE1/dx = e1, de1/dx = -e1
    const float x1_b = e1 * (E1_b - e1_b);
    k_b += x1_b * tau;
    tau_b += x1_b * k;
    const float xn_b = Tn * (En_b - Tn_b);
    tau_b += xn_b * mu0_inv;
    // k = sqrt(max(kk, 1e-12)), kk = 2 omw kq
    const float kk_b = kk_on ? k_b * 0.5f * rk : 0.f;
    omw_b += kk_b * 2.f * kq;
    w0_b += kk_b * 2.f * omw * (-.5f * (1.f + 3.f * g));
    g_b += kk_b * 2.f * omw * (-1.5f * w0);
    // a1, a2, g1..g4
    g1_b += a1_b * g4 + a2_b * g3;
    g4_b += a1_b * g1 + a2_b * g2;
    g2_b += a1_b * g3 + a2_b * g4;
    g3_b += a1_b * g2 + a2_b * g1;
    g3_b -= g4_b;
    g_b += g3_b * (-.75f * mu0);
    w0_b += g2_b * .75f * (1.f - g) - g1_b * (5.f + 3.f * g) * .25f;
    g_b += -g2_b * .75f * w0 - g1_b * .75f * w0;
    // omw = 1 - w0 (formed separately for accuracy): total derivative along w0
    const float taub = tau_b, w0b = w0_b - omw_b, gb = g_b;

    const bool okt = tau > 2.f * FLT_MIN;
    const float ts = w0 * tau;
    const bool oks = ts > 3.f * FLT_MIN;
    const float itau = okt ? __fdividef(1.f, tau) : 0.f;
    const float its = oks ? __fdividef(1.f, ts) : 0.f;
    LocalAdj r;
    r.ta = taub - w0b * w0 * itau;
    r.tr = taub + w0b * omw * itau - gb * g * its;
    r.tc = taub - w0b * w0 * itau;
    r.tsc = w0b * itau - gb * g * its;
    r.tsg = gb * its;
    return r;
}

// Adjoint of one (layer, g-point) through the two-stream (sw_local_adjoint) and the gas optics:
// the absorption tau_bar through the major and minor interpolation (as tau_abs_adjoint of
// adjoint_common.cuh) and the Rayleigh tau_bar through col_rayl * (fm . krayl corners).  The
// table corners are read first, so their latency overlaps the two-stream adjoint.  Out of
// line: the caller's per-layer loops are unrolled 8 times and, inlined, these bodies made the
// kernel's code outgrow the instruction cache (10% of the kernel time).
struct LayerAdj {
    float t, h, o;          // d/dT, d/d vmr_h2o, d/d vmr_o3
    float tc, tsc, tsg;     // adjoints of the cloud tau, tau*ssa, tau*ssa*g
};

template <bool DENSE>
__device__ __noinline__ LayerAdj sw_layer_adjoint(const float4* __restrict__ kmaj4, const float2* __restrict__ kmin,
                                                  const float2* __restrict__ krayl2, const Rec* Rc, const DRec* DR,
                                                  const float4* sc4, const int* gx, int g, int4 mg, int nmax,
                                                  float tau, float w0, float omw, float gasy, float mu0, float mu0_inv,
                                                  float Rb, float Tb, float Rdb, float Tdb, float Tnb, float Afb,
                                                  float Arb)
{
    const float4 c0 = __ldg(kmaj4 + (Rc->kb.x + g));
    const float4 c1 = __ldg(kmaj4 + (Rc->kb.y + g));
    float4 cr[3];
#pragma unroll
    for (int n = 0; n < 3; ++n) {
        cr[n] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (n < nmax) {
            const int c = minor_code(mg, n) >> kScalBits;
            const float2 lo = __ldg(kmin + (Rc->kb.z + c));
            const float2 hi = __ldg(kmin + (Rc->kb.w + c));
            cr[n] = make_float4(lo.x, lo.y, hi.x, hi.y);
        }
    }
    const float2 r0 = __ldg(krayl2 + (Rc->kr[0] + g));
    const float2 r1 = __ldg(krayl2 + (Rc->kr[1] + g));

    const LocalAdj la = sw_local_adjoint(tau, w0, omw, gasy, mu0, mu0_inv, Rb, Tb, Rdb, Tdb, Tnb, Afb, Arb);

    float dT = dot4(DR->wT0, c0) + dot4(DR->wT1, c1);
    float dH = dot4(DR->wH0, c0) + dot4(DR->wH1, c1);
    float dO = dot4(DR->wO0, c0) + dot4(DR->wO1, c1);
    auto minor_term = [&](int code, const float4& crn, bool on) {
        const float M = dot4(Rc->fm, crn);
        const float4 S = sc4[code & (kMaxScal - 1)];   // scaling, d ln / dT, d / d h2o, d / d o3
        const float tT = S.x * (S.y * M + dot4(DR->fmT, crn));
        const float tH = S.z * M + S.x * dot4(DR->fmH, crn);
        const float tO = S.w * M + S.x * dot4(DR->fmO, crn);
        dT += on ? tT : 0.f;
        dH += on ? tH : 0.f;
        dO += on ? tO : 0.f;
    };
#pragma unroll
    for (int n = 0; n < 3; ++n)
        if (n < nmax) minor_term(minor_code(mg, n), cr[n], n < mg.x);
    if constexpr (DENSE) {   // more than three intervals over some g-point
        for (int n = 3; n < nmax; ++n) {
            const int code = n < mg.x ? gx[n - 3] : mg.y;
            const int c = code >> kScalBits;
            const float2 lo = __ldg(kmin + (Rc->kb.z + c));
            const float2 hi = __ldg(kmin + (Rc->kb.w + c));
            minor_term(code, make_float4(lo.x, lo.y, hi.x, hi.y), n < mg.x);
        }
    }
    const float tab = la.ta, trb = la.tr;
    LayerAdj r{tab * dT, tab * dH, tab * dO, la.tc, la.tsc, la.tsg};
    const float4 kr = make_float4(r0.x, r0.y, r1.x, r1.y);
    const float colr = Rc->aux.x;
    r.t += trb * colr * dot4(DR->fmT, kr);
    r.h += trb * (colr * dot4(DR->fmH, kr) + DR->dB.x * dot4(Rc->fm, kr));
    r.o += trb * colr * dot4(DR->fmO, kr);
    return r;
}

// Forward optical properties and two-stream coefficients of one (layer, g-point), as the
// forward kernel's pass 1 (sw_column.cuh), out of line for the same reason.
struct LayerFwd { float tau, w0, omw, gasy, R, T, Rdir, Tdir, Tn, adif, adir; };

template <bool DENSE>
__device__ __noinline__ LayerFwd sw_layer_forward(const float4* __restrict__ kmaj4, const float2* __restrict__ kmin,
                                                  const float2* __restrict__ krayl2, const Rec* Rc, const float4* sc4,
                                                  const int* gx, int g, int4 mg, int nmax, float mu0, float mu0_inv)
{
    const float4 c0 = __ldg(kmaj4 + (Rc->kb.x + g));
    const float4 c1 = __ldg(kmaj4 + (Rc->kb.y + g));
    float ta = dot4(Rc->wmaj0, c0) + dot4(Rc->wmaj1, c1);
    auto minor_term = [&](int code, bool on) {
        const int c = code >> kScalBits;
        const float2 lo = __ldg(kmin + (Rc->kb.z + c));
        const float2 hi = __ldg(kmin + (Rc->kb.w + c));
        const float t = sc4[code & (kMaxScal - 1)].x *
                        (Rc->fm.x * lo.x + Rc->fm.y * lo.y + Rc->fm.z * hi.x + Rc->fm.w * hi.y);
        ta += on ? t : 0.f;
    };
#pragma unroll
    for (int n = 0; n < 3; ++n)
        if (n < nmax) minor_term(minor_code(mg, n), n < mg.x);
    if constexpr (DENSE)
        for (int n = 3; n < nmax; ++n) minor_term(n < mg.x ? gx[n - 3] : mg.y, n < mg.x);
    LayerFwd o;
    const float2 r0 = __ldg(krayl2 + (Rc->kr[0] + g));
    const float2 r1 = __ldg(krayl2 + (Rc->kr[1] + g));
    const float tr = (Rc->fm.x * r0.x + Rc->fm.y * r0.y + Rc->fm.z * r1.x + Rc->fm.w * r1.y) * Rc->aux.x;
    o.tau = ta + tr + Rc->aux.y;
    const float ts = tr + Rc->aux.z;
    o.w0 = 0.f;
    o.omw = 1.f;
    if (o.tau > 2.f * FLT_MIN) {
        const float inv = __fdividef(1.f, o.tau);
        o.w0 = ts * inv;
        o.omw = (ta + Rc->aux2) * inv;
    }
    o.gasy = __fdividef(Rc->aux.w, fmaxf(ts, 3.f * FLT_MIN));
    sw_layer_fast(o.tau, o.w0, o.omw, o.gasy, mu0, mu0_inv, o.R, o.T, o.Rdir, o.Tdir, o.Tn, o.adif, o.adir);
    return o;
}

// Cloud optics of band b (2str, optionally delta-scaled) as duals over (lwp, iwp, rel, rei):
// returns tau', tau' ssa', tau' ssa' g' as used by the SW record.
__device__ __forceinline__ void cloud_sw_dual(const CloudLut<float>& L, int delta, float lwp, float iwp, float rel,
                                              float rei, int b, D4& tau, D4& ts, D4& tsg)
{
    const CloudPoint<float> c = cloud_point(L, lwp, iwp, rel, rei);
    const size_t nl = size_t(L.nband) * L.nsl, ni = size_t(L.nband) * L.nsi;
    D4 lt = dconst<4>(0.f), lts = dconst<4>(0.f), ltg = dconst<4>(0.f);
    D4 it = dconst<4>(0.f), its = dconst<4>(0.f), itg = dconst<4>(0.f);
    auto lerp = [](const float* t, int i, const D4& f) {
        const float d = t[i + 1] - t[i];
        D4 r;
        r.v = t[i] + f.v * d;
#pragma unroll
        for (int q = 0; q < 4; ++q) r.d[q] = f.d[q] * d;
        return r;
    };
    if (c.lwp > 0.f) {
        D4 fl = dconst<4>(c.fl);
        fl.d[2] = 1.f / L.liq_step;
        const float* le = L.lut + size_t(b) * L.nsl;
        lt = dvar<4>(c.lwp, 0) * lerp(le, c.il, fl);
        lts = lt * lerp(le + nl, c.il, fl);
        ltg = lts * lerp(le + 2 * nl, c.il, fl);
    }
    if (c.iwp > 0.f) {
        D4 fi = dconst<4>(c.fi);
        fi.d[3] = 1.f / L.ice_step;
        const float* ie = L.lut + 3 * nl + size_t(b) * L.nsi;
        it = dvar<4>(c.iwp, 1) * lerp(ie, c.ii, fi);
        its = it * lerp(ie + ni, c.ii, fi);
        itg = its * lerp(ie + 2 * ni, c.ii, fi);
    }
    const float eps = FLT_EPSILON;
    D4 t = lt + it;
    const D4 s_num = lts + its;
    D4 ssa = ddiv(s_num, t.v > eps ? t : dconst<4>(eps), false);
    D4 g = ddiv(ltg + itg, s_num.v > eps ? s_num : dconst<4>(eps), false);
    if (delta) {
        const float e3 = 3.f * FLT_MIN;
        const D4 f = g * g;
        const D4 wf = ssa * f;
        t = t * (1.f - wf);
        const D4 d1 = 1.f - wf, d2 = 1.f - f;
        ssa = ddiv(ssa - wf, d1.v > e3 ? d1 : dconst<4>(e3), false);
        g = ddiv(g - f, d2.v > e3 ? d2 : dconst<4>(e3), false);
    }
    tau = t;
    ts = t * ssa;
    tsg = ts * g;
}

struct SwAdjLayout {
    size_t state, cg, scal, aer, seeds, clsum, albacc, x1, x2, x3, x4, x5, recs, drecs, total;
};

// aer: aerosol values per (band, local layer) when aerosols are present (aerosol_point).
__host__ __device__ __forceinline__ SwAdjLayout sw_adj_layout(int ngas, int nband, int mgb, int CS, int WPC,
                                                              int nbuf, int nscal, bool aer)
{
    SwAdjLayout L;
    L.state = 0;
    L.cg = align16(L.state + sizeof(LayerState) * kLPC);
    L.scal = align16(L.cg + sizeof(float) * size_t(ngas + 1) * kLPC);
    L.aer = align16(L.scal + sizeof(float4) * size_t(nscal) * kLPC);
    L.seeds = align16(L.aer + (aer ? sizeof(float4) * size_t(nband) * kLPC : 0));
    L.clsum = align16(L.seeds + sizeof(float) * (4 * (kLPC + 1)));
    L.albacc = align16(L.clsum + sizeof(float) * size_t(nband) * kLPC * 3);
    L.x1 = align16(L.albacc + sizeof(double) * size_t(nband) * 2);
    // chunk maps of every chunk of the cluster (each warp pushes its map to all CTAs)
    const size_t nw = size_t(WPC) * CS * 32;
    L.x2 = align16(L.x1 + sizeof(float) * nw);
    L.x3 = align16(L.x2 + (sizeof(float4) + sizeof(float)) * nw);
    L.x4 = align16(L.x3 + sizeof(float2) * nw);
    L.x5 = align16(L.x4 + (sizeof(float4) + sizeof(float)) * nw);
    L.recs = align16(L.x5 + sizeof(float2) * nw);
    L.drecs = align16(L.recs + sizeof(Rec) * size_t(kLPC) * mgb * nbuf);
    L.total = align16(L.drecs + sizeof(DRec) * size_t(kLPC) * mgb * nbuf);
    return L;
}

template <typename Tp>
__device__ __forceinline__ Tp* remote(cg::cluster_group& cl, Tp* p, int rank)
{
    return cl.map_shared_rank(p, rank);
}

// CL layers per warp, kLPC / CL warps per CTA: CL = 8 gives 8 warps with up to 255 registers,
// CL = 4 gives 16 warps at 128 registers (half the per-layer values per thread).
// DENSE: more than three minor intervals over some g-point (sw_layer_forward/adjoint).
template <int CL, bool FLUX, bool PAIR, bool DENSE>
__global__ void __launch_bounds__(kLPC / CL * 32, 1)
sw_adjoint_kernel(const KdistView<float> k, const GasSet<float> gs, const SwCloudArgs cld, int ncol, int nlay, int CS,
                  int idx_o3, int cd_internal, const float* __restrict__ play, const float* __restrict__ plev,
                  const float* __restrict__ tlay, const float* __restrict__ col_dry_in,
                  const float* __restrict__ mu0_in, const float* __restrict__ tsi_scaling,
                  const float* __restrict__ alb_dir, const float* __restrict__ alb_dif,
                  const float* __restrict__ seed_up, const float* __restrict__ seed_dn,
                  const float* __restrict__ seed_dir, const float* __restrict__ seed_hr, const SwAdjOut out,
                  const SwAerosolArgs aer)
{
    constexpr int WPC = kLPC / CL;   // warps per CTA
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = int(cluster.block_rank());
    const int icol = blockIdx.x / CS;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int Wg = rank * WPC + w;
    const int NWt = CS * WPC;
    const int L_end = NWt * CL;
    const int j0 = rank * kLPC;          // first global layer of this CTA
    const int nband = k.nband, mgb = k.max_group_bands;
    const SwAdjLayout SL = sw_adj_layout(k.ngas, nband, mgb, CS, WPC, PAIR ? 2 : 1, k.max_nscal, aer.present != 0);
    LayerState* st = reinterpret_cast<LayerState*>(smem_raw + SL.state);
    float* sm_cg = reinterpret_cast<float*>(smem_raw + SL.cg);
    float4* sm_sc4 = reinterpret_cast<float4*>(smem_raw + SL.scal);   // [local layer][scaling kind]
    float4* sm_aer = reinterpret_cast<float4*>(smem_raw + SL.aer);    // [band][local layer] (aerosols)
    float* sm_al = reinterpret_cast<float*>(smem_raw + SL.seeds);   // seed F_up per local level (0..64)
    float* sm_be = sm_al + (kLPC + 1);                                // seed F_dn
    float* sm_ga = sm_be + (kLPC + 1);                                // seed F_dir
    float* sm_hh = sm_ga + (kLPC + 1);                                // h per local layer
    float* sm_cl = reinterpret_cast<float*>(smem_raw + SL.clsum);     // [band][layer][3] cloud adjoint sums
    double* sm_alb = reinterpret_cast<double*>(smem_raw + SL.albacc); // [band][2]
    float* sm_x1 = reinterpret_cast<float*>(smem_raw + SL.x1);
    float4* sm_x2a = reinterpret_cast<float4*>(smem_raw + SL.x2);
    float* sm_x2b = reinterpret_cast<float*>(sm_x2a + NWt * 32);
    float2* sm_x3 = reinterpret_cast<float2*>(smem_raw + SL.x3);
    float4* sm_x4a = reinterpret_cast<float4*>(smem_raw + SL.x4);
    float* sm_x4b = reinterpret_cast<float*>(sm_x4a + NWt * 32);
    float2* sm_x5 = reinterpret_cast<float2*>(smem_raw + SL.x5);
    Rec* const recs0 = reinterpret_cast<Rec*>(smem_raw + SL.recs) + w * CL * mgb;
    DRec* const drecs0 = reinterpret_cast<DRec*>(smem_raw + SL.drecs) + w * CL * mgb;

    const bool top_at_1 = play[icol] < play[icol + size_t(nlay - 1) * ncol];
    const float mu0 = mu0_in[icol];
    const float mu0_inv = 1.f / mu0;
    const float tsi = tsi_scaling ? tsi_scaling[icol] : 1.f;
    auto seed_at = [&](const float* s, int lev) -> float {   // global level (top down) -> seed
        if (!s || lev > nlay) return 0.f;
        return s[icol + size_t(top_at_1 ? lev : nlay - lev) * ncol];
    };

    // ---- per-CTA set-up: its 64 layers ----
    for (int jl = threadIdx.x; jl < kLPC; jl += blockDim.x) {
        const int j = j0 + jl;
        if (j >= nlay) continue;
        const int l = top_at_1 ? j : nlay - 1 - j;
        const size_t cl = icol + size_t(l) * ncol;
        const float p = play[cl], t = tlay[cl];
        fill_col_gas(k, gs, ncol, nlay, icol, l, plev, col_dry_in, sm_cg + jl, kLPC);
        const LayerInterp<float> li = layer_interp(k, p, t);
        const int lt = top_at_1 ? j : nlay - j, lb = top_at_1 ? j + 1 : nlay - 1 - j;
        LayerState s;
        s.jt = li.jt; s.jp = li.jp; s.itropo = li.itropo; s.pad = 0;
        s.ftemp = li.ftemp; s.fpress = li.fpress; s.p = p; s.t = t;
        s.t_top = 0.f; s.t_bot = 0.f;
        s.dp = fabsf(plev[icol + size_t(lb) * ncol] - plev[icol + size_t(lt) * ncol]);
        s.pad2 = 0.f;
        st[jl] = s;
    }
    for (int ll = threadIdx.x; ll <= kLPC; ll += blockDim.x) {
        sm_al[ll] = seed_at(seed_up, j0 + ll);
        sm_be[ll] = seed_at(seed_dn, j0 + ll);
        sm_ga[ll] = seed_at(seed_dir, j0 + ll);
    }
    for (int i = threadIdx.x; i < nband * kLPC * 3; i += blockDim.x) sm_cl[i] = 0.f;
    for (int i = threadIdx.x; i < nband * 2; i += blockDim.x) sm_alb[i] = 0.0;
    __syncthreads();
    layer_minor_scalings_d(k, st, sm_cg, kLPC, sm_sc4, max(0, min(kLPC, nlay - j0)), idx_o3, cd_internal, threadIdx.x,
                           blockDim.x);
    if (aer.present) {
        const int nloc = max(0, min(kLPC, nlay - j0));
        for (int idx = threadIdx.x; idx < nloc * nband; idx += blockDim.x) {
            const int jl = idx % nloc, b = idx / nloc, j = j0 + jl;
            sm_aer[b * kLPC + jl] = aerosol_point(aer, ncol, icol, top_at_1 ? j : nlay - 1 - j, st[jl].dp, b);
        }
    }
    for (int jl = threadIdx.x; jl < kLPC; jl += blockDim.x) {
        const int j = j0 + jl;
        float h = 0.f;
        if (j < nlay && seed_hr) {
            const int l = top_at_1 ? j : nlay - 1 - j;
            h = float(9.80665 / 1004.64 * 86400.0 * double(seed_hr[icol + size_t(l) * ncol]) / double(st[jl].dp));
        }
        sm_hh[jl] = h;
    }
    __syncthreads();

    const int ngpt = k.ngpt;
    // top / bottom boundary seeds (every thread walks the whole column)
    const float al0 = seed_at(seed_up, 0);
    const float alN = seed_at(seed_up, nlay), beN = seed_at(seed_dn, nlay), gaN = seed_at(seed_dir, nlay);
    double acc_q = 0.0;   // reduce-scatter of [T | H | O | -] x CL: see the output section
    // forward fluxes (FLUX): as the forward kernel, lane L holds value L >> 1 of the chunk's
    // [levels | layers]: acc_fa direct / direct absorbed, acc_fb up / diffuse absorbed,
    // acc_fc diffuse down
    double acc_fa = 0.0, acc_fb = 0.0, acc_fc = 0.0;
    double acc_sfc_dir = 0.0, acc_sfc_dn = 0.0, acc_sfc_up = 0.0;
    constexpr float m_dry = 0.028964f, m_h2o = 0.018016f;

    for (int gg = 0; gg < k.ngroups; ++gg) {
        const int g = 32 * gg + lane;
        const bool gv = g < ngpt;
        const int b0 = k.group_band0[gg];
        const int gband = gv ? k.gpt2band[g] : b0;
        const int slot = gband - b0;
        const int4 mg0 = minor_entry(k.minor_g[0], g, gv);
        const int4 mg1 = minor_entry(k.minor_g[1], g, gv);
        const int nm0 = __reduce_max_sync(0xffffffffu, mg0.x);
        const int nm1 = __reduce_max_sync(0xffffffffu, mg1.x);
        const float ad = gv ? __ldg(alb_dir + gband + size_t(icol) * nband) : 0.f;
        const float af = gv ? __ldg(alb_dif + gband + size_t(icol) * nband) : 0.f;

        // Records (forward and derivative) of every (layer, band) of the group.  With PAIR, the
        // records of groups gg and gg + 1 are built together at even gg into two buffers: with
        // 8 layers and 2 bands a group has 16 records per warp, so one group alone leaves half
        // the lanes idle.
        Rec* const recs = recs0 + (PAIR ? (gg & 1) : 0) * kLPC * mgb;
        DRec* const drecs = drecs0 + (PAIR ? (gg & 1) : 0) * kLPC * mgb;
        if (!PAIR || (gg & 1) == 0) {
            const int nrec = CL * mgb;
            for (int t = lane; t < (PAIR ? 2 : 1) * nrec; t += 32) {
                const int gq = gg + t / nrec, r = t % nrec;
                if (gq >= k.ngroups) continue;
                const int jl = w * CL + (r % CL);
                const int jj = j0 + jl;
                const int b = k.group_band0[gq] + r / CL;
                if (jj < nlay && b < nband && k.band_lims[2 * b] < 32 * gq + 32) {
                    const int qb = PAIR ? (gq & 1) : 0;
                    const int l = top_at_1 ? jj : nlay - 1 - jj;
                    const LayerState s = st[jl];
                    build_sw_record(k, recs0[qb * kLPC * mgb + r], s, sm_cg + jl, kLPC, b, cld, icol + size_t(l) * ncol,
                                    aer.present ? sm_aer + b * kLPC + jl : nullptr);
                    DRec& DR = drecs0[qb * kLPC * mgb + r];
                    build_drec<false>(k, DR, s, sm_cg + jl, kLPC, b, idx_o3, cd_internal);
                    const float cd = sm_cg[jl];
                    const float vh = sm_cg[k.idx_h2o * kLPC + jl] / cd;
                    const float dcd_h = cd_internal ? -cd * m_h2o / (m_dry + m_h2o * vh) : 0.f;
                    DR.dB = make_float4(dcd_h * (1.f + vh) + cd, 0.f, 0.f, 0.f);   // d col_rayl / d vmr_h2o
                }
            }
        }
        __syncwarp();

        // ---- forward pass 1 (recomputed): optical properties and two-stream per layer ----
        float vTau[CL], vW0[CL], vOmw[CL], vG[CL];
        float vR[CL], vT[CL], vRd[CL], vTd[CL], vTn[CL], vAf[CL], vAr[CL], vP[CL];
        float P = 1.f;
        float cRu = 0.f, cRd = 0.f, cT = 1.f, cU = 0.f, cD = 0.f;
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            const int jl = w * CL + i;
            const int j = j0 + jl;
            float R = 0.f, T = 1.f, Rdir = 0.f, Tdir = 0.f, Tn = 1.f, adif = 0.f, adir = 0.f;
            float tau = 0.f, w0 = 0.f, omw = 1.f, gasy = 0.f;
            if (j < nlay && gv) {
                const Rec& Rc = recs[slot * CL + i];
                const LayerFwd lf = sw_layer_forward<DENSE>(k.kmaj4, k.kmin2[Rc.a], k.krayl2, &Rc, sm_sc4 + jl * k.max_nscal,
                                                     k.minor_gx[Rc.a] + size_t(g) * k.minor_gx_stride, g,
                                                     Rc.a ? mg1 : mg0, Rc.a ? nm1 : nm0, mu0, mu0_inv);
                tau = lf.tau; w0 = lf.w0; omw = lf.omw; gasy = lf.gasy;
                R = lf.R; T = lf.T; Rdir = lf.Rdir; Tdir = lf.Tdir; Tn = lf.Tn; adif = lf.adif; adir = lf.adir;
            }
            vTau[i] = tau; vW0[i] = w0; vOmw[i] = omw; vG[i] = gasy;
            vR[i] = R; vT[i] = T; vRd[i] = Rdir; vTd[i] = Tdir; vTn[i] = Tn; vAf[i] = adif; vAr[i] = adir;
            vP[i] = P;
            const float su = Rdir * P, sd = Tdir * P;
            const float den = __fdividef(1.f, fmaf(-cRd, R, 1.f));
            const float nRu = cRu + cT * cT * R * den;
            const float nRd = R + T * T * cRd * den;
            const float nU = cU + cT * (su + R * cD) * den;
            const float nD = sd + T * (cD + cRd * su) * den;
            cT = cT * T * den;
            cRu = nRu; cRd = nRd; cU = nU; cD = nD;
            P *= Tn;
        }
        for (int rr = 0; rr < CS; ++rr) remote(cluster, sm_x1, rr)[Wg * 32 + lane] = P;
        cluster.sync();

        // ---- X1: direct flux at the chunk top and the surface ----
        const float toa = gv ? __ldg(k.solar_source + g) * tsi * mu0 : 0.f;
        float dtop = toa;
        for (int c = 0; c < Wg; ++c) dtop *= sm_x1[c * 32 + lane];
        float dsfc = dtop;
        for (int c = Wg; c < NWt; ++c) dsfc *= sm_x1[c * 32 + lane];
        for (int rr = 0; rr < CS; ++rr) {
            remote(cluster, sm_x2a, rr)[Wg * 32 + lane] = make_float4(cRu, cRd, cT, cU * dtop);
            remote(cluster, sm_x2b, rr)[Wg * 32 + lane] = cD * dtop;
        }
        cluster.sync();

        // ---- X2: albedo / source at the chunk bottom, incident diffuse flux at its top ----
        float alb = af, src = dsfc * ad;
        float alb_in = af, src_in = src;
        float fa = 1.f, fb = 0.f;
        for (int c = NWt - 1; c >= 0; --c) {
            if (c == Wg) {
                alb_in = alb;
                src_in = src;
                if (Wg == 0) break;
            }
            const float4 m = sm_x2a[c * 32 + lane];
            const float Dc = sm_x2b[c * 32 + lane];
            const float den = __fdividef(1.f, fmaf(-m.y, alb, 1.f));
            if (c < Wg) {
                const float F = m.z * den, G = fmaf(m.y, src, Dc) * den;
                fb = fmaf(fa, G, fb);
                fa *= F;
            }
            const float nalb = m.x + m.z * m.z * alb * den;
            src = m.w + m.z * fmaf(alb, Dc, src) * den;
            alb = nalb;
        }
        // direct flux per level (level i = top of layer i)
        float vDir[CL];
#pragma unroll
        for (int i = 0; i < CL; ++i) vDir[i] = dtop * vP[i];

        // ---- forward pass 2 (bottom up): albedo a_i and source s_i per level ----
        float vA[CL], vS[CL];
        {
            float a = alb_in, s = src_in;
#pragma unroll
            for (int i = CL - 1; i >= 0; --i) {
                const float su = vRd[i] * vDir[i], sd = vTd[i] * vDir[i];
                const float den = __fdividef(1.f, fmaf(-vR[i], a, 1.f));
                const float na = vR[i] + vT[i] * vT[i] * a * den;
                const float ns = su + vT[i] * fmaf(a, sd, s) * den;
                vA[i] = na;
                vS[i] = ns;
                a = na;
                s = ns;
            }
        }
        // ---- forward pass 3 (top down): diffuse downward flux fd per level ----
        float vFd[CL];
        float fd = fb;
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            vFd[i] = fd;
            const float a_n = (i + 1 < CL) ? vA[i + 1] : alb_in;
            const float s_n = (i + 1 < CL) ? vS[i + 1] : src_in;
            const float den = __fdividef(1.f, fmaf(-vR[i], a_n, 1.f));
            fd = (vT[i] * fd + vR[i] * s_n + vTd[i] * vDir[i]) * den;
        }
        const float fd_bot = fd;
        if (FLUX) {
            float v[2 * CL];
#pragma unroll
            for (int i = 0; i < CL; ++i) {
                v[i] = vDir[i];
                v[CL + i] = vDir[i] * vAr[i];
            }
            ReduceScatter<2 * CL, 16>::run(v, lane);
            acc_fa += double(v[0]);
#pragma unroll
            for (int i = 0; i < CL; ++i) {
                const float a_n = (i + 1 < CL) ? vA[i + 1] : alb_in;
                const float s_n = (i + 1 < CL) ? vS[i + 1] : src_in;
                const float fd_n = (i + 1 < CL) ? vFd[i + 1] : fd_bot;
                v[i] = fmaf(vFd[i], vA[i], vS[i]);
                v[CL + i] = (vFd[i] + fmaf(fd_n, a_n, s_n)) * vAf[i];
            }
            ReduceScatter<2 * CL, 16>::run(v, lane);
            acc_fb += double(v[0]);
#pragma unroll
            for (int i = 0; i < CL; ++i) {
                v[i] = vFd[i];
                v[CL + i] = 0.f;
            }
            ReduceScatter<2 * CL, 16>::run(v, lane);
            acc_fc += double(v[0]);
            if (Wg == NWt - 1) {
                acc_sfc_dir += double(warp_sum(dsfc));
                acc_sfc_dn += double(warp_sum(fd_bot));
                acc_sfc_up += double(warp_sum(fmaf(fd_bot, alb_in, src_in)));
            }
        }

        // ---- R3 composite (Fraw bottom -> top of chunk) ----
        {
            float A3 = 1.f, B3 = 0.f;
#pragma unroll
            for (int i = CL - 1; i >= 0; --i) {
                const int jl = w * CL + i;
                const float a_n = (i + 1 < CL) ? vA[i + 1] : alb_in;
                const float den = __fdividef(1.f, fmaf(-vR[i], a_n, 1.f));
                const float c = vT[i] * den;
                const float h = sm_hh[jl];
                const float off = c * h * vAf[i] * a_n + sm_be[jl] + h * vAf[i] + sm_al[jl] * vA[i];
                A3 *= c;
                B3 = c * B3 + off;
            }
            for (int rr = 0; rr < CS; ++rr) remote(cluster, sm_x3, rr)[Wg * 32 + lane] = make_float2(A3, B3);
        }
        cluster.sync();
        float Fraw = (L_end == nlay) ? beN + alN * af : 0.f;
        for (int c = NWt - 1; c > Wg; --c) {
            const float2 m = sm_x3[c * 32 + lane];
            Fraw = m.x * Fraw + m.y;
        }
        // R3 resweep: complete F at the bottom level of every layer
        float vFc[CL];
#pragma unroll
        for (int i = CL - 1; i >= 0; --i) {
            const int jl = w * CL + i;
            const float a_n = (i + 1 < CL) ? vA[i + 1] : alb_in;
            const float den = __fdividef(1.f, fmaf(-vR[i], a_n, 1.f));
            const float h = sm_hh[jl];
            const float Fc = Fraw + h * vAf[i] * a_n;
            vFc[i] = Fc;
            Fraw = vT[i] * den * Fc + sm_be[jl] + h * vAf[i] + sm_al[jl] * vA[i];
        }

        // ---- R2 composite (top -> bottom of chunk), (Abar, Sbar) ----
        {
            float cP = 1.f, cQ = 0.f, cR = 1.f, cUo = 0.f, cV = 0.f;
#pragma unroll
            for (int i = 0; i < CL; ++i) {
                const int jl = w * CL + i;
                const float a_n = (i + 1 < CL) ? vA[i + 1] : alb_in;
                const float s_n = (i + 1 < CL) ? vS[i + 1] : src_in;
                const float fd_n = (i + 1 < CL) ? vFd[i + 1] : fd_bot;
                const float den = __fdividef(1.f, fmaf(-vR[i], a_n, 1.f));
                const float td = vT[i] * den;
                const float ub = sm_al[jl + 1] + sm_hh[jl] * vAf[i];
                const float p = td * td, q = td * den * (vTd[i] * vDir[i] + vR[i] * s_n), r = td;
                const float u = fd_n * (vR[i] * den * vFc[i] + ub), v = vFc[i] * vR[i] * den + ub;
                const float nP = p * cP, nQ = p * cQ + q * cR, nU = p * cUo + q * cV + u;
                const float nR = r * cR, nV = r * cV + v;
                cP = nP; cQ = nQ; cUo = nU; cR = nR; cV = nV;
            }
            for (int rr = 0; rr < CS; ++rr) {
                remote(cluster, sm_x4a, rr)[Wg * 32 + lane] = make_float4(cP, cQ, cR, cUo);
                remote(cluster, sm_x4b, rr)[Wg * 32 + lane] = cV;
            }
        }
        cluster.sync();
        float Ab = 0.f, Sb = al0, Ab_in = 0.f, Sb_in = al0;
        for (int c = 0; c < NWt; ++c) {
            if (c == Wg) { Ab_in = Ab; Sb_in = Sb; }
            const float4 m = sm_x4a[c * 32 + lane];
            const float v = sm_x4b[c * 32 + lane];
            const float nA = m.x * Ab + m.y * Sb + m.w;
            Sb = m.z * Sb + v;
            Ab = nA;
        }
        const float AbN = Ab, SbN = Sb;   // at level nlay (padding is the identity)
        // R2 resweep: layer adjoints of R, T, sup, sdn
        float vRb[CL], vTb[CL], vSub[CL], vSdb[CL], vAfb[CL];
        {
            float A_ = Ab_in, S_ = Sb_in;
#pragma unroll
            for (int i = 0; i < CL; ++i) {
                const int jl = w * CL + i;
                const float a_n = (i + 1 < CL) ? vA[i + 1] : alb_in;
                const float s_n = (i + 1 < CL) ? vS[i + 1] : src_in;
                const float fd_n = (i + 1 < CL) ? vFd[i + 1] : fd_bot;
                const float den = __fdividef(1.f, fmaf(-vR[i], a_n, 1.f));
                const float T = vT[i], R = vR[i], sdn = vTd[i] * vDir[i], Fc = vFc[i];
                const float num_fd = T * vFd[i] + R * s_n + sdn;              // fd_(i+1) / den
                const float denb = A_ * T * T * a_n + S_ * T * (s_n + a_n * sdn) + Fc * num_fd;
                vRb[i] = A_ + denb * a_n * den * den + Fc * s_n * den;
                vTb[i] = A_ * 2.f * T * a_n * den + S_ * den * (s_n + a_n * sdn) + Fc * vFd[i] * den;
                vSub[i] = S_;
                vSdb[i] = S_ * T * den * a_n + Fc * den;
                const float fu_n = fd_n * a_n + s_n;
                vAfb[i] = sm_hh[jl] * (vFd[i] + fu_n);
                // advance to level i + 1
                const float td = T * den;
                const float ub = sm_al[jl + 1] + sm_hh[jl] * vAf[i];
                const float nA = td * td * A_ + td * den * (sdn + R * s_n) * S_ + fd_n * (R * den * Fc + ub);
                S_ = td * S_ + Fc * R * den + ub;
                A_ = nA;
            }
        }
        // surface albedo adjoints (same in every warp; one warp of one CTA accumulates them)
        if (rank == 0 && w == 0) {
            const float gad = SbN * dsfc, gaf = AbN;
            for (int s = 0; s < 2; ++s) {
                const float vd = warp_sum((gv && slot == s) ? gad : 0.f);
                const float vf = warp_sum((gv && slot == s) ? gaf : 0.f);
                const int b = b0 + s;
                if (lane == 0 && s < mgb && b < nband && k.band_lims[2 * b] < 32 * gg + 32) {
                    sm_alb[2 * b] += double(vd);
                    sm_alb[2 * b + 1] += double(vf);
                }
            }
        }

        // ---- R1 composite (Dbar bottom -> top of chunk) ----
        {
            float A5 = 1.f, B5 = 0.f;
#pragma unroll
            for (int i = CL - 1; i >= 0; --i) {
                const int jl = w * CL + i;
                const float e = sm_be[jl] + sm_ga[jl] + sm_hh[jl] * vAr[i] + vSub[i] * vRd[i] + vSdb[i] * vTd[i];
                A5 *= vTn[i];
                B5 = vTn[i] * B5 + e;
            }
            for (int rr = 0; rr < CS; ++rr) remote(cluster, sm_x5, rr)[Wg * 32 + lane] = make_float2(A5, B5);
        }
        cluster.sync();
        float Db = SbN * ad + ((L_end == nlay) ? beN + gaN : 0.f);
        for (int c = NWt - 1; c > Wg; --c) {
            const float2 m = sm_x5[c * 32 + lane];
            Db = m.x * Db + m.y;
        }

        // ---- R1 resweep + local adjoints per layer ----
        float gT[CL], gH[CL], gO[CL], gC0[CL], gC1[CL], gC2[CL];
#pragma unroll
        for (int i = CL - 1; i >= 0; --i) {
            const int jl = w * CL + i;
            const int j = j0 + jl;
            const float dir = vDir[i];
            const float Tnb = Db * dir, Rdb = vSub[i] * dir, Tdb = vSdb[i] * dir, Arb = sm_hh[jl] * dir;
            Db = sm_be[jl] + sm_ga[jl] + sm_hh[jl] * vAr[i] + vSub[i] * vRd[i] + vSdb[i] * vTd[i] + vTn[i] * Db;
            gT[i] = 0.f; gH[i] = 0.f; gO[i] = 0.f; gC0[i] = 0.f; gC1[i] = 0.f; gC2[i] = 0.f;
            if (j < nlay && gv) {
                const Rec& Rc = recs[slot * CL + i];
                const LayerAdj la = sw_layer_adjoint<DENSE>(k.kmaj4, k.kmin2[Rc.a], k.krayl2, &Rc, &drecs[slot * CL + i],
                                                     sm_sc4 + jl * k.max_nscal,
                                                     k.minor_gx[Rc.a] + size_t(g) * k.minor_gx_stride, g,
                                                     Rc.a ? mg1 : mg0, Rc.a ? nm1 : nm0, vTau[i], vW0[i], vOmw[i],
                                                     vG[i], mu0, mu0_inv, vRb[i], vTb[i], Rdb, Tdb, Tnb, vAfb[i], Arb);
                gT[i] = la.t; gH[i] = la.h; gO[i] = la.o;
                gC0[i] = la.tc; gC1[i] = la.tsc; gC2[i] = la.tsg;
            }
        }

        // ---- sums over the 32 g-points ----
        {
            float v[4 * CL];   // [T | H | O | -] x CL
#pragma unroll
            for (int i = 0; i < CL; ++i) { v[i] = gT[i]; v[CL + i] = gH[i]; v[2 * CL + i] = gO[i]; v[3 * CL + i] = 0.f; }
            ReduceScatter<4 * CL, 16>::run(v, lane);
            acc_q += double(v[0]);
        }
        {
            // cloud: [tc s0 | tc s1 | tsc s0 | tsc s1] then [tsg s0 | tsg s1], CL layers each
            constexpr int SH4 = (4 * CL == 32) ? 0 : 1;   // lane L holds value L >> SH4 of 4 CL
            constexpr int SH2 = SH4 + 1;                  // ... and value L >> SH2 of 2 CL
            float v[4 * CL];
#pragma unroll
            for (int i = 0; i < CL; ++i) {
                v[i] = slot == 0 ? gC0[i] : 0.f;
                v[CL + i] = slot == 1 ? gC0[i] : 0.f;
                v[2 * CL + i] = slot == 0 ? gC1[i] : 0.f;
                v[3 * CL + i] = slot == 1 ? gC1[i] : 0.f;
            }
            ReduceScatter<4 * CL, 16>::run(v, lane);
            {
                const int vi = lane >> SH4;
                const int q = vi / (2 * CL), sl = (vi / CL) & 1, jl = w * CL + (vi % CL), b = b0 + sl;
                if ((lane & ((1 << SH4) - 1)) == 0 && j0 + jl < nlay && b < nband &&
                    k.band_lims[2 * b] < 32 * gg + 32)
                    sm_cl[(b * kLPC + jl) * 3 + q] += v[0];
            }
            float u[2 * CL];
#pragma unroll
            for (int i = 0; i < CL; ++i) { u[i] = slot == 0 ? gC2[i] : 0.f; u[CL + i] = slot == 1 ? gC2[i] : 0.f; }
            ReduceScatter<2 * CL, 16>::run(u, lane);
            {
                const int vi = lane >> SH2, sl = vi / CL, jl = w * CL + (vi % CL), b = b0 + sl;
                if ((lane & ((1 << SH2) - 1)) == 0 && j0 + jl < nlay && b < nband &&
                    k.band_lims[2 * b] < 32 * gg + 32)
                    sm_cl[(b * kLPC + jl) * 3 + 2] += u[0];
            }
        }
        // No barrier closes the group: each exchange buffer is rewritten in the next group only
        // after a cluster barrier that every reader of this group's values has passed (a warp
        // reads buffer k between barriers k and k + 1, and the next group writes it after that
        // group's barrier k - 1 at the earliest); records and cloud sums are per warp.  (With
        // the FP64 code in the kernel, a closing barrier measured faster at 60 layers by
        // keeping the warps in the same code; without it the kernel is 2-4% faster at 60, 128
        // and 256 layers.)
    }

    // ---- outputs ----
    __syncthreads();   // the cloud sums of the last group are read below by other warps
    if (FLUX) {
        constexpr int SHF = (2 * CL == 16) ? 1 : 2;   // lane L holds value L >> SHF of 2 CL
        const int v = lane >> SHF;
        const double g0_cp = 9.80665 / 1004.64;
        if ((lane & ((1 << SHF) - 1)) == 0) {
            if (v < CL) {
                const int j = j0 + w * CL + v;
                if (j < nlay) {
                    const size_t o = icol + size_t(top_at_1 ? j : nlay - j) * ncol;
                    const double dn = acc_fc + acc_fa;
                    out.flux_up[o] = float(acc_fb);
                    out.flux_dn[o] = float(dn);
                    out.flux_dir[o] = float(acc_fa);
                    out.flux_net[o] = float(dn - acc_fb);
                }
            } else {
                const int jl = w * CL + v - CL, j = j0 + jl;
                if (j < nlay) {
                    const size_t o = icol + size_t(top_at_1 ? j : nlay - 1 - j) * ncol;
                    out.heating_rate[o] = float(g0_cp * 86400.0 * (acc_fa + acc_fb) / double(st[jl].dp));
                }
            }
        }
        if (Wg == NWt - 1 && lane == 0) {
            const size_t o = icol + size_t(top_at_1 ? nlay : 0) * ncol;
            const double dn = acc_sfc_dn + acc_sfc_dir;
            out.flux_up[o] = float(acc_sfc_up);
            out.flux_dn[o] = float(dn);
            out.flux_dir[o] = float(acc_sfc_dir);
            out.flux_net[o] = float(dn - acc_sfc_up);
        }
    }
    {
        constexpr int SHQ = (4 * CL == 32) ? 0 : 1;   // lane L holds value L >> SHQ of 4 CL
        const int vi = lane >> SHQ;
        const int q = vi / CL, jl = w * CL + (vi % CL), j = j0 + jl;
        if ((lane & ((1 << SHQ) - 1)) == 0 && q < 3 && j < nlay) {
            const size_t o = icol + size_t(top_at_1 ? j : nlay - 1 - j) * ncol;
            float* dst = q == 0 ? out.tlay : (q == 1 ? out.h2o : out.o3);
            if (dst) dst[o] = float(acc_q);
        }
    }
    for (int jl = threadIdx.x; jl < kLPC; jl += blockDim.x) {
        const int j = j0 + jl;
        if (j >= nlay) continue;
        const int l = top_at_1 ? j : nlay - 1 - j;
        const size_t cl = icol + size_t(l) * ncol;
        float gl = 0.f, gi = 0.f, grl = 0.f, gri = 0.f;
        if (cld.present) {
            const float lw = cld.lwp[cl], iw = cld.iwp[cl], rl = cld.rel[cl], ri = cld.rei[cl];
            for (int b = 0; b < nband; ++b) {
                const float* sb = sm_cl + (b * kLPC + jl) * 3;
                if (sb[0] == 0.f && sb[1] == 0.f && sb[2] == 0.f) continue;
                D4 tc, tsc, tsg;
                cloud_sw_dual(cld.L, cld.delta, lw, iw, rl, ri, b, tc, tsc, tsg);
                gl += sb[0] * tc.d[0] + sb[1] * tsc.d[0] + sb[2] * tsg.d[0];
                gi += sb[0] * tc.d[1] + sb[1] * tsc.d[1] + sb[2] * tsg.d[1];
                grl += sb[0] * tc.d[2] + sb[1] * tsc.d[2] + sb[2] * tsg.d[2];
                gri += sb[0] * tc.d[3] + sb[1] * tsc.d[3] + sb[2] * tsg.d[3];
            }
        }
        if (out.lwp) out.lwp[cl] = gl;
        if (out.iwp) out.iwp[cl] = gi;
        if (out.rel) out.rel[cl] = grl;
        if (out.rei) out.rei[cl] = gri;
    }
    if (rank == 0) {
        for (int b = threadIdx.x; b < nband; b += blockDim.x) {
            if (out.alb_dir) out.alb_dir[b + size_t(icol) * nband] = float(sm_alb[2 * b]);
            if (out.alb_dif) out.alb_dif[b + size_t(icol) * nband] = float(sm_alb[2 * b + 1]);
        }
    }
    cluster.sync();   // no CTA leaves while its shared memory may still be read remotely
}

}  // namespace

// a: aerosol tables or NULL (no aerosols); aerosols, naer, rh, delta_aerosol as
// rrtmgp_b200_forward_sw_aer_f32.  The aerosol optics enter the recomputed forward; they depend
// on none of the differentiated inputs, so no aerosol gradient is formed.
int adjoint_sw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay, const float* play, const float* plev,
                   const float* tlay, const float* col_dry, const rrtmgp_b200_gas_conc* gases, int ngases,
                   const float* lwp, const float* iwp, const float* rel, const float* rei, int delta_cloud,
                   const float* mu0, const float* tsi_scaling, const float* sfc_alb_dir, const float* sfc_alb_dif,
                   const float* seed_up, const float* seed_dn, const float* seed_dir, const float* seed_hr,
                   float* g_tlay, float* g_h2o, float* g_o3, float* g_lwp, float* g_iwp, float* g_rel, float* g_rei,
                   float* g_alb_dir, float* g_alb_dif, float* flux_up, float* flux_dn, float* flux_dir,
                   float* flux_net, float* heating_rate, void* stream, rrtmgp_b200_aerosol a = nullptr,
                   const rrtmgp_b200_gas_conc* aerosols = nullptr, int naer = 0, const float* rh = nullptr,
                   int delta_aerosol = 0)
{
    RB_CHECK_ARG(k && !k->info.is_longwave, "adjoint_sw: need a shortwave k-distribution");
    if (const int dst = check_device(k->device, "adjoint_sw")) return dst;
    const bool with_flux = flux_up != nullptr;
    RB_CHECK_ARG(!with_flux || (flux_dn && flux_dir && flux_net && heating_rate), "forward_adjoint_sw: null flux array");
    RB_CHECK_ARG(ncol > 0 && nlay > 1, "adjoint_sw: ncol > 0 and nlay > 1 required");
    RB_CHECK_ARG(play && plev && tlay && mu0 && sfc_alb_dir && sfc_alb_dif, "adjoint_sw: null input array");
    RB_CHECK_ARG(!c || (lwp && iwp && rel && rei), "adjoint_sw: cloud arrays required with a cloud handle");
    RB_CHECK_ARG(!c || c->nband == k->info.nband, "adjoint_sw: cloud and gas band counts differ");
    const KdistView<float>& v = k->v32;
    if (!fused_layout_ok(v, true, 2))
        return fail(RRTMGP_B200_ERR_UNSUPPORTED, "adjoint_sw: k-distribution layout not supported by the adjoint kernel");
    const int CS = (nlay + kLPC - 1) / kLPC;
    RB_CHECK_ARG(CS <= 8, "adjoint_sw: nlay too large (at most 512 layers)");
    GasSet<float> gs;
    int st = make_gas_set<float>(k, ncol, nlay, gases, ngases, gs);
    if (st) return st;
    int idx_o3 = 0;
    for (size_t i = 0; i < k->gas_names.size(); ++i)
        if (k->gas_names[i] == "o3") idx_o3 = int(i) + 1;
    SwAerosolArgs aer{};
    if (a) {
        RB_CHECK_ARG(rh, "adjoint_sw: rh required with aerosol tables");
        aer.L = aerosol_lut32(a);
        RB_CHECK_ARG(aer.L.nband == k->info.nband, "adjoint_sw: aerosol and gas band counts differ");
        st = make_aerosol_set<float>(ncol, nlay, aerosols, naer, aer.s);
        if (st) return st;
        aer.rh = rh;
        aer.present = 1;
        aer.delta = delta_aerosol;
    }
    constexpr int CL = kSwAdjointChunk;
    // two record buffers (records of two groups built at once) when they fit
    const bool wa = aer.present != 0;
    const size_t smem2 = sw_adj_layout(v.ngas, v.nband, v.max_group_bands, CS, kLPC / CL, 2, v.max_nscal, wa).total;
    const bool pair = smem2 <= 227 * 1024;
    const size_t smem =
        pair ? smem2 : sw_adj_layout(v.ngas, v.nband, v.max_group_bands, CS, kLPC / CL, 1, v.max_nscal, wa).total;
    if (smem > 227 * 1024) return fail(RRTMGP_B200_ERR_UNSUPPORTED, "adjoint_sw: shared memory need exceeds 227 KB");
    static PerDeviceOnce attr;
    const int ast = attr.run([] {
        for (auto fn : {sw_adjoint_kernel<CL, false, false, false>, sw_adjoint_kernel<CL, true, false, false>,
                        sw_adjoint_kernel<CL, false, true, false>, sw_adjoint_kernel<CL, true, true, false>,
                        sw_adjoint_kernel<CL, false, false, true>, sw_adjoint_kernel<CL, true, false, true>,
                        sw_adjoint_kernel<CL, false, true, true>, sw_adjoint_kernel<CL, true, true, true>}) {
            const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }, "adjoint_sw attribute");
    if (ast) return ast;
    SwCloudArgs ca{};
    if (c) {
        ca.L = CloudLut<float>{c->nband, c->nsize_liq, c->nsize_ice, float(c->radliq_lwr), float(c->liq_step),
                               float(c->radice_lwr), float(c->ice_step), c->lut32};
        ca.lwp = lwp; ca.iwp = iwp; ca.rel = rel; ca.rei = rei;
        ca.present = 1;
        ca.delta = delta_cloud;
    }
    const SwAdjOut out{g_tlay, g_h2o, g_o3, g_lwp, g_iwp, g_rel, g_rei, g_alb_dir, g_alb_dif,
                       flux_up, flux_dn, flux_dir, flux_net, heating_rate};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(ncol) * CS);
    cfg.blockDim = dim3(kLPC / CL * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = as_stream(stream);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = unsigned(CS);
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const bool dense = v.max_minor_per_g > 3;
    const auto kernel =
        dense ? (with_flux ? (pair ? sw_adjoint_kernel<CL, true, true, true> : sw_adjoint_kernel<CL, true, false, true>)
                           : (pair ? sw_adjoint_kernel<CL, false, true, true> : sw_adjoint_kernel<CL, false, false, true>))
              : (with_flux ? (pair ? sw_adjoint_kernel<CL, true, true, false> : sw_adjoint_kernel<CL, true, false, false>)
                           : (pair ? sw_adjoint_kernel<CL, false, true, false>
                                   : sw_adjoint_kernel<CL, false, false, false>));
    RB_CUDA(cudaLaunchKernelEx(&cfg, kernel, v, gs, ca, ncol, nlay, CS, idx_o3, col_dry ? 0 : 1, play, plev,
                               tlay, col_dry, mu0, tsi_scaling, sfc_alb_dir, sfc_alb_dif, seed_up, seed_dn, seed_dir,
                               seed_hr, out, aer),
            "sw_adjoint_kernel launch");
    return RRTMGP_B200_OK;
}

}  // namespace rrtmgp_b200

extern "C" int rrtmgp_b200_adjoint_sw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp, const float* rel,
        const float* rei, int delta_cloud, const float* mu0, const float* tsi_scaling, const float* sfc_alb_dir,
        const float* sfc_alb_dif, const float* seed_flux_up, const float* seed_flux_dn, const float* seed_flux_dn_dir,
        const float* seed_heating_rate, float* grad_tlay, float* grad_h2o, float* grad_o3, float* grad_lwp,
        float* grad_iwp, float* grad_rel, float* grad_rei, float* grad_sfc_alb_dir, float* grad_sfc_alb_dif,
        void* stream)
{
    return rrtmgp_b200::adjoint_sw_f32(k, c, ncol, nlay, play, plev, tlay, col_dry, gases, ngases, lwp, iwp, rel, rei,
                                       delta_cloud, mu0, tsi_scaling, sfc_alb_dir, sfc_alb_dif, seed_flux_up,
                                       seed_flux_dn, seed_flux_dn_dir, seed_heating_rate, grad_tlay, grad_h2o, grad_o3,
                                       grad_lwp, grad_iwp, grad_rel, grad_rei, grad_sfc_alb_dir, grad_sfc_alb_dif,
                                       nullptr, nullptr, nullptr, nullptr, nullptr, stream);
}

extern "C" int rrtmgp_b200_forward_adjoint_sw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp, const float* rel,
        const float* rei, int delta_cloud, const float* mu0, const float* tsi_scaling, const float* sfc_alb_dir,
        const float* sfc_alb_dif, const float* seed_flux_up, const float* seed_flux_dn, const float* seed_flux_dn_dir,
        const float* seed_heating_rate, float* grad_tlay, float* grad_h2o, float* grad_o3, float* grad_lwp,
        float* grad_iwp, float* grad_rel, float* grad_rei, float* grad_sfc_alb_dir, float* grad_sfc_alb_dif,
        float* flux_up, float* flux_dn, float* flux_dn_dir, float* flux_net, float* heating_rate, void* stream)
{
    RB_CHECK_ARG(flux_up, "forward_adjoint_sw: null flux array");
    return rrtmgp_b200::adjoint_sw_f32(k, c, ncol, nlay, play, plev, tlay, col_dry, gases, ngases, lwp, iwp, rel, rei,
                                       delta_cloud, mu0, tsi_scaling, sfc_alb_dir, sfc_alb_dif, seed_flux_up,
                                       seed_flux_dn, seed_flux_dn_dir, seed_heating_rate, grad_tlay, grad_h2o, grad_o3,
                                       grad_lwp, grad_iwp, grad_rel, grad_rei, grad_sfc_alb_dir, grad_sfc_alb_dif,
                                       flux_up, flux_dn, flux_dn_dir, flux_net, heating_rate, stream);
}

extern "C" int rrtmgp_b200_forward_adjoint_sw_aer_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c,
        rrtmgp_b200_aerosol a, int ncol, int nlay, const float* play, const float* plev, const float* tlay,
        const float* col_dry, const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp,
        const float* rel, const float* rei, int delta_cloud, const rrtmgp_b200_gas_conc* aerosols, int naer,
        const float* rh, int delta_aerosol, const float* mu0, const float* tsi_scaling, const float* sfc_alb_dir,
        const float* sfc_alb_dif, const float* seed_flux_up, const float* seed_flux_dn, const float* seed_flux_dn_dir,
        const float* seed_heating_rate, float* grad_tlay, float* grad_h2o, float* grad_o3, float* grad_lwp,
        float* grad_iwp, float* grad_rel, float* grad_rei, float* grad_sfc_alb_dir, float* grad_sfc_alb_dif,
        float* flux_up, float* flux_dn, float* flux_dn_dir, float* flux_net, float* heating_rate, void* stream)
{
    RB_CHECK_ARG(a, "forward_adjoint_sw_aer: null aerosol handle");
    return rrtmgp_b200::adjoint_sw_f32(k, c, ncol, nlay, play, plev, tlay, col_dry, gases, ngases, lwp, iwp, rel, rei,
                                       delta_cloud, mu0, tsi_scaling, sfc_alb_dir, sfc_alb_dif, seed_flux_up,
                                       seed_flux_dn, seed_flux_dn_dir, seed_heating_rate, grad_tlay, grad_h2o, grad_o3,
                                       grad_lwp, grad_iwp, grad_rel, grad_rei, grad_sfc_alb_dir, grad_sfc_alb_dif,
                                       flux_up, flux_dn, flux_dn_dir, flux_net, heating_rate, stream, a, aerosols,
                                       naer, rh, delta_aerosol);
}
