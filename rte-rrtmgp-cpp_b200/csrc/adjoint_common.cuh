// Building blocks of the hand-written adjoint (reverse-mode) column kernels.
//
// Gas optics of one (layer, band) is a function of a few per-layer scalars -- the layer
// temperature, and the volume mixing ratios of h2o and o3 (through the gas columns, the
// flavour mixing fraction eta and the dry-air column) -- applied to table rows that are
// constant within an interpolation cell.  Its adjoint per (layer, g-point) is therefore
// x_bar += tau_bar * dtau/dx with dtau/dx a fixed linear combination of the same table
// corners the forward reads.  A derivative record (DRec) holds those combinations for one
// (layer, band); it is built once per group of 32 g-points next to the forward record.
//
// Derivation (interpolation_kernel and gas_optical_depths_major/minor_kernel,
// gas_optics_rrtmgp_kernels.cu:215-476), per temperature row it in {0, 1}:
//   ftt_0 = 1 - ftemp, ftt_1 = ftemp,  ftemp = (T - T_ref[jt]) / dT
//   cm = c1 + r c2,  eta = c1 / cm,  feta = eta (neta-1) - (j-1)   (FP32 rule, continuous)
//   tau_it = ftt cm [ (1-feta) Kp(e) + feta Kp(e+1) ],  Kp(e) = (1-fp) k(e,p) + fp k(e,p+1)
// so that, with q = neta - j and the cell (j, jt, jp) fixed,
//   dtau_it/dftemp = sign(it) cm [ (1-feta) Kp(e) + feta Kp(e+1) ]
//   dtau_it/dc1    = ftt [ (1-q) Kp(e) + q Kp(e+1) ]
//   dtau_it/dc2    = ftt r [ j Kp(e) - (j-1) Kp(e+1) ]
// (cm * feta = c1 (neta-1) - cm (j-1) is linear in c1, c2).  Planck fractions and minor
// absorbers use the same weights without cm, so their eta dependence goes through
//   dfeta/dc1 = (neta-1) r c2 / cm^2,  dfeta/dc2 = -(neta-1) r c1 / cm^2.
// Gas columns: col_k = vmr_k col_dry, col_0 = col_dry, and when col_dry is computed from
// the levels, col_dry = C dp / (m_dry + m_h2o vmr_h2o) (get_col_dry,
// Gas_optics_rrtmgp.cpp:764-792), so dcol_dry/dvmr_h2o = -col_dry m_h2o / (m_dry + m_h2o vmr_h2o).
// Minor scaling (gas_optical_depths_minor_kernel :396-417): col_minor [* 0.01 p / T
// [* q or (1 - q)]], q = vmr_s / (1 + vmr_h2o).
#pragma once

#include "fused_common.cuh"

namespace rrtmgp_b200 {
namespace fused {

struct __align__(16) DRec {
    float4 wT0, wT1;    // d tau_major / dT on kmaj4 rows 0 / 1
    float4 wH0, wH1;    // d tau_major / d vmr_h2o
    float4 wO0, wO1;    // d tau_major / d vmr_o3
    float4 pT0, pT1;    // d pfrac / dT on pfrac4 rows (LW; unused in SW)
    float4 pH0, pH1;
    float4 pO0, pO1;
    float4 fmT, fmH, fmO;   // d fminor / dx on the minor corners (lo.x, lo.y, hi.x, hi.y)
    float4 dB;              // LW: dB/dT of the band Planck function at T_lay, T_top, T_bot, T_sfc
                            // SW: d col_rayl / d vmr_h2o in x
    float4 pad;             // 272 bytes: an odd number of 16-byte units (bank-conflict-free stores
                            // of consecutive records, as Rec)
};                          // (minor scalings and their derivatives: layer_minor_scalings_d)
static_assert(sizeof(DRec) == 272, "DRec stride");

__device__ __forceinline__ float dot4(const float4& a, const float4& b)
{
    return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}

// Slope of the piecewise-linear interpolate1D table at val.
__device__ __forceinline__ float interpolate1D_slope(float val, float offset, float delta, int len,
                                                     const float* __restrict__ table)
{
    const float val0 = (val - offset) / delta;
    const int idx = min(len - 1, max(1, int(val0) + 1));
    return (table[idx] - table[idx - 1]) / delta;
}

// Derivative record of band b at layer state s (cg: gas columns of the layer, stride cgs).
// It does not read the forward record, so both can be built at once.  idx_o3: col_gas
// index of o3 (0: absent).
// cd_internal: col_dry was computed from h2o and the level pressures.  PFRAC: also the
// Planck-fraction weights pT/pH/pO (longwave only).
template <bool PFRAC = true>
__device__ __forceinline__ void build_drec(const KdistView<float>& k, DRec& D, const LayerState& s, const float* cg,
                                           int cgs, int b, int idx_o3, int cd_internal)
{
    const float delta = k.temp_ref_delta;
    const int a = s.itropo;
    const int flav = k.band_flav[2 * b + a];
    const int gas1 = k.flavor[2 * flav], gas2 = k.flavor[2 * flav + 1];
    const float cd = cg[0];
    const float vh = cg[k.idx_h2o * cgs] / cd;
    constexpr float m_dry = 0.028964f, m_h2o = 0.018016f;
    const float dcd_h = cd_internal ? -cd * m_h2o / (m_dry + m_h2o * vh) : 0.f;
    // d col_gas[gi] / d vmr of col_gas index xi (xi = idx_h2o or idx_o3)
    auto dcol = [&](int gi, int xi) -> float {
        if (xi <= 0) return 0.f;
        float d = 0.f;
        if (xi == k.idx_h2o) d = (gi == 0 ? 1.f : cg[gi * cgs] / cd) * dcd_h;
        if (gi == xi) d += cd;
        return d;
    };
    const float c1 = cg[gas1 * cgs], c2 = cg[gas2 * cgs];
    const float dc1[2] = {dcol(gas1, k.idx_h2o), dcol(gas1, idx_o3)};
    const float dc2[2] = {dcol(gas2, k.idx_h2o), dcol(gas2, idx_o3)};
    const float fp = s.fpress, f1 = 1.f - s.fpress;
    const float two_tmin = 2.f * FLT_MIN;
    float fmT[4], fmX[2][4];
#pragma unroll
    for (int it = 0; it < 2; ++it) {
        const float* vr = k.vmr_ref + size_t(s.jt - 1 + it) * (k.ngas + 1) * 2 + a;
        const float r = vr[2 * gas1] / vr[2 * gas2];
        const float cm = c1 + r * c2;
        const float eta = cm > two_tmin ? c1 / cm : 0.5f;
        const float loceta = eta * float(k.neta - 1);
        const int j = max(1, min(int(loceta) + 1, k.neta - 1));
        const float feta = loceta - float(j - 1);
        const float ftt = it ? s.ftemp : 1.f - s.ftemp;
        const float sg = it ? 1.f : -1.f;
        const float4 wb = make_float4(f1 * (1.f - feta), f1 * feta, fp * (1.f - feta), fp * feta);
        const float cT = sg * cm / delta, pTs = sg / delta;
        const float4 wT = make_float4(cT * wb.x, cT * wb.y, cT * wb.z, cT * wb.w);
        const float4 pT = make_float4(pTs * wb.x, pTs * wb.y, pTs * wb.z, pTs * wb.w);
        const float q = float(k.neta - j), jf = float(j);
        const float4 u1 = make_float4(f1 * (1.f - q), f1 * q, fp * (1.f - q), fp * q);
        const float4 u2 = make_float4(r * f1 * jf, -r * f1 * (jf - 1.f), r * fp * jf, -r * fp * (jf - 1.f));
        float4 wX[2], pX[2];
#pragma unroll
        for (int x = 0; x < 2; ++x) {
            const float a1 = ftt * dc1[x], a2 = ftt * dc2[x];
            wX[x] = make_float4(a1 * u1.x + a2 * u2.x, a1 * u1.y + a2 * u2.y, a1 * u1.z + a2 * u2.z,
                                a1 * u1.w + a2 * u2.w);
            // (neta-1) r (c2 dc1 - c1 dc2) / cm^2, in ratios: columns ~1e25 overflow FP32 when squared
            const float dfeta = cm > two_tmin
                                    ? float(k.neta - 1) * r * ((c2 / cm) * (dc1[x] / cm) - (c1 / cm) * (dc2[x] / cm))
                                    : 0.f;
            const float e = ftt * dfeta;
            pX[x] = make_float4(-e * f1, e * f1, -e * fp, e * fp);
            fmX[x][2 * it] = -e;
            fmX[x][2 * it + 1] = e;
        }
        fmT[2 * it] = sg * (1.f - feta) / delta;
        fmT[2 * it + 1] = sg * feta / delta;
        if (it == 0) {
            D.wT0 = wT; D.wH0 = wX[0]; D.wO0 = wX[1];
            if (PFRAC) { D.pT0 = pT; D.pH0 = pX[0]; D.pO0 = pX[1]; }
        } else {
            D.wT1 = wT; D.wH1 = wX[0]; D.wO1 = wX[1];
            if (PFRAC) { D.pT1 = pT; D.pH1 = pX[0]; D.pO1 = pX[1]; }
        }
    }
    D.fmT = make_float4(fmT[0], fmT[1], fmT[2], fmT[3]);
    D.fmH = make_float4(fmX[0][0], fmX[0][1], fmX[0][2], fmX[0][3]);
    D.fmO = make_float4(fmX[1][0], fmX[1][1], fmX[1][2], fmX[1][3]);
}

// Minor scalings of every scaling kind of layers 0 .. nloc - 1 with their derivatives:
// sc4[jl * k.max_nscal + sid] = (scaling, d ln(scaling) / dT, d scaling / d vmr_h2o,
// d scaling / d vmr_o3) (kind_scaling; zero past the layer's atmosphere's kind count).  Threads
// tid, tid + nthr, ... of the calling team take one (layer, kind) each.
__device__ __forceinline__ void layer_minor_scalings_d(const KdistView<float>& k, const LayerState* st,
                                                       const float* cg_all, int cgs, float4* sc4, int nloc,
                                                       int idx_o3, int cd_internal, int tid, int nthr)
{
    const int ns = k.max_nscal;
    constexpr float m_dry = 0.028964f, m_h2o = 0.018016f;
    for (int idx = tid; idx < nloc * ns; idx += nthr) {
        const int jl = idx / ns, sid = idx - jl * ns;
        const LayerState& s = st[jl];
        const int a = s.itropo;
        if (sid >= k.nscal[a]) {
            sc4[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
            continue;
        }
        const float* cg = cg_all + jl;
        const float cd = cg[0];
        const float vh = cg[k.idx_h2o * cgs] / cd;
        const float dcd_h = cd_internal ? -cd * m_h2o / (m_dry + m_h2o * vh) : 0.f;
        // d col_gas[gi] / d vmr of col_gas index xi (as build_drec)
        auto dcol = [&](int gi, int xi) -> float {
            if (xi <= 0) return 0.f;
            float d = 0.f;
            if (xi == k.idx_h2o) d = (gi == 0 ? 1.f : cg[gi * cgs] / cd) * dcd_h;
            if (gi == xi) d += cd;
            return d;
        };
        const int flags = k.scal_flags[a][sid];
        const int mg = k.scal_gas[a][sid];
        const float colm = cg[mg * cgs];
        float Dd = 1.f, Q = 1.f, dQh = 0.f, dQo = 0.f, dsT = 0.f;
        if (flags & 1) {
            Dd = 0.01f * s.p / s.t;
            dsT = -1.f / s.t;
            const int sgi = k.scal_sgas[a][sid];
            if (sgi > 0) {
                const float vs = cg[sgi * cgs] / cd;
                const float q0 = vs / (1.f + vh);
                const float sign = (flags & 2) ? -1.f : 1.f;
                Q = (flags & 2) ? 1.f - q0 : q0;
                // dq0/dvmr_sg = 1 / (1 + vh); dq0/dvmr_h2o = -vs / (1 + vh)^2
                float dqh = -vs / ((1.f + vh) * (1.f + vh)), dqo = 0.f;
                if (sgi == k.idx_h2o) dqh += 1.f / (1.f + vh);
                if (idx_o3 > 0 && sgi == idx_o3) dqo = 1.f / (1.f + vh);
                dQh = sign * dqh;
                dQo = sign * dqo;
            }
        }
        sc4[idx] = make_float4(kind_scaling(k, a, sid, cg, cgs, s.p, s.t), dsT,
                               Dd * (Q * dcol(mg, k.idx_h2o) + colm * dQh), Dd * (Q * dcol(mg, idx_o3) + colm * dQo));
    }
}

// Adjoint of tau_abs for g-point g: accumulates tau_bar * dtau/dx into gT, gH, gO.  c0, c1:
// the g-point's kmaj4 corners of the record's two rows (loaded by the caller, early); sc4:
// the layer's scaling table (layer_minor_scalings_d).  DENSE as tau_abs.
template <bool DENSE = false>
__device__ __forceinline__ void tau_abs_adjoint(const KdistView<float>& k, const Rec& R, const DRec& D, int g,
                                                int4 mg, int nmax, float tb, const float4& c0, const float4& c1,
                                                const float4* sc4, float& gT, float& gH, float& gO)
{
    float dT = dot4(D.wT0, c0) + dot4(D.wT1, c1);
    float dH = dot4(D.wH0, c0) + dot4(D.wH1, c1);
    float dO = dot4(D.wO0, c0) + dot4(D.wO1, c1);
    const float2* kn = k.kmin2[R.a];
    auto term = [&](int code, bool on) {
        const int c = code >> kScalBits;
        const float2 lo = __ldg(kn + (R.kb.z + c));
        const float2 hi = __ldg(kn + (R.kb.w + c));
        const float4 cr = make_float4(lo.x, lo.y, hi.x, hi.y);
        const float M = dot4(R.fm, cr);
        const float4 S = sc4[code & (kMaxScal - 1)];
        const float tT = S.x * (S.y * M + dot4(D.fmT, cr));
        const float tH = S.z * M + S.x * dot4(D.fmH, cr);
        const float tO = S.w * M + S.x * dot4(D.fmO, cr);
        dT += on ? tT : 0.f;
        dH += on ? tH : 0.f;
        dO += on ? tO : 0.f;
    };
#pragma unroll
    for (int n = 0; n < 3; ++n)
        if (n < nmax) term(n == 0 ? mg.y : (n == 1 ? mg.z : mg.w), n < mg.x);
    if constexpr (DENSE)
        for (int n = 3; n < nmax; ++n) term(minor_code_at(k, R.a, mg, g, n), n < mg.x);
    gT += tb * dT;
    gH += tb * dH;
    gO += tb * dO;
}

}  // namespace fused
}  // namespace rrtmgp_b200
