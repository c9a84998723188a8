// Hand-written adjoint of the fused longwave column forward (forward_lw.cu): gradients of
//   L = sum_l (seed_up_l F_up,l + seed_dn_l F_dn,l) + sum_i seed_hr_i HR_i
// with respect to the layer temperatures, the level temperatures, the surface temperature,
// the h2o and o3 volume mixing ratios and the cloud water paths / effective radii.  No
// reference counterpart exists (the reference has only the dormant surface Jacobian of
// lw_transport_noscat_kernel, rte_solver_kernels.cu:56-91, disabled at Rte_lw.cu:133).
//
// The optical properties are not stored between forward and backward: per group of 32
// g-points the kernel recomputes the forward (records, pass 1, chunk exchange, pass 2) and
// then runs the reverse sweeps.  Both reverse sweeps are affine recurrences in the same layer
// transmissivities t_i = 1 - omt_i as the forward ones, so their chunk maps are published in
// the same barrier as the forward maps:
//   U_bar(l+1) = t_l U_bar(l) + pi a_(l+1) + h_l omt_l       (top down,  U_bar(0) = pi a_0)
//   I_bar(l)   = t_l I_bar(l+1) + pi b_l + h_l omt_l         (bottom up,
//                I_bar(N) = pi b_N + (1 - emis) U_bar(N))
// (a, b: seeds of F_up, F_dn; h_i = g/cp 86400 pi seed_hr_i / dp_i; HR uses the per-layer
// divergence d_i = omt_i (I_i + U_(i+1)) - S_dn,i - S_up,i of the forward).  Per layer:
//   omt_bar = h (I_i + U_(i+1)) - I_bar(i+1) I_i - U_bar(i) U_(i+1)
//   Sdn_bar = I_bar(i+1) - h,  Sup_bar = U_bar(i) - h,  S_sfc_bar = emis U_bar(N)
// then through the linear-in-tau sources (omt(x), fact(x), x = tau D), the Planck fraction
// and band Planck functions, and the gas-optics interpolation (adjoint_common.cuh).
#include <cooperative_groups.h>

#include "adjoint_common.cuh"

namespace cg = cooperative_groups;

namespace rrtmgp_b200 {
namespace {

using namespace fused;

struct AdjCloud {
    CloudLut<float> L;
    const float* lwp;
    const float* iwp;
    const float* rel;
    const float* rei;
    int present;
};

struct AdjOut {
    float* tlay;
    float* tlev;
    float* tsfc;
    float* h2o;
    float* o3;
    float* lwp;
    float* iwp;
    float* rel;
    float* rei;
    // forward fluxes, written when the kernel is instantiated with FLUX (else unused)
    float* flux_up;
    float* flux_dn;
    float* flux_net;
    float* heating_rate;
};

// omt = 1 - exp(-x), fact = omt / x - exp(-x) and their x-derivatives (series below 0.1, as
// lw_layer_fast in the forward).
__device__ __forceinline__ void lw_terms(float x, float& omt, float& fact, float& domt, float& dfact)
{
    const float s_omt = x * (1.f + x * (-0.5f + x * (1.f / 6.f + x * (-1.f / 24.f + x * (1.f / 120.f +
                        x * (-1.f / 720.f + x * (1.f / 5040.f)))))));
    const float s_fact = x * (0.5f + x * (-1.f / 3.f + x * (0.125f + x * (-1.f / 30.f + x * (1.f / 144.f -
                         x * (1.f / 840.f))))));
    const float s_dfact = 0.5f + x * (-2.f / 3.f + x * (0.375f + x * (-2.f / 15.f + x * (5.f / 144.f +
                          x * (-1.f / 140.f + x * (49.f / 40320.f))))));
    const float e = __expf(-x);
    const float e_omt = 1.f - e;
    const float e_fact = __fdividef(e_omt, x) - e;
    const float e_dfact = e - __fdividef(e_fact, x);
    const bool thin = x < 0.1f;
    omt = thin ? s_omt : e_omt;
    fact = thin ? s_fact : e_fact;
    dfact = thin ? s_dfact : e_dfact;
    domt = thin ? 1.f - s_omt : e;
}

__device__ __forceinline__ void lw_layer_terms(float tau, float D, float lay, float ldn, float lup, float& omt,
                                               float& sdn, float& sup)
{
    float fact, domt, dfact;
    lw_terms(tau * D, omt, fact, domt, dfact);
    sdn = omt * ldn + 2.f * fact * (lay - ldn);
    sup = omt * lup + 2.f * fact * (lay - lup);
}

// Cloud 1scl partials of band b: dtau/dlwp, dtau/diwp, dtau/drel, dtau/drei (zero where the
// water path is not positive, the forward's mask).
__device__ __forceinline__ float4 cloud_1scl_partials(const CloudLut<float>& L, float lwp, float iwp, float rel,
                                                      float rei, int b)
{
    const CloudPoint<float> c = cloud_point(L, lwp, iwp, rel, rei);
    const size_t nl = size_t(L.nband) * L.nsl, ni = size_t(L.nband) * L.nsi;
    float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c.lwp > 0.f) {
        const float* le = L.lut + size_t(b) * L.nsl;
        const float* ls = le + nl;
        const float e = lut_lerp(le, c.il, c.fl), s = lut_lerp(ls, c.il, c.fl);
        const float de = (le[c.il + 1] - le[c.il]) / L.liq_step, ds = (ls[c.il + 1] - ls[c.il]) / L.liq_step;
        d.x = e * (1.f - s);
        d.z = c.lwp * (de * (1.f - s) - e * ds);
    }
    if (c.iwp > 0.f) {
        const float* ie = L.lut + 3 * nl + size_t(b) * L.nsi;
        const float* is = ie + ni;
        const float e = lut_lerp(ie, c.ii, c.fi), s = lut_lerp(is, c.ii, c.fi);
        const float de = (ie[c.ii + 1] - ie[c.ii]) / L.ice_step, ds = (is[c.ii + 1] - is[c.ii]) / L.ice_step;
        d.y = e * (1.f - s);
        d.w = c.iwp * (de * (1.f - s) - e * ds);
    }
    return d;
}

struct AdjLayout {
    size_t state, cg, scal, cld, taubar, seeds, levbot, maps, sfc, recs, drecs, total;
};

// Shared memory of one CTA: LPC local layers (LPC + 1 local levels), maps of all NWt chunks of
// the column, records of its NWc warps.
__host__ __device__ __forceinline__ AdjLayout adj_layout(int LPC, int ngas, int nband, int NWc, int NWt, int CL,
                                                         int mgb, int nbuf, int nscal)
{
    AdjLayout L;
    L.state = 0;
    L.cg = align16(L.state + sizeof(LayerState) * size_t(LPC));
    L.scal = align16(L.cg + sizeof(float) * size_t(ngas + 1) * LPC);
    L.cld = align16(L.scal + sizeof(float4) * size_t(nscal) * LPC);
    L.taubar = align16(L.cld + sizeof(float) * size_t(nband) * LPC);
    L.seeds = align16(L.taubar + sizeof(float) * size_t(nband) * LPC);
    L.levbot = align16(L.seeds + sizeof(float) * size_t(3 * LPC + 2));
    L.maps = align16(L.levbot + sizeof(double) * 16);
    L.sfc = align16(L.maps + sizeof(float4) * size_t(NWt) * 32 * 2 * nbuf);
    L.recs = align16(L.sfc + sizeof(float) * 32 * nbuf);
    L.drecs = align16(L.recs + sizeof(Rec) * size_t(NWc) * CL * mgb);
    L.total = align16(L.drecs + sizeof(DRec) * size_t(NWc) * CL * mgb);
    return L;
}

template <typename Tp>
__device__ __forceinline__ Tp* remote(cg::cluster_group& cl, Tp* p, int rank)
{
    return cl.map_shared_rank(p, rank);
}

// CL = 16: at most 8 warps (128 layers) with up to 255 registers per thread; CL = 8: up to 16
// warps per CTA at 128 registers.
// One column per cluster of CS CTAs (CLUSTER = false: CS = 1, a plain launch compiled without
// the cluster code).  CTA r of the cluster owns the layers [r LPC, (r + 1) LPC), LPC = NWc CL,
// as NWc warps of CL layers; chunk maps and the surface source are pushed to every CTA of the
// cluster through distributed shared memory.
// DENSE: more than three minor intervals over some g-point (tau_abs).
template <int CL, bool CLUSTER, bool FLUX, bool DENSE>
__global__ void __launch_bounds__(CL == 16 ? 256 : 512, 1)
lw_adjoint_kernel(const KdistView<float> k, const GasSet<float> gs, const AdjCloud cld, int ncol, int nlay, int CS,
                  int idx_o3, int cd_internal, const float* __restrict__ play, const float* __restrict__ plev,
                  const float* __restrict__ tlay, const float* __restrict__ tlev, const float* __restrict__ tsfc,
                  const float* __restrict__ col_dry_in, const float* __restrict__ sfc_emis,
                  const float* __restrict__ seed_up, const float* __restrict__ seed_dn,
                  const float* __restrict__ seed_hr, const AdjOut out)
{
    static_assert(CL == 8 || CL == 16, "chunk length");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    if (!CLUSTER) CS = 1;
    const int rank = CLUSTER ? int(cluster.block_rank()) : 0;
    const int icol = blockIdx.x / CS;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int NWc = blockDim.x >> 5;       // warps of this CTA
    const int NWt = CS * NWc;               // chunks of the column
    const int LPC = NWc * CL;               // layers per CTA
    const int Wg = rank * NWc + w;          // this warp's chunk
    const int j0 = rank * LPC;              // first layer of this CTA
    const int nband = k.nband, nlev = nlay + 1;
    const int mgb = k.max_group_bands;
    // One-CTA columns double-buffer the chunk maps and the surface source by group parity, so
    // no barrier is needed at the end of a group; clusters (maps of every chunk in every CTA)
    // keep one buffer and that barrier.
    const AdjLayout SL = adj_layout(LPC, k.ngas, nband, NWc, NWt, CL, mgb, CLUSTER ? 1 : 2, k.max_nscal);
    LayerState* st = reinterpret_cast<LayerState*>(smem_raw + SL.state);
    float* sm_cg = reinterpret_cast<float*>(smem_raw + SL.cg);
    float4* sm_sc4 = reinterpret_cast<float4*>(smem_raw + SL.scal);   // [local layer][scaling kind]
    float* sm_cld = reinterpret_cast<float*>(smem_raw + SL.cld);
    float* sm_tb = reinterpret_cast<float*>(smem_raw + SL.taubar);
    float* sm_a = reinterpret_cast<float*>(smem_raw + SL.seeds);   // pi * seed_up per local level
    float* sm_b = sm_a + (LPC + 1);                                // pi * seed_dn per local level
    float* sm_h = sm_b + (LPC + 1);                                // h per local layer
    double* sm_levbot = reinterpret_cast<double*>(smem_raw + SL.levbot);
    float4* const sm_map0 = reinterpret_cast<float4*>(smem_raw + SL.maps);
    float* const sm_sfc0 = reinterpret_cast<float*>(smem_raw + SL.sfc);
    Rec* recs = reinterpret_cast<Rec*>(smem_raw + SL.recs) + w * CL * mgb;
    DRec* drecs = reinterpret_cast<DRec*>(smem_raw + SL.drecs) + w * CL * mgb;
    auto at_rank = [&](auto* p, int rr) { return CLUSTER ? remote(cluster, p, rr) : p; };
    auto csync = [&]() {
        if (CLUSTER)
            cluster.sync();
        else
            __syncthreads();
    };

    const double pi = 3.14159265358979323846;
    const bool top_at_1 = play[icol] < play[icol + size_t(nlay - 1) * ncol];
    const float ts = tsfc[icol];
    auto seed_at = [&](const float* sd, int lev) -> float {   // global level (top down) -> pi * seed
        if (!sd || lev > nlay) return 0.f;
        return float(pi) * sd[icol + size_t(top_at_1 ? lev : nlay - lev) * ncol];
    };
    setup_layer_range(k, gs, ncol, nlay, icol, top_at_1, play, plev, tlay, tlev, col_dry_in, st, sm_cg, LPC, j0, LPC,
                      threadIdx.x, blockDim.x);
    for (int idx = threadIdx.x; idx < LPC * nband; idx += blockDim.x) {
        const int jl = idx % LPC, b = idx / LPC, j = j0 + jl;
        float tau = 0.f, s, g;
        if (cld.present && j < nlay) {
            const int l = top_at_1 ? j : nlay - 1 - j;
            const size_t cl = icol + size_t(l) * ncol;
            const CloudPoint<float> cp = cloud_point(cld.L, cld.lwp[cl], cld.iwp[cl], cld.rel[cl], cld.rei[cl]);
            cloud_band<float, false>(cld.L, cp, b, tau, s, g);
        }
        sm_cld[b * LPC + jl] = tau;
        sm_tb[b * LPC + jl] = 0.f;
    }
    for (int ll = threadIdx.x; ll <= LPC; ll += blockDim.x) {
        sm_a[ll] = seed_at(seed_up, j0 + ll);
        sm_b[ll] = seed_at(seed_dn, j0 + ll);
    }
    if (threadIdx.x < 16) sm_levbot[threadIdx.x] = 0.0;
    __syncthreads();
    layer_minor_scalings_d(k, st, sm_cg, LPC, sm_sc4, max(0, min(LPC, nlay - j0)), idx_o3, cd_internal, threadIdx.x,
                           blockDim.x);
    for (int jl = threadIdx.x; jl < LPC; jl += blockDim.x) {
        const int j = j0 + jl;
        float h = 0.f;
        if (j < nlay && seed_hr) {
            const int l = top_at_1 ? j : nlay - 1 - j;
            const double g0_cp = 9.80665 / 1004.64;
            h = float(g0_cp * 86400.0 * pi * double(seed_hr[icol + size_t(l) * ncol]) / double(st[jl].dp));
        }
        sm_h[jl] = h;
    }
    __syncthreads();

    const float D = 1.66f;
    const int ngpt = k.ngpt;
    const int L_end = NWt * CL;
    const float a_top = seed_at(seed_up, 0);      // pi a_0: U_bar at the top level
    const float b_bot = seed_at(seed_dn, nlay);   // pi b_N
    constexpr int QPR = 32 / CL;          // quantities per 32-value reduce-scatter
    constexpr int NRS = 4 / QPR;          // reduce-scatters per group for the 4 per-layer quantities
    double acc[NRS];
#pragma unroll
    for (int r = 0; r < NRS; ++r) acc[r] = 0.0;
    double acc_levbot = 0.0, acc_tsfc = 0.0;
    // forward fluxes (FLUX), as the forward kernel: level radiances [up | down] and layer
    // divergences reduce-scattered over the group's g-points, the bottom level separately
    double acc_flev = 0.0, acc_fdiv = 0.0, acc_fbot_up = 0.0, acc_fbot_dn = 0.0;

    for (int gg = 0; gg < k.ngroups; ++gg) {
        const int pb = CLUSTER ? 0 : (gg & 1);
        float4* const sm_mapA = sm_map0 + pb * NWt * 32 * 2;                 // (A, Bd, Bu, BUbar) per chunk
        float* const sm_mapB = reinterpret_cast<float*>(sm_mapA + NWt * 32);  // BIbar per chunk
        float* const sm_sfc = sm_sfc0 + pb * 32;
        const int g = 32 * gg + lane;
        const bool gv = g < ngpt;
        const int b0 = k.group_band0[gg];
        const int gband = gv ? k.gpt2band[g] : b0;
        const int slot = gband - b0;
        const int4 mg0 = minor_entry(k.minor_g[0], g, gv);
        const int4 mg1 = minor_entry(k.minor_g[1], g, gv);
        const int nm0 = __reduce_max_sync(0xffffffffu, mg0.x);
        const int nm1 = __reduce_max_sync(0xffffffffu, mg1.x);
        const float emis = gv ? __ldg(sfc_emis + gband + size_t(icol) * nband) : 0.f;

        for (int r = lane; r < CL * mgb; r += 32) {
            const int jl = w * CL + (r % CL);
            const int jj = j0 + jl;
            const int b = b0 + r / CL;
            if (jj < nlay && b < nband && k.band_lims[2 * b] < 32 * gg + 32) {
                Rec& R = recs[r];
                DRec& DR = drecs[r];
                const LayerState s = st[jl];
                record_weights(k, R, s, sm_cg + jl, LPC, b);
                const float* tp = k.totplnk + size_t(b) * k.nplanck;
                const bool bottom = jj == nlay - 1;
                R.aux = make_float4(interpolate1D(s.t, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp),
                                    interpolate1D(s.t_top, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp),
                                    interpolate1D(s.t_bot, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp),
                                    sm_cld[b * LPC + jl]);
                R.aux2 = bottom ? interpolate1D(ts, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp) : 0.f;
                build_drec(k, DR, s, sm_cg + jl, LPC, b, idx_o3, cd_internal);
                DR.dB = make_float4(interpolate1D_slope(s.t, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp),
                                    interpolate1D_slope(s.t_top, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp),
                                    interpolate1D_slope(s.t_bot, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp),
                                    bottom ? interpolate1D_slope(ts, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp)
                                           : 0.f);
            }
        }
        __syncwarp();

        // ---- forward pass 1 (recomputed) ----
        float vtau[CL], vpf[CL], omt[CL], sdn[CL], sup[CL];
        float A = 1.f, Bd = 0.f;
        float pf_bottom = 0.f;
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            const int jl = w * CL + i;
            const int j = j0 + jl;
            vtau[i] = 0.f; vpf[i] = 0.f; omt[i] = 0.f; sdn[i] = 0.f; sup[i] = 0.f;
            if (j < nlay && gv) {
                const Rec& R = recs[slot * CL + i];
                const float tau = tau_abs<DENSE>(k, R, g, R.a ? mg1 : mg0, R.a ? nm1 : nm0,
                                          &sm_sc4[jl * k.max_nscal].x, 4) + R.aux.w;
                const float4 p0 = __ldg(k.pfrac4 + (R.kb.x + g));
                const float4 p1 = __ldg(k.pfrac4 + (R.kb.y + g));
                const float pfrac = dot4(R.wpl0, p0) + dot4(R.wpl1, p1);
                vtau[i] = tau;
                vpf[i] = pfrac;
                lw_layer_terms(tau, D, pfrac * R.aux.x, pfrac * R.aux.z, pfrac * R.aux.y, omt[i], sdn[i], sup[i]);
                if (j == nlay - 1) {
                    for (int rr = 0; rr < CS; ++rr) at_rank(sm_sfc, rr)[lane] = pfrac * R.aux2;
                    pf_bottom = pfrac;
                }
            } else if (j == nlay - 1) {
                for (int rr = 0; rr < CS; ++rr) at_rank(sm_sfc, rr)[lane] = 0.f;
            }
            A = (1.f - omt[i]) * A;
            Bd = (1.f - omt[i]) * Bd + sdn[i];
        }
        float Bu = 0.f;
#pragma unroll
        for (int i = CL - 1; i >= 0; --i) Bu = (1.f - omt[i]) * Bu + sup[i];
        // reverse maps of the chunk
        float BU = 0.f;   // U_bar: top -> bottom of chunk
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            const int jl = w * CL + i;
            const int j = j0 + jl;
            const float a_next = (j + 1 < nlev) ? sm_a[jl + 1] : 0.f;
            const float hj = (j < nlay) ? sm_h[jl] : 0.f;
            BU = (1.f - omt[i]) * BU + a_next + hj * omt[i];
        }
        float BI = 0.f;   // I_bar: bottom -> top of chunk
#pragma unroll
        for (int i = CL - 1; i >= 0; --i) {
            const int jl = w * CL + i;
            const int j = j0 + jl;
            const float b_here = (j < nlev) ? sm_b[jl] : 0.f;
            const float hj = (j < nlay) ? sm_h[jl] : 0.f;
            BI = (1.f - omt[i]) * BI + b_here + hj * omt[i];
        }
        for (int rr = 0; rr < CS; ++rr) {
            at_rank(sm_mapA, rr)[Wg * 32 + lane] = make_float4(A, Bd, Bu, BU);
            at_rank(sm_mapB, rr)[Wg * 32 + lane] = BI;
        }
        csync();

        // ---- exchange ----
        float x = 0.f, xin = 0.f, u = a_top, uin = 0.f;
        for (int c = 0; c < NWt; ++c) {
            if (c == Wg) { xin = x; uin = u; }
            const float4 m = sm_mapA[c * 32 + lane];
            x = m.x * x + m.y;
            u = m.x * u + m.w;
        }
        // x = I at L_end (= I_N), u = U_bar at L_end (= U_bar_N)
        const float Ssrc = sm_sfc[lane];
        float y = x * (1.f - emis) + emis * Ssrc;
        float ib = (1.f - emis) * u + (L_end == nlay ? b_bot : 0.f);
        for (int c = NWt - 1; c > Wg; --c) {
            const float4 m = sm_mapA[c * 32 + lane];
            y = m.x * y + m.z;
            ib = m.x * ib + sm_mapB[c * 32 + lane];
        }
        const float Sbar = emis * u;

        // ---- forward pass 2: level radiances ----
        float vI[CL + 1], vU[CL + 1];
        vI[0] = xin;
#pragma unroll
        for (int i = 0; i < CL; ++i) vI[i + 1] = (1.f - omt[i]) * vI[i] + sdn[i];
        vU[CL] = y;
#pragma unroll
        for (int i = CL - 1; i >= 0; --i) vU[i] = (1.f - omt[i]) * vU[i + 1] + sup[i];
        if (FLUX) {
            float v[2 * CL], dv[CL];
#pragma unroll
            for (int i = 0; i < CL; ++i) {
                v[i] = vU[i];
                v[CL + i] = vI[i];
                dv[i] = omt[i] * (vI[i] + vU[i + 1]) - sdn[i] - sup[i];
            }
            ReduceScatter<2 * CL, 16>::run(v, lane);
            ReduceScatter<CL, 16>::run(dv, lane);
            acc_flev += double(v[0]);
            acc_fdiv += double(dv[0]);
            if (Wg == NWt - 1) {
                acc_fbot_up += double(warp_sum(vU[CL]));
                acc_fbot_dn += double(warp_sum(vI[CL]));
            }
        }
        // ---- reverse: U_bar per level (top down) ----
        float vUb[CL];
        {
            float ub = uin;
#pragma unroll
            for (int i = 0; i < CL; ++i) {
                vUb[i] = ub;
                const int jl = w * CL + i;
                const int j = j0 + jl;
                const float a_next = (j + 1 < nlev) ? sm_a[jl + 1] : 0.f;
                const float hj = (j < nlay) ? sm_h[jl] : 0.f;
                ub = (1.f - omt[i]) * ub + a_next + hj * omt[i];
            }
        }
        // ---- reverse: I_bar (bottom up) and the local chain per layer ----
        float gT[CL], gH[CL], gO[CL], gL[CL + 1], gS[CL];
#pragma unroll
        for (int i = 0; i <= CL; ++i) gL[i] = 0.f;
        float gTs = 0.f;
#pragma unroll
        for (int i = CL - 1; i >= 0; --i) {
            const int jl = w * CL + i;
            const int j = j0 + jl;
            const float hj = (j < nlay) ? sm_h[jl] : 0.f;
            const float omtb = hj * (vI[i] + vU[i + 1]) - ib * vI[i] - vUb[i] * vU[i + 1];
            const float sdnb = ib - hj, supb = vUb[i] - hj;
            const float b_here = (j < nlev) ? sm_b[jl] : 0.f;
            ib = (1.f - omt[i]) * ib + b_here + hj * omt[i];
            gT[i] = 0.f; gH[i] = 0.f; gO[i] = 0.f; gS[i] = 0.f;
            if (j < nlay && gv) {
                const Rec& R = recs[slot * CL + i];
                const DRec& DR = drecs[slot * CL + i];
                // table corners first: their latency overlaps the layer terms below
                const float4 c0 = __ldg(k.kmaj4 + (R.kb.x + g));
                const float4 c1 = __ldg(k.kmaj4 + (R.kb.y + g));
                const float4 p0 = __ldg(k.pfrac4 + (R.kb.x + g));
                const float4 p1 = __ldg(k.pfrac4 + (R.kb.y + g));
                const float pf = vpf[i];
                const float lay = pf * R.aux.x, ldn = pf * R.aux.z, lup = pf * R.aux.y;
                float om, fact, domt, dfact;
                lw_terms(vtau[i] * D, om, fact, domt, dfact);
                const float xb = sdnb * (domt * ldn + 2.f * dfact * (lay - ldn)) +
                                 supb * (domt * lup + 2.f * dfact * (lay - lup)) + omtb * domt;
                const float tb = D * xb;
                const float layb = 2.f * fact * (sdnb + supb);
                const float ldnb = sdnb * (om - 2.f * fact);
                const float lupb = supb * (om - 2.f * fact);
                float pfb = layb * R.aux.x + ldnb * R.aux.z + lupb * R.aux.y;
                float gt = layb * pf * DR.dB.x;
                gL[i] += lupb * pf * DR.dB.y;       // level above layer i
                gL[i + 1] += ldnb * pf * DR.dB.z;   // level below layer i
                if (j == nlay - 1) {
                    pfb += Sbar * R.aux2;
                    gTs += Sbar * pf_bottom * DR.dB.w;
                }
                float gh = 0.f, go = 0.f;
                tau_abs_adjoint<DENSE>(k, R, DR, g, R.a ? mg1 : mg0, R.a ? nm1 : nm0, tb, c0, c1, sm_sc4 + jl * k.max_nscal,
                                gt, gh, go);
                gt += pfb * (dot4(DR.pT0, p0) + dot4(DR.pT1, p1));
                gh += pfb * (dot4(DR.pH0, p0) + dot4(DR.pH1, p1));
                go += pfb * (dot4(DR.pO0, p0) + dot4(DR.pO1, p1));
                gT[i] = gt;
                gH[i] = gh;
                gO[i] = go;
                gS[i] = tb;   // cloud tau_bar of this lane's band (slot)
            }
        }

        // ---- sums over the 32 g-points ----
        {
            float v[32];
            // quantity order: T, H, O, level
            if (CL == 8) {
#pragma unroll
                for (int i = 0; i < CL; ++i) { v[i] = gT[i]; v[8 + i] = gH[i]; v[16 + i] = gO[i]; v[24 + i] = gL[i]; }
                ReduceScatter<32, 16>::run(v, lane);
                acc[0] += double(v[0]);
            } else {
#pragma unroll
                for (int i = 0; i < CL; ++i) { v[i] = gT[i]; v[CL + i] = gH[i]; }
                ReduceScatter<32, 16>::run(v, lane);
                acc[0] += double(v[0]);
#pragma unroll
                for (int i = 0; i < CL; ++i) { v[i] = gO[i]; v[CL + i] = gL[i]; }
                ReduceScatter<32, 16>::run(v, lane);
                acc[NRS - 1] += double(v[0]);
            }
        }
        {
            float v[2 * CL];
#pragma unroll
            for (int i = 0; i < CL; ++i) { v[i] = slot == 0 ? gS[i] : 0.f; v[CL + i] = slot == 1 ? gS[i] : 0.f; }
            ReduceScatter<2 * CL, 16>::run(v, lane);
            constexpr int SH = (CL == 16) ? 0 : 1;
            const int vi = lane >> SH;
            const int sl = vi / CL, jl = w * CL + (vi % CL);
            const int b = b0 + sl;
            if ((lane & ((1 << SH) - 1)) == 0 && j0 + jl < nlay && b < nband && k.band_lims[2 * b] < 32 * gg + 32)
                sm_tb[b * LPC + jl] += v[0];
        }
        acc_levbot += double(warp_sum(gL[CL]));
        if (Wg == (nlay - 1) / CL) acc_tsfc += double(warp_sum(gTs));
        if (CLUSTER) csync();   // maps and the surface source are rewritten by the next group
    }

    // ---- outputs ----
    if (FLUX) {
        constexpr int SH_LEV = (CL == 16) ? 0 : 1;   // lane L holds value L >> SH_LEV
        constexpr int SH_DIV = (CL == 16) ? 1 : 2;
        const int vidx = lane >> SH_LEV;
        const double other = __shfl_xor_sync(0xffffffffu, acc_flev, CL << SH_LEV);
        if ((lane & ((1 << SH_LEV) - 1)) == 0 && vidx < CL) {
            const int j = j0 + w * CL + vidx;
            if (j < nlay) {
                const size_t o = icol + size_t(top_at_1 ? j : nlay - j) * ncol;
                const double up = pi * acc_flev, dn = pi * other;
                out.flux_up[o] = float(up);
                out.flux_dn[o] = float(dn);
                out.flux_net[o] = float(dn - up);
            }
        }
        if ((lane & ((1 << SH_DIV) - 1)) == 0 && (lane >> SH_DIV) < CL) {
            const int jl = w * CL + (lane >> SH_DIV), j = j0 + jl;
            if (j < nlay) {
                const double g0_cp = 9.80665 / 1004.64;
                out.heating_rate[icol + size_t(top_at_1 ? j : nlay - 1 - j) * ncol] =
                    float(g0_cp * 86400.0 * pi * acc_fdiv / double(st[jl].dp));
            }
        }
        if (Wg == NWt - 1 && lane == 0) {
            const size_t o = icol + size_t(top_at_1 ? nlay : 0) * ncol;
            out.flux_up[o] = float(pi * acc_fbot_up);
            out.flux_dn[o] = float(pi * acc_fbot_dn);
            out.flux_net[o] = float(pi * (acc_fbot_dn - acc_fbot_up));
        }
    }
    if (lane == 0) sm_levbot[w] = acc_levbot;
    csync();
    // level gradient of the bottom level of the previous chunk (another CTA's for w = 0)
    double prev_levbot = 0.0;
    if (w > 0)
        prev_levbot = sm_levbot[w - 1];
    else if (CLUSTER && rank > 0)
        prev_levbot = remote(cluster, sm_levbot, rank - 1)[NWc - 1];
#pragma unroll
    for (int r = 0; r < NRS; ++r) {
        const int vi = lane;                         // RS<32>: lane L holds value L
        const int q = r * QPR + vi / CL;             // 0 T, 1 H, 2 O, 3 level
        const int jl = w * CL + (vi % CL);
        const int j = j0 + jl;
        const double val = acc[r];
        if (q < 3) {
            if (j < nlay) {
                const size_t o = icol + size_t(top_at_1 ? j : nlay - 1 - j) * ncol;
                float* dst = q == 0 ? out.tlay : (q == 1 ? out.h2o : out.o3);
                if (dst) dst[o] = float(val);
            }
        } else if (j <= nlay && out.tlev) {
            double v = val;
            if ((vi % CL) == 0 && Wg > 0) v += prev_levbot;
            out.tlev[icol + size_t(top_at_1 ? j : nlay - j) * ncol] = float(v);
        }
    }
    if (Wg == NWt - 1 && lane == 0) {
        if (L_end == nlay && out.tlev)
            out.tlev[icol + size_t(top_at_1 ? nlay : 0) * ncol] = float(sm_levbot[w]);
    }
    if (Wg == (nlay - 1) / CL && lane == 0 && out.tsfc) out.tsfc[icol] = float(acc_tsfc);
    // cloud gradients: sum over bands of tau_bar(band) * dtau_cloud(band)/dx
    for (int jl = threadIdx.x; jl < LPC; jl += blockDim.x) {
        const int j = j0 + jl;
        if (j >= nlay) break;
        const int l = top_at_1 ? j : nlay - 1 - j;
        const size_t cl = icol + size_t(l) * ncol;
        float4 gsum = make_float4(0.f, 0.f, 0.f, 0.f);
        if (cld.present) {
            const float lw = cld.lwp[cl], iw = cld.iwp[cl], rl = cld.rel[cl], ri = cld.rei[cl];
            for (int b = 0; b < nband; ++b) {
                const float tb = sm_tb[b * LPC + jl];
                const float4 d = cloud_1scl_partials(cld.L, lw, iw, rl, ri, b);
                gsum.x += tb * d.x;
                gsum.y += tb * d.y;
                gsum.z += tb * d.z;
                gsum.w += tb * d.w;
            }
        }
        if (out.lwp) out.lwp[cl] = gsum.x;
        if (out.iwp) out.iwp[cl] = gsum.y;
        if (out.rel) out.rel[cl] = gsum.z;
        if (out.rei) out.rei[cl] = gsum.w;
    }
    if (CLUSTER) cluster.sync();   // no CTA leaves while its shared memory may still be read remotely
}

// Up to 128 layers (CL = 8) or 256 (CL = 16, if the records fit) one CTA of ceil(nlay / CL)
// warps per column; beyond, clusters of CS = ceil(nlay / 128) CTAs of 16 warps (CL = 8).
template <int CL, bool FLUX, bool DENSE>
int launch_lw_adjoint(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay, int idx_o3, const float* play,
                      const float* plev, const float* tlay, const float* tlev, const float* tsfc, const float* col_dry,
                      const GasSet<float>& gs, const float* lwp, const float* iwp, const float* rel, const float* rei,
                      const float* emis, const float* su, const float* sd, const float* sh, const AdjOut& out,
                      cudaStream_t stream)
{
    const KdistView<float>& v = k->v32;
    const int NW1 = (nlay + CL - 1) / CL;
    const size_t smem1 = adj_layout(NW1 * CL, v.ngas, v.nband, NW1, NW1, CL, v.max_group_bands, 2, v.max_nscal).total;
    RB_CHECK_ARG(CL == 8 || NW1 <= 8, "adjoint_lw: chunk 16 covers at most 128 layers");
    int CS = 1, NWc = NW1;
    size_t smem = smem1;
    if (NW1 > 16 || smem1 > 227 * 1024) {
        RB_CHECK_ARG(CL == 8, "adjoint_lw: columns deeper than one CTA holds need chunk 8");
        NWc = 16;
        CS = (nlay + 16 * CL - 1) / (16 * CL);
        RB_CHECK_ARG(CS <= 8, "adjoint_lw: at most 1024 layers");
        smem = adj_layout(16 * CL, v.ngas, v.nband, 16, CS * 16, CL, v.max_group_bands, 1, v.max_nscal).total;
    }
    if (smem > 227 * 1024) return fail(RRTMGP_B200_ERR_UNSUPPORTED, "adjoint_lw: shared memory need exceeds 227 KB");
    static PerDeviceOnce attr;
    const int ast = attr.run([] {
        const cudaError_t e = cudaFuncSetAttribute(lw_adjoint_kernel<CL, false, FLUX, DENSE>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        if (e != cudaSuccess) return e;
        return cudaFuncSetAttribute(lw_adjoint_kernel<8, true, FLUX, DENSE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    227 * 1024);
    }, "adjoint_lw attribute");
    if (ast) return ast;
    AdjCloud ca{};
    if (c) {
        ca.L = CloudLut<float>{c->nband, c->nsize_liq, c->nsize_ice, float(c->radliq_lwr), float(c->liq_step),
                               float(c->radice_lwr), float(c->ice_step), c->lut32};
        ca.lwp = lwp; ca.iwp = iwp; ca.rel = rel; ca.rei = rei;
        ca.present = 1;
    }
    if (CS == 1) {
        lw_adjoint_kernel<CL, false, FLUX, DENSE><<<ncol, NWc * 32, smem, stream>>>(v, gs, ca, ncol, nlay, 1, idx_o3, col_dry ? 0 : 1,
                                                                  play, plev, tlay, tlev, tsfc, col_dry, emis, su, sd,
                                                                  sh, out);
        RB_LAUNCH("lw_adjoint_kernel");
        return RRTMGP_B200_OK;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(ncol) * CS);
    cfg.blockDim = dim3(NWc * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = unsigned(CS);
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    RB_CUDA(cudaLaunchKernelEx(&cfg, lw_adjoint_kernel<8, true, FLUX, DENSE>, v, gs, ca, ncol, nlay, CS, idx_o3, col_dry ? 0 : 1, play,
                               plev, tlay, tlev, tsfc, col_dry, emis, su, sd, sh, out),
            "lw_adjoint_kernel launch");
    return RRTMGP_B200_OK;
}

}  // namespace

int adjoint_lw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay, const float* play, const float* plev,
                   const float* tlay, const float* tlev, const float* tsfc, const float* col_dry,
                   const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp, const float* rel,
                   const float* rei, const float* sfc_emis, const float* seed_up, const float* seed_dn,
                   const float* seed_hr, float* g_tlay, float* g_tlev, float* g_tsfc, float* g_h2o, float* g_o3,
                   float* g_lwp, float* g_iwp, float* g_rel, float* g_rei, float* flux_up, float* flux_dn,
                   float* flux_net, float* heating_rate, int chunk, void* stream)
{
    RB_CHECK_ARG(k && k->info.is_longwave, "adjoint_lw: need a longwave k-distribution");
    if (const int dst = check_device(k->device, "adjoint_lw")) return dst;
    const bool with_flux = flux_up != nullptr;
    RB_CHECK_ARG(!with_flux || (flux_dn && flux_net && heating_rate), "forward_adjoint_lw: null flux array");
    RB_CHECK_ARG(ncol > 0 && nlay > 1, "adjoint_lw: ncol > 0 and nlay > 1 required");
    RB_CHECK_ARG(play && plev && tlay && tlev && tsfc && sfc_emis, "adjoint_lw: null input array");
    RB_CHECK_ARG(!c || (lwp && iwp && rel && rei), "adjoint_lw: cloud arrays required with a cloud handle");
    RB_CHECK_ARG(!c || c->nband == k->info.nband, "adjoint_lw: cloud and gas band counts differ");
    const KdistView<float>& v = k->v32;
    if (!fused_layout_ok(v, false, 2))
        return fail(RRTMGP_B200_ERR_UNSUPPORTED, "adjoint_lw: k-distribution layout not supported by the adjoint kernel");
    GasSet<float> gs;
    int st = make_gas_set<float>(k, ncol, nlay, gases, ngases, gs);
    if (st) return st;
    int idx_o3 = 0;
    for (size_t i = 0; i < k->gas_names.size(); ++i)
        if (k->gas_names[i] == "o3") idx_o3 = int(i) + 1;
    const AdjOut out{g_tlay, g_tlev, g_tsfc, g_h2o, g_o3, g_lwp, g_iwp, g_rel, g_rei,
                     flux_up, flux_dn, flux_net, heating_rate};
    cudaStream_t s = as_stream(stream);
    const bool dense = v.max_minor_per_g > 3;
#define RB_LW_ADJ(CLv, F, D)                                                                                        \
    launch_lw_adjoint<CLv, F, D>(k, c, ncol, nlay, idx_o3, play, plev, tlay, tlev, tsfc, col_dry, gs, lwp, iwp, rel, \
                                 rei, sfc_emis, seed_up, seed_dn, seed_hr, out, s)
    if (dense) {
        if (chunk == 16) return with_flux ? RB_LW_ADJ(16, true, true) : RB_LW_ADJ(16, false, true);
        return with_flux ? RB_LW_ADJ(8, true, true) : RB_LW_ADJ(8, false, true);
    }
    if (chunk == 16) return with_flux ? RB_LW_ADJ(16, true, false) : RB_LW_ADJ(16, false, false);
    return with_flux ? RB_LW_ADJ(8, true, false) : RB_LW_ADJ(8, false, false);
#undef RB_LW_ADJ
}

}  // namespace rrtmgp_b200

extern "C" int rrtmgp_b200_adjoint_lw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* tlev, const float* tsfc,
        const float* col_dry, const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp,
        const float* rel, const float* rei, const float* sfc_emis, const float* seed_flux_up,
        const float* seed_flux_dn, const float* seed_heating_rate, float* grad_tlay, float* grad_tlev,
        float* grad_tsfc, float* grad_h2o, float* grad_o3, float* grad_lwp, float* grad_iwp, float* grad_rel,
        float* grad_rei, int chunk, void* stream)
{
    return rrtmgp_b200::adjoint_lw_f32(k, c, ncol, nlay, play, plev, tlay, tlev, tsfc, col_dry, gases, ngases, lwp, iwp,
                                       rel, rei, sfc_emis, seed_flux_up, seed_flux_dn, seed_heating_rate, grad_tlay,
                                       grad_tlev, grad_tsfc, grad_h2o, grad_o3, grad_lwp, grad_iwp, grad_rel, grad_rei,
                                       nullptr, nullptr, nullptr, nullptr, chunk, stream);
}

extern "C" int rrtmgp_b200_forward_adjoint_lw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* tlev, const float* tsfc,
        const float* col_dry, const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp,
        const float* rel, const float* rei, const float* sfc_emis, const float* seed_flux_up,
        const float* seed_flux_dn, const float* seed_heating_rate, float* grad_tlay, float* grad_tlev,
        float* grad_tsfc, float* grad_h2o, float* grad_o3, float* grad_lwp, float* grad_iwp, float* grad_rel,
        float* grad_rei, float* flux_up, float* flux_dn, float* flux_net, float* heating_rate, int chunk,
        void* stream)
{
    RB_CHECK_ARG(flux_up, "forward_adjoint_lw: null flux array");
    return rrtmgp_b200::adjoint_lw_f32(k, c, ncol, nlay, play, plev, tlay, tlev, tsfc, col_dry, gases, ngases, lwp, iwp,
                                       rel, rei, sfc_emis, seed_flux_up, seed_flux_dn, seed_heating_rate, grad_tlay,
                                       grad_tlev, grad_tsfc, grad_h2o, grad_o3, grad_lwp, grad_iwp, grad_rel, grad_rei,
                                       flux_up, flux_dn, flux_net, heating_rate, chunk, stream);
}
