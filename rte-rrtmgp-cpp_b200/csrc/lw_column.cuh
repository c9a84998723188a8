// Fused longwave forward: gas optics + cloud optics (1scl, added by band) + no-scattering
// solver + broadband fluxes + heating rates for whole columns, without materialising any
// (ncol, nlay, ngpt) array.  The staged equivalent is the sequence of
// Radiation_solver_longwave::solve_gpu (src_test/Radiation_solver.cu:467-615).
//
// Per group of 32 g-points (see fused_common.cuh for the thread mapping):
//   1. each warp writes the records of its layer chunk;
//   2. pass 1: per (layer, g-point) tau, Planck fraction, 1 - transmissivity and the two
//      linear-in-tau sources (lw_solver_noscat step 1) stay in registers; the warp composes
//      its chunk's affine down and up maps x -> A x + B and publishes them;
//   3. after one barrier every thread composes the maps of the other chunks to get its
//      chunk's incoming down and up radiances (surface: radn_dn * (1 - emis) + emis * sfc_src);
//   4. pass 2 re-sweeps the registers: level radiances and the per-layer absorbed radiance
//      omt * (I_dn(top) + I_up(bottom)) - S_dn - S_up, which gives heating rates without
//      differencing two nearly equal FP32 level fluxes;
//   5. a warp reduce-scatter (31 shuffles per 32 values) sums over the 32 g-points and every
//      lane accumulates one level (or layer) in FP64.
#pragma once
#include "fused_common.cuh"

namespace rrtmgp_b200 {
namespace fused {

struct CloudArgs {
    CloudLut<float> L;
    const float* lwp;
    const float* iwp;
    const float* rel;
    const float* rei;
    int present;
};

// Arguments of the per-grid longwave kernel (passed by value: kernel parameters).
struct LwGridIo {
    int ncol_, nlay_;
    const float *play_, *plev_, *tlay_, *tlev_, *tsfc_, *col_dry_, *emis_;
    float *up_, *dn_, *net_, *hr_;
    GasSet<float> gs_;
    CloudArgs cld_;
    __device__ __forceinline__ int ncol() const { return ncol_; }
    __device__ __forceinline__ int nlay() const { return nlay_; }
    __device__ __forceinline__ const float* play() const { return play_; }
    __device__ __forceinline__ const float* plev() const { return plev_; }
    __device__ __forceinline__ const float* tlay() const { return tlay_; }
    __device__ __forceinline__ const float* tlev() const { return tlev_; }
    __device__ __forceinline__ const float* tsfc() const { return tsfc_; }
    __device__ __forceinline__ const float* col_dry() const { return col_dry_; }
    __device__ __forceinline__ const float* emis() const { return emis_; }
    __device__ __forceinline__ float* up() const { return up_; }
    __device__ __forceinline__ float* dn() const { return dn_; }
    __device__ __forceinline__ float* net() const { return net_; }
    __device__ __forceinline__ float* hr() const { return hr_; }
    __device__ __forceinline__ const GasSet<float>& gs() const { return gs_; }
    __device__ __forceinline__ const CloudArgs& cloud() const { return cld_; }
};

__device__ __forceinline__ void build_lw_record(const KdistView<float>& k, Rec& R, const LayerState& s,
                                                const float* cg, int nlay, int b, float tau_cld, bool bottom,
                                                float tsfc)
{
    record_weights(k, R, s, cg, nlay, b);
    const float* tp = k.totplnk + size_t(b) * k.nplanck;
    R.aux = make_float4(interpolate1D(s.t, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp),
                        interpolate1D(s.t_top, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp),
                        interpolate1D(s.t_bot, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp), tau_cld);
    R.aux2 = bottom ? interpolate1D(tsfc, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp) : 0.f;
}

// One column by the warps that context cx names (cx.nwarps() warps of CL layers each,
// nlay <= cx.nwarps() * CL; chunks past nlay are identity layers).  Context and arguments are
// read through accessors at every use (cx: column index, warp, shared memory, barrier; io: grid
// sizes, arrays, gas set, cloud arrays) so that the batched kernel, which keeps them in shared
// memory, holds no register for them across the column (see LwGridIo / CtaCtx for the per-grid
// kernel, where they are launch constants).
// PAIR (8-layer chunks): the records of groups gg and gg + 1 are built together at even gg
// into two buffers (one group's 16 records per warp leave half the lanes idle).
template <int CL, bool PAIR = false, bool DENSE = false, class Cx, class Io>
__device__ __forceinline__ void lw_forward_column(const Cx& cx, const KdistView<float>& k, const Io& io)
{
    static_assert(CL == 8 || CL == 16, "chunk length");
    constexpr bool P2 = PAIR && CL == 8;
    const int lane = threadIdx.x & 31;
    const int nband = k.nband;
    // layer state of the layers [L0, L0 + NL) in this CTA's shared memory, indexed j - L0
    const int L0 = cx.layer0(), NL = cx.nloc(io.nlay());
    const int NWloc = cx.nthreads() >> 5;
    // sized by capacity (NWloc CL layers), the same in every CTA of a cluster: the chunk maps
    // stored into another CTA's shared memory land at the offset this CTA uses
    const SmemLayout SL = smem_layout(NWloc * CL, k.ngas, nband, 1, cx.nwarps(), 2, CL,
                                      k.max_group_bands * (P2 ? 2 : 1), k.max_nscal, NWloc);
    unsigned char* const smem_raw = cx.smem();
    LayerState* st = reinterpret_cast<LayerState*>(smem_raw + SL.state);
    float* sm_cg = reinterpret_cast<float*>(smem_raw + SL.cg);
    float* sm_sc = reinterpret_cast<float*>(smem_raw + SL.scal);   // [layer][scaling kind]
    float* sm_cld = reinterpret_cast<float*>(smem_raw + SL.cloud);
    // chunk maps and surface source are double-buffered by group parity, so a warp can
    // start the next group while others still read this group's (one barrier per group)
    float4* const sm_maps0 = reinterpret_cast<float4*>(smem_raw + SL.maps);
    float* const sm_sfc0 = reinterpret_cast<float*>(smem_raw + SL.sfc);
    Rec* const recs0 = reinterpret_cast<Rec*>(smem_raw + SL.recs) + cx.lwarp() * CL * k.max_group_bands;
    const int rbuf = NWloc * CL * k.max_group_bands;   // records per buffer

    bool top_at_1;
    float ts;
    {
        const int icol = cx.icol(), ncol = io.ncol(), nlay = io.nlay();
        const float* play = io.play();
        top_at_1 = play[icol] < play[icol + size_t(nlay - 1) * ncol];
        ts = io.tsfc()[icol];
        setup_layer_range(k, io.gs(), ncol, nlay, icol, top_at_1, play, io.plev(), io.tlay(), io.tlev(), io.col_dry(),
                          st, sm_cg, NL, L0, NL, cx.tid(), cx.nthreads());
        const CloudArgs cld = io.cloud();
        for (int idx = cx.tid(); idx < NL * nband; idx += cx.nthreads()) {
            const int jl = idx % NL, b = idx / NL, j = L0 + jl;
            float tau = 0.f, s, g;
            if (cld.present) {
                const int l = top_at_1 ? j : nlay - 1 - j;
                const size_t cl = icol + size_t(l) * ncol;
                const CloudPoint<float> cp = cloud_point(cld.L, cld.lwp[cl], cld.iwp[cl], cld.rel[cl], cld.rei[cl]);
                cloud_band<float, false>(cld.L, cp, b, tau, s, g);
            }
            sm_cld[b * NL + jl] = tau;
        }
    }
    cx.sync();
    layer_minor_scalings(k, st, sm_cg, NL, sm_sc, NL, cx.tid(), cx.nthreads());
    cx.sync();

    const float D = 1.66f;                 // single-angle secant (Rte_lw.cpp:101-113)
    const int ngpt = k.ngpt;
    double acc_lev = 0.0, acc_div = 0.0, acc_bot_up = 0.0, acc_bot_dn = 0.0;

    for (int gg = 0; gg < k.ngroups; ++gg) {
        const int nlay = io.nlay();
        float4* const sm_maps = sm_maps0 + (gg & 1) * cx.nwarps() * 32;
        float* const sm_sfc = sm_sfc0 + (gg & 1) * 32;
        const int g = 32 * gg + lane;
        const bool gv = g < ngpt;
        const int b0 = k.group_band0[gg];
        const int gband = gv ? k.gpt2band[g] : b0;
        const int slot = gband - b0;
        const int4 mg0 = minor_entry(k.minor_g[0], g, gv);
        const int4 mg1 = minor_entry(k.minor_g[1], g, gv);
        const int nm0 = __reduce_max_sync(0xffffffffu, mg0.x);
        const int nm1 = __reduce_max_sync(0xffffffffu, mg1.x);

        // 1. records of this warp's chunk
        Rec* const recs = recs0 + (P2 ? (gg & 1) : 0) * rbuf;
        if (!P2 || (gg & 1) == 0) {
            const int nrec = CL * k.max_group_bands;
            for (int t = lane; t < (P2 ? 2 : 1) * nrec; t += 32) {
                const int gq = gg + t / nrec, r = t % nrec;
                if (gq >= k.ngroups) continue;
                const int jj = cx.warp() * CL + (r % CL), jl = jj - L0;
                const int b = k.group_band0[gq] + r / CL;
                if (jj < nlay && b < nband && k.band_lims[2 * b] < 32 * gq + 32)
                    build_lw_record(k, recs0[(P2 ? (gq & 1) : 0) * rbuf + r], st[jl], sm_cg + jl, NL, b,
                                    sm_cld[b * NL + jl], jj == nlay - 1, ts);
            }
        }
        __syncwarp();

        // 2. pass 1
        float omt[CL], sdn[CL], sup[CL];
        float Ad = 1.f, Bd = 0.f;
        const int j0 = cx.warp() * CL;
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            const int j = j0 + i;
            omt[i] = 0.f; sdn[i] = 0.f; sup[i] = 0.f;
            if (j < nlay && gv) {
                const Rec& R = recs[slot * CL + i];
                const float tau =
                    tau_abs<DENSE>(k, R, g, R.a ? mg1 : mg0, R.a ? nm1 : nm0, sm_sc + (j - L0) * k.max_nscal) +
                    R.aux.w;
                const float4 p0 = __ldg(k.pfrac4 + (R.kb.x + g));
                const float4 p1 = __ldg(k.pfrac4 + (R.kb.y + g));
                const float pfrac = (R.wpl0.x * p0.x + R.wpl0.y * p0.y + R.wpl0.z * p0.z + R.wpl0.w * p0.w) +
                                    (R.wpl1.x * p1.x + R.wpl1.y * p1.y + R.wpl1.z * p1.z + R.wpl1.w * p1.w);
                lw_layer_fast(tau, D, pfrac * R.aux.x, pfrac * R.aux.z, pfrac * R.aux.y, omt[i], sdn[i], sup[i]);
                if (j == nlay - 1) cx.put(&sm_sfc[lane], pfrac * R.aux2);
            } else if (j == nlay - 1) {
                cx.put(&sm_sfc[lane], 0.f);
            }
            Ad = (1.f - omt[i]) * Ad;
            Bd = (1.f - omt[i]) * Bd + sdn[i];
        }
        float Au = 1.f, Bu = 0.f;
#pragma unroll
        for (int i = CL - 1; i >= 0; --i) {
            Au = (1.f - omt[i]) * Au;
            Bu = (1.f - omt[i]) * Bu + sup[i];
        }
        cx.put(&sm_maps[cx.warp() * 32 + lane], make_float4(Ad, Bd, Au, Bu));
        cx.sync();

        // 3. incoming radiances of the chunk (no incident longwave flux at the top)
        const int w = cx.warp(), NW = cx.nwarps();
        float x = 0.f, xin = 0.f;
        for (int c = 0; c < NW; ++c) {
            if (c == w) xin = x;
            const float4 m = sm_maps[c * 32 + lane];
            x = m.x * x + m.y;
        }
        const float emis = gv ? __ldg(io.emis() + gband + size_t(cx.icol()) * nband) : 0.f;
        const float S = x * (1.f - emis) + emis * sm_sfc[lane];
        float y = S;
        for (int c = NW - 1; c > w; --c) {
            const float4 m = sm_maps[c * 32 + lane];
            y = m.z * y + m.w;
        }

        // 4. pass 2
        float v[2 * CL], dv[CL];
        float rd = xin;
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            v[CL + i] = rd;  // down radiance at the top of layer i
            rd = (1.f - omt[i]) * rd + sdn[i];
        }
        float ru = y;
#pragma unroll
        for (int i = CL - 1; i >= 0; --i) {
            dv[i] = omt[i] * (v[CL + i] + ru) - sdn[i] - sup[i];
            ru = (1.f - omt[i]) * ru + sup[i];
            v[i] = ru;       // up radiance at the top of layer i
        }
        // 5. sums over the 32 g-points of the group
        ReduceScatter<2 * CL, 16>::run(v, lane);
        ReduceScatter<CL, 16>::run(dv, lane);
        acc_lev += double(v[0]);
        acc_div += double(dv[0]);
        if (w == NW - 1) {
            acc_bot_up += double(warp_sum(S));
            acc_bot_dn += double(warp_sum(rd));
        }
    }

    // Outputs.  Fluxes = 2 pi w * (sum of radiances) with w = 0.5.
    const int w = cx.warp(), NW = cx.nwarps(), icol = cx.icol(), ncol = io.ncol(), nlay = io.nlay();
    float* const flux_up = io.up();
    float* const flux_dn = io.dn();
    float* const flux_net = io.net();
    float* const heating_rate = io.hr();
    const double pi = 3.14159265358979323846;
    constexpr int SH_LEV = (CL == 16) ? 0 : 1;   // lane L holds value L >> SH_LEV
    constexpr int SH_DIV = (CL == 16) ? 1 : 2;
    const int vidx = lane >> SH_LEV;
    const double other = __shfl_xor_sync(0xffffffffu, acc_lev, CL << SH_LEV);
    if ((lane & ((1 << SH_LEV) - 1)) == 0 && vidx < CL) {
        const int jl = w * CL + vidx;
        if (jl < nlay) {
            const int al = top_at_1 ? jl : nlay - jl;
            const size_t o = icol + size_t(al) * ncol;
            const double up = pi * acc_lev, dn = pi * other;
            flux_up[o] = float(up);
            flux_dn[o] = float(dn);
            flux_net[o] = float(dn - up);
        }
    }
    if ((lane & ((1 << SH_DIV) - 1)) == 0) {
        const int jl = w * CL + (lane >> SH_DIV);
        if (jl < nlay && (lane >> SH_DIV) < CL) {
            const int l = top_at_1 ? jl : nlay - 1 - jl;
            const double g0_cp = 9.80665 / 1004.64;
            heating_rate[icol + size_t(l) * ncol] = float(g0_cp * 86400.0 * pi * acc_div / double(st[jl - L0].dp));
        }
    }
    if (w == NW - 1 && lane == 0) {
        const int al = top_at_1 ? nlay : 0;
        const size_t o = icol + size_t(al) * ncol;
        flux_up[o] = float(pi * acc_bot_up);
        flux_dn[o] = float(pi * acc_bot_dn);
        flux_net[o] = float(pi * (acc_bot_dn - acc_bot_up));
    }
}

}  // namespace fused
}  // namespace rrtmgp_b200
