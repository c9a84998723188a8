// Fused shortwave forward: gas optics (major + minor absorption, Rayleigh) + cloud optics
// (2str, delta-scaled, added by band) + two-stream layer coefficients + adding method +
// broadband fluxes + heating rates for whole columns, with no (ncol, nlay, ngpt) array.
// The staged equivalent is Radiation_solver_shortwave::solve_gpu
// (src_test/Radiation_solver.cu:683-950) followed by the heating-rate formula.
//
// Thread mapping as in the longwave kernel (fused_common.cuh): one CTA per column, lane =
// g-point of the current group of 32, warp w = layer chunk [w*CL, (w+1)*CL) from the top.
//
// Per group of 32 g-points:
//   1. pass 1 (per layer, in registers): optical properties, two-stream coefficients
//      (R, T, Rdir, Tdir, Tnoscat) and the layer absorptances; the chunk's direct-beam
//      transmission product PT and its adding composite (R_up, R_dn, T, U, D) with sources
//      relative to a unit direct flux at the chunk top;
//   2. barrier; every warp forms its direct flux at the chunk top from the PT of the chunks
//      above, emits the direct fluxes and direct absorption of its layers and scales its
//      composite's sources to absolute values;
//   3. barrier; every warp walks the composites from the surface up: albedo and upward
//      source at its chunk bottom, and the affine maps fd_bot = F fd_top + G of the chunks
//      above it, composed into its incident diffuse flux;
//   4. pass 2 (bottom-up within the chunk): albedo and source per level (adding_kernel);
//      pass 3 (top-down): diffuse down/up fluxes per level and per-layer diffuse absorption;
//   5. warp reduce-scatter over the 32 g-points, FP64 accumulation per lane.
// Heating rates use the per-layer absorbed flux (direct: F_dir (1 - Tn - Rdir - Tdir);
// diffuse: (F_dn(top) + F_up(bottom)) (1 - R - T)), which equals the net-flux divergence of
// the adding solution but keeps its relative accuracy in the ~0.1 Pa top layers.
#pragma once
#include "sw_common.cuh"

namespace rrtmgp_b200 {
namespace fused {

// Arguments of the per-grid shortwave kernel (passed by value: kernel parameters).
struct SwGridIo {
    int ncol_, nlay_;
    const float *play_, *plev_, *tlay_, *col_dry_, *mu0_, *tsi_, *alb_dir_, *alb_dif_;
    float *up_, *dn_, *dir_, *net_, *hr_;
    GasSet<float> gs_;
    SwCloudArgs cld_;
    SwAerosolArgs aer_;
    __device__ __forceinline__ int ncol() const { return ncol_; }
    __device__ __forceinline__ int nlay() const { return nlay_; }
    __device__ __forceinline__ const float* play() const { return play_; }
    __device__ __forceinline__ const float* plev() const { return plev_; }
    __device__ __forceinline__ const float* tlay() const { return tlay_; }
    __device__ __forceinline__ const float* col_dry() const { return col_dry_; }
    __device__ __forceinline__ const float* mu0() const { return mu0_; }
    __device__ __forceinline__ const float* tsi() const { return tsi_; }
    __device__ __forceinline__ const float* alb_dir() const { return alb_dir_; }
    __device__ __forceinline__ const float* alb_dif() const { return alb_dif_; }
    __device__ __forceinline__ float* up() const { return up_; }
    __device__ __forceinline__ float* dn() const { return dn_; }
    __device__ __forceinline__ float* dir() const { return dir_; }
    __device__ __forceinline__ float* net() const { return net_; }
    __device__ __forceinline__ float* hr() const { return hr_; }
    __device__ __forceinline__ const GasSet<float>& gs() const { return gs_; }
    __device__ __forceinline__ const SwCloudArgs& cloud() const { return cld_; }
    __device__ __forceinline__ const SwAerosolArgs& aerosol() const { return aer_; }
};

// One column by the warps that context cx names (cx.nwarps() warps of CL layers each,
// nlay <= cx.nwarps() * CL; chunks past nlay are identity layers).  Context and arguments are
// read through accessors at every use, as in lw_forward_column.
// PAIR (8-layer chunks): the records of groups gg and gg + 1 are built together at even gg
// into two buffers (one group's 16 records per warp leave half the lanes idle).
template <int CL, bool PAIR = false, bool DENSE = false, class Cx, class Io>
__device__ __forceinline__ void sw_forward_column(const Cx& cx, const KdistView<float>& k, const Io& io)
{
    static_assert(CL == 8 || CL == 16, "chunk length");
    constexpr bool P2 = PAIR && CL == 8;
    const int lane = threadIdx.x & 31;
    const int nband = k.nband;
    const bool with_aer = io.aerosol().present != 0;
    // the "cloud" region holds the aerosol (tau, tau ssa, tau ssa g, tau (1 - ssa)) per (band, layer)
    // layer state of the layers [L0, L0 + NL) in this CTA's shared memory, indexed j - L0
    const int L0 = cx.layer0(), NL = cx.nloc(io.nlay());
    const int NWloc = cx.nthreads() >> 5;
    // sized by capacity (NWloc CL layers), the same in every CTA of a cluster (as lw_forward_column)
    const SmemLayout SL = smem_layout(NWloc * CL, k.ngas, nband, with_aer ? 4 : 0, cx.nwarps(), 3, CL,
                                      k.max_group_bands * (P2 ? 2 : 1), k.max_nscal, NWloc);
    unsigned char* const smem_raw = cx.smem();
    LayerState* st = reinterpret_cast<LayerState*>(smem_raw + SL.state);
    float* sm_cg = reinterpret_cast<float*>(smem_raw + SL.cg);
    float* sm_sc = reinterpret_cast<float*>(smem_raw + SL.scal);   // [layer][scaling kind]
    float* sm_pt = reinterpret_cast<float*>(smem_raw + SL.maps);                            // [NW][32]
    float4* sm_comp = reinterpret_cast<float4*>(smem_raw + SL.maps) + cx.nwarps() * 32;     // [NW][32]
    float* sm_compd = reinterpret_cast<float*>(sm_comp + cx.nwarps() * 32);                 // [NW][32]
    Rec* const recs0 = reinterpret_cast<Rec*>(smem_raw + SL.recs) + cx.lwarp() * CL * k.max_group_bands;
    const int rbuf = NWloc * CL * k.max_group_bands;   // records per buffer

    bool top_at_1;
    float mu0, tsi;
    {
        const int icol = cx.icol(), ncol = io.ncol(), nlay = io.nlay();
        const float* play = io.play();
        top_at_1 = play[icol] < play[icol + size_t(nlay - 1) * ncol];
        mu0 = io.mu0()[icol];
        tsi = io.tsi() ? io.tsi()[icol] : 1.f;
        setup_layer_range(k, io.gs(), ncol, nlay, icol, top_at_1, play, io.plev(), io.tlay(), nullptr, io.col_dry(),
                          st, sm_cg, NL, L0, NL, cx.tid(), cx.nthreads());
    }
    const float mu0_inv = 1.f / mu0;
    cx.sync();
    layer_minor_scalings(k, st, sm_cg, NL, sm_sc, NL, cx.tid(), cx.nthreads());
    float4* const sm_aer = reinterpret_cast<float4*>(smem_raw + SL.cloud);   // [band][local layer]
    if (with_aer) {
        const int nlay = io.nlay();
        for (int idx = cx.tid(); idx < NL * nband; idx += cx.nthreads()) {
            const int jl = idx % NL, b = idx / NL, j = L0 + jl;
            sm_aer[idx] = aerosol_point(io.aerosol(), io.ncol(), cx.icol(), top_at_1 ? j : nlay - 1 - j, st[jl].dp, b);
        }
    }
    cx.sync();

    const int ngpt = k.ngpt;
    constexpr int SH = (CL == 16) ? 0 : 1;          // lane L holds reduced value L >> SH
    double acc_a = 0.0, acc_b = 0.0, acc_c = 0.0;   // see the output section
    double acc_sfc_dir = 0.0, acc_sfc_dn = 0.0, acc_sfc_up = 0.0;

    for (int gg = 0; gg < k.ngroups; ++gg) {
        const int nlay = io.nlay();
        const int g = 32 * gg + lane;
        const bool gv = g < ngpt;
        const int b0 = k.group_band0[gg];
        const int gband = gv ? k.gpt2band[g] : b0;
        const int slot = gband - b0;
        const int4 mg0 = minor_entry(k.minor_g[0], g, gv);
        const int4 mg1 = minor_entry(k.minor_g[1], g, gv);
        const int nm0 = __reduce_max_sync(0xffffffffu, mg0.x);
        const int nm1 = __reduce_max_sync(0xffffffffu, mg1.x);

        Rec* const recs = recs0 + (P2 ? (gg & 1) : 0) * rbuf;
        if (!P2 || (gg & 1) == 0) {
            const int nrec = CL * k.max_group_bands;
            for (int t = lane; t < (P2 ? 2 : 1) * nrec; t += 32) {
                const int gq = gg + t / nrec, r = t % nrec;
                if (gq >= k.ngroups) continue;
                const int jj = cx.warp() * CL + (r % CL);
                const int b = k.group_band0[gq] + r / CL;
                if (jj < nlay && b < nband && k.band_lims[2 * b] < 32 * gq + 32) {
                    const int l = top_at_1 ? jj : nlay - 1 - jj;
                    build_sw_record(k, recs0[(P2 ? (gq & 1) : 0) * rbuf + r], st[jj - L0], sm_cg + (jj - L0), NL, b,
                                    io.cloud(), cx.icol() + size_t(l) * io.ncol(),
                                    with_aer ? sm_aer + b * NL + (jj - L0) : nullptr);
                }
            }
        }
        __syncwarp();

        // 1. pass 1
        float vR[CL], vT[CL], vSu[CL], vSd[CL], vAd[CL], vP[CL], vAdir[CL];
        float P = 1.f;
        float cRu = 0.f, cRd = 0.f, cT = 1.f, cU = 0.f, cD = 0.f;
        const int j0 = cx.warp() * CL;
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            const int j = j0 + i;
            float R = 0.f, T = 1.f, Rdir = 0.f, Tdir = 0.f, Tn = 1.f, adif = 0.f, adir = 0.f;
            if (j < nlay && gv) {
                const Rec& Rc = recs[slot * CL + i];
                const float ta =
                    tau_abs<DENSE>(k, Rc, g, Rc.a ? mg1 : mg0, Rc.a ? nm1 : nm0, sm_sc + (j - L0) * k.max_nscal);
                const float2 r0 = __ldg(k.krayl2 + (Rc.kr[0] + g));
                const float2 r1 = __ldg(k.krayl2 + (Rc.kr[1] + g));
                const float tr = (Rc.fm.x * r0.x + Rc.fm.y * r0.y + Rc.fm.z * r1.x + Rc.fm.w * r1.y) * Rc.aux.x;
                const float tau = ta + tr + Rc.aux.y;
                const float ts = tr + Rc.aux.z;
                float w0 = 0.f, omw = 1.f;
                if (tau > 2.f * FLT_MIN) {
                    const float inv = __fdividef(1.f, tau);
                    w0 = ts * inv;
                    omw = (ta + Rc.aux2) * inv;
                }
                const float gasy = __fdividef(Rc.aux.w, fmaxf(ts, 3.f * FLT_MIN));
                sw_layer_fast(tau, w0, omw, gasy, mu0, mu0_inv, R, T, Rdir, Tdir, Tn, adif, adir);
            }
            vR[i] = R;
            vT[i] = T;
            vP[i] = P;
            vSu[i] = Rdir * P;
            vSd[i] = Tdir * P;
            vAd[i] = adif;
            vAdir[i] = adir * P;
            // Add layer i below the composite of layers 0..i-1.
            const float den = __fdividef(1.f, fmaf(-cRd, R, 1.f));
            const float nRu = cRu + cT * cT * R * den;
            const float nRd = R + T * T * cRd * den;
            const float nU = cU + cT * (vSu[i] + R * cD) * den;
            const float nD = vSd[i] + T * (cD + cRd * vSu[i]) * den;
            cT = cT * T * den;
            cRu = nRu;
            cRd = nRd;
            cU = nU;
            cD = nD;
            P *= Tn;
        }
        cx.put(&sm_pt[cx.warp() * 32 + lane], P);
        cx.sync();

        // 2. direct flux at the chunk top and at the surface
        const int w = cx.warp(), NW = cx.nwarps();
        const float toa = gv ? __ldg(k.solar_source + g) * tsi * mu0 : 0.f;
        float dtop = toa;
        for (int c = 0; c < w; ++c) dtop *= sm_pt[c * 32 + lane];
        float dsfc = dtop;
        for (int c = w; c < NW; ++c) dsfc *= sm_pt[c * 32 + lane];
        {
            float v[2 * CL];
#pragma unroll
            for (int i = 0; i < CL; ++i) {
                v[i] = dtop * vP[i];
                v[CL + i] = dtop * vAdir[i];
            }
            ReduceScatter<2 * CL, 16>::run(v, lane);
            acc_a += double(v[0]);
        }
        cx.put(&sm_comp[w * 32 + lane], make_float4(cRu, cRd, cT, cU * dtop));
        cx.put(&sm_compd[w * 32 + lane], cD * dtop);
        cx.sync();

        // 3. albedo and source at this chunk's bottom; incident diffuse flux at its top.  Chunk 0's
        //    warp scans the composites of all chunks: from the surface up, the albedo and source
        //    at each chunk bottom and the chunk's transfer of the diffuse flux (flux at its bottom
        //    = F * flux at its top + G); then from the top down, the diffuse flux entering each
        //    chunk (no diffuse flux at the top of the atmosphere).  The results replace the
        //    composites (each slot read before it is rewritten, through put for every CTA of a
        //    cluster), and every warp reads its own chunk's after one more barrier: with every
        //    warp scanning the chunks itself the scans were O(chunks^2) per group.
        const float ad = gv ? __ldg(io.alb_dir() + gband + size_t(cx.icol()) * nband) : 0.f;
        const float af = gv ? __ldg(io.alb_dif() + gband + size_t(cx.icol()) * nband) : 0.f;
        if (w == 0) {
            float alb = af, src = dsfc * ad;
            for (int c = NW - 1; c >= 0; --c) {
                const float4 m = sm_comp[c * 32 + lane];
                const float D = sm_compd[c * 32 + lane];
                const float den = __fdividef(1.f, fmaf(-m.y, alb, 1.f));
                cx.put(&sm_comp[c * 32 + lane], make_float4(alb, src, m.z * den, fmaf(m.y, src, D) * den));
                const float nalb = m.x + m.z * m.z * alb * den;
                src = m.w + m.z * fmaf(alb, D, src) * den;
                alb = nalb;
            }
            float f = 0.f;
            for (int c = 0; c < NW; ++c) {
                cx.put(&sm_compd[c * 32 + lane], f);
                const float4 r = sm_comp[c * 32 + lane];
                f = fmaf(r.z, f, r.w);
            }
        }
        cx.sync();
        const float4 own = sm_comp[w * 32 + lane];
        const float alb_in = own.x, src_in = own.y, fb = sm_compd[w * 32 + lane];

        // 4. pass 2 (bottom-up): albedo and upward source per level
        float vA[CL];
        {
            float a = alb_in, s = src_in;
#pragma unroll
            for (int i = CL - 1; i >= 0; --i) {
                const float su = vSu[i] * dtop, sd = vSd[i] * dtop;
                const float den = __fdividef(1.f, fmaf(-vR[i], a, 1.f));
                const float na = vR[i] + vT[i] * vT[i] * a * den;
                const float ns = su + vT[i] * fmaf(a, sd, s) * den;
                vSd[i] = sd;
                vSu[i] = ns;
                vA[i] = na;
                a = na;
                s = ns;
            }
        }
        // pass 3 (top-down): diffuse fluxes and diffuse absorption
        float vUp[2 * CL], vDn[2 * CL];
        float fd = fb;
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            const float a_n = (i + 1 < CL) ? vA[i + 1] : alb_in;
            const float s_n = (i + 1 < CL) ? vSu[i + 1] : src_in;
            const float fu = fmaf(fd, vA[i], vSu[i]);
            const float den = __fdividef(1.f, fmaf(-vR[i], a_n, 1.f));
            const float fdn = (vT[i] * fd + vR[i] * s_n + vSd[i]) * den;
            const float fun = fmaf(fdn, a_n, s_n);
            vUp[i] = fu;
            vUp[CL + i] = (fd + fun) * vAd[i];
            vDn[i] = fd;
            vDn[CL + i] = 0.f;
            fd = fdn;
        }
        if (w == NW - 1) {
            acc_sfc_dir += double(warp_sum(dsfc));
            acc_sfc_dn += double(warp_sum(fd));
            acc_sfc_up += double(warp_sum(fmaf(fd, alb_in, src_in)));
        }
        ReduceScatter<2 * CL, 16>::run(vUp, lane);
        ReduceScatter<2 * CL, 16>::run(vDn, lane);
        acc_b += double(vUp[0]);
        acc_c += double(vDn[0]);
    }

    // Outputs.  Lane L holds value v = L >> SH of the reduced arrays: v < CL is level
    // w*CL + v (acc_a: direct, acc_b: up, acc_c: diffuse down), v >= CL is layer
    // w*CL + v - CL (acc_a + acc_b: absorbed flux).
    const int w = cx.warp(), NW = cx.nwarps(), icol = cx.icol(), ncol = io.ncol(), nlay = io.nlay();
    float* const flux_up = io.up();
    float* const flux_dn = io.dn();
    float* const flux_dir = io.dir();
    float* const flux_net = io.net();
    float* const heating_rate = io.hr();
    const int v = lane >> SH;
    if ((lane & ((1 << SH) - 1)) == 0) {
        if (v < CL) {
            const int jl = w * CL + v;
            if (jl < nlay) {
                const int al = top_at_1 ? jl : nlay - jl;
                const size_t o = icol + size_t(al) * ncol;
                const double dn = acc_c + acc_a;
                flux_up[o] = float(acc_b);
                flux_dn[o] = float(dn);
                flux_dir[o] = float(acc_a);
                flux_net[o] = float(dn - acc_b);
            }
        } else {
            const int jl = w * CL + v - CL;
            if (jl < nlay) {
                const int l = top_at_1 ? jl : nlay - 1 - jl;
                const double g0_cp = 9.80665 / 1004.64;
                heating_rate[icol + size_t(l) * ncol] =
                    float(g0_cp * 86400.0 * (acc_a + acc_b) / double(st[jl - L0].dp));
            }
        }
    }
    if (w == NW - 1 && lane == 0) {
        const int al = top_at_1 ? nlay : 0;
        const size_t o = icol + size_t(al) * ncol;
        const double dn = acc_sfc_dn + acc_sfc_dir;
        flux_up[o] = float(acc_sfc_up);
        flux_dn[o] = float(dn);
        flux_dir[o] = float(acc_sfc_dir);
        flux_net[o] = float(dn - acc_sfc_up);
    }
}

}  // namespace fused
}  // namespace rrtmgp_b200
