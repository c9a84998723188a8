// Fused longwave forward: gas optics + cloud optics (1scl, added by band) + no-scattering
// solver + broadband fluxes + heating rates for whole columns, without materialising any
// (ncol, nlay, ngpt) array.  The staged equivalent is the sequence of
// Radiation_solver_longwave::solve_gpu (src_test/Radiation_solver.cu:467-615).
//
// Mapping: one CTA per column.  Lane l of every warp handles g-point 32*group + l, so the
// table gathers of a warp are two contiguous 64-byte runs (one per band).  Warp w owns the
// layer chunk [w*CL, (w+1)*CL) (counted from the top of the atmosphere).  For each group of
// 32 g-points:
//   1. each warp builds one record per (layer, band) of its chunk in shared memory: table
//      offsets and interpolation weights (interpolation_kernel), minor-absorber scalings,
//      band Planck functions and the cloud optical depth;
//   2. pass 1: per (layer, g-point) tau, Planck fraction, transmissivity and the two
//      linear-in-tau sources (lw_solver_noscat step 1) stay in registers; the warp composes
//      its chunk's affine down and up maps x -> A x + B and publishes them;
//   3. after one barrier every thread composes the maps of the other chunks to get its
//      chunk's incoming down and up radiances (the surface term is the reference's
//      radn_dn * (1 - emis) + emis * sfc_src);
//   4. pass 2 re-sweeps the registers, producing the level radiances and the per-layer
//      absorbed radiance omt * (I_dn(top) + I_up(bottom)) - S_dn - S_up, which gives heating
//      rates without differencing two nearly equal level fluxes;
//   5. a warp reduce-scatter (31 shuffles per 32 values) sums over the 32 g-points and every
//      lane accumulates one level (or layer) in FP64.
#include <cfloat>
#include <cmath>

#include "common.cuh"
#include "rte_device.cuh"

namespace rrtmgp_b200 {
namespace {

constexpr int kMaxMinor = 6;

struct LwRec {
    int kb0, kb1;        // offsets of corners (t0, p0, e0) and (t1, p0, e1) in [t][p][eta][g]
    int r0, r2;          // kminor row offsets of (t0, e0) and (t1, e1) in [t][eta][c]
    int nmin, nc;        // minor intervals in this (band, atmosphere), contributors
    int mgs[kMaxMinor], mge[kMaxMinor], mks[kMaxMinor];
    int a, pad;
    float wmaj[8];       // col_mix x fmajor
    float wpl[8];        // fmajor (Planck fractions)
    float fm[4];         // fminor
    float scal[kMaxMinor];
    float pl_lay, pl_top, pl_bot, pl_sfc, tau_cld;
    float pad2[3];
};

struct CloudArgs {
    CloudLut<float> L;
    const float* lwp;
    const float* iwp;
    const float* rel;
    const float* rei;
    int present;
};

// Reduce-scatter of N per-lane values over the 32 lanes: afterwards lane L holds in v[0] the
// warp total of value L >> log2(32/N) (N <= 32).
template <int N, int OFF>
struct ReduceScatter {
    static __device__ __forceinline__ void run(float* v, int lane)
    {
        constexpr int H = N / 2;
        const bool upper = (lane & OFF) != 0;
#pragma unroll
        for (int i = 0; i < H; ++i) {
            const float send = upper ? v[i] : v[i + H];
            const float keep = upper ? v[i + H] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, OFF);
        }
        ReduceScatter<H, OFF / 2>::run(v, lane);
    }
};
template <int OFF>
struct ReduceScatter<1, OFF> {
    static __device__ __forceinline__ void run(float* v, int lane)
    {
        v[0] += __shfl_xor_sync(0xffffffffu, v[0], OFF);
        ReduceScatter<1, OFF / 2>::run(v, lane);
    }
};
template <>
struct ReduceScatter<1, 0> {
    static __device__ __forceinline__ void run(float*, int) {}
};

__device__ __forceinline__ void build_record(const KdistView<float>& k, LwRec& R, int jj, int b, int nlay,
                                             const int* sm_i, const float* sm_f, const float* sm_cg,
                                             const float* sm_cld, float tsfc)
{
    LayerInterp<float> li;
    li.jt = sm_i[4 * jj + 0];
    li.jp = sm_i[4 * jj + 1];
    li.itropo = sm_i[4 * jj + 2];
    li.ftemp = sm_f[8 * jj + 0];
    li.fpress = sm_f[8 * jj + 1];
    const float p = sm_f[8 * jj + 2], t = sm_f[8 * jj + 3];
    const float* cg = sm_cg + jj;
    const int flav = k.band_flav[2 * b + li.itropo];
    const FlavorWeights<float> fw = flavor_weights(k, flav, li, cg, nlay);
    const MajorCorners<float> mc = major_corners(k, k.kmajor, li, fw);
    R.kb0 = int(mc.c[0] - k.kmajor);
    R.kb1 = int(mc.c[4] - k.kmajor);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        R.wmaj[q] = fw.cm[q / 4] * mc.fmaj[q];
        R.wpl[q] = mc.fmaj[q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) R.fm[q] = fw.fm[q];
    const int a = li.itropo;
    const int nc = k.ncontrib[a];
    R.a = a;
    R.nc = nc;
    R.r0 = ((li.jt - 1) * k.neta + fw.j0 - 1) * nc;
    R.r2 = (li.jt * k.neta + fw.j1 - 1) * nc;
    int n = 0;
    for (int ii = k.band_minor_begin[a][b]; ii < k.band_minor_begin[a][b + 1] && n < kMaxMinor; ++ii, ++n) {
        const int im = k.band_minor_list[a][ii];
        R.scal[n] = minor_scaling(k, a, im, cg, nlay, p, t);
        R.mgs[n] = k.minor_gstart[a][im];
        R.mge[n] = k.minor_gend[a][im];
        R.mks[n] = k.minor_kstart[a][im];
    }
    R.nmin = n;
    const float* tp = k.totplnk + size_t(b) * k.nplanck;
    R.pl_lay = interpolate1D(t, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
    R.pl_top = interpolate1D(sm_f[8 * jj + 4], k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
    R.pl_bot = interpolate1D(sm_f[8 * jj + 5], k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
    R.pl_sfc = (jj == nlay - 1) ? interpolate1D(tsfc, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp) : 0.f;
    R.tau_cld = sm_cld ? sm_cld[b * nlay + jj] : 0.f;
}

// Word offset of the chunk-map area, rounded up to 4 words so that it is float4 aligned.
__host__ __device__ __forceinline__ int lw_maps_offset(int nlay, int ngas, int nband)
{
    return ((12 + ngas + 1 + nband) * nlay + 3) & ~3;
}

template <int CL>
__global__ void __launch_bounds__(512)
lw_forward_kernel(const KdistView<float> k, const GasSet<float> gs, const CloudArgs cld, int ncol, int nlay,
                  const float* __restrict__ play, const float* __restrict__ plev, const float* __restrict__ tlay,
                  const float* __restrict__ tlev, const float* __restrict__ tsfc,
                  const float* __restrict__ col_dry_in, const float* __restrict__ sfc_emis,
                  float* __restrict__ flux_up, float* __restrict__ flux_dn, float* __restrict__ flux_net,
                  float* __restrict__ heating_rate)
{
    static_assert(CL == 8 || CL == 16, "chunk length");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int icol = blockIdx.x;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int NW = blockDim.x >> 5;
    const int nband = k.nband;

    // Shared memory carve-up (4-byte words).
    int* sm_i = reinterpret_cast<int*>(smem_raw);                 // [nlay][4]: jt, jp, itropo
    float* sm_f = reinterpret_cast<float*>(sm_i + 4 * nlay);      // [nlay][8]: ftemp, fpress, p, t, Ttop, Tbot, dp
    float* sm_cg = sm_f + 8 * nlay;                               // [ngas+1][nlay]
    float* sm_cld = sm_cg + (k.ngas + 1) * nlay;                  // [nband][nlay]
    float* sm_maps = reinterpret_cast<float*>(smem_raw) + lw_maps_offset(nlay, k.ngas, nband);  // [NW][32][4]
    float* sm_sfc = sm_maps + NW * 32 * 4;                        // [32]
    LwRec* recs = reinterpret_cast<LwRec*>(sm_sfc + 32);
    const int nrec_w = CL * k.max_group_bands;
    LwRec* myrecs = recs + w * nrec_w;

    const bool top_at_1 = play[icol] < play[icol + size_t(nlay - 1) * ncol];
    const float ts = tsfc[icol];

    // Per-layer state, layers counted from the top (j).
    for (int j = threadIdx.x; j < nlay; j += blockDim.x) {
        const int l = top_at_1 ? j : nlay - 1 - j;
        const size_t cl = icol + size_t(l) * ncol;
        const float p = play[cl], t = tlay[cl];
        fill_col_gas(k, gs, ncol, nlay, icol, l, plev, col_dry_in, sm_cg + j, nlay);
        const LayerInterp<float> li = layer_interp(k, p, t);
        sm_i[4 * j + 0] = li.jt;
        sm_i[4 * j + 1] = li.jp;
        sm_i[4 * j + 2] = li.itropo;
        const int lt = top_at_1 ? j : nlay - j, lb = top_at_1 ? j + 1 : nlay - 1 - j;
        sm_f[8 * j + 0] = li.ftemp;
        sm_f[8 * j + 1] = li.fpress;
        sm_f[8 * j + 2] = p;
        sm_f[8 * j + 3] = t;
        sm_f[8 * j + 4] = tlev[icol + size_t(lt) * ncol];
        sm_f[8 * j + 5] = tlev[icol + size_t(lb) * ncol];
        sm_f[8 * j + 6] = fabsf(plev[icol + size_t(lb) * ncol] - plev[icol + size_t(lt) * ncol]);
    }
    for (int idx = threadIdx.x; idx < nlay * nband; idx += blockDim.x) {
        const int j = idx % nlay, b = idx / nlay;
        float tau = 0.f, s, g;
        if (cld.present) {
            const int l = top_at_1 ? j : nlay - 1 - j;
            const size_t cl = icol + size_t(l) * ncol;
            const CloudPoint<float> cp = cloud_point(cld.L, cld.lwp[cl], cld.iwp[cl], cld.rel[cl], cld.rei[cl]);
            cloud_band<float, false>(cld.L, cp, b, tau, s, g);
        }
        sm_cld[b * nlay + j] = tau;
    }
    __syncthreads();

    const float D = 1.66f;                 // single-angle secant (Rte_lw.cpp:101-113)
    const int ngpt = k.ngpt;
    const int o1 = ngpt, o2 = k.neta * ngpt, o3 = o2 + ngpt;
    double acc_lev = 0.0, acc_div = 0.0, acc_bot_up = 0.0, acc_bot_dn = 0.0;

    for (int gg = 0; gg < k.ngroups; ++gg) {
        const int g = 32 * gg + lane;
        const bool gv = g < ngpt;
        const int b0 = k.group_band0[gg];
        const int gband = gv ? k.gpt2band[g] : b0;
        const int slot = gband - b0;

        // 1. records of this warp's chunk
        for (int r = lane; r < nrec_w; r += 32) {
            const int jj = w * CL + (r % CL);
            const int b = b0 + r / CL;
            if (jj < nlay && b < nband && k.band_lims[2 * b] < 32 * gg + 32)
                build_record(k, myrecs[r], jj, b, nlay, sm_i, sm_f, sm_cg, sm_cld, ts);
        }
        __syncwarp();

        // 2. pass 1: optical properties and sources in registers, chunk maps
        float omt[CL], sdn[CL], sup[CL];
        float Ad = 1.f, Bd = 0.f;
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            const int j = w * CL + i;
            omt[i] = 0.f; sdn[i] = 0.f; sup[i] = 0.f;
            if (j < nlay && gv) {
                const LwRec& R = myrecs[slot * CL + i];
                const float* KM = k.kmajor;
                float tau = R.wmaj[0] * __ldg(KM + R.kb0 + g) + R.wmaj[1] * __ldg(KM + R.kb0 + o1 + g) +
                            R.wmaj[2] * __ldg(KM + R.kb0 + o2 + g) + R.wmaj[3] * __ldg(KM + R.kb0 + o3 + g) +
                            R.wmaj[4] * __ldg(KM + R.kb1 + g) + R.wmaj[5] * __ldg(KM + R.kb1 + o1 + g) +
                            R.wmaj[6] * __ldg(KM + R.kb1 + o2 + g) + R.wmaj[7] * __ldg(KM + R.kb1 + o3 + g);
                const float* KN = k.kminor[R.a];
                for (int n = 0; n < R.nmin; ++n) {
                    if (g >= R.mgs[n] && g < R.mge[n]) {
                        const int c = R.mks[n] + g - R.mgs[n];
                        tau += R.scal[n] * (R.fm[0] * __ldg(KN + R.r0 + c) + R.fm[1] * __ldg(KN + R.r0 + R.nc + c) +
                                            R.fm[2] * __ldg(KN + R.r2 + c) + R.fm[3] * __ldg(KN + R.r2 + R.nc + c));
                    }
                }
                tau += R.tau_cld;
                const float* PF = k.planck_frac;
                const float pfrac =
                    (R.wpl[0] * __ldg(PF + R.kb0 + g) + R.wpl[1] * __ldg(PF + R.kb0 + o1 + g) +
                     R.wpl[2] * __ldg(PF + R.kb0 + o2 + g) + R.wpl[3] * __ldg(PF + R.kb0 + o3 + g)) +
                    (R.wpl[4] * __ldg(PF + R.kb1 + g) + R.wpl[5] * __ldg(PF + R.kb1 + o1 + g) +
                     R.wpl[6] * __ldg(PF + R.kb1 + o2 + g) + R.wpl[7] * __ldg(PF + R.kb1 + o3 + g));
                lw_layer_omt(tau, D, pfrac * R.pl_lay, pfrac * R.pl_bot, pfrac * R.pl_top, omt[i], sdn[i], sup[i]);
                if (j == nlay - 1) sm_sfc[lane] = pfrac * R.pl_sfc;
            } else if (j == nlay - 1) {
                sm_sfc[lane] = 0.f;
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
        reinterpret_cast<float4*>(sm_maps)[w * 32 + lane] = make_float4(Ad, Bd, Au, Bu);
        __syncthreads();

        // 3. incoming radiances of the chunk
        float x = 0.f;  // no incident longwave flux at the top
        float xin = 0.f;
        for (int c = 0; c < NW; ++c) {
            if (c == w) xin = x;
            const float4 m = reinterpret_cast<const float4*>(sm_maps)[c * 32 + lane];
            x = m.x * x + m.y;
        }
        const float emis = gv ? sfc_emis[gband + size_t(icol) * nband] : 0.f;
        const float S = x * (1.f - emis) + emis * sm_sfc[lane];
        float y = S;
        for (int c = NW - 1; c > w; --c) {
            const float4 m = reinterpret_cast<const float4*>(sm_maps)[c * 32 + lane];
            y = m.z * y + m.w;
        }

        // 4. pass 2: level radiances and layer absorption
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
            float bu = S, bd = rd;
#pragma unroll
            for (int off = 16; off >= 1; off >>= 1) {
                bu += __shfl_xor_sync(0xffffffffu, bu, off);
                bd += __shfl_xor_sync(0xffffffffu, bd, off);
            }
            acc_bot_up += double(bu);
            acc_bot_dn += double(bd);
        }
        __syncthreads();
    }

    // Outputs.  Fluxes = 2 pi w * sum of radiances with w = 0.5.
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
            heating_rate[icol + size_t(l) * ncol] = float(g0_cp * 86400.0 * pi * acc_div / double(sm_f[8 * jl + 6]));
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

template <int CL>
size_t lw_forward_smem(const KdistView<float>& v, int nlay)
{
    const int NW = (nlay + CL - 1) / CL;
    return sizeof(float) * (size_t(lw_maps_offset(nlay, v.ngas, v.nband)) + NW * 32 * 4 + 32) +
           sizeof(LwRec) * size_t(NW) * CL * v.max_group_bands;
}

template <int CL>
int launch_lw_forward(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay, const float* play,
                      const float* plev, const float* tlay, const float* tlev, const float* tsfc, const float* col_dry,
                      const GasSet<float>& gs, const float* lwp, const float* iwp, const float* rel, const float* rei,
                      const float* emis, float* up, float* dn, float* net, float* hr, cudaStream_t stream)
{
    const KdistView<float>& v = k->v32;
    const int NW = (nlay + CL - 1) / CL;
    RB_CHECK_ARG(NW <= 16, "forward_lw: nlay too large for the fused kernel (at most 16 chunks)");
    const size_t smem = lw_forward_smem<CL>(v, nlay);
    if (smem > 220 * 1024) return fail(RRTMGP_B200_ERR_UNSUPPORTED, "forward_lw: shared memory need exceeds 220 KB");
    static bool attr = false;
    if (!attr) {
        RB_CUDA(cudaFuncSetAttribute(lw_forward_kernel<CL>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024),
                "forward_lw attribute");
        attr = true;
    }
    CloudArgs ca{};
    if (c) {
        ca.L = CloudLut<float>{c->nband, c->nsize_liq, c->nsize_ice, float(c->radliq_lwr), float(c->liq_step),
                               float(c->radice_lwr), float(c->ice_step), c->lut32};
        ca.lwp = lwp; ca.iwp = iwp; ca.rel = rel; ca.rei = rei;
        ca.present = 1;
    }
    lw_forward_kernel<CL><<<ncol, NW * 32, smem, stream>>>(v, gs, ca, ncol, nlay, play, plev, tlay, tlev, tsfc,
                                                             col_dry, emis, up, dn, net, hr);
    RB_LAUNCH("lw_forward_kernel");
    return RRTMGP_B200_OK;
}

}  // namespace

int forward_lw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay, const float* play,
                   const float* plev, const float* tlay, const float* tlev, const float* tsfc, const float* col_dry,
                   const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp,
                   const float* rel, const float* rei, const float* sfc_emis, float* flux_up, float* flux_dn,
                   float* flux_net, float* heating_rate, int chunk, void* stream)
{
    RB_CHECK_ARG(k && k->info.is_longwave, "forward_lw: need a longwave k-distribution");
    RB_CHECK_ARG(ncol > 0 && nlay > 1, "forward_lw: ncol > 0 and nlay > 1 required");
    RB_CHECK_ARG(play && plev && tlay && tlev && tsfc && sfc_emis && flux_up && flux_dn && flux_net && heating_rate,
                 "forward_lw: null array");
    RB_CHECK_ARG(!c || (lwp && iwp && rel && rei), "forward_lw: cloud arrays required with a cloud handle");
    RB_CHECK_ARG(!c || c->nband == k->info.nband, "forward_lw: cloud and gas band counts differ");
    const KdistView<float>& v = k->v32;
    if (!v.minor_in_band || v.max_band_minor > kMaxMinor || v.max_group_bands > 32 / 4)
        return fail(RRTMGP_B200_ERR_UNSUPPORTED, "forward_lw: k-distribution layout not supported by the fused kernel");
    GasSet<float> gs;
    int st = make_gas_set<float>(k, ncol, nlay, gases, ngases, gs);
    if (st) return st;
    cudaStream_t s = as_stream(stream);
    if (chunk == 8)
        return launch_lw_forward<8>(k, c, ncol, nlay, play, plev, tlay, tlev, tsfc, col_dry, gs, lwp, iwp, rel, rei,
                                    sfc_emis, flux_up, flux_dn, flux_net, heating_rate, s);
    return launch_lw_forward<16>(k, c, ncol, nlay, play, plev, tlay, tlev, tsfc, col_dry, gs, lwp, iwp, rel, rei,
                                 sfc_emis, flux_up, flux_dn, flux_net, heating_rate, s);
}

}  // namespace rrtmgp_b200

extern "C" int rrtmgp_b200_forward_lw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* tlev, const float* tsfc,
        const float* col_dry, const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp,
        const float* rel, const float* rei, const float* sfc_emis, float* flux_up, float* flux_dn, float* flux_net,
        float* heating_rate, int chunk, void* stream)
{
    return rrtmgp_b200::forward_lw_f32(k, c, ncol, nlay, play, plev, tlay, tlev, tsfc, col_dry, gases, ngases, lwp,
                                       iwp, rel, rei, sfc_emis, flux_up, flux_dn, flux_net, heating_rate, chunk, stream);
}
