// Gas optics kernels: col_dry, interpolation, major + minor absorption, Rayleigh, Planck.
//
// One thread per (column, layer); a warp covers 32 consecutive columns of one layer, so the
// (ncol, nlay, ngpt) outputs are written with 128-byte coalesced stores per g-point.  The
// interpolation (jtemp, jpress, jeta, weights) is computed once per (column, layer, band)
// in registers instead of being materialised (the reference's interpolation_kernel,
// gas_optics_rrtmgp_kernels.cu:215-293, stores 14 values per flavor and re-reads them in
// every later kernel).  Tables are g-point fastest, so the 16 g-points of a band at one
// (T, p, eta) corner are one 64-byte run.
#include <cfloat>
#include <cmath>
#include <type_traits>

#include "common.cuh"
#include "fused_common.cuh"
#include "gas_optics_device.cuh"

namespace rrtmgp_b200 {

namespace {

constexpr int kBX = 32, kBY = 4, kThreads = kBX * kBY;

// Longwave: tau and Planck sources (gas_optical_depths_major/minor + Planck_source_kernel).
template <typename T>
__global__ void __launch_bounds__(kThreads)
gas_optics_lw_kernel(const KdistView<T> k, const GasSet<T> gases, int ncol, int nlay,
                     const T* __restrict__ play, const T* __restrict__ plev,
                     const T* __restrict__ tlay, const T* __restrict__ tsfc,
                     const T* __restrict__ tlev, const T* __restrict__ col_dry_in,
                     T* __restrict__ tau, T* __restrict__ lay_src, T* __restrict__ lev_inc,
                     T* __restrict__ lev_dec, T* __restrict__ sfc_src, T* __restrict__ sfc_jac)
{
    extern __shared__ unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int tid = threadIdx.x + threadIdx.y * kBX;
    T* cg = smem + tid;                                  // col_gas[(ngas+1)] stride kThreads
    T* acc = smem + (k.ngas + 1) * kThreads + tid;       // tau accumulator [kMaxBandGpt]

    const int icol = blockIdx.x * kBX + threadIdx.x;
    const int ilay = blockIdx.y * kBY + threadIdx.y;
    if (icol >= ncol || ilay >= nlay) return;
    const size_t cl = size_t(icol) + size_t(ilay) * ncol;
    const size_t ncl = size_t(ncol) * nlay;

    const T p = play[cl], t = tlay[cl];
    fill_col_gas(k, gases, ncol, nlay, icol, ilay, plev, col_dry_in, cg, kThreads);
    LayerInterp<T> li = layer_interp(k, p, t);

    const int sfc_lay = play[icol] > play[icol + size_t(nlay - 1) * ncol] ? 0 : nlay - 1;
    const bool at_sfc = ilay == sfc_lay;
    const T tl_up = tlev[icol + size_t(ilay + 1) * ncol];
    const T tl_dn = tlev[cl];
    const T ts = tsfc[icol];

    for (int b = 0; b < k.nband; ++b) {
        const int g0 = k.band_lims[2 * b], g1 = k.band_lims[2 * b + 1];
        const int flav = k.band_flav[2 * b + li.itropo];
        FlavorWeights<T> fw = flavor_weights(k, flav, li, cg, kThreads);
        MajorCorners<T> mc = major_corners(k, k.kmajor, li, fw);

        for (int g = g0; g < g1; ++g) acc[(g - g0) * kThreads] = major_tau(mc, fw, li, g);
        add_minor(k, li, fw, flav, cg, kThreads, p, t, b, g0, g1, acc, kThreads);
        for (int g = g0; g < g1; ++g) tau[cl + size_t(g) * ncl] = acc[(g - g0) * kThreads];

        // Planck sources: band Planck function at T_lay, T_lev(ilay+1), T_lev(ilay).
        const T* tp = k.totplnk + size_t(b) * k.nplanck;
        const T pl = interpolate1D(t, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
        const T pinc = interpolate1D(tl_up, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
        const T pdec = interpolate1D(tl_dn, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
        T ps = T(0), ps2 = T(0);
        if (at_sfc) {
            ps = interpolate1D(ts, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
            ps2 = interpolate1D(ts + T(1), k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
        }
        MajorCorners<T> pc = major_corners(k, k.planck_frac, li, fw);
        for (int g = g0; g < g1; ++g) {
            const T pfrac = planck_fraction(pc, fw, li, g);
            const size_t o = cl + size_t(g) * ncl;
            lay_src[o] = pfrac * pl;
            lev_inc[o] = pfrac * pinc;
            lev_dec[o] = pfrac * pdec;
            if (at_sfc) {
                sfc_src[icol + size_t(g) * ncol] = pfrac * ps;
                sfc_jac[icol + size_t(g) * ncol] = pfrac * (ps2 - ps);
            }
        }
    }
}

// Shortwave: tau, ssa, g with Rayleigh (compute_tau_rayleigh_kernel + combine_abs_and_rayleigh).
template <typename T>
__global__ void __launch_bounds__(kThreads)
gas_optics_sw_kernel(const KdistView<T> k, const GasSet<T> gases, int ncol, int nlay,
                     const T* __restrict__ play, const T* __restrict__ plev,
                     const T* __restrict__ tlay, const T* __restrict__ col_dry_in,
                     T* __restrict__ tau, T* __restrict__ ssa, T* __restrict__ gasy)
{
    extern __shared__ unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int tid = threadIdx.x + threadIdx.y * kBX;
    T* cg = smem + tid;
    T* acc = smem + (k.ngas + 1) * kThreads + tid;

    const int icol = blockIdx.x * kBX + threadIdx.x;
    const int ilay = blockIdx.y * kBY + threadIdx.y;
    if (icol >= ncol || ilay >= nlay) return;
    const size_t cl = size_t(icol) + size_t(ilay) * ncol;
    const size_t ncl = size_t(ncol) * nlay;

    const T p = play[cl], t = tlay[cl];
    fill_col_gas(k, gases, ncol, nlay, icol, ilay, plev, col_dry_in, cg, kThreads);
    LayerInterp<T> li = layer_interp(k, p, t);
    const T col_rayl = cg[k.idx_h2o * kThreads] + cg[0];
    const T two_tmin = T(2) * tiny_value<T>();

    for (int b = 0; b < k.nband; ++b) {
        const int g0 = k.band_lims[2 * b], g1 = k.band_lims[2 * b + 1];
        const int flav = k.band_flav[2 * b + li.itropo];
        FlavorWeights<T> fw = flavor_weights(k, flav, li, cg, kThreads);
        MajorCorners<T> mc = major_corners(k, k.kmajor, li, fw);
        for (int g = g0; g < g1; ++g) acc[(g - g0) * kThreads] = major_tau(mc, fw, li, g);
        add_minor(k, li, fw, flav, cg, kThreads, p, t, b, g0, g1, acc, kThreads);
        const T* kr = k.krayl + size_t(li.itropo) * k.ntemp * k.neta * k.ngpt;
        for (int g = g0; g < g1; ++g) {
            const T tr = rayleigh_k(k, kr, li, fw, g) * col_rayl;
            const T tt = acc[(g - g0) * kThreads] + tr;
            const size_t o = cl + size_t(g) * ncl;
            tau[o] = tt;
            ssa[o] = tt > two_tmin ? tr / tt : T(0);
            gasy[o] = T(0);
        }
    }
}

// FP32 variants on the corner-packed tables of the fused kernels (KdistView::kmaj4, pfrac4,
// kmin2, krayl2, minor_g).  Same thread mapping and outputs; per (column, layer, g-point) the
// major interpolation is two 16-byte loads instead of eight 4-byte ones (the Planck fraction
// likewise), each minor interval one 8-byte pair per eta corner, and the sum over minor
// intervals stays in registers instead of a shared-memory accumulator.  The per-band weights
// are the records of the fused kernels (fused::record_weights) held in registers.  The minor
// scalings are computed once per (column, layer) for every scaling kind (not per band) and
// are indexed per g-point, so they sit in shared memory, one column of max_nscal values per
// thread (stride kThreads: no bank conflicts).
// Usable when the tables satisfy the fused kernels' layout conditions (packed_tables_ok).
// I32: every (column, layer, g-point) offset fits in 31 bits (packed_index32), so the output
// offsets are 32-bit (one multiply-add per store address instead of 64-bit arithmetic and
// fewer live registers at the occupancy's register cap).
__host__ __device__ inline size_t packed_smem_bytes(int ngas, int nscal)
{
    return sizeof(float) * size_t(ngas + 1 + nscal) * kThreads;
}

inline bool packed_tables_ok(const KdistView<float>& v, bool lw)
{
    return fused::fused_layout_ok(v, !lw, 1 << 30) && v.minor_g[0] && v.minor_g[1];
}

inline bool packed_index32(int ncol, int nlay, int ngpt)
{
    return size_t(ncol) * size_t(nlay) * size_t(ngpt) < (size_t(1) << 31);
}

// minor_g row of g-point g (unused slots already repeat the first one), zeros past the end.
__device__ __forceinline__ int4 next_minor_row(const int4* mgt, int g, int ngpt)
{
    return g < ngpt ? __ldg(mgt + g) : make_int4(0, 0, 0, 0);
}

__device__ __forceinline__ fused::LayerState thread_layer_state(const LayerInterp<float>& li, float p, float t)
{
    fused::LayerState s;
    s.jt = li.jt;
    s.jp = li.jp;
    s.itropo = li.itropo;
    s.pad = 0;
    s.ftemp = li.ftemp;
    s.fpress = li.fpress;
    s.p = p;
    s.t = t;
    s.t_top = s.t_bot = s.dp = s.pad2 = 0.f;
    return s;
}

template <bool DENSE, bool I32>
__global__ void __launch_bounds__(kThreads, 7)
gas_optics_lw_packed_kernel(const KdistView<float> k, const GasSet<float> gases, int ncol, int nlay,
                            const float* __restrict__ play, const float* __restrict__ plev,
                            const float* __restrict__ tlay, const float* __restrict__ tsfc,
                            const float* __restrict__ tlev, const float* __restrict__ col_dry_in,
                            float* __restrict__ tau, float* __restrict__ lay_src, float* __restrict__ lev_inc,
                            float* __restrict__ lev_dec, float* __restrict__ sfc_src, float* __restrict__ sfc_jac)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x + threadIdx.y * kBX;
    float* cg = reinterpret_cast<float*>(smem_raw) + tid;                       // [ngas + 1]
    float* scal = reinterpret_cast<float*>(smem_raw) + (k.ngas + 1) * kThreads + tid;   // [max_nscal]

    using Idx = typename std::conditional<I32, unsigned, size_t>::type;
    const int icol = blockIdx.x * kBX + threadIdx.x;
    const int ilay = blockIdx.y * kBY + threadIdx.y;
    if (icol >= ncol || ilay >= nlay) return;
    const Idx cl = Idx(icol) + Idx(ilay) * Idx(ncol);
    const Idx ncl = Idx(ncol) * Idx(nlay);

    const float p = play[cl], t = tlay[cl];
    fill_col_gas(k, gases, ncol, nlay, icol, ilay, plev, col_dry_in, cg, kThreads);
    const fused::LayerState s = thread_layer_state(layer_interp(k, p, t), p, t);
    for (int sid = 0; sid < k.nscal[s.itropo]; ++sid)
        scal[sid * kThreads] = fused::kind_scaling(k, s.itropo, sid, cg, kThreads, p, t);

    const int sfc_lay = play[icol] > play[icol + size_t(nlay - 1) * ncol] ? 0 : nlay - 1;
    const bool at_sfc = ilay == sfc_lay;
    const float tl_up = tlev[icol + size_t(ilay + 1) * ncol];
    const float tl_dn = tlev[cl];
    const float ts = tsfc[icol];

    // minor_g entries of the layer's own atmosphere (s.itropo), those of the next g-point
    // loaded one iteration ahead, so that the kminor loads of an iteration do not wait on a
    // dependent table load; the minor loop runs to this atmosphere's count
    const int4* const mgt = k.minor_g[s.itropo];
    int4 nx = __ldg(mgt);
    for (int b = 0; b < k.nband; ++b) {
        const int g0 = k.band_lims[2 * b], g1 = k.band_lims[2 * b + 1];
        fused::Rec R;
        fused::record_weights(k, R, s, cg, kThreads, b);
        const float4 wp0 = R.wpl0, wp1 = R.wpl1;

        const float* tp = k.totplnk + size_t(b) * k.nplanck;
        const float pl = interpolate1D(t, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
        const float pinc = interpolate1D(tl_up, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
        const float pdec = interpolate1D(tl_dn, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
        float ps = 0.f, ps2 = 0.f;
        if (at_sfc) {
            ps = interpolate1D(ts, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
            ps2 = interpolate1D(ts + 1.f, k.temp_ref_min, k.totplnk_delta, k.nplanck, tp);
        }
        // two g-points per iteration: their table loads overlap (LW 1.89 -> 1.77 ms at 8192 x 128)
#pragma unroll 2
        for (int g = g0; g < g1; ++g) {
            const int4 mg = nx;
            nx = next_minor_row(mgt, g + 1, k.ngpt);
            const float ta = fused::tau_abs<DENSE>(k, R, g, mg, mg.x, scal, kThreads);
            const float4 p0 = __ldg(k.pfrac4 + (R.kb.x + g));
            const float4 p1 = __ldg(k.pfrac4 + (R.kb.y + g));
            const float pfrac = (wp0.x * p0.x + wp0.y * p0.y + wp0.z * p0.z + wp0.w * p0.w) +
                                (wp1.x * p1.x + wp1.y * p1.y + wp1.z * p1.z + wp1.w * p1.w);
            const Idx o = cl + Idx(g) * ncl;
            tau[o] = ta;
            lay_src[o] = pfrac * pl;
            lev_inc[o] = pfrac * pinc;
            lev_dec[o] = pfrac * pdec;
            if (at_sfc) {
                sfc_src[Idx(icol) + Idx(g) * Idx(ncol)] = pfrac * ps;
                sfc_jac[Idx(icol) + Idx(g) * Idx(ncol)] = pfrac * (ps2 - ps);
            }
        }
    }
}

template <bool DENSE, bool I32>
__global__ void __launch_bounds__(kThreads, 8)
gas_optics_sw_packed_kernel(const KdistView<float> k, const GasSet<float> gases, int ncol, int nlay,
                            const float* __restrict__ play, const float* __restrict__ plev,
                            const float* __restrict__ tlay, const float* __restrict__ col_dry_in,
                            float* __restrict__ tau, float* __restrict__ ssa, float* __restrict__ gasy)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x + threadIdx.y * kBX;
    float* cg = reinterpret_cast<float*>(smem_raw) + tid;                       // [ngas + 1]
    float* scal = reinterpret_cast<float*>(smem_raw) + (k.ngas + 1) * kThreads + tid;   // [max_nscal]

    using Idx = typename std::conditional<I32, unsigned, size_t>::type;
    const int icol = blockIdx.x * kBX + threadIdx.x;
    const int ilay = blockIdx.y * kBY + threadIdx.y;
    if (icol >= ncol || ilay >= nlay) return;
    const Idx cl = Idx(icol) + Idx(ilay) * Idx(ncol);
    const Idx ncl = Idx(ncol) * Idx(nlay);

    const float p = play[cl], t = tlay[cl];
    fill_col_gas(k, gases, ncol, nlay, icol, ilay, plev, col_dry_in, cg, kThreads);
    const fused::LayerState s = thread_layer_state(layer_interp(k, p, t), p, t);
    for (int sid = 0; sid < k.nscal[s.itropo]; ++sid)
        scal[sid * kThreads] = fused::kind_scaling(k, s.itropo, sid, cg, kThreads, p, t);
    const float col_rayl = cg[k.idx_h2o * kThreads] + cg[0];
    const float two_tmin = 2.f * FLT_MIN;

    const int4* const mgt = k.minor_g[s.itropo];   // as the longwave kernel
    int4 nx = __ldg(mgt);
    for (int b = 0; b < k.nband; ++b) {
        const int g0 = k.band_lims[2 * b], g1 = k.band_lims[2 * b + 1];
        fused::Rec R;
        fused::record_weights(k, R, s, cg, kThreads, b);
        const int kr0 = R.kr[0], kr1 = R.kr[1];
        // two g-points per iteration, as the longwave kernel
#pragma unroll 2
        for (int g = g0; g < g1; ++g) {
            const int4 mg = nx;
            nx = next_minor_row(mgt, g + 1, k.ngpt);
            const float ta = fused::tau_abs<DENSE>(k, R, g, mg, mg.x, scal, kThreads);
            const float2 r0 = __ldg(k.krayl2 + (kr0 + g));
            const float2 r1 = __ldg(k.krayl2 + (kr1 + g));
            const float tr = (R.fm.x * r0.x + R.fm.y * r0.y + R.fm.z * r1.x + R.fm.w * r1.y) * col_rayl;
            const float tt = ta + tr;
            const Idx o = cl + Idx(g) * ncl;
            tau[o] = tt;
            // approximate division (2 ulp for normal divisors; tt is far below 2^126)
            ssa[o] = tt > two_tmin ? __fdividef(tr, tt) : 0.f;
            gasy[o] = 0.f;
        }
    }
}

template <typename T>
__global__ void spread_solar_kernel(int ncol, int ngpt, const T* __restrict__ src, T* __restrict__ toa)
{
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < size_t(ncol) * ngpt) toa[i] = src[i / ncol];
}

// get_col_dry: compute_delta_plev + compute_m_air + compute_col_dry in one pass
// (src_cuda/Gas_optics_rrtmgp.cu:806-866).
template <typename T>
__global__ void col_dry_kernel(int ncol, int nlay, const T* __restrict__ h2o,
                               const T* __restrict__ plev, T* __restrict__ col_dry)
{
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= size_t(ncol) * nlay) return;
    col_dry[i] = col_dry_value(plev[i], plev[i + ncol], h2o[i]);
}

// Range check of Gas_optics_rrtmgp::gas_optics (src/Gas_optics_rrtmgp.cpp:812-827).
template <typename T>
__global__ void range_kernel(size_t n, const T* __restrict__ x, T lo, T hi, int bit, int* flags)
{
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T v = x[i];
    if (!(v >= lo && v <= hi)) atomicOr(flags, bit);
}

template <typename T>
int gas_optics_lw(rrtmgp_b200_kdist k, int ncol, int nlay, const T* play, const T* plev,
                  const T* tlay, const T* tsfc, const T* tlev, const T* col_dry,
                  const rrtmgp_b200_gas_conc* gases, int ngases, T* tau, T* lay_src, T* lev_inc,
                  T* lev_dec, T* sfc_src, T* sfc_jac, void* stream)
{
    RB_CHECK_ARG(k, "gas_optics_lw: null kdist");
    RB_CHECK_ARG(k->info.is_longwave, "gas_optics_lw: k-distribution has no internal source");
    RB_CHECK_ARG(ncol > 0 && nlay > 0, "gas_optics_lw: ncol and nlay must be > 0");
    RB_CHECK_ARG(play && plev && tlay && tsfc && tlev && tau && lay_src && lev_inc && lev_dec && sfc_src &&
                 sfc_jac, "gas_optics_lw: null array");
    if (const int dst = check_device(k->device, "gas_optics_lw")) return dst;
    GasSet<T> gs;
    int st = make_gas_set<T>(k, ncol, nlay, gases, ngases, gs);
    if (st) return st;
    const dim3 block(kBX, kBY), grid(ceil_div(ncol, kBX), ceil_div(nlay, kBY));
    if constexpr (std::is_same<T, float>::value) {
        if (packed_tables_ok(k->v32, true)) {
            const size_t psm = packed_smem_bytes(k->info.ngas, k->v32.max_nscal);
            const bool dense = k->v32.max_minor_per_g > 3, i32 = packed_index32(ncol, nlay, k->info.ngpt);
            const auto kernel = dense ? (i32 ? gas_optics_lw_packed_kernel<true, true>
                                             : gas_optics_lw_packed_kernel<true, false>)
                                      : (i32 ? gas_optics_lw_packed_kernel<false, true>
                                             : gas_optics_lw_packed_kernel<false, false>);
            kernel<<<grid, block, psm, as_stream(stream)>>>(k->v32, gs, ncol, nlay, play, plev, tlay, tsfc, tlev,
                                                            col_dry, tau, lay_src, lev_inc, lev_dec, sfc_src, sfc_jac);
            RB_LAUNCH("gas_optics_lw_packed_kernel");
            return RRTMGP_B200_OK;
        }
    }
    const size_t smem = size_t(k->info.ngas + 1 + kMaxBandGpt) * kThreads * sizeof(T);
    if (smem > 48 * 1024) {   // many gases in FP64: opt in to more than the default 48 KB
        static PerDeviceOnce attr;
        const int ast = attr.run([] { return cudaFuncSetAttribute(gas_optics_lw_kernel<T>,
                                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                                  227 * 1024); }, "gas_optics_lw attribute");
        if (ast) return ast;
    }
    gas_optics_lw_kernel<T><<<grid, block, smem, as_stream(stream)>>>(
        view<T>(k), gs, ncol, nlay, play, plev, tlay, tsfc, tlev, col_dry, tau, lay_src, lev_inc,
        lev_dec, sfc_src, sfc_jac);
    RB_LAUNCH("gas_optics_lw_kernel");
    return RRTMGP_B200_OK;
}

template <typename T>
int gas_optics_sw(rrtmgp_b200_kdist k, int ncol, int nlay, const T* play, const T* plev,
                  const T* tlay, const T* col_dry, const rrtmgp_b200_gas_conc* gases, int ngases,
                  T* tau, T* ssa, T* g, T* toa_src, void* stream)
{
    RB_CHECK_ARG(k, "gas_optics_sw: null kdist");
    RB_CHECK_ARG(!k->info.is_longwave, "gas_optics_sw: k-distribution has no external source");
    RB_CHECK_ARG(ncol > 0 && nlay > 0, "gas_optics_sw: ncol and nlay must be > 0");
    RB_CHECK_ARG(play && plev && tlay && tau && ssa && g && toa_src, "gas_optics_sw: null array");
    RB_CHECK_ARG(k->info.has_rayleigh, "gas_optics_sw: Rayleigh tables required");
    if (const int dst = check_device(k->device, "gas_optics_sw")) return dst;
    GasSet<T> gs;
    int st = make_gas_set<T>(k, ncol, nlay, gases, ngases, gs);
    if (st) return st;
    const dim3 block(kBX, kBY), grid(ceil_div(ncol, kBX), ceil_div(nlay, kBY));
    bool packed = false;
    if constexpr (std::is_same<T, float>::value) {
        if (packed_tables_ok(k->v32, false)) {
            const size_t psm = packed_smem_bytes(k->info.ngas, k->v32.max_nscal);
            const bool dense = k->v32.max_minor_per_g > 3, i32 = packed_index32(ncol, nlay, k->info.ngpt);
            const auto kernel = dense ? (i32 ? gas_optics_sw_packed_kernel<true, true>
                                             : gas_optics_sw_packed_kernel<true, false>)
                                      : (i32 ? gas_optics_sw_packed_kernel<false, true>
                                             : gas_optics_sw_packed_kernel<false, false>);
            kernel<<<grid, block, psm, as_stream(stream)>>>(k->v32, gs, ncol, nlay, play, plev, tlay, col_dry, tau,
                                                            ssa, g);
            RB_LAUNCH("gas_optics_sw_packed_kernel");
            packed = true;
        }
    }
    if (!packed) {
        const size_t smem = size_t(k->info.ngas + 1 + kMaxBandGpt) * kThreads * sizeof(T);
        if (smem > 48 * 1024) {
            static PerDeviceOnce attr;
            const int ast = attr.run([] { return cudaFuncSetAttribute(gas_optics_sw_kernel<T>,
                                                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                                      227 * 1024); }, "gas_optics_sw attribute");
            if (ast) return ast;
        }
        gas_optics_sw_kernel<T><<<grid, block, smem, as_stream(stream)>>>(
            view<T>(k), gs, ncol, nlay, play, plev, tlay, col_dry, tau, ssa, g);
        RB_LAUNCH("gas_optics_sw_kernel");
    }
    const size_t n = size_t(ncol) * k->info.ngpt;
    spread_solar_kernel<T><<<ceil_div(long(n), 256), 256, 0, as_stream(stream)>>>(
        ncol, k->info.ngpt, view<T>(k).solar_source, toa_src);
    RB_LAUNCH("spread_solar_kernel");
    return RRTMGP_B200_OK;
}

template <typename T>
int get_col_dry(int ncol, int nlay, const T* h2o, const T* plev, T* col_dry, void* stream)
{
    RB_CHECK_ARG(ncol > 0 && nlay > 0 && h2o && plev && col_dry, "get_col_dry: bad argument");
    const size_t n = size_t(ncol) * nlay;
    col_dry_kernel<T><<<ceil_div(long(n), 256), 256, 0, as_stream(stream)>>>(ncol, nlay, h2o, plev, col_dry);
    RB_LAUNCH("col_dry_kernel");
    return RRTMGP_B200_OK;
}

template <typename T>
int check_range(rrtmgp_b200_kdist k, int ncol, int nlay, const T* play, const T* plev,
                const T* tlay, const T* tlev, const T* tsfc, const T* col_dry, void* stream)
{
    RB_CHECK_ARG(k && ncol > 0 && nlay > 0 && play && plev && tlay, "check_range: bad argument");
    int* d_flags = k->d_flags;
    RB_CUDA(cudaMemsetAsync(d_flags, 0, sizeof(int), as_stream(stream)), "check_range memset");
    const T pmin = T(k->info.press_ref_min), pmax = T(k->info.press_ref_max);
    const T tmin = T(k->info.temp_ref_min), tmax = T(k->info.temp_ref_max);
    auto run = [&](size_t n, const T* x, T lo, T hi, int bit) {
        if (!x) return;
        range_kernel<T><<<ceil_div(long(n), 256), 256, 0, as_stream(stream)>>>(n, x, lo, hi, bit, d_flags);
    };
    const size_t ncl = size_t(ncol) * nlay;
    run(ncl, play, pmin, pmax, 1);
    run(ncl + ncol, plev, pmin, pmax, 2);
    run(ncl, tlay, tmin, tmax, 4);
    run(ncl + ncol, tlev, tmin, tmax, 8);
    run(size_t(ncol), tsfc, tmin, tmax, 16);
    run(ncl, col_dry, T(0), T(INFINITY), 32);
    int flags = 0;
    RB_LAUNCH("range_kernel");
    RB_CUDA(cudaMemcpyAsync(&flags, d_flags, sizeof(int), cudaMemcpyDeviceToHost, as_stream(stream)), "check_range copy");
    RB_CUDA(cudaStreamSynchronize(as_stream(stream)), "check_range sync");
    static const char* names[] = {"play", "plev", "tlay", "tlev", "tsfc", "col_dry"};
    for (int i = 0; i < 6; ++i)
        if (flags & (1 << i)) return fail(RRTMGP_B200_ERR_RANGE, std::string(names[i]) + " is out of range");
    return RRTMGP_B200_OK;
}

}  // namespace
}  // namespace rrtmgp_b200

using namespace rrtmgp_b200;

extern "C" {

int rrtmgp_b200_get_col_dry_f32(int ncol, int nlay, const float* h2o, const float* plev, float* cd, void* s)
{ return get_col_dry<float>(ncol, nlay, h2o, plev, cd, s); }
int rrtmgp_b200_get_col_dry_f64(int ncol, int nlay, const double* h2o, const double* plev, double* cd, void* s)
{ return get_col_dry<double>(ncol, nlay, h2o, plev, cd, s); }

int rrtmgp_b200_gas_optics_lw_f32(rrtmgp_b200_kdist k, int ncol, int nlay, const float* play,
        const float* plev, const float* tlay, const float* tsfc, const float* tlev, const float* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases, float* tau, float* lay_src, float* lev_src_inc,
        float* lev_src_dec, float* sfc_src, float* sfc_src_jac, void* stream)
{
    return gas_optics_lw<float>(k, ncol, nlay, play, plev, tlay, tsfc, tlev, col_dry, gases, ngases, tau,
                                lay_src, lev_src_inc, lev_src_dec, sfc_src, sfc_src_jac, stream);
}
int rrtmgp_b200_gas_optics_lw_f64(rrtmgp_b200_kdist k, int ncol, int nlay, const double* play,
        const double* plev, const double* tlay, const double* tsfc, const double* tlev, const double* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases, double* tau, double* lay_src, double* lev_src_inc,
        double* lev_src_dec, double* sfc_src, double* sfc_src_jac, void* stream)
{
    return gas_optics_lw<double>(k, ncol, nlay, play, plev, tlay, tsfc, tlev, col_dry, gases, ngases, tau,
                                 lay_src, lev_src_inc, lev_src_dec, sfc_src, sfc_src_jac, stream);
}
int rrtmgp_b200_gas_optics_sw_f32(rrtmgp_b200_kdist k, int ncol, int nlay, const float* play,
        const float* plev, const float* tlay, const float* col_dry, const rrtmgp_b200_gas_conc* gases,
        int ngases, float* tau, float* ssa, float* g, float* toa_src, void* stream)
{ return gas_optics_sw<float>(k, ncol, nlay, play, plev, tlay, col_dry, gases, ngases, tau, ssa, g, toa_src, stream); }
int rrtmgp_b200_gas_optics_sw_f64(rrtmgp_b200_kdist k, int ncol, int nlay, const double* play,
        const double* plev, const double* tlay, const double* col_dry, const rrtmgp_b200_gas_conc* gases,
        int ngases, double* tau, double* ssa, double* g, double* toa_src, void* stream)
{ return gas_optics_sw<double>(k, ncol, nlay, play, plev, tlay, col_dry, gases, ngases, tau, ssa, g, toa_src, stream); }

int rrtmgp_b200_check_range_f32(rrtmgp_b200_kdist k, int ncol, int nlay, const float* play,
        const float* plev, const float* tlay, const float* tlev, const float* tsfc, const float* col_dry, void* s)
{ return check_range<float>(k, ncol, nlay, play, plev, tlay, tlev, tsfc, col_dry, s); }
int rrtmgp_b200_check_range_f64(rrtmgp_b200_kdist k, int ncol, int nlay, const double* play,
        const double* plev, const double* tlay, const double* tlev, const double* tsfc, const double* col_dry, void* s)
{ return check_range<double>(k, ncol, nlay, play, plev, tlay, tlev, tsfc, col_dry, s); }

}  // extern "C"
