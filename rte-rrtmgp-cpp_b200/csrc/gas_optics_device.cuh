// Device building blocks of the RRTMGP gas optics, shared by the per-stage kernels and the
// fused forward kernels.  Arithmetic follows the reference kernels
// (src_kernels_cuda/gas_optics_rrtmgp_kernels.cu) step by step; only the data layout and the
// granularity (per band instead of per g-point / per flavor) differ.
#pragma once

#include <cfloat>

#include "common.cuh"

namespace rrtmgp_b200 {

template <typename T> __device__ __forceinline__ T tiny_value();
template <> __device__ __forceinline__ float tiny_value<float>() { return FLT_MIN; }
template <> __device__ __forceinline__ double tiny_value<double>() { return DBL_MIN; }

// interpolate1D (gas_optics_rrtmgp_kernels.cu:1-12).
template <typename T>
__device__ __forceinline__ T interpolate1D(T val, T offset, T delta, int len, const T* __restrict__ table)
{
    const T val0 = (val - offset) / delta;
    const T frac = val0 - T(int(val0));
    const int idx = min(len - 1, max(1, int(val0) + 1));
    return table[idx - 1] + frac * (table[idx] - table[idx - 1]);
}

// Dry-air column of one layer (get_col_dry, src/Gas_optics_rrtmgp.cpp:764-792).
template <typename T>
__device__ __forceinline__ T col_dry_value(T plev0, T plev1, T h2o)
{
    constexpr T g0 = T(9.80665), avogad = T(6.02214076e23), m_dry = T(0.028964), m_h2o = T(0.018016);
    const T dp = fabs(plev0 - plev1);
    const T m_air = (m_dry + m_h2o * h2o) / (T(1) + h2o);
    T cd = T(10) * dp * avogad / (T(1000) * m_air * T(100) * g0);
    return cd / (T(1) + h2o);
}

template <typename T>
__device__ __forceinline__ T gas_vmr(const GasSet<T>& gs, int i, int ncol, int icol, int ilay)
{
    const int m = gs.mode[i];
    const T* v = gs.vmr[i];
    return m == 0 ? v[0] : (m == 1 ? v[ilay] : v[size_t(icol) + size_t(ilay) * ncol]);
}

// col_gas(0) = col_dry, col_gas(i) = vmr_i * col_dry (compute_gas_taus fill,
// src_cuda/Gas_optics_rrtmgp.cu:393-422); cg is strided by `s`.
template <typename T>
__device__ __forceinline__ void fill_col_gas(const KdistView<T>& k, const GasSet<T>& gs, int ncol, int nlay,
                                             int icol, int ilay, const T* __restrict__ plev,
                                             const T* __restrict__ col_dry_in, T* cg, int s)
{
    const size_t cl = size_t(icol) + size_t(ilay) * ncol;
    T cd;
    if (col_dry_in) cd = col_dry_in[cl];
    else cd = col_dry_value(plev[cl], plev[cl + ncol], gas_vmr(gs, k.idx_h2o - 1, ncol, icol, ilay));
    cg[0] = cd;
    for (int i = 0; i < k.ngas; ++i) cg[(i + 1) * s] = gas_vmr(gs, i, ncol, icol, ilay) * cd;
}

template <typename T>
struct LayerInterp {
    int jt, jp, itropo;  // jtemp, jpress (1-based), 0 = lower atmosphere (tropo), 1 = upper
    T ftemp, fpress;
};

// Temperature / pressure part of interpolation_kernel (gas_optics_rrtmgp_kernels.cu:245-254).
template <typename T>
__device__ __forceinline__ LayerInterp<T> layer_interp(const KdistView<T>& k, T p, T t)
{
    LayerInterp<T> li;
    int jt = int((t - (k.temp_ref_min - k.temp_ref_delta)) / k.temp_ref_delta);
    jt = min(k.ntemp - 1, max(1, jt));
    li.jt = jt;
    li.ftemp = (t - k.temp_ref[jt - 1]) / k.temp_ref_delta;
    const T lp = log(p);
    const T locpress = T(1) + (lp - k.press_ref_log0) / k.press_ref_log_delta;
    const int jp = min(k.npres - 1, max(1, int(locpress)));
    li.jp = jp;
    li.fpress = locpress - T(jp);
    li.itropo = (lp > k.press_ref_trop_log) ? 0 : 1;
    return li;
}

// Fractional eta position inside cell j (1-based).  FP64 keeps the reference's
// fmod(loceta, 1) (gas_optics_rrtmgp_kernels.cu:277).  That expression drops to 0 when
// loceta reaches neta-1 while jeta stays clamped at neta-1, a jump from the value at the
// last eta node to the one below it; in FP32 eta = 1 - 2e-9 rounds to exactly 1 (e.g. the
// (h2o, o3) flavor near the surface) and the jump changes tau by up to 40%.  The FP32 path
// therefore uses loceta - (j - 1), which equals fmod(loceta, 1) for every loceta < neta-1
// and is continuous at eta = 1.
template <typename T> __device__ __forceinline__ T eta_fraction(T loceta, int j);
template <> __device__ __forceinline__ double eta_fraction<double>(double loceta, int) { return fmod(loceta, 1.0); }
template <> __device__ __forceinline__ float eta_fraction<float>(float loceta, int j) { return loceta - float(j - 1); }

template <typename T>
struct FlavorWeights {
    int j0, j1;    // jeta for the two temperatures (1-based)
    T fm[4];       // fminor: (itemp 0: 1-feta, feta), (itemp 1: 1-feta, feta) x ftemp terms
    T cm[2];       // col_mix for the two temperatures
};

// Flavor part of interpolation_kernel (gas_optics_rrtmgp_kernels.cu:256-291).
template <typename T>
__device__ __forceinline__ FlavorWeights<T> flavor_weights(const KdistView<T>& k, int flav,
                                                           const LayerInterp<T>& li, const T* cg, int s)
{
    FlavorWeights<T> w;
    const int gas1 = k.flavor[2 * flav], gas2 = k.flavor[2 * flav + 1];
    const T c1 = cg[gas1 * s], c2 = cg[gas2 * s];
    const T two_tmin = T(2) * tiny_value<T>();
#pragma unroll
    for (int itemp = 0; itemp < 2; ++itemp) {
        const T* vr = k.vmr_ref + size_t(li.jt - 1 + itemp) * (k.ngas + 1) * 2 + li.itropo;
        const T ratio = vr[2 * gas1] / vr[2 * gas2];
        const T cm = c1 + ratio * c2;
        const T eta = cm > two_tmin ? c1 / cm : T(0.5);
        const T loceta = eta * T(k.neta - 1);
        // max(1, .) only guards memory for invalid (negative) concentrations; for valid
        // inputs eta lies in [0, 1] and this is the reference's min(int(loceta)+1, neta-1).
        const int j = max(1, min(int(loceta) + 1, k.neta - 1));
        const T feta = eta_fraction<T>(loceta, j);
        const T ftt = T(1 - itemp) + T(2 * itemp - 1) * li.ftemp;
        w.fm[2 * itemp] = (T(1) - feta) * ftt;
        w.fm[2 * itemp + 1] = feta * ftt;
        w.cm[itemp] = cm;
        if (itemp == 0) w.j0 = j; else w.j1 = j;
    }
    return w;
}

// The 8 (T, eta, p) corners of a g-point-fastest [t][p][eta][g] table, in the reference's
// fmajor order, plus the fmajor weights.
template <typename T>
struct MajorCorners {
    const T* c[8];
    T fmaj[8];
};

template <typename T>
__device__ __forceinline__ MajorCorners<T> major_corners(const KdistView<T>& k, const T* __restrict__ table,
                                                         const LayerInterp<T>& li, const FlavorWeights<T>& w)
{
    MajorCorners<T> mc;
    const int np1 = k.npres + 1;
    const int p0 = li.jp + li.itropo - 1;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int t = li.jt - 1 + i;
        const int e0 = (i == 0 ? w.j0 : w.j1) - 1;
        const size_t b00 = ((size_t(t) * np1 + p0) * k.neta + e0) * k.ngpt;
        const size_t dp = size_t(k.neta) * k.ngpt;
        mc.c[4 * i + 0] = table + b00;
        mc.c[4 * i + 1] = table + b00 + k.ngpt;
        mc.c[4 * i + 2] = table + b00 + dp;
        mc.c[4 * i + 3] = table + b00 + dp + k.ngpt;
        const T f0 = w.fm[2 * i], f1 = w.fm[2 * i + 1];
        mc.fmaj[4 * i + 0] = (T(1) - li.fpress) * f0;
        mc.fmaj[4 * i + 1] = (T(1) - li.fpress) * f1;
        mc.fmaj[4 * i + 2] = li.fpress * f0;
        mc.fmaj[4 * i + 3] = li.fpress * f1;
    }
    return mc;
}

// gas_optical_depths_major_kernel (gas_optics_rrtmgp_kernels.cu:330-339).
template <typename T>
__device__ __forceinline__ T major_tau(const MajorCorners<T>& mc, const FlavorWeights<T>& w,
                                       const LayerInterp<T>&, int g)
{
    T acc = T(0);
#pragma unroll
    for (int i = 0; i < 2; ++i)
        acc += w.cm[i] * (mc.fmaj[4 * i + 0] * __ldg(mc.c[4 * i + 0] + g) + mc.fmaj[4 * i + 1] * __ldg(mc.c[4 * i + 1] + g) +
                          mc.fmaj[4 * i + 2] * __ldg(mc.c[4 * i + 2] + g) + mc.fmaj[4 * i + 3] * __ldg(mc.c[4 * i + 3] + g));
    return acc;
}

// Planck fraction (Planck_source_kernel, gas_optics_rrtmgp_kernels.cu:181-190).
template <typename T>
__device__ __forceinline__ T planck_fraction(const MajorCorners<T>& pc, const FlavorWeights<T>&,
                                             const LayerInterp<T>&, int g)
{
    return (pc.fmaj[0] * __ldg(pc.c[0] + g) + pc.fmaj[1] * __ldg(pc.c[1] + g) + pc.fmaj[2] * __ldg(pc.c[2] + g) +
            pc.fmaj[3] * __ldg(pc.c[3] + g)) +
           (pc.fmaj[4] * __ldg(pc.c[4] + g) + pc.fmaj[5] * __ldg(pc.c[5] + g) + pc.fmaj[6] * __ldg(pc.c[6] + g) +
            pc.fmaj[7] * __ldg(pc.c[7] + g));
}

// Rayleigh absorption coefficient (compute_tau_rayleigh_kernel, :597-611); kr = krayl of the
// layer's atmosphere, layout [t][eta][g].
template <typename T>
__device__ __forceinline__ T rayleigh_k(const KdistView<T>& k, const T* __restrict__ kr, const LayerInterp<T>& li,
                                        const FlavorWeights<T>& w, int g)
{
    const size_t st = size_t(k.neta) * k.ngpt;
    const T* r0 = kr + (li.jt - 1) * st + size_t(w.j0 - 1) * k.ngpt;
    const T* r1 = kr + size_t(li.jt) * st + size_t(w.j1 - 1) * k.ngpt;
    return w.fm[0] * __ldg(r0 + g) + w.fm[1] * __ldg(r0 + k.ngpt + g) + w.fm[2] * __ldg(r1 + g) +
           w.fm[3] * __ldg(r1 + k.ngpt + g);
}

// Minor-absorber scaling of one interval (gas_optical_depths_minor_kernel, :396-417).
template <typename T>
__device__ __forceinline__ T minor_scaling(const KdistView<T>& k, int a, int im, const T* cg, int s, T p, T t)
{
    const int flags = k.minor_flags[a][im];
    T scaling = cg[k.minor_gas[a][im] * s];
    if (flags & 1) {
        const T PaTohPa = T(0.01);
        scaling *= PaTohPa * p / t;
        const int sg = k.minor_sgas[a][im];
        if (sg > 0) {
            const T vmr_fact = T(1) / cg[0];
            const T dry_fact = T(1) / (T(1) + cg[k.idx_h2o * s] * vmr_fact);
            if (flags & 2) scaling *= (T(1) - cg[sg * s] * vmr_fact * dry_fact);
            else scaling *= cg[sg * s] * vmr_fact * dry_fact;
        }
    }
    return scaling;
}

// Minor contribution to the g-points [g0, g1) of band b (gas_optical_depths_minor_kernel,
// :428-472): acc[(g - g0) * as] += scaling * 4-point interpolation of kminor.
template <typename T>
__device__ __forceinline__ void add_minor(const KdistView<T>& k, const LayerInterp<T>& li,
                                          const FlavorWeights<T>& fw, int flav, const T* cg, int s,
                                          T p, T t, int b, int g0, int g1, T* acc, int as)
{
    const int a = li.itropo;
    const int nc = k.ncontrib[a];
    const T* __restrict__ km = k.kminor[a];
    for (int ii = k.band_minor_begin[a][b]; ii < k.band_minor_begin[a][b + 1]; ++ii) {
        const int im = k.band_minor_list[a][ii];
        const T scaling = minor_scaling(k, a, im, cg, s, p, t);
        const FlavorWeights<T> w = (k.minor_flav[a][im] == flav) ? fw
                                   : flavor_weights(k, k.minor_flav[a][im], li, cg, s);
        const int gs = k.minor_gstart[a][im], ge = k.minor_gend[a][im];
        const int kst = k.minor_kstart[a][im];
        const T* r0 = km + (size_t(li.jt - 1) * k.neta + (w.j0 - 1)) * nc;
        const T* r1 = km + (size_t(li.jt - 1) * k.neta + w.j0) * nc;
        const T* r2 = km + (size_t(li.jt) * k.neta + (w.j1 - 1)) * nc;
        const T* r3 = km + (size_t(li.jt) * k.neta + w.j1) * nc;
        const int lo = max(gs, g0), hi = min(ge, g1);
        for (int g = lo; g < hi; ++g) {
            const int c = kst + (g - gs);
            const T lt = w.fm[0] * __ldg(r0 + c) + w.fm[1] * __ldg(r1 + c) + w.fm[2] * __ldg(r2 + c) +
                         w.fm[3] * __ldg(r3 + c);
            acc[(g - g0) * as] += lt * scaling;
        }
    }
}

}  // namespace rrtmgp_b200
