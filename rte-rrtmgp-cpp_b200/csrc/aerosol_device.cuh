// Aerosol optics (shortwave two-stream) on the device: the band look-up tables of
// Aerosol_optics_gpu (src_cuda/Aerosol_optics.cu:11-168) as a per-(column, layer) function that
// the standalone kernel and the fused shortwave kernels share.
#pragma once

#include "common.cuh"

namespace rrtmgp_b200 {

constexpr int kNAerosol = 11;   // aermr01 .. aermr11

// Device tables of one precision: rh_upper [nhum], then the hydrophobic tables
// [mext, ssa, g][nphobic][nband], then the hydrophilic ones [mext, ssa, g][nphilic][nhum][nband]
// (the netCDF file order of load_and_init_aerosol_optics, src_test/Radiation_solver.cu:366-401).
template <typename T>
struct AerosolLut {
    int nband, nhum, nphilic, nphobic;
    const T* tab;
    __host__ __device__ const T* rh_upper() const { return tab; }
    __host__ __device__ const T* phobic(int q) const { return tab + nhum + size_t(q) * nphobic * nband; }
    __host__ __device__ const T* philic(int q) const
    {
        return tab + nhum + size_t(3) * nphobic * nband + size_t(q) * nphilic * nhum * nband;
    }
};

// Mass mixing ratios of the 11 species as given (mode 0 scalar, 1 profile, 2 field), like GasSet.
template <typename T>
struct AerosolSet {
    const T* mmr[kNAerosol];
    int mode[kNAerosol];
};

template <typename T>
__device__ __forceinline__ T aerosol_mmr(const AerosolSet<T>& s, int i, int ncol, int icol, int l)
{
    const T* p = s.mmr[i];
    const int m = s.mode[i];
    return m == 0 ? p[0] : (m == 1 ? p[l] : p[icol + size_t(l) * ncol]);
}

// Humidity class: the first rh_upper entry not below rh (find_rh_class,
// src_cuda/Aerosol_optics.cu:11-23), clamped to the last class (the reference reads past the
// table for rh above its last entry).
template <typename T>
__device__ __forceinline__ int aerosol_rh_class(const AerosolLut<T>& L, T rh)
{
    const T* ru = L.rh_upper();
    int i = 0;
    while (i < L.nhum - 1 && ru[i] < rh) ++i;
    return i;
}

// tau, tau*ssa, tau*ssa*g of band b summed over the species, in the reference kernel's order
// DU1 DU2 DU3 BC1 BC2 SS1 SS2 SS3 SU OM1 OM2 (compute_from_table_kernel,
// src_cuda/Aerosol_optics.cu:58-168).  mmr[i] holds aermr(i+1); dpg = |dp| / 9.81.
template <typename T>
__device__ __forceinline__ void aerosol_band(const AerosolLut<T>& L, const T mmr[kNAerosol], int ihum, T dpg, int b,
                                             T& tau, T& taussa, T& taussag)
{
    // species: aermr index (0-based), hydrophilic?, table type (0-based)
    constexpr int kMmr[kNAerosol] = {3, 4, 5, 8, 9, 0, 1, 2, 10, 7, 6};
    constexpr int kPhilic[kNAerosol] = {0, 0, 0, 0, 0, 1, 1, 1, 1, 0, 1};
    constexpr int kType[kNAerosol] = {0, 7, 5, 10, 10, 0, 1, 2, 4, 9, 3};
    tau = T(0);
    taussa = T(0);
    taussag = T(0);
#pragma unroll
    for (int s = 0; s < kNAerosol; ++s) {
        size_t idx;
        const T* me;
        const T* ss;
        const T* gg;
        if (kPhilic[s]) {
            idx = b + size_t(ihum) * L.nband + size_t(kType[s]) * L.nband * L.nhum;
            me = L.philic(0);
            ss = L.philic(1);
            gg = L.philic(2);
        } else {
            idx = b + size_t(kType[s]) * L.nband;
            me = L.phobic(0);
            ss = L.phobic(1);
            gg = L.phobic(2);
        }
        const T od = mmr[kMmr[s]] * dpg * me[idx];
        tau += od;
        taussa += od * ss[idx];
        taussag += od * ss[idx] * gg[idx];
    }
}

// The same sums plus the absorption optical depth sum_s od_s (1 - ssa_s) of band b, formed per
// species (the fused shortwave kernels carry 1 - ssa as absorption over extinction, which a
// difference tau - tau*ssa would lose for nearly conservative scattering).
template <typename T>
__device__ __forceinline__ void aerosol_band_abs(const AerosolLut<T>& L, const T mmr[kNAerosol], int ihum, T dpg,
                                                 int b, T& tau, T& taussa, T& taussag, T& tauabs)
{
    constexpr int kMmr[kNAerosol] = {3, 4, 5, 8, 9, 0, 1, 2, 10, 7, 6};
    constexpr int kPhilic[kNAerosol] = {0, 0, 0, 0, 0, 1, 1, 1, 1, 0, 1};
    constexpr int kType[kNAerosol] = {0, 7, 5, 10, 10, 0, 1, 2, 4, 9, 3};
    tau = T(0);
    taussa = T(0);
    taussag = T(0);
    tauabs = T(0);
#pragma unroll
    for (int s = 0; s < kNAerosol; ++s) {
        const size_t idx = kPhilic[s] ? b + size_t(ihum) * L.nband + size_t(kType[s]) * L.nband * L.nhum
                                      : b + size_t(kType[s]) * L.nband;
        const T* me = kPhilic[s] ? L.philic(0) : L.phobic(0);
        const T* ss = kPhilic[s] ? L.philic(1) : L.phobic(1);
        const T* gg = kPhilic[s] ? L.philic(2) : L.phobic(2);
        const T od = mmr[kMmr[s]] * dpg * me[idx];
        const T w = ss[idx];
        tau += od;
        taussa += od * w;
        taussag += od * w * gg[idx];
        tauabs += od * (T(1) - w);
    }
}

// Host-side helpers of aerosol.cu used by the fused shortwave launchers.
template <typename T>
int make_aerosol_set(int ncol, int nlay, const rrtmgp_b200_gas_conc* aer, int naer, AerosolSet<T>& out);
AerosolLut<float> aerosol_lut32(const rrtmgp_b200_aerosol_t* a);

}  // namespace rrtmgp_b200
