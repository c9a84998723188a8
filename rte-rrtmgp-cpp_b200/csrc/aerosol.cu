// Aerosol optics (shortwave, two-stream): Aerosol_optics_gpu (include/Aerosol_optics.h:64-86,
// src_cuda/Aerosol_optics.cu:188-279).  One thread per (column, layer): the humidity class,
// the layer mass and the 11 mass mixing ratios are read once and every band is written
// (column-fastest, coalesced), with ssa and g formed directly (combine_and_store_kernel,
// :170-186) instead of through three (ncol, nlay, nband) temporaries.
#include <cfloat>
#include <limits>

#include "aerosol_device.cuh"

struct rrtmgp_b200_aerosol_t {
    int nband = 0, nhum = 0, nphilic = 0, nphobic = 0;
    float* lut32 = nullptr;
    double* lut64 = nullptr;
};

namespace rrtmgp_b200 {
namespace {

template <typename T>
AerosolLut<T> lut_view(const rrtmgp_b200_aerosol_t* a);
template <>
AerosolLut<float> lut_view<float>(const rrtmgp_b200_aerosol_t* a)
{
    return AerosolLut<float>{a->nband, a->nhum, a->nphilic, a->nphobic, a->lut32};
}
template <>
AerosolLut<double> lut_view<double>(const rrtmgp_b200_aerosol_t* a)
{
    return AerosolLut<double>{a->nband, a->nhum, a->nphilic, a->nphobic, a->lut64};
}

// One thread per (column, layer).  The block first copies the tables (a few thousand values)
// into shared memory: the per-band lookups of the 11 species then cost shared-memory loads
// (same address across the warp for the hydrophobic species, distinct banks for the
// hydrophilic ones, whose rows differ by nband per humidity class) instead of L1 gathers.
template <typename T>
__global__ void __launch_bounds__(512) aerosol_optics_kernel(const AerosolLut<T> Lg, const AerosolSet<T> as, int ncol,
                                                             int nlay, const T* __restrict__ rh,
                                                             const T* __restrict__ plev, T* __restrict__ tau,
                                                             T* __restrict__ ssa, T* __restrict__ g)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* tab = reinterpret_cast<T*>(smem_raw);
    const int n = Lg.nhum + 3 * Lg.nphobic * Lg.nband + 3 * Lg.nphilic * Lg.nhum * Lg.nband;
    for (int i = threadIdx.x; i < n; i += blockDim.x) tab[i] = Lg.tab[i];
    __syncthreads();
    const AerosolLut<T> L{Lg.nband, Lg.nhum, Lg.nphilic, Lg.nphobic, tab};
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t ncl = size_t(ncol) * nlay;
    if (i >= ncl) return;
    const int icol = int(i % ncol), l = int(i / ncol);
    const int ihum = aerosol_rh_class(L, rh[i]);
    const T dpg = fabs(plev[i] - plev[i + ncol]) / T(9.81);
    T mmr[kNAerosol];
#pragma unroll
    for (int s = 0; s < kNAerosol; ++s) mmr[s] = aerosol_mmr(as, s, ncol, icol, l);
    const T eps = std::numeric_limits<T>::epsilon();
    for (int b = 0; b < L.nband; ++b) {
        T t, ts, tsg;
        aerosol_band(L, mmr, ihum, dpg, b, t, ts, tsg);
        const size_t o = i + size_t(b) * ncl;
        tau[o] = t;
        ssa[o] = ts / (t > eps ? t : eps);
        g[o] = tsg / (ts > eps ? ts : eps);
    }
}

template <typename T>
size_t aerosol_smem(const rrtmgp_b200_aerosol_t* a)
{
    return sizeof(T) * (size_t(a->nhum) + 3 * size_t(a->nphobic) * a->nband + 3 * size_t(a->nphilic) * a->nhum * a->nband);
}

}  // namespace

// Aerosol species of a gas_conc list (names aermr01 .. aermr11, like Aerosol_concs =
// Gas_concs, include/Aerosol_optics.h:35-36); every species is required (the reference's
// get_vmr throws for a missing one).
template <typename T>
int make_aerosol_set(int ncol, int nlay, const rrtmgp_b200_gas_conc* aer, int naer, AerosolSet<T>& out)
{
    RB_CHECK_ARG(naer >= 0 && (naer == 0 || aer), "aerosol_optics: null aerosol list");
    for (int s = 0; s < kNAerosol; ++s) {
        char name[8];
        snprintf(name, sizeof(name), "aermr%02d", s + 1);
        int found = -1;
        for (int j = 0; j < naer; ++j)
            if (aer[j].name && std::string(aer[j].name) == name) found = j;
        if (found < 0) return fail(RRTMGP_B200_ERR_MISSING_GAS, std::string("aerosol_optics: ") + name + " not found");
        const rrtmgp_b200_gas_conc& c = aer[found];
        RB_CHECK_ARG(c.vmr != nullptr, std::string("aerosol_optics: null array for ") + name);
        out.mmr[s] = static_cast<const T*>(c.vmr);
        if (c.dim1 == 1 && c.dim2 == 1) out.mode[s] = 0;
        else if (c.dim1 == 1 && c.dim2 == nlay) out.mode[s] = 1;
        else if (c.dim1 == ncol && c.dim2 == nlay) out.mode[s] = 2;
        else return fail(RRTMGP_B200_ERR_ARG, std::string("aerosol_optics: bad dimensions for ") + name);
    }
    return RRTMGP_B200_OK;
}

template int make_aerosol_set<float>(int, int, const rrtmgp_b200_gas_conc*, int, AerosolSet<float>&);
template int make_aerosol_set<double>(int, int, const rrtmgp_b200_gas_conc*, int, AerosolSet<double>&);

AerosolLut<float> aerosol_lut32(const rrtmgp_b200_aerosol_t* a) { return lut_view<float>(a); }

namespace {

template <typename T>
int aerosol_optics(rrtmgp_b200_aerosol a, int ncol, int nlay, const rrtmgp_b200_gas_conc* aer, int naer, const T* rh,
                   const T* plev, T* tau, T* ssa, T* g, void* stream)
{
    RB_CHECK_ARG(a, "aerosol_optics: null handle");
    RB_CHECK_ARG(ncol > 0 && nlay > 0, "aerosol_optics: ncol, nlay > 0 required");
    RB_CHECK_ARG(rh && plev && tau && ssa && g, "aerosol_optics: null array");
    AerosolSet<T> as;
    int st = make_aerosol_set<T>(ncol, nlay, aer, naer, as);
    if (st) return st;
    const size_t n = size_t(ncol) * nlay;
    const int threads = 512;
    const size_t smem = aerosol_smem<T>(a);
    RB_CHECK_ARG(smem <= 227 * 1024, "aerosol_optics: tables exceed shared memory");
    if (smem > 48 * 1024)
        RB_CUDA(cudaFuncSetAttribute(aerosol_optics_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
                "aerosol_optics attribute");
    aerosol_optics_kernel<T><<<unsigned((n + threads - 1) / threads), threads, smem, as_stream(stream)>>>(
        lut_view<T>(a), as, ncol, nlay, rh, plev, tau, ssa, g);
    RB_LAUNCH("aerosol_optics_kernel");
    return RRTMGP_B200_OK;
}

}  // namespace
}  // namespace rrtmgp_b200

using namespace rrtmgp_b200;

extern "C" {

int rrtmgp_b200_aerosol_create(const rrtmgp_b200_aerosol_tables* t, rrtmgp_b200_aerosol* out)
{
    RB_CHECK_ARG(t && out, "aerosol_create: null argument");
    *out = nullptr;
    RB_CHECK_ARG(t->nband > 0 && t->nhum > 0, "aerosol_create: bad table dimensions");
    RB_CHECK_ARG(t->nphobic >= 11 && t->nphilic >= 5,
                 "aerosol_create: need 11 hydrophobic and 5 hydrophilic species types");
    RB_CHECK_ARG(t->rh_upper && t->mext_phobic && t->ssa_phobic && t->g_phobic && t->mext_philic && t->ssa_philic &&
                 t->g_philic, "aerosol_create: missing table");
    const size_t nph = size_t(t->nphobic) * t->nband, npl = size_t(t->nphilic) * t->nhum * t->nband;
    const size_t n = t->nhum + 3 * nph + 3 * npl;
    std::vector<double> h(n);
    size_t o = 0;
    for (int i = 0; i < t->nhum; ++i) h[o++] = t->rh_upper[i];
    for (const double* src : {t->mext_phobic, t->ssa_phobic, t->g_phobic})
        for (size_t i = 0; i < nph; ++i) h[o++] = src[i];
    for (const double* src : {t->mext_philic, t->ssa_philic, t->g_philic})
        for (size_t i = 0; i < npl; ++i) h[o++] = src[i];
    std::vector<float> hf(h.begin(), h.end());
    auto* a = new rrtmgp_b200_aerosol_t();
    a->nband = t->nband;
    a->nhum = t->nhum;
    a->nphilic = t->nphilic;
    a->nphobic = t->nphobic;
    if (cudaMalloc(&a->lut64, n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&a->lut32, n * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        rrtmgp_b200_aerosol_destroy(a);
        return fail(RRTMGP_B200_ERR_ALLOC, "aerosol_create: cudaMalloc failed");
    }
    if (cudaMemcpy(a->lut64, h.data(), n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(a->lut32, hf.data(), n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        const int st = cuda_status(cudaGetLastError(), "aerosol_create");
        rrtmgp_b200_aerosol_destroy(a);
        return st;
    }
    *out = a;
    return RRTMGP_B200_OK;
}

void rrtmgp_b200_aerosol_destroy(rrtmgp_b200_aerosol a)
{
    if (!a) return;
    if (a->lut32) cudaFree(a->lut32);
    if (a->lut64) cudaFree(a->lut64);
    delete a;
}

int rrtmgp_b200_aerosol_optics_f32(rrtmgp_b200_aerosol a, int ncol, int nlay, const rrtmgp_b200_gas_conc* aerosols,
                                   int naerosols, const float* rh, const float* plev, float* tau, float* ssa,
                                   float* g, void* stream)
{
    return aerosol_optics<float>(a, ncol, nlay, aerosols, naerosols, rh, plev, tau, ssa, g, stream);
}

int rrtmgp_b200_aerosol_optics_f64(rrtmgp_b200_aerosol a, int ncol, int nlay, const rrtmgp_b200_gas_conc* aerosols,
                                   int naerosols, const double* rh, const double* plev, double* tau, double* ssa,
                                   double* g, void* stream)
{
    return aerosol_optics<double>(a, ncol, nlay, aerosols, naerosols, rh, plev, tau, ssa, g, stream);
}

}  // extern "C"
