// Flux reductions: broadband and by-band g-point sums, net fluxes, heating rates.
//
// Sums over g-points are compensated: FP32 inputs are accumulated in FP64, FP64 inputs with a
// Neumaier (Kahan-Babuska) sum.  The reference sums naively in g order
// (fluxes_kernels.cu:26-62).
#include "common.cuh"

namespace rrtmgp_b200 {
namespace {

template <typename T> struct Acc;
template <> struct Acc<float> {
    double s = 0.;
    __device__ void add(float x) { s += double(x); }
    __device__ float get() const { return float(s); }
    __device__ double get_d() const { return s; }
};
template <> struct Acc<double> {
    double s = 0., c = 0.;
    __device__ void add(double x)
    {
        const double t = s + x;
        c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
        s = t;
    }
    __device__ double get() const { return s + c; }
    __device__ double get_d() const { return s + c; }
};

// sum_broadband_kernel + net_broadband_precalc_kernel (fluxes_kernels.cu:26-62).
template <typename T>
__global__ void broadband_kernel(size_t ncl, int ngpt, const T* __restrict__ up, const T* __restrict__ dn,
                                 const T* __restrict__ dir, T* __restrict__ bup, T* __restrict__ bdn,
                                 T* __restrict__ bdir, T* __restrict__ bnet)
{
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= ncl) return;
    Acc<T> au, ad, ar;
    for (int g = 0; g < ngpt; ++g) {
        au.add(up[i + g * ncl]);
        ad.add(dn[i + g * ncl]);
        if (dir) ar.add(dir[i + g * ncl]);
    }
    bup[i] = au.get();
    bdn[i] = ad.get();
    bnet[i] = T(ad.get_d() - au.get_d());
    if (dir && bdir) bdir[i] = ar.get();
}

// sum_byband / net_byband_full over band_lims(1,b)..band_lims(2,b) inclusive, as the F90
// (mo_fluxes_byband_kernels.F90:21-79).
template <typename T>
__global__ void byband_kernel(size_t ncl, int nband, const int* __restrict__ band_lims, const T* __restrict__ up,
                              const T* __restrict__ dn, const T* __restrict__ dir, T* __restrict__ bup,
                              T* __restrict__ bdn, T* __restrict__ bdir, T* __restrict__ bnet)
{
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (i >= ncl || b >= nband) return;
    Acc<T> au, ad, ar, an;
    for (int g = band_lims[2 * b]; g < band_lims[2 * b + 1]; ++g) {
        const T u = up[i + g * ncl], d = dn[i + g * ncl];
        au.add(u);
        ad.add(d);
        an.add(d - u);
        if (dir) ar.add(dir[i + g * ncl]);
    }
    const size_t o = i + size_t(b) * ncl;
    bup[o] = au.get();
    bdn[o] = ad.get();
    bnet[o] = an.get();
    if (dir && bdir) bdir[o] = ar.get();
}

// Heating rate [K/day] = g0 / cp * (Fnet(l) - Fnet(l+1)) / (p(l+1) - p(l)) * 86400.
template <typename T>
__global__ void heating_rate_kernel(int ncol, int nlay, const T* __restrict__ up, const T* __restrict__ dn,
                                    const T* __restrict__ plev, T* __restrict__ hr)
{
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= size_t(ncol) * nlay) return;
    const size_t j = i + ncol;
    const double fa = double(dn[i]) - double(up[i]);
    const double fb = double(dn[j]) - double(up[j]);
    hr[i] = T(9.80665 / 1004.64 * (fa - fb) / (double(plev[j]) - double(plev[i])) * 86400.);
}

template <typename T>
int broadband(int ncol, int nlev, int ngpt, const T* up, const T* dn, const T* dir, T* bup, T* bdn, T* bdir,
              T* bnet, void* stream)
{
    RB_CHECK_ARG(ncol > 0 && nlev > 0 && ngpt > 0 && up && dn && bup && bdn && bnet, "fluxes_broadband: bad argument");
    RB_CHECK_ARG(!dir || bdir, "fluxes_broadband: flux_dn_dir required with gpt_flux_dn_dir");
    const size_t ncl = size_t(ncol) * nlev;
    broadband_kernel<T><<<ceil_div(long(ncl), 256), 256, 0, as_stream(stream)>>>(ncl, ngpt, up, dn, dir, bup, bdn, bdir, bnet);
    RB_LAUNCH("broadband_kernel");
    return RRTMGP_B200_OK;
}

template <typename T>
int byband(rrtmgp_b200_bands b, int ncol, int nlev, const T* up, const T* dn, const T* dir, T* bup, T* bdn,
           T* bdir, T* bnet, void* stream)
{
    RB_CHECK_ARG(b && ncol > 0 && nlev > 0 && up && dn && bup && bdn && bnet, "fluxes_byband: bad argument");
    RB_CHECK_ARG(!dir || bdir, "fluxes_byband: bnd_flux_dn_dir required with gpt_flux_dn_dir");
    const size_t ncl = size_t(ncol) * nlev;
    const dim3 grid(ceil_div(long(ncl), 256), b->nband);
    byband_kernel<T><<<grid, 256, 0, as_stream(stream)>>>(ncl, b->nband, b->d_band_lims, up, dn, dir, bup, bdn, bdir, bnet);
    RB_LAUNCH("byband_kernel");
    return RRTMGP_B200_OK;
}

template <typename T>
int heating_rate(int ncol, int nlay, const T* up, const T* dn, const T* plev, T* hr, void* stream)
{
    RB_CHECK_ARG(ncol > 0 && nlay > 0 && up && dn && plev && hr, "heating_rate: bad argument");
    const size_t n = size_t(ncol) * nlay;
    heating_rate_kernel<T><<<ceil_div(long(n), 256), 256, 0, as_stream(stream)>>>(ncol, nlay, up, dn, plev, hr);
    RB_LAUNCH("heating_rate_kernel");
    return RRTMGP_B200_OK;
}

}  // namespace
}  // namespace rrtmgp_b200

using namespace rrtmgp_b200;

extern "C" {

int rrtmgp_b200_fluxes_broadband_f32(int ncol, int nlev, int ngpt, const float* up, const float* dn,
        const float* dir, float* bup, float* bdn, float* bdir, float* bnet, void* s)
{ return broadband<float>(ncol, nlev, ngpt, up, dn, dir, bup, bdn, bdir, bnet, s); }
int rrtmgp_b200_fluxes_broadband_f64(int ncol, int nlev, int ngpt, const double* up, const double* dn,
        const double* dir, double* bup, double* bdn, double* bdir, double* bnet, void* s)
{ return broadband<double>(ncol, nlev, ngpt, up, dn, dir, bup, bdn, bdir, bnet, s); }
int rrtmgp_b200_fluxes_byband_f32(rrtmgp_b200_bands b, int ncol, int nlev, const float* up, const float* dn,
        const float* dir, float* bup, float* bdn, float* bdir, float* bnet, void* s)
{ return byband<float>(b, ncol, nlev, up, dn, dir, bup, bdn, bdir, bnet, s); }
int rrtmgp_b200_fluxes_byband_f64(rrtmgp_b200_bands b, int ncol, int nlev, const double* up, const double* dn,
        const double* dir, double* bup, double* bdn, double* bdir, double* bnet, void* s)
{ return byband<double>(b, ncol, nlev, up, dn, dir, bup, bdn, bdir, bnet, s); }
int rrtmgp_b200_heating_rate_f32(int ncol, int nlay, const float* up, const float* dn, const float* plev, float* hr, void* s)
{ return heating_rate<float>(ncol, nlay, up, dn, plev, hr, s); }
int rrtmgp_b200_heating_rate_f64(int ncol, int nlay, const double* up, const double* dn, const double* plev, double* hr, void* s)
{ return heating_rate<double>(ncol, nlay, up, dn, plev, hr, s); }

}  // extern "C"
