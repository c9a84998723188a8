// Heating rates of the per-stage (class-API) path from per-layer absorbed flux.
//
// The reference has no heating-rate routine; a caller differences its broadband level fluxes.
// In the top layers of a model atmosphere (Delta p ~ 0.1 Pa) one FP32 rounding of a
// ~1000 W/m2 level flux is worth ~1 K/day, so a difference of FP32 level fluxes cannot give
// 0.01 K/day there.  These kernels form the heating rate of layer l from the flux the layer
// absorbs, summed over g-points in FP64:
//   longwave  A_g = (1 - T) (F_dn,g(top) + F_up,g(bottom)) - pi (S_dn + S_up)   (one angle,
//             D = 1.66, weight 0.5: the per-stage solver's transmissivity and linear-in-tau
//             sources recomputed from tau and the Planck sources);
//   shortwave A_g = F_dir,g(top) (1 - Tn - Rdir - Tdir) + (F_dif,g(top) + F_up,g(bottom)) (1 - R - T)
//             (the per-stage solver's two-stream coefficients recomputed from tau, ssa, g, mu0;
//             F_dif = F_dn - F_dir).
// These equal the net-flux divergence of the solvers' recurrences exactly, but every FP32
// rounding of a level flux enters multiplied by the layer's absorptance, which is small
// exactly where the layers are thin.  HR = g/cp 86400 sum_g A_g / |Delta p| as
// heating_rate_kernel.  One thread per (column, layer), lanes over consecutive columns; the
// inputs of g-point g + 1 are loaded while g-point g is computed (in the plain loop every
// g-point waited for its own loads from memory), with 32-bit offsets (I32) when every
// (column, level, g-point) offset fits in 31 bits.
#include <cfloat>
#include <type_traits>

#include "common.cuh"
#include "rte_device.cuh"
#include "sw_common.cuh"

namespace rrtmgp_b200 {
namespace {

constexpr double kG0OverCp = 9.80665 / 1004.64;

// 1 - T and the layer sources: FP32 as the solvers (lw_layer_fast); FP64 the reference
// expressions with 1 - T = -expm1(-tau D).
template <typename T>
__device__ __forceinline__ void lw_layer_terms(T tau, T D, T lay, T ldn, T lup, T& omt, T& sdn, T& sup);
template <>
__device__ __forceinline__ void lw_layer_terms<float>(float tau, float D, float lay, float ldn, float lup, float& omt,
                                                      float& sdn, float& sup)
{
    lw_layer_fast(tau, D, lay, ldn, lup, omt, sdn, sup);
}
template <>
__device__ __forceinline__ void lw_layer_terms<double>(double tau, double D, double lay, double ldn, double lup,
                                                       double& omt, double& sdn, double& sup)
{
    double trans;
    lw_layer(tau, D, lay, ldn, lup, trans, sdn, sup);
    omt = -expm1(-tau * D);
}

inline bool hr_index32(int ncol, int nlay, int ngpt)
{
    return size_t(ncol) * size_t(nlay + 1) * size_t(ngpt) < (size_t(1) << 31);
}

template <typename T, bool I32>
__global__ void heating_rate_lw_layers_kernel(int ncol, int nlay, int ngpt, int top_at_1, const T* __restrict__ tau,
                                              const T* __restrict__ lay_src, const T* __restrict__ lev_inc,
                                              const T* __restrict__ lev_dec, const T* __restrict__ up,
                                              const T* __restrict__ dn, const T* __restrict__ plev,
                                              T* __restrict__ hr)
{
    using Idx = typename std::conditional<I32, unsigned, size_t>::type;
    const int icol = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = blockIdx.y;
    if (icol >= ncol) return;
    const Idx ncl = Idx(ncol) * Idx(nlay), ncv = Idx(ncol) * Idx(nlay + 1);
    const Idx cl = Idx(icol) + Idx(l) * Idx(ncol);
    const int lt = top_at_1 ? l : l + 1, lb = top_at_1 ? l + 1 : l;
    const T* lev_dn = top_at_1 ? lev_inc : lev_dec;
    const T* lev_up = top_at_1 ? lev_dec : lev_inc;
    const T D = T(1.66), pi = pi_value<T>();
    Idx i = cl, ot = Idx(icol) + Idx(lt) * Idx(ncol), ob = Idx(icol) + Idx(lb) * Idx(ncol);
    T n_tau = tau[i], n_lay = lay_src[i], n_ldn = lev_dn[i], n_lup = lev_up[i], n_dn = dn[ot], n_up = up[ob];
    double acc = 0.0;
    for (int g = 0; g < ngpt; ++g) {
        const T t = n_tau, ly = n_lay, ldn = n_ldn, lup = n_lup, fdn = n_dn, fup = n_up;
        if (g + 1 < ngpt) {
            i += ncl;
            ot += ncv;
            ob += ncv;
            n_tau = tau[i];
            n_lay = lay_src[i];
            n_ldn = lev_dn[i];
            n_lup = lev_up[i];
            n_dn = dn[ot];
            n_up = up[ob];
        }
        T omt, sdn, sup;
        lw_layer_terms<T>(t, D, ly, ldn, lup, omt, sdn, sup);
        acc += double(omt * (fdn + fup) - pi * (sdn + sup));
    }
    const double dp = fabs(double(plev[icol + size_t(lb) * ncol]) - double(plev[icol + size_t(lt) * ncol]));
    hr[cl] = T(kG0OverCp * 86400.0 * acc / dp);
}

// Two-stream coefficients and the layer's direct and diffuse absorptances, as the per-stage
// shortwave solver computes them.
template <typename T>
__device__ __forceinline__ void sw_absorptances(T tau, T ssa, T g, T mu0, T& adir, T& adif);
template <>
__device__ __forceinline__ void sw_absorptances<float>(float tau, float ssa, float g, float mu0, float& adir,
                                                       float& adif)
{
    float R, Tt, Rdir, Tdir, Tn;
    fused::sw_layer_fast(tau, ssa, 1.f - ssa, g, mu0, 1.f / mu0, R, Tt, Rdir, Tdir, Tn, adif, adir);
}
template <>
__device__ __forceinline__ void sw_absorptances<double>(double tau, double ssa, double g, double mu0, double& adir,
                                                        double& adif)
{
    double R, Tt, Rdir, Tdir, Tn;
    sw_two_stream<double>(tau, ssa, g, mu0, R, Tt, Rdir, Tdir, Tn);
    adif = 1. - R - Tt;
    adir = 1. - Tn - Rdir - Tdir;
}

template <typename T, bool I32>
__global__ void heating_rate_sw_layers_kernel(int ncol, int nlay, int ngpt, int top_at_1, const T* __restrict__ tau,
                                              const T* __restrict__ ssa, const T* __restrict__ gasy,
                                              const T* __restrict__ mu0, const T* __restrict__ up,
                                              const T* __restrict__ dn, const T* __restrict__ dir,
                                              const T* __restrict__ plev, T* __restrict__ hr)
{
    using Idx = typename std::conditional<I32, unsigned, size_t>::type;
    const int icol = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = blockIdx.y;
    if (icol >= ncol) return;
    const Idx ncl = Idx(ncol) * Idx(nlay), ncv = Idx(ncol) * Idx(nlay + 1);
    const Idx cl = Idx(icol) + Idx(l) * Idx(ncol);
    const int lt = top_at_1 ? l : l + 1, lb = top_at_1 ? l + 1 : l;
    const T m0 = mu0[icol];
    Idx i = cl, ot = Idx(icol) + Idx(lt) * Idx(ncol), ob = Idx(icol) + Idx(lb) * Idx(ncol);
    T n_tau = tau[i], n_ssa = ssa[i], n_g = gasy[i], n_dir = dir[ot], n_dn = dn[ot], n_up = up[ob];
    double acc = 0.0;
    for (int g = 0; g < ngpt; ++g) {
        const T t = n_tau, w = n_ssa, gy = n_g, fdir = n_dir, fdn = n_dn, fup = n_up;
        if (g + 1 < ngpt) {
            i += ncl;
            ot += ncv;
            ob += ncv;
            n_tau = tau[i];
            n_ssa = ssa[i];
            n_g = gasy[i];
            n_dir = dir[ot];
            n_dn = dn[ot];
            n_up = up[ob];
        }
        T adir, adif;
        sw_absorptances<T>(t, w, gy, m0, adir, adif);
        acc += double(fdir * adir + ((fdn - fdir) + fup) * adif);
    }
    const double dp = fabs(double(plev[icol + size_t(lb) * ncol]) - double(plev[icol + size_t(lt) * ncol]));
    hr[cl] = T(kG0OverCp * 86400.0 * acc / dp);
}

// Heating rate from the per-(layer, g-point) absorbed flux that rte_sw_abs writes: the sum over
// g-points in FP64 per (column, layer), over |Delta p|.  The next g-point's row is loaded while
// the current one is added.
template <bool I32>
__global__ void heating_rate_from_layer_abs_kernel(int ncol, int nlay, int ngpt, const float* __restrict__ layer_abs,
                                                   const float* __restrict__ plev, float* __restrict__ hr)
{
    using Idx = typename std::conditional<I32, unsigned, size_t>::type;
    const int icol = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = blockIdx.y;
    if (icol >= ncol) return;
    const Idx ncl = Idx(ncol) * Idx(nlay);
    const Idx cl = Idx(icol) + Idx(l) * Idx(ncol);
    Idx i = cl;
    float next = layer_abs[i];
    double acc = 0.0;
    for (int g = 0; g < ngpt; ++g) {
        const float v = next;
        if (g + 1 < ngpt) {
            i += ncl;
            next = layer_abs[i];
        }
        acc += double(v);
    }
    const double dp = fabs(double(plev[icol + size_t(l + 1) * ncol]) - double(plev[icol + size_t(l) * ncol]));
    hr[cl] = float(kG0OverCp * 86400.0 * acc / dp);
}

int hr_from_layer_abs(int ncol, int nlay, int ngpt, const float* layer_abs, const float* plev, float* hr,
                      void* stream)
{
    RB_CHECK_ARG(ncol > 0 && nlay > 0 && ngpt > 0, "heating_rate_from_layer_abs: ncol, nlay and ngpt must be > 0");
    RB_CHECK_ARG(layer_abs && plev && hr, "heating_rate_from_layer_abs: null array");
    const dim3 grid(ceil_div(ncol, 128), nlay);
    const auto kernel = hr_index32(ncol, nlay, ngpt) ? heating_rate_from_layer_abs_kernel<true>
                                                     : heating_rate_from_layer_abs_kernel<false>;
    kernel<<<grid, 128, 0, as_stream(stream)>>>(ncol, nlay, ngpt, layer_abs, plev, hr);
    RB_LAUNCH("heating_rate_from_layer_abs_kernel");
    return RRTMGP_B200_OK;
}

template <typename T>
int hr_lw_layers(int ncol, int nlay, int ngpt, int top_at_1, const T* tau, const T* lay, const T* inc, const T* dec,
                 const T* up, const T* dn, const T* plev, T* hr, void* stream)
{
    RB_CHECK_ARG(ncol > 0 && nlay > 0 && ngpt > 0, "heating_rate_lw_layers: ncol, nlay and ngpt must be > 0");
    RB_CHECK_ARG(tau && lay && inc && dec && up && dn && plev && hr, "heating_rate_lw_layers: null array");
    const dim3 grid(ceil_div(ncol, 128), nlay);
    const auto kernel = hr_index32(ncol, nlay, ngpt) ? heating_rate_lw_layers_kernel<T, true>
                                                     : heating_rate_lw_layers_kernel<T, false>;
    kernel<<<grid, 128, 0, as_stream(stream)>>>(ncol, nlay, ngpt, top_at_1, tau, lay, inc, dec, up, dn, plev, hr);
    RB_LAUNCH("heating_rate_lw_layers_kernel");
    return RRTMGP_B200_OK;
}

template <typename T>
int hr_sw_layers(int ncol, int nlay, int ngpt, int top_at_1, const T* tau, const T* ssa, const T* g, const T* mu0,
                 const T* up, const T* dn, const T* dir, const T* plev, T* hr, void* stream)
{
    RB_CHECK_ARG(ncol > 0 && nlay > 0 && ngpt > 0, "heating_rate_sw_layers: ncol, nlay and ngpt must be > 0");
    RB_CHECK_ARG(tau && ssa && g && mu0 && up && dn && dir && plev && hr, "heating_rate_sw_layers: null array");
    const dim3 grid(ceil_div(ncol, 128), nlay);
    const auto kernel = hr_index32(ncol, nlay, ngpt) ? heating_rate_sw_layers_kernel<T, true>
                                                     : heating_rate_sw_layers_kernel<T, false>;
    kernel<<<grid, 128, 0, as_stream(stream)>>>(ncol, nlay, ngpt, top_at_1, tau, ssa, g, mu0, up, dn, dir, plev, hr);
    RB_LAUNCH("heating_rate_sw_layers_kernel");
    return RRTMGP_B200_OK;
}

}  // namespace
}  // namespace rrtmgp_b200

using namespace rrtmgp_b200;

extern "C" {

int rrtmgp_b200_heating_rate_lw_layers_f32(int ncol, int nlay, int ngpt, int top_at_1, const float* tau,
        const float* lay_src, const float* lev_src_inc, const float* lev_src_dec, const float* gpt_flux_up,
        const float* gpt_flux_dn, const float* plev, float* heating_rate, void* s)
{ return hr_lw_layers<float>(ncol, nlay, ngpt, top_at_1, tau, lay_src, lev_src_inc, lev_src_dec, gpt_flux_up, gpt_flux_dn, plev, heating_rate, s); }
int rrtmgp_b200_heating_rate_lw_layers_f64(int ncol, int nlay, int ngpt, int top_at_1, const double* tau,
        const double* lay_src, const double* lev_src_inc, const double* lev_src_dec, const double* gpt_flux_up,
        const double* gpt_flux_dn, const double* plev, double* heating_rate, void* s)
{ return hr_lw_layers<double>(ncol, nlay, ngpt, top_at_1, tau, lay_src, lev_src_inc, lev_src_dec, gpt_flux_up, gpt_flux_dn, plev, heating_rate, s); }
int rrtmgp_b200_heating_rate_sw_layers_f32(int ncol, int nlay, int ngpt, int top_at_1, const float* tau,
        const float* ssa, const float* g, const float* mu0, const float* gpt_flux_up, const float* gpt_flux_dn,
        const float* gpt_flux_dir, const float* plev, float* heating_rate, void* s)
{ return hr_sw_layers<float>(ncol, nlay, ngpt, top_at_1, tau, ssa, g, mu0, gpt_flux_up, gpt_flux_dn, gpt_flux_dir, plev, heating_rate, s); }
int rrtmgp_b200_heating_rate_sw_layers_f64(int ncol, int nlay, int ngpt, int top_at_1, const double* tau,
        const double* ssa, const double* g, const double* mu0, const double* gpt_flux_up, const double* gpt_flux_dn,
        const double* gpt_flux_dir, const double* plev, double* heating_rate, void* s)
{ return hr_sw_layers<double>(ncol, nlay, ngpt, top_at_1, tau, ssa, g, mu0, gpt_flux_up, gpt_flux_dn, gpt_flux_dir, plev, heating_rate, s); }

int rrtmgp_b200_heating_rate_from_layer_abs_f32(int ncol, int nlay, int ngpt, const float* layer_abs,
        const float* plev, float* heating_rate, void* s)
{ return hr_from_layer_abs(ncol, nlay, ngpt, layer_abs, plev, heating_rate, s); }

}  // extern "C"
