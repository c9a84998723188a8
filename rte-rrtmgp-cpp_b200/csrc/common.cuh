// Internal definitions shared by the rrtmgp_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "rrtmgp_b200.h"

namespace rrtmgp_b200 {

// ---------------------------------------------------------------------------------------
// Error reporting: every C-ABI entry point returns a status and stores a message here.
// ---------------------------------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_status(cudaError_t err, const char* where);

#define RB_CHECK_ARG(cond, msg) \
    do { if (!(cond)) return ::rrtmgp_b200::fail(RRTMGP_B200_ERR_ARG, (msg)); } while (0)
#define RB_CUDA(call, where) \
    do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return ::rrtmgp_b200::cuda_status(e_, (where)); } while (0)
#define RB_LAUNCH(where) \
    do { cudaError_t e_ = cudaGetLastError(); if (e_ != cudaSuccess) return ::rrtmgp_b200::cuda_status(e_, (where)); } while (0)

inline int ceil_div(long a, long b) { return int((a + b - 1) / b); }

// Per-device one-time set-up (cudaFuncSetAttribute and the like act on the current device's
// context only).  run(f) calls f once for every device that is current when run is called,
// from any host thread; a failed f is retried on the next call.
class PerDeviceOnce {
public:
    template <class F>
    int run(F&& f, const char* where)
    {
        int dev = 0;
        RB_CUDA(cudaGetDevice(&dev), where);
        if (dev < 0 || dev >= 64) return fail(RRTMGP_B200_ERR_UNSUPPORTED, std::string(where) + ": device ordinal >= 64");
        std::lock_guard<std::mutex> lock(mu_);
        if ((done_ >> dev) & 1ull) return RRTMGP_B200_OK;
        RB_CUDA(f(), where);
        done_ |= 1ull << dev;
        return RRTMGP_B200_OK;
    }

private:
    std::mutex mu_;
    unsigned long long done_ = 0;
};

// Handles hold device pointers of the device they were created on: a call made while another
// device is current is refused.
inline int check_device(int handle_device, const char* where)
{
    int dev = 0;
    RB_CUDA(cudaGetDevice(&dev), where);
    if (dev != handle_device)
        return fail(RRTMGP_B200_ERR_ARG, std::string(where) + ": the handle's tables live on device " +
                                             std::to_string(handle_device) + ", the current device is " +
                                             std::to_string(dev));
    return RRTMGP_B200_OK;
}

constexpr int kMaxGases = 24;          // gases in one k-distribution after reduction
constexpr int kMaxBandGpt = 32;        // g-points per band handled in registers/shared mem
constexpr int kMaxBands = 64;

// ---------------------------------------------------------------------------------------
// Device-resident k-distribution in one precision.  All tables are g-point fastest so that
// the g-points of a band at one (T, p, eta) corner are contiguous.
// ---------------------------------------------------------------------------------------
template <typename T>
struct KdistView {
    int ngas, nband, ngpt, ntemp, npres, neta, nflav, nplanck;
    int idx_h2o;                    // 1-based index into col_gas (0 = dry air)
    int has_rayleigh, is_lw;
    T press_ref_log0, press_ref_log_delta, press_ref_trop_log;
    T temp_ref_min, temp_ref_delta, totplnk_delta;
    const T* temp_ref;              // [ntemp]
    const T* vmr_ref;               // [ntemp][ngas+1][2]
    const int* flavor;              // [nflav][2]   gas indices (0 = dry air)
    const int* band_flav;           // [nband][2]   0-based flavor per band and atmosphere
    const int* band_lims;           // [nband][2]   0-based [start, end)
    const int* gpt2band;            // [ngpt]       0-based
    const T* kmajor;                // [ntemp][npres+1][neta][ngpt]
    const T* planck_frac;           // [ntemp][npres+1][neta][ngpt]
    const T* totplnk;               // [nband][nplanck]
    const T* krayl;                 // [2][ntemp][neta][ngpt]
    const T* solar_source;          // [ngpt]
    // Minor absorbers, per atmosphere a = 0 (lower, tropo) / 1 (upper).
    int nminor[2];
    int ncontrib[2];
    const int* minor_gstart[2];     // [nminor]   0-based
    const int* minor_gend[2];       // [nminor]   exclusive
    const int* minor_kstart[2];     // [nminor]   0-based contributor offset
    const int* minor_flav[2];       // [nminor]   0-based flavor (of g-point gstart)
    const int* minor_gas[2];        // [nminor]   col_gas index
    const int* minor_sgas[2];       // [nminor]   col_gas index of scaling gas, <= 0 none
    const int* minor_flags[2];      // [nminor]   bit0 scales_with_density, bit1 complement
    const int* band_minor_begin[2]; // [nband+1]  CSR into band_minor_list
    const int* band_minor_list[2];  // intervals overlapping each band
    const T* kminor[2];             // [ntemp][neta][ncontrib]
    int minor_in_band;              // every interval lies inside one band
    // Fused-kernel metadata: g-points are processed in groups of 32 (one per lane).
    int ngroups;                    // ceil(ngpt / 32)
    int max_group_bands;            // most bands touched by one group
    int max_band_minor;             // most minor intervals in one (band, atmosphere)
    const int* group_band0;         // [ngroups] first band of each group
    // Corner-packed copies for the fused FP32 kernels (NULL in the FP64 view):
    //   kmaj4/pfrac4 [t][p][eta][g], p < npres, eta < neta-1: (k(e,p), k(e+1,p), k(e,p+1), k(e+1,p+1))
    //   kmin2[a]     [t][eta][c], eta < neta-1: (k(e), k(e+1))
    //   krayl2       [a][t][eta][g], eta < neta-1: (k(e), k(e+1))
    //   minor_g[a]   [g]: x = number of intervals covering g, y/z/w = the first three codes
    //                (c << kScalBits) | sid, c = contributor, sid = scaling kind of the
    //                interval (below); unused slots repeat y (0 when no interval covers g).
    //   minor_gx[a]  [g][minor_gx_stride]: codes 4, 5, ... of g (NULL when no g-point has
    //                more than three intervals).
    const float4* kmaj4;
    const float4* pfrac4;
    const float2* kmin2[2];
    const float2* krayl2;
    const int4* minor_g[2];
    const int* minor_gx[2];
    int minor_gx_stride;
    int max_minor_per_g;            // most intervals covering one g-point
    // Scaling kinds: intervals whose scaling (gas_optical_depths_minor_kernel,
    // gas_optics_rrtmgp_kernels.cu:396-417) is the same function of the layer -- same minor
    // gas, and with density scaling the same scaling gas and complement flag -- share one
    // kind, so the fused kernels evaluate each kind once per layer instead of once per
    // (layer, interval).  scal_gas/sgas/flags [a][sid] as minor_gas/sgas/flags.
    int nscal[2];
    int max_nscal;                  // max(nscal[0], nscal[1], 1)
    const int* scal_gas[2];
    const int* scal_sgas[2];
    const int* scal_flags[2];
};

constexpr int kScalBits = 6;                    // bits of a scaling kind in a minor code
constexpr int kMaxScal = 1 << kScalBits;        // scaling kinds per atmosphere (fused kernels)

}  // namespace rrtmgp_b200

// Opaque handle structs (C ABI).
struct rrtmgp_b200_bands_t {
    int nband = 0, ngpt = 0;
    std::vector<int> band_lims_host;  // (nband, 2) 1-based
    int* d_band_lims = nullptr;       // [nband][2] 0-based [start, end)
    int* d_gpt2band = nullptr;        // [ngpt] 0-based
    bool owned_by_parent = false;
};

struct rrtmgp_b200_kdist_t {
    rrtmgp_b200_kdist_info info{};
    std::vector<std::string> gas_names;  // reduced, trimmed
    rrtmgp_b200_bands_t bands;
    rrtmgp_b200::KdistView<float> v32{};
    rrtmgp_b200::KdistView<double> v64{};
    std::vector<void*> allocations;
    std::vector<double> solar_quiet, solar_fac, solar_spot, solar_source;
    float* d_solar32 = nullptr;
    double* d_solar64 = nullptr;
    int* d_flags = nullptr;   // range-check result word
    int device = 0;
};

struct rrtmgp_b200_cloud_t {
    int nband = 0, nsize_liq = 0, nsize_ice = 0;
    double radliq_lwr = 0, radice_lwr = 0, liq_step = 0, ice_step = 0;
    float* lut32 = nullptr;   // [6][nband][nsize]: extliq, ssaliq, asyliq (nsize_liq) then ice
    double* lut64 = nullptr;
    rrtmgp_b200_bands_t bands;  // one g-point per band
};

namespace rrtmgp_b200 {
template <typename T> const KdistView<T>& view(const rrtmgp_b200_kdist_t* k);
template <> inline const KdistView<float>& view<float>(const rrtmgp_b200_kdist_t* k) { return k->v32; }
template <> inline const KdistView<double>& view<double>(const rrtmgp_b200_kdist_t* k) { return k->v64; }

template <typename T> const T* cloud_lut(const rrtmgp_b200_cloud_t* c);
template <> inline const float* cloud_lut<float>(const rrtmgp_b200_cloud_t* c) { return c->lut32; }
template <> inline const double* cloud_lut<double>(const rrtmgp_b200_cloud_t* c) { return c->lut64; }

// Gas concentration descriptors passed to kernels by value.
template <typename T>
struct GasSet {
    const T* vmr[kMaxGases];   // indexed by reduced gas (0-based)
    int mode[kMaxGases];       // 0 scalar, 1 profile (per layer), 2 field (ncol, nlay)
};

template <typename T>
int make_gas_set(const rrtmgp_b200_kdist_t* k, int ncol, int nlay,
                 const rrtmgp_b200_gas_conc* gases, int ngases, GasSet<T>& out);

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace rrtmgp_b200
