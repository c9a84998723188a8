// Glue between the C++ class API and the C ABI (rrtmgp_b200.h): status codes become
// exceptions (the reference throws std::runtime_error from its classes), Float selects the
// _f32/_f64 entry points, and all launches go to one stream (the default stream unless
// set_stream was called), as the reference issues every launch on the default stream.
#ifndef RRTMGP_B200_CPP_GLUE_H
#define RRTMGP_B200_CPP_GLUE_H

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "../rrtmgp_b200.h"
#include "types.h"

namespace rrtmgp_b200_cpp {

inline cudaStream_t& stream_ref()
{
    static thread_local cudaStream_t s = nullptr;
    return s;
}

// Stream used by every call of the class API made from this host thread.
inline void set_stream(cudaStream_t s) { stream_ref() = s; }
inline void* stream() { return static_cast<void*>(stream_ref()); }

inline void check(int status)
{
    if (status == RRTMGP_B200_OK) return;
    const std::string msg = rrtmgp_b200_last_error();
    if (status == RRTMGP_B200_ERR_RANGE) throw std::range_error(msg);
    throw std::runtime_error(msg);
}

inline void check_cuda(cudaError_t e, const char* where)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
}

// Precision dispatch: one overload pair (float -> _f32, double -> _f64) per C-ABI entry.
inline int get_col_dry(int ncol, int nlay, const float* h2o, const float* plev, float* cd)
{ return rrtmgp_b200_get_col_dry_f32(ncol, nlay, h2o, plev, cd, stream()); }
inline int get_col_dry(int ncol, int nlay, const double* h2o, const double* plev, double* cd)
{ return rrtmgp_b200_get_col_dry_f64(ncol, nlay, h2o, plev, cd, stream()); }

inline int gas_optics_lw(rrtmgp_b200_kdist k, int ncol, int nlay, const float* play, const float* plev,
                         const float* tlay, const float* tsfc, const float* tlev, const float* col_dry,
                         const rrtmgp_b200_gas_conc* g, int ng, float* tau, float* lay, float* inc, float* dec,
                         float* sfc, float* jac)
{ return rrtmgp_b200_gas_optics_lw_f32(k, ncol, nlay, play, plev, tlay, tsfc, tlev, col_dry, g, ng, tau, lay, inc,
                                       dec, sfc, jac, stream()); }
inline int gas_optics_lw(rrtmgp_b200_kdist k, int ncol, int nlay, const double* play, const double* plev,
                         const double* tlay, const double* tsfc, const double* tlev, const double* col_dry,
                         const rrtmgp_b200_gas_conc* g, int ng, double* tau, double* lay, double* inc, double* dec,
                         double* sfc, double* jac)
{ return rrtmgp_b200_gas_optics_lw_f64(k, ncol, nlay, play, plev, tlay, tsfc, tlev, col_dry, g, ng, tau, lay, inc,
                                       dec, sfc, jac, stream()); }

inline int gas_optics_sw(rrtmgp_b200_kdist k, int ncol, int nlay, const float* play, const float* plev,
                         const float* tlay, const float* col_dry, const rrtmgp_b200_gas_conc* g, int ng, float* tau,
                         float* ssa, float* gg, float* toa)
{ return rrtmgp_b200_gas_optics_sw_f32(k, ncol, nlay, play, plev, tlay, col_dry, g, ng, tau, ssa, gg, toa, stream()); }
inline int gas_optics_sw(rrtmgp_b200_kdist k, int ncol, int nlay, const double* play, const double* plev,
                         const double* tlay, const double* col_dry, const rrtmgp_b200_gas_conc* g, int ng,
                         double* tau, double* ssa, double* gg, double* toa)
{ return rrtmgp_b200_gas_optics_sw_f64(k, ncol, nlay, play, plev, tlay, col_dry, g, ng, tau, ssa, gg, toa, stream()); }

inline int cloud_1scl(rrtmgp_b200_cloud c, int ncol, int nlay, const float* lwp, const float* iwp, const float* rl,
                      const float* ri, float* tau)
{ return rrtmgp_b200_cloud_optics_1scl_f32(c, ncol, nlay, lwp, iwp, rl, ri, tau, stream()); }
inline int cloud_1scl(rrtmgp_b200_cloud c, int ncol, int nlay, const double* lwp, const double* iwp, const double* rl,
                      const double* ri, double* tau)
{ return rrtmgp_b200_cloud_optics_1scl_f64(c, ncol, nlay, lwp, iwp, rl, ri, tau, stream()); }
inline int aerosol_optics(rrtmgp_b200_aerosol a, int ncol, int nlay, const rrtmgp_b200_gas_conc* aer, int naer,
                          const float* rh, const float* plev, float* tau, float* ssa, float* g)
{
    return rrtmgp_b200_aerosol_optics_f32(a, ncol, nlay, aer, naer, rh, plev, tau, ssa, g, stream());
}
inline int aerosol_optics(rrtmgp_b200_aerosol a, int ncol, int nlay, const rrtmgp_b200_gas_conc* aer, int naer,
                          const double* rh, const double* plev, double* tau, double* ssa, double* g)
{
    return rrtmgp_b200_aerosol_optics_f64(a, ncol, nlay, aer, naer, rh, plev, tau, ssa, g, stream());
}
inline int cloud_2str(rrtmgp_b200_cloud c, int ncol, int nlay, const float* lwp, const float* iwp, const float* rl,
                      const float* ri, float* tau, float* ssa, float* g)
{ return rrtmgp_b200_cloud_optics_2str_f32(c, ncol, nlay, lwp, iwp, rl, ri, tau, ssa, g, stream()); }
inline int cloud_2str(rrtmgp_b200_cloud c, int ncol, int nlay, const double* lwp, const double* iwp, const double* rl,
                      const double* ri, double* tau, double* ssa, double* g)
{ return rrtmgp_b200_cloud_optics_2str_f64(c, ncol, nlay, lwp, iwp, rl, ri, tau, ssa, g, stream()); }

inline int delta_scale(int ncol, int nlay, int ngpt, float* t, float* s, float* g)
{ return rrtmgp_b200_delta_scale_2str_f32(ncol, nlay, ngpt, t, s, g, stream()); }
inline int delta_scale(int ncol, int nlay, int ngpt, double* t, double* s, double* g)
{ return rrtmgp_b200_delta_scale_2str_f64(ncol, nlay, ngpt, t, s, g, stream()); }

inline int add_to_1scl(rrtmgp_b200_bands b, int ncol, int nlay, float* t, const float* ti, int ngi)
{ return rrtmgp_b200_add_to_1scl_f32(b, ncol, nlay, t, ti, ngi, stream()); }
inline int add_to_1scl(rrtmgp_b200_bands b, int ncol, int nlay, double* t, const double* ti, int ngi)
{ return rrtmgp_b200_add_to_1scl_f64(b, ncol, nlay, t, ti, ngi, stream()); }
inline int add_to_2str(rrtmgp_b200_bands b, int ncol, int nlay, float* t, float* s, float* g, const float* ti,
                       const float* si, const float* gi, int ngi)
{ return rrtmgp_b200_add_to_2str_f32(b, ncol, nlay, t, s, g, ti, si, gi, ngi, stream()); }
inline int add_to_2str(rrtmgp_b200_bands b, int ncol, int nlay, double* t, double* s, double* g, const double* ti,
                       const double* si, const double* gi, int ngi)
{ return rrtmgp_b200_add_to_2str_f64(b, ncol, nlay, t, s, g, ti, si, gi, ngi, stream()); }

inline int rte_lw(rrtmgp_b200_bands b, int ncol, int nlay, int top, const float* tau, const float* lay,
                  const float* inc, const float* dec, const float* sfc, const float* emis, const float* incf, int nmu,
                  float* up, float* dn)
{ return rrtmgp_b200_rte_lw_f32(b, ncol, nlay, top, tau, lay, inc, dec, sfc, emis, incf, nmu, up, dn, stream()); }
inline int rte_lw(rrtmgp_b200_bands b, int ncol, int nlay, int top, const double* tau, const double* lay,
                  const double* inc, const double* dec, const double* sfc, const double* emis, const double* incf,
                  int nmu, double* up, double* dn)
{ return rrtmgp_b200_rte_lw_f64(b, ncol, nlay, top, tau, lay, inc, dec, sfc, emis, incf, nmu, up, dn, stream()); }
inline int rte_lw_jac(rrtmgp_b200_bands b, int ncol, int nlay, int top, const float* tau, const float* lay,
                      const float* inc, const float* dec, const float* sfc, const float* sfc_jac, const float* emis,
                      const float* incf, int nmu, float* up, float* dn, float* up_jac)
{ return rrtmgp_b200_rte_lw_jac_f32(b, ncol, nlay, top, tau, lay, inc, dec, sfc, sfc_jac, emis, incf, nmu, up, dn, up_jac, stream()); }
inline int rte_lw_jac(rrtmgp_b200_bands b, int ncol, int nlay, int top, const double* tau, const double* lay,
                      const double* inc, const double* dec, const double* sfc, const double* sfc_jac,
                      const double* emis, const double* incf, int nmu, double* up, double* dn, double* up_jac)
{ return rrtmgp_b200_rte_lw_jac_f64(b, ncol, nlay, top, tau, lay, inc, dec, sfc, sfc_jac, emis, incf, nmu, up, dn, up_jac, stream()); }

inline int rte_sw(rrtmgp_b200_bands b, int ncol, int nlay, int top, const float* tau, const float* ssa,
                  const float* g, const float* mu0, const float* idir, const float* ad, const float* af,
                  const float* idif, float* up, float* dn, float* dir, void* ws, size_t wsb)
{ return rrtmgp_b200_rte_sw_f32(b, ncol, nlay, top, tau, ssa, g, mu0, idir, ad, af, idif, up, dn, dir, ws, wsb,
                                stream()); }
inline int rte_sw(rrtmgp_b200_bands b, int ncol, int nlay, int top, const double* tau, const double* ssa,
                  const double* g, const double* mu0, const double* idir, const double* ad, const double* af,
                  const double* idif, double* up, double* dn, double* dir, void* ws, size_t wsb)
{ return rrtmgp_b200_rte_sw_f64(b, ncol, nlay, top, tau, ssa, g, mu0, idir, ad, af, idif, up, dn, dir, ws, wsb,
                                stream()); }

inline int broadband(int ncol, int nlev, int ngpt, const float* up, const float* dn, const float* dir, float* fu,
                     float* fd, float* fdir, float* fn)
{ return rrtmgp_b200_fluxes_broadband_f32(ncol, nlev, ngpt, up, dn, dir, fu, fd, fdir, fn, stream()); }
inline int broadband(int ncol, int nlev, int ngpt, const double* up, const double* dn, const double* dir, double* fu,
                     double* fd, double* fdir, double* fn)
{ return rrtmgp_b200_fluxes_broadband_f64(ncol, nlev, ngpt, up, dn, dir, fu, fd, fdir, fn, stream()); }

inline int byband(rrtmgp_b200_bands b, int ncol, int nlev, const float* up, const float* dn, const float* dir,
                  float* bu, float* bd, float* bdir, float* bn)
{ return rrtmgp_b200_fluxes_byband_f32(b, ncol, nlev, up, dn, dir, bu, bd, bdir, bn, stream()); }
inline int byband(rrtmgp_b200_bands b, int ncol, int nlev, const double* up, const double* dn, const double* dir,
                  double* bu, double* bd, double* bdir, double* bn)
{ return rrtmgp_b200_fluxes_byband_f64(b, ncol, nlev, up, dn, dir, bu, bd, bdir, bn, stream()); }

}  // namespace rrtmgp_b200_cpp

#endif
