// Longwave radiative transfer on the GPU: Rte_lw_gpu::rte_lw of the reference
// (include/Rte_lw.h:61-80): no-scattering solver with n_gauss_angles Gauss quadrature angles
// (1..4), surface emissivity per band (nband, ncol), optional incident flux (ncol, ngpt; an
// empty array means none).  Outputs g-point fluxes (ncol, nlay+1, ngpt).
#ifndef RRTMGP_B200_CPP_RTE_LW_H
#define RRTMGP_B200_CPP_RTE_LW_H

#include <memory>

#include "Source_functions.h"

class Rte_lw_gpu
{
  public:
    void rte_lw(const std::unique_ptr<Optical_props_arry_gpu>& optical_props, const Bool top_at_1,
                const Source_func_lw_gpu& sources, const Array_gpu<Float, 2>& sfc_emis,
                const Array_gpu<Float, 2>& inc_flux, Array_gpu<Float, 3>& gpt_flux_up, Array_gpu<Float, 3>& gpt_flux_dn,
                const int n_gauss_angles)
    {
        const int ncol = optical_props->get_ncol(), nlay = optical_props->get_nlay();
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::rte_lw(
            optical_props->bands_handle(), ncol, nlay, int(top_at_1 != 0), optical_props->get_tau().ptr(),
            sources.get_lay_source().ptr(), sources.get_lev_source_inc().ptr(), sources.get_lev_source_dec().ptr(),
            sources.get_sfc_source().ptr(), sfc_emis.ptr(), inc_flux.size() ? inc_flux.ptr() : nullptr,
            n_gauss_angles, gpt_flux_up.ptr(), gpt_flux_dn.ptr()));
    }

    // The same solve plus the surface-temperature Jacobian gpt_flux_up_jac (ncol, nlay+1,
    // ngpt) from the sources' sfc_source_jac: the output the reference computes in
    // lw_solver_noscat when do_jacobians is set (src_cuda/Rte_lw.cu:125-148 keeps it off).
    void rte_lw(const std::unique_ptr<Optical_props_arry_gpu>& optical_props, const Bool top_at_1,
                const Source_func_lw_gpu& sources, const Array_gpu<Float, 2>& sfc_emis,
                const Array_gpu<Float, 2>& inc_flux, Array_gpu<Float, 3>& gpt_flux_up, Array_gpu<Float, 3>& gpt_flux_dn,
                Array_gpu<Float, 3>& gpt_flux_up_jac, const int n_gauss_angles)
    {
        const int ncol = optical_props->get_ncol(), nlay = optical_props->get_nlay();
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::rte_lw_jac(
            optical_props->bands_handle(), ncol, nlay, int(top_at_1 != 0), optical_props->get_tau().ptr(),
            sources.get_lay_source().ptr(), sources.get_lev_source_inc().ptr(), sources.get_lev_source_dec().ptr(),
            sources.get_sfc_source().ptr(), sources.get_sfc_source_jac().ptr(), sfc_emis.ptr(),
            inc_flux.size() ? inc_flux.ptr() : nullptr, n_gauss_angles, gpt_flux_up.ptr(), gpt_flux_dn.ptr(),
            gpt_flux_up_jac.ptr()));
    }
};

#endif
