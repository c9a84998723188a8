// Shortwave radiative transfer on the GPU: Rte_sw_gpu::rte_sw of the reference
// (include/Rte_sw.h:61-81): two-stream coefficients and adding, mu0 (ncol), incident direct
// flux (ncol, ngpt), albedos per band (nband, ncol), optional incident diffuse flux (an empty
// array means none).  Outputs up, dn (diffuse + direct) and direct g-point fluxes
// (ncol, nlay+1, ngpt).  The solver's scratch (only columns deeper than the on-chip solver's
// limit need one) is kept by this object and grown on demand.
#ifndef RRTMGP_B200_CPP_RTE_SW_H
#define RRTMGP_B200_CPP_RTE_SW_H

#include <limits>
#include <memory>
#include <stdexcept>

#include "Optical_props.h"

class Rte_sw_gpu
{
  public:
    void rte_sw(const std::unique_ptr<Optical_props_arry_gpu>& optical_props, const Bool top_at_1,
                const Array_gpu<Float, 1>& mu0, const Array_gpu<Float, 2>& inc_flux_dir,
                const Array_gpu<Float, 2>& sfc_alb_dir, const Array_gpu<Float, 2>& sfc_alb_dif,
                const Array_gpu<Float, 2>& inc_flux_dif, Array_gpu<Float, 3>& gpt_flux_up,
                Array_gpu<Float, 3>& gpt_flux_dn, Array_gpu<Float, 3>& gpt_flux_dir)
    {
        const int ncol = optical_props->get_ncol(), nlay = optical_props->get_nlay();
        const int ngpt = optical_props->get_ngpt();
        const size_t need = rrtmgp_b200_rte_sw_workspace_bytes(ncol, nlay, ngpt, sizeof(Float) == 8);
        const size_t words = (need + sizeof(double) - 1) / sizeof(double);
        if (words > size_t(std::numeric_limits<int>::max()))
            throw std::runtime_error("Rte_sw_gpu: solver workspace too large; split the columns");
        if (size_t(ws_.size()) < words) ws_ = Array_gpu<double, 1>({int(words)});
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::rte_sw(
            optical_props->bands_handle(), ncol, nlay, int(top_at_1 != 0), optical_props->get_tau().ptr(),
            optical_props->get_ssa().ptr(), optical_props->get_g().ptr(), mu0.ptr(), inc_flux_dir.ptr(),
            sfc_alb_dir.ptr(), sfc_alb_dif.ptr(), inc_flux_dif.size() ? inc_flux_dif.ptr() : nullptr,
            gpt_flux_up.ptr(), gpt_flux_dn.ptr(), gpt_flux_dir.ptr(), words ? ws_.ptr() : nullptr,
            sizeof(double) * size_t(ws_.size())));
    }

  private:
    Array_gpu<double, 1> ws_;
};

#endif
