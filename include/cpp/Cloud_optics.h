// Cloud optics from the liquid/ice lookup tables on the GPU: Cloud_optics_gpu of the
// reference (include/Cloud_optics.h:80-131).  One value per band (ncol, nlay, nband); ice
// roughness index 2 as in the reference.  LUT arrays as load_and_init_cloud_optics
// (src_test/Radiation_solver.cpp:287-330) builds them: liquid {nsize_liq, nband}, ice
// {nsize_ice, nband, nrghice}.
#ifndef RRTMGP_B200_CPP_CLOUD_OPTICS_H
#define RRTMGP_B200_CPP_CLOUD_OPTICS_H

#include <memory>
#include <vector>

#include "Optical_props.h"

class Cloud_optics_gpu : public Optical_props_gpu
{
  public:
    Cloud_optics_gpu(const Array<Float, 2>& band_lims_wvn, const Float radliq_lwr, const Float radliq_upr,
                     const Float radliq_fac, const Float radice_lwr, const Float radice_upr, const Float radice_fac,
                     const Array<Float, 2>& lut_extliq, const Array<Float, 2>& lut_ssaliq,
                     const Array<Float, 2>& lut_asyliq, const Array<Float, 3>& lut_extice,
                     const Array<Float, 3>& lut_ssaice, const Array<Float, 3>& lut_asyice)
        : Optical_props_gpu(band_lims_wvn)
    {
        auto dbl = [](const std::vector<Float>& v) { return std::vector<double>(v.begin(), v.end()); };
        const std::vector<double> wvn = dbl(band_lims_wvn.v()), el = dbl(lut_extliq.v()), sl = dbl(lut_ssaliq.v()),
                                  al = dbl(lut_asyliq.v()), ei = dbl(lut_extice.v()), si = dbl(lut_ssaice.v()),
                                  ai = dbl(lut_asyice.v());
        rrtmgp_b200_cloud_tables t{};
        t.nband = band_lims_wvn.dim(2);
        t.nsize_liq = lut_extliq.dim(1);
        t.nsize_ice = lut_extice.dim(1);
        t.nrghice = lut_extice.dim(3);
        t.band_lims_wvn = wvn.data();
        t.radliq_lwr = radliq_lwr;
        t.radliq_upr = radliq_upr;
        t.radliq_fac = radliq_fac;
        t.radice_lwr = radice_lwr;
        t.radice_upr = radice_upr;
        t.radice_fac = radice_fac;
        t.lut_extliq = el.data();
        t.lut_ssaliq = sl.data();
        t.lut_asyliq = al.data();
        t.lut_extice = ei.data();
        t.lut_ssaice = si.data();
        t.lut_asyice = ai.data();
        rrtmgp_b200_cloud h = nullptr;
        rrtmgp_b200_cpp::check(rrtmgp_b200_cloud_create(&t, &h));
        c_ = std::shared_ptr<rrtmgp_b200_cloud_t>(h, [](rrtmgp_b200_cloud p) { rrtmgp_b200_cloud_destroy(p); });
    }

    // Absorption optical depth only (longwave).
    void cloud_optics(const Array_gpu<Float, 2>& clwp, const Array_gpu<Float, 2>& ciwp,
                      const Array_gpu<Float, 2>& reliq, const Array_gpu<Float, 2>& reice,
                      Optical_props_1scl_gpu& optical_props)
    {
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::cloud_1scl(c_.get(), clwp.dim(1), clwp.dim(2), clwp.ptr(), ciwp.ptr(),
                                                           reliq.ptr(), reice.ptr(), optical_props.get_tau().ptr()));
    }

    // tau, ssa, g (shortwave).
    void cloud_optics(const Array_gpu<Float, 2>& clwp, const Array_gpu<Float, 2>& ciwp,
                      const Array_gpu<Float, 2>& reliq, const Array_gpu<Float, 2>& reice,
                      Optical_props_2str_gpu& optical_props)
    {
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::cloud_2str(c_.get(), clwp.dim(1), clwp.dim(2), clwp.ptr(), ciwp.ptr(),
                                                           reliq.ptr(), reice.ptr(), optical_props.get_tau().ptr(),
                                                           optical_props.get_ssa().ptr(),
                                                           optical_props.get_g().ptr()));
    }

    rrtmgp_b200_cloud cloud_handle() const { return c_.get(); }

  private:
    std::shared_ptr<rrtmgp_b200_cloud_t> c_;
};

#endif
