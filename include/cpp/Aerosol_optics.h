// Aerosol optics from the band look-up tables on the GPU: Aerosol_optics_gpu of the
// reference (include/Aerosol_optics.h:64-86, src_cuda/Aerosol_optics.cu:188-279).  Tables as
// load_and_init_aerosol_optics (src_test/Radiation_solver.cu:366-401) builds them: hydrophobic
// {nband, nphobic}, hydrophilic {nband, nhum, nphilic}, rh_upper {nhum}.  The species are the
// Aerosol_concs_gpu (= Gas_concs_gpu) entries aermr01 .. aermr11.
#ifndef RRTMGP_B200_CPP_AEROSOL_OPTICS_H
#define RRTMGP_B200_CPP_AEROSOL_OPTICS_H

#include <memory>
#include <vector>

#include "Gas_concs.h"
#include "Optical_props.h"

using Aerosol_concs = Gas_concs;
using Aerosol_concs_gpu = Gas_concs_gpu;

class Aerosol_optics_gpu : public Optical_props_gpu
{
  public:
    Aerosol_optics_gpu(const Array<Float, 2>& band_lims_wvn, const Array<Float, 1>& rh_upper,
                       const Array<Float, 2>& mext_phobic, const Array<Float, 2>& ssa_phobic,
                       const Array<Float, 2>& g_phobic, const Array<Float, 3>& mext_philic,
                       const Array<Float, 3>& ssa_philic, const Array<Float, 3>& g_philic)
        : Optical_props_gpu(band_lims_wvn)
    {
        auto dbl = [](const std::vector<Float>& v) { return std::vector<double>(v.begin(), v.end()); };
        const std::vector<double> ru = dbl(rh_upper.v()), mp = dbl(mext_phobic.v()), sp = dbl(ssa_phobic.v()),
                                  gp = dbl(g_phobic.v()), ml = dbl(mext_philic.v()), sl = dbl(ssa_philic.v()),
                                  gl = dbl(g_philic.v());
        rrtmgp_b200_aerosol_tables t{};
        t.nband = mext_phobic.dim(1);
        t.nphobic = mext_phobic.dim(2);
        t.nhum = mext_philic.dim(2);
        t.nphilic = mext_philic.dim(3);
        t.rh_upper = ru.data();
        t.mext_phobic = mp.data();
        t.ssa_phobic = sp.data();
        t.g_phobic = gp.data();
        t.mext_philic = ml.data();
        t.ssa_philic = sl.data();
        t.g_philic = gl.data();
        rrtmgp_b200_aerosol h = nullptr;
        rrtmgp_b200_cpp::check(rrtmgp_b200_aerosol_create(&t, &h));
        a_ = std::shared_ptr<rrtmgp_b200_aerosol_t>(h, [](rrtmgp_b200_aerosol p) { rrtmgp_b200_aerosol_destroy(p); });
    }

    // tau, ssa, g (ncol, nlay, nband) of the aerosol mixture; rh (ncol, nlay), plev (ncol, nlay+1).
    void aerosol_optics(Aerosol_concs_gpu& aerosol_concs, const Array_gpu<Float, 2>& rh,
                        const Array_gpu<Float, 2>& plev, Optical_props_2str_gpu& optical_props)
    {
        const std::vector<rrtmgp_b200_gas_conc> d = aerosol_concs.descriptors();
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::aerosol_optics(
            a_.get(), rh.dim(1), rh.dim(2), d.data(), int(d.size()), rh.ptr(), plev.ptr(),
            optical_props.get_tau().ptr(), optical_props.get_ssa().ptr(), optical_props.get_g().ptr()));
    }

    rrtmgp_b200_aerosol aerosol_handle() const { return a_.get(); }

  private:
    std::shared_ptr<rrtmgp_b200_aerosol_t> a_;
};

#endif
