// RRTMGP gas optics on the GPU with the reference's class interface
// (include/Gas_optics.h:87-127, include/Gas_optics_rrtmgp.h:289-551): the longwave and
// shortwave constructors take the host tables exactly as load_and_init_gas_optics
// (src_test/Radiation_solver.cpp:70-284) builds them from the netCDF file; gas_optics()
// fills optical properties and sources (LW) or toa_src (SW).  The work is done by the C ABI
// (rrtmgp_b200_kdist_create, rrtmgp_b200_gas_optics_lw/sw_*), which re-lays the tables out
// on the device once, in the constructor.
#ifndef RRTMGP_B200_CPP_GAS_OPTICS_RRTMGP_H
#define RRTMGP_B200_CPP_GAS_OPTICS_RRTMGP_H

#include <memory>
#include <string>
#include <vector>

#include "Gas_concs.h"
#include "Optical_props.h"
#include "Source_functions.h"

class Gas_optics_gpu : public Optical_props_gpu
{
  public:
    Gas_optics_gpu(const Array<Float, 2>& band_lims_wvn, const Array<int, 2>& band_lims_gpt)
        : Optical_props_gpu(band_lims_wvn, band_lims_gpt)
    {}
    virtual ~Gas_optics_gpu() {}

    virtual bool source_is_internal() const = 0;
    virtual bool source_is_external() const = 0;
    virtual Float get_press_ref_min() const = 0;
    virtual Float get_press_ref_max() const = 0;
    virtual Float get_temp_min() const = 0;
    virtual Float get_temp_max() const = 0;

    virtual void gas_optics(const Array_gpu<Float, 2>& play, const Array_gpu<Float, 2>& plev,
                            const Array_gpu<Float, 2>& tlay, const Array_gpu<Float, 1>& tsfc,
                            const Gas_concs_gpu& gas_desc, std::unique_ptr<Optical_props_arry_gpu>& optical_props,
                            Source_func_lw_gpu& sources, const Array_gpu<Float, 2>& col_dry,
                            const Array_gpu<Float, 2>& tlev) = 0;
    virtual void gas_optics(const Array_gpu<Float, 2>& play, const Array_gpu<Float, 2>& plev,
                            const Array_gpu<Float, 2>& tlay, const Gas_concs_gpu& gas_desc,
                            std::unique_ptr<Optical_props_arry_gpu>& optical_props, Array_gpu<Float, 2>& toa_src,
                            const Array_gpu<Float, 2>& col_dry) = 0;
};

namespace rrtmgp_b200_cpp {

// Owns double copies of the host tables and the C-ABI descriptor that points into them.
struct Kdist_table_copy {
    rrtmgp_b200_kdist_tables t{};
    std::vector<std::vector<double>> f;
    std::vector<std::vector<int>> i;
    std::vector<std::vector<std::string>> s;
    std::vector<std::vector<const char*>> sp;

    template <int N>
    const double* fl(const Array<Float, N>& a)
    {
        if (a.size() == 0) return nullptr;
        f.emplace_back(a.v().begin(), a.v().end());
        return f.back().data();
    }
    template <typename B, int N>
    const int* in(const Array<B, N>& a)
    {
        if (a.size() == 0) return nullptr;
        i.emplace_back(a.v().begin(), a.v().end());
        return i.back().data();
    }
    const char* const* str(const Array<std::string, 1>& a)
    {
        s.emplace_back(a.v().begin(), a.v().end());
        sp.emplace_back();
        for (const auto& x : s.back()) sp.back().push_back(x.c_str());
        return sp.back().data();
    }
    Kdist_table_copy()
    {
        f.reserve(32);
        i.reserve(32);
        s.reserve(16);
        sp.reserve(16);
    }
};

}  // namespace rrtmgp_b200_cpp

class Gas_optics_rrtmgp_gpu : public Gas_optics_gpu
{
  public:
    // Longwave variant.
    Gas_optics_rrtmgp_gpu(
        const Gas_concs_gpu& available_gases, const Array<std::string, 1>& gas_names,
        const Array<int, 3>& key_species, const Array<int, 2>& band2gpt, const Array<Float, 2>& band_lims_wavenum,
        const Array<Float, 1>& press_ref, const Float press_ref_trop, const Array<Float, 1>& temp_ref,
        const Float temp_ref_p, const Float temp_ref_t, const Array<Float, 3>& vmr_ref, const Array<Float, 4>& kmajor,
        const Array<Float, 3>& kminor_lower, const Array<Float, 3>& kminor_upper,
        const Array<std::string, 1>& gas_minor, const Array<std::string, 1>& identifier_minor,
        const Array<std::string, 1>& minor_gases_lower, const Array<std::string, 1>& minor_gases_upper,
        const Array<int, 2>& minor_limits_gpt_lower, const Array<int, 2>& minor_limits_gpt_upper,
        const Array<Bool, 1>& minor_scales_with_density_lower, const Array<Bool, 1>& minor_scales_with_density_upper,
        const Array<std::string, 1>& scaling_gas_lower, const Array<std::string, 1>& scaling_gas_upper,
        const Array<Bool, 1>& scale_by_complement_lower, const Array<Bool, 1>& scale_by_complement_upper,
        const Array<int, 1>& kminor_start_lower, const Array<int, 1>& kminor_start_upper,
        const Array<Float, 2>& totplnk, const Array<Float, 4>& planck_frac, const Array<Float, 3>& rayl_lower,
        const Array<Float, 3>& rayl_upper)
        : Gas_optics_gpu(band_lims_wavenum, band2gpt)
    {
        rrtmgp_b200_cpp::Kdist_table_copy c;
        common(c, gas_names, key_species, band2gpt, band_lims_wavenum, press_ref, press_ref_trop, temp_ref,
               temp_ref_p, temp_ref_t, vmr_ref, kmajor, kminor_lower, kminor_upper, gas_minor, identifier_minor,
               minor_gases_lower, minor_gases_upper, minor_limits_gpt_lower, minor_limits_gpt_upper,
               minor_scales_with_density_lower, minor_scales_with_density_upper, scaling_gas_lower,
               scaling_gas_upper, scale_by_complement_lower, scale_by_complement_upper, kminor_start_lower,
               kminor_start_upper, rayl_lower, rayl_upper);
        c.t.nplanck_temp = totplnk.dim(1);
        c.t.totplnk = c.fl(totplnk);
        c.t.planck_frac = c.fl(planck_frac);
        create(c, available_gases);
    }

    // Shortwave variant.
    Gas_optics_rrtmgp_gpu(
        const Gas_concs_gpu& available_gases, const Array<std::string, 1>& gas_names,
        const Array<int, 3>& key_species, const Array<int, 2>& band2gpt, const Array<Float, 2>& band_lims_wavenum,
        const Array<Float, 1>& press_ref, const Float press_ref_trop, const Array<Float, 1>& temp_ref,
        const Float temp_ref_p, const Float temp_ref_t, const Array<Float, 3>& vmr_ref, const Array<Float, 4>& kmajor,
        const Array<Float, 3>& kminor_lower, const Array<Float, 3>& kminor_upper,
        const Array<std::string, 1>& gas_minor, const Array<std::string, 1>& identifier_minor,
        const Array<std::string, 1>& minor_gases_lower, const Array<std::string, 1>& minor_gases_upper,
        const Array<int, 2>& minor_limits_gpt_lower, const Array<int, 2>& minor_limits_gpt_upper,
        const Array<Bool, 1>& minor_scales_with_density_lower, const Array<Bool, 1>& minor_scales_with_density_upper,
        const Array<std::string, 1>& scaling_gas_lower, const Array<std::string, 1>& scaling_gas_upper,
        const Array<Bool, 1>& scale_by_complement_lower, const Array<Bool, 1>& scale_by_complement_upper,
        const Array<int, 1>& kminor_start_lower, const Array<int, 1>& kminor_start_upper,
        const Array<Float, 1>& solar_src_quiet, const Array<Float, 1>& solar_src_facular,
        const Array<Float, 1>& solar_src_sunspot, const Float tsi_default, const Float mg_default,
        const Float sb_default, const Array<Float, 3>& rayl_lower, const Array<Float, 3>& rayl_upper)
        : Gas_optics_gpu(band_lims_wavenum, band2gpt)
    {
        rrtmgp_b200_cpp::Kdist_table_copy c;
        common(c, gas_names, key_species, band2gpt, band_lims_wavenum, press_ref, press_ref_trop, temp_ref,
               temp_ref_p, temp_ref_t, vmr_ref, kmajor, kminor_lower, kminor_upper, gas_minor, identifier_minor,
               minor_gases_lower, minor_gases_upper, minor_limits_gpt_lower, minor_limits_gpt_upper,
               minor_scales_with_density_lower, minor_scales_with_density_upper, scaling_gas_lower,
               scaling_gas_upper, scale_by_complement_lower, scale_by_complement_upper, kminor_start_lower,
               kminor_start_upper, rayl_lower, rayl_upper);
        c.t.solar_source_quiet = c.fl(solar_src_quiet);
        c.t.solar_source_facular = c.fl(solar_src_facular);
        c.t.solar_source_sunspot = c.fl(solar_src_sunspot);
        c.t.tsi_default = tsi_default;
        c.t.mg_default = mg_default;
        c.t.sb_default = sb_default;
        create(c, available_gases);
    }

    // Dry-air column amount from the level pressures and h2o (molecules / cm2).
    static void get_col_dry(Array_gpu<Float, 2>& col_dry, const Array_gpu<Float, 2>& vmr_h2o,
                            const Array_gpu<Float, 2>& plev)
    {
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::get_col_dry(vmr_h2o.dim(1), vmr_h2o.dim(2), vmr_h2o.ptr(), plev.ptr(),
                                                             col_dry.ptr()));
    }

    bool source_is_internal() const { return info().is_longwave != 0; }
    bool source_is_external() const { return info().is_longwave == 0; }
    Float get_press_ref_min() const { return Float(info().press_ref_min); }
    Float get_press_ref_max() const { return Float(info().press_ref_max); }
    Float get_temp_min() const { return Float(info().temp_ref_min); }
    Float get_temp_max() const { return Float(info().temp_ref_max); }
    int get_nflav() const { return info().nflav; }
    int get_neta() const { return info().neta; }
    int get_npres() const { return info().npres; }
    int get_ntemp() const { return info().ntemp; }
    int get_nPlanckTemp() const { return info().nplanck_temp; }
    int get_ngas() const { return info().ngas; }
    Float get_tsi() const { return Float(info().tsi); }

    void set_solar_variability(const Float md_index, const Float sb_index)
    {
        rrtmgp_b200_cpp::check(rrtmgp_b200_kdist_set_solar_variability(k_.get(), double(md_index), double(sb_index)));
    }

    // Longwave variant: tau into optical_props; lay/lev/sfc sources into sources.  col_dry and
    // tlev may be empty arrays (col_dry is then computed from h2o and plev).
    void gas_optics(const Array_gpu<Float, 2>& play, const Array_gpu<Float, 2>& plev, const Array_gpu<Float, 2>& tlay,
                    const Array_gpu<Float, 1>& tsfc, const Gas_concs_gpu& gas_desc,
                    std::unique_ptr<Optical_props_arry_gpu>& optical_props, Source_func_lw_gpu& sources,
                    const Array_gpu<Float, 2>& col_dry, const Array_gpu<Float, 2>& tlev)
    {
        const int ncol = play.dim(1), nlay = play.dim(2);
        const std::vector<rrtmgp_b200_gas_conc> d = gas_desc.descriptors();
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::gas_optics_lw(
            k_.get(), ncol, nlay, play.ptr(), plev.ptr(), tlay.ptr(), tsfc.ptr(), tlev.size() ? tlev.ptr() : nullptr,
            col_dry.size() ? col_dry.ptr() : nullptr, d.data(), int(d.size()), optical_props->get_tau().ptr(),
            sources.get_lay_source().ptr(), sources.get_lev_source_inc().ptr(), sources.get_lev_source_dec().ptr(),
            sources.get_sfc_source().ptr(), sources.get_sfc_source_jac().ptr()));
    }

    // Shortwave variant: tau, ssa, g into optical_props (a 2str object) and the solar source
    // per column and g-point into toa_src.
    void gas_optics(const Array_gpu<Float, 2>& play, const Array_gpu<Float, 2>& plev, const Array_gpu<Float, 2>& tlay,
                    const Gas_concs_gpu& gas_desc, std::unique_ptr<Optical_props_arry_gpu>& optical_props,
                    Array_gpu<Float, 2>& toa_src, const Array_gpu<Float, 2>& col_dry)
    {
        const int ncol = play.dim(1), nlay = play.dim(2);
        const std::vector<rrtmgp_b200_gas_conc> d = gas_desc.descriptors();
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::gas_optics_sw(
            k_.get(), ncol, nlay, play.ptr(), plev.ptr(), tlay.ptr(), col_dry.size() ? col_dry.ptr() : nullptr,
            d.data(), int(d.size()), optical_props->get_tau().ptr(), optical_props->get_ssa().ptr(),
            optical_props->get_g().ptr(), toa_src.ptr()));
    }

    // C-ABI k-distribution handle (for the fused column kernels and the batched driver).
    rrtmgp_b200_kdist kdist_handle() const { return k_.get(); }

  private:
    void common(rrtmgp_b200_cpp::Kdist_table_copy& c, const Array<std::string, 1>& gas_names,
                const Array<int, 3>& key_species, const Array<int, 2>& band2gpt,
                const Array<Float, 2>& band_lims_wavenum, const Array<Float, 1>& press_ref, const Float press_ref_trop,
                const Array<Float, 1>& temp_ref, const Float temp_ref_p, const Float temp_ref_t,
                const Array<Float, 3>& vmr_ref, const Array<Float, 4>& kmajor, const Array<Float, 3>& kminor_lower,
                const Array<Float, 3>& kminor_upper, const Array<std::string, 1>& gas_minor,
                const Array<std::string, 1>& identifier_minor, const Array<std::string, 1>& minor_gases_lower,
                const Array<std::string, 1>& minor_gases_upper, const Array<int, 2>& minor_limits_gpt_lower,
                const Array<int, 2>& minor_limits_gpt_upper, const Array<Bool, 1>& msd_lower,
                const Array<Bool, 1>& msd_upper, const Array<std::string, 1>& scaling_gas_lower,
                const Array<std::string, 1>& scaling_gas_upper, const Array<Bool, 1>& sbc_lower,
                const Array<Bool, 1>& sbc_upper, const Array<int, 1>& kminor_start_lower,
                const Array<int, 1>& kminor_start_upper, const Array<Float, 3>& rayl_lower,
                const Array<Float, 3>& rayl_upper)
    {
        rrtmgp_b200_kdist_tables& t = c.t;
        t.ngas = gas_names.dim(1);
        t.nband = band2gpt.dim(2);
        t.ngpt = kmajor.dim(1);
        t.neta = kmajor.dim(2);
        t.npres = kmajor.dim(3) - 1;
        t.ntemp = kmajor.dim(4);
        t.nminor_absorber = gas_minor.size();
        t.nint_lower = minor_limits_gpt_lower.size() / 2;
        t.nint_upper = minor_limits_gpt_upper.size() / 2;
        t.ncontrib_lower = kminor_lower.size() ? kminor_lower.dim(1) : 0;
        t.ncontrib_upper = kminor_upper.size() ? kminor_upper.dim(1) : 0;
        t.gas_names = c.str(gas_names);
        t.key_species = c.in(key_species);
        t.band_lims_gpt = c.in(band2gpt);
        t.band_lims_wvn = c.fl(band_lims_wavenum);
        t.press_ref = c.fl(press_ref);
        t.press_ref_trop = press_ref_trop;
        t.temp_ref = c.fl(temp_ref);
        t.temp_ref_p = temp_ref_p;
        t.temp_ref_t = temp_ref_t;
        t.vmr_ref = c.fl(vmr_ref);
        t.kmajor = c.fl(kmajor);
        t.kminor_lower = c.fl(kminor_lower);
        t.kminor_upper = c.fl(kminor_upper);
        t.gas_minor = c.str(gas_minor);
        t.identifier_minor = c.str(identifier_minor);
        t.minor_gases_lower = c.str(minor_gases_lower);
        t.minor_gases_upper = c.str(minor_gases_upper);
        t.minor_limits_gpt_lower = c.in(minor_limits_gpt_lower);
        t.minor_limits_gpt_upper = c.in(minor_limits_gpt_upper);
        t.minor_scales_with_density_lower = c.in(msd_lower);
        t.minor_scales_with_density_upper = c.in(msd_upper);
        t.scaling_gas_lower = c.str(scaling_gas_lower);
        t.scaling_gas_upper = c.str(scaling_gas_upper);
        t.scale_by_complement_lower = c.in(sbc_lower);
        t.scale_by_complement_upper = c.in(sbc_upper);
        t.kminor_start_lower = c.in(kminor_start_lower);
        t.kminor_start_upper = c.in(kminor_start_upper);
        t.rayl_lower = c.fl(rayl_lower);
        t.rayl_upper = c.fl(rayl_upper);
    }

    void create(rrtmgp_b200_cpp::Kdist_table_copy& c, const Gas_concs_gpu& available_gases)
    {
        const std::vector<std::string> names = available_gases.get_gas_names();
        std::vector<const char*> p;
        for (const auto& n : names) p.push_back(n.c_str());
        rrtmgp_b200_kdist h = nullptr;
        rrtmgp_b200_cpp::check(rrtmgp_b200_kdist_create(&c.t, p.data(), int(p.size()), &h));
        k_ = std::shared_ptr<rrtmgp_b200_kdist_t>(h, [](rrtmgp_b200_kdist q) { rrtmgp_b200_kdist_destroy(q); });
    }

    rrtmgp_b200_kdist_info info() const
    {
        rrtmgp_b200_kdist_info i{};
        rrtmgp_b200_cpp::check(rrtmgp_b200_kdist_get_info(k_.get(), &i));
        return i;
    }

    std::shared_ptr<rrtmgp_b200_kdist_t> k_;
};

#endif
