// Test driver of the C++ class API (include/cpp): the LW and SW column solves written the way
// a reference caller writes them (Radiation_solver_longwave/shortwave::solve_gpu,
// src_test/Radiation_solver.cu:419-950 of rte-rrtmgp-cpp) -- host Array tables into the
// Gas_optics_rrtmgp_gpu and Cloud_optics_gpu constructors, Gas_concs_gpu, gas_optics,
// cloud_optics (+ delta_scale) and add_to, Rte_lw_gpu / Rte_sw_gpu, Fluxes_broadband_gpu.
// Built twice (Float = double, and Float = float with RTE_USE_SP) as shared libraries whose
// extern "C" entry points the parity tests call with the synthetic tables and atmospheres.
// Test infrastructure only.
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "Aerosol_optics.h"
#include "Cloud_optics.h"
#include "Fluxes.h"
#include "Gas_optics_rrtmgp.h"
#include "Rte_lw.h"
#include "Rte_sw.h"

namespace {

template <int N>
Array<Float, N> farr(const double* p, const std::array<int, N>& dims)
{
    Array<Float, N> a(dims);
    for (int i = 0; i < a.size(); ++i) a.v()[i] = Float(p[i]);
    return a;
}

template <typename T, int N>
Array<T, N> iarr(const int* p, const std::array<int, N>& dims)
{
    Array<T, N> a(dims);
    for (int i = 0; i < a.size(); ++i) a.v()[i] = T(p[i]);
    return a;
}

Array<std::string, 1> sarr(const char* const* p, int n)
{
    Array<std::string, 1> a({n});
    for (int i = 0; i < n; ++i) a.v()[i] = p[i];
    return a;
}

// The netCDF-file tables (C order) as the reference's loader puts them into Fortran-order
// Arrays: dimensions reversed, memory unchanged.
struct Tables {
    Array<std::string, 1> gas_names, gas_minor, identifier_minor, minor_gases_lower, minor_gases_upper,
        scaling_gas_lower, scaling_gas_upper;
    Array<int, 3> key_species;
    Array<int, 2> band2gpt, minor_limits_gpt_lower, minor_limits_gpt_upper;
    Array<Float, 2> band_lims;
    Array<Float, 1> press_ref, temp_ref;
    Array<Float, 3> vmr_ref, kminor_lower, kminor_upper, rayl_lower, rayl_upper;
    Array<Float, 4> kmajor;
    Array<Bool, 1> msd_lower, msd_upper, sbc_lower, sbc_upper;
    Array<int, 1> kminor_start_lower, kminor_start_upper;

    explicit Tables(const rrtmgp_b200_kdist_tables& t)
    {
        const int nb = t.nband, ng = t.ngpt, nt = t.ntemp, np = t.npres, ne = t.neta;
        gas_names = sarr(t.gas_names, t.ngas);
        key_species = iarr<int, 3>(t.key_species, {2, 2, nb});
        band2gpt = iarr<int, 2>(t.band_lims_gpt, {2, nb});
        band_lims = farr<2>(t.band_lims_wvn, {2, nb});
        press_ref = farr<1>(t.press_ref, {np});
        temp_ref = farr<1>(t.temp_ref, {nt});
        vmr_ref = farr<3>(t.vmr_ref, {2, t.ngas + 1, nt});
        kmajor = farr<4>(t.kmajor, {ng, ne, np + 1, nt});
        kminor_lower = farr<3>(t.kminor_lower, {t.ncontrib_lower, ne, nt});
        kminor_upper = farr<3>(t.kminor_upper, {t.ncontrib_upper, ne, nt});
        gas_minor = sarr(t.gas_minor, t.nminor_absorber);
        identifier_minor = sarr(t.identifier_minor, t.nminor_absorber);
        minor_gases_lower = sarr(t.minor_gases_lower, t.nint_lower);
        minor_gases_upper = sarr(t.minor_gases_upper, t.nint_upper);
        minor_limits_gpt_lower = iarr<int, 2>(t.minor_limits_gpt_lower, {2, t.nint_lower});
        minor_limits_gpt_upper = iarr<int, 2>(t.minor_limits_gpt_upper, {2, t.nint_upper});
        msd_lower = iarr<Bool, 1>(t.minor_scales_with_density_lower, {t.nint_lower});
        msd_upper = iarr<Bool, 1>(t.minor_scales_with_density_upper, {t.nint_upper});
        scaling_gas_lower = sarr(t.scaling_gas_lower, t.nint_lower);
        scaling_gas_upper = sarr(t.scaling_gas_upper, t.nint_upper);
        sbc_lower = iarr<Bool, 1>(t.scale_by_complement_lower, {t.nint_lower});
        sbc_upper = iarr<Bool, 1>(t.scale_by_complement_upper, {t.nint_upper});
        kminor_start_lower = iarr<int, 1>(t.kminor_start_lower, {t.nint_lower});
        kminor_start_upper = iarr<int, 1>(t.kminor_start_upper, {t.nint_upper});
        if (t.rayl_lower) {
            rayl_lower = farr<3>(t.rayl_lower, {ng, ne, nt});
            rayl_upper = farr<3>(t.rayl_upper, {ng, ne, nt});
        }
    }
};

Gas_optics_rrtmgp_gpu make_lw(const rrtmgp_b200_kdist_tables* tk, const Tables& t, const Gas_concs_gpu& gases)
{
    return Gas_optics_rrtmgp_gpu(
        gases, t.gas_names, t.key_species, t.band2gpt, t.band_lims, t.press_ref, Float(tk->press_ref_trop),
        t.temp_ref, Float(tk->temp_ref_p), Float(tk->temp_ref_t), t.vmr_ref, t.kmajor, t.kminor_lower,
        t.kminor_upper, t.gas_minor, t.identifier_minor, t.minor_gases_lower, t.minor_gases_upper,
        t.minor_limits_gpt_lower, t.minor_limits_gpt_upper, t.msd_lower, t.msd_upper, t.scaling_gas_lower,
        t.scaling_gas_upper, t.sbc_lower, t.sbc_upper, t.kminor_start_lower, t.kminor_start_upper,
        farr<2>(tk->totplnk, {tk->nplanck_temp, tk->nband}),
        farr<4>(tk->planck_frac, {tk->ngpt, tk->neta, tk->npres + 1, tk->ntemp}), t.rayl_lower, t.rayl_upper);
}

std::unique_ptr<Cloud_optics_gpu> make_cloud(const rrtmgp_b200_cloud_tables& c)
{
    return std::make_unique<Cloud_optics_gpu>(
        farr<2>(c.band_lims_wvn, {2, c.nband}), Float(c.radliq_lwr), Float(c.radliq_upr), Float(c.radliq_fac),
        Float(c.radice_lwr), Float(c.radice_upr), Float(c.radice_fac),
        farr<2>(c.lut_extliq, {c.nsize_liq, c.nband}), farr<2>(c.lut_ssaliq, {c.nsize_liq, c.nband}),
        farr<2>(c.lut_asyliq, {c.nsize_liq, c.nband}), farr<3>(c.lut_extice, {c.nsize_ice, c.nband, c.nrghice}),
        farr<3>(c.lut_ssaice, {c.nsize_ice, c.nband, c.nrghice}),
        farr<3>(c.lut_asyice, {c.nsize_ice, c.nband, c.nrghice}));
}

Gas_concs make_gases(int ngas, const char* const* names, const double* const* vmr, const int* dims)
{
    Gas_concs g;
    for (int i = 0; i < ngas; ++i) {
        const int d1 = dims[2 * i], d2 = dims[2 * i + 1];
        if (d1 == 1 && d2 == 1)
            g.set_vmr(names[i], Float(vmr[i][0]));
        else if (d1 == 1)
            g.set_vmr(names[i], farr<1>(vmr[i], {d2}));
        else
            g.set_vmr(names[i], farr<2>(vmr[i], {d1, d2}));
    }
    return g;
}

void out2(const Array_gpu<Float, 2>& a, double* o)
{
    const Array<Float, 2> h(a);
    for (int i = 0; i < h.size(); ++i) o[i] = double(h.v()[i]);
}

void out3(const Array_gpu<Float, 3>& a, double* o)
{
    const Array<Float, 3> h(a);
    for (int i = 0; i < h.size(); ++i) o[i] = double(h.v()[i]);
}

int fail(const std::exception& e, char* err, int errlen)
{
    std::strncpy(err, e.what(), size_t(errlen) - 1);
    err[errlen - 1] = '\0';
    return 1;
}

}  // namespace

extern "C" {

// Longwave: gas optics + optional clouds (1scl, added by band) + rte_lw + broadband fluxes.
int class_api_forward_lw(const rrtmgp_b200_kdist_tables* tk, const rrtmgp_b200_cloud_tables* tc, int ncol, int nlay,
                         const double* play_in, const double* plev_in, const double* tlay_in, const double* tlev_in,
                         const double* tsfc_in, const double* emis_in, int ngas, const char* const* gas_names,
                         const double* const* gas_vmr, const int* gas_dims, const double* lwp_in,
                         const double* iwp_in, const double* rel_in, const double* rei_in, int n_gauss_angles,
                         double* flux_up, double* flux_dn, double* flux_net, char* err, int errlen)
{
    try {
        const int nlev = nlay + 1;
        const Tables t(*tk);
        const Gas_concs gas_concs = make_gases(ngas, gas_names, gas_vmr, gas_dims);
        const Gas_concs_gpu gas_concs_gpu(gas_concs);
        Gas_optics_rrtmgp_gpu kdist = make_lw(tk, t, gas_concs_gpu);

        const Array<Float, 2> p_lay = farr<2>(play_in, {ncol, nlay});
        const Array_gpu<Float, 2> p_lay_g(p_lay), p_lev_g(farr<2>(plev_in, {ncol, nlev})),
            t_lay_g(farr<2>(tlay_in, {ncol, nlay})), t_lev_g(farr<2>(tlev_in, {ncol, nlev}));
        const Array_gpu<Float, 1> t_sfc_g(farr<1>(tsfc_in, {ncol}));
        const Array_gpu<Float, 2> emis_g(farr<2>(emis_in, {kdist.get_nband(), ncol}));
        const Bool top_at_1 = p_lay({1, 1}) < p_lay({1, nlay});

        std::unique_ptr<Optical_props_arry_gpu> optical_props =
            std::make_unique<Optical_props_1scl_gpu>(ncol, nlay, kdist);
        Source_func_lw_gpu sources(ncol, nlay, kdist);
        kdist.gas_optics(p_lay_g, p_lev_g, t_lay_g, t_sfc_g, gas_concs_gpu, optical_props, sources,
                         Array_gpu<Float, 2>(), t_lev_g);

        if (tc) {
            std::unique_ptr<Cloud_optics_gpu> cloud = make_cloud(*tc);
            Optical_props_1scl_gpu cloud_props(ncol, nlay, *cloud);
            cloud->cloud_optics(Array_gpu<Float, 2>(farr<2>(lwp_in, {ncol, nlay})),
                                Array_gpu<Float, 2>(farr<2>(iwp_in, {ncol, nlay})),
                                Array_gpu<Float, 2>(farr<2>(rel_in, {ncol, nlay})),
                                Array_gpu<Float, 2>(farr<2>(rei_in, {ncol, nlay})), cloud_props);
            add_to(dynamic_cast<Optical_props_1scl_gpu&>(*optical_props), cloud_props);
        }

        Array_gpu<Float, 3> gpt_flux_up({ncol, nlev, kdist.get_ngpt()}), gpt_flux_dn({ncol, nlev, kdist.get_ngpt()});
        Rte_lw_gpu rte_lw;
        rte_lw.rte_lw(optical_props, top_at_1, sources, emis_g, Array_gpu<Float, 2>(), gpt_flux_up, gpt_flux_dn,
                      n_gauss_angles);
        Fluxes_broadband_gpu fluxes(ncol, nlev);
        fluxes.reduce(gpt_flux_up, gpt_flux_dn, optical_props, top_at_1);
        out2(fluxes.get_flux_up(), flux_up);
        out2(fluxes.get_flux_dn(), flux_dn);
        out2(fluxes.get_flux_net(), flux_net);
        return 0;
    } catch (const std::exception& e) {
        return fail(e, err, errlen);
    }
}

// Shortwave: gas optics + toa_src x tsi_scaling + optional clouds (2str, delta-scaled, added by
// band) + rte_sw + broadband fluxes (with the direct beam).
int class_api_forward_sw(const rrtmgp_b200_kdist_tables* tk, const rrtmgp_b200_cloud_tables* tc, int ncol, int nlay,
                         const double* play_in, const double* plev_in, const double* tlay_in, const double* mu0_in,
                         const double* tsi_in, const double* alb_dir_in, const double* alb_dif_in, int ngas,
                         const char* const* gas_names, const double* const* gas_vmr, const int* gas_dims,
                         const double* lwp_in, const double* iwp_in, const double* rel_in, const double* rei_in,
                         double* flux_up, double* flux_dn, double* flux_dn_dir, double* flux_net, char* err,
                         int errlen)
{
    try {
        const int nlev = nlay + 1;
        const Tables t(*tk);
        const Gas_concs gas_concs = make_gases(ngas, gas_names, gas_vmr, gas_dims);
        const Gas_concs_gpu gas_concs_gpu(gas_concs);
        Gas_optics_rrtmgp_gpu kdist(
            gas_concs_gpu, t.gas_names, t.key_species, t.band2gpt, t.band_lims, t.press_ref, Float(tk->press_ref_trop),
            t.temp_ref, Float(tk->temp_ref_p), Float(tk->temp_ref_t), t.vmr_ref, t.kmajor, t.kminor_lower,
            t.kminor_upper, t.gas_minor, t.identifier_minor, t.minor_gases_lower, t.minor_gases_upper,
            t.minor_limits_gpt_lower, t.minor_limits_gpt_upper, t.msd_lower, t.msd_upper, t.scaling_gas_lower,
            t.scaling_gas_upper, t.sbc_lower, t.sbc_upper, t.kminor_start_lower, t.kminor_start_upper,
            farr<1>(tk->solar_source_quiet, {tk->ngpt}), farr<1>(tk->solar_source_facular, {tk->ngpt}),
            farr<1>(tk->solar_source_sunspot, {tk->ngpt}), Float(tk->tsi_default), Float(tk->mg_default),
            Float(tk->sb_default), t.rayl_lower, t.rayl_upper);

        const int ngpt = kdist.get_ngpt(), nband = kdist.get_nband();
        const Array<Float, 2> p_lay = farr<2>(play_in, {ncol, nlay});
        const Array_gpu<Float, 2> p_lay_g(p_lay), p_lev_g(farr<2>(plev_in, {ncol, nlev})),
            t_lay_g(farr<2>(tlay_in, {ncol, nlay}));
        const Array_gpu<Float, 1> mu0_g(farr<1>(mu0_in, {ncol}));
        const Array_gpu<Float, 2> alb_dir_g(farr<2>(alb_dir_in, {nband, ncol})),
            alb_dif_g(farr<2>(alb_dif_in, {nband, ncol}));
        const Bool top_at_1 = p_lay({1, 1}) < p_lay({1, nlay});

        std::unique_ptr<Optical_props_arry_gpu> optical_props =
            std::make_unique<Optical_props_2str_gpu>(ncol, nlay, kdist);
        Array_gpu<Float, 2> toa_src({ncol, ngpt});
        kdist.gas_optics(p_lay_g, p_lev_g, t_lay_g, gas_concs_gpu, optical_props, toa_src, Array_gpu<Float, 2>());

        // toa_src x tsi_scaling per column (Radiation_solver.cu:44-69, done here on the host).
        Array<Float, 2> toa(toa_src);
        for (int g = 1; g <= ngpt; ++g)
            for (int c = 1; c <= ncol; ++c) toa({c, g}) *= Float(tsi_in[c - 1]);
        toa_src = Array_gpu<Float, 2>(toa);

        if (tc) {
            std::unique_ptr<Cloud_optics_gpu> cloud = make_cloud(*tc);
            Optical_props_2str_gpu cloud_props(ncol, nlay, *cloud);
            cloud->cloud_optics(Array_gpu<Float, 2>(farr<2>(lwp_in, {ncol, nlay})),
                                Array_gpu<Float, 2>(farr<2>(iwp_in, {ncol, nlay})),
                                Array_gpu<Float, 2>(farr<2>(rel_in, {ncol, nlay})),
                                Array_gpu<Float, 2>(farr<2>(rei_in, {ncol, nlay})), cloud_props);
            cloud_props.delta_scale();
            add_to(dynamic_cast<Optical_props_2str_gpu&>(*optical_props), cloud_props);
        }

        Array_gpu<Float, 3> up({ncol, nlev, ngpt}), dn({ncol, nlev, ngpt}), dir({ncol, nlev, ngpt});
        Rte_sw_gpu rte_sw;
        rte_sw.rte_sw(optical_props, top_at_1, mu0_g, toa_src, alb_dir_g, alb_dif_g, Array_gpu<Float, 2>(), up, dn,
                      dir);
        Fluxes_broadband_gpu fluxes(ncol, nlev);
        fluxes.reduce(up, dn, dir, optical_props, top_at_1);
        out2(fluxes.get_flux_up(), flux_up);
        out2(fluxes.get_flux_dn(), flux_dn);
        out2(fluxes.get_flux_dn_dir(), flux_dn_dir);
        out2(fluxes.get_flux_net(), flux_net);
        return 0;
    } catch (const std::exception& e) {
        return fail(e, err, errlen);
    }
}

// Error path: a k-distribution whose key species is not among the available gases must throw
// from the constructor (Gas_optics_rrtmgp.cpp:241-243).  Returns 0 when it threw.
int class_api_missing_gas_throws(const rrtmgp_b200_kdist_tables* tk, char* err, int errlen)
{
    try {
        const Tables t(*tk);
        Gas_concs g;
        g.set_vmr("h2o", Float(0.01));
        const Gas_concs_gpu gg(g);
        Gas_optics_rrtmgp_gpu kdist = make_lw(tk, t, gg);
        return 1;
    } catch (const std::runtime_error& e) {
        fail(e, err, errlen);
        return 0;
    }
}

// Aerosol optics through Aerosol_optics_gpu, tables as load_and_init_aerosol_optics builds them
// (src_test/Radiation_solver.cu:366-401); the species are Aerosol_concs entries aermr01 ..
// aermr11.  tau, ssa, g (ncol, nlay, nband).
int class_api_aerosol_optics(const rrtmgp_b200_aerosol_tables* ta, int ncol, int nlay, const double* rh_in,
                             const double* plev_in, int naer, const char* const* names, const double* const* mmr,
                             const int* dims, double* tau, double* ssa, double* g, char* err, int errlen)
{
    try {
        const int nb = ta->nband, nh = ta->nhum, npl = ta->nphilic, nph = ta->nphobic;
        Aerosol_optics_gpu aerosol(Array<Float, 2>({2, nb}), farr<1>(ta->rh_upper, {nh}),
                                   farr<2>(ta->mext_phobic, {nb, nph}), farr<2>(ta->ssa_phobic, {nb, nph}),
                                   farr<2>(ta->g_phobic, {nb, nph}), farr<3>(ta->mext_philic, {nb, nh, npl}),
                                   farr<3>(ta->ssa_philic, {nb, nh, npl}), farr<3>(ta->g_philic, {nb, nh, npl}));
        const Aerosol_concs concs = make_gases(naer, names, mmr, dims);
        Aerosol_concs_gpu concs_gpu(concs);
        Optical_props_2str_gpu props(ncol, nlay, aerosol);
        aerosol.aerosol_optics(concs_gpu, Array_gpu<Float, 2>(farr<2>(rh_in, {ncol, nlay})),
                               Array_gpu<Float, 2>(farr<2>(plev_in, {ncol, nlay + 1})), props);
        out3(props.get_tau(), tau);
        out3(props.get_ssa(), ssa);
        out3(props.get_g(), g);
        return 0;
    } catch (const std::exception& e) {
        return fail(e, err, errlen);
    }
}

int class_api_float_bytes(void) { return int(sizeof(Float)); }

}  // extern "C"
