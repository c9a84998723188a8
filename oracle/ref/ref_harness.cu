// ORACLE -- test infrastructure only.
//
// C entry points over the reference's own GPU classes (rte-rrtmgp-cpp src_cuda/ +
// src_kernels_cuda/, compiled from the reference sources by oracle/ref/Makefile into
// oracle/_ref/libref_rrtmgp_f64.so).  Used once, on the GPU box, by
// tests/golden/make_ref_golden.py to produce fixtures that pin the FP64 oracle to the
// reference implementation.  All arrays are host double arrays in the reference layouts;
// tables come in the netCDF layout of load_and_init_gas_optics
// (src_test/Radiation_solver.cpp:70-284).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "Array.h"
#include "Cloud_optics.h"
#include "Aerosol_optics.h"
#include "Fluxes.h"
#include "Gas_concs.h"
#include "Gas_optics_rrtmgp.h"
#include "Optical_props.h"
#include "Rte_lw.h"
#include "Rte_sw.h"
#include "Source_functions.h"
#include "../../include/rrtmgp_b200.h"

namespace {

thread_local std::string g_err;

template <typename T, int N>
Array<T, N> host(const T* p, const std::array<int, N>& dims)
{
    size_t n = 1;
    for (int d : dims) n *= size_t(d);
    return Array<T, N>(std::vector<T>(p, p + n), dims);
}

Array<std::string, 1> strs(const char* const* p, int n)
{
    std::vector<std::string> v;
    for (int i = 0; i < n; ++i) v.push_back(p[i]);
    return Array<std::string, 1>(v, {n});
}

template <typename T, int N>
Array_gpu<T, N> dev(const T* p, const std::array<int, N>& dims)
{
    return Array_gpu<T, N>(host<T, N>(p, dims));
}

template <typename T, int N>
void out(const Array_gpu<T, N>& a, T* dst)
{
    if (!dst) return;
    cudaDeviceSynchronize();
    cudaMemcpy(dst, a.ptr(), a.size() * sizeof(T), cudaMemcpyDeviceToHost);
}

Gas_concs gas_concs(const rrtmgp_b200_gas_conc* g, int n, int ncol, int nlay)
{
    Gas_concs gc;
    for (int i = 0; i < n; ++i) {
        const double* v = static_cast<const double*>(g[i].vmr);
        if (g[i].dim1 == 1 && g[i].dim2 == 1) gc.set_vmr(g[i].name, v[0]);
        else gc.set_vmr(g[i].name, host<double, 2>(v, {g[i].dim1, g[i].dim2}));
    }
    return gc;
}

std::unique_ptr<Gas_optics_rrtmgp_gpu> make_kdist(const rrtmgp_b200_kdist_tables* t, const Gas_concs_gpu& avail)
{
    const int ngas = t->ngas, nb = t->nband, ng = t->ngpt, nt = t->ntemp, np = t->npres, ne = t->neta;
    auto gas_names = strs(t->gas_names, ngas);
    auto key = host<int, 3>(t->key_species, {2, 2, nb});
    auto b2g = host<int, 2>(t->band_lims_gpt, {2, nb});
    auto blw = host<double, 2>(t->band_lims_wvn, {2, nb});
    auto pref = host<double, 1>(t->press_ref, {np});
    auto tref = host<double, 1>(t->temp_ref, {nt});
    auto vmr = host<double, 3>(t->vmr_ref, {2, ngas + 1, nt});
    auto kmaj = host<double, 4>(t->kmajor, {ng, ne, np + 1, nt});
    auto kmlo = host<double, 3>(t->kminor_lower, {t->ncontrib_lower, ne, nt});
    auto kmup = host<double, 3>(t->kminor_upper, {t->ncontrib_upper, ne, nt});
    auto gmin = strs(t->gas_minor, t->nminor_absorber);
    auto idmin = strs(t->identifier_minor, t->nminor_absorber);
    auto mglo = strs(t->minor_gases_lower, t->nint_lower);
    auto mgup = strs(t->minor_gases_upper, t->nint_upper);
    auto mllo = host<int, 2>(t->minor_limits_gpt_lower, {2, t->nint_lower});
    auto mlup = host<int, 2>(t->minor_limits_gpt_upper, {2, t->nint_upper});
    auto dlo = host<int, 1>(t->minor_scales_with_density_lower, {t->nint_lower});
    auto dup = host<int, 1>(t->minor_scales_with_density_upper, {t->nint_upper});
    auto sglo = strs(t->scaling_gas_lower, t->nint_lower);
    auto sgup = strs(t->scaling_gas_upper, t->nint_upper);
    auto clo = host<int, 1>(t->scale_by_complement_lower, {t->nint_lower});
    auto cup = host<int, 1>(t->scale_by_complement_upper, {t->nint_upper});
    auto kslo = host<int, 1>(t->kminor_start_lower, {t->nint_lower});
    auto ksup = host<int, 1>(t->kminor_start_upper, {t->nint_upper});
    if (t->totplnk) {
        auto tp = host<double, 2>(t->totplnk, {t->nplanck_temp, nb});
        auto pf = host<double, 4>(t->planck_frac, {ng, ne, np + 1, nt});
        return std::make_unique<Gas_optics_rrtmgp_gpu>(
            avail, gas_names, key, b2g, blw, pref, t->press_ref_trop, tref, t->temp_ref_p, t->temp_ref_t, vmr, kmaj,
            kmlo, kmup, gmin, idmin, mglo, mgup, mllo, mlup, dlo, dup, sglo, sgup, clo, cup, kslo, ksup, tp, pf,
            Array<double, 3>(), Array<double, 3>());
    }
    auto sq = host<double, 1>(t->solar_source_quiet, {ng});
    auto sf = host<double, 1>(t->solar_source_facular, {ng});
    auto ss = host<double, 1>(t->solar_source_sunspot, {ng});
    auto rlo = host<double, 3>(t->rayl_lower, {ng, ne, nt});
    auto rup = host<double, 3>(t->rayl_upper, {ng, ne, nt});
    return std::make_unique<Gas_optics_rrtmgp_gpu>(
        avail, gas_names, key, b2g, blw, pref, t->press_ref_trop, tref, t->temp_ref_p, t->temp_ref_t, vmr, kmaj, kmlo,
        kmup, gmin, idmin, mglo, mgup, mllo, mlup, dlo, dup, sglo, sgup, clo, cup, kslo, ksup, sq, sf, ss,
        t->tsi_default, t->mg_default, t->sb_default, rlo, rup);
}

Optical_props_gpu bands_of(int nband, const int* lims)
{
    std::vector<double> wvn(2 * nband);
    for (int i = 0; i < 2 * nband; ++i) wvn[i] = double(i + 1);
    return Optical_props_gpu(Array<double, 2>(wvn, {2, nband}), host<int, 2>(lims, {2, nband}));
}

template <typename F>
int guarded(F&& f)
{
    try {
        f();
        cudaDeviceSynchronize();
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { g_err = cudaGetErrorString(e); return 4; }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    } catch (...) {
        g_err = "reference threw a non-std exception";
        return 1;
    }
}

Cloud_optics_gpu make_cloud(const rrtmgp_b200_cloud_tables* c)
{
    const int nb = c->nband;
    return Cloud_optics_gpu(host<double, 2>(c->band_lims_wvn, {2, nb}), c->radliq_lwr, c->radliq_upr, c->radliq_fac,
                            c->radice_lwr, c->radice_upr, c->radice_fac,
                            host<double, 2>(c->lut_extliq, {c->nsize_liq, nb}),
                            host<double, 2>(c->lut_ssaliq, {c->nsize_liq, nb}),
                            host<double, 2>(c->lut_asyliq, {c->nsize_liq, nb}),
                            host<double, 3>(c->lut_extice, {c->nsize_ice, nb, c->nrghice}),
                            host<double, 3>(c->lut_ssaice, {c->nsize_ice, nb, c->nrghice}),
                            host<double, 3>(c->lut_asyice, {c->nsize_ice, nb, c->nrghice}));
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

// Gas_optics_rrtmgp_gpu::gas_optics, longwave (src_cuda/Gas_optics_rrtmgp.cu:907-943); col_dry
// from get_col_dry when NULL (as Radiation_solver_longwave::solve_gpu does).
int ref_gas_optics_lw(const rrtmgp_b200_kdist_tables* t, const rrtmgp_b200_gas_conc* gases, int ngases, int ncol,
                      int nlay, const double* play, const double* plev, const double* tlay, const double* tsfc,
                      const double* tlev, const double* col_dry, double* tau, double* lay_src, double* lev_inc,
                      double* lev_dec, double* sfc_src, double* sfc_jac)
{
    return guarded([&] {
        Gas_concs gc = gas_concs(gases, ngases, ncol, nlay);
        Gas_concs_gpu gcg(gc);
        auto kd = make_kdist(t, gcg);
        std::unique_ptr<Optical_props_arry_gpu> ops = std::make_unique<Optical_props_1scl_gpu>(ncol, nlay, *kd);
        Source_func_lw_gpu src(ncol, nlay, *kd);
        auto p = dev<double, 2>(play, {ncol, nlay});
        auto pl = dev<double, 2>(plev, {ncol, nlay + 1});
        auto tl = dev<double, 2>(tlay, {ncol, nlay});
        auto ts = dev<double, 1>(tsfc, {ncol});
        auto tv = dev<double, 2>(tlev, {ncol, nlay + 1});
        Array_gpu<double, 2> cd({ncol, nlay});
        if (col_dry) cd = dev<double, 2>(col_dry, {ncol, nlay});
        else Gas_optics_rrtmgp_gpu::get_col_dry(cd, gcg.get_vmr("h2o"), pl);
        kd->gas_optics(p, pl, tl, ts, gcg, ops, src, cd, tv);
        out(ops->get_tau(), tau);
        out(src.get_lay_source(), lay_src);
        out(src.get_lev_source_inc(), lev_inc);
        out(src.get_lev_source_dec(), lev_dec);
        out(src.get_sfc_source(), sfc_src);
        out(src.get_sfc_source_jac(), sfc_jac);
    });
}

// Gas_optics_rrtmgp_gpu::gas_optics, shortwave (src_cuda/Gas_optics_rrtmgp.cu:947-977).
int ref_gas_optics_sw(const rrtmgp_b200_kdist_tables* t, const rrtmgp_b200_gas_conc* gases, int ngases, int ncol,
                      int nlay, const double* play, const double* plev, const double* tlay, const double* col_dry,
                      double* tau, double* ssa, double* g, double* toa_src)
{
    return guarded([&] {
        Gas_concs gc = gas_concs(gases, ngases, ncol, nlay);
        Gas_concs_gpu gcg(gc);
        auto kd = make_kdist(t, gcg);
        std::unique_ptr<Optical_props_arry_gpu> ops = std::make_unique<Optical_props_2str_gpu>(ncol, nlay, *kd);
        auto p = dev<double, 2>(play, {ncol, nlay});
        auto pl = dev<double, 2>(plev, {ncol, nlay + 1});
        auto tl = dev<double, 2>(tlay, {ncol, nlay});
        Array_gpu<double, 2> cd({ncol, nlay});
        if (col_dry) cd = dev<double, 2>(col_dry, {ncol, nlay});
        else Gas_optics_rrtmgp_gpu::get_col_dry(cd, gcg.get_vmr("h2o"), pl);
        Array_gpu<double, 2> toa({ncol, kd->get_ngpt()});
        kd->gas_optics(p, pl, tl, gcg, ops, toa, cd);
        out(ops->get_tau(), tau);
        out(ops->get_ssa(), ssa);
        out(ops->get_g(), g);
        out(toa, toa_src);
    });
}

// Cloud_optics_gpu::cloud_optics 2str / 1scl (src_cuda/Cloud_optics.cu:181-329), optionally
// followed by Optical_props_2str_gpu::delta_scale.
int ref_cloud_optics(const rrtmgp_b200_cloud_tables* c, int ncol, int nlay, const double* clwp, const double* ciwp,
                     const double* reliq, const double* reice, int two_stream, int delta, double* tau, double* ssa,
                     double* g)
{
    return guarded([&] {
        const int nb = c->nband;
        Cloud_optics_gpu co(host<double, 2>(c->band_lims_wvn, {2, nb}), c->radliq_lwr, c->radliq_upr, c->radliq_fac,
                            c->radice_lwr, c->radice_upr, c->radice_fac,
                            host<double, 2>(c->lut_extliq, {c->nsize_liq, nb}),
                            host<double, 2>(c->lut_ssaliq, {c->nsize_liq, nb}),
                            host<double, 2>(c->lut_asyliq, {c->nsize_liq, nb}),
                            host<double, 3>(c->lut_extice, {c->nsize_ice, nb, c->nrghice}),
                            host<double, 3>(c->lut_ssaice, {c->nsize_ice, nb, c->nrghice}),
                            host<double, 3>(c->lut_asyice, {c->nsize_ice, nb, c->nrghice}));
        auto l = dev<double, 2>(clwp, {ncol, nlay});
        auto i = dev<double, 2>(ciwp, {ncol, nlay});
        auto rl = dev<double, 2>(reliq, {ncol, nlay});
        auto ri = dev<double, 2>(reice, {ncol, nlay});
        if (two_stream) {
            Optical_props_2str_gpu o(ncol, nlay, co);
            co.cloud_optics(l, i, rl, ri, o);
            if (delta) o.delta_scale();
            out(o.get_tau(), tau);
            out(o.get_ssa(), ssa);
            out(o.get_g(), g);
        } else {
            Optical_props_1scl_gpu o(ncol, nlay, co);
            co.cloud_optics(l, i, rl, ri, o);
            out(o.get_tau(), tau);
        }
    });
}

// add_to(Optical_props_2str_gpu&, const Optical_props_2str_gpu&) by band (Optical_props.cu:119-145).
int ref_add_to_2str_bybnd(int ncol, int nlay, int nband, const int* band_lims, double* tau, double* ssa, double* g,
                          const double* tau2, const double* ssa2, const double* g2)
{
    return guarded([&] {
        Optical_props_gpu b = bands_of(nband, band_lims);
        Optical_props_gpu bb = bands_of(nband, [&] {
            static std::vector<int> l;
            l.assign(2 * nband, 0);
            for (int i = 0; i < nband; ++i) { l[2 * i] = i + 1; l[2 * i + 1] = i + 1; }
            return l.data();
        }());
        Optical_props_2str_gpu a(ncol, nlay, b), c(ncol, nlay, bb);
        const int ngpt = b.get_ngpt();
        const size_t na = size_t(ncol) * nlay * ngpt, nc = size_t(ncol) * nlay * nband;
        cudaMemcpy(a.get_tau().ptr(), tau, na * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(a.get_ssa().ptr(), ssa, na * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(a.get_g().ptr(), g, na * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(c.get_tau().ptr(), tau2, nc * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(c.get_ssa().ptr(), ssa2, nc * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(c.get_g().ptr(), g2, nc * 8, cudaMemcpyHostToDevice);
        add_to(a, c);
        out(a.get_tau(), tau);
        out(a.get_ssa(), ssa);
        out(a.get_g(), g);
    });
}

// Rte_lw_gpu::rte_lw (src_cuda/Rte_lw.cu:81-152), single angle.
int ref_rte_lw(int ncol, int nlay, int nband, const int* band_lims, int top_at_1, const double* tau,
               const double* lay_src, const double* lev_inc, const double* lev_dec, const double* sfc_src,
               const double* sfc_emis, double* flux_up, double* flux_dn)
{
    return guarded([&] {
        Optical_props_gpu b = bands_of(nband, band_lims);
        const int ngpt = b.get_ngpt();
        std::unique_ptr<Optical_props_arry_gpu> ops = std::make_unique<Optical_props_1scl_gpu>(ncol, nlay, b);
        Source_func_lw_gpu src(ncol, nlay, b);
        const size_t n3 = size_t(ncol) * nlay * ngpt, n2 = size_t(ncol) * ngpt;
        cudaMemcpy(ops->get_tau().ptr(), tau, n3 * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(src.get_lay_source().ptr(), lay_src, n3 * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(src.get_lev_source_inc().ptr(), lev_inc, n3 * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(src.get_lev_source_dec().ptr(), lev_dec, n3 * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(src.get_sfc_source().ptr(), sfc_src, n2 * 8, cudaMemcpyHostToDevice);
        auto emis = dev<double, 2>(sfc_emis, {nband, ncol});
        Array_gpu<double, 3> up({ncol, nlay + 1, ngpt}), dn({ncol, nlay + 1, ngpt});
        Rte_lw_gpu rte;
        rte.rte_lw(ops, top_at_1, src, emis, Array_gpu<double, 2>(), up, dn, 1);
        out(up, flux_up);
        out(dn, flux_dn);
    });
}

// Rte_sw_gpu::rte_sw (src_cuda/Rte_sw.cu:116-161).
int ref_rte_sw(int ncol, int nlay, int nband, const int* band_lims, int top_at_1, const double* tau,
               const double* ssa, const double* g, const double* mu0, const double* inc_dir,
               const double* alb_dir, const double* alb_dif, double* flux_up, double* flux_dn, double* flux_dir)
{
    return guarded([&] {
        Optical_props_gpu b = bands_of(nband, band_lims);
        const int ngpt = b.get_ngpt();
        std::unique_ptr<Optical_props_arry_gpu> ops = std::make_unique<Optical_props_2str_gpu>(ncol, nlay, b);
        const size_t n3 = size_t(ncol) * nlay * ngpt;
        cudaMemcpy(ops->get_tau().ptr(), tau, n3 * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(ops->get_ssa().ptr(), ssa, n3 * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(ops->get_g().ptr(), g, n3 * 8, cudaMemcpyHostToDevice);
        auto m0 = dev<double, 1>(mu0, {ncol});
        auto inc = dev<double, 2>(inc_dir, {ncol, ngpt});
        auto ad = dev<double, 2>(alb_dir, {nband, ncol});
        auto af = dev<double, 2>(alb_dif, {nband, ncol});
        Array_gpu<double, 3> up({ncol, nlay + 1, ngpt}), dn({ncol, nlay + 1, ngpt}), dr({ncol, nlay + 1, ngpt});
        Rte_sw_gpu rte;
        rte.rte_sw(ops, top_at_1, m0, inc, ad, af, Array_gpu<double, 2>(), up, dn, dr);
        out(up, flux_up);
        out(dn, flux_dn);
        out(dr, flux_dir);
    });
}

// Fluxes_broadband_gpu::reduce (3-array overload) and Fluxes_byband_gpu::reduce
// (src_cuda/Fluxes.cu:39-136).
int ref_fluxes(int ncol, int nlev, int nband, const int* band_lims, const double* up, const double* dn,
               const double* dir, double* bb_up, double* bb_dn, double* bb_dir, double* bb_net, double* bnd_up,
               double* bnd_dn, double* bnd_net)
{
    return guarded([&] {
        Optical_props_gpu b = bands_of(nband, band_lims);
        const int ngpt = b.get_ngpt();
        std::unique_ptr<Optical_props_arry_gpu> ops = std::make_unique<Optical_props_1scl_gpu>(ncol, nlev - 1, b);
        auto u = dev<double, 3>(up, {ncol, nlev, ngpt});
        auto d = dev<double, 3>(dn, {ncol, nlev, ngpt});
        auto r = dev<double, 3>(dir, {ncol, nlev, ngpt});
        Fluxes_broadband_gpu fb(ncol, nlev);
        fb.reduce(u, d, r, ops, true);
        out(fb.get_flux_up(), bb_up);
        out(fb.get_flux_dn(), bb_dn);
        out(fb.get_flux_dn_dir(), bb_dir);
        out(fb.get_flux_net(), bb_net);
        Fluxes_byband_gpu fy(ncol, nlev, nband);
        fy.reduce(u, d, ops, true);
        out(fy.get_bnd_flux_up(), bnd_up);
        out(fy.get_bnd_flux_dn(), bnd_dn);
        out(fy.get_bnd_flux_net(), bnd_net);
    });
}

// Aerosol_optics_gpu::aerosol_optics (src_cuda/Aerosol_optics.cu:220-279), tables as
// load_and_init_aerosol_optics builds them (src_test/Radiation_solver.cu:366-401: netCDF order
// read into Fortran-order arrays of the reversed dimensions, band_lims_wvn left zero).
int ref_aerosol_optics(const rrtmgp_b200_aerosol_tables* t, const rrtmgp_b200_gas_conc* aer, int naer, int ncol,
                       int nlay, const double* rh, const double* plev, double* tau, double* ssa, double* g)
{
    return guarded([&] {
        const int nb = t->nband, nh = t->nhum, npl = t->nphilic, nph = t->nphobic;
        Array<double, 2> band_lims({2, nb});
        auto rhu = host<double, 1>(t->rh_upper, {nh});
        auto mp = host<double, 2>(t->mext_phobic, {nb, nph});
        auto sp = host<double, 2>(t->ssa_phobic, {nb, nph});
        auto gp = host<double, 2>(t->g_phobic, {nb, nph});
        auto ml = host<double, 3>(t->mext_philic, {nb, nh, npl});
        auto sl = host<double, 3>(t->ssa_philic, {nb, nh, npl});
        auto gl = host<double, 3>(t->g_philic, {nb, nh, npl});
        Aerosol_optics_gpu ao(band_lims, rhu, mp, sp, gp, ml, sl, gl);
        Gas_concs gc = gas_concs(aer, naer, ncol, nlay);
        Gas_concs_gpu gcg(gc);
        Optical_props_2str_gpu ops(ncol, nlay, ao);
        auto r = dev<double, 2>(rh, {ncol, nlay});
        auto pl = dev<double, 2>(plev, {ncol, nlay + 1});
        ao.aerosol_optics(gcg, r, pl, ops);
        out(ops.get_tau(), tau);
        out(ops.get_ssa(), ssa);
        out(ops.get_g(), g);
    });
}


// Times the reference's all-sky forward on the GPU the way its test driver runs it
// (Radiation_solver_longwave/shortwave::solve_gpu, src_test/Radiation_solver.cu:419-950):
// columns in blocks of ncol_block; per block the column subsets of the inputs, get_col_dry,
// gas_optics, cloud_optics (LW 1scl; SW 2str + delta_scale) added by band, rte_lw / rte_sw
// and Fluxes_broadband::reduce.  The k-distributions, cloud tables and input arrays are
// built once, outside the timing (the driver keeps them in its solver objects).  One
// untimed warm-up step, then nsteps timed with CUDA events per domain; ms_lw, ms_sw are the
// mean times per step.  The broadband fluxes of the last step go to the (ncol, nlev) outputs
// (NULL to skip).  tsi scaling is 1.
int ref_time_forward(const rrtmgp_b200_kdist_tables* tlw, const rrtmgp_b200_kdist_tables* tsw,
                     const rrtmgp_b200_cloud_tables* clw, const rrtmgp_b200_cloud_tables* csw,
                     const rrtmgp_b200_gas_conc* gases, int ngases, int ncol, int nlay, int ncol_block,
                     const double* play, const double* plev, const double* tlay, const double* tlev,
                     const double* tsfc, const double* emis, const double* mu0, const double* alb_dir,
                     const double* alb_dif, const double* lwp, const double* iwp, const double* rel,
                     const double* rei, int nsteps, double* ms_lw, double* ms_sw, double* lw_up, double* lw_dn,
                     double* sw_up, double* sw_dn)
{
    return guarded([&] {
        const int nlev = nlay + 1;
        Gas_concs gc = gas_concs(gases, ngases, ncol, nlay);
        Gas_concs_gpu gcg(gc);
        auto klw = make_kdist(tlw, gcg);
        auto ksw = make_kdist(tsw, gcg);
        Cloud_optics_gpu colw = make_cloud(clw), cosw = make_cloud(csw);
        const int nblw = klw->get_nband(), nbsw = ksw->get_nband();
        const auto P = dev<double, 2>(play, {ncol, nlay});
        const auto PL = dev<double, 2>(plev, {ncol, nlev});
        const auto TL = dev<double, 2>(tlay, {ncol, nlay});
        const auto TV = dev<double, 2>(tlev, {ncol, nlev});
        const auto TS = dev<double, 1>(tsfc, {ncol});
        const auto EM = dev<double, 2>(emis, {nblw, ncol});
        const auto M0 = dev<double, 1>(mu0, {ncol});
        const auto AD = dev<double, 2>(alb_dir, {nbsw, ncol});
        const auto AF = dev<double, 2>(alb_dif, {nbsw, ncol});
        const auto LW = dev<double, 2>(lwp, {ncol, nlay});
        const auto IW = dev<double, 2>(iwp, {ncol, nlay});
        const auto RL = dev<double, 2>(rel, {ncol, nlay});
        const auto RI = dev<double, 2>(rei, {ncol, nlay});
        const Bool top_at_1 = play[0] < play[size_t(nlay - 1) * ncol];
        Rte_lw_gpu rte_lw;
        Rte_sw_gpu rte_sw;
        cudaEvent_t e0, e1, e2;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventCreate(&e2);
        double tot_lw = 0., tot_sw = 0.;
        for (int step = 0; step <= nsteps; ++step) {
            const bool last = step == nsteps;
            cudaEventRecord(e0);
            for (int c0 = 0; c0 < ncol; c0 += ncol_block) {
                const int nb = std::min(ncol_block, ncol - c0), cs = c0 + 1, ce = c0 + nb;
                Gas_concs_gpu gsub(gcg, cs, nb);
                auto pl = PL.subset({{{cs, ce}, {1, nlev}}});
                Array_gpu<double, 2> cd({nb, nlay});
                Gas_optics_rrtmgp_gpu::get_col_dry(cd, gsub.get_vmr("h2o"), pl);
                std::unique_ptr<Optical_props_arry_gpu> ops = std::make_unique<Optical_props_1scl_gpu>(nb, nlay, *klw);
                Source_func_lw_gpu src(nb, nlay, *klw);
                klw->gas_optics(P.subset({{{cs, ce}, {1, nlay}}}), pl, TL.subset({{{cs, ce}, {1, nlay}}}),
                                TS.subset({{{cs, ce}}}), gsub, ops, src, cd, TV.subset({{{cs, ce}, {1, nlev}}}));
                Optical_props_1scl_gpu cop(nb, nlay, colw);
                colw.cloud_optics(LW.subset({{{cs, ce}, {1, nlay}}}), IW.subset({{{cs, ce}, {1, nlay}}}),
                                  RL.subset({{{cs, ce}, {1, nlay}}}), RI.subset({{{cs, ce}, {1, nlay}}}), cop);
                add_to(dynamic_cast<Optical_props_1scl_gpu&>(*ops), cop);
                Array_gpu<double, 3> up({nb, nlev, klw->get_ngpt()}), dn({nb, nlev, klw->get_ngpt()});
                rte_lw.rte_lw(ops, top_at_1, src, EM.subset({{{1, nblw}, {cs, ce}}}), Array_gpu<double, 2>(), up, dn, 1);
                Fluxes_broadband_gpu fl(nb, nlev);
                fl.reduce(up, dn, ops, top_at_1);
                if (last && lw_up && lw_dn) {
                    cudaDeviceSynchronize();
                    for (int l = 0; l < nlev; ++l) {
                        cudaMemcpy(lw_up + size_t(l) * ncol + c0, fl.get_flux_up().ptr() + size_t(l) * nb, nb * 8,
                                   cudaMemcpyDeviceToHost);
                        cudaMemcpy(lw_dn + size_t(l) * ncol + c0, fl.get_flux_dn().ptr() + size_t(l) * nb, nb * 8,
                                   cudaMemcpyDeviceToHost);
                    }
                }
            }
            cudaEventRecord(e1);
            for (int c0 = 0; c0 < ncol; c0 += ncol_block) {
                const int nb = std::min(ncol_block, ncol - c0), cs = c0 + 1, ce = c0 + nb;
                Gas_concs_gpu gsub(gcg, cs, nb);
                auto pl = PL.subset({{{cs, ce}, {1, nlev}}});
                Array_gpu<double, 2> cd({nb, nlay});
                Gas_optics_rrtmgp_gpu::get_col_dry(cd, gsub.get_vmr("h2o"), pl);
                std::unique_ptr<Optical_props_arry_gpu> ops = std::make_unique<Optical_props_2str_gpu>(nb, nlay, *ksw);
                Array_gpu<double, 2> toa({nb, ksw->get_ngpt()});
                ksw->gas_optics(P.subset({{{cs, ce}, {1, nlay}}}), pl, TL.subset({{{cs, ce}, {1, nlay}}}), gsub, ops,
                                toa, cd);
                Optical_props_2str_gpu cop(nb, nlay, cosw);
                cosw.cloud_optics(LW.subset({{{cs, ce}, {1, nlay}}}), IW.subset({{{cs, ce}, {1, nlay}}}),
                                  RL.subset({{{cs, ce}, {1, nlay}}}), RI.subset({{{cs, ce}, {1, nlay}}}), cop);
                cop.delta_scale();
                add_to(dynamic_cast<Optical_props_2str_gpu&>(*ops), cop);
                const int ng = ksw->get_ngpt();
                Array_gpu<double, 3> up({nb, nlev, ng}), dn({nb, nlev, ng}), dr({nb, nlev, ng});
                rte_sw.rte_sw(ops, top_at_1, M0.subset({{{cs, ce}}}), toa, AD.subset({{{1, nbsw}, {cs, ce}}}),
                              AF.subset({{{1, nbsw}, {cs, ce}}}), Array_gpu<double, 2>(), up, dn, dr);
                Fluxes_broadband_gpu fl(nb, nlev);
                fl.reduce(up, dn, dr, ops, top_at_1);
                if (last && sw_up && sw_dn) {
                    cudaDeviceSynchronize();
                    for (int l = 0; l < nlev; ++l) {
                        cudaMemcpy(sw_up + size_t(l) * ncol + c0, fl.get_flux_up().ptr() + size_t(l) * nb, nb * 8,
                                   cudaMemcpyDeviceToHost);
                        cudaMemcpy(sw_dn + size_t(l) * ncol + c0, fl.get_flux_dn().ptr() + size_t(l) * nb, nb * 8,
                                   cudaMemcpyDeviceToHost);
                    }
                }
            }
            cudaEventRecord(e2);
            cudaEventSynchronize(e2);
            float a = 0.f, b = 0.f;
            cudaEventElapsedTime(&a, e0, e1);
            cudaEventElapsedTime(&b, e1, e2);
            if (step > 0 && !last) { tot_lw += a; tot_sw += b; }
            if (step == 0 && nsteps == 0) { tot_lw = a; tot_sw = b; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(e2);
        const int n = std::max(nsteps - 1, 1);
        *ms_lw = tot_lw / n;
        *ms_sw = tot_sw / n;
    });
}

}  // extern "C"
