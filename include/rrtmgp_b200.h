/*
 * rrtmgp_b200.h -- C ABI of the B200 column-radiation hot path (RTE+RRTMGP).
 *
 * Plain C: opaque handles, plain pointers and sizes, an int status return, a cudaStream_t
 * passed as void*.  Every array argument of a compute entry point is a DEVICE pointer in
 * the reference's layout: Fortran order with the column index fastest, i.e. the flat
 * memory of the reference's Array_gpu<Float,N> (include/Array.h:41-63 of rte-rrtmgp-cpp):
 *
 *   (ncol, nlay)        p_lay, t_lay, col_dry, vmr fields, lwp, iwp, re_liq, re_ice
 *   (ncol, nlev)        p_lev, t_lev, broadband fluxes
 *   (ncol, nlay, ngpt)  tau, ssa, g, Planck sources      (ngpt may be nband for clouds)
 *   (ncol, nlev, ngpt)  g-point fluxes
 *   (ncol, ngpt)        surface sources, toa_src, incident fluxes
 *   (nband, ncol)       sfc_emis, sfc_alb_dir, sfc_alb_dif (band fastest, as the reference)
 *
 * Entry points come in _f32 (the product arithmetic) and _f64 (same kernels instantiated in
 * double: the "plain FP64 GPU forward" baseline) variants.  Nothing here allocates device
 * memory inside a compute call: tables live in handles created once, temporaries come from
 * a caller-supplied workspace whose size a *_workspace_bytes() query returns.  No call
 * synchronises the stream; errors in arguments are reported synchronously by the status
 * code and rrtmgp_b200_last_error().
 *
 * Each declaration names the reference interface it replaces (file:line in rte-rrtmgp-cpp).
 */
#ifndef RRTMGP_B200_H
#define RRTMGP_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RRTMGP_B200_ABI_VERSION 1

enum rrtmgp_b200_status {
    RRTMGP_B200_OK = 0,
    RRTMGP_B200_ERR_ARG = 1,          /* null pointer, bad shape, bad enum             */
    RRTMGP_B200_ERR_RANGE = 2,        /* input outside the table range (range check)   */
    RRTMGP_B200_ERR_MISSING_GAS = 3,  /* key species or h2o absent                     */
    RRTMGP_B200_ERR_CUDA = 4,         /* CUDA runtime error (launch / copy)            */
    RRTMGP_B200_ERR_ALLOC = 5,        /* allocation failed at handle creation          */
    RRTMGP_B200_ERR_UNSUPPORTED = 6,  /* option not supported                          */
    RRTMGP_B200_ERR_WORKSPACE = 7     /* caller workspace missing or too small         */
};

/* Message of the last failing call on this host thread ("" if none). */
const char* rrtmgp_b200_last_error(void);
int rrtmgp_b200_abi_version(void);

/* ------------------------------------------------------------------------------------ */
/* Coefficient tables, as read from an RRTMGP k-distribution netCDF file.                */
/* Replaces the 35-argument constructors Gas_optics_rrtmgp_gpu::Gas_optics_rrtmgp_gpu    */
/* (include/Gas_optics_rrtmgp.h:293-364) fed by load_and_init_gas_optics                 */
/* (src_test/Radiation_solver.cpp:70-284).  Host pointers, double, C order = netCDF     */
/* dimension order (the memory the reference's Array<Float,N> holds after reading).      */
/* ------------------------------------------------------------------------------------ */
typedef struct rrtmgp_b200_kdist_tables {
    int ngas;                /* absorber                                                 */
    int nband, ngpt;         /* bnd, gpt                                                 */
    int ntemp, npres, neta;  /* temperature, pressure, mixing_fraction                  */
    int nminor_absorber;     /* minor_absorber                                           */
    int nint_lower, nint_upper;           /* minor_absorber_intervals_lower/upper        */
    int ncontrib_lower, ncontrib_upper;   /* contributors_lower/upper                    */
    int nplanck_temp;        /* temperature_Planck (0 for a shortwave file)              */

    const char* const* gas_names;          /* [ngas]                                     */
    const int* key_species;                /* (nband, 2 atmos_layer, 2 pair), 1-based    */
    const int* band_lims_gpt;              /* (nband, 2), 1-based inclusive, covering    */
                                           /* 1..ngpt in order without gaps              */
    const double* band_lims_wvn;           /* (nband, 2)                                 */
    const double* press_ref;               /* [npres], Pa, decreasing                    */
    double press_ref_trop;
    const double* temp_ref;                /* [ntemp], K, increasing                     */
    double temp_ref_p, temp_ref_t;
    const double* vmr_ref;                 /* (ntemp, ngas+1, 2); index 0 = dry air      */
    const double* kmajor;                  /* (ntemp, npres+1, neta, ngpt)               */
    const double* kminor_lower;            /* (ntemp, neta, ncontrib_lower)              */
    const double* kminor_upper;            /* (ntemp, neta, ncontrib_upper)              */
    const char* const* gas_minor;          /* [nminor_absorber]                          */
    const char* const* identifier_minor;   /* [nminor_absorber]                          */
    const char* const* minor_gases_lower;  /* [nint_lower]                               */
    const char* const* minor_gases_upper;  /* [nint_upper]                               */
    const int* minor_limits_gpt_lower;     /* (nint_lower, 2), 1-based                   */
    const int* minor_limits_gpt_upper;     /* (nint_upper, 2)                            */
    const int* minor_scales_with_density_lower;  /* [nint_lower] 0/1                     */
    const int* minor_scales_with_density_upper;
    const char* const* scaling_gas_lower;  /* [nint_lower] ("" = none)                   */
    const char* const* scaling_gas_upper;
    const int* scale_by_complement_lower;  /* [nint_lower] 0/1                           */
    const int* scale_by_complement_upper;
    const int* kminor_start_lower;         /* [nint_lower], 1-based                      */
    const int* kminor_start_upper;
    /* longwave only (NULL for shortwave) */
    const double* totplnk;                 /* (nband, nplanck_temp)                      */
    const double* planck_frac;             /* (ntemp, npres+1, neta, ngpt)               */
    /* shortwave only (NULL for longwave) */
    const double* solar_source_quiet;      /* [ngpt]                                     */
    const double* solar_source_facular;    /* [ngpt]                                     */
    const double* solar_source_sunspot;    /* [ngpt]                                     */
    double tsi_default, mg_default, sb_default;
    const double* rayl_lower;              /* (ntemp, neta, ngpt) or NULL                */
    const double* rayl_upper;              /* (ntemp, neta, ngpt) or NULL                */
} rrtmgp_b200_kdist_tables;

typedef struct rrtmgp_b200_kdist_t* rrtmgp_b200_kdist;
typedef struct rrtmgp_b200_cloud_t* rrtmgp_b200_cloud;
typedef struct rrtmgp_b200_bands_t* rrtmgp_b200_bands;

/* Gas_optics_rrtmgp_gpu ctor + init_abs_coeffs (src/Gas_optics_rrtmgp.cpp:391-742,
 * src_cuda/Gas_optics_rrtmgp.cu:427-803): keeps the gases also listed in available_gases,
 * drops absent minor absorbers, builds flavors/gpoint_flavor, re-lays the tables out
 * g-point fastest in FP32 and FP64 on the current device.  Errors: MISSING_GAS when a key
 * species is not available ("Gas optics: required gas X is missing", :241-243); ARG for
 * missing tables, more than 32 g-points in a band, or band limits that do not cover
 * 1..ngpt in order without gaps (checked before any device allocation). */
int rrtmgp_b200_kdist_create(const rrtmgp_b200_kdist_tables* tables,
                             const char* const* available_gases, int n_available,
                             rrtmgp_b200_kdist* out);
void rrtmgp_b200_kdist_destroy(rrtmgp_b200_kdist k);

typedef struct rrtmgp_b200_kdist_info {
    int ngas, nflav, nband, ngpt, ntemp, npres, neta, nplanck_temp;
    int nminor_lower, nminor_upper;        /* after reduction                            */
    int is_longwave;                        /* source_is_internal()                       */
    int has_rayleigh;
    double press_ref_min, press_ref_max;   /* get_press_ref_min/max (Gas_optics_rrtmgp.h) */
    double temp_ref_min, temp_ref_max;     /* get_temp_min/max                           */
    double tsi;                             /* get_tsi() (Gas_optics_rrtmgp.cpp:1347-1356) */
} rrtmgp_b200_kdist_info;
int rrtmgp_b200_kdist_get_info(rrtmgp_b200_kdist k, rrtmgp_b200_kdist_info* info);
/* Name of reduced gas i (0-based) into buf. */
int rrtmgp_b200_kdist_gas_name(rrtmgp_b200_kdist k, int i, char* buf, int buflen);
/* Band/g-point discretisation of the k-distribution (Optical_props_gpu base). */
rrtmgp_b200_bands rrtmgp_b200_kdist_bands(rrtmgp_b200_kdist k);
/* set_solar_variability (Gas_optics_rrtmgp.cpp:745-760); SW only. */
int rrtmgp_b200_kdist_set_solar_variability(rrtmgp_b200_kdist k, double mg_index, double sb_index);
/* Host copy of solar_source [ngpt] (double); SW only. */
int rrtmgp_b200_kdist_solar_source(rrtmgp_b200_kdist k, double* out_host);

/* Band / g-point discretisation: Optical_props_gpu(band_lims_wvn, band_lims_gpt)
 * (include/Optical_props.h:176-211).  band_lims_gpt host (nband, 2), 1-based. */
int rrtmgp_b200_bands_create(int nband, const int* band_lims_gpt_host, rrtmgp_b200_bands* out);
void rrtmgp_b200_bands_destroy(rrtmgp_b200_bands b);
int rrtmgp_b200_bands_get(rrtmgp_b200_bands b, int* nband, int* ngpt);

/* Gas concentration entry: the reference's Gas_concs_gpu map name -> Array_gpu<Float,2>
 * (include/Gas_concs.h:67-91).  dim1 x dim2 = 1x1 (scalar), 1 x nlay (profile) or
 * ncol x nlay (field), column fastest; vmr is a device pointer of the call's precision. */
typedef struct rrtmgp_b200_gas_conc {
    const char* name;
    const void* vmr;
    int dim1, dim2;
} rrtmgp_b200_gas_conc;

/* ------------------------------------------------------------------------------------ */
/* Gas optics                                                                            */
/* ------------------------------------------------------------------------------------ */
/* Gas_optics_rrtmgp_gpu::get_col_dry (src_cuda/Gas_optics_rrtmgp.cu:806-903). */
int rrtmgp_b200_get_col_dry_f32(int ncol, int nlay, const float* vmr_h2o, const float* plev,
                                float* col_dry, void* stream);
int rrtmgp_b200_get_col_dry_f64(int ncol, int nlay, const double* vmr_h2o, const double* plev,
                                double* col_dry, void* stream);

/* Longwave gas_optics (include/Gas_optics_rrtmgp.h:389-398; src_cuda/Gas_optics_rrtmgp.cu
 * :907-943 + compute_gas_taus :980-1148 + source :1167-1202).  col_dry may be NULL (then
 * computed in-kernel from h2o and plev exactly as get_col_dry).  Outputs: tau, lay_src,
 * lev_src_inc, lev_src_dec (ncol,nlay,ngpt); sfc_src, sfc_src_jac (ncol,ngpt). */
int rrtmgp_b200_gas_optics_lw_f32(rrtmgp_b200_kdist k, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* tsfc,
        const float* tlev, const float* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases,
        float* tau, float* lay_src, float* lev_src_inc, float* lev_src_dec,
        float* sfc_src, float* sfc_src_jac, void* stream);
int rrtmgp_b200_gas_optics_lw_f64(rrtmgp_b200_kdist k, int ncol, int nlay,
        const double* play, const double* plev, const double* tlay, const double* tsfc,
        const double* tlev, const double* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases,
        double* tau, double* lay_src, double* lev_src_inc, double* lev_src_dec,
        double* sfc_src, double* sfc_src_jac, void* stream);

/* Shortwave gas_optics (include/Gas_optics_rrtmgp.h:400-408; Gas_optics_rrtmgp.cu:947-977).
 * Outputs tau, ssa, g (ncol,nlay,ngpt) and toa_src (ncol,ngpt) = solar_source spread. */
int rrtmgp_b200_gas_optics_sw_f32(rrtmgp_b200_kdist k, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases,
        float* tau, float* ssa, float* g, float* toa_src, void* stream);
int rrtmgp_b200_gas_optics_sw_f64(rrtmgp_b200_kdist k, int ncol, int nlay,
        const double* play, const double* plev, const double* tlay, const double* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases,
        double* tau, double* ssa, double* g, double* toa_src, void* stream);

/* Range check of Gas_optics_rrtmgp::gas_optics (src/Gas_optics_rrtmgp.cpp:812-827), which
 * the reference GPU path skips.  tlev/tsfc may be NULL (shortwave).  Synchronises the
 * stream; returns RRTMGP_B200_ERR_RANGE with the failing field named in last_error. */
int rrtmgp_b200_check_range_f32(rrtmgp_b200_kdist k, int ncol, int nlay, const float* play,
        const float* plev, const float* tlay, const float* tlev, const float* tsfc,
        const float* col_dry, void* stream);
int rrtmgp_b200_check_range_f64(rrtmgp_b200_kdist k, int ncol, int nlay, const double* play,
        const double* plev, const double* tlay, const double* tlev, const double* tsfc,
        const double* col_dry, void* stream);

/* ------------------------------------------------------------------------------------ */
/* Cloud optics: Cloud_optics_gpu (include/Cloud_optics.h:80-131; src_cuda/Cloud_optics.cu) */
/* ------------------------------------------------------------------------------------ */
typedef struct rrtmgp_b200_cloud_tables {
    int nband, nsize_liq, nsize_ice, nrghice;
    const double* band_lims_wvn;     /* (nband, 2)                                        */
    double radliq_lwr, radliq_upr, radliq_fac;
    double radice_lwr, radice_upr, radice_fac;
    const double* lut_extliq;        /* (nband, nsize_liq)                                */
    const double* lut_ssaliq;
    const double* lut_asyliq;
    const double* lut_extice;        /* (nrghice, nband, nsize_ice)                       */
    const double* lut_ssaice;
    const double* lut_asyice;
} rrtmgp_b200_cloud_tables;

/* Cloud_optics_gpu ctor (src_cuda/Cloud_optics.cu:130-179): ice roughness icergh = 2. */
int rrtmgp_b200_cloud_create(const rrtmgp_b200_cloud_tables* t, rrtmgp_b200_cloud* out);
void rrtmgp_b200_cloud_destroy(rrtmgp_b200_cloud c);

/* cloud_optics 1scl (Cloud_optics.cu:257-329): tau (ncol,nlay,nband) = absorption tau. */
int rrtmgp_b200_cloud_optics_1scl_f32(rrtmgp_b200_cloud c, int ncol, int nlay,
        const float* clwp, const float* ciwp, const float* reliq, const float* reice,
        float* tau, void* stream);
int rrtmgp_b200_cloud_optics_1scl_f64(rrtmgp_b200_cloud c, int ncol, int nlay,
        const double* clwp, const double* ciwp, const double* reliq, const double* reice,
        double* tau, void* stream);
/* cloud_optics 2str (Cloud_optics.cu:181-253): tau, ssa, g (ncol,nlay,nband). */
int rrtmgp_b200_cloud_optics_2str_f32(rrtmgp_b200_cloud c, int ncol, int nlay,
        const float* clwp, const float* ciwp, const float* reliq, const float* reice,
        float* tau, float* ssa, float* g, void* stream);
int rrtmgp_b200_cloud_optics_2str_f64(rrtmgp_b200_cloud c, int ncol, int nlay,
        const double* clwp, const double* ciwp, const double* reliq, const double* reice,
        double* tau, double* ssa, double* g, void* stream);

/* ------------------------------------------------------------------------------------ */
/* Aerosol optics (shortwave, two-stream).  Replaces Aerosol_optics_gpu                  */
/* (include/Aerosol_optics.h:64-86, src_cuda/Aerosol_optics.cu:188-279) built by          */
/* load_and_init_aerosol_optics (src_test/Radiation_solver.cu:366-401).  Host tables,     */
/* double, C order = netCDF dimension order.                                              */
/* ------------------------------------------------------------------------------------ */
typedef struct rrtmgp_b200_aerosol_tables {
    int nband, nhum, nphilic, nphobic;   /* band_sw, relative_humidity, hydrophilic (>= 5),  */
                                         /* hydrophobic (>= 11)                              */
    const double* rh_upper;              /* [nhum] "relative_humidity2", increasing          */
    const double* mext_phobic;           /* (nphobic, nband) "mass_ext_sw_hydrophobic", m2/kg */
    const double* ssa_phobic;            /* (nphobic, nband)                                 */
    const double* g_phobic;              /* (nphobic, nband)                                 */
    const double* mext_philic;           /* (nphilic, nhum, nband)                           */
    const double* ssa_philic;
    const double* g_philic;
} rrtmgp_b200_aerosol_tables;

typedef struct rrtmgp_b200_aerosol_t* rrtmgp_b200_aerosol;

int rrtmgp_b200_aerosol_create(const rrtmgp_b200_aerosol_tables* t, rrtmgp_b200_aerosol* out);
void rrtmgp_b200_aerosol_destroy(rrtmgp_b200_aerosol a);

/* Aerosol_optics_gpu::aerosol_optics: tau, ssa, g (ncol, nlay, nband) of the 11 species
 * aermr01 .. aermr11 (mass mixing ratios, kg/kg: sea salt 1-3, dust 1-3, hydrophilic and
 * hydrophobic organic matter, black carbon 1-2, sulphate), passed as gas_conc entries with
 * those names and shape (1,1), (1,nlay) or (ncol,nlay); rh (ncol, nlay) relative humidity
 * as a fraction, plev (ncol, nlay+1).  Layer mass |dp| / 9.81 as the reference GPU kernel.
 * Divergence: rh above the last rh_upper entry uses the last class (the reference reads
 * past its table). */
int rrtmgp_b200_aerosol_optics_f32(rrtmgp_b200_aerosol a, int ncol, int nlay,
        const rrtmgp_b200_gas_conc* aerosols, int naerosols, const float* rh, const float* plev,
        float* tau, float* ssa, float* g, void* stream);
int rrtmgp_b200_aerosol_optics_f64(rrtmgp_b200_aerosol a, int ncol, int nlay,
        const rrtmgp_b200_gas_conc* aerosols, int naerosols, const double* rh, const double* plev,
        double* tau, double* ssa, double* g, void* stream);

/* ------------------------------------------------------------------------------------ */
/* Optical-property arithmetic (src_cuda/Optical_props.cu:93-165)                        */
/* ------------------------------------------------------------------------------------ */
/* Optical_props_2str_gpu::delta_scale with f = g^2 (optical_props_kernels.cu:139-160). */
int rrtmgp_b200_delta_scale_2str_f32(int ncol, int nlay, int ngpt, float* tau, float* ssa,
                                     float* g, void* stream);
int rrtmgp_b200_delta_scale_2str_f64(int ncol, int nlay, int ngpt, double* tau, double* ssa,
                                     double* g, void* stream);
/* add_to(Optical_props_1scl_gpu&, const Optical_props_1scl_gpu&) (Optical_props.cu:93-116):
 * ngpt_in == ngpt adds g-point by g-point, ngpt_in == nband broadcasts by band through
 * the bands' g-point limits; anything else is ERR_ARG (the reference's runtime_error). */
int rrtmgp_b200_add_to_1scl_f32(rrtmgp_b200_bands b, int ncol, int nlay, float* tau_inout,
                                const float* tau_in, int ngpt_in, void* stream);
int rrtmgp_b200_add_to_1scl_f64(rrtmgp_b200_bands b, int ncol, int nlay, double* tau_inout,
                                const double* tau_in, int ngpt_in, void* stream);
/* add_to(Optical_props_2str_gpu&, const Optical_props_2str_gpu&) (Optical_props.cu:119-145). */
int rrtmgp_b200_add_to_2str_f32(rrtmgp_b200_bands b, int ncol, int nlay,
        float* tau_inout, float* ssa_inout, float* g_inout,
        const float* tau_in, const float* ssa_in, const float* g_in, int ngpt_in, void* stream);
int rrtmgp_b200_add_to_2str_f64(rrtmgp_b200_bands b, int ncol, int nlay,
        double* tau_inout, double* ssa_inout, double* g_inout,
        const double* tau_in, const double* ssa_in, const double* g_in, int ngpt_in, void* stream);

/* ------------------------------------------------------------------------------------ */
/* Solvers                                                                               */
/* ------------------------------------------------------------------------------------ */
/* Rte_lw_gpu::rte_lw (include/Rte_lw.h:65-73; src_cuda/Rte_lw.cu:81-152) with the
 * no-scattering solver (rte_solver_kernels.cu:16-185; mo_rte_solver_kernels.F90:58-265).
 * sfc_emis (nband, ncol); inc_flux (ncol, ngpt) or NULL (zero); n_gauss_angles 1..4
 * (Gauss-Jacobi secants and weights of Rte_lw.cu:87-101; the reference GPU path supports
 * only 1).  Outputs gpt_flux_up, gpt_flux_dn (ncol, nlay+1, ngpt). */
int rrtmgp_b200_rte_lw_f32(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1,
        const float* tau, const float* lay_src, const float* lev_src_inc,
        const float* lev_src_dec, const float* sfc_src, const float* sfc_emis,
        const float* inc_flux, int n_gauss_angles, float* gpt_flux_up, float* gpt_flux_dn,
        void* stream);
int rrtmgp_b200_rte_lw_f64(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1,
        const double* tau, const double* lay_src, const double* lev_src_inc,
        const double* lev_src_dec, const double* sfc_src, const double* sfc_emis,
        const double* inc_flux, int n_gauss_angles, double* gpt_flux_up, double* gpt_flux_dn,
        void* stream);
/* The same solve with the surface-temperature Jacobian: the reference's do_jacobians path of
 * lw_solver_noscat (rte_solver_kernels.cu:56,65,82,91 and the step-3 scaling; wired through
 * src_cuda/Rte_lw.cu:125-148, where the reference disables it).  sfc_src_jac (ncol, ngpt) is
 * the gas optics' sfc_source_jac (Planck source at Tsfc + 1 K minus at Tsfc);
 * gpt_flux_up_jac (ncol, nlay+1, ngpt) receives 2 pi w sum over angles of the upward
 * radiance that the surface term sfc_emis * sfc_src_jac alone produces at every level, i.e.
 * d gpt_flux_up / d Tsfc in the reference's finite-difference form. */
int rrtmgp_b200_rte_lw_jac_f32(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1,
        const float* tau, const float* lay_src, const float* lev_src_inc,
        const float* lev_src_dec, const float* sfc_src, const float* sfc_src_jac,
        const float* sfc_emis, const float* inc_flux, int n_gauss_angles, float* gpt_flux_up,
        float* gpt_flux_dn, float* gpt_flux_up_jac, void* stream);
int rrtmgp_b200_rte_lw_jac_f64(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1,
        const double* tau, const double* lay_src, const double* lev_src_inc,
        const double* lev_src_dec, const double* sfc_src, const double* sfc_src_jac,
        const double* sfc_emis, const double* inc_flux, int n_gauss_angles, double* gpt_flux_up,
        double* gpt_flux_dn, double* gpt_flux_up_jac, void* stream);

/* No reference counterpart.  Kernels that copy their inputs with TMA tile loads wait for each
 * copy for at most 2 s; a copy that has not landed by then ends the kernel early (its outputs
 * are then incomplete) and is counted on the current device.  *count receives that count
 * since the library was loaded (0 in normal operation); the call synchronises the device. */
int rrtmgp_b200_device_wait_timeouts(unsigned int* count);

/* Rte_sw_gpu::rte_sw (include/Rte_sw.h:65-75; src_cuda/Rte_sw.cu:116-161), two-stream +
 * adding (rte_solver_kernels.cu:188-278,535-647; F90 :512-606,996-1228).  mu0 (ncol);
 * inc_flux_dir (ncol, ngpt); sfc_alb_dir/dif (nband, ncol); inc_flux_dif (ncol, ngpt) or
 * NULL.  Outputs gpt_flux_up, gpt_flux_dn (total = diffuse + direct), gpt_flux_dir
 * (ncol, nlay+1, ngpt).  workspace: device scratch of rrtmgp_b200_rte_sw_workspace_bytes()
 * bytes.  Only columns deeper than 256 layers (FP32) or 128 layers (FP64) use it; for
 * shallower ones the kernel keeps the adding recurrences on chip, the query returns 0 and
 * workspace may be NULL. */
size_t rrtmgp_b200_rte_sw_workspace_bytes(int ncol, int nlay, int ngpt, int fp64);
int rrtmgp_b200_rte_sw_f32(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1,
        const float* tau, const float* ssa, const float* g, const float* mu0,
        const float* inc_flux_dir, const float* sfc_alb_dir, const float* sfc_alb_dif,
        const float* inc_flux_dif, float* gpt_flux_up, float* gpt_flux_dn, float* gpt_flux_dir,
        void* workspace, size_t workspace_bytes, void* stream);
/* rte_sw (FP32) that also returns the flux every layer absorbs (no reference counterpart):
 * layer_abs (ncol, nlay, ngpt), laid out as tau, receives per g-point
 * F_dir(top)(1 - Tn - Rdir - Tdir) + (F_dn(top) - F_dir(top) + F_up(bottom))(1 - R - T) with the
 * solver's own two-stream terms, for rrtmgp_b200_heating_rate_from_layer_abs_f32.  The fluxes
 * are those of rrtmgp_b200_rte_sw_f32.  Columns of up to 128 layers; deeper ones return
 * RRTMGP_B200_ERR_UNSUPPORTED (use rte_sw and heating_rate_sw_layers).  No workspace. */
int rrtmgp_b200_rte_sw_abs_f32(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1,
        const float* tau, const float* ssa, const float* g, const float* mu0,
        const float* inc_flux_dir, const float* sfc_alb_dir, const float* sfc_alb_dif,
        const float* inc_flux_dif, float* gpt_flux_up, float* gpt_flux_dn, float* gpt_flux_dir,
        float* layer_abs, void* stream);
int rrtmgp_b200_rte_sw_f64(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1,
        const double* tau, const double* ssa, const double* g, const double* mu0,
        const double* inc_flux_dir, const double* sfc_alb_dir, const double* sfc_alb_dif,
        const double* inc_flux_dif, double* gpt_flux_up, double* gpt_flux_dn,
        double* gpt_flux_dir, void* workspace, size_t workspace_bytes, void* stream);

/* Shortwave solver that allocates nothing and needs no workspace argument.  No counterpart
 * in the reference.  It is for callers that cannot obtain device memory themselves -- for
 * example a Fortran or C host model bound through this ABI whose device memory is owned by
 * its OpenACC/OpenMP runtime or by a fixed memory plan, where an extra cudaMalloc is not
 * available or would synchronise the device.  Same arguments and results as
 * rrtmgp_b200_rte_sw_f32 minus the workspace; the scratch is a 16 MiB array compiled into
 * this library, which every GPU that loads the library holds until the process exits.
 * Limit: ncol * nlay * ngpt <= RRTMGP_B200_SW_STATIC_SCRATCH_MAX_ELEMS, else
 * RRTMGP_B200_ERR_WORKSPACE and nothing is launched (split the columns into smaller calls).
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before any stream capture.  The address is kept
 * per device ordinal for the life of the process and belongs to the context that was current
 * at that first call (normally the device's primary context, which the CUDA runtime uses):
 * it does not survive cudaDeviceReset, and a caller that makes another context current must
 * not use this entry point.  All calls share the
 * one array, so calls that overlap on the GPU (concurrent streams, or several host threads)
 * race and must be serialised by the caller.  No slot of the scratch needs to start at zero:
 * each call writes every slot it reads. */
#define RRTMGP_B200_SW_STATIC_SCRATCH_MAX_ELEMS (1048576)
int rrtmgp_b200_rte_sw_static_scratch_f32(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1,
        const float* tau, const float* ssa, const float* g, const float* mu0,
        const float* inc_flux_dir, const float* sfc_alb_dir, const float* sfc_alb_dif,
        const float* inc_flux_dif, float* gpt_flux_up, float* gpt_flux_dn, float* gpt_flux_dir,
        void* stream);

/* ------------------------------------------------------------------------------------ */
/* Flux reductions (src_cuda/Fluxes.cu:39-136; fluxes_kernels.cu:26-113)                 */
/* ------------------------------------------------------------------------------------ */
/* Fluxes_broadband_gpu::reduce: sums over g (compensated), net = dn - up.  gpt_flux_dn_dir
 * and flux_dn_dir may be NULL (the 2-array overload). */
int rrtmgp_b200_fluxes_broadband_f32(int ncol, int nlev, int ngpt, const float* gpt_flux_up,
        const float* gpt_flux_dn, const float* gpt_flux_dn_dir, float* flux_up, float* flux_dn,
        float* flux_dn_dir, float* flux_net, void* stream);
int rrtmgp_b200_fluxes_broadband_f64(int ncol, int nlev, int ngpt, const double* gpt_flux_up,
        const double* gpt_flux_dn, const double* gpt_flux_dn_dir, double* flux_up,
        double* flux_dn, double* flux_dn_dir, double* flux_net, void* stream);
/* Fluxes_byband_gpu::reduce: band sums over band_lims_gpt(1,b)..band_lims_gpt(2,b)
 * inclusive, as mo_fluxes_byband_kernels.F90:21-79 (the reference CUDA kernel
 * fluxes_kernels.cu:78-86 starts one g-point late).  Outputs (ncol, nlev, nband); the
 * dn_dir pair may be NULL. */
int rrtmgp_b200_fluxes_byband_f32(rrtmgp_b200_bands b, int ncol, int nlev,
        const float* gpt_flux_up, const float* gpt_flux_dn, const float* gpt_flux_dn_dir,
        float* bnd_flux_up, float* bnd_flux_dn, float* bnd_flux_dn_dir, float* bnd_flux_net,
        void* stream);
int rrtmgp_b200_fluxes_byband_f64(rrtmgp_b200_bands b, int ncol, int nlev,
        const double* gpt_flux_up, const double* gpt_flux_dn, const double* gpt_flux_dn_dir,
        double* bnd_flux_up, double* bnd_flux_dn, double* bnd_flux_dn_dir,
        double* bnd_flux_net, void* stream);
/* Heating rate [K/day] per layer from broadband fluxes (no reference counterpart):
 * HR(l) = g0 / cp_dry * (Fnet(l) - Fnet(l+1)) / (p(l+1) - p(l)) * 86400, i.e. the net
 * downward flux converging in the layer over its mass, for either vertical orientation;
 * Fnet = dn - up, g0 = 9.80665 m s-2, cp_dry = 1004.64 J kg-1 K-1. */
int rrtmgp_b200_heating_rate_f32(int ncol, int nlay, const float* flux_up, const float* flux_dn,
        const float* plev, float* heating_rate, void* stream);
int rrtmgp_b200_heating_rate_f64(int ncol, int nlay, const double* flux_up,
        const double* flux_dn, const double* plev, double* heating_rate, void* stream);
/* Heating rates from per-layer absorbed flux (no reference counterpart; the reference leaves
 * heating rates to the caller): the per-stage solvers' layer terms are recomputed from their
 * inputs and the absorbed flux sum_g A_g is accumulated in FP64, so FP32 inputs keep their
 * accuracy in layers of ~0.1 Pa where a difference of FP32 level fluxes loses ~1 K/day.
 * Longwave (one angle, as rte_lw with n_gauss_angles = 1): A_g = (1 - T)(F_dn(top) +
 * F_up(bottom)) - pi (S_dn + S_up) from tau and the Planck sources; shortwave: A_g =
 * F_dir(top)(1 - Tn - Rdir - Tdir) + (F_dn(top) - F_dir(top) + F_up(bottom))(1 - R - T) from
 * tau, ssa, g and mu0.  g-point arrays as rte_lw / rte_sw; heating_rate (ncol, nlay) K/day. */
int rrtmgp_b200_heating_rate_lw_layers_f32(int ncol, int nlay, int ngpt, int top_at_1,
        const float* tau, const float* lay_src, const float* lev_src_inc, const float* lev_src_dec,
        const float* gpt_flux_up, const float* gpt_flux_dn, const float* plev, float* heating_rate,
        void* stream);
int rrtmgp_b200_heating_rate_lw_layers_f64(int ncol, int nlay, int ngpt, int top_at_1,
        const double* tau, const double* lay_src, const double* lev_src_inc,
        const double* lev_src_dec, const double* gpt_flux_up, const double* gpt_flux_dn,
        const double* plev, double* heating_rate, void* stream);
int rrtmgp_b200_heating_rate_sw_layers_f32(int ncol, int nlay, int ngpt, int top_at_1,
        const float* tau, const float* ssa, const float* g, const float* mu0, const float* gpt_flux_up,
        const float* gpt_flux_dn, const float* gpt_flux_dir, const float* plev, float* heating_rate,
        void* stream);
int rrtmgp_b200_heating_rate_sw_layers_f64(int ncol, int nlay, int ngpt, int top_at_1,
        const double* tau, const double* ssa, const double* g, const double* mu0,
        const double* gpt_flux_up, const double* gpt_flux_dn, const double* gpt_flux_dir,
        const double* plev, double* heating_rate, void* stream);
/* Heating rate [K/day] from the per-layer absorbed flux of rrtmgp_b200_rte_sw_abs_f32 (no
 * reference counterpart): sum over g-points of layer_abs in FP64, times g0 / cp_dry * 86400,
 * over |p(l+1) - p(l)|; the same quantity as heating_rate_sw_layers without recomputing the
 * two-stream or re-reading the optical properties and g-point fluxes. */
int rrtmgp_b200_heating_rate_from_layer_abs_f32(int ncol, int nlay, int ngpt, const float* layer_abs,
        const float* plev, float* heating_rate, void* stream);

/* ------------------------------------------------------------------------------------ */
/* Fused column forward (FP32 product path)                                              */
/* ------------------------------------------------------------------------------------ */
/* Longwave column forward: the sequence of Radiation_solver_longwave::solve_gpu
 * (src_test/Radiation_solver.cu:467-615) -- gas_optics, cloud_optics (1scl, added by band;
 * skipped when cloud is NULL), rte_lw (one angle) and Fluxes_broadband::reduce -- plus heating
 * rates, in one kernel that keeps every (layer, g-point) quantity on chip.  Outputs
 * flux_up, flux_dn, flux_net (ncol, nlay+1) and heating_rate (ncol, nlay) [K/day].  The
 * vertical orientation is taken per column from play.  chunk: layers per warp (8 or 16;
 * 0 picks the tuned default).  Up to 16 chunks (16 * chunk layers) a column is one CTA; deeper
 * columns run on a thread-block cluster of ceil(chunks / 16) CTAs, nlay <= 128 * chunk. */
int rrtmgp_b200_forward_lw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud cloud, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* tlev,
        const float* tsfc, const float* col_dry, const rrtmgp_b200_gas_conc* gases, int ngases,
        const float* lwp, const float* iwp, const float* rel, const float* rei,
        const float* sfc_emis, float* flux_up, float* flux_dn, float* flux_net,
        float* heating_rate, int chunk, void* stream);
/* Shortwave column forward: the sequence of Radiation_solver_shortwave::solve_gpu
 * (src_test/Radiation_solver.cu:683-950) -- gas_optics with Rayleigh, toa_src scaled by
 * tsi_scaling (NULL: 1), cloud_optics (2str; delta-scaled when delta_cloud != 0; skipped when
 * cloud is NULL) added by band, rte_sw (two-stream + adding, no incident diffuse flux) and
 * Fluxes_broadband::reduce -- plus heating rates, in one kernel.  mu0 (ncol) > 0; surface
 * albedos (nband, ncol) in the reference's column-fastest order.  Outputs flux_up, flux_dn
 * (direct included), flux_dn_dir, flux_net (ncol, nlay+1) and heating_rate (ncol, nlay).
 * chunk: layers per warp (8 or 16; 0: 8 up to 128 layers, else 16).  Columns of more than 16
 * chunks run on a thread-block cluster of ceil(chunks / 16) CTAs; nlay <= 128 * chunk. */
int rrtmgp_b200_forward_sw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud cloud, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp,
        const float* rel, const float* rei, int delta_cloud, const float* mu0,
        const float* tsi_scaling, const float* sfc_alb_dir, const float* sfc_alb_dif,
        float* flux_up, float* flux_dn, float* flux_dn_dir, float* flux_net,
        float* heating_rate, int chunk, void* stream);
/* The same shortwave column forward with aerosols, the reference's switch_aerosol_optics
 * step (src_test/Radiation_solver.cu:794-807): Aerosol_optics_gpu::aerosol_optics of the
 * tables a (rrtmgp_b200_aerosol_create) for the mass mixing ratios aermr01 .. aermr11
 * (aerosols, naer; scalars, profiles or fields as gases) and relative humidity rh
 * (ncol, nlay), delta-scaled when delta_aerosol != 0, added by band after the clouds -- all
 * inside the kernel, per (layer, band).  a must not be NULL. */
int rrtmgp_b200_forward_sw_aer_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud cloud, rrtmgp_b200_aerosol a,
        int ncol, int nlay, const float* play, const float* plev, const float* tlay,
        const float* col_dry, const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp,
        const float* iwp, const float* rel, const float* rei, int delta_cloud,
        const rrtmgp_b200_gas_conc* aerosols, int naer, const float* rh, int delta_aerosol,
        const float* mu0, const float* tsi_scaling, const float* sfc_alb_dir,
        const float* sfc_alb_dif, float* flux_up, float* flux_dn, float* flux_dn_dir,
        float* flux_net, float* heating_rate, int chunk, void* stream);

/* Longwave adjoint of rrtmgp_b200_forward_lw_f32 (no reference counterpart; the reference
 * has only the disabled surface Jacobian of lw_transport_noscat_kernel,
 * rte_solver_kernels.cu:56-91, Rte_lw.cu:133).  Same inputs as the forward plus the seeds of
 * L = sum(seed_flux_up * flux_up + seed_flux_dn * flux_dn) + sum(seed_heating_rate * HR)
 * ((ncol, nlay+1), (ncol, nlay+1), (ncol, nlay); NULL = zero; fold a flux_net seed in as
 * dn += s, up -= s).  Writes dL/dx for x = tlay, h2o and o3 volume mixing ratios (ncol, nlay),
 * tlev (ncol, nlay+1), tsfc (ncol), and lwp, iwp, rel, rei (ncol, nlay; zero where the water
 * path is not positive).  Any output may be NULL.  The vmr gradients treat each gas as a
 * (ncol, nlay) field whatever its given shape; with col_dry == NULL the dry-air column's
 * dependence on h2o is included.  Forward optical properties are recomputed per group of
 * 32 g-points on chip, nothing is stored between forward and adjoint.  chunk: 8 or 16
 * layers per warp (0 = 8); the k-distribution's bands must hold 16 or more g-points each.
 * One CTA per column up to 128 layers (chunk 16: up to what its shared memory holds); deeper
 * columns (chunk 8, nlay <= 512) run on a thread-block cluster of ceil(nlay / 128) CTAs. */
int rrtmgp_b200_adjoint_lw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud cloud, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* tlev,
        const float* tsfc, const float* col_dry, const rrtmgp_b200_gas_conc* gases, int ngases,
        const float* lwp, const float* iwp, const float* rel, const float* rei,
        const float* sfc_emis, const float* seed_flux_up, const float* seed_flux_dn,
        const float* seed_heating_rate, float* grad_tlay, float* grad_tlev, float* grad_tsfc,
        float* grad_h2o, float* grad_o3, float* grad_lwp, float* grad_iwp, float* grad_rel,
        float* grad_rei, int chunk, void* stream);

/* Shortwave adjoint of rrtmgp_b200_forward_sw_f32 (no reference counterpart).  Same inputs as
 * the forward plus the seeds of L = sum(seed_flux_up * flux_up + seed_flux_dn * flux_dn +
 * seed_flux_dn_dir * flux_dn_dir) + sum(seed_heating_rate * HR) ((ncol, nlay+1) x 3,
 * (ncol, nlay); NULL = zero; flux_dn includes the direct beam; fold a flux_net seed in as
 * dn += s, up -= s).  Writes dL/dx for x = tlay, h2o and o3 volume mixing ratios, lwp, iwp,
 * rel, rei (ncol, nlay) and the surface albedos (nband, ncol).  Any output may be NULL.  One
 * thread-block cluster of ceil(nlay / 64) CTAs per column (nlay <= 512); the forward optical
 * properties are recomputed on chip per group of 32 g-points. */
int rrtmgp_b200_adjoint_sw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud cloud, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp,
        const float* rel, const float* rei, int delta_cloud, const float* mu0,
        const float* tsi_scaling, const float* sfc_alb_dir, const float* sfc_alb_dif,
        const float* seed_flux_up, const float* seed_flux_dn, const float* seed_flux_dn_dir,
        const float* seed_heating_rate, float* grad_tlay, float* grad_h2o, float* grad_o3,
        float* grad_lwp, float* grad_iwp, float* grad_rel, float* grad_rei,
        float* grad_sfc_alb_dir, float* grad_sfc_alb_dif, void* stream);

/* Forward + adjoint in one pass per domain (no reference counterpart): the adjoint kernels
 * above also emit the forward fluxes they recompute, so a caller that needs both (a
 * variational step, a Jacobian-vector product with its primal) makes one launch per domain
 * instead of a forward and an adjoint.  Arguments as rrtmgp_b200_adjoint_lw_f32 /
 * rrtmgp_b200_adjoint_sw_f32, plus the outputs of rrtmgp_b200_forward_lw_f32 /
 * rrtmgp_b200_forward_sw_f32 (all required; the same values to FP32 rounding). */
int rrtmgp_b200_forward_adjoint_lw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud cloud, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* tlev,
        const float* tsfc, const float* col_dry, const rrtmgp_b200_gas_conc* gases, int ngases,
        const float* lwp, const float* iwp, const float* rel, const float* rei,
        const float* sfc_emis, const float* seed_flux_up, const float* seed_flux_dn,
        const float* seed_heating_rate, float* grad_tlay, float* grad_tlev, float* grad_tsfc,
        float* grad_h2o, float* grad_o3, float* grad_lwp, float* grad_iwp, float* grad_rel,
        float* grad_rei, float* flux_up, float* flux_dn, float* flux_net, float* heating_rate,
        int chunk, void* stream);
int rrtmgp_b200_forward_adjoint_sw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud cloud, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp,
        const float* rel, const float* rei, int delta_cloud, const float* mu0,
        const float* tsi_scaling, const float* sfc_alb_dir, const float* sfc_alb_dif,
        const float* seed_flux_up, const float* seed_flux_dn, const float* seed_flux_dn_dir,
        const float* seed_heating_rate, float* grad_tlay, float* grad_h2o, float* grad_o3,
        float* grad_lwp, float* grad_iwp, float* grad_rel, float* grad_rei,
        float* grad_sfc_alb_dir, float* grad_sfc_alb_dif, float* flux_up, float* flux_dn,
        float* flux_dn_dir, float* flux_net, float* heating_rate, void* stream);
/* Shortwave forward + adjoint with aerosols: rrtmgp_b200_forward_adjoint_sw_f32 with the
 * aerosol arguments of rrtmgp_b200_forward_sw_aer_f32 (a not NULL).  The aerosol optics enter
 * the recomputed forward; they depend on none of the differentiated inputs (rh is an input of
 * its own), so no aerosol gradient is formed.  The flux outputs may all be NULL (adjoint only). */
int rrtmgp_b200_forward_adjoint_sw_aer_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud cloud,
        rrtmgp_b200_aerosol a, int ncol, int nlay, const float* play, const float* plev,
        const float* tlay, const float* col_dry, const rrtmgp_b200_gas_conc* gases, int ngases,
        const float* lwp, const float* iwp, const float* rel, const float* rei, int delta_cloud,
        const rrtmgp_b200_gas_conc* aerosols, int naer, const float* rh, int delta_aerosol,
        const float* mu0, const float* tsi_scaling, const float* sfc_alb_dir,
        const float* sfc_alb_dif, const float* seed_flux_up, const float* seed_flux_dn,
        const float* seed_flux_dn_dir, const float* seed_heating_rate, float* grad_tlay,
        float* grad_h2o, float* grad_o3, float* grad_lwp, float* grad_iwp, float* grad_rel,
        float* grad_rei, float* grad_sfc_alb_dir, float* grad_sfc_alb_dif, float* flux_up,
        float* flux_dn, float* flux_dn_dir, float* flux_net, float* heating_rate, void* stream);

/* ---- Batched forward of many independent column grids ------------------------------------
 * No reference counterpart as one call: the reference's driver runs one grid at a time and
 * splits its columns into blocks of n_col_block (src_test/Radiation_solver.cu:467-615 and
 * :683-950 called per block from src_test/test_rte_rrtmgp.cu).  A batch describes up to
 * thousands of grids of uneven ncol / nlay whose device arrays stay fixed; one run computes
 * the longwave and shortwave forwards of every grid (the same results as
 * rrtmgp_b200_forward_lw_f32 / _sw_f32 per grid) in ONE persistent kernel launch: each CTA
 * takes tiles of (grid, domain, columns) from a device work counter, ordered by decreasing
 * tile cost.  A tile runs columns_per_cta columns side by side, each on
 * ceil(nlay / chunk) warps with its own hardware barrier.  The tile shape (chunk, columns)
 * of every (domain, 8-layer bin) comes from a built-in heuristic, from
 * rrtmgp_b200_batch_autotune, or from rrtmgp_b200_batch_set_plan (a cached result). */
typedef struct rrtmgp_b200_batch_grid {
    int ncol, nlay;                    /* nlay <= 256                                        */
    const float* play;                 /* (ncol, nlay), column fastest, device                */
    const float* plev;                 /* (ncol, nlay+1)                                      */
    const float* tlay;                 /* (ncol, nlay)                                        */
    const float* tlev;                 /* (ncol, nlay+1), longwave only                       */
    const float* tsfc;                 /* (ncol), longwave only                               */
    const float* col_dry;              /* (ncol, nlay) or NULL (from h2o and plev)            */
    const rrtmgp_b200_gas_conc* gases; /* host array, read by rrtmgp_b200_batch_create;        */
    int ngases;                        /* the vmr arrays it points to must stay valid          */
    const float* lwp;                  /* (ncol, nlay) x 4, or all NULL: clear sky             */
    const float* iwp;
    const float* rel;
    const float* rei;
    const float* sfc_emis;             /* (nband_lw, ncol)                                    */
    float* lw_flux_up;                 /* (ncol, nlay+1) x 3 and (ncol, nlay); lw_flux_up     */
    float* lw_flux_dn;                 /* NULL: no longwave for this grid                     */
    float* lw_flux_net;
    float* lw_heating_rate;
    const float* mu0;                  /* (ncol) > 0                                          */
    const float* tsi_scaling;          /* (ncol) or NULL                                      */
    const float* sfc_alb_dir;          /* (nband_sw, ncol)                                    */
    const float* sfc_alb_dif;
    float* sw_flux_up;                 /* (ncol, nlay+1) x 4 and (ncol, nlay); sw_flux_up     */
    float* sw_flux_dn;                 /* NULL: no shortwave for this grid                    */
    float* sw_flux_dn_dir;
    float* sw_flux_net;
    float* sw_heating_rate;
} rrtmgp_b200_batch_grid;

typedef struct rrtmgp_b200_batch_t* rrtmgp_b200_batch;

#define RRTMGP_B200_BATCH_PERSISTENT 0  /* one persistent launch (work counter reset first)  */
#define RRTMGP_B200_BATCH_GRAPH 1       /* the same, replayed from a captured CUDA graph     */
#define RRTMGP_B200_BATCH_PER_GRID 2    /* one fused launch per grid and domain (comparison) */

/* k_lw / k_sw: longwave / shortwave k-distributions (either may be NULL when no grid needs
 * that domain); cloud_lw / cloud_sw: cloud LUTs (NULL: clear sky for every grid). */
int rrtmgp_b200_batch_create(rrtmgp_b200_kdist k_lw, rrtmgp_b200_cloud cloud_lw,
        rrtmgp_b200_kdist k_sw, rrtmgp_b200_cloud cloud_sw, int delta_cloud,
        const rrtmgp_b200_batch_grid* grids, int ngrids, rrtmgp_b200_batch* out);
int rrtmgp_b200_batch_destroy(rrtmgp_b200_batch b);
/* Runs every grid once on stream (mode: RRTMGP_B200_BATCH_*).  One run may be in flight per
 * batch.  The first GRAPH run (and the first after a plan change) captures the graph. */
int rrtmgp_b200_batch_run(rrtmgp_b200_batch b, int mode, void* stream);
/* Times every candidate tile shape of every (domain, 8-layer bin) that the batch holds on a
 * replicated sample of its widest grid in that bin (persistent launches on stream, `reps`
 * timed runs each, the fastest counts) and keeps the fastest.  Synchronous.  Run it with the
 * inputs filled: the sample writes the outputs of the sampled grids. */
int rrtmgp_b200_batch_autotune(rrtmgp_b200_batch b, int reps, void* stream);
/* Tile shape of domain (0 longwave, 1 shortwave) for nlay in [8 bin - 7, 8 bin], bin 1..32:
 * chunk (8 or 16 layers per warp), columns per CTA, and the time of one tile in
 * microseconds (the work order key; 0 before any autotune).  set_plan validates the shape. */
int rrtmgp_b200_batch_get_plan(rrtmgp_b200_batch b, int domain, int bin, int* chunk, int* columns,
        float* tile_us);
int rrtmgp_b200_batch_set_plan(rrtmgp_b200_batch b, int domain, int bin, int chunk, int columns,
        float tile_us);
/* Work description of the current plan: total tiles, persistent CTAs, dynamic shared memory
 * per CTA (bytes) and kernel launches per run of each mode (persistent, per grid). */
int rrtmgp_b200_batch_stats(rrtmgp_b200_batch b, long long* ntiles, int* ctas, int* smem_bytes,
        int* launches_persistent, int* launches_per_grid);

/* No reference counterpart: FP32 FMA throughput probe used as the FP32-pipe roofline
 * denominator by the benchmark.  blocks x 512 threads, iters x 128 FMAs per thread
 * (FLOP = blocks * 512 * iters * 256); out (blocks floats) is written only in a case that
 * does not occur. */
int rrtmgp_b200_fp32_fma_probe(int blocks, int iters, float* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RRTMGP_B200_H */
