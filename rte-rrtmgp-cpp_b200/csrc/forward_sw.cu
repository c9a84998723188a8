// Fused shortwave forward kernel (one CTA per column) and its launcher; the per-column
// algorithm is in sw_column.cuh.
#include "sw_column.cuh"

namespace rrtmgp_b200 {
namespace {

using namespace fused;

// DENSE: tables with more than three minor intervals over some g-point (tau_abs).
template <int CL, bool DENSE>
__global__ void __launch_bounds__(512) sw_forward_kernel(const KdistView<float> k, const SwGridIo io)
{
    sw_forward_column<CL, true, DENSE>(CtaCtx{}, k, io);
}

// Columns of more than 16 chunks: one thread-block cluster of cs CTAs per column (ClusterCtx).
template <int CL, bool DENSE>
__global__ void __launch_bounds__(512) sw_forward_cluster_kernel(const KdistView<float> k, const SwGridIo io, int cs)
{
    sw_forward_column<CL, true, DENSE>(ClusterCtx<CL>{cs}, k, io);
    cooperative_groups::this_cluster().sync();   // no CTA leaves while another may store into its shared memory
}

template <int CL, bool DENSE>
int launch_sw_forward(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay, const float* play,
                      const float* plev, const float* tlay, const float* col_dry, const GasSet<float>& gs,
                      const float* lwp, const float* iwp, const float* rel, const float* rei, int delta,
                      const float* mu0, const float* tsi, const float* alb_dir, const float* alb_dif, float* up,
                      float* dn, float* dir, float* net, float* hr, const SwAerosolArgs& aer, cudaStream_t stream)
{
    const KdistView<float>& v = k->v32;
    const int NW = (nlay + CL - 1) / CL;
    // more than 16 chunks: a cluster of CS CTAs of NWc warps per column
    const int CS = (NW + 15) / 16, NWc = (NW + CS - 1) / CS;
    RB_CHECK_ARG(CS <= 8, "forward_sw: nlay too large for the fused kernel (at most 128 chunks)");
    const size_t smem = smem_layout(NWc * CL, v.ngas, v.nband, aer.present ? 4 : 0, CS * NWc, 3, CL,
                                    v.max_group_bands * (CL == 8 ? 2 : 1), v.max_nscal, NWc).total;
    if (smem > 220 * 1024) return fail(RRTMGP_B200_ERR_UNSUPPORTED, "forward_sw: shared memory need exceeds 220 KB");
    static PerDeviceOnce attr;
    int st = attr.run([] {
        const cudaError_t e = cudaFuncSetAttribute(sw_forward_kernel<CL, DENSE>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
        if (e != cudaSuccess) return e;
        return cudaFuncSetAttribute(sw_forward_cluster_kernel<CL, DENSE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    220 * 1024);
    }, "forward_sw attribute");
    if (st) return st;
    SwCloudArgs ca{};
    if (c) {
        ca.L = CloudLut<float>{c->nband, c->nsize_liq, c->nsize_ice, float(c->radliq_lwr), float(c->liq_step),
                               float(c->radice_lwr), float(c->ice_step), c->lut32};
        ca.lwp = lwp; ca.iwp = iwp; ca.rel = rel; ca.rei = rei;
        ca.present = 1;
        ca.delta = delta;
    }
    SwGridIo io{ncol, nlay, play, plev, tlay, col_dry, mu0, tsi, alb_dir, alb_dif, up, dn, dir, net, hr, gs, ca, aer};
    if (CS == 1) {
        sw_forward_kernel<CL, DENSE><<<ncol, NW * 32, smem, stream>>>(v, io);
        RB_LAUNCH("sw_forward_kernel");
        return RRTMGP_B200_OK;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(ncol) * CS);
    cfg.blockDim = dim3(NWc * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = unsigned(CS);
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    RB_CUDA(cudaLaunchKernelEx(&cfg, sw_forward_cluster_kernel<CL, DENSE>, v, io, CS), "sw_forward_cluster_kernel");
    return RRTMGP_B200_OK;
}

}  // namespace

// a: aerosol tables (NULL: no aerosols); aerosols/naer: aermr01 .. aermr11; rh (ncol, nlay).
int forward_sw_aer_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, rrtmgp_b200_aerosol a, int ncol, int nlay,
                       const float* play, const float* plev, const float* tlay, const float* col_dry,
                       const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp,
                       const float* rel, const float* rei, int delta_cloud, const rrtmgp_b200_gas_conc* aerosols,
                       int naer, const float* rh, int delta_aerosol, const float* mu0, const float* tsi_scaling,
                       const float* sfc_alb_dir, const float* sfc_alb_dif, float* flux_up, float* flux_dn,
                       float* flux_dn_dir, float* flux_net, float* heating_rate, int chunk, void* stream)
{
    RB_CHECK_ARG(k && !k->info.is_longwave, "forward_sw: need a shortwave k-distribution");
    if (const int dst = check_device(k->device, "forward_sw")) return dst;
    RB_CHECK_ARG(ncol > 0 && nlay > 1, "forward_sw: ncol > 0 and nlay > 1 required");
    RB_CHECK_ARG(play && plev && tlay && mu0 && sfc_alb_dir && sfc_alb_dif && flux_up && flux_dn && flux_dn_dir &&
                 flux_net && heating_rate, "forward_sw: null array");
    RB_CHECK_ARG(!c || (lwp && iwp && rel && rei), "forward_sw: cloud arrays required with a cloud handle");
    RB_CHECK_ARG(!c || c->nband == k->info.nband, "forward_sw: cloud and gas band counts differ");
    const KdistView<float>& v = k->v32;
    if (!fused_layout_ok(v, true, 8))
        return fail(RRTMGP_B200_ERR_UNSUPPORTED, "forward_sw: k-distribution layout not supported by the fused kernel");
    GasSet<float> gs;
    int st = make_gas_set<float>(k, ncol, nlay, gases, ngases, gs);
    if (st) return st;
    SwAerosolArgs aer{};
    if (a) {
        RB_CHECK_ARG(rh, "forward_sw: rh required with aerosol tables");
        aer.L = aerosol_lut32(a);
        RB_CHECK_ARG(aer.L.nband == k->info.nband, "forward_sw: aerosol and gas band counts differ");
        st = make_aerosol_set<float>(ncol, nlay, aerosols, naer, aer.s);
        if (st) return st;
        aer.rh = rh;
        aer.present = 1;
        aer.delta = delta_aerosol;
    }
    cudaStream_t s = as_stream(stream);
    const int cl = chunk ? chunk : (nlay > 128 ? 16 : 8);
    const bool dense = v.max_minor_per_g > 3;
#define RB_SW_FWD(CLv, D)                                                                                           \
    launch_sw_forward<CLv, D>(k, c, ncol, nlay, play, plev, tlay, col_dry, gs, lwp, iwp, rel, rei, delta_cloud, mu0, \
                              tsi_scaling, sfc_alb_dir, sfc_alb_dif, flux_up, flux_dn, flux_dn_dir, flux_net,         \
                              heating_rate, aer, s)
    if (cl == 16) return dense ? RB_SW_FWD(16, true) : RB_SW_FWD(16, false);
    return dense ? RB_SW_FWD(8, true) : RB_SW_FWD(8, false);
#undef RB_SW_FWD
}

int forward_sw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay, const float* play,
                   const float* plev, const float* tlay, const float* col_dry, const rrtmgp_b200_gas_conc* gases,
                   int ngases, const float* lwp, const float* iwp, const float* rel, const float* rei,
                   int delta_cloud, const float* mu0, const float* tsi_scaling, const float* sfc_alb_dir,
                   const float* sfc_alb_dif, float* flux_up, float* flux_dn, float* flux_dn_dir, float* flux_net,
                   float* heating_rate, int chunk, void* stream)
{
    return forward_sw_aer_f32(k, c, nullptr, ncol, nlay, play, plev, tlay, col_dry, gases, ngases, lwp, iwp, rel, rei,
                              delta_cloud, nullptr, 0, nullptr, 0, mu0, tsi_scaling, sfc_alb_dir, sfc_alb_dif, flux_up,
                              flux_dn, flux_dn_dir, flux_net, heating_rate, chunk, stream);
}

}  // namespace rrtmgp_b200

extern "C" int rrtmgp_b200_forward_sw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp, const float* rel,
        const float* rei, int delta_cloud, const float* mu0, const float* tsi_scaling, const float* sfc_alb_dir,
        const float* sfc_alb_dif, float* flux_up, float* flux_dn, float* flux_dn_dir, float* flux_net,
        float* heating_rate, int chunk, void* stream)
{
    return rrtmgp_b200::forward_sw_f32(k, c, ncol, nlay, play, plev, tlay, col_dry, gases, ngases, lwp, iwp, rel, rei,
                                       delta_cloud, mu0, tsi_scaling, sfc_alb_dir, sfc_alb_dif, flux_up, flux_dn,
                                       flux_dn_dir, flux_net, heating_rate, chunk, stream);
}

extern "C" int rrtmgp_b200_forward_sw_aer_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, rrtmgp_b200_aerosol a,
        int ncol, int nlay, const float* play, const float* plev, const float* tlay, const float* col_dry,
        const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp, const float* rel,
        const float* rei, int delta_cloud, const rrtmgp_b200_gas_conc* aerosols, int naer, const float* rh,
        int delta_aerosol, const float* mu0, const float* tsi_scaling, const float* sfc_alb_dir,
        const float* sfc_alb_dif, float* flux_up, float* flux_dn, float* flux_dn_dir, float* flux_net,
        float* heating_rate, int chunk, void* stream)
{
    RB_CHECK_ARG(a, "forward_sw_aer: null aerosol handle (use rrtmgp_b200_forward_sw_f32 without aerosols)");
    return rrtmgp_b200::forward_sw_aer_f32(k, c, a, ncol, nlay, play, plev, tlay, col_dry, gases, ngases, lwp, iwp,
                                           rel, rei, delta_cloud, aerosols, naer, rh, delta_aerosol, mu0, tsi_scaling,
                                           sfc_alb_dir, sfc_alb_dif, flux_up, flux_dn, flux_dn_dir, flux_net,
                                           heating_rate, chunk, stream);
}
