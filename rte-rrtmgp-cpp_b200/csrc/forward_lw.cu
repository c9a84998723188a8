// Fused longwave forward kernel (one CTA per column) and its launcher; the per-column
// algorithm is in lw_column.cuh.
#include "lw_column.cuh"

namespace rrtmgp_b200 {
namespace {

using namespace fused;

// DENSE: tables with more than three minor intervals over some g-point (tau_abs).
template <int CL, bool DENSE>
__global__ void __launch_bounds__(512) lw_forward_kernel(const KdistView<float> k, const LwGridIo io)
{
    lw_forward_column<CL, true, DENSE>(CtaCtx{}, k, io);
}

// Columns of more than 16 chunks: one thread-block cluster of cs CTAs per column (ClusterCtx).
template <int CL, bool DENSE>
__global__ void __launch_bounds__(512) lw_forward_cluster_kernel(const KdistView<float> k, const LwGridIo io, int cs)
{
    lw_forward_column<CL, true, DENSE>(ClusterCtx<CL>{cs}, k, io);
    cooperative_groups::this_cluster().sync();   // no CTA leaves while another may store into its shared memory
}

template <int CL, bool DENSE>
int launch_lw_forward(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay, const float* play,
                      const float* plev, const float* tlay, const float* tlev, const float* tsfc, const float* col_dry,
                      const GasSet<float>& gs, const float* lwp, const float* iwp, const float* rel, const float* rei,
                      const float* emis, float* up, float* dn, float* net, float* hr, cudaStream_t stream)
{
    const KdistView<float>& v = k->v32;
    const int NW = (nlay + CL - 1) / CL;
    // more than 16 chunks: a cluster of CS CTAs of NWc warps per column
    const int CS = (NW + 15) / 16, NWc = (NW + CS - 1) / CS;
    RB_CHECK_ARG(CS <= 8, "forward_lw: nlay too large for the fused kernel (at most 128 chunks)");
    const size_t smem = smem_layout(NWc * CL, v.ngas, v.nband, 1, CS * NWc, 2, CL,
                                    v.max_group_bands * (CL == 8 ? 2 : 1), v.max_nscal, NWc).total;
    if (smem > 220 * 1024) return fail(RRTMGP_B200_ERR_UNSUPPORTED, "forward_lw: shared memory need exceeds 220 KB");
    static PerDeviceOnce attr;
    int st = attr.run([] {
        const cudaError_t e = cudaFuncSetAttribute(lw_forward_kernel<CL, DENSE>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
        if (e != cudaSuccess) return e;
        return cudaFuncSetAttribute(lw_forward_cluster_kernel<CL, DENSE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    220 * 1024);
    }, "forward_lw attribute");
    if (st) return st;
    CloudArgs ca{};
    if (c) {
        ca.L = CloudLut<float>{c->nband, c->nsize_liq, c->nsize_ice, float(c->radliq_lwr), float(c->liq_step),
                               float(c->radice_lwr), float(c->ice_step), c->lut32};
        ca.lwp = lwp; ca.iwp = iwp; ca.rel = rel; ca.rei = rei;
        ca.present = 1;
    }
    LwGridIo io{ncol, nlay, play, plev, tlay, tlev, tsfc, col_dry, emis, up, dn, net, hr, gs, ca};
    if (CS == 1) {
        lw_forward_kernel<CL, DENSE><<<ncol, NW * 32, smem, stream>>>(v, io);
        RB_LAUNCH("lw_forward_kernel");
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
    RB_CUDA(cudaLaunchKernelEx(&cfg, lw_forward_cluster_kernel<CL, DENSE>, v, io, CS), "lw_forward_cluster_kernel");
    return RRTMGP_B200_OK;
}

}  // namespace

int forward_lw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay, const float* play,
                   const float* plev, const float* tlay, const float* tlev, const float* tsfc, const float* col_dry,
                   const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp,
                   const float* rel, const float* rei, const float* sfc_emis, float* flux_up, float* flux_dn,
                   float* flux_net, float* heating_rate, int chunk, void* stream)
{
    RB_CHECK_ARG(k && k->info.is_longwave, "forward_lw: need a longwave k-distribution");
    if (const int dst = check_device(k->device, "forward_lw")) return dst;
    RB_CHECK_ARG(ncol > 0 && nlay > 1, "forward_lw: ncol > 0 and nlay > 1 required");
    RB_CHECK_ARG(play && plev && tlay && tlev && tsfc && sfc_emis && flux_up && flux_dn && flux_net && heating_rate,
                 "forward_lw: null array");
    RB_CHECK_ARG(!c || (lwp && iwp && rel && rei), "forward_lw: cloud arrays required with a cloud handle");
    RB_CHECK_ARG(!c || c->nband == k->info.nband, "forward_lw: cloud and gas band counts differ");
    const KdistView<float>& v = k->v32;
    if (!fused_layout_ok(v, false, 8))
        return fail(RRTMGP_B200_ERR_UNSUPPORTED, "forward_lw: k-distribution layout not supported by the fused kernel");
    GasSet<float> gs;
    int st = make_gas_set<float>(k, ncol, nlay, gases, ngases, gs);
    if (st) return st;
    cudaStream_t s = as_stream(stream);
    const bool dense = v.max_minor_per_g > 3;
#define RB_LW_FWD(CLv, D)                                                                                          \
    launch_lw_forward<CLv, D>(k, c, ncol, nlay, play, plev, tlay, tlev, tsfc, col_dry, gs, lwp, iwp, rel, rei, \
                              sfc_emis, flux_up, flux_dn, flux_net, heating_rate, s)
    if (chunk == 8) return dense ? RB_LW_FWD(8, true) : RB_LW_FWD(8, false);
    return dense ? RB_LW_FWD(16, true) : RB_LW_FWD(16, false);
#undef RB_LW_FWD
}

}  // namespace rrtmgp_b200

extern "C" int rrtmgp_b200_forward_lw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay,
        const float* play, const float* plev, const float* tlay, const float* tlev, const float* tsfc,
        const float* col_dry, const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp,
        const float* rel, const float* rei, const float* sfc_emis, float* flux_up, float* flux_dn, float* flux_net,
        float* heating_rate, int chunk, void* stream)
{
    return rrtmgp_b200::forward_lw_f32(k, c, ncol, nlay, play, plev, tlay, tlev, tsfc, col_dry, gases, ngases, lwp,
                                       iwp, rel, rei, sfc_emis, flux_up, flux_dn, flux_net, heating_rate, chunk, stream);
}
