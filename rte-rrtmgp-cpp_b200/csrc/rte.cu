// Per-stage RTE solvers: longwave no-scattering (Gauss quadrature) and shortwave two-stream
// with adding.  One thread per (column, g-point); a block is a run of consecutive columns at
// one g-point, so every layer read and level write is a coalesced row of the column-fastest
// (ncol, nlay|nlev, ngpt) arrays.  No temporaries are allocated: the longwave up-sweep
// inputs are kept in shared memory (or recomputed when nlay is too large), and the
// shortwave adding recurrences use a caller workspace plus the output arrays themselves.
#include <algorithm>
#include <cfloat>
#include <mutex>

#include "common.cuh"
#include "rte_device.cuh"

namespace rrtmgp_b200 {
namespace {

// Longwave no-scattering solver (lw_solver_noscat steps 1-3 + lw_transport_noscat_kernel,
// rte_solver_kernels.cu:35-185; F90 lw_solver_noscat / _GaussQuad :58-380).  Stash: trans
// and source_up of the down sweep kept in shared memory [nlay][blockDim] for the up sweep.
template <typename T, bool Stash>
__global__ void lw_solver_kernel(int ncol, int nlay, int nband, int top_at_1, int nmus,
                                 const int* __restrict__ gpt2band, const T* __restrict__ tau,
                                 const T* __restrict__ lay_src, const T* __restrict__ lev_inc,
                                 const T* __restrict__ lev_dec, const T* __restrict__ sfc_src,
                                 const T* __restrict__ sfc_emis, const T* __restrict__ inc_flux,
                                 T* __restrict__ flux_up, T* __restrict__ flux_dn)
{
    extern __shared__ unsigned char smem_raw[];
    T* st_tr = reinterpret_cast<T*>(smem_raw);
    T* st_su = st_tr + size_t(nlay) * blockDim.x;
    const int icol = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    if (icol >= ncol) return;
    const size_t ncl = size_t(ncol) * nlay, ncv = size_t(ncol) * (nlay + 1);
    const size_t base = icol + size_t(g) * ncl;
    const size_t fbase = icol + size_t(g) * ncv;
    const T emis = sfc_emis[gpt2band[g] + size_t(icol) * nband];
    const T ssrc = sfc_src[icol + size_t(g) * ncol];
    const T inc = inc_flux ? inc_flux[icol + size_t(g) * ncol] : T(0);
    const T* lev_dn = top_at_1 ? lev_inc : lev_dec;
    const T* lev_up = top_at_1 ? lev_dec : lev_inc;
    const int top = top_at_1 ? 0 : nlay, sfc = top_at_1 ? nlay : 0;

    for (int imu = 0; imu < nmus; ++imu) {
        const T D = T(kGaussDs[nmus - 1][imu]);
        const T w = T(kGaussWts[nmus - 1][imu]);
        const T two_pi_w = T(2) * pi_value<T>() * w;
        T radn = inc / two_pi_w;
        // Downward sweep.
        if (imu == 0) flux_dn[fbase + size_t(top) * ncol] = two_pi_w * radn;
        else flux_dn[fbase + size_t(top) * ncol] += two_pi_w * radn;
#pragma unroll 4
        for (int j = 0; j < nlay; ++j) {
            const int l = top_at_1 ? j : nlay - 1 - j;
            const size_t i = base + size_t(l) * ncol;
            T tr, sdn, sup;
            lw_layer(tau[i], D, lay_src[i], lev_dn[i], lev_up[i], tr, sdn, sup);
            radn = tr * radn + sdn;
            if (Stash) {
                st_tr[size_t(j) * blockDim.x + threadIdx.x] = tr;
                st_su[size_t(j) * blockDim.x + threadIdx.x] = sup;
            }
            const size_t o = fbase + size_t(top_at_1 ? l + 1 : l) * ncol;
            if (imu == 0) flux_dn[o] = two_pi_w * radn;
            else flux_dn[o] += two_pi_w * radn;
        }
        // Surface reflection and emission.
        T rup = radn * (T(1) - emis) + emis * ssrc;
        if (imu == 0) flux_up[fbase + size_t(sfc) * ncol] = two_pi_w * rup;
        else flux_up[fbase + size_t(sfc) * ncol] += two_pi_w * rup;
        // Upward sweep.
#pragma unroll 4
        for (int j = nlay - 1; j >= 0; --j) {
            const int l = top_at_1 ? j : nlay - 1 - j;
            T tr, sup;
            if (Stash) {
                tr = st_tr[size_t(j) * blockDim.x + threadIdx.x];
                sup = st_su[size_t(j) * blockDim.x + threadIdx.x];
            } else {
                const size_t i = base + size_t(l) * ncol;
                T sdn;
                lw_layer(tau[i], D, lay_src[i], lev_dn[i], lev_up[i], tr, sdn, sup);
            }
            rup = tr * rup + sup;
            const size_t o = fbase + size_t(top_at_1 ? l : l + 1) * ncol;
            if (imu == 0) flux_up[o] = two_pi_w * rup;
            else flux_up[o] += two_pi_w * rup;
        }
    }
}

// Shortwave two-stream + adding (sw_source_2stream_kernel + sw_adding_kernel,
// rte_solver_kernels.cu:188-278,587-647; F90 sw_solver_2stream / sw_dif_and_source / adding
// :512-606,996-1228).  Workspace ws = [Rdif, Tdif, src_dn, src_up->denom] x (ncol,nlay,ngpt);
// during the adding the albedo / source of each level are parked in flux_up / flux_dn.
// C is the precision of the two-stream coefficients and of the adding denominators.
template <typename T, typename C>
__global__ void sw_solver_kernel(int ncol, int nlay, int ngpt, int nband, int top_at_1,
                                 const int* __restrict__ gpt2band, const T* __restrict__ tau,
                                 const T* __restrict__ ssa, const T* __restrict__ gasy,
                                 const T* __restrict__ mu0, const T* __restrict__ inc_dir,
                                 const T* __restrict__ alb_dir, const T* __restrict__ alb_dif,
                                 const T* __restrict__ inc_dif, T* __restrict__ flux_up,
                                 T* __restrict__ flux_dn, T* __restrict__ flux_dir, T* __restrict__ ws)
{
    const int icol = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    if (icol >= ncol) return;
    const size_t ncl = size_t(ncol) * nlay, ncv = size_t(ncol) * (nlay + 1);
    const size_t ntot = ncl * ngpt;
    T* rdif = ws;
    T* tdif = ws + ntot;
    T* sdn = ws + 2 * ntot;
    T* sup = ws + 3 * ntot;   // source_up, then denominator
    const size_t base = icol + size_t(g) * ncl;
    const size_t fb = icol + size_t(g) * ncv;
    const int band = gpt2band[g];
    const T m0 = mu0[icol];
    const T ad = alb_dir[band + size_t(icol) * nband];
    const T af = alb_dif[band + size_t(icol) * nband];
    const int top = top_at_1 ? 0 : nlay, sfc = top_at_1 ? nlay : 0;
    const T fd_top = inc_dif ? inc_dif[icol + size_t(g) * ncol] : T(0);

    // Direct beam and layer coefficients, from the top down.
    T dir = inc_dir[icol + size_t(g) * ncol] * m0;
    flux_dir[fb + size_t(top) * ncol] = dir;
    for (int j = 0; j < nlay; ++j) {
        const int l = top_at_1 ? j : nlay - 1 - j;
        const size_t i = base + size_t(l) * ncol;
        C Rd, Td, Rr, Tr, Tn;
        sw_two_stream<C>(C(tau[i]), C(ssa[i]), C(gasy[i]), C(m0), Rd, Td, Rr, Tr, Tn);
        rdif[i] = T(Rd);
        tdif[i] = T(Td);
        sup[i] = T(Rr) * dir;
        sdn[i] = T(Tr) * dir;
        dir = T(Tn) * dir;
        flux_dir[fb + size_t(top_at_1 ? l + 1 : l) * ncol] = dir;
    }
    // Adding, surface upward: albedo -> flux_up, src -> flux_dn (levels), denom -> sup.
    T alb = af, src = dir * ad;
    flux_up[fb + size_t(sfc) * ncol] = alb;
    flux_dn[fb + size_t(sfc) * ncol] = src;
    for (int j = nlay - 1; j >= 0; --j) {
        const int l = top_at_1 ? j : nlay - 1 - j;
        const size_t i = base + size_t(l) * ncol;
        const T R = rdif[i], Tt = tdif[i];
        const T den = T(C(1) / (C(1) - C(R) * C(alb)));
        const T alb_n = R + Tt * Tt * alb * den;
        const T src_n = sup[i] + Tt * den * (src + alb * sdn[i]);
        sup[i] = den;
        alb = alb_n;
        src = src_n;
        const size_t o = fb + size_t(top_at_1 ? l : l + 1) * ncol;
        flux_up[o] = alb;
        flux_dn[o] = src;
    }
    // Top of the domain, then downward.
    T fd = fd_top;
    flux_up[fb + size_t(top) * ncol] = fd * alb + src;
    flux_dn[fb + size_t(top) * ncol] = fd + flux_dir[fb + size_t(top) * ncol];
    for (int j = 0; j < nlay; ++j) {
        const int l = top_at_1 ? j : nlay - 1 - j;
        const size_t i = base + size_t(l) * ncol;
        const size_t o = fb + size_t(top_at_1 ? l + 1 : l) * ncol;
        const T a = flux_up[o], s = flux_dn[o];
        fd = (tdif[i] * fd + rdif[i] * s + sdn[i]) * sup[i];
        flux_up[o] = fd * a + s;
        flux_dn[o] = fd + flux_dir[o];
    }
}

template <typename T>
int lw_smem_block(int nlay, size_t* smem)
{
    const size_t per_thread = size_t(nlay) * 2 * sizeof(T);
    for (int bs : {128, 64, 32}) {
        if (per_thread * bs <= 96 * 1024) { *smem = per_thread * bs; return bs; }
    }
    *smem = 0;
    return 0;
}

template <typename T>
int rte_lw(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const T* tau, const T* lay_src,
           const T* lev_inc, const T* lev_dec, const T* sfc_src, const T* sfc_emis, const T* inc_flux,
           int nmus, T* flux_up, T* flux_dn, void* stream)
{
    RB_CHECK_ARG(b, "rte_lw: null bands");
    RB_CHECK_ARG(ncol > 0 && nlay > 0, "rte_lw: ncol and nlay must be > 0");
    RB_CHECK_ARG(nmus >= 1 && nmus <= 4, "rte_lw: n_gauss_angles must be 1..4");
    RB_CHECK_ARG(tau && lay_src && lev_inc && lev_dec && sfc_src && sfc_emis && flux_up && flux_dn,
                 "rte_lw: null array");
    size_t smem = 0;
    const int bs = lw_smem_block<T>(nlay, &smem);
    if (bs > 0) {
        static bool attr_set = false;
        if (!attr_set) {
            RB_CUDA(cudaFuncSetAttribute(lw_solver_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         96 * 1024), "rte_lw attribute");
            attr_set = true;
        }
        const dim3 grid(ceil_div(ncol, bs), b->ngpt);
        lw_solver_kernel<T, true><<<grid, bs, smem, as_stream(stream)>>>(
            ncol, nlay, b->nband, top_at_1, nmus, b->d_gpt2band, tau, lay_src, lev_inc, lev_dec, sfc_src, sfc_emis,
            inc_flux, flux_up, flux_dn);
    } else {
        const dim3 grid(ceil_div(ncol, 64), b->ngpt);
        lw_solver_kernel<T, false><<<grid, 64, 0, as_stream(stream)>>>(
            ncol, nlay, b->nband, top_at_1, nmus, b->d_gpt2band, tau, lay_src, lev_inc, lev_dec, sfc_src, sfc_emis,
            inc_flux, flux_up, flux_dn);
    }
    RB_LAUNCH("lw_solver_kernel");
    return RRTMGP_B200_OK;
}

size_t sw_ws_bytes(int ncol, int nlay, int ngpt, int fp64)
{
    return size_t(4) * ncol * nlay * ngpt * (fp64 ? sizeof(double) : sizeof(float));
}

template <typename T>
int rte_sw(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const T* tau, const T* ssa, const T* g,
           const T* mu0, const T* inc_dir, const T* alb_dir, const T* alb_dif, const T* inc_dif, T* flux_up,
           T* flux_dn, T* flux_dir, void* ws, size_t ws_bytes, void* stream)
{
    RB_CHECK_ARG(b, "rte_sw: null bands");
    RB_CHECK_ARG(ncol > 0 && nlay > 0, "rte_sw: ncol and nlay must be > 0");
    RB_CHECK_ARG(tau && ssa && g && mu0 && inc_dir && alb_dir && alb_dif && flux_up && flux_dn && flux_dir,
                 "rte_sw: null array");
    const size_t need = sw_ws_bytes(ncol, nlay, b->ngpt, sizeof(T) == 8);
    if (!ws || ws_bytes < need)
        return fail(RRTMGP_B200_ERR_WORKSPACE, "rte_sw: workspace of " + std::to_string(need) + " bytes required");
    const dim3 grid(ceil_div(ncol, 64), b->ngpt);
    sw_solver_kernel<T, double><<<grid, 64, 0, as_stream(stream)>>>(
        ncol, nlay, b->ngpt, b->nband, top_at_1, b->d_gpt2band, tau, ssa, g, mu0, inc_dir, alb_dir, alb_dif,
        inc_dif, flux_up, flux_dn, flux_dir, static_cast<T*>(ws));
    RB_LAUNCH("sw_solver_kernel");
    return RRTMGP_B200_OK;
}

// Shortwave solver scratch for callers that cannot allocate device memory themselves.
// Lives in this file-scope device array: RRTMGP_B200_SW_STATIC_SCRATCH_MAX_ELEMS entries per
// workspace slice, four slices, i.e. 16 MiB that every GPU which loads this library keeps
// until the process exits.  Host code must not hand the array's name to a kernel (on the host
// it is only a stand-in); the device address is looked up once per device below.
constexpr size_t kSwStaticElems = RRTMGP_B200_SW_STATIC_SCRATCH_MAX_ELEMS;
static __device__ __align__(256) float g_sw_static_scratch[4 * kSwStaticElems];

std::mutex g_sw_static_mu;
float* g_sw_static_ptr[64] = {};

// Device address of g_sw_static_scratch on the current device, resolved with
// cudaGetSymbolAddress on the first call made with that device current.
int sw_static_scratch(float** out)
{
    int dev = 0;
    RB_CUDA(cudaGetDevice(&dev), "rte_sw_static_scratch: cudaGetDevice");
    if (dev < 0 || dev >= 64) return fail(RRTMGP_B200_ERR_UNSUPPORTED, "rte_sw_static_scratch: device ordinal >= 64");
    std::lock_guard<std::mutex> lock(g_sw_static_mu);
    if (!g_sw_static_ptr[dev]) {
        void* p = nullptr;
        RB_CUDA(cudaGetSymbolAddress(&p, g_sw_static_scratch), "rte_sw_static_scratch: cudaGetSymbolAddress");
        g_sw_static_ptr[dev] = static_cast<float*>(p);
    }
    *out = g_sw_static_ptr[dev];
    return RRTMGP_B200_OK;
}

int rte_sw_static(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const float* tau, const float* ssa,
                  const float* g, const float* mu0, const float* inc_dir, const float* alb_dir,
                  const float* alb_dif, const float* inc_dif, float* flux_up, float* flux_dn, float* flux_dir,
                  void* stream)
{
    RB_CHECK_ARG(b, "rte_sw_static_scratch: null bands");
    RB_CHECK_ARG(ncol > 0 && nlay > 0, "rte_sw_static_scratch: ncol and nlay must be > 0");
    const size_t elems = size_t(ncol) * nlay * b->ngpt;
    if (elems > kSwStaticElems)
        return fail(RRTMGP_B200_ERR_WORKSPACE,
                    "rte_sw_static_scratch: ncol*nlay*ngpt = " + std::to_string(elems) + " exceeds the built-in "
                    "scratch of " + std::to_string(kSwStaticElems) + " elements; split the columns or use rte_sw_f32");
    RB_CHECK_ARG(tau && ssa && g && mu0 && inc_dir && alb_dir && alb_dif && flux_up && flux_dn && flux_dir,
                 "rte_sw_static_scratch: null array");
    float* ws = nullptr;
    const int st = sw_static_scratch(&ws);
    if (st != RRTMGP_B200_OK) return st;
    // The kernel reads the four slices with a stride of ncol*nlay*ngpt, so the slices are
    // packed at that stride inside the static array; every slot is written before it is read
    // within the call, so nothing needs clearing.
    const dim3 grid(ceil_div(ncol, 64), b->ngpt);
    sw_solver_kernel<float, double><<<grid, 64, 0, as_stream(stream)>>>(
        ncol, nlay, b->ngpt, b->nband, top_at_1, b->d_gpt2band, tau, ssa, g, mu0, inc_dir, alb_dir, alb_dif,
        inc_dif, flux_up, flux_dn, flux_dir, ws);
    RB_LAUNCH("sw_solver_kernel (static scratch)");
    return RRTMGP_B200_OK;
}

}  // namespace
}  // namespace rrtmgp_b200

using namespace rrtmgp_b200;

extern "C" {

int rrtmgp_b200_rte_lw_f32(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const float* tau,
        const float* lay_src, const float* lev_src_inc, const float* lev_src_dec, const float* sfc_src,
        const float* sfc_emis, const float* inc_flux, int n_gauss_angles, float* up, float* dn, void* s)
{ return rte_lw<float>(b, ncol, nlay, top_at_1, tau, lay_src, lev_src_inc, lev_src_dec, sfc_src, sfc_emis, inc_flux, n_gauss_angles, up, dn, s); }
int rrtmgp_b200_rte_lw_f64(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const double* tau,
        const double* lay_src, const double* lev_src_inc, const double* lev_src_dec, const double* sfc_src,
        const double* sfc_emis, const double* inc_flux, int n_gauss_angles, double* up, double* dn, void* s)
{ return rte_lw<double>(b, ncol, nlay, top_at_1, tau, lay_src, lev_src_inc, lev_src_dec, sfc_src, sfc_emis, inc_flux, n_gauss_angles, up, dn, s); }

size_t rrtmgp_b200_rte_sw_workspace_bytes(int ncol, int nlay, int ngpt, int fp64)
{ return sw_ws_bytes(ncol, nlay, ngpt, fp64); }

int rrtmgp_b200_rte_sw_f32(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const float* tau,
        const float* ssa, const float* g, const float* mu0, const float* inc_flux_dir, const float* sfc_alb_dir,
        const float* sfc_alb_dif, const float* inc_flux_dif, float* up, float* dn, float* dir, void* ws,
        size_t ws_bytes, void* s)
{ return rte_sw<float>(b, ncol, nlay, top_at_1, tau, ssa, g, mu0, inc_flux_dir, sfc_alb_dir, sfc_alb_dif, inc_flux_dif, up, dn, dir, ws, ws_bytes, s); }
int rrtmgp_b200_rte_sw_f64(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const double* tau,
        const double* ssa, const double* g, const double* mu0, const double* inc_flux_dir,
        const double* sfc_alb_dir, const double* sfc_alb_dif, const double* inc_flux_dif, double* up,
        double* dn, double* dir, void* ws, size_t ws_bytes, void* s)
{ return rte_sw<double>(b, ncol, nlay, top_at_1, tau, ssa, g, mu0, inc_flux_dir, sfc_alb_dir, sfc_alb_dif, inc_flux_dif, up, dn, dir, ws, ws_bytes, s); }

int rrtmgp_b200_rte_sw_static_scratch_f32(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const float* tau,
        const float* ssa, const float* g, const float* mu0, const float* inc_flux_dir, const float* sfc_alb_dir,
        const float* sfc_alb_dif, const float* inc_flux_dif, float* up, float* dn, float* dir, void* s)
{ return rte_sw_static(b, ncol, nlay, top_at_1, tau, ssa, g, mu0, inc_flux_dir, sfc_alb_dir, sfc_alb_dif, inc_flux_dif, up, dn, dir, s); }

}  // extern "C"
