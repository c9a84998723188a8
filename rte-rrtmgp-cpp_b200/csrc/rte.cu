// Per-stage RTE solvers: longwave no-scattering (Gauss quadrature) and shortwave two-stream
// with adding, over the reference's column-fastest (ncol, nlay|nlev, ngpt) arrays.
//   * Up to 256 layers (one angle for the longwave; FP64 shortwave up to 128): the chunked
//     kernels below -- a warp is 32 consecutive columns x a chunk of layers at one g-point,
//     the chunks of a column are the warps of a block and exchange affine maps through shared
//     memory -- read every input once and write every level once (no workspace, no stash).
//   * Otherwise one thread per (column, g-point), a block being a run of consecutive columns
//     at one g-point: the longwave up-sweep inputs are kept in shared memory (or recomputed
//     when nlay is too large), and the shortwave adding recurrences use the caller workspace
//     plus the output arrays themselves.
// Every layer read and level write is a coalesced row either way.  The shortwave workspace is
// needed only by the second kind.  The FP32 longwave solver up to 192 layers stages its layer
// inputs through shared memory with TMA tile copies (lw_solver_tma).  The FP32 shortwave solver
// up to 128 layers can also write the flux each layer absorbs per g-point (rte_sw_abs), from
// which heating.cu forms heating rates without a second pass over the g-point arrays.
#include <algorithm>
#include <cfloat>
#include <mutex>
#include <type_traits>

#include "common.cuh"
#include "rte_device.cuh"
#include "sw_common.cuh"
#include "tma.cuh"

namespace rrtmgp_b200 {
namespace {

// Longwave no-scattering solver (lw_solver_noscat steps 1-3 + lw_transport_noscat_kernel,
// rte_solver_kernels.cu:35-185; F90 lw_solver_noscat / _GaussQuad :58-380).  Stash: trans
// and source_up of the down sweep kept in shared memory [nlay][blockDim] for the up sweep.
// Surface-temperature Jacobian (the reference's do_jacobians path of
// lw_transport_noscat_kernel, rte_solver_kernels.cu:56,65,82,91 and step 3): when flux_up_jac
// is not NULL, flux_up_jac = 2 pi w sum over angles of the upward radiance a surface source
// sfc_emis * sfc_src_jac produces with no other source, i.e. that source attenuated by the
// transmissivities of the layers between the surface and the level.
template <typename T, bool Stash>
__global__ void lw_solver_kernel(int ncol, int nlay, int nband, int top_at_1, int nmus,
                                 const int* __restrict__ gpt2band, const T* __restrict__ tau,
                                 const T* __restrict__ lay_src, const T* __restrict__ lev_inc,
                                 const T* __restrict__ lev_dec, const T* __restrict__ sfc_src,
                                 const T* __restrict__ sfc_emis, const T* __restrict__ inc_flux,
                                 T* __restrict__ flux_up, T* __restrict__ flux_dn,
                                 const T* __restrict__ sfc_src_jac, T* __restrict__ flux_up_jac)
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
        T rjac = flux_up_jac ? emis * sfc_src_jac[icol + size_t(g) * ncol] : T(0);
        if (flux_up_jac) {
            if (imu == 0) flux_up_jac[fbase + size_t(sfc) * ncol] = two_pi_w * rjac;
            else flux_up_jac[fbase + size_t(sfc) * ncol] += two_pi_w * rjac;
        }
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
            if (flux_up_jac) {
                rjac *= tr;
                if (imu == 0) flux_up_jac[o] = two_pi_w * rjac;
                else flux_up_jac[o] += two_pi_w * rjac;
            }
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

// ---- Chunked solvers (nlay <= 16 CL) ----
// A warp is 32 consecutive columns x one chunk of CL layers at one g-point, and the chunks of a
// column are the warps of one block (blockDim = 32 ceil(nlay / CL)).  Each thread reads its
// layers once (coalesced 128-byte rows, all loads of the chunk in flight together), composes
// the chunk's affine maps in registers, the chunks exchange the maps through shared memory,
// and a re-sweep of the registers writes every level once: the HBM traffic is the algorithmic
// one (inputs read once, outputs written once), with no shared-memory stash or workspace.

// Arguments of the chunked longwave solvers other than the layer inputs.
template <typename T>
struct LwChunkArgs {
    int ncol, nlay, nband, top_at_1;
    const int* gpt2band;
    const T *sfc_src, *sfc_emis, *inc_flux, *sfc_src_jac;
    T *flux_up, *flux_dn, *flux_up_jac;
};

// Layer inputs (tau, Planck sources; tr/sdn/sup are overwritten with the transmissivity and
// the layer sources) -> the chunk's maps: the down sweep x -> A x + Bd and the up sweep
// x -> A x + Bu, stored at [w][lane] of sm_a, sm_bd, sm_bu.  One angle (D = 1.66, weight 0.5:
// Rte_lw.cpp:101-113).
template <typename T, int CL>
__device__ __forceinline__ void lw_chunk_maps(T (&tr)[CL], const T (&lay)[CL], T (&sdn)[CL], T (&sup)[CL], T* sm_a,
                                              T* sm_bd, T* sm_bu, int w, int lane)
{
    const T D = T(1.66);
    T A = T(1), Bd = T(0), Bu = T(0);
#pragma unroll
    for (int i = 0; i < CL; ++i) {
        lw_layer(tr[i], D, lay[i], sdn[i], sup[i], tr[i], sdn[i], sup[i]);   // tau -> trans (1 for padding)
        A *= tr[i];
        Bd = tr[i] * Bd + sdn[i];
    }
#pragma unroll
    for (int i = CL - 1; i >= 0; --i) Bu = tr[i] * Bu + sup[i];
    sm_a[w * 32 + lane] = A;
    sm_bd[w * 32 + lane] = Bd;
    sm_bu[w * 32 + lane] = Bu;
}

// After the maps of all nw chunks are visible, one warp (warp 0) turns them into the radiances
// entering every chunk, each slot of the maps read before it is rewritten: from the top, the
// downward radiance at each chunk top (into sm_bd); from the surface, the upward radiance at
// each chunk bottom (into sm_bu; the last chunk's is the radiance leaving the surface) and,
// with the Jacobian, the surface term carried to each chunk bottom (into sm_a).  With every
// warp scanning the chunks above and below itself, the scans were O(chunks^2) loads per tile.
template <typename T>
__device__ __forceinline__ void lw_chunk_scan(const LwChunkArgs<T>& a, T* sm_a, T* sm_bd, T* sm_bu, int nw, int lane,
                                              int ic, int g)
{
    const int ncol = a.ncol;
    T x = (a.inc_flux ? a.inc_flux[ic + size_t(g) * ncol] : T(0)) / pi_value<T>();
    for (int c = 0; c < nw; ++c) {
        const T A = sm_a[c * 32 + lane], B = sm_bd[c * 32 + lane];
        sm_bd[c * 32 + lane] = x;
        x = A * x + B;
    }
    const T emis = a.sfc_emis[a.gpt2band[g] + size_t(ic) * a.nband];
    T y = x * (T(1) - emis) + emis * a.sfc_src[ic + size_t(g) * ncol];   // leaving the surface
    T yj = a.flux_up_jac ? emis * a.sfc_src_jac[ic + size_t(g) * ncol] : T(0);
    for (int c = nw - 1; c >= 0; --c) {
        const T A = sm_a[c * 32 + lane], B = sm_bu[c * 32 + lane];
        sm_bu[c * 32 + lane] = y;
        sm_a[c * 32 + lane] = yj;
        y = A * y + B;
        yj *= A;
    }
}

// After lw_chunk_scan: re-sweeps writing every level of the chunk (column ic, g-point g; level
// j0 + i is the top of layer j0 + i).
template <typename T, int CL>
__device__ __forceinline__ void lw_chunk_levels(const LwChunkArgs<T>& a, const T (&tr)[CL], const T (&sdn)[CL],
                                                const T (&sup)[CL], const T* sm_a, const T* sm_bd, const T* sm_bu,
                                                int w, int lane, int ic, int g)
{
    const int ncol = a.ncol, nlay = a.nlay;
    const size_t ncv = size_t(ncol) * (nlay + 1);
    const T two_pi_w = pi_value<T>();
    const int j0 = w * CL;
    T radn = sm_bd[w * 32 + lane];          // entering the chunk at its top
    T rup = sm_bu[w * 32 + lane];           // entering the chunk at its bottom
    const T rsfc = rup;                     // for the last chunk: leaving the surface
    T rjac = sm_a[w * 32 + lane];           // surface-temperature Jacobian at the chunk bottom
    const T jsfc = rjac;
    T* const dn = a.flux_dn + ic + size_t(g) * ncv;
    T* const up = a.flux_up + ic + size_t(g) * ncv;
    const ptrdiff_t step = a.top_at_1 ? ptrdiff_t(ncol) : -ptrdiff_t(ncol);
    const ptrdiff_t o0 = a.top_at_1 ? ptrdiff_t(j0) * ncol : ptrdiff_t(nlay - j0) * ncol;   // level j0
    if (w == 0) dn[o0] = two_pi_w * radn;
#pragma unroll
    for (int i = 0; i < CL; ++i) {
        radn = tr[i] * radn + sdn[i];
        if (j0 + i < nlay) dn[o0 + (i + 1) * step] = two_pi_w * radn;
    }
    if (j0 <= nlay - 1 && nlay - 1 < j0 + CL) up[o0 + (nlay - j0) * step] = two_pi_w * rsfc;
#pragma unroll
    for (int i = CL - 1; i >= 0; --i) {
        rup = tr[i] * rup + sup[i];
        if (j0 + i < nlay) up[o0 + i * step] = two_pi_w * rup;
    }
    if (a.flux_up_jac) {
        T* const uj = a.flux_up_jac + ic + size_t(g) * ncv;
        if (j0 <= nlay - 1 && nlay - 1 < j0 + CL) uj[o0 + (nlay - j0) * step] = two_pi_w * jsfc;
#pragma unroll
        for (int i = CL - 1; i >= 0; --i) {
            rjac *= tr[i];
            if (j0 + i < nlay) uj[o0 + i * step] = two_pi_w * rjac;
        }
    }
}

template <typename T, int CL, int MAXT>
__global__ void __launch_bounds__(MAXT) lw_solver_chunked(const LwChunkArgs<T> a, const T* __restrict__ tau,
                                                          const T* __restrict__ lay_src, const T* __restrict__ lev_inc,
                                                          const T* __restrict__ lev_dec)
{
    __shared__ T sm_a[16 * 32], sm_bd[16 * 32], sm_bu[16 * 32];   // chunk maps [chunk][lane]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int ncol = a.ncol, nlay = a.nlay;
    const int icol = blockIdx.x * 32 + lane;
    const bool cv = icol < ncol;
    const int ic = cv ? icol : 0;
    const int g = blockIdx.y;
    const size_t ncl = size_t(ncol) * nlay;
    const T* lev_dn = a.top_at_1 ? lev_inc : lev_dec;
    const T* lev_up = a.top_at_1 ? lev_dec : lev_inc;
    const int j0 = w * CL;

    // every input of the chunk is read before any is used (the layer terms branch, and loads
    // are not moved above a branch: read in the loop, one layer's rows would be in flight)
    T tr[CL], sdn[CL], sup[CL], lay[CL];
#pragma unroll
    for (int i = 0; i < CL; ++i) {
        const int j = j0 + i;
        tr[i] = T(0); lay[i] = T(0); sdn[i] = T(0); sup[i] = T(0);
        if (cv && j < nlay) {
            const size_t x = ic + size_t(g) * ncl + size_t(a.top_at_1 ? j : nlay - 1 - j) * ncol;
            tr[i] = tau[x];
            lay[i] = lay_src[x];
            sdn[i] = lev_dn[x];
            sup[i] = lev_up[x];
        }
    }
    lw_chunk_maps<T, CL>(tr, lay, sdn, sup, sm_a, sm_bd, sm_bu, w, lane);
    __syncthreads();
    if (w == 0) lw_chunk_scan<T>(a, sm_a, sm_bd, sm_bu, nw, lane, ic, g);
    __syncthreads();
    if (!cv) return;
    lw_chunk_levels<T, CL>(a, tr, sdn, sup, sm_a, sm_bd, sm_bu, w, lane, ic, g);
}

// TMA-staged FP32 variant (nlay <= kLwTmaMaxLay).  A tile is the (32 columns x nlay layers)
// block of the four layer inputs at one g-point; tiles are numbered g-point by g-point, column
// tile fastest, and a persistent block takes every gridDim.x-th tile.  One shared-memory stage
// per block, several blocks per SM: the block copies its layers of tile k from the stage into
// registers, frees the stage, and thread 0 has the TMA unit copy tile k + 1 into it while the
// block computes tile k (as lw_solver_chunked), so HBM reads continue through the compute and
// store phases (the one-tile-per-block kernel above has its loads in flight only between its
// start and its first use).  Lane = column: the stage reads are conflict-free rows.  Four
// barriers per tile: after thread 0's wait (hands out its outcome), after the stage reads
// (frees the stage), after the maps (publishes them), after warp 0's scan of the maps
// (lw_chunk_scan: publishes the radiances entering every chunk).
// Shared memory: [array 4][layer nlay][32] floats, maps [3][nw][32], one mbarrier.
constexpr int kLwTmaMaxLay = 192;

__device__ unsigned int g_tma_wait_timeouts;   // tiles whose copy did not complete in time

inline size_t lw_tma_smem_bytes(int nlay, int nw)
{
    return 128 /* alignment slack */ + size_t(4) * 32 * nlay * sizeof(float) + size_t(3) * nw * 32 * sizeof(float) +
           sizeof(uint64_t);
}

template <int CL>
__global__ void __launch_bounds__(512, CL == 8 ? 2 : 1) lw_solver_tma(const __grid_constant__ CUtensorMap m_tau,
                                                                     const __grid_constant__ CUtensorMap m_lay,
                                                                     const __grid_constant__ CUtensorMap m_dn,
                                                                     const __grid_constant__ CUtensorMap m_up,
                                                                     const LwChunkArgs<float> a, int ngpt)
{
    extern __shared__ unsigned char smem_dyn[];
    __shared__ int s_ok;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int ncol = a.ncol, nlay = a.nlay;
    const int tile_floats = 32 * nlay;
    float* const stage = reinterpret_cast<float*>(
        (reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~uintptr_t(127));   // 128-byte aligned tiles
    float* const sm_a = stage + 4 * tile_floats;
    float* const sm_bd = sm_a + nw * 32;
    float* const sm_bu = sm_bd + nw * 32;
    uint64_t* const bar = reinterpret_cast<uint64_t*>(sm_bu + nw * 32);   // 8-byte aligned: nw * 32 floats
    const int nct = (ncol + 31) >> 5;
    const unsigned tx_bytes = 4u * unsigned(tile_floats) * 4u;
    // Tile cursor (g-point g, column tile ct): the block visits tiles blockIdx.x + k gridDim.x
    // of g * nct + ct; one division at the start, then 32-bit steps (the host keeps
    // nct * ngpt below 2^31).
    const int dg = int(gridDim.x) / nct, dct = int(gridDim.x) - dg * nct;
    auto advance = [&](int& gq, int& cq) {
        cq += dct;
        gq += dg;
        if (cq >= nct) {
            cq -= nct;
            ++gq;
        }
    };
    int g = int(blockIdx.x) / nct, ct = int(blockIdx.x) - g * nct;   // current tile
    int gn = g, ctn = ct;                                              // next tile
    advance(gn, ctn);

    auto issue = [&](int gq, int cq) {
        const int x = cq * 32;
        tma::mbar_arrive_expect_tx(bar, tx_bytes);
        tma::load_3d(stage, &m_tau, x, 0, gq, bar);
        tma::load_3d(stage + tile_floats, &m_lay, x, 0, gq, bar);
        tma::load_3d(stage + 2 * tile_floats, &m_dn, x, 0, gq, bar);
        tma::load_3d(stage + 3 * tile_floats, &m_up, x, 0, gq, bar);
    };
    if (threadIdx.x == 0) {
        tma::prefetch_map(&m_tau);
        tma::prefetch_map(&m_lay);
        tma::prefetch_map(&m_dn);
        tma::prefetch_map(&m_up);
        tma::mbar_init(bar, 1);
        tma::fence_mbar_init();
        if (g < ngpt) issue(g, ct);
    }
    for (int k = 0; g < ngpt; ++k) {
        if (threadIdx.x == 0) s_ok = tma::mbar_wait(bar, k & 1);
        __syncthreads();
        if (!s_ok) {
            // the copy of tile k did not complete: count it, let it land (bounded) before the
            // block's shared memory is released, and stop
            if (threadIdx.x == 0) {
                atomicAdd(&g_tma_wait_timeouts, 1u);
                tma::mbar_wait(bar, k & 1);
            }
            return;
        }
        const int j0 = w * CL;
        float tr[CL], sdn[CL], sup[CL], lay[CL];
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            const int j = j0 + i;
            tr[i] = 0.f; lay[i] = 0.f; sdn[i] = 0.f; sup[i] = 0.f;
            if (j < nlay) {
                const int x = (a.top_at_1 ? j : nlay - 1 - j) * 32 + lane;
                tr[i] = stage[x];
                lay[i] = stage[tile_floats + x];
                sdn[i] = stage[2 * tile_floats + x];
                sup[i] = stage[3 * tile_floats + x];
            }
        }
        __syncthreads();   // every read of the stage done
        if (threadIdx.x == 0 && gn < ngpt) {
            tma::fence_proxy_async_smem();
            issue(gn, ctn);
        }
        const int icol = ct * 32 + lane;
        lw_chunk_maps<float, CL>(tr, lay, sdn, sup, sm_a, sm_bd, sm_bu, w, lane);
        __syncthreads();   // maps visible
        if (w == 0) lw_chunk_scan<float>(a, sm_a, sm_bd, sm_bu, nw, lane, icol < ncol ? icol : 0, g);
        __syncthreads();   // entering radiances visible
        if (icol < ncol) lw_chunk_levels<float, CL>(a, tr, sdn, sup, sm_a, sm_bd, sm_bu, w, lane, icol, g);
        g = gn;
        ct = ctn;
        advance(gn, ctn);
    }
}

// Two-stream layer coefficients of the chunked shortwave solver: FP32 uses the fused kernels'
// rearranged FP32 expressions (sw_layer_fast; 1 - ssa is exact in FP32 for ssa >= 1/2), FP64
// the reference expressions.
template <typename T>
__device__ __forceinline__ void sw_layer_coeffs(T tau, T ssa, T g, T mu0, T mu0_inv, T& R, T& Tt, T& Rdir, T& Tdir,
                                                T& Tn);
template <>
__device__ __forceinline__ void sw_layer_coeffs<float>(float tau, float ssa, float g, float mu0, float mu0_inv,
                                                       float& R, float& Tt, float& Rdir, float& Tdir, float& Tn)
{
    float adif, adir;
    fused::sw_layer_fast(tau, ssa, 1.f - ssa, g, mu0, mu0_inv, R, Tt, Rdir, Tdir, Tn, adif, adir);
}
template <>
__device__ __forceinline__ void sw_layer_coeffs<double>(double tau, double ssa, double g, double mu0, double,
                                                        double& R, double& Tt, double& Rdir, double& Tdir, double& Tn)
{
    sw_two_stream<double>(tau, ssa, g, mu0, R, Tt, Rdir, Tdir, Tn);
}
// FP32 coefficients together with the layer's diffuse and direct absorptances (1 - R - T and
// 1 - Tn - Rdir - Tdir in sw_layer_fast's cancellation-free form).
__device__ __forceinline__ void sw_layer_coeffs_abs(float tau, float ssa, float g, float mu0, float mu0_inv, float& R,
                                                    float& Tt, float& Rdir, float& Tdir, float& Tn, float& adif,
                                                    float& adir)
{
    fused::sw_layer_fast(tau, ssa, 1.f - ssa, g, mu0, mu0_inv, R, Tt, Rdir, Tdir, Tn, adif, adir);
}

template <typename T>
__device__ __forceinline__ T adding_den(T R, T a) { return T(1) / (T(1) - R * a); }
template <>
__device__ __forceinline__ float adding_den<float>(float R, float a) { return __fdividef(1.f, fmaf(-R, a, 1.f)); }

// Arguments of the chunked shortwave solvers other than the layer optical properties.
template <typename T>
struct SwChunkArgs {
    int ncol, nlay, nband, top_at_1;
    const int* gpt2band;
    const T *mu0, *inc_dir, *alb_dir, *alb_dif, *inc_dif;
    T *flux_up, *flux_dn, *flux_dir;
    T* layer_abs = nullptr;   // ABS solvers: absorbed flux per (layer, g-point), laid out as tau
};

// Per-thread state of one chunk: its layers' diffuse reflectance and transmittance, direct
// sources relative to the chunk top, direct-beam product above each layer, and the adding
// composite of the chunk (R_up, R_dn, T, U, D) with its direct-beam product P.
template <typename T, int CL>
struct SwChunk {
    T vR[CL], vT[CL], vSu[CL], vSd[CL], vP[CL];
    T P = T(1), cRu = T(0), cRd = T(0), cT = T(1), cU = T(0), cD = T(0);

    __device__ __forceinline__ void add_layer(int i, T R, T Tt, T Rdir, T Tdir, T Tn)
    {
        vR[i] = R;
        vT[i] = Tt;
        vP[i] = P;
        vSu[i] = Rdir * P;
        vSd[i] = Tdir * P;
        const T den = adding_den(cRd, R);
        const T nRu = cRu + cT * cT * R * den;
        const T nRd = R + Tt * Tt * cRd * den;
        const T nU = cU + cT * (vSu[i] + R * cD) * den;
        const T nD = vSd[i] + Tt * (cD + cRd * vSu[i]) * den;
        cT = cT * Tt * den;
        cRu = nRu;
        cRd = nRd;
        cU = nU;
        cD = nD;
        P *= Tn;
    }
};

// Shared-memory arrays of the chunk exchange, [chunk][lane] each.
template <typename T>
struct SwChunkSmem {
    T *p, *ru, *rd, *t, *u, *d;
};

// After every layer of the chunk is added (column ic, g-point g): the direct beam and the
// adding composites exchanged between the chunks (three barriers), albedo and source at the
// chunk bottom, and the level outputs.  Threads of columns past ncol take part in the
// barriers and write nothing.  Idx: the signed type of the output offsets (int when every
// (column, level, g-point) offset fits in 31 bits).  ABS: also the flux every layer absorbs,
// F_dir(top) adir + (F_dif(top) + F_up(bottom)) adif, with the layer's absorptances read from
// sm_abs ([2 i] adif, [2 i + 1] adir of chunk layer i, stride blockDim.x, this thread's slot).
template <typename T, int CL, typename Idx, bool ABS = false>
__device__ __forceinline__ void sw_chunk_finish(const SwChunkArgs<T>& a, SwChunk<T, CL>& c, const SwChunkSmem<T>& sm,
                                                int w, int nw, int lane, bool cv, int ic, int g, T dir_toa, T fd_toa,
                                                T ad, T af, const T* sm_abs = nullptr)
{
    const int ncol = a.ncol, nlay = a.nlay;
    const int j0 = w * CL;
    sm.p[w * 32 + lane] = c.P;
    __syncthreads();
    // 2. direct beam at the chunk top and at the surface
    T dtop = dir_toa;
    for (int q = 0; q < w; ++q) dtop *= sm.p[q * 32 + lane];
    T dsfc = dtop;
    for (int q = w; q < nw; ++q) dsfc *= sm.p[q * 32 + lane];
    sm.ru[w * 32 + lane] = c.cRu;
    sm.rd[w * 32 + lane] = c.cRd;
    sm.t[w * 32 + lane] = c.cT;
    sm.u[w * 32 + lane] = c.cU * dtop;
    sm.d[w * 32 + lane] = c.cD * dtop;
    __syncthreads();
    // 3. One warp scans the chunk composites: from the surface up, the albedo and source at the
    //    bottom of every chunk and the transfer of the diffuse flux through it (flux at the
    //    chunk bottom = F * flux at its top + G); then from the top down, the diffuse flux
    //    entering every chunk.  The results replace the composites in shared memory (a slot is
    //    read before it is rewritten) and every warp reads its own chunk's after one more
    //    barrier: with every warp scanning all chunks itself, the scans were O(chunks^2) loads
    //    and divisions per tile.
    if (w == 0) {
        T alb = af, src = dsfc * ad;
        for (int q = nw - 1; q >= 0; --q) {
            const int x = q * 32 + lane;
            const T mRu = sm.ru[x], mRd = sm.rd[x], mT = sm.t[x], mU = sm.u[x], mD = sm.d[x];
            const T den = adding_den(mRd, alb);
            sm.ru[x] = mT * den;                 // F
            sm.rd[x] = (mRd * src + mD) * den;   // G
            sm.t[x] = alb;                       // albedo and source at the chunk bottom
            sm.u[x] = src;
            const T nalb = mRu + mT * mT * alb * den;
            src = mU + mT * (alb * mD + src) * den;
            alb = nalb;
        }
        T f = fd_toa;
        for (int q = 0; q < nw; ++q) {
            const int x = q * 32 + lane;
            sm.d[x] = f;                         // diffuse flux at the chunk top
            f = sm.ru[x] * f + sm.rd[x];
        }
    }
    __syncthreads();
    const T alb_in = sm.t[w * 32 + lane], src_in = sm.u[w * 32 + lane], fd_in = sm.d[w * 32 + lane];
    // 4. albedo and upward source at the top of every layer (bottom-up)
    T vA[CL];
    {
        T al = alb_in, so = src_in;
#pragma unroll
        for (int i = CL - 1; i >= 0; --i) {
            const T su = c.vSu[i] * dtop, sd = c.vSd[i] * dtop;
            const T den = adding_den(c.vR[i], al);
            const T na = c.vR[i] + c.vT[i] * c.vT[i] * al * den;
            const T ns = su + c.vT[i] * (al * sd + so) * den;
            c.vSd[i] = sd;
            c.vSu[i] = ns;
            vA[i] = na;
            al = na;
            so = ns;
        }
    }
    // 5. diffuse fluxes (top-down) and the level outputs
    if (!cv) return;
    const Idx off = Idx(ic) + Idx(g) * Idx(ncol) * Idx(nlay + 1);
    const Idx step = a.top_at_1 ? Idx(ncol) : -Idx(ncol);
    const Idx o0 = off + (a.top_at_1 ? Idx(j0) * Idx(ncol) : Idx(nlay - j0) * Idx(ncol));   // level j0
    T* const up = a.flux_up;
    T* const dn = a.flux_dn;
    T* const dr = a.flux_dir;
    T fd = fd_in;
    if constexpr (!ABS) {
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            const T a_n = (i + 1 < CL) ? vA[i + 1] : alb_in;
            const T s_n = (i + 1 < CL) ? c.vSu[i + 1] : src_in;
            if (j0 + i < nlay) {
                const T dir = dtop * c.vP[i];
                up[o0 + i * step] = fd * vA[i] + c.vSu[i];
                dn[o0 + i * step] = fd + dir;
                dr[o0 + i * step] = dir;
            }
            const T den = adding_den(c.vR[i], a_n);
            fd = (c.vT[i] * fd + c.vR[i] * s_n + c.vSd[i]) * den;
        }
    } else {
        const Idx lstep = a.top_at_1 ? Idx(ncol) : -Idx(ncol);
        const Idx l0 = Idx(ic) + Idx(g) * Idx(ncol) * Idx(nlay) +
                       (a.top_at_1 ? Idx(j0) * Idx(ncol) : Idx(nlay - 1 - j0) * Idx(ncol));   // layer j0
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            const T a_n = (i + 1 < CL) ? vA[i + 1] : alb_in;
            const T s_n = (i + 1 < CL) ? c.vSu[i + 1] : src_in;
            const T dir = dtop * c.vP[i];
            if (j0 + i < nlay) {
                up[o0 + i * step] = fd * vA[i] + c.vSu[i];
                dn[o0 + i * step] = fd + dir;
                dr[o0 + i * step] = dir;
            }
            const T den = adding_den(c.vR[i], a_n);
            const T fdb = (c.vT[i] * fd + c.vR[i] * s_n + c.vSd[i]) * den;   // diffuse down at the layer bottom
            if (j0 + i < nlay) {
                const T adif = sm_abs[(2 * i) * blockDim.x + threadIdx.x];
                const T adir = sm_abs[(2 * i + 1) * blockDim.x + threadIdx.x];
                a.layer_abs[l0 + i * lstep] = dir * adir + (fd + fdb * a_n + s_n) * adif;
            }
            fd = fdb;
        }
    }
    if (j0 <= nlay - 1 && nlay - 1 < j0 + CL) {
        // fd is now at the chunk bottom (padding layers are the identity): the surface level
        const Idx o = o0 + Idx(nlay - j0) * step;
        up[o] = fd * alb_in + src_in;
        dn[o] = fd + dsfc;
        dr[o] = dsfc;
    }
}

// I32: every (column, level, g-point) offset fits in 31 bits (sw_index32).  ABS (FP32): also
// the flux every layer absorbs per g-point (a.layer_abs); the layers' absorptances wait in
// shared memory (2 CL values per thread: kept in registers they spilled at the register cap).
template <typename T, int CL, int MAXT, int MINB = 1, bool I32 = false, bool ABS = false>
__global__ void __launch_bounds__(MAXT, MINB) sw_solver_chunked(const SwChunkArgs<T> a, const T* __restrict__ tau,
                                                                const T* __restrict__ ssa, const T* __restrict__ gasy)
{
    using Idx = typename std::conditional<I32, int, ptrdiff_t>::type;
    __shared__ T sm_p[16 * 32];                                      // direct-beam product per chunk
    __shared__ T sm_ru[16 * 32], sm_rd[16 * 32], sm_t[16 * 32], sm_u[16 * 32], sm_d[16 * 32];   // composites
    __shared__ T sm_abs[ABS ? 2 * CL * MAXT : 1];                    // [2 CL][thread] absorptances
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int ncol = a.ncol, nlay = a.nlay;
    const int icol = blockIdx.x * 32 + lane;
    const bool cv = icol < ncol;
    const int ic = cv ? icol : 0;
    const int g = blockIdx.y;
    const Idx base = Idx(ic) + Idx(g) * Idx(ncol) * Idx(nlay);
    const int band = a.gpt2band[g];
    const T m0 = a.mu0[ic], m0_inv = T(1) / m0;
    const T ad = a.alb_dir[band + size_t(ic) * a.nband], af = a.alb_dif[band + size_t(ic) * a.nband];
    const T dir_toa = a.inc_dir[ic + size_t(g) * ncol] * m0;
    const T fd_toa = a.inc_dif ? a.inc_dif[ic + size_t(g) * ncol] : T(0);
    const int j0 = w * CL;

    // 1. layer coefficients; direct beam relative to the chunk top; adding composite of the chunk.
    //    The optical properties of layer i + 1 are loaded while layer i is computed, from an
    //    address clamped to the column's last layer (ic is a valid column for every thread and
    //    j0 < nlay for every warp), so the loads are unconditional: inside the per-layer branch
    //    each layer waited for its own loads from memory.
    const auto layer_at = [&](int j) {
        const int jc = min(j, nlay - 1);
        return base + Idx(a.top_at_1 ? jc : nlay - 1 - jc) * Idx(ncol);
    };
    SwChunk<T, CL> c;
    Idx x = layer_at(j0);
    T nt = tau[x], ns = ssa[x], ng = gasy[x];
#pragma unroll
    for (int i = 0; i < CL; ++i) {
        const int j = j0 + i;
        const T tj = nt, sj = ns, gj = ng;
        if (i + 1 < CL) {
            x = layer_at(j + 1);
            nt = tau[x];
            ns = ssa[x];
            ng = gasy[x];
        }
        T R = T(0), Tt = T(1), Rdir = T(0), Tdir = T(0), Tn = T(1);
        if constexpr (!ABS) {
            if (cv && j < nlay) sw_layer_coeffs<T>(tj, sj, gj, m0, m0_inv, R, Tt, Rdir, Tdir, Tn);
        } else {
            T adif = T(0), adir = T(0);
            if (cv && j < nlay) sw_layer_coeffs_abs(tj, sj, gj, m0, m0_inv, R, Tt, Rdir, Tdir, Tn, adif, adir);
            sm_abs[(2 * i) * blockDim.x + threadIdx.x] = adif;
            sm_abs[(2 * i + 1) * blockDim.x + threadIdx.x] = adir;
        }
        c.add_layer(i, R, Tt, Rdir, Tdir, Tn);
    }
    sw_chunk_finish<T, CL, Idx, ABS>(a, c, SwChunkSmem<T>{sm_p, sm_ru, sm_rd, sm_t, sm_u, sm_d}, w, nw, lane, cv, ic,
                                     g, dir_toa, fd_toa, ad, af, sm_abs);
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

// The TMA variant needs 16-byte row strides (ncol a multiple of 4) and 16-byte aligned arrays.
inline bool lw_tma_ok(int ncol, int nlay, int ngpt, const float* tau, const float* lay, const float* dn,
                      const float* up)
{
    auto al = [](const float* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    return nlay <= kLwTmaMaxLay && ncol % 4 == 0 && (long long)ceil_div(ncol, 32) * ngpt < (1ll << 31) - 1024 &&
           al(tau) && al(lay) && al(dn) && al(up);
}

int lw_solver_tma_launch(const LwChunkArgs<float>& a, int ngpt, const float* tau, const float* lay,
                         const float* lev_dn, const float* lev_up, void* stream)
{
    CUtensorMap m[4];
    const float* src[4] = {tau, lay, lev_dn, lev_up};
    for (int q = 0; q < 4; ++q) {
        const int st = encode_map_3d_f32(&m[q], src[q], a.ncol, a.nlay, ngpt, 32, a.nlay);
        if (st) return st;
    }
    const int cl = a.nlay <= 8 * 16 ? 8 : 16;
    const int nw = ceil_div(a.nlay, cl);
    const size_t smem = lw_tma_smem_bytes(a.nlay, nw);
    const auto kernel = cl == 8 ? lw_solver_tma<8> : lw_solver_tma<16>;
    static PerDeviceOnce attr;
    const int ast = attr.run([] {
        // the largest request: 192 layers in 16-layer chunks (the 8-layer kernel stops at 128)
        const int most = int(lw_tma_smem_bytes(kLwTmaMaxLay, kLwTmaMaxLay / 16));
        cudaError_t e = cudaFuncSetAttribute(lw_solver_tma<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(lw_solver_tma<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
        return e;
    }, "rte_lw TMA attribute");
    if (ast) return ast;
    int dev = 0, nsm = 0, per_sm = 0;
    RB_CUDA(cudaGetDevice(&dev), "rte_lw");
    RB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "rte_lw");
    RB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * nw, smem), "rte_lw");
    const long long ntiles = (long long)ceil_div(a.ncol, 32) * ngpt;
    const int grid = int(std::min<long long>(ntiles, (long long)nsm * std::max(per_sm, 1)));
    kernel<<<grid, 32 * nw, smem, as_stream(stream)>>>(m[0], m[1], m[2], m[3], a, ngpt);
    RB_LAUNCH("lw_solver_tma");
    return RRTMGP_B200_OK;
}

template <typename T>
int rte_lw(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const T* tau, const T* lay_src,
           const T* lev_inc, const T* lev_dec, const T* sfc_src, const T* sfc_emis, const T* inc_flux,
           int nmus, T* flux_up, T* flux_dn, void* stream, const T* sfc_src_jac = nullptr, T* flux_up_jac = nullptr)
{
    RB_CHECK_ARG(b, "rte_lw: null bands");
    RB_CHECK_ARG(ncol > 0 && nlay > 0, "rte_lw: ncol and nlay must be > 0");
    RB_CHECK_ARG(nmus >= 1 && nmus <= 4, "rte_lw: n_gauss_angles must be 1..4");
    RB_CHECK_ARG(tau && lay_src && lev_inc && lev_dec && sfc_src && sfc_emis && flux_up && flux_dn,
                 "rte_lw: null array");
    if (nmus == 1 && nlay <= 16 * 16) {
        const LwChunkArgs<T> a{ncol, nlay, b->nband, top_at_1, b->d_gpt2band, sfc_src, sfc_emis, inc_flux,
                               sfc_src_jac, flux_up, flux_dn, flux_up_jac};
        const T* lev_dn = top_at_1 ? lev_inc : lev_dec;
        const T* lev_up = top_at_1 ? lev_dec : lev_inc;
        if constexpr (sizeof(T) == 4) {
            if (lw_tma_ok(ncol, nlay, b->ngpt, tau, lay_src, lev_dn, lev_up))
                return lw_solver_tma_launch(a, b->ngpt, tau, lay_src, lev_dn, lev_up, stream);
        }
        const dim3 grid(ceil_div(ncol, 32), b->ngpt);
        // FP32 up to 128 layers: 8-layer chunks (more warps with fewer rows in flight each
        // measured faster than 16 at 8192 x 128); FP64 and deeper columns: 16-layer chunks
        if (sizeof(T) == 4 && nlay <= 8 * 16)
            lw_solver_chunked<T, 8, 512><<<grid, 32 * ceil_div(nlay, 8), 0, as_stream(stream)>>>(
                a, tau, lay_src, lev_inc, lev_dec);
        else
            lw_solver_chunked<T, 16, 512><<<grid, 32 * ceil_div(nlay, 16), 0, as_stream(stream)>>>(
                a, tau, lay_src, lev_inc, lev_dec);
        RB_LAUNCH("lw_solver_chunked");
        return RRTMGP_B200_OK;
    }
    size_t smem = 0;
    const int bs = lw_smem_block<T>(nlay, &smem);
    if (bs > 0) {
        static PerDeviceOnce attr;
        const int ast = attr.run([] { return cudaFuncSetAttribute(lw_solver_kernel<T, true>,
                                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                                  96 * 1024); }, "rte_lw attribute");
        if (ast) return ast;
        const dim3 grid(ceil_div(ncol, bs), b->ngpt);
        lw_solver_kernel<T, true><<<grid, bs, smem, as_stream(stream)>>>(
            ncol, nlay, b->nband, top_at_1, nmus, b->d_gpt2band, tau, lay_src, lev_inc, lev_dec, sfc_src, sfc_emis,
            inc_flux, flux_up, flux_dn, sfc_src_jac, flux_up_jac);
    } else {
        const dim3 grid(ceil_div(ncol, 64), b->ngpt);
        lw_solver_kernel<T, false><<<grid, 64, 0, as_stream(stream)>>>(
            ncol, nlay, b->nband, top_at_1, nmus, b->d_gpt2band, tau, lay_src, lev_inc, lev_dec, sfc_src, sfc_emis,
            inc_flux, flux_up, flux_dn, sfc_src_jac, flux_up_jac);
    }
    RB_LAUNCH("lw_solver_kernel");
    return RRTMGP_B200_OK;
}

// Columns up to this depth run the chunked shortwave solver, which needs no workspace.
constexpr int sw_chunked_max_nlay(bool fp64) { return fp64 ? 128 : 256; }

// Every (column, level, g-point) offset of the shortwave fluxes fits in 31 bits.
inline bool sw_index32(int ncol, int nlay, int ngpt)
{
    return size_t(ncol) * size_t(nlay + 1) * size_t(ngpt) < (size_t(1) << 31);
}

size_t sw_ws_bytes(int ncol, int nlay, int ngpt, int fp64)
{
    if (ncol <= 0 || nlay <= 0 || ngpt <= 0 || nlay <= sw_chunked_max_nlay(fp64 != 0)) return 0;
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
    // Chunked solver up to 256 layers (FP64: 128; its deeper columns would spill registers).
    constexpr bool fp64 = sizeof(T) == 8;
    if (nlay <= sw_chunked_max_nlay(fp64)) {
        const SwChunkArgs<T> a{ncol, nlay, b->nband, top_at_1, b->d_gpt2band, mu0, inc_dir, alb_dir, alb_dif,
                               inc_dif, flux_up, flux_dn, flux_dir};
        const dim3 grid(ceil_div(ncol, 32), b->ngpt);
        const bool i32 = sw_index32(ncol, nlay, b->ngpt);
        if constexpr (fp64) {
            sw_solver_chunked<T, 16, 256><<<grid, 32 * ceil_div(nlay, 16), 0, as_stream(stream)>>>(a, tau, ssa, g);
        } else if (nlay <= 128) {
            const auto kernel = i32 ? sw_solver_chunked<T, 8, 512, 2, true> : sw_solver_chunked<T, 8, 512, 2, false>;
            kernel<<<grid, 32 * ceil_div(nlay, 8), 0, as_stream(stream)>>>(a, tau, ssa, g);
        } else {
            const auto kernel = i32 ? sw_solver_chunked<T, 16, 512, 1, true> : sw_solver_chunked<T, 16, 512, 1, false>;
            kernel<<<grid, 32 * ceil_div(nlay, 16), 0, as_stream(stream)>>>(a, tau, ssa, g);
        }
        RB_LAUNCH("sw_solver_chunked");
        return RRTMGP_B200_OK;
    }
    const size_t need = sw_ws_bytes(ncol, nlay, b->ngpt, fp64);
    if (!ws || ws_bytes < need)
        return fail(RRTMGP_B200_ERR_WORKSPACE, "rte_sw: workspace of " + std::to_string(need) + " bytes required");
    const dim3 grid(ceil_div(ncol, 64), b->ngpt);
    sw_solver_kernel<T, double><<<grid, 64, 0, as_stream(stream)>>>(
        ncol, nlay, b->ngpt, b->nband, top_at_1, b->d_gpt2band, tau, ssa, g, mu0, inc_dir, alb_dir, alb_dif,
        inc_dif, flux_up, flux_dn, flux_dir, static_cast<T*>(ws));
    RB_LAUNCH("sw_solver_kernel");
    return RRTMGP_B200_OK;
}

// rte_sw (FP32, chunked solver, nlay <= 128) that also writes the flux every layer absorbs per
// g-point, for heating rates summed from it (heating.cu: heating_rate_from_layer_abs) instead
// of recomputing the two-stream from tau, ssa and g and re-reading six g-point rows.
int rte_sw_abs(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const float* tau, const float* ssa,
               const float* g, const float* mu0, const float* inc_dir, const float* alb_dir, const float* alb_dif,
               const float* inc_dif, float* flux_up, float* flux_dn, float* flux_dir, float* layer_abs, void* stream)
{
    RB_CHECK_ARG(b, "rte_sw_abs: null bands");
    RB_CHECK_ARG(ncol > 0 && nlay > 0, "rte_sw_abs: ncol and nlay must be > 0");
    RB_CHECK_ARG(tau && ssa && g && mu0 && inc_dir && alb_dir && alb_dif && flux_up && flux_dn && flux_dir &&
                 layer_abs, "rte_sw_abs: null array");
    if (nlay > 128)
        return fail(RRTMGP_B200_ERR_UNSUPPORTED,
                    "rte_sw_abs: more than 128 layers (use rte_sw and heating_rate_sw_layers)");
    SwChunkArgs<float> a{ncol, nlay, b->nband, top_at_1, b->d_gpt2band, mu0, inc_dir, alb_dir, alb_dif,
                         inc_dif, flux_up, flux_dn, flux_dir};
    a.layer_abs = layer_abs;
    const dim3 grid(ceil_div(ncol, 32), b->ngpt);
    const auto kernel = sw_index32(ncol, nlay, b->ngpt) ? sw_solver_chunked<float, 8, 512, 2, true, true>
                                                        : sw_solver_chunked<float, 8, 512, 2, false, true>;
    kernel<<<grid, 32 * ceil_div(nlay, 8), 0, as_stream(stream)>>>(a, tau, ssa, g);
    RB_LAUNCH("sw_solver_chunked (absorbed flux)");
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

int rrtmgp_b200_rte_lw_jac_f32(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const float* tau,
        const float* lay_src, const float* lev_src_inc, const float* lev_src_dec, const float* sfc_src,
        const float* sfc_src_jac, const float* sfc_emis, const float* inc_flux, int n_gauss_angles, float* up,
        float* dn, float* up_jac, void* s)
{
    RB_CHECK_ARG(sfc_src_jac && up_jac, "rte_lw_jac: null Jacobian array");
    return rte_lw<float>(b, ncol, nlay, top_at_1, tau, lay_src, lev_src_inc, lev_src_dec, sfc_src, sfc_emis, inc_flux,
                         n_gauss_angles, up, dn, s, sfc_src_jac, up_jac);
}
int rrtmgp_b200_rte_lw_jac_f64(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const double* tau,
        const double* lay_src, const double* lev_src_inc, const double* lev_src_dec, const double* sfc_src,
        const double* sfc_src_jac, const double* sfc_emis, const double* inc_flux, int n_gauss_angles, double* up,
        double* dn, double* up_jac, void* s)
{
    RB_CHECK_ARG(sfc_src_jac && up_jac, "rte_lw_jac: null Jacobian array");
    return rte_lw<double>(b, ncol, nlay, top_at_1, tau, lay_src, lev_src_inc, lev_src_dec, sfc_src, sfc_emis,
                          inc_flux, n_gauss_angles, up, dn, s, sfc_src_jac, up_jac);
}

size_t rrtmgp_b200_rte_sw_workspace_bytes(int ncol, int nlay, int ngpt, int fp64)
{ return sw_ws_bytes(ncol, nlay, ngpt, fp64); }

int rrtmgp_b200_rte_sw_f32(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const float* tau,
        const float* ssa, const float* g, const float* mu0, const float* inc_flux_dir, const float* sfc_alb_dir,
        const float* sfc_alb_dif, const float* inc_flux_dif, float* up, float* dn, float* dir, void* ws,
        size_t ws_bytes, void* s)
{ return rte_sw<float>(b, ncol, nlay, top_at_1, tau, ssa, g, mu0, inc_flux_dir, sfc_alb_dir, sfc_alb_dif, inc_flux_dif, up, dn, dir, ws, ws_bytes, s); }
int rrtmgp_b200_rte_sw_abs_f32(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const float* tau,
        const float* ssa, const float* g, const float* mu0, const float* inc_flux_dir, const float* sfc_alb_dir,
        const float* sfc_alb_dif, const float* inc_flux_dif, float* up, float* dn, float* dir, float* layer_abs,
        void* s)
{ return rte_sw_abs(b, ncol, nlay, top_at_1, tau, ssa, g, mu0, inc_flux_dir, sfc_alb_dir, sfc_alb_dif, inc_flux_dif, up, dn, dir, layer_abs, s); }
int rrtmgp_b200_rte_sw_f64(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const double* tau,
        const double* ssa, const double* g, const double* mu0, const double* inc_flux_dir,
        const double* sfc_alb_dir, const double* sfc_alb_dif, const double* inc_flux_dif, double* up,
        double* dn, double* dir, void* ws, size_t ws_bytes, void* s)
{ return rte_sw<double>(b, ncol, nlay, top_at_1, tau, ssa, g, mu0, inc_flux_dir, sfc_alb_dir, sfc_alb_dif, inc_flux_dif, up, dn, dir, ws, ws_bytes, s); }

int rrtmgp_b200_rte_sw_static_scratch_f32(rrtmgp_b200_bands b, int ncol, int nlay, int top_at_1, const float* tau,
        const float* ssa, const float* g, const float* mu0, const float* inc_flux_dir, const float* sfc_alb_dir,
        const float* sfc_alb_dif, const float* inc_flux_dif, float* up, float* dn, float* dir, void* s)
{ return rte_sw_static(b, ncol, nlay, top_at_1, tau, ssa, g, mu0, inc_flux_dir, sfc_alb_dir, sfc_alb_dif, inc_flux_dif, up, dn, dir, s); }

int rrtmgp_b200_device_wait_timeouts(unsigned int* count)
{
    RB_CHECK_ARG(count, "device_wait_timeouts: null count");
    RB_CUDA(cudaMemcpyFromSymbol(count, g_tma_wait_timeouts, sizeof(unsigned int)), "device_wait_timeouts");
    return RRTMGP_B200_OK;
}

}  // extern "C"
