// Building blocks shared by the fused FP32 column-forward kernels (longwave and shortwave).
//
// Mapping (both kernels): one CTA per column; lane l of every warp handles g-point
// 32*group + l; warp w owns the layer chunk [w*CL, (w+1)*CL) counted from the top of the
// atmosphere.  Per group of 32 g-points each warp first writes one record per (layer, band)
// of its chunk to shared memory (table offsets and interpolation weights of
// interpolation_kernel, minor scalings, band Planck values, cloud properties); the per
// (layer, g-point) work then reads its record with 128-bit shared loads and the tables with
// 128-bit corner-packed global loads (KdistView::kmaj4 & co.).
#pragma once

#include <cooperative_groups.h>

#include <cfloat>
#include <cmath>

#include "common.cuh"
#include "rte_device.cuh"

namespace rrtmgp_b200 {
namespace fused {

// Per-layer state kept in shared memory for the whole kernel (layers counted from the top).
struct __align__(16) LayerState {
    int jt, jp, itropo, pad;
    float ftemp, fpress, p, t;
    float t_top, t_bot, dp, pad2;
};

// Per (layer, band) record.
struct __align__(16) Rec {
    int4 kb;          // x, y: element offsets (row * ngpt) of the kmaj4/pfrac4 rows of
                      //       (t0, p0, e0) and (t1, p0, e1); z, w: kmin2 row offsets of (t0, e0), (t1, e1)
    float4 wmaj0, wmaj1;   // col_mix x fmajor (major absorption weights)
    float4 wpl0, wpl1;     // fmajor (Planck fractions; SW: unused)
    float4 fm;             // fminor (minor and Rayleigh weights)
    float4 aux;            // LW: pl_lay, pl_top, pl_bot, tau_cloud
                           // SW: col_dry + col_h2o (Rayleigh), cloud tau, ssa, g
    float aux2;            // LW: surface Planck function (bottom layer only)
                           // SW: cloud absorption optical depth tau_c * (1 - ssa_c)
    int a;                 // 0 lower / 1 upper atmosphere
    int kr[2];             // element offsets (row * ngpt) of the krayl2 rows of (a, t0, e0), (a, t1, e1)
    int4 pad;              // 144 bytes: an odd number of 16-byte units, so that the 128-bit stores of
                           // 32 lanes building consecutive records spread over all 32 banks
};
static_assert(sizeof(Rec) == 144, "Rec stride");

// Reduce-scatter of N per-lane values over 32 lanes: afterwards lane L holds in v[0] the warp
// total of value L >> log2(32 / N) (N <= 32, a power of two).
template <int N, int OFF>
struct ReduceScatter {
    static __device__ __forceinline__ void run(float* v, int lane)
    {
        constexpr int H = N / 2;
        const bool upper = (lane & OFF) != 0;
#pragma unroll
        for (int i = 0; i < H; ++i) {
            const float send = upper ? v[i] : v[i + H];
            const float keep = upper ? v[i + H] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, OFF);
        }
        ReduceScatter<H, OFF / 2>::run(v, lane);
    }
};
template <int OFF>
struct ReduceScatter<1, OFF> {
    static __device__ __forceinline__ void run(float* v, int lane)
    {
        v[0] += __shfl_xor_sync(0xffffffffu, v[0], OFF);
        ReduceScatter<1, OFF / 2>::run(v, lane);
    }
};
template <>
struct ReduceScatter<1, 0> {
    static __device__ __forceinline__ void run(float*, int) {}
};

__device__ __forceinline__ float warp_sum(float x)
{
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    return x;
}

// Interpolation part of a record (interpolation_kernel, gas_optics_rrtmgp_kernels.cu:256-291)
// for band b at layer state s.  The minor scalings are per layer, not per record
// (layer_minor_scalings).
__device__ __forceinline__ void record_weights(const KdistView<float>& k, Rec& R, const LayerState& s,
                                               const float* cg, int cgs, int b)
{
    LayerInterp<float> li;
    li.jt = s.jt;
    li.jp = s.jp;
    li.itropo = s.itropo;
    li.ftemp = s.ftemp;
    li.fpress = s.fpress;
    const int flav = k.band_flav[2 * b + li.itropo];
    const FlavorWeights<float> fw = flavor_weights(k, flav, li, cg, cgs);
    const int ne1 = k.neta - 1, np = k.npres;
    const int p0 = li.jp + li.itropo - 1;
    R.kb.x = (((li.jt - 1) * np + p0) * ne1 + (fw.j0 - 1)) * k.ngpt;
    R.kb.y = ((li.jt * np + p0) * ne1 + (fw.j1 - 1)) * k.ngpt;
    const int a = li.itropo;
    const int nc = k.ncontrib[a] > 0 ? k.ncontrib[a] : 1;
    // kmin2 rows; the Rayleigh rows (krayl2, [a][t][eta][g]) follow the same (t, eta) corners.
    R.kb.z = ((li.jt - 1) * ne1 + (fw.j0 - 1)) * nc;
    R.kb.w = (li.jt * ne1 + (fw.j1 - 1)) * nc;
    const float fp = li.fpress, f1 = 1.f - li.fpress;
    R.wpl0 = make_float4(f1 * fw.fm[0], f1 * fw.fm[1], fp * fw.fm[0], fp * fw.fm[1]);
    R.wpl1 = make_float4(f1 * fw.fm[2], f1 * fw.fm[3], fp * fw.fm[2], fp * fw.fm[3]);
    R.wmaj0 = make_float4(fw.cm[0] * R.wpl0.x, fw.cm[0] * R.wpl0.y, fw.cm[0] * R.wpl0.z, fw.cm[0] * R.wpl0.w);
    R.wmaj1 = make_float4(fw.cm[1] * R.wpl1.x, fw.cm[1] * R.wpl1.y, fw.cm[1] * R.wpl1.z, fw.cm[1] * R.wpl1.w);
    R.fm = make_float4(fw.fm[0], fw.fm[1], fw.fm[2], fw.fm[3]);
    R.a = a;
    R.kr[0] = ((a * k.ntemp + li.jt - 1) * ne1 + (fw.j0 - 1)) * k.ngpt;
    R.kr[1] = ((a * k.ntemp + li.jt) * ne1 + (fw.j1 - 1)) * k.ngpt;
}

// Minor scaling of scaling kind sid of atmosphere a at a layer (minor_scaling: the same
// arithmetic, gas_optical_depths_minor_kernel :396-417).
__device__ __forceinline__ float kind_scaling(const KdistView<float>& k, int a, int sid, const float* cg, int cgs,
                                              float p, float t)
{
    const int flags = k.scal_flags[a][sid];
    float scaling = cg[k.scal_gas[a][sid] * cgs];
    if (flags & 1) {
        scaling *= 0.01f * p / t;
        const int sg = k.scal_sgas[a][sid];
        if (sg > 0) {
            const float vmr_fact = 1.f / cg[0];
            const float dry_fact = 1.f / (1.f + cg[k.idx_h2o * cgs] * vmr_fact);
            if (flags & 2) scaling *= (1.f - cg[sg * cgs] * vmr_fact * dry_fact);
            else scaling *= cg[sg * cgs] * vmr_fact * dry_fact;
        }
    }
    return scaling;
}

// Scalings of every kind of layers 0 .. nloc - 1 (layer state st[], gas columns cg with
// stride cgs) into sc[jl * k.max_nscal + sid]; threads tid, tid + nthr, ... of the calling
// team take one (layer, kind) each.  Kinds past the layer's atmosphere's count are set to 0.
__device__ __forceinline__ void layer_minor_scalings(const KdistView<float>& k, const LayerState* st, const float* cg,
                                                     int cgs, float* sc, int nloc, int tid, int nthr)
{
    const int ns = k.max_nscal;
    for (int idx = tid; idx < nloc * ns; idx += nthr) {
        const int jl = idx / ns, sid = idx - jl * ns;
        const LayerState& s = st[jl];
        sc[idx] = sid < k.nscal[s.itropo] ? kind_scaling(k, s.itropo, sid, cg + jl, cgs, s.p, s.t) : 0.f;
    }
}

// Code n of g-point g's minor-interval list (minor_g / minor_gx; n < count, or a code that
// repeats the first one for n < 3).
__device__ __forceinline__ int minor_code_at(const KdistView<float>& k, int a, const int4& mg, int g, int n)
{
    if (n < 3) return n == 0 ? mg.y : (n == 1 ? mg.z : mg.w);
    return n < mg.x ? __ldg(k.minor_gx[a] + size_t(g) * k.minor_gx_stride + (n - 3)) : mg.y;
}

// Absorption optical depth of g-point g from a record: major (8 corners via two float4 loads)
// plus the minor intervals covering g (minor_g list), as gas_optical_depths_major/minor.
// nmax = most intervals over the warp's lanes (warp-uniform loop bound); lanes with fewer
// intervals read a valid entry and discard it with a select, so the loop does not diverge.
// sc: the layer's scalings, kind sid at sc[sid * sst].  DENSE: tables with more than three
// intervals over some g-point (KdistView::max_minor_per_g > 3); the loop over the further
// intervals is compiled only then, so that for the usual layouts the whole function stays
// straight-line code whose table loads the caller's unrolled layer loop can overlap.
template <bool DENSE = false>
__device__ __forceinline__ float tau_abs(const KdistView<float>& k, const Rec& R, int g, int4 mg, int nmax,
                                         const float* sc, int sst = 1)
{
    const float4 c0 = __ldg(k.kmaj4 + (R.kb.x + g));
    const float4 c1 = __ldg(k.kmaj4 + (R.kb.y + g));
    float tau = R.wmaj0.x * c0.x + R.wmaj0.y * c0.y + R.wmaj0.z * c0.z + R.wmaj0.w * c0.w +
                R.wmaj1.x * c1.x + R.wmaj1.y * c1.y + R.wmaj1.z * c1.z + R.wmaj1.w * c1.w;
    const float2* kn = k.kmin2[R.a];
#pragma unroll
    for (int n = 0; n < 3; ++n) {
        if (n < nmax) {
            const int code = n == 0 ? mg.y : (n == 1 ? mg.z : mg.w);
            const int c = code >> kScalBits;
            const float2 lo = __ldg(kn + (R.kb.z + c));
            const float2 hi = __ldg(kn + (R.kb.w + c));
            const float t = sc[(code & (kMaxScal - 1)) * sst] *
                            (R.fm.x * lo.x + R.fm.y * lo.y + R.fm.z * hi.x + R.fm.w * hi.y);
            tau += (n < mg.x) ? t : 0.f;
        }
    }
    if constexpr (DENSE) {
        for (int n = 3; n < nmax; ++n) {
            const int code = minor_code_at(k, R.a, mg, g, n);
            const int c = code >> kScalBits;
            const float2 lo = __ldg(kn + (R.kb.z + c));
            const float2 hi = __ldg(kn + (R.kb.w + c));
            const float t = sc[(code & (kMaxScal - 1)) * sst] *
                            (R.fm.x * lo.x + R.fm.y * lo.y + R.fm.z * hi.x + R.fm.w * hi.y);
            tau += (n < mg.x) ? t : 0.f;
        }
    }
    return tau;
}

// minor_g entry of g-point g with unused slots set to the first used one (or to contributor 0,
// slot 0), so that tau_abs can read every slot below the warp's maximum count.
__device__ __forceinline__ int4 minor_entry(const int4* mgt, int g, bool valid)
{
    int4 m = valid ? __ldg(mgt + g) : make_int4(0, 0, 0, 0);
    if (m.x < 2) m.z = m.y;
    if (m.x < 3) m.w = m.y;
    return m;
}

// Context of a fused column computation.  Members: icol(); warp() = the chunk this warp owns
// and nwarps() = the chunks of the column; lwarp() = the warp within the CTA (or team) that
// holds its shared memory; tid() / nthreads() of that CTA (team); smem(); sync() = the barrier
// of every warp of the column; layer0() / nloc(nlay) = the layers whose state that shared
// memory holds; put(p, v) stores v at p in the shared memory of every CTA that reads it.
// CtaCtx: the whole CTA computes column blockIdx.x; every value is a special register or a
// launch constant, so none occupies a register across the column.  The batched kernel
// supplies its own context type with the same members.
struct CtaCtx {
    __device__ __forceinline__ int icol() const { return blockIdx.x; }
    __device__ __forceinline__ int warp() const { return threadIdx.x >> 5; }
    __device__ __forceinline__ int nwarps() const { return blockDim.x >> 5; }
    __device__ __forceinline__ int lwarp() const { return threadIdx.x >> 5; }
    __device__ __forceinline__ int tid() const { return threadIdx.x; }
    __device__ __forceinline__ int nthreads() const { return blockDim.x; }
    __device__ __forceinline__ int layer0() const { return 0; }
    __device__ __forceinline__ int nloc(int nlay) const { return nlay; }
    __device__ __forceinline__ unsigned char* smem() const
    {
        extern __shared__ __align__(16) unsigned char smem_raw[];
        return smem_raw;
    }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    template <class T>
    __device__ __forceinline__ void put(T* p, const T& v) const { *p = v; }
};

// One column on a thread-block cluster of cs CTAs (columns deeper than one CTA holds): CTA r
// of the cluster owns the chunks [r W, (r + 1) W) (W = its warps) and the state of their
// layers [r W CL, (r + 1) W CL); the chunk quantities every warp reads are stored into the
// shared memory of all CTAs of the cluster (distributed shared memory) and the barrier is the
// cluster's.
template <int CL>
struct ClusterCtx {
    int cs;
    __device__ __forceinline__ int rank() const { return int(cooperative_groups::this_cluster().block_rank()); }
    __device__ __forceinline__ int icol() const { return blockIdx.x / cs; }
    __device__ __forceinline__ int warp() const { return rank() * int(blockDim.x >> 5) + int(threadIdx.x >> 5); }
    __device__ __forceinline__ int nwarps() const { return cs * int(blockDim.x >> 5); }
    __device__ __forceinline__ int lwarp() const { return threadIdx.x >> 5; }
    __device__ __forceinline__ int tid() const { return threadIdx.x; }
    __device__ __forceinline__ int nthreads() const { return blockDim.x; }
    __device__ __forceinline__ int layer0() const { return rank() * int(blockDim.x >> 5) * CL; }
    __device__ __forceinline__ int nloc(int nlay) const
    {
        return max(0, min(int(blockDim.x >> 5) * CL, nlay - layer0()));
    }
    __device__ __forceinline__ unsigned char* smem() const
    {
        extern __shared__ __align__(16) unsigned char smem_raw[];
        return smem_raw;
    }
    __device__ __forceinline__ void sync() const { cooperative_groups::this_cluster().sync(); }
    template <class T>
    __device__ __forceinline__ void put(T* p, const T& v) const
    {
        cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
        for (int r = 0; r < cs; ++r) *cl.map_shared_rank(p, r) = v;
    }
};

// Fill the per-layer state and col_gas of layers j0 .. j0 + nloc - 1 (counted from the top,
// those below nlay) of column icol into st[j - j0] and cg[(gas) * cg_stride + j - j0]; threads
// tid, tid + nthr, ... of the calling team take one layer each.
__device__ __forceinline__ void setup_layer_range(const KdistView<float>& k, const GasSet<float>& gs, int ncol,
                                                  int nlay, int icol, bool top_at_1, const float* __restrict__ play,
                                                  const float* __restrict__ plev, const float* __restrict__ tlay,
                                                  const float* __restrict__ tlev, const float* __restrict__ col_dry,
                                                  LayerState* st, float* cg, int cg_stride, int j0, int nloc,
                                                  int tid, int nthr)
{
    for (int jl = tid; jl < nloc; jl += nthr) {
        const int j = j0 + jl;
        if (j >= nlay) break;
        const int l = top_at_1 ? j : nlay - 1 - j;
        const size_t cl = icol + size_t(l) * ncol;
        const float p = play[cl], t = tlay[cl];
        fill_col_gas(k, gs, ncol, nlay, icol, l, plev, col_dry, cg + jl, cg_stride);
        const LayerInterp<float> li = layer_interp(k, p, t);
        const int lt = top_at_1 ? j : nlay - j, lb = top_at_1 ? j + 1 : nlay - 1 - j;
        LayerState s;
        s.jt = li.jt;
        s.jp = li.jp;
        s.itropo = li.itropo;
        s.pad = 0;
        s.ftemp = li.ftemp;
        s.fpress = li.fpress;
        s.p = p;
        s.t = t;
        s.t_top = tlev ? tlev[icol + size_t(lt) * ncol] : 0.f;
        s.t_bot = tlev ? tlev[icol + size_t(lb) * ncol] : 0.f;
        s.dp = fabsf(plev[icol + size_t(lb) * ncol] - plev[icol + size_t(lt) * ncol]);
        s.pad2 = 0.f;
        st[jl] = s;
    }
}

// The whole column (layers 0 .. nlay - 1, cg stride nlay).
__device__ __forceinline__ void setup_layers(const KdistView<float>& k, const GasSet<float>& gs, int ncol,
                                             int nlay, int icol, bool top_at_1, const float* __restrict__ play,
                                             const float* __restrict__ plev, const float* __restrict__ tlay,
                                             const float* __restrict__ tlev, const float* __restrict__ col_dry,
                                             LayerState* st, float* cg, int tid, int nthr)
{
    setup_layer_range(k, gs, ncol, nlay, icol, top_at_1, play, plev, tlay, tlev, col_dry, st, cg, nlay, 0, nlay, tid,
                      nthr);
}

// Table layouts the corner-packed FP32 kernels take: minor intervals inside one band (their
// interpolation weights are the band's), at most kMaxScal scaling kinds per atmosphere, and
// a group of 32 g-points touching at most max_bands bands.  Any number of minor intervals per
// band or per g-point is accepted.
inline bool fused_layout_ok(const KdistView<float>& v, bool sw, int max_bands)
{
    return v.kmaj4 && v.minor_in_band && v.nscal[0] <= kMaxScal && v.nscal[1] <= kMaxScal &&
           v.max_group_bands <= max_bands && (sw ? v.krayl2 != nullptr : v.pfrac4 != nullptr);
}

// Shared-memory offsets (bytes) of the fused kernels, all 16-byte aligned.
struct SmemLayout {
    size_t state, cg, scal, cloud, maps, sfc, recs, total;
};

__host__ __device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// nlay: layers whose state the CTA holds; NW: chunks of the column (maps); NWloc: warps of
// the CTA (records).
__host__ __device__ __forceinline__ SmemLayout smem_layout(int nlay, int ngas, int nband, int ncloud_vals, int NW,
                                                           int nmaps, int CL, int nbands_per_group, int nscal,
                                                           int NWloc = -1)
{
    if (NWloc < 0) NWloc = NW;
    SmemLayout L;
    L.state = 0;
    L.cg = align16(L.state + sizeof(LayerState) * size_t(nlay));
    L.scal = align16(L.cg + sizeof(float) * size_t(ngas + 1) * nlay);
    L.cloud = align16(L.scal + sizeof(float) * size_t(nscal) * nlay);
    L.maps = align16(L.cloud + sizeof(float) * size_t(ncloud_vals) * nband * nlay);
    L.sfc = align16(L.maps + sizeof(float4) * size_t(NW) * 32 * nmaps);
    L.recs = align16(L.sfc + sizeof(float) * 64);
    L.total = align16(L.recs + sizeof(Rec) * size_t(NWloc) * CL * nbands_per_group);
    return L;
}

}  // namespace fused
}  // namespace rrtmgp_b200
