// Batched forward of many independent column grids of uneven ncol / nlay in one persistent
// launch (rrtmgp_b200_batch_* in rrtmgp_b200.h).
//
// Work decomposition.  An item is one (grid, spectral domain) pair.  Its columns are cut into
// tiles of P columns; a tile runs on one CTA of 16 warps as P teams of W = ceil(nlay / CL)
// warps, each team computing one column with the fused per-column code of lw_column.cuh /
// sw_column.cuh on its own slice of shared memory and its own hardware barrier (ids 1..P).
// Tiles are numbered item by item, items in order of decreasing tile time, and the
// persistent CTAs (one per SM at 128 registers x 512 threads) take the next tile from a
// device counter, so long tiles go first and the short ones fill the tail.
//
// The reference has no batching of grids: its driver loops over column blocks of one grid
// (src_test/Radiation_solver.cu:467-615 longwave, :683-950 shortwave) and its runtime
// autotuner (include/tuner.h:78-182) times block sizes per kernel on the first call.  Here the
// autotuner times the tile shapes (CL, P) per (domain, 8-layer bin) on the persistent kernel
// itself and keeps the measured tile time as the work-order key.
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>

#include "lw_column.cuh"
#include "sw_column.cuh"

namespace rrtmgp_b200 {
namespace {

using namespace fused;

constexpr int kBatchThreads = 512;   // 16 warps per persistent CTA
constexpr int kBatchWarps = kBatchThreads / 32;
constexpr int kMaxBins = 32;         // nlay <= 256 in 8-layer bins
constexpr int kMaxTeams = 15;        // hardware barriers 1..15 (0 is __syncthreads)

// One (grid, domain) work item as the persistent kernel reads it.
struct BatchItem {
    int ncol, nlay;
    int domain;        // 0 longwave, 1 shortwave
    int cl, W, P;      // chunk length, warps per column, columns per tile
    int team_smem;     // bytes of shared memory per team (16-byte multiple)
    int cloudy, delta;
    CloudLut<float> lut;
    const float *play, *plev, *tlay, *tlev, *tsfc, *col_dry;
    const float *lwp, *iwp, *rel, *rei;
    const float *emis;                           // longwave
    const float *mu0, *tsi, *alb_dir, *alb_dif;  // shortwave
    float *up, *dn, *dir, *net, *hr;
    GasSet<float> gs;
};

// Per-warp view of the current tile: which column the warp's team computes, where the team's
// warps and shared memory start, its hardware barrier.
struct WarpSlot {
    int icol, first_warp, nwarps, bar, smem_off, active, pad0, pad1;
};

// The current tile's item and warp slots, staged in shared memory at every tile.
__shared__ BatchItem g_item;
__shared__ WarpSlot g_slot[kBatchWarps];

__device__ __forceinline__ int warp_uniform(int v) { return __reduce_max_sync(0xffffffffu, v); }

// Team context.  Its values are made warp-uniform (redux) once per tile, so that the compiler
// keeps them in uniform registers and the column code keeps its uniform branches and address
// arithmetic, as with blockIdx / blockDim in the per-grid kernels.
struct TeamCtx {
    int ic, fw, nw, bar, soff;
    __device__ __forceinline__ int icol() const { return ic; }
    __device__ __forceinline__ int warp() const { return int(threadIdx.x >> 5) - fw; }
    __device__ __forceinline__ int nwarps() const { return nw; }
    __device__ __forceinline__ int lwarp() const { return int(threadIdx.x >> 5) - fw; }
    __device__ __forceinline__ int tid() const { return int(threadIdx.x) - 32 * fw; }
    __device__ __forceinline__ int nthreads() const { return 32 * nw; }
    __device__ __forceinline__ int layer0() const { return 0; }
    __device__ __forceinline__ int nloc(int nlay) const { return nlay; }
    template <class T>
    __device__ __forceinline__ void put(T* p, const T& v) const { *p = v; }
    __device__ __forceinline__ unsigned char* smem() const
    {
        extern __shared__ __align__(16) unsigned char smem_raw[];
        return smem_raw + soff;
    }
    __device__ __forceinline__ void sync() const
    {
        asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(32 * nw) : "memory");
    }
};

// Item arguments: the sizes as warp-uniform values, the arrays read from the staged item where
// they are used (setup, once per group of g-points, outputs).
struct ItemIo {
    int nc, nl;
    __device__ __forceinline__ int ncol() const { return nc; }
    __device__ __forceinline__ int nlay() const { return nl; }
    __device__ __forceinline__ const float* play() const { return g_item.play; }
    __device__ __forceinline__ const float* plev() const { return g_item.plev; }
    __device__ __forceinline__ const float* tlay() const { return g_item.tlay; }
    __device__ __forceinline__ const float* tlev() const { return g_item.tlev; }
    __device__ __forceinline__ const float* tsfc() const { return g_item.tsfc; }
    __device__ __forceinline__ const float* col_dry() const { return g_item.col_dry; }
    __device__ __forceinline__ const float* emis() const { return g_item.emis; }
    __device__ __forceinline__ const float* mu0() const { return g_item.mu0; }
    __device__ __forceinline__ const float* tsi() const { return g_item.tsi; }
    __device__ __forceinline__ const float* alb_dir() const { return g_item.alb_dir; }
    __device__ __forceinline__ const float* alb_dif() const { return g_item.alb_dif; }
    __device__ __forceinline__ float* up() const { return g_item.up; }
    __device__ __forceinline__ float* dn() const { return g_item.dn; }
    __device__ __forceinline__ float* dir() const { return g_item.dir; }
    __device__ __forceinline__ float* net() const { return g_item.net; }
    __device__ __forceinline__ float* hr() const { return g_item.hr; }
    __device__ __forceinline__ const GasSet<float>& gs() const { return g_item.gs; }
    __device__ __forceinline__ CloudArgs cloud() const
    {
        return CloudArgs{g_item.lut, g_item.lwp, g_item.iwp, g_item.rel, g_item.rei, g_item.cloudy};
    }
};

struct SwItemIo : ItemIo {
    __device__ __forceinline__ SwAerosolArgs aerosol() const { return SwAerosolArgs{}; }   // no aerosols
    __device__ __forceinline__ SwCloudArgs cloud() const
    {
        return SwCloudArgs{g_item.lut, g_item.lwp, g_item.iwp, g_item.rel, g_item.rei, g_item.cloudy, g_item.delta};
    }
};

// DENSE: a k-distribution with more than three minor intervals over some g-point (tau_abs).
template <bool DENSE>
__global__ void __launch_bounds__(kBatchThreads, 1)
batch_forward_kernel(const KdistView<float> klw, const KdistView<float> ksw, const BatchItem* __restrict__ items,
                     const long long* __restrict__ tile_start, const int* __restrict__ tile_item, int nitems,
                     unsigned long long* __restrict__ counter)
{
    __shared__ long long s_tile;
    __shared__ int s_item;
    const long long ntiles = tile_start[nitems];
    for (;;) {
        if (threadIdx.x == 0) {
            const long long t = (long long)atomicAdd(counter, 1ull);
            s_tile = t;
            s_item = t < ntiles ? __ldg(tile_item + t) : 0;   // the item of tile t: one load
        }
        __syncthreads();
        const long long t = s_tile;
        const int ii = s_item;
        if (t >= ntiles) break;
        // stage the item and the warp slots of this tile
        const int* src = reinterpret_cast<const int*>(items + ii);
        for (int q = threadIdx.x; q < int(sizeof(BatchItem) / 4); q += blockDim.x)
            reinterpret_cast<int*>(&g_item)[q] = __ldg(src + q);
        if (threadIdx.x < kBatchWarps) {
            const BatchItem& it = items[ii];
            const int team = int(threadIdx.x) / it.W;
            const int icol = int(t - tile_start[ii]) * it.P + team;
            WarpSlot sl;
            sl.icol = icol;
            sl.first_warp = team * it.W;
            sl.nwarps = it.W;
            sl.bar = 1 + team;
            sl.smem_off = team * it.team_smem;
            sl.active = team < it.P && icol < it.ncol;
            sl.pad0 = sl.pad1 = 0;
            g_slot[threadIdx.x] = sl;
        }
        __syncthreads();
        const WarpSlot& q = g_slot[threadIdx.x >> 5];
        if (warp_uniform(q.active)) {
            // The shared-memory offset is rebuilt from a 16-byte count so that the compiler knows
            // its alignment (with an unknown low part, the column code ran ~15% slower).
            const TeamCtx cx{warp_uniform(q.icol), warp_uniform(q.first_warp), warp_uniform(q.nwarps),
                             warp_uniform(q.bar), warp_uniform(q.smem_off >> 4) << 4};
            const int domain = warp_uniform(g_item.domain), cl = warp_uniform(g_item.cl);
            const int nc = warp_uniform(g_item.ncol), nl = warp_uniform(g_item.nlay);
            if (domain == 0) {
                const ItemIo io{nc, nl};
                if (cl == 8)
                    lw_forward_column<8, false, DENSE>(cx, klw, io);
                else
                    lw_forward_column<16, false, DENSE>(cx, klw, io);
            } else {
                const SwItemIo io{{nc, nl}};
                if (cl == 8)
                    sw_forward_column<8, true, DENSE>(cx, ksw, io);
                else
                    sw_forward_column<16, false, DENSE>(cx, ksw, io);
            }
        }
        __syncthreads();
    }
}

struct TileShape {
    int cl = 0, P = 0;
    float tile_us = 0.f;   // measured time of one tile; 0 = not measured
};

int ceil_div_i(int a, int b) { return (a + b - 1) / b; }

CloudLut<float> lut_of(rrtmgp_b200_cloud c)
{
    if (!c) return CloudLut<float>{};
    return CloudLut<float>{c->nband, c->nsize_liq, c->nsize_ice, float(c->radliq_lwr), float(c->liq_step),
                           float(c->radice_lwr), float(c->ice_step), c->lut32};
}

}  // namespace

// Single-grid fused forwards (forward_lw.cu, forward_sw.cu), the per-grid comparison path.
int forward_lw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay, const float* play,
                   const float* plev, const float* tlay, const float* tlev, const float* tsfc, const float* col_dry,
                   const rrtmgp_b200_gas_conc* gases, int ngases, const float* lwp, const float* iwp,
                   const float* rel, const float* rei, const float* sfc_emis, float* flux_up, float* flux_dn,
                   float* flux_net, float* heating_rate, int chunk, void* stream);
int forward_sw_f32(rrtmgp_b200_kdist k, rrtmgp_b200_cloud c, int ncol, int nlay, const float* play,
                   const float* plev, const float* tlay, const float* col_dry, const rrtmgp_b200_gas_conc* gases,
                   int ngases, const float* lwp, const float* iwp, const float* rel, const float* rei,
                   int delta_cloud, const float* mu0, const float* tsi_scaling, const float* sfc_alb_dir,
                   const float* sfc_alb_dif, float* flux_up, float* flux_dn, float* flux_dn_dir, float* flux_net,
                   float* heating_rate, int chunk, void* stream);

namespace {

bool batch_layout_ok(const KdistView<float>& v, bool sw) { return fused_layout_ok(v, sw, 8); }

}  // namespace
}  // namespace rrtmgp_b200

using namespace rrtmgp_b200;

struct rrtmgp_b200_batch_t {
    rrtmgp_b200_kdist k[2] = {nullptr, nullptr};
    rrtmgp_b200_cloud c[2] = {nullptr, nullptr};
    int delta = 1;
    std::vector<rrtmgp_b200_batch_grid> grids;
    std::vector<std::vector<rrtmgp_b200_gas_conc>> gases;   // per grid, copies of the host arrays
    std::vector<std::vector<std::string>> gas_names;
    std::vector<BatchItem> items;      // unplanned items (cl, W, P, team_smem set by plan())
    TileShape shape[2][kMaxBins + 1];  // [domain][bin]
    int nsm = 0, device = 0;
    bool dense = false;                // a k-distribution needs the DENSE kernel
    int max_smem = 0;                  // dynamic shared memory per CTA the kernel may use
    // planned state
    bool dirty = true;
    std::vector<BatchItem> order;      // planned items in work order
    std::vector<long long> starts;
    long long ntiles = 0;
    int ctas = 0;
    size_t smem = 0;
    BatchItem* d_items = nullptr;
    long long* d_starts = nullptr;
    int* d_tile_item = nullptr;        // item of every tile (work order)
    size_t cap_tiles = 0;
    size_t cap_items = 0;
    unsigned long long* d_counter = nullptr;
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace rrtmgp_b200 {
namespace {

size_t team_smem_bytes(const rrtmgp_b200_batch_t* b, int domain, int nlay, int cl)
{
    const KdistView<float>& v = b->k[domain]->v32;
    const int W = ceil_div_i(nlay, cl);
    // as the column code lays it out: by capacity, W cl layers
    const SmemLayout L = domain == 0 ? smem_layout(W * cl, v.ngas, v.nband, 1, W, 2, cl, v.max_group_bands, v.max_nscal)
                                     : smem_layout(W * cl, v.ngas, v.nband, 0, W, 3, cl,
                                                   v.max_group_bands * (cl == 8 ? 2 : 1), v.max_nscal);
    return align16(L.total);
}

// Largest P for a shape, 0 when the chunk length cannot hold nlay.
int max_columns(const rrtmgp_b200_batch_t* b, int domain, int nlay, int cl)
{
    const int W = ceil_div_i(nlay, cl);
    if (W > kBatchWarps) return 0;
    const size_t per = team_smem_bytes(b, domain, nlay, cl);
    return int(std::min<size_t>(std::min(kBatchWarps / W, kMaxTeams), size_t(b->max_smem) / per));
}

// Shape of (domain, bin) for a grid of nlay layers: the stored shape when it fits, else the
// heuristic (most busy warps, then the shorter chunk).
TileShape shape_for(const rrtmgp_b200_batch_t* b, int domain, int nlay)
{
    const int bin = ceil_div_i(nlay, 8);
    TileShape s = b->shape[domain][bin];
    if (s.cl && s.P >= 1 && s.P <= max_columns(b, domain, nlay, s.cl)) return s;
    TileShape best;
    int best_busy = -1;
    for (int cl : {8, 16}) {
        const int P = max_columns(b, domain, nlay, cl);
        if (P < 1) continue;
        const int busy = P * ceil_div_i(nlay, cl);
        if (busy > best_busy) {
            best_busy = busy;
            best.cl = cl;
            best.P = P;
        }
    }
    return best;
}

// Relative tile time used to order work when no measurement exists: the serial sweep length
// (chunk) plus the composition over the column's chunks.
float tile_cost(const TileShape& s, int nlay)
{
    if (s.tile_us > 0.f) return s.tile_us;
    return float(s.cl) + 0.5f * float(ceil_div_i(nlay, s.cl));
}

BatchItem planned(const rrtmgp_b200_batch_t* b, const BatchItem& in, const TileShape& s)
{
    BatchItem it = in;
    it.cl = s.cl;
    it.P = s.P;
    it.W = ceil_div_i(it.nlay, s.cl);
    it.team_smem = int(team_smem_bytes(b, it.domain, it.nlay, s.cl));
    return it;
}

void release_graph(rrtmgp_b200_batch_t* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

int ensure_capacity(rrtmgp_b200_batch_t* b, size_t n)
{
    if (n <= b->cap_items) return RRTMGP_B200_OK;
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_starts) cudaFree(b->d_starts);
    b->d_items = nullptr;
    b->d_starts = nullptr;
    b->cap_items = 0;
    if (cudaMalloc(&b->d_items, sizeof(BatchItem) * n) != cudaSuccess ||
        cudaMalloc(&b->d_starts, sizeof(long long) * (n + 1)) != cudaSuccess) {
        cudaGetLastError();
        return fail(RRTMGP_B200_ERR_ALLOC, "batch: device work table allocation failed");
    }
    b->cap_items = n;
    return RRTMGP_B200_OK;
}

// Uploads a work list (already in work order) and returns its tile count and shared memory.
int upload(rrtmgp_b200_batch_t* b, const std::vector<BatchItem>& list, long long& ntiles, size_t& smem)
{
    std::vector<long long> starts(list.size() + 1, 0);
    smem = 0;
    for (size_t i = 0; i < list.size(); ++i) {
        starts[i + 1] = starts[i] + ceil_div_i(list[i].ncol, list[i].P);
        smem = std::max(smem, size_t(list[i].P) * size_t(list[i].team_smem));
    }
    ntiles = starts.back();
    int st = ensure_capacity(b, std::max<size_t>(list.size(), 1));
    if (st) return st;
    std::vector<int> tile_item(size_t(std::max<long long>(ntiles, 1)), 0);
    for (size_t i = 0; i < list.size(); ++i)
        std::fill(tile_item.begin() + starts[i], tile_item.begin() + starts[i + 1], int(i));
    if (tile_item.size() > b->cap_tiles) {
        if (b->d_tile_item) cudaFree(b->d_tile_item);
        b->d_tile_item = nullptr;
        b->cap_tiles = 0;
        if (cudaMalloc(&b->d_tile_item, sizeof(int) * tile_item.size()) != cudaSuccess) {
            cudaGetLastError();
            return fail(RRTMGP_B200_ERR_ALLOC, "batch: tile table allocation failed");
        }
        b->cap_tiles = tile_item.size();
    }
    RB_CUDA(cudaMemcpy(b->d_tile_item, tile_item.data(), sizeof(int) * tile_item.size(), cudaMemcpyHostToDevice),
            "batch: tile table upload");
    RB_CUDA(cudaMemcpy(b->d_items, list.data(), sizeof(BatchItem) * list.size(), cudaMemcpyHostToDevice),
            "batch: work table upload");
    RB_CUDA(cudaMemcpy(b->d_starts, starts.data(), sizeof(long long) * starts.size(), cudaMemcpyHostToDevice),
            "batch: work table upload");
    return RRTMGP_B200_OK;
}

int plan(rrtmgp_b200_batch_t* b)
{
    if (!b->dirty) return RRTMGP_B200_OK;
    release_graph(b);
    std::vector<std::pair<float, BatchItem>> keyed;
    keyed.reserve(b->items.size());
    for (const BatchItem& in : b->items) {
        const TileShape s = shape_for(b, in.domain, in.nlay);
        if (!s.cl) return fail(RRTMGP_B200_ERR_UNSUPPORTED, "batch: no tile shape holds nlay = " +
                                                                std::to_string(in.nlay));
        keyed.emplace_back(tile_cost(s, in.nlay), planned(b, in, s));
    }
    std::stable_sort(keyed.begin(), keyed.end(),
                     [](const std::pair<float, BatchItem>& x, const std::pair<float, BatchItem>& y) {
                         return x.first > y.first;
                     });
    b->order.clear();
    for (auto& kv : keyed) b->order.push_back(kv.second);
    int st = upload(b, b->order, b->ntiles, b->smem);
    if (st) return st;
    b->ctas = int(std::min<long long>(b->nsm, std::max<long long>(b->ntiles, 1)));
    b->dirty = false;
    return RRTMGP_B200_OK;
}

int launch_persistent(rrtmgp_b200_batch_t* b, const BatchItem* d_items, const long long* d_starts, int nitems,
                      long long ntiles, size_t smem, cudaStream_t s)
{
    RB_CUDA(cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), s), "batch: counter reset");
    const int ctas = int(std::min<long long>(b->nsm, std::max<long long>(ntiles, 1)));
    const KdistView<float> klw = b->k[0] ? b->k[0]->v32 : KdistView<float>{};
    const KdistView<float> ksw = b->k[1] ? b->k[1]->v32 : KdistView<float>{};
    if (b->dense)
        batch_forward_kernel<true><<<ctas, kBatchThreads, smem, s>>>(klw, ksw, d_items, d_starts, b->d_tile_item, nitems,
                                                                     b->d_counter);
    else
        batch_forward_kernel<false><<<ctas, kBatchThreads, smem, s>>>(klw, ksw, d_items, d_starts, b->d_tile_item,
                                                                      nitems, b->d_counter);
    RB_LAUNCH("batch_forward_kernel");
    return RRTMGP_B200_OK;
}

int run_per_grid(rrtmgp_b200_batch_t* b, cudaStream_t s)
{
    for (const rrtmgp_b200_batch_grid& g : b->grids) {
        const bool cloudy = g.lwp != nullptr;
        if (g.lw_flux_up) {
            int st = forward_lw_f32(b->k[0], cloudy ? b->c[0] : nullptr, g.ncol, g.nlay, g.play, g.plev, g.tlay,
                                    g.tlev, g.tsfc, g.col_dry, g.gases, g.ngases, g.lwp, g.iwp, g.rel, g.rei,
                                    g.sfc_emis, g.lw_flux_up, g.lw_flux_dn, g.lw_flux_net, g.lw_heating_rate,
                                    0, s);
            if (st) return st;
        }
        if (g.sw_flux_up) {
            int st = forward_sw_f32(b->k[1], cloudy ? b->c[1] : nullptr, g.ncol, g.nlay, g.play, g.plev, g.tlay,
                                    g.col_dry, g.gases, g.ngases, g.lwp, g.iwp, g.rel, g.rei, b->delta, g.mu0,
                                    g.tsi_scaling, g.sfc_alb_dir, g.sfc_alb_dif, g.sw_flux_up, g.sw_flux_dn,
                                    g.sw_flux_dn_dir, g.sw_flux_net, g.sw_heating_rate, 0, s);
            if (st) return st;
        }
    }
    return RRTMGP_B200_OK;
}

int batch_create(rrtmgp_b200_kdist klw, rrtmgp_b200_cloud clw, rrtmgp_b200_kdist ksw, rrtmgp_b200_cloud csw,
                 int delta, const rrtmgp_b200_batch_grid* grids, int ngrids, rrtmgp_b200_batch* out)
{
    RB_CHECK_ARG(out, "batch_create: null output handle");
    *out = nullptr;
    RB_CHECK_ARG(grids && ngrids > 0, "batch_create: no grids");
    RB_CHECK_ARG(!klw || klw->info.is_longwave, "batch_create: k_lw is not a longwave k-distribution");
    RB_CHECK_ARG(!ksw || !ksw->info.is_longwave, "batch_create: k_sw is not a shortwave k-distribution");
    RB_CHECK_ARG(!clw || (klw && clw->nband == klw->info.nband), "batch_create: longwave cloud bands differ");
    RB_CHECK_ARG(!csw || (ksw && csw->nband == ksw->info.nband), "batch_create: shortwave cloud bands differ");
    if ((klw && !batch_layout_ok(klw->v32, false)) || (ksw && !batch_layout_ok(ksw->v32, true)))
        return fail(RRTMGP_B200_ERR_UNSUPPORTED, "batch_create: k-distribution layout not supported");
    std::unique_ptr<rrtmgp_b200_batch_t> b(new rrtmgp_b200_batch_t);
    b->k[0] = klw;
    b->k[1] = ksw;
    b->c[0] = clw;
    b->c[1] = csw;
    b->delta = delta;
    for (int i = 0; i < ngrids; ++i) {
        const rrtmgp_b200_batch_grid& g = grids[i];
        const std::string at = "batch_create: grid " + std::to_string(i) + ": ";
        RB_CHECK_ARG(g.ncol > 0 && g.nlay > 1 && g.nlay <= 8 * kMaxBins, at + "need ncol > 0 and 1 < nlay <= 256");
        RB_CHECK_ARG(g.play && g.plev && g.tlay, at + "null atmosphere array");
        const bool cloudy = g.lwp != nullptr;
        RB_CHECK_ARG(!cloudy || (g.iwp && g.rel && g.rei), at + "cloud arrays must be all set or all NULL");
        RB_CHECK_ARG(g.lw_flux_up || g.sw_flux_up, at + "neither longwave nor shortwave outputs");
        BatchItem base{};
        base.delta = delta;
        base.ncol = g.ncol;
        base.nlay = g.nlay;
        base.play = g.play;
        base.plev = g.plev;
        base.tlay = g.tlay;
        base.col_dry = g.col_dry;
        base.lwp = g.lwp;
        base.iwp = g.iwp;
        base.rel = g.rel;
        base.rei = g.rei;
        if (g.lw_flux_up) {
            RB_CHECK_ARG(klw, at + "longwave outputs without a longwave k-distribution");
            RB_CHECK_ARG(g.tlev && g.tsfc && g.sfc_emis && g.lw_flux_dn && g.lw_flux_net && g.lw_heating_rate,
                         at + "null longwave array");
            BatchItem it = base;
            it.domain = 0;
            it.cloudy = cloudy && clw;
            it.lut = lut_of(clw);
            it.tlev = g.tlev;
            it.tsfc = g.tsfc;
            it.emis = g.sfc_emis;
            it.up = g.lw_flux_up;
            it.dn = g.lw_flux_dn;
            it.net = g.lw_flux_net;
            it.hr = g.lw_heating_rate;
            int st = make_gas_set<float>(klw, g.ncol, g.nlay, g.gases, g.ngases, it.gs);
            if (st) return st;
            b->items.push_back(it);
        }
        if (g.sw_flux_up) {
            RB_CHECK_ARG(ksw, at + "shortwave outputs without a shortwave k-distribution");
            RB_CHECK_ARG(g.mu0 && g.sfc_alb_dir && g.sfc_alb_dif && g.sw_flux_dn && g.sw_flux_dn_dir &&
                         g.sw_flux_net && g.sw_heating_rate, at + "null shortwave array");
            BatchItem it = base;
            it.domain = 1;
            it.cloudy = cloudy && csw;
            it.lut = lut_of(csw);
            it.mu0 = g.mu0;
            it.tsi = g.tsi_scaling;
            it.alb_dir = g.sfc_alb_dir;
            it.alb_dif = g.sfc_alb_dif;
            it.up = g.sw_flux_up;
            it.dn = g.sw_flux_dn;
            it.dir = g.sw_flux_dn_dir;
            it.net = g.sw_flux_net;
            it.hr = g.sw_heating_rate;
            int st = make_gas_set<float>(ksw, g.ncol, g.nlay, g.gases, g.ngases, it.gs);
            if (st) return st;
            b->items.push_back(it);
        }
        b->gas_names.emplace_back();
        b->gases.emplace_back();
        for (int j = 0; j < g.ngases; ++j) b->gas_names.back().push_back(g.gases[j].name ? g.gases[j].name : "");
        for (int j = 0; j < g.ngases; ++j) {
            rrtmgp_b200_gas_conc c = g.gases[j];
            c.name = b->gas_names.back()[j].c_str();
            b->gases.back().push_back(c);
        }
        b->grids.push_back(g);
    }
    for (size_t i = 0; i < b->grids.size(); ++i) b->grids[i].gases = b->gases[i].data();
    RB_CUDA(cudaGetDevice(&b->device), "batch_create");
    RB_CUDA(cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->device), "batch_create");
    int optin = 0;
    RB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device), "batch_create");
    b->dense = (klw && klw->v32.max_minor_per_g > 3) || (ksw && ksw->v32.max_minor_per_g > 3);
    const auto kernel = b->dense ? batch_forward_kernel<true> : batch_forward_kernel<false>;
    cudaFuncAttributes fa{};
    RB_CUDA(cudaFuncGetAttributes(&fa, kernel), "batch_create");
    b->max_smem = optin - int(fa.sharedSizeBytes);
    RB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, b->max_smem),
            "batch_create: kernel attribute");
    for (const BatchItem& it : b->items)
        if (!shape_for(b.get(), it.domain, it.nlay).cl)
            return fail(RRTMGP_B200_ERR_UNSUPPORTED, "batch_create: shared memory need too large for nlay = " +
                                                         std::to_string(it.nlay));
    if (cudaMalloc(&b->d_counter, sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        return fail(RRTMGP_B200_ERR_ALLOC, "batch_create: counter allocation failed");
    }
    *out = b.release();
    return RRTMGP_B200_OK;
}

int batch_autotune(rrtmgp_b200_batch_t* b, int reps, cudaStream_t s)
{
    RB_CHECK_ARG(reps >= 1 && reps <= 100, "batch_autotune: reps must be in 1..100");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    RB_CUDA(cudaEventCreate(&e0), "batch_autotune");
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_status(cudaGetLastError(), "batch_autotune");
    }
    int st = RRTMGP_B200_OK;
    for (int domain = 0; domain < 2 && !st; ++domain) {
        // widest grid of each bin (then the deepest) is the sample
        std::map<int, const BatchItem*> sample;
        for (const BatchItem& it : b->items) {
            if (it.domain != domain) continue;
            const BatchItem*& cur = sample[ceil_div_i(it.nlay, 8)];
            if (!cur || it.ncol > cur->ncol || (it.ncol == cur->ncol && it.nlay > cur->nlay)) cur = &it;
        }
        for (const auto& kv : sample) {
            const BatchItem& rep_item = *kv.second;
            TileShape best;
            float best_col_us = 0.f;
            for (int cl : {8, 16}) {
                const int pmax = max_columns(b, domain, rep_item.nlay, cl);
                for (int P = 1; P <= pmax && !st; ++P) {
                    TileShape cand;
                    cand.cl = cl;
                    cand.P = P;
                    const BatchItem it = planned(b, rep_item, cand);
                    const int tiles_per_copy = ceil_div_i(it.ncol, P);
                    const int copies = std::min(256, std::max(1, ceil_div_i(3 * b->nsm, tiles_per_copy)));
                    const std::vector<BatchItem> list(size_t(copies), it);
                    long long ntiles = 0;
                    size_t smem = 0;
                    st = upload(b, list, ntiles, smem);
                    if (st) break;
                    float ms_min = 0.f;
                    for (int r = -1; r < reps && !st; ++r) {   // r = -1: warm-up
                        cudaEventRecord(e0, s);
                        st = launch_persistent(b, b->d_items, b->d_starts, copies, ntiles, smem, s);
                        cudaEventRecord(e1, s);
                        if (st) break;
                        if (cudaEventSynchronize(e1) != cudaSuccess) {
                            st = cuda_status(cudaGetLastError(), "batch_autotune: sample run");
                            break;
                        }
                        float ms = 0.f;
                        cudaEventElapsedTime(&ms, e0, e1);
                        if (r >= 0 && (r == 0 || ms < ms_min)) ms_min = ms;
                    }
                    if (st) break;
                    const float col_us = 1000.f * ms_min / float(copies * it.ncol);
                    if (!best.cl || col_us < best_col_us) {
                        const int ctas = int(std::min<long long>(b->nsm, ntiles));
                        best = cand;
                        best.tile_us = 1000.f * ms_min * float(ctas) / float(ntiles);
                        best_col_us = col_us;
                    }
                }
            }
            if (st) break;
            b->shape[domain][kv.first] = best;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->dirty = true;
    return st;
}

}  // namespace
}  // namespace rrtmgp_b200

extern "C" int rrtmgp_b200_batch_create(rrtmgp_b200_kdist k_lw, rrtmgp_b200_cloud cloud_lw, rrtmgp_b200_kdist k_sw,
                                        rrtmgp_b200_cloud cloud_sw, int delta_cloud,
                                        const rrtmgp_b200_batch_grid* grids, int ngrids, rrtmgp_b200_batch* out)
{
    return batch_create(k_lw, cloud_lw, k_sw, cloud_sw, delta_cloud, grids, ngrids, out);
}

extern "C" int rrtmgp_b200_batch_destroy(rrtmgp_b200_batch b)
{
    if (!b) return RRTMGP_B200_OK;
    release_graph(b);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_starts) cudaFree(b->d_starts);
    if (b->d_tile_item) cudaFree(b->d_tile_item);
    if (b->d_counter) cudaFree(b->d_counter);
    delete b;
    return RRTMGP_B200_OK;
}

extern "C" int rrtmgp_b200_batch_run(rrtmgp_b200_batch b, int mode, void* stream)
{
    RB_CHECK_ARG(b, "batch_run: null batch");
    cudaStream_t s = as_stream(stream);
    if (mode == RRTMGP_B200_BATCH_PER_GRID) return run_per_grid(b, s);
    RB_CHECK_ARG(mode == RRTMGP_B200_BATCH_PERSISTENT || mode == RRTMGP_B200_BATCH_GRAPH, "batch_run: bad mode");
    int st = plan(b);
    if (st) return st;
    if (mode == RRTMGP_B200_BATCH_PERSISTENT)
        return launch_persistent(b, b->d_items, b->d_starts, int(b->order.size()), b->ntiles, b->smem, s);
    if (!b->exec) {
        if (!b->cap_stream) RB_CUDA(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking), "batch graph");
        RB_CUDA(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal), "batch graph capture");
        st = launch_persistent(b, b->d_items, b->d_starts, int(b->order.size()), b->ntiles, b->smem, b->cap_stream);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->cap_stream, &g);
        if (st) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        RB_CUDA(e, "batch graph capture");
        b->graph = g;
        RB_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0), "batch graph instantiate");
    }
    RB_CUDA(cudaGraphLaunch(b->exec, s), "batch graph launch");
    return RRTMGP_B200_OK;
}

extern "C" int rrtmgp_b200_batch_autotune(rrtmgp_b200_batch b, int reps, void* stream)
{
    RB_CHECK_ARG(b, "batch_autotune: null batch");
    return batch_autotune(b, reps, as_stream(stream));
}

extern "C" int rrtmgp_b200_batch_get_plan(rrtmgp_b200_batch b, int domain, int bin, int* chunk, int* columns,
                                          float* tile_us)
{
    RB_CHECK_ARG(b && chunk && columns && tile_us, "batch_get_plan: null argument");
    RB_CHECK_ARG((domain == 0 || domain == 1) && b->k[domain], "batch_get_plan: domain not in the batch");
    RB_CHECK_ARG(bin >= 1 && bin <= kMaxBins, "batch_get_plan: bin must be in 1..32");
    const TileShape s = shape_for(b, domain, 8 * bin);
    *chunk = s.cl;
    *columns = s.P;
    *tile_us = s.tile_us;
    return RRTMGP_B200_OK;
}

extern "C" int rrtmgp_b200_batch_set_plan(rrtmgp_b200_batch b, int domain, int bin, int chunk, int columns,
                                          float tile_us)
{
    RB_CHECK_ARG(b, "batch_set_plan: null batch");
    RB_CHECK_ARG((domain == 0 || domain == 1) && b->k[domain], "batch_set_plan: domain not in the batch");
    RB_CHECK_ARG(bin >= 1 && bin <= kMaxBins, "batch_set_plan: bin must be in 1..32");
    RB_CHECK_ARG(chunk == 8 || chunk == 16, "batch_set_plan: chunk must be 8 or 16");
    RB_CHECK_ARG(columns >= 1 && columns <= max_columns(b, domain, 8 * bin, chunk),
                 "batch_set_plan: columns per CTA do not fit the warps, barriers or shared memory");
    RB_CHECK_ARG(tile_us >= 0.f, "batch_set_plan: negative tile time");
    TileShape& t = b->shape[domain][bin];
    t.cl = chunk;
    t.P = columns;
    t.tile_us = tile_us;
    b->dirty = true;
    return RRTMGP_B200_OK;
}

extern "C" int rrtmgp_b200_batch_stats(rrtmgp_b200_batch b, long long* ntiles, int* ctas, int* smem_bytes,
                                       int* launches_persistent, int* launches_per_grid)
{
    RB_CHECK_ARG(b, "batch_stats: null batch");
    int st = plan(b);
    if (st) return st;
    if (ntiles) *ntiles = b->ntiles;
    if (ctas) *ctas = b->ctas;
    if (smem_bytes) *smem_bytes = int(b->smem);
    if (launches_persistent) *launches_persistent = 1;
    if (launches_per_grid) *launches_per_grid = int(b->items.size());
    return RRTMGP_B200_OK;
}
