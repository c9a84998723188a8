// Cloud optics LUT, delta scaling and add_to (optical-property arithmetic).
#include <cfloat>
#include <cstdint>

#include "common.cuh"
#include "optics_device.cuh"

namespace rrtmgp_b200 {
namespace {

// Cloud_optics_gpu::cloud_optics (src_cuda/Cloud_optics.cu:30-126): one thread per
// (column, layer); the LUT index and weight depend only on r_eff, so they are computed once
// and reused for every band (the reference recomputes them per band and stores six
// (ncol, nlay, nband) temporaries).
template <typename T, bool TwoStream>
__global__ void cloud_optics_kernel(int ncol, int nlay, int nband, int nsl, int nsi,
                                    T liq_lwr, T liq_step, T ice_lwr, T ice_step,
                                    const T* __restrict__ lut, const T* __restrict__ clwp,
                                    const T* __restrict__ ciwp, const T* __restrict__ reliq,
                                    const T* __restrict__ reice, T* __restrict__ tau,
                                    T* __restrict__ ssa, T* __restrict__ g)
{
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t ncl = size_t(ncol) * nlay;
    if (i >= ncl) return;
    const CloudLut<T> L{nband, nsl, nsi, liq_lwr, liq_step, ice_lwr, ice_step, lut};
    const CloudPoint<T> cp = cloud_point(L, clwp[i], ciwp[i], reliq[i], reice[i]);
    for (int b = 0; b < nband; ++b) {
        T t, s, gg;
        cloud_band<T, TwoStream>(L, cp, b, t, s, gg);
        tau[i + size_t(b) * ncl] = t;
        if (TwoStream) {
            ssa[i + size_t(b) * ncl] = s;
            g[i + size_t(b) * ncl] = gg;
        }
    }
}

// delta_scale_2str_k_kernel (optical_props_kernels.cu:139-160).
template <typename T>
__global__ void delta_scale_kernel(size_t n, T* __restrict__ tau, T* __restrict__ ssa, T* __restrict__ g)
{
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T t = tau[i], s = ssa[i], a = g[i];
    delta_scale_point(t, s, a);
    tau[i] = t; ssa[i] = s; g[i] = a;
}

// increment_1scalar_by_1scalar / inc_1scalar_by_1scalar_bybnd (optical_props_kernels.cu:30-98);
// bybnd uses gpt2band instead of scanning all bands per element.
// add_to kernels: grid (column-layer blocks, g-point), so no thread divides its flat index;
// 16 bytes per array and thread (4 FP32 / 2 FP64 values) when ncl and the pointers allow.
template <typename T>
struct alignas(16) Vec16 {
    T v[16 / sizeof(T)];
};

// increment_1scalar_by_1scalar / inc_1scalar_by_1scalar_bybnd (optical_props_kernels.cu:30-43).
template <typename T, bool VEC>
__global__ void add_1scl_kernel(size_t ncl, T* __restrict__ tau1, const T* __restrict__ tau2,
                                const int* __restrict__ gpt2band)
{
    constexpr int V = VEC ? 16 / sizeof(T) : 1;
    const int gpt = blockIdx.y;
    const size_t src = size_t(gpt2band ? gpt2band[gpt] : gpt);
    const size_t i = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) * V;
    if (i >= ncl) return;
    T* const t1 = tau1 + size_t(gpt) * ncl + i;
    const T* const t2 = tau2 + src * ncl + i;
    if constexpr (VEC) {
        Vec16<T> a = *reinterpret_cast<const Vec16<T>*>(t1);
        const Vec16<T> b = *reinterpret_cast<const Vec16<T>*>(t2);
#pragma unroll
        for (int q = 0; q < V; ++q) a.v[q] = a.v[q] + b.v[q];
        *reinterpret_cast<Vec16<T>*>(t1) = a;
    } else {
        t1[0] = t1[0] + t2[0];
    }
}

// increment_2stream_by_2stream / inc_2stream_by_2stream_bybnd (:44-136).
template <typename T, bool VEC>
__global__ void add_2str_kernel(size_t ncl, T* __restrict__ tau1, T* __restrict__ ssa1, T* __restrict__ g1,
                                const T* __restrict__ tau2, const T* __restrict__ ssa2, const T* __restrict__ g2,
                                const int* __restrict__ gpt2band)
{
    constexpr int V = VEC ? 16 / sizeof(T) : 1;
    const int gpt = blockIdx.y;
    const size_t src = size_t(gpt2band ? gpt2band[gpt] : gpt);
    const size_t i = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) * V;
    if (i >= ncl) return;
    const size_t o1 = size_t(gpt) * ncl + i, o2 = src * ncl + i;
    if constexpr (VEC) {
        using W = Vec16<T>;
        W t = *reinterpret_cast<const W*>(tau1 + o1), s = *reinterpret_cast<const W*>(ssa1 + o1),
          a = *reinterpret_cast<const W*>(g1 + o1);
        const W t2 = *reinterpret_cast<const W*>(tau2 + o2), s2 = *reinterpret_cast<const W*>(ssa2 + o2),
                a2 = *reinterpret_cast<const W*>(g2 + o2);
#pragma unroll
        for (int q = 0; q < V; ++q) add_2str_point(t.v[q], s.v[q], a.v[q], t2.v[q], s2.v[q], a2.v[q]);
        *reinterpret_cast<W*>(tau1 + o1) = t;
        *reinterpret_cast<W*>(ssa1 + o1) = s;
        *reinterpret_cast<W*>(g1 + o1) = a;
    } else {
        T t = tau1[o1], s = ssa1[o1], a = g1[o1];
        add_2str_point(t, s, a, tau2[o2], ssa2[o2], g2[o2]);
        tau1[o1] = t; ssa1[o1] = s; g1[o1] = a;
    }
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <typename T>
int cloud_optics(rrtmgp_b200_cloud c, int ncol, int nlay, const T* clwp, const T* ciwp, const T* reliq,
                 const T* reice, T* tau, T* ssa, T* g, bool two_stream, void* stream)
{
    RB_CHECK_ARG(c, "cloud_optics: null cloud handle");
    RB_CHECK_ARG(ncol > 0 && nlay > 0, "cloud_optics: ncol and nlay must be > 0");
    RB_CHECK_ARG(clwp && ciwp && reliq && reice && tau && (!two_stream || (ssa && g)), "cloud_optics: null array");
    const size_t n = size_t(ncol) * nlay;
    const int grid = ceil_div(long(n), 128);
    if (two_stream)
        cloud_optics_kernel<T, true><<<grid, 128, 0, as_stream(stream)>>>(
            ncol, nlay, c->nband, c->nsize_liq, c->nsize_ice, T(c->radliq_lwr), T(c->liq_step), T(c->radice_lwr),
            T(c->ice_step), cloud_lut<T>(c), clwp, ciwp, reliq, reice, tau, ssa, g);
    else
        cloud_optics_kernel<T, false><<<grid, 128, 0, as_stream(stream)>>>(
            ncol, nlay, c->nband, c->nsize_liq, c->nsize_ice, T(c->radliq_lwr), T(c->liq_step), T(c->radice_lwr),
            T(c->ice_step), cloud_lut<T>(c), clwp, ciwp, reliq, reice, tau, nullptr, nullptr);
    RB_LAUNCH("cloud_optics_kernel");
    return RRTMGP_B200_OK;
}

template <typename T>
int delta_scale(int ncol, int nlay, int ngpt, T* tau, T* ssa, T* g, void* stream)
{
    RB_CHECK_ARG(ncol > 0 && nlay > 0 && ngpt > 0 && tau && ssa && g, "delta_scale: bad argument");
    const size_t n = size_t(ncol) * nlay * ngpt;
    delta_scale_kernel<T><<<ceil_div(long(n), 256), 256, 0, as_stream(stream)>>>(n, tau, ssa, g);
    RB_LAUNCH("delta_scale_kernel");
    return RRTMGP_B200_OK;
}

// add_to dispatch (src/Optical_props.cpp:218-268): same g-points, or band broadcast.
inline int resolve_add(rrtmgp_b200_bands b, int ngpt_in, const int** g2b)
{
    RB_CHECK_ARG(b, "add_to: null bands");
    RB_CHECK_ARG(b->ngpt <= 65535, "add_to: more than 65535 g-points");
    if (ngpt_in == b->ngpt) { *g2b = nullptr; return RRTMGP_B200_OK; }
    if (ngpt_in == b->nband) { *g2b = b->d_gpt2band; return RRTMGP_B200_OK; }
    return fail(RRTMGP_B200_ERR_ARG, "Cannot add optical properties with incompatible band - gpoint combination");
}

template <typename T>
int add_to_1scl(rrtmgp_b200_bands b, int ncol, int nlay, T* tau1, const T* tau2, int ngpt_in, void* stream)
{
    const int* g2b = nullptr;
    int st = resolve_add(b, ngpt_in, &g2b);
    if (st) return st;
    RB_CHECK_ARG(ncol > 0 && nlay > 0 && tau1 && tau2, "add_to_1scl: bad argument");
    const size_t ncl = size_t(ncol) * nlay;
    constexpr size_t V = 16 / sizeof(T);
    if (ncl % V == 0 && aligned16(tau1) && aligned16(tau2))
        add_1scl_kernel<T, true><<<dim3(unsigned(ceil_div(long(ncl / V), 256)), b->ngpt), 256, 0, as_stream(stream)>>>(
            ncl, tau1, tau2, g2b);
    else
        add_1scl_kernel<T, false><<<dim3(unsigned(ceil_div(long(ncl), 256)), b->ngpt), 256, 0, as_stream(stream)>>>(
            ncl, tau1, tau2, g2b);
    RB_LAUNCH("add_1scl_kernel");
    return RRTMGP_B200_OK;
}

template <typename T>
int add_to_2str(rrtmgp_b200_bands b, int ncol, int nlay, T* tau1, T* ssa1, T* g1, const T* tau2,
                const T* ssa2, const T* g2, int ngpt_in, void* stream)
{
    const int* g2b = nullptr;
    int st = resolve_add(b, ngpt_in, &g2b);
    if (st) return st;
    RB_CHECK_ARG(ncol > 0 && nlay > 0 && tau1 && ssa1 && g1 && tau2 && ssa2 && g2, "add_to_2str: bad argument");
    const size_t ncl = size_t(ncol) * nlay;
    constexpr size_t V = 16 / sizeof(T);
    if (ncl % V == 0 && aligned16(tau1) && aligned16(ssa1) && aligned16(g1) && aligned16(tau2) && aligned16(ssa2) &&
        aligned16(g2))
        add_2str_kernel<T, true><<<dim3(unsigned(ceil_div(long(ncl / V), 256)), b->ngpt), 256, 0, as_stream(stream)>>>(
            ncl, tau1, ssa1, g1, tau2, ssa2, g2, g2b);
    else
        add_2str_kernel<T, false><<<dim3(unsigned(ceil_div(long(ncl), 256)), b->ngpt), 256, 0, as_stream(stream)>>>(
            ncl, tau1, ssa1, g1, tau2, ssa2, g2, g2b);
    RB_LAUNCH("add_2str_kernel");
    return RRTMGP_B200_OK;
}

}  // namespace
}  // namespace rrtmgp_b200

using namespace rrtmgp_b200;

extern "C" {

int rrtmgp_b200_cloud_optics_1scl_f32(rrtmgp_b200_cloud c, int ncol, int nlay, const float* clwp,
        const float* ciwp, const float* reliq, const float* reice, float* tau, void* s)
{ return cloud_optics<float>(c, ncol, nlay, clwp, ciwp, reliq, reice, tau, nullptr, nullptr, false, s); }
int rrtmgp_b200_cloud_optics_1scl_f64(rrtmgp_b200_cloud c, int ncol, int nlay, const double* clwp,
        const double* ciwp, const double* reliq, const double* reice, double* tau, void* s)
{ return cloud_optics<double>(c, ncol, nlay, clwp, ciwp, reliq, reice, tau, nullptr, nullptr, false, s); }
int rrtmgp_b200_cloud_optics_2str_f32(rrtmgp_b200_cloud c, int ncol, int nlay, const float* clwp,
        const float* ciwp, const float* reliq, const float* reice, float* tau, float* ssa, float* g, void* s)
{ return cloud_optics<float>(c, ncol, nlay, clwp, ciwp, reliq, reice, tau, ssa, g, true, s); }
int rrtmgp_b200_cloud_optics_2str_f64(rrtmgp_b200_cloud c, int ncol, int nlay, const double* clwp,
        const double* ciwp, const double* reliq, const double* reice, double* tau, double* ssa, double* g, void* s)
{ return cloud_optics<double>(c, ncol, nlay, clwp, ciwp, reliq, reice, tau, ssa, g, true, s); }

int rrtmgp_b200_delta_scale_2str_f32(int ncol, int nlay, int ngpt, float* tau, float* ssa, float* g, void* s)
{ return delta_scale<float>(ncol, nlay, ngpt, tau, ssa, g, s); }
int rrtmgp_b200_delta_scale_2str_f64(int ncol, int nlay, int ngpt, double* tau, double* ssa, double* g, void* s)
{ return delta_scale<double>(ncol, nlay, ngpt, tau, ssa, g, s); }

int rrtmgp_b200_add_to_1scl_f32(rrtmgp_b200_bands b, int ncol, int nlay, float* t1, const float* t2, int n, void* s)
{ return add_to_1scl<float>(b, ncol, nlay, t1, t2, n, s); }
int rrtmgp_b200_add_to_1scl_f64(rrtmgp_b200_bands b, int ncol, int nlay, double* t1, const double* t2, int n, void* s)
{ return add_to_1scl<double>(b, ncol, nlay, t1, t2, n, s); }
int rrtmgp_b200_add_to_2str_f32(rrtmgp_b200_bands b, int ncol, int nlay, float* t1, float* s1, float* g1,
        const float* t2, const float* s2, const float* g2, int n, void* s)
{ return add_to_2str<float>(b, ncol, nlay, t1, s1, g1, t2, s2, g2, n, s); }
int rrtmgp_b200_add_to_2str_f64(rrtmgp_b200_bands b, int ncol, int nlay, double* t1, double* s1, double* g1,
        const double* t2, const double* s2, const double* g2, int n, void* s)
{ return add_to_2str<double>(b, ncol, nlay, t1, s1, g1, t2, s2, g2, n, s); }

}  // extern "C"
