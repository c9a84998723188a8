// FP32 FMA throughput probe: the denominator of the FP32-pipe roofline of the fused
// column-forward kernels.  Every thread runs 8 independent FMA chains, so the FMA pipe, not
// latency, is the limit; the result is written so that the chains are not eliminated.
#include "common.cuh"

namespace rrtmgp_b200 {
namespace {

__global__ void __launch_bounds__(512) fma_probe_kernel(int iters, float* __restrict__ out)
{
    float a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = float(threadIdx.x + i) * 1.0e-3f;
    const float m = 0.999999f, c = 1.0e-7f;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = fmaf(a[i], m, c);
        }
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += a[i];
    if (s == 12345.678f) out[blockIdx.x] = s;   // practically never true; keeps the chains live
}

}  // namespace
}  // namespace rrtmgp_b200

// No reference counterpart: measurement helper.  Launches blocks x 512 threads, each doing
// iters x 128 FMAs (2 FLOP each); FLOP = blocks * 512 * iters * 256.
extern "C" int rrtmgp_b200_fp32_fma_probe(int blocks, int iters, float* out, void* stream)
{
    RB_CHECK_ARG(blocks > 0 && iters > 0 && out, "fp32_fma_probe: blocks, iters > 0 and out required");
    rrtmgp_b200::fma_probe_kernel<<<blocks, 512, 0, rrtmgp_b200::as_stream(stream)>>>(iters, out);
    RB_LAUNCH("fma_probe_kernel");
    return RRTMGP_B200_OK;
}
