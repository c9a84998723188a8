// Tensor-memory-accelerator (TMA) tile loads into shared memory, completed on an mbarrier,
// with waits bounded in time.
//
// A tile is one box of a tensor map (cuTensorMapEncodeTiled, made on the host per call):
// cp.async.bulk.tensor copies it from global to shared memory and adds its bytes to the
// mbarrier's transaction count; the mbarrier phase completes when the one expected arrival
// (arrive.expect_tx by the issuing thread) and all bytes have landed.  Loads only, never with
// cluster multicast: every tile is read by the CTA that asked for it.
//
// Waits: one thread polls the mbarrier (try_wait.parity) for at most kWaitLimitNs of the
// global timer, so a copy that never completes ends the kernel with an error count instead of
// hanging the GPU; callers drain their other copies in flight (again bounded) before exiting.
#pragma once

#include <cuda.h>   // CUtensorMap, CUtensorMapDataType (types only; no driver call is linked)

#include <cstdint>

#include "common.cuh"

namespace rrtmgp_b200 {
namespace tma {

constexpr unsigned long long kWaitLimitNs = 2000000000ull;   // 2 s

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes initialised mbarriers visible to the async proxy (the TMA unit).
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses (after a barrier: the
// block's) before later async-proxy writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void prefetch_map(const CUtensorMap* map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Box of `map` at element coordinates (x, y, z) -> dst (16-byte aligned shared memory); x is a
// multiple of 4 elements (16 bytes) for 32-bit data.
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase with parity `parity` of bar; false if it has not completed after
// kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    do {
        if (mbar_try_wait(bar, parity)) return true;
    } while (global_ns() - t0 < kWaitLimitNs);
    return false;
}

}  // namespace tma

// Host: a rank-3 FP32 tensor map over a column-fastest (n0, n1, n2) array with box
// (b0, b1, 1).  Returns RRTMGP_B200_OK or an error status (the driver's encoder rejected the
// map, or it could not be found).
int encode_map_3d_f32(CUtensorMap* map, const float* base, unsigned long long n0, unsigned long long n1,
                      unsigned long long n2, unsigned b0, unsigned b1);

}  // namespace rrtmgp_b200
