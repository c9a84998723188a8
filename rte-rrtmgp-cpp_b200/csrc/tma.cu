// Host side of the TMA tile loads (tma.cuh): tensor maps encoded with the driver's
// cuTensorMapEncodeTiled, found once through the runtime's driver entry-point query (the
// library links only the CUDA runtime).
#include <cudaTypedefs.h>

#include <mutex>

#include "tma.cuh"

namespace rrtmgp_b200 {
namespace {

PFN_cuTensorMapEncodeTiled_v12000 encoder()
{
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();   // leave no sticky query error behind
    });
    return fn;
}

}  // namespace

int encode_map_3d_f32(CUtensorMap* map, const float* base, unsigned long long n0, unsigned long long n1,
                      unsigned long long n2, unsigned b0, unsigned b1)
{
    const auto fn = encoder();
    if (!fn) return fail(RRTMGP_B200_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[3] = {n0, n1, n2};
    const cuuint64_t strides[2] = {n0 * sizeof(float), n0 * n1 * sizeof(float)};   // bytes, dims 1 and 2
    const cuuint32_t box[3] = {b0, b1, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(RRTMGP_B200_ERR_CUDA, "cuTensorMapEncodeTiled rejected a map (error " + std::to_string(int(r)) + ")");
    return RRTMGP_B200_OK;
}

}  // namespace rrtmgp_b200
