// TMA tensor-map encoding via cudaGetDriverEntryPoint.
#include "tma.hpp"

#include <mutex>

#include "status.hpp"

namespace gatlas {

namespace {
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
std::once_flag g_once;
EncodeTiledFn g_encode = nullptr;

void resolve() {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_encode = reinterpret_cast<EncodeTiledFn>(fn);
}
}  // namespace

int make_tensor_map(CUtensorMap *map, CUtensorMapDataType dtype, int rank, void *base,
                    const uint64_t *dims, const uint64_t *strides_bytes, const uint32_t *box,
                    CUtensorMapSwizzle swizzle) {
    std::call_once(g_once, resolve);
    if (!g_encode) return set_error(GATLAS_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0)
        return set_error(GATLAS_ERR_INVALID, "tensor map base not 16-byte aligned");
    for (int i = 0; i + 1 < rank; ++i)
        if (strides_bytes[i] % 16 != 0)
            return set_error(GATLAS_ERR_INVALID, "tensor map stride %d not a multiple of 16 bytes", i);
    cuuint64_t d[5];
    cuuint64_t s[4];
    cuuint32_t b[5], e[5];
    for (int i = 0; i < rank; ++i) {
        d[i] = dims[i];
        b[i] = box[i];
        e[i] = 1;
    }
    for (int i = 0; i + 1 < rank; ++i) s[i] = strides_bytes[i];
    CUresult r = g_encode(map, dtype, (cuuint32_t)rank, base, d, s, b, e, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(GATLAS_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return GATLAS_OK;
}

}  // namespace gatlas
