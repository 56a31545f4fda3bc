// Image engine for matmul: SIMT math fed by TMA tensor-map tile loads.
#include "../common.cuh"
#include "gemm_engines.hpp"

namespace gatlas {

int matmul_image_f32(const gatlas_matmul_desc *, const Geometry &, const float *, const float *, float *,
                     cudaStream_t) {
    return set_error(GATLAS_ERR_UNSUPPORTED, "matmul: image engine not built yet");
}

int matmul_image_f64(const gatlas_matmul_desc *, const Geometry &, const double *, const double *, double *,
                     cudaStream_t) {
    return set_error(GATLAS_ERR_UNSUPPORTED, "matmul: image engine not built yet");
}

int image_supported(int, const gatlas_matmul_desc *) { return 0; }

}  // namespace gatlas
