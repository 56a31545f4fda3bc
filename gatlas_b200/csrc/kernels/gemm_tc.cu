// Tensor-core (tcgen05) matmul engines.
#include "../common.cuh"
#include "gemm_engines.hpp"

namespace gatlas {

int matmul_tc(const gatlas_matmul_desc *, const Geometry &, const float *, const float *, float *, void *,
              size_t, cudaStream_t) {
    return set_error(GATLAS_ERR_UNSUPPORTED, "matmul: tensor-core engines not built yet");
}

int tc_supported(const gatlas_matmul_desc *) { return 0; }

size_t tc_workspace_bytes(const gatlas_matmul_desc *, const Geometry &) { return 0; }

}  // namespace gatlas
