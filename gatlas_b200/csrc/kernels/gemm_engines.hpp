// Matmul engine interfaces shared by the dispatcher (gemm.cu) and the
// image (TMA) and tensor-core engines.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../../include/gatlas.h"

namespace gatlas {

// Dense-default-resolved matmul geometry (element strides).
struct Geometry {
    int64_t M, N, K;
    bool ta, tb;
    int64_t lda, ldb, ldc;
    int64_t batch, stride_a, stride_b, stride_c;
};

bool resolve_geometry(const gatlas_matmul_desc *d, Geometry *g);

// FP64 residual of C against alpha*op(A)*op(B) (+ beta*Cin when gemm and Cin):
// out = {||C-Cref||_F, ||Cref||_F, max|C-Cref|, sum|C-Cref|}; batch 1 geometry.
int matmul_residual(const Geometry &g, double alpha, double beta, int gemm, const float *A, const float *B,
                    const float *Cin, const float *C, double *out_host, cudaStream_t stream);

// image engine: SIMT math on TMA tensor-map tile loads (gemm_image.cu)
int matmul_image_f32(const gatlas_matmul_desc *d, const Geometry &g, const float *A, const float *B,
                     float *C, cudaStream_t stream);
int matmul_image_f64(const gatlas_matmul_desc *d, const Geometry &g, const double *A, const double *B,
                     double *C, cudaStream_t stream);
int image_supported(int scalar, const gatlas_matmul_desc *d);

template <typename T>
inline int matmul_image(const gatlas_matmul_desc *d, const Geometry &g, const T *A, const T *B, T *C,
                        cudaStream_t stream);
template <>
inline int matmul_image<float>(const gatlas_matmul_desc *d, const Geometry &g, const float *A,
                               const float *B, float *C, cudaStream_t stream) {
    return matmul_image_f32(d, g, A, B, C, stream);
}
template <>
inline int matmul_image<double>(const gatlas_matmul_desc *d, const Geometry &g, const double *A,
                                const double *B, double *C, cudaStream_t stream) {
    return matmul_image_f64(d, g, A, B, C, stream);
}

// tensor-core engines (gemm_tc.cu)
int matmul_tc(const gatlas_matmul_desc *d, const Geometry &g, const float *A, const float *B, float *C,
              void *ws, size_t ws_bytes, cudaStream_t stream);
int tc_supported(const gatlas_matmul_desc *d);
size_t tc_workspace_bytes(const gatlas_matmul_desc *d, const Geometry &g);
namespace tcg {
// host-buffer pipeline of the tensor-core engines (gemm_tc.cu)
bool host_pipeline_ok(const gatlas_matmul_desc *d, const Geometry &g);
size_t host_pipeline_bytes(const gatlas_matmul_desc *d, const Geometry &g);
int host_pipeline(const gatlas_matmul_desc *d, const Geometry &g, const float *hA, const float *hB, float *hC,
                  void *dev, cudaStream_t caller);
}  // namespace tcg

}  // namespace gatlas
