// Device reference computations used by the plugin layer's paranoid check.
// fused: the generated kernels' mad chain (fma); otherwise every product and
// sum rounded separately, as the reference's host check loops are.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace gatlas {

template <typename T>
int ref_matmul(const T *A, const T *B, const T *Cin, T *C, size_t packed, size_t M, size_t N, size_t K, bool ta,
               bool tb, bool gemm, T alpha, T beta, cudaStream_t s, bool fused = true);
template <typename T>
int ref_matvec(const T *A, const T *b, const T *cin, T *c, size_t packed, size_t M, size_t N, bool ta, bool gemv,
               T alpha, T beta, cudaStream_t s, bool fused = true);
template <typename T>
int ref_saxpy(const T *x, const T *y, T *z, size_t n, T alpha, cudaStream_t s, bool fused = true);

}  // namespace gatlas
