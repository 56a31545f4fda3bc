// Registry of the compiled SIMT GEMM instantiations (one per tuning point).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace gatlas {
namespace simt {

struct LaunchArgs {
    const void *A;
    const void *B;
    void *C;
    int64_t M, N, K, lda, ldb, ldc, stride_a, stride_b, stride_c, batch;
    double alpha, beta;
    int gemm;
    cudaStream_t stream;
};

using LaunchFn = int (*)(const LaunchArgs &);

struct Entry {
    int scalar;  // 0 float, 1 double
    int ta, tb, gh, gw, bh, bw, vl;
    LaunchFn launch;
};

// Tables defined in gemm_simt_f32_nn_{a,b}.cu, gemm_simt_f32_tx.cu, gemm_simt_f64.cu.
const Entry *table_f32_nn_a(size_t *n);
const Entry *table_f32_nn_b(size_t *n);
const Entry *table_f32_tx(size_t *n);
const Entry *table_f64(size_t *n);

// Finds an entry for the exact point, or nullptr.
const Entry *find(int scalar, int ta, int tb, int gh, int gw, int bh, int bw, int vl);

}  // namespace simt
}  // namespace gatlas
