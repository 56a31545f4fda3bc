// Device reference computations for the plugin layer's paranoid check.
//
// The reference's paranoid check recomputes the result on the host in the
// kernel's own precision, accumulating k = 0..K-1 in order
// (KernelMatmulBuffer.hpp:108-147, KernelMatvecBuffer.hpp:106-142,
// KernelSaxpyBuffer.hpp:106-121), and passes iff absdiff < 1/length
// (OCLAppUtil.hpp:212-264).  These kernels recompute the same quantity on the
// device, one thread per output element, so that the check stays affordable
// at full size, in one of two arithmetics:
//  - unfused: every product and every sum rounded separately, as the
//    reference's host loops compile (g++ -O2 on x86-64, no FMA): acc += a*b,
//    then alpha*acc + beta*c (KernelMatmulBuffer.hpp:124-143,
//    KernelMatvecBuffer.hpp:122-138, KernelSaxpyBuffer.hpp:118-120);
//  - fused: the mad chain of the generated kernels, acc = fma(a, b, acc),
//    then fma(alpha, acc, beta*c) (KernelMatmulBuffer.hpp:302-337), which is
//    the arithmetic the SIMT engines here reproduce bit for bit.
// The __f*_rn / __d*_rn intrinsics keep the compiler from contracting the
// unfused form into FMAs.
#include "gatlas.h"

#include "../common.cuh"
#include "reference.hpp"

namespace gatlas {

template <typename T>
struct Arith;
template <>
struct Arith<float> {
    static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
};
template <>
struct Arith<double> {
    static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
};

// acc <- a*b + acc in the chosen arithmetic
template <typename T, bool Fused>
__device__ __forceinline__ T step(T a, T b, T acc) {
    return Fused ? Arith<T>::fma(a, b, acc) : Arith<T>::add(acc, Arith<T>::mul(a, b));
}

// alpha*acc + beta*c; c is not read when beta == 0 on the fused form (the
// generated kernels' convention); the unfused form reads it as the
// reference's host loop does
template <typename T, bool Fused>
__device__ __forceinline__ T epilogue(T alpha, T acc, T beta, const T *cin, int64_t o) {
    if (Fused) return Arith<T>::fma(alpha, acc, beta == T(0) ? T(0) : Arith<T>::mul(beta, cin[o]));
    return Arith<T>::add(Arith<T>::mul(alpha, acc), Arith<T>::mul(beta, cin[o]));
}

template <typename T, bool Fused>
__global__ void ref_matmul_kernel(const T *A, const T *B, const T *Cin, T *C, int64_t M, int64_t N, int64_t K,
                                  int ta, int tb, int gemm, T alpha, T beta) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t i = blockIdx.y;
    const int64_t p = blockIdx.z;
    if (j >= N) return;
    const T *Ap = A + p * M * K;
    const T *Bp = B + p * K * N;
    T acc = T(0);
    for (int64_t k = 0; k < K; ++k) {
        const T a = ta ? Ap[k * M + i] : Ap[i * K + k];
        const T b = tb ? Bp[j * K + k] : Bp[k * N + j];
        acc = step<T, Fused>(a, b, acc);
    }
    const int64_t o = p * M * N + i * N + j;
    C[o] = gemm ? epilogue<T, Fused>(alpha, acc, beta, Cin, o) : acc;
}

template <typename T, bool Fused>
__global__ void ref_matvec_kernel(const T *A, const T *b, const T *cin, T *c, int64_t M, int64_t N, int ta,
                                  int gemv, T alpha, T beta) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t p = blockIdx.y;
    if (i >= M) return;
    const T *Ap = A + p * M * N;
    T acc = T(0);
    for (int64_t j = 0; j < N; ++j) acc = step<T, Fused>(ta ? Ap[j * M + i] : Ap[i * N + j], b[p * N + j], acc);
    const int64_t o = p * M + i;
    c[o] = gemv ? epilogue<T, Fused>(alpha, acc, beta, cin, o) : acc;
}

template <typename T, bool Fused>
__global__ void ref_saxpy_kernel(const T *x, const T *y, T *z, int64_t n, T alpha) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) z[i] = Fused ? Arith<T>::fma(alpha, x[i], y[i]) : Arith<T>::add(Arith<T>::mul(alpha, x[i]), y[i]);
}

template <typename T>
int ref_matmul(const T *A, const T *B, const T *Cin, T *C, size_t packed, size_t M, size_t N, size_t K, bool ta,
               bool tb, bool gemm, T alpha, T beta, cudaStream_t s, bool fused) {
    if (M == 0 || N == 0) return GATLAS_OK;
    if (M > 65535 || packed > 65535) return set_error(GATLAS_ERR_INVALID, "reference matmul: M or packed > 65535");
    dim3 grid((unsigned)((N + 127) / 128), (unsigned)M, (unsigned)packed);
    if (fused) ref_matmul_kernel<T, true><<<grid, 128, 0, s>>>(A, B, Cin, C, M, N, K, ta, tb, gemm, alpha, beta);
    else ref_matmul_kernel<T, false><<<grid, 128, 0, s>>>(A, B, Cin, C, M, N, K, ta, tb, gemm, alpha, beta);
    return check_launch("ref_matmul_kernel");
}

template <typename T>
int ref_matvec(const T *A, const T *b, const T *cin, T *c, size_t packed, size_t M, size_t N, bool ta, bool gemv,
               T alpha, T beta, cudaStream_t s, bool fused) {
    if (M == 0) return GATLAS_OK;
    if (packed > 65535) return set_error(GATLAS_ERR_INVALID, "reference matvec: packed > 65535");
    dim3 grid((unsigned)((M + 127) / 128), (unsigned)packed);
    if (fused) ref_matvec_kernel<T, true><<<grid, 128, 0, s>>>(A, b, cin, c, M, N, ta, gemv, alpha, beta);
    else ref_matvec_kernel<T, false><<<grid, 128, 0, s>>>(A, b, cin, c, M, N, ta, gemv, alpha, beta);
    return check_launch("ref_matvec_kernel");
}

template <typename T>
int ref_saxpy(const T *x, const T *y, T *z, size_t n, T alpha, cudaStream_t s, bool fused) {
    if (n == 0) return GATLAS_OK;
    const unsigned grid = (unsigned)((n + 255) / 256);
    if (fused) ref_saxpy_kernel<T, true><<<grid, 256, 0, s>>>(x, y, z, n, alpha);
    else ref_saxpy_kernel<T, false><<<grid, 256, 0, s>>>(x, y, z, n, alpha);
    return check_launch("ref_saxpy_kernel");
}

template int ref_matmul<float>(const float *, const float *, const float *, float *, size_t, size_t, size_t, size_t,
                               bool, bool, bool, float, float, cudaStream_t, bool);
template int ref_matmul<double>(const double *, const double *, const double *, double *, size_t, size_t, size_t,
                                size_t, bool, bool, bool, double, double, cudaStream_t, bool);
template int ref_matvec<float>(const float *, const float *, const float *, float *, size_t, size_t, size_t, bool,
                               bool, float, float, cudaStream_t, bool);
template int ref_matvec<double>(const double *, const double *, const double *, double *, size_t, size_t, size_t,
                                bool, bool, double, double, cudaStream_t, bool);
template int ref_saxpy<float>(const float *, const float *, float *, size_t, float, cudaStream_t, bool);
template int ref_saxpy<double>(const double *, const double *, double *, size_t, double, cudaStream_t, bool);

}  // namespace gatlas

// ---------------------------------------------------------------------------
// C ABI: the paranoid check's device reference, callable on its own
// ---------------------------------------------------------------------------
namespace {

bool dense_matmul(const gatlas_matmul_desc *d) {
    const uint64_t lda = d->trans_a ? d->m : d->k, ldb = d->trans_b ? d->k : d->n;
    return (!d->lda || d->lda == lda) && (!d->ldb || d->ldb == ldb) && (!d->ldc || d->ldc == d->n) &&
           (!d->stride_a || d->stride_a == d->m * d->k) && (!d->stride_b || d->stride_b == d->k * d->n) &&
           (!d->stride_c || d->stride_c == d->m * d->n);
}

bool dense_matvec(const gatlas_matvec_desc *d) {
    const uint64_t lda = d->trans_a ? d->m : d->n;
    return (!d->lda || d->lda == lda) && (!d->stride_a || d->stride_a == d->m * d->n) &&
           (!d->stride_x || d->stride_x == d->n) && (!d->stride_y || d->stride_y == d->m);
}

}  // namespace

extern "C" int gatlas_reference_matmul(int scalar, int fused, const gatlas_matmul_desc *d, const void *A,
                                       const void *B, const void *Cin, void *C, void *stream) {
    using namespace gatlas;
    if (!d || (scalar != 0 && scalar != 1)) return set_error(GATLAS_ERR_INVALID, "reference matmul: bad arguments");
    if (!dense_matmul(d)) return set_error(GATLAS_ERR_INVALID, "reference matmul: dense packed layouts only");
    const size_t P = d->batch ? d->batch : 1;
    if (d->m == 0 || d->n == 0) return GATLAS_OK;
    const bool reads_c = d->gemm && (!fused || d->beta != 0.0);
    if (!C || (d->k && (!A || !B)) || (reads_c && !Cin)) return set_error(GATLAS_ERR_INVALID, "reference matmul: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    if (scalar == 0)
        return ref_matmul<float>((const float *)A, (const float *)B, (const float *)Cin, (float *)C, P, d->m, d->n, d->k,
                                 d->trans_a, d->trans_b, d->gemm, (float)d->alpha, (float)d->beta, s, fused != 0);
    return ref_matmul<double>((const double *)A, (const double *)B, (const double *)Cin, (double *)C, P, d->m, d->n,
                              d->k, d->trans_a, d->trans_b, d->gemm, d->alpha, d->beta, s, fused != 0);
}

extern "C" int gatlas_reference_matvec(int scalar, int fused, const gatlas_matvec_desc *d, const void *A,
                                       const void *x, const void *yin, void *y, void *stream) {
    using namespace gatlas;
    if (!d || (scalar != 0 && scalar != 1)) return set_error(GATLAS_ERR_INVALID, "reference matvec: bad arguments");
    if (!dense_matvec(d)) return set_error(GATLAS_ERR_INVALID, "reference matvec: dense packed layouts only");
    const size_t P = d->batch ? d->batch : 1;
    if (d->m == 0) return GATLAS_OK;
    const bool reads_y = d->gemv && (!fused || d->beta != 0.0);
    if (!y || (d->n && (!A || !x)) || (reads_y && !yin)) return set_error(GATLAS_ERR_INVALID, "reference matvec: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    if (scalar == 0)
        return ref_matvec<float>((const float *)A, (const float *)x, (const float *)yin, (float *)y, P, d->m, d->n,
                                 d->trans_a, d->gemv, (float)d->alpha, (float)d->beta, s, fused != 0);
    return ref_matvec<double>((const double *)A, (const double *)x, (const double *)yin, (double *)y, P, d->m, d->n,
                              d->trans_a, d->gemv, d->alpha, d->beta, s, fused != 0);
}

extern "C" int gatlas_reference_saxpy(int scalar, int fused, size_t n, double alpha, const void *x, const void *y,
                                      void *z, void *stream) {
    using namespace gatlas;
    if (scalar != 0 && scalar != 1) return set_error(GATLAS_ERR_INVALID, "reference saxpy: bad scalar type");
    if (n == 0) return GATLAS_OK;
    if (!x || !y || !z) return set_error(GATLAS_ERR_INVALID, "reference saxpy: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    if (scalar == 0)
        return ref_saxpy<float>((const float *)x, (const float *)y, (float *)z, n, (float)alpha, s, fused != 0);
    return ref_saxpy<double>((const double *)x, (const double *)y, (double *)z, n, alpha, s, fused != 0);
}
