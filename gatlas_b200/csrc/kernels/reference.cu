// Device reference computations for the plugin layer's paranoid check.
//
// The reference's paranoid check recomputes the result on the host in the
// kernel's own precision, accumulating k = 0..K-1 in order
// (KernelMatmulBuffer.hpp:108-147, KernelMatvecBuffer.hpp:106-142,
// KernelSaxpyBuffer.hpp:106-121), and passes iff absdiff < 1/length
// (OCLAppUtil.hpp:212-264).  These kernels recompute the same quantity on the
// device, one thread per output element, with the fused mad chain of the
// generated kernels, so that the check stays affordable at full size.
#include "../common.cuh"
#include "reference.hpp"

namespace gatlas {

template <typename T>
__device__ __forceinline__ T fma_rn_t(T a, T b, T c);
template <>
__device__ __forceinline__ float fma_rn_t<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <>
__device__ __forceinline__ double fma_rn_t<double>(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename T>
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
        acc = fma_rn_t<T>(a, b, acc);
    }
    const int64_t o = p * M * N + i * N + j;
    if (gemm) {
        const T bc = (beta == T(0)) ? T(0) : beta * Cin[o];
        C[o] = fma_rn_t<T>(alpha, acc, bc);
    } else {
        C[o] = acc;
    }
}

template <typename T>
__global__ void ref_matvec_kernel(const T *A, const T *b, const T *cin, T *c, int64_t M, int64_t N, int ta,
                                  int gemv, T alpha, T beta) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t p = blockIdx.y;
    if (i >= M) return;
    const T *Ap = A + p * M * N;
    T acc = T(0);
    for (int64_t j = 0; j < N; ++j) acc = fma_rn_t<T>(ta ? Ap[j * M + i] : Ap[i * N + j], b[p * N + j], acc);
    const int64_t o = p * M + i;
    if (gemv) {
        const T bc = (beta == T(0)) ? T(0) : beta * cin[o];
        c[o] = fma_rn_t<T>(alpha, acc, bc);
    } else {
        c[o] = acc;
    }
}

template <typename T>
__global__ void ref_saxpy_kernel(const T *x, const T *y, T *z, int64_t n, T alpha) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) z[i] = fma_rn_t<T>(alpha, x[i], y[i]);
}

template <typename T>
int ref_matmul(const T *A, const T *B, const T *Cin, T *C, size_t packed, size_t M, size_t N, size_t K, bool ta,
               bool tb, bool gemm, T alpha, T beta, cudaStream_t s) {
    if (M == 0 || N == 0) return GATLAS_OK;
    if (M > 65535 || packed > 65535) return set_error(GATLAS_ERR_INVALID, "reference matmul: M or packed > 65535");
    dim3 grid((unsigned)((N + 127) / 128), (unsigned)M, (unsigned)packed);
    ref_matmul_kernel<T><<<grid, 128, 0, s>>>(A, B, Cin, C, M, N, K, ta, tb, gemm, alpha, beta);
    return check_launch("ref_matmul_kernel");
}

template <typename T>
int ref_matvec(const T *A, const T *b, const T *cin, T *c, size_t packed, size_t M, size_t N, bool ta, bool gemv,
               T alpha, T beta, cudaStream_t s) {
    if (M == 0) return GATLAS_OK;
    if (packed > 65535) return set_error(GATLAS_ERR_INVALID, "reference matvec: packed > 65535");
    dim3 grid((unsigned)((M + 127) / 128), (unsigned)packed);
    ref_matvec_kernel<T><<<grid, 128, 0, s>>>(A, b, cin, c, M, N, ta, gemv, alpha, beta);
    return check_launch("ref_matvec_kernel");
}

template <typename T>
int ref_saxpy(const T *x, const T *y, T *z, size_t n, T alpha, cudaStream_t s) {
    if (n == 0) return GATLAS_OK;
    ref_saxpy_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x, y, z, n, alpha);
    return check_launch("ref_saxpy_kernel");
}

template int ref_matmul<float>(const float *, const float *, const float *, float *, size_t, size_t, size_t, size_t,
                               bool, bool, bool, float, float, cudaStream_t);
template int ref_matmul<double>(const double *, const double *, const double *, double *, size_t, size_t, size_t,
                                size_t, bool, bool, bool, double, double, cudaStream_t);
template int ref_matvec<float>(const float *, const float *, const float *, float *, size_t, size_t, size_t, bool,
                               bool, float, float, cudaStream_t);
template int ref_matvec<double>(const double *, const double *, const double *, double *, size_t, size_t, size_t,
                                bool, bool, double, double, cudaStream_t);
template int ref_saxpy<float>(const float *, const float *, float *, size_t, float, cudaStream_t);
template int ref_saxpy<double>(const double *, const double *, double *, size_t, double, cudaStream_t);

}  // namespace gatlas
