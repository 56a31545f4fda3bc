// Instantiation helper for SIMT GEMM tuning points.
#pragma once

#include "../common.cuh"
#include "gemm_simt.cuh"
#include "gemm_simt_registry.hpp"

namespace gatlas {
namespace simt {

constexpr int kBK = 8;

template <typename T, bool TA, bool TB, int GH, int GW, int BH, int BW, int VL>
int launch_point(const LaunchArgs &l) {
    using TT = Tile<T, TA, TB, GH, GW, BH, BW, VL, kBK>;
    GemmArgs<T> a;
    a.A = static_cast<const T *>(l.A);
    a.B = static_cast<const T *>(l.B);
    a.C = static_cast<T *>(l.C);
    a.M = l.M;
    a.N = l.N;
    a.K = l.K;
    a.lda = l.lda;
    a.ldb = l.ldb;
    a.ldc = l.ldc;
    a.stride_a = l.stride_a;
    a.stride_b = l.stride_b;
    a.stride_c = l.stride_c;
    a.alpha = (T)l.alpha;
    a.beta = (T)l.beta;
    a.gemm = l.gemm;
    const int64_t gx = (l.N + TT::BN - 1) / TT::BN;
    const int64_t gy = (l.M + TT::BM - 1) / TT::BM;
    if (gx > 0x7fffffff || gy > 65535 || l.batch > 65535)
        return set_error(GATLAS_ERR_INVALID, "matmul: grid (%lld, %lld, %lld) too large", (long long)gx,
                         (long long)gy, (long long)l.batch);
    dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)l.batch);
    gemm_simt_kernel<T, TA, TB, GH, GW, BH, BW, VL, kBK><<<grid, TT::NT, 0, l.stream>>>(a);
    return check_launch("gemm_simt_kernel");
}

}  // namespace simt
}  // namespace gatlas

#define GATLAS_SIMT_ENTRY(T, SC, TA, TB, GH, GW, BH, BW, VL)                                      \
    {SC, TA, TB, GH, GW, BH, BW, VL,                                                              \
     &gatlas::simt::launch_point<T, (TA) != 0, (TB) != 0, GH, GW, BH, BW, VL>}
