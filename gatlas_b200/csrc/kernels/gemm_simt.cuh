// SIMT GEMM kernel template (FP32 / FP64), buffer engine.
//
// Reference: KernelMatmulBuffer<SCALAR,VL>::print (KernelMatmulBuffer.hpp:174-342).
// A (group_h x group_w) work group computes a (group_h*block_h) x
// (group_w*block_w) tile of C; per K step every work item copies part of the
// A and B tiles into padded __local memory (KernelMatmulBuffer.hpp:261-281),
// barriers, and runs block_h x VL x VL mad chains from local memory
// (:302-321); the store writes block_h rows of VL-vectors (:325-337).
//
// B200 design, same parameter point:
//  * thread block = group_h x group_w threads, CTA tile BM x BN with
//    BM = group_h*block_h, BN = group_w*block_w, K step BK = 8;
//  * global loads are VL-wide vectors on the operand's contiguous dimension,
//    staged in registers one K step ahead (software pipelining) and stored
//    to a double-buffered, k-major shared tile (transposed on store where the
//    operand is k-contiguous), padded by 4 elements so both the transposed
//    stores and the 16-byte fragment reads are bank-conflict free;
//  * each thread's block_h x block_w micro-tile is split into 4-wide groups
//    strided by 4*group_h rows / 4*group_w columns (conflict-free 16-byte
//    fragment reads);
//  * every output element is one fused multiply-add chain over k = 0..K-1,
//    the order of the reference's mad chain, so FP32 results are bit-exact
//    against a sequential fmaf chain;
//  * epilogue C = fma(alpha, acc, beta*C) (the reference's
//    mad(alpha, accum, beta*C)), C unread when beta == 0.
// Edges are predicated (zero-filled loads, guarded stores), so any M, N, K
// works; the reference's divisibility rules are enforced above this layer.
#pragma once

// This header is also compiled at run time by NVRTC (for parameter points
// without a prebuilt instantiation), where no system headers are available.
#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#else
typedef long long int64_t;
typedef unsigned long long uintptr_t;
#endif

namespace gatlas {
namespace simt {

template <typename T>
struct GemmArgs {
    const T *A;
    const T *B;
    T *C;
    int64_t M, N, K;
    int64_t lda, ldb, ldc;
    int64_t stride_a, stride_b, stride_c;
    T alpha, beta;
    int gemm;
};

template <typename T, int N>
struct alignas(sizeof(T) * N) VecN {
    T v[N];
};

__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// Two round-to-nearest fused multiply-adds in one packed instruction
// (fma.rn.f32x2, sm_100): d0 = a*b0 + d0 and d1 = a*b1 + d1, each exactly
// what __fmaf_rn gives.
__device__ __forceinline__ void fma2_rn(float &d0, float &d1, float a, float b0, float b1) {
    asm("{.reg .b64 pa, pb, pd;\n\t"
        "mov.b64 pa, {%2, %2};\n\t"
        "mov.b64 pb, {%3, %4};\n\t"
        "mov.b64 pd, {%0, %1};\n\t"
        "fma.rn.f32x2 pd, pa, pb, pd;\n\t"
        "mov.b64 {%0, %1}, pd;}"
        : "+f"(d0), "+f"(d1)
        : "f"(a), "f"(b0), "f"(b1));
}

// The micro-tile update acc[i][j] = fma(af[i], bf[j], acc[i][j]) of one k.
// FP32 pairs of neighbouring columns take one packed instruction: every
// element still gets one round-to-nearest fused multiply-add per k, in k
// order, so results are unchanged, while the FMA instructions the kernel
// issues halve (it is bound by instruction issue, not by the FP32 pipe).
template <typename T, int BH, int BW>
__device__ __forceinline__ void micro_update(T (&acc)[BH][BW], const T (&af)[BH], const T (&bf)[BW]) {
    if constexpr (sizeof(T) == 4 && BW % 2 == 0) {
#pragma unroll
        for (int i = 0; i < BH; ++i)
#pragma unroll
            for (int j = 0; j < BW; j += 2) fma2_rn(acc[i][j], acc[i][j + 1], af[i], bf[j], bf[j + 1]);
    } else {
#pragma unroll
        for (int i = 0; i < BH; ++i)
#pragma unroll
            for (int j = 0; j < BW; ++j) acc[i][j] = fma_rn(af[i], bf[j], acc[i][j]);
    }
}

// Index of micro-tile row i (of BH) for thread row ty.
template <int G, int BH>
__device__ __forceinline__ int micro_index(int t, int i) {
    if constexpr (BH % 4 == 0) {
        return (i / 4) * (G * 4) + t * 4 + (i % 4);
    } else {
        return t * BH + i;
    }
}

constexpr int kPad = 4;

template <typename T, bool TA, bool TB, int GH, int GW, int BH, int BW, int VL, int BK>
struct Tile {
    static constexpr int NT = GH * GW;
    static constexpr int BM = GH * BH;
    static constexpr int BN = GW * BW;
    static constexpr int LDA_S = BM + kPad;
    static constexpr int LDB_S = BN + kPad;
    static constexpr int A_VECS = BM * BK / VL;
    static constexpr int B_VECS = BN * BK / VL;
    static constexpr int LA = (A_VECS + NT - 1) / NT;
    static constexpr int LB = (B_VECS + NT - 1) / NT;
    static constexpr int SMEM_ELEMS = 2 * BK * (LDA_S + LDB_S);
    // vectors run along each operand's contiguous dimension
    static_assert(BK % VL == 0, "vector width must divide the K step");
    static_assert(!TA || BM % VL == 0, "vector width must divide the A tile rows");
    static_assert(TB || BN % VL == 0, "vector width must divide the B tile columns");
};

// FP32 points with micro-tiles of at most 64 elements are capped at 128
// registers so that 512 threads fit per SM; larger micro-tiles take up to 255
// registers at one CTA per SM, with the ILP of their accumulators instead.
template <typename T, int NT, int MICRO>
constexpr int min_blocks() {
    return (sizeof(T) == 4 && NT <= 512 && MICRO <= 64) ? 512 / NT : 1;
}

template <typename T, bool TA, bool TB, int GH, int GW, int BH, int BW, int VL, int BK>
__global__ void __launch_bounds__(GH *GW, min_blocks<T, GH * GW, BH * BW>())
    gemm_simt_kernel(GemmArgs<T> a) {
    using TT = Tile<T, TA, TB, GH, GW, BH, BW, VL, BK>;
    constexpr int NT = TT::NT, BM = TT::BM, BN = TT::BN;
    constexpr int LDA_S = TT::LDA_S, LDB_S = TT::LDB_S;
    using V = VecN<T, VL>;

    __shared__ __align__(16) T As[2][BK][LDA_S];
    __shared__ __align__(16) T Bs[2][BK][LDB_S];

    const int tid = threadIdx.x;
    const int tx = tid % GW, ty = tid / GW;
    const int64_t m0 = (int64_t)blockIdx.y * BM;
    const int64_t n0 = (int64_t)blockIdx.x * BN;
    const int64_t p = blockIdx.z;
    const T *A = a.A + p * a.stride_a;
    const T *B = a.B + p * a.stride_b;
    T *C = a.C + p * a.stride_c;

    V ra[TT::LA], rb[TT::LB];

    auto load_tile = [&](int64_t k0) {
#pragma unroll
        for (int it = 0; it < TT::LA; ++it) {
            const int v = tid + it * NT;
            V val;
#pragma unroll
            for (int e = 0; e < VL; ++e) val.v[e] = T(0);
            if (v < TT::A_VECS) {
                if constexpr (!TA) {  // A row-major M x K: vectors along k
                    const int kv = v % (BK / VL), m = v / (BK / VL);
                    const int64_t gr = m0 + m, gc = k0 + kv * VL;
                    if (gr < a.M && gc < a.K) val = *reinterpret_cast<const V *>(A + gr * a.lda + gc);
                } else {  // A stored K x M: vectors along m
                    const int mv = v % (BM / VL), k = v / (BM / VL);
                    const int64_t gr = k0 + k, gc = m0 + mv * VL;
                    if (gr < a.K && gc < a.M) val = *reinterpret_cast<const V *>(A + gr * a.lda + gc);
                }
            }
            ra[it] = val;
        }
#pragma unroll
        for (int it = 0; it < TT::LB; ++it) {
            const int v = tid + it * NT;
            V val;
#pragma unroll
            for (int e = 0; e < VL; ++e) val.v[e] = T(0);
            if (v < TT::B_VECS) {
                if constexpr (!TB) {  // B row-major K x N: vectors along n
                    const int nv = v % (BN / VL), k = v / (BN / VL);
                    const int64_t gr = k0 + k, gc = n0 + nv * VL;
                    if (gr < a.K && gc < a.N) val = *reinterpret_cast<const V *>(B + gr * a.ldb + gc);
                } else {  // B stored N x K: vectors along k
                    const int kv = v % (BK / VL), n = v / (BK / VL);
                    const int64_t gr = n0 + n, gc = k0 + kv * VL;
                    if (gr < a.N && gc < a.K) val = *reinterpret_cast<const V *>(B + gr * a.ldb + gc);
                }
            }
            rb[it] = val;
        }
    };

    auto store_tile = [&](int buf) {
#pragma unroll
        for (int it = 0; it < TT::LA; ++it) {
            const int v = tid + it * NT;
            if (v < TT::A_VECS) {
                if constexpr (!TA) {
                    const int kv = v % (BK / VL), m = v / (BK / VL);
#pragma unroll
                    for (int e = 0; e < VL; ++e) As[buf][kv * VL + e][m] = ra[it].v[e];
                } else {
                    const int mv = v % (BM / VL), k = v / (BM / VL);
                    *reinterpret_cast<V *>(&As[buf][k][mv * VL]) = ra[it];
                }
            }
        }
#pragma unroll
        for (int it = 0; it < TT::LB; ++it) {
            const int v = tid + it * NT;
            if (v < TT::B_VECS) {
                if constexpr (!TB) {
                    const int nv = v % (BN / VL), k = v / (BN / VL);
                    *reinterpret_cast<V *>(&Bs[buf][k][nv * VL]) = rb[it];
                } else {
                    const int kv = v % (BK / VL), n = v / (BK / VL);
#pragma unroll
                    for (int e = 0; e < VL; ++e) Bs[buf][kv * VL + e][n] = rb[it].v[e];
                }
            }
        }
    };


    // L2 prefetch of the operand vectors of a later K step: it holds no
    // registers, and the register-staged loads of that step then hit L2
    // instead of waiting on DRAM
    auto prefetch_tile = [&](int64_t k0) {
#pragma unroll
        for (int it = 0; it < TT::LA; ++it) {
            const int v = tid + it * NT;
            if (v < TT::A_VECS) {
                const T *ptr = nullptr;
                if constexpr (!TA) {
                    const int kv = v % (BK / VL), m = v / (BK / VL);
                    const int64_t gr = m0 + m, gc = k0 + kv * VL;
                    if (gr < a.M && gc < a.K) ptr = A + gr * a.lda + gc;
                } else {
                    const int mv = v % (BM / VL), k = v / (BM / VL);
                    const int64_t gr = k0 + k, gc = m0 + mv * VL;
                    if (gr < a.K && gc < a.M) ptr = A + gr * a.lda + gc;
                }
                if (ptr) asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
            }
        }
#pragma unroll
        for (int it = 0; it < TT::LB; ++it) {
            const int v = tid + it * NT;
            if (v < TT::B_VECS) {
                const T *ptr = nullptr;
                if constexpr (!TB) {
                    const int nv = v % (BN / VL), k = v / (BN / VL);
                    const int64_t gr = k0 + k, gc = n0 + nv * VL;
                    if (gr < a.K && gc < a.N) ptr = B + gr * a.ldb + gc;
                } else {
                    const int kv = v % (BK / VL), n = v / (BK / VL);
                    const int64_t gr = n0 + n, gc = k0 + kv * VL;
                    if (gr < a.N && gc < a.K) ptr = B + gr * a.ldb + gc;
                }
                if (ptr) asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
            }
        }
    };

    T acc[BH][BW];
#pragma unroll
    for (int i = 0; i < BH; ++i)
#pragma unroll
        for (int j = 0; j < BW; ++j) acc[i][j] = T(0);

    const int64_t KT = (a.K + BK - 1) / BK;
    if (KT > 0) {
        load_tile(0);
        store_tile(0);
    }
    __syncthreads();

    for (int64_t kt = 0; kt < KT; ++kt) {
        const int cur = (int)(kt & 1);
        // two K steps ahead, for FP32 points that run two CTAs per SM under
        // the 128-register cap (8192^3 default point 47.9 -> 50.6 TFLOP/s);
        // one-CTA points (8x16 x 16x8: 47.5 -> 44.7) and FP64 (21.1 -> 20.4
        // at 4096^3) ran slower with it and go without
        if constexpr (sizeof(T) == 4 && min_blocks<T, NT, BH * BW>() > 1)
            if (kt + 2 < KT) prefetch_tile((kt + 2) * BK);
        if (kt + 1 < KT) load_tile((kt + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T af[BH], bf[BW];
            if constexpr (BH % 4 == 0) {
#pragma unroll
                for (int g = 0; g < BH / 4; ++g) {
                    const VecN<T, 4> q = *reinterpret_cast<const VecN<T, 4> *>(&As[cur][kk][g * GH * 4 + ty * 4]);
#pragma unroll
                    for (int e = 0; e < 4; ++e) af[g * 4 + e] = q.v[e];
                }
            } else {
#pragma unroll
                for (int i = 0; i < BH; ++i) af[i] = As[cur][kk][ty * BH + i];
            }
            if constexpr (BW % 4 == 0) {
#pragma unroll
                for (int g = 0; g < BW / 4; ++g) {
                    const VecN<T, 4> q = *reinterpret_cast<const VecN<T, 4> *>(&Bs[cur][kk][g * GW * 4 + tx * 4]);
#pragma unroll
                    for (int e = 0; e < 4; ++e) bf[g * 4 + e] = q.v[e];
                }
            } else {
#pragma unroll
                for (int j = 0; j < BW; ++j) bf[j] = Bs[cur][kk][tx * BW + j];
            }
            micro_update<T, BH, BW>(acc, af, bf);
        }
        if (kt + 1 < KT) store_tile(cur ^ 1);
        __syncthreads();
    }

    // epilogue
    const bool vec_store = (BW % 4 == 0) && (sizeof(T) == 4) && (a.ldc % 4 == 0) &&
                           ((reinterpret_cast<uintptr_t>(C) & 15) == 0);
#pragma unroll
    for (int i = 0; i < BH; ++i) {
        const int64_t row = m0 + micro_index<GH, BH>(ty, i);
        if (row >= a.M) continue;
        T *crow = C + row * a.ldc;
        if constexpr (BW % 4 == 0) {
#pragma unroll
            for (int g = 0; g < BW / 4; ++g) {
                const int64_t col = n0 + g * GW * 4 + tx * 4;
                T out[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const T acc_v = acc[i][g * 4 + e];
                    if (a.gemm) {
                        const T bc = (a.beta == T(0) || col + e >= a.N) ? T(0) : a.beta * crow[col + e];
                        out[e] = fma_rn(a.alpha, acc_v, bc);
                    } else {
                        out[e] = acc_v;
                    }
                }
                if (vec_store && col + 3 < a.N) {
                    *reinterpret_cast<VecN<T, 4> *>(crow + col) = *reinterpret_cast<VecN<T, 4> *>(out);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        if (col + e < a.N) crow[col + e] = out[e];
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < BW; ++j) {
                const int64_t col = n0 + tx * BW + j;
                if (col >= a.N) continue;
                const T acc_v = acc[i][j];
                if (a.gemm) {
                    const T bc = (a.beta == T(0)) ? T(0) : a.beta * crow[col];
                    crow[col] = fma_rn(a.alpha, acc_v, bc);
                } else {
                    crow[col] = acc_v;
                }
            }
        }
    }
}

}  // namespace simt
}  // namespace gatlas
