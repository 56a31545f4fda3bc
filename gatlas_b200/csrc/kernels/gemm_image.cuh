// SIMT GEMM fed by TMA tensor-map tiles (the "image" engine), FP32 / FP64.
//
// Reference: KernelMatmulImage<SCALAR,VL>::print (KernelMatmulImage.hpp:192-313)
// samples A and B from RGBA images (read_imagef, nearest, unnormalised) and
// runs the same blockHeight x VL x VL mad chains as the buffer kernel.
//
// B200 design, same parameter point (work group GH x GW, micro-tile BH x BW):
//  * A and B are described by 3-D tensor maps (inner dimension, rows, packed
//    instance); one thread issues cp.async.bulk.tensor loads of BK-deep
//    tiles into an S-stage mbarrier ring;
//  * a tile whose stored layout is k-major (A stored K x M, B stored K x N)
//    is used where it lands; an m-major tile (A stored M x K, B stored N x K)
//    arrives 128-byte swizzled and is transposed once into a padded k-major
//    buffer (conflict-free on both sides);
//  * the math is the buffer kernel's: every element is one fused
//    multiply-add chain over k = 0..K-1, bit-exact against a sequential fmaf
//    chain; epilogue C = fma(alpha, acc, beta*C).
// Waits are bounded in wall time; a timeout sets the fault word and stops.
// This header is also compiled at run time by NVRTC for points without a
// prebuilt instantiation, so it is self-contained.
#pragma once

#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#else
typedef long long int64_t;
typedef unsigned long long uint64_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef unsigned long long uintptr_t;
#endif

namespace gatlas {
namespace img {

template <typename T>
struct ImgArgs {
    T *C;
    int64_t M, N, K, ldc, stride_c;
    T alpha, beta;
    int gemm;
    int *fault;
};

// Tensor-map descriptors are passed as opaque, 64-byte aligned 128-byte blocks.
struct __align__(64) TmapBlob {
    unsigned long long w[16];
};

template <typename T> struct Bk;
template <> struct Bk<float> { static constexpr int value = 32; };   // 128-byte rows
template <> struct Bk<double> { static constexpr int value = 16; };

template <typename T, bool TA, bool TB, int GH, int GW, int BH, int BW>
struct ImgTile {
    static constexpr int BK = Bk<T>::value;
    static constexpr int NT = GH * GW;
    static constexpr int BM = GH * BH, BN = GW * BW;
    static constexpr int S = 2;  // two stages and two CTAs per SM hide the TMA latency
    static constexpr int ALIGN = 1024 / (int)sizeof(T);                // raw tiles start on 1 KiB
    static constexpr int A_BOX = BM * BK, B_BOX = BN * BK;             // elements delivered per stage
    static constexpr int A_RAW = (A_BOX + ALIGN - 1) / ALIGN * ALIGN;  // padded slots
    static constexpr int B_RAW = (B_BOX + ALIGN - 1) / ALIGN * ALIGN;
    static constexpr int PA = TA ? BM : BM + 4;                        // pitch of the k-major A tile
    static constexpr int PB = TB ? BN + 4 : BN;
    static constexpr int SMEM = (S * (A_RAW + B_RAW) + (TA ? 0 : BK * PA) + (TB ? BK * PB : 0)) * (int)sizeof(T) + 1024;
};

template <typename T>
struct alignas(4 * sizeof(T)) Quad {
    T v[4];
};

template <typename T>
struct alignas(16) Chunk {
    T v[16 / sizeof(T)];
};

// Transposes a swizzled m-major raw tile (rows x BK) into a k-major tile with
// pitch P: thread e copies one 16-byte chunk of one row; eight consecutive
// threads read eight rows of the same logical chunk, which the swizzle spreads
// over all banks, and write consecutive rows of the k-major tile.
template <typename T, int BK, int ROWS, int P, int NT>
__device__ __forceinline__ void transpose_tile(const T *rawt, T *km, int tid) {
    constexpr int PER = 16 / (int)sizeof(T);
    constexpr int CHUNKS = BK / PER;
    for (int e = tid; e < ROWS * CHUNKS; e += NT) {
        const int r = e % ROWS, c = e / ROWS;
        const Chunk<T> q = *reinterpret_cast<const Chunk<T> *>(rawt + r * BK + ((c ^ (r & 7)) * PER));
#pragma unroll
        for (int j = 0; j < PER; ++j) km[(c * PER + j) * P + r] = q.v[j];
    }
}

__device__ __forceinline__ uint32_t img_smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t img_globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool img_wait(uint64_t *bar, uint32_t parity, volatile int *abort) {
    const uint64_t t0 = img_globaltimer();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(img_smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (*abort) return false;
        if (img_globaltimer() - t0 > 1000000000ull) return false;
    }
}

__device__ __forceinline__ void img_load(void *dst, const TmapBlob *map, int32_t x, int32_t y, int32_t z,
                                         uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(img_smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(img_smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ float img_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double img_fma(double a, double b, double c) { return __fma_rn(a, b, c); }

// Two round-to-nearest fused multiply-adds in one packed instruction
// (fma.rn.f32x2, sm_100): d0 = a*b0 + d0 and d1 = a*b1 + d1, each exactly
// what __fmaf_rn gives.
__device__ __forceinline__ void img_fma2(float &d0, float &d1, float a, float b0, float b1) {
    asm("{.reg .b64 pa, pb, pd;\n\t"
        "mov.b64 pa, {%2, %2};\n\t"
        "mov.b64 pb, {%3, %4};\n\t"
        "mov.b64 pd, {%0, %1};\n\t"
        "fma.rn.f32x2 pd, pa, pb, pd;\n\t"
        "mov.b64 {%0, %1}, pd;}"
        : "+f"(d0), "+f"(d1)
        : "f"(a), "f"(b0), "f"(b1));
}

template <typename T, bool TA, bool TB, int GH, int GW, int BH, int BW>
__global__ void __launch_bounds__(GH *GW, (GH * GW <= 256) ? 2 : 1)
    gemm_image_kernel(const __grid_constant__ TmapBlob mapA, const __grid_constant__ TmapBlob mapB, ImgArgs<T> a) {
    using L = ImgTile<T, TA, TB, GH, GW, BH, BW>;
    constexpr int BK = L::BK, BM = L::BM, BN = L::BN, S = L::S, NT = L::NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // 128-byte swizzled tiles must start on 1 KiB boundaries; the launch adds
    // 1 KiB of slack for this alignment
    T *raw = reinterpret_cast<T *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    T *kmA = raw + S * (L::A_RAW + L::B_RAW);
    T *kmB = kmA + (TA ? 0 : BK * L::PA);
    __shared__ __align__(8) uint64_t full[S];
    __shared__ volatile int abort_flag;

    const int tid = threadIdx.x, tx = tid % GW, ty = tid / GW;
    const int64_t m0 = (int64_t)blockIdx.y * BM, n0 = (int64_t)blockIdx.x * BN;
    const int z = blockIdx.z;
    const int64_t KT = (a.K + BK - 1) / BK;
    const uint32_t stage_bytes = (uint32_t)((L::A_BOX + L::B_BOX) * sizeof(T));

    if (tid == 0) {
        for (int s = 0; s < S; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(img_smem_u32(&full[s])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    __syncthreads();

    auto issue = [&](int64_t kt) {
        const int s = (int)(kt % S);
        T *ra = raw + s * (L::A_RAW + L::B_RAW);
        T *rb = ra + L::A_RAW;
        asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(img_smem_u32(&full[s])),
                     "r"(stage_bytes)
                     : "memory");
        const int32_t k0 = (int32_t)(kt * BK);
        if (TA) img_load(ra, &mapA, (int32_t)m0, k0, z, &full[s]);   // [k][m]
        else img_load(ra, &mapA, k0, (int32_t)m0, z, &full[s]);      // [m][k], swizzled
        if (TB) img_load(rb, &mapB, k0, (int32_t)n0, z, &full[s]);   // [n][k], swizzled
        else img_load(rb, &mapB, (int32_t)n0, k0, z, &full[s]);      // [k][n]
    };

    if (tid == 0)
        for (int64_t kt = 0; kt < S - 1 && kt < KT; ++kt) issue(kt);

    T acc[BH][BW];
#pragma unroll
    for (int i = 0; i < BH; ++i)
#pragma unroll
        for (int j = 0; j < BW; ++j) acc[i][j] = T(0);

    int64_t kt = 0;
    for (; kt < KT; ++kt) {
        const int s = (int)(kt % S);
        if (tid == 0 && kt + S - 1 < KT) issue(kt + S - 1);
        if (!img_wait(&full[s], (uint32_t)(kt / S) & 1u, &abort_flag)) {
            if (a.fault && !abort_flag) atomicOr(a.fault, 1 << 2);
            abort_flag = 1;
        }
        __syncthreads();
        if (abort_flag) break;
        const T *ra = raw + s * (L::A_RAW + L::B_RAW);
        const T *rb = ra + L::A_RAW;
        const T *Ak = ra;
        const T *Bk = rb;
        if (!TA || TB) {
            // transpose the m-major tiles into their k-major buffers
            if (!TA) transpose_tile<T, BK, BM, L::PA, NT>(ra, kmA, tid);
            if (TB) transpose_tile<T, BK, BN, L::PB, NT>(rb, kmB, tid);
            __syncthreads();
            if (!TA) Ak = kmA;
            if (TB) Bk = kmB;
        }
        constexpr int PA = L::PA, PB = L::PB;
#pragma unroll 4
        for (int kk = 0; kk < BK; ++kk) {
            T af[BH], bf[BW];
            if constexpr (BH % 4 == 0) {
#pragma unroll
                for (int g = 0; g < BH / 4; ++g) {
                    const Quad<T> q = *reinterpret_cast<const Quad<T> *>(Ak + kk * PA + g * GH * 4 + ty * 4);
#pragma unroll
                    for (int e = 0; e < 4; ++e) af[g * 4 + e] = q.v[e];
                }
            } else {
#pragma unroll
                for (int i = 0; i < BH; ++i) af[i] = Ak[kk * PA + ty * BH + i];
            }
            if constexpr (BW % 4 == 0) {
#pragma unroll
                for (int g = 0; g < BW / 4; ++g) {
                    const Quad<T> q = *reinterpret_cast<const Quad<T> *>(Bk + kk * PB + g * GW * 4 + tx * 4);
#pragma unroll
                    for (int e = 0; e < 4; ++e) bf[g * 4 + e] = q.v[e];
                }
            } else {
#pragma unroll
                for (int j = 0; j < BW; ++j) bf[j] = Bk[kk * PB + tx * BW + j];
            }
            // FP32 column pairs in one packed instruction: the same fused
            // multiply-add chain per element, half the FMA instructions
            if constexpr (sizeof(T) == 4 && BW % 2 == 0) {
#pragma unroll
                for (int i = 0; i < BH; ++i)
#pragma unroll
                    for (int j = 0; j < BW; j += 2) img_fma2(acc[i][j], acc[i][j + 1], af[i], bf[j], bf[j + 1]);
            } else {
#pragma unroll
                for (int i = 0; i < BH; ++i)
#pragma unroll
                    for (int j = 0; j < BW; ++j) acc[i][j] = img_fma(af[i], bf[j], acc[i][j]);
            }
        }
        __syncthreads();
    }
    if (abort_flag) {
        // bounded wait for the tiles still landing in shared memory
        if (tid == 0) {
            volatile int never = 0;
            for (int64_t k = kt; k < KT && k < kt + S; ++k) img_wait(&full[k % S], (uint32_t)(k / S) & 1u, &never);
        }
        return;
    }
    T *C = a.C + (int64_t)z * a.stride_c;
#pragma unroll
    for (int i = 0; i < BH; ++i) {
        const int r = (BH % 4 == 0) ? (i / 4) * (GH * 4) + ty * 4 + (i % 4) : ty * BH + i;
        const int64_t row = m0 + r;
        if (row >= a.M) continue;
#pragma unroll
        for (int j = 0; j < BW; ++j) {
            const int c = (BW % 4 == 0) ? (j / 4) * (GW * 4) + tx * 4 + (j % 4) : tx * BW + j;
            const int64_t col = n0 + c;
            if (col >= a.N) continue;
            T *p = C + row * a.ldc + col;
            if (a.gemm) {
                const T bc = (a.beta == T(0)) ? T(0) : a.beta * *p;
                *p = img_fma(a.alpha, acc[i][j], bc);
            } else {
                *p = acc[i][j];
            }
        }
    }
}

}  // namespace img
}  // namespace gatlas
