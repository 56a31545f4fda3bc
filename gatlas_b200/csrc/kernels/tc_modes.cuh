// Shared pieces of the tensor-core engines: tile shape, per-mode operand
// formats and shared-memory layouts, and the FP32 -> BF16 piece split.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "../tcgen05.cuh"

namespace gatlas {
namespace tcg {

constexpr int BM = 128, BN = 256;

// Default promotion interval for the BF16 modes: 4 slices of 32, i.e.
// K = 128 per TMEM segment (selectable per call through the descriptor's
// extra field).  The FP8 mode promotes every slice (one scale block).
constexpr int kDefaultSegKblocks = 4;
// One-product BF16 promotes every 16 slices (K = 512): its MMA segment of 4
// slices is shorter than the drain, and the longer TMEM accumulation adds
// nothing measurable next to BF16's own input rounding (2^-9).
constexpr int kDefaultSegKblocksBf16 = 16;
__host__ __device__ constexpr int default_seg_kblocks(int mode) {
    return mode == 0 ? kDefaultSegKblocksBf16 : kDefaultSegKblocks;
}
// FP8: most 128-deep blocks per tile (K <= 131072), and by default at most
// 4 equally scaled blocks accumulate in TMEM before promotion.
constexpr int kMaxFp8Blocks = 1024;

// MODE 0: one BF16 piece, one product; 1: two pieces, three products;
// 2: three pieces, six products; 3: FP8 E4M3 codes with one FP32 scale per
// 128 x 128 block of each operand.  Every mode stages K slices of 32 bytes
// per MMA instruction: K = 16 BF16 or K = 32 E4M3 elements.
template <int MODE>
struct Mode;
template <>
struct Mode<0> {
    static constexpr int NP = 1, NPROD = 1, STAGES = 8, ELEM = 2, BKE = 32;
    static constexpr bool SCALED = false;
    __device__ static constexpr int pa(int) { return 0; }
    __device__ static constexpr int pb(int) { return 0; }
};
template <>
struct Mode<1> {
    static constexpr int NP = 2, NPROD = 3, STAGES = 4, ELEM = 2, BKE = 32;
    static constexpr bool SCALED = false;
    // hi*hi, hi*lo, lo*hi
    __device__ static constexpr int pa(int j) { return j == 2 ? 1 : 0; }
    __device__ static constexpr int pb(int j) { return j == 1 ? 1 : 0; }
};
template <>
struct Mode<2> {
    static constexpr int NP = 3, NPROD = 6, STAGES = 3, ELEM = 2, BKE = 32;
    static constexpr bool SCALED = false;
    // hi*hi, hi*mid, mid*hi, mid*mid, hi*lo, lo*hi
    __device__ static constexpr int pa(int j) { return j == 2 || j == 3 ? 1 : (j == 5 ? 2 : 0); }
    __device__ static constexpr int pb(int j) { return j == 1 || j == 3 ? 1 : (j == 4 ? 2 : 0); }
};
template <>
struct Mode<3> {
    static constexpr int NP = 1, NPROD = 1, STAGES = 4, ELEM = 1, BKE = 128;
    static constexpr bool SCALED = true;
    __device__ static constexpr int pa(int) { return 0; }
    __device__ static constexpr int pb(int) { return 0; }
};

template <int MODE>
struct Layout {
    using MD = Mode<MODE>;
    static constexpr int NP = MD::NP;
    static constexpr int STAGES = MD::STAGES;
    static constexpr int BK = MD::BKE;                              // elements per K slice
    static constexpr uint32_t ROW_BYTES = BK * MD::ELEM;            // 64 (BF16) or 128 (FP8)
    static constexpr uint32_t SWIZZLE = ROW_BYTES == 128 ? tc::kSwizzle128B : tc::kSwizzle64B;
    static constexpr uint32_t SBO = 8 * ROW_BYTES;                  // 8-row core-matrix groups
    static constexpr uint32_t A_TILE = BM * ROW_BYTES;
    static constexpr uint32_t B_TILE = BN * ROW_BYTES;
    static constexpr int KSTEPS = ROW_BYTES / 32;                   // MMA instructions per slice
    static constexpr uint32_t STAGE_BYTES = NP * (A_TILE + B_TILE);
    // FP8: per-block scale products of the tile's two column halves, compacted
    // in place into per-segment scales, and one segment-start flag per block
    static constexpr uint32_t PLAN_BYTES = MD::SCALED ? (2 * 4 + 1) * 1024 : 0;
    static constexpr uint32_t SMEM_BYTES = STAGES * STAGE_BYTES + PLAN_BYTES + 1024;  // + alignment slack
    static constexpr uint32_t IDESC = MD::SCALED ? tc::idesc_e4m3_f32(BM, BN) : tc::idesc_bf16_f32(BM, BN);
};

// CTA-pair layout (cta_group::2): one 256 x 256 tile per pair of CTAs.  Each
// CTA stages its 128 rows of A and its 128-row half of B per K slice, and
// holds its 128 rows of the accumulator in its own TMEM.
template <int MODE>
struct PairLayout {
    using L1 = Layout<MODE>;
    using MD = Mode<MODE>;
    static constexpr int NP = MD::NP;
    static constexpr int BK = L1::BK;
    static constexpr uint32_t ROW_BYTES = L1::ROW_BYTES;
    static constexpr uint32_t SWIZZLE = L1::SWIZZLE;
    static constexpr uint32_t SBO = L1::SBO;
    static constexpr int KSTEPS = L1::KSTEPS;
    static constexpr int PM = 256, PN = 256;                 // pair tile
    static constexpr uint32_t A_TILE = 128 * ROW_BYTES;      // this CTA's rows of A
    static constexpr uint32_t B_TILE = 128 * ROW_BYTES;      // this CTA's half of B
    static constexpr uint32_t STAGE_BYTES = NP * (A_TILE + B_TILE);
    static constexpr uint32_t PLAN_BYTES = L1::PLAN_BYTES;
    static constexpr uint32_t BUDGET = 226 * 1024;          // dynamic shared memory per CTA
    static constexpr int STAGES = (int)((BUDGET - PLAN_BYTES - 1024) / STAGE_BYTES);
    static constexpr uint32_t SMEM_BYTES = STAGES * STAGE_BYTES + PLAN_BYTES + 1024;
    static constexpr uint32_t IDESC = MD::SCALED ? tc::idesc_e4m3_f32(PM, PN) : tc::idesc_bf16_f32(PM, PN);
    static_assert(STAGES >= 3, "pair pipeline depth");
};

template <int NP>
__device__ __forceinline__ void split_value(float x, __nv_bfloat16 (&out)[3]) {
    const __nv_bfloat16 hi = __float2bfloat16_rn(x);
    out[0] = hi;
    if constexpr (NP >= 2) {
        const float r1 = x - __bfloat162float(hi);  // exact
        const __nv_bfloat16 mid = __float2bfloat16_rn(r1);
        out[1] = mid;
        if constexpr (NP >= 3) {
            const float r2 = r1 - __bfloat162float(mid);  // exact
            out[2] = __float2bfloat16_rn(r2);
        }
    }
}

}  // namespace tcg
}  // namespace gatlas
