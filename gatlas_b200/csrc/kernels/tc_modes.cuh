// Shared pieces of the tensor-core engines: tile shape, per-mode operand
// formats and shared-memory layouts, and the FP32 -> BF16 piece split.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "../tcgen05.cuh"

namespace gatlas {
namespace tcg {

constexpr int BM = 128, BN = 256;

// Default promotion intervals, in K slices of each mode (selectable per call
// through the descriptor's extra field): split3 promotes every K = 256
// (4 slices of 64), split6 every K = 128 (4 slices of 32).  Each promotion
// is a round trip between the MMA issuer and the drain warps (of both CTAs
// of a pair); at 8192^3, split3 with K = 256 runs 5 % faster than with
// K = 128 while its normwise error grows from 3.81e-6 to 3.87e-6.
// One-product BF16 accumulates all of K in TMEM (kSegAll): the tensor core's
// FP32 accumulation error stays far below BF16's own input rounding (2^-9),
// and without promotion a 256 x 256 tile fits one CTA.  FP8 accumulates runs
// of at most 16 equally scaled 128-deep blocks (K = 2048): at 8192^3 on
// sign * 2^e operands, which E4M3 holds exactly, the normwise error is
// 1.2e-6 (3.2e-7 with runs of 4, below SIMT FP32's 1.6e-6 either way), on
// uniform operands E4M3's own rounding (0.033) is unchanged, and the
// contraction takes 0.490 ms instead of 0.517.
constexpr int kSegAll = 1 << 30;
__host__ __device__ constexpr int default_seg_kblocks(int mode) {
    return mode == 0 ? kSegAll : mode == 3 ? 16 : 4;
}
// FP8: most 128-deep blocks per tile (K <= 131072).
constexpr int kMaxFp8Blocks = 1024;

// MODE 0: one BF16 piece, one product; 1: two pieces, three products;
// 2: three pieces, six products; 3: FP8 E4M3 codes with one FP32 scale per
// 128 x 128 block of each operand.  Each MMA instruction consumes 32 bytes
// of K per row (K = 16 BF16 or K = 32 E4M3 elements); a pipeline slice is
// one ROWB-byte row per operand row: 128 bytes (128-byte swizzle) where the
// ring still holds at least two slices, 64 bytes (64-byte swizzle) for the
// six-product mode, whose three pieces per operand would leave one.  On
// B200 the tensor core streams 128-byte-swizzled rows markedly faster: the
// one-product BF16 kernel runs 993 instead of 630 TFLOP/s at 8192^3.
template <int MODE>
struct Mode;
template <>
struct Mode<0> {
    static constexpr int NP = 1, NPROD = 1, ELEM = 2, ROWB = 128;
    static constexpr bool SCALED = false;
    __device__ static constexpr int pa(int) { return 0; }
    __device__ static constexpr int pb(int) { return 0; }
};
template <>
struct Mode<1> {
    static constexpr int NP = 2, NPROD = 3, ELEM = 2, ROWB = 128;
    static constexpr bool SCALED = false;
    // hi*hi, hi*lo, lo*hi
    __device__ static constexpr int pa(int j) { return j == 2 ? 1 : 0; }
    __device__ static constexpr int pb(int j) { return j == 1 ? 1 : 0; }
};
template <>
struct Mode<2> {
    static constexpr int NP = 3, NPROD = 6, ELEM = 2, ROWB = 64;
    static constexpr bool SCALED = false;
    // hi*hi, hi*mid, mid*hi, mid*mid, hi*lo, lo*hi
    __device__ static constexpr int pa(int j) { return j == 2 || j == 3 ? 1 : (j == 5 ? 2 : 0); }
    __device__ static constexpr int pb(int j) { return j == 1 || j == 3 ? 1 : (j == 4 ? 2 : 0); }
};
template <>
struct Mode<3> {
    static constexpr int NP = 1, NPROD = 1, ELEM = 1, ROWB = 128;
    static constexpr bool SCALED = true;
    __device__ static constexpr int pa(int) { return 0; }
    __device__ static constexpr int pb(int) { return 0; }
};

// Single-CTA layout (128 x 256 tiles) with ROWB-byte K slices; the ring
// takes as many stages as 226 KB of shared memory hold, at most 8.
template <int MODE, uint32_t ROWB = Mode<MODE>::ROWB>
struct Layout {
    using MD = Mode<MODE>;
    static constexpr int NP = MD::NP;
    static constexpr uint32_t ROW_BYTES = ROWB;                     // 64 or 128
    static constexpr int BK = (int)(ROWB / MD::ELEM);               // elements per K slice
    static constexpr uint32_t SWIZZLE = ROW_BYTES == 128 ? tc::kSwizzle128B : tc::kSwizzle64B;
    static constexpr uint32_t SBO = 8 * ROW_BYTES;                  // 8-row core-matrix groups
    static constexpr uint32_t A_TILE = BM * ROW_BYTES;
    static constexpr uint32_t B_TILE = BN * ROW_BYTES;
    static constexpr int KSTEPS = ROW_BYTES / 32;                   // MMA instructions per slice
    static constexpr uint32_t STAGE_BYTES = NP * (A_TILE + B_TILE);
    // FP8: per-block scale products of the tile's two column halves, compacted
    // in place into per-segment scales, and one segment-start flag per block
    static constexpr uint32_t PLAN_BYTES = MD::SCALED ? (2 * 4 + 1) * 1024 : 0;
    static constexpr uint32_t BUDGET = 226 * 1024;
    static constexpr int FIT = (int)((BUDGET - PLAN_BYTES - 1024) / STAGE_BYTES);
    static constexpr int STAGES = FIT < 8 ? FIT : 8;
    static_assert(STAGES >= 2, "tensor-core pipeline depth");
    static_assert(ROWB == 64 || ROWB == 128, "K slice of 64 or 128 bytes");
    static constexpr uint32_t SMEM_BYTES = STAGES * STAGE_BYTES + PLAN_BYTES + 1024;  // + alignment slack
    static constexpr uint32_t IDESC = MD::SCALED ? tc::idesc_e4m3_f32(BM, BN) : tc::idesc_bf16_f32(BM, BN);
};

// Persistent layout: the ring, then one 32 x 32 FP32 staging
// tile per drain warp for the TMA-store epilogue, which runs while the ring
// already feeds the next tile.  PAIR: a 256 x 256 tile per cluster of two
// CTAs, each staging its 128 rows of A and its 128-row half of B.
constexpr uint32_t kEpiTileBytes = 32 * 32 * 4;
constexpr uint32_t kEpiBytes = 8 * kEpiTileBytes;
template <int MODE, bool PAIR, uint32_t ROWB = Mode<MODE>::ROWB>
struct PersistentLayout {
    using MD = Mode<MODE>;
    static constexpr int NP = MD::NP;
    static constexpr uint32_t ROW_BYTES = ROWB;
    static constexpr int BK = (int)(ROWB / MD::ELEM);
    static constexpr uint32_t SWIZZLE = ROWB == 128 ? tc::kSwizzle128B : tc::kSwizzle64B;
    static constexpr uint32_t SBO = 8 * ROWB;
    static constexpr int KSTEPS = (int)(ROWB / 32);
    static constexpr int TM = PAIR ? 256 : 128;                    // rows of C per tile
    static constexpr uint32_t A_TILE = 128 * ROWB;                 // this CTA's rows of A
    static constexpr uint32_t B_TILE = (PAIR ? 128u : 256u) * ROWB;  // B's 256 rows, or this CTA's half
    static constexpr uint32_t STAGE_BYTES = NP * (A_TILE + B_TILE);
    static constexpr uint32_t BUDGET = 226 * 1024;
    static constexpr int FIT = (int)((BUDGET - kEpiBytes - 1024) / STAGE_BYTES);
    static constexpr int STAGES = FIT < 8 ? FIT : 8;
    static constexpr uint32_t EPI_OFFSET = STAGES * STAGE_BYTES;
    static constexpr uint32_t SMEM_BYTES = EPI_OFFSET + kEpiBytes + 1024;  // + alignment slack
    static constexpr uint32_t IDESC = MD::SCALED ? tc::idesc_e4m3_f32(TM, 256) : tc::idesc_bf16_f32(TM, 256);
    static_assert(STAGES >= 2, "tensor-core pipeline depth");
};

// Wide layout (one-product BF16 accumulated over all of K): one CTA computes
// a 256 x 256 tile as two M = 128 accumulators, all 512 TMEM columns, so a K
// slice stages 256 rows of A and 256 of B (64 KiB) for 8 MMAs: a third fewer
// bytes per MMA than a 128 x 256 tile, without a CTA pair's round trips.
struct WideLayout {
    static constexpr uint32_t ROW_BYTES = 128;
    static constexpr int BK = 64;                  // BF16 elements per K slice
    static constexpr uint32_t SWIZZLE = tc::kSwizzle128B;
    static constexpr uint32_t SBO = 8 * ROW_BYTES;
    static constexpr int KSTEPS = (int)(ROW_BYTES / 32);
    static constexpr int TM = 256;
    static constexpr uint32_t A_TILE = 256 * ROW_BYTES;  // rows 0..127, then 128..255
    static constexpr uint32_t A_HALF = 128 * ROW_BYTES;
    static constexpr uint32_t B_TILE = 256 * ROW_BYTES;
    static constexpr uint32_t STAGE_BYTES = A_TILE + B_TILE;
    static constexpr uint32_t BUDGET = 226 * 1024;
    static constexpr int STAGES = (int)((BUDGET - kEpiBytes - 1024) / STAGE_BYTES);
    static constexpr uint32_t EPI_OFFSET = STAGES * STAGE_BYTES;
    static constexpr uint32_t SMEM_BYTES = EPI_OFFSET + kEpiBytes + 1024;  // + alignment slack
    static constexpr uint32_t IDESC = tc::idesc_bf16_f32(128, 256);
    static_assert(STAGES >= 3, "wide pipeline depth");
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
