// Grouped tensor-core matmul: hundreds of instances of different shapes and
// layouts (C_i = alpha_i * op(A_i) op(B_i) + beta_i * C_i) in one persistent
// launch.
//
// No reference counterpart as one kernel: the reference batches only equal
// shapes (packedCalc, KernelMatmulBuffer.hpp:229-230) and otherwise runs one
// kernel per problem.  Design for B200:
//  1. pack pass (one launch for all instances): every FP32 operand is split
//     into BF16 pieces and written tile-major in the exact shared-memory
//     image the MMA descriptors read: A as [mt][kt][128 rows x 128 B], B as
//     [nt][kt][BN rows x 128 B], each tile 128-byte swizzled (16-byte chunk
//     c of row r stored at chunk c ^ (r & 7)), zero padded past M, N, K.
//     The contraction then streams every tile with one 1-D bulk copy: no
//     per-instance tensor maps.  The pack itself stages its source tiles
//     with 16-byte async copies through a 3-stage shared-memory ring;
//  2. contraction: one CTA per SM walks a statically balanced list of
//     output tiles (longest first, greedy onto the least-loaded CTA) across
//     instances.  Warp 0 streams tiles through the mbarrier ring, warp 1
//     issues tcgen05.mma (N = the instance's tile width), warps 2..9 promote
//     the TMEM segments into FP32 registers and write C, overlapping the
//     epilogue of one tile with the main loop of the next (two TMEM
//     accumulators).
// The tile width BN (64, 128 or 256) is chosen per instance, by default from
// a per-size-bucket table that the autotuner fills.
// Every wait is bounded; a timeout sets the device fault word, stops the
// pipeline, drains the copies in flight and frees TMEM.
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <queue>
#include <vector>

#include "../common.cuh"
#include "../device_state.cuh"
#include "../tcgen05.cuh"
#include "gemm_engines.hpp"
#include "grouped.hpp"
#include "tc_modes.cuh"

namespace gatlas {
namespace grp {

using tcg::BM;
constexpr int kPackBK = 64;              // K elements per pack item
constexpr uint32_t kPackRowBytes = 128;   // one pack item's row of one BF16 piece
constexpr uint32_t kRowBytes = 128;       // one contraction K slice of one row (128-byte swizzle)
constexpr int kBK = kRowBytes / 2;        // BF16 elements per contraction K slice
constexpr int kSlicesPerItem = (int)(kPackRowBytes / kRowBytes);
constexpr uint32_t kATileBytes = BM * kRowBytes;
constexpr int kDrainWarps = 8;            // a multiple of 4: kDrainParts warps per TMEM lane quarter
constexpr int kThreads = 32 * (2 + kDrainWarps);
constexpr int kDrainParts = kDrainWarps / 4;          // column parts of a tile per lane quarter
constexpr int kPartGroups = 256 / kDrainParts / 8;    // 8-column groups in a part of the widest tile
constexpr int kAccRegs = 2 * kPartGroups * 4;         // accumulator registers per drain thread
constexpr uint32_t kTmemCols = 512;       // two accumulators of up to 256 columns
constexpr uint64_t kWaitNs = 2000000000ull;
constexpr int kPackRows = 128;            // rows per pack item
constexpr int kEpiBatch = 8;              // 8-column groups of C loaded together by the epilogue
static_assert(kDrainWarps % 4 == 0 && kPartGroups % kEpiBatch == 0, "drain layout");
// The grouped engine stages 64-byte K slices (its packed tiles carry the
// 64-byte swizzle), so that a ring of 48 KiB stages holds four split3 K slices
// of a 128 x 256 tile, and promotes after the same K as the single-instance
// engine (all of K for one-product BF16, 256 for split3), issuing the same
// MMA sequence (16-deep K steps in order, the products of each in order), so
// that each instance's result is bit-identical to it.
// Ring layout: a stage holds every piece of a 128-row A tile and of BROWS
// rows of B (one K slice): all 256 rows of the widest tile on a single CTA,
// its 128-row half on each CTA of a pair.
template <int MODE, int BROWS>
struct GLayout {
    using MD = tcg::Mode<MODE>;
    static constexpr int BK = kRowBytes / MD::ELEM;
    static constexpr uint32_t SWIZZLE = kRowBytes == 128 ? tc::kSwizzle128B : tc::kSwizzle64B;
    static constexpr uint32_t SBO = 8 * kRowBytes;
    static constexpr int KSTEPS = kRowBytes / 32;
    static constexpr uint32_t A_TILE = BM * kRowBytes;
    static constexpr uint32_t B_TILE = BROWS * kRowBytes;
    static constexpr uint32_t STAGE_BYTES = MD::NP * (A_TILE + B_TILE);
    static constexpr int FIT = (int)((226 * 1024 - 1024) / STAGE_BYTES);
    static constexpr int STAGES = FIT < 8 ? FIT : 8;
    static constexpr uint32_t SMEM_BYTES = STAGES * STAGE_BYTES + 1024;  // + alignment slack
    static_assert(STAGES >= 2, "grouped pipeline depth");
};
template <int MODE, bool PAIR>
using GLayoutOf = GLayout<MODE, PAIR ? 128 : 256>;
constexpr int grouped_seg_kblocks(int mode) { return mode == 0 ? tcg::kSegAll : 256 / kBK; }

// Packed byte offset of 16-byte chunk c (0..7) of row `row` of pack item kb
// (K elements 64 kb .. 64 kb + 63) in an operand of kt items per row block of
// tr rows.  Each row block is a run of K slices, each slice tr rows of
// kRowBytes; 16-byte chunk j of row r sits at chunk j ^ (r & 7) (128-byte
// swizzle) or j ^ ((r >> 1) & 3) (64-byte swizzle), the layouts the MMA's
// shared-memory descriptors read.
__device__ __forceinline__ int64_t packed_offset(int64_t row, int kb, int c, int tr, int kt) {
    constexpr int per = (int)(kRowBytes / 16);  // chunks per slice row
    const int s = kb * kSlicesPerItem + c / per, j = c % per;
    const int swz = kRowBytes == 128 ? (int)(row & 7) : (int)((row >> 1) & 3);
    return ((row / tr) * (int64_t)(kt * kSlicesPerItem) + s) * (int64_t)tr * kRowBytes + (row % tr) * kRowBytes +
           ((j ^ swz) << 4);
}

// ---------------------------------------------------------------------------
// pack pass
// ---------------------------------------------------------------------------
// Item space: segment s = 2*instance + operand covers rows/128 x kt items,
// ordered row block major, K slice minor.  CTA b packs the contiguous items
// [b*per_cta, (b+1)*per_cta): one binary search for its first segment, then
// an incremental walk, and neighbouring items read neighbouring memory.
// Where item `it` of segment `sg` reads and writes.
struct PackItem {
    const Inst *I;
    int op, kb, tr;
    int64_t r0, k0, rows, rows_alloc, ld, K;
    const float *src;
    bool transposed, vec;
};

__device__ __forceinline__ PackItem pack_item(const Inst *insts, const int64_t *seg_start, int sgi, int64_t it) {
    PackItem q;
    q.I = insts + (sgi >> 1);
    const Inst &I = *q.I;
    q.op = sgi & 1;
    const int64_t local = it - seg_start[sgi];
    q.kb = (int)(local % I.kt);
    q.r0 = (local / I.kt) * kPackRows;
    q.k0 = (int64_t)q.kb * kPackBK;
    q.rows = q.op ? I.N : I.M;
    q.tr = q.op ? I.bn : BM;
    q.rows_alloc = q.op ? (int64_t)I.nt * I.bn : (int64_t)I.mt * BM;
    q.transposed = q.op ? (I.tb == 0) : (I.ta != 0);
    q.src = q.op ? I.src_b : I.src_a;
    q.ld = q.op ? I.ldb : I.lda;
    q.vec = (q.ld % 4 == 0) && ((reinterpret_cast<uintptr_t>(q.src) & 15) == 0);
    q.K = I.K;
    return q;
}

// Stage layout: [128 rows][64 k] floats (rows of 256 B) for row-major
// sources, [64 k][128 rows] (k rows of 512 B) for transposed ones, where the
// 16-byte chunk of rows 4q..4q+3 in k row k sits at chunk q ^ ((k >> 3) & 7),
// so that the eight k-runs one warp reads per row land in distinct banks.
constexpr uint32_t kPackTileBytes = kPackRows * kPackBK * 4;
constexpr int kPackStages = 3;
constexpr uint32_t kPackSmemBytes = kPackStages * kPackTileBytes;
constexpr int kPackChunks = (int)(kPackTileBytes / 16) / 256;  // 16-byte chunks per thread per item

__device__ __forceinline__ void cp_async16(void *smem_dst, const void *src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(smem_dst)), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem_dst, const void *src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(smem_dst)), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Thread `tid` copies its 16-byte chunks of item q into `stage` with async
// copies (no registers held while they fly); bytes past M, N or K are
// zero-filled by the copies themselves.
__device__ __forceinline__ void pack_issue(const PackItem &q, uint8_t *stage, int tid) {
#pragma unroll
    for (int j = 0; j < kPackChunks; ++j) {
        const int e = j * 256 + tid;
        int64_t outer, inner, outer_lim, inner_lim;
        if (!q.transposed) {  // stage[r][k]: 16 chunks per 256-byte row
            outer = q.r0 + (e >> 4), inner = q.k0 + (e & 15) * 4, outer_lim = q.rows, inner_lim = q.K;
        } else {              // stage[k][r]: 32 chunks per 512-byte k row
            outer = q.k0 + (e >> 5), inner = q.r0 + (e & 31) * 4, outer_lim = q.K, inner_lim = q.rows;
        }
        int64_t valid = outer < outer_lim ? inner_lim - inner : 0;
        valid = valid < 0 ? 0 : (valid > 4 ? 4 : valid);
        const float *src = valid > 0 ? q.src + outer * q.ld + inner : q.src;
        uint8_t *dst = !q.transposed ? stage + (size_t)e * 16
                                     : stage + (size_t)(e >> 5) * 512 + (((e & 31) ^ ((e >> 8) & 7)) << 4);
        if (q.vec) {
            cp_async16(dst, src, (uint32_t)valid * 4);
        } else {
#pragma unroll
            for (int v = 0; v < 4; ++v) cp_async4(dst + 4 * v, v < valid ? src + v : q.src, v < valid ? 4u : 0u);
        }
    }
}

// One walk per CTA over its items: every thread keeps kPackStages - 1 items
// of async copies in flight while the CTA splits the current item from
// shared memory into BF16 pieces and writes them with 16-byte swizzled
// stores.
template <int NP>
__global__ void __launch_bounds__(256, 2) grouped_pack_kernel(const Inst *insts, const int64_t *seg_start, int nseg,
                                                           int64_t per_cta) {
    extern __shared__ __align__(128) uint8_t pack_smem[];
    const int tid = threadIdx.x;
    const int64_t nitems = seg_start[nseg];
    const int64_t it0 = (int64_t)blockIdx.x * per_cta;
    const int64_t it1 = it0 + per_cta < nitems ? it0 + per_cta : nitems;
    if (it0 >= it1) return;
    int sgi = 0;
    {
        int lo = 0, hi = nseg - 1;  // last segment whose start is <= it0
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (seg_start[mid] <= it0) lo = mid;
            else hi = mid - 1;
        }
        sgi = lo;
    }
    while (it0 >= seg_start[sgi + 1]) ++sgi;
    auto stage_of = [&](int64_t it) { return pack_smem + (size_t)((it - it0) % kPackStages) * kPackTileBytes; };

    // issue cursor: one commit group per item (empty past the range), so that
    // wait_group counts items
    int psgi = sgi;
    int64_t pit = it0;
    auto issue_next = [&]() {
        if (pit < it1) {
            while (pit >= seg_start[psgi + 1]) ++psgi;
            pack_issue(pack_item(insts, seg_start, psgi, pit), stage_of(pit), tid);
        }
        cp_async_commit();
        ++pit;
    };
    for (int i = 0; i < kPackStages - 1; ++i) issue_next();

    for (int64_t it = it0; it < it1; ++it) {
        issue_next();  // into the stage the previous iteration released
        cp_async_wait<kPackStages - 1>();  // this thread's copies of item `it` have landed
        __syncthreads();                   // and every other thread's
        while (it >= seg_start[sgi + 1]) ++sgi;
        const PackItem cur = pack_item(insts, seg_start, sgi, it);
        const float *tile = reinterpret_cast<const float *>(stage_of(it));
        uint8_t *const *dst = cur.op ? cur.I->pb : cur.I->pa;
#pragma unroll
        for (int pass = 0; pass < kPackRows * (kPackBK / 8) / 256; ++pass) {
            const int e = pass * 256 + tid;
            // 8 threads per row (coalesced 128-byte runs of pieces), 4 rows per warp
            const int r = e >> 3, c = e & 7;
            const int64_t row = cur.r0 + r;
            if (row >= cur.rows_alloc) continue;
            float x[8];
            if (!cur.transposed) {
                // the upper four threads read their second half first: no bank conflicts
                const int h = (c >> 2) & 1;
                const float4 u = *reinterpret_cast<const float4 *>(tile + r * kPackBK + c * 8 + 4 * h);
                const float4 v = *reinterpret_cast<const float4 *>(tile + r * kPackBK + c * 8 + 4 * (h ^ 1));
                const float4 lo = h ? v : u, hi = h ? u : v;
                x[0] = lo.x, x[1] = lo.y, x[2] = lo.z, x[3] = lo.w, x[4] = hi.x, x[5] = hi.y, x[6] = hi.z, x[7] = hi.w;
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int k = c * 8 + j;  // (k >> 3) & 7 == c
                    x[j] = tile[k * kPackRows + ((((r >> 2) ^ c) << 2) | (r & 3))];
                }
            }
            __nv_bfloat16 pcs[8][3];
#pragma unroll
            for (int j = 0; j < 8; ++j) tcg::split_value<NP>(x[j], pcs[j]);
            const int64_t off = packed_offset(row, cur.kb, c, cur.tr, cur.I->kt);
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                uint32_t w[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    __nv_bfloat162 v = __halves2bfloat162(pcs[2 * j][i], pcs[2 * j + 1][i]);
                    w[j] = *reinterpret_cast<uint32_t *>(&v);
                }
                *reinterpret_cast<uint4 *>(dst[i] + off) = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
        __syncthreads();  // this stage is read: the next issue may refill it
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// persistent contraction
// ---------------------------------------------------------------------------
struct Params {
    const TileRec *tiles;
    const int32_t *cta_start;  // tiles of CTA (pair kernel: cluster) b: [cta_start[b], cta_start[b+1])
    int seg_kblocks;
    int *fault;
};

// PAIR: a cluster of two CTAs runs 256 x bn tiles (an instance's row blocks
// in pairs), the leader issuing cta_group::2 MMAs (M = 256) on both CTAs'
// shared memory: each CTA stages its own 128-row A tile and half of the B
// tile's rows, so at bn = 256 a CTA moves a third fewer operand bytes per MMA
// than on a single-CTA 128 x 256 tile.
// Each CTA's copies complete on its own barrier; the peer's warp 1 relays
// every landed stage to the leader's barrier, which the MMA issuer waits on.
// The leader's MMAs commit to both CTAs' ring and accumulator barriers; both
// CTAs' drain warps (each on its own 128 rows of TMEM) arrive on the leader's.
//
// VEC: every instance's C takes 8-byte vector accesses (even N and ldc, C
// 8-byte aligned), so the epilogue is built without its scalar path.  That
// path, even never taken, costs the epilogue registers and instruction
// fetch: the contraction of the 1024-instance mix ran 2.08 ms (BF16) with
// it and 1.67 ms without.
template <int MODE, bool PAIR, bool VEC>
__global__ void __launch_bounds__(kThreads, 1) grouped_gemm_kernel(Params p) {
    using L = GLayoutOf<MODE, PAIR>;
    using MD = tcg::Mode<MODE>;
    constexpr int S = L::STAGES;
    static_assert(L::BK == kBK, "grouped engine stages BF16 slices of kBK");
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[S], empty[S], tfull[2], tempty[2], mma_done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    __shared__ int ring_issued, ring_consumed, mma_aborted;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = PAIR ? tc::cluster_ctarank() : 0u;
    const bool leader = rank == 0;
    const int unit = PAIR ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
    const int t_begin = p.cta_start[unit], t_end = p.cta_start[unit + 1];
    auto wait = [&](uint64_t *bar, uint32_t parity, uint64_t limit) {
        return PAIR ? tc::wait_timed_cluster(bar, parity, limit, &abort_flag)
                    : tc::wait_timed(bar, parity, limit, &abort_flag);
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            // the leader's stage completes on its own copies and the peer's relay
            mbar_init(&full[s], PAIR && leader ? 2 : 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], (PAIR ? 2 : 1) * kDrainWarps);
        }
        mbar_init(&mma_done, 1);
        fence_mbarrier_init();
        abort_flag = 0;
        ring_issued = ring_consumed = 0;
        mma_aborted = 0;
    }
    if (warp == 0) {
        if constexpr (PAIR) {
            tc::tmem_alloc_pair(&tmem_base, kTmemCols);
            tc::tmem_relinquish_pair();
        } else {
            tc::tmem_alloc(&tmem_base, kTmemCols);
            tc::tmem_relinquish();
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if constexpr (PAIR) tc::cluster_sync();  // both CTAs' barriers exist before any signal crosses the pair
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;

    auto a_tile = [&](int s, int piece) { return smem + s * L::STAGE_BYTES + piece * L::A_TILE; };
    auto b_tile = [&](int s, int piece) { return smem + s * L::STAGE_BYTES + MD::NP * L::A_TILE + piece * L::B_TILE; };

    if (warp == 0) {
        if (lane == 0) {
            // ---- producer: one bulk copy per piece tile ----
            int ring = 0;
            bool stop = false;
            TileRec cur;
            if (t_begin < t_end) cur = p.tiles[t_begin];
            for (int t = t_begin; t < t_end && !stop; ++t) {
                // the next record loads while this tile's copies are issued
                const TileRec next = p.tiles[t + 1 < t_end ? t + 1 : t];
                // a slice of the B tile is bn rows, and a pair CTA copies its half of
                // them; rank 1's A tile is the next row block, or (in a tile of 128
                // rows or fewer) rank 0's again, whose products are never stored
                const uint32_t b_slice = (uint32_t)cur.bn * kRowBytes;
                const uint32_t b_bytes = PAIR ? b_slice / 2 : b_slice;
                const int64_t a_off = (PAIR && rank == 1 && cur.rows > BM) ? (int64_t)cur.kt * kATileBytes : 0;
                const int64_t b_off = PAIR ? (int64_t)rank * b_bytes : 0;
                for (int kb = 0; kb < cur.kt; ++kb, ++ring) {
                    const int s = ring % S;
                    if (!wait(&empty[s], ((uint32_t)(ring / S) & 1u) ^ 1u, kWaitNs)) {
                        if (!abort_flag) report_fault(p.fault, kFaultTcProducerWait);
                        abort_flag = 1;
                        stop = true;
                        break;
                    }
                    mbar_arrive_expect_tx(&full[s], MD::NP * (kATileBytes + b_bytes));
                    for (int i = 0; i < MD::NP; ++i) {
                        bulk_g2s(a_tile(s, i), cur.a[i] + a_off + (int64_t)kb * kATileBytes, kATileBytes, &full[s]);
                        bulk_g2s(b_tile(s, i), cur.b[i] + b_off + (int64_t)kb * b_slice, b_bytes, &full[s]);
                    }
                }
                cur = next;
            }
            ring_issued = ring;
        }
        __syncwarp();
    } else if (warp == 1) {
        if (PAIR && !leader && lane == 0) {
            // ---- relay: each landed stage of this CTA, to the leader's barrier ----
            const uint32_t full_leader = tc::mapa_shared(smem_u32(&full[0]), 0);
            int ring = 0;
            bool stop = false;
            for (int t = t_begin; t < t_end && !stop; ++t) {
                const int kt = p.tiles[t].kt;
                for (int kb = 0; kb < kt; ++kb, ++ring) {
                    const int s = ring % S;
                    if (!wait(&full[s], (uint32_t)(ring / S) & 1u, kWaitNs)) {
                        if (!abort_flag) report_fault(p.fault, kFaultTcProducerWait);
                        abort_flag = 1;
                        stop = true;
                        break;
                    }
                    tc::mbar_arrive_remote(full_leader + (uint32_t)(s * sizeof(uint64_t)));
                }
            }
        } else if (lane == 0) {
            // ---- MMA issuer ----
            const uint32_t empty_self = PAIR ? tc::mapa_shared(smem_u32(&empty[0]), 0) : 0u;
            const uint32_t empty_peer = PAIR ? tc::mapa_shared(smem_u32(&empty[0]), 1) : 0u;
            const uint32_t tfull_self = PAIR ? tc::mapa_shared(smem_u32(&tfull[0]), 0) : 0u;
            const uint32_t tfull_peer = PAIR ? tc::mapa_shared(smem_u32(&tfull[0]), 1) : 0u;
            int ring = 0, seg = 0;
            bool stop = false;
            int2 cur = make_int2(0, 0);  // (kt, bn)
            if (t_begin < t_end) cur = make_int2(p.tiles[t_begin].kt, p.tiles[t_begin].bn);
            for (int t = t_begin; t < t_end && !stop; ++t) {
                const int tn = t + 1 < t_end ? t + 1 : t;
                const int2 next = make_int2(p.tiles[tn].kt, p.tiles[tn].bn);
                const int kt = cur.x;
                const uint32_t idesc = tc::idesc_bf16_f32(PAIR ? 2 * BM : BM, cur.y);
                cur = next;
                for (int kb = 0; kb < kt; ++kb, ++ring) {
                    const int b = seg & 1;
                    const bool seg_first = (kb % p.seg_kblocks) == 0;
                    const bool seg_last = (kb % p.seg_kblocks) == p.seg_kblocks - 1 || kb == kt - 1;
                    if (seg_first) {
                        if (!wait(&tempty[b], ((uint32_t)(seg >> 1) & 1u) ^ 1u, kWaitNs)) {
                            if (!abort_flag) report_fault(p.fault, kFaultTcMmaWait);
                            abort_flag = 1;
                            stop = true;
                            break;
                        }
                        tc::fence_after_sync();
                    }
                    const int s = ring % S;
                    if (!wait(&full[s], (uint32_t)(ring / S) & 1u, kWaitNs)) {
                        if (!abort_flag) report_fault(p.fault, kFaultTcMmaWait);
                        abort_flag = 1;
                        stop = true;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint32_t d = tmem + (uint32_t)(b * 256);
#pragma unroll
                    for (int kk = 0; kk < L::KSTEPS; ++kk) {
#pragma unroll
                        for (int j = 0; j < MD::NPROD; ++j) {
                            const uint32_t a_addr = smem_u32(a_tile(s, MD::pa(j))) + kk * 32;
                            const uint32_t b_addr = smem_u32(b_tile(s, MD::pb(j))) + kk * 32;
                            const uint64_t ad = tc::smem_desc_kmajor(a_addr, L::SBO, L::SWIZZLE);
                            const uint64_t bd = tc::smem_desc_kmajor(b_addr, L::SBO, L::SWIZZLE);
                            const uint32_t accum = (seg_first && kk == 0 && j == 0) ? 0u : 1u;
                            if constexpr (PAIR) tc::mma_bf16_pair(d, ad, bd, idesc, accum);
                            else tc::mma_bf16(d, ad, bd, idesc, accum);
                        }
                    }
                    if constexpr (PAIR) {
                        const uint32_t so = (uint32_t)(s * sizeof(uint64_t)), bo = (uint32_t)(b * sizeof(uint64_t));
                        tc::commit_pair_to(empty_self + so);
                        tc::commit_pair_to(empty_peer + so);
                        if (seg_last) {
                            tc::commit_pair_to(tfull_self + bo);
                            tc::commit_pair_to(tfull_peer + bo);
                        }
                    } else {
                        tc::commit_to(&empty[s]);
                        if (seg_last) tc::commit_to(&tfull[b]);
                    }
                    if (seg_last) ++seg;
                }
            }
            ring_consumed = ring;
            if (stop) {
                // every MMA issued before the abort completes before TMEM is freed
                mma_aborted = 1;
                if constexpr (PAIR) tc::commit_pair_to(tc::mapa_shared(smem_u32(&mma_done), 0));
                else tc::commit_to(&mma_done);
            }
        }
        __syncwarp();
    } else {
        // ---- drain + epilogue ----
        const int quarter = warp & 3, part = (warp - 2) >> 2;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        const int row_off = PAIR ? (int)rank * 128 : 0;  // a pair CTA's rows of the 256-row tile
        const uint32_t tempty_leader = PAIR ? tc::mapa_shared(smem_u32(&tempty[0]), 0) : 0u;
        int seg = 0;
        bool ok = true;
        for (int t = t_begin; t < t_end && ok; ++t) {
            const TileRec *R = p.tiles + t;
            const int bn = R->bn, kt = R->kt;
            const int hw = bn / kDrainParts;   // columns of this warp's part of the tile
            const int nseg = (kt + p.seg_kblocks - 1) / p.seg_kblocks;
            // Accumulator fragments in the 16x256b layout: for row slab rs (TMEM
            // lanes 16*rs .. 16*rs+15 of this warp's quarter) and column group
            // cg (8 columns), acc[(rs*kPartGroups + cg)*4 + e] holds row
            // 16*rs + lane/4 (e = 0, 1) or 16*rs + lane/4 + 8 (e = 2, 3), column
            // 8*cg + 2*(lane%4) + (e & 1) of this warp's part of the tile.  Four
            // neighbouring lanes then hold 32 contiguous bytes of one row of C,
            // so each store request covers whole sectors of eight rows.
            float acc[kAccRegs];
#pragma unroll
            for (int j = 0; j < kAccRegs; ++j) acc[j] = 0.0f;
            const int ngroups = hw >> 3;         // 8-column groups of this warp's part: 2 to kPartGroups
            {
                // C is read by the epilogue (beta != 0): pull this warp's rows
                // of it into L2 while the tile's MMAs run
                const int r = row_off + quarter * 32 + lane;
                if (R->gemm && R->beta != 0.0f && r < R->rows) {
                    const int left = R->cols - part * hw;
                    const int ncols = left < hw ? left : hw;
                    const char *row = reinterpret_cast<const char *>(R->C + (int64_t)r * R->ldc + part * hw);
                    for (int off = 0; off < ncols * 4; off += 128)
                        asm volatile("prefetch.global.L2 [%0];" ::"l"(row + off));
                }
            }
            for (int sg = 0; sg < nseg; ++sg, ++seg) {
                const int b = seg & 1;
                if (!wait(&tfull[b], (uint32_t)(seg >> 1) & 1u, 2 * kWaitNs)) {
                    if (!abort_flag) report_fault(p.fault, kFaultTcEpilogueWait);
                    abort_flag = 1;
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                const uint32_t col_base = tmem + lane_base + (uint32_t)(b * 256 + part * hw);
#pragma unroll
                for (int rs = 0; rs < 2; ++rs) {
                    const uint32_t slab = col_base + ((uint32_t)(rs * 16) << 16);
                    if (ngroups >= 4) {
#pragma unroll
                        for (int c = 0; c < kPartGroups / 4; ++c) {   // 32 columns per load
                            if (c * 4 < ngroups) {
                                uint32_t r[16];
                                tc::tmem_ld_16x256b_x4(slab + (uint32_t)(c * 32), r);
                                tc::tmem_ld_wait();
#pragma unroll
                                for (int j = 0; j < 16; ++j) {
                                    const int idx = (rs * kPartGroups + c * 4) * 4 + j;
                                    acc[idx] = __fadd_rn(acc[idx], __uint_as_float(r[j]));
                                }
                            }
                        }
                    } else {   // a 16-column part (64-wide tiles split four ways)
                        uint32_t r[8];
                        tc::tmem_ld_16x256b_x2(slab, r);
                        tc::tmem_ld_wait();
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const int idx = rs * kPartGroups * 4 + j;
                            acc[idx] = __fadd_rn(acc[idx], __uint_as_float(r[j]));
                        }
                    }
                }
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) {
                    if (!PAIR || leader) mbar_arrive(&tempty[b]);
                    else tc::mbar_arrive_remote(tempty_leader + (uint32_t)(b * sizeof(uint64_t)));
                }
            }
            if (!ok || abort_flag) break;
            const int left = R->cols - part * hw;
            const int ncols = left < hw ? left : hw;  // valid columns of this part
            const bool gemm = R->gemm != 0;
            const float alpha = R->alpha, beta = gemm ? R->beta : 0.0f;
            const bool vec_ok = ((R->ldc & 1) == 0) && ((reinterpret_cast<uintptr_t>(R->C) & 7) == 0) &&
                                ((part * hw) % 2 == 0);
            const int cl = 2 * (lane & 3);
#pragma unroll
            for (int rs = 0; rs < 2; ++rs) {
#pragma unroll
                for (int rr = 0; rr < 2; ++rr) {
                    const int row = row_off + quarter * 32 + rs * 16 + (lane >> 2) + 8 * rr;
                    if (row >= R->rows) continue;
                    float *cp = R->C + (int64_t)row * R->ldc + part * hw;
                    // kEpiBatch 8-column groups at a time: their loads of C
                    // (beta != 0) are issued together, then their stores
#pragma unroll
                    for (int g0 = 0; g0 < kPartGroups; g0 += kEpiBatch) {
                        if (g0 >= ngroups) break;
                        float2 c2[kEpiBatch];
#pragma unroll
                        for (int q = 0; q < kEpiBatch; ++q) {
                            const int col = (g0 + q) * 8 + cl;
                            c2[q] = make_float2(0.0f, 0.0f);
                            if (beta != 0.0f && vec_ok && col + 1 < ncols)
                                c2[q] = *reinterpret_cast<const float2 *>(cp + col);
                        }
#pragma unroll
                        for (int q = 0; q < kEpiBatch; ++q) {
                            const int col = (g0 + q) * 8 + cl;
                            const int idx = (rs * kPartGroups + g0 + q) * 4 + 2 * rr;
                            if (col >= ncols) continue;
                            if (vec_ok && col + 1 < ncols) {
                                float2 v;
                                v.x = gemm ? __fmaf_rn(alpha, acc[idx], beta == 0.0f ? 0.0f : beta * c2[q].x)
                                           : acc[idx];
                                v.y = gemm ? __fmaf_rn(alpha, acc[idx + 1], beta == 0.0f ? 0.0f : beta * c2[q].y)
                                           : acc[idx + 1];
                                *reinterpret_cast<float2 *>(cp + col) = v;
                            } else if constexpr (!VEC) {
#pragma unroll
                                for (int e = 0; e < 2; ++e) {
                                    if (col + e < ncols) {
                                        const float bc = beta == 0.0f ? 0.0f : beta * cp[col + e];
                                        cp[col + e] = gemm ? __fmaf_rn(alpha, acc[idx + e], bc) : acc[idx + e];
                                    }
                                }
                            }
                        }
                    }
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0 && abort_flag) {
        if constexpr (PAIR) {
            // a pair's stages complete on two CTAs' barriers: give every copy in
            // flight time to land (microseconds), then the MMAs issued before the abort
            const uint64_t t0 = tc::globaltimer();
            while (tc::globaltimer() - t0 < 20000000ull) {
            }
            if (leader && mma_aborted) tc::wait_timed(&mma_done, 0, kWaitNs, nullptr);
        } else {
            // bounded waits for the copies still landing and the MMAs issued before the abort
            for (int r = ring_consumed; r < ring_issued; ++r)
                tc::wait_timed(&full[r % S], (uint32_t)(r / S) & 1u, kWaitNs, nullptr);
            if (mma_aborted) tc::wait_timed(&mma_done, 0, kWaitNs, nullptr);
        }
    }
    __syncthreads();
    if constexpr (PAIR) {
        tc::cluster_sync();  // neither CTA leaves while the pair can still touch its memory
        if (warp == 0) tc::tmem_dealloc_pair(tmem, kTmemCols);
    } else {
        if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
    }
}

}  // namespace grp

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

std::mutex g_table_mu;
// per-bucket tile width, indexed [engine is split3][bucket]
int32_t g_tile_table[2][kGroupedBuckets] = {{64, 128, 256, 256}, {64, 128, 256, 256}};

int engine_slot(int engine) { return engine == GATLAS_ENGINE_TC_SPLIT3 ? 1 : 0; }

std::atomic<int> g_pair_mode{0};

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

int32_t grouped_bucket(int64_t m, int64_t n, int64_t k) {
    (void)m;
    (void)k;
    if (n <= 64) return 0;
    if (n <= 128) return 1;
    if (n <= 256) return 2;
    return 3;
}

int grouped_set_pair(int mode) {
    if (mode < 0 || mode > 1) return set_error(GATLAS_ERR_INVALID, "grouped_pair: %d (0 single CTAs, 1 CTA pairs)", mode);
    g_pair_mode.store(mode);
    return GATLAS_OK;
}

int grouped_get_pair() { return g_pair_mode.load(); }

// Clusters of two that fit at once (occupancy query, once per device).
template <int MODE>
static int pair_units_cap() {
    static thread_local int cap_dev = -1, cap = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (cap_dev != dev) {
        auto kern = grp::grouped_gemm_kernel<MODE, true, false>;
        cap = sm_count() / 2;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)grp::GLayoutOf<MODE, true>::SMEM_BYTES) == cudaSuccess) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = 2;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(2 * (unsigned)cap, 1, 1);
            cfg.blockDim = dim3(grp::kThreads, 1, 1);
            cfg.dynamicSmemBytes = grp::GLayoutOf<MODE, true>::SMEM_BYTES;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int n = 0;
            if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) == cudaSuccess && n > 0) cap = n;
        }
        cudaGetLastError();
        cap_dev = dev;
    }
    return std::max(cap, 1);
}

int grouped_set_tile_table(int engine, const int32_t *t, int32_t nb) {
    if (engine != GATLAS_ENGINE_TC_BF16 && engine != GATLAS_ENGINE_TC_SPLIT3)
        return set_error(GATLAS_ERR_UNSUPPORTED, "grouped: engine %d has no grouped kernel", engine);
    if (!t || nb != kGroupedBuckets) return set_error(GATLAS_ERR_INVALID, "grouped: tile table needs %d entries", kGroupedBuckets);
    for (int i = 0; i < nb; ++i)
        if (t[i] != 64 && t[i] != 128 && t[i] != 256) return set_error(GATLAS_ERR_INVALID, "grouped: tile width %d", t[i]);
    std::lock_guard<std::mutex> lk(g_table_mu);
    for (int i = 0; i < nb; ++i) g_tile_table[engine_slot(engine)][i] = t[i];
    return GATLAS_OK;
}

int grouped_get_tile_table(int engine, int32_t *t, int32_t nb) {
    if (engine != GATLAS_ENGINE_TC_BF16 && engine != GATLAS_ENGINE_TC_SPLIT3)
        return set_error(GATLAS_ERR_UNSUPPORTED, "grouped: engine %d has no grouped kernel", engine);
    if (!t || nb != kGroupedBuckets) return set_error(GATLAS_ERR_INVALID, "grouped: tile table needs %d entries", kGroupedBuckets);
    std::lock_guard<std::mutex> lk(g_table_mu);
    for (int i = 0; i < nb; ++i) t[i] = g_tile_table[engine_slot(engine)][i];
    return GATLAS_OK;
}

static int resolve_instance(const gatlas_grouped_instance &in, int slot, InstPlan *o) {
    if (in.m < 0 || in.n < 0 || in.k < 0) return set_error(GATLAS_ERR_INVALID, "grouped: negative dimension");
    o->M = in.m, o->N = in.n, o->K = in.k;
    const int64_t a_inner = in.trans_a ? in.m : in.k, b_inner = in.trans_b ? in.k : in.n;
    o->lda = in.lda ? in.lda : std::max<int64_t>(a_inner, 1);
    o->ldb = in.ldb ? in.ldb : std::max<int64_t>(b_inner, 1);
    o->ldc = in.ldc ? in.ldc : std::max<int64_t>(in.n, 1);
    if (o->lda < a_inner || o->ldb < b_inner || o->ldc < in.n)
        return set_error(GATLAS_ERR_INVALID, "grouped: leading dimension below the stored row length");
    int bn = in.tile_n;
    if (bn == 0) {
        std::lock_guard<std::mutex> lk(g_table_mu);
        bn = g_tile_table[slot][grouped_bucket(in.m, in.n, in.k)];
    }
    if (bn != 64 && bn != 128 && bn != 256) return set_error(GATLAS_ERR_INVALID, "grouped: tile width %d", bn);
    o->bn = bn;
    o->mt = (int)((in.m + grp::BM - 1) / grp::BM);
    o->nt = (int)((in.n + bn - 1) / bn);
    o->kt = (int)((in.k + grp::kPackBK - 1) / grp::kPackBK);
    if (in.m == 0 || in.n == 0) o->mt = o->nt = 0;
    if (o->mt > 65535 || o->kt > (1 << 24)) return set_error(GATLAS_ERR_INVALID, "grouped: instance too large");
    o->a_piece = round_up((size_t)o->mt * o->kt * grp::BM * grp::kPackRowBytes, 1024);
    o->b_piece = round_up((size_t)o->nt * o->kt * bn * grp::kPackRowBytes, 1024);
    return GATLAS_OK;
}

static bool grouped_engine_ok(int engine) {
    return engine == GATLAS_ENGINE_TC_BF16 || engine == GATLAS_ENGINE_TC_SPLIT3;
}

int grouped_instance_bytes(int engine, const gatlas_grouped_instance &in, size_t *bytes) {
    if (!grouped_engine_ok(engine))
        return set_error(GATLAS_ERR_UNSUPPORTED, "grouped: engine %d has no grouped kernel (tc_bf16, tc_split3)", engine);
    InstPlan o{};
    const int rc = resolve_instance(in, engine_slot(engine), &o);
    if (rc) return rc;
    const int np = engine == GATLAS_ENGINE_TC_SPLIT3 ? 2 : 1;
    *bytes = np * (o.a_piece + o.b_piece);
    return GATLAS_OK;
}

int grouped_build(int engine, const gatlas_grouped_instance *in, int32_t count, uint8_t *base,
                  uint8_t *const *packed, GroupedTables *t) {
    if (!grouped_engine_ok(engine))
        return set_error(GATLAS_ERR_UNSUPPORTED, "grouped: engine %d has no grouped kernel (tc_bf16, tc_split3)", engine);
    if (count < 0 || (count > 0 && !in)) return set_error(GATLAS_ERR_INVALID, "grouped: invalid instance list");
    t->engine = engine;
    t->np = engine == GATLAS_ENGINE_TC_SPLIT3 ? 2 : 1;
    t->mode = engine == GATLAS_ENGINE_TC_SPLIT3 ? 1 : 0;
    t->ip.assign(count, InstPlan{});
    t->inst.assign(std::max(count, 1), grp::Inst{});
    t->seg.assign(2 * (size_t)count + 1, 0);
    t->flops = 0;
    t->packed_bytes = 0;
    struct Cand {
        int64_t cost;
        grp::TileRec r;
    };
    std::vector<Cand> cands;
    for (int i = 0; i < count; ++i) {
        int rc = resolve_instance(in[i], engine_slot(engine), &t->ip[i]);
        if (rc) return rc;
    }
    t->pair = g_pair_mode.load() == 1;
    // the vector-only epilogue serves the launch when every C takes 8-byte
    // accesses: even N and ldc, 8-byte aligned base
    t->vec = true;
    for (int i = 0; i < count; ++i)
        if (in[i].m > 0 && in[i].n > 0)
            t->vec = t->vec && (t->ip[i].N % 2 == 0) && (t->ip[i].ldc % 2 == 0) &&
                     ((reinterpret_cast<uintptr_t>(in[i].c) & 7) == 0);
    const int step_m = t->pair ? 2 : 1;
    size_t off = 0;
    for (int i = 0; i < count; ++i) {
        InstPlan &o = t->ip[i];
        const gatlas_grouped_instance &q = in[i];
        if (q.m > 0 && q.n > 0 && (!q.c || (q.k > 0 && (!q.a || !q.b))))
            return set_error(GATLAS_ERR_INVALID, "grouped: instance %d has a null pointer", i);
        uint8_t *pb = packed ? packed[i] : (base ? base + off : nullptr);
        off += t->np * (o.a_piece + o.b_piece);
        t->packed_bytes += t->np * (o.a_piece + o.b_piece);
        t->flops += 2.0 * (double)q.m * (double)q.n * (double)q.k;
        grp::Inst &I = t->inst[i];
        std::memset(&I, 0, sizeof(I));
        I.src_a = q.a;
        I.src_b = q.b;
        for (int j = 0; j < t->np && pb; ++j) {
            I.pa[j] = pb + j * o.a_piece;
            I.pb[j] = pb + t->np * o.a_piece + j * o.b_piece;
        }
        I.C = q.c;
        I.M = o.M, I.N = o.N, I.K = o.K, I.lda = o.lda, I.ldb = o.ldb, I.ldc = o.ldc;
        I.ta = q.trans_a != 0, I.tb = q.trans_b != 0, I.gemm = q.gemm != 0;
        I.bn = o.bn, I.mt = o.mt, I.nt = o.nt, I.kt = o.kt;
        I.alpha = (float)q.alpha;
        I.beta = (float)q.beta;
        const int64_t a_items = o.kt ? (int64_t)o.mt * o.kt : 0;  // 128 A rows per item = one A tile row block
        const int64_t b_items = o.kt ? ((int64_t)o.nt * o.bn + grp::kPackRows - 1) / grp::kPackRows * o.kt : 0;
        t->seg[2 * i + 1] = t->seg[2 * i] + a_items;
        t->seg[2 * i + 2] = t->seg[2 * i + 1] + b_items;
        // cost in bytes moved: operand tiles through shared memory plus the C
        // tile (read too when beta != 0), plus a fixed per-tile overhead
        // (a pair tile: both CTAs' halves, as one unit of its cluster's time)
        const int64_t c_bytes = (int64_t)step_m * grp::BM * o.bn * 4 * ((q.gemm && q.beta != 0.0) ? 2 : 1);
        const int64_t cost = (int64_t)o.kt * t->np * (step_m * grp::BM + o.bn) * grp::kPackRowBytes + c_bytes + 16384;
        // grouped raster inside the instance: 16 tile rows per group, so the
        // tiles that run at the same time share A and B rows through L2
        for (int g0 = 0; g0 < o.mt; g0 += 16)
            for (int tn = 0; tn < o.nt; ++tn)
                for (int tm = g0; tm < std::min(o.mt, g0 + 16); tm += step_m) {
                grp::TileRec r;
                std::memset(&r, 0, sizeof(r));
                for (int j = 0; j < t->np && pb; ++j) {
                    r.a[j] = I.pa[j] + (size_t)tm * o.kt * grp::BM * grp::kPackRowBytes;
                    r.b[j] = I.pb[j] + (size_t)tn * o.kt * o.bn * grp::kPackRowBytes;
                }
                r.C = q.c + (int64_t)tm * grp::BM * o.ldc + (int64_t)tn * o.bn;
                r.ldc = o.ldc;
                r.kt = o.kt * grp::kSlicesPerItem;  // contraction K slices
                r.bn = o.bn;
                r.rows = (int32_t)std::min<int64_t>(step_m * grp::BM, o.M - (int64_t)tm * grp::BM);
                r.cols = (int32_t)std::min<int64_t>(o.bn, o.N - (int64_t)tn * o.bn);
                r.alpha = (float)q.alpha;
                r.beta = (float)q.beta;
                r.gemm = q.gemm != 0;
                cands.push_back(Cand{cost, r});
            }
    }
    t->nseg = 2 * count;
    t->nitems = t->seg.back();
    t->ntiles = (int64_t)cands.size();
    // longest first onto the least-loaded CTA
    std::stable_sort(cands.begin(), cands.end(), [](const Cand &a, const Cand &b) { return a.cost > b.cost; });
    const int units = t->pair ? (t->mode == 1 ? pair_units_cap<1>() : pair_units_cap<0>()) : sm_count();
    t->grid = (int)std::min<int64_t>(units, std::max<int64_t>(t->ntiles, 1));
    std::vector<int> owner(cands.size());
    std::vector<int32_t> count_per(t->grid, 0);
    {
        using E = std::pair<int64_t, int>;
        std::priority_queue<E, std::vector<E>, std::greater<E>> heap;
        for (int b = 0; b < t->grid; ++b) heap.push({0, b});
        for (size_t c = 0; c < cands.size(); ++c) {
            E e = heap.top();
            heap.pop();
            owner[c] = e.second;
            ++count_per[e.second];
            heap.push({e.first + cands[c].cost, e.second});
        }
    }
    t->cta.assign(t->grid + 1, 0);
    for (int b = 0; b < t->grid; ++b) t->cta[b + 1] = t->cta[b] + count_per[b];
    t->tiles.assign(std::max<size_t>(cands.size(), 1), grp::TileRec{});
    std::vector<int32_t> fill(t->cta.begin(), t->cta.end() - 1);
    for (size_t c = 0; c < cands.size(); ++c) t->tiles[fill[owner[c]]++] = cands[c].r;
    return GATLAS_OK;
}

// Shared-memory attribute of the pack kernels, once per device (also before
// a graph capture, since attribute changes are not captured).
static void grouped_pack_attributes() {
    static thread_local int attr_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_dev == dev) return;
    cudaFuncSetAttribute(grp::grouped_pack_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)grp::kPackSmemBytes);
    cudaFuncSetAttribute(grp::grouped_pack_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)grp::kPackSmemBytes);
    attr_dev = dev;
}

int grouped_launch_pack(const GroupedTables &t, const GroupedDevice &d, cudaStream_t stream) {
    if (t.nitems == 0) return GATLAS_OK;
    // two resident CTAs per SM (96 KiB of staging each), one item range per CTA
    grouped_pack_attributes();
    const int64_t grid = std::min<int64_t>(t.nitems, (int64_t)sm_count() * 2);
    const int64_t per_cta = (t.nitems + grid - 1) / grid;
    if (t.np == 2)
        grp::grouped_pack_kernel<2><<<(unsigned)grid, 256, grp::kPackSmemBytes, stream>>>(d.inst, d.seg, t.nseg,
                                                                                          per_cta);
    else
        grp::grouped_pack_kernel<1><<<(unsigned)grid, 256, grp::kPackSmemBytes, stream>>>(d.inst, d.seg, t.nseg,
                                                                                          per_cta);
    return check_launch("grouped_pack_kernel");
}

// Shared-memory attributes of the four contraction kernels, once per device
// (also before a graph capture, since attribute changes are not captured).
static int grouped_gemm_attributes() {
    static thread_local int attr_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_dev == dev) return GATLAS_OK;
    const cudaError_t e[8] = {
        cudaFuncSetAttribute(grp::grouped_gemm_kernel<0, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)grp::GLayoutOf<0, false>::SMEM_BYTES),
        cudaFuncSetAttribute(grp::grouped_gemm_kernel<1, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)grp::GLayoutOf<1, false>::SMEM_BYTES),
        cudaFuncSetAttribute(grp::grouped_gemm_kernel<0, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)grp::GLayoutOf<0, true>::SMEM_BYTES),
        cudaFuncSetAttribute(grp::grouped_gemm_kernel<1, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)grp::GLayoutOf<1, true>::SMEM_BYTES),
        cudaFuncSetAttribute(grp::grouped_gemm_kernel<0, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)grp::GLayoutOf<0, false>::SMEM_BYTES),
        cudaFuncSetAttribute(grp::grouped_gemm_kernel<1, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)grp::GLayoutOf<1, false>::SMEM_BYTES),
        cudaFuncSetAttribute(grp::grouped_gemm_kernel<0, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)grp::GLayoutOf<0, true>::SMEM_BYTES),
        cudaFuncSetAttribute(grp::grouped_gemm_kernel<1, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)grp::GLayoutOf<1, true>::SMEM_BYTES)};
    for (cudaError_t x : e)
        if (x != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "grouped smem attribute: %s", cudaGetErrorString(x));
    attr_dev = dev;
    return GATLAS_OK;
}

template <int MODE, bool PAIR, bool VEC>
static int launch_grouped(const GroupedTables &t, const GroupedDevice &d, cudaStream_t stream) {
    grp::Params prm;
    prm.tiles = d.tiles;
    prm.cta_start = d.cta;
    prm.seg_kblocks = grp::grouped_seg_kblocks(MODE);
    prm.fault = device_fault_word();
    const int rc = grouped_gemm_attributes();
    if (rc) return rc;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((PAIR ? 2 : 1) * t.grid), 1, 1);
    cfg.blockDim = dim3(grp::kThreads, 1, 1);
    cfg.dynamicSmemBytes = grp::GLayoutOf<MODE, PAIR>::SMEM_BYTES;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = PAIR ? 1 : 0;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, grp::grouped_gemm_kernel<MODE, PAIR, VEC>, prm);
    if (e != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "grouped_gemm_kernel: %s", cudaGetErrorString(e));
    return check_launch("grouped_gemm_kernel");
}

int grouped_launch_contract(const GroupedTables &t, const GroupedDevice &d, cudaStream_t stream) {
    if (t.ntiles == 0) return GATLAS_OK;
    if (t.vec) {
        if (t.pair)
            return t.mode == 1 ? launch_grouped<1, true, true>(t, d, stream) : launch_grouped<0, true, true>(t, d, stream);
        return t.mode == 1 ? launch_grouped<1, false, true>(t, d, stream) : launch_grouped<0, false, true>(t, d, stream);
    }
    if (t.pair)
        return t.mode == 1 ? launch_grouped<1, true, false>(t, d, stream) : launch_grouped<0, true, false>(t, d, stream);
    return t.mode == 1 ? launch_grouped<1, false, false>(t, d, stream) : launch_grouped<0, false, false>(t, d, stream);
}

struct GroupedPlan {
    int count = 0;
    std::vector<gatlas_grouped_instance> in;
    GroupedTables t;
    GroupedDevice d;
    void *dev_tables = nullptr;
    void *ws = nullptr;
    bool owns_ws = false;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
};

size_t grouped_workspace_bytes(int engine, const gatlas_grouped_instance *in, int32_t count) {
    if (!grouped_engine_ok(engine) || !in || count < 0) return 0;
    size_t total = 0;
    for (int i = 0; i < count; ++i) {
        size_t b = 0;
        if (grouped_instance_bytes(engine, in[i], &b)) return 0;
        total += b;
    }
    return total;
}

static void free_plan(GroupedPlan *p) {
    for (auto &g : p->graph)
        if (g) cudaGraphExecDestroy(g);
    cudaFree(p->dev_tables);
    if (p->owns_ws) cudaFree(p->ws);
    delete p;
}

// Byte layout of the device tables: [inst][seg][tiles][cta], 256-byte aligned parts.
static size_t table_layout(const GroupedTables &t, size_t off[4]) {
    const size_t sz[4] = {t.inst.size() * sizeof(grp::Inst), t.seg.size() * sizeof(int64_t),
                          t.tiles.size() * sizeof(grp::TileRec), t.cta.size() * sizeof(int32_t)};
    size_t o = 0;
    for (int i = 0; i < 4; ++i) {
        off[i] = o;
        o += round_up(sz[i], 256);
    }
    return o;
}

size_t grouped_tables_bytes(const GroupedTables &t) {
    size_t off[4];
    return table_layout(t, off);
}

void grouped_tables_serialise(const GroupedTables &t, void *host_dst) {
    size_t off[4];
    table_layout(t, off);
    uint8_t *h = static_cast<uint8_t *>(host_dst);
    std::memcpy(h + off[0], t.inst.data(), t.inst.size() * sizeof(grp::Inst));
    std::memcpy(h + off[1], t.seg.data(), t.seg.size() * sizeof(int64_t));
    std::memcpy(h + off[2], t.tiles.data(), t.tiles.size() * sizeof(grp::TileRec));
    std::memcpy(h + off[3], t.cta.data(), t.cta.size() * sizeof(int32_t));
}

GroupedDevice grouped_tables_device(const GroupedTables &t, const void *dev_base) {
    size_t off[4];
    table_layout(t, off);
    const uint8_t *b = static_cast<const uint8_t *>(dev_base);
    GroupedDevice d;
    d.inst = reinterpret_cast<const grp::Inst *>(b + off[0]);
    d.seg = reinterpret_cast<const int64_t *>(b + off[1]);
    d.tiles = reinterpret_cast<const grp::TileRec *>(b + off[2]);
    d.cta = reinterpret_cast<const int32_t *>(b + off[3]);
    return d;
}

int grouped_create(int engine, const gatlas_grouped_instance *in, int32_t count, void *ws, size_t ws_bytes,
                   GroupedPlan **out) {
    if (!out) return set_error(GATLAS_ERR_INVALID, "grouped: null plan pointer");
    *out = nullptr;
    GroupedPlan *p = new GroupedPlan();
    p->count = count;
    if (count > 0 && in) p->in.assign(in, in + count);
    // validate and size before any device work
    int rc = grouped_build(engine, in, count, nullptr, nullptr, &p->t);
    if (rc) {
        delete p;
        return rc;
    }
    const size_t total = p->t.packed_bytes;
    if (ws) {
        if (ws_bytes < total) {
            delete p;
            return set_error(GATLAS_ERR_INVALID, "grouped: workspace %zu < %zu bytes", ws_bytes, total);
        }
        if (!aligned_to(ws, 1024)) {
            delete p;
            return set_error(GATLAS_ERR_INVALID, "grouped: workspace must be 1024-byte aligned");
        }
        p->ws = ws;
    } else if (total) {
        if (cudaMalloc(&p->ws, total) != cudaSuccess) {
            cudaGetLastError();
            delete p;
            return set_error(GATLAS_ERR_NOMEM, "grouped: workspace of %zu bytes", total);
        }
        p->owns_ws = true;
    }
    rc = grouped_build(engine, in, count, static_cast<uint8_t *>(p->ws), nullptr, &p->t);
    if (rc) {
        free_plan(p);
        return rc;
    }
    const size_t tb = grouped_tables_bytes(p->t);
    std::vector<uint8_t> host(tb);
    grouped_tables_serialise(p->t, host.data());
    if (cudaMalloc(&p->dev_tables, tb) != cudaSuccess ||
        cudaMemcpy(p->dev_tables, host.data(), tb, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        free_plan(p);
        return set_error(GATLAS_ERR_NOMEM, "grouped: device tables");
    }
    p->d = grouped_tables_device(p->t, p->dev_tables);
    *out = p;
    return GATLAS_OK;
}

int grouped_prepare(GroupedPlan *p, cudaStream_t stream) {
    if (!p) return set_error(GATLAS_ERR_INVALID, "grouped: null plan");
    return grouped_launch_pack(p->t, p->d, stream);
}

int grouped_run(GroupedPlan *p, cudaStream_t stream) {
    if (!p) return set_error(GATLAS_ERR_INVALID, "grouped: null plan");
    return grouped_launch_contract(p->t, p->d, stream);
}

int grouped_launch_graph(GroupedPlan *p, int with_prepare, cudaStream_t stream) {
    if (!p) return set_error(GATLAS_ERR_INVALID, "grouped: null plan");
    const int slot = with_prepare ? 1 : 0;
    if (!p->graph[slot]) {
        cudaStream_t cap;
        if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
            return set_error(GATLAS_ERR_CUDA, "grouped: capture stream");
        // attribute changes are not captured: set them before the capture
        const int arc = grouped_gemm_attributes();
        if (arc) {
            cudaStreamDestroy(cap);
            return arc;
        }
        grouped_pack_attributes();
        device_fault_word();
        cudaGraph_t graph = nullptr;
        int rc = GATLAS_OK;
        if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaStreamDestroy(cap);
            return set_error(GATLAS_ERR_CUDA, "grouped: begin capture");
        }
        if (with_prepare) rc = grouped_prepare(p, cap);
        if (!rc) rc = grouped_run(p, cap);
        cudaError_t e = cudaStreamEndCapture(cap, &graph);
        cudaStreamDestroy(cap);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess || !graph) return set_error(GATLAS_ERR_CUDA, "grouped: end capture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&p->graph[slot], graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            p->graph[slot] = nullptr;
            return set_error(GATLAS_ERR_CUDA, "grouped: graph instantiate: %s", cudaGetErrorString(e));
        }
    }
    if (cudaGraphLaunch(p->graph[slot], stream) != cudaSuccess) return check_launch("grouped graph launch");
    return GATLAS_OK;
}

static gatlas_matmul_desc instance_desc(const GroupedPlan *p, int i) {
    const gatlas_grouped_instance &q = p->in[i];
    gatlas_matmul_desc d;
    std::memset(&d, 0, sizeof(d));
    d.engine = p->t.engine;
    d.gemm = q.gemm;
    d.trans_a = q.trans_a;
    d.trans_b = q.trans_b;
    d.m = q.m, d.n = q.n, d.k = q.k;
    d.lda = p->t.ip[i].lda, d.ldb = p->t.ip[i].ldb, d.ldc = p->t.ip[i].ldc;
    d.batch = 1;
    d.alpha = q.alpha;
    d.beta = q.beta;
    return d;
}

// The comparator: one engine call (split A, split B, contraction) per
// instance, through the library's scratch buffer, grown once up front.
int grouped_run_each(GroupedPlan *p, cudaStream_t stream) {
    if (!p) return set_error(GATLAS_ERR_INVALID, "grouped: null plan");
    size_t need = 0;
    for (int i = 0; i < p->count; ++i) {
        const gatlas_matmul_desc d = instance_desc(p, i);
        need = std::max(need, gatlas_matmul_workspace_size(&d));
    }
    if (need && !device_scratch(need)) return set_error(GATLAS_ERR_NOMEM, "grouped: scratch of %zu bytes", need);
    for (int i = 0; i < p->count; ++i) {
        const gatlas_grouped_instance &q = p->in[i];
        if (q.m == 0 || q.n == 0) continue;
        const gatlas_matmul_desc d = instance_desc(p, i);
        const int rc = gatlas_matmul_f32(&d, q.a, q.b, q.c, nullptr, 0, stream);
        if (rc) return rc;
    }
    return GATLAS_OK;
}

int grouped_info(const GroupedPlan *p, int64_t *tiles, int32_t *ctas, double *flops, int64_t *items) {
    if (!p) return set_error(GATLAS_ERR_INVALID, "grouped: null plan");
    if (tiles) *tiles = p->t.ntiles;
    if (ctas) *ctas = p->t.grid * (p->t.pair ? 2 : 1);
    if (flops) *flops = p->t.flops;
    if (items) *items = p->t.nitems;
    return GATLAS_OK;
}

void grouped_destroy(GroupedPlan *p) {
    if (p) free_plan(p);
}

}  // namespace gatlas

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

size_t gatlas_grouped_workspace_size(int engine, const gatlas_grouped_instance *inst, int32_t count) {
    return gatlas::grouped_workspace_bytes(engine, inst, count);
}

int gatlas_grouped_create(int engine, const gatlas_grouped_instance *inst, int32_t count, void *workspace,
                          size_t workspace_bytes, gatlas_grouped_plan **plan) {
    gatlas::clear_error();
    return gatlas::grouped_create(engine, inst, count, workspace, workspace_bytes,
                                  reinterpret_cast<gatlas::GroupedPlan **>(plan));
}

int gatlas_grouped_prepare(gatlas_grouped_plan *plan, void *stream) {
    gatlas::clear_error();
    return gatlas::grouped_prepare(reinterpret_cast<gatlas::GroupedPlan *>(plan), (cudaStream_t)stream);
}

int gatlas_grouped_run(gatlas_grouped_plan *plan, void *stream) {
    gatlas::clear_error();
    return gatlas::grouped_run(reinterpret_cast<gatlas::GroupedPlan *>(plan), (cudaStream_t)stream);
}

int gatlas_grouped_launch_graph(gatlas_grouped_plan *plan, int32_t with_prepare, void *stream) {
    gatlas::clear_error();
    return gatlas::grouped_launch_graph(reinterpret_cast<gatlas::GroupedPlan *>(plan), with_prepare,
                                        (cudaStream_t)stream);
}

int gatlas_grouped_run_each(gatlas_grouped_plan *plan, void *stream) {
    gatlas::clear_error();
    return gatlas::grouped_run_each(reinterpret_cast<gatlas::GroupedPlan *>(plan), (cudaStream_t)stream);
}

int gatlas_grouped_info(const gatlas_grouped_plan *plan, int64_t *tiles, int32_t *ctas, double *flops,
                        int64_t *pack_items) {
    gatlas::clear_error();
    return gatlas::grouped_info(reinterpret_cast<const gatlas::GroupedPlan *>(plan), tiles, ctas, flops, pack_items);
}

void gatlas_grouped_destroy(gatlas_grouped_plan *plan) {
    gatlas::grouped_destroy(reinterpret_cast<gatlas::GroupedPlan *>(plan));
}

int32_t gatlas_grouped_bucket(int64_t m, int64_t n, int64_t k) { return gatlas::grouped_bucket(m, n, k); }

int gatlas_grouped_set_tile_table(int engine, const int32_t *bucket_tile_n, int32_t nbuckets) {
    gatlas::clear_error();
    return gatlas::grouped_set_tile_table(engine, bucket_tile_n, nbuckets);
}

int gatlas_grouped_get_tile_table(int engine, int32_t *bucket_tile_n, int32_t nbuckets) {
    gatlas::clear_error();
    return gatlas::grouped_get_tile_table(engine, bucket_tile_n, nbuckets);
}

}  // extern "C"
