// Tensor-core (tcgen05) matmul engines: BF16 operands with FP32 accumulation,
// and FP32-accurate contractions of FP32 operands split into BF16 pieces.
//
// No reference counterpart: the reference's matmul kernels are SIMT mad
// chains (KernelMatmulBuffer.hpp:302-321).  These engines compute the same
// C = op(A)·op(B) (alpha/beta, packed batches, all four layouts) on the
// 5th-generation tensor cores:
//
//  1. split pass: every FP32 operand element x is split into BF16 pieces
//     (x = hi + lo + r with hi = bf16(x), lo = bf16(x - hi), |r| <= 2^-17|x|;
//     three pieces hi + mid + lo represent x exactly) written K-major
//     ([rows][Kp], Kp = K rounded up to 8, zero padded), transposing the
//     operands whose stored layout is not K-major;
//  2. contraction (BF16, split3, split6): a persistent kernel, one CTA per
//     SM over 128 x 256 tiles of C, or one cluster of two CTAs per SM pair
//     over 256 x 256 tiles (cta_group::2).  Warp 0 lane 0 streams K slices
//     of 128 bytes per row (64 BF16; 64 bytes for split6) of every piece
//     of A and B with 3-D TMA tensor-map loads (128-byte swizzle) into a
//     multi-stage mbarrier ring; warp 1 lane 0 issues tcgen05.mma kind::f16
//     (M = 128 or 256, N = 256, K = 16) for each product of pieces (hi*hi,
//     hi*lo, lo*hi for 3 products; the six leading products of three pieces
//     for 6), accumulating in FP32 in two TMEM buffers of 256 columns; eight
//     drain warps promote each segment into round-to-nearest FP32 registers
//     and, at the end of a tile, apply C = fma(alpha, acc, beta*C) and store
//     C through TMA while the next tile already runs.  FP8 E4M3 (per-block
//     scales) runs the same persistent kernel, on single CTAs or pairs, its
//     segments planned per tile by fp8_plan_kernel.
// Every mbarrier wait is bounded in wall time; a timeout sets the device
// fault word, stops the pipeline, drains the copies in flight and frees TMEM.
#include <cuda.h>

#include <algorithm>
#include <cstring>
#include <vector>
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include "../common.cuh"
#include "../device_state.cuh"
#include "../tcgen05.cuh"
#include "../tma.hpp"
#include "gemm_engines.hpp"
#include "grouped.hpp"
#include "tc_modes.cuh"

namespace gatlas {
namespace tcg {

constexpr int kGroupM = 16;  // tile rows per raster group (128-row tiles)
// Rows of C per raster group: 2048, i.e. 16 single-CTA or 8 pair tiles, so
// that the tiles in flight at once (one per SM) cover a near-square block of
// C whose A rows and B columns stay in L2.
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s bound on any single wait

struct Params {
    float *C;
    int64_t M, N, ldc, stride_c;
    int kblocks;
    int seg_kblocks;  // K slices accumulated in TMEM before promotion
    float alpha, beta;
    int gemm;
    int *fault;
    // FP8 only: block scales [batch][row blocks][kblocks] of A and of B
    const float *scale_a, *scale_b;
    int64_t scale_a_stride, scale_b_stride;  // per instance
    int nblocks_n;                           // 128-column blocks of N
    int nblocks_m;                           // 128-row blocks of M
    // persistent kernels: tiles per instance and instances; tma_store = 1
    // when C leaves through the C tensor map (beta == 0, 16-byte aligned)
    int tiles_m, tiles_n, batch;
    int tma_store;
    int group_tiles;  // tile rows per raster group
    // 1: A's loads evict-last in L2 (A is reused by every tile column of a
    // raster group, B by the group's tile rows at about the same time)
    int l2_hint;
    // FP8 persistent kernel: per tile (instance-major, then tile row, then
    // tile column) the segment count, one segment-start bit per 128-deep
    // block (plan_words words), and each segment's scale products of the
    // tile's two column halves (kblocks entries reserved per tile)
    const int *plan_nseg;
    const uint32_t *plan_bits;
    const float2 *plan_q;
    int plan_words;
};

// Warp roles: warp 0 = TMA producer (lane 0), warp 1 = MMA issuer (lane 0),
// warps 2..9 = accumulator drain + epilogue.  Drain warp w reads TMEM lane
// quarter (w % 4) and column half (w - 2) / 4.
constexpr int kDrainWarps = 8;
constexpr int kThreads2 = 32 * (2 + kDrainWarps);
constexpr uint32_t kTmemCols2 = 2 * BN;  // two accumulator buffers

// ---------------------------------------------------------------------------
// Persistent contraction: one CTA (or CTA pair) per SM walks
// the tiles t = unit, unit + units, ... in the grouped raster order.  The
// ring, the MMA issue and the TMEM double buffer run on across tile
// boundaries, so one tile's last promotions and its C stores overlap the
// next tile's loads and MMAs; each drain warp stages its 32 x 128 block of C
// through a 32 x 32 shared-memory tile (128-byte swizzle) and a TMA store,
// which also clips the tile at M and N.
// FP8 (MODE 3): segments follow the per-tile plan written by fp8_plan_kernel
// (runs of equally scaled 128-deep blocks); the MMA issuer reads its
// segment-start bits a 32-block word ahead, the drain scales each segment as
// it promotes it (on a pair, with the products of its own CTA's rows).
//
// PAIR (cta_group::2, one 256 x 256 tile per cluster of two CTAs):
// Each CTA streams 128 rows of A and its 128-row half of B per K slice
// (instead of 128 + 256 rows for a 128 x 256 tile), so the operand bytes
// moved from L2 per FLOP fall by a third and the ring gets deeper for the
// same shared memory.  Roles per CTA as in tc_gemm_persistent_kernel; only the leader
// (rank 0) issues MMAs, M = 256 split by rows across the two TMEMs.
// Barriers (no multicast forms anywhere):
//  * full[s] of the leader: both producers' TMA loads complete on it; the
//    leader's producer arrives once with the pair's byte count;
//  * empty[s] and tfull[b] of each CTA: the leader's MMA commits to its own
//    barrier and to the peer's;
//  * tempty[b] of the leader: 16 arrivals, the 8 drain warps of each CTA.
// Every wait is bounded; after an abort each CTA lets in-flight copies land
// before the closing cluster barrier, so neither CTA leaves while the pair's
// MMAs or copies can still touch its shared memory.
// ---------------------------------------------------------------------------
template <int MODE, bool PAIR>
__global__ void __launch_bounds__(kThreads2, 1)
    tc_gemm_persistent_kernel(const __grid_constant__ CUtensorMap ta0, const __grid_constant__ CUtensorMap ta1,
                              const __grid_constant__ CUtensorMap ta2, const __grid_constant__ CUtensorMap tb0,
                              const __grid_constant__ CUtensorMap tb1, const __grid_constant__ CUtensorMap tb2,
                              const __grid_constant__ CUtensorMap tcout, Params p) {
    using L = PersistentLayout<MODE, PAIR>;
    using MD = Mode<MODE>;
    constexpr int S = L::STAGES;
    constexpr int BK = L::BK;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[S], empty[S], tfull[2], tempty[2], mma_done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    __shared__ int mma_aborted;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = PAIR ? tc::cluster_ctarank() : 0u;
    const bool leader = rank == 0;
    const int unit = PAIR ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
    const int units = PAIR ? (int)(gridDim.x >> 1) : (int)gridDim.x;
    const int64_t per_batch = (int64_t)p.tiles_m * p.tiles_n;
    const int64_t total = per_batch * p.batch;
    const CUtensorMap *tA[3] = {&ta0, &ta1, &ta2};
    const CUtensorMap *tB[3] = {&tb0, &tb1, &tb2};

    // tile t -> (tile row, tile column, instance), grouped raster within an instance
    auto decode = [&](int64_t t, int &tm, int &tn, int &z) {
        z = (int)(t / per_batch);
        const int bid = (int)(t - (int64_t)z * per_batch);
        const int G = p.group_tiles;
        const int per_group = G * p.tiles_n;
        const int first_m = (bid / per_group) * G;
        const int gm = min(p.tiles_m - first_m, G);
        const int r = bid % per_group;
        tm = first_m + r % gm;
        tn = r / gm;
    };
    auto wait = [&](uint64_t *bar, uint32_t parity, uint64_t limit) {
        return PAIR ? tc::wait_timed_cluster(bar, parity, limit, &abort_flag)
                    : tc::wait_timed(bar, parity, limit, &abort_flag);
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], (PAIR ? 2 : 1) * kDrainWarps);
        }
        mbar_init(&mma_done, 1);
        fence_mbarrier_init();
        abort_flag = 0;
        mma_aborted = 0;
        for (int i = 0; i < MD::NP; ++i) {
            prefetch_tmap(tA[i]);
            prefetch_tmap(tB[i]);
        }
        if (p.tma_store) prefetch_tmap(&tcout);
    }
    if (warp == 0) {
        if constexpr (PAIR) {
            tc::tmem_alloc_pair(&tmem_base, kTmemCols2);
            tc::tmem_relinquish_pair();
        } else {
            tc::tmem_alloc(&tmem_base, kTmemCols2);
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
            // ---- TMA producer: one ring position per K slice, across tiles ----
            const uint32_t full_leader = PAIR ? tc::mapa_shared(smem_u32(&full[0]), 0) : 0u;
            const uint64_t pol_a = tc::l2_policy_evict_last();
            int s = 0;
            uint32_t ph = 0;
            bool stop = false;
            for (int64_t t = unit; t < total && !stop; t += units) {
                int tm, tn, z;
                decode(t, tm, tn, z);
                const int m0 = tm * L::TM + (int)rank * 128;
                const int nb = tn * BN + (int)rank * (PAIR ? 128 : 0);
                for (int kb = 0; kb < p.kblocks; ++kb) {
                    if (!wait(&empty[s], ph ^ 1u, kWaitNs)) {
                        if (!abort_flag) report_fault(p.fault, kFaultTcProducerWait);
                        abort_flag = 1;
                        stop = true;
                        break;
                    }
                    if constexpr (PAIR) {
                        if (leader) mbar_arrive_expect_tx(&full[s], 2 * L::STAGE_BYTES);
                        const uint32_t bar = full_leader + (uint32_t)(s * sizeof(uint64_t));
                        for (int i = 0; i < MD::NP; ++i) {
                            if (p.l2_hint) tc::tma_load_3d_pair_hint(a_tile(s, i), tA[i], kb * BK, m0, z, bar, pol_a);
                            else tc::tma_load_3d_pair(a_tile(s, i), tA[i], kb * BK, m0, z, bar);
                            tc::tma_load_3d_pair(b_tile(s, i), tB[i], kb * BK, nb, z, bar);
                        }
                    } else {
                        mbar_arrive_expect_tx(&full[s], L::STAGE_BYTES);
                        for (int i = 0; i < MD::NP; ++i) {
                            if (p.l2_hint) tc::tma_load_3d_hint(a_tile(s, i), tA[i], kb * BK, m0, z, &full[s], pol_a);
                            else tma_load_3d(a_tile(s, i), tA[i], kb * BK, m0, z, &full[s]);
                            tma_load_3d(b_tile(s, i), tB[i], kb * BK, nb, z, &full[s]);
                        }
                    }
                    if (++s == S) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0 && leader) {
            // ---- MMA issuer: segment g (counted across tiles) accumulates into TMEM buffer g & 1 ----
            constexpr uint32_t idesc = L::IDESC;
            const uint32_t empty_self = PAIR ? tc::mapa_shared(smem_u32(&empty[0]), 0) : 0u;
            const uint32_t empty_peer = PAIR ? tc::mapa_shared(smem_u32(&empty[0]), 1) : 0u;
            const uint32_t tfull_self = PAIR ? tc::mapa_shared(smem_u32(&tfull[0]), 0) : 0u;
            const uint32_t tfull_peer = PAIR ? tc::mapa_shared(smem_u32(&tfull[0]), 1) : 0u;
            int s = 0, seg = -1;
            uint32_t ph = 0;
            bool stop = false;
            for (int64_t t = unit; t < total && !stop; t += units) {
                const uint32_t *wb = nullptr;
                uint32_t wcur = 0, wnext = 0;
                if constexpr (MD::SCALED) {
                    int tm, tn, z;
                    decode(t, tm, tn, z);
                    wb = p.plan_bits + (((int64_t)z * p.tiles_m + tm) * p.tiles_n + tn) * p.plan_words;
                    wcur = __ldg(wb);
                    wnext = p.plan_words > 1 ? __ldg(wb + 1) : 0u;
                }
                for (int kb = 0; kb < p.kblocks; ++kb) {
                    bool seg_first, seg_last;
                    if constexpr (MD::SCALED) {
                        if (kb > 0 && (kb & 31) == 0) {  // next word; the one after it loads meanwhile
                            wcur = wnext;
                            wnext = (kb >> 5) + 1 < p.plan_words ? __ldg(wb + (kb >> 5) + 1) : 0u;
                        }
                        const int k1 = kb + 1;
                        seg_first = ((wcur >> (kb & 31)) & 1u) != 0;
                        seg_last = k1 == p.kblocks || (((k1 & 31) ? (wcur >> (k1 & 31)) : wnext) & 1u) != 0;
                    } else {
                        seg_first = (kb % p.seg_kblocks) == 0;
                        seg_last = (kb % p.seg_kblocks) == p.seg_kblocks - 1 || kb == p.kblocks - 1;
                    }
                    if (seg_first) ++seg;
                    const int b = seg & 1;
                    if (seg_first) {
                        // the drain of this buffer's previous segment (both CTAs' for a pair) is done
                        if (!wait(&tempty[b], ((uint32_t)(seg >> 1) & 1u) ^ 1u, kWaitNs)) {
                            if (!abort_flag) report_fault(p.fault, kFaultTcMmaWait);
                            abort_flag = 1;
                            stop = true;
                            break;
                        }
                        tc::fence_after_sync();
                    }
                    if (!wait(&full[s], ph, kWaitNs)) {
                        if (!abort_flag) report_fault(p.fault, kFaultTcMmaWait);
                        abort_flag = 1;
                        stop = true;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint32_t d = tmem + (uint32_t)(b * BN);
#pragma unroll
                    for (int kk = 0; kk < L::KSTEPS; ++kk) {
#pragma unroll
                        for (int j = 0; j < MD::NPROD; ++j) {
                            // 32 bytes of K per instruction inside the swizzled rows
                            const uint32_t a_addr = smem_u32(a_tile(s, MD::pa(j))) + kk * 32;
                            const uint32_t b_addr = smem_u32(b_tile(s, MD::pb(j))) + kk * 32;
                            const uint64_t ad = tc::smem_desc_kmajor(a_addr, L::SBO, L::SWIZZLE);
                            const uint64_t bd = tc::smem_desc_kmajor(b_addr, L::SBO, L::SWIZZLE);
                            const uint32_t accum = (seg_first && kk == 0 && j == 0) ? 0u : 1u;
                            if constexpr (MD::SCALED && PAIR) tc::mma_f8_pair(d, ad, bd, idesc, accum);
                            else if constexpr (MD::SCALED) tc::mma_f8(d, ad, bd, idesc, accum);
                            else if constexpr (PAIR) tc::mma_bf16_pair(d, ad, bd, idesc, accum);
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
                    if (++s == S) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
            if (stop) {
                // every MMA issued before the abort completes before TMEM is freed
                mma_aborted = 1;
                if constexpr (PAIR) tc::commit_pair_to(tc::mapa_shared(smem_u32(&mma_done), 0));
                else tc::commit_to(&mma_done);
            }
        }
        __syncwarp();
    } else {
        // ---- drain: promote each segment into round-to-nearest FP32 sums; then C ----
        const int quarter = warp & 3, half = (warp - 2) >> 2;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        const uint32_t tempty_leader = PAIR ? tc::mapa_shared(smem_u32(&tempty[0]), 0) : 0u;
        uint8_t *stage = smem + L::EPI_OFFSET + (warp - 2) * kEpiTileBytes;
        const int nseg = (p.kblocks + p.seg_kblocks - 1) / p.seg_kblocks;
        const bool vec_ok = (p.ldc % 4 == 0) && ((reinterpret_cast<uintptr_t>(p.C) & 15) == 0) && (p.stride_c % 4 == 0);
        int seg = -1;
        bool ok = true;
        for (int64_t t = unit; t < total && ok; t += units) {
            int tm, tn, z;
            decode(t, tm, tn, z);
            const int64_t m0 = (int64_t)tm * L::TM + (int64_t)rank * 128;
            const int64_t n0 = (int64_t)tn * BN;
            int tile_nseg = nseg;
            const float2 *tile_q = nullptr;
            if constexpr (MD::SCALED) {
                const int64_t pidx = ((int64_t)z * p.tiles_m + tm) * p.tiles_n + tn;
                tile_nseg = __ldg(p.plan_nseg + pidx);
                // a pair's plan holds the products of both CTAs' rows per segment
                tile_q = p.plan_q + pidx * p.kblocks * (PAIR ? 2 : 1) + (PAIR ? rank : 0);
            }
            float acc[BN / 2];
#pragma unroll
            for (int j = 0; j < BN / 2; ++j) acc[j] = 0.0f;
            for (int g = 0; g < tile_nseg; ++g) {
                ++seg;
                const int b = seg & 1;
                float scale = 1.0f;
                if constexpr (MD::SCALED) {
                    const float2 q = __ldg(tile_q + (PAIR ? 2 * g : g));  // this half's scale block product
                    scale = half ? q.y : q.x;
                }
                if (!wait(&tfull[b], (uint32_t)(seg >> 1) & 1u, 2 * kWaitNs)) {
                    if (!abort_flag) report_fault(p.fault, kFaultTcEpilogueWait);
                    abort_flag = 1;
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                // 16-column loads keep the drain within the 168-register cap
#pragma unroll
                for (int c = 0; c < BN / 2 / 16; ++c) {
                    uint32_t r[16];
                    tc::tmem_ld_32x32b_x16(tmem + lane_base + (uint32_t)(b * BN + half * (BN / 2) + c * 16), r);
                    tc::tmem_ld_wait();
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        if constexpr (MD::SCALED)
                            acc[c * 16 + j] = __fmaf_rn(__uint_as_float(r[j]), scale, acc[c * 16 + j]);
                        else
                            acc[c * 16 + j] = __fadd_rn(acc[c * 16 + j], __uint_as_float(r[j]));
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
            const int64_t row0 = m0 + quarter * 32;
            const int64_t col0 = n0 + half * (BN / 2);
            if (p.tma_store) {
                // 32 x 32 chunks: row `lane` into the staging tile (128-byte
                // swizzle: 16-byte chunk j of row r at (j ^ (r & 7))), then one
                // TMA store; C = alpha * acc when gemm (beta is 0 on this path)
#pragma unroll
                for (int c = 0; c < BN / 2 / 32; ++c) {
                    if (lane == 0) bulk_wait_read<0>();  // the previous store has read the staging tile
                    __syncwarp();
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        float v[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const float a = acc[c * 32 + j * 4 + e];
                            v[e] = p.gemm ? __fmaf_rn(p.alpha, a, 0.0f) : a;
                        }
                        *reinterpret_cast<float4 *>(stage + lane * 128 + ((j ^ (lane & 7)) << 4)) =
                            make_float4(v[0], v[1], v[2], v[3]);
                    }
                    fence_proxy_async_shared();
                    __syncwarp();
                    if (lane == 0 && row0 < p.M && col0 + c * 32 < p.N) {
                        tma_store_3d(&tcout, stage, (int32_t)(col0 + c * 32), (int32_t)row0, z);
                        bulk_commit();
                    }
                }
            } else {
                const int64_t row = row0 + lane;
                float *crow = p.C + (int64_t)z * p.stride_c + row * p.ldc;
                if (row < p.M) {
#pragma unroll
                    for (int j = 0; j < BN / 2; j += 4) {
                        float v[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const int64_t col = col0 + j + e;
                            if (p.gemm) {
                                const float bc = (p.beta == 0.0f || col >= p.N) ? 0.0f : p.beta * crow[col];
                                v[e] = __fmaf_rn(p.alpha, acc[j + e], bc);
                            } else {
                                v[e] = acc[j + e];
                            }
                        }
                        if (vec_ok && col0 + j + 3 < p.N) {
                            *reinterpret_cast<float4 *>(crow + col0 + j) = make_float4(v[0], v[1], v[2], v[3]);
                        } else {
#pragma unroll
                            for (int e = 0; e < 4; ++e)
                                if (col0 + j + e < p.N) crow[col0 + j + e] = v[e];
                        }
                    }
                }
            }
        }
        if (lane == 0) bulk_wait<0>();  // this warp's C stores are complete
        __syncwarp();
    }
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0 && abort_flag) {
        // Copies complete on the leader's barrier and cannot be awaited from
        // a pair's second CTA: give every copy in flight time to land (they
        // take microseconds).  The MMA issuer's CTA also waits for the MMAs
        // issued before its abort.
        const uint64_t t0 = tc::globaltimer();
        while (tc::globaltimer() - t0 < 20000000ull) {
        }
        if (leader && mma_aborted) tc::wait_timed(&mma_done, 0, kWaitNs, nullptr);
    }
    __syncthreads();
    if constexpr (PAIR) {
        tc::cluster_sync();  // neither CTA leaves while the pair can still touch its memory
        if (warp == 0) tc::tmem_dealloc_pair(tmem, kTmemCols2);
    } else {
        if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols2);
    }
}

// ---------------------------------------------------------------------------
// Wide contraction (one-product BF16 accumulated over all of K): persistent,
// one CTA per SM over 256 x 256 tiles, two M = 128 accumulators in all 512
// TMEM columns.  With no promotion there is nothing to double-buffer: the
// drain warps stream each tile's accumulators out through the staging tiles
// and TMA stores, then free TMEM for the next tile (whose K slices the ring
// has meanwhile prefetched).  The MMA sequence per output element is that of
// tc_gemm_persistent_kernel<0> with one segment, so the results are
// bit-identical.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads2, 1)
    tc_gemm_wide_kernel(const __grid_constant__ CUtensorMap ta0, const __grid_constant__ CUtensorMap tb0,
                        const __grid_constant__ CUtensorMap tcout, Params p) {
    using L = WideLayout;
    constexpr int S = L::STAGES;
    constexpr int BK = L::BK;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[S], empty[S], tfull, tempty, mma_done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    __shared__ int mma_aborted;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int unit = (int)blockIdx.x, units = (int)gridDim.x;
    const int64_t per_batch = (int64_t)p.tiles_m * p.tiles_n;
    const int64_t total = per_batch * p.batch;
    auto decode = [&](int64_t t, int &tm, int &tn, int &z) {
        z = (int)(t / per_batch);
        const int bid = (int)(t - (int64_t)z * per_batch);
        const int G = p.group_tiles;
        const int per_group = G * p.tiles_n;
        const int first_m = (bid / per_group) * G;
        const int gm = min(p.tiles_m - first_m, G);
        const int r = bid % per_group;
        tm = first_m + r % gm;
        tn = r / gm;
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&tfull, 1);
        mbar_init(&tempty, kDrainWarps);
        mbar_init(&mma_done, 1);
        fence_mbarrier_init();
        abort_flag = 0;
        mma_aborted = 0;
        prefetch_tmap(&ta0);
        prefetch_tmap(&tb0);
        if (p.tma_store) prefetch_tmap(&tcout);
    }
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, kTmemCols2);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    auto a_tile = [&](int s) { return smem + s * L::STAGE_BYTES; };
    auto b_tile = [&](int s) { return smem + s * L::STAGE_BYTES + L::A_TILE; };

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer: one ring position per K slice, across tiles ----
            int s = 0;
            uint32_t ph = 0;
            bool stop = false;
            for (int64_t t = unit; t < total && !stop; t += units) {
                int tm, tn, z;
                decode(t, tm, tn, z);
                for (int kb = 0; kb < p.kblocks; ++kb) {
                    if (!tc::wait_timed(&empty[s], ph ^ 1u, kWaitNs, &abort_flag)) {
                        if (!abort_flag) report_fault(p.fault, kFaultTcProducerWait);
                        abort_flag = 1;
                        stop = true;
                        break;
                    }
                    mbar_arrive_expect_tx(&full[s], L::STAGE_BYTES);
                    tma_load_3d(a_tile(s), &ta0, kb * BK, tm * L::TM, z, &full[s]);
                    tma_load_3d(b_tile(s), &tb0, kb * BK, tn * BN, z, &full[s]);
                    if (++s == S) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer: each tile accumulates over all of K in TMEM ----
            constexpr uint32_t idesc = L::IDESC;
            int s = 0;
            uint32_t ph = 0, tph = 0;
            bool stop = false;
            for (int64_t t = unit; t < total && !stop; t += units, tph ^= 1u) {
                // the drain has read the previous tile's accumulators
                if (!tc::wait_timed(&tempty, tph ^ 1u, kWaitNs, &abort_flag)) {
                    if (!abort_flag) report_fault(p.fault, kFaultTcMmaWait);
                    abort_flag = 1;
                    stop = true;
                    break;
                }
                tc::fence_after_sync();
                for (int kb = 0; kb < p.kblocks; ++kb) {
                    if (!tc::wait_timed(&full[s], ph, kWaitNs, &abort_flag)) {
                        if (!abort_flag) report_fault(p.fault, kFaultTcMmaWait);
                        abort_flag = 1;
                        stop = true;
                        break;
                    }
                    tc::fence_after_sync();
#pragma unroll
                    for (int kk = 0; kk < L::KSTEPS; ++kk) {
                        const uint32_t a_addr = smem_u32(a_tile(s)) + kk * 32;
                        const uint32_t b_addr = smem_u32(b_tile(s)) + kk * 32;
                        const uint64_t bd = tc::smem_desc_kmajor(b_addr, L::SBO, L::SWIZZLE);
                        const uint32_t accum = (kb == 0 && kk == 0) ? 0u : 1u;
                        tc::mma_bf16(tmem, tc::smem_desc_kmajor(a_addr, L::SBO, L::SWIZZLE), bd, idesc, accum);
                        tc::mma_bf16(tmem + (uint32_t)BN, tc::smem_desc_kmajor(a_addr + L::A_HALF, L::SBO, L::SWIZZLE),
                                     bd, idesc, accum);
                    }
                    tc::commit_to(&empty[s]);
                    if (++s == S) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (!stop) tc::commit_to(&tfull);
            }
            if (stop) {
                // every MMA issued before the abort completes before TMEM is freed
                mma_aborted = 1;
                tc::commit_to(&mma_done);
            }
        }
        __syncwarp();
    } else {
        // ---- drain: stream each tile's accumulators out ----
        // warp (quarter q, half h) reads TMEM lanes 32q..32q+31 of accumulator h:
        // tile rows 128h + 32q + lane, all 256 columns, in chunks of 32
        const int quarter = warp & 3, half = (warp - 2) >> 2;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        uint8_t *stage = smem + L::EPI_OFFSET + (warp - 2) * kEpiTileBytes;
        const bool vec_ok = (p.ldc % 4 == 0) && ((reinterpret_cast<uintptr_t>(p.C) & 15) == 0) && (p.stride_c % 4 == 0);
        uint32_t tph = 0;
        for (int64_t t = unit; t < total; t += units, tph ^= 1u) {
            int tm, tn, z;
            decode(t, tm, tn, z);
            if (!tc::wait_timed(&tfull, tph, 2 * kWaitNs, &abort_flag)) {
                if (!abort_flag) report_fault(p.fault, kFaultTcEpilogueWait);
                abort_flag = 1;
                break;
            }
            tc::fence_after_sync();
            const int64_t row0 = (int64_t)tm * L::TM + half * 128 + quarter * 32;
            const int64_t n0 = (int64_t)tn * BN;
#pragma unroll 1
            for (int c = 0; c < BN / 32; ++c) {
                uint32_t r[32];
                {
                    uint32_t (&lo)[16] = *reinterpret_cast<uint32_t (*)[16]>(&r[0]);
                    uint32_t (&hi)[16] = *reinterpret_cast<uint32_t (*)[16]>(&r[16]);
                    const uint32_t col = tmem + lane_base + (uint32_t)(half * BN + c * 32);
                    tc::tmem_ld_32x32b_x16(col, lo);
                    tc::tmem_ld_32x32b_x16(col + 16, hi);
                    tc::tmem_ld_wait();
                }
                if (c == BN / 32 - 1) {
                    // every accumulator column of this warp is read: TMEM is free
                    tc::fence_before_sync();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&tempty);
                }
                const int64_t col0 = n0 + c * 32;
                if (p.tma_store) {
                    if (lane == 0) bulk_wait_read<0>();  // the previous store has read the staging tile
                    __syncwarp();
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        float v[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const float a = __uint_as_float(r[j * 4 + e]);
                            v[e] = p.gemm ? __fmaf_rn(p.alpha, a, 0.0f) : a;
                        }
                        *reinterpret_cast<float4 *>(stage + lane * 128 + ((j ^ (lane & 7)) << 4)) =
                            make_float4(v[0], v[1], v[2], v[3]);
                    }
                    fence_proxy_async_shared();
                    __syncwarp();
                    if (lane == 0 && row0 < p.M && col0 < p.N) {
                        tma_store_3d(&tcout, stage, (int32_t)col0, (int32_t)row0, z);
                        bulk_commit();
                    }
                } else {
                    const int64_t row = row0 + lane;
                    if (row < p.M) {
                        float *crow = p.C + (int64_t)z * p.stride_c + row * p.ldc;
#pragma unroll
                        for (int j = 0; j < 32; j += 4) {
                            float v[4];
#pragma unroll
                            for (int e = 0; e < 4; ++e) {
                                const int64_t col = col0 + j + e;
                                const float a = __uint_as_float(r[j + e]);
                                if (p.gemm) {
                                    const float bc = (p.beta == 0.0f || col >= p.N) ? 0.0f : p.beta * crow[col];
                                    v[e] = __fmaf_rn(p.alpha, a, bc);
                                } else {
                                    v[e] = a;
                                }
                            }
                            if (vec_ok && col0 + j + 3 < p.N) {
                                *reinterpret_cast<float4 *>(crow + col0 + j) = make_float4(v[0], v[1], v[2], v[3]);
                            } else {
#pragma unroll
                                for (int e = 0; e < 4; ++e)
                                    if (col0 + j + e < p.N) crow[col0 + j + e] = v[e];
                            }
                        }
                    }
                }
            }
        }
        if (lane == 0) bulk_wait<0>();  // this warp's C stores are complete
        __syncwarp();
    }
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0 && abort_flag) {
        // copies in flight land (microseconds); the MMAs issued before an abort complete
        const uint64_t t0 = tc::globaltimer();
        while (tc::globaltimer() - t0 < 20000000ull) {
        }
        if (mma_aborted) tc::wait_timed(&mma_done, 0, kWaitNs, nullptr);
    }
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols2);
}

// ---------------------------------------------------------------------------
// split pass: FP32 -> NP BF16 pieces, K-major [batch][rows][Kp]
// ---------------------------------------------------------------------------
struct SplitArgs {
    const float *src;
    int64_t rows, K, Kp, ld, src_stride;  // src element (r,k): src[r*ld + k] (direct) or src[k*ld + r] (transposed)
    __nv_bfloat16 *out[3];
    int64_t piece_stride;                 // elements per instance in each piece: rows*Kp
};

// Stores the NP pieces of 8 consecutive elements of one K-major row: one
// 16-byte store per piece (Kp is a multiple of 8, so every run is aligned).
template <int NP>
__device__ __forceinline__ void store_pieces8(const SplitArgs &a, int64_t z, int64_t r, int64_t k, const float (&x)[8]) {
    __nv_bfloat16 pcs[8][3];
#pragma unroll
    for (int e = 0; e < 8; ++e) split_value<NP>(x[e], pcs[e]);
#pragma unroll
    for (int i = 0; i < NP; ++i) {
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            __nv_bfloat162 v = __halves2bfloat162(pcs[2 * j][i], pcs[2 * j + 1][i]);
            w[j] = *reinterpret_cast<uint32_t *>(&v);
        }
        *reinterpret_cast<uint4 *>(a.out[i] + z * a.piece_stride + r * a.Kp + k) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// Source stored rows x K (element (r,k) at src[r*ld + k]): each thread
// splits runs of 8 consecutive k, read as two 16-byte loads where aligned.
template <int NP>
__global__ void __launch_bounds__(256) split_direct_kernel(SplitArgs a) {
    const int64_t runs_per_row = a.Kp / 8;
    const int64_t total = a.rows * runs_per_row;
    const int64_t z = blockIdx.y;
    const float *src = a.src + z * a.src_stride;
    const bool vec = (a.ld % 4 == 0) && ((reinterpret_cast<uintptr_t>(src) & 15) == 0);
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = q / runs_per_row, k = (q % runs_per_row) * 8;
        const float *ptr = src + r * a.ld + k;
        float x[8];
        if (vec && k + 7 < a.K) {
            const float4 u = __ldcs(reinterpret_cast<const float4 *>(ptr));
            const float4 v = __ldcs(reinterpret_cast<const float4 *>(ptr + 4));
            x[0] = u.x, x[1] = u.y, x[2] = u.z, x[3] = u.w, x[4] = v.x, x[5] = v.y, x[6] = v.z, x[7] = v.w;
        } else {
#pragma unroll
            for (int e = 0; e < 8; ++e) x[e] = (k + e < a.K) ? ptr[e] : 0.0f;
        }
        store_pieces8<NP>(a, z, r, k, x);
    }
}

// Source stored K x rows (element (r,k) at src[k*ld + r]): 64 x 64 tiles
// transposed through shared memory.  Reads are 16-byte loads along rows;
// writes are 16-byte runs of 8 k, eight threads covering one 128-byte row
// segment per piece.
template <int NP>
__global__ void __launch_bounds__(256) split_transpose_kernel(SplitArgs a) {
    __shared__ float tile[64][65];  // [k][r]
    const int tid = threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.x * 64, k0 = (int64_t)blockIdx.y * 64;
    const int64_t z = blockIdx.z;
    const float *src = a.src + z * a.src_stride;
    const bool vec = (a.ld % 4 == 0) && ((reinterpret_cast<uintptr_t>(src) & 15) == 0);
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int kk = p * 16 + (tid >> 4), rr = (tid & 15) * 4;
        const int64_t k = k0 + kk, r = r0 + rr;
        float v[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (k < a.K) {
            const float *ptr = src + k * a.ld + r;
            if (vec && r + 3 < a.rows) {
                const float4 u = __ldcs(reinterpret_cast<const float4 *>(ptr));
                v[0] = u.x, v[1] = u.y, v[2] = u.z, v[3] = u.w;
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    if (r + e < a.rows) v[e] = ptr[e];
            }
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) tile[kk][rr + e] = v[e];
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const int rr = p * 32 + (tid >> 3), c = tid & 7;
        const int64_t r = r0 + rr, k = k0 + c * 8;
        if (r < a.rows && k < a.Kp) {
            float x[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = tile[c * 8 + j][rr];
            store_pieces8<NP>(a, z, r, k, x);
        }
    }
}

// ---------------------------------------------------------------------------
// FP8 pass: FP32 -> E4M3 codes, K-major [batch][rows][Kp], with one FP32
// scale per 128 x 128 block: s = the smallest power of two with
// amax / s <= 448, code = e4m3_rn_satfinite(x / s) (x / s is exact; all
// codes 0 and s = 0 for an all-zero block).  Power-of-two scales keep the
// scaling, the scale product sa * sb and the dequantisation exact.
// ---------------------------------------------------------------------------
constexpr int kQBlock = 128;

struct QuantArgs {
    const float *src;
    int64_t rows, K, Kp, ld, src_stride;
    int transposed;   // element (r,k) at src[k*ld + r] instead of src[r*ld + k]
    int vec;          // 16-byte loads allowed: ld and src_stride multiples of 4, base 16-byte aligned
    uint8_t *codes;   // [batch][rows][Kp]
    float *scales;    // [batch][rblocks][kblocks]
    int64_t rblocks, kblocks;
};

// Staged code words: row r (0..127) holds 32 words of 4 codes; word w is
// stored at w ^ (r >> 2) so that both the staging stores (a warp covers 32
// words of one row, or one word of 32 row quads) and the row-wise copy-out
// hit 32 distinct banks.
__device__ __forceinline__ int qt_index(int r, int w) { return r * 32 + (w ^ ((r >> 2) & 31)); }

// x / s for the block scale s, a power of two.  Where 1/s is a normal power
// of two (r != 0), x * r and x / s are the correctly rounded values of the
// same real number, hence identical; elsewhere (s subnormal or huge) divide.
__device__ __forceinline__ float scale_down(float x, float s, float r) { return r != 0.0f ? x * r : __fdiv_rn(x, s); }

__device__ __forceinline__ uint32_t e4m3_pack4(float s, float r, float x0, float x1, float x2, float x3) {
    if (s == 0.0f) return 0u;
    const uint32_t b0 = __nv_cvt_float_to_fp8(scale_down(x0, s, r), __NV_SATFINITE, __NV_E4M3);
    const uint32_t b1 = __nv_cvt_float_to_fp8(scale_down(x1, s, r), __NV_SATFINITE, __NV_E4M3);
    const uint32_t b2 = __nv_cvt_float_to_fp8(scale_down(x2, s, r), __NV_SATFINITE, __NV_E4M3);
    const uint32_t b3 = __nv_cvt_float_to_fp8(scale_down(x3, s, r), __NV_SATFINITE, __NV_E4M3);
    return b0 | (b1 << 8) | (b2 << 16) | (b3 << 24);
}

constexpr int kQThreads = 512;  // 32 values per thread; two CTAs (1024 threads) per SM

__global__ void __launch_bounds__(kQThreads, 2) quant_fp8_kernel(QuantArgs a) {
    constexpr int G = kQBlock * kQBlock / 4 / kQThreads;  // groups of 4 values per thread
    __shared__ uint32_t qt[kQBlock * 32];
    __shared__ float red[kQThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t r0 = (int64_t)blockIdx.y * kQBlock, k0 = (int64_t)blockIdx.x * kQBlock, z = blockIdx.z;
    const float *src = a.src + z * a.src_stride;
    // 4*G values per thread as G groups of 4 consecutive elements of the
    // stored inner dimension (k for direct sources, rows for transposed ones)
    float v[4 * G];
    float amax = 0.0f;
#pragma unroll
    for (int i = 0; i < G; ++i) {
        int64_t outer, inner;  // stored coordinates of the group's first element
        if (!a.transposed) {
            const int idx = i * kQThreads + tid;            // row idx/32, k quad idx%32
            outer = r0 + (idx >> 5);
            inner = k0 + (idx & 31) * 4;
        } else {
            const int blk = (i >> 2) * kQThreads + tid;     // 4x4 block: row quad blk%32, k quad blk/32
            outer = k0 + (blk >> 5) * 4 + (i & 3);
            inner = r0 + (blk & 31) * 4;
        }
        const int64_t outer_lim = a.transposed ? a.K : a.rows, inner_lim = a.transposed ? a.rows : a.K;
        float x[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (outer < outer_lim) {
            const float *ptr = src + outer * a.ld + inner;
            if (a.vec && inner + 3 < inner_lim) {
                const float4 q = __ldcs(reinterpret_cast<const float4 *>(ptr));
                x[0] = q.x, x[1] = q.y, x[2] = q.z, x[3] = q.w;
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    if (inner + e < inner_lim) x[e] = ptr[e];
            }
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            v[i * 4 + e] = x[e];
            amax = fmaxf(amax, fabsf(x[e]));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    if (lane == 0) red[warp] = amax;
    __syncthreads();
    amax = red[0];
#pragma unroll
    for (int w = 1; w < kQThreads / 32; ++w) amax = fmaxf(amax, red[w]);
    // s = 2^ceil(log2(amax / 448)), the smallest power of two with amax / s <= 448:
    // with amax = f * 2^e, f in [0.5, 1), that is 2^(e - 9) for f <= 0.875, else 2^(e - 8)
    float s = 0.0f, rcp = 0.0f;
    if (amax > 0.0f) {
        int e;
        const float f = frexpf(amax, &e);
        const int j = e - 9 + (f > 0.875f ? 1 : 0);  // s = 2^j
        s = ldexpf(1.0f, j);
        if (isfinite(amax) && j >= -126 && j <= 126) rcp = ldexpf(1.0f, -j);  // 1/s, exact and normal
    }
    if (tid == 0) a.scales[(z * a.rblocks + blockIdx.y) * a.kblocks + blockIdx.x] = s;
    if (!a.transposed) {
#pragma unroll
        for (int i = 0; i < G; ++i) {
            const int idx = i * kQThreads + tid;
            qt[qt_index(idx >> 5, idx & 31)] = e4m3_pack4(s, rcp, v[i * 4], v[i * 4 + 1], v[i * 4 + 2], v[i * 4 + 3]);
        }
    } else {
#pragma unroll
        for (int j = 0; j < G / 4; ++j) {
            const int blk = j * kQThreads + tid;
            const int rq = blk & 31, kq = blk >> 5;
            // v[(j*4 + kk)*4 + e] is element (row 4*rq + e, k 4*kq + kk)
#pragma unroll
            for (int e = 0; e < 4; ++e)
                qt[qt_index(rq * 4 + e, kq)] = e4m3_pack4(s, rcp, v[(j * 4 + 0) * 4 + e], v[(j * 4 + 1) * 4 + e],
                                                          v[(j * 4 + 2) * 4 + e], v[(j * 4 + 3) * 4 + e]);
        }
    }
    __syncthreads();
    uint8_t *codes = a.codes + z * a.rows * a.Kp;
#pragma unroll
    for (int i = 0; i < kQBlock * 32 / kQThreads; ++i) {
        const int idx = i * kQThreads + tid;
        const int r = idx >> 5, w = idx & 31;
        const int64_t row = r0 + r, k = k0 + w * 4;
        if (row < a.rows && k < a.Kp)
            *reinterpret_cast<uint32_t *>(codes + row * a.Kp + k) = qt[qt_index(r, w)];
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct Plan {
    int mode;  // 0 bf16, 1 split3, 2 split6, 3 fp8
    int np;    // operand pieces
    int elem;  // bytes per staged element
    int64_t Kp;
    size_t a_piece_bytes, b_piece_bytes;
    // FP8: scale blocks, and the per-tile segment plan of the contraction
    int64_t mblocks, nblocks, kblocks;
    size_t sa_bytes, sb_bytes;
    size_t plan_nseg_bytes, plan_bits_bytes, plan_q_bytes;
    size_t total;
};

static inline size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

static bool make_plan(const gatlas_matmul_desc *d, const Geometry &g, Plan *pl) {
    pl->elem = 2;
    switch (d->engine) {
        case GATLAS_ENGINE_TC_BF16: pl->mode = 0; pl->np = 1; break;
        case GATLAS_ENGINE_TC_SPLIT3: pl->mode = 1; pl->np = 2; break;
        case GATLAS_ENGINE_TC_SPLIT6: pl->mode = 2; pl->np = 3; break;
        case GATLAS_ENGINE_TC_FP8: pl->mode = 3; pl->np = 1; pl->elem = 1; break;
        default: return false;
    }
    const size_t K = (size_t)(g.K > 0 ? g.K : 1);
    // rows of 16 bytes at least (TMA row pitch), zero padded to Kp
    pl->Kp = (int64_t)round_up(K, 16 / pl->elem);
    pl->a_piece_bytes = round_up((size_t)g.batch * (size_t)g.M * (size_t)pl->Kp * pl->elem, 1024);
    pl->b_piece_bytes = round_up((size_t)g.batch * (size_t)g.N * (size_t)pl->Kp * pl->elem, 1024);
    pl->mblocks = pl->nblocks = pl->kblocks = 0;
    pl->sa_bytes = pl->sb_bytes = 0;
    pl->plan_nseg_bytes = pl->plan_bits_bytes = pl->plan_q_bytes = 0;
    if (pl->mode == 3) {
        pl->mblocks = (g.M + kQBlock - 1) / kQBlock;
        pl->nblocks = (g.N + kQBlock - 1) / kQBlock;
        pl->kblocks = (int64_t)((K + kQBlock - 1) / kQBlock);
        pl->sa_bytes = round_up((size_t)g.batch * pl->mblocks * pl->kblocks * 4, 1024);
        pl->sb_bytes = round_up((size_t)g.batch * pl->nblocks * pl->kblocks * 4, 1024);
        // per tile a segment count, one bit per block and the scale products
        // of every possible segment: tiles of 128 x 256 (single CTAs, two
        // products) or 256 x 256 (CTA pairs, four); sized for either
        const size_t tn = (size_t)((g.N + BN - 1) / BN) * (size_t)g.batch;
        const size_t tiles = (size_t)((g.M + BM - 1) / BM) * tn;
        const size_t pair_tiles = (size_t)((g.M + 2 * BM - 1) / (2 * BM)) * tn;
        pl->plan_nseg_bytes = round_up(tiles * 4, 256);
        pl->plan_bits_bytes = round_up(tiles * (size_t)((pl->kblocks + 31) / 32) * 4, 256);
        pl->plan_q_bytes = round_up(std::max(tiles, 2 * pair_tiles) * (size_t)pl->kblocks * 8, 1024);
    }
    pl->total = pl->np * (pl->a_piece_bytes + pl->b_piece_bytes) + pl->sa_bytes + pl->sb_bytes +
                pl->plan_nseg_bytes + pl->plan_bits_bytes + pl->plan_q_bytes;
    return true;
}

static int launch_quant(bool transposed, const float *src, int64_t rows, int64_t K, int64_t Kp, int64_t ld,
                        int64_t src_stride, int64_t batch, uint8_t *codes, float *scales, cudaStream_t stream) {
    QuantArgs a;
    a.src = src;
    a.rows = rows;
    a.K = K;
    a.Kp = Kp;
    a.ld = ld;
    a.src_stride = src_stride;
    a.transposed = transposed ? 1 : 0;
    a.vec = (ld % 4 == 0) && aligned16(src) && (batch == 1 || src_stride % 4 == 0);
    a.codes = codes;
    a.scales = scales;
    a.rblocks = (rows + kQBlock - 1) / kQBlock;
    a.kblocks = (K + kQBlock - 1) / kQBlock;
    if (a.rblocks > 65535) return set_error(GATLAS_ERR_INVALID, "matmul: too many rows for the FP8 pass");
    dim3 gr((unsigned)a.kblocks, (unsigned)a.rblocks, (unsigned)batch);
    quant_fp8_kernel<<<gr, kQThreads, 0, stream>>>(a);
    return check_launch("quant_fp8_kernel");
}

static int launch_split(int np, bool transposed, const float *src, int64_t rows, int64_t K, int64_t Kp,
                        int64_t ld, int64_t src_stride, int64_t batch, __nv_bfloat16 *const out[3],
                        cudaStream_t stream) {
    SplitArgs a;
    a.src = src;
    a.rows = rows;
    a.K = K;
    a.Kp = Kp;
    a.ld = ld;
    a.src_stride = src_stride;
    for (int i = 0; i < 3; ++i) a.out[i] = out[i];
    a.piece_stride = rows * Kp;
    if (!transposed) {
        const int64_t total = rows * (Kp / 8);
        int64_t grid = (total + 255) / 256;
        const int64_t cap = (int64_t)sm_count() * 16;
        if (grid > cap) grid = cap;
        dim3 gr((unsigned)(grid > 0 ? grid : 1), (unsigned)batch);
        if (np == 1) split_direct_kernel<1><<<gr, 256, 0, stream>>>(a);
        else if (np == 2) split_direct_kernel<2><<<gr, 256, 0, stream>>>(a);
        else split_direct_kernel<3><<<gr, 256, 0, stream>>>(a);
    } else {
        const int64_t gx = (rows + 63) / 64, gy = (Kp + 63) / 64;
        if (gy > 65535) return set_error(GATLAS_ERR_INVALID, "matmul: K too large for the transposing split");
        dim3 gr((unsigned)gx, (unsigned)gy, (unsigned)batch);
        if (np == 1) split_transpose_kernel<1><<<gr, 256, 0, stream>>>(a);
        else if (np == 2) split_transpose_kernel<2><<<gr, 256, 0, stream>>>(a);
        else split_transpose_kernel<3><<<gr, 256, 0, stream>>>(a);
    }
    return check_launch("split kernel");
}

// Operand pointers inside a prepared workspace: [A pieces][B pieces], then
// for FP8 [A scales][B scales].
struct WsPtrs {
    void *a[3], *b[3];
    float *sa, *sb;
    int *plan_nseg;  // FP8: per-tile segment plan (fp8_plan_kernel)
    uint32_t *plan_bits;
    float2 *plan_q;
};

static WsPtrs ws_ptrs(const Plan &pl, void *ws) {
    uint8_t *base = static_cast<uint8_t *>(ws);
    WsPtrs w;
    for (int i = 0; i < 3; ++i) {
        w.a[i] = w.b[i] = nullptr;
        if (i < pl.np) {
            w.a[i] = base + i * pl.a_piece_bytes;
            w.b[i] = base + pl.np * pl.a_piece_bytes + i * pl.b_piece_bytes;
        }
    }
    uint8_t *sc = base + pl.np * (pl.a_piece_bytes + pl.b_piece_bytes);
    w.sa = pl.mode == 3 ? reinterpret_cast<float *>(sc) : nullptr;
    w.sb = pl.mode == 3 ? reinterpret_cast<float *>(sc + pl.sa_bytes) : nullptr;
    uint8_t *pp = sc + pl.sa_bytes + pl.sb_bytes;
    w.plan_nseg = pl.mode == 3 ? reinterpret_cast<int *>(pp) : nullptr;
    w.plan_bits = pl.mode == 3 ? reinterpret_cast<uint32_t *>(pp + pl.plan_nseg_bytes) : nullptr;
    w.plan_q = pl.mode == 3 ? reinterpret_cast<float2 *>(pp + pl.plan_nseg_bytes + pl.plan_bits_bytes) : nullptr;
    return w;
}

// Tiling of C for M > 128 ("tc_pair"): 1 = what measures fastest on B200 --
// CTA pairs for the split engines (17-19 % fewer cycles per 8192^3 launch
// than 128 x 256 single CTAs), 256 x 256 single-CTA tiles for one-product
// BF16 over all of K (35 % fewer), 128 x 256 single CTAs for FP8 (pairs
// measured 30 % slower); 2 = CTA pairs always; 0 = 128 x 256 always.
static int g_tc_pair = 1;
// Rows of C per raster group of the persistent kernels (multiple of 128).
static int g_tc_group_rows = kGroupM * 128;
// A's loads evict-last in the persistent kernel (Params::l2_hint): at 8192^3
// split3 on CTA pairs, 2.54 GB of DRAM reads per launch instead of 3.45, at the
// same speed.
static int g_tc_l2_hint = 1;

// FP8 segment plan, one thread per tile: a run of at most seg_kblocks
// 128-deep blocks whose scale products sa * sb are equal for every 128 x 128
// block of the tile accumulates in TMEM and is promoted, scaled once (exact:
// the scales are powers of two).  Writes the tile's segment count, its
// segment-start bits and each segment's scale products.  Single CTAs
// (pair == 0) have 128 x 256 tiles: one A block, two column halves, products
// (a b0, a b1) per segment.  CTA pairs (pair == 1) have 256 x 256 tiles: the
// MMAs of both CTAs share their segments, so a run ends where any of the four
// products changes; per segment the plan holds (a0 b0, a0 b1) for the
// leader's rows and (a1 b0, a1 b1) for the peer's.
__global__ void __launch_bounds__(128)
    fp8_plan_kernel(const float *scale_a, const float *scale_b, int64_t sa_stride, int64_t sb_stride, int tiles_m,
                    int tiles_n, int batch, int kblocks, int nblocks_m, int nblocks_n, int seg_kblocks, int words,
                    int pair, int *nseg, uint32_t *bits, float2 *q) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)tiles_m * tiles_n * batch) return;
    const int tn = (int)(idx % tiles_n);
    const int64_t rest = idx / tiles_n;
    const int tm = (int)(rest % tiles_m);
    const int64_t z = rest / tiles_m;
    const int ma0 = pair ? 2 * tm : tm, ma1 = 2 * tm + 1;
    const float *sa0 = scale_a + z * sa_stride + (int64_t)ma0 * kblocks;
    const float *sa1 = pair && ma1 < nblocks_m ? scale_a + z * sa_stride + (int64_t)ma1 * kblocks : nullptr;
    const int nb0 = 2 * tn, nb1 = 2 * tn + 1;
    const float *sb0 = nb0 < nblocks_n ? scale_b + z * sb_stride + (int64_t)nb0 * kblocks : nullptr;
    const float *sb1 = nb1 < nblocks_n ? scale_b + z * sb_stride + (int64_t)nb1 * kblocks : nullptr;
    uint32_t *wb = bits + idx * words;
    float2 *qt = q + idx * kblocks * (pair ? 2 : 1);
    int s = -1, run = 0;
    float prev[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    uint32_t w = 0;
    for (int kb = 0; kb < kblocks; ++kb) {
        const float a0 = sa0[kb], a1 = sa1 ? sa1[kb] : 0.0f;
        const float b0 = sb0 ? sb0[kb] : 0.0f, b1 = sb1 ? sb1[kb] : 0.0f;
        const float cur[4] = {sb0 ? __fmul_rn(a0, b0) : 0.0f, sb1 ? __fmul_rn(a0, b1) : 0.0f,
                              sa1 && sb0 ? __fmul_rn(a1, b0) : 0.0f, sa1 && sb1 ? __fmul_rn(a1, b1) : 0.0f};
        bool start = kb == 0 || run == seg_kblocks;
        for (int i = 0; i < 4; ++i) start = start || cur[i] != prev[i];
        if (start) {
            ++s;
            run = 0;
            if (pair) {
                qt[2 * s] = make_float2(cur[0], cur[1]);
                qt[2 * s + 1] = make_float2(cur[2], cur[3]);
            } else {
                qt[s] = make_float2(cur[0], cur[1]);
            }
            w |= 1u << (kb & 31);
        }
        ++run;
        for (int i = 0; i < 4; ++i) prev[i] = cur[i];
        if ((kb & 31) == 31 || kb == kblocks - 1) {
            wb[kb >> 5] = w;
            w = 0;
        }
    }
    nseg[idx] = s + 1;
}

// Encodes the tensor map of C for the TMA-store epilogue (32 x 32 boxes,
// 128-byte swizzle) when C allows it; p.tma_store says whether it did.
static void c_tensor_map(const Geometry &g, Params &p, CUtensorMap *tcout) {
    p.tma_store = 0;
    const bool c_ok = (!p.gemm || p.beta == 0.0f) && aligned_to(p.C, 16) && p.ldc % 4 == 0 &&
                      (g.batch == 1 || p.stride_c % 4 == 0) && g.N < ((int64_t)1 << 31) && g.M < ((int64_t)1 << 31);
    if (!c_ok) return;
    const uint64_t cdims[3] = {(uint64_t)g.N, (uint64_t)g.M, (uint64_t)g.batch};
    const uint64_t cstr[2] = {(uint64_t)p.ldc * 4, (uint64_t)(g.batch > 1 ? p.stride_c : g.M * p.ldc) * 4};
    const uint32_t cbox[3] = {32, 32, 1};
    if (make_tensor_map(tcout, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, p.C, cdims, cstr, cbox,
                        CU_TENSOR_MAP_SWIZZLE_128B) == GATLAS_OK)
        p.tma_store = 1;
}

// Persistent launch: as many CTAs (CTA pairs) as fit on the GPU at once, at
// most one per tile.  C leaves through a TMA tensor map unless beta is used
// or C is not 16-byte aligned in rows and instances.
template <int MODE, bool PAIR>
static int launch_persistent(const CUtensorMap *ta, const CUtensorMap *tb, const Geometry &g, Params p,
                             cudaStream_t stream) {
    using PL = PersistentLayout<MODE, PAIR>;
    auto kern = tc_gemm_persistent_kernel<MODE, PAIR>;
    const int smem = (int)PL::SMEM_BYTES;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "tc persistent smem attribute: %s", cudaGetErrorString(e));
    const int64_t tiles_m = (g.M + PL::TM - 1) / PL::TM, tiles_n = (g.N + BN - 1) / BN;
    const int64_t total = tiles_m * tiles_n * g.batch;
    if (tiles_m * tiles_n > 0x7fffffff || total > ((int64_t)1 << 40))
        return set_error(GATLAS_ERR_INVALID, "matmul: too many tensor-core tiles");
    p.tiles_m = (int)tiles_m;
    p.tiles_n = (int)tiles_n;
    p.batch = (int)g.batch;
    p.group_tiles = std::max(1, g_tc_group_rows / PL::TM);
    p.l2_hint = g_tc_l2_hint;
    CUtensorMap tcout = ta[0];  // unused unless tma_store
    c_tensor_map(g, p, &tcout);
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(kThreads2, 1, 1);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = PAIR ? 2 : 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = PAIR ? 1 : 0;
    // resident units: CTAs (one per SM) or clusters of two, as the occupancy query reports
    static thread_local int cap_dev = -1, cap = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (cap_dev != dev) {
        cap = PAIR ? sm_count() / 2 : sm_count();
        if (PAIR) {
            cfg.gridDim = dim3(2 * (unsigned)cap, 1, 1);
            int n = 0;
            if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) == cudaSuccess && n > 0) cap = n;
            cudaGetLastError();
        }
        cap_dev = dev;
    }
    const int units = (int)std::min<int64_t>(total, std::max(cap, 1));
    cfg.gridDim = dim3((unsigned)((PAIR ? 2 : 1) * units), 1, 1);
    e = cudaLaunchKernelEx(&cfg, kern, ta[0], ta[1], ta[2], tb[0], tb[1], tb[2], tcout, p);
    if (e != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "tc_gemm_persistent_kernel: %s", cudaGetErrorString(e));
    return check_launch("tc_gemm_persistent_kernel");
}

// Wide launch (one-product BF16 over all of K): one CTA per SM, at most one
// per 256 x 256 tile; A and B tensor maps with 256-row boxes.
static int launch_wide(const Geometry &g, const Plan &pl, const WsPtrs &w, Params p, cudaStream_t stream) {
    using L = WideLayout;
    CUtensorMap ta, tb, tcout;
    const uint64_t row_bytes = (uint64_t)pl.Kp * pl.elem;
    const uint64_t adims[3] = {(uint64_t)pl.Kp, (uint64_t)g.M, (uint64_t)g.batch};
    const uint64_t astr[2] = {row_bytes, row_bytes * (uint64_t)g.M};
    const uint64_t bdims[3] = {(uint64_t)pl.Kp, (uint64_t)g.N, (uint64_t)g.batch};
    const uint64_t bstr[2] = {row_bytes, row_bytes * (uint64_t)g.N};
    const uint32_t box[3] = {(uint32_t)L::BK, 256, 1};
    int rc = make_tensor_map(&ta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, w.a[0], adims, astr, box, CU_TENSOR_MAP_SWIZZLE_128B);
    if (!rc) rc = make_tensor_map(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, w.b[0], bdims, bstr, box, CU_TENSOR_MAP_SWIZZLE_128B);
    if (rc) return rc;
    const int smem = (int)L::SMEM_BYTES;
    cudaError_t e = cudaFuncSetAttribute(tc_gemm_wide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "tc wide smem attribute: %s", cudaGetErrorString(e));
    const int64_t tiles_m = (g.M + L::TM - 1) / L::TM, tiles_n = (g.N + BN - 1) / BN;
    const int64_t total = tiles_m * tiles_n * g.batch;
    if (tiles_m * tiles_n > 0x7fffffff || total > ((int64_t)1 << 40))
        return set_error(GATLAS_ERR_INVALID, "matmul: too many tensor-core tiles");
    p.tiles_m = (int)tiles_m;
    p.tiles_n = (int)tiles_n;
    p.batch = (int)g.batch;
    p.group_tiles = std::max(1, g_tc_group_rows / L::TM);
    tcout = ta;  // unused unless tma_store
    c_tensor_map(g, p, &tcout);
    const int units = (int)std::min<int64_t>(total, sm_count());
    tc_gemm_wide_kernel<<<(unsigned)units, kThreads2, smem, stream>>>(ta, tb, tcout, p);
    return check_launch("tc_gemm_wide_kernel");
}

template <int MODE>
static int launch_tc(const Geometry &g, const Plan &pl, const WsPtrs &w, float *C, double alpha, double beta,
                     int gemm, int seg_kblocks, cudaStream_t stream) {
    using L = Layout<MODE>;
    const bool pair = g.M > BM && (g_tc_pair == 2 || (g_tc_pair == 1 && (MODE == 1 || MODE == 2)));
    CUtensorMap ta[3], tb[3];
    const uint64_t row_bytes = (uint64_t)pl.Kp * pl.elem;
    const uint64_t adims[3] = {(uint64_t)pl.Kp, (uint64_t)g.M, (uint64_t)g.batch};
    const uint64_t astr[2] = {row_bytes, row_bytes * (uint64_t)g.M};
    const uint64_t bdims[3] = {(uint64_t)pl.Kp, (uint64_t)g.N, (uint64_t)g.batch};
    const uint64_t bstr[2] = {row_bytes, row_bytes * (uint64_t)g.N};
    // a CTA of a pair stages 128 rows of B (its half of the pair's 256 columns)
    const uint32_t abox[3] = {(uint32_t)L::BK, BM, 1}, bbox[3] = {(uint32_t)L::BK, pair ? 128u : (uint32_t)BN, 1};
    const CUtensorMapDataType dt = MODE == 3 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    const CUtensorMapSwizzle swz = L::ROW_BYTES == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
    for (int i = 0; i < 3; ++i) {
        const int src = i < pl.np ? i : 0;  // unused slots alias piece 0
        int rc = make_tensor_map(&ta[i], dt, 3, w.a[src], adims, astr, abox, swz);
        if (rc) return rc;
        rc = make_tensor_map(&tb[i], dt, 3, w.b[src], bdims, bstr, bbox, swz);
        if (rc) return rc;
    }
    Params p;
    std::memset(&p, 0, sizeof(p));
    p.C = C;
    p.M = g.M;
    p.N = g.N;
    p.ldc = g.ldc;
    p.stride_c = g.stride_c;
    p.kblocks = (int)((pl.Kp + L::BK - 1) / L::BK);
    p.seg_kblocks = seg_kblocks > 0 ? seg_kblocks : default_seg_kblocks(MODE);
    p.alpha = (float)alpha;
    p.beta = (float)beta;
    p.gemm = gemm;
    p.fault = device_fault_word();
    p.scale_a = w.sa;
    p.scale_b = w.sb;
    p.scale_a_stride = pl.mblocks * pl.kblocks;
    p.scale_b_stride = pl.nblocks * pl.kblocks;
    p.nblocks_n = (int)pl.nblocks;
    p.nblocks_m = (int)pl.mblocks;
    if (MODE == 3 && p.kblocks != pl.kblocks) return set_error(GATLAS_ERR_INVALID, "matmul: FP8 slice count");
    if (MODE == 3 && p.kblocks > kMaxFp8Blocks)
        return set_error(GATLAS_ERR_UNSUPPORTED, "matmul: FP8 engine takes K <= %d", kMaxFp8Blocks * 128);
    if constexpr (MODE != 3) {
        // one-product BF16 accumulated over all of K: 256 x 256 tiles on single
        // CTAs, once there are at least as many of them as SMs (smaller products
        // keep the twice as many 128 x 256 tiles; the results are identical)
        const int64_t wide_tiles = ((g.M + 255) / 256) * ((g.N + BN - 1) / BN) * g.batch;
        if (MODE == 0 && g_tc_pair == 1 && g.M > BM && p.seg_kblocks >= p.kblocks && wide_tiles >= sm_count())
            return launch_wide(g, pl, w, p, stream);
        return pair ? launch_persistent<MODE, true>(ta, tb, g, p, stream)
                    : launch_persistent<MODE, false>(ta, tb, g, p, stream);
    } else {
        // plan every tile's segments (256 x 256 tiles on CTA pairs, 128 x 256
        // on single CTAs), then the persistent kernel
        const int64_t tm_rows = pair ? 2 * BM : BM;
        const int64_t tiles_m = (g.M + tm_rows - 1) / tm_rows, tiles_n = (g.N + BN - 1) / BN;
        const int64_t tiles = tiles_m * tiles_n * g.batch;
        if (tiles > 0) {
            const int words = (int)((p.kblocks + 31) / 32);
            fp8_plan_kernel<<<(unsigned)((tiles + 127) / 128), 128, 0, stream>>>(
                w.sa, w.sb, p.scale_a_stride, p.scale_b_stride, (int)tiles_m, (int)tiles_n, (int)g.batch,
                p.kblocks, p.nblocks_m, p.nblocks_n, p.seg_kblocks, words, pair ? 1 : 0, w.plan_nseg, w.plan_bits,
                w.plan_q);
            int rc = check_launch("fp8_plan_kernel");
            if (rc) return rc;
            p.plan_nseg = w.plan_nseg;
            p.plan_bits = w.plan_bits;
            p.plan_q = w.plan_q;
            p.plan_words = words;
        }
        return pair ? launch_persistent<MODE, true>(ta, tb, g, p, stream)
                    : launch_persistent<MODE, false>(ta, tb, g, p, stream);
    }
}

static int check_ws(const Plan &pl, const void *ws, size_t ws_bytes) {
    if (!ws) return set_error(GATLAS_ERR_INVALID, "matmul: null workspace");
    if (ws_bytes < pl.total) return set_error(GATLAS_ERR_INVALID, "matmul: workspace %zu < %zu bytes", ws_bytes, pl.total);
    if (!aligned_to(ws, 1024)) return set_error(GATLAS_ERR_INVALID, "matmul: workspace must be 1024-byte aligned");
    return GATLAS_OK;
}

int tc_prepare(const gatlas_matmul_desc *d, const Geometry &g, const float *A, const float *B, void *ws,
               size_t ws_bytes, cudaStream_t stream) {
    Plan pl;
    if (!make_plan(d, g, &pl)) return set_error(GATLAS_ERR_UNSUPPORTED, "matmul: tensor-core engine %d not built", d->engine);
    int rc = check_ws(pl, ws, ws_bytes);
    if (rc) return rc;
    const WsPtrs w = ws_ptrs(pl, ws);
    // A is K-major already when not transposed; B is K-major when transposed.
    if (pl.mode == 3) {
        rc = launch_quant(g.ta, A, g.M, g.K, pl.Kp, g.lda, g.stride_a, g.batch, static_cast<uint8_t *>(w.a[0]), w.sa,
                          stream);
        if (rc) return rc;
        return launch_quant(!g.tb, B, g.N, g.K, pl.Kp, g.ldb, g.stride_b, g.batch, static_cast<uint8_t *>(w.b[0]),
                            w.sb, stream);
    }
    __nv_bfloat16 *ap[3], *bp[3];
    for (int i = 0; i < 3; ++i) {
        ap[i] = static_cast<__nv_bfloat16 *>(w.a[i]);
        bp[i] = static_cast<__nv_bfloat16 *>(w.b[i]);
    }
    rc = launch_split(pl.np, g.ta, A, g.M, g.K, pl.Kp, g.lda, g.stride_a, g.batch, ap, stream);
    if (rc) return rc;
    return launch_split(pl.np, !g.tb, B, g.N, g.K, pl.Kp, g.ldb, g.stride_b, g.batch, bp, stream);
}

int tc_run(const gatlas_matmul_desc *d, const Geometry &g, const void *ws, size_t ws_bytes, float *C,
           cudaStream_t stream) {
    Plan pl;
    if (!make_plan(d, g, &pl)) return set_error(GATLAS_ERR_UNSUPPORTED, "matmul: tensor-core engine %d not built", d->engine);
    int rc = check_ws(pl, ws, ws_bytes);
    if (rc) return rc;
    if (g.K == 0) return set_error(GATLAS_ERR_INVALID, "matmul: K == 0 has no prepared operands");
    const WsPtrs w = ws_ptrs(pl, const_cast<void *>(ws));
    switch (pl.mode) {
        case 0: return launch_tc<0>(g, pl, w, C, d->alpha, d->beta, d->gemm, (int)d->extra, stream);
        case 1: return launch_tc<1>(g, pl, w, C, d->alpha, d->beta, d->gemm, (int)d->extra, stream);
        case 2: return launch_tc<2>(g, pl, w, C, d->alpha, d->beta, d->gemm, (int)d->extra, stream);
        default: return launch_tc<3>(g, pl, w, C, d->alpha, d->beta, d->gemm, (int)d->extra, stream);
    }
}

// ---------------------------------------------------------------------------
// host-buffer contraction: uploads, preparation and contraction, and
// downloads of row blocks of A run on three streams, one per role, so that
// the host link carries uploads back to back while earlier blocks are
// contracted and their C rows travel back
// ---------------------------------------------------------------------------
// Rows of A per pipelined block: a multiple of 256 (CTA pairs) and of 128
// (FP8 scale blocks); option "host_block_rows".
static int64_t g_host_block_rows = 512;

// Prepares rows [r0, r1) of A (K-major pieces or codes and scales).
static int prepare_a_rows(const Plan &pl, const Geometry &g, const float *A, int64_t r0, int64_t r1,
                          const WsPtrs &w, cudaStream_t s) {
    const float *src = g.ta ? A + r0 : A + r0 * g.lda;  // stored K x M: a column block
    const int64_t rows = r1 - r0;
    if (pl.mode == 3)
        return launch_quant(g.ta, src, rows, g.K, pl.Kp, g.lda, 0, 1, static_cast<uint8_t *>(w.a[0]) + r0 * pl.Kp,
                            w.sa + (r0 / kQBlock) * pl.kblocks, s);
    __nv_bfloat16 *ap[3];
    for (int i = 0; i < 3; ++i)
        ap[i] = w.a[i] ? static_cast<__nv_bfloat16 *>(w.a[i]) + r0 * pl.Kp : nullptr;
    return launch_split(pl.np, g.ta, src, rows, g.K, pl.Kp, g.lda, 0, 1, ap, s);
}

static int prepare_b(const Plan &pl, const Geometry &g, const float *B, const WsPtrs &w, cudaStream_t s) {
    if (pl.mode == 3)
        return launch_quant(!g.tb, B, g.N, g.K, pl.Kp, g.ldb, 0, 1, static_cast<uint8_t *>(w.b[0]), w.sb, s);
    __nv_bfloat16 *bp[3];
    for (int i = 0; i < 3; ++i) bp[i] = static_cast<__nv_bfloat16 *>(w.b[i]);
    return launch_split(pl.np, !g.tb, B, g.N, g.K, pl.Kp, g.ldb, 0, 1, bp, s);
}

// Contracts rows [r0, r1) of A against all of B into rows [r0, r1) of C.
static int run_rows(const gatlas_matmul_desc *d, const Plan &pl, const Geometry &g, const WsPtrs &w, int64_t r0,
                    int64_t r1, float *C, cudaStream_t s) {
    Geometry gb = g;
    gb.M = r1 - r0;
    Plan pb = pl;
    pb.mblocks = (gb.M + kQBlock - 1) / kQBlock;
    WsPtrs wb = w;
    for (int i = 0; i < 3; ++i)
        if (wb.a[i]) wb.a[i] = static_cast<uint8_t *>(wb.a[i]) + r0 * pl.Kp * pl.elem;
    if (wb.sa) wb.sa += (r0 / kQBlock) * pl.kblocks;
    if (pl.mode == 3) {  // the block's tiles in the plan of the whole product
        const int64_t first = (r0 / BM) * ((g.N + BN - 1) / BN);
        wb.plan_nseg += first;
        wb.plan_bits += first * ((pl.kblocks + 31) / 32);
        wb.plan_q += first * pl.kblocks;
    }
    float *Cb = C + r0 * g.ldc;
    switch (pl.mode) {
        case 0: return launch_tc<0>(gb, pb, wb, Cb, d->alpha, d->beta, d->gemm, (int)d->extra, s);
        case 1: return launch_tc<1>(gb, pb, wb, Cb, d->alpha, d->beta, d->gemm, (int)d->extra, s);
        case 2: return launch_tc<2>(gb, pb, wb, Cb, d->alpha, d->beta, d->gemm, (int)d->extra, s);
        default: return launch_tc<3>(gb, pb, wb, Cb, d->alpha, d->beta, d->gemm, (int)d->extra, s);
    }
}

// Bytes of device memory the pipeline needs: copies of A, B, C and the workspace.
size_t host_pipeline_bytes(const gatlas_matmul_desc *d, const Geometry &g) {
    Plan pl;
    if (!make_plan(d, g, &pl)) return 0;
    const int64_t a_rows = g.ta ? g.K : g.M, b_rows = g.tb ? g.N : g.K;
    return round_up((size_t)(a_rows * g.lda) * 4, 1024) + round_up((size_t)(b_rows * g.ldb) * 4, 1024) +
           round_up((size_t)(g.M * g.ldc) * 4, 1024) + pl.total;
}

bool host_pipeline_ok(const gatlas_matmul_desc *d, const Geometry &g) {
    Plan pl;
    return make_plan(d, g, &pl) && g.batch == 1 && g.K > 0 && g.M >= 2 * g_host_block_rows &&
           (pl.mode != 3 || (g.K + kQBlock - 1) / kQBlock <= kMaxFp8Blocks);
}

int host_pipeline(const gatlas_matmul_desc *d, const Geometry &g, const float *hA, const float *hB, float *hC,
                  void *dev, cudaStream_t caller) {
    Plan pl;
    if (!make_plan(d, g, &pl)) return set_error(GATLAS_ERR_UNSUPPORTED, "matmul: tensor-core engine %d not built", d->engine);
    const int64_t a_rows = g.ta ? g.K : g.M, b_rows = g.tb ? g.N : g.K;
    uint8_t *base = static_cast<uint8_t *>(dev);
    float *dA = reinterpret_cast<float *>(base);
    float *dB = reinterpret_cast<float *>(base + round_up((size_t)(a_rows * g.lda) * 4, 1024));
    float *dC = reinterpret_cast<float *>(reinterpret_cast<uint8_t *>(dB) + round_up((size_t)(b_rows * g.ldb) * 4, 1024));
    void *ws = reinterpret_cast<uint8_t *>(dC) + round_up((size_t)(g.M * g.ldc) * 4, 1024);
    const WsPtrs w = ws_ptrs(pl, ws);
    // roles: uploads, preparation + contraction, downloads
    cudaStream_t up = pool_stream(0), comp = pool_stream(1), down = pool_stream(2);
    if (!up || !comp || !down) return set_error(GATLAS_ERR_CUDA, "matmul: library streams");
    const int64_t nblk = (g.M + g_host_block_rows - 1) / g_host_block_rows;
    std::vector<cudaEvent_t> evs;
    auto event = [&]() -> cudaEvent_t {
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
        evs.push_back(e);
        return e;
    };
    int rc = GATLAS_OK;
    auto cuda = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == GATLAS_OK) rc = set_error(GATLAS_ERR_CUDA, "matmul host path: %s: %s", what, cudaGetErrorString(e));
    };
    // rows of C (or of a row-major operand) as one linear copy when they are
    // dense: the copy engines move one large copy faster than many row copies
    auto copy_rows = [&](float *dst, const float *src, int64_t pitch, int64_t width, int64_t rows, cudaMemcpyKind kind,
                         cudaStream_t s) {
        if (pitch == width) return cudaMemcpyAsync(dst, src, (size_t)(rows * width) * 4, kind, s);
        return cudaMemcpy2DAsync(dst, pitch * 4, src, pitch * 4, width * 4, rows, kind, s);
    };
    cudaEvent_t ev_start = event(), ev_b = event(), ev_up_end = event(), ev_comp_end = event(), ev_down_end = event();
    std::vector<cudaEvent_t> ev_up(nblk), ev_done(nblk);
    for (int64_t b = 0; b < nblk; ++b) {
        ev_up[b] = event();
        ev_done[b] = event();
    }
    for (cudaEvent_t e : evs)
        if (!e) rc = set_error(GATLAS_ERR_CUDA, "matmul host path: events");
    if (!rc) {
        cuda(cudaEventRecord(ev_start, caller), "record");
        for (cudaStream_t s : {up, comp, down}) cuda(cudaStreamWaitEvent(s, ev_start, 0), "wait");
        // uploads: B, then every row block of A (and of C when beta is used), back to back
        // exact extents: the last stored row holds only the inner dimension
        const int64_t b_inner = g.tb ? g.K : g.N;
        cuda(cudaMemcpyAsync(dB, hB, (size_t)((b_rows - 1) * g.ldb + b_inner) * 4, cudaMemcpyHostToDevice, up),
             "upload B");
        cuda(cudaEventRecord(ev_b, up), "record");
        const bool read_c = d->gemm && d->beta != 0.0;
        for (int64_t b = 0; b < nblk; ++b) {
            const int64_t r0 = b * g_host_block_rows, rows = std::min(g.M, r0 + g_host_block_rows) - r0;
            if (g.ta)  // stored K x M: rows r0..r1 of op(A) are a column block of every stored row
                cuda(cudaMemcpy2DAsync(dA + r0, g.lda * 4, hA + r0, g.lda * 4, rows * 4, g.K, cudaMemcpyHostToDevice,
                                       up),
                     "upload A");
            else
                cuda(cudaMemcpyAsync(dA + r0 * g.lda, hA + r0 * g.lda, (size_t)((rows - 1) * g.lda + g.K) * 4,
                                     cudaMemcpyHostToDevice, up),
                     "upload A");
            if (read_c)
                cuda(copy_rows(dC + r0 * g.ldc, hC + r0 * g.ldc, g.ldc, g.N, rows, cudaMemcpyHostToDevice, up),
                     "upload C");
            cuda(cudaEventRecord(ev_up[b], up), "record");
        }
        // preparation and contraction, block by block as the uploads land
        cuda(cudaStreamWaitEvent(comp, ev_b, 0), "wait");
        if (!rc) rc = prepare_b(pl, g, dB, w, comp);
        for (int64_t b = 0; b < nblk && !rc; ++b) {
            const int64_t r0 = b * g_host_block_rows, r1 = std::min(g.M, r0 + g_host_block_rows);
            cuda(cudaStreamWaitEvent(comp, ev_up[b], 0), "wait");
            if (!rc) rc = prepare_a_rows(pl, g, dA, r0, r1, w, comp);
            if (!rc) rc = run_rows(d, pl, g, w, r0, r1, dC, comp);
            cuda(cudaEventRecord(ev_done[b], comp), "record");
        }
        // downloads of C, block by block as the contractions finish.  Each
        // download also waits for the next block's upload to land, so that
        // the two directions of the host link start their copies together:
        // downloads started in the middle of an upload measured about 7 %
        // slower in total on B200 (the contraction finishes well before the
        // next upload does, so this costs no time)
        for (int64_t b = 0; b < nblk && !rc; ++b) {
            const int64_t r0 = b * g_host_block_rows, rows = std::min(g.M, r0 + g_host_block_rows) - r0;
            cuda(cudaStreamWaitEvent(down, ev_done[b], 0), "wait");
            if (b + 1 < nblk) cuda(cudaStreamWaitEvent(down, ev_up[b + 1], 0), "wait");
            cuda(copy_rows(hC + r0 * g.ldc, dC + r0 * g.ldc, g.ldc, g.N, rows, cudaMemcpyDeviceToHost, down),
                 "download C");
        }
    }
    // the caller's stream resumes when every role is done (also after an
    // error, so that no copy into the library's buffers is still in flight)
    cudaEventRecord(ev_up_end, up);
    cudaEventRecord(ev_comp_end, comp);
    cudaEventRecord(ev_down_end, down);
    cudaStreamWaitEvent(caller, ev_up_end, 0);
    cudaStreamWaitEvent(caller, ev_comp_end, 0);
    cudaStreamWaitEvent(caller, ev_down_end, 0);
    for (cudaEvent_t e : evs)
        if (e) cudaEventDestroy(e);
    return rc;
}

}  // namespace tcg

size_t tc_workspace_bytes(const gatlas_matmul_desc *d, const Geometry &g) {
    tcg::Plan pl;
    if (!tcg::make_plan(d, g, &pl)) return 0;
    return pl.total;
}

int tc_supported(const gatlas_matmul_desc *d) {
    return d->engine == GATLAS_ENGINE_TC_BF16 || d->engine == GATLAS_ENGINE_TC_SPLIT3 ||
           d->engine == GATLAS_ENGINE_TC_SPLIT6 || d->engine == GATLAS_ENGINE_TC_FP8;
}

int matmul_tc(const gatlas_matmul_desc *d, const Geometry &g, const float *A, const float *B, float *C, void *ws,
              size_t ws_bytes, cudaStream_t stream) {
    using namespace tcg;
    Plan pl;
    if (!make_plan(d, g, &pl))
        return set_error(GATLAS_ERR_UNSUPPORTED, "matmul: tensor-core engine %d not built", d->engine);
    if (g.K == 0) {
        // empty contraction: C = beta*C (gemm) or 0; handled by the SIMT path
        gatlas_matmul_desc s = *d;
        s.engine = GATLAS_ENGINE_BUFFER;
        s.group_h = s.group_w = s.block_h = s.block_w = s.vector_length = 0;
        return gatlas_matmul_f32(&s, A, B, C, nullptr, 0, stream);
    }
    if (!ws) {
        ws = device_scratch(pl.total);
        if (!ws) return set_error(GATLAS_ERR_NOMEM, "matmul: scratch of %zu bytes", pl.total);
        ws_bytes = pl.total;
    }
    int rc = tc_prepare(d, g, A, B, ws, ws_bytes, stream);
    if (rc) return rc;
    return tc_run(d, g, ws, ws_bytes, C, stream);
}

}  // namespace gatlas

extern "C" int gatlas_set_option(const char *name, int64_t value) {
    using namespace gatlas;
    if (!name) return set_error(GATLAS_ERR_INVALID, "set_option: null name");
    if (std::strcmp(name, "tc_pair") == 0) {
        if (value < 0 || value > 2) return set_error(GATLAS_ERR_INVALID, "set_option: tc_pair is 0, 1 or 2");
        tcg::g_tc_pair = (int)value;
        return GATLAS_OK;
    }
    if (std::strcmp(name, "host_block_rows") == 0) {
        if (value < 256 || value > 65536 || value % 256 != 0)
            return set_error(GATLAS_ERR_INVALID, "set_option: host_block_rows is a multiple of 256 in [256, 65536]");
        tcg::g_host_block_rows = value;
        return GATLAS_OK;
    }
    if (std::strcmp(name, "tc_group_rows") == 0) {
        if (value < 128 || value > 65536 || value % 128 != 0)
            return set_error(GATLAS_ERR_INVALID, "set_option: tc_group_rows is a multiple of 128 in [128, 65536]");
        tcg::g_tc_group_rows = (int)value;
        return GATLAS_OK;
    }
    if (std::strcmp(name, "tc_l2_hint") == 0) {
        if (value < 0 || value > 1) return set_error(GATLAS_ERR_INVALID, "set_option: tc_l2_hint is 0 or 1");
        tcg::g_tc_l2_hint = (int)value;
        return GATLAS_OK;
    }
    if (std::strcmp(name, "grouped_pair") == 0) return grouped_set_pair((int)std::max<int64_t>(-1, std::min<int64_t>(value, 3)));
    return set_error(GATLAS_ERR_INVALID, "set_option: unknown option %s", name);
}

extern "C" int gatlas_get_option(const char *name, int64_t *value) {
    using namespace gatlas;
    if (!name || !value) return set_error(GATLAS_ERR_INVALID, "get_option: null argument");
    if (std::strcmp(name, "tc_pair") == 0) {
        *value = tcg::g_tc_pair;
        return GATLAS_OK;
    }
    if (std::strcmp(name, "tc_group_rows") == 0) {
        *value = tcg::g_tc_group_rows;
        return GATLAS_OK;
    }
    if (std::strcmp(name, "host_block_rows") == 0) {
        *value = tcg::g_host_block_rows;
        return GATLAS_OK;
    }
    if (std::strcmp(name, "tc_l2_hint") == 0) {
        *value = tcg::g_tc_l2_hint;
        return GATLAS_OK;
    }
    if (std::strcmp(name, "grouped_pair") == 0) {
        *value = grouped_get_pair();
        return GATLAS_OK;
    }
    return set_error(GATLAS_ERR_INVALID, "get_option: unknown option %s", name);
}

extern "C" int gatlas_matmul_tc_prepare(const gatlas_matmul_desc *d, const float *A, const float *B, void *workspace,
                                        size_t workspace_bytes, void *stream) {
    using namespace gatlas;
    if (!d) return set_error(GATLAS_ERR_INVALID, "matmul_tc_prepare: null descriptor");
    Geometry g;
    if (!resolve_geometry(d, &g)) return set_error(GATLAS_ERR_INVALID, "matmul_tc_prepare: invalid dimensions");
    if (!A || !B) return set_error(GATLAS_ERR_INVALID, "matmul_tc_prepare: null operand");
    if (g.M == 0 || g.N == 0 || g.K == 0) return GATLAS_OK;
    return tcg::tc_prepare(d, g, A, B, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" int gatlas_matmul_tc_run(const gatlas_matmul_desc *d, const void *workspace, size_t workspace_bytes,
                                    float *C, void *stream) {
    using namespace gatlas;
    if (!d) return set_error(GATLAS_ERR_INVALID, "matmul_tc_run: null descriptor");
    Geometry g;
    if (!resolve_geometry(d, &g)) return set_error(GATLAS_ERR_INVALID, "matmul_tc_run: invalid dimensions");
    if (g.M == 0 || g.N == 0) return GATLAS_OK;
    if (!C) return set_error(GATLAS_ERR_INVALID, "matmul_tc_run: null C");
    if (g.batch > 65535) return set_error(GATLAS_ERR_INVALID, "matmul_tc_run: batch > 65535");
    return tcg::tc_run(d, g, workspace, workspace_bytes, C, (cudaStream_t)stream);
}
