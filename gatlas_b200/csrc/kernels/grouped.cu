// Grouped tensor-core matmul: hundreds of instances of different shapes and
// layouts (C_i = alpha_i * op(A_i) op(B_i) + beta_i * C_i) in one persistent
// launch.
//
// No reference counterpart as one kernel: the reference batches only equal
// shapes (packedCalc, KernelMatmulBuffer.hpp:229-230) and otherwise runs one
// kernel per problem.  Design for B200:
//  1. pack pass (one launch for all instances): every FP32 operand is split
//     into BF16 pieces and written tile-major in the exact shared-memory
//     image the MMA descriptors read: A as [mt][kt][128 rows x 64 B], B as
//     [nt][kt][BN rows x 64 B], each tile 64-byte swizzled (16-byte chunk c
//     of row r stored at chunk c ^ ((r >> 1) & 3)), zero padded past M, N, K.
//     The contraction then streams every tile with one 1-D bulk copy: no
//     per-instance tensor maps;
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
constexpr int kBK = 32;                  // BF16 elements per K slice
constexpr uint32_t kRowBytes = 64;        // one K slice of one row
constexpr uint32_t kATileBytes = BM * kRowBytes;
constexpr int kDrainWarps = 8;
constexpr int kThreads = 32 * (2 + kDrainWarps);
constexpr uint32_t kTmemCols = 512;       // two accumulators of up to 256 columns
constexpr uint64_t kWaitNs = 2000000000ull;
constexpr int kPackRows = 128;            // rows per pack item

// Per-instance device record.
struct Inst {
    const float *src_a, *src_b;
    uint8_t *pa[2], *pb[2];  // packed pieces
    float *C;
    int64_t M, N, K, lda, ldb, ldc;
    int32_t ta, tb, gemm, bn, mt, nt, kt, pad;
    float alpha, beta;
};

// Self-contained record of one output tile, in the order its CTA runs it:
// the producer, the MMA issuer and the epilogue read nothing else.
struct TileRec {
    const uint8_t *a[2];  // piece tiles of this row block: [kt][128 rows x 64 B]
    const uint8_t *b[2];  // piece tiles of this column block: [kt][bn rows x 64 B]
    float *C;             // C at the tile's origin
    int64_t ldc;
    int32_t kt, bn, rows, cols;  // valid rows / columns of the tile
    float alpha, beta;
    int32_t gemm, pad;
};
static_assert(sizeof(TileRec) == 80, "tile record layout");

// Packed byte offset of 16-byte chunk c of row `row` in K slice kb.
__device__ __forceinline__ int64_t packed_offset(int64_t row, int kb, int c, int tr, int kt) {
    return ((row / tr) * kt + kb) * (int64_t)tr * kRowBytes + (row % tr) * kRowBytes +
           ((c ^ (int)((row >> 1) & 3)) << 4);
}

// ---------------------------------------------------------------------------
// pack pass
// ---------------------------------------------------------------------------
// Item space: segment s = 2*instance + operand covers rows/128 x kt items,
// ordered row block major, K slice minor.  CTA b packs the contiguous items
// [b*per_cta, (b+1)*per_cta): one binary search for its first segment, then
// an incremental walk, and neighbouring items read neighbouring memory.
template <int NP>
__global__ void __launch_bounds__(256) grouped_pack_kernel(const Inst *insts, const int64_t *seg_start, int nseg,
                                                           int64_t per_cta) {
    __shared__ float tile[kPackRows][kBK + 1];
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
    int64_t seg_end = seg_start[sgi + 1];
    for (int64_t it = it0; it < it1; ++it) {
        while (it >= seg_end) seg_end = seg_start[++sgi + 1];
        const Inst &I = insts[sgi >> 1];
        const int op = sgi & 1;
        const int64_t local = it - seg_start[sgi];
        const int kb = (int)(local % I.kt);
        const int64_t r0 = (local / I.kt) * kPackRows;
        const int64_t k0 = (int64_t)kb * kBK;
        const int64_t rows = op ? I.N : I.M;
        const int tr = op ? I.bn : BM;
        const int64_t rows_alloc = op ? (int64_t)I.nt * I.bn : (int64_t)I.mt * BM;
        const bool transposed = op ? (I.tb == 0) : (I.ta != 0);
        const float *src = op ? I.src_b : I.src_a;
        const int64_t ld = op ? I.ldb : I.lda;
        const bool vec = (ld % 4 == 0) && ((reinterpret_cast<uintptr_t>(src) & 15) == 0);
        const int64_t K = I.K;
        __syncthreads();  // the previous item's reads of the tile are done
        if (!transposed) {
            // element (r, k) at src[r*ld + k]: 8 threads x 4 consecutive k per row
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int e = i * 256 + tid;
                const int r = e >> 3, k = (e & 7) * 4;
                const int64_t gr = r0 + r, gk = k0 + k;
                float x[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                if (gr < rows) {
                    const float *ptr = src + gr * ld + gk;
                    if (vec && gk + 3 < K) {
                        const float4 q = __ldcs(reinterpret_cast<const float4 *>(ptr));
                        x[0] = q.x, x[1] = q.y, x[2] = q.z, x[3] = q.w;
                    } else {
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            if (gk + j < K) x[j] = ptr[j];
                    }
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) tile[r][k + j] = x[j];
            }
        } else {
            // element (r, k) at src[k*ld + r]: 32 threads x 4 consecutive rows per k
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int e = i * 256 + tid;
                const int k = e >> 5, r = (e & 31) * 4;
                const int64_t gr = r0 + r, gk = k0 + k;
                float x[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                if (gk < K) {
                    const float *ptr = src + gk * ld + gr;
                    if (vec && gr + 3 < rows) {
                        const float4 q = __ldcs(reinterpret_cast<const float4 *>(ptr));
                        x[0] = q.x, x[1] = q.y, x[2] = q.z, x[3] = q.w;
                    } else {
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            if (gr + j < rows) x[j] = ptr[j];
                    }
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) tile[r + j][k] = x[j];
            }
        }
        __syncthreads();
        uint8_t *const *dst = op ? I.pb : I.pa;
        for (int e = tid; e < kPackRows * 4; e += 256) {
            const int r = e >> 2, c = e & 3;
            const int64_t row = r0 + r;
            if (row >= rows_alloc) continue;
            __nv_bfloat16 pcs[8][3];
#pragma unroll
            for (int j = 0; j < 8; ++j) tcg::split_value<NP>(tile[r][c * 8 + j], pcs[j]);
            const int64_t off = packed_offset(row, kb, c, tr, I.kt);
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                uint4 u;
                uint32_t w[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    __nv_bfloat162 v = __halves2bfloat162(pcs[2 * j][i], pcs[2 * j + 1][i]);
                    w[j] = *reinterpret_cast<uint32_t *>(&v);
                }
                u.x = w[0], u.y = w[1], u.z = w[2], u.w = w[3];
                *reinterpret_cast<uint4 *>(dst[i] + off) = u;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// persistent contraction
// ---------------------------------------------------------------------------
struct Params {
    const TileRec *tiles;
    const int32_t *cta_start;  // tiles of CTA b: [cta_start[b], cta_start[b+1])
    int seg_kblocks;
    int *fault;
};

template <int MODE>
__global__ void __launch_bounds__(kThreads, 1) grouped_gemm_kernel(Params p) {
    using L = tcg::Layout<MODE>;
    using MD = tcg::Mode<MODE>;
    constexpr int S = L::STAGES;
    static_assert(L::ROW_BYTES == kRowBytes, "grouped engine stages BF16 slices of 32");
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[S], empty[S], tfull[2], tempty[2], mma_done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    __shared__ int ring_issued, ring_consumed, mma_aborted;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t_begin = p.cta_start[blockIdx.x], t_end = p.cta_start[blockIdx.x + 1];

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], kDrainWarps);
        }
        mbar_init(&mma_done, 1);
        fence_mbarrier_init();
        abort_flag = 0;
        ring_issued = ring_consumed = 0;
        mma_aborted = 0;
    }
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, kTmemCols);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
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
                const uint32_t b_bytes = (uint32_t)cur.bn * kRowBytes;
                for (int kb = 0; kb < cur.kt; ++kb, ++ring) {
                    const int s = ring % S;
                    if (!tc::wait_timed(&empty[s], ((uint32_t)(ring / S) & 1u) ^ 1u, kWaitNs, &abort_flag)) {
                        if (!abort_flag) report_fault(p.fault, kFaultTcProducerWait);
                        abort_flag = 1;
                        stop = true;
                        break;
                    }
                    mbar_arrive_expect_tx(&full[s], MD::NP * (kATileBytes + b_bytes));
                    for (int i = 0; i < MD::NP; ++i) {
                        bulk_g2s(a_tile(s, i), cur.a[i] + (int64_t)kb * kATileBytes, kATileBytes, &full[s]);
                        bulk_g2s(b_tile(s, i), cur.b[i] + (int64_t)kb * b_bytes, b_bytes, &full[s]);
                    }
                }
                cur = next;
            }
            ring_issued = ring;
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer ----
            int ring = 0, seg = 0;
            bool stop = false;
            int2 cur = make_int2(0, 0);  // (kt, bn)
            if (t_begin < t_end) cur = make_int2(p.tiles[t_begin].kt, p.tiles[t_begin].bn);
            for (int t = t_begin; t < t_end && !stop; ++t) {
                const int tn = t + 1 < t_end ? t + 1 : t;
                const int2 next = make_int2(p.tiles[tn].kt, p.tiles[tn].bn);
                const int kt = cur.x;
                const uint32_t idesc = tc::idesc_bf16_f32(BM, cur.y);
                cur = next;
                for (int kb = 0; kb < kt; ++kb, ++ring) {
                    const int b = seg & 1;
                    const bool seg_first = (kb % p.seg_kblocks) == 0;
                    const bool seg_last = (kb % p.seg_kblocks) == p.seg_kblocks - 1 || kb == kt - 1;
                    if (seg_first) {
                        if (!tc::wait_timed(&tempty[b], ((uint32_t)(seg >> 1) & 1u) ^ 1u, kWaitNs, &abort_flag)) {
                            if (!abort_flag) report_fault(p.fault, kFaultTcMmaWait);
                            abort_flag = 1;
                            stop = true;
                            break;
                        }
                        tc::fence_after_sync();
                    }
                    const int s = ring % S;
                    if (!tc::wait_timed(&full[s], (uint32_t)(ring / S) & 1u, kWaitNs, &abort_flag)) {
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
                            tc::mma_bf16(d, tc::smem_desc_kmajor(a_addr, L::SBO, L::SWIZZLE),
                                         tc::smem_desc_kmajor(b_addr, L::SBO, L::SWIZZLE), idesc,
                                         (seg_first && kk == 0 && j == 0) ? 0u : 1u);
                        }
                    }
                    tc::commit_to(&empty[s]);
                    if (seg_last) {
                        tc::commit_to(&tfull[b]);
                        ++seg;
                    }
                }
            }
            ring_consumed = ring;
            if (stop) {
                // every MMA issued before the abort completes before TMEM is freed
                mma_aborted = 1;
                tc::commit_to(&mma_done);
            }
        }
        __syncwarp();
    } else {
        // ---- drain + epilogue ----
        const int quarter = warp & 3, half = (warp - 2) >> 2;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        int seg = 0;
        bool ok = true;
        for (int t = t_begin; t < t_end && ok; ++t) {
            const TileRec *R = p.tiles + t;
            const int bn = R->bn, kt = R->kt;
            const int hw = bn >> 1;            // columns of this warp's half
            const int nchunks = hw >> 5;       // 1, 2 or 4 chunks of 32 columns
            const int nseg = (kt + p.seg_kblocks - 1) / p.seg_kblocks;
            float acc[128];
#pragma unroll
            for (int j = 0; j < 128; ++j) acc[j] = 0.0f;
            for (int sg = 0; sg < nseg; ++sg, ++seg) {
                const int b = seg & 1;
                if (!tc::wait_timed(&tfull[b], (uint32_t)(seg >> 1) & 1u, 2 * kWaitNs, &abort_flag)) {
                    if (!abort_flag) report_fault(p.fault, kFaultTcEpilogueWait);
                    abort_flag = 1;
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                const uint32_t col_base = tmem + lane_base + (uint32_t)(b * 256 + half * hw);
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    if (c < 2 * nchunks) {
                        uint32_t r[16];
                        tc::tmem_ld_32x32b_x16(col_base + (uint32_t)(c * 16), r);
                        tc::tmem_ld_wait();
#pragma unroll
                        for (int j = 0; j < 16; ++j) acc[c * 16 + j] = __fadd_rn(acc[c * 16 + j], __uint_as_float(r[j]));
                    }
                }
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[b]);
            }
            if (!ok || abort_flag) break;
            const int r = quarter * 32 + lane;
            if (r < R->rows) {
                const int left = R->cols - half * hw;
                const int ncols = left < hw ? left : hw;  // valid columns of this half
                float *cp = R->C + (int64_t)r * R->ldc + half * hw;
                const bool vec_ok = ((reinterpret_cast<uintptr_t>(cp) & 15) == 0);
                const bool gemm = R->gemm != 0;
                const float alpha = R->alpha, beta = gemm ? R->beta : 0.0f;
#pragma unroll
                for (int q = 0; q < 32; ++q) {
                    const int jc = q * 4;
                    if (jc >= ncols) break;
                    float v[4];
                    if (vec_ok && jc + 3 < ncols) {
                        float4 c4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        if (beta != 0.0f) c4 = *reinterpret_cast<const float4 *>(cp + jc);
                        const float cv[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
                        for (int e = 0; e < 4; ++e)
                            v[e] = gemm ? __fmaf_rn(alpha, acc[jc + e], beta == 0.0f ? 0.0f : beta * cv[e]) : acc[jc + e];
                        *reinterpret_cast<float4 *>(cp + jc) = make_float4(v[0], v[1], v[2], v[3]);
                    } else {
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            if (jc + e < ncols) {
                                const float bc = beta == 0.0f ? 0.0f : beta * cp[jc + e];
                                cp[jc + e] = gemm ? __fmaf_rn(alpha, acc[jc + e], bc) : acc[jc + e];
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
        // bounded waits for the copies still landing and the MMAs issued before the abort
        for (int r = ring_consumed; r < ring_issued; ++r)
            tc::wait_timed(&full[r % S], (uint32_t)(r / S) & 1u, kWaitNs, nullptr);
        if (mma_aborted) tc::wait_timed(&mma_done, 0, kWaitNs, nullptr);
    }
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
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

// Resolved geometry of one instance.
struct InstPlan {
    int64_t M, N, K, lda, ldb, ldc;
    int bn, mt, nt, kt;
    size_t a_piece, b_piece;  // bytes per piece
};

static int resolve_instance(const gatlas_grouped_instance &in, int np, int slot, InstPlan *o) {
    (void)np;
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
    o->kt = (int)((in.k + grp::kBK - 1) / grp::kBK);
    if (in.m == 0 || in.n == 0) o->mt = o->nt = 0;
    o->a_piece = round_up((size_t)o->mt * o->kt * grp::kATileBytes, 1024);
    o->b_piece = round_up((size_t)o->nt * o->kt * bn * grp::kRowBytes, 1024);
    return GATLAS_OK;
}

struct GroupedPlan {
    int engine = 0, np = 1, mode = 0;
    int count = 0;
    std::vector<gatlas_grouped_instance> in;
    std::vector<InstPlan> ip;
    std::vector<grp::Inst> host_inst;
    grp::Inst *d_inst = nullptr;
    int64_t *d_seg = nullptr;
    grp::TileRec *d_tiles = nullptr;
    int32_t *d_cta = nullptr;
    void *ws = nullptr;
    bool owns_ws = false;
    size_t ws_bytes = 0;
    int64_t ntiles = 0, nitems = 0;
    int grid = 0, nseg = 0;
    double flops = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int device = 0;
};

size_t grouped_workspace_bytes(int engine, const gatlas_grouped_instance *in, int32_t count) {
    if ((engine != GATLAS_ENGINE_TC_BF16 && engine != GATLAS_ENGINE_TC_SPLIT3) || !in || count < 0) return 0;
    const int np = engine == GATLAS_ENGINE_TC_SPLIT3 ? 2 : 1;
    size_t total = 0;
    for (int i = 0; i < count; ++i) {
        InstPlan o{};
        if (resolve_instance(in[i], np, engine_slot(engine), &o)) return 0;
        total += np * (o.a_piece + o.b_piece);
    }
    return total;
}

static void free_plan(GroupedPlan *p) {
    for (auto &g : p->graph)
        if (g) cudaGraphExecDestroy(g);
    cudaFree(p->d_inst);
    cudaFree(p->d_seg);
    cudaFree(p->d_tiles);
    cudaFree(p->d_cta);
    if (p->owns_ws) cudaFree(p->ws);
    delete p;
}

int grouped_create(int engine, const gatlas_grouped_instance *in, int32_t count, void *ws, size_t ws_bytes,
                   GroupedPlan **out) {
    if (!out) return set_error(GATLAS_ERR_INVALID, "grouped: null plan pointer");
    *out = nullptr;
    if (engine != GATLAS_ENGINE_TC_BF16 && engine != GATLAS_ENGINE_TC_SPLIT3)
        return set_error(GATLAS_ERR_UNSUPPORTED, "grouped: engine %d has no grouped kernel (tc_bf16, tc_split3)", engine);
    if (count < 0 || (count > 0 && !in)) return set_error(GATLAS_ERR_INVALID, "grouped: invalid instance list");
    GroupedPlan *p = new GroupedPlan();
    p->engine = engine;
    p->np = engine == GATLAS_ENGINE_TC_SPLIT3 ? 2 : 1;
    p->mode = engine == GATLAS_ENGINE_TC_SPLIT3 ? 1 : 0;
    p->count = count;
    p->in.assign(in, in + count);
    p->ip.resize(count);
    cudaGetDevice(&p->device);
    size_t total = 0;
    for (int i = 0; i < count; ++i) {
        int rc = resolve_instance(in[i], p->np, engine_slot(engine), &p->ip[i]);
        if (rc) {
            delete p;
            return rc;
        }
        const gatlas_grouped_instance &q = in[i];
        if (q.m > 0 && q.n > 0 && (!q.c || (q.k > 0 && (!q.a || !q.b)))) {
            delete p;
            return set_error(GATLAS_ERR_INVALID, "grouped: instance %d has a null pointer", i);
        }
        if (p->ip[i].mt > 65535 || p->ip[i].kt > (1 << 24)) {
            delete p;
            return set_error(GATLAS_ERR_INVALID, "grouped: instance %d is too large", i);
        }
        total += p->np * (p->ip[i].a_piece + p->ip[i].b_piece);
        p->flops += 2.0 * (double)q.m * (double)q.n * (double)q.k;
    }
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
    p->ws_bytes = total;

    // instance records, pack segments and output tiles
    p->host_inst.resize(std::max(count, 1));
    std::vector<int64_t> seg(2 * (size_t)count + 1, 0);
    struct Cand {
        int64_t cost;
        grp::TileRec t;
    };
    std::vector<Cand> tiles;
    uint8_t *base = static_cast<uint8_t *>(p->ws);
    size_t off = 0;
    for (int i = 0; i < count; ++i) {
        const InstPlan &o = p->ip[i];
        const gatlas_grouped_instance &q = in[i];
        grp::Inst &I = p->host_inst[i];
        std::memset(&I, 0, sizeof(I));
        I.src_a = q.a;
        I.src_b = q.b;
        for (int j = 0; j < p->np; ++j) {
            I.pa[j] = base + off + j * o.a_piece;
            I.pb[j] = base + off + p->np * o.a_piece + j * o.b_piece;
        }
        off += p->np * (o.a_piece + o.b_piece);
        I.C = q.c;
        I.M = o.M, I.N = o.N, I.K = o.K, I.lda = o.lda, I.ldb = o.ldb, I.ldc = o.ldc;
        I.ta = q.trans_a != 0, I.tb = q.trans_b != 0, I.gemm = q.gemm != 0;
        I.bn = o.bn, I.mt = o.mt, I.nt = o.nt, I.kt = o.kt;
        I.alpha = (float)q.alpha;
        I.beta = (float)q.beta;
        const int64_t a_items = o.kt ? (int64_t)o.mt * o.kt : 0;  // 128 A rows per item = one A tile row block
        const int64_t b_items = o.kt ? ((int64_t)o.nt * o.bn + grp::kPackRows - 1) / grp::kPackRows * o.kt : 0;
        seg[2 * i + 1] = seg[2 * i] + a_items;
        seg[2 * i + 2] = seg[2 * i + 1] + b_items;
        // cost in bytes moved: operand tiles through shared memory plus the C
        // tile (read too when beta != 0), plus a fixed per-tile overhead
        const int64_t c_bytes = (int64_t)grp::BM * o.bn * 4 * ((q.gemm && q.beta != 0.0) ? 2 : 1);
        const int64_t cost = (int64_t)o.kt * p->np * (grp::BM + o.bn) * grp::kRowBytes + c_bytes + 16384;
        for (int tm = 0; tm < o.mt; ++tm)
            for (int tn = 0; tn < o.nt; ++tn) {
                grp::TileRec r;
                std::memset(&r, 0, sizeof(r));
                for (int j = 0; j < p->np; ++j) {
                    r.a[j] = I.pa[j] + (size_t)tm * o.kt * grp::kATileBytes;
                    r.b[j] = I.pb[j] + (size_t)tn * o.kt * o.bn * grp::kRowBytes;
                }
                r.C = q.c + (int64_t)tm * grp::BM * o.ldc + (int64_t)tn * o.bn;
                r.ldc = o.ldc;
                r.kt = o.kt;
                r.bn = o.bn;
                r.rows = (int32_t)std::min<int64_t>(grp::BM, o.M - (int64_t)tm * grp::BM);
                r.cols = (int32_t)std::min<int64_t>(o.bn, o.N - (int64_t)tn * o.bn);
                r.alpha = (float)q.alpha;
                r.beta = (float)q.beta;
                r.gemm = q.gemm != 0;
                tiles.push_back(Cand{cost, r});
            }
    }
    p->nseg = 2 * count;
    p->nitems = seg.back();
    p->ntiles = (int64_t)tiles.size();
    // longest first onto the least-loaded CTA
    std::stable_sort(tiles.begin(), tiles.end(), [](const Cand &a, const Cand &b) { return a.cost > b.cost; });
    p->grid = (int)std::min<int64_t>(sm_count(), std::max<int64_t>(p->ntiles, 1));
    std::vector<std::vector<grp::TileRec>> per(p->grid);
    {
        using E = std::pair<int64_t, int>;
        std::priority_queue<E, std::vector<E>, std::greater<E>> heap;
        for (int b = 0; b < p->grid; ++b) heap.push({0, b});
        for (const Cand &c : tiles) {
            E e = heap.top();
            heap.pop();
            per[e.second].push_back(c.t);
            heap.push({e.first + c.cost, e.second});
        }
    }
    std::vector<grp::TileRec> flat;
    std::vector<int32_t> cta(p->grid + 1, 0);
    flat.reserve(tiles.size());
    for (int b = 0; b < p->grid; ++b) {
        cta[b] = (int32_t)flat.size();
        flat.insert(flat.end(), per[b].begin(), per[b].end());
    }
    cta[p->grid] = (int32_t)flat.size();
    if (flat.empty()) flat.push_back(grp::TileRec{});
    bool ok = cudaMalloc(&p->d_inst, p->host_inst.size() * sizeof(grp::Inst)) == cudaSuccess &&
              cudaMalloc(&p->d_seg, seg.size() * sizeof(int64_t)) == cudaSuccess &&
              cudaMalloc(&p->d_tiles, flat.size() * sizeof(grp::TileRec)) == cudaSuccess &&
              cudaMalloc(&p->d_cta, cta.size() * sizeof(int32_t)) == cudaSuccess;
    ok = ok && cudaMemcpy(p->d_inst, p->host_inst.data(), p->host_inst.size() * sizeof(grp::Inst),
                          cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(p->d_seg, seg.data(), seg.size() * sizeof(int64_t), cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(p->d_tiles, flat.data(), flat.size() * sizeof(grp::TileRec), cudaMemcpyHostToDevice) ==
                   cudaSuccess;
    ok = ok && cudaMemcpy(p->d_cta, cta.data(), cta.size() * sizeof(int32_t), cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        free_plan(p);
        return set_error(GATLAS_ERR_NOMEM, "grouped: device tables");
    }
    *out = p;
    return GATLAS_OK;
}

int grouped_prepare(GroupedPlan *p, cudaStream_t stream) {
    if (!p) return set_error(GATLAS_ERR_INVALID, "grouped: null plan");
    if (p->nitems == 0) return GATLAS_OK;
    const int64_t grid = std::min<int64_t>(p->nitems, (int64_t)sm_count() * 8);
    const int64_t per_cta = (p->nitems + grid - 1) / grid;
    if (p->np == 2)
        grp::grouped_pack_kernel<2><<<(unsigned)grid, 256, 0, stream>>>(p->d_inst, p->d_seg, p->nseg, per_cta);
    else
        grp::grouped_pack_kernel<1><<<(unsigned)grid, 256, 0, stream>>>(p->d_inst, p->d_seg, p->nseg, per_cta);
    return check_launch("grouped_pack_kernel");
}

template <int MODE>
static int launch_grouped(GroupedPlan *p, int seg_kblocks, cudaStream_t stream) {
    using L = tcg::Layout<MODE>;
    grp::Params prm;
    prm.tiles = p->d_tiles;
    prm.cta_start = p->d_cta;
    prm.seg_kblocks = seg_kblocks > 0 ? seg_kblocks : tcg::kDefaultSegKblocks;
    prm.fault = device_fault_word();
    const int smem = (int)L::SMEM_BYTES;
    cudaError_t e = cudaFuncSetAttribute(grp::grouped_gemm_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "grouped smem attribute: %s", cudaGetErrorString(e));
    grp::grouped_gemm_kernel<MODE><<<p->grid, grp::kThreads, smem, stream>>>(prm);
    return check_launch("grouped_gemm_kernel");
}

int grouped_run(GroupedPlan *p, cudaStream_t stream) {
    if (!p) return set_error(GATLAS_ERR_INVALID, "grouped: null plan");
    if (p->ntiles == 0) return GATLAS_OK;
    return p->mode == 1 ? launch_grouped<1>(p, 0, stream) : launch_grouped<0>(p, 0, stream);
}

int grouped_launch_graph(GroupedPlan *p, int with_prepare, cudaStream_t stream) {
    if (!p) return set_error(GATLAS_ERR_INVALID, "grouped: null plan");
    const int slot = with_prepare ? 1 : 0;
    if (!p->graph[slot]) {
        cudaStream_t cap;
        if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
            return set_error(GATLAS_ERR_CUDA, "grouped: capture stream");
        // attribute changes are not captured: set them before the capture
        cudaFuncSetAttribute(grp::grouped_gemm_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tcg::Layout<0>::SMEM_BYTES);
        cudaFuncSetAttribute(grp::grouped_gemm_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tcg::Layout<1>::SMEM_BYTES);
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
    d.engine = p->engine;
    d.gemm = q.gemm;
    d.trans_a = q.trans_a;
    d.trans_b = q.trans_b;
    d.m = q.m, d.n = q.n, d.k = q.k;
    d.lda = p->ip[i].lda, d.ldb = p->ip[i].ldb, d.ldc = p->ip[i].ldc;
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
    if (tiles) *tiles = p->ntiles;
    if (ctas) *ctas = p->grid;
    if (flops) *flops = p->flops;
    if (items) *items = p->nitems;
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
