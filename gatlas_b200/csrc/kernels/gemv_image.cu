// GEMV image engine: A streamed through shared memory by TMA tensor-map loads.
//
// Reference: KernelMatvecImage<SCALAR,VL> (KernelMatvecImage.hpp:188-295)
// reads A and b through read_imagef texture fetches, one work item per
// blockHeight rows.  On B200 the "image" path is the TMA engine: a 2-D
// tensor map describes A, and tiles of it land in shared memory through an
// mbarrier ring; warps compute from shared memory.
//
//  * row-major A (y = A·x): persistent CTAs take blocks of 16 rows; a
//    producer warp streams 16 x 256-element boxes of A and the matching
//    256-element chunk of x (1-D bulk copy) through an 8-stage ring; each of
//    8 consumer warps owns 2 rows, accumulates fmaf chains per lane and
//    reduces with a fixed butterfly at the end of the row block.
//  * column-major A (y = A^T·x): a CTA owns 256 columns and a segment of the
//    rows; boxes of 32 rows x 256 columns stream through a 4-stage ring, lane l
//    of every warp owns columns 8l..8l+7, warps take interleaved rows, and the
//    partial sums are combined across warps in shared memory and across
//    segments as in the buffer engine (fixed order, last CTA per column block).
// Every wait is bounded (fault word on timeout).  Float only; the operand
// must have 16-byte aligned rows (lda % 4 == 0) and 16-byte aligned bases.
#include <cuda.h>

#include <algorithm>

#include "../common.cuh"
#include "../device_state.cuh"
#include "../tcgen05.cuh"
#include "../tma.hpp"

namespace gatlas {
namespace gvi {

constexpr int kConsumerWarps = 8;
constexpr int kThreads = 32 * (kConsumerWarps + 1);  // + producer warp
constexpr uint64_t kWaitNs = 1000000000ull;

// ---- row-major -------------------------------------------------------------
constexpr int RB = 16;     // rows per block (box height)
constexpr int RC = 256;    // columns per chunk (box width)
constexpr int RS = 8;      // stages
constexpr uint32_t kRowTile = RB * RC * 4;   // 16 KiB
constexpr uint32_t kRowStage = kRowTile + RC * 4;

struct RowArgs {
    float *y;
    const float *x;
    int64_t M, N;
    float alpha, beta;
    int gemv;
    int *fault;
};

__global__ void __launch_bounds__(kThreads, 1)
    gemv_rows_tma_kernel(const __grid_constant__ CUtensorMap tmA, RowArgs a) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[RS], empty[RS];
    __shared__ volatile int abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t nblocks = (a.M + RB - 1) / RB;
    const int64_t nchunks = (a.N + RC - 1) / RC;
    // this CTA's row blocks: blockIdx.x, +gridDim.x, ...
    const int64_t my_blocks = blockIdx.x < nblocks ? (nblocks - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const int64_t items = my_blocks * nchunks;
    if (threadIdx.x == 0) {
        for (int s = 0; s < RS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kConsumerWarps);
        }
        fence_mbarrier_init();
        abort_flag = 0;
        prefetch_tmap(&tmA);
    }
    __syncthreads();

    if (warp == kConsumerWarps) {
        if (lane == 0) {
            int64_t it = 0;
            for (; it < items; ++it) {
                const int s = (int)(it % RS);
                const uint32_t ph = (uint32_t)(it / RS) & 1u;
                if (!tc::wait_timed(&empty[s], ph ^ 1u, kWaitNs, &abort_flag)) {
                    if (!abort_flag) report_fault(a.fault, kFaultGemvTmaWait);
                    abort_flag = 1;
                    break;
                }
                const int64_t rb = blockIdx.x + (it / nchunks) * gridDim.x, c = it % nchunks;
                const int64_t c0 = c * RC;
                const uint32_t xbytes = (uint32_t)((a.N - c0 < RC ? a.N - c0 : RC) * 4);
                uint8_t *st = smem + s * kRowStage;
                mbar_arrive_expect_tx(&full[s], kRowTile + xbytes);
                tma_load_2d(st, &tmA, (int32_t)c0, (int32_t)(rb * RB), &full[s]);
                bulk_g2s(st + kRowTile, a.x + c0, xbytes, &full[s]);
            }
            // the last load issued into each stage has landed before the CTA can exit
            for (int64_t k = it > RS ? it - RS : 0; k < it; ++k)
                tc::wait_timed(&full[k % RS], (uint32_t)(k / RS) & 1u, kWaitNs, nullptr);
        }
        return;
    }

    // consumers: warp w owns rows 2w, 2w+1 of each block
    float acc0 = 0.f, acc1 = 0.f;
    for (int64_t it = 0; it < items; ++it) {
        const int s = (int)(it % RS);
        const uint32_t ph = (uint32_t)(it / RS) & 1u;
        if (!tc::wait_timed(&full[s], ph, kWaitNs, &abort_flag)) {
            if (!abort_flag) report_fault(a.fault, kFaultGemvTmaWait);
            abort_flag = 1;
            break;
        }
        const int64_t c = it % nchunks;
        const int64_t c0 = c * RC;
        const float *tile = reinterpret_cast<const float *>(smem + s * kRowStage);
        const float *xs = reinterpret_cast<const float *>(smem + s * kRowStage + kRowTile);
        const bool last = (c == nchunks - 1);
#pragma unroll
        for (int j = 0; j < RC / 128; ++j) {
            const int col = j * 128 + lane * 4;
            if (!last || c0 + col < a.N) {  // N % 4 == 0: a vector is all in or all out
                const float4 xv = *reinterpret_cast<const float4 *>(xs + col);
                const float4 a0 = *reinterpret_cast<const float4 *>(tile + (2 * warp) * RC + col);
                const float4 a1 = *reinterpret_cast<const float4 *>(tile + (2 * warp + 1) * RC + col);
                acc0 = __fmaf_rn(a0.x, xv.x, acc0);
                acc0 = __fmaf_rn(a0.y, xv.y, acc0);
                acc0 = __fmaf_rn(a0.z, xv.z, acc0);
                acc0 = __fmaf_rn(a0.w, xv.w, acc0);
                acc1 = __fmaf_rn(a1.x, xv.x, acc1);
                acc1 = __fmaf_rn(a1.y, xv.y, acc1);
                acc1 = __fmaf_rn(a1.z, xv.z, acc1);
                acc1 = __fmaf_rn(a1.w, xv.w, acc1);
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (last) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                acc0 += __shfl_xor_sync(0xffffffffu, acc0, off);
                acc1 += __shfl_xor_sync(0xffffffffu, acc1, off);
            }
            const int64_t rb = blockIdx.x + (it / nchunks) * gridDim.x;
            if (lane < 2) {
                const int64_t row = rb * RB + 2 * warp + lane;
                const float v = lane == 0 ? acc0 : acc1;
                if (row < a.M) {
                    float out = v;
                    if (a.gemv) {
                        const float bc = (a.beta == 0.f) ? 0.f : a.beta * a.y[row];
                        out = __fmaf_rn(a.alpha, v, bc);
                    }
                    a.y[row] = out;
                }
            }
            acc0 = acc1 = 0.f;
        }
    }
}

// ---- column-major --------------------------------------------------------
constexpr int CC = 256;    // columns per block (box width)
constexpr int CR = 32;     // rows per box
constexpr int CS = 4;      // stages
constexpr uint32_t kColTile = CC * CR * 4;  // 32 KiB
constexpr uint32_t kColStage = kColTile + CR * 4;

struct ColArgs {
    float *y;
    const float *x;
    int64_t M, N;
    int64_t seg_len;
    int nseg;
    float alpha, beta;
    int gemv;
    float *partial;
    unsigned *counters;
    int *fault;
};

__global__ void __launch_bounds__(kThreads, 1)
    gemv_cols_tma_kernel(const __grid_constant__ CUtensorMap tmA, ColArgs a) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[CS], empty[CS];
    __shared__ volatile int abort_flag;
    __shared__ __align__(16) float red[kConsumerWarps][CC];
    __shared__ unsigned ticket;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t cb = blockIdx.x, seg = blockIdx.y;
    const int64_t col0 = cb * CC;
    const int64_t j0 = seg * a.seg_len;
    const int64_t j1 = (j0 + a.seg_len < a.N) ? j0 + a.seg_len : a.N;
    const int64_t nboxes = j1 > j0 ? (j1 - j0 + CR - 1) / CR : 0;
    if (threadIdx.x == 0) {
        for (int s = 0; s < CS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kConsumerWarps);
        }
        fence_mbarrier_init();
        abort_flag = 0;
        prefetch_tmap(&tmA);
    }
    __syncthreads();

    float acc[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) acc[v] = 0.f;
    if (warp == kConsumerWarps) {
        if (lane == 0) {
            int64_t b = 0;
            for (; b < nboxes; ++b) {
                const int s = (int)(b % CS);
                const uint32_t ph = (uint32_t)(b / CS) & 1u;
                if (!tc::wait_timed(&empty[s], ph ^ 1u, kWaitNs, &abort_flag)) {
                    if (!abort_flag) report_fault(a.fault, kFaultGemvTmaWait);
                    abort_flag = 1;
                    break;
                }
                const int64_t r0 = j0 + b * CR;
                const int64_t rows = (j1 - r0 < CR) ? j1 - r0 : CR;
                // x rows of the box: copy whole 16-byte groups, the tail is masked
                const uint32_t xbytes = (uint32_t)(((rows * 4) + 15) / 16 * 16);
                uint8_t *st = smem + s * kColStage;
                const bool x_in = (r0 * 4) % 16 == 0 && (uint64_t)(r0 * 4 + xbytes) <= (uint64_t)(a.N * 4);
                mbar_arrive_expect_tx(&full[s], kColTile + (x_in ? xbytes : 0));
                tma_load_2d(st, &tmA, (int32_t)col0, (int32_t)r0, &full[s]);
                if (x_in) bulk_g2s(st + kColTile, a.x + r0, xbytes, &full[s]);
            }
            for (int64_t k = b > CS ? b - CS : 0; k < b; ++k)
                tc::wait_timed(&full[k % CS], (uint32_t)(k / CS) & 1u, kWaitNs, nullptr);
        }
    } else {
        for (int64_t b = 0; b < nboxes; ++b) {
            const int s = (int)(b % CS);
            const uint32_t ph = (uint32_t)(b / CS) & 1u;
            if (!tc::wait_timed(&full[s], ph, kWaitNs, &abort_flag)) {
                if (!abort_flag) report_fault(a.fault, kFaultGemvTmaWait);
                abort_flag = 1;
                break;
            }
            const int64_t r0 = j0 + b * CR;
            const int64_t rows = (j1 - r0 < CR) ? j1 - r0 : CR;
            const float *tile = reinterpret_cast<const float *>(smem + s * kColStage);
            const float *xs = reinterpret_cast<const float *>(smem + s * kColStage + kColTile);
            const bool x_in = (r0 * 4) % 16 == 0 && (uint64_t)(r0 * 4 + (((rows * 4) + 15) / 16 * 16)) <=
                                                         (uint64_t)(a.N * 4);
            for (int r = warp; r < rows; r += kConsumerWarps) {
                const float xv = x_in ? xs[r] : __ldg(a.x + r0 + r);
                const float4 v0 = *reinterpret_cast<const float4 *>(tile + r * CC + lane * 8);
                const float4 v1 = *reinterpret_cast<const float4 *>(tile + r * CC + lane * 8 + 4);
                acc[0] = __fmaf_rn(v0.x, xv, acc[0]);
                acc[1] = __fmaf_rn(v0.y, xv, acc[1]);
                acc[2] = __fmaf_rn(v0.z, xv, acc[2]);
                acc[3] = __fmaf_rn(v0.w, xv, acc[3]);
                acc[4] = __fmaf_rn(v1.x, xv, acc[4]);
                acc[5] = __fmaf_rn(v1.y, xv, acc[5]);
                acc[6] = __fmaf_rn(v1.z, xv, acc[6]);
                acc[7] = __fmaf_rn(v1.w, xv, acc[7]);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
        }
#pragma unroll
        for (int v = 0; v < 8; ++v) red[warp][lane * 8 + v] = acc[v];
    }
    __syncthreads();
    if (warp != 0 || abort_flag) return;
    float tot[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
        float t = red[0][lane * 8 + v];
#pragma unroll
        for (int w = 1; w < kConsumerWarps; ++w) t += red[w][lane * 8 + v];
        tot[v] = t;
    }
    auto finish = [&](int v, float t) {
        const int64_t col = col0 + lane * 8 + v;
        if (col >= a.M) return;
        float out = t;
        if (a.gemv) {
            const float bc = (a.beta == 0.f) ? 0.f : a.beta * a.y[col];
            out = __fmaf_rn(a.alpha, t, bc);
        }
        a.y[col] = out;
    };
    if (a.nseg == 1) {
#pragma unroll
        for (int v = 0; v < 8; ++v) finish(v, tot[v]);
        return;
    }
    float *part = a.partial + seg * a.M;
#pragma unroll
    for (int v = 0; v < 8; ++v)
        if (col0 + lane * 8 + v < a.M) part[col0 + lane * 8 + v] = tot[v];
    __threadfence();
    __syncwarp();
    if (lane == 0) ticket = atomicAdd(a.counters + cb, 1u);
    __syncwarp();
    if (ticket != (unsigned)(a.nseg - 1)) return;
    __threadfence();
#pragma unroll
    for (int v = 0; v < 8; ++v) {
        const int64_t col = col0 + lane * 8 + v;
        if (col >= a.M) continue;
        float t = 0.f;
        for (int ss = 0; ss < a.nseg; ++ss) {
            const float pv = __ldcg(a.partial + (int64_t)ss * a.M + col);
            t = (ss == 0) ? pv : t + pv;
        }
        finish(v, t);
    }
}

// Row segments per column block of the column-major kernel.  One CTA per SM
// at a time runs ceil(ncb * nseg / sms) rounds of seg_len rows plus a fixed
// cost per CTA (ring fill, partial sums; about 128 rows' worth), so the
// segment count chosen is the one whose rounds waste the least SM time
// (fewest segments among equals).  64 column blocks of 16384 rows on 148 SMs:
// 9 segments in 4 rounds rather than 5 segments in 3 rounds, the last of them
// one-sixth full.  The workspace query and the launch both call this, so a
// workspace sized by the query always fits the launch.
struct ColSegments {
    int64_t ncb, nseg, seg_len;
    size_t part_bytes, cnt_bytes;  // both 0 when nseg == 1 (no partial sums)
};

ColSegments col_segments(int64_t M, int64_t N, int sms) {
    ColSegments s{(M + CC - 1) / CC, 1, 0, 0, 0};
    const int64_t max_seg = std::min<int64_t>((N + CR - 1) / CR, 256);
    double best = -1.0;
    for (int64_t cand = 1; cand <= max_seg; ++cand) {
        int64_t len = (N + cand - 1) / cand;
        len = (len + CR - 1) / CR * CR;  // whole boxes per segment
        const int64_t segs = (N + len - 1) / len;
        const int64_t rounds = (s.ncb * segs + sms - 1) / sms;
        const double eff = (double)(s.ncb * N) / ((double)sms * (double)rounds * (double)(len + 128));
        if (eff > best + 1e-3) {
            best = eff;
            s.nseg = segs;
            s.seg_len = len;
        }
    }
    if (s.nseg > 1) {
        s.part_bytes = ((size_t)s.nseg * M * 4 + 255) & ~(size_t)255;
        s.cnt_bytes = ((size_t)s.ncb * 4 + 255) & ~(size_t)255;
    }
    return s;
}

}  // namespace gvi

size_t matvec_image_ws_bytes(const gatlas_matvec_desc *d) {
    using namespace gvi;
    if (!d || !d->trans_a || d->n == 0 || d->m == 0) return 0;
    const ColSegments s = col_segments((int64_t)d->m, (int64_t)d->n, sm_count());
    return s.part_bytes + s.cnt_bytes;
}

int matvec_image_f32(const gatlas_matvec_desc *d, const float *A, const float *x, float *y, void *ws,
                     size_t ws_bytes, cudaStream_t stream) {
    using namespace gvi;
    if (d->m == 0) return GATLAS_OK;
    if (!A || !x || !y) return set_error(GATLAS_ERR_INVALID, "matvec: null pointer");
    const size_t batch = d->batch ? d->batch : 1;
    if (batch != 1) return set_error(GATLAS_ERR_UNSUPPORTED, "matvec image engine: batch must be 1");
    const int64_t M = (int64_t)d->m, N = (int64_t)d->n;
    const int64_t lda = d->lda ? (int64_t)d->lda : (d->trans_a ? M : N);
    const int64_t inner = d->trans_a ? M : N;
    if (lda < inner) return set_error(GATLAS_ERR_INVALID, "matvec: lda too small");
    if (lda % 4 || !aligned16(A) || !aligned16(x) || inner % 4)
        return set_error(GATLAS_ERR_UNSUPPORTED,
                         "matvec image engine: needs 16-byte aligned rows (lda and the inner dimension multiples of 4)");
    if (N == 0) {
        gatlas_matvec_desc b = *d;
        b.engine = GATLAS_ENGINE_BUFFER;
        return gatlas_matvec_f32(&b, A, x, y, ws, ws_bytes, stream);
    }
    CUtensorMap tm;
    const uint64_t dims[2] = {(uint64_t)inner, (uint64_t)(d->trans_a ? N : M)};
    const uint64_t strides[1] = {(uint64_t)lda * 4};
    const int sms = sm_count();
    if (!d->trans_a) {
        const uint32_t box[2] = {RC, RB};
        int rc = make_tensor_map(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(A), dims, strides, box,
                                 CU_TENSOR_MAP_SWIZZLE_NONE);
        if (rc) return rc;
        RowArgs a{y, x, M, N, (float)d->alpha, (float)d->beta, d->gemv, device_fault_word()};
        const int smem = RS * (int)kRowStage;
        cudaFuncSetAttribute(gemv_rows_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        const int64_t nblocks = (M + RB - 1) / RB;
        const int grid = (int)(nblocks < sms ? nblocks : sms);
        gemv_rows_tma_kernel<<<grid, kThreads, smem, stream>>>(tm, a);
        return check_launch("gemv_rows_tma_kernel");
    }
    const uint32_t box[2] = {CC, CR};
    int rc = make_tensor_map(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(A), dims, strides, box,
                             CU_TENSOR_MAP_SWIZZLE_NONE);
    if (rc) return rc;
    const ColSegments seg = col_segments(M, N, sms);
    const int64_t ncb = seg.ncb, nseg = seg.nseg, seg_len = seg.seg_len;
    float *partial = nullptr;
    unsigned *counters = nullptr;
    if (nseg > 1) {
        const size_t part_bytes = seg.part_bytes, cnt_bytes = seg.cnt_bytes;
        if (!ws) {
            ws = device_scratch(part_bytes + cnt_bytes);
            if (!ws) return set_error(GATLAS_ERR_NOMEM, "matvec: scratch");
        } else if (ws_bytes < part_bytes + cnt_bytes || !aligned_to(ws, 256)) {
            return set_error(GATLAS_ERR_INVALID, "matvec: workspace too small or not 256-byte aligned");
        }
        partial = static_cast<float *>(ws);
        counters = reinterpret_cast<unsigned *>(static_cast<char *>(ws) + part_bytes);
        cudaError_t e = cudaMemsetAsync(counters, 0, cnt_bytes, stream);
        if (e != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "matvec: %s", cudaGetErrorString(e));
    }
    ColArgs a{y, x, M, N, seg_len, (int)nseg, (float)d->alpha, (float)d->beta, d->gemv, partial, counters,
              device_fault_word()};
    const int smem = CS * (int)kColStage;
    cudaFuncSetAttribute(gemv_cols_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    dim3 grid((unsigned)ncb, (unsigned)nseg);
    gemv_cols_tma_kernel<<<grid, kThreads, smem, stream>>>(tm, a);
    return check_launch("gemv_cols_tma_kernel");
}

}  // namespace gatlas
