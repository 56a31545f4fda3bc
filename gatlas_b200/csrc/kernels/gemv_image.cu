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
// Every wait is bounded (fault word on timeout).  Float and double (the
// reference's floatimg and doubleimg, KernelMatvecImage.hpp:61-65): a box row
// is 1 KiB (256 floats or 128 doubles) and every shared-memory read a 16-byte
// vector, so the operand needs 16-byte aligned rows (lda a multiple of 4
// floats or 2 doubles) and a 16-byte aligned base.
#include <cuda.h>
#include <string.h>

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

// Element-type traits: every box row is 1 KiB and every shared-memory read a
// 16-byte vector (float4 of floats or double2 of doubles).
template <typename T>
struct Elem {
    static constexpr int V = 16 / (int)sizeof(T);         // elements per 16-byte vector
    static constexpr int ROW = 1024 / (int)sizeof(T);     // elements per 1 KiB box row
};
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
template <typename T>
__device__ __forceinline__ void ld16(const T *p, T (&v)[Elem<T>::V]) {
    const uint4 raw = *reinterpret_cast<const uint4 *>(p);
    memcpy(v, &raw, 16);
}

// ---- row-major -------------------------------------------------------------
constexpr int RB = 16;     // rows per block (box height)
constexpr int RS = 8;      // stages
constexpr uint32_t kRowTile = RB * 1024;   // 16 KiB
constexpr uint32_t kRowStage = kRowTile + 1024;

template <typename T>
struct RowArgs {
    T *y;
    const T *x;
    int64_t M, N;
    T alpha, beta;
    int gemv;
    int *fault;
};

template <typename T>
__global__ void __launch_bounds__(kThreads, 1)
    gemv_rows_tma_kernel(const __grid_constant__ CUtensorMap tmA, RowArgs<T> a) {
    constexpr int RC = Elem<T>::ROW, V = Elem<T>::V;
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
                const uint32_t xbytes = (uint32_t)((a.N - c0 < RC ? a.N - c0 : RC) * (int64_t)sizeof(T));
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

    // consumers: warp w owns rows 2w, 2w+1 of each block; lane l reads the
    // 16-byte vectors l, l + 32 of every chunk
    T acc0 = T(0), acc1 = T(0);
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
        const T *tile = reinterpret_cast<const T *>(smem + s * kRowStage);
        const T *xs = reinterpret_cast<const T *>(smem + s * kRowStage + kRowTile);
        const bool last = (c == nchunks - 1);
#pragma unroll
        for (int j = 0; j < RC / (32 * V); ++j) {
            const int col = j * 32 * V + lane * V;
            if (!last || c0 + col < a.N) {  // N % V == 0: a vector is all in or all out
                T xv[V], a0[V], a1[V];
                ld16(xs + col, xv);
                ld16(tile + (2 * warp) * RC + col, a0);
                ld16(tile + (2 * warp + 1) * RC + col, a1);
#pragma unroll
                for (int e = 0; e < V; ++e) acc0 = fma_rn(a0[e], xv[e], acc0);
#pragma unroll
                for (int e = 0; e < V; ++e) acc1 = fma_rn(a1[e], xv[e], acc1);
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
                const T v = lane == 0 ? acc0 : acc1;
                if (row < a.M) {
                    T out = v;
                    if (a.gemv) {
                        const T bc = (a.beta == T(0)) ? T(0) : a.beta * a.y[row];
                        out = fma_rn(a.alpha, v, bc);
                    }
                    a.y[row] = out;
                }
            }
            acc0 = acc1 = T(0);
        }
    }
}

// ---- column-major --------------------------------------------------------
constexpr int CR = 32;     // rows per box
constexpr int CS = 4;      // stages
constexpr uint32_t kColTile = CR * 1024;  // 32 KiB
constexpr uint32_t kColStage = kColTile + CR * 8;

template <typename T>
struct ColArgs {
    T *y;
    const T *x;
    int64_t M, N;
    int64_t seg_len;
    int nseg;
    T alpha, beta;
    int gemv;
    T *partial;
    unsigned *counters;
    int *fault;
};

template <typename T>
__global__ void __launch_bounds__(kThreads, 1)
    gemv_cols_tma_kernel(const __grid_constant__ CUtensorMap tmA, ColArgs<T> a) {
    constexpr int CC = Elem<T>::ROW;          // columns per block (box width)
    constexpr int EPL = CC / 32;              // columns per lane: two 16-byte vectors
    constexpr int V = Elem<T>::V;
    constexpr int TS = (int)sizeof(T);
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[CS], empty[CS];
    __shared__ volatile int abort_flag;
    __shared__ __align__(16) T red[kConsumerWarps][CC];
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

    T acc[EPL];
#pragma unroll
    for (int v = 0; v < EPL; ++v) acc[v] = T(0);
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
                const uint32_t xbytes = (uint32_t)(((rows * TS) + 15) / 16 * 16);
                uint8_t *st = smem + s * kColStage;
                const bool x_in = (r0 * TS) % 16 == 0 && (uint64_t)(r0 * TS + xbytes) <= (uint64_t)(a.N * TS);
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
            const T *tile = reinterpret_cast<const T *>(smem + s * kColStage);
            const T *xs = reinterpret_cast<const T *>(smem + s * kColStage + kColTile);
            const bool x_in = (r0 * TS) % 16 == 0 && (uint64_t)(r0 * TS + (((rows * TS) + 15) / 16 * 16)) <=
                                                          (uint64_t)(a.N * TS);
            for (int r = warp; r < rows; r += kConsumerWarps) {
                const T xv = x_in ? xs[r] : __ldg(a.x + r0 + r);
                T v0[V], v1[V];
                ld16(tile + r * CC + lane * EPL, v0);
                ld16(tile + r * CC + lane * EPL + V, v1);
#pragma unroll
                for (int e = 0; e < V; ++e) acc[e] = fma_rn(v0[e], xv, acc[e]);
#pragma unroll
                for (int e = 0; e < V; ++e) acc[V + e] = fma_rn(v1[e], xv, acc[V + e]);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
        }
#pragma unroll
        for (int v = 0; v < EPL; ++v) red[warp][lane * EPL + v] = acc[v];
    }
    __syncthreads();
    if (warp != 0 || abort_flag) return;
    T tot[EPL];
#pragma unroll
    for (int v = 0; v < EPL; ++v) {
        T t = red[0][lane * EPL + v];
#pragma unroll
        for (int w = 1; w < kConsumerWarps; ++w) t += red[w][lane * EPL + v];
        tot[v] = t;
    }
    auto finish = [&](int v, T t) {
        const int64_t col = col0 + lane * EPL + v;
        if (col >= a.M) return;
        T out = t;
        if (a.gemv) {
            const T bc = (a.beta == T(0)) ? T(0) : a.beta * a.y[col];
            out = fma_rn(a.alpha, t, bc);
        }
        a.y[col] = out;
    };
    if (a.nseg == 1) {
#pragma unroll
        for (int v = 0; v < EPL; ++v) finish(v, tot[v]);
        return;
    }
    T *part = a.partial + seg * a.M;
#pragma unroll
    for (int v = 0; v < EPL; ++v)
        if (col0 + lane * EPL + v < a.M) part[col0 + lane * EPL + v] = tot[v];
    __threadfence();
    __syncwarp();
    if (lane == 0) ticket = atomicAdd(a.counters + cb, 1u);
    __syncwarp();
    if (ticket != (unsigned)(a.nseg - 1)) return;
    __threadfence();
#pragma unroll
    for (int v = 0; v < EPL; ++v) {
        const int64_t col = col0 + lane * EPL + v;
        if (col >= a.M) continue;
        T t = T(0);
        for (int ss = 0; ss < a.nseg; ++ss) {
            const T pv = __ldcg(a.partial + (int64_t)ss * a.M + col);
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

// cc: columns per block, ts: bytes per element (partial sums are elements).
ColSegments col_segments(int64_t M, int64_t N, int sms, int64_t cc, size_t ts) {
    ColSegments s{(M + cc - 1) / cc, 1, 0, 0, 0};
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
        s.part_bytes = ((size_t)s.nseg * M * ts + 255) & ~(size_t)255;
        s.cnt_bytes = ((size_t)s.ncb * 4 + 255) & ~(size_t)255;
    }
    return s;
}

template <typename T>
struct TmaType;
template <>
struct TmaType<float> {
    static constexpr CUtensorMapDataType value = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
};
template <>
struct TmaType<double> {
    static constexpr CUtensorMapDataType value = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
};

}  // namespace gvi

size_t matvec_image_ws_bytes(const gatlas_matvec_desc *d, size_t elem_bytes) {
    using namespace gvi;
    if (!d || !d->trans_a || d->n == 0 || d->m == 0) return 0;
    const ColSegments s =
        col_segments((int64_t)d->m, (int64_t)d->n, sm_count(), 1024 / (int64_t)elem_bytes, elem_bytes);
    return s.part_bytes + s.cnt_bytes;
}

template <typename T>
int matvec_image(const gatlas_matvec_desc *d, const T *A, const T *x, T *y, void *ws, size_t ws_bytes,
                 cudaStream_t stream) {
    using namespace gvi;
    constexpr int V = Elem<T>::V, ROW = Elem<T>::ROW;
    constexpr size_t TS = sizeof(T);
    if (d->m == 0) return GATLAS_OK;
    if (!A || !x || !y) return set_error(GATLAS_ERR_INVALID, "matvec: null pointer");
    const size_t batch = d->batch ? d->batch : 1;
    if (batch != 1) return set_error(GATLAS_ERR_UNSUPPORTED, "matvec image engine: batch must be 1");
    const int64_t M = (int64_t)d->m, N = (int64_t)d->n;
    const int64_t lda = d->lda ? (int64_t)d->lda : (d->trans_a ? M : N);
    const int64_t inner = d->trans_a ? M : N;
    if (lda < inner) return set_error(GATLAS_ERR_INVALID, "matvec: lda too small");
    if (lda % V || !aligned16(A) || !aligned16(x) || inner % V)
        return set_error(GATLAS_ERR_UNSUPPORTED,
                         "matvec image engine: needs 16-byte aligned rows (lda and the inner dimension multiples "
                         "of %d)", V);
    if (N == 0) {
        gatlas_matvec_desc b = *d;
        b.engine = GATLAS_ENGINE_BUFFER;
        if constexpr (sizeof(T) == 4) return gatlas_matvec_f32(&b, A, x, y, ws, ws_bytes, stream);
        else return gatlas_matvec_f64(&b, A, x, y, ws, ws_bytes, stream);
    }
    CUtensorMap tm;
    const uint64_t dims[2] = {(uint64_t)inner, (uint64_t)(d->trans_a ? N : M)};
    const uint64_t strides[1] = {(uint64_t)lda * TS};
    const int sms = sm_count();
    if (!d->trans_a) {
        const uint32_t box[2] = {(uint32_t)ROW, RB};
        int rc = make_tensor_map(&tm, TmaType<T>::value, 2, const_cast<T *>(A), dims, strides, box,
                                 CU_TENSOR_MAP_SWIZZLE_NONE);
        if (rc) return rc;
        RowArgs<T> a{y, x, M, N, (T)d->alpha, (T)d->beta, d->gemv, device_fault_word()};
        const int smem = RS * (int)kRowStage;
        cudaFuncSetAttribute(gemv_rows_tma_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        const int64_t nblocks = (M + RB - 1) / RB;
        const int grid = (int)(nblocks < sms ? nblocks : sms);
        gemv_rows_tma_kernel<T><<<grid, kThreads, smem, stream>>>(tm, a);
        return check_launch("gemv_rows_tma_kernel");
    }
    const uint32_t box[2] = {(uint32_t)ROW, CR};
    int rc = make_tensor_map(&tm, TmaType<T>::value, 2, const_cast<T *>(A), dims, strides, box,
                             CU_TENSOR_MAP_SWIZZLE_NONE);
    if (rc) return rc;
    const ColSegments seg = col_segments(M, N, sms, ROW, TS);
    const int64_t ncb = seg.ncb, nseg = seg.nseg, seg_len = seg.seg_len;
    T *partial = nullptr;
    unsigned *counters = nullptr;
    if (nseg > 1) {
        const size_t part_bytes = seg.part_bytes, cnt_bytes = seg.cnt_bytes;
        if (!ws) {
            ws = device_scratch(part_bytes + cnt_bytes);
            if (!ws) return set_error(GATLAS_ERR_NOMEM, "matvec: scratch");
        } else if (ws_bytes < part_bytes + cnt_bytes || !aligned_to(ws, 256)) {
            return set_error(GATLAS_ERR_INVALID, "matvec: workspace too small or not 256-byte aligned");
        }
        partial = static_cast<T *>(ws);
        counters = reinterpret_cast<unsigned *>(static_cast<char *>(ws) + part_bytes);
        cudaError_t e = cudaMemsetAsync(counters, 0, cnt_bytes, stream);
        if (e != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "matvec: %s", cudaGetErrorString(e));
    }
    ColArgs<T> a{y, x, M, N, seg_len, (int)nseg, (T)d->alpha, (T)d->beta, d->gemv, partial, counters,
                 device_fault_word()};
    const int smem = CS * (int)kColStage;
    cudaFuncSetAttribute(gemv_cols_tma_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    dim3 grid((unsigned)ncb, (unsigned)nseg);
    gemv_cols_tma_kernel<T><<<grid, kThreads, smem, stream>>>(tm, a);
    return check_launch("gemv_cols_tma_kernel");
}

int matvec_image_f32(const gatlas_matvec_desc *d, const float *A, const float *x, float *y, void *ws,
                     size_t ws_bytes, cudaStream_t stream) {
    return matvec_image<float>(d, A, x, y, ws, ws_bytes, stream);
}

int matvec_image_f64(const gatlas_matvec_desc *d, const double *A, const double *x, double *y, void *ws,
                     size_t ws_bytes, cudaStream_t stream) {
    return matvec_image<double>(d, A, x, y, ws, ws_bytes, stream);
}

}  // namespace gatlas
