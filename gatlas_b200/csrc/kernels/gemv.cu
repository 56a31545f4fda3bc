// GEMV: y = A·x or y = alpha·A·x + beta·y, HBM streaming (buffer engine).
//
// Reference: KernelMatvecBuffer<SCALAR,VL>::print (KernelMatvecBuffer.hpp:180-325):
// one work item owns blockHeight rows and walks N/VL vectors of its rows and
// of b, accumulating with mad; transposeA reads A column-major
// (KernelMatvecBuffer.hpp:288-291).  Row-per-thread reads are uncoalesced for
// row-major A.
//
// B200 design (both layouts read every byte of A exactly once, 16-byte loads):
//  * trans_a == 0 (row-major): for long rows (at least 4 x 256 vectors) a CTA
//    owns two rows at a time and its 256 threads stride across them in
//    16-byte vectors, reduced in a fixed order (warp butterfly, then the 8
//    warps in shared memory); otherwise a warp owns ROWS rows at a time, its
//    lanes striding across the row with UNROLL loads per row in flight and a
//    fixed butterfly shuffle reduction.  x is read through the L1-cached
//    read-only path.
//  * trans_a == 1 (column-major): a CTA owns 32*VW adjacent columns (one
//    16-byte vector per lane) and one segment of the rows; its 8 warps take
//    interleaved rows, partial sums are combined across warps in a fixed order
//    in shared memory, and across the S row segments by the last CTA of each
//    column block (partials in a workspace, arrival counter per column block).
// Results are deterministic: the order depends only on (M, N) and the SM count.
#include <algorithm>

#include "../common.cuh"
#include "../device_state.cuh"

namespace gatlas {

template <typename T, int VW> struct VecT;
template <> struct VecT<float, 4> { using type = float4; };
template <> struct VecT<float, 1> { using type = float; };
template <> struct VecT<double, 2> { using type = double2; };
template <> struct VecT<double, 1> { using type = double; };

__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// acc = fma chain over the vector's components in order.
__device__ __forceinline__ float dot_acc(float acc, float4 a, float4 x) {
    acc = fma_rn(a.x, x.x, acc);
    acc = fma_rn(a.y, x.y, acc);
    acc = fma_rn(a.z, x.z, acc);
    return fma_rn(a.w, x.w, acc);
}
__device__ __forceinline__ double dot_acc(double acc, double2 a, double2 x) {
    acc = fma_rn(a.x, x.x, acc);
    return fma_rn(a.y, x.y, acc);
}
__device__ __forceinline__ float dot_acc(float acc, float a, float x) { return fma_rn(a, x, acc); }
__device__ __forceinline__ double dot_acc(double acc, double a, double x) { return fma_rn(a, x, acc); }

template <typename T>
__device__ __forceinline__ T epilogue(int gemv, T alpha, T beta, T acc, const T *yold) {
    if (!gemv) return acc;
    const T bc = (beta == T(0)) ? T(0) : beta * (*yold);
    return fma_rn(alpha, acc, bc);
}

struct GemvArgs {
    const void *A;
    const void *x;
    void *y;
    size_t M, N, lda;
    size_t stride_a, stride_x, stride_y;
    double alpha, beta;
    int gemv;
};

constexpr int kGemvThreads = 256;
constexpr int kGemvWarps = kGemvThreads / 32;

// ---------------------------------------------------------------------------
// row-major A
// ---------------------------------------------------------------------------
template <typename T, int VW, int ROWS, int UNROLL>
__global__ void __launch_bounds__(kGemvThreads)
    gemv_rows_kernel(GemvArgs a) {
    using V = typename VecT<T, VW>::type;
    const int lane = threadIdx.x & 31;
    const size_t warp = (size_t)blockIdx.x * kGemvWarps + (threadIdx.x >> 5);
    const size_t nwarps = (size_t)gridDim.x * kGemvWarps;
    const size_t p = blockIdx.y;
    const T *A = static_cast<const T *>(a.A) + p * a.stride_a;
    const V *x = reinterpret_cast<const V *>(static_cast<const T *>(a.x) + p * a.stride_x);
    T *y = static_cast<T *>(a.y) + p * a.stride_y;
    const size_t nvec = a.N / VW;
    const size_t ldv = a.lda / VW;
    const T alpha = (T)a.alpha, beta = (T)a.beta;

    for (size_t row0 = warp * ROWS; row0 < a.M; row0 += nwarps * ROWS) {
        T acc[ROWS];
        const V *arow[ROWS];
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            acc[r] = T(0);
            const size_t row = (row0 + r < a.M) ? row0 + r : a.M - 1;  // clamp; result discarded
            arow[r] = reinterpret_cast<const V *>(A + row * a.lda);
        }
        (void)ldv;
        size_t c = lane;
        for (; c + (UNROLL - 1) * 32 < nvec; c += UNROLL * 32) {
            V av[ROWS][UNROLL], xv[UNROLL];
#pragma unroll
            for (int u = 0; u < UNROLL; ++u) xv[u] = __ldg(x + c + u * 32);
#pragma unroll
            for (int r = 0; r < ROWS; ++r)
#pragma unroll
                for (int u = 0; u < UNROLL; ++u) av[r][u] = __ldcs(arow[r] + c + u * 32);
#pragma unroll
            for (int u = 0; u < UNROLL; ++u)
#pragma unroll
                for (int r = 0; r < ROWS; ++r) acc[r] = dot_acc(acc[r], av[r][u], xv[u]);
        }
        for (; c < nvec; c += 32) {
            const V xv = __ldg(x + c);
#pragma unroll
            for (int r = 0; r < ROWS; ++r) acc[r] = dot_acc(acc[r], __ldcs(arow[r] + c), xv);
        }
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], off);
        }
        if (lane < ROWS) {
            T v = acc[0];
#pragma unroll
            for (int r = 1; r < ROWS; ++r)
                if (lane == r) v = acc[r];
            const size_t row = row0 + lane;
            if (row < a.M) y[row] = epilogue<T>(a.gemv, alpha, beta, v, y + row);
        }
    }
}

// Long rows: a CTA owns RB rows at a time and all 256 threads stride across
// each of them in 16-byte vectors (UNROLL per row in flight, x reused from
// registers across the RB rows); the per-thread chains are combined by a
// fixed butterfly per warp and a fixed-order sum over the 8 warps in shared
// memory.  The units are 8 times smaller than a warp's rows, so a 16384^2
// product is thousands of CTAs and the last partial wave costs little.
template <typename T, int VW, int RB, int UNROLL>
__global__ void __launch_bounds__(kGemvThreads)
    gemv_rowblock_kernel(GemvArgs a) {
    using V = typename VecT<T, VW>::type;
    __shared__ T red[RB][kGemvWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const size_t p = blockIdx.y;
    const T *A = static_cast<const T *>(a.A) + p * a.stride_a;
    const V *x = reinterpret_cast<const V *>(static_cast<const T *>(a.x) + p * a.stride_x);
    T *y = static_cast<T *>(a.y) + p * a.stride_y;
    const size_t nvec = a.N / VW;
    const T alpha = (T)a.alpha, beta = (T)a.beta;
    const size_t nblocks = (a.M + RB - 1) / RB;
    for (size_t rb = blockIdx.x; rb < nblocks; rb += gridDim.x) {
        const size_t row0 = rb * RB;
        T acc[RB];
        const V *arow[RB];
#pragma unroll
        for (int r = 0; r < RB; ++r) {
            acc[r] = T(0);
            const size_t row = (row0 + r < a.M) ? row0 + r : a.M - 1;  // clamp; result discarded
            arow[r] = reinterpret_cast<const V *>(A + row * a.lda);
        }
        size_t c = threadIdx.x;
        for (; c + (UNROLL - 1) * kGemvThreads < nvec; c += UNROLL * kGemvThreads) {
            V av[RB][UNROLL], xv[UNROLL];
#pragma unroll
            for (int u = 0; u < UNROLL; ++u) xv[u] = __ldg(x + c + u * kGemvThreads);
#pragma unroll
            for (int r = 0; r < RB; ++r)
#pragma unroll
                for (int u = 0; u < UNROLL; ++u) av[r][u] = __ldcs(arow[r] + c + u * kGemvThreads);
#pragma unroll
            for (int u = 0; u < UNROLL; ++u)
#pragma unroll
                for (int r = 0; r < RB; ++r) acc[r] = dot_acc(acc[r], av[r][u], xv[u]);
        }
        for (; c < nvec; c += kGemvThreads) {
            const V xv = __ldg(x + c);
#pragma unroll
            for (int r = 0; r < RB; ++r) acc[r] = dot_acc(acc[r], __ldcs(arow[r] + c), xv);
        }
#pragma unroll
        for (int r = 0; r < RB; ++r) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], off);
        }
        if (lane == 0)
#pragma unroll
            for (int r = 0; r < RB; ++r) red[r][w] = acc[r];
        __syncthreads();
        if (threadIdx.x < RB) {
            const int r = threadIdx.x;
            T v = red[r][0];
#pragma unroll
            for (int ww = 1; ww < kGemvWarps; ++ww) v += red[r][ww];
            const size_t row = row0 + r;
            if (row < a.M) y[row] = epilogue<T>(a.gemv, alpha, beta, v, y + row);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// column-major A
// ---------------------------------------------------------------------------
template <typename T, int VW, int UNROLL>
__global__ void __launch_bounds__(kGemvThreads)
    gemv_cols_kernel(GemvArgs a, int nseg, size_t seg_len, T *partial, unsigned *counters) {
    using V = typename VecT<T, VW>::type;
    __shared__ __align__(16) T red[kGemvWarps][32 * VW];
    __shared__ unsigned ticket;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const size_t cb = blockIdx.x, s = blockIdx.y, p = blockIdx.z;
    const size_t ncb = gridDim.x;
    const size_t col0 = cb * 32 * VW + (size_t)lane * VW;
    const bool active = col0 < a.M;  // M % VW == 0 is guaranteed when VW > 1
    const T *A = static_cast<const T *>(a.A) + p * a.stride_a;
    const T *x = static_cast<const T *>(a.x) + p * a.stride_x;
    T *y = static_cast<T *>(a.y) + p * a.stride_y;
    const size_t j0 = s * seg_len;
    const size_t j1 = (j0 + seg_len < a.N) ? j0 + seg_len : a.N;

    T acc[VW];
#pragma unroll
    for (int v = 0; v < VW; ++v) acc[v] = T(0);

    if (active) {
        size_t j = j0 + w;
        for (; j + (size_t)(UNROLL - 1) * kGemvWarps < j1; j += (size_t)UNROLL * kGemvWarps) {
            V av[UNROLL];
            T xv[UNROLL];
#pragma unroll
            for (int u = 0; u < UNROLL; ++u) {
                const size_t jj = j + (size_t)u * kGemvWarps;
                av[u] = __ldcs(reinterpret_cast<const V *>(A + jj * a.lda + col0));
                xv[u] = __ldg(x + jj);
            }
#pragma unroll
            for (int u = 0; u < UNROLL; ++u) {
                const T *e = reinterpret_cast<const T *>(&av[u]);
#pragma unroll
                for (int v = 0; v < VW; ++v) acc[v] = fma_rn(e[v], xv[u], acc[v]);
            }
        }
        for (; j < j1; j += kGemvWarps) {
            const V av = __ldcs(reinterpret_cast<const V *>(A + j * a.lda + col0));
            const T xv = __ldg(x + j);
            const T *e = reinterpret_cast<const T *>(&av);
#pragma unroll
            for (int v = 0; v < VW; ++v) acc[v] = fma_rn(e[v], xv, acc[v]);
        }
    }
#pragma unroll
    for (int v = 0; v < VW; ++v) red[w][lane * VW + v] = acc[v];
    __syncthreads();
    if (w != 0) return;

    T tot[VW];
#pragma unroll
    for (int v = 0; v < VW; ++v) {
        T t = red[0][lane * VW + v];
#pragma unroll
        for (int ww = 1; ww < kGemvWarps; ++ww) t += red[ww][lane * VW + v];
        tot[v] = t;
    }
    const T alpha = (T)a.alpha, beta = (T)a.beta;
    if (nseg == 1) {
        if (active)
#pragma unroll
            for (int v = 0; v < VW; ++v) y[col0 + v] = epilogue<T>(a.gemv, alpha, beta, tot[v], y + col0 + v);
        return;
    }
    // publish this segment's partial, then the last CTA of the column block sums
    T *part = partial + (p * nseg + s) * a.M;
    if (active)
#pragma unroll
        for (int v = 0; v < VW; ++v) part[col0 + v] = tot[v];
    __threadfence();
    __syncwarp();
    if (lane == 0) ticket = atomicAdd(counters + p * ncb + cb, 1u);
    __syncwarp();
    if (ticket != (unsigned)(nseg - 1)) return;
    __threadfence();
    if (!active) return;
#pragma unroll
    for (int v = 0; v < VW; ++v) {
        T t = T(0);
        for (int ss = 0; ss < nseg; ++ss) {
            const T pv = __ldcg(partial + (p * nseg + ss) * a.M + col0 + v);
            t = (ss == 0) ? pv : t + pv;
        }
        y[col0 + v] = epilogue<T>(a.gemv, alpha, beta, t, y + col0 + v);
    }
}

// ---------------------------------------------------------------------------
// launch
// ---------------------------------------------------------------------------
int matvec_image_f32(const gatlas_matvec_desc *d, const float *A, const float *x, float *y, void *ws,
                     size_t ws_bytes, cudaStream_t stream);
int matvec_image_f64(const gatlas_matvec_desc *d, const double *A, const double *x, double *y, void *ws,
                     size_t ws_bytes, cudaStream_t stream);
size_t matvec_image_ws_bytes(const gatlas_matvec_desc *d, size_t elem_bytes);

template <typename T>
static int matvec_image_dispatch(const gatlas_matvec_desc *d, const T *A, const T *x, T *y, void *ws,
                                 size_t ws_bytes, cudaStream_t stream) {
    if constexpr (sizeof(T) == 4) return matvec_image_f32(d, A, x, y, ws, ws_bytes, stream);
    else return matvec_image_f64(d, A, x, y, ws, ws_bytes, stream);
}

struct ColsPlan {
    int vw;
    size_t ncb, nseg, seg_len, part_bytes, counter_bytes;
};

template <typename T>
static ColsPlan cols_plan(const gatlas_matvec_desc *d, bool vec_ok) {
    ColsPlan pl{};
    const size_t batch = d->batch ? d->batch : 1;
    pl.vw = vec_ok ? (int)(16 / sizeof(T)) : 1;
    pl.ncb = (d->m + 32 * pl.vw - 1) / (32 * pl.vw);
    const size_t target = (size_t)sm_count() * 4;
    size_t per_batch = (target + batch - 1) / batch;
    size_t nseg = (per_batch + pl.ncb - 1) / pl.ncb;
    const size_t max_seg = (d->n + 31) / 32;
    if (nseg > max_seg) nseg = max_seg;
    if (nseg < 1) nseg = 1;
    if (nseg > 4096) nseg = 4096;
    if (d->n == 0) {
        pl.seg_len = 0;
        pl.nseg = 1;
    } else {
        pl.seg_len = (d->n + nseg - 1) / nseg;
        pl.nseg = (d->n + pl.seg_len - 1) / pl.seg_len;
    }
    if (pl.nseg > 1) {
        pl.part_bytes = (batch * pl.nseg * d->m * sizeof(T) + 255) & ~(size_t)255;
        pl.counter_bytes = (batch * pl.ncb * sizeof(unsigned) + 255) & ~(size_t)255;
    }
    return pl;
}

template <typename T>
static bool gemv_vec_ok(const gatlas_matvec_desc *d, const T *A, const T *x) {
    const size_t vw = 16 / sizeof(T);
    const size_t lda = d->lda ? d->lda : (d->trans_a ? d->m : d->n);
    const size_t inner = d->trans_a ? d->m : d->n;
    const size_t batch = d->batch ? d->batch : 1;
    bool ok = aligned16(A) && (lda % vw == 0) && (inner % vw == 0);
    if (!d->trans_a) ok = ok && aligned16(x);
    if (batch > 1) {
        const size_t sa = d->stride_a ? d->stride_a : lda * (d->trans_a ? d->n : d->m);
        const size_t sx = d->stride_x ? d->stride_x : d->n;
        ok = ok && (sa % vw == 0) && (d->trans_a || sx % vw == 0);
    }
    return ok;
}

template <typename T>
static size_t matvec_ws(const gatlas_matvec_desc *d, const void *A, const void *x) {
    if (!d || !d->trans_a) return 0;
    if (d->engine == GATLAS_ENGINE_IMAGE) return matvec_image_ws_bytes(d, sizeof(T));
    const ColsPlan pl = cols_plan<T>(d, gemv_vec_ok<T>(d, (const T *)A, (const T *)x));
    return pl.part_bytes + pl.counter_bytes;
}

template <typename T>
static int matvec_launch(const gatlas_matvec_desc *d, const T *A, const T *x, T *y, void *ws,
                         size_t ws_bytes, cudaStream_t stream) {
    if (!d) return set_error(GATLAS_ERR_INVALID, "matvec: null descriptor");
    if (d->engine == GATLAS_ENGINE_IMAGE) return matvec_image_dispatch<T>(d, A, x, y, ws, ws_bytes, stream);
    if (d->engine != GATLAS_ENGINE_BUFFER)
        return set_error(GATLAS_ERR_INVALID, "matvec: engine %d is not buffer/image", d->engine);
    if (d->m == 0) return GATLAS_OK;
    if (!A || !x || !y) return set_error(GATLAS_ERR_INVALID, "matvec: null pointer");
    const size_t batch = d->batch ? d->batch : 1;
    if (batch > 65535) return set_error(GATLAS_ERR_INVALID, "matvec: batch %zu > 65535", batch);
    const size_t lda = d->lda ? d->lda : (d->trans_a ? d->m : d->n);
    if ((!d->trans_a && lda < d->n) || (d->trans_a && lda < d->m))
        return set_error(GATLAS_ERR_INVALID, "matvec: lda %zu too small", lda);

    GemvArgs a;
    a.A = A;
    a.x = x;
    a.y = y;
    a.M = d->m;
    a.N = d->n;
    a.lda = lda;
    a.stride_a = d->stride_a ? d->stride_a : lda * (d->trans_a ? d->n : d->m);
    a.stride_x = d->stride_x ? d->stride_x : d->n;
    a.stride_y = d->stride_y ? d->stride_y : d->m;
    a.alpha = d->alpha;
    a.beta = d->beta;
    a.gemv = d->gemv;

    const bool vec_ok = gemv_vec_ok<T>(d, A, x);
    const int sms = sm_count();
    if (!d->trans_a) {
        constexpr int UNROLL = 4;
        constexpr int VWV = 16 / sizeof(T);
        if (vec_ok && d->n / VWV >= (size_t)UNROLL * kGemvThreads) {
            // long rows: a CTA per RB rows (see gemv_rowblock_kernel)
            constexpr int RB = 2;
            const size_t nblocks = (d->m + RB - 1) / RB;
            const size_t cap = (size_t)sms * 64 / (batch < 8 ? batch : 8);
            dim3 g((unsigned)(nblocks < cap ? nblocks : cap), (unsigned)batch);
            gemv_rowblock_kernel<T, VWV, RB, UNROLL><<<g, kGemvThreads, 0, stream>>>(a);
            return check_launch("gemv_rowblock_kernel");
        }
        constexpr int ROWS = 2;
        const size_t warps_needed = (d->m + ROWS - 1) / ROWS;
        size_t grid = (warps_needed + kGemvWarps - 1) / kGemvWarps;
        const size_t cap = (size_t)sms * 8 / (batch < 8 ? batch : 8);
        if (grid > cap) grid = cap ? cap : 1;
        dim3 g((unsigned)grid, (unsigned)batch);
        if (vec_ok) {
            constexpr int VW = 16 / sizeof(T);
            gemv_rows_kernel<T, VW, ROWS, 4><<<g, kGemvThreads, 0, stream>>>(a);
        } else {
            gemv_rows_kernel<T, 1, ROWS, 4><<<g, kGemvThreads, 0, stream>>>(a);
        }
        return check_launch("gemv_rows_kernel");
    }

    const ColsPlan pl = cols_plan<T>(d, vec_ok);
    T *partial = nullptr;
    unsigned *counters = nullptr;
    if (pl.nseg > 1) {
        const size_t need = pl.part_bytes + pl.counter_bytes;
        if (!ws) {
            ws = device_scratch(need);
            if (!ws) return set_error(GATLAS_ERR_NOMEM, "matvec: scratch of %zu bytes", need);
        } else if (ws_bytes < need) {
            return set_error(GATLAS_ERR_INVALID, "matvec: workspace %zu < %zu bytes", ws_bytes, need);
        } else if (!aligned_to(ws, 256)) {
            return set_error(GATLAS_ERR_INVALID, "matvec: workspace must be 256-byte aligned");
        }
        partial = static_cast<T *>(ws);
        counters = reinterpret_cast<unsigned *>(static_cast<char *>(ws) + pl.part_bytes);
        cudaError_t e = cudaMemsetAsync(counters, 0, pl.counter_bytes, stream);
        if (e != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "matvec: memset counters: %s", cudaGetErrorString(e));
    }
    dim3 g((unsigned)pl.ncb, (unsigned)pl.nseg, (unsigned)batch);
    if (pl.ncb > 0x7fffffffu || pl.nseg > 65535)
        return set_error(GATLAS_ERR_INVALID, "matvec: grid too large");
    if (pl.vw > 1) {
        constexpr int VW = 16 / sizeof(T);
        gemv_cols_kernel<T, VW, 4><<<g, kGemvThreads, 0, stream>>>(a, (int)pl.nseg, pl.seg_len, partial, counters);
    } else {
        gemv_cols_kernel<T, 1, 4><<<g, kGemvThreads, 0, stream>>>(a, (int)pl.nseg, pl.seg_len, partial, counters);
    }
    return check_launch("gemv_cols_kernel");
}

}  // namespace gatlas

extern "C" size_t gatlas_matvec_workspace_size(const gatlas_matvec_desc *d) {
    // The largest need over both element types and both load widths, so the
    // answer holds whichever path the launch picks.
    if (!d || !d->trans_a) return 0;
    size_t best = 0;
    for (int vec = 0; vec < 2; ++vec) {
        const gatlas::ColsPlan f = gatlas::cols_plan<float>(d, vec != 0);
        const gatlas::ColsPlan g = gatlas::cols_plan<double>(d, vec != 0);
        const size_t a = f.part_bytes + f.counter_bytes, b = g.part_bytes + g.counter_bytes;
        if (a > best) best = a;
        if (b > best) best = b;
    }
    const size_t img = std::max(gatlas::matvec_image_ws_bytes(d, 4), gatlas::matvec_image_ws_bytes(d, 8));
    return img > best ? img : best;
}

extern "C" int gatlas_matvec_f32(const gatlas_matvec_desc *d, const float *A, const float *x, float *y,
                                 void *workspace, size_t workspace_bytes, void *stream) {
    return gatlas::matvec_launch<float>(d, A, x, y, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" int gatlas_matvec_f64(const gatlas_matvec_desc *d, const double *A, const double *x,
                                 double *y, void *workspace, size_t workspace_bytes, void *stream) {
    return gatlas::matvec_launch<double>(d, A, x, y, workspace, workspace_bytes, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Allocation-free GEMV entry point.
//
// For callers that cannot call cudaMalloc: code that runs inside a host
// framework which owns all device memory (or has reserved it for its own
// pool), and code on a latency-critical path that must not trigger the
// device-wide synchronisation cudaMalloc/cudaFree imply.  The column-major
// path needs scratch for per-segment partial sums and arrival counters; this
// entry point takes it from a fixed 1 MiB array in device memory that this
// file owns, instead of from a workspace or the library's allocation cache.
// ---------------------------------------------------------------------------
#include <mutex>

namespace gatlas {
namespace {

constexpr size_t kNoAllocScratchBytes = GATLAS_MATVEC_NOALLOC_SCRATCH_BYTES;

// One copy per GPU that loads this library, held until the process exits.
// Host code may not use this name as a device address: the device address is
// looked up once per device with cudaGetSymbolAddress.
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch for the current device (looked up on
// the first call on each device, with that device current).
int noalloc_scratch(void **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "matvec_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return set_error(GATLAS_ERR_INVALID, "matvec_noalloc: device %d", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return set_error(GATLAS_ERR_CUDA, "matvec_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return GATLAS_OK;
}

}  // namespace
}  // namespace gatlas

extern "C" int gatlas_matvec_f32_noalloc(const gatlas_matvec_desc *d, const float *A, const float *x, float *y,
                                         void *stream) {
    using namespace gatlas;
    if (!d) return set_error(GATLAS_ERR_INVALID, "matvec_noalloc: null descriptor");
    const size_t need = matvec_ws<float>(d, A, x);
    if (need > kNoAllocScratchBytes)
        return set_error(GATLAS_ERR_INVALID,
                         "matvec_noalloc: this problem needs %zu bytes of scratch, more than the %zu-byte "
                         "static scratch of the allocation-free entry point; call gatlas_matvec_f32 with a "
                         "workspace instead",
                         need, kNoAllocScratchBytes);
    void *scratch = nullptr;
    const int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    return matvec_launch<float>(d, A, x, y, scratch, kNoAllocScratchBytes, (cudaStream_t)stream);
}
