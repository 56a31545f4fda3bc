// SAXPY / DAXPY: z = fma(alpha, x, y), HBM streaming.
//
// Reference: KernelSaxpyBuffer<SCALAR,VL>::print (KernelSaxpyBuffer.hpp:143-225)
// emits Z = mad(alpha, X, Y) over 1-D or 2-D work groups; KernelSaxpyImage
// (KernelSaxpyImage.hpp:148-233) reads X and Y through texture fetches.
//
// B200 design:
//  * buffer engine: grid-stride loop over 16-byte vectors (float4 / double2),
//    UNROLL independent vectors per stream in flight per thread, streaming
//    (evict-first) loads and stores, grid = SMs x 8 blocks of 256 threads.
//  * image engine: persistent CTAs stream 16 KiB chunks of x and y into shared
//    memory with 1-D bulk async copies (cp.async.bulk, TMA engine) through a
//    6-stage mbarrier pipeline (loads four chunks ahead), compute in place,
//    and write back with bulk shared->global copies.
// Both compute __fma_rn(alpha, x, y): bit-exact against a per-element fmaf.
#include "../common.cuh"
#include "../device_state.cuh"

namespace gatlas {

template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; static constexpr int n = 4; };
template <> struct Vec16<double> { using type = double2; static constexpr int n = 2; };

__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

__device__ __forceinline__ float4 axpy_vec(float a, float4 x, float4 y) {
    return make_float4(fma_rn(a, x.x, y.x), fma_rn(a, x.y, y.y), fma_rn(a, x.z, y.z),
                       fma_rn(a, x.w, y.w));
}
__device__ __forceinline__ double2 axpy_vec(double a, double2 x, double2 y) {
    return make_double2(fma_rn(a, x.x, y.x), fma_rn(a, x.y, y.y));
}

constexpr int kSaxpyThreads = 256;
constexpr int kSaxpyUnroll = 4;

template <typename T>
__global__ void __launch_bounds__(kSaxpyThreads)
    saxpy_vec_kernel(size_t nvec, T alpha, const typename Vec16<T>::type *__restrict__ x,
                     const typename Vec16<T>::type *y, typename Vec16<T>::type *z) {
    using V = typename Vec16<T>::type;
    const size_t stride = (size_t)gridDim.x * kSaxpyThreads * kSaxpyUnroll;
    for (size_t base = (size_t)blockIdx.x * kSaxpyThreads * kSaxpyUnroll + threadIdx.x; base < nvec;
         base += stride) {
        V xv[kSaxpyUnroll], yv[kSaxpyUnroll];
#pragma unroll
        for (int u = 0; u < kSaxpyUnroll; ++u) {
            const size_t i = base + (size_t)u * kSaxpyThreads;
            if (i < nvec) {
                xv[u] = ld_stream(x + i);
                yv[u] = ld_stream(y + i);
            }
        }
#pragma unroll
        for (int u = 0; u < kSaxpyUnroll; ++u) {
            const size_t i = base + (size_t)u * kSaxpyThreads;
            if (i < nvec) st_stream(z + i, axpy_vec(alpha, xv[u], yv[u]));
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kSaxpyThreads)
    saxpy_scalar_kernel(size_t n, T alpha, const T *x, const T *y, T *z) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        z[i] = fma_rn(alpha, x[i], y[i]);
}

// ---------------------------------------------------------------------------
// image engine: bulk-copy pipeline
// ---------------------------------------------------------------------------
constexpr int kBulkThreads = 256;
constexpr int kBulkStages = 6;
// Loads run kBulkAhead chunks ahead, so the stage a new load reuses was last
// stored from two chunks ago: the producer waits only for that older bulk
// store to finish reading shared memory (wait_group.read 1), never for the
// store just committed.
constexpr int kBulkAhead = kBulkStages - 2;
constexpr uint32_t kBulkChunkBytes = 16384;  // per operand per stage

template <typename T>
__global__ void __launch_bounds__(kBulkThreads, 1)
    saxpy_bulk_kernel(size_t n, T alpha, const T *x, const T *y, T *z, int *fault) {
    extern __shared__ __align__(128) unsigned char smem[];
    using V = typename Vec16<T>::type;
    constexpr uint32_t kElems = kBulkChunkBytes / sizeof(T);
    unsigned char *xs = smem;
    unsigned char *ys = smem + kBulkStages * kBulkChunkBytes;
    __shared__ __align__(8) uint64_t full[kBulkStages];
    __shared__ int abort_flag;

    const size_t nfull16 = (n * sizeof(T)) / 16;                 // whole 16-byte vectors
    const size_t nchunks = (nfull16 * 16 + kBulkChunkBytes - 1) / kBulkChunkBytes;
    // chunks owned by this CTA: blockIdx.x, blockIdx.x + gridDim.x, ...
    const size_t mine = (blockIdx.x < nchunks) ? (nchunks - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kBulkStages; ++s) mbar_init(&full[s], 1);
        fence_mbarrier_init();
        abort_flag = 0;
    }
    __syncthreads();

    auto chunk_bytes = [&](size_t c) -> uint32_t {
        const size_t off = c * kBulkChunkBytes;
        const size_t rem = nfull16 * 16 - off;
        return rem < kBulkChunkBytes ? (uint32_t)rem : kBulkChunkBytes;
    };
    auto issue = [&](size_t i) {
        const size_t c = blockIdx.x + i * gridDim.x;
        const int s = (int)(i % kBulkStages);
        const uint32_t bytes = chunk_bytes(c);
        const size_t off = c * kBulkChunkBytes;
        mbar_arrive_expect_tx(&full[s], 2 * bytes);
        bulk_g2s(xs + s * kBulkChunkBytes, reinterpret_cast<const unsigned char *>(x) + off, bytes,
                 &full[s]);
        bulk_g2s(ys + s * kBulkChunkBytes, reinterpret_cast<const unsigned char *>(y) + off, bytes,
                 &full[s]);
    };

    size_t issued = 0;  // meaningful in thread 0 only
    if (threadIdx.x == 0)
        for (; issued < (size_t)kBulkAhead && issued < mine; ++issued) issue(issued);

    size_t i = 0;
    for (; i < mine; ++i) {
        const int s = (int)(i % kBulkStages);
        if (threadIdx.x == 0 && i + kBulkAhead < mine) {
            // stage (i - 2) % S is reused: the bulk store of chunk i - 2 (every
            // committed group but the newest) must have finished reading smem
            bulk_wait_read<1>();
            issue(i + kBulkAhead);
            issued = i + kBulkAhead + 1;
        }
        if (!mbar_wait_bounded(&full[s], (uint32_t)((i / kBulkStages) & 1), 1u << 22)) {
            report_fault(fault, kFaultSaxpyBulkWait);
            abort_flag = 1;
        }
        __syncthreads();
        if (abort_flag) break;
        const size_t c = blockIdx.x + i * gridDim.x;
        const uint32_t bytes = chunk_bytes(c);
        const V *xv = reinterpret_cast<const V *>(xs + s * kBulkChunkBytes);
        V *yv = reinterpret_cast<V *>(ys + s * kBulkChunkBytes);
        for (uint32_t k = threadIdx.x; k < bytes / 16; k += kBulkThreads) yv[k] = axpy_vec(alpha, xv[k], yv[k]);
        fence_proxy_async_shared();
        __syncthreads();
        if (threadIdx.x == 0) {
            bulk_s2g(reinterpret_cast<unsigned char *>(z) + c * kBulkChunkBytes, yv, bytes);
            bulk_commit();
        }
    }
    if (threadIdx.x == 0) {
        // after an abort, wait (bounded) for the loads still in flight into smem
        for (size_t j = i; j < issued; ++j)
            mbar_wait_bounded(&full[j % kBulkStages], (uint32_t)((j / kBulkStages) & 1), 1u << 22);
        bulk_wait<0>();
    }
    (void)kElems;

    // elements past the last whole 16-byte vector
    if (blockIdx.x == 0) {
        const size_t first = nfull16 * 16 / sizeof(T);
        for (size_t i = first + threadIdx.x; i < n; i += kBulkThreads) z[i] = fma_rn(alpha, x[i], y[i]);
    }
}

template <typename T>
static int saxpy_launch(int engine, size_t n, T alpha, const T *x, const T *y, T *z,
                        cudaStream_t stream) {
    if (n == 0) return GATLAS_OK;
    if (!x || !y || !z) return set_error(GATLAS_ERR_INVALID, "saxpy: null pointer");
    if (engine != GATLAS_ENGINE_BUFFER && engine != GATLAS_ENGINE_IMAGE)
        return set_error(GATLAS_ERR_INVALID, "saxpy: engine %d is not buffer/image", engine);
    const int sms = sm_count();
    const bool vec_ok = aligned16(x) && aligned16(y) && aligned16(z);
    if (engine == GATLAS_ENGINE_IMAGE && vec_ok) {
        const int smem = 2 * kBulkStages * (int)kBulkChunkBytes;
        cudaFuncSetAttribute(saxpy_bulk_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        const size_t nchunks = (n * sizeof(T) / 16 * 16 + kBulkChunkBytes - 1) / kBulkChunkBytes;
        size_t grid = (size_t)sms;
        if (nchunks < grid) grid = nchunks ? nchunks : 1;
        saxpy_bulk_kernel<T><<<(unsigned)grid, kBulkThreads, smem, stream>>>(n, alpha, x, y, z,
                                                                             device_fault_word());
        return check_launch("saxpy_bulk_kernel");
    }
    if (vec_ok) {
        using V = typename Vec16<T>::type;
        const size_t nvec = n / Vec16<T>::n;
        if (nvec) {
            size_t grid = (nvec + kSaxpyThreads * kSaxpyUnroll - 1) / (kSaxpyThreads * kSaxpyUnroll);
            const size_t cap = (size_t)sms * 8;
            if (grid > cap) grid = cap;
            saxpy_vec_kernel<T><<<(unsigned)grid, kSaxpyThreads, 0, stream>>>(
                nvec, alpha, reinterpret_cast<const V *>(x), reinterpret_cast<const V *>(y),
                reinterpret_cast<V *>(z));
            int rc = check_launch("saxpy_vec_kernel");
            if (rc) return rc;
        }
        const size_t done = nvec * Vec16<T>::n;
        if (done < n) {
            saxpy_scalar_kernel<T><<<1, kSaxpyThreads, 0, stream>>>(n - done, alpha, x + done,
                                                                    y + done, z + done);
            return check_launch("saxpy_scalar_kernel");
        }
        return GATLAS_OK;
    }
    size_t grid = (n + kSaxpyThreads - 1) / kSaxpyThreads;
    if (grid > (size_t)sms * 8) grid = (size_t)sms * 8;
    saxpy_scalar_kernel<T><<<(unsigned)grid, kSaxpyThreads, 0, stream>>>(n, alpha, x, y, z);
    return check_launch("saxpy_scalar_kernel");
}

}  // namespace gatlas

extern "C" int gatlas_saxpy_f32(int engine, size_t n, float alpha, const float *x, const float *y,
                                float *z, void *stream) {
    return gatlas::saxpy_launch<float>(engine, n, alpha, x, y, z, (cudaStream_t)stream);
}

extern "C" int gatlas_saxpy_f64(int engine, size_t n, double alpha, const double *x, const double *y,
                                double *z, void *stream) {
    return gatlas::saxpy_launch<double>(engine, n, alpha, x, y, z, (cudaStream_t)stream);
}
