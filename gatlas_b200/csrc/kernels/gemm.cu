// Matmul entry points: argument checks, engine dispatch, FP64 residual.
//
// Reference: the KernelMatmul{Buffer,Image} launch path (GatlasBenchmark.cpp:
// 221-236 -> OCLApp::enqueueKernel) with the layout rules of
// KernelMatmulBuffer.hpp:131-136 and the paranoid check of
// KernelMatmulBuffer.hpp:104-147 / OCLAppUtil.hpp:212-264.
#include <cmath>

#include "../common.cuh"
#include "../device_state.cuh"
#include "gemm_engines.hpp"
#include "gemm_simt.cuh"
#include "gemm_simt_registry.hpp"
#include "jit.hpp"

namespace gatlas {

namespace simt {

const Entry *find(int scalar, int ta, int tb, int gh, int gw, int bh, int bw, int vl) {
    const Entry *(*tables[])(size_t *) = {table_f32_nn_a, table_f32_nn_b, table_f32_tx, table_f64};
    for (auto tf : tables) {
        size_t n = 0;
        const Entry *t = tf(&n);
        for (size_t i = 0; i < n; ++i) {
            const Entry &e = t[i];
            if (e.scalar == scalar && e.ta == ta && e.tb == tb && e.gh == gh && e.gw == gw &&
                e.bh == bh && e.bw == bw && e.vl == vl)
                return &e;
        }
    }
    return nullptr;
}

}  // namespace simt

// Normalised matmul geometry (dense defaults filled in).
bool resolve_geometry(const gatlas_matmul_desc *d, Geometry *g) {
    g->M = (int64_t)d->m;
    g->N = (int64_t)d->n;
    g->K = (int64_t)d->k;
    g->ta = d->trans_a != 0;
    g->tb = d->trans_b != 0;
    g->lda = d->lda ? (int64_t)d->lda : (g->ta ? g->M : g->K);
    g->ldb = d->ldb ? (int64_t)d->ldb : (g->tb ? g->K : g->N);
    g->ldc = d->ldc ? (int64_t)d->ldc : g->N;
    g->batch = d->batch ? (int64_t)d->batch : 1;
    const int64_t a_rows = g->ta ? g->K : g->M, b_rows = g->tb ? g->N : g->K;
    g->stride_a = d->stride_a ? (int64_t)d->stride_a : g->lda * a_rows;
    g->stride_b = d->stride_b ? (int64_t)d->stride_b : g->ldb * b_rows;
    g->stride_c = d->stride_c ? (int64_t)d->stride_c : g->ldc * g->M;
    if (g->M < 0 || g->N < 0 || g->K < 0) return false;
    if (g->lda < (g->ta ? g->M : g->K) || g->ldb < (g->tb ? g->K : g->N) || g->ldc < g->N) return false;
    return true;
}

// Largest vector width <= want that every operand's contiguous dimension,
// leading dimension, batch stride and base pointer allow.
static int feasible_vl(const Geometry &g, const void *A, const void *B, size_t elem, int want) {
    for (int vl = want; vl >= 1; vl /= 2) {
        const int64_t a_inner = g.ta ? g.M : g.K, b_inner = g.tb ? g.K : g.N;
        bool ok = (a_inner % vl == 0) && (g.lda % vl == 0) && (b_inner % vl == 0) &&
                  (g.ldb % vl == 0) && aligned_to(A, elem * vl) && aligned_to(B, elem * vl);
        if (g.batch > 1) ok = ok && (g.stride_a % vl == 0) && (g.stride_b % vl == 0);
        if (ok) return vl;
    }
    return 1;
}

// A point without a prebuilt instantiation: compile it at run time.
template <typename T>
static int matmul_simt_jit(const gatlas_matmul_desc *d, const Geometry &g, const T *A, const T *B, T *C,
                           const jit::Point &pt, cudaStream_t stream) {
    void *fn = nullptr;
    const int rc = jit::simt_function(pt, &fn);
    if (rc) return rc;
    simt::GemmArgs<T> a;
    a.A = A;
    a.B = B;
    a.C = C;
    a.M = g.M;
    a.N = g.N;
    a.K = g.K;
    a.lda = g.lda;
    a.ldb = g.ldb;
    a.ldc = g.ldc;
    a.stride_a = g.stride_a;
    a.stride_b = g.stride_b;
    a.stride_c = g.stride_c;
    a.alpha = (T)d->alpha;
    a.beta = (T)d->beta;
    a.gemm = d->gemm;
    const int64_t BM = (int64_t)pt.gh * pt.bh, BN = (int64_t)pt.gw * pt.bw;
    const int64_t gx = (g.N + BN - 1) / BN, gy = (g.M + BM - 1) / BM;
    if (gx > 0x7fffffff || gy > 65535) return set_error(GATLAS_ERR_INVALID, "matmul: grid too large");
    return jit::launch(fn, (unsigned)gx, (unsigned)gy, (unsigned)g.batch, (unsigned)(pt.gh * pt.gw), &a, stream);
}

template <typename T>
static int matmul_simt(const gatlas_matmul_desc *d, const Geometry &g, const T *A, const T *B, T *C,
                       cudaStream_t stream) {
    const int scalar = sizeof(T) == 8 ? 1 : 0;
    int gh = (int)d->group_h, gw = (int)d->group_w, bh = (int)d->block_h, bw = (int)d->block_w;
    int vl = (int)d->vector_length;
    const bool defaulted = (gh == 0 && gw == 0 && bh == 0 && bw == 0);
    if (defaulted) {
        // the fastest measured points: 16 x 16 x 8 x 8 for float, 8 x 16 x 8 x 8 for double
        gh = scalar ? 8 : 16;
        gw = 16;
        bh = bw = 8;
    }
    const int vmax = scalar ? 2 : 4;
    const int fv = feasible_vl(g, A, B, sizeof(T), vl ? vl : vmax);
    if (vl && fv != vl)
        return set_error(GATLAS_ERR_INVALID,
                         "matmul: vector length %d not allowed by the operand layout/alignment", vl);
    vl = fv;
    const simt::Entry *e = simt::find(scalar, g.ta, g.tb, gh, gw, bh, bw, vl);
    if (!e && defaulted) {
        for (int v = vl; v >= 1 && !e; v /= 2) e = simt::find(scalar, g.ta, g.tb, gh, gw, bh, bw, v);
        if (!e) e = simt::find(scalar, g.ta, g.tb, 16, 16, 4, 4, 1);
    }
    if (!e) return matmul_simt_jit<T>(d, g, A, B, C, jit::Point{scalar, g.ta, g.tb, gh, gw, bh, bw, vl}, stream);
    simt::LaunchArgs l;
    l.A = A;
    l.B = B;
    l.C = C;
    l.M = g.M;
    l.N = g.N;
    l.K = g.K;
    l.lda = g.lda;
    l.ldb = g.ldb;
    l.ldc = g.ldc;
    l.stride_a = g.stride_a;
    l.stride_b = g.stride_b;
    l.stride_c = g.stride_c;
    l.batch = g.batch;
    l.alpha = d->alpha;
    l.beta = d->beta;
    l.gemm = d->gemm;
    l.stream = stream;
    return e->launch(l);
}

template <typename T>
static int matmul_dispatch(const gatlas_matmul_desc *d, const T *A, const T *B, T *C, void *ws,
                           size_t ws_bytes, cudaStream_t stream) {
    if (!d) return set_error(GATLAS_ERR_INVALID, "matmul: null descriptor");
    Geometry g;
    if (!resolve_geometry(d, &g)) return set_error(GATLAS_ERR_INVALID, "matmul: invalid dimensions or leading dimensions");
    if (g.M == 0 || g.N == 0) return GATLAS_OK;
    if (!C || (g.K > 0 && (!A || !B))) return set_error(GATLAS_ERR_INVALID, "matmul: null pointer");
    if (g.batch > 65535) return set_error(GATLAS_ERR_INVALID, "matmul: batch > 65535");
    switch (d->engine) {
        case GATLAS_ENGINE_BUFFER: return matmul_simt<T>(d, g, A, B, C, stream);
        case GATLAS_ENGINE_IMAGE: return matmul_image<T>(d, g, A, B, C, stream);
        case GATLAS_ENGINE_TC_BF16:
        case GATLAS_ENGINE_TC_SPLIT3:
        case GATLAS_ENGINE_TC_SPLIT6:
        case GATLAS_ENGINE_TC_FP8:
            if (sizeof(T) != 4) return set_error(GATLAS_ERR_UNSUPPORTED, "matmul: tensor-core engines take float operands");
            return matmul_tc(d, g, reinterpret_cast<const float *>(A), reinterpret_cast<const float *>(B),
                             reinterpret_cast<float *>(C), ws, ws_bytes, stream);
        default: return set_error(GATLAS_ERR_INVALID, "matmul: unknown engine %d", d->engine);
    }
}

// ---------------------------------------------------------------------------
// FP64 residual on the device
// ---------------------------------------------------------------------------
constexpr int kResTile = 32;

__global__ void __launch_bounds__(256) residual_kernel(const float *A, const float *B, const float *Cin,
                                                       const float *C, int64_t M, int64_t N, int64_t K,
                                                       int64_t lda, int64_t ldb, int64_t ldc, int ta, int tb,
                                                       double alpha, double beta, int gemm, double *stats) {
    __shared__ double As[kResTile][kResTile + 1];
    __shared__ double Bs[kResTile][kResTile + 1];
    __shared__ double red[3][256];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int64_t m0 = (int64_t)blockIdx.y * kResTile, n0 = (int64_t)blockIdx.x * kResTile;
    double acc[2][2] = {{0, 0}, {0, 0}};
    for (int64_t k0 = 0; k0 < K; k0 += kResTile) {
        for (int t = threadIdx.x; t < kResTile * kResTile; t += 256) {
            const int r = t / kResTile, c = t % kResTile;
            const int64_t gi = m0 + r, gk = k0 + c;
            double va = 0;
            if (gi < M && gk < K) va = ta ? (double)A[gk * lda + gi] : (double)A[gi * lda + gk];
            As[r][c] = va;
            const int64_t gkk = k0 + r, gj = n0 + c;
            double vb = 0;
            if (gkk < K && gj < N) vb = tb ? (double)B[gj * ldb + gkk] : (double)B[gkk * ldb + gj];
            Bs[r][c] = vb;
        }
        __syncthreads();
        for (int kk = 0; kk < kResTile; ++kk)
            for (int i = 0; i < 2; ++i)
                for (int j = 0; j < 2; ++j) acc[i][j] += As[ty + 16 * i][kk] * Bs[kk][tx + 16 * j];
        __syncthreads();
    }
    double s2 = 0, r2 = 0, mx = 0, s1 = 0;
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) {
            const int64_t r = m0 + ty + 16 * i, c = n0 + tx + 16 * j;
            if (r < M && c < N) {
                double ref = gemm ? alpha * acc[i][j] : acc[i][j];
                if (gemm && Cin && beta != 0.0) ref += beta * (double)Cin[r * ldc + c];
                const double dlt = (double)C[r * ldc + c] - ref;
                s2 += dlt * dlt;
                r2 += ref * ref;
                s1 += fabs(dlt);
                mx = fmax(mx, fabs(dlt));
            }
        }
    red[0][threadIdx.x] = s2;
    red[1][threadIdx.x] = r2;
    red[2][threadIdx.x] = s1;
    // max via integer atomics on the non-negative double's bits
    atomicMax(reinterpret_cast<unsigned long long *>(stats + 2), (unsigned long long)__double_as_longlong(mx));
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(stats + 0, red[0][0]);
        atomicAdd(stats + 1, red[1][0]);
        atomicAdd(stats + 3, red[2][0]);
    }
}

}  // namespace gatlas

extern "C" size_t gatlas_matmul_workspace_size(const gatlas_matmul_desc *d) {
    if (!d) return 0;
    gatlas::Geometry g;
    if (!gatlas::resolve_geometry(d, &g)) return 0;
    return gatlas::tc_workspace_bytes(d, g);
}

extern "C" int gatlas_matmul_f32(const gatlas_matmul_desc *d, const float *A, const float *B, float *C,
                                 void *workspace, size_t workspace_bytes, void *stream) {
    return gatlas::matmul_dispatch<float>(d, A, B, C, workspace, workspace_bytes, (cudaStream_t)stream);
}

// Host buffers in, host buffer out (the reference's bus-transfer timing
// modes, GatlasBenchmark.cpp:198-265, as one call).  Tensor-core engines with
// one instance and at least two row blocks (option "host_block_rows", 512 by
// default) run as a pipeline on three library streams: uploads of B and of
// the row blocks of A, preparation and contraction of each block as it
// lands, downloads of each block's rows of C.  Everything else uploads the
// operands, runs the engine and downloads C on `stream`.
extern "C" int gatlas_matmul_f32_host(const gatlas_matmul_desc *d, const float *A, const float *B, float *C,
                                      void *stream) {
    using namespace gatlas;
    if (!d) return set_error(GATLAS_ERR_INVALID, "matmul_host: null descriptor");
    Geometry g;
    if (!resolve_geometry(d, &g)) return set_error(GATLAS_ERR_INVALID, "matmul_host: invalid dimensions");
    if (g.M == 0 || g.N == 0) return GATLAS_OK;
    if (!C || (g.K > 0 && (!A || !B))) return set_error(GATLAS_ERR_INVALID, "matmul_host: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    const bool tc = d->engine >= GATLAS_ENGINE_TC_BF16 && d->engine <= GATLAS_ENGINE_TC_FP8;
    if (tc && tcg::host_pipeline_ok(d, g)) {
        void *dev = device_scratch(tcg::host_pipeline_bytes(d, g), 1);
        if (!dev) return set_error(GATLAS_ERR_NOMEM, "matmul_host: device copies");
        return tcg::host_pipeline(d, g, A, B, C, dev, s);
    }
    // Exact extents: the last stored row of an operand holds only its inner
    // dimension, so the caller's buffer may end there.  Copies read and write
    // nothing outside [0, extent) of each host buffer, and C comes back row by
    // row (ldc may exceed N; padding columns and gaps between instances stay
    // as the caller left them).
    const int64_t a_rows = g.ta ? g.K : g.M, a_inner = g.ta ? g.M : g.K;
    const int64_t b_rows = g.tb ? g.N : g.K, b_inner = g.tb ? g.K : g.N;
    auto extent = [&](int64_t stride, int64_t rows, int64_t ld, int64_t inner) {
        return (size_t)((g.batch - 1) * stride + (rows - 1) * ld + inner);
    };
    const size_t a_el = g.K ? extent(g.stride_a, a_rows, g.lda, a_inner) : 0;
    const size_t b_el = g.K ? extent(g.stride_b, b_rows, g.ldb, b_inner) : 0;
    const size_t c_el = extent(g.stride_c, g.M, g.ldc, g.N);
    auto r1k = [](size_t b) { return (b + 1023) / 1024 * 1024; };
    uint8_t *dev = static_cast<uint8_t *>(device_scratch(r1k(a_el * 4) + r1k(b_el * 4) + r1k(c_el * 4) + 1024, 1));
    if (!dev) return set_error(GATLAS_ERR_NOMEM, "matmul_host: device copies");
    float *dA = reinterpret_cast<float *>(dev), *dB = reinterpret_cast<float *>(dev + r1k(a_el * 4));
    float *dC = reinterpret_cast<float *>(dev + r1k(a_el * 4) + r1k(b_el * 4));
    if ((a_el && cudaMemcpyAsync(dA, A, a_el * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) ||
        (b_el && cudaMemcpyAsync(dB, B, b_el * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) ||
        (d->gemm && d->beta != 0.0 && cudaMemcpyAsync(dC, C, c_el * 4, cudaMemcpyHostToDevice, s) != cudaSuccess))
        return check_launch("matmul_host upload");
    const int rc = gatlas_matmul_f32(d, dA, dB, dC, nullptr, 0, stream);
    if (rc) return rc;
    for (int64_t p = 0; p < g.batch; ++p) {
        const int64_t off = p * g.stride_c;
        const cudaError_t e =
            g.ldc == g.N ? cudaMemcpyAsync(C + off, dC + off, (size_t)(g.M * g.N) * 4, cudaMemcpyDeviceToHost, s)
                         : cudaMemcpy2DAsync(C + off, g.ldc * 4, dC + off, g.ldc * 4, g.N * 4, g.M,
                                             cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) return check_launch("matmul_host download");
    }
    return GATLAS_OK;
}

extern "C" int gatlas_matmul_f64(const gatlas_matmul_desc *d, const double *A, const double *B, double *C,
                                 void *workspace, size_t workspace_bytes, void *stream) {
    return gatlas::matmul_dispatch<double>(d, A, B, C, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" int gatlas_matmul_supported(int scalar, const gatlas_matmul_desc *d) {
    if (!d) return 0;
    if (d->engine == GATLAS_ENGINE_BUFFER) {
        if (d->group_h == 0 && d->group_w == 0 && d->block_h == 0 && d->block_w == 0) return 1;
        const int vl = d->vector_length ? (int)d->vector_length : 1;
        if (gatlas::simt::find(scalar, d->trans_a != 0, d->trans_b != 0, (int)d->group_h, (int)d->group_w,
                               (int)d->block_h, (int)d->block_w, vl) != nullptr)
            return 1;
        const gatlas::jit::Point pt{scalar, d->trans_a != 0, d->trans_b != 0, (int)d->group_h, (int)d->group_w,
                                    (int)d->block_h, (int)d->block_w, vl};
        return gatlas::jit::available() && gatlas::jit::point_ok(pt) ? 2 : 0;
    }
    if (d->engine == GATLAS_ENGINE_IMAGE) return gatlas::image_supported(scalar, d);
    return scalar == 0 && gatlas::tc_supported(d);
}

namespace gatlas {

int matmul_residual(const Geometry &g, double alpha, double beta, int gemm, const float *A, const float *B,
                    const float *Cin, const float *C, double *out_host, cudaStream_t stream) {
    double *stats = static_cast<double *>(device_scratch(4 * sizeof(double)));
    if (!stats) return set_error(GATLAS_ERR_NOMEM, "residual: scratch");
    cudaError_t e = cudaMemsetAsync(stats, 0, 4 * sizeof(double), stream);
    if (e != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "residual: %s", cudaGetErrorString(e));
    dim3 grid((unsigned)((g.N + kResTile - 1) / kResTile), (unsigned)((g.M + kResTile - 1) / kResTile));
    residual_kernel<<<grid, 256, 0, stream>>>(A, B, Cin, C, g.M, g.N, g.K, g.lda, g.ldb, g.ldc, g.ta, g.tb, alpha,
                                              beta, gemm, stats);
    int rc = check_launch("residual_kernel");
    if (rc) return rc;
    double h[4];
    e = cudaMemcpyAsync(h, stats, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "residual: %s", cudaGetErrorString(e));
    out_host[0] = std::sqrt(h[0]);
    out_host[1] = std::sqrt(h[1]);
    out_host[2] = h[2];
    out_host[3] = h[3];
    return GATLAS_OK;
}

}  // namespace gatlas

extern "C" int gatlas_matmul_residual_f32(const gatlas_matmul_desc *d, const float *A, const float *B,
                                          const float *C, double *out_host, void *stream_) {
    using namespace gatlas;
    if (!d || !out_host) return set_error(GATLAS_ERR_INVALID, "residual: null argument");
    Geometry g;
    if (!resolve_geometry(d, &g)) return set_error(GATLAS_ERR_INVALID, "residual: invalid dimensions");
    if (g.batch != 1) return set_error(GATLAS_ERR_INVALID, "residual: batch must be 1");
    if (d->gemm && d->beta != 0.0)
        return set_error(GATLAS_ERR_INVALID, "residual: beta must be 0 (C holds the product)");
    return matmul_residual(g, d->alpha, 0.0, d->gemm, A, B, nullptr, C, out_host, (cudaStream_t)stream_);
}
