/*
 * Oracle for the GATLAS GEMM / GEMV / SAXPY hot path (CPU restatement).
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline legs as the checker or the timed CPU baseline,
 * never by the product library.
 *
 * Build: oracle/Makefile.  It must be compiled with -ffp-contract=off so that
 * ORACLE_REFHOST rounds every product and every sum separately, as the
 * reference's own g++ -O2 x86-64 build of its host loops does.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ----------------------------------------------------------------------- */
/* random streams                                                           */
/* ----------------------------------------------------------------------- */

/* The reference never seeds drand48 (OCLAppUtil.hpp:28-33).  glibc's
 * never-seeded generator starts from state X0 = 0 with the standard
 * multiplier 0x5DEECE66D and addend 0xB (first value 11 / 2^48); seed48 with
 * a zero state restores exactly that stream. */
void oracle_drand48_reset(void) {
    unsigned short s[3] = {0, 0, 0};
    seed48(s);
}

double oracle_drand48(void) { return drand48(); }

/* posrand<float>: `SCALAR_TYPE a; while (0 == (a = drand48())) ;`
 * (OCLAppUtil.hpp:28-33).  The double is rounded to float before the test. */
float oracle_posrand_f32(void) {
    float a;
    while (0 == (a = (float)drand48())) ;
    return a;
}

double oracle_posrand_f64(void) {
    double a;
    while (0 == (a = drand48())) ;
    return a;
}

/* fillrand (OCLAppUtil.hpp:35-39) */
void oracle_fillrand_f32(float *out, size_t n) {
    for (size_t i = 0; i < n; i++) out[i] = oracle_posrand_f32();
}

void oracle_fillrand_f64(double *out, size_t n) {
    for (size_t i = 0; i < n; i++) out[i] = oracle_posrand_f64();
}

uint64_t oracle_splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* Element i of a seeded stream: splitmix64(splitmix64(seed) + offset + i).
 * Uniform [-1,1) floats carry 24 random bits and are formed exactly:
 * ((x >> 40) - 2^23) * 2^-23. */
void oracle_fill_uniform_f32(float *out, size_t n, uint64_t seed, uint64_t offset) {
    const uint64_t key = oracle_splitmix64(seed);
    for (size_t i = 0; i < n; i++) {
        const uint64_t x = oracle_splitmix64(key + offset + i);
        const int64_t q = (int64_t)(x >> 40) - (int64_t)(1 << 23);
        out[i] = (float)q * 0x1p-23f;
    }
}

void oracle_fill_uniform_f64(double *out, size_t n, uint64_t seed, uint64_t offset) {
    const uint64_t key = oracle_splitmix64(seed);
    for (size_t i = 0; i < n; i++) {
        const uint64_t x = oracle_splitmix64(key + offset + i);
        const int64_t q = (int64_t)(x >> 11) - ((int64_t)1 << 52);
        out[i] = (double)q * 0x1p-52;
    }
}

/* sign * 2^e with e uniform in [-8, 8]. */
void oracle_fill_pow2_f32(float *out, size_t n, uint64_t seed, uint64_t offset) {
    const uint64_t key = oracle_splitmix64(seed);
    for (size_t i = 0; i < n; i++) {
        const uint64_t x = oracle_splitmix64(key + offset + i);
        const int e = (int)((x >> 8) % 17) - 8;
        const float v = ldexpf(1.0f, e);
        out[i] = (x & 1) ? -v : v;
    }
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static int nthreads(int threads) {
    if (threads <= 0) return oracle_max_threads();
    return threads;
}

/* ----------------------------------------------------------------------- */
/* matmul                                                                   */
/* ----------------------------------------------------------------------- */

/* Element (i,k) of A and (k,j) of B for packed instance p, with the
 * reference's transpose index formulas (KernelMatmulBuffer.hpp:131-136):
 *   A: tA ? A[p*M*K + k*M + i] : A[p*M*K + i*K + k]
 *   B: tB ? B[p*K*N + j*K + k] : B[p*K*N + k*N + j]                          */
#define AIDX(p, i, k) ((p) * M * K + (tA ? (k) * M + (i) : (i) * K + (k)))
#define BIDX(p, k, j) ((p) * K * N + (tB ? (j) * K + (k) : (k) * N + (j)))

int oracle_matmul_f32(int mode, size_t packed, int gemm, size_t M, size_t N, size_t K,
                      int tA, int tB, const float *A, const float *B, const float *Cin,
                      float alpha, float beta, float *C, int threads) {
    if (mode != ORACLE_REFHOST && mode != ORACLE_FMA) return -1;
    const long rows = (long)(packed * M);
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (long r = 0; r < rows; r++) {
        const size_t p = (size_t)r / M, i = (size_t)r % M;
        for (size_t j = 0; j < N; j++) {
            float acc = 0;  /* fillconst(_paranoidC, 0) (KernelMatmulBuffer.hpp:121) */
            if (mode == ORACLE_REFHOST) {
                for (size_t k = 0; k < K; k++) {
                    const float prod = A[AIDX(p, i, k)] * B[BIDX(p, k, j)];
                    acc = acc + prod;
                }
            } else {
                for (size_t k = 0; k < K; k++)
                    acc = fmaf(A[AIDX(p, i, k)], B[BIDX(p, k, j)], acc);
            }
            const size_t o = p * M * N + i * N + j;
            if (gemm) {
                if (mode == ORACLE_REFHOST) {
                    /* alpha * C + beta * Cin (KernelMatmulBuffer.hpp:139-142) */
                    const float t1 = alpha * acc;
                    const float t2 = beta * Cin[o];
                    C[o] = t1 + t2;
                } else {
                    /* mad(alpha, accum, beta * C) (KernelMatmulBuffer.hpp:328-335);
                     * C is not read when beta == 0 (BLAS convention). */
                    const float bc = (beta == 0.0f) ? 0.0f : beta * Cin[o];
                    C[o] = fmaf(alpha, acc, bc);
                }
            } else {
                C[o] = acc;
            }
        }
    }
    return 0;
}

int oracle_matmul_f32_acc64(size_t packed, int gemm, size_t M, size_t N, size_t K,
                            int tA, int tB, const float *A, const float *B, const float *Cin,
                            double alpha, double beta, double *C, int threads) {
    const long rows = (long)(packed * M);
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (long r = 0; r < rows; r++) {
        const size_t p = (size_t)r / M, i = (size_t)r % M;
        for (size_t j = 0; j < N; j++) {
            double acc = 0;
            for (size_t k = 0; k < K; k++)
                acc += (double)A[AIDX(p, i, k)] * (double)B[BIDX(p, k, j)];
            const size_t o = p * M * N + i * N + j;
            C[o] = gemm ? alpha * acc + (beta == 0.0 ? 0.0 : beta * (double)Cin[o]) : acc;
        }
    }
    return 0;
}

int oracle_matmul_f64(int mode, size_t packed, int gemm, size_t M, size_t N, size_t K,
                      int tA, int tB, const double *A, const double *B, const double *Cin,
                      double alpha, double beta, double *C, int threads) {
    if (mode != ORACLE_REFHOST && mode != ORACLE_FMA) return -1;
    const long rows = (long)(packed * M);
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (long r = 0; r < rows; r++) {
        const size_t p = (size_t)r / M, i = (size_t)r % M;
        for (size_t j = 0; j < N; j++) {
            double acc = 0;
            if (mode == ORACLE_REFHOST) {
                for (size_t k = 0; k < K; k++) {
                    const double prod = A[AIDX(p, i, k)] * B[BIDX(p, k, j)];
                    acc = acc + prod;
                }
            } else {
                for (size_t k = 0; k < K; k++)
                    acc = fma(A[AIDX(p, i, k)], B[BIDX(p, k, j)], acc);
            }
            const size_t o = p * M * N + i * N + j;
            if (gemm) {
                if (mode == ORACLE_REFHOST) {
                    const double t1 = alpha * acc;
                    const double t2 = beta * Cin[o];
                    C[o] = t1 + t2;
                } else {
                    const double bc = (beta == 0.0) ? 0.0 : beta * Cin[o];
                    C[o] = fma(alpha, acc, bc);
                }
            } else {
                C[o] = acc;
            }
        }
    }
    return 0;
}

/* The generated buffer kernel's own algorithm on host cores: one output tile
 * of tile_m x tile_n per work group (KernelBaseMatmul.cpp:364-376), work groups
 * run in parallel, every element accumulated as a fused mad chain over
 * k = 0..K-1 (KernelMatmulBuffer.hpp:257-323).  Results equal ORACLE_FMA.
 * Rows [row_begin, row_end) bound the work for timed samples. */
int oracle_matmul_tiled_f32(size_t M, size_t N, size_t K, int tA, int tB,
                            const float *A, const float *B, float *C,
                            size_t tile_m, size_t tile_n, size_t row_begin, size_t row_end,
                            int threads) {
    if (tile_m == 0 || tile_n == 0 || tile_m > 256 || tile_n > 256) return -1;
    if (row_end > M) row_end = M;
    if (row_begin >= row_end) return 0;
    const size_t p = 0;
    const size_t tiles_m = (row_end - row_begin + tile_m - 1) / tile_m;
    const size_t tiles_n = (N + tile_n - 1) / tile_n;
    const long tiles = (long)(tiles_m * tiles_n);
#pragma omp parallel num_threads(nthreads(threads))
    {
        float *acc = (float *)malloc(sizeof(float) * tile_m * tile_n);
        float *brow = (float *)malloc(sizeof(float) * tile_n);
#pragma omp for schedule(dynamic, 1)
        for (long t = 0; t < tiles; t++) {
            const size_t i0 = row_begin + ((size_t)t / tiles_n) * tile_m;
            const size_t j0 = ((size_t)t % tiles_n) * tile_n;
            const size_t im = (i0 + tile_m <= row_end) ? tile_m : row_end - i0;
            const size_t jn = (j0 + tile_n <= N) ? tile_n : N - j0;
            memset(acc, 0, sizeof(float) * tile_m * tile_n);
            for (size_t k = 0; k < K; k++) {
                for (size_t jj = 0; jj < jn; jj++) brow[jj] = B[BIDX(p, k, j0 + jj)];
                for (size_t ii = 0; ii < im; ii++) {
                    const float a = A[AIDX(p, i0 + ii, k)];
                    float *row = acc + ii * tile_n;
                    for (size_t jj = 0; jj < jn; jj++) row[jj] = fmaf(a, brow[jj], row[jj]);
                }
            }
            for (size_t ii = 0; ii < im; ii++)
                memcpy(C + (i0 + ii) * N + j0, acc + ii * tile_n, sizeof(float) * jn);
        }
        free(acc);
        free(brow);
    }
    return 0;
}

#undef AIDX
#undef BIDX

/* ----------------------------------------------------------------------- */
/* matvec                                                                   */
/* ----------------------------------------------------------------------- */

/* A element (i,j) of packed instance p (KernelMatvecBuffer.hpp:128-131):
 *   tA ? A[p*M*N + j*M + i] : A[p*M*N + i*N + j]                           */
#define VIDX(p, i, j) ((p) * M * N + (tA ? (j) * M + (i) : (i) * N + (j)))

int oracle_matvec_f32(int mode, size_t packed, int gemv, size_t M, size_t N, int tA,
                      const float *A, const float *b, const float *cin,
                      float alpha, float beta, float *c, int threads) {
    if (mode != ORACLE_REFHOST && mode != ORACLE_FMA) return -1;
    const long rows = (long)(packed * M);
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (long r = 0; r < rows; r++) {
        const size_t p = (size_t)r / M, i = (size_t)r % M;
        float acc = 0;
        if (mode == ORACLE_REFHOST) {
            for (size_t j = 0; j < N; j++) {
                const float prod = A[VIDX(p, i, j)] * b[p * N + j];
                acc = acc + prod;
            }
        } else {
            for (size_t j = 0; j < N; j++) acc = fmaf(A[VIDX(p, i, j)], b[p * N + j], acc);
        }
        const size_t o = p * M + i;
        if (gemv) {
            if (mode == ORACLE_REFHOST) {
                const float t1 = alpha * acc;
                const float t2 = beta * cin[o];
                c[o] = t1 + t2;
            } else {
                const float bc = (beta == 0.0f) ? 0.0f : beta * cin[o];
                c[o] = fmaf(alpha, acc, bc);
            }
        } else {
            c[o] = acc;
        }
    }
    return 0;
}

int oracle_matvec_f32_acc64(size_t packed, int gemv, size_t M, size_t N, int tA,
                            const float *A, const float *b, const float *cin,
                            double alpha, double beta, double *c, int threads) {
    const long rows = (long)(packed * M);
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (long r = 0; r < rows; r++) {
        const size_t p = (size_t)r / M, i = (size_t)r % M;
        double acc = 0;
        for (size_t j = 0; j < N; j++) acc += (double)A[VIDX(p, i, j)] * (double)b[p * N + j];
        const size_t o = p * M + i;
        c[o] = gemv ? alpha * acc + (beta == 0.0 ? 0.0 : beta * (double)cin[o]) : acc;
    }
    return 0;
}

int oracle_matvec_f64(int mode, size_t packed, int gemv, size_t M, size_t N, int tA,
                      const double *A, const double *b, const double *cin,
                      double alpha, double beta, double *c, int threads) {
    if (mode != ORACLE_REFHOST && mode != ORACLE_FMA) return -1;
    const long rows = (long)(packed * M);
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (long r = 0; r < rows; r++) {
        const size_t p = (size_t)r / M, i = (size_t)r % M;
        double acc = 0;
        if (mode == ORACLE_REFHOST) {
            for (size_t j = 0; j < N; j++) {
                const double prod = A[VIDX(p, i, j)] * b[p * N + j];
                acc = acc + prod;
            }
        } else {
            for (size_t j = 0; j < N; j++) acc = fma(A[VIDX(p, i, j)], b[p * N + j], acc);
        }
        const size_t o = p * M + i;
        if (gemv) {
            if (mode == ORACLE_REFHOST) {
                const double t1 = alpha * acc;
                const double t2 = beta * cin[o];
                c[o] = t1 + t2;
            } else {
                const double bc = (beta == 0.0) ? 0.0 : beta * cin[o];
                c[o] = fma(alpha, acc, bc);
            }
        } else {
            c[o] = acc;
        }
    }
    return 0;
}

#undef VIDX

/* ----------------------------------------------------------------------- */
/* saxpy                                                                    */
/* ----------------------------------------------------------------------- */

/* REFHOST: Z[i] = alpha * X[i] + Y[i] (KernelSaxpyBuffer.hpp:118-120).
 * FMA:     Z = mad(alpha, X, Y)        (KernelSaxpyBuffer.hpp:186-190).
 * z may alias y (in-place y <- a*x + y). */
int oracle_saxpy_f32(int mode, size_t n, float alpha, const float *x, const float *y,
                     float *z, int threads) {
    if (mode != ORACLE_REFHOST && mode != ORACLE_FMA) return -1;
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (long i = 0; i < (long)n; i++) {
        if (mode == ORACLE_REFHOST) {
            const float t = alpha * x[i];
            z[i] = t + y[i];
        } else {
            z[i] = fmaf(alpha, x[i], y[i]);
        }
    }
    return 0;
}

int oracle_saxpy_f64(int mode, size_t n, double alpha, const double *x, const double *y,
                     double *z, int threads) {
    if (mode != ORACLE_REFHOST && mode != ORACLE_FMA) return -1;
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (long i = 0; i < (long)n; i++) {
        if (mode == ORACLE_REFHOST) {
            const double t = alpha * x[i];
            z[i] = t + y[i];
        } else {
            z[i] = fma(alpha, x[i], y[i]);
        }
    }
    return 0;
}

/* ----------------------------------------------------------------------- */
/* checks                                                                   */
/* ----------------------------------------------------------------------- */

/* absdiff: sum |m1 - m2| in long double (OCLAppUtil.hpp:47-53).  The
 * paranoid check passes iff absdiff < 1/length (OCLAppUtil.hpp:212-264). */
long double oracle_absdiff_f32(const float *a, const float *b, size_t n) {
    long double acc = 0;
    for (size_t i = 0; i < n; i++) acc += fabsl((long double)(a[i] - b[i]));
    return acc;
}

long double oracle_absdiff_f64(const double *a, const double *b, size_t n) {
    long double acc = 0;
    for (size_t i = 0; i < n; i++) acc += fabsl((long double)(a[i] - b[i]));
    return acc;
}

/* checkArray: every element equals the test value (OCLAppUtil.hpp:55-61). */
int oracle_check_pattern_f32(const float *a, size_t n, float value) {
    for (size_t i = 0; i < n; i++)
        if (a[i] != value) return 0;
    return 1;
}

int oracle_check_pattern_f64(const double *a, size_t n, double value) {
    for (size_t i = 0; i < n; i++)
        if (a[i] != value) return 0;
    return 1;
}

/* ----------------------------------------------------------------------- */
/* FP8 E4M3 block quantisation and the dequantised product                  */
/* ----------------------------------------------------------------------- */

uint8_t oracle_e4m3_encode(float x) {
    if (isnan(x)) return 0x7F;
    const uint8_t sign = signbit(x) ? 0x80 : 0x00;
    const double a = fabs((double)x);
    if (a >= 448.0) return sign | 0x7E; /* saturate */
    int code;
    if (a < 0x1p-6) {
        /* subnormal quantum 2^-9; a result of 8 is the smallest normal 0x08 */
        code = (int)nearbyint(a * 0x1p9);
    } else {
        int e;
        frexp(a, &e);            /* a = f * 2^e, f in [0.5, 1) */
        const int E = e - 1;     /* floor(log2 a), in [-6, 8] */
        const int mm = (int)nearbyint(ldexp(a, 3 - E)); /* 8..16; 16 carries into the exponent */
        code = ((E + 7) << 3) + mm - 8;
    }
    return sign | (uint8_t)code;
}

float oracle_e4m3_decode(uint8_t c) {
    const int e = (c >> 3) & 15, m = c & 7;
    if (e == 15 && m == 7) return NAN;
    const double v = e == 0 ? ldexp((double)m, -9) : ldexp((double)(8 + m), e - 10);
    return (float)((c & 0x80) ? -v : v);
}

void oracle_e4m3_encode_n(const float *x, uint8_t *out, size_t n) {
    for (size_t i = 0; i < n; i++) out[i] = oracle_e4m3_encode(x[i]);
}

void oracle_e4m3_decode_n(const uint8_t *c, float *out, size_t n) {
    for (size_t i = 0; i < n; i++) out[i] = oracle_e4m3_decode(c[i]);
}

#define QB 128

int oracle_quant_fp8(size_t batch, size_t rows, size_t K, size_t Kp, int transposed, size_t ld,
                     size_t src_stride, const float *src, uint8_t *codes, float *scales) {
    if (Kp < K) return -1;
    const size_t rblocks = (rows + QB - 1) / QB, kblocks = (K + QB - 1) / QB;
    for (size_t z = 0; z < batch; z++) {
        const float *s0 = src + z * src_stride;
        uint8_t *c0 = codes + z * rows * Kp;
        for (size_t rb = 0; rb < rblocks; rb++)
            for (size_t kb = 0; kb < kblocks; kb++) {
                const size_t r_end = rb * QB + QB < rows ? rb * QB + QB : rows;
                const size_t k_end = kb * QB + QB < K ? kb * QB + QB : K;
                float amax = 0.0f;
                for (size_t r = rb * QB; r < r_end; r++)
                    for (size_t k = kb * QB; k < k_end; k++) {
                        const float x = transposed ? s0[k * ld + r] : s0[r * ld + k];
                        const float ax = fabsf(x);
                        if (ax > amax) amax = ax;
                    }
                /* smallest power of two with amax / s <= 448 */
                float s = 0.0f;
                if (amax > 0.0f) {
                    int e;
                    const float f = frexpf(amax, &e);
                    s = ldexpf(1.0f, e - 9 + (f > 0.875f ? 1 : 0));
                }
                scales[(z * rblocks + rb) * kblocks + kb] = s;
                /* codes of this block, including the zero padding up to Kp
                 * that falls inside the last block */
                const size_t kc_end = kb + 1 == kblocks ? Kp : kb * QB + QB;
                for (size_t r = rb * QB; r < r_end; r++)
                    for (size_t k = kb * QB; k < kc_end; k++) {
                        const float x = k < K ? (transposed ? s0[k * ld + r] : s0[r * ld + k]) : 0.0f;
                        c0[r * Kp + k] = s == 0.0f ? 0 : oracle_e4m3_encode(x / s);
                    }
            }
    }
    return 0;
}

int oracle_matmul_fp8_dequant(size_t batch, int gemm, size_t M, size_t N, size_t K, size_t Kp,
                              const uint8_t *qa, const float *sa, const uint8_t *qb, const float *sb,
                              double alpha, double beta, const float *Cin, double *out) {
    const size_t kblocks = (K + QB - 1) / QB, mblocks = (M + QB - 1) / QB, nblocks = (N + QB - 1) / QB;
    float lut[256];
    for (int c = 0; c < 256; c++) lut[c] = oracle_e4m3_decode((uint8_t)c);
#pragma omp parallel for collapse(2) schedule(static)
    for (size_t z = 0; z < batch; z++)
        for (size_t m = 0; m < M; m++) {
            const uint8_t *arow = qa + (z * M + m) * Kp;
            for (size_t n = 0; n < N; n++) {
                const uint8_t *brow = qb + (z * N + n) * Kp;
                double acc = 0.0;
                for (size_t kb = 0; kb < kblocks; kb++) {
                    double part = 0.0;
                    const size_t k_end = kb * QB + QB < K ? kb * QB + QB : K;
                    for (size_t k = kb * QB; k < k_end; k++) part += (double)lut[arow[k]] * (double)lut[brow[k]];
                    acc += part * (double)sa[(z * mblocks + m / QB) * kblocks + kb] *
                           (double)sb[(z * nblocks + n / QB) * kblocks + kb];
                }
                const size_t o = (z * M + m) * N + n;
                out[o] = gemm ? alpha * acc + beta * (double)Cin[o] : acc;
            }
        }
    return 0;
}
