/*
 * Oracle for the GATLAS GEMM / GEMV / SAXPY hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a CPU restatement of the reference's
 * host-side reference computations and of its kernels' accumulation order.
 * Only tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg and
 * its --impl reference arm) may load it, and only as the checker or as the
 * timed CPU baseline.  The product library never links or calls it.
 *
 * Reference files are cited by their path inside the GATLAS project.
 *
 * Arithmetic modes (all accumulate k = 0..K-1 sequentially per output, the
 * order the reference's host loop and its generated kernels both use):
 *   ORACLE_REFHOST : product and sum rounded separately in the kernel's own
 *                    precision, exactly the reference's paranoid host loop
 *                    (KernelMatmulBuffer.hpp:124-143, KernelMatvecBuffer.hpp:122-138,
 *                    KernelSaxpyBuffer.hpp:118-120) compiled without FMA contraction.
 *   ORACLE_FMA     : one fused multiply-add per step, what the generated OpenCL
 *                    `mad` chain computes on a device with fused mad
 *                    (KernelMatmulBuffer.hpp:302-337, KernelMatvecBuffer.hpp:281-320,
 *                    KernelSaxpyBuffer.hpp:186-190).
 *   ORACLE_F64     : the same products accumulated in double (FP64 oracle).
 */
#ifndef GATLAS_ORACLE_H
#define GATLAS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_REFHOST = 0, ORACLE_FMA = 1, ORACLE_F64 = 2 };

/* ---- random streams -------------------------------------------------- */
void   oracle_drand48_reset(void);
double oracle_drand48(void);
float  oracle_posrand_f32(void);
double oracle_posrand_f64(void);
void   oracle_fillrand_f32(float *out, size_t n);
void   oracle_fillrand_f64(double *out, size_t n);

/* Counter-based seeded generators shared with the device generators. */
uint64_t oracle_splitmix64(uint64_t x);
void oracle_fill_uniform_f32(float *out, size_t n, uint64_t seed, uint64_t offset);
void oracle_fill_uniform_f64(double *out, size_t n, uint64_t seed, uint64_t offset);
void oracle_fill_pow2_f32(float *out, size_t n, uint64_t seed, uint64_t offset);

/* ---- matmul ------------------------------------------------------------ */
int oracle_matmul_f32(int mode, size_t packed, int gemm, size_t M, size_t N, size_t K,
                      int tA, int tB, const float *A, const float *B, const float *Cin,
                      float alpha, float beta, float *C, int threads);
int oracle_matmul_f32_acc64(size_t packed, int gemm, size_t M, size_t N, size_t K,
                            int tA, int tB, const float *A, const float *B, const float *Cin,
                            double alpha, double beta, double *C, int threads);
int oracle_matmul_f64(int mode, size_t packed, int gemm, size_t M, size_t N, size_t K,
                      int tA, int tB, const double *A, const double *B, const double *Cin,
                      double alpha, double beta, double *C, int threads);
int oracle_matmul_tiled_f32(size_t M, size_t N, size_t K, int tA, int tB,
                            const float *A, const float *B, float *C,
                            size_t tile_m, size_t tile_n, size_t row_begin, size_t row_end,
                            int threads);

/* ---- matvec ------------------------------------------------------------ */
int oracle_matvec_f32(int mode, size_t packed, int gemv, size_t M, size_t N, int tA,
                      const float *A, const float *b, const float *cin,
                      float alpha, float beta, float *c, int threads);
int oracle_matvec_f32_acc64(size_t packed, int gemv, size_t M, size_t N, int tA,
                            const float *A, const float *b, const float *cin,
                            double alpha, double beta, double *c, int threads);
int oracle_matvec_f64(int mode, size_t packed, int gemv, size_t M, size_t N, int tA,
                      const double *A, const double *b, const double *cin,
                      double alpha, double beta, double *c, int threads);

/* ---- saxpy ------------------------------------------------------------- */
int oracle_saxpy_f32(int mode, size_t n, float alpha, const float *x, const float *y,
                     float *z, int threads);
int oracle_saxpy_f64(int mode, size_t n, double alpha, const double *x, const double *y,
                     double *z, int threads);

/* ---- checks (OCLAppUtil.hpp:47-61, 212-264) ---------------------------- */
long double oracle_absdiff_f32(const float *a, const float *b, size_t n);
long double oracle_absdiff_f64(const double *a, const double *b, size_t n);
int oracle_check_pattern_f32(const float *a, size_t n, float value);
int oracle_check_pattern_f64(const double *a, size_t n, double value);
int oracle_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
