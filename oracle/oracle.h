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
/* FP8 E4M3 operands of the tensor-core FP8 engine (no reference
 * counterpart: the reference has no 8-bit path).  Encoding: 1 sign, 4
 * exponent bits (bias 7), 3 mantissa bits, no infinities, 0x7F/0xFF NaN,
 * largest finite 448; rounding to nearest even with saturation to +-448.
 * Block quantisation: one FP32 scale per 128 x 128 block of the K-major
 * operand (rows x K), s = the smallest power of two with amax / s <= 448,
 * code = e4m3(x / s), s = 0 and all codes 0 for an all-zero block; codes
 * laid out [batch][rows][Kp], zero for k >= K. */
uint8_t oracle_e4m3_encode(float x);
float   oracle_e4m3_decode(uint8_t c);
void    oracle_e4m3_encode_n(const float *x, uint8_t *out, size_t n);
void    oracle_e4m3_decode_n(const uint8_t *c, float *out, size_t n);
int oracle_quant_fp8(size_t batch, size_t rows, size_t K, size_t Kp, int transposed, size_t ld,
                     size_t src_stride, const float *src, uint8_t *codes, float *scales);
/* C = sum over K blocks of sa*sb * (sum of decoded code products), in FP64,
 * with alpha/beta applied when gemm != 0 (Cin read then). */
int oracle_matmul_fp8_dequant(size_t batch, int gemm, size_t M, size_t N, size_t K, size_t Kp,
                              const uint8_t *qa, const float *sa, const uint8_t *qb, const float *sb,
                              double alpha, double beta, const float *Cin, double *out);

long double oracle_absdiff_f32(const float *a, const float *b, size_t n);
long double oracle_absdiff_f64(const double *a, const double *b, size_t n);
int oracle_check_pattern_f32(const float *a, size_t n, float value);
int oracle_check_pattern_f64(const double *a, size_t n, double value);
int oracle_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
