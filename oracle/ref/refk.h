/* C interface of the reference's generated kernels compiled for the host CPU.
 *
 * TEST INFRASTRUCTURE: gen_kernels.py emits, for every kernel point it
 * builds, two entry points refk_<id>_fma and refk_<id>_sep (mad fused, or
 * rounded as a separate product and sum) with this signature.  Operands are
 * row-major host arrays in the reference's layouts; image operands are the
 * same arrays read as RGBA texels (clshim.hpp).  M, N, K and the work sizes
 * are fixed when the kernel is generated.
 */
#ifndef GATLAS_ORACLE_REFK_H
#define GATLAS_ORACLE_REFK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct refk_args {
    const void *A, *B; /* matmul A, B; matvec A, x; saxpy X, Y */
    void *C;           /* matmul C, matvec y, saxpy Z (read too when the kernel reads it: GEMM/GEMV) */
    double alpha, beta;
    /* work groups to run: [begin, end) per dimension; end 0 = all */
    size_t group_begin[2], group_end[2];
    int threads; /* 0 = every OpenMP thread */
} refk_args;

typedef struct refk_launch {
    size_t global[2], local[2];
    size_t group_begin[2], group_end[2];
    size_t local_bytes[2]; /* __local arguments tmpA, tmpB */
    int uses_barrier;
    int threads;
} refk_launch;

typedef void (*refk_body)(void *arg, void *local0, void *local1);

/* Runs every work item of the selected work groups; 0 on success. */
int refk_run_groups(const refk_launch *launch, refk_body body, void *arg);

#ifdef __cplusplus
}
#endif

#endif
