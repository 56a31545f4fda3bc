/*
 * gatlas_b200 — C ABI of the B200-native GEMM / GEMV / SAXPY hot path.
 *
 * Plain C: no C++ or torch types cross this boundary.  Every entry point
 * returns an int status (GATLAS_OK == 0, negative on error) unless stated
 * otherwise; gatlas_last_error() returns the calling thread's last message.
 * Device pointers are caller-owned CUDA device memory on the current device;
 * `stream` is a cudaStream_t passed as void* (NULL = the legacy default stream).
 *
 * Each declaration cites the reference (GATLAS) interface it replaces.  The
 * reference has no C ABI: its plugin boundary is the C++ virtual interface
 * KernelInterface (GatlasBenchmark.hpp:28-58) plus the KernelBase* setters,
 * and its device boundary is clEnqueueNDRangeKernel on generated OpenCL C.
 */
#ifndef GATLAS_B200_H
#define GATLAS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status ------------------------------------------------------------ */
#define GATLAS_OK 0
#define GATLAS_ERR_INVALID (-1)     /* invalid argument or parameter point */
#define GATLAS_ERR_CUDA (-2)        /* CUDA runtime / driver error */
#define GATLAS_ERR_UNSUPPORTED (-3) /* valid point with no kernel built for it */
#define GATLAS_ERR_TIMEOUT (-4)     /* a bounded device wait expired */
#define GATLAS_ERR_NOMEM (-5)       /* allocation failed */
#define GATLAS_ERR_CHECK (-6)       /* output check failed */
#define GATLAS_ERR_STATE (-7)       /* call out of order (e.g. run before set_args) */

int gatlas_version(void);
const char *gatlas_status_string(int status);
/* Copies the calling thread's last error message; returns its length. */
size_t gatlas_last_error(char *buf, size_t len);

/* ---- enums ------------------------------------------------------------- */
/* Engines.  BUFFER and IMAGE are the reference's two kernel families
 * ("matmulbuffer", "matmulimage", ...); on B200 the image family loads its
 * operands with TMA tensor-map / bulk copies instead of texture fetches.
 * The TC_* engines are tcgen05 tensor-core contractions (no reference
 * counterpart): BF16 operands with FP32 accumulation, FP32 operands split
 * into BF16 pieces (3 or 6 products), FP8 E4M3 with FP32 block scales. */
enum {
    GATLAS_ENGINE_BUFFER = 0,
    GATLAS_ENGINE_IMAGE = 1,
    GATLAS_ENGINE_TC_BF16 = 2,
    GATLAS_ENGINE_TC_SPLIT3 = 3,
    GATLAS_ENGINE_TC_SPLIT6 = 4,
    GATLAS_ENGINE_TC_FP8 = 5
};

enum { GATLAS_DIST_UNIFORM = 0, GATLAS_DIST_POW2 = 1, GATLAS_DIST_CONST = 2 };

/* ---- SAXPY --------------------------------------------------------------
 * z[i] = fma(alpha, x[i], y[i]) for i < n; z may alias y (in place).
 * Replaces KernelSaxpyBuffer<float,VL> / KernelSaxpyImage<float,4>
 * (KernelSaxpyBuffer.hpp:143-225, KernelSaxpyImage.hpp:148-233), whose
 * generated kernels compute Z = mad(alpha, X, Y).  Results are bit-exact
 * against a per-element fmaf. */
int gatlas_saxpy_f32(int engine, size_t n, float alpha, const float *x, const float *y, float *z,
                     void *stream);
int gatlas_saxpy_f64(int engine, size_t n, double alpha, const double *x, const double *y,
                     double *z, void *stream);

/* ---- GEMV ---------------------------------------------------------------
 * y[p] = A[p]·x[p] (gemv == 0) or alpha·A[p]·x[p] + beta·y[p] (gemv == 1)
 * for p < batch.  trans_a == 0: A is M×N row-major (element (i,j) at
 * A[i*lda + j], lda >= N); trans_a == 1: A is stored column-major (element
 * (i,j) at A[j*lda + i], lda >= M), the reference's transposeA layout
 * (KernelMatvecBuffer.hpp:128-131).  Replaces KernelMatvecBuffer<float,VL>
 * and KernelMatvecImage<float,4> (KernelMatvecBuffer.hpp:180-325,
 * KernelMatvecImage.hpp:188-295).  Deterministic: the summation order
 * depends only on (M, N, engine) and the device's SM count.
 * `workspace` may be NULL, in which case the library uses an internal
 * per-device buffer; gatlas_matvec_workspace_size() gives the bytes needed
 * (the most that either engine, float or double, needs for these sizes on
 * the current device), and a workspace must start on a 256-byte boundary.
 * Calls that use the internal per-device buffers (here, gatlas_matmul_* with
 * no workspace, gatlas_matmul_f32_host) share them: calls on one device that
 * overlap on the GPU (several streams or host threads) race; serialise them or
 * pass workspaces. */
typedef struct gatlas_matvec_desc {
    int32_t engine;  /* GATLAS_ENGINE_BUFFER or GATLAS_ENGINE_IMAGE */
    int32_t gemv;
    int32_t trans_a;
    int32_t reserved0;
    uint64_t m, n, lda;
    uint64_t batch;                      /* packedCalc; 0 means 1 */
    uint64_t stride_a, stride_x, stride_y; /* elements between instances; 0 = dense */
    double alpha, beta;
} gatlas_matvec_desc;

size_t gatlas_matvec_workspace_size(const gatlas_matvec_desc *d);
int gatlas_matvec_f32(const gatlas_matvec_desc *d, const float *A, const float *x, float *y,
                      void *workspace, size_t workspace_bytes, void *stream);
int gatlas_matvec_f64(const gatlas_matvec_desc *d, const double *A, const double *x, double *y,
                      void *workspace, size_t workspace_bytes, void *stream);

/* Allocation-free float GEMV.  No counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc -- code inside a host framework that
 * owns all device memory, and latency-critical code that must not trigger the
 * device-wide synchronisation of cudaMalloc/cudaFree.  Same arguments and
 * results as gatlas_matvec_f32 without the workspace: the scratch of the
 * column-major path (per-segment partial sums and arrival counters) comes
 * from a fixed GATLAS_MATVEC_NOALLOC_SCRATCH_BYTES array of device memory
 * inside the library, which every GPU that loads the library holds until the
 * process exits.  The first call on each device looks the array's device
 * address up (cudaGetSymbolAddress), so make that first call before any stream
 * capture.  Problems that need more scratch are rejected with
 * GATLAS_ERR_INVALID.  All calls share the one array and each call clears
 * the counters it needs, so calls that overlap on the GPU (concurrent streams,
 * several host threads) race; serialise them. */
#define GATLAS_MATVEC_NOALLOC_SCRATCH_BYTES ((size_t)1 << 20)
int gatlas_matvec_f32_noalloc(const gatlas_matvec_desc *d, const float *A, const float *x, float *y,
                              void *stream);

/* ---- GEMM ---------------------------------------------------------------
 * C[p] = op(A[p])·op(B[p]) (gemm == 0) or alpha·op(A[p])·op(B[p]) + beta·C[p]
 * (gemm == 1; C is not read when beta == 0).  Layouts follow the reference
 * (KernelMatmulBuffer.hpp:131-136): trans_a == 0 → A is M×K row-major
 * (lda >= K); trans_a == 1 → A stored K×M row-major (lda >= M); trans_b == 0
 * → B is K×N row-major (ldb >= N); trans_b == 1 → B stored N×K row-major
 * (ldb >= K); C is M×N row-major (ldc >= N).  ld* == 0 means dense.
 * The SIMT tile is the reference's work-group × inner-blocking point
 * (KernelBaseMatmul.hpp:85-140): a group_h × group_w thread block computes a
 * (group_h·block_h) × (group_w·block_w) tile; vector_length is the width of
 * the global loads; extra is the reference's extra parameter (recorded, no
 * effect on the arithmetic).  Zeros select the tuned default.
 * Replaces KernelMatmulBuffer<SCALAR,VL> and KernelMatmulImage<SCALAR,VL>
 * (KernelMatmulBuffer.hpp:174-342, KernelMatmulImage.hpp:192-313).
 * SIMT engines accumulate k = 0..K-1 as one fused multiply-add chain per
 * element, bit-exact against a sequential fmaf chain.  For the TC_* engines
 * the tile fields are ignored and `extra` is the promotion interval: the
 * tensor cores accumulate `extra` K slices in TMEM before the partial sum is
 * added into round-to-nearest FP32 registers.  A slice is K = 64 for TC_BF16
 * and TC_SPLIT3 and K = 32 for TC_SPLIT6; 0 selects all of K for TC_BF16
 * (accumulated in TMEM; with M > 128 on 256 x 256 single-CTA tiles), K = 256
 * for TC_SPLIT3 and K = 128 for TC_SPLIT6.
 * GATLAS_ENGINE_TC_FP8 quantises each operand to E4M3 with one power-of-two
 * FP32 scale per 128 x 128 block (the smallest power of two s with
 * amax / s <= 448); runs of up to `extra` (0 selects 16) 128-deep blocks
 * whose scale products sa * sb are equal accumulate in TMEM and are promoted
 * scaled once, exactly (powers of two), K <= 131072; its
 * tc_prepare workspace holds [A codes][B codes][A scales][B scales][plan],
 * codes K-major [batch][rows][Kp] (Kp = K rounded up to 16), scales
 * [batch][rows/128][K/128], each part 1024-byte aligned; tc_run writes the
 * plan (each 128 x 256 tile's runs of equally scaled blocks) before it
 * contracts. */
typedef struct gatlas_matmul_desc {
    int32_t engine;
    int32_t gemm;
    int32_t trans_a, trans_b;
    uint64_t m, n, k;
    uint64_t lda, ldb, ldc;
    uint64_t batch;                       /* packedCalc; 0 means 1 */
    uint64_t stride_a, stride_b, stride_c; /* elements between instances; 0 = dense */
    double alpha, beta;
    uint32_t group_h, group_w, block_h, block_w, vector_length, extra;
} gatlas_matmul_desc;

/* Bytes of scratch the engine needs (split / quantised operand copies for the
 * TC_* engines, 0 for SIMT).  workspace may be NULL: the library then uses an
 * internal per-device buffer; otherwise it is 1024-byte aligned and at least
 * this size. */
size_t gatlas_matmul_workspace_size(const gatlas_matmul_desc *d);
int gatlas_matmul_f32(const gatlas_matmul_desc *d, const float *A, const float *B, float *C,
                      void *workspace, size_t workspace_bytes, void *stream);
int gatlas_matmul_f64(const gatlas_matmul_desc *d, const double *A, const double *B, double *C,
                      void *workspace, size_t workspace_bytes, void *stream);
/* Tensor-core engines in two steps, for operands that stay resident: prepare
 * writes the BF16 pieces of A and B into the workspace
 * (gatlas_matmul_workspace_size bytes, 1024-byte aligned); run contracts the
 * prepared pieces into C and may be repeated.  gatlas_matmul_f32 with a TC_*
 * engine is prepare followed by run.  No reference counterpart (the reference
 * regenerates and re-uploads operands per run, KernelMatmulBuffer.hpp:83-171). */
int gatlas_matmul_tc_prepare(const gatlas_matmul_desc *d, const float *A, const float *B, void *workspace,
                             size_t workspace_bytes, void *stream);
int gatlas_matmul_tc_run(const gatlas_matmul_desc *d, const void *workspace, size_t workspace_bytes, float *C,
                         void *stream);

/* Host buffers in and out: uploads op(A), op(B) (and C when gemm and
 * beta != 0), contracts and downloads C, ordered on `stream` (the call
 * returns before the work completes: keep A, B and C allocated and A and B
 * unchanged until the stream has completed, and synchronise it before
 * reading C).  Replaces the reference's bus-transfer timing modes -s/-r
 * (GatlasBenchmark.cpp:198-265).  Tensor-core engines with one instance and
 * M of at least two blocks (option "host_block_rows", 512 rows by default)
 * pipeline the transfers on three library streams: uploads (B, then A block
 * by block, back to back), preparation and contraction
 * of each block as it lands, and the download of each block's C rows as
 * its contraction finishes.  Use pinned host memory for the copies to
 * overlap.  Results are bit-identical to gatlas_matmul_f32. */
int gatlas_matmul_f32_host(const gatlas_matmul_desc *d, const float *A, const float *B, float *C, void *stream);

/* Library options.  "tc_pair": how tensor-core contractions with M > 128
 * tile C.  1 (default): CTA pairs (cta_group::2, a 256 x 256 tile per pair,
 * each CTA staging half of B) for split3 and split6; 256 x 256 tiles on
 * single CTAs for one-product BF16 over all of K once there are at least as
 * many such tiles as SMs; one CTA per 128 x 256 tile otherwise.  2: CTA
 * pairs always.  0: 128 x 256 tiles always.  Results are bit-identical in
 * every case (same pieces, same MMA order, same promotion).
 * "tc_group_rows": rows of C per raster group of the persistent
 * tensor-core contraction, a multiple of 128 (default 2048): the
 * tiles in flight cover a block of that height, whose operands share L2.
 * "host_block_rows": rows of A per pipelined block of gatlas_matmul_f32_host,
 * a multiple of 256 (default 512).
 * "tc_l2_hint": 1 (default) loads A's tiles in the persistent tensor-core
 * contraction with an evict-last L2 priority (A is reused by every tile
 * column of a raster group); 0 loads them plainly.  Results are identical.
 * "grouped_pair": how grouped contractions tile C.  0 (default): 128-row
 * tiles on single CTAs.  1: 256-row tiles on CTA pairs (an instance's row
 * blocks two at a time, each CTA staging half of the B tile; the second half
 * of an odd instance's last pair is computed and not stored).  Results are
 * bit-identical.  On the 1024-instance log-uniform mix pairs are slower
 * (split3 3.9 vs 3.5 ms, BF16 3.0 vs 2.3 ms).  Read when a plan is created. */
int gatlas_set_option(const char *name, int64_t value);
int gatlas_get_option(const char *name, int64_t *value);

/* 1 if a prebuilt kernel exists for (scalar 0=float/1=double, desc); 2 if
 * the SIMT point has no prebuilt instantiation but will be compiled on first
 * use (NVRTC, cached per device); 0 if it cannot run. */
int gatlas_matmul_supported(int scalar, const gatlas_matmul_desc *d);

/* ---- grouped GEMM --------------------------------------------------------
 * Many instances of different shapes and layouts in one persistent
 * tensor-core launch (engines GATLAS_ENGINE_TC_BF16 and
 * GATLAS_ENGINE_TC_SPLIT3).  Replaces what the reference can only do with
 * one kernel per problem: packedCalc batches equal shapes only
 * (KernelMatmulBuffer.hpp:229-230, benchMatmul.cpp -C).
 *
 * Lifetime: create (validates, lays out the packed workspace, balances the
 * output tiles over the SMs and uploads the tables; synchronous), then
 * prepare (one launch packing every operand into BF16 piece tiles) and run
 * (one launch contracting every instance), or launch_graph, which captures
 * [prepare +] run once into a CUDA graph and replays it.  Operand and C
 * pointers are bound at create and must stay valid.  run_each is the
 * comparator: one gatlas_matmul_f32 call per instance. */
#define GATLAS_GROUPED_BUCKETS 4

typedef struct gatlas_grouped_instance {
    const float *a, *b; /* device operands, layouts as in gatlas_matmul_desc */
    float *c;
    int64_t m, n, k;
    int64_t lda, ldb, ldc; /* 0 = dense */
    int32_t trans_a, trans_b;
    int32_t gemm;   /* 1: C = alpha*op(A)op(B) + beta*C; 0: C = op(A)op(B) */
    int32_t tile_n; /* output tile width 64, 128 or 256; 0 = the tuned width of the instance's bucket */
    double alpha, beta;
} gatlas_grouped_instance;

typedef struct gatlas_grouped_plan gatlas_grouped_plan;

/* Packed workspace bytes for the instances (0 on invalid input). */
size_t gatlas_grouped_workspace_size(int engine, const gatlas_grouped_instance *inst, int32_t count);
/* workspace == NULL: the plan allocates and owns it; otherwise 1024-byte
 * aligned and at least gatlas_grouped_workspace_size bytes. */
int gatlas_grouped_create(int engine, const gatlas_grouped_instance *inst, int32_t count, void *workspace,
                          size_t workspace_bytes, gatlas_grouped_plan **plan);
int gatlas_grouped_prepare(gatlas_grouped_plan *plan, void *stream);
int gatlas_grouped_run(gatlas_grouped_plan *plan, void *stream);
int gatlas_grouped_launch_graph(gatlas_grouped_plan *plan, int32_t with_prepare, void *stream);
int gatlas_grouped_run_each(gatlas_grouped_plan *plan, void *stream);
int gatlas_grouped_info(const gatlas_grouped_plan *plan, int64_t *tiles, int32_t *ctas, double *flops,
                        int64_t *pack_items);
void gatlas_grouped_destroy(gatlas_grouped_plan *plan);

/* Size buckets for the tuned tile width: by n, [0,64], (64,128], (128,256],
 * (256, inf).  The table (one width per bucket and engine) starts at
 * {64, 128, 256, 256}; the autotuner (gatlas_grouped_autotune) rewrites it. */
int32_t gatlas_grouped_bucket(int64_t m, int64_t n, int64_t k);
int gatlas_grouped_set_tile_table(int engine, const int32_t *bucket_tile_n, int32_t nbuckets);
int gatlas_grouped_get_tile_table(int engine, int32_t *bucket_tile_n, int32_t nbuckets);

/* Autotunes the tile width of every bucket.  One seeded synthetic group
 * holds 48 instances per bucket (m, k log-uniform in [16,4096], n
 * log-uniform in the bucket, multiples of 16, random layouts).  Bucket by
 * bucket, the whole group is timed over `trials` runs with that bucket at
 * each width 64/128/256 and the others at their current widths, and the
 * fastest width stays (a width pays off or not beside the other buckets'
 * work).  The final table is installed (and copied to out_table when not
 * NULL).  Every timing is recorded in the journal at journal_path (NULL or
 * "": none) with the reference's run states (GatlasBenchmark.cpp:185-288)
 * under the key "grouped<engine>_<bucket>_<width>_192_<seed>_<t0>_<t1>_<t2>_
 * <t3>_" (t = the table timed); recorded times are replayed, crashed ones
 * skipped. */
int gatlas_grouped_autotune(int engine, const char *journal_path, int32_t trials, uint64_t seed,
                            int32_t *out_table);

/* ---- serving ---------------------------------------------------------------
 * A request loop over mixed GEMM / GEMV / SAXPY solves (no reference
 * counterpart: the reference times one kernel at a time).  A trace of
 * requests with arrival times is replayed in real time.  Continuous mode:
 * FIFO admission into a device arena of budget_bytes (a request that does
 * not fit waits, and later arrivals do not overtake it), operands generated
 * from each request's seed on a prep stream, every admitted GEMM batched
 * into one grouped tensor-core launch whenever fewer than two GEMM batches
 * are on the device (at most max_batch GEMMs, or about batch_target_ms of
 * estimated work), GEMVs and SAXPYs launched as admitted on a second
 * stream.  Serial mode: one request at a time, one engine call each,
 * synchronised.  Results of the same request are bit-identical in both modes
 * and alone or in any mix. */
enum { GATLAS_REQ_GEMM = 0, GATLAS_REQ_GEMV = 1, GATLAS_REQ_SAXPY = 2 };
enum { GATLAS_SERVE_CONTINUOUS = 0, GATLAS_SERVE_SERIAL = 1 };

typedef struct gatlas_request {
    int32_t kind;             /* GATLAS_REQ_* */
    int32_t trans_a, trans_b; /* GEMM layouts; GEMV: trans_a = column-major A */
    int32_t retain;           /* keep the result (and the request's memory) until gatlas_server_release */
    int64_t m, n, k;          /* GEMM m x n x k; GEMV A m x n (y = alpha*A*x + beta*y); SAXPY length n */
    double alpha, beta;       /* GEMM C = alpha*op(A)op(B) + beta*C; SAXPY y = alpha*x + y */
    uint64_t seed;            /* operands: uniform[-1,1) streams 4*seed, 4*seed+1, 4*seed+2 (initial result) */
    int64_t arrival_ns;       /* from the start of the run, non-decreasing */
} gatlas_request;

typedef struct gatlas_request_result {
    int64_t admit_ns, start_ns, done_ns; /* from the start of the run; done on the device timeline */
    int32_t status;                      /* GATLAS_OK or the request's error */
    int32_t batch;                       /* GEMM batch index, -1 for single launches */
    float *result;                       /* retained device result (C, y), else NULL */
    int64_t result_elems;
} gatlas_request_result;

typedef struct gatlas_server_config {
    size_t budget_bytes;         /* device-memory admission budget (one arena) */
    int32_t gemm_engine;         /* GATLAS_ENGINE_TC_SPLIT3 or GATLAS_ENGINE_TC_BF16 */
    int32_t max_batch;           /* most GEMMs per grouped launch (0: 256) */
    double batch_target_ms;      /* estimated device time per GEMM batch (0: 20 ms) */
    double gemm_tflops_estimate; /* rate behind that estimate, FP32-equivalent TFLOP/s (0: 300) */
} gatlas_server_config;

typedef struct gatlas_server_stats_t {
    size_t budget_bytes, peak_bytes, used_bytes;
    int64_t gemm_batches, batched_gemms;
    int64_t host_busy_ns; /* host time spent in loop iterations that did work */
    int64_t iterations;   /* loop iterations */
    /* host ns per phase: harvest, admission (incl. operand generation),
     * single launches, GEMM batch tables, GEMM batch launches */
    int64_t phase_ns[5];
    /* host ns spent inside the operand-generation launches of admission, and
     * their count: a launch blocks while the device's launch queue is full,
     * so generation time far above a few microseconds per launch is the
     * device pushing back, not host work */
    int64_t generate_ns, generate_launches;
} gatlas_server_stats_t;

typedef struct gatlas_server gatlas_server;

int gatlas_server_create(const gatlas_server_config *cfg, gatlas_server **srv);
/* Blocks until every request is done; results[i] belongs to reqs[i]. */
int gatlas_server_run(gatlas_server *srv, const gatlas_request *reqs, int32_t count, int32_t mode,
                      gatlas_request_result *results);
int gatlas_server_release(gatlas_server *srv, float *result);
/* Copies elems floats of a retained result to host memory (synchronous). */
int gatlas_server_read(gatlas_server *srv, const float *result, float *host_dst, int64_t elems);
int gatlas_server_stats(const gatlas_server *srv, gatlas_server_stats_t *out);
void gatlas_server_destroy(gatlas_server *srv);

/* ---- data generation and residuals ---------------------------------------
 * Seeded device-side generators (splitmix64 counter streams shared with the
 * host oracle): uniform [-1,1), sign·2^e (e in [-8,8]) or a constant. */
int gatlas_fill_f32(float *out, size_t n, int dist, uint64_t seed, uint64_t offset, float value,
                    void *stream);
int gatlas_fill_f64(double *out, size_t n, int dist, uint64_t seed, uint64_t offset, double value,
                    void *stream);

/* FP64 residual of a float result against an FP64 reference product computed
 * on the GPU (the paranoid check, OCLAppUtil.hpp:212-264, moved to the device):
 * out[0] = ||C - Cref||_F, out[1] = ||Cref||_F, out[2] = max |C - Cref|,
 * out[3] = sum |C - Cref| (the reference's absdiff), with Cref = op(A)·op(B)
 * accumulated in double.  Only the dense, batch == 1 layout is accepted. */
int gatlas_matmul_residual_f32(const gatlas_matmul_desc *d, const float *A, const float *B,
                               const float *C, double *out_host, void *stream);

/* The paranoid check's device reference (the reference's host check loops,
 * KernelMatmulBuffer.hpp:108-147, KernelMatvecBuffer.hpp:106-142 and
 * KernelSaxpyBuffer.hpp:106-121, moved to the GPU, one thread per output
 * element, accumulating k = 0..K-1 in order).  scalar: 0 float, 1 double.
 * fused == 0: every product and sum rounded separately, the arithmetic of the
 * reference's g++ -O2 x86-64 host loops (alpha*acc + beta*c reads c even
 * when beta == 0); fused != 0: the generated kernels' mad chain
 * (KernelMatmulBuffer.hpp:302-337, KernelSaxpyBuffer.hpp:186-190), which the
 * SIMT and image engines reproduce bit for bit.  Dense packed layouts only
 * (leading dimensions and strides 0 or dense); engine and tiling fields of
 * the descriptors are ignored. */
int gatlas_reference_matmul(int scalar, int fused, const gatlas_matmul_desc *d, const void *A, const void *B,
                            const void *Cin, void *C, void *stream);
int gatlas_reference_matvec(int scalar, int fused, const gatlas_matvec_desc *d, const void *A, const void *x,
                            const void *yin, void *y, void *stream);
int gatlas_reference_saxpy(int scalar, int fused, size_t n, double alpha, const void *x, const void *y, void *z,
                           void *stream);

/* ---- plugin surface: KernelInterface objects -------------------------------
 * One object per kernel family and -T type, with the reference's parameter
 * vector, validity rules, names, flop counts and work-item shapes
 * (KernelInterface, GatlasBenchmark.hpp:28-58; KernelBase{Matmul,Matvec,
 * Saxpy}).  op is "matmul", "matvec" or "saxpy"; type is a -T name of the
 * reference's tools (float1|float2|float4|double1|double2|double4|floatimg|
 * doubleimg), or tcbf16|split3|split6|fp8 for the tensor-core matmul engines.
 * String and vector getters return the full length and copy at most
 * len - 1 characters / cap elements. */
typedef struct gatlas_kernel gatlas_kernel;
int gatlas_kernel_create(const char *op, const char *type, gatlas_kernel **out);
void gatlas_kernel_destroy(gatlas_kernel *k);
size_t gatlas_kernel_name(const gatlas_kernel *k, char *buf, size_t len);          /* kernelName */
int gatlas_kernel_set_params(gatlas_kernel *k, const size_t *params, size_t n);    /* setParams */
/* getParams: returns 1 and the vector when the point is valid (validParams), else 0 */
int gatlas_kernel_get_params(const gatlas_kernel *k, size_t *params, size_t cap, size_t *n);
size_t gatlas_kernel_number_flops(const gatlas_kernel *k);                          /* numberFlops */
size_t gatlas_kernel_total_variations(const gatlas_kernel *k);
size_t gatlas_kernel_extra_param_detail(const gatlas_kernel *k, size_t *out, size_t cap);
size_t gatlas_kernel_global_work_items(const gatlas_kernel *k, size_t *out, size_t cap);
size_t gatlas_kernel_local_work_items(const gatlas_kernel *k, size_t *out, size_t cap);
size_t gatlas_kernel_print(const gatlas_kernel *k, char *buf, size_t len);         /* print */
void gatlas_kernel_paranoid_check(gatlas_kernel *k);                                /* paranoidCheck */
/* Arithmetic of the paranoid check's reference: fused != 0 (the default) the
 * generated kernels' mad chain, fused == 0 the reference's separately rounded
 * host loops (see gatlas_reference_matmul).  The pass rule is the
 * reference's either way: absdiff < 1/length (OCLAppUtil.hpp:212-264). */
void gatlas_kernel_paranoid_fused(gatlas_kernel *k, int fused);
/* absdiff (or, for the tensor-core engines and GEMV, the normwise error) of
 * the last paranoid check. */
double gatlas_kernel_last_check(const gatlas_kernel *k);
/* Bench::run (GatlasBenchmark.cpp:178-289): set params, journal the build and
 * run states when `journal` is a path, set args, time `trials` launches (with
 * the host<->device copies when bus_to_device / bus_from_device), check the
 * output.  *usec = elapsed microseconds, 0 when the point failed. */
int gatlas_bench_run(gatlas_kernel *k, const char *journal, size_t trials, const size_t *params, size_t n,
                     int bus_to_device, int bus_from_device, size_t *usec);

/* ---- devices --------------------------------------------------------------
 * Device selection for callers that do not link the CUDA runtime themselves
 * (the library carries its own).  Replaces the reference's device choice by
 * -d cpu|gpu|accN (GatlasAppUtil.cpp:30-60). */
int gatlas_device_count(int *count);
int gatlas_set_device(int device);

/* ---- device faults ------------------------------------------------------
 * Kernels that wait on asynchronous copies (mbarrier waits) give up after a
 * bounded number of polls, set a bit in the current device's fault word and
 * return instead of hanging.  Reads the word after synchronising the device;
 * clears it when `clear` is non-zero.  No reference counterpart (the
 * reference detects hangs only through its journal, GatlasBenchmark.cpp:178-289). */
int gatlas_device_faults(int *flags, int clear);

/* Exercises that mechanism without a fault: one thread waits on an mbarrier
 * with the library's bounded poll, limited to limit_ns (at most 2 s).  With
 * arrive != 0 the phase completes first and *completed = 1; with arrive == 0
 * nothing completes it, the wait runs out, the fault word gets bit 6 (1 << 6)
 * and *completed = 0, and the device stays usable.  Synchronises `stream`.
 * No reference counterpart. */
int gatlas_selftest_bounded_wait(int64_t limit_ns, int arrive, int *completed, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* GATLAS_B200_H */
