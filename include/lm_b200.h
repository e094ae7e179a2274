/*
 * lm_b200.h — C ABI of the B200 (sm_100a) dense-solve library.
 *
 * This is the drop-in boundary for linear-massiv's dense solve path.  Every
 * entry point is `extern "C"`, takes plain pointers and sizes, and returns an
 * int status:
 *     0            success
 *     > 0          LAPACK-style info: k + 1 where k is the first zero pivot
 *                  (LU) or first non-positive diagonal (Cholesky).  The
 *                  outputs are still written, with the Inf/NaN the reference's
 *                  own arithmetic produces in that case.
 *     < 0          LM_ERR_* below (argument, CUDA or device-wait error).
 * Errors never cross the ABI as exceptions.
 *
 * Layout convention (the reference's massiv `Array P Ix2 Double`): row-major,
 * element (i, j) at ptr[i * ld + j], ld >= number of columns.
 *
 * Device-pointer entry points (lm_d*) leave matrices resident in HBM and run
 * asynchronously on the context's stream unless an `info` host pointer is
 * passed (then they synchronise to report it).  Host-buffer entry points
 * (lm_*_host) are what a pure binding of the reference's functions calls:
 * they copy in, compute, copy out and synchronise.
 *
 * References in comments are to linear-massiv source files:
 *   L3.hs  src/Numeric/LinearAlgebra/Massiv/BLAS/Level3.hs
 *   L2.hs  src/Numeric/LinearAlgebra/Massiv/BLAS/Level2.hs
 *   LU.hs  src/Numeric/LinearAlgebra/Massiv/Solve/LU.hs
 *   Chol.hs src/Numeric/LinearAlgebra/Massiv/Solve/Cholesky.hs
 *   K.hs   src/Numeric/LinearAlgebra/Massiv/Internal/Kernel.hs
 */
#ifndef LM_B200_H
#define LM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LM_OK 0
#define LM_ERR_ARG (-1)           /* invalid argument (size, stride, null)      */
#define LM_ERR_CUDA (-2)          /* CUDA runtime/driver error                  */
#define LM_ERR_UNSUPPORTED (-3)   /* configuration not supported                */
#define LM_ERR_TIMEOUT (-4)       /* a bounded device-side wait gave up         */
#define LM_ERR_NOMEM (-5)         /* device or pinned allocation failed         */
#define LM_ERR_NOT_CONVERGED (-6) /* iterative refinement did not converge      */

typedef struct lm_ctx lm_ctx;

/* ---- context ------------------------------------------------------------
 * One context per device and calling thread (Haskell capability).  A context
 * owns a CUDA stream, a grow-only device workspace and a pinned staging
 * buffer.  Calls on one context are serialised by an internal lock. */
int lm_ctx_create(lm_ctx** ctx, int device);
int lm_ctx_destroy(lm_ctx* ctx);
/* Use an external cudaStream_t (passed as void*) instead of the own stream. */
int lm_ctx_set_stream(lm_ctx* ctx, void* stream);
void* lm_ctx_get_stream(lm_ctx* ctx);
int lm_ctx_synchronize(lm_ctx* ctx);
/* Device status of the last call on this context (checks the device error
 * flag, e.g. a bounded wait that timed out); synchronises. */
int lm_ctx_check(lm_ctx* ctx);
const char* lm_status_string(int status);
/* Thread-local text of the last error raised by this library. */
const char* lm_last_error(void);
/* Number of kernel launches this library has issued in this process. */
long long lm_launch_count(void);

/* ---- per-phase tracing ----------------------------------------------------
 * When enabled, every kernel of the named phases is bracketed by CUDA events
 * on the context's stream; lm_ctx_profile_read aggregates them per phase:
 * launches, device milliseconds, algorithmic FLOPs and bytes.
 * Phases: 0 GEMM (trailing updates, solve updates), 1 panel (LU leaf,
 * Cholesky diagonal block), 2 row interchanges, 3 triangular block solves,
 * 4 other (copies, residuals). */
#define LM_PHASES 5
int lm_ctx_profile(lm_ctx* ctx, int enable);
/* Synchronises; fills arrays of LM_PHASES entries (any may be NULL) and
 * clears the records. */
int lm_ctx_profile_read(lm_ctx* ctx, long long* launches, double* ms, double* flops, double* bytes);

/* ---- memory (device buffers stay resident between calls) -------------- */
int lm_dmalloc(lm_ctx* ctx, void** ptr, size_t bytes);
int lm_dfree(lm_ctx* ctx, void* ptr);
int lm_h2d(lm_ctx* ctx, void* dst_device, const void* src_host, size_t bytes);
int lm_d2h(lm_ctx* ctx, void* dst_host, const void* src_device, size_t bytes);

/* ---- BLAS-3 ---------------------------------------------------------------
 * gemm alpha A B beta C (L3.hs:102-131); with alpha = 1, beta = 0 this is
 * matMul / matMulP (L3.hs:144-147, 183-207) and matMulPPar (L3.hs:214-294),
 * whose work rawGemmKernel (K.hs:145-806) does on the CPU.
 * C (m x n) = alpha * A (m x k) * B (k x n) + beta * C, device pointers. */
int lm_dgemm(lm_ctx* ctx, int m, int n, int k, double alpha, const double* A, int lda,
             const double* B, int ldb, double beta, double* C, int ldc);

/* ---- LU with partial pivoting ---------------------------------------------
 * lm_dgetrf: in-place PA = LU of the n x n matrix A (device).  Replaces the
 * factor phase of luSolveP, panelLUFactor (LU.hs:265-357) with its kernels
 * rawPivotSearch / rawSwapRows / rawLUEliminateColumnTo (K.hs:1414-1556),
 * rawTriSolvePanelTrail (LU.hs:364-407) and the trailing GEMM; also the
 * factor of `lu` (LU.hs:121-167).  Pivot rule: largest |a_ik|, first
 * (lowest) row on ties (K.hs:1541-1556).  Rows are swapped across all n
 * columns, as the reference does.
 * ipiv (device, n ints): swap list, 0-based — step k swapped rows k and
 * ipiv[k] (the reference's [(k, pivRow)] list, LU.hs:283,326).
 * info (host, may be NULL): if given, the call synchronises and stores the
 * LAPACK-style info there; the return value carries the same. */
int lm_dgetrf(lm_ctx* ctx, int n, double* A, int lda, int* ipiv, int* info);

/* lm_dgetrs: solve A X = B with the output of lm_dgetrf, B (n x nrhs, ldb)
 * overwritten by X.  Replaces applyPivotsForward, rawForwardSubUnitPackedSIMD
 * and rawBackSubPackedSIMD (LU.hs:493-507, K.hs:2205-2314); nrhs > 1 solves
 * each column as luSolveP would. */
int lm_dgetrs(lm_ctx* ctx, int n, int nrhs, const double* LU, int lda, const int* ipiv, double* B,
              int ldb);

/* lm_dgesv: luSolveP (LU.hs:265-304) on device buffers: A is overwritten by
 * its LU factors, B by the solution. */
int lm_dgesv(lm_ctx* ctx, int n, int nrhs, double* A, int lda, int* ipiv, double* B, int ldb,
             int* info);

/* ---- Cholesky ---------------------------------------------------------------
 * lm_dpotrf: A = G G^T from the lower triangle of A (device), G written to
 * the lower triangle and the strict upper triangle zeroed, as `cholesky`
 * returns it (Chol.hs:114-147).  Replaces panelCholFactor with
 * rawCholColumnSIMD(From) (Chol.hs:279-321, K.hs:2071-2195). */
int lm_dpotrf(lm_ctx* ctx, int n, double* A, int lda, int* info);

/* lm_dpotrs: solve with G from lm_dpotrf; B (n x nrhs) overwritten by X.
 * Replaces rawForwardSubCholPackedSIMD and rawBackSubCholTPackedSIMD
 * (K.hs:2319-2430). */
int lm_dpotrs(lm_ctx* ctx, int n, int nrhs, const double* G, int lda, double* B, int ldb);

/* lm_dposv: choleskySolveP (Chol.hs:241-273) on device buffers. */
int lm_dposv(lm_ctx* ctx, int n, int nrhs, double* A, int lda, double* B, int ldb, int* info);

/* ---- host-buffer entry points (pure functions of the reference) ------------
 * Inputs are read-only host arrays (row-major, dense: lda = n, ldb = nrhs);
 * outputs are written to host arrays.  These are the calls a Haskell
 * `foreign import ccall safe` binding of luSolve / choleskySolve / matMul /
 * lu / cholesky makes. */
int lm_lu_solve_host(lm_ctx* ctx, int n, int nrhs, const double* A, const double* B, double* X,
                     int* info);
int lm_chol_solve_host(lm_ctx* ctx, int n, int nrhs, const double* A, const double* B, double* X,
                       int* info);
int lm_matmul_host(lm_ctx* ctx, int m, int n, int k, const double* A, const double* B, double* C);
int lm_gemm_host(lm_ctx* ctx, int m, int n, int k, double alpha, const double* A, const double* B,
                 double beta, const double* C0, double* C);
/* lu (LU.hs:121-122): packed LU (n x n) and the permutation vector form of
 * the pivots, perm[i] = original row of A that ends up at row i. */
int lm_lu_host(lm_ctx* ctx, int n, const double* A, double* LU, int* perm, int* info);
/* cholesky (Chol.hs:114-115): G with zeros above the diagonal. */
int lm_cholesky_host(lm_ctx* ctx, int n, const double* A, double* G, int* info);
/* det (LU.hs:534-545): product of U's diagonal times the pivot sign. */
int lm_det_host(lm_ctx* ctx, int n, const double* A, double* det);

/* Host helper: swap list -> permutation vector (the reference's `lu` form). */
int lm_ipiv_to_perm(int n, const int* ipiv, int* perm);

/* ---- mixed precision with iterative refinement -----------------------------
 * No counterpart in the reference (its solves are FP64 throughout).  A is
 * rounded to FP32 and factored with partial pivoting, every Schur-complement
 * update on the tcgen05 tensor cores in TF32 with FP32 accumulation; the
 * solution is then refined in FP64 (residual r = B - A X with the original A,
 * correction from the FP32 factors, X += d) until the normwise backward error
 * ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) of every column is <= tol
 * (tol <= 0 selects 1e-15 * n).  A and B are not modified; X (n x nrhs,
 * nrhs <= 64) receives the solution.  Returns LM_ERR_NOT_CONVERGED (with X the
 * last iterate) when max_iter corrections do not reach tol, e.g. for
 * condition numbers beyond what FP32/TF32 factors can precondition. */
int lm_dgesv_ir(lm_ctx* ctx, int n, int nrhs, const double* A, int lda, const double* B, int ldb, double* X,
                int ldx, double tol, int max_iter, int* iters, double* berr, int* info);
/* Host-buffer form of lm_dgesv_ir (dense row-major host arrays). */
int lm_lu_solve_ir_host(lm_ctx* ctx, int n, int nrhs, const double* A, const double* B, double* X, double tol,
                        int max_iter, int* iters, double* berr, int* info);

/* Factorisation used by the mixed-precision solves of a context (lm_dgesv_ir,
 * lm_lu_solve_ir_host and the serving loop's large requests).
 *   LM_IR_GEPP (default): FP32 LU with partial pivoting (the FP64 path's pivot
 *     rule), every Schur-complement update as 3xTF32 on the tensor cores, with
 *     look-ahead; the FP32 substitutions solve their diagonal blocks by
 *     substitution, so each correction is backward stable in FP32.
 *   LM_IR_RBT: A is mixed by two random depth-2 butterfly transforms,
 *     Ar = U^T A V (Baboulin, Dongarra, Herrmann, Tomov 2013), and Ar is
 *     factored in FP32 without pivoting, so that everything but the 128 x 128
 *     diagonal blocks runs on the tensor cores; corrections are V Ar^-1 U^T r.
 *     Fast on matrices whose leading blocks stay well conditioned, but without
 *     pivoting it stalls on dense ill-conditioned ones: if its refinement
 *     stalls (two steps in a row do not reduce the worst backward error, or its
 *     contraction rate cannot reach tol within max_iter) or runs out of steps,
 *     the solve is redone with LM_IR_GEPP, and only that result is reported.
 * The stopping test, tolerance and FP64 residual are the same for both. */
#define LM_IR_RBT 0
#define LM_IR_GEPP 1
/* Precision of the partial-pivoting factor's trailing updates (lm_dgesv_ir_prec):
 *   LM_IR_PREC_TF32X3  three TF32 products per element (close to FP32), refined
 *                      by classical refinement (the default of lm_dgesv_ir);
 *   LM_IR_PREC_TF32    one TF32 product (kind::tf32), refined by GMRES-IR;
 *   LM_IR_PREC_BF16    one BF16 product (kind::f16), refined by GMRES-IR.
 * GMRES-IR (Carson and Higham): each correction solves A d = r with
 * right-preconditioned flexible GMRES in FP64 (up to 30 steps, until the
 * correction's residual falls by 1e-4), the low-precision LU applied in FP32
 * as the preconditioner; the outer residual, update and stopping test are those
 * of lm_dgesv_ir.  Lower precision trades factor speed for refinement steps
 * and a smaller range of condition numbers. */
#define LM_IR_PREC_TF32X3 0
#define LM_IR_PREC_TF32 1
#define LM_IR_PREC_BF16 2
int lm_ctx_set_ir_method(lm_ctx* ctx, int method);
/* lm_dgesv_ir with the factor precision `prec` (LM_IR_PREC_*) and partial
 * pivoting whatever the context's method; iters counts the outer refinement
 * steps. */
int lm_dgesv_ir_prec(lm_ctx* ctx, int n, int nrhs, const double* A, int lda, const double* B, int ldb, double* X,
                     int ldx, int prec, double tol, int max_iter, int* iters, double* berr, int* info);
/* Method that produced the last mixed-precision result on this context
 * (LM_IR_RBT, or LM_IR_GEPP after a fallback); -1 before the first solve. */
int lm_ctx_ir_last_method(lm_ctx* ctx, int* method);
/* Convergence record of the context's last mixed-precision solve: the worst
 * normwise backward error after each refinement step, over both methods in
 * the order they ran (randomised first, then partial pivoting after a
 * fallback).  *steps receives the number of steps; up to max_steps values are
 * written to berr. */
int lm_ctx_ir_history(lm_ctx* ctx, double* berr, int max_steps, int* steps);

/* ---- factorisation without allocation -----------------------------------------
 * No counterpart in the reference.  lm_dpotrf without any allocation: for
 * callers that cannot call cudaMalloc at call time (a runtime whose memory
 * pool owns every allocation, a real-time loop that forbids allocation, a
 * plugin host that only hands out pre-registered buffers).  Same result as
 * lm_dpotrf on `stream` (cudaStream_t as void*, 0 = legacy default stream),
 * on the current device; it synchronises `stream` to report info.  Its
 * scratch is one static device array of the library, about 4.3 MB per
 * device, reserved when the first call on that device looks up its address
 * (CUDA loads device code lazily by default) and held until exit: make that
 * first call (n = 0 does only this) before any region that must not
 * allocate and before any stream capture.  The array limits n to 4096
 * (larger n returns LM_ERR_ARG) and A must be 16-byte aligned with an even
 * lda.  All calls share the array: calls that overlap on the GPU race and
 * must be serialised by the caller. */
int lm_dpotrf_noalloc(void* stream, int n, double* A, int lda, int* info);

/* ---- batched uneven-size solves in one persistent launch -----------------------
 * No counterpart in the reference (its solves take one system at a time).
 * A plan fixes the sizes of `count` independent systems A_i X_i = B_i:
 * n_i in [0, 256], nrhs_i in [0, 16], kind_i LM_BATCH_GENERAL (LU with partial
 * pivoting, luSolveP, LU.hs:265-357) or LM_BATCH_SPD (Cholesky,
 * choleskySolveP, Chol.hs:241-321).  Inputs are packed back to back in the
 * caller's order: A_i at A + a_off[i] (n_i x n_i row-major), B_i and X_i at
 * + b_off[i] (n_i x nrhs_i row-major); lm_batch_offsets returns the offsets
 * (count + 1 entries each, host arrays).  lm_batch_solve runs the whole batch
 * as one persistent kernel (captured in a CUDA graph after its first call):
 * A and B are read-only device buffers, X (device) receives the solutions.
 * precision LM_PREC_FP64: factor and solve in FP64.  LM_PREC_FP32_IR: factor
 * in FP32 and refine in FP64 until each instance's normwise backward error is
 * <= tol (tol <= 0 selects 1e-15 * n_i per instance); an instance not
 * converged after max_iter corrections is redone in FP64.
 * lm_batch_results copies per-instance info (LAPACK-style, 0 = ok), the
 * number of corrections (-1 = FP64 fallback, 0 for LM_PREC_FP64) and the
 * final backward error (IR only) to host arrays (any may be NULL); it
 * synchronises.  Panel widths per size bucket come from the context's tuning
 * table (lm_batch_tune). */
#define LM_BATCH_GENERAL 0
#define LM_BATCH_SPD 1
#define LM_PREC_FP64 0
#define LM_PREC_FP32_IR 1
typedef struct lm_batch lm_batch;
int lm_batch_create(lm_ctx* ctx, lm_batch** plan, int count, const int* n, const int* nrhs, const int* kind,
                    int precision);
int lm_batch_destroy(lm_batch* plan);
int lm_batch_offsets(const lm_batch* plan, long long* a_off, long long* b_off);
int lm_batch_solve(lm_batch* plan, const double* A, const double* B, double* X, double tol, int max_iter);
int lm_batch_results(lm_batch* plan, int* info, int* iters, double* berr);
/* Device pointers of the plan's factor workspace (instance i's LU or G at
 * F + a_off[i], FP64 plans) and swap lists (instance i's at ipiv + p_off[i],
 * p_off[i] = sum of n_j, j < i); valid until the next solve or destroy. */
int lm_batch_factors(const lm_batch* plan, const double** F, const int** ipiv);
/* Host-buffer form: copies the packed A and B in, solves, copies X out. */
int lm_batch_solve_host(lm_batch* plan, const double* A, const double* B, double* X, double tol, int max_iter);
/* Project-written autotuner: for each size bucket (n <= 32, 64, 128, 256)
 * times the batch kernel on a seeded synthetic batch of that bucket with each
 * candidate panel width (8, 16, 32) and keeps the fastest in the context's
 * table; `path` (may be NULL) receives the table as JSON.  lm_batch_tune_get /
 * lm_batch_tune_set read and write the table (nb[precision][bucket]). */
int lm_batch_tune(lm_ctx* ctx, int precision, const char* path);
int lm_batch_tune_get(lm_ctx* ctx, int* nb /* [2][4] */);
int lm_batch_tune_set(lm_ctx* ctx, const int* nb /* [2][4] */);

/* ---- serving loop: continuous batching of arriving solves -----------------------
 * No counterpart in the reference.  A server owns a device arena of
 * `hbm_budget` bytes (0 = a quarter of the free memory after start-up) from
 * which every admitted request takes one block (its A, B, X, factor and
 * pivots).  Requests are admitted as soon as an execution slot and a block are
 * free; small ones (n <= small_max_n, nrhs <= 16) run on the device-resident
 * request loop (device_loop, below) or as micro-batches of the persistent
 * batch kernel (batch_lanes streams, each micro-batch taking every small
 * request queued when its lane frees up), larger ones each take
 * one of `large_workers` contexts (own stream; workspaces pre-grown at start-up
 * for max_n x max_nrhs).  Every large request is solved at a padded order (n
 * rounded up to a multiple of 64, 128 or 256, the system embedded with a
 * diagonal block max_i |a_ii| I and zero right-hand-side rows), so that
 * requests of nearby orders replay the same captured CUDA graphs: by FP64 LU
 * (general, n <= lu_fp64_max_n) or FP64 Cholesky (SPD, n <= chol_fp64_max_n),
 * and above those orders, with large_precision LM_PREC_FP32_IR, by the
 * mixed-precision solve of lm_dgesv_ir (FP32 factor + FP64 refinement, for
 * general and SPD matrices alike, method ir_method, stopping test of the
 * original order), then FP64 LU or Cholesky at the original order when
 * refinement does not converge; with LM_PREC_FP64 always FP64.  A, B (read)
 * and X (written) are the
 * caller's host buffers (pinned for asynchronous copies) and must stay valid
 * until the request completes.  Status of a completed request: 0, LAPACK-style
 * info > 0, or < 0 on error / cancellation. */
typedef struct {
  size_t hbm_budget;    /* bytes of the request arena (0 = 1/4 of free memory) */
  int large_workers;    /* concurrent large solves (default 8) */
  int batch_lanes;      /* concurrent micro-batches (default 2) */
  int small_max_n;      /* largest n sent to the batch kernel (default 256, <= 256) */
  int small_precision;  /* LM_PREC_FP64 (default) or LM_PREC_FP32_IR */
  int large_precision;  /* LM_PREC_FP32_IR (default) or LM_PREC_FP64 */
  int max_batch;        /* most requests per micro-batch (default 4096) */
  int max_n;            /* largest admissible order (default 4096) */
  int max_nrhs;         /* most right-hand sides (default 64, <= 64) */
  int nb[4];            /* batch-kernel panel width per size bucket (default 16) */
  int ir_method;        /* factorisation of the large mixed-precision solves: LM_IR_GEPP
                           (default: FP32 partial pivoting, the same result for a request
                           alone and in any mix) or LM_IR_RBT (the randomised factor
                           without pivoting, redone with partial pivoting whenever its
                           refinement stalls) */
  int device_loop;      /* 1 (default): small requests run on the device-resident loop, a
                           persistent kernel of loop_ctas CTAs that claims each posted
                           request from a ring in device memory as soon as its data has
                           arrived, and returns after a few ms without work (relaunched
                           when work arrives); 0: micro-batches of the batch kernel on the
                           batch lanes.  The loop solves in FP64 (small_precision
                           LM_PREC_FP64). */
  int loop_ctas;        /* CTAs of the device-resident loop (default 16, which leaves every GPC
                           room for the large solves' thread-block clusters) */
  int lu_fp64_max_n;    /* general requests above small_max_n and up to this order are solved
                           by FP64 LU at the bucket order instead of the mixed-precision solve
                           (default 2048: below it both factorisations are bound by the same
                           column chain, and FP64 needs no refinement) */
  int chol_fp64_max_n;  /* SPD requests up to this order by FP64 Cholesky at the bucket order
                           (default 4096) */
} lm_server_config;
typedef struct {
  long long completed, rejected, cancelled, failed, fp64_fallbacks;
  long long queue_peak, pending, micro_batches, small_solved;
  int inflight, inflight_peak;
  size_t arena_bytes, arena_peak_bytes, fixed_bytes;
  double p50_ms, p99_ms, mean_ms, max_ms; /* submit -> X in the host buffer */
  double span_s, solves_per_s, tflops;    /* first submission to last completion */
  /* large requests solved by lm_dgesv_ir, how many of those needed its partial-
   * pivoting fallback (LM_IR_GEPP), and their refinement steps in all */
  long long ir_solves, ir_gepp, ir_iterations;
} lm_server_stats_t;
int lm_server_default_config(lm_server_config* cfg);
typedef struct lm_server lm_server;
int lm_server_create(lm_server** server, int device, const lm_server_config* cfg);
/* Queue one request; *id identifies it.  LM_ERR_ARG for sizes outside the
 * configuration, LM_ERR_NOMEM for a request larger than the whole arena. */
int lm_server_submit(lm_server* server, int n, int nrhs, int kind, const double* A, const double* B, double* X,
                     long long* id);
/* Non-blocking: *done = 1 once X is written (the id is then released). */
int lm_server_test(lm_server* server, long long id, int* done, int* status, double* latency_ms);
/* Blocking (timeout_s <= 0: no limit; LM_ERR_TIMEOUT when it expires). */
int lm_server_wait(lm_server* server, long long id, int* status, double* latency_ms, double timeout_s);
/* Remove a request that is still queued (LM_ERR_UNSUPPORTED once admitted). */
int lm_server_cancel(lm_server* server, long long id);
int lm_server_drain(lm_server* server, double timeout_s);
int lm_server_stats(lm_server* server, lm_server_stats_t* stats);
int lm_server_reset_stats(lm_server* server);
/* Finishes admitted requests, cancels queued ones, frees everything. */
int lm_server_destroy(lm_server* server);

/* ---- matvec and norms ----------------------------------------------------------
 * lm_dgemv: y (m) = A (m x n, lda) x (n), device pointers, asynchronous on the
 * context's stream.  Replaces matvec / matvecP (L2.hs:123-139, rewritten to
 * matvecP by the RULE "matvec/P/Double") and rawGemv / rawDot
 * (K.hs:84-134), in their floating-point order: every y_i is bitwise the
 * reference's (four FMA accumulators over j = 4s + l, combined as
 * ((a0 + a1) + a2) + a3, the last n mod 4 columns added with separately
 * rounded products). */
int lm_dgemv(lm_ctx* ctx, int m, int n, const double* A, int lda, const double* x, double* y);
/* Host-buffer form of lm_dgemv (matvec on host arrays, A dense row-major). */
int lm_matvec_host(lm_ctx* ctx, int m, int n, const double* A, const double* x, double* y);
/* lm_dnorm_inf: normInf (Norms.hs:135-141), the largest row sum of |a_ij|,
 * each row a left fold from 0 in column order (bitwise the reference's); A on
 * the device, *result on the host (synchronises).  vnormInf (Norms.hs:94-96)
 * of a vector x is lm_dnorm_inf of x as an n x 1 matrix.  0 for an empty A. */
int lm_dnorm_inf(lm_ctx* ctx, int m, int n, const double* A, int lda, double* result);
int lm_norm_inf_host(lm_ctx* ctx, int m, int n, const double* A, double* result);

/* ---- adjacent solvers -------------------------------------------------------------
 * lm_dgetrf_nopiv: luNoPivot (LU.hs:196-214), LU without row interchanges of
 * the n x n device matrix A in place (unit L below the diagonal, U on and
 * above), blocked: 128 x 128 diagonal blocks factored without interchanges,
 * the panels and the trailing update on the DMMA GEMM.  As in the reference
 * the caller must supply a matrix that needs no pivoting (e.g. diagonally
 * dominant); a zero pivot is reported as info = k + 1 and, like the
 * reference's division by it, leaves Inf/NaN in the result. */
int lm_dgetrf_nopiv(lm_ctx* ctx, int n, double* A, int lda, int* info);
/* Host-buffer form: LU (n x n) receives the packed factor. */
int lm_lu_nopivot_host(lm_ctx* ctx, int n, const double* A, double* LU, int* info);
/* choleskyGaxpy (Chol.hs:173-204): the same G as cholesky (lower, zeros
 * above), from the device Cholesky factorisation; host buffers. */
int lm_cholesky_gaxpy_host(lm_ctx* ctx, int n, const double* A, double* G, int* info);
/* lm_dtridiag_solve: tridiagSolve (Solve/Banded.hs:292-342), x = A^-1 b for
 * the symmetric positive definite tridiagonal A with diagonal diag (n) and
 * superdiagonal supdiag (entries 0 .. n-2 are read), device pointers, by
 * parallel cyclic reduction: ceil(log2 n) fully parallel elimination steps
 * instead of the reference's sequential LDL^T sweep (the same solution to
 * within rounding). */
int lm_dtridiag_solve(lm_ctx* ctx, int n, const double* diag, const double* supdiag, const double* b, double* x);
int lm_tridiag_solve_host(lm_ctx* ctx, int n, const double* diag, const double* supdiag, const double* b,
                          double* x);

/* ---- residual (IR and the reference's scaled residual) ---------------------
 * R = B - A X in FP64 (device), n x nrhs; replaces matvec / rawGemv
 * (L2.hs:123-144, K.hs:119-134) on the refinement path. */
int lm_dresidual(lm_ctx* ctx, int n, int nrhs, const double* A, int lda, const double* X, int ldx,
                 const double* B, int ldb, double* R, int ldr);

#ifdef __cplusplus
}
#endif

#endif /* LM_B200_H */
