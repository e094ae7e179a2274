// Internal (non-ABI) interfaces shared by the library's translation units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <functional>
#include <vector>

#include "lm_b200.h"

namespace lm {

constexpr int kMaxDevices = 64;

struct Ctx;

// --- context accessors (api.cu) ---------------------------------------------
void count_launch(int n);  // process-wide kernel launch counter
int* ctx_status(Ctx& c);        // device int[4]: error code, info, ticket, spare
int ctx_num_sms(Ctx& c);
int ctx_device(Ctx& c);
// Grow-only device workspace owned by the context (slot 0..kWsSlots-1).
constexpr int kWsSlots = 4;
int ctx_workspace(Ctx& c, int slot, size_t bytes, void** ptr);
// The context's look-ahead stream (highest priority, created on first use,
// which must not be inside a stream capture) and its fork / join events.
int ctx_aux(Ctx& c, cudaStream_t* aux, cudaEvent_t* fork, cudaEvent_t* join);
// Whether the factorisations may fork onto the look-ahead stream (false for
// the borrowed contexts of the entry points without allocation).
bool ctx_lookahead(Ctx& c);
// Worst backward error after each refinement step of the context's last
// mixed-precision solve (both methods, in order).
std::vector<double>& ctx_ir_history(Ctx& c);
// Grow-only pinned host buffer owned by the context (not inside a capture).
int ctx_pinned(Ctx& c, size_t bytes, void** ptr);

// Per-phase CUDA-event tracing (enabled by lm_ctx_profile).  A Prof scope
// brackets the kernels launched inside it with events on stream `st`.
enum Phase { kPhaseGemm = 0, kPhasePanel = 1, kPhaseSwap = 2, kPhaseTrsm = 3, kPhaseOther = 4, kNumPhases = 5 };
struct Prof {
  Prof(Ctx& c, int phase, double flops, double bytes, cudaStream_t st);
  ~Prof();
  Ctx& c;
  int phase;
  double flops, bytes;
  cudaStream_t st;
  cudaEvent_t a = nullptr;
};

// TMA descriptor for a row-major 2D view: `inner` elements per row (contiguous),
// `outer` rows, row stride `ld` elements; box of box_inner x box_outer.
int make_tmap_2d(CUtensorMap* tm, CUtensorMapDataType dt, int elem_bytes, const void* base,
                 long long inner, long long outer, long long ld, int box_inner, int box_outer,
                 CUtensorMapSwizzle swz);

// --- few-rhs persistent substitutions (trsv.cu) ------------------------------
// Elements of one factor's diagonal-block inverses for order n.
template <typename T>
size_t trsv_inv_elems(int n);
// DinvL / DinvU <- inverses of the diagonal blocks of the packed LU factor's
// unit-lower L and upper U (16-byte aligned, trsv_inv_elems<T>(n) each).
template <typename T>
int tri_inv_blocks(const T* LU, long long lda, int n, T* DinvL, T* DinvU, cudaStream_t st);
// X (n x nrhs) <- U^-1 L^-1 X, two persistent launches per pass (FP64:
// nrhs <= 4; FP32: any nrhs, in passes of 16 beyond 4); `sync` is 4 ints of
// device scratch.  FP64, and FP32 with `exact`, solve the diagonal blocks by
// substitution; FP32 otherwise multiplies by the block inverses, and corr
// (two flags per 128-row block: L, U), when given, limits the diagonal-block
// correction step to flagged blocks.
// unit_lower = false reads L's stored diagonal (a Cholesky factor G packed
// with G^T above the diagonal).
template <typename T>
int trsv_lu(const T* LU, long long lda, int n, int nrhs, const T* DinvL, const T* DinvU, T* X, long long ldx,
            int* sync, int* status, cudaStream_t st, const int* corr = nullptr, bool exact = false,
            bool unit_lower = true);

// --- FP64 GEMM (dgemm.cu) ----------------------------------------------------
// C = alpha * op(A) * op(B) + beta * C, row-major.
//   a_trans = false: A is m x k (lda)  | true: A^T is stored, k x m (lda)
//   b_trans = false: B is k x n (ldb)  | true: B^T is stored, n x k (ldb)
// lower_only: only C(i,j) with j <= i is read or written (requires m == n).
// max_sms: SMs the persistent grid may occupy (0 = all of them).
struct GemmDesc {
  int m = 0, n = 0, k = 0;
  double alpha = 1.0, beta = 0.0;
  const double* A = nullptr;
  long long lda = 0;
  const double* B = nullptr;
  long long ldb = 0;
  double* C = nullptr;
  long long ldc = 0;
  bool a_trans = false, b_trans = false, lower_only = false;
  int max_sms = 0;
};
int dgemm(Ctx& c, const GemmDesc& d, cudaStream_t st);

// --- shared kernels (blas_aux.cu) --------------------------------------------
// Apply row interchanges ipiv[k0..k1) in order (row s <-> row ipiv[s]) to the
// columns [ca0, ca1) and [cb0, cb1) of A (nrows rows).  A pivot row outside
// [0, nrows) is skipped and recorded as LM_DEVERR_BOUNDS in status[0].
// `plan` (kSwapPlanInts ints of device scratch, or null) lets wide updates
// compose the interchanges once instead of in every column block.
constexpr int kSwapPlanInts = 1 + 2 * 256 + 15;
template <typename T>
int laswp(T* A, long long lda, int nrows, const int* ipiv, int k0, int k1, int ca0, int ca1, int cb0, int cb1,
          int* status, cudaStream_t st, int* plan = nullptr);

// All interchanges ipiv[0..n) on a narrow n x nrhs block B at once (one
// parallel gather into W, n x nrhs scratch, then copied back).
template <typename T>
int laswp_narrow(T* B, long long ldb, int n, int nrhs, const int* ipiv, T* W, int* status, cudaStream_t st);
// The composed row permutation of a swap list, once per factorisation
// (perm[i] = sigma(i), the row laswp_narrow would bring to row i), and the
// gather that applies it to a narrow block (W: n x nrhs scratch).
int perm_from_swaps(const int* ipiv, int n, int* perm, int* status, cudaStream_t st);
template <typename T>
int laswp_perm(T* B, long long ldb, int n, int nrhs, const int* perm, T* W, cudaStream_t st);

// In-place triangular solve with a w x w block (w <= 128) of Tri (ldt) on the
// w x ncols block B (ldb):  op(Tri) X = B.
//   lower/unit describe Tri as stored; trans solves with Tri^T.
template <typename T>
int trsm_left(const T* Tri, long long ldt, int w, bool lower, bool unit, bool trans, T* B,
              long long ldb, int ncols, cudaStream_t st);

// Inverse of a lower-triangular block of order w <= 128 (diag.cu): Xout
// (w x w, ldx) <- inv(L) with zeros above the diagonal; `unit` ignores the
// stored diagonal.  For float with `lo` given, Xout receives the TF32 high
// part and lo the remainder (the 3xTF32 operand split).  One CTA.
template <typename T>
int tri_inv_lower(const T* L, long long ldl, int w, bool unit, T* Xout, long long ldx, T* lo, cudaStream_t st);

// B (w x ncols, ldb) <- inv(lower triangle of L) B in one launch, for
// w <= 64 and ncols <= 128 (the block solves inside a panel; diag.cu).
template <typename T>
int trsm_lower_small(const T* L, long long ldl, int w, bool unit, T* B, long long ldb, int ncols, cudaStream_t st);

// LU without pivoting of the w x w (w <= 128) FP32 block A11 in place, with
// split(inv(L11)) into Lhi/Llo and split(inv(U11)^T) into UThi/UTlo (w x w,
// ld ldi), inv(L11) / inv(U11) as 128 x 128 identity-padded blocks into
// DinvL / DinvU, and split(L11) (unit diagonal) / split(U11^T) into
// LFhi/LFlo / UFThi/UFTlo (w x w, ld ldi); the first zero or NaN pivot is
// recorded as base + k + 1 in status[1] (diag.cu).  The inverses are formed
// in FP64; refine[0] / refine[1] are set to 1 when L11 / U11 is
// ill-conditioned enough for the products with its inverse to need a
// correction step.
int nopiv_diag(float* A11, long long lda, int w, int base, float* Lhi, float* Llo, float* UThi, float* UTlo,
               long long ldi, float* DinvL, float* DinvU, float* LFhi, float* LFlo, float* UFThi, float* UFTlo,
               int* refine, int* status, cudaStream_t st);

// 2D copy (rows x cols) between strided buffers on the device.
template <typename T>
int copy2d(T* dst, long long ldd, const T* src, long long lds, int rows, int cols, cudaStream_t st);

// Set a rows x cols block to the identity (1 on the diagonal, 0 elsewhere).
template <typename T>
int set_identity(T* A, long long lda, int rows, int cols, cudaStream_t st);

// Zero the strict upper triangle of an n x n matrix.
template <typename T>
int zero_upper(T* A, long long lda, int n, cudaStream_t st);

// --- adjacent entry points (aux_solvers.cu) -----------------------------------
// y = A x in rawGemv's floating-point order (bitwise the reference's matvecP).
int dgemv_exact(int m, int n, const double* A, long long lda, const double* x, double* y, cudaStream_t st);
// normInf of A (bitwise the reference's row folds) as the bits of a
// non-negative double in *out (device).
int dnorm_inf_exact(int m, int n, const double* A, long long lda, unsigned long long* out, cudaStream_t st);
// LU without interchanges of one w x w block (w <= 128) in place; the first
// zero pivot goes to status[1] as base + k + 1.
int lu_nopiv_block(double* A, long long lda, int w, int base, int* status, cudaStream_t st);
// P (n x n) = G on and below the diagonal, G^T above it.
int pack_lower_sym(double* P, long long ldp, const double* G, long long ldg, int n, cudaStream_t st);
// dst (w x w) = src^T.
int transpose_block(double* dst, long long ldd, const double* src, long long lds, int w, cudaStream_t st);
// SPD tridiagonal solve by parallel cyclic reduction; W is 8 n doubles.
int dtridiag_pcr(int n, const double* diag, const double* sup, const double* rhs, double* x, double* W,
                 cudaStream_t st);

// --- factorisations and solves ---------------------------------------------
int dgetrf(Ctx& c, int n, double* A, long long lda, int* ipiv, cudaStream_t st);
int dgetrf_nopiv(Ctx& c, int n, double* A, long long lda, cudaStream_t st);
int dgetrs(Ctx& c, int n, int nrhs, const double* LU, long long lda, const int* ipiv, double* B,
           long long ldb, cudaStream_t st);
int dpotrf(Ctx& c, int n, double* A, long long lda, cudaStream_t st);
int dpotrs(Ctx& c, int n, int nrhs, const double* G, long long lda, double* B, long long ldb,
           cudaStream_t st);

// Panel factorisation kernels (panel.cu): LU of rows [c0, n) x columns
// [c0, c0 + w) in place, w <= 32, recording ipiv[c0 .. c0 + w) (global rows)
// and the first zero pivot in status[1].  The leaf's row interchanges are
// also applied to the other columns of the enclosing panel [pc0, pc0 + pw)
// (pw <= 128); columns outside it are left to the caller.
template <typename T>
int panel_leaf(Ctx& c, T* A, long long lda, int n, int c0, int w, int pc0, int pw, int* ipiv, cudaStream_t st);
int panel_leaf_max_width_for(Ctx& c, int rows);  // widest leaf one cluster holds for `rows`

// Cholesky of a w x w diagonal block (w <= 128) in place, lower triangle;
// records the first non-positive pivot (global index base + j + 1) in status[1].
template <typename T>
int potrf_block(Ctx& c, T* A, long long lda, int w, int base, cudaStream_t st);

// Mixed precision (ir.cu): FP32 LU with TF32 tensor-core updates, FP32
// substitutions, FP64 refinement.  `factor_runner` runs the factorisation
// body (so the caller can capture it into a CUDA graph).
int sgetrf(Ctx& c, int n, float* A, long long lda, int* ipiv, cudaStream_t st, int prec = LM_IR_PREC_TF32X3);
int sgetrs(Ctx& c, int n, int nrhs, const float* LU, long long lda, const int* ipiv, float* X, long long ldx,
           cudaStream_t st);
// Runs a fixed launch sequence tagged "factor" or "iter" (the caller maps the
// tag and the solve's buffers to a CUDA-graph key, or runs it eagerly).
using IrRunner = std::function<int(const char* tag, const std::function<int(cudaStream_t)>& body)>;
// prec (LM_IR_PREC_*): the factor's trailing-update precision; TF32 and
// BF16 factors are refined by GMRES-IR, 3xTF32 by classical refinement.
int dgesv_ir(Ctx& c, int n, int nrhs, const double* A, long long lda, const double* B, long long ldb, double* X,
             long long ldx, double tol, int max_iter, int* iters_out, double* berr_out, cudaStream_t st,
             const IrRunner& run, int prec = LM_IR_PREC_TF32X3);

// Randomised variant (ir.cu, rbt.cu): depth-2 random butterflies on both
// sides, FP32 LU without pivoting on the tensor cores, FP64 refinement.
// Returns LM_ERR_NOT_CONVERGED when refinement stalls (the caller falls back
// to dgesv_ir).
int dgesv_rbt_ir(Ctx& c, int n, int nrhs, const double* A, long long lda, const double* B, long long ldb, double* X,
                 long long ldx, double tol, int max_iter, int* iters_out, double* berr_out, cudaStream_t st,
                 const IrRunner& run);
int sgetrf_nopiv(Ctx& c, int n, float* A, long long lda, float* DinvL, float* DinvU, int* rflag, cudaStream_t st);
// Depth-2 recursive butterflies (rbt.cu); np is a multiple of 4.
int rbt_diagonals(double* du, double* dv, int np, cudaStream_t st);
int rbt_transform(float* Ar, long long ldr, const double* A, long long lda, int n, int np, const double* du,
                  const double* dv, cudaStream_t st);
int rbt_rows(float* D, long long ldd, int np, int nrhs, const double* d, bool transposed, cudaStream_t st);

// Run dpotrf with caller-provided device scratch (workspace slot 1) and
// status words instead of a context's own allocations (api.cu).
int dpotrf_borrowed(int device, int num_sms, cudaStream_t st, int n, double* A, long long lda, int* d_status,
                    void* scratch, size_t scratch_bytes);

// r = b - A x for nrhs columns (FP64), and max-norm helpers (resid.cu).
int dresidual(Ctx& c, int n, int nrhs, const double* A, long long lda, const double* X, long long ldx,
              const double* B, long long ldb, double* R, long long ldr, cudaStream_t st);


// Turn CUDA-graph capture of repeated call sequences on or off for a context
// (api.cu); the serving loop's workers run each request on fresh arena
// addresses, where capture would not pay.
void ctx_set_graphs(lm_ctx* ctx, bool on);
// Most captured graphs a context keeps (oldest evicted first; default 16).
void ctx_set_graph_cache(lm_ctx* ctx, int max_graphs);

// --- batched persistent factor + solve (batch.cu) ------------------------------
struct BatchLimits {
  static constexpr int kMaxN = 256;    // largest order per instance
  static constexpr int kMaxRhs = 16;   // most right-hand sides per instance
  static constexpr int kBuckets = 4;   // size buckets n <= 32, 64, 128, 256
};
inline int batch_bucket(int n) { return n <= 32 ? 0 : n <= 64 ? 1 : n <= 128 ? 2 : 3; }

// One instance, in schedule order (largest first).
struct BatchItem {
  long long a_off;  // A_i at A + a_off: n x n row-major, ld n
  long long b_off;  // B_i at B + b_off: n x nrhs row-major, ld nrhs
  long long x_off;  // X_i at X + x_off (same shape)
  long long f_off;  // factor workspace at F + f_off: n * n doubles
  long long p_off;  // swap list at ipiv + p_off: n ints
  int n, nrhs, kind, nb, index;
};

struct BatchArgs {
  const BatchItem* items;
  int count;
  int prec;             // LM_PREC_FP64 or LM_PREC_FP32_IR
  int nmax, rmax, nbmax;
  const double* A;
  const double* B;
  double* X;
  double* F;
  int* ipiv;
  int* info;
  int* iters;
  double* berr;
  int* ticket;
  double tol;
  int max_iter;
};
// Ring of posted requests of the device-resident serving loop: descriptors
// in device memory (items[seq % cap]), the next sequence number to claim
// (head) and the number posted (tail), a stop word, and per slot in pinned
// host memory the info and the completion word (seq + 1 when done).
struct ServeRing {
  const BatchItem* items;
  int cap;
  int* head;
  const int* tail;
  const int* stop;
  int* h_info;
  int* h_done;
};
// Launch the device-resident loop (FP64 solves of the posted requests).
int serve_loop_launch(const BatchArgs& g, const ServeRing& rg, int grid, size_t smem, cudaStream_t st);

// Dynamic shared memory of the batch kernel for the given maxima.
size_t batch_smem_bytes(int nmax, int rmax, int nbmax);
// Resident CTAs per SM of the batch kernel at that shared-memory size.
int batch_occupancy(size_t smem, int* per_sm);
// Reset the ticket and launch `grid` persistent CTAs on `st`.
int batch_launch(const BatchArgs& g, int grid, size_t smem, cudaStream_t st);

}  // namespace lm
