// Host-side drivers of the FP64 factorisations and triangular solves.
//
// dgetrf — right-looking blocked LU, outer panels of kNB = 128 columns so the
//   trailing update is a k = 128 DMMA GEMM (compute-bound on B200, unlike the
//   reference's k = 32 update, LU.hs:311-357).  Each 128-wide panel is
//   factored recursively (halves down to a cluster leaf of <= 32 columns):
//     left half -> swap right half -> U12 = L11^-1 A12 -> A22 -= L21 U12 ->
//     right half -> swap left half.
//   Row interchanges are applied to every column of A, matching the
//   reference's full-row rawSwapRows (fromCol = 0, LU.hs:324-325).
//   Every U12 = L11^-1 A12 (rawTriSolvePanelTrail, LU.hs:364-407) runs as
//   inv(L11) (one CTA, blocked inversion in shared memory) times a copy of A12
//   on the DMMA GEMM: the multipliers are bounded by 1 under partial
//   pivoting, so the explicit inverse of the unit-lower block is well scaled,
//   and the block solve leaves the latency-bound substitution kernel.
// dpotrf — right-looking blocked Cholesky, kNB = 128: diagonal block in SMEM,
//   L21 = A21 L11^-T (inverse block times the panel, on the tensor cores), then
//   A22 -= L21 L21^T as a lower-triangle-only GEMM (SYRK tile skip).  Same
//   mathematics as the reference's left-looking panelCholFactor
//   (Chol.hs:279-321), different association.
// dgetrs / dpotrs — blocked substitutions: a 128 x 128 triangular block
//   solve, then the rest of the right-hand side updated by GEMM; dgetrs with
//   at most 4 right-hand sides runs one persistent launch per direction
//   (trsv.cu).
#include <algorithm>

#include "common.cuh"
#include "internal.h"

namespace lm {

namespace {

constexpr int kNB = 128;

// Scratch of the inverse-based block solves: inv(L11) (kNB x kNB) and the
// row-interchange plan.
struct TrsmScratch {
  double* Linv;
  int* plan;  // kSwapPlanInts
};

// B (w x ncols, ldb) <- inv(unit lower L11) B.  Small blocks (inside a panel)
// in one fused launch; the panel's row block as inv(L11) times B on the
// tensor cores, written in place: with m = w <= 128 there is one row of
// output tiles, so each CTA reads exactly the columns of B that it later
// overwrites, all of them before its epilogue, and no other CTA reads them.
// With have_inv, s.Linv already holds inv(L11).
int trsm_unit_lower_gemm(Ctx& c, const double* L11, long long lda, int w, double* B, long long ldb, int ncols,
                         const TrsmScratch& s, cudaStream_t st, bool have_inv = false) {
  if (w <= 0 || ncols <= 0) return LM_OK;
  if (w <= 64 && ncols <= 128 && !have_inv) {
    Prof p(c, kPhaseTrsm, (double)w * w * ncols, 8.0 * ((double)w * w / 2 + 2.0 * w * ncols), st);
    return trsm_lower_small<double>(L11, lda, w, true, B, ldb, ncols, st);
  }
  if (!have_inv) {
    Prof p(c, kPhaseTrsm, (double)w * w * w / 3.0, 8.0 * (double)w * w, st);
    LM_TRY(tri_inv_lower<double>(L11, lda, w, true, s.Linv, kNB, nullptr, st));
  }
  GemmDesc d;
  d.m = w; d.n = ncols; d.k = w;
  d.alpha = 1.0; d.beta = 0.0;
  d.A = s.Linv; d.lda = kNB;
  d.B = B; d.ldb = ldb;
  d.C = B; d.ldc = ldb;
  return dgemm(c, d, st);
}

// gemm_sms caps the SMs of the panel's own GEMMs (0 = no cap), so that a
// panel factored beside a trailing update fits on the SMs that update leaves.
int getrf_panel_rec(Ctx& c, double* A, long long lda, int n, int c0, int w, int pc0, int pw, int* ipiv,
                    const TrsmScratch& s, cudaStream_t st, int gemm_sms = 0) {
  const int R = n - c0;
  const int wmax = panel_leaf_max_width_for(c, R);
  if (wmax <= 0) return LM_ERR_UNSUPPORTED;
  if (w <= wmax) {
    // the leaf also swaps the rest of the panel [pc0, pc0 + pw)
    Prof p(c, kPhasePanel, (double)R * w * w, 16.0 * R * w, st);
    return panel_leaf<double>(c, A, lda, n, c0, w, pc0, pw, ipiv, st);
  }
  // Split so that column offsets stay multiples of 4 (16-byte TMA alignment).
  int w1 = (w >= 16) ? std::max(8, (w / 2) & ~7) : std::max(4, (w / 2) & ~3);
  if (w1 >= w) w1 = w - 4;
  const int w2 = w - w1;
  LM_TRY(getrf_panel_rec(c, A, lda, n, c0, w1, pc0, pw, ipiv, s, st, gemm_sms));
  double* A11 = A + (long long)c0 * lda + c0;
  LM_TRY(trsm_unit_lower_gemm(c, A11, lda, w1, A11 + w1, lda, w2, s, st));
  GemmDesc d;
  d.m = R - w1; d.n = w2; d.k = w1;
  d.alpha = -1.0; d.beta = 1.0;
  d.A = A11 + (long long)w1 * lda; d.lda = lda;
  d.B = A11 + w1; d.ldb = lda;
  d.C = A11 + (long long)w1 * lda + w1; d.ldc = lda;
  d.max_sms = gemm_sms;
  LM_TRY(dgemm(c, d, st));
  return getrf_panel_rec(c, A, lda, n, c0 + w1, w2, pc0, pw, ipiv, s, st, gemm_sms);
}

}  // namespace

// SMs left to a panel factored beside the trailing update (the widest panel
// leaf is a cluster of 16 CTAs of one SM each), and the order from which that
// look-ahead is used.
constexpr int kLookaheadSms = 16;
constexpr int kLookaheadMinN = 2048;

int dgetrf(Ctx& c, int n, double* A, long long lda, int* ipiv, cudaStream_t st) {
  TrsmScratch s;
  {
    void* ws = nullptr;
    LM_TRY(ctx_workspace(c, 1, sizeof(double) * (size_t)kNB * kNB + sizeof(int) * kSwapPlanInts, &ws));
    s.Linv = static_cast<double*>(ws);
    s.plan = reinterpret_cast<int*>(s.Linv + (size_t)kNB * kNB);
  }
  // Look-ahead: once the next panel's columns are updated, that panel is
  // factored on the priority stream while the rest of the trailing update
  // runs with a grid that leaves kLookaheadSms SMs free.  Its own GEMMs are
  // capped to fit there.  Nothing waits across the two streams inside a
  // kernel; at worst the panel starts when the update ends.
  const int nsm = ctx_num_sms(c);
  const bool la = n >= kLookaheadMinN && nsm > 2 * kLookaheadSms && ctx_lookahead(c);
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  if (la) LM_TRY(ctx_aux(c, &aux, &ev_fork, &ev_join));
  const int panel_sms = kLookaheadSms;
  const int rest_sms = nsm - kLookaheadSms;
  LM_TRY(getrf_panel_rec(c, A, lda, n, 0, std::min(kNB, n), 0, std::min(kNB, n), ipiv, s, st));
  for (int k0 = 0; k0 < n; k0 += kNB) {
    const int w = std::min(kNB, n - k0);
    // panel k is factored: its interchanges on the columns left and right of it
    {
      Prof p(c, kPhaseSwap, 0.0, 32.0 * w * (n - w), st);
      LM_TRY(laswp<double>(A, lda, n, ipiv, k0, k0 + w, 0, k0, k0 + w, n, ctx_status(c), st, s.plan));
    }
    if (k0 + w >= n) break;
    const int m = n - k0 - w;
    const int wn = std::min(kNB, m);  // next panel
    double* A11 = A + (long long)k0 * lda + k0;
    // with look-ahead, inv(L11) of this panel was formed beside the previous update
    LM_TRY(trsm_unit_lower_gemm(c, A11, lda, w, A11 + w, lda, m, s, st, la && k0 > 0));
    GemmDesc d;  // A22 -= L21 U12, the next panel's columns first
    d.m = m; d.n = wn; d.k = w;
    d.alpha = -1.0; d.beta = 1.0;
    d.A = A11 + (long long)w * lda; d.lda = lda;
    d.B = A11 + w; d.ldb = lda;
    d.C = A11 + (long long)w * lda + w; d.ldc = lda;
    LM_TRY(dgemm(c, d, st));
    GemmDesc r = d;  // the rest of the columns
    r.n = m - wn;
    r.B = A11 + w + wn;
    r.C = A11 + (long long)w * lda + w + wn;
    if (la) {
      LM_CUDA_TRY(cudaEventRecord(ev_fork, st));
      LM_CUDA_TRY(cudaStreamWaitEvent(aux, ev_fork, 0));
      LM_TRY(getrf_panel_rec(c, A, lda, n, k0 + w, wn, k0 + w, wn, ipiv, s, aux, panel_sms));
      if (k0 + w + wn < n) {
        // the next step's block solve needs inv(L11) of this panel; the
        // current step's product with the old inverse has already run
        Prof p(c, kPhaseTrsm, (double)wn * wn * wn / 3.0, 8.0 * (double)wn * wn, aux);
        LM_TRY(tri_inv_lower<double>(A + (long long)(k0 + w) * lda + k0 + w, lda, wn, true, s.Linv, kNB, nullptr, aux));
      }
      LM_CUDA_TRY(cudaEventRecord(ev_join, aux));
      if (r.n > 0) {
        r.max_sms = rest_sms;
        LM_TRY(dgemm(c, r, st));
      }
      LM_CUDA_TRY(cudaStreamWaitEvent(st, ev_join, 0));
    } else {
      if (r.n > 0) LM_TRY(dgemm(c, r, st));
      LM_TRY(getrf_panel_rec(c, A, lda, n, k0 + w, wn, k0 + w, wn, ipiv, s, st));
    }
  }
  return LM_OK;
}

namespace {

// L21 = A21 inv(L11)^T for the block column at j0 (w wide, R rows below):
// inv(L11) in one CTA, then the product with a copy of A21 on the DMMA GEMM.
int potrf_panel(Ctx& c, double* A, long long lda, int j0, int w, int R, double* Linv, double* W21, cudaStream_t st,
                int max_sms = 0) {
  double* A11 = A + (long long)j0 * lda + j0;
  double* A21 = A11 + (long long)w * lda;
  {
    Prof p(c, kPhaseTrsm, (double)w * w * w / 3.0, 16.0 * w * w, st);
    LM_TRY(tri_inv_lower<double>(A11, lda, w, false, Linv, kNB, nullptr, st));
  }
  {
    Prof p(c, kPhaseOther, 0.0, 16.0 * R * w, st);
    LM_TRY(copy2d<double>(W21, kNB, A21, lda, R, w, st));
  }
  GemmDesc t;  // L21 = A21 * L11^-T
  t.m = R; t.n = w; t.k = w; t.alpha = 1.0; t.beta = 0.0;
  t.A = W21; t.lda = kNB; t.B = Linv; t.ldb = kNB; t.b_trans = true;
  t.C = A21; t.ldc = lda;
  t.max_sms = max_sms;
  return dgemm(c, t, st);
}

}  // namespace

// Right-looking blocked Cholesky with look-ahead: once the trailing update
// has reached the next block column (its diagonal block and everything
// below), that column is factored on the priority stream (diagonal block,
// inverse, L21) while the rest of the lower-triangle update runs on the
// other SMs.  The two streams touch disjoint columns: the update reads the
// current L21 and writes columns right of the next block column.
int dpotrf(Ctx& c, int n, double* A, long long lda, cudaStream_t st) {
  const size_t blk = (size_t)kNB * kNB;
  void* ws = nullptr;
  LM_TRY(ctx_workspace(c, 1, sizeof(double) * (blk + (size_t)n * kNB), &ws));
  double* Linv = static_cast<double*>(ws);
  double* W21 = Linv + blk;
  const int nsm = ctx_num_sms(c);
  const bool la = n >= kLookaheadMinN && nsm > 2 * kLookaheadSms && ctx_lookahead(c);
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  if (la) LM_TRY(ctx_aux(c, &aux, &ev_fork, &ev_join));
  auto factor_column = [&](int j0, cudaStream_t s, int max_sms) {
    const int w = std::min(kNB, n - j0);
    const int R = n - j0 - w;
    {
      Prof p(c, kPhasePanel, (double)w * w * w / 3.0, 8.0 * w * w, s);
      LM_TRY(potrf_block<double>(c, A + (long long)j0 * lda + j0, lda, w, j0, s));
    }
    if (R > 0) LM_TRY(potrf_panel(c, A, lda, j0, w, R, Linv, W21, s, max_sms));
    return LM_OK;
  };
  LM_TRY(factor_column(0, st, 0));
  for (int j0 = 0; j0 < n; j0 += kNB) {
    const int w = std::min(kNB, n - j0);
    const int R = n - j0 - w;
    if (R <= 0) break;
    double* A21 = A + (long long)(j0 + w) * lda + j0;
    double* A22 = A21 + w;
    const int wn = std::min(kNB, R);  // next block column
    // A22 -= L21 L21^T: the next block column first (all R rows of it)
    GemmDesc d;
    d.m = R; d.n = wn; d.k = w; d.alpha = -1.0; d.beta = 1.0;
    d.A = A21; d.lda = lda; d.B = A21; d.ldb = lda; d.b_trans = true;
    d.C = A22; d.ldc = lda;
    LM_TRY(dgemm(c, d, st));
    const int rest = R - wn;
    GemmDesc r;  // then the lower triangle right of it
    r.m = rest; r.n = rest; r.k = w; r.alpha = -1.0; r.beta = 1.0;
    r.A = A21 + (long long)wn * lda; r.lda = lda; r.B = r.A; r.ldb = lda; r.b_trans = true;
    r.lower_only = true;
    r.C = A22 + (long long)wn * lda + wn; r.ldc = lda;
    if (la) {
      LM_CUDA_TRY(cudaEventRecord(ev_fork, st));
      LM_CUDA_TRY(cudaStreamWaitEvent(aux, ev_fork, 0));
      LM_TRY(factor_column(j0 + w, aux, kLookaheadSms));
      LM_CUDA_TRY(cudaEventRecord(ev_join, aux));
      if (rest > 0) {
        r.max_sms = nsm - kLookaheadSms;
        LM_TRY(dgemm(c, r, st));
      }
      LM_CUDA_TRY(cudaStreamWaitEvent(st, ev_join, 0));
    } else {
      if (rest > 0) LM_TRY(dgemm(c, r, st));
      LM_TRY(factor_column(j0 + w, st, 0));
    }
  }
  return zero_upper<double>(A, lda, n, st);
}

// luNoPivot (LU.hs:196-214) blocked: right-looking with 128-wide diagonal
// blocks, each factored without interchanges in one CTA (registers); then
// U12 = inv(L11) A12 and L21 = A21 inv(U11) as products with the blocks'
// inverses on the DMMA GEMM (the reference's precondition, e.g. diagonal
// dominance, keeps the diagonal blocks well conditioned), and
// A22 -= L21 U12.  A zero pivot is recorded in status[1] and, as in the
// reference, the division by it still happens.
int dgetrf_nopiv(Ctx& c, int n, double* A, long long lda, cudaStream_t st) {
  void* ws = nullptr;
  const size_t blk = (size_t)kNB * kNB;
  LM_TRY(ctx_workspace(c, 1, sizeof(double) * (3 * blk + (size_t)n * kNB) + sizeof(int) * kSwapPlanInts, &ws));
  double* Linv = static_cast<double*>(ws);
  double* Ut = Linv + blk;
  double* Uinv = Ut + blk;
  double* W21 = Uinv + blk;
  TrsmScratch s;
  s.Linv = Linv;
  s.plan = reinterpret_cast<int*>(W21 + (size_t)n * kNB);
  for (int j0 = 0; j0 < n; j0 += kNB) {
    const int w = std::min(kNB, n - j0);
    const int R = n - j0 - w;
    double* A11 = A + (long long)j0 * lda + j0;
    {
      Prof p(c, kPhasePanel, 2.0 / 3.0 * w * w * w, 16.0 * w * w, st);
      LM_TRY(lu_nopiv_block(A11, lda, w, j0, ctx_status(c), st));
    }
    if (R <= 0) break;
    double* A12 = A11 + w;
    double* A21 = A11 + (long long)w * lda;
    LM_TRY(trsm_unit_lower_gemm(c, A11, lda, w, A12, lda, R, s, st));
    {
      Prof p(c, kPhaseTrsm, (double)w * w * w / 3.0, 24.0 * (double)w * w, st);
      LM_TRY(transpose_block(Ut, kNB, A11, lda, w, st));
      LM_TRY(tri_inv_lower<double>(Ut, kNB, w, false, Uinv, kNB, nullptr, st));
    }
    {
      Prof p(c, kPhaseOther, 0.0, 16.0 * R * w, st);
      LM_TRY(copy2d<double>(W21, kNB, A21, lda, R, w, st));
    }
    GemmDesc t;  // L21 = A21 inv(U11) = W21 (inv(U11^T))^T
    t.m = R; t.n = w; t.k = w; t.alpha = 1.0; t.beta = 0.0;
    t.A = W21; t.lda = kNB; t.B = Uinv; t.ldb = kNB; t.b_trans = true;
    t.C = A21; t.ldc = lda;
    LM_TRY(dgemm(c, t, st));
    GemmDesc d;  // A22 -= L21 U12
    d.m = R; d.n = R; d.k = w; d.alpha = -1.0; d.beta = 1.0;
    d.A = A21; d.lda = lda; d.B = A12; d.ldb = lda;
    d.C = A21 + w; d.ldc = lda;
    LM_TRY(dgemm(c, d, st));
  }
  return LM_OK;
}

namespace {

// Copy to even-stride, 16-byte aligned buffers when the caller's are not
// (TMA row alignment); returns the buffers to use.
struct SolveBufs {
  const double* M;
  long long ldm;
  double* X;
  long long ldx;
  bool copied_x;
};

int solve_bufs(Ctx& c, int n, int nrhs, const double* M, long long ldm, double* B, long long ldb,
               SolveBufs& sb, cudaStream_t st) {
  sb.M = M; sb.ldm = ldm; sb.X = B; sb.ldx = ldb; sb.copied_x = false;
  const bool m_ok = !(reinterpret_cast<uintptr_t>(M) & 15) && !(ldm & 1);
  const bool x_ok = !(reinterpret_cast<uintptr_t>(B) & 15) && !(ldb & 1);
  const long long ldm2 = m_ok ? 0 : (n + 7) / 8 * 8;
  const long long ldx2 = x_ok ? 0 : (nrhs + 7) / 8 * 8;
  const size_t bytes = sizeof(double) * ((size_t)n * ldm2 + (size_t)n * ldx2);
  if (bytes == 0) return LM_OK;
  void* ws = nullptr;
  LM_TRY(ctx_workspace(c, 2, bytes, &ws));
  double* p = static_cast<double*>(ws);
  if (!m_ok) {
    LM_TRY(copy2d<double>(p, ldm2, M, ldm, n, n, st));
    sb.M = p; sb.ldm = ldm2;
    p += (size_t)n * ldm2;
  }
  if (!x_ok) {
    LM_TRY(copy2d<double>(p, ldx2, B, ldb, n, nrhs, st));
    sb.X = p; sb.ldx = ldx2; sb.copied_x = true;
  }
  return LM_OK;
}

// Forward substitution with the lower triangle of M (unit or not), blocked.
int forward_blocked(Ctx& c, int n, int nrhs, const double* M, long long ldm, bool unit, double* X,
                    long long ldx, cudaStream_t st) {
  for (int i0 = 0; i0 < n; i0 += kNB) {
    const int w = std::min(kNB, n - i0);
    const double* Mii = M + (long long)i0 * ldm + i0;
    {
      Prof p(c, kPhaseTrsm, (double)w * w * nrhs, 8.0 * ((double)w * w / 2 + 2.0 * w * nrhs), st);
      LM_TRY(trsm_left<double>(Mii, ldm, w, true, unit, false, X + (long long)i0 * ldx, ldx, nrhs, st));
    }
    if (i0 + w < n) {
      GemmDesc d;
      d.m = n - i0 - w; d.n = nrhs; d.k = w; d.alpha = -1.0; d.beta = 1.0;
      d.A = Mii + (long long)w * ldm; d.lda = ldm;
      d.B = X + (long long)i0 * ldx; d.ldb = ldx;
      d.C = X + (long long)(i0 + w) * ldx; d.ldc = ldx;
      LM_TRY(dgemm(c, d, st));
    }
  }
  return LM_OK;
}

}  // namespace

int dgetrs(Ctx& c, int n, int nrhs, const double* LU, long long lda, const int* ipiv, double* B,
           long long ldb, cudaStream_t st) {
  if (nrhs <= 4) {
    // few right-hand sides: P b, then one persistent launch per direction
    void* ws = nullptr;
    LM_TRY(ctx_workspace(c, 2, 64 + sizeof(double) * (size_t)n * nrhs, &ws));
    {
      Prof p(c, kPhaseSwap, 0.0, 32.0 * n * nrhs, st);
      LM_TRY(laswp_narrow<double>(B, ldb, n, nrhs, ipiv, reinterpret_cast<double*>(static_cast<char*>(ws) + 64),
                                  ctx_status(c), st));
    }
    Prof p(c, kPhaseTrsm, 2.0 * n * n * nrhs, 8.0 * n * n, st);
    return trsv_lu<double>(LU, lda, n, nrhs, nullptr, nullptr, B, ldb, static_cast<int*>(ws), ctx_status(c), st);
  }
  SolveBufs sb;
  LM_TRY(solve_bufs(c, n, nrhs, LU, lda, B, ldb, sb, st));
  // P b (applyPivotsForward, LU.hs:493-507)
  {
    Prof p(c, kPhaseSwap, 0.0, 32.0 * n * nrhs, st);
    LM_TRY(laswp<double>(sb.X, sb.ldx, n, ipiv, 0, n, 0, nrhs, 0, 0, ctx_status(c), st));
  }
  LM_TRY(forward_blocked(c, n, nrhs, sb.M, sb.ldm, true, sb.X, sb.ldx, st));
  const int nblk = (n + kNB - 1) / kNB;
  for (int b = nblk - 1; b >= 0; --b) {
    const int i0 = b * kNB;
    const int w = std::min(kNB, n - i0);
    const double* Uii = sb.M + (long long)i0 * sb.ldm + i0;
    {
      Prof p(c, kPhaseTrsm, (double)w * w * nrhs, 8.0 * ((double)w * w / 2 + 2.0 * w * nrhs), st);
      LM_TRY(trsm_left<double>(Uii, sb.ldm, w, false, false, false, sb.X + (long long)i0 * sb.ldx, sb.ldx, nrhs,
                               st));
    }
    if (i0 > 0) {
      GemmDesc d;
      d.m = i0; d.n = nrhs; d.k = w; d.alpha = -1.0; d.beta = 1.0;
      d.A = sb.M + i0; d.lda = sb.ldm;
      d.B = sb.X + (long long)i0 * sb.ldx; d.ldb = sb.ldx;
      d.C = sb.X; d.ldc = sb.ldx;
      LM_TRY(dgemm(c, d, st));
    }
  }
  if (sb.copied_x) LM_TRY(copy2d<double>(B, ldb, sb.X, sb.ldx, n, nrhs, st));
  return LM_OK;
}

int dpotrs(Ctx& c, int n, int nrhs, const double* G, long long lda, double* B, long long ldb,
           cudaStream_t st) {
  if (nrhs <= 4) {
    // few right-hand sides: G packed with G^T above the diagonal, then one
    // persistent launch per direction (the same kernels as dgetrs, with the
    // stored diagonal of G)
    const long long ldp = (n + 7) / 8 * 8;
    void* ws = nullptr;
    LM_TRY(ctx_workspace(c, 2, 256 + sizeof(double) * (size_t)n * ldp, &ws));
    int* sync = static_cast<int*>(ws);
    double* P = reinterpret_cast<double*>(static_cast<char*>(ws) + 256);
    {
      Prof p(c, kPhaseOther, 0.0, 16.0 * n * n, st);
      LM_TRY(pack_lower_sym(P, ldp, G, lda, n, st));
    }
    Prof p(c, kPhaseTrsm, 2.0 * n * n * nrhs, 8.0 * n * n, st);
    return trsv_lu<double>(P, ldp, n, nrhs, nullptr, nullptr, B, ldb, sync, ctx_status(c), st, nullptr, true, false);
  }
  SolveBufs sb;
  LM_TRY(solve_bufs(c, n, nrhs, G, lda, B, ldb, sb, st));
  LM_TRY(forward_blocked(c, n, nrhs, sb.M, sb.ldm, false, sb.X, sb.ldx, st));
  // G^T x = y, bottom-up; the off-diagonal update uses G's row block transposed.
  const int nblk = (n + kNB - 1) / kNB;
  for (int b = nblk - 1; b >= 0; --b) {
    const int i0 = b * kNB;
    const int w = std::min(kNB, n - i0);
    const double* Gii = sb.M + (long long)i0 * sb.ldm + i0;
    {
      Prof p(c, kPhaseTrsm, (double)w * w * nrhs, 8.0 * ((double)w * w / 2 + 2.0 * w * nrhs), st);
      LM_TRY(trsm_left<double>(Gii, sb.ldm, w, true, false, true, sb.X + (long long)i0 * sb.ldx, sb.ldx, nrhs,
                               st));
    }
    if (i0 > 0) {
      GemmDesc d;
      d.m = i0; d.n = nrhs; d.k = w; d.alpha = -1.0; d.beta = 1.0;
      d.A = sb.M + (long long)i0 * sb.ldm; d.lda = sb.ldm; d.a_trans = true;
      d.B = sb.X + (long long)i0 * sb.ldx; d.ldb = sb.ldx;
      d.C = sb.X; d.ldc = sb.ldx;
      LM_TRY(dgemm(c, d, st));
    }
  }
  if (sb.copied_x) LM_TRY(copy2d<double>(B, ldb, sb.X, sb.ldx, n, nrhs, st));
  return LM_OK;
}

}  // namespace lm
