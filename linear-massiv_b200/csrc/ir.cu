// Mixed precision: FP32 LU with TF32 tensor-core updates, FP64 iterative
// refinement.  No counterpart in linear-massiv (its luSolveP, LU.hs:265-304, is
// FP64 throughout); the refinement recovers FP64-accurate solutions:
//
//   A32 = fl32(A);  P A32 = L U   (panel leaves and TRSM in FP32, all
//                                  Schur-complement GEMMs on tcgen05 TF32)
//   x = 0, r = b
//   repeat:  d = U^-1 L^-1 P fl32(r)       (FP32 substitutions)
//            x = x + d                     (FP64)
//            r = b - A x                   (FP64, original A)
//   until  ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol  (per column)
//
// The stopping metric is the reference test suite's scaledResidualLinear
// without the n*eps guard (test/Test/Residuals.hs:69-78).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace lm {

void count_launch(int n);
// C = alpha A Bt^T + beta C on tcgen05 (sgemm_tc.cu); max_ctas caps the
// persistent grid (0 = one CTA per SM); with gate set the launch does
// nothing when *gate == 0 (a device-side switch inside captured sequences).
int sgemm_tf32(Ctx& ctx, int m, int n, int k, float alpha, const float* A, long long lda, const float* Bt,
               long long ldb, float beta, float* C, long long ldc, cudaStream_t st, const float* Alo,
               const float* Btlo, int max_ctas = 0, const int* gate = nullptr);


namespace {

constexpr int kNB = 128;

__global__ void d2s_kernel(float* dst, long long ldd, const double* src, long long lds, int rows, int cols) {
  const long long total = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i % cols);
    dst[(long long)r * ldd + c] = (float)src[(long long)r * lds + c];
  }
}

// High part of the 3xTF32 split: a rounded to the nearest TF32 value (ties
// away from zero), so that the remainder a - hi is exact in FP32 and at most
// 2^-11 |a|; the remainder is rounded the same way before it is stored, and
// the tensor core then reads both parts without further loss.
__device__ __forceinline__ float tf32_hi(float a) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(a));
  return __uint_as_float(r);
}

// Split for 3xTF32: hi = a rounded to TF32, lo = a - hi (exact in FP32)
// rounded to TF32; hi + lo carries a to within 2^-22 |a|.
// dst_hi/dst_lo (cols x rows) = split(src (rows x cols))^T.
// With `gate` given and *gate == 0 nothing is written (a correction step
// switched off on the device, inside a captured sequence, whose consumers are
// gated by the same flag).  With `cpy` given, src is also copied unchanged to
// cpy (rows x cols, ldc).
__global__ void transpose_split_kernel(float* dhi, float* dlo, long long ldd, const float* src, long long lds,
                                       int rows, int cols, const int* gate = nullptr, float* cpy = nullptr,
                                       long long ldc = 0) {
  if (gate != nullptr && *gate == 0) return;
  __shared__ float tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = by + j, c = bx + threadIdx.x;
    if (r < rows && c < cols) {
      const float a = src[(long long)r * lds + c];
      tile[j][threadIdx.x] = a;
      if (cpy != nullptr) cpy[(long long)r * ldc + c] = a;
    }
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = bx + j, c = by + threadIdx.x;
    if (r < cols && c < rows) {
      const float a = tile[threadIdx.x][j];
      const float h = tf32_hi(a);
      dhi[(long long)r * ldd + c] = h;
      dlo[(long long)r * ldd + c] = tf32_hi(a - h);
    }
  }
}

// dst_hi/dst_lo (rows x cols, ldd) = split(src (rows x cols, lds)).
// `gate` and `cpy` as for transpose_split_kernel.
__global__ void split_kernel(float* dhi, float* dlo, long long ldd, const float* src, long long lds, int rows,
                             int cols, const int* gate = nullptr, float* cpy = nullptr, long long ldc = 0) {
  if (gate != nullptr && *gate == 0) return;
  const long long total = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i % cols);
    const float a = src[(long long)r * lds + c];
    if (cpy != nullptr) cpy[(long long)r * ldc + c] = a;
    const float h = tf32_hi(a);
    dhi[(long long)r * ldd + c] = h;
    dlo[(long long)r * ldd + c] = tf32_hi(a - h);
  }
}

// X[m x nrhs] -= M[m x k] * Y[k x nrhs] in FP32 (exact fp32 FMAs), one warp per
// row, nrhs <= 64 (the right-hand-side updates of the FP32 substitutions).
__global__ void sgemm_rhs_kernel(int m, int k, int nrhs, const float* __restrict__ M, long long ldm,
                                 const float* __restrict__ Y, long long ldy, float* X, long long ldx) {
  const int warps = blockDim.x >> 5;
  const int row = blockIdx.x * warps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= m) return;
  const float* mr = M + (long long)row * ldm;
  for (int c0 = 0; c0 < nrhs; c0 += 8) {
    float acc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = 0.f;
    for (int kk = lane; kk < k; kk += 32) {
      const float a = mr[kk];
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c0 + c < nrhs) acc[c] = fmaf(a, Y[(long long)kk * ldy + c0 + c], acc[c]);
    }
#pragma unroll
    for (int c = 0; c < 8; ++c)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    if (lane == 0)
      for (int c = 0; c < 8 && c0 + c < nrhs; ++c) X[(long long)row * ldx + c0 + c] -= acc[c];
  }
}

// X (FP64) += D (FP32); R (FP32) <- fl32(Rd) helpers.
__global__ void add_s2d_kernel(double* X, long long ldx, const float* D, long long ldd, int rows, int cols) {
  const long long total = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i % cols);
    X[(long long)r * ldx + c] += (double)D[(long long)r * ldd + c];
  }
}

// ||A||_inf (max row sum of |a_ij|) into out[0] as the bits of a non-negative
// double (atomicMax on the ordered integer image).
__global__ void norm_inf_rows_kernel(const double* A, long long lda, int n, unsigned long long* out) {
  const int warps = blockDim.x >> 5;
  const int row = blockIdx.x * warps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  double s = 0.0;
  for (int j = lane; j < n; j += 32) s += fabs(A[(long long)row * lda + j]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) atomicMax(out, (unsigned long long)__double_as_longlong(s));
}

// Per column c: max_i |V_ic| into out[c] (ordered-integer atomicMax).
__global__ void colmax_abs_kernel(const double* V, long long ldv, int rows, int cols, unsigned long long* out) {
  const long long total = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i % cols);
    atomicMax(out + c, (unsigned long long)__double_as_longlong(fabs(V[(long long)r * ldv + c])));
  }
}

int grid_of(long long total) { return (int)std::max<long long>(1, std::min<long long>(cdivll(total, 256), 2048)); }

// Scratch for the split operands of the 3xTF32 update: L21 -> Ahi/Alo
// (m x k), U12^T -> Bhi/Blo (n x k); all with leading dimension 128 (k <= 128);
// Lhi/Llo hold split(inv(L11)) for the block solves (128 x 128).
struct SScratch {
  float *Ahi, *Alo, *Bhi, *Blo, *Lhi, *Llo;
  long long ld;
  int* plan;  // row-interchange plan (kSwapPlanInts)
};

// B (w x ncols, ldb) <- inv(unit lower L11) B: small blocks (inside a panel)
// in one fused FP32 launch; otherwise the inverse of the diagonal block (one
// CTA) times B on the tensor cores as 3xTF32.
int s_trsm_unit_lower(Ctx& c, const float* L11, long long lda, int w, float* B, long long ldb, int ncols,
                      SScratch& s, cudaStream_t st, int max_ctas = 0) {
  if (w <= 0 || ncols <= 0) return LM_OK;
  if (w <= 64 && ncols <= 128) {
    Prof p(c, kPhaseTrsm, (double)w * w * ncols, 4.0 * ((double)w * w / 2 + 2.0 * w * ncols), st);
    return trsm_lower_small<float>(L11, lda, w, true, B, ldb, ncols, st);
  }
  {
    Prof p(c, kPhaseTrsm, (double)w * w * w / 3.0, 12.0 * (double)w * w, st);
    LM_TRY(tri_inv_lower<float>(L11, lda, w, true, s.Lhi, kNB, s.Llo, st));
  }
  dim3 tb(32, 8), tg(cdiv(ncols, 32), cdiv(w, 32));
  transpose_split_kernel<<<tg, tb, 0, st>>>(s.Bhi, s.Blo, s.ld, B, ldb, w, ncols);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return sgemm_tf32(c, w, ncols, w, 1.0f, s.Lhi, kNB, s.Bhi, s.ld, 0.0f, B, ldb, st, s.Llo, s.Blo, max_ctas);
}

int s_update(Ctx& c, int m, int n, int k, float* A21, long long lda, const float* U12, float* C, SScratch& s,
             cudaStream_t st, int max_ctas = 0) {
  // C -= A21 (m x k) * U12 (k x n), as 3xTF32 on the tensor cores
  dim3 tb(32, 8), tg(cdiv(n, 32), cdiv(k, 32));
  transpose_split_kernel<<<tg, tb, 0, st>>>(s.Bhi, s.Blo, s.ld, U12, lda, k, n);
  split_kernel<<<grid_of((long long)m * k), 256, 0, st>>>(s.Ahi, s.Alo, s.ld, A21, lda, m, k);
  count_launch(2);
  LM_CUDA_TRY(cudaGetLastError());
  return sgemm_tf32(c, m, n, k, -1.0f, s.Ahi, s.ld, s.Bhi, s.ld, 1.0f, C, lda, st, s.Alo, s.Blo, max_ctas);
}

// max_ctas caps the grids of the panel's own GEMMs (0 = no cap), so that a
// panel factored beside a trailing update fits on the SMs that update leaves.
int sgetrf_panel_rec(Ctx& c, float* A, long long lda, int n, int c0, int w, int pc0, int pw, int* ipiv, SScratch& s,
                     cudaStream_t st, int max_ctas = 0) {
  const int R = n - c0;
  const int wmax = panel_leaf_max_width_for(c, R);
  if (wmax <= 0) return LM_ERR_UNSUPPORTED;
  if (w <= wmax) {
    Prof p(c, kPhasePanel, (double)R * w * w, 8.0 * R * w, st);
    return panel_leaf<float>(c, A, lda, n, c0, w, pc0, pw, ipiv, st);
  }
  int w1 = (w >= 16) ? std::max(8, (w / 2) & ~7) : std::max(4, (w / 2) & ~3);
  if (w1 >= w) w1 = w - 4;
  const int w2 = w - w1;
  LM_TRY(sgetrf_panel_rec(c, A, lda, n, c0, w1, pc0, pw, ipiv, s, st, max_ctas));
  float* A11 = A + (long long)c0 * lda + c0;
  LM_TRY(s_trsm_unit_lower(c, A11, lda, w1, A11 + w1, lda, w2, s, st, max_ctas));
  LM_TRY(s_update(c, R - w1, w2, w1, A11 + (long long)w1 * lda, lda, A11 + w1, A11 + (long long)w1 * lda + w1, s, st,
                  max_ctas));
  return sgetrf_panel_rec(c, A, lda, n, c0 + w1, w2, pc0, pw, ipiv, s, st, max_ctas);
}

// Split-operand scratch set carved from `p` (4 n x 128 + 2 128 x 128 floats,
// then the interchange plan); returns the end of the set.
char* carve_scratch(SScratch& s, char* p, int n) {
  s.ld = kNB;
  s.Ahi = reinterpret_cast<float*>(p);
  s.Alo = s.Ahi + (size_t)n * kNB;
  s.Bhi = s.Alo + (size_t)n * kNB;
  s.Blo = s.Bhi + (size_t)n * kNB;
  s.Lhi = s.Blo + (size_t)n * kNB;
  s.Llo = s.Lhi + (size_t)kNB * kNB;
  s.plan = reinterpret_cast<int*>(s.Llo + (size_t)kNB * kNB);
  return reinterpret_cast<char*>(s.plan) + ((sizeof(int) * kSwapPlanInts + 255) / 256) * 256;
}

size_t scratch_set_bytes(int n) {
  return sizeof(float) * (4 * (size_t)n * kNB + 2 * (size_t)kNB * kNB) + ((sizeof(int) * kSwapPlanInts + 255) / 256) * 256;
}

// SMs left to a panel factored beside the trailing update (the widest panel
// leaf is a cluster of 16 CTAs of one SM each), and the order from which that
// look-ahead is used.
constexpr int kSLookaheadSms = 16;
constexpr int kSLookaheadMinN = 2048;

}  // namespace

// FP32 LU with partial pivoting (the same pivot rule as the FP64 path), 128-
// column panels factored by cluster leaves, U12 = inv(L11) A12 and every
// Schur-complement update as 3xTF32 on tcgen05.  Look-ahead as in dgetrf:
// once the next panel's columns are updated, that panel is factored on the
// priority stream (its own GEMMs capped to the SMs left free) while the rest
// of the trailing update runs; its interchanges reach the columns right of it
// after the join.  The two streams use separate split-operand scratch.
int sgetrf(Ctx& c, int n, float* A, long long lda, int* ipiv, cudaStream_t st) {
  const int nsm = ctx_num_sms(c);
  const bool la = n >= kSLookaheadMinN && nsm > 2 * kSLookaheadSms && ctx_lookahead(c);
  void* ws = nullptr;
  LM_TRY(ctx_workspace(c, 1, (la ? 2 : 1) * scratch_set_bytes(n), &ws));
  SScratch s, sa;
  char* p = carve_scratch(s, static_cast<char*>(ws), n);
  if (la) carve_scratch(sa, p, n);
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  if (la) LM_TRY(ctx_aux(c, &aux, &ev_fork, &ev_join));
  LM_TRY(sgetrf_panel_rec(c, A, lda, n, 0, std::min(kNB, n), 0, std::min(kNB, n), ipiv, s, st));
  for (int k0 = 0; k0 < n; k0 += kNB) {
    const int w = std::min(kNB, n - k0);
    {
      Prof p2(c, kPhaseSwap, 0.0, 16.0 * w * (n - w), st);
      LM_TRY(laswp<float>(A, lda, n, ipiv, k0, k0 + w, 0, k0, k0 + w, n, ctx_status(c), st, s.plan));
    }
    if (k0 + w >= n) break;
    const int m = n - k0 - w;
    const int wn = std::min(kNB, m);  // next panel
    float* A11 = A + (long long)k0 * lda + k0;
    LM_TRY(s_trsm_unit_lower(c, A11, lda, w, A11 + w, lda, m, s, st));
    // A22 -= L21 U12: the next panel's columns first
    LM_TRY(s_update(c, m, wn, w, A11 + (long long)w * lda, lda, A11 + w, A11 + (long long)w * lda + w, s, st));
    const int rest = m - wn;
    if (la) {
      LM_CUDA_TRY(cudaEventRecord(ev_fork, st));
      LM_CUDA_TRY(cudaStreamWaitEvent(aux, ev_fork, 0));
      LM_TRY(sgetrf_panel_rec(c, A, lda, n, k0 + w, wn, k0 + w, wn, ipiv, sa, aux, kSLookaheadSms));
      LM_CUDA_TRY(cudaEventRecord(ev_join, aux));
      if (rest > 0)
        LM_TRY(s_update(c, m, rest, w, A11 + (long long)w * lda, lda, A11 + w + wn, A11 + (long long)w * lda + w + wn,
                        s, st, nsm - kSLookaheadSms));
      LM_CUDA_TRY(cudaStreamWaitEvent(st, ev_join, 0));
    } else {
      if (rest > 0)
        LM_TRY(s_update(c, m, rest, w, A11 + (long long)w * lda, lda, A11 + w + wn, A11 + (long long)w * lda + w + wn,
                        s, st));
      LM_TRY(sgetrf_panel_rec(c, A, lda, n, k0 + w, wn, k0 + w, wn, ipiv, s, st));
    }
  }
  return LM_OK;
}

// Solve with the FP32 factors: X (n x nrhs, FP32, ldx) overwritten.
int sgetrs(Ctx& c, int n, int nrhs, const float* LU, long long lda, const int* ipiv, float* X, long long ldx,
           cudaStream_t st) {
  {
    Prof p(c, kPhaseSwap, 0.0, 16.0 * n * nrhs, st);
    LM_TRY(laswp<float>(X, ldx, n, ipiv, 0, n, 0, nrhs, 0, 0, ctx_status(c), st));
  }
  for (int i0 = 0; i0 < n; i0 += kNB) {
    const int w = std::min(kNB, n - i0);
    const float* Lii = LU + (long long)i0 * lda + i0;
    {
      Prof p(c, kPhaseTrsm, (double)w * w * nrhs, 4.0 * ((double)w * w / 2 + 2.0 * w * nrhs), st);
      LM_TRY(trsm_left<float>(Lii, lda, w, true, true, false, X + (long long)i0 * ldx, ldx, nrhs, st));
    }
    if (i0 + w < n) {
      const int m = n - i0 - w;
      Prof p(c, kPhaseGemm, 2.0 * m * w * nrhs, 4.0 * (double)m * w, st);
      sgemm_rhs_kernel<<<cdiv(m, 8), 256, 0, st>>>(m, w, nrhs, Lii + (long long)w * lda, lda,
                                                   X + (long long)i0 * ldx, ldx, X + (long long)(i0 + w) * ldx, ldx);
      count_launch(1);
      LM_CUDA_TRY(cudaGetLastError());
    }
  }
  const int nblk = (n + kNB - 1) / kNB;
  for (int b = nblk - 1; b >= 0; --b) {
    const int i0 = b * kNB;
    const int w = std::min(kNB, n - i0);
    const float* Uii = LU + (long long)i0 * lda + i0;
    {
      Prof p(c, kPhaseTrsm, (double)w * w * nrhs, 4.0 * ((double)w * w / 2 + 2.0 * w * nrhs), st);
      LM_TRY(trsm_left<float>(Uii, lda, w, false, false, false, X + (long long)i0 * ldx, ldx, nrhs, st));
    }
    if (i0 > 0) {
      Prof p(c, kPhaseGemm, 2.0 * i0 * w * nrhs, 4.0 * (double)i0 * w, st);
      sgemm_rhs_kernel<<<cdiv(i0, 8), 256, 0, st>>>(i0, w, nrhs, LU + i0, lda, X + (long long)i0 * ldx, ldx, X,
                                                    ldx);
      count_launch(1);
      LM_CUDA_TRY(cudaGetLastError());
    }
  }
  return LM_OK;
}

int convert_d2s(float* dst, long long ldd, const double* src, long long lds, int rows, int cols, cudaStream_t st) {
  d2s_kernel<<<grid_of((long long)rows * cols), 256, 0, st>>>(dst, ldd, src, lds, rows, cols);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

namespace {

// Refinement loop shared by both low-precision factorisations.  R (n x ldr
// FP64), D (np x ldr FP32, np >= n) and nrm (2 + 3 * 64 words, nrm[0] and
// nrm[1..] already hold ||A||_inf and ||B_c||_inf) are device scratch.
// `correct(D, s)` turns D = fl32(r) (rows n..np-1 zero) into the correction.
// With stall_exit the loop gives up after two steps in a row that fail to
// reduce the worst backward error, or when the observed contraction rate
// could not reach tol within max_iter, so that a poor factor hands over to
// the next method early.
int refine(Ctx& c, int n, int np, int nrhs, const double* A, long long lda, const double* B, long long ldb, double* X,
           long long ldx, double tol, int max_iter, bool stall_exit, double* R, long long ldr, float* D,
           unsigned long long* nrm, int* iters_out, double* berr_out, cudaStream_t st, const IrRunner& run,
           const std::function<int(float*, cudaStream_t)>& correct) {
  // x = 0, r = b
  LM_CUDA_TRY(cudaMemset2DAsync(X, sizeof(double) * ldx, 0, sizeof(double) * nrhs, n, st));
  LM_TRY(copy2d<double>(R, ldr, B, ldb, n, nrhs, st));
  const size_t hwords = 1 + 3 * 64;
  unsigned long long* h = nullptr;  // pinned: the copy below is part of the iteration's graph
  LM_TRY(ctx_pinned(c, sizeof(unsigned long long) * hwords, reinterpret_cast<void**>(&h)));
  int it = 0;
  double worst = 0.0, prev = 1e300;
  int flat = 0;  // consecutive steps without progress
  for (it = 1; it <= max_iter; ++it) {
    // one correction step as a fixed launch sequence (captured and replayed
    // by the runner), ending with the norms copied to the host
    LM_TRY(run("iter", [&](cudaStream_t s) {
      LM_TRY(convert_d2s(D, ldr, R, ldr, n, nrhs, s));
      if (np > n) LM_CUDA_TRY(cudaMemsetAsync(D + (size_t)n * ldr, 0, sizeof(float) * (size_t)(np - n) * ldr, s));
      LM_TRY(correct(D, s));
      add_s2d_kernel<<<grid_of((long long)n * nrhs), 256, 0, s>>>(X, ldx, D, ldr, n, nrhs);
      count_launch(1);
      LM_TRY(dresidual(c, n, nrhs, A, lda, X, ldx, B, ldb, R, ldr, s));
      LM_CUDA_TRY(cudaMemsetAsync(nrm + 1 + 64, 0, sizeof(unsigned long long) * 128, s));
      colmax_abs_kernel<<<grid_of((long long)n * nrhs), 256, 0, s>>>(R, ldr, n, nrhs, nrm + 1 + 64);
      colmax_abs_kernel<<<grid_of((long long)n * nrhs), 256, 0, s>>>(X, ldx, n, nrhs, nrm + 1 + 128);
      count_launch(2);
      LM_CUDA_TRY(cudaMemcpyAsync(h, nrm, sizeof(unsigned long long) * hwords, cudaMemcpyDeviceToHost, s));
      return LM_OK;
    }));
    LM_CUDA_TRY(cudaStreamSynchronize(st));
    auto dbl = [](unsigned long long u) {
      double d;
      std::memcpy(&d, &u, sizeof d);
      return d;
    };
    const double anorm = dbl(h[0]);
    worst = 0.0;
    for (int col = 0; col < nrhs; ++col) {
      const double rn = dbl(h[1 + 64 + col]), xn = dbl(h[1 + 128 + col]), bn = dbl(h[1 + col]);
      const double den = anorm * xn + bn;
      const double be = den > 0 ? rn / den : (rn > 0 ? 1.0 : 0.0);
      worst = std::max(worst, (be != be) ? 1e300 : be);
    }
    ctx_ir_history(c).push_back(worst);
    if (worst <= tol) break;
    if (stall_exit && it >= 2) {
      // give up after two steps in a row without progress, or when the
      // observed contraction cannot reach tol within max_iter
      const double rate = worst / prev;
      flat = rate < 1.0 ? 0 : flat + 1;
      if (flat >= 2 || !(worst == worst)) break;
      if (rate < 1.0 && rate > 0.5 && it + std::log(tol / worst) / std::log(rate) > max_iter) break;
    }
    prev = worst;
  }
  if (iters_out) *iters_out = std::min(it, max_iter);
  if (berr_out) *berr_out = worst;
  return worst <= tol ? LM_OK : LM_ERR_NOT_CONVERGED;
}

// ||A||_inf and ||B_c||_inf (FP64, from the original data) into nrm.
int input_norms(int n, int nrhs, const double* A, long long lda, const double* B, long long ldb,
                unsigned long long* nrm, size_t nrm_bytes, cudaStream_t st) {
  LM_CUDA_TRY(cudaMemsetAsync(nrm, 0, nrm_bytes, st));
  norm_inf_rows_kernel<<<cdiv(n, 8), 256, 0, st>>>(A, lda, n, nrm);
  colmax_abs_kernel<<<grid_of((long long)n * nrhs), 256, 0, st>>>(B, ldb, n, nrhs, nrm + 1);
  count_launch(2);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

}  // namespace

// Iterative refinement driver.  A, B, X are FP64 device buffers; X receives
// the solution.  Returns info (> 0 if the FP32 factor hit a zero pivot),
// LM_ERR_NOT_CONVERGED if some column misses tol after max_iter steps.
int dgesv_ir(Ctx& c, int n, int nrhs, const double* A, long long lda, const double* B, long long ldb, double* X,
             long long ldx, double tol, int max_iter, int* iters_out, double* berr_out, cudaStream_t st,
             const IrRunner& run) {
  const long long lda32 = (n + 31) / 32 * 32;
  const long long ldr = (nrhs + 7) / 8 * 8;
  const size_t a32_bytes = sizeof(float) * (size_t)n * lda32;
  const size_t piv_bytes = sizeof(int) * (size_t)((n + 63) / 64 * 64);
  const size_t r_bytes = sizeof(double) * (size_t)n * ldr;
  const size_t d_bytes = sizeof(float) * (size_t)n * ldr;
  const size_t nrm_bytes = sizeof(unsigned long long) * (size_t)(2 + 3 * 64);  // 16-byte multiple
  const size_t sync_bytes = 64;
  const size_t w_bytes = sizeof(float) * (size_t)n * ldr;  // gather scratch of the interchanges
  void* ws = nullptr;
  LM_TRY(ctx_workspace(c, 0, a32_bytes + piv_bytes + r_bytes + d_bytes + nrm_bytes + sync_bytes + w_bytes, &ws));
  char* p = static_cast<char*>(ws);
  float* A32 = reinterpret_cast<float*>(p);
  int* ipiv = reinterpret_cast<int*>(p + a32_bytes);
  double* R = reinterpret_cast<double*>(p + a32_bytes + piv_bytes);
  float* D = reinterpret_cast<float*>(p + a32_bytes + piv_bytes + r_bytes);
  unsigned long long* nrm = reinterpret_cast<unsigned long long*>(p + a32_bytes + piv_bytes + r_bytes + d_bytes);
  int* tsync = reinterpret_cast<int*>(p + a32_bytes + piv_bytes + r_bytes + d_bytes + nrm_bytes);
  float* Wg = reinterpret_cast<float*>(p + a32_bytes + piv_bytes + r_bytes + d_bytes + nrm_bytes + sync_bytes);
  if (nrhs > 64) return LM_ERR_UNSUPPORTED;

  LM_TRY(input_norms(n, nrhs, A, lda, B, ldb, nrm, nrm_bytes, st));
  // factor fl32(A)
  LM_TRY(run("factor", [&](cudaStream_t s) {
    LM_TRY(convert_d2s(A32, lda32, A, lda, n, n, s));
    return sgetrf(c, n, A32, lda32, ipiv, s);
  }));
  return refine(c, n, n, nrhs, A, lda, B, ldb, X, ldx, tol, max_iter, false, R, ldr, D, nrm, iters_out, berr_out, st, run,
                [&](float* Dd, cudaStream_t s) {
                  {
                    Prof pp(c, kPhaseSwap, 0.0, 16.0 * n * nrhs, s);
                    LM_TRY(laswp_narrow<float>(Dd, ldr, n, nrhs, ipiv, Wg, ctx_status(c), s));
                  }
                  // diagonal blocks by substitution: with partial pivoting U's
                  // blocks carry the small pivots of an ill-conditioned A, and a
                  // product with their inverse would not be backward stable
                  Prof pt(c, kPhaseTrsm, 2.0 * n * n * nrhs, 4.0 * n * n, s);
                  return trsv_lu<float>(A32, lda32, n, nrhs, nullptr, nullptr, Dd, ldr, tsync, ctx_status(c), s,
                                        nullptr, true);
                });
}

// LU without pivoting of the FP32 matrix A (n x n, lda), right-looking in
// super-steps of two 128-column blocks a and b, so that the trailing update
// is one k = 256 GEMM: it reads and writes A22 once per 256 columns, which
// halves the HBM traffic that bounds it.  Everything but the 128 x 128
// diagonal blocks runs on the tensor cores (3xTF32):
//   a: diagonal block (nopiv_diag: LU in one CTA, then the FP64 inverses);
//      L_a = A[below a, a] inv(U_aa),  U_a = inv(L_aa) A[a, right of a],
//      each with one correction step (X += (B - X U) inv(U)), for n > 4096, when the
//      diagonal factor's 1-norm condition number exceeds kRefineCond: without
//      pivoting a few diagonal blocks are ill-conditioned, and a plain product
//      with their explicit inverse loses accuracy by that condition (the
//      diagonal kernel sets the per-block flags; a switched-off correction
//      adds zero);
//      block b's column and row panels -= L_a U_a (k = 128);
//   b: diagonal block, L_b and U_b likewise;
//   A22 -= [L_a L_b] [U_a; U_b]  (k = 256).
// Look-ahead: each diagonal block is factored on the priority stream, on the
// two SMs that the concurrent GEMMs leave free (146 of 148 CTAs; the LU takes
// one, the two triangle inversions one each): block b beside
// the rest of its panels' update, the next super-step's block a beside the
// trailing update.  DinvL / DinvU receive the diagonal-block inverses in the
// layout of the persistent substitutions, rflag (2 ints per 128-column block:
// L, U) the ill-conditioning flags that the substitutions' correction step
// follows too.  A zero pivot is recorded in status[1].
constexpr int kBlockCorrMinN = 4096;

int sgetrf_nopiv(Ctx& c, int n, float* A, long long lda, float* DinvL, float* DinvU, int* rflag, cudaStream_t st) {
  constexpr int SW = 2 * kNB;  // super-step width
  const size_t blk = (size_t)kNB * kNB;
  const long long ldk = SW;     // K-major operands of the k = 256 update
  void* ws = nullptr;
  const long long ldr = (n + 3) / 4 * 4;  // rows of the transposed residual
  LM_TRY(ctx_workspace(c, 1,
                       sizeof(float) * (4 * (size_t)n * SW + 5 * (size_t)n * kNB + 16 * blk + 2 * (size_t)kNB * ldr),
                       &ws));
  float* Ahi = static_cast<float*>(ws);  // [L_a | L_b] split, n x 256 (row i <-> row k0 + wa + i)
  float* Alo = Ahi + (size_t)n * SW;
  float* Bhi = Alo + (size_t)n * SW;     // [U_a | U_b]^T split, n x 256 (row j <-> column k0 + wa + j)
  float* Blo = Bhi + (size_t)n * SW;
  float* Thi = Blo + (size_t)n * SW;     // operands of the inverse products, n x 128
  float* Tlo = Thi + (size_t)n * kNB;
  float* Xhi = Tlo + (size_t)n * kNB;    // split first products, n x 128
  float* Xlo = Xhi + (size_t)n * kNB;
  float* Rb = Xlo + (size_t)n * kNB;     // residual of L_a (n x 128)
  // two sets of diagonal-block operands (split inverses, then split factors):
  // the look-ahead factors the next block while this one's are still read
  float* inv[2][8];
  for (int q2 = 0; q2 < 2; ++q2)
    for (int q = 0; q < 8; ++q) inv[q2][q] = Rb + (size_t)n * kNB + (size_t)(8 * q2 + q) * blk;
  float* Rt = inv[1][7] + blk;           // residual of U_a (128 x ldr)
  cudaStream_t aux;
  cudaEvent_t ev_fork, ev_join;
  LM_TRY(ctx_aux(c, &aux, &ev_fork, &ev_join));
  const int nsm = ctx_num_sms(c);
  auto diag = [&](int k0, cudaStream_t ds) {
    const int w = std::min(kNB, n - k0);
    float** d = inv[(k0 / kNB) & 1];
    Prof p(c, kPhasePanel, 2.0 / 3.0 * w * w * w, 8.0 * w * w, ds);
    return nopiv_diag(A + (long long)k0 * lda + k0, lda, w, k0, d[0], d[1], d[2], d[3], kNB,
                      DinvL + (size_t)(k0 / kNB) * blk, DinvU + (size_t)(k0 / kNB) * blk, d[4], d[5], d[6], d[7],
                      rflag + 2 * (k0 / kNB), ctx_status(c), ds);
  };
  auto split_rows = [&](float* hi, float* lo, long long ldd, const float* src, int rows, int cols, cudaStream_t ss,
                        long long lds = 0, const int* gate = nullptr, float* cpy = nullptr, long long ldc = 0) {
    split_kernel<<<grid_of((long long)rows * cols), 256, 0, ss>>>(hi, lo, ldd, src, lds ? lds : lda, rows, cols,
                                                                  gate, cpy, ldc);
    count_launch(1);
    LM_CUDA_TRY(cudaGetLastError());
    return LM_OK;
  };
  auto split_cols = [&](float* hi, float* lo, long long ldd, const float* src, int rows, int cols, cudaStream_t ss,
                        long long lds = 0, const int* gate = nullptr, float* cpy = nullptr, long long ldc = 0) {
    dim3 tb(32, 8), tg(cdiv(cols, 32), cdiv(rows, 32));
    transpose_split_kernel<<<tg, tb, 0, ss>>>(hi, lo, ldd, src, lds ? lds : lda, rows, cols, gate, cpy, ldc);
    count_launch(1);
    LM_CUDA_TRY(cudaGetLastError());
    return LM_OK;
  };
  // Block at k0 (w wide, diagonal block factored): L = A[k0+w:, k0:k0+w] inv(U)
  // and U = inv(L) A[k0:k0+w, k0+w:] in place, m = n - k0 - w; then their
  // splits into column `col` of the k = 256 operands, rows from `row0`.
  // Below this order the first-step errors of the uncorrected factor stay
  // small (5e-5 at n = 4096 for kappa = 1e2), and the correction chain's five
  // launches per block part, switched off or not, cost more than they save.
  const bool block_corr = n > kBlockCorrMinN;
  auto block_solves = [&](int k0, int w, int m, float* ahi, float* alo, float* bhi, float* blo) {
    float** d = inv[(k0 / kNB) & 1];
    float* A11 = A + (long long)k0 * lda + k0;
    float* A21 = A11 + (long long)w * lda;
    float* A12 = A11 + w;
    // L = B inv(U): X0 = B inv(U), R = B - X0 U, X = X0 + R inv(U); the
    // correction (all launches after the first product) runs only when the
    // diagonal kernel flagged U11 as ill-conditioned (gl), and likewise for
    // U with L11 (gu)
    const int* gu = rflag + 2 * (k0 / kNB);
    const int* gl = gu + 1;
    {
      Prof p(c, kPhaseTrsm, 2.0 * m * w * w, 8.0 * m * w, st);
      LM_TRY(split_rows(Thi, Tlo, kNB, A21, m, w, st, 0, nullptr, block_corr ? Rb : nullptr, kNB));
    }
    LM_TRY(sgemm_tf32(c, m, w, w, 1.0f, Thi, kNB, d[2], kNB, 0.0f, A21, lda, st, Tlo, d[3]));
    if (block_corr) {
      LM_TRY(split_rows(Xhi, Xlo, kNB, A21, m, w, st, 0, gl));
      LM_TRY(sgemm_tf32(c, m, w, w, -1.0f, Xhi, kNB, d[6], kNB, 1.0f, Rb, kNB, st, Xlo, d[7], 0, gl));
      LM_TRY(split_rows(Thi, Tlo, kNB, Rb, m, w, st, kNB, gl));
      LM_TRY(sgemm_tf32(c, m, w, w, 1.0f, Thi, kNB, d[2], kNB, 1.0f, A21, lda, st, Tlo, d[3], 0, gl));
    }
    // U = inv(L) B likewise, with B^T as the K-major operand
    {
      Prof p(c, kPhaseTrsm, 2.0 * m * w * w, 8.0 * m * w, st);
      LM_TRY(split_cols(Thi, Tlo, kNB, A12, w, m, st, 0, nullptr, block_corr ? Rt : nullptr, ldr));
    }
    LM_TRY(sgemm_tf32(c, w, m, w, 1.0f, d[0], kNB, Thi, kNB, 0.0f, A12, lda, st, d[1], Tlo));
    if (block_corr) {
      LM_TRY(split_cols(Xhi, Xlo, kNB, A12, w, m, st, 0, gu));
      LM_TRY(sgemm_tf32(c, w, m, w, -1.0f, d[4], kNB, Xhi, kNB, 1.0f, Rt, ldr, st, d[5], Xlo, 0, gu));
      LM_TRY(split_cols(Thi, Tlo, kNB, Rt, w, m, st, ldr, gu));
      LM_TRY(sgemm_tf32(c, w, m, w, 1.0f, d[0], kNB, Thi, kNB, 1.0f, A12, lda, st, d[1], Tlo, 0, gu));
    }
    LM_TRY(split_rows(ahi, alo, ldk, A21, m, w, st));
    return split_cols(bhi, blo, ldk, A12, w, m, st);
  };
  LM_TRY(diag(0, st));
  for (int k0 = 0; k0 < n; k0 += SW) {
    const int wa = std::min(kNB, n - k0);
    const int ma = n - k0 - wa;  // rows below / columns right of block a
    if (ma <= 0) break;
    const int wb = std::min(kNB, ma);
    const int mb = ma - wb;      // rows below / columns right of block b
    // ---- block a ----
    LM_TRY(block_solves(k0, wa, ma, Ahi, Alo, Bhi, Blo));
    float* Abb = A + (long long)(k0 + wa) * lda + k0 + wa;
    // b's diagonal block first, then its factorisation beside the rest of b's panels
    LM_TRY(sgemm_tf32(c, wb, wb, wa, -1.0f, Ahi, ldk, Bhi, ldk, 1.0f, Abb, lda, st, Alo, Blo));
    LM_CUDA_TRY(cudaEventRecord(ev_fork, st));
    LM_CUDA_TRY(cudaStreamWaitEvent(aux, ev_fork, 0));
    LM_TRY(diag(k0 + wa, aux));
    LM_CUDA_TRY(cudaEventRecord(ev_join, aux));
    if (mb > 0) {
      // column panel of b below its diagonal block, row panel of b right of it
      LM_TRY(sgemm_tf32(c, mb, wb, wa, -1.0f, Ahi + (size_t)wb * ldk, ldk, Bhi, ldk, 1.0f, Abb + (long long)wb * lda, lda,
                        st, Alo + (size_t)wb * ldk, Blo, nsm - 2));
      LM_TRY(sgemm_tf32(c, wb, mb, wa, -1.0f, Ahi, ldk, Bhi + (size_t)wb * ldk, ldk, 1.0f, Abb + wb, lda, st, Alo,
                        Blo + (size_t)wb * ldk, nsm - 2));
    }
    LM_CUDA_TRY(cudaStreamWaitEvent(st, ev_join, 0));
    if (mb <= 0) break;
    // ---- block b ----  (its splits go to column 128 of the operands, rows from wb)
    LM_TRY(block_solves(k0 + wa, wb, mb, Ahi + (size_t)wb * ldk + kNB, Alo + (size_t)wb * ldk + kNB,
                        Bhi + (size_t)wb * ldk + kNB, Blo + (size_t)wb * ldk + kNB));
    // ---- trailing update, k = wa + wb ----
    const int kk = wa + wb;
    const float* ah = Ahi + (size_t)wb * ldk;
    const float* al = Alo + (size_t)wb * ldk;
    const float* bh = Bhi + (size_t)wb * ldk;
    const float* bl = Blo + (size_t)wb * ldk;
    float* A22 = Abb + (long long)wb * lda + wb;
    const int w2 = std::min(kNB, mb);
    LM_TRY(sgemm_tf32(c, w2, w2, kk, -1.0f, ah, ldk, bh, ldk, 1.0f, A22, lda, st, al, bl));
    LM_CUDA_TRY(cudaEventRecord(ev_fork, st));
    LM_CUDA_TRY(cudaStreamWaitEvent(aux, ev_fork, 0));
    LM_TRY(diag(k0 + kk, aux));
    LM_CUDA_TRY(cudaEventRecord(ev_join, aux));
    if (mb > w2) {
      LM_TRY(sgemm_tf32(c, w2, mb - w2, kk, -1.0f, ah, ldk, bh + (size_t)w2 * ldk, ldk, 1.0f, A22 + w2, lda, st, al,
                        bl + (size_t)w2 * ldk, nsm - 2));
      LM_TRY(sgemm_tf32(c, mb - w2, mb, kk, -1.0f, ah + (size_t)w2 * ldk, ldk, bh, ldk, 1.0f, A22 + (long long)w2 * lda,
                        lda, st, al + (size_t)w2 * ldk, bl, nsm - 2));
    }
    LM_CUDA_TRY(cudaStreamWaitEvent(st, ev_join, 0));
  }
  return LM_OK;
}

// Randomised mixed-precision solve: Ar = fl32(U^T A V) with depth-2 random
// butterflies U, V (rbt.cu), Ar = L U without pivoting (sgetrf_nopiv), then
// FP64 refinement with the original A where each correction is
// V U^-1 L^-1 U^T fl32(r).  Returns LM_ERR_NOT_CONVERGED when the refinement
// stalls or runs out of steps; the caller then falls back to partial pivoting.
int dgesv_rbt_ir(Ctx& c, int n, int nrhs, const double* A, long long lda, const double* B, long long ldb, double* X,
                 long long ldx, double tol, int max_iter, int* iters_out, double* berr_out, cudaStream_t st,
                 const IrRunner& run) {
  if (nrhs > 64) return LM_ERR_UNSUPPORTED;
  const int np = (n + 3) / 4 * 4;
  const long long lda32 = (np + 31) / 32 * 32;
  const long long ldr = (nrhs + 7) / 8 * 8;
  const size_t a32_bytes = sizeof(float) * (size_t)np * lda32;
  const size_t r_bytes = sizeof(double) * (size_t)n * ldr;
  const size_t d_bytes = (sizeof(float) * (size_t)np * ldr + 15) / 16 * 16;
  const size_t nrm_bytes = sizeof(unsigned long long) * (size_t)(2 + 3 * 64);
  const size_t inv_elems = trsv_inv_elems<float>(np);
  const size_t inv_bytes = 2 * sizeof(float) * inv_elems;
  const size_t diag_bytes = 4 * sizeof(double) * (size_t)np;
  const size_t sync_bytes = 64;
  const size_t flag_bytes = sizeof(int) * 2 * (size_t)((np + 127) / 128);
  void* ws = nullptr;
  LM_TRY(ctx_workspace(c, 0, a32_bytes + r_bytes + d_bytes + nrm_bytes + inv_bytes + diag_bytes + sync_bytes + flag_bytes,
                       &ws));
  char* p = static_cast<char*>(ws);
  float* A32 = reinterpret_cast<float*>(p);
  p += a32_bytes;
  double* R = reinterpret_cast<double*>(p);
  p += r_bytes;
  float* D = reinterpret_cast<float*>(p);
  p += d_bytes;
  unsigned long long* nrm = reinterpret_cast<unsigned long long*>(p);
  p += nrm_bytes;
  float* DinvL = reinterpret_cast<float*>(p);
  float* DinvU = DinvL + inv_elems;
  p += inv_bytes;
  double* du = reinterpret_cast<double*>(p);
  double* dv = du + 2 * (size_t)np;
  p += diag_bytes;
  int* tsync = reinterpret_cast<int*>(p);
  p += sync_bytes;
  int* rflag = reinterpret_cast<int*>(p);
  LM_TRY(input_norms(n, nrhs, A, lda, B, ldb, nrm, nrm_bytes, st));
  LM_TRY(run("factor", [&](cudaStream_t s) {
    LM_TRY(rbt_diagonals(du, dv, np, s));
    LM_TRY(rbt_transform(A32, lda32, A, lda, n, np, du, dv, s));
    return sgetrf_nopiv(c, np, A32, lda32, DinvL, DinvU, rflag, s);
  }));
  return refine(c, n, np, nrhs, A, lda, B, ldb, X, ldx, tol, max_iter, true, R, ldr, D, nrm, iters_out, berr_out, st, run,
                [&](float* Dd, cudaStream_t s) {
                  LM_TRY(rbt_rows(Dd, ldr, np, nrhs, du, true, s));
                  {
                    Prof pt(c, kPhaseTrsm, 2.0 * np * np * nrhs, 4.0 * np * np, s);
                    LM_TRY(trsv_lu<float>(A32, lda32, np, nrhs, DinvL, DinvU, Dd, ldr, tsync, ctx_status(c), s,
                                          rflag));
                  }
                  return rbt_rows(Dd, ldr, np, nrhs, dv, false, s);
                });
}

}  // namespace lm
