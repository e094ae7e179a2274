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

#include <cuda_bf16.h>

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
// The same with BF16 operands (kind::f16), FP32 C and accumulation.
int sgemm_bf16(Ctx& ctx, int m, int n, int k, float alpha, const void* A, long long lda, const void* Bt,
               long long ldb, float beta, float* C, long long ldc, cudaStream_t st, int max_ctas = 0);


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

// BF16 operands of the low-precision update: dst (rows x cols, ldd) =
// bf16(src), and the transposed form dst (cols x rows) = bf16(src)^T.
__global__ void to_bf16_kernel(__nv_bfloat16* dst, long long ldd, const float* src, long long lds, int rows,
                               int cols) {
  const long long total = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i % cols);
    dst[(long long)r * ldd + c] = __float2bfloat16_rn(src[(long long)r * lds + c]);
  }
}
__global__ void transpose_to_bf16_kernel(__nv_bfloat16* dst, long long ldd, const float* src, long long lds, int rows,
                                         int cols) {
  __shared__ float tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = by + j, c = bx + threadIdx.x;
    if (r < rows && c < cols) tile[j][threadIdx.x] = src[(long long)r * lds + c];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = bx + j, c = by + threadIdx.x;
    if (r < cols && c < rows) dst[(long long)r * ldd + c] = __float2bfloat16_rn(tile[threadIdx.x][j]);
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
    __syncwarp();
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
  __syncwarp();
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
             cudaStream_t st, int max_ctas = 0, int prec = LM_IR_PREC_TF32X3) {
  // C -= A21 (m x k) * U12 (k x n) on the tensor cores: 3xTF32, one TF32 or
  // one BF16 product per element
  dim3 tb(32, 8), tg(cdiv(n, 32), cdiv(k, 32));
  if (prec == LM_IR_PREC_BF16) {
    auto* ab = reinterpret_cast<__nv_bfloat16*>(s.Ahi);
    auto* bb = reinterpret_cast<__nv_bfloat16*>(s.Bhi);
    transpose_to_bf16_kernel<<<tg, tb, 0, st>>>(bb, s.ld, U12, lda, k, n);
    to_bf16_kernel<<<grid_of((long long)m * k), 256, 0, st>>>(ab, s.ld, A21, lda, m, k);
    count_launch(2);
    LM_CUDA_TRY(cudaGetLastError());
    return sgemm_bf16(c, m, n, k, -1.0f, ab, s.ld, bb, s.ld, 1.0f, C, lda, st, max_ctas);
  }
  if (prec == LM_IR_PREC_TF32) {
    transpose_split_kernel<<<tg, tb, 0, st>>>(s.Bhi, s.Blo, s.ld, U12, lda, k, n);
    split_kernel<<<grid_of((long long)m * k), 256, 0, st>>>(s.Ahi, s.Alo, s.ld, A21, lda, m, k);
    count_launch(2);
    LM_CUDA_TRY(cudaGetLastError());
    return sgemm_tf32(c, m, n, k, -1.0f, s.Ahi, s.ld, s.Bhi, s.ld, 1.0f, C, lda, st, nullptr, nullptr, max_ctas);
  }
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
// column panels factored by cluster leaves, U12 = inv(L11) A12 and the
// updates inside a panel as 3xTF32 on tcgen05; the trailing Schur-complement
// update, where the flops are, at `prec` (3xTF32, TF32 or BF16).  Look-ahead as in dgetrf:
// once the next panel's columns are updated, that panel is factored on the
// priority stream (its own GEMMs capped to the SMs left free) while the rest
// of the trailing update runs; its interchanges reach the columns right of it
// after the join.  The two streams use separate split-operand scratch.
int sgetrf(Ctx& c, int n, float* A, long long lda, int* ipiv, cudaStream_t st, int prec) {
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
    // A22 -= L21 U12 (at the factorisation's precision): the next panel's columns first
    LM_TRY(s_update(c, m, wn, w, A11 + (long long)w * lda, lda, A11 + w, A11 + (long long)w * lda + w, s, st, 0,
                    prec));
    const int rest = m - wn;
    if (la) {
      LM_CUDA_TRY(cudaEventRecord(ev_fork, st));
      LM_CUDA_TRY(cudaStreamWaitEvent(aux, ev_fork, 0));
      LM_TRY(sgetrf_panel_rec(c, A, lda, n, k0 + w, wn, k0 + w, wn, ipiv, sa, aux, kSLookaheadSms));
      LM_CUDA_TRY(cudaEventRecord(ev_join, aux));
      if (rest > 0)
        LM_TRY(s_update(c, m, rest, w, A11 + (long long)w * lda, lda, A11 + w + wn, A11 + (long long)w * lda + w + wn,
                        s, st, nsm - kSLookaheadSms, prec));
      LM_CUDA_TRY(cudaStreamWaitEvent(st, ev_join, 0));
    } else {
      if (rest > 0)
        LM_TRY(s_update(c, m, rest, w, A11 + (long long)w * lda, lda, A11 + w + wn, A11 + (long long)w * lda + w + wn,
                        s, st, 0, prec));
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

// Normwise backward error of one column from its norms: a NaN in the
// residual or in the solution (whose max-abs reductions return NaN) is never
// converged, and a zero denominator counts only an exact zero residual.
inline double backward_error(double rn, double xn, double den) {
  if (rn != rn || xn != xn || den != den) return 1e300;
  if (den > 0) return rn / den;
  return rn > 0 ? 1e300 : 0.0;
}

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
      const double be = backward_error(rn, xn, den);
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

// ---- GMRES-IR ------------------------------------------------------------------
// Correction equations A d = r solved by right-preconditioned flexible GMRES in
// FP64 (Carson and Higham's GMRES-IR), the preconditioner being the low-
// precision LU applied in FP32.  The columns of a multi-right-hand-side solve
// run in lockstep, each with its own Krylov basis and Hessenberg matrix; the
// Givens rotations and the small triangular solves run on the host.
constexpr int kGmresM = 30;             // inner steps per correction
constexpr double kGmresInnerTol = 1e-4; // relative residual of one correction
constexpr int kDotBlocks = 128;         // CTAs of the deterministic dot products

// partial[blk][p] = sum over this CTA's rows of V_i[r][c] W[r][c], p = i * nrhs + c
// (i < count), one thread per (i, c) pair, rows in a fixed order.
__global__ void gm_dots_kernel(int count, const double* V, long long vstride, const double* W, long long ldr, int n,
                               int nrhs, double* partial) {
  const int pairs = count * nrhs;
  const int rows_per = (n + gridDim.x - 1) / gridDim.x;
  const int r0 = blockIdx.x * rows_per, r1 = min(n, r0 + rows_per);
  for (int p = threadIdx.x; p < pairs; p += blockDim.x) {
    const int i = p / nrhs, c = p % nrhs;
    const double* v = V + (long long)i * vstride;
    double acc = 0.0;
    for (int r = r0; r < r1; ++r) acc = fma(v[(long long)r * ldr + c], W[(long long)r * ldr + c], acc);
    partial[(long long)blockIdx.x * pairs + p] = acc;
  }
}
__global__ void gm_reduce_kernel(const double* partial, int blocks, int pairs, double* out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < pairs; p += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int b = 0; b < blocks; ++b) acc += partial[(long long)b * pairs + p];
    out[p] = acc;
  }
}
// W[r][c] (ldw) = sw * W[r][c] + sum_i coef[i * nrhs + c] * V_i[r][c] (ldr), i < count.
__global__ void gm_combine_kernel(int count, const double* V, long long vstride, long long ldr, const double* coef,
                                  double sw, double* W, long long ldw, int n, int nrhs) {
  const long long total = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e / nrhs), c = (int)(e % nrhs);
    double acc = sw * W[(long long)r * ldw + c];
    for (int i = 0; i < count; ++i) acc = fma(coef[i * nrhs + c], V[(long long)i * vstride + (long long)r * ldr + c], acc);
    W[(long long)r * ldw + c] = acc;
  }
}
// Z (FP64) = D (FP32), n x nrhs, both with leading dimension ld.
__global__ void s2d_kernel(double* Z, const float* D, long long ld, int n, int nrhs) {
  const long long total = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long o = (e / nrhs) * ld + e % nrhs;
    Z[o] = (double)D[o];
  }
}

struct GmresBufs {
  double *V, *Z, *W, *zero, *partial, *dots, *coef;
  long long vstride;
  double* hdots;  // pinned host copy of dots
};

// Outer FP64 refinement with GMRES corrections.  R, D, nrm as in refine();
// precond(D) turns D (FP32, n x ldr) into M^-1 D.  Returns LM_OK when every
// column's normwise backward error is <= tol within max_iter corrections.
int refine_gmres(Ctx& c, int n, int nrhs, const double* A, long long lda, const double* B, long long ldb, double* X,
                 long long ldx, double tol, int max_iter, double* R, long long ldr, float* D, unsigned long long* nrm,
                 GmresBufs& g, int* iters_out, double* berr_out, cudaStream_t st,
                 const std::function<int(float*, cudaStream_t)>& precond) {
  const int M = kGmresM;
  const size_t hwords = 1 + 3 * 64;
  unsigned long long* h = nullptr;
  LM_TRY(ctx_pinned(c, sizeof(unsigned long long) * hwords + sizeof(double) * (size_t)(M + 1) * 64 * 2,
                    reinterpret_cast<void**>(&h)));
  double* hd = reinterpret_cast<double*>(h + hwords);       // dots from the device
  double* hc = hd + (size_t)(M + 1) * 64;                    // coefficients to the device
  auto dbl = [](unsigned long long u) {
    double d;
    std::memcpy(&d, &u, sizeof d);
    return d;
  };
  LM_CUDA_TRY(cudaMemset2DAsync(X, sizeof(double) * ldx, 0, sizeof(double) * nrhs, n, st));
  LM_TRY(copy2d<double>(R, ldr, B, ldb, n, nrhs, st));
  LM_CUDA_TRY(cudaMemsetAsync(g.zero, 0, sizeof(double) * (size_t)n * ldr, st));
  const int gr = grid_of((long long)n * nrhs);
  // per-column dot products of W with V_0 .. V_{count-1} into hd (synchronises)
  auto dots = [&](int count, const double* V, const double* W) -> int {
    gm_dots_kernel<<<kDotBlocks, 256, 0, st>>>(count, V, g.vstride, W, ldr, n, nrhs, g.partial);
    gm_reduce_kernel<<<cdiv(count * nrhs, 256), 256, 0, st>>>(g.partial, kDotBlocks, count * nrhs, g.dots);
    count_launch(2);
    LM_CUDA_TRY(cudaGetLastError());
    LM_CUDA_TRY(cudaMemcpyAsync(hd, g.dots, sizeof(double) * count * nrhs, cudaMemcpyDeviceToHost, st));
    LM_CUDA_TRY(cudaStreamSynchronize(st));
    return LM_OK;
  };
  // W = sw W + sum_i hc[i] V_i
  auto combine = [&](int count, const double* V, double sw, double* W, long long ldw) -> int {
    LM_CUDA_TRY(cudaMemcpyAsync(g.coef, hc, sizeof(double) * count * nrhs, cudaMemcpyHostToDevice, st));
    gm_combine_kernel<<<gr, 256, 0, st>>>(count, V, g.vstride, ldr, g.coef, sw, W, ldw, n, nrhs);
    count_launch(1);
    LM_CUDA_TRY(cudaGetLastError());
    return LM_OK;
  };
  std::vector<double> H((size_t)nrhs * (M + 1) * M), cs((size_t)nrhs * M), sn((size_t)nrhs * M),
      gv((size_t)nrhs * (M + 1)), beta(nrhs), y((size_t)nrhs * M);
  double worst = 0.0;
  int it = 0;
  for (it = 1; it <= max_iter; ++it) {
    // ---- one correction: d ~ A^-1 r by FGMRES(M) ----
    LM_TRY(copy2d<double>(g.V, ldr, R, ldr, n, nrhs, st));
    LM_TRY(dots(1, g.V, g.V));
    for (int col = 0; col < nrhs; ++col) {
      beta[col] = std::sqrt(std::max(hd[col], 0.0));
      hc[col] = beta[col] > 0 ? 1.0 / beta[col] : 0.0;
    }
    LM_TRY(combine(1, g.V, 0.0, g.V, ldr));  // V_0 = r / beta
    std::fill(H.begin(), H.end(), 0.0);
    std::fill(gv.begin(), gv.end(), 0.0);
    for (int col = 0; col < nrhs; ++col) gv[(size_t)col * (M + 1)] = beta[col];
    int k = 0;
    for (int j = 0; j < M; ++j) {
      double* Vj = g.V + (long long)j * g.vstride;
      double* Zj = g.Z + (long long)j * g.vstride;
      // z_j = M^-1 v_j in FP32
      LM_TRY(convert_d2s(D, ldr, Vj, ldr, n, nrhs, st));
      LM_TRY(precond(D, st));
      s2d_kernel<<<gr, 256, 0, st>>>(Zj, D, ldr, n, nrhs);
      count_launch(1);
      // w = A z_j (as -(0 - A z_j))
      LM_TRY(dresidual(c, n, nrhs, A, lda, Zj, ldr, g.zero, ldr, g.W, ldr, st));
      // classical Gram-Schmidt, twice: h = V^T w, w -= V h
      for (int pass = 0; pass < 2; ++pass) {
        LM_TRY(dots(j + 1, g.V, g.W));  // V^T (-w)
        for (int col = 0; col < nrhs; ++col)
          for (int i = 0; i <= j; ++i) {
            const double hij = -hd[i * nrhs + col];
            H[((size_t)col * (M + 1) + i) * M + j] += hij;
            hc[i * nrhs + col] = hij;  // w -= h v, i.e. W = -w gains + h v
          }
        LM_TRY(combine(j + 1, g.V, 1.0, g.W, ldr));  // W = -w + ... stays the negated vector
      }
      LM_TRY(dots(1, g.W, g.W));
      bool all_done = true;
      for (int col = 0; col < nrhs; ++col) {
        const double hn = std::sqrt(std::max(hd[col], 0.0));
        H[((size_t)col * (M + 1) + j + 1) * M + j] = hn;
        hc[col] = hn > 0 ? -1.0 / hn : 0.0;  // V_{j+1} = w / hn = -W / hn
        // Givens rotations of this column's Hessenberg
        double* Hcol = &H[(size_t)col * (M + 1) * M];
        for (int i = 0; i < j; ++i) {
          const double a = Hcol[i * M + j], b = Hcol[(i + 1) * M + j];
          Hcol[i * M + j] = cs[(size_t)col * M + i] * a + sn[(size_t)col * M + i] * b;
          Hcol[(i + 1) * M + j] = -sn[(size_t)col * M + i] * a + cs[(size_t)col * M + i] * b;
        }
        const double a = Hcol[j * M + j], b = Hcol[(j + 1) * M + j];
        const double rr = std::hypot(a, b);
        const double cc = rr > 0 ? a / rr : 1.0, ss = rr > 0 ? b / rr : 0.0;
        cs[(size_t)col * M + j] = cc;
        sn[(size_t)col * M + j] = ss;
        Hcol[j * M + j] = rr;
        Hcol[(j + 1) * M + j] = 0.0;
        double* gc = &gv[(size_t)col * (M + 1)];
        gc[j + 1] = -ss * gc[j];
        gc[j] = cc * gc[j];
        if (!(std::fabs(gc[j + 1]) <= kGmresInnerTol * beta[col]) && hn > 0) all_done = false;
      }
      k = j + 1;
      if (all_done || k == M) break;
      // V_{j+1} = -W / ||W||
      double* Vn = g.V + (long long)(j + 1) * g.vstride;
      LM_CUDA_TRY(cudaMemsetAsync(Vn, 0, sizeof(double) * (size_t)n * ldr, st));
      LM_CUDA_TRY(cudaMemcpyAsync(g.coef, hc, sizeof(double) * nrhs, cudaMemcpyHostToDevice, st));
      gm_combine_kernel<<<gr, 256, 0, st>>>(1, g.W, 0, ldr, g.coef, 0.0, Vn, ldr, n, nrhs);
      count_launch(1);
      LM_CUDA_TRY(cudaGetLastError());
    }
    // y = H^-1 g (k x k upper triangular per column), x += Z y
    for (int col = 0; col < nrhs; ++col) {
      const double* Hcol = &H[(size_t)col * (M + 1) * M];
      const double* gc = &gv[(size_t)col * (M + 1)];
      for (int i = k - 1; i >= 0; --i) {
        double v = gc[i];
        for (int l = i + 1; l < k; ++l) v -= Hcol[i * M + l] * y[(size_t)col * M + l];
        y[(size_t)col * M + i] = Hcol[i * M + i] != 0 ? v / Hcol[i * M + i] : 0.0;
      }
      for (int i = 0; i < k; ++i) hc[i * nrhs + col] = y[(size_t)col * M + i];
    }
    LM_TRY(combine(k, g.Z, 1.0, X, ldx));
    // ---- r = b - A x in FP64 and the stopping test ----
    LM_TRY(dresidual(c, n, nrhs, A, lda, X, ldx, B, ldb, R, ldr, st));
    LM_CUDA_TRY(cudaMemsetAsync(nrm + 1 + 64, 0, sizeof(unsigned long long) * 128, st));
    colmax_abs_kernel<<<grid_of((long long)n * nrhs), 256, 0, st>>>(R, ldr, n, nrhs, nrm + 1 + 64);
    colmax_abs_kernel<<<grid_of((long long)n * nrhs), 256, 0, st>>>(X, ldx, n, nrhs, nrm + 1 + 128);
    count_launch(2);
    LM_CUDA_TRY(cudaMemcpyAsync(h, nrm, sizeof(unsigned long long) * hwords, cudaMemcpyDeviceToHost, st));
    LM_CUDA_TRY(cudaStreamSynchronize(st));
    const double anorm = dbl(h[0]);
    worst = 0.0;
    for (int col = 0; col < nrhs; ++col) {
      const double rn = dbl(h[1 + 64 + col]), xn = dbl(h[1 + 128 + col]), bn = dbl(h[1 + col]);
      const double den = anorm * xn + bn;
      const double be = backward_error(rn, xn, den);
      worst = std::max(worst, (be != be) ? 1e300 : be);
    }
    ctx_ir_history(c).push_back(worst);
    if (worst <= tol) break;
  }
  if (iters_out) *iters_out = std::min(it, max_iter);
  if (berr_out) *berr_out = worst;
  return worst <= tol ? LM_OK : LM_ERR_NOT_CONVERGED;
}

}  // namespace

// Iterative refinement driver.  A, B, X are FP64 device buffers; X receives
// the solution.  Returns info (> 0 if the FP32 factor hit a zero pivot),
// LM_ERR_NOT_CONVERGED if some column misses tol after max_iter steps.
int dgesv_ir(Ctx& c, int n, int nrhs, const double* A, long long lda, const double* B, long long ldb, double* X,
             long long ldx, double tol, int max_iter, int* iters_out, double* berr_out, cudaStream_t st,
             const IrRunner& run, int prec) {
  const long long lda32 = (n + 31) / 32 * 32;
  const long long ldr = (nrhs + 7) / 8 * 8;
  const size_t a32_bytes = sizeof(float) * (size_t)n * lda32;
  const size_t piv_bytes = 2 * sizeof(int) * (size_t)((n + 63) / 64 * 64);  // ipiv, then its composed permutation
  const size_t r_bytes = sizeof(double) * (size_t)n * ldr;
  const size_t d_bytes = sizeof(float) * (size_t)n * ldr;
  const size_t nrm_bytes = sizeof(unsigned long long) * (size_t)(2 + 3 * 64);  // 16-byte multiple
  const size_t sync_bytes = 64;
  const size_t w_bytes = sizeof(float) * (size_t)n * ldr;  // gather scratch of the interchanges
  // GMRES-IR (low-precision factors): Krylov bases V (M + 1) and Z (M), W, a
  // zero block, dot-product partials and coefficients
  const bool gmres = prec != LM_IR_PREC_TF32X3;
  const long long vstride = (long long)n * ldr;
  const size_t gm_bytes =
      gmres ? sizeof(double) * ((size_t)(2 * kGmresM + 3) * vstride + (size_t)kDotBlocks * (kGmresM + 1) * 64 +
                                2 * (size_t)(kGmresM + 1) * 64)
            : 0;
  void* ws = nullptr;
  LM_TRY(ctx_workspace(c, 0, a32_bytes + piv_bytes + r_bytes + d_bytes + nrm_bytes + sync_bytes + w_bytes + gm_bytes,
                       &ws));
  char* p = static_cast<char*>(ws);
  float* A32 = reinterpret_cast<float*>(p);
  int* ipiv = reinterpret_cast<int*>(p + a32_bytes);
  int* perm = ipiv + (n + 63) / 64 * 64;
  double* R = reinterpret_cast<double*>(p + a32_bytes + piv_bytes);
  float* D = reinterpret_cast<float*>(p + a32_bytes + piv_bytes + r_bytes);
  unsigned long long* nrm = reinterpret_cast<unsigned long long*>(p + a32_bytes + piv_bytes + r_bytes + d_bytes);
  int* tsync = reinterpret_cast<int*>(p + a32_bytes + piv_bytes + r_bytes + d_bytes + nrm_bytes);
  float* Wg = reinterpret_cast<float*>(p + a32_bytes + piv_bytes + r_bytes + d_bytes + nrm_bytes + sync_bytes);
  if (nrhs > 64) return LM_ERR_UNSUPPORTED;
  GmresBufs gb{};
  if (gmres) {
    double* q = reinterpret_cast<double*>(p + a32_bytes + piv_bytes + r_bytes + d_bytes + nrm_bytes + sync_bytes +
                                          w_bytes);
    gb.vstride = vstride;
    gb.V = q;
    gb.Z = gb.V + (size_t)(kGmresM + 1) * vstride;
    gb.W = gb.Z + (size_t)kGmresM * vstride;
    gb.zero = gb.W + vstride;
    gb.partial = gb.zero + vstride;
    gb.dots = gb.partial + (size_t)kDotBlocks * (kGmresM + 1) * 64;
    gb.coef = gb.dots + (size_t)(kGmresM + 1) * 64;
  }

  LM_TRY(input_norms(n, nrhs, A, lda, B, ldb, nrm, nrm_bytes, st));
  // factor fl32(A)
  LM_TRY(run(gmres ? (prec == LM_IR_PREC_BF16 ? "factor_bf16" : "factor_tf32") : "factor", [&](cudaStream_t s) {
    LM_TRY(convert_d2s(A32, lda32, A, lda, n, n, s));
    LM_TRY(sgetrf(c, n, A32, lda32, ipiv, s, prec));
    // the interchanges composed once; every correction then gathers with them
    return perm_from_swaps(ipiv, n, perm, ctx_status(c), s);
  }));
  auto precond = [&](float* Dd, cudaStream_t s) {
    LM_TRY(laswp_perm<float>(Dd, ldr, n, nrhs, perm, Wg, s));
    return trsv_lu<float>(A32, lda32, n, nrhs, nullptr, nullptr, Dd, ldr, tsync, ctx_status(c), s, nullptr, true);
  };
  if (gmres)  // the host steers the Krylov steps: these run without graph capture
    return refine_gmres(c, n, nrhs, A, lda, B, ldb, X, ldx, tol, max_iter, R, ldr, D, nrm, gb, iters_out, berr_out,
                        st, precond);
  return refine(c, n, n, nrhs, A, lda, B, ldb, X, ldx, tol, max_iter, false, R, ldr, D, nrm, iters_out, berr_out, st, run,
                [&](float* Dd, cudaStream_t s) {
                  {
                    Prof pp(c, kPhaseSwap, 0.0, 16.0 * n * nrhs, s);
                    LM_TRY(laswp_perm<float>(Dd, ldr, n, nrhs, perm, Wg, s));
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
