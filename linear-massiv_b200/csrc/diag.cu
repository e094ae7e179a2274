// Diagonal-block kernels of the blocked factorisations (blocks of order <= 128).
//
// tri_inv_lower  — inverse of a lower-triangular block (unit or not), so that
//   the block triangular solves of the factorisations become tensor-core
//   GEMMs:  U12 = inv(L11) A12  replaces the column-by-column substitution of
//   rawTriSolvePanelTrail (LU.hs:364-407) for the row block of every panel.
// nopiv_diag     — LU without pivoting of one diagonal block, both factors'
//   inverses (and inv(U)^T), for the randomised mixed-precision solver.
//
// Blocked inversion in shared memory (order 128, 512 threads):
//   1. four warps invert the four 32 x 32 diagonal blocks, lane j holding
//      column j of its block's inverse in registers (row sweep, the triangle
//      read as shared-memory broadcasts);
//   2. twice (h = 32, then 64) the 2h x 2h blocks are completed by
//      X21 = -X22 (L21 X11), two small matrix products per level.
// About 4 x 512 + 2 x 8 x 64 multiply-adds per thread instead of the 128
// dependent steps of a plain substitution sweep.
#include "common.cuh"
#include "internal.h"

namespace lm {

void count_launch(int n);

namespace {

constexpr int DB = 128;       // block order handled by one CTA
constexpr int DLD = DB + 4;   // shared-memory leading dimension (rows 16-byte aligned)
constexpr int TLD = 64 + 4;   // scratch leading dimension
// 1-norm condition number of a no-pivot diagonal factor beyond which the
// block solves that use its inverse take a correction step (measured: the
// correction helps ill-conditioned blocks and slightly hurts well-conditioned
// ones of graded matrices, so it is applied per block)
constexpr double kRefineCond = 1e4;

__device__ __forceinline__ void group_bar(int id, int nthreads) {
  if (id == 0)
    __syncthreads();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Four consecutive elements of a shared-memory row (16-byte aligned for
// FP32, 32 bytes as two 16-byte loads for FP64).
template <typename T>
__device__ __forceinline__ void lds4(T (&v)[4], const T* p) {
  if constexpr (sizeof(T) == 4) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
  } else {
    const double2 q0 = *reinterpret_cast<const double2*>(p);
    const double2 q1 = *reinterpret_cast<const double2*>(p + 2);
    v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
  }
}

// C (m x n) = C0 + sign * A (m x kdim) B (kdim x n), all row-major in shared
// memory, m and n multiples of 4 and every row start 16-byte aligned.
// 4 x 4 register tiles, nthreads threads from t = 0; consecutive threads take
// consecutive column tiles, so a warp reads A as broadcasts and B as
// contiguous 16-byte vectors (about half a shared-memory wavefront per FMA
// instruction instead of two).  With `acc_c` C0 = C, else C0 = 0.
template <typename T>
__device__ __forceinline__ void smem_mm4(T* C, int ldc, const T* A, int lda, const T* B, int ldb, int m, int n,
                                         int kdim, T sign, bool acc_c, int t, int nthreads) {
  const int tn = n / 4, tiles = (m / 4) * tn;
  for (int tt = t; tt < tiles; tt += nthreads) {
    const int r0 = (tt / tn) * 4, c0 = (tt % tn) * 4;
    T acc[4][4];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[p][q] = T(0);
#pragma unroll 4
    for (int k = 0; k < kdim; ++k) {
      T b[4];
      lds4<T>(b, B + k * ldb + c0);
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const T a = A[(r0 + p) * lda + k];
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = fma(a, b[q], acc[p][q]);
      }
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      T* cr = C + (r0 + p) * ldc + c0;
#pragma unroll
      for (int q = 0; q < 4; ++q) cr[q] = acc_c ? fma(sign, acc[p][q], cr[q]) : sign * acc[p][q];
    }
  }
}

// One doubling level of the blocked inversion: for each 2H x 2H diagonal
// block p, X21 = -X22 (L21 X11), with tmp receiving L21 X11 (register-tiled
// products).  Upper triangles of the diagonal blocks must hold zeros.
template <typename T, int H>
__device__ __forceinline__ void inv_combine(T* S, T* tmp, int t, int bar) {
  constexpr int NB = DB / (2 * H);
  constexpr int PER = 512 / NB;  // the blocks split the threads evenly
  const int p = t / PER, tl = t % PER;
  const int q0 = p * 2 * H;
  smem_mm4<T>(tmp + p * H * TLD, TLD, S + (q0 + H) * DLD + q0, DLD, S + q0 * DLD + q0, DLD, H, H, H, T(1), false, tl,
              PER);
  group_bar(bar, 512);
  smem_mm4<T>(S + (q0 + H) * DLD + q0, DLD, S + (q0 + H) * DLD + q0 + H, DLD, tmp + p * H * TLD, TLD, H, H, H, T(-1),
              false, tl, PER);
  group_bar(bar, 512);
}

// Inverse of the lower-triangular 32 x 32 block at blk (leading dimension
// DLD) in place, by one warp: lane j computes column j column-oriented (once
// x[k] is final it is applied to every later row at once).  Out of line so
// that x[] is register-allocated apart from the caller.
template <typename T>
__device__ __noinline__ void inv32_warp(T* blk, bool unit, int j) {
  T x[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) x[i] = (i == j) ? T(1) : T(0);
#pragma unroll 32
  for (int k = 0; k < 32; ++k) {
    if (!unit) x[k] = x[k] / blk[k * DLD + k];
#pragma unroll 32
    for (int i = k + 1; i < 32; ++i) x[i] = fma(-blk[i * DLD + k], x[k], x[i]);
  }
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 32; ++i)
    if (i >= j) blk[i * DLD + j] = x[i];
}

// In-place inverse of the lower triangle of S (DB x DB, leading dimension
// DLD): on exit S(i, j), j <= i, holds inv(L)(i, j) (1 on the diagonal when
// `unit`).  The strict upper triangle must hold zeros and keeps them; with
// `unit` the stored diagonal is ignored.  `tmp` holds 64 x TLD elements.
// When `half` is set only the leading 64 x 64 block is inverted (the rest of
// S must then be the identity).  Run by the 512 threads t = 0..511 of a group
// synchronised with barrier `bar` (0 = the whole CTA of 512 threads).
template <typename T>
__device__ void inv_lower_smem(T* S, T* tmp, bool unit, bool half, int t, int bar) {
  const int lane = t & 31, warp = t >> 5;
  if (warp < (half ? 2 : 4)) inv32_warp<T>(S + warp * 32 * DLD + warp * 32, unit, lane);
  group_bar(bar, 512);
  inv_combine<T, 32>(S, tmp, t, bar);
  if (!half) inv_combine<T, 64>(S, tmp, t, bar);
}

// High part of the 3xTF32 split: a rounded to the nearest TF32 value (ties
// away from zero), so that the remainder a - hi is exact in FP32 and at most
// 2^-11 |a|; the remainder is rounded the same way before it is stored, and
// the tensor core then reads both parts without further loss.
__device__ __forceinline__ float tf32_hi_part(float a) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(a));
  return __uint_as_float(r);
}

// Xout (w x w, ldx) <- inv(lower triangle of L) with zeros above the
// diagonal; for FP32 with `lo` given, Xout receives the TF32 high part and
// lo the remainder (3xTF32 operand split).
// Fused form (B given, w <= 64, ncols <= 128): B (w x ncols, ldb) <-
// inv(L) B in place and Xout is not written — the small block solves inside
// a panel in one launch.
template <typename T>
__global__ void __launch_bounds__(512, 1)
    tri_inv_lower_kernel(const T* __restrict__ L, long long ldl, int w, int unit, T* Xout, long long ldx, T* lo,
                         T* B, long long ldb, int ncols) {
  extern __shared__ __align__(16) unsigned char dsm[];
  T* S = reinterpret_cast<T*>(dsm);
  T* tmp = S + DB * DLD;
  const int t = threadIdx.x;
#pragma unroll 8
  for (int e = t; e < DB * DB; e += 512) {
    const int i = e / DB, j = e % DB;
    T v = T(0);
    if (i < w && j <= i) v = L[(long long)i * ldl + j];
    if (i == j && i >= w) v = T(1);
    S[i * DLD + j] = v;
  }
  __syncthreads();
  inv_lower_smem<T>(S, tmp, unit != 0, w <= 64, t, 0);
  if (B) {
    // X = inv(L) B, 64 columns at a time through tmp
    for (int c0 = 0; c0 < ncols; c0 += 64) {
#pragma unroll 8
      for (int e = t; e < 64 * 64; e += 512) {
        const int r = e / 64, c = e % 64;
        tmp[r * TLD + c] = (r < w && c0 + c < ncols) ? B[(long long)r * ldb + c0 + c] : T(0);
      }
      __syncthreads();
      // X = inv(L)[0:64, 0:64] tmp: 4 x 4 register tiles, written to B directly
      if (t < 256) {
        const int r0 = (t / 16) * 4, cq = (t % 16) * 4;
        T acc[4][4];
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[p][q] = T(0);
#pragma unroll 4
        for (int k = 0; k < 64; ++k) {
          T b[4];
          lds4<T>(b, tmp + k * TLD + cq);
#pragma unroll
          for (int p = 0; p < 4; ++p) {
            const T a = S[(r0 + p) * DLD + k];
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[p][q] = fma(a, b[q], acc[p][q]);
          }
        }
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (r0 + p < w && c0 + cq + q < ncols) B[(long long)(r0 + p) * ldb + c0 + cq + q] = acc[p][q];
      }
      __syncthreads();
    }
    return;
  }
#pragma unroll 4
  for (int e = t; e < w * w; e += 512) {
    const int i = e / w, j = e % w;
    const T v = (j <= i) ? S[i * DLD + j] : T(0);
    if constexpr (sizeof(T) == 4) {
      if (lo) {
        const float h = tf32_hi_part(v);
        Xout[(long long)i * ldx + j] = h;
        lo[(long long)i * ldx + j] = tf32_hi_part(v - h);
        continue;
      }
    }
    Xout[(long long)i * ldx + j] = v;
  }
}

// x U = row (U the upper triangle of the 32 x 32 block d, leading dimension
// DLD), in place on the row: column-oriented in registers.
__device__ __noinline__ void row_solve32(float* row, const float* d) {
  float x[32];
#pragma unroll
  for (int j = 0; j < 32; j += 4) {
    const float4 q = *reinterpret_cast<const float4*>(row + j);
    x[j] = q.x; x[j + 1] = q.y; x[j + 2] = q.z; x[j + 3] = q.w;
  }
#pragma unroll 32
  for (int j = 0; j < 32; ++j) {
    x[j] = x[j] / d[j * DLD + j];
#pragma unroll 32
    for (int jj = j + 1; jj < 32; ++jj) x[jj] = fmaf(-x[j], d[j * DLD + jj], x[jj]);
  }
#pragma unroll
  for (int j = 0; j < 32; j += 4) *reinterpret_cast<float4*>(row + j) = make_float4(x[j], x[j + 1], x[j + 2], x[j + 3]);
}

// L y = col (L the unit lower triangle of d), in place on a column of
// stride DLD: column-oriented in registers.
__device__ __noinline__ void col_solve32(float* col, const float* d) {
  float y[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) y[i] = col[i * DLD];
#pragma unroll 32
  for (int i = 0; i < 32; ++i) {
#pragma unroll 32
    for (int ii = i + 1; ii < 32; ++ii) y[ii] = fmaf(-d[ii * DLD + i], y[i], y[ii]);
  }
#pragma unroll
  for (int i = 1; i < 32; ++i) col[i * DLD] = y[i];
}

// LU without pivoting of a 32 x 32 block (leading dimension DLD) by one
// warp: lane i holds row i in registers, row k reaches the other lanes by
// shuffles.  Kept out of line so that its registers are allocated apart from
// the rest of the kernel.  The first zero or NaN pivot (global column
// base + o + k < base + w) is recorded in status[1].
__device__ __noinline__ void lu32_warp(float* blk, int o, int w, int base, int* status) {
  const int i = threadIdx.x & 31;
  float* ri = blk + i * DLD;
  float r[32];
#pragma unroll
  for (int j = 0; j < 32; j += 4) {
    const float4 q = *reinterpret_cast<const float4*>(ri + j);
    r[j] = q.x; r[j + 1] = q.y; r[j + 2] = q.z; r[j + 3] = q.w;
  }
#pragma unroll 32
  for (int k = 0; k < 32; ++k) {
    const float piv = __shfl_sync(0xffffffffu, r[k], k);
    if (i == 0 && o + k < w && (piv == 0.f || piv != piv)) atomicCAS(status + 1, 0, base + o + k + 1);
    __syncwarp();  // the rare branch above must not leave the warp split for the shuffles
    const float l = r[k] / piv;
    if (i > k) r[k] = l;
#pragma unroll 32
    for (int j = k + 1; j < 32; ++j) {
      const float u = __shfl_sync(0xffffffffu, r[j], k);
      if (i > k) r[j] = fmaf(-l, u, r[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < 32; j += 4) *reinterpret_cast<float4*>(ri + j) = make_float4(r[j], r[j + 1], r[j + 2], r[j + 3]);
}

// LU without pivoting of the w x w block A11 (w <= 128) in place, then
//   Lhi/Llo   = split(inv(L11))        (w x w, ld ldi, zeros above the diagonal)
//   UThi/UTlo = split(inv(U11)^T)      (w x w, ld ldi, zeros above the diagonal)
//   DinvL / DinvU = inv(L11) / inv(U11) as DB x DB blocks padded with the
//                   identity (the layout of the persistent substitutions).
// The first zero or NaN pivot is recorded as base + k + 1 in status[1].
// 512 threads; L and U^T are inverted one after the other.
__global__ void __launch_bounds__(512, 1)
    nopiv_diag_kernel(float* A11, long long lda, int w, int base, float* Lhi, float* Llo, float* UThi, float* UTlo,
                      long long ldi, float* DinvL, float* DinvU, float* LFhi, float* LFlo, float* UFThi,
                      float* UFTlo, int* status) {
  extern __shared__ __align__(16) unsigned char dsm[];
  float* S = reinterpret_cast<float*>(dsm);   // L \ U
  const int t = threadIdx.x;
#pragma unroll 8
  for (int e = t; e < DB * DB; e += 512) {
    const int i = e / DB, j = e % DB;
    float v = 0.f;
    if (i < w && j < w)
      v = A11[(long long)i * lda + j];
    else if (i == j)
      v = 1.f;
    S[i * DLD + j] = v;
  }
  __syncthreads();
  // Blocked right-looking LU in 32-column steps:
  //   (a) one warp factors the 32 x 32 diagonal block (lane i owns row i);
  //   (b) L10 = A10 U00^-1 row by row and U01 = L00^-1 A01 column by column,
  //       one thread per row / column;
  //   (c) A11 -= L10 U01 over the whole CTA.
  for (int kb = 0; kb < DB / 32; ++kb) {
    const int o = kb * 32;
    const int rem = DB - o - 32;
    if (t < 32) lu32_warp(S + o * DLD + o, o, w, base, status);
    __syncthreads();
    if (rem <= 0) break;
    // both solves column-oriented in registers: each finished unknown is
    // applied to all later ones at once (independent FMAs per step)
    if (t < rem)
      row_solve32(S + (o + 32 + t) * DLD + o, S + o * DLD + o);
    else if (t >= 256 && t < 256 + rem)
      col_solve32(S + o * DLD + o + 32 + (t - 256), S + o * DLD + o);
    __syncthreads();
    smem_mm4<float>(S + (o + 32) * DLD + o + 32, DLD, S + (o + 32) * DLD + o, DLD, S + o * DLD + o + 32, DLD, rem,
                    rem, 32, -1.f, true, t, 512);
    __syncthreads();
  }
  for (int e = t; e < w * w; e += 512) {
    const int i = e / w, j = e % w;
    A11[(long long)i * lda + j] = S[i * DLD + j];
  }
  // split factors themselves (unit L, U^T) for the refinement of the block solves
  for (int e = t; e < w * w; e += 512) {
    const int i = e / w, j = e % w;
    const float lf = (j < i) ? S[i * DLD + j] : (i == j ? 1.f : 0.f);
    const float uf = (j <= i) ? S[j * DLD + i] : 0.f;
    const float lh = tf32_hi_part(lf), uh = tf32_hi_part(uf);
    LFhi[(long long)i * ldi + j] = lh;
    LFlo[(long long)i * ldi + j] = tf32_hi_part(lf - lh);
    UFThi[(long long)i * ldi + j] = uh;
    UFTlo[(long long)i * ldi + j] = tf32_hi_part(uf - uh);
  }
}

// inv(L11) and inv(U11) of the FP32 factor just written to A11, computed in
// FP64 (one CTA per triangle, so the two run side by side) and rounded once:
// without pivoting the diagonal blocks can be ill-conditioned, and an inverse
// formed in FP32 would be too inaccurate for the correction steps of the
// block solves and substitutions that use it.  Outputs as nopiv_diag.
__global__ void __launch_bounds__(512, 1)
    nopiv_inv_kernel(const float* __restrict__ A11, long long lda, int w, float* Lhi, float* Llo, float* UThi,
                     float* UTlo, long long ldi, float* DinvL, float* DinvU, int* refine) {
  extern __shared__ __align__(16) unsigned char dsm[];
  double* S = reinterpret_cast<double*>(dsm);
  double* tmp = S + DB * DLD;
  __shared__ double colsum[DB];
  __shared__ double norm_f;
  const int t = threadIdx.x;
  // 1-norm (largest column sum) of the lower triangle held in S
  auto norm1 = [&]() {
    if (t < DB) {
      double sum = 0.0;
      for (int i = t; i < DB; ++i) sum += fabs(S[i * DLD + t]);
      colsum[t] = sum;
    }
    __syncthreads();
    if (t < 32) {
      double m = 0.0;
      for (int j = t; j < DB; j += 32) m = fmax(m, colsum[j]);
      __syncwarp();
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (t == 0) colsum[0] = m;
    }
    __syncthreads();
    const double r = colsum[0];
    __syncthreads();
    return r;
  };
  {
    // CTA 0: unit-lower L; CTA 1: U^T (lower, U's diagonal)
    const int pass = blockIdx.x;
#pragma unroll 8
    for (int e = t; e < DB * DB; e += 512) {
      const int i = e / DB, j = e % DB;
      double v = 0.0;
      if (i < w && j < w) {
        if (pass == 0)
          v = (j < i) ? (double)A11[(long long)i * lda + j] : (i == j ? 1.0 : 0.0);
        else
          v = (j <= i) ? (double)A11[(long long)j * lda + i] : 0.0;
      } else if (i == j) {
        v = 1.0;
      }
      S[i * DLD + j] = v;
    }
    __syncthreads();
    const double nf = norm1();
    if (t == 0) norm_f = nf;
    inv_lower_smem<double>(S, tmp, pass == 0, false, t, 0);
    __syncthreads();
    const double ni = norm1();
    // refine[0]: the products with inv(L) (U_a), refine[1]: with inv(U) (L_a)
    if (t == 0) refine[pass] = (norm_f * ni > kRefineCond || !(norm_f * ni == norm_f * ni)) ? 1 : 0;
    for (int e = t; e < DB * DB; e += 512) {
      const int i = e / DB, j = e % DB;
      if (pass == 0) {
        const float li = (j <= i) ? (float)S[i * DLD + j] : 0.f;  // inv(L)(i, j)
        DinvL[e] = li;
        if (i < w && j < w) {
          const float lh = tf32_hi_part(li);
          Lhi[(long long)i * ldi + j] = lh;
          Llo[(long long)i * ldi + j] = tf32_hi_part(li - lh);
        }
      } else {
        const float ut = (j <= i) ? (float)S[i * DLD + j] : 0.f;  // inv(U)^T(i, j)
        DinvU[e] = (i <= j) ? (float)S[j * DLD + i] : 0.f;        // inv(U)(i, j)
        if (i < w && j < w) {
          const float uh = tf32_hi_part(ut);
          UThi[(long long)i * ldi + j] = uh;
          UTlo[(long long)i * ldi + j] = tf32_hi_part(ut - uh);
        }
      }
    }
    __syncthreads();
  }
}

template <typename T>
constexpr size_t inv_smem_bytes() {
  return sizeof(T) * ((size_t)DB * DLD + (size_t)64 * TLD);
}
constexpr size_t nopiv_smem_bytes() { return sizeof(float) * (size_t)DB * DLD; }

}  // namespace

template <typename T>
int tri_inv_lower(const T* L, long long ldl, int w, bool unit, T* Xout, long long ldx, T* lo, cudaStream_t st) {
  if (w <= 0) return LM_OK;
  if (w > DB) return LM_ERR_ARG;
  static bool attr_set[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(tri_inv_lower_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)inv_smem_bytes<T>()));
    attr_set[dev] = true;
  }
  tri_inv_lower_kernel<T><<<1, 512, inv_smem_bytes<T>(), st>>>(L, ldl, w, unit ? 1 : 0, Xout, ldx, lo, nullptr, 0,
                                                                 0);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

template <typename T>
int trsm_lower_small(const T* L, long long ldl, int w, bool unit, T* B, long long ldb, int ncols, cudaStream_t st) {
  if (w <= 0 || ncols <= 0) return LM_OK;
  if (w > 64 || ncols > 128) return LM_ERR_ARG;
  static bool attr_set[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(tri_inv_lower_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)inv_smem_bytes<T>()));
    attr_set[dev] = true;
  }
  tri_inv_lower_kernel<T><<<1, 512, inv_smem_bytes<T>(), st>>>(L, ldl, w, unit ? 1 : 0, nullptr, 0, nullptr, B, ldb,
                                                                 ncols);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

int nopiv_diag(float* A11, long long lda, int w, int base, float* Lhi, float* Llo, float* UThi, float* UTlo,
               long long ldi, float* DinvL, float* DinvU, float* LFhi, float* LFlo, float* UFThi, float* UFTlo,
               int* refine, int* status, cudaStream_t st) {
  if (w <= 0) return LM_OK;
  if (w > DB) return LM_ERR_ARG;
  static bool attr_set[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(nopiv_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)nopiv_smem_bytes()));
    LM_CUDA_TRY(cudaFuncSetAttribute(nopiv_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)inv_smem_bytes<double>()));
    attr_set[dev] = true;
  }
  nopiv_diag_kernel<<<1, 512, nopiv_smem_bytes(), st>>>(A11, lda, w, base, Lhi, Llo, UThi, UTlo, ldi, DinvL, DinvU,
                                                         LFhi, LFlo, UFThi, UFTlo, status);
  nopiv_inv_kernel<<<2, 512, inv_smem_bytes<double>(), st>>>(A11, lda, w, Lhi, Llo, UThi, UTlo, ldi, DinvL, DinvU,
                                                             refine);
  count_launch(2);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

template int tri_inv_lower<double>(const double*, long long, int, bool, double*, long long, double*, cudaStream_t);
template int trsm_lower_small<double>(const double*, long long, int, bool, double*, long long, int, cudaStream_t);
template int trsm_lower_small<float>(const float*, long long, int, bool, float*, long long, int, cudaStream_t);
template int tri_inv_lower<float>(const float*, long long, int, bool, float*, long long, float*, cudaStream_t);

}  // namespace lm
