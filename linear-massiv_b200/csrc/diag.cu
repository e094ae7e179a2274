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
constexpr int DLD = DB + 1;   // shared-memory leading dimension
constexpr int TLD = 64 + 1;   // scratch leading dimension

__device__ __forceinline__ void group_bar(int id, int nthreads) {
  if (id == 0)
    __syncthreads();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// One doubling level of the blocked inversion: for each 2H x 2H diagonal
// block p, X21 = -X22 (L21 X11), with tmp receiving L21 X11.  Thread t owns
// column j = t % H and the rows ig + 8 r (r < H / 8) of its block, so every
// k step loads one value of the right operand and H / 8 broadcast values of
// the left one for H / 8 independent accumulations.  Upper triangles of the
// diagonal blocks must hold zeros.
template <typename T, int H>
__device__ __forceinline__ void inv_combine(T* S, T* tmp, int t, int bar) {
  constexpr int R = H / 8;
  const int j = t % H, rest = t / H;
  const int p = rest / 8, ig = rest % 8;
  const int q0 = p * 2 * H;
  T acc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = T(0);
#pragma unroll 8
  for (int k = 0; k < H; ++k) {
    const T b = S[(q0 + k) * DLD + q0 + j];  // X11(k, j)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = fma(S[(q0 + H + ig + 8 * r) * DLD + q0 + k], b, acc[r]);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) tmp[(p * H + ig + 8 * r) * TLD + j] = acc[r];
  group_bar(bar, 512);
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = T(0);
#pragma unroll 8
  for (int k = 0; k < H; ++k) {
    const T b = tmp[(p * H + k) * TLD + j];  // (L21 X11)(k, j)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = fma(S[(q0 + H + ig + 8 * r) * DLD + q0 + H + k], b, acc[r]);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) S[(q0 + H + ig + 8 * r) * DLD + q0 + j] = -acc[r];
  group_bar(bar, 512);
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
  if (warp < (half ? 2 : 4)) {
    const int b0 = warp * 32, j = lane;
    T x[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      T acc = (i == j) ? T(1) : T(0);
#pragma unroll
      for (int k = 0; k < i; ++k) acc = fma(-S[(b0 + i) * DLD + b0 + k], x[k], acc);
      if (!unit) acc = acc / S[(b0 + i) * DLD + b0 + i];
      x[i] = (i < j) ? T(0) : acc;
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 32; ++i)
      if (i >= j) S[(b0 + i) * DLD + b0 + j] = x[i];
  }
  group_bar(bar, 512);
  inv_combine<T, 32>(S, tmp, t, bar);
  if (!half) inv_combine<T, 64>(S, tmp, t, bar);
}

__device__ __forceinline__ float tf32_hi_part(float a) { return __uint_as_float(__float_as_uint(a) & 0xFFFFE000u); }

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
    const int j = t % 64, ig = t / 64;
    for (int c0 = 0; c0 < ncols; c0 += 64) {
#pragma unroll 8
      for (int e = t; e < 64 * 64; e += 512) {
        const int r = e / 64, c = e % 64;
        tmp[r * TLD + c] = (r < w && c0 + c < ncols) ? B[(long long)r * ldb + c0 + c] : T(0);
      }
      __syncthreads();
      T acc[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) acc[r] = T(0);
#pragma unroll 8
      for (int k = 0; k < 64; ++k) {
        const T b = tmp[k * TLD + j];
#pragma unroll
        for (int r = 0; r < 8; ++r) acc[r] = fma(S[(ig + 8 * r) * DLD + k], b, acc[r]);
      }
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int i = ig + 8 * r;
        if (i < w && c0 + j < ncols) B[(long long)i * ldb + c0 + j] = acc[r];
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
        lo[(long long)i * ldx + j] = v - h;
        continue;
      }
    }
    Xout[(long long)i * ldx + j] = v;
  }
}

// LU without pivoting of the w x w block A11 (w <= 128) in place, then
//   Lhi/Llo   = split(inv(L11))        (w x w, ld ldi, zeros above the diagonal)
//   UThi/UTlo = split(inv(U11)^T)      (w x w, ld ldi, zeros above the diagonal)
//   DinvL / DinvU = inv(L11) / inv(U11) as DB x DB blocks padded with the
//                   identity (the layout of the persistent substitutions).
// The first zero or NaN pivot is recorded as base + k + 1 in status[1].
// 1024 threads: the factorisation uses all of them; then threads 0..511
// invert L and 512..1023 invert U^T concurrently (named barriers 1 and 2).
__global__ void __launch_bounds__(1024, 1)
    nopiv_diag_kernel(float* A11, long long lda, int w, int base, float* Lhi, float* Llo, float* UThi, float* UTlo,
                      long long ldi, float* DinvL, float* DinvU, int* status) {
  extern __shared__ __align__(16) unsigned char dsm[];
  float* S = reinterpret_cast<float*>(dsm);   // L \ U, then inv(L)
  float* S2 = S + DB * DLD;                    // U^T, then inv(U^T)
  float* tmp = S2 + DB * DLD;                  // 2 x 64 x TLD
  const int t = threadIdx.x;
  for (int e = t; e < DB * DB; e += 1024) {
    const int i = e / DB, j = e % DB;
    float v = 0.f;
    if (i < w && j < w)
      v = A11[(long long)i * lda + j];
    else if (i == j)
      v = 1.f;
    S[i * DLD + j] = v;
  }
  __syncthreads();
  for (int k = 0; k < w; ++k) {
    const float piv = S[k * DLD + k];
    if (t == 0 && (piv == 0.f || piv != piv)) atomicCAS(status + 1, 0, base + k + 1);
    const int m = DB - k - 1;
    for (int i = t; i < m; i += 1024) S[(k + 1 + i) * DLD + k] = S[(k + 1 + i) * DLD + k] / piv;
    __syncthreads();
    for (int e = t; e < m * m; e += 1024) {
      const int i = k + 1 + e / m, j = k + 1 + e % m;
      S[i * DLD + j] = fmaf(-S[i * DLD + k], S[k * DLD + j], S[i * DLD + j]);
    }
    __syncthreads();
  }
  for (int e = t; e < w * w; e += 1024) {
    const int i = e / w, j = e % w;
    A11[(long long)i * lda + j] = S[i * DLD + j];
  }
  // S2 = U^T (lower, with U's diagonal); then S keeps only L (zero upper)
  for (int e = t; e < DB * DB; e += 1024) {
    const int i = e / DB, j = e % DB;
    S2[i * DLD + j] = (j <= i) ? S[j * DLD + i] : 0.f;
  }
  __syncthreads();
  for (int e = t; e < DB * DB; e += 1024) {
    const int i = e / DB, j = e % DB;
    if (j > i) S[i * DLD + j] = 0.f;
  }
  __syncthreads();
  if (t < 512)
    inv_lower_smem<float>(S, tmp, true, false, t, 1);
  else
    inv_lower_smem<float>(S2, tmp + 64 * TLD, false, false, t - 512, 2);
  __syncthreads();
  for (int e = t; e < DB * DB; e += 1024) {
    const int i = e / DB, j = e % DB;
    const float li = (j <= i) ? S[i * DLD + j] : 0.f;    // inv(L)(i, j)
    const float ut = (j <= i) ? S2[i * DLD + j] : 0.f;   // inv(U)^T(i, j) = inv(U)(j, i)
    const float ui = (i <= j) ? S2[j * DLD + i] : 0.f;   // inv(U)(i, j)
    DinvL[e] = li;
    DinvU[e] = ui;
    if (i < w && j < w) {
      const float lh = tf32_hi_part(li), uh = tf32_hi_part(ut);
      Lhi[(long long)i * ldi + j] = lh;
      Llo[(long long)i * ldi + j] = li - lh;
      UThi[(long long)i * ldi + j] = uh;
      UTlo[(long long)i * ldi + j] = ut - uh;
    }
  }
}

template <typename T>
constexpr size_t inv_smem_bytes() {
  return sizeof(T) * ((size_t)DB * DLD + (size_t)64 * TLD);
}
constexpr size_t nopiv_smem_bytes() { return sizeof(float) * (2 * (size_t)DB * DLD + 2 * (size_t)64 * TLD); }

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
               long long ldi, float* DinvL, float* DinvU, int* status, cudaStream_t st) {
  if (w <= 0) return LM_OK;
  if (w > DB) return LM_ERR_ARG;
  static bool attr_set[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(nopiv_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)nopiv_smem_bytes()));
    attr_set[dev] = true;
  }
  nopiv_diag_kernel<<<1, 1024, nopiv_smem_bytes(), st>>>(A11, lda, w, base, Lhi, Llo, UThi, UTlo, ldi, DinvL, DinvU,
                                                         status);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

template int tri_inv_lower<double>(const double*, long long, int, bool, double*, long long, double*, cudaStream_t);
template int trsm_lower_small<double>(const double*, long long, int, bool, double*, long long, int, cudaStream_t);
template int trsm_lower_small<float>(const float*, long long, int, bool, float*, long long, int, cudaStream_t);
template int tri_inv_lower<float>(const float*, long long, int, bool, float*, long long, float*, cudaStream_t);

}  // namespace lm
