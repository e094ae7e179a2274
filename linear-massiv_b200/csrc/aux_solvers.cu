// Kernels of the reference's adjacent entry points on the dense path:
//
//   gemv_exact_kernel     matvecP -> rawGemv (BLAS/Level2.hs:131-139,
//                         Internal/Kernel.hs:119-134), in the reference's own
//                         floating-point order, so results are bitwise equal:
//                         per row, four FMA accumulators over the columns
//                         j = 4s + l (j < n - n mod 4), combined as
//                         ((a0 + a1) + a2) + a3, then the remaining columns
//                         with a separately rounded multiply and add.
//   norm_inf_exact_kernel normInf (Norms.hs:135-141): each row's sum of |a_ij|
//                         as a left fold from 0 in column order (bitwise the
//                         reference's), the maximum over rows.
//   lu_nopiv_block_kernel luNoPivot (Solve/LU.hs:196-214) of one <= 128 x 128
//                         diagonal block, register resident.
//   pcr_step_kernel       tridiagSolve (Solve/Banded.hs:292-342) as parallel
//                         cyclic reduction: ceil(log2 n) steps of one thread
//                         per equation instead of the sequential LDL^T sweep.
#include <algorithm>

#include "common.cuh"
#include "internal.h"

namespace lm {

void count_launch(int n);

namespace {

constexpr unsigned kFull = 0xffffffffu;

__global__ void __launch_bounds__(256) gemv_exact_kernel(int m, int n, const double* __restrict__ A, long long lda,
                                                         const double* __restrict__ x, double* __restrict__ y) {
  const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long row = gt >> 2;
  const int l = threadIdx.x & 3;
  const bool ok = row < m;
  const double* ar = A + (ok ? row : 0) * lda;
  const int n4 = n - n % 4;
  double acc = 0.0;
#pragma unroll 8
  for (int j = l; j < n4; j += 4) acc = fma(ar[j], x[j], acc);
  __syncwarp();
  // lane 0 of the quad gathers the four accumulators in the reference's order
  const double a1 = __shfl_down_sync(kFull, acc, 1, 4);
  const double a2 = __shfl_down_sync(kFull, acc, 2, 4);
  const double a3 = __shfl_down_sync(kFull, acc, 3, 4);
  if (ok && l == 0) {
    double s = __dadd_rn(__dadd_rn(__dadd_rn(acc, a1), a2), a3);
    for (int j = n4; j < n; ++j) s = __dadd_rn(s, __dmul_rn(ar[j], x[j]));
    y[row] = s;
  }
}

// 32 rows per CTA; column chunks of 128 staged through shared memory so the
// loads are coalesced, each row then folded by one lane in column order.
constexpr int kNormRows = 32, kNormCols = 128;

__global__ void __launch_bounds__(256) norm_inf_exact_kernel(int m, int n, const double* __restrict__ A,
                                                             long long lda, unsigned long long* out) {
  __shared__ double tile[kNormRows][kNormCols + 1];
  const int r0 = blockIdx.x * kNormRows;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double acc = 0.0;
  for (int c0 = 0; c0 < n; c0 += kNormCols) {
#pragma unroll
    for (int rr = 0; rr < kNormRows / 8; ++rr) {
      const int r = warp * (kNormRows / 8) + rr;
#pragma unroll
      for (int q = 0; q < kNormCols / 32; ++q) {
        const int c = c0 + q * 32 + lane;
        tile[r][q * 32 + lane] = (r0 + r < m && c < n) ? A[(long long)(r0 + r) * lda + c] : 0.0;
      }
    }
    __syncthreads();
    if (warp == 0) {
      const int lim = min(kNormCols, n - c0);
      for (int c = 0; c < lim; ++c) acc = __dadd_rn(acc, fabs(tile[lane][c]));
    }
    __syncthreads();
  }
  if (warp == 0 && r0 + lane < m) atomicMax(out, (unsigned long long)__double_as_longlong(acc));
}

// luNoPivot of the w x w block at A (w <= 128) in place: thread (ty, tx) of a
// 16 x 32 grid holds elements (ty + 16 a, tx + 32 b), a < 8, b < 4, in
// registers.  Step k: the owners of row k publish it, the owners of column k
// form the multipliers a_ik / a_kk (as products with 1 / a_kk, within an ulp
// of the quotients), every thread subtracts l_ik * u_kj with a
// separately rounded product (the reference's `aij - aik * akj`).  Rows and
// columns past w are the identity.  The first zero pivot is recorded as
// base + k + 1 in status[1]; the division still runs, as in the reference.
__global__ void __launch_bounds__(512) lu_nopiv_block_kernel(double* A, long long lda, int w, int base, int* status) {
  __shared__ double urow[2][128];
  __shared__ double lcol[2][128];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  double v[8][4];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int i = ty + 16 * a, j = tx + 32 * b;
      v[a][b] = (i < w && j < w) ? A[(long long)i * lda + j] : (i == j ? 1.0 : 0.0);
    }
#pragma unroll 1
  for (int k = 0; k < w; ++k) {
    const int buf = k & 1;
    const int ak = k >> 4, bk = k >> 5;
    if (ty == (k & 15)) {
#pragma unroll
      for (int a = 0; a < 8; ++a)
        if (a == ak)
#pragma unroll
          for (int b = 0; b < 4; ++b) urow[buf][tx + 32 * b] = v[a][b];
    }
    __syncthreads();
    const double ukk = urow[buf][k];
    if (tx == (k & 31)) {
      if (ty == 0 && ukk == 0.0) atomicCAS(status + 1, 0, base + k + 1);
      const double rkk = 1.0 / ukk;  // one division per column: the multipliers are products with it
#pragma unroll
      for (int b = 0; b < 4; ++b)
        if (b == bk)
#pragma unroll
          for (int a = 0; a < 8; ++a) {
            const int i = ty + 16 * a;
            if (i > k) {
              const double lik = v[a][b] * rkk;
              v[a][b] = lik;
              lcol[buf][i] = lik;
            }
          }
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int i = ty + 16 * a;
      if (i > k) {
        const double lik = lcol[buf][i];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int j = tx + 32 * b;
          if (j > k) v[a][b] = __dsub_rn(v[a][b], __dmul_rn(lik, urow[buf][j]));
        }
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int i = ty + 16 * a, j = tx + 32 * b;
      if (i < w && j < w) A[(long long)i * lda + j] = v[a][b];
    }
}

// Transposed copy of a w x w block: dst(j, i) = src(i, j).
__global__ void transpose_block_kernel(double* dst, long long ldd, const double* src, long long lds, int w) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < w * w; e += gridDim.x * blockDim.x) {
    const int i = e / w, j = e % w;
    dst[(long long)j * ldd + i] = src[(long long)i * lds + j];
  }
}

// One step of parallel cyclic reduction on a_i x_{i-s} + b_i x_i + c_i x_{i+s} = d_i.
__global__ void pcr_step_kernel(int n, int s, const double* __restrict__ a, const double* __restrict__ b,
                                const double* __restrict__ c, const double* __restrict__ d, double* __restrict__ a2,
                                double* __restrict__ b2, double* __restrict__ c2, double* __restrict__ d2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double na = 0.0, nb = b[i], nc = 0.0, nd = d[i];
    if (i - s >= 0) {
      const double k1 = a[i] / b[i - s];
      na = -a[i - s] * k1;
      nb -= c[i - s] * k1;
      nd -= d[i - s] * k1;
    }
    if (i + s < n) {
      const double k2 = c[i] / b[i + s];
      nc = -c[i + s] * k2;
      nb -= a[i + s] * k2;
      nd -= d[i + s] * k2;
    }
    a2[i] = na, b2[i] = nb, c2[i] = nc, d2[i] = nd;
  }
}

// a_i = supdiag[i-1], b_i = diag[i], c_i = supdiag[i] (0 past the ends), d = rhs.
__global__ void pcr_init_kernel(int n, const double* diag, const double* sup, const double* rhs, double* a, double* b,
                                double* c, double* d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    a[i] = i > 0 ? sup[i - 1] : 0.0;
    b[i] = diag[i];
    c[i] = i < n - 1 ? sup[i] : 0.0;
    d[i] = rhs[i];
  }
}

__global__ void pcr_finish_kernel(int n, const double* b, const double* d, double* x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = d[i] / b[i];
}

// P = G on and below the diagonal, G^T above it (n x n), from the lower
// triangle of G: 32 x 32 tiles, the tiles above the diagonal transposed
// through shared memory so both the reads and the writes are coalesced.
__global__ void pack_lower_sym_kernel(double* P, long long ldp, const double* G, long long ldg, int n) {
  __shared__ double t[32][33];
  const int bi = blockIdx.y * 32, bj = blockIdx.x * 32;  // tile of P
  const bool upper = bj > bi;
  const int si = upper ? bj : bi, sj = upper ? bi : bj;  // tile of G that it comes from
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = si + r, j = sj + threadIdx.x;
    t[r][threadIdx.x] = (i < n && j < n) ? G[(long long)i * ldg + j] : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = bi + r, j = bj + threadIdx.x;
    if (i >= n || j >= n) continue;
    P[(long long)i * ldp + j] = upper ? t[threadIdx.x][r] : (j <= i ? t[r][threadIdx.x] : G[(long long)j * ldg + i]);
  }
}

int grid_for(long long total, int per) { return (int)std::max<long long>(1, std::min<long long>(cdivll(total, per), 4096)); }

}  // namespace

int dgemv_exact(int m, int n, const double* A, long long lda, const double* x, double* y, cudaStream_t st) {
  if (m <= 0) return LM_OK;
  gemv_exact_kernel<<<(int)cdivll(4LL * m, 256), 256, 0, st>>>(m, n, A, lda, x, y);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

int dnorm_inf_exact(int m, int n, const double* A, long long lda, unsigned long long* out, cudaStream_t st) {
  LM_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(unsigned long long), st));
  if (m <= 0 || n <= 0) return LM_OK;
  norm_inf_exact_kernel<<<cdiv(m, kNormRows), 256, 0, st>>>(m, n, A, lda, out);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

int lu_nopiv_block(double* A, long long lda, int w, int base, int* status, cudaStream_t st) {
  if (w <= 0) return LM_OK;
  if (w > 128) return LM_ERR_ARG;
  lu_nopiv_block_kernel<<<1, 512, 0, st>>>(A, lda, w, base, status);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

int pack_lower_sym(double* P, long long ldp, const double* G, long long ldg, int n, cudaStream_t st) {
  if (n <= 0) return LM_OK;
  dim3 tb(32, 8), tg(cdiv(n, 32), cdiv(n, 32));
  pack_lower_sym_kernel<<<tg, tb, 0, st>>>(P, ldp, G, ldg, n);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

int transpose_block(double* dst, long long ldd, const double* src, long long lds, int w, cudaStream_t st) {
  if (w <= 0) return LM_OK;
  transpose_block_kernel<<<grid_for((long long)w * w, 256), 256, 0, st>>>(dst, ldd, src, lds, w);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

// x = tridiag(supdiag, diag, supdiag)^-1 rhs by parallel cyclic reduction;
// W holds 8 n doubles of scratch.
int dtridiag_pcr(int n, const double* diag, const double* sup, const double* rhs, double* x, double* W,
                 cudaStream_t st) {
  if (n <= 0) return LM_OK;
  double* p[2][4];
  for (int s = 0; s < 2; ++s)
    for (int q = 0; q < 4; ++q) p[s][q] = W + (size_t)(4 * s + q) * n;
  const int g = grid_for(n, 256);
  pcr_init_kernel<<<g, 256, 0, st>>>(n, diag, sup, rhs, p[0][0], p[0][1], p[0][2], p[0][3]);
  int cur = 0, launches = 2;
  for (int s = 1; s < n; s *= 2, ++launches) {
    pcr_step_kernel<<<g, 256, 0, st>>>(n, s, p[cur][0], p[cur][1], p[cur][2], p[cur][3], p[cur ^ 1][0],
                                       p[cur ^ 1][1], p[cur ^ 1][2], p[cur ^ 1][3]);
    cur ^= 1;
  }
  pcr_finish_kernel<<<g, 256, 0, st>>>(n, p[cur][1], p[cur][3], x);
  count_launch(launches);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

}  // namespace lm
