// Recursive butterfly transformation (RBT) of depth 2 for the randomised
// mixed-precision solver.  No counterpart in linear-massiv.
//
// A butterfly of order m is B = (1/sqrt2) [R S; R -S] with R, S diagonal,
// entries exp(r / 10), r uniform in [-1/2, 1/2] (Parker 1995; Baboulin,
// Dongarra, Herrmann and Tomov 2013).  The depth-2 recursive butterfly of
// order np (a multiple of 4) is W = W1 W2: W1 one butterfly of order np, W2
// two butterflies of order np/2 on the diagonal.  With independent U and V,
// Ar = U^T A V can be factored without pivoting with high probability of
// stability; A x = b is solved as Ar y = U^T b, x = V y, and iterative
// refinement with the original A repairs the rest.
//
// Depth 2 couples each row i only with the rows i0 + a*np/4 (a = 0..3,
// i0 = i mod np/4), so every transform is a set of independent 4-point
// butterflies: one thread per (i0, j0) for the matrix, per (i0, column) for
// the right-hand sides.  Matrices of order n not divisible by 4 are padded
// to np with the identity (and right-hand sides with zeros).
//
// Diagonal storage d[2*np] per transform: d[p] (p < np/2) is R of the
// level-1 butterfly, d[np/2 + p] its S; d[np + p] for p in the four quarters
// [0, np/4), ... are R and S of the first level-2 butterfly, then R and S of
// the second.
#include "common.cuh"
#include "internal.h"

namespace lm {

void count_launch(int n);

namespace {

constexpr double kRsqrt2 = 0.70710678118654752440;

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// d[0 .. 2np) of U (which = 0) or V (which = 1) from a fixed seed.
__global__ void rbt_diag_kernel(double* du, double* dv, int np, unsigned long long seed) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 4 * np; i += gridDim.x * blockDim.x) {
    const unsigned long long h = mix64(seed ^ mix64((unsigned long long)i));
    const double r = (double)(h >> 11) * (1.0 / 9007199254740992.0) - 0.5;  // [-1/2, 1/2)
    const double v = exp(r / 10.0);
    if (i < 2 * np)
      du[i] = v;
    else
      dv[i - 2 * np] = v;
  }
}

// y = W^T x for the four partner entries x[a] at positions i0 + a q.
__device__ __forceinline__ void bt_transposed(double (&x)[4], int i0, int q, const double* __restrict__ d) {
  const int np = 4 * q;
  const double t0 = d[i0] * (x[0] + x[2]) * kRsqrt2;
  const double t1 = d[i0 + q] * (x[1] + x[3]) * kRsqrt2;
  const double b0 = d[2 * q + i0] * (x[0] - x[2]) * kRsqrt2;
  const double b1 = d[3 * q + i0] * (x[1] - x[3]) * kRsqrt2;
  x[0] = d[np + i0] * (t0 + t1) * kRsqrt2;
  x[1] = d[np + q + i0] * (t0 - t1) * kRsqrt2;
  x[2] = d[np + 2 * q + i0] * (b0 + b1) * kRsqrt2;
  x[3] = d[np + 3 * q + i0] * (b0 - b1) * kRsqrt2;
}

// x = W y for the four partner entries.
__device__ __forceinline__ void bt_forward(double (&y)[4], int i0, int q, const double* __restrict__ d) {
  const int np = 4 * q;
  const double z0 = (d[np + i0] * y[0] + d[np + q + i0] * y[1]) * kRsqrt2;
  const double z1 = (d[np + i0] * y[0] - d[np + q + i0] * y[1]) * kRsqrt2;
  const double z2 = (d[np + 2 * q + i0] * y[2] + d[np + 3 * q + i0] * y[3]) * kRsqrt2;
  const double z3 = (d[np + 2 * q + i0] * y[2] - d[np + 3 * q + i0] * y[3]) * kRsqrt2;
  y[0] = (d[i0] * z0 + d[2 * q + i0] * z2) * kRsqrt2;
  y[1] = (d[i0 + q] * z1 + d[3 * q + i0] * z3) * kRsqrt2;
  y[2] = (d[i0] * z0 - d[2 * q + i0] * z2) * kRsqrt2;
  y[3] = (d[i0 + q] * z1 - d[3 * q + i0] * z3) * kRsqrt2;
}

// Ar (np x np, FP32, ldr) = fl32(U^T A V) with A (n x n, FP64) padded to np
// with the identity.  Thread (i0, j0): the 16 entries at (i0 + a q, j0 + b q).
__global__ void __launch_bounds__(256) rbt_transform_kernel(float* __restrict__ Ar, long long ldr,
                                                            const double* __restrict__ A, long long lda, int n,
                                                            int np, const double* __restrict__ du,
                                                            const double* __restrict__ dv) {
  const int q = np / 4;
  const int j0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = blockIdx.y;
  if (j0 >= q) return;
  double m[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = i0 + a * q;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int j = j0 + b * q;
      m[a][b] = (i < n && j < n) ? A[(long long)i * lda + j] : (i == j ? 1.0 : 0.0);
    }
  }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    double x[4] = {m[0][b], m[1][b], m[2][b], m[3][b]};
    bt_transposed(x, i0, q, du);
#pragma unroll
    for (int a = 0; a < 4; ++a) m[a][b] = x[a];
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    double x[4] = {m[a][0], m[a][1], m[a][2], m[a][3]};
    bt_transposed(x, j0, q, dv);
#pragma unroll
    for (int b = 0; b < 4; ++b) Ar[(long long)(i0 + a * q) * ldr + j0 + b * q] = (float)x[b];
  }
}

// In place on the np x nrhs FP32 block D: D = W^T D (transposed = 1) or W D.
__global__ void rbt_rows_kernel(float* D, long long ldd, int np, int nrhs, const double* __restrict__ d,
                                int transposed) {
  const int q = np / 4;
  const long long total = (long long)q * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(e / nrhs), c = (int)(e % nrhs);
    double x[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) x[a] = D[(long long)(i0 + a * q) * ldd + c];
    if (transposed)
      bt_transposed(x, i0, q, d);
    else
      bt_forward(x, i0, q, d);
#pragma unroll
    for (int a = 0; a < 4; ++a) D[(long long)(i0 + a * q) * ldd + c] = (float)x[a];
  }
}

}  // namespace

int rbt_diagonals(double* du, double* dv, int np, cudaStream_t st) {
  if (np <= 0 || np % 4) return LM_ERR_ARG;
  rbt_diag_kernel<<<(4 * np + 255) / 256, 256, 0, st>>>(du, dv, np, 0x6C696E6D61737369ull);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

int rbt_transform(float* Ar, long long ldr, const double* A, long long lda, int n, int np, const double* du,
                  const double* dv, cudaStream_t st) {
  if (np <= 0 || np % 4 || n > np) return LM_ERR_ARG;
  const int q = np / 4;
  dim3 grid((q + 255) / 256, q);
  rbt_transform_kernel<<<grid, 256, 0, st>>>(Ar, ldr, A, lda, n, np, du, dv);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

int rbt_rows(float* D, long long ldd, int np, int nrhs, const double* d, bool transposed, cudaStream_t st) {
  if (np <= 0 || np % 4) return LM_ERR_ARG;
  const long long total = (long long)(np / 4) * nrhs;
  const int grid = (int)std::min<long long>((total + 255) / 256, 1184);
  rbt_rows_kernel<<<grid, 256, 0, st>>>(D, ldd, np, nrhs, d, transposed ? 1 : 0);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

}  // namespace lm
