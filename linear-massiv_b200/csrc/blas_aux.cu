// Row interchanges, triangular block solves, copies and the FP64 residual.
//
// laswp      : the row-swap half of rawSwapRows (K.hs:1507-1537) applied to
//              the columns outside the current panel, and applyPivotsForward
//              (LU.hs:493-507) on right-hand sides.
// trsm_left  : the w x w triangular block solves of the blocked factorisations
//              and substitutions — rawTriSolvePanelTrail (LU.hs:364-407) for
//              U12, and the diagonal blocks of rawForwardSubUnitPackedSIMD,
//              rawBackSubPackedSIMD, rawForwardSubCholPackedSIMD and
//              rawBackSubCholTPackedSIMD (K.hs:2205-2430).
// dresidual  : r = b - A x in FP64, the GEMV of matvecP / rawGemv
//              (L2.hs:131-139, K.hs:119-134) on the refinement path.
#include <climits>

#include "common.cuh"
#include "internal.h"

namespace lm {

void count_launch(int n);

namespace {

// Each thread owns one column and applies the swaps in groups of 8: all rows a
// group touches are loaded first (independent loads), the swaps are replayed
// in order on registers, and the touched rows are stored once.
template <typename T>
__global__ void laswp_kernel(T* A, long long lda, int nrows, const int* __restrict__ ipiv, int k0, int k1,
                             int ca0, int ca1, int cb0, int cb1, int* status) {
  const int na = ca1 - ca0, nb = cb1 - cb0;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= na + nb) return;
  const int col = t < na ? ca0 + t : cb0 + (t - na);
  T* base = A + col;
  constexpr int G = 8;
  for (int s0 = k0; s0 < k1; s0 += G) {
    const int cnt = min(G, k1 - s0);
    T v[2 * G];
    int slot_of_piv[G];
    int extra_row[G];
    int nextra = 0;
#pragma unroll
    for (int q = 0; q < G; ++q)
      if (q < cnt) v[q] = base[(long long)(s0 + q) * lda];
#pragma unroll
    for (int q = 0; q < G; ++q) {
      if (q < cnt) {
        int p = __ldg(ipiv + s0 + q);
        if (p < 0 || p >= nrows) {  // a bad swap list: record it, treat as no swap
          atomicCAS(status, 0, LM_DEVERR_BOUNDS);
          p = s0 + q;
        }
        int slot = -1;
        if (p >= s0 && p < s0 + cnt) {
          slot = p - s0;
        } else {
          for (int e = 0; e < nextra; ++e)
            if (extra_row[e] == p) slot = G + e;
          if (slot < 0) {
            extra_row[nextra] = p;
            slot = G + nextra;
            v[slot] = base[(long long)p * lda];
            ++nextra;
          }
        }
        slot_of_piv[q] = slot;
      }
    }
    for (int q = 0; q < cnt; ++q) {
      const int s = slot_of_piv[q];
      const T tmp = v[q];
      v[q] = v[s];
      v[s] = tmp;
    }
#pragma unroll
    for (int q = 0; q < G; ++q)
      if (q < cnt) base[(long long)(s0 + q) * lda] = v[q];
    for (int e = 0; e < nextra; ++e) base[(long long)extra_row[e] * lda] = v[G + e];
  }
}

// op(Tri) X = B for one w x 64 column block of B per CTA.  The w x w block of
// Tri and the B block are staged in shared memory; step k finalises x_k and
// applies it to the rows still to be solved (one barrier per step); the
// divisions by the diagonal are applied once at the end.
template <typename T>
__global__ void __launch_bounds__(256) trsm_left_kernel(const T* __restrict__ Tri, long long ldt, int w,
                                                       int lower, int unit, int trans, T* B, long long ldb,
                                                       int ncols) {
  extern __shared__ __align__(16) unsigned char sm[];
  const int ldts = w + 1;
  T* Ts = reinterpret_cast<T*>(sm);
  T* Bs = Ts + (size_t)w * ldts;  // w x 64, ld 65
  const int c0 = blockIdx.x * 64;
  const int nc = min(64, ncols - c0);
  for (int i = threadIdx.x; i < w * w; i += blockDim.x) {
    const int r = i / w, c = i % w;
    Ts[r * ldts + c] = Tri[(long long)r * ldt + c];
  }
  for (int i = threadIdx.x; i < w * 64; i += blockDim.x) {
    const int r = i / 64, c = i % 64;
    Bs[r * 65 + c] = (c < nc) ? B[(long long)r * ldb + c0 + c] : T(0);
  }
  __syncthreads();
  const bool upper_op = (lower == 0) != (trans != 0);
  const int c = threadIdx.x & 63;
  const int rg = threadIdx.x >> 6;
  const int ng = blockDim.x >> 6;
  for (int step = 0; step < w; ++step) {
    const int k = upper_op ? (w - 1 - step) : step;
    T xk = Bs[k * 65 + c];
    if (!unit) xk = xk / Ts[k * ldts + k];
    if (!upper_op) {
      for (int i = k + 1 + ((rg - (k + 1)) % ng + ng) % ng; i < w; i += ng) {
        const T tik = trans ? Ts[k * ldts + i] : Ts[i * ldts + k];
        Bs[i * 65 + c] = fma(-tik, xk, Bs[i * 65 + c]);
      }
    } else {
      for (int i = rg; i < k; i += ng) {
        const T tik = trans ? Ts[k * ldts + i] : Ts[i * ldts + k];
        Bs[i * 65 + c] = fma(-tik, xk, Bs[i * 65 + c]);
      }
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < w * 64; i += blockDim.x) {
    const int r = i / 64, cc = i % 64;
    if (cc < nc) {
      T x = Bs[r * 65 + cc];
      if (!unit) x = x / Ts[r * ldts + r];
      B[(long long)r * ldb + c0 + cc] = x;
    }
  }
}

template <typename T>
__global__ void copy2d_kernel(T* dst, long long ldd, const T* src, long long lds, int rows, int cols) {
  const long long total = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i % cols);
    dst[(long long)r * ldd + c] = src[(long long)r * lds + c];
  }
}

template <typename T>
__global__ void identity_kernel(T* A, long long lda, int rows, int cols) {
  const long long total = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i % cols);
    A[(long long)r * lda + c] = (r == c) ? T(1) : T(0);
  }
}

template <typename T>
__global__ void zero_upper_kernel(T* A, long long lda, int n) {
  const long long total = (long long)n * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / n), c = (int)(i % n);
    if (c > r) A[(long long)r * lda + c] = T(0);
  }
}

// One warp per row: r_i = b_i - sum_j a_ij x_j for up to 8 right-hand sides.
template <int NR>
__global__ void residual_kernel(int n, int nrhs, const double* __restrict__ A, long long lda,
                                const double* __restrict__ X, long long ldx, const double* __restrict__ B,
                                long long ldb, double* R, long long ldr) {
  const int warps = blockDim.x >> 5;
  const int row = blockIdx.x * warps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  double acc[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) acc[r] = 0.0;
  const double* arow = A + (long long)row * lda;
  for (int j = lane; j < n; j += 32) {
    const double a = arow[j];
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if (r < nrhs) acc[r] = fma(a, X[(long long)j * ldx + r], acc[r]);
  }
#pragma unroll
  for (int r = 0; r < NR; ++r)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
  if (lane == 0) {
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if (r < nrhs) R[(long long)row * ldr + r] = B[(long long)row * ldb + r] - acc[r];
  }
}

int grid_for(long long total, int threads, int sms) {
  long long g = cdivll(total, threads);
  return (int)std::max<long long>(1, std::min<long long>(g, 8LL * sms > 0 ? 8LL * sms : 1184));
}

}  // namespace

template <typename T>
int laswp(T* A, long long lda, int nrows, const int* ipiv, int k0, int k1, int ca0, int ca1, int cb0, int cb1,
          int* status, cudaStream_t st) {
  const int cols = std::max(0, ca1 - ca0) + std::max(0, cb1 - cb0);
  if (cols == 0 || k1 <= k0) return LM_OK;
  laswp_kernel<T><<<cdiv(cols, 128), 128, 0, st>>>(A, lda, nrows, ipiv, k0, k1, ca0, std::max(ca0, ca1), cb0,
                                                   std::max(cb0, cb1), status);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

template <typename T>
int trsm_left(const T* Tri, long long ldt, int w, bool lower, bool unit, bool trans, T* B, long long ldb,
              int ncols, cudaStream_t st) {
  if (w <= 0 || ncols <= 0) return LM_OK;
  if (w > 128) return LM_ERR_ARG;
  const size_t smem = sizeof(T) * ((size_t)w * (w + 1) + (size_t)w * 65);
  static bool attr_set[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(trsm_left_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(sizeof(T) * (128 * 129 + 128 * 65))));
    attr_set[dev] = true;
  }
  trsm_left_kernel<T><<<cdiv(ncols, 64), 256, smem, st>>>(Tri, ldt, w, lower ? 1 : 0, unit ? 1 : 0,
                                                          trans ? 1 : 0, B, ldb, ncols);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

template <typename T>
int copy2d(T* dst, long long ldd, const T* src, long long lds, int rows, int cols, cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return LM_OK;
  copy2d_kernel<T><<<grid_for((long long)rows * cols, 256, 148), 256, 0, st>>>(dst, ldd, src, lds, rows, cols);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

template <typename T>
int set_identity(T* A, long long lda, int rows, int cols, cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return LM_OK;
  identity_kernel<T><<<grid_for((long long)rows * cols, 256, 148), 256, 0, st>>>(A, lda, rows, cols);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

template <typename T>
int zero_upper(T* A, long long lda, int n, cudaStream_t st) {
  if (n <= 1) return LM_OK;
  zero_upper_kernel<T><<<grid_for((long long)n * n, 256, 148), 256, 0, st>>>(A, lda, n);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

int dresidual(Ctx& c, int n, int nrhs, const double* A, long long lda, const double* X, long long ldx,
              const double* B, long long ldb, double* R, long long ldr, cudaStream_t st) {
  if (nrhs <= 8) {
    const int warps = 8;
    residual_kernel<8><<<cdiv(n, warps), warps * 32, 0, st>>>(n, nrhs, A, lda, X, ldx, B, ldb, R, ldr);
    count_launch(1);
    LM_CUDA_TRY(cudaGetLastError());
    return LM_OK;
  }
  // Wide right-hand sides: R = B, then R -= A X on the tensor cores.
  const bool ok = !((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(X)) & 15) && !(lda & 1) &&
                  !(ldx & 1);
  const double* A2 = A;
  const double* X2 = X;
  long long lda2 = lda, ldx2 = ldx;
  if (!ok) {
    lda2 = (n + 7) / 8 * 8;
    ldx2 = (nrhs + 7) / 8 * 8;
    void* ws = nullptr;
    LM_TRY(ctx_workspace(c, 1, sizeof(double) * ((size_t)n * lda2 + (size_t)n * ldx2), &ws));
    double* a = static_cast<double*>(ws);
    double* x = a + (size_t)n * lda2;
    LM_TRY(copy2d<double>(a, lda2, A, lda, n, n, st));
    LM_TRY(copy2d<double>(x, ldx2, X, ldx, n, nrhs, st));
    A2 = a;
    X2 = x;
  }
  LM_TRY(copy2d<double>(R, ldr, B, ldb, n, nrhs, st));
  GemmDesc d;
  d.m = n; d.n = nrhs; d.k = n; d.alpha = -1.0; d.beta = 1.0;
  d.A = A2; d.lda = lda2; d.B = X2; d.ldb = ldx2; d.C = R; d.ldc = ldr;
  return dgemm(c, d, st);
}

template int laswp<double>(double*, long long, int, const int*, int, int, int, int, int, int, int*, cudaStream_t);
template int laswp<float>(float*, long long, int, const int*, int, int, int, int, int, int, int*, cudaStream_t);
template int trsm_left<double>(const double*, long long, int, bool, bool, bool, double*, long long, int,
                               cudaStream_t);
template int trsm_left<float>(const float*, long long, int, bool, bool, bool, float*, long long, int,
                              cudaStream_t);
template int copy2d<double>(double*, long long, const double*, long long, int, int, cudaStream_t);
template int copy2d<float>(float*, long long, const float*, long long, int, int, cudaStream_t);
template int set_identity<double>(double*, long long, int, int, cudaStream_t);
template int set_identity<float>(float*, long long, int, int, cudaStream_t);
template int zero_upper<double>(double*, long long, int, cudaStream_t);
template int zero_upper<float>(float*, long long, int, cudaStream_t);

}  // namespace lm
