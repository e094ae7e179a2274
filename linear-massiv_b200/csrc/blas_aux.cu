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

// Row interchanges as one composed permutation.  The swaps ipiv[k0..k1)
// (at most kSwapChunk of them) touch at most 2 * kSwapChunk rows.  Thread 0
// replays them on row indices in shared memory (rows k0..k1-1 in fixed
// slots, other pivot rows found through a small open-addressing table),
// giving for every touched row r the row src(r) whose data ends up in it.
// The CTA then gathers all sources of its 32-column block into shared memory
// (coalesced along the columns, many independent loads per thread) and
// scatters them to their rows.
constexpr int kSwapChunk = 128;
constexpr int kSwapThreads = 256;
constexpr int kHash = 512;

template <typename T>
__global__ void __launch_bounds__(kSwapThreads) laswp_kernel(T* A, long long lda, int nrows,
                                                             const int* __restrict__ ipiv, int k0, int k1, int ca0,
                                                             int ca1, int cb0, int cb1, int* status) {
  __shared__ int rows[2 * kSwapChunk];
  __shared__ int src[2 * kSwapChunk];
  __shared__ int piv[kSwapChunk];
  __shared__ int hkey[kHash];
  __shared__ short hval[kHash];
  __shared__ int list_r[2 * kSwapChunk];
  __shared__ int list_s[2 * kSwapChunk];
  __shared__ int m_sh, mm_sh;
  extern __shared__ __align__(16) unsigned char sm[];
  T* stage = reinterpret_cast<T*>(sm);  // [2 * kSwapChunk][32]
  const int tid = threadIdx.x;
  const int cnt = k1 - k0;
  for (int i = tid; i < kHash; i += kSwapThreads) hkey[i] = -1;
  for (int i = tid; i < cnt; i += kSwapThreads) {
    rows[i] = k0 + i;
    src[i] = k0 + i;
    piv[i] = __ldg(ipiv + k0 + i);
  }
  if (tid == 0) mm_sh = 0;
  __syncthreads();
  if (tid == 0) {
    int m = cnt;
    for (int q = 0; q < cnt; ++q) {
      const int k = k0 + q;
      const int p = piv[q];
      if (p < 0 || p >= nrows) {  // a bad swap list: record it, treat as no swap
        atomicCAS(status, 0, LM_DEVERR_BOUNDS);
        continue;
      }
      if (p == k) continue;
      int sp;
      if (p >= k0 && p < k1) {
        sp = p - k0;
      } else {
        unsigned h = ((unsigned)p * 2654435761u) & (kHash - 1);
        while (hkey[h] != -1 && hkey[h] != p) h = (h + 1) & (kHash - 1);
        if (hkey[h] == p) {
          sp = hval[h];
        } else {
          hkey[h] = p;
          hval[h] = (short)m;
          rows[m] = p;
          src[m] = p;
          sp = m++;
        }
      }
      const int t = src[q];
      src[q] = src[sp];
      src[sp] = t;
    }
    m_sh = m;
  }
  __syncthreads();
  // compact to the rows that actually change
  for (int i = tid; i < m_sh; i += kSwapThreads)
    if (src[i] != rows[i]) {
      const int at = atomicAdd(&mm_sh, 1);
      list_r[at] = rows[i];
      list_s[at] = src[i];
    }
  __syncthreads();
  const int mm = mm_sh;
  const int na = ca1 - ca0, ncols = na + (cb1 - cb0);
  const int lane = tid & 31, warp = tid >> 5;
  const int t = blockIdx.x * 32 + lane;
  const bool active = t < ncols;
  const int col = t < na ? ca0 + t : cb0 + (t - na);
#pragma unroll 4
  for (int i = warp; i < mm; i += kSwapThreads / 32)
    if (active) stage[i * 32 + lane] = A[(long long)list_s[i] * lda + col];
  __syncthreads();
#pragma unroll 4
  for (int i = warp; i < mm; i += kSwapThreads / 32)
    if (active) A[(long long)list_r[i] * lda + col] = stage[i * 32 + lane];
}

// The same interchanges split in two launches for wide matrices: one CTA
// composes the swaps ipiv[k0..k1) into the list of (row, source row) pairs
// that change (plan[0] = count, then rows, then sources, 2 * kSwapChunk
// each), so that the column blocks need no serial prologue of their own.
// Every touched row (the swap positions k0..k1-1 and the distinct pivot rows
// outside them) is a thread, which finds its source by walking the swap list
// backwards: source(r) = tau_k0(tau_k0+1(... tau_k1-1(r))).
__global__ void __launch_bounds__(2 * kSwapChunk) swap_plan_kernel(int nrows, const int* __restrict__ ipiv, int k0,
                                                                   int k1, int* plan, int* status) {
  __shared__ int piv[kSwapChunk];
  __shared__ int mm_sh;
  const int tid = threadIdx.x;
  const int cnt = k1 - k0;
  if (tid < cnt) {
    int p = __ldg(ipiv + k0 + tid);
    if (p < 0 || p >= nrows) {  // a bad swap list: record it, treat as no swap
      atomicCAS(status, 0, LM_DEVERR_BOUNDS);
      p = k0 + tid;
    }
    piv[tid] = p;
  }
  if (tid == 0) mm_sh = 0;
  __syncthreads();
  int r = -1;
  if (tid < cnt) {
    r = k0 + tid;
  } else if (tid < 2 * cnt) {
    const int q = tid - cnt;
    const int p = piv[q];
    bool first = p < k0 || p >= k1;  // swap positions are covered above
    for (int e = 0; e < q && first; ++e) first = piv[e] != p;
    if (first) r = p;
  }
  if (r >= 0) {
    int x = r;
    for (int q = cnt - 1; q >= 0; --q) {
      const int k = k0 + q, p = piv[q];
      x = (x == k) ? p : ((x == p) ? k : x);
    }
    if (x != r) {
      const int at = atomicAdd(&mm_sh, 1);
      plan[1 + at] = r;
      plan[1 + 2 * kSwapChunk + at] = x;
    }
  }
  __syncthreads();
  if (tid == 0) plan[0] = mm_sh;
}

// Gather every changing row's source over a 32-column block into shared
// memory, then scatter (the plan of swap_plan_kernel).
template <typename T>
__global__ void __launch_bounds__(kSwapThreads) swap_apply_kernel(T* A, long long lda, const int* __restrict__ plan,
                                                                  int ca0, int ca1, int cb0, int cb1) {
  __shared__ int list_r[2 * kSwapChunk];
  __shared__ int list_s[2 * kSwapChunk];
  extern __shared__ __align__(16) unsigned char sm[];
  T* stage = reinterpret_cast<T*>(sm);  // [2 * kSwapChunk][32]
  const int tid = threadIdx.x;
  const int mm = __ldg(plan);
  for (int i = tid; i < mm; i += kSwapThreads) {
    list_r[i] = __ldg(plan + 1 + i);
    list_s[i] = __ldg(plan + 1 + 2 * kSwapChunk + i);
  }
  __syncthreads();
  const int na = ca1 - ca0, ncols = na + (cb1 - cb0);
  const int lane = tid & 31, warp = tid >> 5;
  const int t = blockIdx.x * 32 + lane;
  const bool active = t < ncols;
  const int col = t < na ? ca0 + t : cb0 + (t - na);
#pragma unroll 8
  for (int i = warp; i < mm; i += kSwapThreads / 32)
    if (active) stage[i * 32 + lane] = A[(long long)list_s[i] * lda + col];
  __syncthreads();
#pragma unroll 8
  for (int i = warp; i < mm; i += kSwapThreads / 32)
    if (active) A[(long long)list_r[i] * lda + col] = stage[i * 32 + lane];
}

// All interchanges ipiv[0..n) on a narrow block B (n x nrhs) at once:
// W(i, :) = B(sigma(i), :) with sigma(i) = tau_0(tau_1(... tau_{n-1}(i))),
// tau_k the transposition (k, ipiv[k]).  Thread i walks the swap list
// backwards (ipiv staged through shared memory, read as broadcasts), so the
// n sequential swaps of applyPivotsForward (LU.hs:493-507) become one
// parallel gather; an out-of-range pivot row records LM_DEVERR_BOUNDS.
template <typename T>
__global__ void __launch_bounds__(128) perm_gather_kernel(const T* __restrict__ B, long long ldb, int n, int nrhs,
                                                          const int* __restrict__ ipiv, T* W, long long ldw,
                                                          int* status) {
  constexpr int CH = 4096;
  __shared__ int sp[CH];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int r = i;
  bool bad = false;
  for (int c0 = ((n - 1) / CH) * CH; c0 >= 0; c0 -= CH) {
    const int cnt = min(CH, n - c0);
    __syncthreads();
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) sp[e] = __ldg(ipiv + c0 + e);
    __syncthreads();
#pragma unroll 8
    for (int k = cnt - 1; k >= 0; --k) {
      const int p = sp[k];
      const int kk = c0 + k;
      r = (r == kk) ? p : ((r == p) ? kk : r);
    }
  }
  if (i < n) {
    if (r < 0 || r >= n) bad = true;
    if (bad) {
      atomicCAS(status, 0, LM_DEVERR_BOUNDS);
      r = i;
    }
    for (int c = 0; c < nrhs; ++c) W[(long long)i * ldw + c] = B[(long long)r * ldb + c];
  }
}

// sigma of the swap list ipiv[0..n) (as perm_gather_kernel walks it), once
// per factorisation: perm[i] = sigma(i), so that every later application of
// the interchanges to a right-hand side (applyPivotsForward, LU.hs:493-507)
// is a plain gather; an out-of-range pivot row records LM_DEVERR_BOUNDS and
// maps i to itself.
__global__ void __launch_bounds__(128) perm_from_swaps_kernel(const int* __restrict__ ipiv, int n, int* perm,
                                                              int* status) {
  constexpr int CH = 4096;
  __shared__ int sp[CH];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int r = i;
  for (int c0 = ((n - 1) / CH) * CH; c0 >= 0; c0 -= CH) {
    const int cnt = min(CH, n - c0);
    __syncthreads();
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) sp[e] = __ldg(ipiv + c0 + e);
    __syncthreads();
#pragma unroll 8
    for (int k = cnt - 1; k >= 0; --k) {
      const int p = sp[k];
      const int kk = c0 + k;
      r = (r == kk) ? p : ((r == p) ? kk : r);
    }
  }
  if (i < n) {
    if (r < 0 || r >= n) {
      atomicCAS(status, 0, LM_DEVERR_BOUNDS);
      r = i;
    }
    perm[i] = r;
  }
}

// W(i, :) = B(perm[i], :) for a narrow block (n x nrhs).
template <typename T>
__global__ void gather_rows_kernel(const T* __restrict__ B, long long ldb, int n, int nrhs,
                                   const int* __restrict__ perm, T* W, long long ldw) {
  const long long total = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / nrhs), c = (int)(e % nrhs);
    W[(long long)i * ldw + c] = B[(long long)__ldg(perm + i) * ldb + c];
  }
}

// op(Tri) X = B for one w x 32 column block of B per CTA (w <= 128).  The
// triangle of op(Tri) is staged packed in shared memory (w(w+1)/2 entries,
// so two CTAs fit per SM in FP64) together with the block.  Rows are solved
// in 16-row blocks: warp 0 solves a diagonal block (lane = column,
// sequential over its 16 rows), then all warps apply the block to the rows
// still to be solved (a rank-16 update).  Two barriers per 16 rows.
__device__ __forceinline__ int tri_idx(bool upper, int w, int i, int k) {
  return upper ? i * w - (i * (i - 1)) / 2 + (k - i) : (i * (i + 1)) / 2 + k;
}

template <typename T>
__global__ void __launch_bounds__(256) trsm_left_kernel(const T* __restrict__ Tri, long long ldt, int w,
                                                       int lower, int unit, int trans, T* B, long long ldb,
                                                       int ncols) {
  extern __shared__ __align__(16) unsigned char sm[];
  const bool upper_op = (lower == 0) != (trans != 0);
  T* Ts = reinterpret_cast<T*>(sm);
  T* Bs = Ts + ((w * (w + 1) / 2 + 1) & ~1);  // w x 32, ld 33
  const int c0 = blockIdx.x * 32;
  const int nc = min(32, ncols - c0);
#pragma unroll 8
  for (int i = threadIdx.x; i < w * w; i += blockDim.x) {
    const int r = i / w, c = i % w;
    if (lower ? (c <= r) : (c >= r)) {
      const int oi = trans ? c : r, ok = trans ? r : c;
      Ts[tri_idx(upper_op, w, oi, ok)] = Tri[(long long)r * ldt + c];
    }
  }
#pragma unroll 8
  for (int i = threadIdx.x; i < w * 32; i += blockDim.x) {
    const int r = i >> 5, c = i & 31;
    Bs[r * 33 + c] = (c < nc) ? B[(long long)r * ldb + c0 + c] : T(0);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int nb = (w + 15) / 16;
  for (int bi = 0; bi < nb; ++bi) {
    const int b = upper_op ? nb - 1 - bi : bi;
    const int r0 = b * 16, r1 = min(r0 + 16, w);
    if (warp == 0) {
      if (!upper_op) {
        for (int r = r0; r < r1; ++r) {
          const T* trow = Ts + tri_idx(false, w, r, 0);
          T x = Bs[r * 33 + lane];
          for (int q = r0; q < r; ++q) x = fma(-trow[q], Bs[q * 33 + lane], x);
          if (!unit) x = x / trow[r];
          Bs[r * 33 + lane] = x;
        }
      } else {
        for (int r = r1 - 1; r >= r0; --r) {
          const T* trow = Ts + tri_idx(true, w, r, r) - r;  // trow[q] = op(T)(r, q), q >= r
          T x = Bs[r * 33 + lane];
          for (int q = r + 1; q < r1; ++q) x = fma(-trow[q], Bs[q * 33 + lane], x);
          if (!unit) x = x / trow[r];
          Bs[r * 33 + lane] = x;
        }
      }
    }
    __syncthreads();
    // rank-(r1-r0) update of the unsolved rows
    const int u0 = upper_op ? 0 : r1, u1 = upper_op ? r0 : w;
    for (int i = u0 + warp; i < u1; i += nwarps) {
      const T* trow = upper_op ? Ts + tri_idx(true, w, i, i) - i : Ts + tri_idx(false, w, i, 0);
      T acc = Bs[i * 33 + lane];
      for (int q = r0; q < r1; ++q) acc = fma(-trow[q], Bs[q * 33 + lane], acc);
      Bs[i * 33 + lane] = acc;
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < w * 32; i += blockDim.x) {
    const int r = i >> 5, c = i & 31;
    if (c < nc) B[(long long)r * ldb + c0 + c] = Bs[r * 33 + c];
  }
}

template <typename T>
__global__ void copy2d_kernel(T* dst, long long ldd, const T* src, long long lds, int rows, int cols) {
  const long long total = (long long)rows * cols;
#pragma unroll 4
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
#pragma unroll 8
  for (int j = lane; j < n; j += 32) {
    const double a = arow[j];
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if (r < nrhs) acc[r] = fma(a, X[(long long)j * ldx + r], acc[r]);
  }
  __syncwarp();  // lanes leave the strided loop at different trip counts
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
          int* status, cudaStream_t st, int* plan) {
  ca1 = std::max(ca0, ca1);
  cb1 = std::max(cb0, cb1);
  const int cols = (ca1 - ca0) + (cb1 - cb0);
  if (cols == 0 || k1 <= k0) return LM_OK;
  const size_t smem = sizeof(T) * 2 * kSwapChunk * 32;
  static bool attr_set[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(laswp_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    LM_CUDA_TRY(cudaFuncSetAttribute(swap_apply_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set[dev] = true;
  }
  // wide: plan once, then the column blocks; narrow: one self-contained launch
  const bool planned = plan != nullptr && cols > 4 * 32;
  for (int s0 = k0; s0 < k1; s0 += kSwapChunk) {
    const int s1 = std::min(k1, s0 + kSwapChunk);
    if (planned) {
      swap_plan_kernel<<<1, 2 * kSwapChunk, 0, st>>>(nrows, ipiv, s0, s1, plan, status);
      swap_apply_kernel<T><<<cdiv(cols, 32), kSwapThreads, smem, st>>>(A, lda, plan, ca0, ca1, cb0, cb1);
      count_launch(2);
    } else {
      laswp_kernel<T><<<cdiv(cols, 32), kSwapThreads, smem, st>>>(A, lda, nrows, ipiv, s0, s1, ca0, ca1, cb0, cb1,
                                                                  status);
      count_launch(1);
    }
    LM_CUDA_TRY(cudaGetLastError());
  }
  return LM_OK;
}

int perm_from_swaps(const int* ipiv, int n, int* perm, int* status, cudaStream_t st) {
  if (n <= 0) return LM_OK;
  perm_from_swaps_kernel<<<cdiv(n, 128), 128, 0, st>>>(ipiv, n, perm, status);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

template <typename T>
int laswp_perm(T* B, long long ldb, int n, int nrhs, const int* perm, T* W, cudaStream_t st) {
  if (n <= 0 || nrhs <= 0) return LM_OK;
  const long long total = (long long)n * nrhs;
  gather_rows_kernel<T><<<(int)std::min<long long>((total + 255) / 256, 4096), 256, 0, st>>>(B, ldb, n, nrhs, perm,
                                                                                            W, nrhs);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return copy2d<T>(B, ldb, W, nrhs, n, nrhs, st);
}

template <typename T>
int laswp_narrow(T* B, long long ldb, int n, int nrhs, const int* ipiv, T* W, int* status, cudaStream_t st) {
  if (n <= 0 || nrhs <= 0) return LM_OK;
  perm_gather_kernel<T><<<cdiv(n, 128), 128, 0, st>>>(B, ldb, n, nrhs, ipiv, W, nrhs, status);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return copy2d<T>(B, ldb, W, nrhs, n, nrhs, st);
}

template <typename T>
int trsm_left(const T* Tri, long long ldt, int w, bool lower, bool unit, bool trans, T* B, long long ldb,
              int ncols, cudaStream_t st) {
  if (w <= 0 || ncols <= 0) return LM_OK;
  if (w > 128) return LM_ERR_ARG;
  const size_t smem = sizeof(T) * ((size_t)((w * (w + 1) / 2 + 1) & ~1) + (size_t)w * 33);
  static bool attr_set[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(trsm_left_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(sizeof(T) * (128 * 129 / 2 + 1 + 128 * 33))));
    attr_set[dev] = true;
  }
  trsm_left_kernel<T><<<cdiv(ncols, 32), 256, smem, st>>>(Tri, ldt, w, lower ? 1 : 0, unit ? 1 : 0,
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

template int laswp<double>(double*, long long, int, const int*, int, int, int, int, int, int, int*, cudaStream_t,
                           int*);
template int laswp<float>(float*, long long, int, const int*, int, int, int, int, int, int, int*, cudaStream_t, int*);
template int laswp_narrow<double>(double*, long long, int, int, const int*, double*, int*, cudaStream_t);
template int laswp_narrow<float>(float*, long long, int, int, const int*, float*, int*, cudaStream_t);
template int laswp_perm<double>(double*, long long, int, int, const int*, double*, cudaStream_t);
template int laswp_perm<float>(float*, long long, int, int, const int*, float*, cudaStream_t);
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
