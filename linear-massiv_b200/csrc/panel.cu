// Panel kernels: the latency-bound, column-by-column parts of LU and Cholesky.
//
// panel_leaf  — partial-pivoting LU of a tall panel (rows [c0, n), up to 32
//   columns), the B200 replacement for the per-column loop of panelLUFactor
//   (LU.hs:320-327): rawPivotSearch (K.hs:1541-1556), rawSwapRows
//   (K.hs:1507-1537) and rawLUEliminateColumnTo (K.hs:1464-1503).
//   The panel is held in the shared memory of a thread-block cluster (up to 16
//   CTAs, each owning a contiguous slab of rows, column-major in SMEM).  Per
//   column: each CTA reduces its slab's |a_ij| with warp shuffles, publishes
//   (value, row, candidate row, row j) in a double-buffered mailbox, one
//   cluster barrier, then every CTA reads all mailboxes over distributed shared
//   memory, picks the pivot (largest |a|, lowest row on ties — the reference's
//   strict '>' scan), swaps and eliminates its own rows, fusing the next
//   column's local argmax into the elimination pass.
//   NaN rule of the reference scan: if |a_jj| is NaN it stays the pivot; NaNs
//   below it never win.
//
// potrf_block — Cholesky of one <=128 x 128 diagonal block in SMEM
//   (rawCholColumnSIMDFrom, K.hs:2137-2195, for a diagonal panel).
#include <climits>

#include "common.cuh"
#include "internal.h"

namespace lm {

void count_launch(int n);

namespace {

constexpr int kLeafThreads = 512;
constexpr int kLeafRowsTimesW = 16384;  // rows per CTA * leaf width (128 KB of FP64)

template <typename T, int W>
struct alignas(16) Mailbox {
  T val;
  int idx;
  int jnan;
  T cand[W];
  T rowj[W];
};

template <typename T>
__device__ __forceinline__ bool better(T v1, int i1, T v2, int i2) {
  return v1 > v2 || (v1 == v2 && i1 < i2);
}

template <typename T>
__device__ __forceinline__ T absval(T x) {
  T a = x < T(0) ? -x : x;
  return (a != a) ? T(-1) : a;  // NaN never wins the scan
}

template <typename T, int W>
struct LeafSmem {
  static constexpr size_t mb_off = 0;
  static constexpr size_t mb_bytes = 2 * sizeof(Mailbox<T, W>);
  static constexpr size_t cand_off = (mb_off + mb_bytes + 15) / 16 * 16;
  static constexpr size_t rowj_off = cand_off + 16 * W * sizeof(T);
  static constexpr size_t cval_off = rowj_off + W * sizeof(T);
  static constexpr size_t cidx_off = cval_off + 16 * sizeof(T);
  static constexpr size_t misc_off = cidx_off + 16 * sizeof(int);
  static constexpr size_t wval_off = (misc_off + 4 * sizeof(int) + 15) / 16 * 16;
  static constexpr size_t widx_off = wval_off + 16 * sizeof(T);
  static constexpr size_t p_off = (widx_off + 16 * sizeof(int) + 15) / 16 * 16;
  static size_t bytes(int rpc) { return p_off + (size_t)W * (rpc + 1) * sizeof(T); }
};

template <typename T, int W>
__global__ void __launch_bounds__(kLeafThreads, 1)
    panel_leaf_kernel(T* A, long long lda, int n, int c0, int w, int rpc, int* ipiv, int* status) {
  using L = LeafSmem<T, W>;
  extern __shared__ __align__(16) unsigned char sm[];
  Mailbox<T, W>* mb = reinterpret_cast<Mailbox<T, W>*>(sm + L::mb_off);
  T* cand_all = reinterpret_cast<T*>(sm + L::cand_off);
  T* rowj_st = reinterpret_cast<T*>(sm + L::rowj_off);
  T* cval = reinterpret_cast<T*>(sm + L::cval_off);
  int* cidx = reinterpret_cast<int*>(sm + L::cidx_off);
  int* misc = reinterpret_cast<int*>(sm + L::misc_off);
  T* wval = reinterpret_cast<T*>(sm + L::wval_off);
  int* widx = reinterpret_cast<int*>(sm + L::widx_off);
  T* P = reinterpret_cast<T*>(sm + L::p_off);
  const int ldp = rpc + 1;

  const int q = (int)cluster_ctarank();
  const int C = (int)cluster_nctarank();
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int R = n - c0;
  const int rbeg = q * rpc;
  const int rcnt = max(0, min(rpc, R - rbeg));
  constexpr int RPT = (kLeafRowsTimesW / W + kLeafThreads - 1) / kLeafThreads;  // rows per thread

  // Load this CTA's slab, column-major: P[c * ldp + r].
  for (int i = tid; i < rcnt * W; i += kLeafThreads) {
    const int r = i / W, c = i % W;
    P[c * ldp + r] = (c < w) ? A[(long long)(c0 + rbeg + r) * lda + c0 + c] : T(0);
  }
  __syncthreads();

  // Local argmax of column 0.
  T bv = T(-1);
  int bi = INT_MAX;
#pragma unroll
  for (int u = 0; u < RPT; ++u) {
    const int r = tid + u * kLeafThreads;
    if (r < rcnt) {
      const T v = absval(P[r]);
      if (better(v, rbeg + r, bv, bi)) { bv = v; bi = rbeg + r; }
    }
  }

  for (int j = 0; j < w; ++j) {
    // ---- CTA-level reduction of (bv, bi) ----
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const T ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
    }
    if (lane == 0) { wval[warp] = bv; widx[warp] = bi; }
    __syncthreads();
    Mailbox<T, W>& m = mb[j & 1];
    if (warp == 0) {
      T v = lane < kLeafThreads / 32 ? wval[lane] : T(-1);
      int i = lane < kLeafThreads / 32 ? widx[lane] : INT_MAX;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, i, o);
        if (better(ov, oi, v, i)) { v = ov; i = oi; }
      }
      if (lane == 0) { m.val = v; m.idx = i; }
      if (i != INT_MAX && lane < W) m.cand[lane] = P[lane * ldp + (i - rbeg)];
      if (j >= rbeg && j < rbeg + rcnt) {
        if (lane < W) m.rowj[lane] = P[lane * ldp + (j - rbeg)];
        if (lane == 0) {
          const T d = P[j * ldp + (j - rbeg)];
          m.jnan = (d != d) ? 1 : 0;
        }
      }
    }
    cluster_sync_all();

    // ---- gather every CTA's candidate over distributed shared memory ----
    const int owner_j = j / rpc;
    // items: [0, C) values+rows, [C, C + C*W) candidate rows, then row j, then jnan
    for (int it = tid; it < C + C * W + W + 1; it += kLeafThreads) {
      if (it < C) {
        cval[it] = dsmem_ld<T>(dsmem_map(&m.val, it));
        cidx[it] = dsmem_ld_s32(dsmem_map(&m.idx, it));
      } else if (it < C + C * W) {
        const int src = (it - C) / W, e = (it - C) % W;
        cand_all[src * W + e] = dsmem_ld<T>(dsmem_map(&m.cand[e], src));
      } else if (it < C + C * W + W) {
        const int e = it - (C + C * W);
        rowj_st[e] = dsmem_ld<T>(dsmem_map(&m.rowj[e], owner_j));
      } else {
        misc[0] = dsmem_ld_s32(dsmem_map(&m.jnan, owner_j));
      }
    }
    __syncthreads();

    int qw = 0;
    T vb = cval[0];
    int ib = cidx[0];
    for (int s = 1; s < C; ++s)
      if (better(cval[s], cidx[s], vb, ib)) { vb = cval[s]; ib = cidx[s]; qw = s; }
    int p;
    const T* prow;
    if (misc[0]) {
      p = j;
      prow = rowj_st;
    } else {
      p = ib;
      prow = cand_all + qw * W;
    }
    const T piv = prow[j];
    if (q == 0 && tid == 0) {
      ipiv[c0 + j] = c0 + p;
      if (piv == T(0)) atomicCAS(status + 1, 0, c0 + j + 1);
    }

    // ---- swap, eliminate own rows, and scan column j+1 ----
    bv = T(-1);
    bi = INT_MAX;
#pragma unroll
    for (int u = 0; u < RPT; ++u) {
      const int r = tid + u * kLeafThreads;
      if (r < rcnt) {
        const int gr = rbeg + r;
        if (gr == j) {
#pragma unroll
          for (int c = 0; c < W; ++c) P[c * ldp + r] = prow[c];
        } else if (gr == p) {
#pragma unroll
          for (int c = 0; c < W; ++c) P[c * ldp + r] = rowj_st[c];
        }
        if (gr > j) {
          const T mult = P[j * ldp + r] / piv;
          P[j * ldp + r] = mult;
#pragma unroll
          for (int c = 1; c < W; ++c)
            if (c > j && c < w) P[c * ldp + r] = fma(-mult, prow[c], P[c * ldp + r]);
          if (j + 1 < w) {
            const T v = absval(P[(j + 1) * ldp + r]);
            if (better(v, gr, bv, bi)) { bv = v; bi = gr; }
          }
        }
      }
    }
  }
  // Nobody may leave while others can still read its mailbox.
  cluster_sync_all();
  __syncthreads();
  for (int i = tid; i < rcnt * W; i += kLeafThreads) {
    const int r = i / W, c = i % W;
    if (c < w) A[(long long)(c0 + rbeg + r) * lda + c0 + c] = P[c * ldp + r];
  }
}

int g_max_cluster[kMaxDevices] = {};

template <typename T, int W>
int launch_leaf(Ctx& c, T* A, long long lda, int n, int c0, int w, int* ipiv, cudaStream_t st) {
  const int R = n - c0;
  const int rpc_max = kLeafRowsTimesW / W;
  const int C = cdiv(R, rpc_max);
  const int rpc = cdiv(R, C);
  const size_t smem = LeafSmem<T, W>::bytes(rpc);
  auto kern = panel_leaf_kernel<T, W>;
  static bool attr_set[kMaxDevices] = {};
  const int dev = ctx_device(c);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)LeafSmem<T, W>::bytes(rpc_max)));
    LM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    attr_set[dev] = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C, 1, 1);
  cfg.blockDim = dim3(kLeafThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  LM_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, A, lda, n, c0, w, rpc, ipiv, ctx_status(c)));
  count_launch(1);
  return LM_OK;
}

// Largest cluster the device schedules for the leaf kernel (16 when allowed).
int max_cluster(Ctx& c) {
  const int dev = ctx_device(c);
  if (g_max_cluster[dev]) return g_max_cluster[dev];
  int best = 8;
  auto kern = panel_leaf_kernel<double, 16>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)LeafSmem<double, 16>::bytes(kLeafRowsTimesW / 16)) == cudaSuccess &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(16, 1, 1);
    cfg.blockDim = dim3(kLeafThreads, 1, 1);
    cfg.dynamicSmemBytes = LeafSmem<double, 16>::bytes(kLeafRowsTimesW / 16);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 16;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) == cudaSuccess && nclusters > 0) best = 16;
  }
  cudaGetLastError();
  g_max_cluster[dev] = best;
  return best;
}

}  // namespace

int panel_leaf_max_width_for(Ctx& c, int rows) {
  const long long cap = (long long)max_cluster(c) * kLeafRowsTimesW;  // rows * W per cluster
  for (int W = 32; W >= 4; W >>= 1)
    if ((long long)rows * W <= cap) return W;
  return 0;
}

template <typename T>
int panel_leaf(Ctx& c, T* A, long long lda, int n, int c0, int w, int* ipiv, cudaStream_t st) {
  if (w <= 0) return LM_OK;
  const int R = n - c0;
  const int wmax = panel_leaf_max_width_for(c, R);
  if (w > wmax || w > 32) return LM_ERR_UNSUPPORTED;
  // smallest compiled width that holds w
  if (w <= 4 && wmax >= 4) return launch_leaf<T, 4>(c, A, lda, n, c0, w, ipiv, st);
  if (w <= 8 && wmax >= 8) return launch_leaf<T, 8>(c, A, lda, n, c0, w, ipiv, st);
  if (w <= 16 && wmax >= 16) return launch_leaf<T, 16>(c, A, lda, n, c0, w, ipiv, st);
  return launch_leaf<T, 32>(c, A, lda, n, c0, w, ipiv, st);
}

template int panel_leaf<double>(Ctx&, double*, long long, int, int, int, int*, cudaStream_t);
template int panel_leaf<float>(Ctx&, float*, long long, int, int, int, int*, cudaStream_t);

// ---------------------------------------------------------------------------
// Cholesky of one diagonal block (w <= 128), right-looking in SMEM.
// ---------------------------------------------------------------------------
namespace {

template <typename T>
__global__ void __launch_bounds__(512) potrf_block_kernel(T* A, long long lda, int w, int base, int* status) {
  extern __shared__ __align__(16) unsigned char sm[];
  T* S = reinterpret_cast<T*>(sm);
  const int ld = w + 1;
  for (int i = threadIdx.x; i < w * w; i += blockDim.x) {
    const int r = i / w, c = i % w;
    if (c <= r) S[r * ld + c] = A[(long long)r * lda + c];
  }
  __syncthreads();
  for (int k = 0; k < w; ++k) {
    if (threadIdx.x == 0) {
      const T d = S[k * ld + k];
      if (!(d > T(0))) atomicCAS(status + 1, 0, base + k + 1);
      S[k * ld + k] = sqrt(d);
    }
    __syncthreads();
    const T skk = S[k * ld + k];
    for (int i = k + 1 + threadIdx.x; i < w; i += blockDim.x) S[i * ld + k] = S[i * ld + k] / skk;
    __syncthreads();
    const int m = w - k - 1;
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
      const int i = k + 1 + idx / m, jj = k + 1 + idx % m;
      if (jj <= i) S[i * ld + jj] = fma(-S[i * ld + k], S[jj * ld + k], S[i * ld + jj]);
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < w * w; i += blockDim.x) {
    const int r = i / w, c = i % w;
    if (c <= r) A[(long long)r * lda + c] = S[r * ld + c];
  }
}

}  // namespace

template <typename T>
int potrf_block(Ctx& c, T* A, long long lda, int w, int base, cudaStream_t st) {
  if (w <= 0) return LM_OK;
  if (w > 128) return LM_ERR_ARG;
  const size_t smem = sizeof(T) * (size_t)w * (w + 1);
  static bool attr_set[kMaxDevices] = {};
  const int dev = ctx_device(c);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(potrf_block_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(sizeof(T) * 128 * 129)));
    attr_set[dev] = true;
  }
  potrf_block_kernel<T><<<1, 512, smem, st>>>(A, lda, w, base, ctx_status(c));
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

template int potrf_block<double>(Ctx&, double*, long long, int, int, cudaStream_t);
template int potrf_block<float>(Ctx&, float*, long long, int, int, cudaStream_t);

}  // namespace lm
