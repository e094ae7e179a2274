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
//   Each thread keeps its rows in registers in a rotating layout (slot 0 is
//   always the current column; finished columns move to the end), so that
//   every column step runs the same compact code: a loop body specialised per
//   column index does not fit the instruction cache and made each step
//   fetch-bound.  Rows never move between threads: each carries its logical
//   row index, an interchange swaps two labels, and the write-back puts every
//   row at its final position.  So only the candidates travel per column; the
//   NaN rule for a_jj rides on the candidate of the CTA holding row j.
//   NaN rule of the reference scan: if |a_jj| is NaN it stays the pivot; NaNs
//   below it never win.
//
// potrf_block — Cholesky of one <=128 x 128 diagonal block in shared memory,
//   by 32-column panels (rawCholColumnSIMDFrom, K.hs:2137-2195, for a
//   diagonal panel).
#include <climits>

#include "common.cuh"
#include "internal.h"

namespace lm {

void count_launch(int n);

namespace {

constexpr int kLeafThreads = 512;
constexpr int kLeafRowsTimesW = 16384;  // rows per CTA * leaf width (128 KB of FP64)
static_assert(kLeafThreads / 32 >= 16, "one pushing warp per CTA of the largest (16-CTA) cluster");

template <typename T>
__device__ __forceinline__ T absval(T x) {
  T a = x < T(0) ? -x : x;
  return (a != a) ? T(-1) : a;  // NaN never wins the scan
}

// The pivot order of the reference's scan (strict '>' from row j down): the
// larger |a| wins, the lower row on ties, NaN never wins.  Scan values
// (absval's: -1 or >= 0) become integers in that order: 0 for -1, 1 for zero
// (either sign), the IEEE bits + 1 above, which grow with the value.  A warp then reduces (key, row) with three redux.sync
// instead of five shuffle rounds of (value, row) pairs.
template <typename T>
__device__ __forceinline__ unsigned long long scan_key(T v) {
  if (!(v >= T(0))) return 0ull;
  if (v == T(0)) return 1ull;
  if constexpr (sizeof(T) == 8)
    return (unsigned long long)__double_as_longlong((double)v) + 1ull;
  else
    return (unsigned long long)__float_as_uint((float)v) + 1ull;
}
// Row j with a NaN a_jj stays the pivot (the reference scan starts at row j
// and NaN never compares greater): its key beats every other.
constexpr unsigned long long kForcedKey = ~0ull;
// A key in the message's T-sized slot, bit for bit (float keys fit 32 bits).
template <typename T>
__device__ __forceinline__ T key_to_msg(unsigned long long k) {
  if constexpr (sizeof(T) == 8)
    return (T)__longlong_as_double((long long)k);
  else
    return (T)__uint_as_float(k == kForcedKey ? 0xffffffffu : (unsigned)k);
}
template <typename T>
__device__ __forceinline__ unsigned long long msg_to_key(T m) {
  if constexpr (sizeof(T) == 8) {
    return (unsigned long long)__double_as_longlong((double)m);
  } else {
    const unsigned b = __float_as_uint((float)m);
    return b == 0xffffffffu ? kForcedKey : (unsigned long long)b;
  }
}
// Every lane receives the warp's best (key, row) in the pivot order: the
// largest key, then the lowest row (rows are >= 0, or INT_MAX for none).
__device__ __forceinline__ void warp_best(unsigned long long& key, int& row) {
  // reconverge first: after the data-dependent branches and bounded spins of
  // a column step a warp can arrive split, and every *_sync below would then
  // serialise its halves
  __syncwarp();
  const unsigned khi = (unsigned)(key >> 32), klo = (unsigned)key;
  const unsigned hi = __reduce_max_sync(0xffffffffu, khi);
  const unsigned lo = __reduce_max_sync(0xffffffffu, khi == hi ? klo : 0u);
  const unsigned long long best = ((unsigned long long)hi << 32) | lo;
  row = (int)__reduce_min_sync(0xffffffffu, key == best ? (unsigned)row : 0xffffffffu);
  key = best;
}

// Per-column message pushed into every CTA of the cluster (T elements), one
// per source CTA: [0] the scan key of its best candidate (bit pattern, see
// scan_key; kForcedKey when that row is row j with a NaN a_jj), [1] that
// row's logical index relative to c0 (or -1), [2..3] unused, [4, 4 + W) the
// row in the rotated register layout.
template <typename T, int W>
struct LeafMsg {
  static constexpr int N = 4 + W;
  static constexpr int BYTES = N * (int)sizeof(T);
  static constexpr int CHUNKS = BYTES / 16;
  static constexpr int PER_CHUNK = 16 / (int)sizeof(T);
  static_assert(BYTES % 16 == 0, "message must be a whole number of 16-byte chunks");
};

template <typename T, int W>
struct LeafSmem {
  using M = LeafMsg<T, W>;
  static constexpr size_t cand_off = 0;                                    // T[2][16][N]
  static constexpr size_t outc_off = cand_off + 2 * 16 * (size_t)M::BYTES;  // T[N] outgoing candidate
  static constexpr size_t bar_off = outc_off + (size_t)M::BYTES;            // uint64_t[2]
  static constexpr size_t wkey_off = bar_off + 16;                          // uint64_t[16] warp best keys
  static constexpr size_t widx_off = wkey_off + 16 * sizeof(unsigned long long);  // int[16] their rows
  static constexpr size_t hist_off = widx_off + 16 * sizeof(int);           // int[W] pivot rows
  static constexpr size_t trow_off = hist_off + W * sizeof(int);            // int[2W] touched rows
  static constexpr size_t tsrc_off = trow_off + 2 * W * sizeof(int);        // int[2W] their sources
  static constexpr size_t tm_off = tsrc_off + 2 * W * sizeof(int);          // int touched count
  static constexpr size_t stage_off = (tm_off + sizeof(int) + 15) / 16 * 16;
  // One region, used twice: first the CTA's slab (rpc rows x W, row stride
  // W + 1) for coalesced loads and write-back, followed by the rows' final
  // logical indices (rpc ints), then the swap staging for the other panel
  // columns (2W rows x up to 128 columns, split over the cluster).
  static constexpr int SLD = W + 1;
  static size_t stage_elems(int C) { return (size_t)(2 * W * 128 + C - 1) / C; }
  __host__ __device__ static size_t slab_elems(int rpc) { return (size_t)rpc * SLD; }
  static size_t region_elems(int rpc, int C) {
    const size_t slab = slab_elems(rpc) + ((size_t)rpc * sizeof(int) + sizeof(T) - 1) / sizeof(T);
    return slab > stage_elems(C) ? slab : stage_elems(C);
  }
  static size_t bytes(int rpc, int C) { return stage_off + region_elems(rpc, C) * sizeof(T); }
};

template <typename T>
__device__ __forceinline__ void pack16(const T* src, uint32_t (&w)[4]) {
  if constexpr (sizeof(T) == 8) {
    const unsigned long long a = (unsigned long long)__double_as_longlong((double)src[0]);
    const unsigned long long b = (unsigned long long)__double_as_longlong((double)src[1]);
    w[0] = (uint32_t)a; w[1] = (uint32_t)(a >> 32); w[2] = (uint32_t)b; w[3] = (uint32_t)(b >> 32);
  } else {
    w[0] = __float_as_uint((float)src[0]); w[1] = __float_as_uint((float)src[1]);
    w[2] = __float_as_uint((float)src[2]); w[3] = __float_as_uint((float)src[3]);
  }
}

// Push a message staged in this CTA's shared memory (`msg`) to the same
// offset `slot` in CTA d of the cluster, completing on its `bar`; one lane
// per 16-byte chunk.
template <typename T, int W>
__device__ __forceinline__ void push_one(const T* msg, T* slot, uint64_t* bar, int d, int lane) {
  using M = LeafMsg<T, W>;
  static_assert(M::CHUNKS <= 32, "one chunk per lane");
  if (lane < M::CHUNKS) {
    uint32_t w4[4];
    pack16<T>(msg + lane * M::PER_CHUNK, w4);
    st_async_16(dsmem_map(slot, d) + lane * 16, dsmem_map(bar, d), w4[0], w4[1], w4[2], w4[3]);
  }
}

template <typename T, int W>
__global__ void __launch_bounds__(kLeafThreads, 1)
    panel_leaf_kernel(T* A, long long lda, int n, int c0, int w, int rpc, int pc0, int pw, int* ipiv,
                      int* status) {
  using L = LeafSmem<T, W>;
  using M = LeafMsg<T, W>;
  extern __shared__ __align__(16) unsigned char sm[];
  T* cand = reinterpret_cast<T*>(sm + L::cand_off);
  T* outc = reinterpret_cast<T*>(sm + L::outc_off);
  uint64_t* rbar = reinterpret_cast<uint64_t*>(sm + L::bar_off);
  unsigned long long* wkey = reinterpret_cast<unsigned long long*>(sm + L::wkey_off);
  int* widx = reinterpret_cast<int*>(sm + L::widx_off);
  int* hist = reinterpret_cast<int*>(sm + L::hist_off);
  int* trow = reinterpret_cast<int*>(sm + L::trow_off);
  int* tsrc = reinterpret_cast<int*>(sm + L::tsrc_off);
  int* tm = reinterpret_cast<int*>(sm + L::tm_off);
  T* stage = reinterpret_cast<T*>(sm + L::stage_off);

  const int q = (int)cluster_ctarank();
  const int C = (int)cluster_nctarank();
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int R = n - c0;
  const int rbeg = q * rpc;
  const int rcnt = max(0, min(rpc, R - rbeg));
  constexpr int RPT = kLeafRowsTimesW / W / kLeafThreads;  // rows per thread (= 32 / W)
  static_assert(RPT * W == kLeafRowsTimesW / kLeafThreads, "slab must split evenly");

  if (tid == 0) {
    mbar_init(&rbar[0], 1);
    mbar_init(&rbar[1], 1);
    fence_barrier_init();
  }
  // This thread's rows of the slab, in registers: row r = tid + u * threads.
  // The slab through shared memory: each warp instruction reads 32 / W whole
  // rows (coalesced), then every thread takes its rows from there.
  constexpr int SLD = L::SLD;
  constexpr int RPI = 32 / W;  // rows per warp instruction
  T* slab = stage;
  for (int r = warp * RPI + lane / W; r < rcnt; r += (kLeafThreads / 32) * RPI) {
    const int c = lane % W;
    slab[r * SLD + c] = c < w ? A[(long long)(c0 + rbeg + r) * lda + c0 + c] : T(0);
  }
  __syncthreads();
  T x[RPT][W];
#pragma unroll
  for (int u = 0; u < RPT; ++u) {
    const int r = tid + u * kLeafThreads;
#pragma unroll
    for (int c = 0; c < W; ++c) x[u][c] = r < rcnt ? slab[r * SLD + c] : T(0);
  }
  cluster_sync_all();  // every CTA's barriers exist before anyone pushes into them

  // logical row (relative to c0) of each of this thread's rows
  int lr[RPT];
#pragma unroll
  for (int u = 0; u < RPT; ++u) lr[u] = rbeg + tid + u * kLeafThreads;
  // this thread's best candidate for the next column: (key, logical row)
  unsigned long long bk = 0ull;
  int bi = INT_MAX;
#pragma unroll
  for (int u = 0; u < RPT; ++u) {
    const int r = tid + u * kLeafThreads;
    if (r < rcnt) {
      const unsigned long long k = scan_key(absval(x[u][0]));
      if (k > bk || (k == bk && lr[u] < bi)) { bk = k; bi = lr[u]; }
    }
  }

  bool timed_out = false;
  // Column j's step.  Register layout of a row at step j: slot c < W - j holds
  // column j + c, slot W - j + i holds the finished column i.
#pragma unroll 1
  for (int j = 0; j < w; ++j) {
    const int par = j & 1;
    if (tid == 0) mbar_arrive_expect_tx(&rbar[par], (uint32_t)(C * M::BYTES));
    // row j with a NaN a_jj is this CTA's candidate whatever else it holds
#pragma unroll
    for (int u = 0; u < RPT; ++u) {
      const int r = tid + u * kLeafThreads;
      if (r < rcnt && lr[u] == j && x[u][0] != x[u][0]) { bk = kForcedKey; bi = j; }
    }
    // ---- CTA argmax: warp reduction, one barrier, every warp reduces ----
    warp_best(bk, bi);
    if (lane == 0) { wkey[warp] = bk; widx[warp] = bi; }
    __syncthreads();
    {
      const unsigned long long k0 = lane < kLeafThreads / 32 ? wkey[lane] : 0ull;
      const int i0 = lane < kLeafThreads / 32 ? widx[lane] : INT_MAX;
      unsigned long long k = k0;
      int i = i0;
      warp_best(k, i);
      // the warp holding the CTA's best row stages and pushes it (warp 0 if none)
      const int wo = i == INT_MAX ? 0 : __ffs(__ballot_sync(0xffffffffu, k0 == k && i0 == i)) - 1;
      if (warp == wo) {
        if (i != INT_MAX) {
#pragma unroll
          for (int u = 0; u < RPT; ++u)
            if (tid + u * kLeafThreads < rcnt && lr[u] == i) {
#pragma unroll
              for (int c = 0; c < W; ++c) outc[4 + c] = x[u][c];
            }
        } else if (lane < W) {
          outc[4 + lane] = T(0);
        }
        if (lane == 0) {
          outc[0] = key_to_msg<T>(k);
          outc[1] = i != INT_MAX ? T(i) : T(-1);
          outc[2] = T(0);
          outc[3] = T(0);
        }
      }
    }
    // the staged candidate goes out from C warps at once: warp d sends it to
    // CTA d, one 16-byte chunk per lane (one warp sending all C copies took
    // about 900 cycles per column)
    __syncthreads();
    if (warp < C) push_one<T, W>(outc, cand + ((size_t)par * 16 + q) * M::N, &rbar[par], warp, lane);
    // ---- wait for the C candidates ----
    if (!timed_out && !mbar_wait_spin(&rbar[par], (uint32_t)((j >> 1) & 1), status)) timed_out = true;

    const T* rc = cand + (size_t)par * 16 * M::N;
    int i = lane < C ? (int)rc[lane * M::N + 1] : INT_MAX;
    if (i < 0) i = INT_MAX;
    int qw;
    {
      const unsigned long long mine = lane < C ? msg_to_key(rc[lane * M::N + 0]) : 0ull;
      const int my_row = i;
      unsigned long long k = mine;
      warp_best(k, i);
      qw = __ffs(__ballot_sync(0xffffffffu, mine == k && my_row == i)) - 1;  // the winning CTA
    }
    // (row j itself is always a candidate, so some CTA wins; the fallback
    // only keeps the indexing in bounds)
    const int p = (i == INT_MAX || qw >= C) ? j : i;
    const T* prow = rc + ((i == INT_MAX || qw >= C) ? 0 : qw) * M::N + 4;
    const T piv = prow[0];
    if (tid == 0) hist[j] = p;
    if (q == 0 && tid == 0) {
      ipiv[c0 + j] = c0 + p;
      if (piv == T(0)) atomicCAS(status + 1, 0, c0 + j + 1);
    }

    // ---- interchange labels, eliminate own rows in registers, scan column j+1 ----
    bk = 0ull;
    bi = INT_MAX;
#pragma unroll
    for (int u = 0; u < RPT; ++u) {
      const int r = tid + u * kLeafThreads;
      if (r < rcnt) {
        if (lr[u] == p)
          lr[u] = j;
        else if (lr[u] == j)
          lr[u] = p;
        if (lr[u] > j) {
          const T mult = x[u][0] / piv;
          x[u][0] = mult;
#pragma unroll
          for (int c = 1; c < W; ++c)
            if (c < W - j) x[u][c] = fma(-mult, prow[c], x[u][c]);
          if (j + 1 < w) {
            const unsigned long long k1 = scan_key(absval(x[u][1]));
            if (k1 > bk || (k1 == bk && lr[u] < bi)) { bk = k1; bi = lr[u]; }
          }
        }
      }
      // column j's final value moves to the end
      const T t0 = x[u][0];
#pragma unroll
      for (int c = 0; c + 1 < W; ++c) x[u][c] = x[u][c + 1];
      x[u][W - 1] = t0;
    }
    // The buffers of this parity are rewritten two columns later; the
    // barrier at the top of the next column orders these reads before this
    // CTA pushes again, and no CTA can run two columns ahead of another.
  }
  // a leaf narrower than W stops w steps into the rotation: finish it
#pragma unroll 1
  for (int k = w; k < W; ++k)
#pragma unroll
    for (int u = 0; u < RPT; ++u) {
      const T t0 = x[u][0];
#pragma unroll
      for (int c = 0; c + 1 < W; ++c) x[u][c] = x[u][c + 1];
      x[u][W - 1] = t0;
    }
  // Nobody may leave while others can still write into it.
  cluster_sync_all();
  // write-back through the slab, coalesced like the load, each row to its
  // logical position
  int* lrow = reinterpret_cast<int*>(slab + L::slab_elems(rpc));
#pragma unroll
  for (int u = 0; u < RPT; ++u) {
    const int r = tid + u * kLeafThreads;
    if (r < rcnt) {
#pragma unroll
      for (int c = 0; c < W; ++c) slab[r * SLD + c] = x[u][c];
      lrow[r] = lr[u];
    }
  }
  __syncthreads();
  for (int r = warp * RPI + lane / W; r < rcnt; r += (kLeafThreads / 32) * RPI) {
    const int c = lane % W;
    if (c < w) A[(long long)(c0 + lrow[r]) * lda + c0 + c] = slab[r * SLD + c];
  }
  __syncthreads();  // the region is the swap staging from here on
  // This leaf's interchanges on the other columns of the enclosing panel
  // [pc0, pc0 + pw): compose them (rows relative to c0), gather every touched
  // row's source over the cluster, barrier, scatter.
  const int ocols = pw - w;
  if (ocols > 0) {
    // Touched rows: 0 .. w-1, then each pivot row >= w in order of first
    // use; the source of row r is tau_0(tau_1(... tau_{w-1}(r))), walking
    // the interchanges backwards.  One warp (w <= 32).
    if (warp == 0) {
      const int pr = lane < w ? hist[lane] : -1;
      bool fresh = lane < w && pr >= w;
      for (int jj = 0; jj < lane && jj < w; ++jj)
        if (hist[jj] == pr) fresh = false;
      __syncwarp();
      const unsigned bal = __ballot_sync(0xffffffffu, fresh);
      if (lane < w) trow[lane] = lane;
      if (fresh) trow[w + __popc(bal & ((1u << lane) - 1u))] = pr;
      const int m = w + __popc(bal);
      __syncwarp();
      for (int e = lane; e < m; e += 32) {
        int r = trow[e];
        for (int jj = w - 1; jj >= 0; --jj) {
          const int h = hist[jj];
          if (r == jj) r = h;
          else if (r == h) r = jj;
        }
        tsrc[e] = r;
      }
      if (lane == 0) *tm = m;
    }
    __syncthreads();
    const int m = *tm;
    const long long total = (long long)m * ocols;
    const long long chunk = (total + C - 1) / C;
    const long long e0 = q * chunk, e1 = min(total, e0 + chunk);
    const int left = c0 - pc0;  // other columns: [pc0, c0) then [c0 + w, pc0 + pw)
#pragma unroll 4
    for (long long e = e0 + tid; e < e1; e += kLeafThreads) {
      const int ii = (int)(e / ocols), oc = (int)(e % ocols);
      const int col = oc < left ? pc0 + oc : c0 + w + (oc - left);
      if (tsrc[ii] != trow[ii]) stage[e - e0] = A[(long long)(c0 + tsrc[ii]) * lda + col];
    }
    cluster_sync_all();
    for (long long e = e0 + tid; e < e1; e += kLeafThreads) {
      const int ii = (int)(e / ocols), oc = (int)(e % ocols);
      const int col = oc < left ? pc0 + oc : c0 + w + (oc - left);
      if (tsrc[ii] != trow[ii]) A[(long long)(c0 + trow[ii]) * lda + col] = stage[e - e0];
    }
  }
}

int g_max_cluster[kMaxDevices] = {};

template <typename T, int W>
int launch_leaf(Ctx& c, T* A, long long lda, int n, int c0, int w, int pc0, int pw, int* ipiv, cudaStream_t st) {
  const int R = n - c0;
  const int rpc_max = kLeafRowsTimesW / W;
  const int C = cdiv(R, rpc_max);
  const int rpc = cdiv(R, C);
  const size_t smem = LeafSmem<T, W>::bytes(rpc, C);
  auto kern = panel_leaf_kernel<T, W>;
  static bool attr_set[kMaxDevices] = {};
  const int dev = ctx_device(c);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)LeafSmem<T, W>::bytes(rpc_max, 1)));
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
  LM_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, A, lda, n, c0, w, rpc, pc0, pw, ipiv, ctx_status(c)));
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
                           (int)LeafSmem<double, 16>::bytes(kLeafRowsTimesW / 16, 1)) == cudaSuccess &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(16, 1, 1);
    cfg.blockDim = dim3(kLeafThreads, 1, 1);
    cfg.dynamicSmemBytes = LeafSmem<double, 16>::bytes(kLeafRowsTimesW / 16, 16);
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
int panel_leaf(Ctx& c, T* A, long long lda, int n, int c0, int w, int pc0, int pw, int* ipiv, cudaStream_t st) {
  if (w <= 0) return LM_OK;
  const int R = n - c0;
  const int wmax = panel_leaf_max_width_for(c, R);
  if (w > wmax || w > 32) return LM_ERR_UNSUPPORTED;
  // smallest compiled width that holds w
  if (pw > 128 || pc0 > c0 || pc0 + pw < c0 + w) return LM_ERR_ARG;
  if (w <= 4 && wmax >= 4) return launch_leaf<T, 4>(c, A, lda, n, c0, w, pc0, pw, ipiv, st);
  if (w <= 8 && wmax >= 8) return launch_leaf<T, 8>(c, A, lda, n, c0, w, pc0, pw, ipiv, st);
  if (w <= 16 && wmax >= 16) return launch_leaf<T, 16>(c, A, lda, n, c0, w, pc0, pw, ipiv, st);
  return launch_leaf<T, 32>(c, A, lda, n, c0, w, pc0, pw, ipiv, st);
}

template int panel_leaf<double>(Ctx&, double*, long long, int, int, int, int, int, int*, cudaStream_t);
template int panel_leaf<float>(Ctx&, float*, long long, int, int, int, int, int, int*, cudaStream_t);

// ---------------------------------------------------------------------------
// Cholesky of one diagonal block (w <= 128), by 32-column panels in shared memory.
// ---------------------------------------------------------------------------
namespace {

// Cholesky of the w x w block at A (w <= 128, lower triangle) in place, in
// shared memory, right-looking by 32-column panels (padded to whole panels
// with the identity).  Per panel c0:
//   1. warp 0 factors the 32 x 32 diagonal block in registers: lane i holds
//      row i; step k broadcasts a_kk, forms r = 1 / sqrt(a_kk), l_ik = a_ik r
//      (l_kk = a_kk r) and subtracts l_ik l_jk from the lanes' later columns
//      with one shuffle per column (steps unrolled at compile time so the row
//      stays in registers: 256 threads leave room for it); r is kept for the
//      panel solve;
//   2. one thread per row below solves x = a L11^-T by the same products
//      (x_k = (a_k - sum_{j<k} x_j l_kj) r_k);
//   3. all threads subtract X X^T from the lower trailing block in 4 x 4
//      register tiles.
// A non-positive (or NaN) pivot is recorded as base + k + 1 in status[1]
// (the first one: panels and steps run in order); the arithmetic continues,
// leaving the NaN the reference's would.
constexpr int kPbLd = 129;  // padded row stride of the shared copy (elements)
constexpr int kPbXt = 96;   // row stride of the transposed panel X^T (elements)
constexpr int kPbThreads = 256;

template <typename T>
constexpr int potrf_block_smem() {
  return (128 * kPbLd + 32 * kPbXt) * (int)sizeof(T);
}

// Step K of the one-warp 32 x 32 Cholesky (lane i holds row i in d), with
// K a compile-time constant so that d stays in registers.
template <typename T, int K>
__device__ __forceinline__ void pb_diag_step(T (&d)[32], int lane, int& bad, T& myr) {
  if constexpr (K < 32) {
    const T dkk = __shfl_sync(0xffffffffu, d[K], K);
    bad = (bad < 0 && !(dkk > T(0))) ? K : bad;  // the same in every lane
    const T r = rsqrt(dkk);
    const T lk = d[K] * r;
    d[K] = lane >= K ? lk : d[K];
    myr = lane == K ? r : myr;
#pragma unroll
    for (int j = K + 1; j < 32; ++j) {
      const T lj = __shfl_sync(0xffffffffu, lk, j);
      d[j] = lane >= j ? fma(-lk, lj, d[j]) : d[j];
    }
    pb_diag_step<T, K + 1>(d, lane, bad, myr);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) potrf_block_kernel(T* A, long long lda, int w, int base, int* status) {
  extern __shared__ __align__(16) unsigned char pb_smem[];
  T* S = reinterpret_cast<T*>(pb_smem);  // 128 x kPbLd, lower triangle
  T* Xt = S + 128 * kPbLd;               // 32 x kPbXt: the solved panel, transposed
  __shared__ T rdiag[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int np = (w + 31) >> 5;  // panels
  const int wp = np << 5;        // padded order
  for (int e = tid; e < wp * wp; e += kPbThreads) {
    const int i = e / wp, j = e % wp;
    T v = T(0);
    if (j <= i) v = (i < w) ? A[(long long)i * lda + j] : (i == j ? T(1) : T(0));
    S[i * kPbLd + j] = v;
  }
  __syncthreads();
#pragma unroll 1
  for (int p = 0; p < np; ++p) {
    const int c0 = p << 5;
    // ---- 1. diagonal block, one warp (selects, not branches: the warp
    //         stays converged for its shuffles) ----
    if (warp == 0) {
      T d[32];
      T* row = S + (c0 + lane) * kPbLd + c0;
#pragma unroll
      for (int j = 0; j < 32; ++j) d[j] = row[j];
      int bad = -1;
      T myr = T(0);
      pb_diag_step<T, 0>(d, lane, bad, myr);
      rdiag[lane] = myr;
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j <= lane) row[j] = d[j];
      if (lane == 0 && bad >= 0 && c0 + bad < w) atomicCAS(status + 1, 0, base + c0 + bad + 1);
    }
    __syncthreads();
    const int m = wp - c0 - 32;  // rows below the diagonal block
    if (m <= 0) break;
    // ---- 2. panel solve, one thread per row: x = a L11^-T ----
    if (tid < m) {
      T* row = S + (c0 + 32 + tid) * kPbLd + c0;
      const T* L = S + c0 * kPbLd + c0;
      T a[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) a[j] = row[j];
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        const T x = a[k] * rdiag[k];
        a[k] = x;
#pragma unroll
        for (int j = k + 1; j < 32; ++j) a[j] = fma(-x, L[j * kPbLd + k], a[j]);
      }
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        row[j] = a[j];
        Xt[j * kPbXt + tid] = a[j];
      }
    }
    __syncthreads();
    // ---- 3. trailing update, 4 x 4 register tiles of the lower triangle ----
    const int tt = m >> 2;                 // tiles per side
    const int ntiles = tt * (tt + 1) / 2;  // tile (ti, tj), tj <= ti, at t = ti (ti + 1) / 2 + tj
    for (int t = tid; t < ntiles; t += kPbThreads) {
      int ti = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
      while (ti > 0 && ti * (ti + 1) / 2 > t) --ti;
      while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
      const int tj = t - ti * (ti + 1) / 2;
      const int ri = 4 * ti, rj = 4 * tj;  // rows within the trailing block
      const int i0 = c0 + 32 + ri, j0 = c0 + 32 + rj;
      T acc[4][4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = S[(i0 + u) * kPbLd + j0 + v];
#pragma unroll 8
      for (int k = 0; k < 32; ++k) {
        T xi[4], xj[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          xi[u] = Xt[k * kPbXt + ri + u];
          xj[u] = Xt[k * kPbXt + rj + u];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[u][v] = fma(-xi[u], xj[v], acc[u][v]);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v)
          if (j0 + v <= i0 + u) S[(i0 + u) * kPbLd + j0 + v] = acc[u][v];
    }
    __syncthreads();
  }
  for (int e = tid; e < w * w; e += kPbThreads) {
    const int i = e / w, j = e % w;
    if (j <= i) A[(long long)i * lda + j] = S[i * kPbLd + j];
  }
}

}  // namespace

template <typename T>
int potrf_block(Ctx& c, T* A, long long lda, int w, int base, cudaStream_t st) {
  if (w <= 0) return LM_OK;
  if (w > 128) return LM_ERR_ARG;
  constexpr int smem = potrf_block_smem<T>();
  static bool attr_set[kMaxDevices] = {};
  const int dev = ctx_device(c);
  if (!attr_set[dev]) {
    LM_CUDA_TRY(cudaFuncSetAttribute(potrf_block_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr_set[dev] = true;
  }
  potrf_block_kernel<T><<<1, kPbThreads, smem, st>>>(A, lda, w, base, ctx_status(c));
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

template int potrf_block<double>(Ctx&, double*, long long, int, int, cudaStream_t);
template int potrf_block<float>(Ctx&, float*, long long, int, int, cudaStream_t);

}  // namespace lm
