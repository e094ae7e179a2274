// Triangular solves with few right-hand sides as one persistent launch per
// direction (the refinement loop's substitutions; counterpart of the packed
// substitutions rawForwardSubUnitPackedSIMD / rawBackSubPackedSIMD,
// K.hs:2205-2314).
//
//   tri_inv_blocks : inverts every BS x BS diagonal block of L (unit lower)
//                    and U (upper) once per factorisation;
//   trsv_kernel    : row-block b (taken in dependency order through an atomic
//                    ticket, so a block only ever waits on blocks that are
//                    already running) accumulates  y_b = rhs_b - sum_j T_bj x_j
//                    over its dependencies in the order they complete, then
//                    x_b = inv(T_bb) y_b, publishes x_b and advances the
//                    direction's progress counter (blocks finish in ticket
//                    order, so one counter says which x_j are ready).
// Each T_bj tile is constant and is loaded before waiting on x_j; the
// right-hand side and inv(T_bb) are loaded before the first wait.  Every wait
// is bounded (kSpinLimit polls, then LM_DEVERR_TIMEOUT).
//
// Diagonal blocks: FP32 multiplies by the precomputed inverse (the refinement
// loop absorbs its rounding); FP64, the drop-in path, solves the diagonal block
// by substitution in one warp (column sweep over a shared-memory copy of
// T_bb), so its accuracy is that of the reference's substitutions
// (LU.hs:493-507, K.hs:2205-2314) rather than that of an explicit inverse.
//
// Block size: 128 rows for FP32 (512 threads), 64 for FP64 (256 threads).
// Thread (r, q) of a block owns row r and, of every tile, the float4/double2
// groups at columns 16 v + 4 q (FP32) so that the four threads of a row read
// 64 contiguous bytes per load instruction.
#include <algorithm>

#include "common.cuh"
#include "internal.h"

namespace lm {

void count_launch(int n);

namespace {

constexpr int MAX_RHS = 4;    // one pass, both precisions
constexpr int WIDE_RHS = 16;  // one pass of the FP32 wide variant

template <typename T>
struct TrsvCfg;
template <>
struct TrsvCfg<float> {
  static constexpr int BS = 128, NT = 512, VEC = 4;  // VEC elements per 16-byte load
};
template <>
struct TrsvCfg<double> {
  static constexpr int BS = 64, NT = 256, VEC = 2;
};

// Dynamic shared memory of trsv_kernel when the diagonal block is solved by
// substitution.  Lane l of the solving warp owns the RPL consecutive rows
// RPL l .. RPL l + RPL - 1; the block is stored as RPL x RPL tiles, tile (l, s)
// (rows of lane l, columns of lane s) at tile index s * 32 + l, padded so that
// the 16-byte loads of one tile row by consecutive lanes hit distinct banks.
template <typename T>
struct TrsvDiag {
  static constexpr int RPL = TrsvCfg<T>::BS / 32;
  static constexpr int TS = RPL * RPL + 16 / (int)sizeof(T);  // tile stride in elements
  T tile[32 * 32 * TS];
  T rdiag[TrsvCfg<T>::BS];  // 1 / T_kk, formed before the first wait
};

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
template <typename T>
__device__ __forceinline__ T ld_volatile(const T* p) {
  return *reinterpret_cast<const volatile T*>(p);
}

// inv of the b-th diagonal block of the unit-lower (lower = 1) or upper
// (lower = 0) factor, row-major BS x BS into Dinv + b * BS * BS.
template <typename T>
__global__ void __launch_bounds__(TrsvCfg<T>::NT) tri_inv_blocks_kernel(const T* __restrict__ LU, long long lda,
                                                                       int n, int lower, T* Dinv) {
  constexpr int BS = TrsvCfg<T>::BS, NT = TrsvCfg<T>::NT, RG = NT / BS;
  extern __shared__ __align__(16) unsigned char inv_smem[];
  T(*Ts)[BS + 1] = reinterpret_cast<T(*)[BS + 1]>(inv_smem);
  T(*Xs)[BS + 1] = Ts + BS;
  const int b = blockIdx.x;
  const int r0 = b * BS;
  const int w = min(BS, n - r0);
  for (int i = threadIdx.x; i < BS * BS; i += NT) {
    const int r = i / BS, c = i % BS;
    T t = T(0);
    if (r < w && c < w) {
      const T v = LU[(long long)(r0 + r) * lda + r0 + c];
      if (lower)
        t = (c < r) ? v : (c == r ? T(1) : T(0));
      else
        t = (c >= r) ? v : T(0);
    } else if (r == c) {
      t = T(1);  // pad the last block with the identity
    }
    Ts[r][c] = t;
    Xs[r][c] = (r == c) ? T(1) : T(0);
  }
  __syncthreads();
  const int c = threadIdx.x % BS;   // column of X this thread updates
  const int rg = threadIdx.x / BS;  // row group
  if (lower) {
    for (int k = 0; k < BS; ++k) {  // rows i > k:  X[i] -= L[i][k] X[k]
      const T xk = Xs[k][c];
      for (int i = k + 1 + ((rg - (k + 1)) % RG + RG) % RG; i < BS; i += RG) Xs[i][c] = fma(-Ts[i][k], xk, Xs[i][c]);
      __syncthreads();
    }
  } else {
    for (int k = BS - 1; k >= 0; --k) {  // X[k] /= U[k][k]; rows i < k: X[i] -= U[i][k] X[k]
      if (threadIdx.x < BS) Xs[k][threadIdx.x] = Xs[k][threadIdx.x] / Ts[k][k];
      __syncthreads();
      const T xk = Xs[k][c];
      for (int i = rg; i < k; i += RG) Xs[i][c] = fma(-Ts[i][k], xk, Xs[i][c]);
      __syncthreads();
    }
  }
  T* D = Dinv + (size_t)b * BS * BS;
  for (int i = threadIdx.x; i < BS * BS; i += NT) D[i] = Xs[i / BS][i % BS];
}

// Loads this thread's share of a BS-wide slice of row `src` (columns c0 ..):
// groups of VEC at c0 + 4 VEC v + VEC q, v = 0 .. BS/(4 VEC) - 1.
template <typename T>
__device__ __forceinline__ void load_row_share(T* out, const T* src, int c0, int q, int n, bool row_ok,
                                               bool vec_ok) {
  constexpr int BS = TrsvCfg<T>::BS, VEC = TrsvCfg<T>::VEC, G = BS / (4 * VEC);
#pragma unroll
  for (int v = 0; v < G; ++v) {
    const int c = c0 + 4 * VEC * v + VEC * q;
    if (vec_ok && row_ok && c + VEC <= n) {
      if constexpr (VEC == 4) {
        const float4 x = *reinterpret_cast<const float4*>(src + c);
        out[4 * v] = x.x, out[4 * v + 1] = x.y, out[4 * v + 2] = x.z, out[4 * v + 3] = x.w;
      } else {
        const double2 x = *reinterpret_cast<const double2*>(src + c);
        out[2 * v] = x.x, out[2 * v + 1] = x.y;
      }
    } else {
#pragma unroll
      for (int e = 0; e < VEC; ++e) out[VEC * v + e] = (row_ok && c + e < n) ? src[c + e] : T(0);
    }
  }
}

// One direction of the blocked substitution.  forward: L unit lower, blocks in
// increasing order; backward: U upper, blocks in decreasing order.
// sync[0] = progress counter, sync[1] = ticket dispenser (both zero at launch).
// EXACT: the diagonal block is solved by substitution (backward stable, as
// the reference's substitutions are); otherwise it is multiplied by its
// precomputed inverse Dinv.
// corr (inverse form only): per-block flags at stride 2; when given, the
// correction step on the diagonal block runs only for blocks whose flag is
// set.  The 16-column variant never takes the correction step.
template <typename T, int RHS, bool EXACT, bool FWD>
__global__ void __launch_bounds__(TrsvCfg<T>::NT) trsv_kernel(const T* __restrict__ LU, long long lda, int n,
                                                             int nrhs, const T* __restrict__ Dinv,
                                                             T* X, long long ldx, int* sync, int* status,
                                                             int vec_ok, const int* corr, int unit_l) {
  constexpr int MAX_RHS = RHS;
  constexpr int BS = TrsvCfg<T>::BS, NT = TrsvCfg<T>::NT, VEC = TrsvCfg<T>::VEC, CP = BS / 4;
  constexpr int RPL = BS / 32;  // rows per lane of the one-warp substitution
  constexpr bool forward = FWD;  // the direction is a compile-time constant
  static_assert(NT == 4 * BS, "four threads per row");
  __shared__ int tk_sh, prog_sh;
  // rows padded by one element: the four threads of a row read columns 4 q
  // apart, which an unpadded power-of-two row length puts in one bank
  constexpr int XS = MAX_RHS + 1;
  __shared__ T xj[2][BS][XS];
  __shared__ T ys[BS][XS];
  extern __shared__ __align__(16) unsigned char trsv_dyn[];
  TrsvDiag<T>& diag = *reinterpret_cast<TrsvDiag<T>*>(trsv_dyn);
  const int nb = (n + BS - 1) / BS;
  if (threadIdx.x == 0) tk_sh = atomicAdd(sync + 1, 1);
  __syncthreads();
  const int t = tk_sh;
  const int b = forward ? t : nb - 1 - t;
  const int r0 = b * BS;
  const int rows = min(BS, n - r0);
  const int r = threadIdx.x >> 2, q = threadIdx.x & 3;
  const bool row_ok = r < rows;
  // column index of the e-th element of this thread's share
  auto col_of = [&](int e) { return 4 * VEC * (e / VEC) + VEC * q + (e % VEC); };

  T rhs[MAX_RHS];
#pragma unroll
  for (int h = 0; h < MAX_RHS; ++h) rhs[h] = (q == 0 && row_ok && h < nrhs) ? X[(long long)(r0 + r) * ldx + h] : T(0);
  T dv[EXACT ? 1 : CP];
  if constexpr (EXACT) {
    // T_bb with the unit (forward) or the stored (backward) diagonal; the
    // padding of a ragged last block is the identity.
    constexpr int TS = TrsvDiag<T>::TS;
    for (int i = threadIdx.x; i < BS * BS; i += NT) {
      const int rr = i / BS, cc = i % BS;
      T v = T(0);
      if (rr < rows && cc < rows) {
        if (forward ? (cc < rr || (!unit_l && cc == rr)) : cc >= rr) v = LU[(long long)(r0 + rr) * lda + r0 + cc];
        if (forward && unit_l && cc == rr) v = T(1);
      } else if (rr == cc) {
        v = T(1);
      }
      diag.tile[((cc / RPL) * 32 + rr / RPL) * TS + (rr % RPL) * RPL + cc % RPL] = v;
      if (rr == cc) diag.rdiag[rr] = T(1) / v;
    }
  } else {
    load_row_share<T>(dv, Dinv + (size_t)b * BS * BS + (size_t)r * BS, 0, q, BS, true, true);
  }

  T acc[MAX_RHS];
#pragma unroll
  for (int h = 0; h < MAX_RHS; ++h) acc[h] = T(0);
  const int ndep = forward ? b : nb - 1 - b;  // dependencies = tickets 0 .. t-1
  int known = 0;
  bool ok = true;
  for (int d = 0; d < ndep; ++d) {
    const int j = forward ? d : nb - 1 - d;  // ticket d, in completion order
    T tv[CP];
    load_row_share<T>(tv, LU + (long long)(r0 + r) * lda, j * BS, q, n, row_ok, vec_ok != 0);
    if (d >= known) {
      if (threadIdx.x == 0) {
        // every waiting block polls the one progress word: a short sleep
        // between polls keeps them from saturating its L2 slice, which the
        // producing block's stores and instruction fetches also go through
        int p = ld_acquire(sync);
        for (uint32_t it = 0; ok && p <= d; p = ld_acquire(sync)) {
          if (++it > kSpinLimit) {
            atomicCAS(status, 0, LM_DEVERR_TIMEOUT);
            ok = false;
          }
          __nanosleep(p + 1 < d ? 512 : 64);
        }
        prog_sh = ok ? p : nb;  // on timeout, run to the end without waiting
      }
      __syncthreads();
      known = prog_sh;
    }
    T(*xs)[XS] = xj[d & 1];
    for (int i = threadIdx.x; i < BS * nrhs; i += NT) {
      const int rr = i / nrhs, h = i % nrhs;
      const int row = j * BS + rr;
      xs[rr][h] = row < n ? ld_volatile(X + (long long)row * ldx + h) : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < CP; ++e) {
      const int cc = col_of(e);
#pragma unroll
      for (int h = 0; h < MAX_RHS; ++h)
        if (h < nrhs) acc[h] = fma(tv[e], xs[cc][h], acc[h]);
    }
    // xj is double-buffered: the next write to this buffer comes after the
    // next iteration's barrier, which every thread reaches after this FMA.
  }
  // y = rhs - T_b,dep x_dep  (the four lanes of a row are adjacent).  The
  // warp is reconverged first: thread 0's bounded poll and the barriers
  // leave it split, and a split warp serialises every shuffle that follows.
  __syncwarp();
#pragma unroll
  for (int h = 0; h < MAX_RHS; ++h) {
    acc[h] += __shfl_xor_sync(0xffffffffu, acc[h], 1);
    acc[h] += __shfl_xor_sync(0xffffffffu, acc[h], 2);
  }
  if (q == 0)
#pragma unroll
    for (int h = 0; h < MAX_RHS; ++h) ys[r][h] = row_ok ? rhs[h] - acc[h] : T(0);
  __syncthreads();
  if constexpr (EXACT) {
    // warp 0: blocked column sweep in 32 dependent steps of RPL rows.  Step s:
    // every lane takes lane s's RPL partial results by shuffles and solves the
    // RPL x RPL diagonal tile with them itself (the same values in every lane,
    // so no lane branches off), then the lanes on the unsolved side subtract
    // tile (l, s) times the solution from their rows.  Tile rows are 16-byte
    // shared-memory loads.
    if (threadIdx.x < 32) {
      constexpr int TS = TrsvDiag<T>::TS;
      static_assert(RPL * sizeof(T) == 16, "a tile row is one 16-byte load");
      const int l = threadIdx.x;
      T y[RPL][MAX_RHS];
#pragma unroll
      for (int i = 0; i < RPL; ++i)
#pragma unroll
        for (int h = 0; h < MAX_RHS; ++h) y[i][h] = ys[RPL * l + i][h];
      const uint32_t tile_base = smem_u32(diag.tile);
      auto load_tile = [&](int row_lane, int col_lane, T (&t)[RPL][RPL]) {
        const uint32_t a = tile_base + (uint32_t)((col_lane * 32 + row_lane) * TS * (int)sizeof(T));
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
          if constexpr (sizeof(T) == 4) {
            float4 v;
            asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                         : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                         : "r"(a + 16u * i));
            t[i][0] = v.x, t[i][1] = v.y, t[i][2] = v.z, t[i][3] = v.w;
          } else {
            double2 v;
            asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a + 16u * i));
            t[i][0] = v.x, t[i][1] = v.y;
          }
        }
      };
      // one converged warp for the whole sweep: entered split (after the
      // divergent ys stores and the barrier), each step's shuffles cost 5x
      __syncwarp();
#pragma unroll 1
      for (int st = 0; st < 32; ++st) {
        const int sl = forward ? st : 31 - st;  // lane whose rows are solved now
        T tl[RPL][RPL], td[RPL][RPL], rdv[RPL];
        load_tile(l, sl, tl);   // this lane's rows, the solved lane's columns
        load_tile(sl, sl, td);  // the diagonal tile (the same address in every lane)
#pragma unroll
        for (int i = 0; i < RPL; ++i) rdv[i] = (forward && unit_l) ? T(1) : diag.rdiag[RPL * sl + i];
#pragma unroll
        for (int h = 0; h < MAX_RHS; ++h) {  // columns past nrhs hold zeros: no branch on nrhs
            T xv[RPL];
#pragma unroll
            for (int j = 0; j < RPL; ++j) xv[j] = __shfl_sync(0xffffffffu, y[j][h], sl);
            if (forward) {
#pragma unroll
              for (int i = 0; i < RPL; ++i) {
                T v = xv[i];
#pragma unroll
                for (int j = 0; j < i; ++j) v = fma(-td[i][j], xv[j], v);
                xv[i] = unit_l ? v : v * rdv[i];
              }
            } else {
#pragma unroll
              for (int i = RPL - 1; i >= 0; --i) {
                T v = xv[i];
#pragma unroll
                for (int j = i + 1; j < RPL; ++j) v = fma(-td[i][j], xv[j], v);
                xv[i] = v * rdv[i];
              }
            }
            const bool below = forward ? l > sl : l < sl;
#pragma unroll
            for (int i = 0; i < RPL; ++i) {
              T v = y[i][h];
#pragma unroll
              for (int j = 0; j < RPL; ++j) v = fma(-tl[i][j], xv[j], v);
              y[i][h] = l == sl ? xv[i] : (below ? v : y[i][h]);
            }
          }
      }
#pragma unroll
      for (int h = 0; h < MAX_RHS; ++h)
        if (h < nrhs)
#pragma unroll
          for (int i = 0; i < RPL; ++i)
            if (RPL * l + i < rows) X[(long long)(r0 + RPL * l + i) * ldx + h] = y[i][h];
    }
  } else {
    // x_b = inv(T_bb) y, then one correction x_b += inv(T_bb) (y - T_bb x_b):
    // the diagonal blocks of a factor without pivoting can be ill-conditioned,
    // and a product with the explicit inverse alone loses accuracy by their
    // condition number
    auto inv_times_ys = [&](T (&out)[MAX_RHS]) {
      __syncwarp();
#pragma unroll
      for (int h = 0; h < MAX_RHS; ++h) out[h] = T(0);
#pragma unroll
      for (int e = 0; e < CP; ++e) {
        const int cc = col_of(e);
#pragma unroll
        for (int h = 0; h < MAX_RHS; ++h)
          if (h < nrhs) out[h] = fma(dv[e], ys[cc][h], out[h]);
      }
#pragma unroll
      for (int h = 0; h < MAX_RHS; ++h) {
        out[h] += __shfl_xor_sync(0xffffffffu, out[h], 1);
        out[h] += __shfl_xor_sync(0xffffffffu, out[h], 2);
      }
    };
    inv_times_ys(acc);
    // The 16-column variant keeps the plain product: the correction's
    // operands do not fit its registers (it spilled in the dependency loop).
    if (RHS > 4 || (corr != nullptr && corr[2 * b] == 0)) {  // uniform over the CTA
      if (q == 0 && row_ok)
#pragma unroll
        for (int h = 0; h < MAX_RHS; ++h)
          if (h < nrhs) X[(long long)(r0 + r) * ldx + h] = acc[h];
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        st_release(sync, t + 1);
      }
      return;
    }
    // this thread's share of row r of T_bb (unit diagonal forward, identity padding)
    T tb[CP];
    load_row_share<T>(tb, LU + (long long)(r0 + (row_ok ? r : 0)) * lda, r0, q, n, row_ok, vec_ok != 0);
#pragma unroll
    for (int e = 0; e < CP; ++e) {
      const int cc = col_of(e);
      const bool keep = row_ok && cc < rows && (forward ? cc < r : cc >= r);
      tb[e] = keep ? tb[e] : ((cc == r && (forward || !row_ok || cc >= rows)) ? T(1) : T(0));
    }
    T(*xb)[XS] = xj[0];
    if (q == 0)
#pragma unroll
      for (int h = 0; h < MAX_RHS; ++h) xb[r][h] = acc[h];
    __syncthreads();
    T rr[MAX_RHS];
#pragma unroll
    for (int h = 0; h < MAX_RHS; ++h) rr[h] = T(0);
#pragma unroll
    for (int e = 0; e < CP; ++e) {
      const int cc = col_of(e);
#pragma unroll
      for (int h = 0; h < MAX_RHS; ++h)
        if (h < nrhs) rr[h] = fma(tb[e], xb[cc][h], rr[h]);
    }
    __syncwarp();
#pragma unroll
    for (int h = 0; h < MAX_RHS; ++h) {
      rr[h] += __shfl_xor_sync(0xffffffffu, rr[h], 1);
      rr[h] += __shfl_xor_sync(0xffffffffu, rr[h], 2);
    }
    __syncthreads();  // every thread has read ys for the first product
    if (q == 0)
#pragma unroll
      for (int h = 0; h < MAX_RHS; ++h) ys[r][h] = row_ok ? ys[r][h] - rr[h] : T(0);
    __syncthreads();
    T dx[MAX_RHS];
    inv_times_ys(dx);
    if (q == 0 && row_ok)
#pragma unroll
      for (int h = 0; h < MAX_RHS; ++h)
        if (h < nrhs) X[(long long)(r0 + r) * ldx + h] = acc[h] + dx[h];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    st_release(sync, t + 1);
  }
}

}  // namespace

template <typename T>
size_t trsv_inv_elems(int n) {
  constexpr int BS = TrsvCfg<T>::BS;
  return (size_t)((n + BS - 1) / BS) * BS * BS;
}

// Inverses of the diagonal blocks of L (unit lower) and U of a packed LU
// factor: DinvL and DinvU each hold trsv_inv_elems<T>(n) elements.
template <typename T>
int tri_inv_blocks(const T* LU, long long lda, int n, T* DinvL, T* DinvU, cudaStream_t st) {
  constexpr int BS = TrsvCfg<T>::BS, NT = TrsvCfg<T>::NT;
  if (n <= 0) return LM_OK;
  const int nb = (n + BS - 1) / BS;
  const int smem = (int)(2 * BS * (BS + 1) * sizeof(T));
  LM_CUDA_TRY(cudaFuncSetAttribute(tri_inv_blocks_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  tri_inv_blocks_kernel<T><<<nb, NT, smem, st>>>(LU, lda, n, 1, DinvL);
  tri_inv_blocks_kernel<T><<<nb, NT, smem, st>>>(LU, lda, n, 0, DinvU);
  count_launch(2);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

// X (n x nrhs) <- U^-1 L^-1 X with the packed factor (L unit lower, or with
// its stored diagonal when unit_lower is false, as for a Cholesky factor
// packed with its transpose).  FP64 and FP32 with `exact` solve the diagonal
// blocks by substitution (DinvL / DinvU unused);
// FP32 otherwise multiplies by the block inverses DinvL / DinvU.  FP64 takes
// nrhs <= 4; FP32 any nrhs (more than 4 in passes of 16 columns).  `sync`
// holds 4 ints of device scratch.  corr (inverse form), when given, holds two
// flags per diagonal block (L, U); only flagged blocks take the correction
// step, all blocks do without it.  Passes of the 16-column variant multiply by
// the inverse only.
template <typename T, int RHS, bool EXACT>
int trsv_pass(const T* LU, long long lda, int n, int nrhs, const T* DinvL, const T* DinvU, T* X, long long ldx,
              int* sync, int* status, cudaStream_t st, const int* corr, int vec_ok, int unit_l) {
  constexpr int BS = TrsvCfg<T>::BS, NT = TrsvCfg<T>::NT;
  const int nb = (n + BS - 1) / BS;
  const int smem = EXACT ? (int)sizeof(TrsvDiag<T>) : 0;
  if (EXACT) {
    static bool attr_set[kMaxDevices] = {};
    int dev = 0;
    LM_CUDA_TRY(cudaGetDevice(&dev));
    if (!attr_set[dev]) {
      LM_CUDA_TRY(cudaFuncSetAttribute(trsv_kernel<T, RHS, EXACT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       smem));
      LM_CUDA_TRY(cudaFuncSetAttribute(trsv_kernel<T, RHS, EXACT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       smem));
      attr_set[dev] = true;
    }
  }
  LM_CUDA_TRY(cudaMemsetAsync(sync, 0, sizeof(int) * 4, st));
  trsv_kernel<T, RHS, EXACT, true><<<nb, NT, smem, st>>>(LU, lda, n, nrhs, DinvL, X, ldx, sync, status, vec_ok, corr,
                                                         unit_l);
  trsv_kernel<T, RHS, EXACT, false><<<nb, NT, smem, st>>>(LU, lda, n, nrhs, DinvU, X, ldx, sync + 2, status, vec_ok,
                                                          corr ? corr + 1 : nullptr, unit_l);
  count_launch(2);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

template <typename T>
int trsv_lu(const T* LU, long long lda, int n, int nrhs, const T* DinvL, const T* DinvU, T* X, long long ldx,
            int* sync, int* status, cudaStream_t st, const int* corr, bool exact, bool unit_lower) {
  constexpr int VEC = TrsvCfg<T>::VEC;
  if (n <= 0 || nrhs <= 0) return LM_OK;
  constexpr bool kF64 = sizeof(T) == 8;
  exact = exact || kF64 || !unit_lower;
  const int ul = unit_lower ? 1 : 0;
  if (!exact && (reinterpret_cast<uintptr_t>(DinvL) % 16 || reinterpret_cast<uintptr_t>(DinvU) % 16))
    return LM_ERR_ARG;
  const int vec_ok = (reinterpret_cast<uintptr_t>(LU) % 16 == 0) && (lda % VEC == 0);
  if (nrhs == 1 && exact)  // the refinement's common case: one column, fewer registers
    return trsv_pass<T, 1, true>(LU, lda, n, nrhs, DinvL, DinvU, X, ldx, sync, status, st, nullptr, vec_ok, ul);
  if (nrhs <= MAX_RHS) {
    if (exact)
      return trsv_pass<T, MAX_RHS, true>(LU, lda, n, nrhs, DinvL, DinvU, X, ldx, sync, status, st, nullptr, vec_ok, ul);
    return trsv_pass<T, MAX_RHS, false>(LU, lda, n, nrhs, DinvL, DinvU, X, ldx, sync, status, st, corr, vec_ok, ul);
  }
  if constexpr (kF64) {
    return LM_ERR_UNSUPPORTED;
  } else {
    // more right-hand sides: the FP32 wide variant, WIDE_RHS columns per pass
    for (int c0 = 0; c0 < nrhs; c0 += WIDE_RHS) {
      const int nc = std::min(WIDE_RHS, nrhs - c0);
      if (exact)
        LM_TRY((trsv_pass<T, WIDE_RHS, true>(LU, lda, n, nc, DinvL, DinvU, X + c0, ldx, sync, status, st, nullptr,
                                             vec_ok, ul)));
      else
        LM_TRY((trsv_pass<T, WIDE_RHS, false>(LU, lda, n, nc, DinvL, DinvU, X + c0, ldx, sync, status, st, corr,
                                              vec_ok, ul)));
    }
    return LM_OK;
  }
}

template size_t trsv_inv_elems<float>(int);
template size_t trsv_inv_elems<double>(int);
template int tri_inv_blocks<float>(const float*, long long, int, float*, float*, cudaStream_t);
template int tri_inv_blocks<double>(const double*, long long, int, double*, double*, cudaStream_t);
template int trsv_lu<float>(const float*, long long, int, int, const float*, const float*, float*, long long, int*,
                            int*, cudaStream_t, const int*, bool, bool);
template int trsv_lu<double>(const double*, long long, int, int, const double*, const double*, double*, long long,
                             int*, int*, cudaStream_t, const int*, bool, bool);

}  // namespace lm
