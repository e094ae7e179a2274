// Batched uneven-size factor + solve in one persistent launch.
//
// Thousands of independent systems A_i X_i = B_i (n_i <= 256, nrhs_i <= 16),
// each general (LU with partial pivoting: luSolveP, LU.hs:265-357, pivot rule
// of rawPivotSearch K.hs:1541-1556) or SPD (Cholesky: choleskySolveP,
// Chol.hs:241-321), are solved by one persistent grid.  Each CTA takes the
// next instance from a ticket counter (the host orders the instances by
// decreasing cost, longest-processing-time first), factors it in a private
// workspace region that stays L2-resident (at most 512 KB per instance), and
// solves.  Inside an instance everything is CTA-local — no grid-wide
// synchronisation and no spin-waits:
//   factor : right-looking, panels of nb columns (nb tuned per size bucket)
//            held in shared memory; pivot search by warp shuffles; row
//            interchanges and the U12 = L11^-1 A12 solve by per-thread
//            columns; the trailing update as a 64 x 64 register-tiled FMA
//            loop with the panel and a staged U12 chunk in shared memory.
//   solve  : 32-row blocks; off-diagonal part as staged dot products, the
//            diagonal block by one warp per right-hand side (lane = row,
//            shuffles carry the solved entry).
//
// Mixed precision (LM_PREC_FP32_IR): the factorisation and the correction
// solves run in FP32; the solution is refined in FP64 inside the same CTA —
// r = B - A X with the original FP64 A, correction from the FP32 factors,
// X += D — until the normwise backward error max_h ||r_h|| / (||A|| ||x_h|| +
// ||b_h||) (infinity norms) is <= tol.  An instance that has not converged
// after max_iter corrections is refactored and solved in FP64 (iters = -1).
#include <cfloat>
#include <climits>

#include "common.cuh"
#include "internal.h"

namespace lm {

namespace {

constexpr int kBT = 256;     // threads per CTA
constexpr int kUC = 64;      // trailing-update column chunk
constexpr int kSB = 32;      // substitution row block
constexpr int kSC = 64;      // substitution column chunk (staged)
constexpr int kFixed = 512;  // bytes of fixed shared scratch ahead of the carved region

__device__ __forceinline__ int tid_() { return threadIdx.x; }

template <typename T>
__device__ __forceinline__ T abs_nan_low(T x) {
  const T a = x < T(0) ? -x : x;
  return (a != a) ? T(-1) : a;  // NaN never wins the pivot scan
}

template <typename T>
__device__ __forceinline__ bool piv_better(T v1, int i1, T v2, int i2) {
  return v1 > v2 || (v1 == v2 && i1 < i2);
}

// Fixed shared scratch (first kFixed bytes of dynamic shared memory).
struct Fixed {
  double rv[8];
  int ri[8];
  double norm[3][BatchLimits::kMaxRhs];  // ||r_h||, ||x_h||, ||b_h||
  double anorm;
  int flag;
};
static_assert(sizeof(Fixed) <= kFixed, "fixed scratch");

// Block-wide argmax of (v, i) (largest v, lowest i on ties); every thread
// returns the winner.  Two barriers.
template <typename T>
__device__ __forceinline__ void block_argmax(T& v, int& i, Fixed* fx) {
  const int lane = tid_() & 31, warp = tid_() >> 5;
  __syncwarp();  // a warp split by earlier branches would serialise the shuffles
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    if (piv_better(ov, oi, v, i)) { v = ov; i = oi; }
  }
  if (lane == 0) { fx->rv[warp] = (double)v; fx->ri[warp] = i; }
  __syncthreads();
  T w = lane < kBT / 32 ? (T)fx->rv[lane] : T(-1);
  int wi = lane < kBT / 32 ? fx->ri[lane] : INT_MAX;
  __syncwarp();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T ov = __shfl_xor_sync(0xffffffffu, w, o);
    const int oi = __shfl_xor_sync(0xffffffffu, wi, o);
    if (piv_better(ov, oi, w, wi)) { w = ov; wi = oi; }
  }
  v = w;
  i = wi;
  __syncthreads();  // the scratch is reused by the next reduction
}

// Block-wide max of a non-negative value (NaN propagates as +inf).
__device__ __forceinline__ double block_max(double v, Fixed* fx) {
  const int lane = tid_() & 31, warp = tid_() >> 5;
  if (v != v) v = DBL_MAX;
  __syncwarp();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if (lane == 0) fx->rv[warp] = v;
  __syncthreads();
  double w = lane < kBT / 32 ? fx->rv[lane] : 0.0;
  __syncwarp();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) w = fmax(w, __shfl_xor_sync(0xffffffffu, w, o));
  __syncthreads();
  return w;
}

// ---------------------------------------------------------------------------
// Factorisations of one instance (F: n x n, ld n, in global memory).
// ---------------------------------------------------------------------------

// Trailing update C (M x Nc) -= L (M x w, shared, ld ldl) * U (w x Nc), with
// U read from global rows u (ld n) through a staged chunk Us, or (lower =
// true, Cholesky) C -= L L^T on the lower triangle with U = L^T from shared.
template <typename T>
__device__ void trailing_update(T* C, int n, int M, int Nc, const T* L, int ldl, const T* U, int w, bool lower,
                                T* Us) {
  const int ty = tid_() >> 4, tx = tid_() & 15;
  for (int c0 = 0; c0 < Nc; c0 += kUC) {
    if (!lower) {
      for (int e = tid_(); e < w * kUC; e += kBT) {
        const int kk = e / kUC, cc = e % kUC;
        Us[e] = (c0 + cc < Nc) ? U[(long long)kk * n + c0 + cc] : T(0);
      }
      __syncthreads();
    }
    for (int rb = lower ? c0 : 0; rb < M; rb += 64) {
      T acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = rb + ty + 16 * i;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int cc = c0 + tx + 16 * j;
          const bool in = r < M && cc < Nc && (!lower || cc <= r);
          acc[i][j] = in ? C[(long long)r * n + cc] : T(0);
        }
      }
      for (int kk = 0; kk < w; ++kk) {
        T a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int r = rb + ty + 16 * i;
          a[i] = r < M ? L[r * ldl + kk] : T(0);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int cc = tx + 16 * j;
          if (lower)
            b[j] = (c0 + cc < M) ? L[(c0 + cc) * ldl + kk] : T(0);
          else
            b[j] = Us[kk * kUC + cc];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fma(-a[i], b[j], acc[i][j]);
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = rb + ty + 16 * i;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int cc = c0 + tx + 16 * j;
          if (r < M && cc < Nc && (!lower || cc <= r)) C[(long long)r * n + cc] = acc[i][j];
        }
      }
    }
    __syncthreads();
  }
}

// LU with partial pivoting in place; ipiv (global, n) receives the swap list
// (0-based).  Returns the LAPACK-style info (first zero pivot + 1, or 0).
template <typename T>
__device__ int lu_factor(T* F, int n, int nb, int* ipiv, unsigned char* region, Fixed* fx) {
  T* P = reinterpret_cast<T*>(region);  // [n][nb + 1]
  const int ldp = nb + 1;
  T* Us = P + (size_t)n * ldp;          // [nb][kUC]
  int* pv = reinterpret_cast<int*>(Us + (size_t)nb * kUC);  // [nb]
  int info = 0;
  for (int k0 = 0; k0 < n; k0 += nb) {
    const int w = min(nb, n - k0), R = n - k0;
    for (int e = tid_(); e < R * w; e += kBT) {
      const int r = e / w, c = e % w;
      P[r * ldp + c] = F[(long long)(k0 + r) * n + k0 + c];
    }
    __syncthreads();
    // column loop: candidate of column j from the rows this thread updated
    T bv = T(-1);
    int bi = INT_MAX;
    for (int r = tid_(); r < R; r += kBT) {
      const T v = abs_nan_low(P[r * ldp]);
      if (piv_better(v, r, bv, bi)) { bv = v; bi = r; }
    }
    for (int j = 0; j < w; ++j) {
      // thread 0 last wrote row j (step j-1 eliminated rows j.. from thread 0
      // up), so it reads a_jj before the argmax's barriers publish the flag
      if (tid_() == 0) fx->flag = (P[j * ldp + j] != P[j * ldp + j]) ? 1 : 0;
      block_argmax(bv, bi, fx);
      const int p = (fx->flag || bi == INT_MAX) ? j : bi;  // NaN diagonal stays the pivot
      if (tid_() == 0) pv[j] = p;
      if (p != j)
        for (int c = tid_(); c < w; c += kBT) {
          const T t = P[j * ldp + c];
          P[j * ldp + c] = P[p * ldp + c];
          P[p * ldp + c] = t;
        }
      __syncthreads();
      const T piv = P[j * ldp + j];
      if (piv == T(0) && info == 0) info = k0 + j + 1;
      bv = T(-1);
      bi = INT_MAX;
      // eliminate rows j+1.. and scan them for column j+1's candidates (the
      // argmax needs the set of candidates, not which thread holds them)
      for (int r = j + 1 + tid_(); r < R; r += kBT) {
        const T m = P[r * ldp + j] / piv;
        P[r * ldp + j] = m;
        for (int c = j + 1; c < w; ++c) P[r * ldp + c] = fma(-m, P[j * ldp + c], P[r * ldp + c]);
        if (j + 1 < w) {
          const T v = abs_nan_low(P[r * ldp + j + 1]);
          if (piv_better(v, r, bv, bi)) { bv = v; bi = r; }
        }
      }
    }
    __syncthreads();  // the last column's multipliers come from every thread
    for (int e = tid_(); e < R * w; e += kBT) {
      const int r = e / w, c = e % w;
      F[(long long)(k0 + r) * n + k0 + c] = P[r * ldp + c];
    }
    for (int j = tid_(); j < w; j += kBT) ipiv[k0 + j] = k0 + pv[j];
    // interchanges on the columns outside the panel: each thread owns columns
    for (int col = tid_(); col < n - w; col += kBT) {
      const int gc = col < k0 ? col : col + w;
      for (int j = 0; j < w; ++j) {
        const int p = pv[j];
        if (p != j) {
          T* a = F + (long long)(k0 + j) * n + gc;
          T* b = F + (long long)(k0 + p) * n + gc;
          const T t = *a;
          *a = *b;
          *b = t;
        }
      }
    }
    __syncthreads();
    if (k0 + w < n) {
      // U12 = L11^-1 A12 (unit lower L11 in P's top w rows), per-thread columns
      for (int col = k0 + w + tid_(); col < n; col += kBT) {
        T u[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) u[i] = i < w ? F[(long long)(k0 + i) * n + col] : T(0);
#pragma unroll
        for (int i = 1; i < 32; ++i)
          if (i < w) {
#pragma unroll
            for (int q = 0; q < i; ++q) u[i] = fma(-P[i * ldp + q], u[q], u[i]);
          }
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (i < w) F[(long long)(k0 + i) * n + col] = u[i];
      }
      __syncthreads();
      trailing_update<T>(F + (long long)(k0 + w) * n + k0 + w, n, R - w, R - w, P + (size_t)w * ldp, ldp,
                         F + (long long)k0 * n + k0 + w, w, false, Us);
    }
  }
  return info;
}

// Cholesky (lower) in place: G in the lower triangle, the strict upper
// triangle left as it was.  Returns the first non-positive pivot + 1, or 0.
template <typename T>
__device__ int chol_factor(T* F, int n, int nb, unsigned char* region, Fixed* fx) {
  T* P = reinterpret_cast<T*>(region);  // [n][nb + 1]
  const int ldp = nb + 1;
  int info = 0;
  for (int k0 = 0; k0 < n; k0 += nb) {
    const int w = min(nb, n - k0), R = n - k0;
    for (int e = tid_(); e < R * w; e += kBT) {
      const int r = e / w, c = e % w;
      P[r * ldp + c] = F[(long long)(k0 + r) * n + k0 + c];
    }
    __syncthreads();
    for (int j = 0; j < w; ++j) {
      const T d = P[j * ldp + j];
      if (!(d > T(0)) && info == 0) info = k0 + j + 1;
      const T s = sqrt(d);
      for (int r = j + 1 + tid_(); r < R; r += kBT) P[r * ldp + j] = P[r * ldp + j] / s;
      __syncthreads();
      if (tid_() == 0) P[j * ldp + j] = s;
      for (int r = j + 1 + tid_(); r < R; r += kBT) {
        const T m = P[r * ldp + j];
        const int ce = min(r, w - 1);
        for (int c = j + 1; c <= ce; ++c) P[r * ldp + c] = fma(-m, P[c * ldp + j], P[r * ldp + c]);
      }
      __syncthreads();
    }
    for (int e = tid_(); e < R * w; e += kBT) {
      const int r = e / w, c = e % w;
      if (r >= w || c <= r) F[(long long)(k0 + r) * n + k0 + c] = P[r * ldp + c];
    }
    __syncthreads();
    if (k0 + w < n)
      trailing_update<T>(F + (long long)(k0 + w) * n + k0 + w, n, R - w, R - w, P + (size_t)w * ldp, ldp, nullptr,
                         w, true, nullptr);
  }
  return info;
}

// ---------------------------------------------------------------------------
// Triangular solves on V (n x r, shared, ld r) with the factor in F.
//   mode 0: unit lower (LU's L)      forward
//   mode 1: upper (LU's U)           backward
//   mode 2: lower G (Cholesky)       forward
//   mode 3: upper G^T (Cholesky)     backward, T(i, k) = G(k, i)
// ---------------------------------------------------------------------------
template <typename TF, typename TV>
__device__ __forceinline__ TF tri_elem(const TF* F, int n, int mode, int i, int k) {
  return mode == 3 ? F[(long long)k * n + i] : F[(long long)i * n + k];
}

template <typename TF, typename TV>
__device__ void tri_solve(const TF* F, int n, int mode, TV* V, int r, TF* Tb) {
  // Tb: [kSB][kSC + 1] staging
  const bool fwd = (mode == 0 || mode == 2);
  const bool unit = (mode == 0);
  const int nblk = (n + kSB - 1) / kSB;
  const int lane = tid_() & 31, warp = tid_() >> 5;
  constexpr int LDT = kSC + 1;
  for (int bi = 0; bi < nblk; ++bi) {
    const int b = fwd ? bi : nblk - 1 - bi;
    const int i0 = b * kSB, bw = min(kSB, n - i0);
    // off-diagonal: V[i0 + ii][h] -= sum_k T(i0 + ii, k) V[k][h] over the solved k
    const int ks = fwd ? 0 : i0 + bw, ke = fwd ? i0 : n;
    TV acc[2] = {TV(0), TV(0)};
    const int pairs = bw * r;
    for (int kc = ks; kc < ke; kc += kSC) {
      const int kw = min(kSC, ke - kc);
      for (int e = tid_(); e < kSB * kSC; e += kBT) {
        int ii, kk;
        if (mode == 3) { ii = e % kSB; kk = e / kSB; }   // contiguous along i for G^T
        else { kk = e % kSC; ii = e / kSC; }             // contiguous along k
        Tb[ii * LDT + kk] = (ii < bw && kk < kw) ? tri_elem<TF, TV>(F, n, mode, i0 + ii, kc + kk) : TF(0);
      }
      __syncthreads();
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int pr = tid_() + s * kBT;
        if (pr < pairs) {
          const int ii = pr / r, h = pr % r;
          TV a = acc[s];
          for (int kk = 0; kk < kw; ++kk) a = fma(-(TV)Tb[ii * LDT + kk], V[(kc + kk) * r + h], a);
          acc[s] = a;
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int pr = tid_() + s * kBT;
      if (pr < pairs && ke > ks) {
        const int ii = pr / r, h = pr % r;
        V[(i0 + ii) * r + h] += acc[s];
      }
    }
    // diagonal block
    for (int e = tid_(); e < kSB * kSB; e += kBT) {
      int ii, kk;
      if (mode == 3) { ii = e % kSB; kk = e / kSB; }
      else { kk = e % kSB; ii = e / kSB; }
      Tb[ii * LDT + kk] = (ii < bw && kk < bw) ? tri_elem<TF, TV>(F, n, mode, i0 + ii, i0 + kk) : TF(0);
    }
    __syncthreads();
    for (int h = warp; h < r; h += kBT / 32) {
      TV y = lane < bw ? V[(i0 + lane) * r + h] : TV(0);
      __syncwarp();  // one converged warp for the column sweep's shuffles
      if (fwd) {
        for (int kk = 0; kk < bw; ++kk) {
          if (!unit && lane == kk) y = y / (TV)Tb[kk * LDT + kk];
          const TV xk = __shfl_sync(0xffffffffu, y, kk);
          if (lane > kk) y = fma(-(TV)Tb[lane * LDT + kk], xk, y);
        }
      } else {
        for (int kk = bw - 1; kk >= 0; --kk) {
          if (lane == kk) y = y / (TV)Tb[kk * LDT + kk];
          const TV xk = __shfl_sync(0xffffffffu, y, kk);
          if (lane < kk) y = fma(-(TV)Tb[lane * LDT + kk], xk, y);
        }
      }
      if (lane < bw) V[(i0 + lane) * r + h] = y;
    }
    __syncthreads();
  }
}

// Apply the swap list to the rows of V in order (applyPivotsForward, LU.hs:493-507).
template <typename TV>
__device__ void apply_pivots(TV* V, int n, int r, const int* ipiv) {
  for (int h = tid_(); h < r; h += kBT)
    for (int j = 0; j < n; ++j) {
      const int p = ipiv[j];
      if (p != j && p >= 0 && p < n) {
        const TV t = V[j * r + h];
        V[j * r + h] = V[p * r + h];
        V[p * r + h] = t;
      }
    }
  __syncthreads();
}

template <typename TF, typename TV>
__device__ void solve_factored(const TF* F, int n, int kind, const int* ipiv, TV* V, int r, TF* Tb) {
  if (kind == LM_BATCH_GENERAL) {
    apply_pivots<TV>(V, n, r, ipiv);
    tri_solve<TF, TV>(F, n, 0, V, r, Tb);
    tri_solve<TF, TV>(F, n, 1, V, r, Tb);
  } else {
    tri_solve<TF, TV>(F, n, 2, V, r, Tb);
    tri_solve<TF, TV>(F, n, 3, V, r, Tb);
  }
}

// Shared-memory carve (byte offsets from the start of dynamic shared memory):
//   [Fixed][Xs: nmax x rmax doubles][union { factor panel P, U12 chunk, pivots |
//                                              D (nmax x rmax floats), staging Tb }]
// Xs holds the FP64 solution across the IR loop and the FP64 fallback.
struct Carve {
  size_t xs, u, d, tb, total;
};
__host__ __device__ inline Carve carve(int nmax, int rmax, int nbmax) {
  Carve c;
  c.xs = kFixed;
  c.u = (c.xs + (size_t)nmax * rmax * 8 + 15) / 16 * 16;
  c.d = c.u;
  c.tb = (c.d + (size_t)nmax * rmax * 4 + 15) / 16 * 16;
  const size_t sol_end = c.tb + (size_t)kSB * (kSC + 1) * 8;
  const size_t fac_end = c.u + (size_t)nmax * (nbmax + 1) * 8 + (size_t)nbmax * kUC * 8 + (size_t)nbmax * 4;
  c.total = (sol_end > fac_end ? sol_end : fac_end);
  return c;
}

// Input loads: L2-only (ld.global.cg) for the device-resident consumer, whose
// CTAs outlive the requests they read (an arena block is reused by later
// requests, and an SM's L1 is not coherent with the copies that refill it).
template <bool CG>
__device__ __forceinline__ double ld_in(const double* p) {
  if constexpr (CG) return __ldcg(p);
  else return *p;
}

// Factor + solve one instance entirely in FP64.
template <bool CG = false>
__device__ void run_fp64(const BatchItem& it, const BatchArgs& g, unsigned char* sm, Fixed* fx, double* Xs,
                         int* info_out) {
  const Carve cv = carve(g.nmax, g.rmax, g.nbmax);
  unsigned char* region = sm + cv.u;
  const int n = it.n, r = it.nrhs;
  double* F = g.F + it.f_off;
  int* ipiv = g.ipiv + it.p_off;
  for (long long e = tid_(); e < (long long)n * n; e += kBT) F[e] = ld_in<CG>(g.A + it.a_off + e);
  __syncthreads();
  const int info = it.kind == LM_BATCH_GENERAL ? lu_factor<double>(F, n, it.nb, ipiv, region, fx)
                                               : chol_factor<double>(F, n, it.nb, region, fx);
  __syncthreads();
  *info_out = info;
  if (r == 0) return;
  double* V = Xs;
  double* Tb = reinterpret_cast<double*>(sm + cv.tb);
  for (int e = tid_(); e < n * r; e += kBT) V[e] = ld_in<CG>(g.B + it.b_off + e);
  __syncthreads();
  solve_factored<double, double>(F, n, it.kind, ipiv, V, r, Tb);
}

// Factor in FP32, refine in FP64.  Returns the number of corrections, or -1
// when it fell back to FP64.
__device__ int run_ir(const BatchItem& it, const BatchArgs& g, unsigned char* sm, Fixed* fx, double* Xd,
                      int* info_out, double* berr_out) {
  const Carve cv = carve(g.nmax, g.rmax, g.nbmax);
  unsigned char* region = sm + cv.u;
  const int n = it.n, r = it.nrhs;
  float* F = reinterpret_cast<float*>(g.F + it.f_off);
  int* ipiv = g.ipiv + it.p_off;
  const double* A = g.A + it.a_off;
  const double* B = g.B + it.b_off;
  const double tol = g.tol > 0.0 ? g.tol : 1e-15 * n;
  for (long long e = tid_(); e < (long long)n * n; e += kBT) F[e] = (float)A[e];
  __syncthreads();
  const int info = it.kind == LM_BATCH_GENERAL ? lu_factor<float>(F, n, it.nb, ipiv, region, fx)
                                               : chol_factor<float>(F, n, it.nb, region, fx);
  __syncthreads();
  float* D = reinterpret_cast<float*>(sm + cv.d);
  float* Tb = reinterpret_cast<float*>(sm + cv.tb);
  const int lane = tid_() & 31, warp = tid_() >> 5;
  // ||A||_inf and ||b_h||_inf
  {
    double m = 0.0;
    for (int i = warp; i < n; i += kBT / 32) {
      double s = 0.0;
      for (int k = lane; k < n; k += 32) s += fabs(A[(long long)i * n + k]);
      __syncwarp();
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      m = fmax(m, s);
    }
    const double an = block_max(m, fx);
    if (tid_() == 0) fx->anorm = an;
    for (int h = 0; h < r; ++h) {
      double bm = 0.0;
      for (int i = tid_(); i < n; i += kBT) bm = fmax(bm, fabs(B[i * r + h]));
      const double bn = block_max(bm, fx);
      if (tid_() == 0) fx->norm[2][h] = bn;
    }
  }
  // x0 from the FP32 factors
  for (int e = tid_(); e < n * r; e += kBT) D[e] = (float)B[e];
  __syncthreads();
  if (info == 0) solve_factored<float, float>(F, n, it.kind, ipiv, D, r, Tb);
  for (int e = tid_(); e < n * r; e += kBT) Xd[e] = (double)D[e];
  __syncthreads();
  int iters = 0;
  bool ok = false;
  double be = 0.0;
  for (;;) {
    // r = B - A X (FP64), one warp per row; ||r_h||, ||x_h||
    double rmax[BatchLimits::kMaxRhs];
#pragma unroll
    for (int h = 0; h < BatchLimits::kMaxRhs; ++h) rmax[h] = 0.0;
    for (int i = warp; i < n; i += kBT / 32) {
      double s[BatchLimits::kMaxRhs];
#pragma unroll
      for (int h = 0; h < BatchLimits::kMaxRhs; ++h) s[h] = 0.0;
      for (int k = lane; k < n; k += 32) {
        const double a = A[(long long)i * n + k];
#pragma unroll
        for (int h = 0; h < BatchLimits::kMaxRhs; ++h)
          if (h < r) s[h] = fma(a, Xd[k * r + h], s[h]);
      }
      __syncwarp();
#pragma unroll
      for (int h = 0; h < BatchLimits::kMaxRhs; ++h)
        if (h < r) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) s[h] += __shfl_xor_sync(0xffffffffu, s[h], o);
          const double res = B[i * r + h] - s[h];
          if (lane == 0) D[i * r + h] = (float)res;
          rmax[h] = fmax(rmax[h], fabs(res) != fabs(res) ? DBL_MAX : fabs(res));
        }
    }
    be = 0.0;
    for (int h = 0; h < r; ++h) {
      const double rn = block_max(rmax[h], fx);
      double xm = 0.0;
      for (int i = tid_(); i < n; i += kBT) xm = fmax(xm, fabs(Xd[i * r + h]));
      const double xn = block_max(xm, fx);
      const double den = fx->anorm * xn + fx->norm[2][h];
      const double bh = den > 0.0 ? rn / den : (rn > 0.0 ? DBL_MAX : 0.0);
      be = fmax(be, bh != bh ? DBL_MAX : bh);
    }
    if (be <= tol) { ok = true; break; }
    if (iters >= g.max_iter || info != 0) break;
    __syncthreads();
    solve_factored<float, float>(F, n, it.kind, ipiv, D, r, Tb);
    for (int e = tid_(); e < n * r; e += kBT) Xd[e] += (double)D[e];
    __syncthreads();
    ++iters;
  }
  __syncthreads();
  if (ok) {
    *info_out = 0;
    *berr_out = be;
    return iters;
  }
  // FP64 fallback: refactor from A in the same workspace (n^2 doubles)
  int info64 = 0;
  run_fp64(it, g, sm, fx, Xd, &info64);
  *info_out = info64;
  *berr_out = be;
  return -1;
}

__global__ void __launch_bounds__(kBT, 2) batch_kernel(const BatchArgs g) {
  extern __shared__ __align__(16) unsigned char sm[];
  Fixed* fx = reinterpret_cast<Fixed*>(sm);
  __shared__ int slot;
  const Carve cv = carve(g.nmax, g.rmax, g.nbmax);
  double* Xs = reinterpret_cast<double*>(sm + cv.xs);
  for (;;) {
    if (tid_() == 0) slot = atomicAdd(g.ticket, 1);
    __syncthreads();
    const int s = slot;
    __syncthreads();
    if (s >= g.count) break;
    const BatchItem it = g.items[s];
    if (it.n <= 0) continue;
    int info = 0;
    int iters = 0;
    double be = 0.0;
    if (g.prec == LM_PREC_FP32_IR) {
      iters = run_ir(it, g, sm, fx, Xs, &info, &be);
    } else {
      run_fp64(it, g, sm, fx, Xs, &info);
    }
    __syncthreads();
    for (int e = tid_(); e < it.n * it.nrhs; e += kBT) g.X[it.x_off + e] = Xs[e];
    if (tid_() == 0) {
      g.info[it.index] = info;
      g.iters[it.index] = iters;
      g.berr[it.index] = be;
    }
    __syncthreads();
  }
}

// Device-resident request loop (the serving loop's small requests): every CTA
// claims the next posted request from a ring in device memory (head < tail),
// solves it in FP64 exactly as batch_kernel would, writes X into the arena and
// publishes info and a completion sequence number into pinned host memory.
// An idle CTA sleeps between polls and returns after kServeIdlePolls polls
// without work (the host relaunches the loop when new work arrives); the stop
// word ends it at once.  No other wait.
constexpr uint32_t kServeIdlePolls = 4000;  // x ~2 us of sleep: ~8 ms idle before returning

__global__ void __launch_bounds__(kBT, 2) serve_loop_kernel(const BatchArgs g, const ServeRing rg) {
  extern __shared__ __align__(16) unsigned char sm[];
  Fixed* fx = reinterpret_cast<Fixed*>(sm);
  __shared__ int slot;
  const Carve cv = carve(g.nmax, g.rmax, g.nbmax);
  double* Xs = reinterpret_cast<double*>(sm + cv.xs);
  for (;;) {
    if (tid_() == 0) {
      int claimed = -1;
      for (uint32_t idle = 0; idle < kServeIdlePolls;) {
        if (*reinterpret_cast<volatile const int*>(rg.stop) != 0) break;
        const int h = *reinterpret_cast<volatile const int*>(rg.head);
        const int t = *reinterpret_cast<volatile const int*>(rg.tail);
        if (h < t) {
          if (atomicCAS(rg.head, h, h + 1) == h) {
            claimed = h;
            break;
          }
          continue;  // another CTA took it: look again at once
        }
        __nanosleep(2000);
        ++idle;
      }
      slot = claimed;
    }
    __syncthreads();
    const int sq = slot;
    __syncthreads();
    if (sq < 0) return;
    const int idx = sq % rg.cap;
    BatchItem it;
    {
      const long long* src = reinterpret_cast<const long long*>(rg.items + idx);
      long long* dst = reinterpret_cast<long long*>(&it);
#pragma unroll
      for (int w = 0; w < (int)(sizeof(BatchItem) / sizeof(long long)); ++w) dst[w] = __ldcg(src + w);
    }
    int info = 0;
    if (it.n > 0) {
      run_fp64<true>(it, g, sm, fx, Xs, &info);
      __syncthreads();
      for (int e = tid_(); e < it.n * it.nrhs; e += kBT) g.X[it.x_off + e] = Xs[e];
    }
    __syncthreads();
    if (tid_() == 0) {
      __threadfence();  // X visible in device memory before the host copies it out
      rg.h_info[idx] = info;
      __threadfence_system();
      *reinterpret_cast<volatile int*>(rg.h_done + idx) = sq + 1;
    }
    __syncthreads();
  }
}

}  // namespace

size_t batch_smem_bytes(int nmax, int rmax, int nbmax) { return carve(nmax, rmax, nbmax).total; }

int serve_loop_launch(const BatchArgs& g, const ServeRing& rg, int grid, size_t smem, cudaStream_t st) {
  static size_t set_to[kMaxDevices] = {};
  int dev = 0;
  LM_CUDA_TRY(cudaGetDevice(&dev));
  if (set_to[dev] < smem) {
    LM_CUDA_TRY(cudaFuncSetAttribute(serve_loop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    set_to[dev] = smem;
  }
  serve_loop_kernel<<<grid, kBT, smem, st>>>(g, rg);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

// Raise the kernel's dynamic shared-memory limit to `smem` (once per size and device).
int batch_set_smem(size_t smem) {
  static size_t set_to[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (set_to[dev] < smem) {
    LM_CUDA_TRY(cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    set_to[dev] = smem;
  }
  return LM_OK;
}

int batch_launch(const BatchArgs& g, int grid, size_t smem, cudaStream_t st) {
  LM_TRY(batch_set_smem(smem));
  LM_CUDA_TRY(cudaMemsetAsync(g.ticket, 0, sizeof(int), st));
  batch_kernel<<<grid, kBT, smem, st>>>(g);
  count_launch(1);
  LM_CUDA_TRY(cudaGetLastError());
  return LM_OK;
}

int batch_occupancy(size_t smem, int* per_sm) {
  LM_TRY(batch_set_smem(smem));
  LM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, batch_kernel, kBT, smem));
  return LM_OK;
}

}  // namespace lm
