// CPU oracle for the dense-solve path: TEST INFRASTRUCTURE ONLY.
//
// A C++ restatement of linear-massiv's CPU algorithms for GEMM, panel LU
// with partial pivoting, panel Cholesky and the packed triangular
// substitutions.  It exists so that tests, the smoke check and the CPU
// baseline leg of the benchmark can compare the CUDA library against the
// reference's arithmetic.  Nothing in the product library links or calls it.
//
// Floating-point order follows the reference exactly:
//   * GHC's fmaddDoubleX4# is a fused multiply-add  -> _mm256_fmadd_pd
//   * scalar `a +## b *## c` is two roundings         -> compiled with
//     -ffp-contract=off so the compiler never fuses them
//   * horizontal sums are ((a + b) + c) + d
// so results are bit-identical to the reference on machines with AVX2+FMA.
//
// File references are relative to the linear-massiv source tree:
//   K.hs   = src/Numeric/LinearAlgebra/Massiv/Internal/Kernel.hs
//   LU.hs  = src/Numeric/LinearAlgebra/Massiv/Solve/LU.hs
//   Chol.hs= src/Numeric/LinearAlgebra/Massiv/Solve/Cholesky.hs
//   Tri.hs = src/Numeric/LinearAlgebra/Massiv/Solve/Triangular.hs
//   L3.hs  = src/Numeric/LinearAlgebra/Massiv/BLAS/Level3.hs
//   L2.hs  = src/Numeric/LinearAlgebra/Massiv/BLAS/Level2.hs

#include <immintrin.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

inline int rem_(int a, int b) { return a % b; }  // Haskell remInt# (truncating)

inline __m256d ld(const double* p) { return _mm256_loadu_pd(p); }
inline void st(double* p, __m256d v) { _mm256_storeu_pd(p, v); }
inline __m256d bc(double x) { return _mm256_set1_pd(x); }
inline __m256d fma4(__m256d a, __m256d b, __m256d c) { return _mm256_fmadd_pd(a, b, c); }
inline double hsum(__m256d v) {  // ((a + b) + c) + d, K.hs:96-97
  alignas(32) double t[4];
  _mm256_store_pd(t, v);
  double s = t[0] + t[1];
  s = s + t[2];
  s = s + t[3];
  return s;
}

// ---------------------------------------------------------------------------
// GEMM: rawGemmBIBJSlice (K.hs:175-406).  C[bi..,bj..] += A * B, A m x k,
// B k x n, C m x n, all row-major and dense (strides k, n, n).
// ---------------------------------------------------------------------------
void gemm_bibj(const double* A, const double* B, double* C, int biStart, int biEnd,
               int bjStart, int bjEnd, int /*m*/, int k, int n) {
  const int bs = 64;  // K.hs:182
  for (int bi = biStart; bi < biEnd; bi += bs) {
    const int iEnd = std::min(bi + bs, biEnd);
    for (int bk = 0; bk < k; bk += bs) {
      const int kEnd = std::min(bk + bs, k);
      for (int bj = bjStart; bj < bjEnd; bj += bs) {
        const int jEnd = std::min(bj + bs, bjEnd);
        // innerBlock (K.hs:203-209)
        const int jSpan = jEnd - bj;
        const int j8End = bj + (jSpan - rem_(jSpan, 8));
        const int j4End = bj + (jSpan - rem_(jSpan, 4));
        const int iSpan = iEnd - bi;
        const int i4End = bi + (iSpan - rem_(iSpan, 4));
        int i = bi;
        for (; i < i4End; i += 4) {  // goI4 (K.hs:212-219)
          // goJScalar4 (K.hs:306-333): separate mul/add accumulators from 0
          for (int j = j4End; j < jEnd; ++j) {
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
            for (int kk = bk; kk < kEnd; ++kk) {
              const double bkj = B[(size_t)kk * n + j];
              a0 = a0 + A[(size_t)i * k + kk] * bkj;
              a1 = a1 + A[(size_t)(i + 1) * k + kk] * bkj;
              a2 = a2 + A[(size_t)(i + 2) * k + kk] * bkj;
              a3 = a3 + A[(size_t)(i + 3) * k + kk] * bkj;
            }
            C[(size_t)i * n + j] = C[(size_t)i * n + j] + a0;
            C[(size_t)(i + 1) * n + j] = C[(size_t)(i + 1) * n + j] + a1;
            C[(size_t)(i + 2) * n + j] = C[(size_t)(i + 2) * n + j] + a2;
            C[(size_t)(i + 3) * n + j] = C[(size_t)(i + 3) * n + j] + a3;
          }
          // goJ4_4x4 (K.hs:277-304)
          for (int j = j8End; j < j4End; j += 4) {
            double* c0p = C + (size_t)i * n + j;
            __m256d c0 = ld(c0p), c1 = ld(c0p + n), c2 = ld(c0p + 2 * (size_t)n),
                    c3 = ld(c0p + 3 * (size_t)n);
            for (int kk = bk; kk < kEnd; ++kk) {
              const __m256d bv = ld(B + (size_t)kk * n + j);
              c0 = fma4(bc(A[(size_t)i * k + kk]), bv, c0);
              c1 = fma4(bc(A[(size_t)(i + 1) * k + kk]), bv, c1);
              c2 = fma4(bc(A[(size_t)(i + 2) * k + kk]), bv, c2);
              c3 = fma4(bc(A[(size_t)(i + 3) * k + kk]), bv, c3);
            }
            st(c0p, c0); st(c0p + n, c1); st(c0p + 2 * (size_t)n, c2); st(c0p + 3 * (size_t)n, c3);
          }
          // goJ8_4x8 + goK4x8 (K.hs:232-275): the 4x8 register-blocked micro-kernel
          for (int j = bj; j < j8End; j += 8) {
            double* r0 = C + (size_t)i * n + j;
            double* r1 = r0 + n;
            double* r2 = r0 + 2 * (size_t)n;
            double* r3 = r0 + 3 * (size_t)n;
            __m256d c00 = ld(r0), c01 = ld(r0 + 4), c10 = ld(r1), c11 = ld(r1 + 4);
            __m256d c20 = ld(r2), c21 = ld(r2 + 4), c30 = ld(r3), c31 = ld(r3 + 4);
            for (int kk = bk; kk < kEnd; ++kk) {
              const double* bp = B + (size_t)kk * n + j;
              const __m256d bv0 = ld(bp), bv1 = ld(bp + 4);
              const __m256d a0 = bc(A[(size_t)i * k + kk]);
              const __m256d a1 = bc(A[(size_t)(i + 1) * k + kk]);
              const __m256d a2 = bc(A[(size_t)(i + 2) * k + kk]);
              const __m256d a3 = bc(A[(size_t)(i + 3) * k + kk]);
              c00 = fma4(a0, bv0, c00); c01 = fma4(a0, bv1, c01);
              c10 = fma4(a1, bv0, c10); c11 = fma4(a1, bv1, c11);
              c20 = fma4(a2, bv0, c20); c21 = fma4(a2, bv1, c21);
              c30 = fma4(a3, bv0, c30); c31 = fma4(a3, bv1, c31);
            }
            st(r0, c00); st(r0 + 4, c01); st(r1, c10); st(r1 + 4, c11);
            st(r2, c20); st(r2 + 4, c21); st(r3, c30); st(r3 + 4, c31);
          }
        }
        for (; i < iEnd; ++i) {  // goI1 (K.hs:222-229)
          for (int j = j4End; j < jEnd; ++j) {  // goJScalar1 (K.hs:385-404)
            double acc = 0.0;
            for (int kk = bk; kk < kEnd; ++kk) acc = acc + A[(size_t)i * k + kk] * B[(size_t)kk * n + j];
            C[(size_t)i * n + j] = C[(size_t)i * n + j] + acc;
          }
          for (int j = j8End; j < j4End; j += 4) {  // goJ4_1x4 (K.hs:367-382)
            __m256d c0 = ld(C + (size_t)i * n + j);
            for (int kk = bk; kk < kEnd; ++kk)
              c0 = fma4(bc(A[(size_t)i * k + kk]), ld(B + (size_t)kk * n + j), c0);
            st(C + (size_t)i * n + j, c0);
          }
          for (int j = bj; j < j8End; j += 8) {  // goJ8_1x8 (K.hs:336-364)
            __m256d c0 = ld(C + (size_t)i * n + j), c1 = ld(C + (size_t)i * n + j + 4);
            for (int kk = bk; kk < kEnd; ++kk) {
              const __m256d av = bc(A[(size_t)i * k + kk]);
              c0 = fma4(av, ld(B + (size_t)kk * n + j), c0);
              c1 = fma4(av, ld(B + (size_t)kk * n + j + 4), c1);
            }
            st(C + (size_t)i * n + j, c0); st(C + (size_t)i * n + j + 4, c1);
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Host threads for the oracle's large cases.  Only row ranges of the trailing
// updates are split, at multiples of rawGemmBIBJSlice's 64-row tile, so every
// element is computed by exactly the same instruction sequence as in the
// single-threaded reference (the tile and 4-row grouping of a row depend only
// on its offset from the start of its 64-row tile).  0 = all hardware threads.
// ---------------------------------------------------------------------------
int g_threads = 0;

int oracle_threads() {
  if (g_threads > 0) return g_threads;
  const unsigned h = std::thread::hardware_concurrency();
  return h > 0 ? (int)h : 1;
}

// fn(r0, r1) over [0, rows) in chunks whose starts are multiples of 64.
template <class F>
void par_rows(int rows, F fn) {
  const int tiles = (rows + 63) / 64;
  const int nt = std::min(oracle_threads(), tiles);
  if (nt <= 1 || (long long)rows * 1 < 256) {
    if (rows > 0) fn(0, rows);
    return;
  }
  std::vector<std::thread> th;
  const int per = (tiles + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    const int r0 = t * per * 64, r1 = std::min(rows, (t + 1) * per * 64);
    if (r0 < r1) th.emplace_back([=] { fn(r0, r1); });
  }
  for (auto& x : th) x.join();
}

// ---------------------------------------------------------------------------
// Packed-B GEMM: rawGemmBISlicePackedBK (K.hs:412-805).  B is packed into
// kc x 8 panels per 64-row k slice (packB, K.hs:573-590); the 4x8 / 1x8
// micro-kernels read the panels, columns past the last full 8-panel use the
// unpacked 4-wide and scalar cleanups over the full row.
// ---------------------------------------------------------------------------
void gemm_packed(const double* A, const double* B, double* C, int biStart, int biEnd, int m,
                 int k, int n) {
  const int bs = 64;
  const int nPanels = n / 8;
  const int j8End = nPanels * 8;
  const int j4End = n - rem_(n, 4);
  if (j8End == 0) {  // goBI_unpacked fallback (K.hs:425-447)
    gemm_bibj(A, B, C, biStart, biEnd, 0, n, m, k, n);
    return;
  }
  std::vector<double> bp;
  for (int bk = 0; bk < k; bk += bs) {  // goBKO (K.hs:560-571)
    const int kEnd = std::min(bk + bs, k);
    const int kc = kEnd - bk;
    bp.assign((size_t)nPanels * kc * 8, 0.0);
    for (int p = 0; p < nPanels; ++p)
      for (int kl = 0; kl < kc; ++kl)
        std::memcpy(&bp[(size_t)p * kc * 8 + (size_t)kl * 8], B + (size_t)(bk + kl) * n + p * 8,
                    8 * sizeof(double));
    for (int bi = biStart; bi < biEnd; bi += bs) {  // goBIO (K.hs:593-603)
      const int iEnd = std::min(bi + bs, biEnd);
      const int iSpan = iEnd - bi;
      const int i4End = bi + (iSpan - rem_(iSpan, 4));
      for (int i = bi; i < i4End; i += 4) {  // goI4P
        for (int j = j4End; j < n; ++j) {   // goJSU4 (K.hs:727-755)
          double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
          for (int kk = bk; kk < kEnd; ++kk) {
            const double bkj = B[(size_t)kk * n + j];
            a0 = a0 + A[(size_t)i * k + kk] * bkj;
            a1 = a1 + A[(size_t)(i + 1) * k + kk] * bkj;
            a2 = a2 + A[(size_t)(i + 2) * k + kk] * bkj;
            a3 = a3 + A[(size_t)(i + 3) * k + kk] * bkj;
          }
          C[(size_t)i * n + j] = C[(size_t)i * n + j] + a0;
          C[(size_t)(i + 1) * n + j] = C[(size_t)(i + 1) * n + j] + a1;
          C[(size_t)(i + 2) * n + j] = C[(size_t)(i + 2) * n + j] + a2;
          C[(size_t)(i + 3) * n + j] = C[(size_t)(i + 3) * n + j] + a3;
        }
        for (int j = j8End; j < j4End; j += 4) {  // goJ4U4 (K.hs:697-724)
          double* c0p = C + (size_t)i * n + j;
          __m256d c0 = ld(c0p), c1 = ld(c0p + n), c2 = ld(c0p + 2 * (size_t)n),
                  c3 = ld(c0p + 3 * (size_t)n);
          for (int kk = bk; kk < kEnd; ++kk) {
            const __m256d bv = ld(B + (size_t)kk * n + j);
            c0 = fma4(bc(A[(size_t)i * k + kk]), bv, c0);
            c1 = fma4(bc(A[(size_t)(i + 1) * k + kk]), bv, c1);
            c2 = fma4(bc(A[(size_t)(i + 2) * k + kk]), bv, c2);
            c3 = fma4(bc(A[(size_t)(i + 3) * k + kk]), bv, c3);
          }
          st(c0p, c0); st(c0p + n, c1); st(c0p + 2 * (size_t)n, c2); st(c0p + 3 * (size_t)n, c3);
        }
        for (int j = 0; j < j8End; j += 8) {  // goJ8P4 + goKP4x8 (K.hs:626-671)
          const double* pan = &bp[(size_t)(j / 8) * kc * 8];
          double* r0 = C + (size_t)i * n + j;
          double* r1 = r0 + n;
          double* r2 = r0 + 2 * (size_t)n;
          double* r3 = r0 + 3 * (size_t)n;
          __m256d c00 = ld(r0), c01 = ld(r0 + 4), c10 = ld(r1), c11 = ld(r1 + 4);
          __m256d c20 = ld(r2), c21 = ld(r2 + 4), c30 = ld(r3), c31 = ld(r3 + 4);
          for (int kl = 0; kl < kc; ++kl) {
            const __m256d bv0 = ld(pan + (size_t)kl * 8), bv1 = ld(pan + (size_t)kl * 8 + 4);
            const int kk = bk + kl;
            const __m256d a0 = bc(A[(size_t)i * k + kk]);
            const __m256d a1 = bc(A[(size_t)(i + 1) * k + kk]);
            const __m256d a2 = bc(A[(size_t)(i + 2) * k + kk]);
            const __m256d a3 = bc(A[(size_t)(i + 3) * k + kk]);
            c00 = fma4(a0, bv0, c00); c01 = fma4(a0, bv1, c01);
            c10 = fma4(a1, bv0, c10); c11 = fma4(a1, bv1, c11);
            c20 = fma4(a2, bv0, c20); c21 = fma4(a2, bv1, c21);
            c30 = fma4(a3, bv0, c30); c31 = fma4(a3, bv1, c31);
          }
          st(r0, c00); st(r0 + 4, c01); st(r1, c10); st(r1 + 4, c11);
          st(r2, c20); st(r2 + 4, c21); st(r3, c30); st(r3 + 4, c31);
        }
      }
      for (int i = i4End; i < iEnd; ++i) {  // goI1P
        for (int j = j4End; j < n; ++j) {   // goJSU1 (K.hs:783-801)
          double acc = 0.0;
          for (int kk = bk; kk < kEnd; ++kk) acc = acc + A[(size_t)i * k + kk] * B[(size_t)kk * n + j];
          C[(size_t)i * n + j] = C[(size_t)i * n + j] + acc;
        }
        for (int j = j8End; j < j4End; j += 4) {  // goJ4U1 (K.hs:758-773)
          __m256d c0 = ld(C + (size_t)i * n + j);
          for (int kk = bk; kk < kEnd; ++kk)
            c0 = fma4(bc(A[(size_t)i * k + kk]), ld(B + (size_t)kk * n + j), c0);
          st(C + (size_t)i * n + j, c0);
        }
        for (int j = 0; j < j8End; j += 8) {  // goJ8P1 + goKP1x8 (K.hs:677-694)
          const double* pan = &bp[(size_t)(j / 8) * kc * 8];
          __m256d c0 = ld(C + (size_t)i * n + j), c1 = ld(C + (size_t)i * n + j + 4);
          for (int kl = 0; kl < kc; ++kl) {
            const __m256d av = bc(A[(size_t)i * k + bk + kl]);
            c0 = fma4(av, ld(pan + (size_t)kl * 8), c0);
            c1 = fma4(av, ld(pan + (size_t)kl * 8 + 4), c1);
          }
          st(C + (size_t)i * n + j, c0); st(C + (size_t)i * n + j + 4, c1);
        }
      }
    }
  }
}

// rawGemmKernel dispatch (K.hs:145-159): packed when min(m,k,n) >= 96.
void gemm_kernel(const double* A, const double* B, double* C, int m, int k, int n) {
  if (m <= 0 || n <= 0) return;
  if (std::min(m, std::min(k, n)) >= 96)
    gemm_packed(A, B, C, 0, m, m, k, n);
  else
    gemm_bibj(A, B, C, 0, m, 0, n, m, k, n);
}

// rawDot (K.hs:84-115)
double raw_dot(const double* x, const double* y, int n) {
  const int n4 = n - rem_(n, 4);
  __m256d acc = _mm256_setzero_pd();
  for (int i = 0; i < n4; i += 4) acc = fma4(ld(x + i), ld(y + i), acc);
  double s = hsum(acc);
  for (int i = n4; i < n; ++i) s = s + x[i] * y[i];
  return s;
}

// ---------------------------------------------------------------------------
// LU kernels (K.hs:1414-1556)
// ---------------------------------------------------------------------------
double absd(double v) { return (v >= 0.0) ? v : -v; }  // K.hs:1549

// rawPivotSearch (K.hs:1541-1556): strict '>' keeps the first maximum.
int pivot_search(const double* A, int n, int k, int fromRow) {
  int best = fromRow;
  double bestVal = absd(A[(size_t)fromRow * n + k]);
  for (int i = fromRow + 1; i < n; ++i) {
    const double av = absd(A[(size_t)i * n + k]);
    if (av > bestVal) { best = i; bestVal = av; }
  }
  return best;
}

// rawSwapRows (K.hs:1507-1537)
void swap_rows(double* A, int n, int r1, int r2, int fromCol) {
  double* a = A + (size_t)r1 * n;
  double* b = A + (size_t)r2 * n;
  for (int j = fromCol; j < n; ++j) std::swap(a[j], b[j]);
}

// rawLUEliminateColumnTo (K.hs:1464-1503); colEnd = n gives rawLUEliminateColumn
// (K.hs:1414-1458).  Multipliers for all rows below, update columns (k, colEnd).
void lu_eliminate_to(double* A, int n, int k, int colEnd) {
  const double akk = A[(size_t)k * n + k];
  const double* krow = A + (size_t)k * n;
  for (int i = k + 1; i < n; ++i) {
    double* irow = A + (size_t)i * n;
    const double mult = irow[k] / akk;
    irow[k] = mult;
    const int jSpan = colEnd - k - 1;
    const int jStart = k + 1;
    const int j4End = jStart + (jSpan - rem_(jSpan, 4));
    const __m256d neg = bc(-mult);
    for (int j = jStart; j < j4End; j += 4) st(irow + j, fma4(neg, ld(krow + j), ld(irow + j)));
    for (int j = j4End; j < colEnd; ++j) irow[j] = irow[j] - mult * krow[j];
  }
}

// rawTriSolvePanelTrail (LU.hs:364-407)
void tri_solve_panel_trail(double* A, int n, int k0, int panelEnd) {
  for (int k = k0; k < panelEnd; ++k) {
    const double* krow = A + (size_t)k * n;
    for (int i = k + 1; i < panelEnd; ++i) {
      double* irow = A + (size_t)i * n;
      const double negLik = -irow[k];
      const __m256d nv = bc(negLik);
      const int jSpan = n - panelEnd;
      const int j4End = panelEnd + (jSpan - rem_(jSpan, 4));
      for (int j = panelEnd; j < j4End; j += 4) st(irow + j, fma4(nv, ld(krow + j), ld(irow + j)));
      for (int j = j4End; j < n; ++j) irow[j] = irow[j] + negLik * krow[j];
    }
  }
}

// panelLUFactor (LU.hs:311-357).  Returns the swap list [(k, pivRow)] in order.
void panel_lu_factor(double* A, int n, int nb, std::vector<int>& pk, std::vector<int>& pr) {
  std::vector<double> bufL, bufU, bufC;
  int k0 = 0;
  while (!(k0 >= n - 1)) {
    const int panelEnd = std::min(k0 + nb, n);
    const int actualNb = panelEnd - k0;
    for (int k = k0; k < panelEnd; ++k) {
      const int piv = pivot_search(A, n, k, k);
      if (piv != k) swap_rows(A, n, k, piv, 0);
      lu_eliminate_to(A, n, k, panelEnd);
      pk.push_back(k);
      pr.push_back(piv);
    }
    if (panelEnd < n) {
      tri_solve_panel_trail(A, n, k0, panelEnd);
      const int mT = n - panelEnd, nT = n - panelEnd;
      // rawCopySubmatrixToDense (LU.hs:411-440): L21 and U12 as dense buffers
      bufL.resize((size_t)mT * actualNb);
      bufU.resize((size_t)actualNb * nT);
      for (int i = 0; i < actualNb; ++i)
        for (int j = 0; j < nT; ++j) bufU[(size_t)i * nT + j] = A[(size_t)(k0 + i) * n + panelEnd + j];
      bufC.resize((size_t)mT * nT);
      // k = actualNb <= 32 < 96: rawGemmKernel takes the unpacked path
      // (rawGemmBIBJSlice over all rows), split here by 64-row tiles
      double* Lp = bufL.data();
      double* Up = bufU.data();
      double* Cp = bufC.data();
      par_rows(mT, [=](int r0, int r1) {
        for (int i = r0; i < r1; ++i)
          for (int j = 0; j < actualNb; ++j) Lp[(size_t)i * actualNb + j] = A[(size_t)(panelEnd + i) * n + k0 + j];
        std::memset(Cp + (size_t)r0 * nT, 0, (size_t)(r1 - r0) * nT * sizeof(double));  // rawZeroDoubles
        gemm_bibj(Lp, Up, Cp, r0, r1, 0, nT, mT, actualNb, nT);
        // rawSubtractFromStrided (LU.hs:444-476): a + (-c) == a - c
        for (int i = r0; i < r1; ++i) {
          double* arow = A + (size_t)(panelEnd + i) * n + panelEnd;
          const double* crow = Cp + (size_t)i * nT;
          for (int j = 0; j < nT; ++j) arow[j] = arow[j] - crow[j];
        }
      });
    }
    k0 = panelEnd;
  }
}

// Factor phase of luSolveP (LU.hs:275-285).
void lu_factor_p(double* A, int n, std::vector<int>& pk, std::vector<int>& pr) {
  if (n >= 64) {
    panel_lu_factor(A, n, 32, pk, pr);
  } else {
    for (int k = 0; k <= n - 2; ++k) {
      const int piv = pivot_search(A, n, k, k);
      if (piv != k) swap_rows(A, n, k, piv, 0);
      lu_eliminate_to(A, n, k, n);
      pk.push_back(k);
      pr.push_back(piv);
    }
  }
}

// rawForwardSubUnitPackedSIMD (K.hs:2205-2256) and the Cholesky variant with a
// non-unit diagonal (K.hs:2319-2371): dot form with two 4-lane accumulators.
void forward_sub_packed(const double* L, int n, double* x, bool unitDiag) {
  for (int i = 0; i < n; ++i) {
    const double* row = L + (size_t)i * n;
    const int dotLen = i;
    const int d8End = dotLen - rem_(dotLen, 8);
    const int d4End = dotLen - rem_(dotLen, 4);
    __m256d acc0 = _mm256_setzero_pd(), acc1 = _mm256_setzero_pd();
    for (int k = 0; k < d8End; k += 8) {
      acc0 = fma4(ld(row + k), ld(x + k), acc0);
      acc1 = fma4(ld(row + k + 4), ld(x + k + 4), acc1);
    }
    for (int k = d8End; k < d4End; k += 4) acc0 = fma4(ld(row + k), ld(x + k), acc0);
    double dot = hsum(_mm256_add_pd(acc0, acc1));
    for (int k = d4End; k < dotLen; ++k) dot = dot + row[k] * x[k];
    if (unitDiag)
      x[i] = x[i] - dot;
    else
      x[i] = (x[i] - dot) / row[i];
  }
}

// rawBackSubPackedSIMD (K.hs:2261-2314)
void back_sub_packed(const double* U, int n, double* x) {
  for (int i = n - 1; i >= 0; --i) {
    const double* row = U + (size_t)i * n;
    const int dotStart = i + 1;
    const int dotLen = n - i - 1;
    const int d8End = dotStart + (dotLen - rem_(dotLen, 8));
    const int d4End = dotStart + (dotLen - rem_(dotLen, 4));
    __m256d acc0 = _mm256_setzero_pd(), acc1 = _mm256_setzero_pd();
    for (int k = dotStart; k < d8End; k += 8) {
      acc0 = fma4(ld(row + k), ld(x + k), acc0);
      acc1 = fma4(ld(row + k + 4), ld(x + k + 4), acc1);
    }
    for (int k = d8End; k < d4End; k += 4) acc0 = fma4(ld(row + k), ld(x + k), acc0);
    double dot = hsum(_mm256_add_pd(acc0, acc1));
    for (int k = d4End; k < n; ++k) dot = dot + row[k] * x[k];
    x[i] = (x[i] - dot) / row[i];
  }
}

// rawBackSubCholTPackedSIMD (K.hs:2378-2430): solves G^T x = y, SAXPY form.
void back_sub_chol_t_packed(const double* G, int n, double* x) {
  for (int j = n - 1; j >= 0; --j) {
    const double* row = G + (size_t)j * n;
    const double xj = x[j] / row[j];
    x[j] = xj;
    const __m256d neg = bc(-xj);
    const int u8End = j - rem_(j, 8);
    const int u4End = j - rem_(j, 4);
    for (int i = 0; i < u8End; i += 8) {
      st(x + i, fma4(neg, ld(row + i), ld(x + i)));
      st(x + i + 4, fma4(neg, ld(row + i + 4), ld(x + i + 4)));
    }
    for (int i = u8End; i < u4End; i += 4) st(x + i, fma4(neg, ld(row + i), ld(x + i)));
    for (int i = u4End; i < j; ++i) x[i] = x[i] - row[i] * xj;
  }
}

// rawCholColumnSIMDFrom (K.hs:2137-2195); fromCol = 0 is rawCholColumnSIMD
// (K.hs:2071-2131), whose loop bounds coincide.
void chol_column_from(double* G, int n, int j, int fromCol) {
  const double* jrow = G + (size_t)j * n;
  const int dotLen = j - fromCol;
  const int dotLen4 = dotLen - rem_(dotLen, 4);
  const int k4End = fromCol + dotLen4;
  for (int i = j; i < n; ++i) {
    const double* irow = G + (size_t)i * n;
    double dot;
    if (fromCol < k4End) {
      __m256d acc = _mm256_setzero_pd();
      for (int k = fromCol; k < k4End; k += 4) acc = fma4(ld(irow + k), ld(jrow + k), acc);
      dot = hsum(acc);
      for (int k = k4End; k < j; ++k) dot = dot + irow[k] * jrow[k];
    } else {
      dot = 0.0;
      for (int k = fromCol; k < j; ++k) dot = dot + irow[k] * jrow[k];
    }
    G[(size_t)i * n + j] = G[(size_t)i * n + j] - dot;
  }
  const double sjj = std::sqrt(G[(size_t)j * n + j]);
  G[(size_t)j * n + j] = sjj;
  for (int i = j + 1; i < n; ++i) G[(size_t)i * n + j] = G[(size_t)i * n + j] / sjj;
}

// panelCholFactor (Chol.hs:279-321): left-looking panels of nb columns.
void panel_chol_factor(double* G, int n, int nb) {
  std::vector<double> bufA, bufBT, bufC;
  for (int j = 0; j < n;) {
    const int jb = std::min(nb, n - j);
    const int nBelow = n - j;
    if (j > 0) {
      bufA.resize((size_t)nBelow * j);  // rawCopyCholSubmatrix (Chol.hs:325-358)
      bufBT.resize((size_t)j * jb);  // rawCopyCholTranspose (Chol.hs:363-384)
      for (int i = 0; i < jb; ++i)
        for (int c = 0; c < j; ++c) bufBT[(size_t)c * jb + i] = G[(size_t)(j + i) * n + c];
      bufC.resize((size_t)nBelow * jb);
      // n = jb <= 32 < 96: the unpacked path, split by 64-row tiles
      double* Ap = bufA.data();
      double* Bp = bufBT.data();
      double* Cp = bufC.data();
      const int jj = j;
      par_rows(nBelow, [=](int r0, int r1) {
        for (int i = r0; i < r1; ++i) std::memcpy(Ap + (size_t)i * jj, G + (size_t)(jj + i) * n, (size_t)jj * sizeof(double));
        std::memset(Cp + (size_t)r0 * jb, 0, (size_t)(r1 - r0) * jb * sizeof(double));
        gemm_bibj(Ap, Bp, Cp, r0, r1, 0, jb, nBelow, jj, jb);
        for (int i = r0; i < r1; ++i)  // rawCholSubtractPanel (Chol.hs:388-416)
          for (int c = 0; c < jb; ++c)
            G[(size_t)(jj + i) * n + jj + c] = G[(size_t)(jj + i) * n + jj + c] - Cp[(size_t)i * jb + c];
      });
    }
    for (int c = j; c < j + jb; ++c) chol_column_from(G, n, c, j);
    j += jb;
  }
}

// Factor phase of choleskySolveP (Chol.hs:241-258): G starts as the lower
// triangle of A with zeros above (copyLowerTriangle, Chol.hs:420-434).
void chol_factor_p(const double* A, double* G, int n) {
  std::memset(G, 0, (size_t)n * n * sizeof(double));
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) G[(size_t)i * n + j] = A[(size_t)i * n + j];
  if (n >= 64)
    panel_chol_factor(G, n, 32);
  else
    for (int j = 0; j < n; ++j) chol_column_from(G, n, j, 0);
}

// Haskell `compare` on Double: LT if x<y, EQ if x==y, else GT (NaN -> GT).
int hs_compare(double x, double y) { return (x < y) ? -1 : ((x == y) ? 0 : 1); }

}  // namespace

extern "C" {

// C += A * B through rawGemmKernel (K.hs:145-153).  Dense row-major.
void orc_gemm_kernel(const double* A, const double* B, double* C, int m, int k, int n) {
  gemm_kernel(A, B, C, m, k, n);
}

// matMulP (L3.hs:183-207): C = A * B with C zero-initialised first.
void orc_matmul_p(const double* A, const double* B, double* C, int m, int k, int n) {
  std::memset(C, 0, (size_t)m * n * sizeof(double));
  gemm_kernel(A, B, C, m, k, n);
}

// matMulPPar (L3.hs:214-294): 2D (or 1D) partition of C over threads, each
// tile computed by rawGemmBIBJSlice.  Elements on the FMA path are bitwise
// identical to matMulP; the set of columns that take the scalar (separately
// rounded) tail depends on where the column chunks start, exactly as in the
// reference, so results can differ from matMulP in the last bits of a few
// columns when chunk widths are not multiples of 4.
void orc_matmul_par(const double* A, const double* B, double* C, int m, int k, int n, int caps) {
  std::memset(C, 0, (size_t)m * n * sizeof(double));
  const int minRowsPerThread = 16;
  const int maxThreads = std::max(1, m / minRowsPerThread);
  const int numThreads = std::min(caps, std::min(m, maxThreads));
  if (numThreads <= 1) {
    gemm_kernel(A, B, C, m, k, n);
    return;
  }
  std::vector<std::thread> th;
  const bool use2D = numThreads >= 4 && m >= 128 && n >= 128;
  if (use2D) {
    // gridDims (L3.hs:280-294)
    int p = numThreads;
    int sq = (int)std::floor(std::sqrt((double)p));
    double target = (double)m / (double)std::max(1, n);
    auto score = [&](int pr, int pc) { return std::fabs((double)pr / std::max(1, pc) - target); };
    int bpr = 1, bpc = p;
    bool first = true;
    for (int i = 1; i <= sq; ++i)
      if (p % i == 0) {
        if (first) { bpr = i; bpc = p / i; first = false; }
        else if (score(bpr, bpc) > score(i, p / i)) { bpr = i; bpc = p / i; }
      }
    if (score(bpc, bpr) < score(bpr, bpc)) std::swap(bpr, bpc);
    const int rChunk = (m + bpr - 1) / bpr, cChunk = (n + bpc - 1) / bpc;
    for (int tr = 0; tr < bpr; ++tr)
      for (int tc = 0; tc < bpc; ++tc) {
        const int b0 = tr * rChunk, b1 = std::min(b0 + rChunk, m);
        const int c0 = tc * cChunk, c1 = std::min(c0 + cChunk, n);
        th.emplace_back([=] { if (b0 < b1 && c0 < c1) gemm_bibj(A, B, C, b0, b1, c0, c1, m, k, n); });
      }
  } else {
    const int chunk = (m + numThreads - 1) / numThreads;
    for (int t = 0; t < numThreads; ++t) {
      const int b0 = t * chunk, b1 = std::min(b0 + chunk, m);
      th.emplace_back([=] { if (b0 < b1) gemm_bibj(A, B, C, b0, b1, 0, n, m, k, n); });
    }
  }
  for (auto& t : th) t.join();
}

// gemm (L3.hs:102-131): C = beta*C0, then 32-blocked ikj accumulation of
// (alpha*a_il)*b_lj with separate roundings.
void orc_gemm_generic(double alpha, const double* A, const double* B, double beta,
                      const double* C0, double* C, int m, int k, int n) {
  const int bs = 32;
  for (size_t i = 0; i < (size_t)m * n; ++i) C[i] = beta * C0[i];
  for (int bi = 0; bi < m; bi += bs)
    for (int bk = 0; bk < k; bk += bs)
      for (int bj = 0; bj < n; bj += bs) {
        const int iE = std::min(bi + bs, m), kE = std::min(bk + bs, k), jE = std::min(bj + bs, n);
        for (int i = bi; i < iE; ++i)
          for (int l = bk; l < kE; ++l) {
            const double aik = alpha * A[(size_t)i * k + l];
            for (int j = bj; j < jE; ++j) C[(size_t)i * n + j] = C[(size_t)i * n + j] + aik * B[(size_t)l * n + j];
          }
      }
}

// In-place LU of luSolveP's factor phase (LU.hs:265-285).  Writes the packed
// LU into A and the swap list (pivot row for step k) into swaps[0..nswaps).
// Returns nswaps (n-1 for n < 64; the panel path may record step n-1 too).
int orc_lu_factor_p(double* A, int n, int* swap_k, int* swap_row) {
  std::vector<int> pk, pr;
  lu_factor_p(A, n, pk, pr);
  for (size_t i = 0; i < pk.size(); ++i) { swap_k[i] = pk[i]; swap_row[i] = pr[i]; }
  return (int)pk.size();
}

// luSolveP (LU.hs:265-304) for nrhs right-hand sides (each column of the n x
// nrhs row-major B solved independently, as a loop over the single-vector API).
// LU (n x n) and the swap list are returned when the pointers are non-null.
int orc_lu_solve_p(const double* A, const double* B, double* X, int n, int nrhs, double* LUout,
                   int* swap_k, int* swap_row) {
  std::vector<double> lu(A, A + (size_t)n * n);
  std::vector<int> pk, pr;
  lu_factor_p(lu.data(), n, pk, pr);
  std::vector<double> x(n);
  for (int c = 0; c < nrhs; ++c) {
    for (int i = 0; i < n; ++i) x[i] = B[(size_t)i * nrhs + c];  // copyVector
    for (size_t s = 0; s < pk.size(); ++s)                        // applyPivotsForward (LU.hs:493-507)
      if (pk[s] != pr[s]) std::swap(x[pk[s]], x[pr[s]]);
    forward_sub_packed(lu.data(), n, x.data(), true);
    back_sub_packed(lu.data(), n, x.data());
    for (int i = 0; i < n; ++i) X[(size_t)i * nrhs + c] = x[i];
  }
  if (LUout) std::memcpy(LUout, lu.data(), (size_t)n * n * sizeof(double));
  if (swap_k)
    for (size_t i = 0; i < pk.size(); ++i) { swap_k[i] = pk[i]; swap_row[i] = pr[i]; }
  return (int)pk.size();
}

// Factor phase of choleskySolveP (Chol.hs:241-258).  G is n x n; the lower
// triangle holds the factor.  Entries above the diagonal inside the 32-wide
// diagonal panels carry the GEMM's side effects exactly as the reference does.
void orc_chol_factor_p(const double* A, double* G, int n) { chol_factor_p(A, G, n); }

// choleskySolveP (Chol.hs:241-273) for nrhs columns of B.
void orc_chol_solve_p(const double* A, const double* B, double* X, int n, int nrhs, double* Gout) {
  std::vector<double> g((size_t)n * n);
  chol_factor_p(A, g.data(), n);
  std::vector<double> x(n);
  for (int c = 0; c < nrhs; ++c) {
    for (int i = 0; i < n; ++i) x[i] = B[(size_t)i * nrhs + c];
    forward_sub_packed(g.data(), n, x.data(), false);
    back_sub_chol_t_packed(g.data(), n, x.data());
    for (int i = 0; i < n; ++i) X[(size_t)i * nrhs + c] = x[i];
  }
  if (Gout) std::memcpy(Gout, g.data(), (size_t)n * n * sizeof(double));
}

// lu (LU.hs:121-167): unblocked outer-product LU.  Pivot by maximumBy on |a|
// (the LAST maximum on ties), row swaps over all columns, elimination skipped
// when the pivot is exactly zero.  perm[i] = original row now at row i.
void orc_lu_generic(const double* A, double* LU, int* perm, int n) {
  std::memcpy(LU, A, (size_t)n * n * sizeof(double));
  for (int i = 0; i < n; ++i) perm[i] = i;
  for (int k = 0; k <= n - 2; ++k) {
    int best = k;
    double bestV = std::fabs(LU[(size_t)k * n + k]);
    for (int i = k + 1; i < n; ++i) {  // maximumBy (comparing snd): keep x only on GT
      const double v = std::fabs(LU[(size_t)i * n + k]);
      if (hs_compare(bestV, v) != 1) { best = i; bestV = v; }
    }
    if (best != k) {
      std::swap(perm[k], perm[best]);
      for (int j = 0; j < n; ++j) std::swap(LU[(size_t)k * n + j], LU[(size_t)best * n + j]);
    }
    const double akk = LU[(size_t)k * n + k];
    if (akk != 0.0) {
      for (int i = k + 1; i < n; ++i) {
        const double mult = LU[(size_t)i * n + k] / akk;
        LU[(size_t)i * n + k] = mult;
        for (int j = k + 1; j < n; ++j)
          LU[(size_t)i * n + j] = LU[(size_t)i * n + j] - mult * LU[(size_t)k * n + j];
      }
    }
  }
}

// luSolve (LU.hs:240-259): lu, then pb[i] = b[perm[i]], forwardSubUnit
// (Tri.hs:187-209) and backSub (Tri.hs:136-160), both column oriented.
void orc_lu_solve_generic(const double* A, const double* b, double* x, int n) {
  std::vector<double> lu((size_t)n * n);
  std::vector<int> perm(n);
  orc_lu_generic(A, lu.data(), perm.data(), n);
  for (int i = 0; i < n; ++i) x[i] = b[perm[i]];
  for (int j = 0; j < n; ++j) {
    const double xj = x[j];
    for (int i = j + 1; i < n; ++i) x[i] = x[i] - lu[(size_t)i * n + j] * xj;
  }
  for (int j = n - 1; j >= 0; --j) {
    const double xj = x[j] / lu[(size_t)j * n + j];
    x[j] = xj;
    for (int i = 0; i < j; ++i) x[i] = x[i] - lu[(size_t)i * n + j] * xj;
  }
}

// cholesky (Chol.hs:114-147): outer-product column loop on the lower
// triangle; the upper triangle of G is zero.
void orc_cholesky_generic(const double* A, double* G, int n) {
  std::memset(G, 0, (size_t)n * n * sizeof(double));
  for (int j = 0; j < n; ++j)
    for (int i = j; i < n; ++i) G[(size_t)i * n + j] = A[(size_t)i * n + j];
  for (int j = 0; j < n; ++j) {
    for (int k = 0; k < j; ++k) {
      const double gjk = G[(size_t)j * n + k];
      for (int i = j; i < n; ++i) G[(size_t)i * n + j] = G[(size_t)i * n + j] - G[(size_t)i * n + k] * gjk;
    }
    const double sjj = std::sqrt(G[(size_t)j * n + j]);
    G[(size_t)j * n + j] = sjj;
    for (int i = j + 1; i < n; ++i) G[(size_t)i * n + j] = G[(size_t)i * n + j] / sjj;
  }
}

// choleskySolve (Chol.hs:229-235): forwardSub with G (Tri.hs:90-112), then
// backSub with G^T (Tri.hs:136-160).
void orc_chol_solve_generic(const double* A, const double* b, double* x, int n) {
  std::vector<double> g((size_t)n * n);
  orc_cholesky_generic(A, g.data(), n);
  for (int i = 0; i < n; ++i) x[i] = b[i];
  for (int j = 0; j < n; ++j) {
    const double xj = x[j] / g[(size_t)j * n + j];
    x[j] = xj;
    for (int i = j + 1; i < n; ++i) x[i] = x[i] - g[(size_t)i * n + j] * xj;
  }
  for (int j = n - 1; j >= 0; --j) {  // gt[i][j] = g[j][i]
    const double xj = x[j] / g[(size_t)j * n + j];
    x[j] = xj;
    for (int i = 0; i < j; ++i) x[i] = x[i] - g[(size_t)j * n + i] * xj;
  }
}

// det (LU.hs:534-557): product of U's diagonal (left fold from 1) times the
// sign of the permutation (countSwaps).
double orc_det(const double* A, int n) {
  std::vector<double> lu((size_t)n * n);
  std::vector<int> perm(n);
  orc_lu_generic(A, lu.data(), perm.data(), n);
  double prod = 1.0;
  for (int i = 0; i < n; ++i) prod = prod * lu[(size_t)i * n + i];
  std::vector<int> p(perm);
  int swaps = 0;
  for (int i = 0; i < n; ++i) {
    if (p[i] == i) continue;
    for (int j = i + 1; j < n; ++j)
      if (p[j] == i) { p[j] = p[i]; break; }
    ++swaps;
  }
  return (swaps % 2 == 0) ? prod : -prod;
}

// matvecP -> rawGemv (L2.hs:131-139, K.hs:119-134): y_i = rawDot(row i, x).
void orc_matvec_p(const double* A, const double* x, double* y, int m, int n) {
  for (int i = 0; i < m; ++i) y[i] = raw_dot(A + (size_t)i * n, x, n);
}

// Generic matvec (L2.hs:123-127): left fold acc + a_ij * x_j from 0.
void orc_matvec_generic(const double* A, const double* x, double* y, int m, int n) {
  for (int i = 0; i < m; ++i) {
    double acc = 0.0;
    for (int j = 0; j < n; ++j) acc = acc + A[(size_t)i * n + j] * x[j];
    y[i] = acc;
  }
}

// Threads used by the row-parallel trailing updates (0 = all hardware threads).
void orc_set_threads(int t) { g_threads = t; }

// luNoPivot (LU.hs:196-214): outer-product LU without pivoting, in place,
// GVL4 Algorithm 3.2.1.  For each k: multipliers a_ik / a_kk for the rows
// below, then a_ij - a_ik * a_kj (separately rounded) for j > k, i > k, with
// j the outer loop; the order inside one k does not change any value.
void orc_lu_nopivot(double* A, int n) {
  for (int k = 0; k <= n - 2; ++k) {
    const double akk = A[(size_t)k * n + k];
    for (int i = k + 1; i < n; ++i) A[(size_t)i * n + k] = A[(size_t)i * n + k] / akk;
    for (int j = k + 1; j < n; ++j) {
      const double akj = A[(size_t)k * n + j];
      for (int i = k + 1; i < n; ++i) A[(size_t)i * n + j] = A[(size_t)i * n + j] - A[(size_t)i * n + k] * akj;
    }
  }
}

// choleskyGaxpy (Chol.hs:173-204), GVL4 Algorithm 4.2.2: G starts as the
// lower triangle of A (zeros above); column j gets g_ij - g_ik * g_jk for
// k = 0 .. j-1 in order, then every g_ij (i >= j) is divided by sqrt(g_jj).
void orc_cholesky_gaxpy(const double* A, double* G, int n) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) G[(size_t)i * n + j] = (i >= j) ? A[(size_t)i * n + j] : 0.0;
  for (int j = 0; j < n; ++j) {
    for (int k = 0; k < j; ++k) {
      const double gjk = G[(size_t)j * n + k];
      for (int i = j; i < n; ++i) G[(size_t)i * n + j] = G[(size_t)i * n + j] - G[(size_t)i * n + k] * gjk;
    }
    const double sjj = std::sqrt(G[(size_t)j * n + j]);
    for (int i = j; i < n; ++i) G[(size_t)i * n + j] = G[(size_t)i * n + j] / sjj;
  }
}

// tridiagSolve (Solve/Banded.hs:292-342), GVL4 Algorithm 4.3.6: LDL^T of the
// SPD tridiagonal (diag, supdiag[0..n-2]) folded with the substitutions.
void orc_tridiag_solve(const double* diag, const double* supdiag, const double* b, double* x, int n) {
  if (n <= 0) return;
  std::vector<double> alpha(diag, diag + n), beta(n, 0.0);
  for (int i = 0; i < n - 1; ++i) beta[i] = supdiag[i];
  for (int i = 0; i < n; ++i) x[i] = b[i];
  for (int k = 1; k < n; ++k) {  // t = beta(k-1), beta(k-1) = t / alpha(k-1), alpha(k) -= t * beta(k-1)
    const double t = beta[k - 1];
    const double bk1 = t / alpha[k - 1];
    beta[k - 1] = bk1;
    alpha[k] = alpha[k] - t * bk1;
  }
  for (int k = 1; k < n; ++k) x[k] = x[k] - beta[k - 1] * x[k - 1];
  x[n - 1] = x[n - 1] / alpha[n - 1];
  for (int k = n - 2; k >= 0; --k) x[k] = x[k] / alpha[k] - beta[k] * x[k + 1];
}

// normInf (Norms.hs:135-141): the largest row sum of |a_ij|, each row summed
// as a left fold from 0 in column order.  vnormInf (Norms.hs:94-96) of x is
// normInf of x as an n x 1 matrix.
double orc_norm_inf(const double* A, int m, int n) {
  double best = 0.0;
  for (int i = 0; i < m; ++i) {
    double acc = 0.0;
    for (int j = 0; j < n; ++j) acc = acc + std::fabs(A[(size_t)i * n + j]);
    best = (i == 0) ? acc : std::max(best, acc);
  }
  return best;
}

// Throughput helper for the CPU baseline: `count` independent luSolveP solves
// of the same n x n system spread over `threads` host threads (the reference's
// luSolveP is single-threaded; independent solves are how it uses more cores).
void orc_lu_solve_p_many(const double* A, const double* b, double* x, int n, int count, int threads) {
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t)
    th.emplace_back([=] {
      std::vector<double> xl(n);
      for (int c = t; c < count; c += threads) orc_lu_solve_p(A, b, xl.data(), n, 1, nullptr, nullptr, nullptr);
      if (t == 0) std::memcpy(x, xl.data(), (size_t)n * sizeof(double));
    });
  for (auto& t : th) t.join();
}

void orc_chol_solve_p_many(const double* A, const double* b, double* x, int n, int count, int threads) {
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t)
    th.emplace_back([=] {
      std::vector<double> xl(n);
      for (int c = t; c < count; c += threads) orc_chol_solve_p(A, b, xl.data(), n, 1, nullptr);
      if (t == 0) std::memcpy(x, xl.data(), (size_t)n * sizeof(double));
    });
  for (auto& t : th) t.join();
}

}  // extern "C"
