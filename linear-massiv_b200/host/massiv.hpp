// massiv.hpp — C++ host mirror of linear-massiv's dense-solve API over the
// C ABI of lm_b200.h.
//
// The reference's types carry their dimensions at the type level
// (`Matrix (m :: Nat) (n :: Nat) r e`, Types.hs:90; `Vector n r e`,
// Types.hs:103) and its functions are pure.  Here:
//   massiv::Matrix<M, N>  — an M x N FP64 matrix resident in device memory,
//                           dimensions checked at compile time;
//   massiv::Vector<N>     — an N-vector resident in device memory;
//   gemm / matMul / lu / luSolve / cholesky / choleskySolve / det
//                         — pure functions: inputs are never modified,
//                           results are fresh device buffers.
// Numerical breakdown follows the reference: no exception, the result holds
// the Inf/NaN its arithmetic produces; the LAPACK-style info is available via
// the *Info variants.  CUDA or argument errors throw massiv::Error (the
// Haskell binding turns the same statuses into exceptions).
//
// Runtime-size values (the reference's SomeMatrix / SomeVector existentials)
// are massiv::SomeMatrix / SomeVector, with someMatrix, forget and reifyDim.
//
// File references: Types.hs, Internal.hs, Norms.hs (src/Numeric/LinearAlgebra/Massiv/),
// L2.hs = BLAS/Level2.hs, L3.hs = BLAS/Level3.hs, LU.hs = Solve/LU.hs,
// Chol.hs = Solve/Cholesky.hs.
#pragma once

#include <lm_b200.h>

#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace massiv {

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& what)
      : std::runtime_error(what + ": " + lm_status_string(s) + " " + lm_last_error()), status(s) {}
};

inline int check(int s, const char* what) {
  if (s < 0) throw Error(s, what);
  return s;
}

// One context per thread (the reference's capabilities); device 0 by default.
inline lm_ctx* context(int device = 0) {
  struct Holder {
    lm_ctx* c = nullptr;
    ~Holder() { if (c) lm_ctx_destroy(c); }
  };
  thread_local Holder h;
  if (!h.c) check(lm_ctx_create(&h.c, device), "lm_ctx_create");
  return h.c;
}

// Device buffer with shared ownership (values are immutable once built, so
// sharing is safe, like massiv's immutable arrays).
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(std::size_t count) : n_(count) {
    void* p = nullptr;
    if (count) check(lm_dmalloc(context(), &p, count * sizeof(double)), "lm_dmalloc");
    p_ = std::shared_ptr<double>(static_cast<double*>(p), [](double* q) { if (q) lm_dfree(context(), q); });
  }
  double* data() const { return p_.get(); }
  std::size_t size() const { return n_; }

 private:
  std::shared_ptr<double> p_;
  std::size_t n_ = 0;
};

template <std::size_t N>
class Vector {
 public:
  Vector() : buf_(N) {}
  // vector (Types.hs:131-140): from host values, N of them.
  static Vector fromHost(const std::vector<double>& v) {
    if (v.size() != N) throw Error(LM_ERR_ARG, "Vector::fromHost: wrong length");
    Vector out;
    if (N) check(lm_h2d(context(), out.data(), v.data(), N * sizeof(double)), "lm_h2d");
    return out;
  }
  std::vector<double> toHost() const {
    std::vector<double> v(N);
    if (N) check(lm_d2h(context(), v.data(), data(), N * sizeof(double)), "lm_d2h");
    return v;
  }
  double* data() const { return buf_.data(); }
  static constexpr std::size_t size() { return N; }

 private:
  DeviceBuffer buf_;
};

template <std::size_t M, std::size_t N>
class Matrix {
 public:
  Matrix() : buf_(M * N) {}
  // matrix (Types.hs:121-130): row-major host values, M*N of them.
  static Matrix fromHost(const std::vector<double>& v) {
    if (v.size() != M * N) throw Error(LM_ERR_ARG, "Matrix::fromHost: wrong size");
    Matrix out;
    if (M * N) check(lm_h2d(context(), out.data(), v.data(), M * N * sizeof(double)), "lm_h2d");
    return out;
  }
  // makeMatrix (Internal.hs:139): element function evaluated on the host.
  template <typename F>
  static Matrix make(F f) {
    std::vector<double> v(M * N);
    for (std::size_t i = 0; i < M; ++i)
      for (std::size_t j = 0; j < N; ++j) v[i * N + j] = f(i, j);
    return fromHost(v);
  }
  std::vector<double> toHost() const {
    std::vector<double> v(M * N);
    if (M * N) check(lm_d2h(context(), v.data(), data(), M * N * sizeof(double)), "lm_d2h");
    return v;
  }
  Matrix clone() const {
    Matrix out;
    if (M * N) out = fromHost(toHost());  // host round trip keeps this header on the ABI only
    return out;
  }
  double* data() const { return buf_.data(); }
  static constexpr std::size_t rows() { return M; }
  static constexpr std::size_t cols() { return N; }

 private:
  DeviceBuffer buf_;
};

// ---- BLAS-3 -----------------------------------------------------------------
// gemm alpha A B beta C (L3.hs:102-131)
template <std::size_t M, std::size_t K, std::size_t N>
Matrix<M, N> gemm(double alpha, const Matrix<M, K>& a, const Matrix<K, N>& b, double beta, const Matrix<M, N>& c) {
  Matrix<M, N> out = Matrix<M, N>::fromHost(c.toHost());
  check(lm_dgemm(context(), (int)M, (int)N, (int)K, alpha, a.data(), (int)K, b.data(), (int)N, beta, out.data(),
                 (int)N),
        "gemm");
  return out;
}

// matMul (L3.hs:144-147) — with the reference's RULE this is matMulP.
template <std::size_t M, std::size_t K, std::size_t N>
Matrix<M, N> matMul(const Matrix<M, K>& a, const Matrix<K, N>& b) {
  Matrix<M, N> out;
  check(lm_dgemm(context(), (int)M, (int)N, (int)K, 1.0, a.data(), (int)K, b.data(), (int)N, 0.0, out.data(),
                 (int)N),
        "matMul");
  return out;
}

// ---- LU -----------------------------------------------------------------------
template <std::size_t N>
struct LUResult {
  Matrix<N, N> lu;          // L strictly below the diagonal, U on and above
  std::vector<int> perm;    // (PA)[i] = A[perm[i]]  (LU.hs:121-122)
  int info;                 // 0, or k+1 for the first zero pivot
};

template <std::size_t N>
LUResult<N> luInfo(const Matrix<N, N>& a) {
  std::vector<double> h = a.toHost(), lu(N * N);
  std::vector<int> perm(N);
  int info = 0;
  check(lm_lu_host(context(), (int)N, h.data(), lu.data(), perm.data(), &info), "lu");
  return {Matrix<N, N>::fromHost(lu), perm, info};
}

// lu :: Matrix n n r e -> (Matrix n n r e, Array P Ix1 Int)  (LU.hs:121-167)
template <std::size_t N>
std::pair<Matrix<N, N>, std::vector<int>> lu(const Matrix<N, N>& a) {
  auto r = luInfo(a);
  return {r.lu, r.perm};
}

// luSolve / luSolveP (LU.hs:240-304)
template <std::size_t N>
Vector<N> luSolve(const Matrix<N, N>& a, const Vector<N>& b) {
  std::vector<double> A = a.toHost(), B = b.toHost(), X(N);
  int info = 0;
  check(lm_lu_solve_host(context(), (int)N, 1, A.data(), B.data(), X.data(), &info), "luSolve");
  return Vector<N>::fromHost(X);
}

// Device-resident variant: the factorisation and the solve stay in HBM.
template <std::size_t N>
Vector<N> luSolveDevice(const Matrix<N, N>& a, const Vector<N>& b, int* info_out = nullptr) {
  Matrix<N, N> work = a.clone();
  Vector<N> x = Vector<N>::fromHost(b.toHost());
  void* ipiv = nullptr;
  check(lm_dmalloc(context(), &ipiv, N * sizeof(int) + 1), "lm_dmalloc");
  int info = 0;
  int s = lm_dgesv(context(), (int)N, 1, work.data(), (int)N, static_cast<int*>(ipiv), x.data(), 1, &info);
  lm_dfree(context(), ipiv);
  check(s, "luSolve");
  if (info_out) *info_out = info;
  return x;
}

// det (LU.hs:534-545)
template <std::size_t N>
double det(const Matrix<N, N>& a) {
  std::vector<double> A = a.toHost();
  double d = 0.0;
  check(lm_det_host(context(), (int)N, A.data(), &d), "det");
  return d;
}

// ---- Cholesky ---------------------------------------------------------------
// cholesky (Chol.hs:114-147): G lower, zeros above.
template <std::size_t N>
Matrix<N, N> cholesky(const Matrix<N, N>& a, int* info_out = nullptr) {
  std::vector<double> A = a.toHost(), G(N * N);
  int info = 0;
  check(lm_cholesky_host(context(), (int)N, A.data(), G.data(), &info), "cholesky");
  if (info_out) *info_out = info;
  return Matrix<N, N>::fromHost(G);
}

// choleskySolve / choleskySolveP (Chol.hs:229-273)
template <std::size_t N>
Vector<N> choleskySolve(const Matrix<N, N>& a, const Vector<N>& b) {
  std::vector<double> A = a.toHost(), B = b.toHost(), X(N);
  int info = 0;
  check(lm_chol_solve_host(context(), (int)N, 1, A.data(), B.data(), X.data(), &info), "choleskySolve");
  return Vector<N>::fromHost(X);
}

// ---- BLAS-2, norms, adjacent solvers -------------------------------------------
// matvec (L2.hs:123-127; matvecP via its RULE, L2.hs:131-144): bitwise the
// reference's rawGemv order.
template <std::size_t M, std::size_t N>
Vector<M> matvec(const Matrix<M, N>& a, const Vector<N>& x) {
  Vector<M> y;
  check(lm_dgemv(context(), (int)M, (int)N, a.data(), (int)N, x.data(), y.data()), "matvec");
  return y;
}

// normInf (Norms.hs:135-141) and vnormInf (Norms.hs:94-96).
template <std::size_t M, std::size_t N>
double normInf(const Matrix<M, N>& a) {
  double r = 0.0;
  check(lm_dnorm_inf(context(), (int)M, (int)N, a.data(), (int)N, &r), "normInf");
  return r;
}
template <std::size_t N>
double vnormInf(const Vector<N>& x) {
  double r = 0.0;
  check(lm_dnorm_inf(context(), (int)N, 1, x.data(), 1, &r), "vnormInf");
  return r;
}

// luNoPivot (LU.hs:196-214): packed unit-L / U, no interchanges.
template <std::size_t N>
Matrix<N, N> luNoPivot(const Matrix<N, N>& a, int* info_out = nullptr) {
  std::vector<double> A = a.toHost(), LU(N * N);
  int info = 0;
  check(lm_lu_nopivot_host(context(), (int)N, A.data(), LU.data(), &info), "luNoPivot");
  if (info_out) *info_out = info;
  return Matrix<N, N>::fromHost(LU);
}

// choleskyGaxpy (Chol.hs:173-204): the same G as cholesky.
template <std::size_t N>
Matrix<N, N> choleskyGaxpy(const Matrix<N, N>& a, int* info_out = nullptr) {
  std::vector<double> A = a.toHost(), G(N * N);
  int info = 0;
  check(lm_cholesky_gaxpy_host(context(), (int)N, A.data(), G.data(), &info), "choleskyGaxpy");
  if (info_out) *info_out = info;
  return Matrix<N, N>::fromHost(G);
}

// tridiagSolve (Solve/Banded.hs:292-342): SPD tridiagonal from its diagonal and
// superdiagonal (entries 0 .. N-2 read).
template <std::size_t N>
Vector<N> tridiagSolve(const Vector<N>& diag, const Vector<N>& supdiag, const Vector<N>& b) {
  Vector<N> x;
  check(lm_dtridiag_solve(context(), (int)N, diag.data(), supdiag.data(), b.data(), x.data()), "tridiagSolve");
  return x;
}

// ---- runtime sizes: SomeMatrix / someMatrix / reifyDim -----------------------------
// The reference wraps arrays whose dimensions are known only at run time in
// existentials (SomeMatrix, SomeVector; someMatrix / someVector, Types.hs:165-178)
// and turns a runtime Int into a type-level Nat with reifyDim / reifyDim2
// (Internal.hs:123-129).  Here SomeMatrix / SomeVector carry their dimensions
// as values (device-resident like Matrix); forget() is the existential's
// constructor, reifyDim<Ns...> recovers a compile-time size from a runtime one
// over a list of candidate sizes (C++ cannot mint a new type at run time), and
// the operations on SomeMatrix check dimensions at run time where the
// reference's checks happen at compile time.
class SomeMatrix {
 public:
  SomeMatrix() = default;
  SomeMatrix(std::size_t rows, std::size_t cols) : rows_(rows), cols_(cols), buf_(rows * cols) {}
  std::size_t rows() const { return rows_; }
  std::size_t cols() const { return cols_; }
  double* data() const { return buf_.data(); }
  std::vector<double> toHost() const {
    std::vector<double> v(rows_ * cols_);
    if (!v.empty()) check(lm_d2h(context(), v.data(), data(), v.size() * sizeof(double)), "lm_d2h");
    return v;
  }

 private:
  std::size_t rows_ = 0, cols_ = 0;
  DeviceBuffer buf_;
};

class SomeVector {
 public:
  SomeVector() = default;
  explicit SomeVector(std::size_t n) : n_(n), buf_(n) {}
  std::size_t size() const { return n_; }
  double* data() const { return buf_.data(); }
  std::vector<double> toHost() const {
    std::vector<double> v(n_);
    if (n_) check(lm_d2h(context(), v.data(), data(), n_ * sizeof(double)), "lm_d2h");
    return v;
  }

 private:
  std::size_t n_ = 0;
  DeviceBuffer buf_;
};

// someMatrix (Types.hs:170-174): wrap row-major host values of a rows x cols array.
inline SomeMatrix someMatrix(std::size_t rows, std::size_t cols, const std::vector<double>& v) {
  if (v.size() != rows * cols) throw Error(LM_ERR_ARG, "someMatrix: wrong size");
  SomeMatrix m(rows, cols);
  if (!v.empty()) check(lm_h2d(context(), m.data(), v.data(), v.size() * sizeof(double)), "lm_h2d");
  return m;
}
// someVector (Types.hs:176-178)
inline SomeVector someVector(const std::vector<double>& v) {
  SomeVector x(v.size());
  if (!v.empty()) check(lm_h2d(context(), x.data(), v.data(), v.size() * sizeof(double)), "lm_h2d");
  return x;
}
// The existential's constructor: forget the static dimensions.
template <std::size_t M, std::size_t N>
SomeMatrix forget(const Matrix<M, N>& a) {
  return someMatrix(M, N, a.toHost());
}

// reifyDim (Internal.hs:123-125): call f(std::integral_constant<size_t, N>{})
// for the candidate N equal to n; Error(LM_ERR_ARG) when none is.
template <std::size_t... Ns, typename F>
auto reifyDim(std::size_t n, F&& f) {
  using R = decltype(f(std::integral_constant<std::size_t, 1>{}));
  bool hit = false;
  if constexpr (std::is_void_v<R>) {
    ((n == Ns ? (f(std::integral_constant<std::size_t, Ns>{}), hit = true) : false), ...);
    if (!hit) throw Error(LM_ERR_ARG, "reifyDim: size not among the candidates");
  } else {
    R out{};
    ((n == Ns ? (out = f(std::integral_constant<std::size_t, Ns>{}), hit = true) : false), ...);
    if (!hit) throw Error(LM_ERR_ARG, "reifyDim: size not among the candidates");
    return out;
  }
}
// Recover a typed Matrix<N, N> from a SomeMatrix whose size is one of Ns.
template <std::size_t N>
Matrix<N, N> unsafeTyped(const SomeMatrix& a) {
  if (a.rows() != N || a.cols() != N) throw Error(LM_ERR_ARG, "typed: dimension mismatch");
  return Matrix<N, N>::fromHost(a.toHost());
}

// Operations on runtime-size values (the reference's functions applied inside
// a SomeMatrix pattern match).
inline SomeVector luSolve(const SomeMatrix& a, const SomeVector& b, int* info_out = nullptr) {
  if (a.rows() != a.cols() || b.size() != a.rows()) throw Error(LM_ERR_ARG, "luSolve: dimension mismatch");
  const int n = (int)a.rows();
  std::vector<double> A = a.toHost(), B = b.toHost(), X(n);
  int info = 0;
  check(lm_lu_solve_host(context(), n, 1, A.data(), B.data(), X.data(), &info), "luSolve");
  if (info_out) *info_out = info;
  return someVector(X);
}
inline SomeVector choleskySolve(const SomeMatrix& a, const SomeVector& b, int* info_out = nullptr) {
  if (a.rows() != a.cols() || b.size() != a.rows()) throw Error(LM_ERR_ARG, "choleskySolve: dimension mismatch");
  const int n = (int)a.rows();
  std::vector<double> A = a.toHost(), B = b.toHost(), X(n);
  int info = 0;
  check(lm_chol_solve_host(context(), n, 1, A.data(), B.data(), X.data(), &info), "choleskySolve");
  if (info_out) *info_out = info;
  return someVector(X);
}
inline SomeMatrix matMul(const SomeMatrix& a, const SomeMatrix& b) {
  if (a.cols() != b.rows()) throw Error(LM_ERR_ARG, "matMul: dimension mismatch");
  SomeMatrix c(a.rows(), b.cols());
  check(lm_dgemm(context(), (int)a.rows(), (int)b.cols(), (int)a.cols(), 1.0, a.data(), (int)a.cols(), b.data(),
                 (int)b.cols(), 0.0, c.data(), (int)b.cols()),
        "matMul");
  return c;
}
inline SomeVector matvec(const SomeMatrix& a, const SomeVector& x) {
  if (a.cols() != x.size()) throw Error(LM_ERR_ARG, "matvec: dimension mismatch");
  SomeVector y(a.rows());
  check(lm_dgemv(context(), (int)a.rows(), (int)a.cols(), a.data(), (int)a.cols(), x.data(), y.data()), "matvec");
  return y;
}

// Earlier host-vector spellings of the runtime-size solves.
struct SomeMatrixHost {
  std::size_t rows = 0, cols = 0;
  std::vector<double> host;  // row-major
};
inline std::vector<double> luSolveSome(const SomeMatrixHost& a, const std::vector<double>& b) {
  return luSolve(someMatrix(a.rows, a.cols, a.host), someVector(b)).toHost();
}
inline std::vector<double> choleskySolveSome(const SomeMatrixHost& a, const std::vector<double>& b) {
  return choleskySolve(someMatrix(a.rows, a.cols, a.host), someVector(b)).toHost();
}

}  // namespace massiv
