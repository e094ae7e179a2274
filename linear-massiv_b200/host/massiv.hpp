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
// File references: Types.hs, Internal.hs (src/Numeric/LinearAlgebra/Massiv/),
// L3.hs = BLAS/Level3.hs, LU.hs = Solve/LU.hs, Chol.hs = Solve/Cholesky.hs.
#pragma once

#include <lm_b200.h>

#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>
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

// ---- runtime sizes: SomeMatrix (Types.hs:165-178) ----------------------------
// A matrix whose dimensions are known only at run time (serving).
struct SomeMatrix {
  std::size_t rows = 0, cols = 0;
  std::vector<double> host;  // row-major
};

inline std::vector<double> luSolveSome(const SomeMatrix& a, const std::vector<double>& b) {
  if (a.rows != a.cols || b.size() != a.rows) throw Error(LM_ERR_ARG, "luSolveSome: dimension mismatch");
  std::vector<double> x(a.rows);
  int info = 0;
  check(lm_lu_solve_host(context(), (int)a.rows, 1, a.host.data(), b.data(), x.data(), &info), "luSolveSome");
  return x;
}

inline std::vector<double> choleskySolveSome(const SomeMatrix& a, const std::vector<double>& b) {
  if (a.rows != a.cols || b.size() != a.rows) throw Error(LM_ERR_ARG, "choleskySolveSome: dimension mismatch");
  std::vector<double> x(a.rows);
  int info = 0;
  check(lm_chol_solve_host(context(), (int)a.rows, 1, a.host.data(), b.data(), x.data(), &info),
        "choleskySolveSome");
  return x;
}

}  // namespace massiv
