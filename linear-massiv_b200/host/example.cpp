// Known-answer checks of the C++ mirror of the reference API, the same cases
// as linear-massiv's test/Test/Solve.hs and test/Test/BLAS.hs.  Exit status 0
// when every check passes.
#include <cmath>
#include <cstdio>

#include "massiv.hpp"

using namespace massiv;

static int failures = 0;
static bool approx(double x, double y) { return std::fabs(x - y) < 1e-8 * (1 + std::fabs(x) + std::fabs(y)); }
static void expect(bool ok, const char* what) {
  std::printf("%s %s\n", ok ? "ok  " : "FAIL", what);
  if (!ok) ++failures;
}

int main() {
  // test_luKnown (test/Test/Solve.hs:107-119)
  auto a = Matrix<3, 3>::fromHost({2, 1, 1, 4, 3, 3, 8, 7, 9});
  auto b = Vector<3>::fromHost({1, 1, 1});
  auto x = luSolve(a, b).toHost();
  expect(approx(x[0], 1) && approx(x[1], -1) && approx(x[2], 0), "luSolve 3x3 known");
  auto xd = luSolveDevice(a, b).toHost();
  expect(approx(xd[0], 1) && approx(xd[1], -1) && approx(xd[2], 0), "luSolve 3x3 known (device resident)");
  // test_matMulKnown (test/Test/BLAS.hs:132-144)
  auto c = matMul(Matrix<2, 2>::fromHost({1, 2, 3, 4}), Matrix<2, 2>::fromHost({5, 6, 7, 8})).toHost();
  expect(c[0] == 19 && c[1] == 22 && c[2] == 43 && c[3] == 50, "matMul 2x2 known");
  // test_gemmLarger (test/Test/BLAS.hs:156-172)
  auto A3 = Matrix<3, 3>::make([](std::size_t i, std::size_t j) { return double(i * 3 + j + 1); });
  auto B3 = Matrix<3, 3>::make([](std::size_t i, std::size_t j) { return double(9 - (i * 3 + j)); });
  auto I3 = Matrix<3, 3>::make([](std::size_t i, std::size_t j) { return i == j ? 1.0 : 0.0; });
  auto g = gemm(2.0, A3, B3, 0.5, I3).toHost();
  const double want[9] = {60.5, 48, 36, 168, 138.5, 108, 276, 228, 180.5};
  bool ok = true;
  for (int i = 0; i < 9; ++i) ok = ok && approx(g[i], want[i]);
  expect(ok, "gemm alpha=2 beta=0.5 3x3 known");
  // test_luHilbert (test/Test/Solve.hs:157-166): scaled residual < 1e-4
  auto H = Matrix<5, 5>::make([](std::size_t i, std::size_t j) { return 1.0 / double(i + j + 1); });
  std::vector<double> hx = {1, 2, 3, 4, 5}, hb(5, 0.0), hh = H.toHost();
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) hb[i] += hh[i * 5 + j] * hx[j];
  auto xs = luSolve(H, Vector<5>::fromHost(hb)).toHost();
  double rmax = 0, an = 0, xn = 0, bn = 0;
  for (int i = 0; i < 5; ++i) {
    double r = -hb[i], rs = 0;
    for (int j = 0; j < 5; ++j) { r += hh[i * 5 + j] * xs[j]; rs += std::fabs(hh[i * 5 + j]); }
    rmax = std::fmax(rmax, std::fabs(r)); an = std::fmax(an, rs);
    xn = std::fmax(xn, std::fabs(xs[i])); bn = std::fmax(bn, std::fabs(hb[i]));
  }
  expect(rmax / (an * xn + bn + 5 * 2.220446049250313e-16) < 1e-4, "luSolve Hilbert 5 residual");
  // cholesky / choleskySolve round trip on an SPD matrix
  auto S = Matrix<4, 4>::make([](std::size_t i, std::size_t j) {
    return (i == j ? double(4 - i) : 0.0) + 0.1;
  });
  auto G = cholesky(S).toHost();
  auto Sh = S.toHost();
  ok = true;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += G[i * 4 + k] * G[j * 4 + k];
      ok = ok && approx(s, Sh[i * 4 + j]) && (j <= i || G[i * 4 + j] == 0.0);
    }
  expect(ok, "cholesky G G^T = A, zeros above");
  auto xc = choleskySolve(S, Vector<4>::fromHost({1, 2, 3, 4})).toHost();
  ok = true;
  for (int i = 0; i < 4; ++i) {
    double s = 0;
    for (int j = 0; j < 4; ++j) s += Sh[i * 4 + j] * xc[j];
    ok = ok && approx(s, i + 1.0);
  }
  expect(ok, "choleskySolve round trip");
  // det (test/Test/Solve.hs:228-238): diag(4,3,2,1) + 0.1
  double d = det(S);
  expect(std::fabs(d - 29.0) / 29.0 < 1e-12, "det diag(4,3,2,1)+0.1 = 29");
  // runtime-size entry (SomeMatrix)
  SomeMatrix sm{3, 3, {2, 1, 1, 4, 3, 3, 8, 7, 9}};
  auto xr = luSolveSome(sm, {1, 1, 1});
  expect(approx(xr[0], 1) && approx(xr[1], -1) && approx(xr[2], 0), "luSolveSome runtime size");
  std::printf("%d failure(s)\n", failures);
  return failures ? 1 : 0;
}
