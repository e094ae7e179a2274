// Known-answer checks of the C++ mirror of the reference API, the same cases
// as linear-massiv's test/Test/Solve.hs and test/Test/BLAS.hs.  Exit status 0
// when every check passes.
#include <cmath>
#include <cstdio>
#include <string>

#include "massiv.hpp"

using namespace massiv;

static int failures = 0;
static bool approx(double x, double y) { return std::fabs(x - y) < 1e-8 * (1 + std::fabs(x) + std::fabs(y)); }
static void expect(bool ok, const char* what) {
  std::printf("%s %s\n", ok ? "ok  " : "FAIL", what);
  if (!ok) ++failures;
}

static int solve_file(const char* in, const char* out);

int main(int argc, char** argv) {
  if (argc == 4 && std::string(argv[1]) == "solve") return solve_file(argv[2], argv[3]);
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
  SomeMatrixHost sm{3, 3, {2, 1, 1, 4, 3, 3, 8, 7, 9}};
  auto xr = luSolveSome(sm, {1, 1, 1});
  expect(approx(xr[0], 1) && approx(xr[1], -1) && approx(xr[2], 0), "luSolveSome runtime size");
  auto xs2 = luSolve(forget(a), someVector({1, 1, 1})).toHost();
  expect(approx(xs2[0], 1) && approx(xs2[1], -1) && approx(xs2[2], 0), "luSolve on forget(Matrix<3,3>)");
  // matvec with the identity (test/Test/BLAS.hs:71-74)
  auto mv = matvec(I3, Vector<3>::fromHost({1.5, -2, 7})).toHost();
  expect(mv[0] == 1.5 && mv[1] == -2 && mv[2] == 7, "matvec identity");
  // normInf / vnormInf
  expect(normInf(Matrix<2, 3>::fromHost({1, -2, 3, -4, 5, -6})) == 15.0, "normInf 2x3 = 15");
  expect(vnormInf(Vector<3>::fromHost({1, -9, 3})) == 9.0, "vnormInf = 9");
  // luNoPivot on test_luKnown's matrix reordered to need no pivoting: L U = A
  auto A4 = Matrix<3, 3>::fromHost({8, 7, 9, 4, 3, 3, 2, 1, 1});
  auto lun = luNoPivot(A4).toHost();
  auto a4 = A4.toHost();
  ok = true;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k <= std::min(i, j); ++k) s += (k == i ? 1.0 : lun[i * 3 + k]) * lun[k * 3 + j];
      ok = ok && approx(s, a4[i * 3 + j]);
    }
  expect(ok, "luNoPivot L U = A");
  auto Gg = choleskyGaxpy(S).toHost();
  ok = true;
  for (int i = 0; i < 16; ++i) ok = ok && approx(Gg[i], G[i]);
  expect(ok, "choleskyGaxpy = cholesky");
  // test_tridiagKnown (test/Test/Solve.hs:138-150)
  auto xt = tridiagSolve(Vector<3>::fromHost({2, 2, 2}), Vector<3>::fromHost({-1, -1, 0}),
                         Vector<3>::fromHost({1, 0, 1})).toHost();
  expect(approx(xt[0], 1) && approx(xt[1], 1) && approx(xt[2], 1), "tridiagSolve known");
  std::printf("%d failure(s)\n", failures);
  return failures ? 1 : 0;
}

// Runtime-size solve of a system read from a file (int32 kind, int32 n, then
// A as n*n and b as n doubles; kind 0 = LU, 1 = Cholesky), written as n
// doubles.  Sizes among the reify candidates go through the typed API after
// reifyDim, the others through the SomeMatrix operations.
static int solve_file(const char* in, const char* out) {
  std::FILE* f = std::fopen(in, "rb");
  if (!f) return 2;
  int hdr[2];
  if (std::fread(hdr, sizeof(int), 2, f) != 2) return 2;
  const std::size_t n = (std::size_t)hdr[1];
  std::vector<double> A(n * n), b(n);
  if (std::fread(A.data(), sizeof(double), n * n, f) != n * n || std::fread(b.data(), sizeof(double), n, f) != n)
    return 2;
  std::fclose(f);
  SomeMatrix sa = someMatrix(n, n, A);
  SomeVector sb = someVector(b);
  std::vector<double> x;
  bool typed = false;
  try {
    x = reifyDim<3, 64, 300>(n, [&](auto N) {
      constexpr std::size_t K = decltype(N)::value;
      auto ta = unsafeTyped<K>(sa);
      auto tb = Vector<K>::fromHost(b);
      return hdr[0] == 0 ? luSolve(ta, tb).toHost() : choleskySolve(ta, tb).toHost();
    });
    typed = true;
  } catch (const Error&) {
    x = (hdr[0] == 0 ? luSolve(sa, sb) : choleskySolve(sa, sb)).toHost();
  }
  std::FILE* g = std::fopen(out, "wb");
  if (!g) return 2;
  std::fwrite(x.data(), sizeof(double), n, g);
  std::fclose(g);
  std::printf("solved n=%zu kind=%d via %s\n", n, hdr[0], typed ? "reifyDim + typed API" : "SomeMatrix");
  return 0;
}
