"""CPU tests of the oracle: pinned against the reference's own known answers
and properties (test/Test/Solve.hs, test/Test/BLAS.hs), against exact rational
solutions, against the second (generic-path) restatement, and against its own
committed regression vectors."""
import numpy as np
import pytest

import oracle as O
from conftest import philox
from helpers import approx_eq, gen_randsvd, gen_uniform


# ---- known answers of the reference's test suite ----------------------------

def test_lu_known(golden_known):
    c = golden_known["test_luKnown"]
    A, b = np.array(c["A"], float), np.array(c["b"], float)
    for x in (O.lu_solve_p(A, b)[0], O.lu_solve_generic(A, b)):
        assert approx_eq(A @ x, b)               # luSolve roundtrip
        assert approx_eq(x, c["x"], 1e-14)        # exact solution


def test_matmul_known(golden_known):
    c = golden_known["test_matMulKnown"]
    A, B = np.array(c["A"], float), np.array(c["B"], float)
    assert np.array_equal(O.matmul_p(A, B), np.array(c["C"], float))
    assert np.array_equal(O.gemm_generic(1.0, A, B, 0.0, np.zeros((2, 2))), np.array(c["C"], float))


def test_gemm_larger(golden_known):
    c = golden_known["test_gemmLarger"]
    got = O.gemm_generic(c["alpha"], np.array(c["A"], float), np.array(c["B"], float), c["beta"],
                         np.array(c["C"], float))
    assert approx_eq(got, c["expected"])
    assert np.array_equal(got, np.array(c["expected"], float))


def test_lu_hilbert(golden_known):
    c = golden_known["test_luHilbert"]
    n = c["n"]
    H = np.array([[1.0 / (i + j + 1) for j in range(n)] for i in range(n)])
    x = np.array(c["x"], float)
    b = O.matvec_generic(H, x)
    for xs in (O.lu_solve_p(H, b)[0], O.lu_solve_generic(H, b)):
        assert O.scaled_residual_linear(H, xs, b) < c["residual_bound"]


def test_det_known(golden_known):
    c = golden_known["test_detEqualsEigenProduct"]
    A = np.array(c["A"])
    d = O.det(A)
    assert abs(d - c["det"]) / (abs(d) + 1e-15) < c["rel_bound"]
    ev = np.linalg.eigvalsh(A)
    assert abs(d - np.prod(ev)) / (abs(d) + 1e-15) < 1e-4


@pytest.mark.parametrize("n", [10, 50, 100])
def test_bench_comparison_matrices(golden_known, n):
    """The reference's benchmark inputs (bench-comparison/Main.hs:43-65) against exact solutions."""
    sol = golden_known["bench_comparison"]["solutions"][str(n)]
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    dd = (i * 7 + j * 3 + 1) / 100.0 + n * (i == j)
    vec = (np.arange(n) + 1) / 10.0
    Bm = (i * n + j + 1) / float(n * n)
    spd = np.eye(n) + Bm @ Bm.T
    assert np.abs(O.lu_solve_p(dd, vec)[0] - sol["lu_x"]).max() < 1e-12
    assert np.abs(O.chol_solve_p(spd, vec)[0] - sol["chol_x"]).max() < 1e-9 * np.abs(sol["chol_x"]).max()


# ---- committed regression vectors (bit-exact) --------------------------------

@pytest.mark.parametrize("n", [3, 10, 63, 64, 65, 100])
def test_regression_lu_chol(golden_regression, n):
    R = golden_regression
    x, LU, ipiv = O.lu_solve_p(R[f"lu{n}_A"], R[f"lu{n}_b"])
    assert np.array_equal(x, R[f"lu{n}_x"])
    assert np.array_equal(ipiv, R[f"lu{n}_ipiv"])
    if f"lu{n}_LU" in R:
        assert np.array_equal(LU, R[f"lu{n}_LU"])
    xc, G = O.chol_solve_p(R[f"ch{n}_A"], R[f"lu{n}_b"])
    assert np.array_equal(xc, R[f"ch{n}_x"])
    if f"ch{n}_G" in R:
        assert np.array_equal(np.tril(G), R[f"ch{n}_G"])


@pytest.mark.parametrize("key", ["mm7x5x3", "mm65x33x70", "mm100x100x101"])
def test_regression_matmul(golden_regression, key):
    R = golden_regression
    assert np.array_equal(O.matmul_p(R[key + "_A"], R[key + "_B"]), R[key + "_C"])


# ---- the reference's properties, on the oracle --------------------------------

@pytest.mark.parametrize("n,seed", [(3, s) for s in range(20)] + [(5, s) for s in range(10)])
def test_lu_reconstruction(n, seed):
    A = gen_uniform(philox(seed), n, -10, 10)        # genMatrix, test/Test/Types.hs:68-73
    LU, perm = O.lu_generic(A)
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    assert approx_eq(A[perm], O.matmul_p(L, U))       # prop_luReconstruction


@pytest.mark.parametrize("seed", range(20))
def test_lu_residual_bound_3(seed):
    g = philox(100 + seed)
    A, b = gen_uniform(g, 3, -10, 10), g.uniform(-10, 10, 3)
    LU, _ = O.lu_generic(A)
    if np.all(np.abs(np.diag(LU)) > 1e-6):
        assert O.scaled_residual_linear(A, O.lu_solve_generic(A, b), b) < 1e-6
        assert O.scaled_residual_linear(A, O.lu_solve_p(A, b)[0], b) < 1e-6


@pytest.mark.parametrize("seed", range(10))
def test_lu_solve_10(seed):
    g = philox(200 + seed)
    A, b = gen_uniform(g, 10, -10, 10), g.uniform(-10, 10, 10)
    assert O.scaled_residual_linear(A, O.lu_solve_p(A, b)[0], b) < 1e-6


@pytest.mark.parametrize("n,seed", [(3, s) for s in range(10)] + [(5, s) for s in range(10)])
def test_cholesky_reconstruction(n, seed):
    Bm = philox(300 + seed).uniform(-5, 5, (n, n))    # genSPDMatrix, test/Test/Types.hs:83-93
    A = Bm @ Bm.T + 0.1 * np.eye(n)
    G = O.cholesky_generic(A)
    assert approx_eq(A, G @ G.T)
    b = philox(400 + seed).uniform(-10, 10, n)
    assert O.scaled_residual_linear(A, O.chol_solve_p(A, b)[0], b) < 1e-6
    assert O.scaled_residual_linear(A, O.chol_solve_generic(A, b), b) < 1e-6


@pytest.mark.parametrize("seed", range(10))
def test_randsvd(seed):
    g = philox(500 + seed)
    A, b = gen_randsvd(g, 5, 100.0), g.uniform(-10, 10, 5)   # prop_luSolveRandsvd
    assert O.scaled_residual_linear(A, O.lu_solve_p(A, b)[0], b) < 0.01
    Q, _ = np.linalg.qr(g.uniform(-10, 10, (5, 5)))           # genSPDMatrixWithCond
    S = (Q * (1e4 ** (-np.arange(5) / 4))) @ Q.T
    S = 0.5 * (S + S.T)
    assert O.scaled_residual_cholesky(S, O.cholesky_generic(S)) < 1000


# ---- P path against the independent generic restatement -----------------------

@pytest.mark.parametrize("n", [10, 63, 64, 65, 97, 130, 300])
def test_p_vs_generic(n):
    g = philox(600 + n)
    A, b = gen_uniform(g, n), g.uniform(-1, 1, n)
    x, LU, ipiv = O.lu_solve_p(A, b)
    LUg, perm = O.lu_generic(A)
    assert np.array_equal(O.ipiv_to_perm(ipiv), perm)           # identical pivots
    assert np.abs(x - O.lu_solve_generic(A, b)).max() / np.abs(x).max() < 1e-11
    assert np.abs(LU - LUg).max() < 1e-10 * max(1.0, np.abs(LUg).max())
    S = A @ A.T + n * np.eye(n)
    xc, G = O.chol_solve_p(S, b)
    assert np.abs(np.tril(G) - O.cholesky_generic(S)).max() < 1e-12 * np.abs(G).max()
    assert np.abs(xc - O.chol_solve_generic(S, b)).max() < 1e-12 * np.abs(xc).max()


@pytest.mark.parametrize("shape", [(200, 200, 203), (256, 96, 130), (17, 300, 9)])
def test_matmul_par_and_numpy(shape):
    m, k, n = shape
    g = philox(700 + m)
    A, B = g.uniform(-1, 1, (m, k)), g.uniform(-1, 1, (k, n))
    C = O.matmul_p(A, B)
    assert np.abs(C - A @ B).max() < 4 * k * 2.2e-16 * (np.abs(A) @ np.abs(B)).max()
    Cp = O.matmul_par(A, B, 8)
    assert np.abs(Cp - C).max() <= 4 * k * 2.2e-16 * (np.abs(A) @ np.abs(B)).max()


def test_pivot_tie_first_wins():
    # rawPivotSearch keeps the first maximum (strict '>'), lu keeps the last.
    A = np.array([[1.0, 2.0], [-1.0, 3.0]])
    _, _, ipiv = O.lu_solve_p(A, np.ones(2))
    assert ipiv[0] == 0
    _, perm = O.lu_generic(A)
    assert list(perm) == [1, 0]


# ---- adjacent solvers: known answers and independent checks ---------------------

def test_tridiag_known_answer():
    # test_tridiagKnown (test/Test/Solve.hs:138-150): x = [1, 1, 1] for
    # A = tridiag(-1, 2, -1), b = [1, 0, 1], with the suite's (~=) tolerance
    x = O.tridiag_solve(np.full(3, 2.0), np.array([-1.0, -1.0, 0.0]), np.array([1.0, 0.0, 1.0]))
    assert np.all(np.abs(x - 1.0) < 1e-8 * (2 + np.abs(x)))


@pytest.mark.parametrize("n", [1, 2, 9, 200])
def test_tridiag_vs_dense_solve(n):
    g = philox(800 + n)
    sup = g.uniform(-1, 1, n)
    d = 2.5 + g.uniform(0, 1, n)
    b = g.uniform(-1, 1, n)
    T = np.diag(d) + np.diag(sup[:n - 1], 1) + np.diag(sup[:n - 1], -1)
    assert np.abs(O.tridiag_solve(d, sup, b) - np.linalg.solve(T, b)).max() < 1e-13


@pytest.mark.parametrize("n", [1, 2, 5, 70])
def test_lu_nopivot_reconstructs(n):
    g = philox(900 + n)
    A = g.uniform(-1, 1, (n, n)) + n * np.eye(n)
    LU = O.lu_nopivot(A)
    L, U = np.tril(LU, -1) + np.eye(n), np.triu(LU)
    assert O.scaled_residual_lu(A, LU, np.arange(n)) < 10
    # without pivoting on a diagonally dominant matrix, GEPP picks the diagonal
    # too, so the P path gives the same factor up to rounding
    _, LUp, ipiv = O.lu_solve_p(A, np.ones(n))
    assert np.array_equal(ipiv, np.arange(n))
    assert np.abs(LU - LUp).max() < 1e-12 * np.abs(LU).max()
    assert np.abs(L @ U - A).max() < 1e-12 * np.abs(A).max()


@pytest.mark.parametrize("n", [1, 3, 40])
def test_cholesky_gaxpy_matches_cholesky(n):
    g = philox(1000 + n)
    B = g.uniform(-1, 1, (n, n))
    S = B @ B.T + n * np.eye(n)
    G = O.cholesky_gaxpy(S)
    assert np.all(np.triu(G, 1) == 0.0)
    assert np.abs(G - O.cholesky_generic(S)).max() < 1e-13 * np.abs(G).max()


def test_norm_inf_matches_numpy():
    g = philox(1100)
    A = g.uniform(-3, 3, (37, 53))
    assert abs(O.norm_inf(A) - np.abs(A).sum(axis=1).max()) < 1e-13 * O.norm_inf(A)
    assert O.norm_inf(np.array([[1.0, -2.0, 3.0], [-4.0, 5.0, -6.0]])) == 15.0
