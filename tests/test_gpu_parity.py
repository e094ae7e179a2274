"""GPU parity of the CUDA path against the CPU oracle (restated reference).

Bars (stated per test):
  * GEMM: elementwise |C - C_oracle| <= 2 k eps (|A||B|)_ij + tiny, the FP64
    bound for two different summation orders.
  * LU: identical pivot sequence (inputs with distinct pivot magnitudes),
    relative forward error vs the oracle <= max(1e-12, 32 kappa eps), normwise
    backward error <= 1e-15 n.
  * Cholesky: G close to the oracle's G, same forward/backward bars.
"""
import numpy as np
import pytest
import torch

import lmb200
import oracle as O
from conftest import philox
from helpers import approx_eq, backward_error, gen_spd, gen_uniform, rel_forward

pytestmark = pytest.mark.gpu
EPS = 2.220446049250313e-16


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def gemm_bound(A, B, k):
    return 2 * max(k, 1) * EPS * (np.abs(A) @ np.abs(B)) + 1e-300


# ---- GEMM ------------------------------------------------------------------------

@pytest.mark.parametrize("m,k,n", [(1, 1, 1), (3, 3, 3), (7, 5, 3), (65, 33, 70), (100, 100, 101),
                                   (128, 128, 128), (129, 17, 257), (257, 129, 300), (300, 1, 64),
                                   (64, 1000, 33), (1000, 1000, 1000)])
def test_gemm_vs_oracle(ctx, m, k, n):
    g = philox(m * 7 + k * 3 + n)
    A, B = g.uniform(-1, 1, (m, k)), g.uniform(-1, 1, (k, n))
    C = host(lmb200.matMul(dev(A), dev(B), ctx))
    ref = O.matmul_p(A, B)
    assert np.all(np.abs(C - ref) <= gemm_bound(A, B, k))


@pytest.mark.parametrize("alpha,beta", [(2.0, 0.5), (-1.0, 1.0), (0.0, 3.0), (1.5, 0.0)])
def test_gemm_alpha_beta(ctx, alpha, beta):
    g = philox(11)
    m, k, n = 190, 77, 130
    A, B, C0 = g.uniform(-1, 1, (m, k)), g.uniform(-1, 1, (k, n)), g.uniform(-1, 1, (m, n))
    C = host(lmb200.gemm(alpha, dev(A), dev(B), beta, dev(C0), ctx))
    ref = O.gemm_generic(alpha, A, B, beta, C0)
    assert np.all(np.abs(C - ref) <= abs(alpha) * gemm_bound(A, B, k) + 4 * EPS * np.abs(beta * C0))


@pytest.mark.parametrize("m,k,n", [(2100, 200, 2050), (1500, 128, 3000), (700, 16, 900)])
def test_gemm_short_k_update_many_tiles(ctx, m, k, n):
    # the trailing-update shape (k <= 256, beta != 0) with several output
    # tiles per persistent CTA and ragged edges
    g = philox(m + 3 * k + 5 * n)
    A, B, C0 = g.uniform(-1, 1, (m, k)), g.uniform(-1, 1, (k, n)), g.uniform(-1, 1, (m, n))
    C = host(lmb200.gemm(-1.0, dev(A), dev(B), 1.0, dev(C0), ctx))
    ref = C0 - A @ B
    assert np.all(np.abs(C - ref) <= gemm_bound(A, B, k) + 4 * EPS * np.abs(C0))


def test_gemm_known_answers(ctx, golden_known):
    c = golden_known["test_gemmLarger"]
    got = host(lmb200.gemm(c["alpha"], dev(np.array(c["A"], float)), dev(np.array(c["B"], float)), c["beta"],
                           dev(np.array(c["C"], float)), ctx))
    assert np.array_equal(got, np.array(c["expected"], float))
    c = golden_known["test_matMulKnown"]
    got = host(lmb200.matMul(dev(np.array(c["A"], float)), dev(np.array(c["B"], float)), ctx))
    assert np.array_equal(got, np.array(c["C"], float))


def test_gemm_strided_and_odd_ld(ctx):
    g = philox(12)
    big = g.uniform(-1, 1, (300, 301))          # odd leading dimension -> staging path
    A = dev(big)[:200, :151]
    B = dev(g.uniform(-1, 1, (151, 99)))
    C = torch.zeros((200, 99), dtype=torch.float64, device="cuda")
    lmb200.dgemm(1.0, A, B, 0.0, C, ctx)
    ref = O.matmul_p(big[:200, :151], host(B))
    assert np.all(np.abs(host(C) - ref) <= gemm_bound(big[:200, :151], host(B), 151))


def test_gemm_host_entry(ctx):
    g = philox(13)
    A, B, C0 = g.uniform(-1, 1, (33, 45)), g.uniform(-1, 1, (45, 21)), g.uniform(-1, 1, (33, 21))
    C = lmb200.gemm_host(0.5, A, B, -2.0, C0, ctx)
    ref = O.gemm_generic(0.5, A, B, -2.0, C0)
    assert np.all(np.abs(C - ref) <= gemm_bound(A, B, 45) + 8 * EPS * np.abs(C0))


# ---- LU ----------------------------------------------------------------------------

LU_SIZES = [1, 2, 3, 4, 10, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129, 200, 255, 256, 257, 500, 777, 1024]


@pytest.mark.parametrize("n", LU_SIZES)
def test_lu_vs_oracle(ctx, n):
    g = philox(5000 + n)
    A, b = gen_uniform(g, n), g.uniform(-1, 1, n)
    LUd, ipiv, info = lmb200.lu_factor(dev(A), ctx)
    x = host(lmb200.luSolve(dev(A), dev(b), ctx))
    xo, LUo, ipo = O.lu_solve_p(A, b)
    assert info == 0
    assert np.array_equal(host(ipiv), ipo), "pivot sequence differs from the oracle"
    kappa = np.linalg.cond(A) if n > 1 else 1.0
    assert rel_forward(x, xo) <= max(1e-12, 32 * kappa * EPS)
    assert backward_error(A, x, b) <= 1e-15 * max(n, 1)
    LU = host(LUd)
    assert np.abs(LU - LUo).max() <= max(1e-12, 64 * kappa * EPS) * max(1.0, np.abs(LUo).max())


@pytest.mark.parametrize("n", [2048, 4096])
def test_lu_large_vs_oracle(ctx, n):
    g = philox(6000 + n)
    A, b = gen_uniform(g, n), g.uniform(-1, 1, n)
    _, ipiv, info = lmb200.lu_factor(dev(A), ctx)
    x = host(lmb200.luSolve(dev(A), dev(b), ctx))
    xo, _, ipo = O.lu_solve_p(A, b)
    assert info == 0
    agree = float(np.mean(host(ipiv) == ipo))
    assert agree == 1.0, f"pivot agreement {agree}"
    assert backward_error(A, x, b) <= 1e-15 * n
    assert rel_forward(x, xo) <= max(1e-12, 32 * np.linalg.cond(A) * EPS)


@pytest.mark.parametrize("n,nrhs", [(100, 64), (300, 7), (513, 64)])
def test_lu_multi_rhs(ctx, n, nrhs):
    g = philox(7000 + n)
    A, B = gen_uniform(g, n), g.uniform(-1, 1, (n, nrhs))
    X = host(lmb200.luSolve(dev(A), dev(B), ctx))
    Xo, _, _ = O.lu_solve_p(A, B)
    kappa = np.linalg.cond(A)
    for c in range(nrhs):
        assert backward_error(A, X[:, c], B[:, c]) <= 1e-15 * n
        assert rel_forward(X[:, c], Xo[:, c]) <= max(1e-12, 32 * kappa * EPS)


def test_lu_known_and_hilbert(ctx, golden_known):
    c = golden_known["test_luKnown"]
    A, b = np.array(c["A"], float), np.array(c["b"], float)
    x = host(lmb200.luSolve(dev(A), dev(b), ctx))
    assert approx_eq(A @ x, b) and approx_eq(x, c["x"], 1e-14)
    h = golden_known["test_luHilbert"]
    n = h["n"]
    H = np.array([[1.0 / (i + j + 1) for j in range(n)] for i in range(n)])
    bh = O.matvec_generic(H, np.array(h["x"], float))
    xh = host(lmb200.luSolve(dev(H), dev(bh), ctx))
    assert O.scaled_residual_linear(H, xh, bh) < h["residual_bound"]


def test_lu_pivot_ties_pick_lowest_row(ctx):
    # |a| ties in the first column: the reference's strict '>' keeps the first.
    A = np.array([[1.0, 2.0, 0.5], [-1.0, 3.0, 1.0], [1.0, -1.0, 2.0]])
    _, ipiv, _ = lmb200.lu_factor(dev(A), ctx)
    _, _, ipo = O.lu_solve_p(A, np.ones(3))
    assert np.array_equal(host(ipiv), ipo)
    assert host(ipiv)[0] == 0


def test_lu_nan_pivot_rule(ctx):
    # NaN at the diagonal stays the pivot; NaN below never wins (K.hs:1541-1556).
    A = np.array([[np.nan, 1.0], [2.0, 3.0]])
    _, ipiv, _ = lmb200.lu_factor(dev(A), ctx)
    assert host(ipiv)[0] == 0
    B = np.array([[1.0, 1.0, 1.0], [np.nan, 2.0, 0.0], [3.0, 0.0, 1.0]])
    _, ipiv, _ = lmb200.lu_factor(dev(B), ctx)
    _, _, ipo = O.lu_solve_p(B, np.ones(3))
    assert host(ipiv)[0] == ipo[0] == 2


def test_lu_singular_reports_info(ctx):
    A = np.array([[1.0, 2.0, 3.0], [2.0, 4.0, 6.0], [1.0, 1.0, 1.0]])
    A[:, 1] = 0.0  # zero column -> zero pivot at step 1
    _, _, info = lmb200.lu_factor(dev(A), ctx)
    assert info == 2


def test_lu_odd_lda_and_host_entries(ctx):
    g = philox(14)
    n = 157
    A, b = gen_uniform(g, n), g.uniform(-1, 1, n)
    x, info = lmb200.lu_solve_host(A, b, ctx)
    xo, LUo, ipo = O.lu_solve_p(A, b)
    assert info == 0 and rel_forward(x, xo) <= max(1e-12, 32 * np.linalg.cond(A) * EPS)
    LU, perm, info = lmb200.lu_host(A, ctx)
    LUg, permg = O.lu_generic(A)
    assert np.array_equal(perm, permg)
    assert np.abs(LU - LUo).max() < 1e-10
    # odd leading dimension on the device path
    big = dev(np.pad(A, ((0, 0), (0, 2))))[:, :n + 1]
    sub = big[:, :n]
    ipiv = torch.empty(n, dtype=torch.int32, device="cuda")
    assert lmb200.dgetrf(sub, ipiv, ctx) == 0
    assert np.array_equal(host(ipiv), ipo)
    assert np.abs(host(sub) - LUo).max() < 1e-10


def test_det(ctx, golden_known):
    c = golden_known["test_detEqualsEigenProduct"]
    d = lmb200.det(dev(np.array(c["A"])), ctx)
    assert abs(d - c["det"]) / abs(c["det"]) < 1e-12


# ---- Cholesky --------------------------------------------------------------------------

@pytest.mark.parametrize("n", [1, 2, 3, 10, 63, 64, 65, 127, 128, 129, 300, 513, 1024])
def test_cholesky_vs_oracle(ctx, n):
    g = philox(8000 + n)
    A, b = gen_spd(g, n), g.uniform(-1, 1, n)
    G = host(lmb200.cholesky(dev(A), ctx))
    x = host(lmb200.choleskySolve(dev(A), dev(b), ctx))
    xo, Go = O.chol_solve_p(A, b)
    assert np.all(np.triu(G, 1) == 0.0)
    assert np.abs(G - np.tril(Go)).max() <= 1e-13 * np.abs(Go).max()
    assert rel_forward(x, xo) <= 1e-12
    assert backward_error(A, x, b) <= 1e-15 * n


@pytest.mark.parametrize("n,nrhs", [(200, 64), (257, 3)])
def test_cholesky_multi_rhs(ctx, n, nrhs):
    g = philox(8100 + n)
    A, B = gen_spd(g, n), g.uniform(-1, 1, (n, nrhs))
    X = host(lmb200.choleskySolve(dev(A), dev(B), ctx))
    Xo, _ = O.chol_solve_p(A, B)
    assert rel_forward(X, Xo) <= 1e-12


def test_cholesky_not_spd_reports_info(ctx):
    A = np.eye(5)
    A[3, 3] = -1.0
    G = dev(A)
    assert lmb200.dpotrf(G, ctx) == 4


def test_cholesky_host_entries(ctx):
    g = philox(15)
    n = 91
    A, b = gen_spd(g, n), g.uniform(-1, 1, n)
    x, info = lmb200.chol_solve_host(A, b, ctx)
    G, info2 = lmb200.cholesky_host(A, ctx)
    assert info == 0 and info2 == 0
    assert rel_forward(x, O.chol_solve_generic(A, b)) < 1e-12
    assert np.abs(G - O.cholesky_generic(A)).max() < 1e-13 * np.abs(G).max()


def test_bench_comparison_matrices(ctx, golden_known):
    """The reference's own benchmark inputs (bench-comparison/Main.hs:43-65)."""
    for n in (10, 50, 100):
        sol = golden_known["bench_comparison"]["solutions"][str(n)]
        i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        dd = (i * 7 + j * 3 + 1) / 100.0 + n * (i == j)
        vec = (np.arange(n) + 1) / 10.0
        Bm = (i * n + j + 1) / float(n * n)
        spd = np.eye(n) + Bm @ Bm.T
        assert np.abs(host(lmb200.luSolve(dev(dd), dev(vec), ctx)) - sol["lu_x"]).max() < 1e-12
        xc = host(lmb200.choleskySolve(dev(spd), dev(vec), ctx))
        assert np.abs(xc - sol["chol_x"]).max() < 1e-9 * np.abs(sol["chol_x"]).max()


# ---- residual ----------------------------------------------------------------------------

@pytest.mark.parametrize("nrhs", [1, 5, 16])
def test_residual(ctx, nrhs):
    g = philox(16 + nrhs)
    n = 300
    A, X, B = g.uniform(-1, 1, (n, n)), g.uniform(-1, 1, (n, nrhs)), g.uniform(-1, 1, (n, nrhs))
    R = torch.empty((n, nrhs), dtype=torch.float64, device="cuda")
    lmb200.dresidual(dev(A), dev(X), dev(B), R, ctx)
    ref = B - A @ X
    assert np.abs(host(R) - ref).max() <= 2 * n * EPS * (np.abs(A) @ np.abs(X)).max()
