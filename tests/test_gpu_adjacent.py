"""GPU parity of the adjacent entry points against the oracle: matvec
(bitwise: the device kernel keeps rawGemv's floating-point order), normInf
(bitwise: the same row folds), the residual of the refinement path, luNoPivot,
choleskyGaxpy and tridiagSolve.

Bars: matvec and normInf bit for bit; luNoPivot within 32 n eps max|LU| of
the oracle (the device association differs: blocked, DMMA GEMMs) and a
reconstruction L U = A within the reference's scaledResidualLU bound;
choleskyGaxpy within 1e-13 max|G|; tridiagSolve relative error <= 1e-13 on
diagonally dominant SPD systems (parallel cyclic reduction reorders the
arithmetic) and the reference's known answer to 1e-8 (test/Test/Solve.hs:138-150).
"""
import ctypes

import numpy as np
import pytest
import torch

import lmb200
import oracle as O
from conftest import philox
from helpers import approx_eq, gen_spd

pytestmark = pytest.mark.gpu
EPS = 2.220446049250313e-16


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


# ---- matvec ------------------------------------------------------------------

@pytest.mark.parametrize("m,n", [(1, 1), (1, 3), (3, 7), (5, 4), (100, 257), (1000, 1003), (4096, 4096),
                                 (16384, 16384)])
def test_matvec_bitwise_vs_oracle(ctx, m, n):
    g = philox(30000 + m + 7 * n)
    A, x = g.uniform(-1, 1, (m, n)), g.uniform(-1, 1, n)
    y = host(lmb200.matvec(dev(A), dev(x), ctx))
    assert np.array_equal(y, O.matvec_p(A, x))


def test_matvec_strided_and_host_entry(ctx):
    g = philox(30001)
    big = g.uniform(-1, 1, (300, 517))
    x = g.uniform(-1, 1, 511)
    y = host(lmb200.matvec(dev(big)[:, :511], dev(x), ctx))
    assert np.array_equal(y, O.matvec_p(big[:, :511], x))
    A = np.ascontiguousarray(big[:, :511])
    yh = np.empty(300)
    s = lmb200.lib().lm_matvec_host(ctx.h, 300, 511, lmb200._np_ptr(A), lmb200._np_ptr(x), lmb200._np_ptr(yh))
    assert s == 0 and np.array_equal(yh, O.matvec_p(A, x))


@pytest.mark.parametrize("nrhs", [1, 5, 16])
def test_residual_vs_oracle_matvec(ctx, nrhs):
    """r = b - A x of the refinement path against b - matvecP(A, x)."""
    g = philox(30100 + nrhs)
    n = 777
    A, X, B = g.uniform(-1, 1, (n, n)), g.uniform(-1, 1, (n, nrhs)), g.uniform(-1, 1, (n, nrhs))
    R = torch.empty((n, nrhs), dtype=torch.float64, device="cuda")
    lmb200.dresidual(dev(A), dev(X), dev(B), R, ctx)
    ref = np.stack([B[:, c] - O.matvec_p(A, X[:, c]) for c in range(nrhs)], axis=1)
    assert np.abs(host(R) - ref).max() <= 2 * n * EPS * (np.abs(A) @ np.abs(X)).max()


# ---- normInf ------------------------------------------------------------------

@pytest.mark.parametrize("m,n", [(1, 1), (2, 3), (33, 129), (1000, 1000), (4099, 301)])
def test_norm_inf_bitwise_vs_oracle(ctx, m, n):
    g = philox(31000 + m + n)
    A = g.uniform(-1, 1, (m, n)) * np.exp(g.uniform(-3, 3, (m, 1)))
    assert lmb200.normInf(dev(A), ctx) == O.norm_inf(A)
    x = g.uniform(-5, 5, m)
    assert lmb200.normInf(dev(x), ctx) == O.norm_inf(x) == np.abs(x).max()


def test_norm_inf_host_entry(ctx):
    A = np.array([[1.0, -2.0, 3.0], [-4.0, 5.0, -6.0]])
    out = np.zeros(1)
    s = lmb200.lib().lm_norm_inf_host(ctx.h, 2, 3, lmb200._np_ptr(A), lmb200._np_ptr(out))
    assert s == 0 and out[0] == 15.0 == O.norm_inf(A)


# ---- luNoPivot ------------------------------------------------------------------

def diag_dominant(g, n):
    return g.uniform(-1, 1, (n, n)) + n * np.eye(n)


@pytest.mark.parametrize("n", [1, 2, 3, 31, 64, 127, 128, 129, 300, 1000, 2049])
def test_lu_nopivot_vs_oracle(ctx, n):
    g = philox(32000 + n)
    A = diag_dominant(g, n)
    LU, info = lmb200.luNoPivot(dev(A), ctx)
    LU = host(LU)
    LUo = O.lu_nopivot(A)
    assert info == 0
    assert np.abs(LU - LUo).max() <= 32 * n * EPS * np.abs(LUo).max()
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    # scaledResidualLU (test/Test/Residuals.hs:167-189) with the identity permutation
    assert np.linalg.norm(A - L @ U) / (np.linalg.norm(A) * n * EPS + EPS) < 10.0


def test_lu_nopivot_zero_pivot_and_host_entry(ctx):
    A = np.array([[0.0, 1.0], [1.0, 1.0]])
    _, info = lmb200.luNoPivot(dev(A), ctx)
    assert info == 1
    g = philox(32100)
    B = diag_dominant(g, 65)
    LU = np.empty_like(B)
    inf = np.zeros(1, dtype=np.int32)
    s = lmb200.lib().lm_lu_nopivot_host(ctx.h, 65, lmb200._np_ptr(B), lmb200._np_ptr(LU),
                                        inf.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    assert s == 0 and inf[0] == 0
    assert np.abs(LU - O.lu_nopivot(B)).max() <= 32 * 65 * EPS * np.abs(LU).max()


# ---- choleskyGaxpy ------------------------------------------------------------------

@pytest.mark.parametrize("n", [1, 2, 17, 128, 129, 500])
def test_cholesky_gaxpy_vs_oracle(ctx, n):
    g = philox(33000 + n)
    A = gen_spd(g, n)
    G = host(lmb200.choleskyGaxpy(dev(A), ctx))
    Go = O.cholesky_gaxpy(A)
    assert np.all(np.triu(G, 1) == 0.0)
    assert np.abs(G - Go).max() <= 1e-13 * np.abs(Go).max()
    Gh = np.empty_like(A)
    inf = np.zeros(1, dtype=np.int32)
    s = lmb200.lib().lm_cholesky_gaxpy_host(ctx.h, n, lmb200._np_ptr(np.ascontiguousarray(A)), lmb200._np_ptr(Gh),
                                            inf.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    assert s == 0 and inf[0] == 0 and np.abs(Gh - Go).max() <= 1e-13 * np.abs(Go).max()


# ---- tridiagSolve ------------------------------------------------------------------

def test_tridiag_known_answer(ctx, golden_known):
    # test_tridiagKnown (test/Test/Solve.hs:138-150): A = tridiag(-1, 2, -1), b = [1, 0, 1], x = [1, 1, 1]
    d = np.full(3, 2.0)
    sup = np.array([-1.0, -1.0, 0.0])
    b = np.array([1.0, 0.0, 1.0])
    x = host(lmb200.tridiagSolve(dev(d), dev(sup), dev(b), ctx))
    assert approx_eq(x, [1.0, 1.0, 1.0])
    assert approx_eq(O.tridiag_solve(d, sup, b), [1.0, 1.0, 1.0])


@pytest.mark.parametrize("n", [1, 2, 5, 64, 1000, 4097, 100000, 1 << 20])
def test_tridiag_vs_oracle(ctx, n):
    g = philox(34000 + n)
    sup = g.uniform(-1, 1, n)
    d = 2.5 + g.uniform(0, 1, n)  # diagonally dominant, SPD
    b = g.uniform(-1, 1, n)
    x = host(lmb200.tridiagSolve(dev(d), dev(sup), dev(b), ctx))
    xo = O.tridiag_solve(d, sup, b)
    assert np.abs(x - xo).max() <= 1e-13 * np.abs(xo).max()
    xh = np.empty(n)
    s = lmb200.lib().lm_tridiag_solve_host(ctx.h, n, lmb200._np_ptr(d), lmb200._np_ptr(sup), lmb200._np_ptr(b),
                                           lmb200._np_ptr(xh))
    assert s == 0 and np.array_equal(xh, x)
