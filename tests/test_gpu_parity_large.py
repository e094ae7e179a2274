"""GPU parity at the full sizes of the plain FP64 workloads, against the oracle.

The plain FP64 workloads are gemm m = n = k = 8192, luSolve n = 8192 and
16384 (nrhs 1 and 64) and cholSolve n = 8192 (nrhs 1 and 64), all with
uniform[-1,1] inputs (SPD: B B^T + n I).  The oracle runs the reference's
algorithms (luSolveP, choleskySolveP, matMulPPar) with its trailing updates
split over host threads by 64-row tiles, which leaves every value bitwise the
same as a single thread.

Bars:
  * LU: identical pivot sequence; relative forward error vs the oracle
    <= max(1e-12, 32 kappa eps) with kappa the 1-norm condition number
    estimated from the oracle's factors (Hager's estimator); normwise backward
    error <= 1e-15 n for every column.
  * Cholesky: G within 1e-13 max|G| of the oracle's; forward error <= 1e-12;
    backward error <= 1e-15 n.
  * GEMM: elementwise |C - C_oracle| <= 2 k eps (|A||B|)_ij.
"""
import os

import numpy as np
import pytest
import scipy.linalg as sla
import torch

import lmb200
import oracle as O
from conftest import philox
from helpers import backward_error, gen_spd, gen_uniform, rel_forward

pytestmark = pytest.mark.gpu
EPS = 2.220446049250313e-16


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def cond1_estimate(A, LU, ipiv):
    """||A||_1 times Hager's estimate of ||A^-1||_1 from the packed LU factor
    and its swap list (LAPACK convention, as scipy's lu_solve takes it)."""
    n = A.shape[0]
    fac = (np.asfortranarray(LU), np.asarray(ipiv, dtype=np.int32))
    x = np.full(n, 1.0 / n)
    est = 0.0
    for _ in range(5):
        y = sla.lu_solve(fac, x, check_finite=False)
        est = np.abs(y).sum()
        z = sla.lu_solve(fac, np.where(y >= 0, 1.0, -1.0), trans=1, check_finite=False)
        j = int(np.argmax(np.abs(z)))
        if np.abs(z[j]) <= z @ x:
            break
        x = np.zeros(n)
        x[j] = 1.0
    return float(np.abs(A).sum(axis=0).max() * est)


def columns_ok(A, X, B, Xo, kappa):
    n = A.shape[0]
    bound = max(1e-12, 32 * kappa * EPS)
    for c in range(X.shape[1]):
        assert backward_error(A, X[:, c], B[:, c]) <= 1e-15 * n, f"column {c}"
        assert rel_forward(X[:, c], Xo[:, c]) <= bound, f"column {c}"


@pytest.mark.parametrize("n,nrhs", [(8192, 1), (8192, 64), (16384, 1)])
def test_lu_solve_full_size_vs_oracle(ctx, n, nrhs):
    O.set_threads(0)
    g = philox(90000 + n + nrhs)
    A, B = gen_uniform(g, n), g.uniform(-1, 1, (n, nrhs))
    dA = dev(A)
    _, ipiv, info = lmb200.lu_factor(dA, ctx)
    X = host(lmb200.luSolve(dA, dev(B), ctx))
    del dA
    Xo, LUo, ipo = O.lu_solve_p(A, B)
    assert info == 0
    agree = float(np.mean(host(ipiv) == ipo))
    assert agree == 1.0, f"pivot agreement {agree}"
    kappa = cond1_estimate(A, LUo, ipo)
    columns_ok(A, X, B, Xo, kappa)


@pytest.mark.parametrize("nrhs", [1, 64])
def test_cholesky_solve_full_size_vs_oracle(ctx, nrhs):
    O.set_threads(0)
    n = 8192
    g = philox(91000 + nrhs)
    A, B = gen_spd(g, n), g.uniform(-1, 1, (n, nrhs))
    dA = dev(A)
    X = host(lmb200.choleskySolve(dA, dev(B), ctx))
    G = host(lmb200.cholesky(dA, ctx)) if nrhs == 1 else None
    del dA
    Xo, Go = O.chol_solve_p(A, B)
    for c in range(nrhs):
        assert backward_error(A, X[:, c], B[:, c]) <= 1e-15 * n
        assert rel_forward(X[:, c], Xo[:, c]) <= 1e-12
    if G is not None:
        assert np.all(np.triu(G, 1) == 0.0)
        assert np.abs(G - np.tril(Go)).max() <= 1e-13 * np.abs(Go).max()


def test_gemm_full_size_vs_oracle(ctx):
    n = 8192
    g = philox(92000)
    A, B = g.uniform(-1, 1, (n, n)), g.uniform(-1, 1, (n, n))
    C = host(lmb200.matMul(dev(A), dev(B), ctx))
    ref = O.matmul_par(A, B, os.cpu_count() or 1)
    bound = 2 * n * EPS * (np.abs(A) @ np.abs(B))
    assert np.all(np.abs(C - ref) <= bound)
