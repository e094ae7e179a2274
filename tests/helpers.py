"""Numerical helpers shared by the tests (metrics of the reference's suite)."""
import numpy as np

EPS = 2.220446049250313e-16  # test/Test/Residuals.hs:57-58


def approx_eq(x, y, tol=1e-8):
    """(~=) of test/Test/Types.hs:44-50: |x-y| < tol*(1+|x|+|y|), elementwise."""
    x, y = np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)
    return bool(np.all(np.abs(x - y) < tol * (1 + np.abs(x) + np.abs(y))))


def backward_error(A, x, b):
    """Normwise backward error ||Ax-b||_inf / (||A||_inf ||x||_inf + ||b||_inf)."""
    A, x, b = (np.asarray(v, dtype=np.float64) for v in (A, x, b))
    r = A @ x - b
    num = np.abs(r).max()
    den = np.abs(A).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max()
    return float(num / den)


def rel_forward(x, xref):
    x, xref = np.asarray(x), np.asarray(xref)
    return float(np.abs(x - xref).max() / np.abs(xref).max())


def gen_uniform(g, n, lo=-1.0, hi=1.0):
    return g.uniform(lo, hi, (n, n))


def gen_spd(g, n):
    """A = B B^T + n I with B uniform[-1,1] (the SPD workload construction)."""
    B = g.uniform(-1.0, 1.0, (n, n))
    return B @ B.T + n * np.eye(n)


def gen_randsvd(g, n, kappa, lo=-10.0, hi=10.0):
    """randsvd of test/Test/Types.hs:196-213: U diag(sigma) V^T, sigma_i = kappa^(-i/(n-1))."""
    U, _ = np.linalg.qr(g.uniform(lo, hi, (n, n)))
    V, _ = np.linalg.qr(g.uniform(lo, hi, (n, n)))
    s = kappa ** (-np.arange(n) / max(n - 1, 1)) if n > 1 else np.ones(1)
    return (U * s) @ V.T
