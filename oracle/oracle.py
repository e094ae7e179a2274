"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates linear-massiv's CPU algorithms for the dense-solve path
(see oracle.cpp for the per-function reference citations).  Only the test
suite, the smoke check and the benchmark's CPU-baseline leg load it, and only
as the checker or as the timed CPU baseline; the CUDA library never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build() -> str:
    """Compile liboracle.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        src = os.path.join(_HERE, "oracle.cpp")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(path)
        i, d = ctypes.c_int, ctypes.c_double
        sig = {
            "orc_gemm_kernel": [_dp, _dp, _dp, i, i, i],
            "orc_matmul_p": [_dp, _dp, _dp, i, i, i],
            "orc_matmul_par": [_dp, _dp, _dp, i, i, i, i],
            "orc_gemm_generic": [d, _dp, _dp, d, _dp, _dp, i, i, i],
            "orc_lu_factor_p": [_dp, i, _ip, _ip],
            "orc_lu_solve_p": [_dp, _dp, _dp, i, i, _dp, _ip, _ip],
            "orc_chol_factor_p": [_dp, _dp, i],
            "orc_chol_solve_p": [_dp, _dp, _dp, i, i, _dp],
            "orc_lu_generic": [_dp, _dp, _ip, i],
            "orc_lu_solve_generic": [_dp, _dp, _dp, i],
            "orc_cholesky_generic": [_dp, _dp, i],
            "orc_chol_solve_generic": [_dp, _dp, _dp, i],
            "orc_det": [_dp, i],
            "orc_matvec_p": [_dp, _dp, _dp, i, i],
            "orc_matvec_generic": [_dp, _dp, _dp, i, i],
            "orc_lu_solve_p_many": [_dp, _dp, _dp, i, i, i],
            "orc_chol_solve_p_many": [_dp, _dp, _dp, i, i, i],
            "orc_set_threads": [i],
            "orc_lu_nopivot": [_dp, i],
            "orc_cholesky_gaxpy": [_dp, _dp, i],
            "orc_tridiag_solve": [_dp, _dp, _dp, _dp, i],
            "orc_norm_inf": [_dp, i, i],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int if name in ("orc_lu_factor_p", "orc_lu_solve_p") else (
                ctypes.c_double if name in ("orc_det", "orc_norm_inf") else None)
        _LIB = L
    return _LIB


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


# --- GEMM -----------------------------------------------------------------

def matmul_p(A, B) -> np.ndarray:
    """matMulP: C = A*B through the reference's 4x8 micro-kernel GEMM."""
    A, B = _c(A), _c(B)
    m, k = A.shape
    n = B.shape[1]
    C = np.empty((m, n))
    lib().orc_matmul_p(_d(A), _d(B), _d(C), m, k, n)
    return C


def matmul_par(A, B, threads: int) -> np.ndarray:
    """matMulPPar with `threads` capabilities (same tiling of C as the reference)."""
    A, B = _c(A), _c(B)
    m, k = A.shape
    n = B.shape[1]
    C = np.empty((m, n))
    lib().orc_matmul_par(_d(A), _d(B), _d(C), m, k, n, threads)
    return C


def gemm_kernel_acc(A, B, C) -> np.ndarray:
    """rawGemmKernel: returns C + A*B (C is not modified)."""
    A, B = _c(A), _c(B)
    C = _c(C).copy()
    m, k = A.shape
    n = B.shape[1]
    lib().orc_gemm_kernel(_d(A), _d(B), _d(C), m, k, n)
    return C


def gemm_generic(alpha, A, B, beta, C0) -> np.ndarray:
    """gemm alpha A B beta C (generic massiv path)."""
    A, B, C0 = _c(A), _c(B), _c(C0)
    m, k = A.shape
    n = B.shape[1]
    C = np.empty((m, n))
    lib().orc_gemm_generic(float(alpha), _d(A), _d(B), float(beta), _d(C0), _d(C), m, k, n)
    return C


# --- LU ---------------------------------------------------------------------

def lu_factor_p(A):
    """Factor phase of luSolveP: (packed LU, swap list as int array of pivot rows).

    The swap list is returned as a length-n array `ipiv` with ipiv[k] = pivot
    row chosen at step k (k itself for steps the reference does not record).
    """
    LU = _c(A).copy()
    n = LU.shape[0]
    sk = np.zeros(max(n, 1), dtype=np.int32)
    sr = np.zeros(max(n, 1), dtype=np.int32)
    cnt = lib().orc_lu_factor_p(_d(LU), n, sk.ctypes.data_as(_ip), sr.ctypes.data_as(_ip))
    ipiv = np.arange(n, dtype=np.int32)
    ipiv[sk[:cnt]] = sr[:cnt]
    return LU, ipiv


def lu_solve_p(A, B):
    """luSolveP for a vector b (n,) or n x nrhs matrix B: returns (x, LU, ipiv)."""
    A = _c(A)
    n = A.shape[0]
    vec = np.ndim(B) == 1
    B2 = _c(B).reshape(n, -1)
    nrhs = B2.shape[1]
    X = np.empty_like(B2)
    LU = np.empty((n, n))
    sk = np.zeros(max(n, 1), dtype=np.int32)
    sr = np.zeros(max(n, 1), dtype=np.int32)
    cnt = lib().orc_lu_solve_p(_d(A), _d(B2), _d(X), n, nrhs, _d(LU), sk.ctypes.data_as(_ip),
                               sr.ctypes.data_as(_ip))
    ipiv = np.arange(n, dtype=np.int32)
    ipiv[sk[:cnt]] = sr[:cnt]
    return (X[:, 0] if vec else X), LU, ipiv


def lu_generic(A):
    """lu: (packed LU, permutation vector perm with (PA)[i] = A[perm[i]])."""
    A = _c(A)
    n = A.shape[0]
    LU = np.empty_like(A)
    perm = np.zeros(n, dtype=np.int32)
    lib().orc_lu_generic(_d(A), _d(LU), perm.ctypes.data_as(_ip), n)
    return LU, perm


def lu_solve_generic(A, b):
    A, b = _c(A), _c(b)
    x = np.empty_like(b)
    lib().orc_lu_solve_generic(_d(A), _d(b), _d(x), A.shape[0])
    return x


def det(A) -> float:
    A = _c(A)
    return lib().orc_det(_d(A), A.shape[0])


# --- Cholesky ---------------------------------------------------------------

def chol_factor_p(A) -> np.ndarray:
    A = _c(A)
    n = A.shape[0]
    G = np.empty_like(A)
    lib().orc_chol_factor_p(_d(A), _d(G), n)
    return G


def chol_solve_p(A, B):
    """choleskySolveP for a vector or n x nrhs matrix: returns (x, G)."""
    A = _c(A)
    n = A.shape[0]
    vec = np.ndim(B) == 1
    B2 = _c(B).reshape(n, -1)
    X = np.empty_like(B2)
    G = np.empty((n, n))
    lib().orc_chol_solve_p(_d(A), _d(B2), _d(X), n, B2.shape[1], _d(G))
    return (X[:, 0] if vec else X), G


def cholesky_generic(A) -> np.ndarray:
    A = _c(A)
    G = np.empty_like(A)
    lib().orc_cholesky_generic(_d(A), _d(G), A.shape[0])
    return G


def chol_solve_generic(A, b):
    A, b = _c(A), _c(b)
    x = np.empty_like(b)
    lib().orc_chol_solve_generic(_d(A), _d(b), _d(x), A.shape[0])
    return x


def set_threads(threads: int) -> None:
    """Host threads of the row-parallel trailing updates (0 = all; bitwise the same result)."""
    lib().orc_set_threads(int(threads))


def lu_nopivot(A) -> np.ndarray:
    """luNoPivot: packed unit-L / U without row interchanges."""
    LU = _c(A).copy()
    lib().orc_lu_nopivot(_d(LU), LU.shape[0])
    return LU


def cholesky_gaxpy(A) -> np.ndarray:
    """choleskyGaxpy: G (lower, zeros above) by the gaxpy column loop."""
    A = _c(A)
    G = np.empty_like(A)
    lib().orc_cholesky_gaxpy(_d(A), _d(G), A.shape[0])
    return G


def tridiag_solve(diag, supdiag, b) -> np.ndarray:
    """tridiagSolve: SPD tridiagonal solve from the diagonal and superdiagonal
    (length n, entries 0..n-2 used)."""
    diag, supdiag, b = _c(diag), _c(supdiag), _c(b)
    x = np.empty_like(b)
    lib().orc_tridiag_solve(_d(diag), _d(supdiag), _d(b), _d(x), b.shape[0])
    return x


# --- BLAS-2 and norms ---------------------------------------------------------

def norm_inf(A) -> float:
    """normInf: largest row sum of |a_ij| (each row a left fold in column order)."""
    A = _c(A)
    if A.ndim == 1:
        A = A.reshape(-1, 1)
    return lib().orc_norm_inf(_d(A), A.shape[0], A.shape[1])


def matvec_p(A, x):
    A, x = _c(A), _c(x)
    y = np.empty(A.shape[0])
    lib().orc_matvec_p(_d(A), _d(x), _d(y), A.shape[0], A.shape[1])
    return y


def matvec_generic(A, x):
    A, x = _c(A), _c(x)
    y = np.empty(A.shape[0])
    lib().orc_matvec_generic(_d(A), _d(x), _d(y), A.shape[0], A.shape[1])
    return y


# --- CPU baseline throughput helpers ----------------------------------------

def lu_solve_p_many(A, b, count: int, threads: int):
    A, b = _c(A), _c(b)
    x = np.empty_like(b)
    lib().orc_lu_solve_p_many(_d(A), _d(b), _d(x), A.shape[0], count, threads)
    return x


def chol_solve_p_many(A, b, count: int, threads: int):
    A, b = _c(A), _c(b)
    x = np.empty_like(b)
    lib().orc_chol_solve_p_many(_d(A), _d(b), _d(x), A.shape[0], count, threads)
    return x


# --- Residual metrics of the reference's test suite --------------------------

MACHINE_EPS = 2.220446049250313e-16  # test/Test/Residuals.hs:57-58


def scaled_residual_linear(A, x, b) -> float:
    """scaledResidualLinear (test/Test/Residuals.hs:69-78)."""
    A, x, b = _c(A), _c(x), _c(b)
    r = matvec_generic(A, x) - b
    n = A.shape[0]
    denom = np.abs(A).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max() + n * MACHINE_EPS
    return float(np.abs(r).max() / denom)


def scaled_residual_lu(A, LU, perm) -> float:
    """scaledResidualLU (test/Test/Residuals.hs:167-189) with a permutation vector."""
    n = A.shape[0]
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    PA = np.asarray(A)[np.asarray(perm)]
    diff = PA - L @ U
    return float(np.linalg.norm(diff) / (np.linalg.norm(A) * n * MACHINE_EPS + MACHINE_EPS))


def scaled_residual_cholesky(A, G) -> float:
    """scaledResidualCholesky (test/Test/Residuals.hs:148-156)."""
    n = A.shape[0]
    G = np.tril(G)
    diff = np.asarray(A) - G @ G.T
    return float(np.linalg.norm(diff) / (np.linalg.norm(A) * n * MACHINE_EPS + MACHINE_EPS))


def ipiv_to_perm(ipiv) -> np.ndarray:
    """Swap list (LAPACK ipiv style) -> permutation vector perm, (PA)[i] = A[perm[i]]."""
    n = len(ipiv)
    perm = np.arange(n)
    for k in range(n):
        p = int(ipiv[k])
        if p != k:
            perm[k], perm[p] = perm[p], perm[k]
    return perm
