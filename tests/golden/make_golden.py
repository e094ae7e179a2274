"""Generate the golden fixtures used by the test suite.

known_answers.json — the known-answer cases of linear-massiv's own test
suite for this path, restated with exact expected values:
  * test_luKnown          test/Test/Solve.hs:107-119
  * test_matMulKnown      test/Test/BLAS.hs:132-144
  * test_gemmLarger       test/Test/BLAS.hs:156-172
  * test_luHilbert        test/Test/Solve.hs:157-166   (scaled residual < 1e-4)
  * test_detEqualsEigenProduct  test/Test/Solve.hs:228-238 (rel. err < 1e-4)
  * the deterministic benchmark matrices mkDDLM / mkSPDLM / mkVecLM
    (bench-comparison/Main.hs:43-65) at n = 10, 50, 100.
Exact answers come from rational arithmetic (fractions), not from the oracle.

oracle_regression.npz — seeded inputs (numpy Philox) and the oracle's
bit-exact outputs for luSolveP, choleskySolveP and matMulP at sizes that hit
every tail path (n < 64 unblocked, n >= 64 panels, packed GEMM above 96).
They pin the oracle build against itself across machines.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def solve_exact(A, b):
    """Gaussian elimination over the rationals."""
    n = len(A)
    M = [[Fraction(A[i][j]) for j in range(n)] + [Fraction(b[i])] for i in range(n)]
    for k in range(n):
        p = next(i for i in range(k, n) if M[i][k] != 0)
        M[k], M[p] = M[p], M[k]
        for i in range(n):
            if i != k and M[i][k] != 0:
                f = M[i][k] / M[k][k]
                M[i] = [a - f * c for a, c in zip(M[i], M[k])]
    return [M[i][n] / M[i][i] for i in range(n)]


def det_exact(A):
    n = len(A)
    M = [[Fraction(x) for x in row] for row in A]
    d = Fraction(1)
    for k in range(n):
        p = next((i for i in range(k, n) if M[i][k] != 0), None)
        if p is None:
            return Fraction(0)
        if p != k:
            M[k], M[p] = M[p], M[k]
            d = -d
        d *= M[k][k]
        for i in range(k + 1, n):
            f = M[i][k] / M[k][k]
            M[i] = [a - f * c for a, c in zip(M[i], M[k])]
    return d


def known_answers():
    cases = {}
    A = [[2, 1, 1], [4, 3, 3], [8, 7, 9]]
    b = [1, 1, 1]
    cases["test_luKnown"] = {"A": A, "b": b, "x": [float(v) for v in solve_exact(A, b)],
                             "source": "test/Test/Solve.hs:107-119"}
    cases["test_matMulKnown"] = {"A": [[1, 2], [3, 4]], "B": [[5, 6], [7, 8]], "C": [[19, 22], [43, 50]],
                                 "source": "test/Test/BLAS.hs:132-144"}
    A3 = [[i * 3 + j + 1 for j in range(3)] for i in range(3)]
    B3 = [[9 - (i * 3 + j) for j in range(3)] for i in range(3)]
    C3 = [[1 if i == j else 0 for j in range(3)] for i in range(3)]
    ref = [[2 * sum(A3[i][l] * B3[l][j] for l in range(3)) + 0.5 * C3[i][j] for j in range(3)] for i in range(3)]
    cases["test_gemmLarger"] = {"alpha": 2.0, "beta": 0.5, "A": A3, "B": B3, "C": C3, "expected": ref,
                                "source": "test/Test/BLAS.hs:156-172"}
    H = [[Fraction(1, i + j + 1) for j in range(5)] for i in range(5)]
    xh = [i + 1 for i in range(5)]
    cases["test_luHilbert"] = {"n": 5, "x": xh, "residual_bound": 1e-4, "source": "test/Test/Solve.hs:157-166"}
    D = [[(Fraction({0: 4, 1: 3, 2: 2}.get(i, 1)) if i == j else 0) + Fraction(1, 10) for j in range(4)]
         for i in range(4)]
    cases["test_detEqualsEigenProduct"] = {"A": [[float(v) for v in r] for r in D], "det": float(det_exact(D)),
                                           "rel_bound": 1e-4, "source": "test/Test/Solve.hs:228-238"}
    bench = {}
    for n in (10, 50, 100):
        dd = [[Fraction(i * 7 + j * 3 + 1, 100) + (n if i == j else 0) for j in range(n)] for i in range(n)]
        vec = [Fraction(i + 1, 10) for i in range(n)]
        Bm = [[Fraction(i * n + j + 1, n * n) for j in range(n)] for i in range(n)]
        spd = [[(1 if i == j else 0) + sum(Bm[i][k] * Bm[j][k] for k in range(n)) for j in range(n)]
               for i in range(n)]
        bench[str(n)] = {
            "lu_x": [float(v) for v in solve_exact(dd, vec)],
            "chol_x": [float(v) for v in solve_exact(spd, vec)],
        }
    cases["bench_comparison"] = {"source": "bench-comparison/Main.hs:43-65", "solutions": bench}
    return cases


def oracle_regression():
    import oracle as O

    out = {}
    for n in (3, 10, 63, 64, 65, 100):
        g = np.random.Generator(np.random.Philox(1000 + n))
        A = g.uniform(-1.0, 1.0, (n, n))
        b = g.uniform(-1.0, 1.0, n)
        x, LU, ipiv = O.lu_solve_p(A, b)
        out[f"lu{n}_A"], out[f"lu{n}_b"], out[f"lu{n}_x"] = A, b, x
        out[f"lu{n}_ipiv"] = ipiv
        if n <= 65:
            out[f"lu{n}_LU"] = LU
        Bm = g.uniform(-1.0, 1.0, (n, n))
        S = Bm @ Bm.T + n * np.eye(n)
        xc, G = O.chol_solve_p(S, b)
        out[f"ch{n}_A"], out[f"ch{n}_x"] = S, xc
        if n <= 65:
            out[f"ch{n}_G"] = np.tril(G)
    for (m, k, n) in ((7, 5, 3), (65, 33, 70), (100, 100, 101)):
        g = np.random.Generator(np.random.Philox(2000 + m))
        A = g.uniform(-1.0, 1.0, (m, k))
        B = g.uniform(-1.0, 1.0, (k, n))
        key = f"mm{m}x{k}x{n}"
        out[key + "_A"], out[key + "_B"], out[key + "_C"] = A, B, O.matmul_p(A, B)
    return out


if __name__ == "__main__":
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(known_answers(), f, indent=1)
    np.savez_compressed(os.path.join(HERE, "oracle_regression.npz"), **oracle_regression())
    print("wrote", os.listdir(HERE))
