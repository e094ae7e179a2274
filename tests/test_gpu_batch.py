"""Batched uneven-size solves (one persistent launch) against the oracle.

Every instance of a mixed batch is checked against the oracle's luSolveP /
choleskySolveP (pivot sequences identical, solutions within the same
kappa-scaled tolerance as the single-system tests); the FP32 + FP64-refinement
plan must reach the normwise backward error 1e-15 n of every instance; an
instance's result is bit-identical alone and inside a large mix.
"""
import json

import numpy as np
import pytest

import lmb200
import oracle as O
from conftest import philox
from helpers import EPS, backward_error, rel_forward

pytestmark = pytest.mark.gpu

EDGE_N = [1, 2, 3, 31, 32, 33, 63, 64, 65, 127, 128, 129, 200, 255, 256]


def make_batch(g, count, nlo=1, nhi=256, rhs_hi=16, edge=True):
    n = g.integers(nlo, nhi + 1, count).astype(np.int32)
    if edge:
        n[:len(EDGE_N)] = EDGE_N[:count]
    nrhs = g.integers(1, rhs_hi + 1, count).astype(np.int32)
    kind = (np.arange(count) % 2).astype(np.int32)  # half general, half SPD
    return n, nrhs, kind


def fill(g, n, nrhs, kind):
    a_off = np.concatenate([[0], np.cumsum(n.astype(np.int64) ** 2)])
    b_off = np.concatenate([[0], np.cumsum(n.astype(np.int64) * nrhs)])
    A = np.empty(a_off[-1])
    B = g.uniform(-1.0, 1.0, b_off[-1])
    for i in range(len(n)):
        m = int(n[i])
        M = g.uniform(-1.0, 1.0, (m, m))
        if kind[i] == lmb200.BATCH_SPD:
            M = M @ M.T + m * np.eye(m)
        A[a_off[i]:a_off[i + 1]] = M.ravel()
    return A, B, a_off, b_off


def view(A, B, X, a_off, b_off, n, nrhs, i):
    m, r = int(n[i]), int(nrhs[i])
    return (A[a_off[i]:a_off[i + 1]].reshape(m, m), B[b_off[i]:b_off[i + 1]].reshape(m, r),
            X[b_off[i]:b_off[i + 1]].reshape(m, r))


def run(plan, A, B, **kw):
    import torch

    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    dX = torch.empty_like(dB)
    plan.solve(dA, dB, dX, **kw)
    return dX.cpu().numpy()


def test_batch_fp64_vs_oracle():
    g = philox(71)
    n, nrhs, kind = make_batch(g, 120)
    A, B, a_off, b_off = fill(g, n, nrhs, kind)
    plan = lmb200.Batch(n, nrhs, kind, lmb200.PREC_FP64)
    assert np.array_equal(plan.a_off, a_off) and np.array_equal(plan.b_off, b_off)
    X = run(plan, A, B)
    info, iters, _ = plan.results()
    assert (info == 0).all() and (iters == 0).all()
    import ctypes

    _, pptr = plan.factors()
    ipiv_all = np.empty(int(n.sum()), dtype=np.int32)
    assert lmb200.lib().lm_d2h(plan.ctx.h, ctypes.c_void_p(ipiv_all.ctypes.data), ctypes.c_void_p(pptr),
                               ipiv_all.nbytes) == 0
    for i in range(len(n)):
        Ai, Bi, Xi = view(A, B, X, a_off, b_off, n, nrhs, i)
        m = int(n[i])
        if kind[i] == lmb200.BATCH_GENERAL:
            Xo, _, ipo = O.lu_solve_p(Ai, Bi)
            assert np.array_equal(ipiv_all[plan.p_off[i]:plan.p_off[i] + m], ipo), f"instance {i}: pivots differ"
        else:
            Xo, _ = O.chol_solve_p(Ai, Bi)
        kappa = np.linalg.cond(Ai) if m > 1 else 1.0
        assert rel_forward(Xi, Xo) <= max(1e-12, 32 * kappa * EPS), f"instance {i} (n={m})"
        for h in range(int(nrhs[i])):
            assert backward_error(Ai, Xi[:, h], Bi[:, h]) <= 1e-15 * m


def test_batch_fp32_ir_reaches_fp64_accuracy():
    g = philox(72)
    n, nrhs, kind = make_batch(g, 100)
    A, B, a_off, b_off = fill(g, n, nrhs, kind)
    plan = lmb200.Batch(n, nrhs, kind, lmb200.PREC_FP32_IR)
    X = run(plan, A, B, tol=0.0, max_iter=10)
    info, iters, berr = plan.results()
    assert (info == 0).all()
    assert (iters >= 0).all(), "no instance should need the FP64 fallback here"
    for i in range(len(n)):
        Ai, Bi, Xi = view(A, B, X, a_off, b_off, n, nrhs, i)
        m = int(n[i])
        worst = max(backward_error(Ai, Xi[:, h], Bi[:, h]) for h in range(int(nrhs[i])))
        assert worst <= 1e-15 * m, f"instance {i} (n={m}) backward error {worst}"
        assert berr[i] <= 1e-15 * m


def test_batch_result_same_alone_and_in_mix():
    g = philox(73)
    n, nrhs, kind = make_batch(g, 600)
    A, B, a_off, b_off = fill(g, n, nrhs, kind)
    for prec in (lmb200.PREC_FP64, lmb200.PREC_FP32_IR):
        X = run(lmb200.Batch(n, nrhs, kind, prec), A, B)
        for i in (0, 5, 17, 333, 599):
            sl_a, sl_b = slice(a_off[i], a_off[i + 1]), slice(b_off[i], b_off[i + 1])
            alone = lmb200.Batch(n[i:i + 1], nrhs[i:i + 1], kind[i:i + 1], prec)
            Xi = run(alone, A[sl_a].copy(), B[sl_b].copy())
            assert np.array_equal(Xi, X[sl_b]), f"instance {i} differs alone vs in the mix (prec {prec})"


def test_batch_edge_cases():
    g = philox(74)
    n = np.array([5, 0, 4, 7, 1, 3], dtype=np.int32)
    nrhs = np.array([2, 3, 1, 0, 1, 16], dtype=np.int32)
    kind = np.array([0, 0, 1, 0, 1, 0], dtype=np.int32)
    A, B, a_off, b_off = fill(g, n, nrhs, kind)
    A[a_off[0]:a_off[1]] = 0.0                      # singular: first pivot is zero
    A[a_off[2]:a_off[3]] = -np.eye(4).ravel()       # not SPD: first diagonal negative
    plan = lmb200.Batch(n, nrhs, kind, lmb200.PREC_FP64)
    X = run(plan, A, B)
    info, _, _ = plan.results()
    assert info[0] == 1 and info[2] == 1 and info[1] == 0 and info[3] == 0
    for i in (4, 5):
        Ai, Bi, Xi = view(A, B, X, a_off, b_off, n, nrhs, i)
        ref = O.lu_solve_p(Ai, Bi)[0] if kind[i] == 0 else O.chol_solve_p(Ai, Bi)[0]
        assert np.allclose(Xi, ref, rtol=1e-13, atol=1e-13)
    empty = lmb200.Batch(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert empty.results()[0].size == 0
    with pytest.raises(lmb200.LMError):
        lmb200.Batch(np.array([257], np.int32), np.array([1], np.int32), np.array([0], np.int32))
    with pytest.raises(lmb200.LMError):
        lmb200.Batch(np.array([8], np.int32), np.array([17], np.int32), np.array([0], np.int32))


def test_batch_host_entry_matches_device():
    g = philox(75)
    n, nrhs, kind = make_batch(g, 50, edge=False)
    A, B, _, _ = fill(g, n, nrhs, kind)
    plan = lmb200.Batch(n, nrhs, kind)
    assert np.array_equal(plan.solve_host(A, B), run(plan, A, B))


def test_batch_full_size_backward_error():
    """The bench's workload shape (n uniform in [8, 256], nrhs in [1, 16], half
    SPD) at 2000 instances: every instance at FP64 accuracy, FP64 and IR."""
    g = philox(76)
    n, nrhs, kind = make_batch(g, 2000, nlo=8, edge=False)
    A, B, a_off, b_off = fill(g, n, nrhs, kind)
    for prec in (lmb200.PREC_FP64, lmb200.PREC_FP32_IR):
        plan = lmb200.Batch(n, nrhs, kind, prec)
        X = run(plan, A, B)
        info, iters, _ = plan.results()
        assert (info == 0).all()
        for i in range(0, len(n), 7):
            Ai, Bi, Xi = view(A, B, X, a_off, b_off, n, nrhs, i)
            r = Ai @ Xi - Bi
            den = np.abs(Ai).sum(axis=1).max() * np.abs(Xi).max(axis=0) + np.abs(Bi).max(axis=0)
            assert (np.abs(r).max(axis=0) / den).max() <= 1e-15 * int(n[i])


def test_batch_autotune_table(tmp_path):
    ctx = lmb200.default_context(0)
    saved = lmb200.batch_tune_get(ctx)
    try:
        path = tmp_path / "tune.json"
        table = lmb200.batch_tune(lmb200.PREC_FP64, str(path), ctx)
        assert all(v in (8, 16, 32) for v in table[0])
        doc = json.loads(path.read_text())
        assert doc["nb"][0] == table[0] and len(doc["best_ms"]) == 4
        g = philox(77)
        n, nrhs, kind = make_batch(g, 40, edge=False)
        A, B, a_off, b_off = fill(g, n, nrhs, kind)
        X = run(lmb200.Batch(n, nrhs, kind), A, B)
        for i in range(len(n)):
            Ai, Bi, Xi = view(A, B, X, a_off, b_off, n, nrhs, i)
            assert backward_error(Ai, Xi[:, 0], Bi[:, 0]) <= 1e-15 * int(n[i])
    finally:
        lmb200.batch_tune_set(saved, ctx)
