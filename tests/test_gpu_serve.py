"""Serving loop (continuous batching, HBM-budget admission) on the GPU.

Requests mix small instances (the device-resident loop or micro-batches of the
persistent batch kernel) and larger ones (FP64 LU or Cholesky at the bucket
order, or the mixed-precision LU + FP64 refinement for general and SPD systems
with FP64 LU or Cholesky as the fallback).  Checked: every result reaches the normwise backward error
1e-15 n; each result is the same alone and in the mix (bitwise: the
per-request computation does not depend on what else runs); admission never
exceeds the arena; small requests overtake a large one in flight; host-side
failures (oversized requests, a producer thread dying mid-stream, cancelled
requests, a singular system) leave the server serving.
"""
import threading
import time

import numpy as np
import pytest

import lmb200
from conftest import philox

pytestmark = pytest.mark.gpu

TOL = 1e-15  # normwise backward error per unit of n


def sigma_matrix(g, n, kappa, spd):
    """U diag(sigma) V^T (V = U for SPD), U and V products of 4 Householder
    reflectors, sigma geometric from 1 to 1/kappa."""
    s = kappa ** (-np.arange(n) / max(n - 1, 1))

    def reflect(M, left):
        for _ in range(4):
            v = g.standard_normal(n)
            v /= np.linalg.norm(v)
            M = M - 2.0 * np.outer(v, v @ M) if left else M - 2.0 * np.outer(M @ v, v)
        return M

    U = reflect(np.eye(n), True)
    V = U if spd else reflect(np.eye(n), True)
    return (U * s) @ V.T


def berr(A, X, B):
    r = np.abs(A @ X - B).max(axis=0)
    den = np.abs(A).sum(axis=1).max() * np.abs(X).max(axis=0) + np.abs(B).max(axis=0)
    return float((r / den).max())


def make_requests(g, count, nmax):
    reqs = []
    for _ in range(count):
        n = int(np.exp(g.uniform(np.log(16), np.log(nmax))))
        nrhs = int(g.choice([1, 8, 32]))
        spd = g.uniform() < 0.3
        kappa = float(np.exp(g.uniform(np.log(1e1), np.log(1e6))))
        A = sigma_matrix(g, n, kappa, spd)
        B = g.uniform(-1.0, 1.0, (n, nrhs))
        reqs.append((A, B, lmb200.BATCH_SPD if spd else lmb200.BATCH_GENERAL))
    return reqs


@pytest.fixture(scope="module", params=["fp64", "ir"])
def server(request):
    """Larger requests by FP64 LU / Cholesky at the bucket order (the default up
    to order 2048 / 4096), or all of them by the mixed-precision solve."""
    limits = {} if request.param == "fp64" else {"lu_fp64_max_n": 0, "chol_fp64_max_n": 0}
    s = lmb200.Server(0, max_n=1024, max_nrhs=64, large_workers=3, batch_lanes=2, hbm_budget=512 << 20, **limits)
    s.route = request.param
    yield s
    s.close()


def test_mix_matches_alone_and_fp64_accuracy(server):
    g = philox(91)
    reqs = make_requests(g, 48, 1024)
    ids = [server.submit(A, B, k) for A, B, k in reqs]
    mixed = []
    for (rid, X), (A, B, k) in zip(ids, reqs):
        st, lat = server.wait(rid, 60.0)
        assert st == 0 and lat > 0
        assert berr(A, X, B) <= TOL * A.shape[0]
        mixed.append(X.copy())
    # each one alone (the server otherwise idle)
    for (A, B, k), Xm in zip(reqs, mixed):
        rid, X = server.submit(A, B, k)
        assert server.wait(rid, 60.0)[0] == 0
        assert np.array_equal(X, Xm), "result differs alone vs in the mix"
    st = server.stats()
    assert st["completed"] >= 96 and st["failed"] == 0
    assert (st["ir_solves"] > 0) == (server.route == "ir")
    assert st["arena_peak_bytes"] <= st["arena_bytes"]
    assert st["micro_batches"] >= 1 and st["small_solved"] >= 1


def test_device_loop_matches_micro_batches():
    """Small requests on the device-resident loop (the default) give the same
    bits as the micro-batch lanes of the batch kernel, and the loop returns to
    the host when idle and is relaunched by the next request."""
    g = philox(97)
    reqs = []
    for _ in range(40):
        n = int(g.integers(8, 257))
        r = int(g.integers(1, 17))
        spd = g.uniform() < 0.5
        M = g.uniform(-1, 1, (n, n))
        M = M @ M.T + n * np.eye(n) if spd else M
        reqs.append((M, g.uniform(-1, 1, (n, r)), lmb200.BATCH_SPD if spd else lmb200.BATCH_GENERAL))
    outs = {}
    for loop in (1, 0):
        s = lmb200.Server(0, max_n=256, max_nrhs=16, large_workers=1, batch_lanes=2, device_loop=loop)
        try:
            ids = [s.submit(A, B, k) for A, B, k in reqs[:20]]
            time.sleep(0.05)  # long enough for an idle loop to return
            ids += [s.submit(A, B, k) for A, B, k in reqs[20:]]
            res = []
            for (rid, X), (A, B, k) in zip(ids, reqs):
                assert s.wait(rid, 60.0)[0] == 0
                assert berr(A, X, B) <= TOL * A.shape[0]
                res.append(X.copy())
            outs[loop] = res
            st = s.stats()
            assert st["small_solved"] == 40 and st["micro_batches"] >= (2 if loop else 1)
        finally:
            s.close()
    for a, b in zip(outs[1], outs[0]):
        assert np.array_equal(a, b)


def test_small_requests_overtake_a_large_one(server):
    g = philox(92)
    A = sigma_matrix(g, 1024, 1e3, False)
    B = g.uniform(-1, 1, (1024, 32))
    big, Xb = server.submit(A, B, lmb200.BATCH_GENERAL)
    small = []
    for _ in range(20):
        n = int(g.integers(16, 128))
        M = g.uniform(-1, 1, (n, n)) + n * np.eye(n)
        b = g.uniform(-1, 1, (n, 4))
        small.append((server.submit(M, b, lmb200.BATCH_GENERAL), M, b))
    done_small = 0
    for (rid, X), M, b in small:
        st, _ = server.wait(rid, 60.0)
        assert st == 0 and berr(M, X, b) <= TOL * M.shape[0]
        done_small += 1
    st, _ = server.wait(big, 60.0)
    assert st == 0 and berr(A, Xb, B) <= TOL * 1024
    assert done_small == 20


def test_admission_respects_budget_and_overlaps():
    g = philox(93)
    # room for about three n=512 requests at a time
    budget = 3 * (512 * 512 * 8 + 2 * 512 * 8 * 8 + 512 * 4 + 4096)
    s = lmb200.Server(0, max_n=512, max_nrhs=8, large_workers=4, batch_lanes=1, hbm_budget=budget)
    try:
        reqs = [(g.uniform(-1, 1, (512, 512)) + 512 * np.eye(512), g.uniform(-1, 1, (512, 8))) for _ in range(10)]
        ids = [s.submit(A, B, lmb200.BATCH_GENERAL) for A, B in reqs]
        for (rid, X), (A, B) in zip(ids, reqs):
            assert s.wait(rid, 60.0)[0] == 0
            assert berr(A, X, B) <= TOL * 512
        st = s.stats()
        assert st["arena_peak_bytes"] <= budget
        assert 2 <= st["inflight_peak"] <= 3, st
    finally:
        s.close()


def test_request_larger_than_the_arena_is_rejected():
    s = lmb200.Server(0, max_n=512, max_nrhs=8, large_workers=1, batch_lanes=1, hbm_budget=1 << 20)
    try:
        with pytest.raises(lmb200.LMError) as e:
            s.submit(np.eye(512), np.ones((512, 8)))
        assert e.value.status == lmb200.LM_ERR_NOMEM
        rid, X = s.submit(np.eye(100) * 2.0, np.ones((100, 1)))  # a small one still fits
        assert s.wait(rid, 60.0)[0] == 0 and np.allclose(X, 0.5)
        assert s.stats()["rejected"] == 1
    finally:
        s.close()


def test_host_side_failures_leave_the_server_serving(server):
    g = philox(94)
    # outside the configured sizes
    with pytest.raises(lmb200.LMError):
        server.submit(np.eye(2048), np.ones(2048))
    # a producer thread that dies mid-stream: what it submitted still completes
    submitted = []

    def producer():
        for i in range(6):
            n = 64 + 16 * i
            M = g.uniform(-1, 1, (n, n)) + n * np.eye(n)
            b = g.uniform(-1, 1, (n, 2))
            submitted.append((server.submit(M, b), M, b))
            if i == 3:
                raise RuntimeError("producer killed")

    t = threading.Thread(target=producer)
    t.start()
    t.join()
    assert len(submitted) == 4
    for (rid, X), M, b in submitted:
        assert server.wait(rid, 60.0)[0] == 0 and berr(M, X, b) <= TOL * M.shape[0]
    # a singular system completes with its LAPACK-style info (FP64 fallback ran)
    Z = np.zeros((300, 300))
    rid, _ = server.submit(Z, np.ones((300, 1)))
    st, _ = server.wait(rid, 60.0)
    assert st == 1
    # requests dropped by their client (never waited for) still complete and free their memory
    for _ in range(5):
        n = 200
        server.submit(g.uniform(-1, 1, (n, n)) + n * np.eye(n), g.uniform(-1, 1, (n, 1)))
    server.drain(60.0)
    st = server.stats()
    assert st["pending"] == 0 and st["inflight"] == 0


def test_cancel_queued_request():
    g = philox(95)
    budget = 520 * 520 * 8 + 4 * 520 * 8 + 8192
    s = lmb200.Server(0, max_n=512, max_nrhs=1, large_workers=1, batch_lanes=1, hbm_budget=budget)
    try:
        reqs = [(g.uniform(-1, 1, (512, 512)) + 512 * np.eye(512), g.uniform(-1, 1, (512, 1))) for _ in range(4)]
        ids = [s.submit(A, B) for A, B in reqs]
        # one worker and room for one request: the last one is still queued
        assert s.cancel(ids[-1][0]) == 0
        for rid, _ in ids[:-1]:
            assert s.wait(rid, 60.0)[0] == 0
        st, _ = s.wait(ids[-1][0], 1.0)
        assert st < 0
        assert s.stats()["cancelled"] == 1
    finally:
        s.close()


def test_destroy_with_queued_work_returns():
    g = philox(96)
    s = lmb200.Server(0, max_n=512, max_nrhs=1, large_workers=1, batch_lanes=1)
    for _ in range(6):
        s.submit(g.uniform(-1, 1, (512, 512)) + 512 * np.eye(512), g.uniform(-1, 1, (512, 1)))
    t0 = time.time()
    s.close()
    assert time.time() - t0 < 60.0
