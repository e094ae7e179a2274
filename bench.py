#!/usr/bin/env python
"""Benchmark of the B200 dense-solve path (one JSON line on rank 0).

Workloads (--workload):
  lu    luSolve, A n x n i.i.d. uniform[-1,1] (numpy Philox, seeded),
        b uniform[-1,1], nrhs right-hand sides; one step = copy A into the
        work buffer (luSolveP's thaw), LU with partial pivoting, solve.
  chol  choleskySolve with A = B B^T + n I, B uniform[-1,1].
  gemm  C = A B, m = n = k.
  ir    (default) mixed precision: FP32 LU with partial pivoting and
        tcgen05 3xTF32 updates, refined in FP64 to the normwise backward error
        1e-15 n; A = U diag(sigma) V^T with U, V dense random orthogonal (Q
        factors of seeded Gaussian matrices; --reflectors k > 0 uses k seeded
        Householder reflectors per side instead) and sigma geometric from 1 to
        1/kappa (--kappa; 0 = uniform[-1,1] A).  The plain FP64 LU solve of the same system is timed
        beside it (the metric's comparison).
The timed region replays the solve's captured CUDA graphs; per-kernel CUDA
events (the roofline's kernel time and the phase breakdown) come from
--profile-steps extra steps after it.
Metric: FP64-accurate solves per second (GEMMs per second for gemm), whole
job.  Multi-GPU: replicas only — every rank solves its own system, no
collective on the data path; value = all solves / max-over-ranks time.

--impl reference times the reference algorithm's CPU implementation (the
oracle restatement of luSolveP / choleskySolveP / matMulP; linear-massiv is
Haskell and no GHC exists here) on the host cores, as independent solves on
every hardware thread, on a bounded-size sample scaled to the workload's n by
the n^3 flop count.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "linear-massiv_b200"))

FLOPS = {
    "lu": lambda n, r: 2.0 / 3.0 * n ** 3 + 2.0 * n * n * r,
    "chol": lambda n, r: 1.0 / 3.0 * n ** 3 + 2.0 * n * n * r,
    "gemm": lambda n, r: 2.0 * n ** 3,
    "ir": lambda n, r: 2.0 / 3.0 * n ** 3 + 2.0 * n * n * r,
}


def gemm_k(a):
    return a.k if a.k > 0 else a.n


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["lu", "chol", "gemm", "ir", "batch", "serve"], default="ir")
    p.add_argument("--rate", type=float, default=2000.0, help="serve: Poisson arrival rate (requests/s)")
    p.add_argument("--duration", type=float, default=60.0, help="serve: seconds of arrivals")
    p.add_argument("--pool", type=int, default=512,
                   help="serve: pregenerated systems (each of its own order, log-uniform)")
    p.add_argument("--max-n", type=int, default=4096, help="serve: largest order")
    p.add_argument("--workers", type=int, default=8, help="serve: concurrent large solves")
    p.add_argument("--lu-fp64-max-n", type=int, default=-1,
                   help="serve: largest general order solved by FP64 LU (default: the server's)")
    p.add_argument("--count", type=int, default=10000, help="batch: number of instances")
    p.add_argument("--precision", choices=["fp64", "ir"], default="fp64", help="batch: FP64 or FP32 + FP64 IR")
    p.add_argument("--tune", action="store_true", help="batch: autotune the panel widths before timing")
    p.add_argument("--kappa", type=float, default=1e6, help="ir: condition number of A (0 = uniform A)")
    p.add_argument("--ir-method", choices=["gepp", "rbt"], default="gepp",
                   help="ir: partial pivoting (default) or random butterflies without pivoting")
    p.add_argument("--prec", choices=["tf32x3", "tf32", "bf16"], default="tf32x3",
                   help="ir: precision of the factor's trailing updates (tf32 and bf16 are refined by GMRES-IR)")
    p.add_argument("--reflectors", type=int, default=0,
                   help="ir: Householder reflectors per side (0 = dense Haar-random orthogonal U, V)")
    p.add_argument("--n", type=int, default=16384)
    p.add_argument("--nrhs", type=int, default=1)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--cpu-full", action="store_true",
                   help="cpu_baseline: one oracle solve at the full n on every host thread instead of the "
                        "single-threaded n <= 2048 sample (minutes at n = 16384)")
    p.add_argument("--no-peak", action="store_true", help="skip the cuBLAS DGEMM peak measurement")
    p.add_argument("--k", type=int, default=0, help="gemm inner dimension (default n); k < n adds beta = 1")
    p.add_argument("--profile-steps", type=int, default=1,
                   help="steps run with per-kernel CUDA events after the timed region (0 = none)")
    return p.parse_args()


def workload_name(a):
    if a.workload == "serve":
        return (f"serving loop, Poisson arrivals at {a.rate:g} req/s for {a.duration:g} s, n log-uniform in "
                f"[16,{a.max_n}], nrhs in {{1,8,32}}, 70% general / 30% SPD, kappa log-uniform in [1e1,1e6] "
                f"(sigma-spectrum, 8 reflectors per side; {a.pool} pregenerated systems of continuous order), "
                f"large requests at padded bucket orders: FP64 LU up to n="
                f"{a.lu_fp64_max_n if a.lu_fp64_max_n >= 0 else 2048} and FP64 Cholesky (SPD), mixed-precision IR "
                f"with FP64 fallback above; small ones on the device-resident loop; HBM-budget admission")
    if a.workload == "batch":
        return (f"batched solves, {a.count} instances in one persistent launch, n uniform in [8,256], nrhs uniform "
                f"in [1,16], half SPD (B B^T + n I, Cholesky) half general (uniform[-1,1], LU), "
                f"{'FP64' if a.precision == 'fp64' else 'FP32 factor + FP64 refinement'}")
    if a.workload == "ir":
        if a.kappa <= 0:
            spec = "A uniform[-1,1]"
        elif a.reflectors <= 0:
            spec = (f"A = U diag(sigma) V^T, kappa={a.kappa:g}, U and V dense random orthogonal "
                    f"(Q of seeded Gaussian, n Householder reflectors each)")
        else:
            spec = f"A = U diag(sigma) V^T, kappa={a.kappa:g}, {a.reflectors} Householder reflectors per side"
        upd = {"tf32x3": "3xTF32 tcgen05 updates, FP64 refinement",
               "tf32": "1xTF32 tcgen05 trailing updates, FP64 GMRES-IR",
               "bf16": "BF16 tcgen05 trailing updates, FP64 GMRES-IR"}[a.prec]
        fac = ("FP32 LU with partial pivoting" if a.ir_method == "gepp" else
               "random butterflies + FP32 LU without pivoting (partial pivoting if refinement stalls)")
        return f"mixed-precision IR luSolve n={a.n} nrhs={a.nrhs}, {spec}, {fac} + {upd}"
    if a.workload == "lu":
        return f"luSolve FP64 n={a.n} nrhs={a.nrhs}, A uniform[-1,1]"
    if a.workload == "chol":
        return f"choleskySolve FP64 n={a.n} nrhs={a.nrhs}, A = B B^T + n I"
    if gemm_k(a) != a.n:
        return f"gemm FP64 m=n={a.n} k={gemm_k(a)} C += A B, uniform[-1,1]"
    return f"gemm FP64 m=n=k={a.n}, uniform[-1,1]"


def metric_name(a):
    return "FP64 GEMMs/s" if a.workload == "gemm" else "FP64-accurate solves/s"


# ---- batched uneven solves ----------------------------------------------------------------

def batch_inputs(a, rank, np):
    """Seeded instances: sizes, kinds and the packed A / B (host, float64)."""
    g = np.random.Generator(np.random.Philox(a.seed + 7919 * rank))
    cnt = a.count
    n = g.integers(8, 257, cnt).astype(np.int32)
    nrhs = g.integers(1, 17, cnt).astype(np.int32)
    kind = (np.arange(cnt) % 2).astype(np.int32)
    a_off = np.concatenate([[0], np.cumsum(n.astype(np.int64) ** 2)])
    b_off = np.concatenate([[0], np.cumsum(n.astype(np.int64) * nrhs)])
    A = np.empty(a_off[-1])
    for i in range(cnt):
        m = int(n[i])
        M = g.uniform(-1.0, 1.0, (m, m))
        if kind[i] == 1:
            M = M @ M.T + m * np.eye(m)
        A[a_off[i]:a_off[i + 1]] = M.ravel()
    B = g.uniform(-1.0, 1.0, b_off[-1])
    return n, nrhs, kind, A, B, a_off, b_off


def batch_flops(n, nrhs, kind):
    n = n.astype(np.float64) if hasattr(n, "astype") else n
    return float(((kind == 0) * (2.0 / 3.0) * n ** 3 + (kind == 1) * (1.0 / 3.0) * n ** 3 + 2.0 * n * n * nrhs).sum())


def run_batch(a, world, rank, local):
    import torch

    import lmb200

    torch.cuda.set_device(local)
    ctx = lmb200.Context(local)
    n, nrhs, kind, A, B, a_off, b_off = batch_inputs(a, rank, np)
    prec = lmb200.PREC_FP64 if a.precision == "fp64" else lmb200.PREC_FP32_IR
    tuned = None
    if a.tune:
        tuned = lmb200.batch_tune(prec, None, ctx)
    plan = lmb200.Batch(n, nrhs, kind, prec, ctx)
    A_h = torch.from_numpy(A).pin_memory()
    B_h = torch.from_numpy(B).pin_memory()
    A_d, B_d = A_h.cuda(), B_h.cuda()
    X_d = torch.empty_like(B_d)
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")  # 256 MB > L2

    def step():
        plan.solve(A_d, B_d, X_d, tol=0.0, max_iter=10)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    info, iters, berr = plan.results()
    # accuracy of the warm-up result on a sample of instances (host FP64)
    Xh = X_d.cpu().numpy()
    worst = 0.0
    for i in range(0, a.count, max(1, a.count // 200)):
        m, r = int(n[i]), int(nrhs[i])
        Ai = A[a_off[i]:a_off[i + 1]].reshape(m, m)
        Bi = B[b_off[i]:b_off[i + 1]].reshape(m, r)
        Xi = Xh[b_off[i]:b_off[i + 1]].reshape(m, r)
        res = np.abs(Ai @ Xi - Bi).max(axis=0)
        den = np.abs(Ai).sum(axis=1).max() * np.abs(Xi).max(axis=0) + np.abs(Bi).max(axis=0)
        worst = max(worst, float((res / den).max() / (1e-15 * m)))
    launches0 = lmb200.launch_count()
    clocks = Clocks(local)
    barrier(world)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    ms = []
    for _ in range(a.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        step()
        e1.record(st)
        ms.append((e0, e1))
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    t_local = sum(e0.elapsed_time(e1) for e0, e1 in ms) * 1e-3
    launches = lmb200.launch_count() - launches0
    t = max_over_ranks(t_local, world)
    value = world * a.count * a.steps / t
    flops = batch_flops(n, nrhs, kind)
    peak = measure_fp64_peak(torch) if (rank == 0 and not a.no_peak) else None
    achieved = flops * a.steps / t_local / 1e12
    # e2e: host (pinned) buffers through lm_batch_solve_host
    Xp = torch.empty_like(B_h).pin_memory()
    P = lmb200._np_ptr
    lib = lmb200.lib()

    def e2e_step():
        stt = lib.lm_batch_solve_host(plan.h, P(A_h.numpy()), P(B_h.numpy()), P(Xp.numpy()), 0.0, 10)
        if stt < 0:
            raise lmb200.LMError(stt, "lm_batch_solve_host")

    e2e_val = None
    if a.e2e_steps > 0:
        e2e_step()
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(a.e2e_steps):
            e2e_step()
        e2e_val = world * a.count * a.e2e_steps / max_over_ranks(time.perf_counter() - t0, world)
    if rank != 0:
        return
    nb = lmb200.batch_tune_get(ctx)
    line = {
        "metric": metric_name(a), "value": value, "unit": metric_name(a), "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * t / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if a.precision == "fp64" else "f32 factor / f64 refinement",
        "data": "synthetic (seeded numpy Philox)",
        "config": {"workload": workload_name(a), "count": a.count, "parallelism": f"replicas x{world}",
                   "l2": "256 MB buffer written between timed steps (L2 flush)",
                   "panel_width_per_bucket": nb[prec], "autotuned": bool(a.tune)},
        "gpu_launches": launches,
        "e2e": {"value": e2e_val, "unit": metric_name(a), "h2d_bytes_per_step": int(A.nbytes + B.nbytes),
                "d2h_bytes_per_step": int(B.nbytes), "steps": a.e2e_steps, "api": "lm_batch_solve_host"},
        "roofline": {"bound": "fp64", "kernel": "batch_kernel (persistent, one CTA per instance)",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": (achieved / peak) if peak else None, "traffic": None,
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 peak; MEASURED_PEAKS.json has no FP64)",
                     "algorithmic_flops_per_step": flops},
        "tflops_whole_step": flops * a.steps / t / 1e12,
        "accuracy": {"worst_backward_error_over_1e-15n": worst, "sampled_instances": len(range(0, a.count, max(1, a.count // 200))),
                     "info_nonzero": int((info != 0).sum()), "fp64_fallbacks": int((iters < 0).sum()),
                     "mean_corrections": float(iters[iters >= 0].mean()) if (iters >= 0).any() else None},
        "clocks": clk,
    }
    if world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_batch(a, n, nrhs, kind, A, B, a_off, b_off)
    print(json.dumps(line), flush=True)


def serve_pool(a, torch):
    """Pregenerated request systems: (A pinned, kind, kappa), n drawn continuously
    log-uniform in [16, max_n] (so almost every system has its own order), A =
    U diag(sigma) V^T with U, V products of 8 seeded Householder reflectors and
    sigma geometric from 1 to 1/kappa (V = U for SPD requests)."""
    g = np.random.Generator(np.random.Philox(a.seed + 4242))
    pool = []
    for _ in range(a.pool):
        n = int(np.exp(g.uniform(np.log(16), np.log(a.max_n + 1))))
        n = max(16, min(n, a.max_n))
        spd = g.uniform() < 0.3
        kappa = float(np.exp(g.uniform(np.log(1e1), np.log(1e6))))
        s = torch.from_numpy(kappa ** (-np.arange(n) / max(n - 1, 1))).cuda()

        def reflectors():
            Q = torch.eye(n, dtype=torch.float64, device="cuda")
            for _ in range(8):
                v = torch.from_numpy(g.standard_normal(n)).cuda()
                v /= torch.linalg.norm(v)
                Q -= 2.0 * torch.outer(v, v @ Q)
            return Q

        U = reflectors()
        V = U if spd else reflectors()
        A = ((U * s) @ V.T).cpu().pin_memory()
        pool.append((A, 1 if spd else 0, kappa))
    return pool


def run_serve(a, world, rank, local):
    import torch

    import lmb200

    torch.cuda.set_device(local)
    pool = serve_pool(a, torch)
    g = np.random.Generator(np.random.Philox(a.seed + 99 + 7919 * rank))
    rhs = {r: torch.from_numpy(g.uniform(-1.0, 1.0, (a.max_n, r))).pin_memory() for r in (1, 8, 32)}
    free_b, _ = torch.cuda.mem_get_info()
    route = {} if a.lu_fp64_max_n < 0 else {"lu_fp64_max_n": a.lu_fp64_max_n}
    srv = lmb200.Server(local, max_n=a.max_n, max_nrhs=32, large_workers=a.workers, batch_lanes=2,
                        hbm_budget=int(min(free_b // 3, 48 << 30)), **route)
    # arrival schedule and request draws (seeded, fixed before the run)
    total = int(a.rate * a.duration)
    gaps = g.exponential(1.0 / a.rate, total)
    picks = g.integers(0, len(pool), total)
    nrhs_of = g.choice([1, 8, 32], total)
    nmax_pool = max(p[0].shape[0] for p in pool)
    # output buffers are recycled round-robin: the timed requests' solutions
    # are not read (accuracy is checked on separate requests below)
    outs = [torch.empty((nmax_pool, 32), dtype=torch.float64).pin_memory() for _ in range(64)]

    def submit_sys(j, r, out):
        A, kind, _ = pool[j]
        n = A.shape[0]
        return srv.submit_raw(n, r, kind, A.data_ptr(), rhs[r].data_ptr(), out.data_ptr())

    def submit(i, out):
        return submit_sys(int(picks[i]), int(nrhs_of[i]), out)

    # warm-up (untimed): every pool system with each right-hand-side count, in
    # two bursts, so that every worker sees the order buckets twice (the first
    # run of a launch sequence is eager, the second is captured as a graph)
    for _ in range(2):
        k = 0
        for j in range(len(pool)):
            for r in (1, 8, 32):
                submit_sys(j, r, outs[k % 64])
                k += 1
        srv.drain(600.0)
    srv.reset_stats()
    clocks = Clocks(local)
    launches0 = lmb200.launch_count()
    ids = []
    t0 = time.perf_counter()
    t_next = t0
    k = 0
    for i in range(total):
        t_next += gaps[i]
        while True:
            d = t_next - time.perf_counter()
            if d <= 0:
                break
            if d > 2e-4:
                time.sleep(d - 1e-4)
        ids.append(submit(i, outs[k]))
        k = (k + 1) % 64
    t_arrivals = time.perf_counter() - t0
    drained = True
    try:
        srv.drain(max(120.0, 2 * a.duration))
    except Exception:
        drained = False
    clk = clocks.stop()
    st = srv.stats()
    launches = lmb200.launch_count() - launches0
    # accuracy on a sample: re-solve a few pool systems through the server and check on the host
    worst = 0.0
    for j in range(min(len(pool), 12)):
        A, kind, _ = pool[j]
        n = A.shape[0]
        out = torch.empty((n, 8), dtype=torch.float64).pin_memory()
        rid = srv.submit_raw(n, 8, kind, A.data_ptr(), rhs[8].data_ptr(), out.data_ptr())
        srv.wait(rid, 120.0)
        An, Xn, Bn = A.numpy(), out.numpy(), rhs[8].numpy().ravel()[:n * 8].reshape(n, 8)
        r = np.abs(An @ Xn - Bn).max(axis=0)
        den = np.abs(An).sum(axis=1).max() * np.abs(Xn).max(axis=0) + np.abs(Bn).max(axis=0)
        worst = max(worst, float((r / den).max() / (1e-15 * n)))
    srv.close()
    if rank != 0:
        return
    value = st["solves_per_s"] * world
    line = {
        "metric": "FP64-accurate solves/s (serving) with p50/p99 latency", "value": value,
        "unit": "FP64-accurate solves/s", "n_gpus": world, "steps": total, "warmup": len(pool),
        "ms_per_step": 1e3 / value if value else None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 factor / f64 refinement (large), f64 (batched small)",
        "data": "synthetic (seeded numpy Philox; sigma-spectrum systems)",
        "config": {"workload": workload_name(a), "parallelism": f"replicas x{world}",
                   "arrivals_offered": total, "arrival_window_s": t_arrivals, "drained": drained,
                   "l2": "inputs far larger than L2 across the pool"},
        "latency_ms": {"p50": st["p50_ms"], "p99": st["p99_ms"], "mean": st["mean_ms"], "max": st["max_ms"]},
        "serving": {k2: st[k2] for k2 in ("completed", "rejected", "failed", "fp64_fallbacks", "queue_peak",
                                          "inflight_peak", "micro_batches", "small_solved", "arena_bytes",
                                          "arena_peak_bytes", "fixed_bytes", "span_s", "tflops", "ir_solves",
                                          "ir_gepp", "ir_iterations")},
        "gpu_launches": launches,
        "e2e": {"value": value, "unit": "FP64-accurate solves/s", "api": "lm_server_submit / lm_server_drain",
                "note": "every request is host-to-host: A, B copied in and X copied out inside its latency"},
        "accuracy": {"worst_backward_error_over_1e-15n": worst, "sampled_systems": min(len(pool), 12)},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_batch(a, n, nrhs, kind, A, B, a_off, b_off):
    """Oracle luSolveP / choleskySolveP on the leading instances for about 10 s, one thread."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    t0 = time.perf_counter()
    done = 0
    for i in range(a.count):
        m, r = int(n[i]), int(nrhs[i])
        Ai = A[a_off[i]:a_off[i + 1]].reshape(m, m)
        Bi = B[b_off[i]:b_off[i + 1]].reshape(m, r)
        if kind[i] == 0:
            O.lu_solve_p(Ai, Bi)
        else:
            O.chol_solve_p(Ai, Bi)
        done += 1
        if time.perf_counter() - t0 > 10.0:
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "FP64-accurate solves/s", "cores": 1, "kind": "port",
            "sample": f"the first {done} instances of the same batch solved one by one by the oracle "
                      f"(luSolveP / choleskySolveP restatement) on one host thread in {dt:.1f} s"}


# ---- clocks sampled during the timed region ----------------------------------------

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(gpu_index)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit()),
                "reasons": reasons, "samples": len(rows)}


# ---- distributed plumbing ------------------------------------------------------------

def dist_init(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if a.impl == "ours":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- inputs ---------------------------------------------------------------------------

def dense_randsvd_matrix(n, kappa, seed, torch):
    """A = U diag(sigma) V^T on the GPU (input preparation, not timed) with U, V
    dense Haar-random orthogonal: the Q factors of seeded Gaussian matrices, each
    a product of n Householder reflectors (the reference's randsvd construction,
    test/Test/Types.hs:196-213); sigma_i = kappa^(-i/(n-1))."""
    gen = torch.Generator(device="cuda")
    gen.manual_seed(int(seed))
    s = kappa ** (-torch.arange(n, dtype=torch.float64, device="cuda") / max(n - 1, 1))
    A = None
    for side in range(2):
        G = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=gen)
        Q, R = torch.linalg.qr(G)
        Q *= torch.sign(torch.diagonal(R)).unsqueeze(0)  # Haar measure
        del G, R
        if side == 0:
            A = Q * s.unsqueeze(0)   # U diag(sigma)
        else:
            A = A @ Q.T              # ... V^T
        del Q
    torch.cuda.empty_cache()
    return A.cpu()


def sigma_spectrum_matrix(n, kappa, reflectors, g, torch, np):
    """A = U diag(sigma) V^T on the GPU (input preparation, not timed): sigma_i =
    kappa^(-i/(n-1)), U and V products of `reflectors` seeded Householder
    reflectors (a nearly diagonal matrix for few reflectors)."""
    s = torch.from_numpy(kappa ** (-np.arange(n) / max(n - 1, 1))).cuda()
    A = torch.diag(s)
    for side in ("left", "right"):
        for _ in range(reflectors):
            v = torch.from_numpy(g.standard_normal(n)).cuda()
            v /= torch.linalg.norm(v)
            if side == "left":   # A <- (I - 2 v v^T) A
                A -= 2.0 * torch.outer(v, v @ A)
            else:                # A <- A (I - 2 v v^T)
                A -= 2.0 * torch.outer(A @ v, v)
    return A.cpu()


def make_inputs(a, rank, torch, np):
    g = np.random.Generator(np.random.Philox(a.seed + 7919 * rank))
    n = a.n
    if a.workload == "ir" and a.kappa > 0 and a.reflectors <= 0:
        A = dense_randsvd_matrix(n, a.kappa, a.seed + 7919 * rank, torch)
    elif a.workload == "ir" and a.kappa > 0:
        A = sigma_spectrum_matrix(n, a.kappa, a.reflectors, g, torch, np)
    else:
        A = torch.from_numpy(g.uniform(-1.0, 1.0, (n, n)))
    if a.workload == "chol":
        Bd = A.cuda()
        S = Bd @ Bd.T  # input preparation only (not timed)
        S.diagonal().add_(float(n))
        S = 0.5 * (S + S.T)
        A = S.cpu()
        del Bd, S
    if a.workload == "gemm" and gemm_k(a) != n:
        A = A[:, :gemm_k(a)].contiguous()
    B = torch.from_numpy(g.uniform(-1.0, 1.0, (gemm_k(a) if a.workload == "gemm" else n,
                                               a.nrhs if a.workload != "gemm" else n)))
    return A.pin_memory(), B.pin_memory()


def measure_fp64_peak(torch):
    """cuBLAS DGEMM 8192^3 throughput on this GPU (the FP64 roofline denominator)."""
    return _measure_peak(torch, torch.float64, False)


def measure_tf32_peak(torch):
    """cuBLAS FP32-storage GEMM with TF32 tensor cores, 8192^3 (the TF32 denominator)."""
    return _measure_peak(torch, torch.float32, True)


def _measure_peak(torch, dtype, tf32):
    n = 8192
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = tf32
    try:
        x = torch.rand((n, n), dtype=dtype, device="cuda")
        y = torch.rand((n, n), dtype=dtype, device="cuda")
        for _ in range(2):
            torch.matmul(x, y)
        best = 0.0
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(x, y)
            e1.record()
            torch.cuda.synchronize()
            best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3))
        del x, y
        torch.cuda.empty_cache()
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old
    return best / 1e12


def cpu_baseline(a):
    """Oracle luSolveP/choleskySolveP/matMulP single-threaded on a bounded sample."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    full = a.cpu_full and a.workload in ("lu", "ir", "chol")
    ns = a.n if full else min(a.n, 2048)
    threads = (os.cpu_count() or 1) if full else 1
    O.set_threads(threads)
    g = np.random.Generator(np.random.Philox(a.seed + 1))
    A = g.uniform(-1.0, 1.0, (ns, ns))
    b = g.uniform(-1.0, 1.0, ns)
    if a.workload == "chol":
        A = A @ A.T + ns * np.eye(ns)
    if full:
        # one solve of the full order; the oracle's trailing updates split
        # their rows over the threads (bitwise the same result as one thread)
        t0 = time.perf_counter()
        {"lu": O.lu_solve_p, "ir": O.lu_solve_p, "chol": O.chol_solve_p}[a.workload](A, b)
        dt = time.perf_counter() - t0
        O.set_threads(1)
        return {"value": 1.0 / dt, "unit": metric_name(a), "cores": threads, "kind": "port",
                "sample": f"one oracle solve at the full n={ns} ({dt:.2f} s) with its trailing updates split over "
                          f"{threads} host threads"}
    fn = {"lu": lambda: O.lu_solve_p(A, b), "ir": lambda: O.lu_solve_p(A, b), "chol": lambda: O.chol_solve_p(A, b),
          "gemm": lambda: O.matmul_p(A, A)}[a.workload]
    fn()
    t0 = time.perf_counter()
    reps = 0
    while True:
        fn()
        reps += 1
        if time.perf_counter() - t0 > 8.0 or reps >= 20:
            break
    dt = (time.perf_counter() - t0) / reps
    scale = FLOPS[a.workload](ns, 1) / FLOPS[a.workload](a.n, a.nrhs)
    return {"value": scale / dt, "unit": metric_name(a), "cores": 1, "kind": "port",
            "sample": f"{reps} single-threaded oracle solves at n={ns} ({dt:.3f} s each), scaled to n={a.n} "
                      f"by the flop count"}


# ---- the reference arm ------------------------------------------------------------------

def run_reference(a, world, rank):
    if rank != 0:
        return
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    threads = os.cpu_count() or 1
    ns = min(a.n, 2048)
    g = np.random.Generator(np.random.Philox(a.seed + 1))
    A = g.uniform(-1.0, 1.0, (ns, ns))
    b = g.uniform(-1.0, 1.0, ns)
    if a.workload == "chol":
        A = A @ A.T + ns * np.eye(ns)

    def step():
        if a.workload in ("lu", "ir"):
            O.lu_solve_p_many(A, b, threads, threads)
        elif a.workload == "chol":
            O.chol_solve_p_many(A, b, threads, threads)
        else:
            O.matmul_par(A, A, threads)

    for _ in range(a.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        step()
    dt = time.perf_counter() - t0
    per_step = threads if a.workload != "gemm" else 1
    scale = FLOPS[a.workload](ns, 1) / FLOPS[a.workload](a.n, a.nrhs)
    value = per_step * a.steps / dt * scale
    sample = (f"each step: {per_step} independent oracle {'solves' if per_step > 1 else 'GEMM (matMulPPar tiling)'} "
              f"at n={ns} on {threads} host threads; scaled to n={a.n} by the flop count")
    line = {"impl": "reference", "metric": metric_name(a), "value": value, "unit": metric_name(a),
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * dt / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded numpy Philox, uniform[-1,1])",
            "config": {"workload": workload_name(a), "n": a.n, "nrhs": a.nrhs, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (8 n^2 bytes per matrix)"},
            "cpu_baseline": {"value": value, "unit": metric_name(a), "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": metric_name(a), "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# DRAM bytes per algorithmic byte of the dominant kernel: dram__bytes_read.sum
# + dram__bytes_write.sum of one captured launch (ncu, one trailing update of
# the same kernel at n = 8192) divided by that launch's algorithmic bytes.  A
# run's per-launch traffic is this ratio times its own algorithmic bytes per
# launch (the traffic of these launches grows in proportion to their size).
DRAM_PER_ALGO_BYTE = {
    "dgemm": 1.11e9 / 1.090e9,
    "sgemm": 481.2e6 / 528.0e6,
}


def measured_hbm_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"


def traffic_per_launch(a, gp, steps):
    key = "dgemm" if a.workload in ("lu", "chol", "gemm") else "sgemm"
    if key is None or key not in DRAM_PER_ALGO_BYTE or not gp.get("launches"):
        return None
    return DRAM_PER_ALGO_BYTE[key] * gp["bytes"] / gp["launches"]


# ---- our arm ------------------------------------------------------------------------------

def run_ours(a, world, rank, local):
    import numpy as np
    import torch

    import lmb200

    torch.cuda.set_device(local)
    ctx = lmb200.Context(local)
    if a.workload == "ir":
        ctx.set_ir_method(lmb200.IR_RBT if a.ir_method == "rbt" else lmb200.IR_GEPP)
    lib = lmb200.lib()
    n, nrhs = a.n, a.nrhs
    A_h, B_h = make_inputs(a, rank, torch, np)
    A_d = A_h.cuda()
    B_d = B_h.cuda()
    work = torch.empty((n, n), dtype=torch.float64, device="cuda")
    X = torch.empty_like(B_d)
    ipiv = torch.empty(n, dtype=torch.int32, device="cuda")
    P = lmb200._ptr

    kk = gemm_k(a)

    ir_stats = {}

    def step():
        if a.workload == "ir":
            it, be, info = ctypes.c_int(0), ctypes.c_double(0.0), ctypes.c_int(0)
            if a.prec == "tf32x3":
                st = lib.lm_dgesv_ir(ctx.h, n, nrhs, P(A_d), n, P(B_d), nrhs, P(X), nrhs, 0.0, 50, ctypes.byref(it),
                                     ctypes.byref(be), ctypes.byref(info))
            else:
                pr = {"tf32": lmb200.IR_PREC_TF32, "bf16": lmb200.IR_PREC_BF16}[a.prec]
                st = lib.lm_dgesv_ir_prec(ctx.h, n, nrhs, P(A_d), n, P(B_d), nrhs, P(X), nrhs, pr, 0.0, 50,
                                          ctypes.byref(it), ctypes.byref(be), ctypes.byref(info))
            ir_stats["iters"] = it.value
            ir_stats["berr"] = be.value
            if st < 0:
                raise lmb200.LMError(st, "ir step")
            return
        if a.workload == "gemm":
            st = lib.lm_dgemm(ctx.h, n, n, kk, 1.0, P(A_d), kk, P(B_d), n, 1.0 if kk != n else 0.0, P(work), n)
        else:
            work.copy_(A_d)
            X.copy_(B_d)
            fn = lib.lm_dgesv if a.workload == "lu" else None
            if a.workload == "lu":
                st = fn(ctx.h, n, nrhs, P(work), n, P(ipiv), P(X), nrhs, None)
            else:
                st = lib.lm_dposv(ctx.h, n, nrhs, P(work), n, P(X), nrhs, None)
        if st < 0:
            raise lmb200.LMError(st, "bench step")

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    ctx.check()
    ir_method = ctx.ir_last_method() if a.workload == "ir" else None
    ir_hist = ctx.ir_history() if a.workload == "ir" else None
    # accuracy of the last warm-up result (FP64 backward error, checked on the GPU)
    accuracy = {}
    if a.workload != "gemm":
        R = B_d - A_d @ X
        num = R.abs().max().item()
        den = A_d.abs().sum(dim=1).max().item() * X.abs().max().item() + B_d.abs().max().item()
        accuracy = {"backward_error": num / den, "bound": 1e-15 * n}
        del R
    peak = None
    tf32_peak = None
    if rank == 0 and not a.no_peak:
        if a.workload == "ir":
            tf32_peak = measure_tf32_peak(torch)
        else:
            peak = measure_fp64_peak(torch)

    # Timed region: the captured CUDA graphs of the solve, no per-kernel events.
    launches0 = lmb200.launch_count()
    clocks = Clocks(local)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    th0 = time.perf_counter()
    for _ in range(a.steps):
        step()
    host_enqueue_ms = (time.perf_counter() - th0) * 1e3 / a.steps
    e1.record()
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    t_local = e0.elapsed_time(e1) * 1e-3
    launches = lmb200.launch_count() - launches0
    t = max_over_ranks(t_local, world)
    value = world * a.steps / t

    # Kernel breakdown: the same step with CUDA events around every kernel
    # group on the launching stream (eager launches), right after the timed
    # region.  The roofline's achieved rate is the dominant kernel's
    # algorithmic work divided by its event-timed duration here.
    phases = None
    prof_ms = None
    if a.profile_steps > 0:
        ctx.profile(True)
        ctx.profile_read()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record()
        for _ in range(a.profile_steps):
            step()
        p1.record()
        torch.cuda.synchronize()
        prof_ms = p0.elapsed_time(p1) / a.profile_steps
        phases = ctx.profile_read()
        ctx.profile(False)

    # IR: time the plain FP64 LU solve of the same system beside it
    fp64_ref = None
    if a.workload == "ir":
        def fp64_step():
            work.copy_(A_d)
            Xf.copy_(B_d)
            st = lib.lm_dgesv(ctx.h, n, nrhs, P(work), n, P(ipiv), P(Xf), nrhs, None)
            if st < 0:
                raise lmb200.LMError(st, "fp64 step")
        Xf = torch.empty_like(B_d)
        # three warm-up solves: a workspace that grows on the first one renews
        # the graph keys, so capture can happen as late as the third
        for _ in range(3):
            fp64_step()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        kf = max(3, a.steps // 2)
        for _ in range(kf):
            fp64_step()
        f1.record()
        torch.cuda.synchronize()
        tf = f0.elapsed_time(f1) * 1e-3 / kf
        R = B_d - A_d @ Xf
        be64 = R.abs().max().item() / (A_d.abs().sum(dim=1).max().item() * Xf.abs().max().item() +
                                      B_d.abs().max().item())
        fwd = ((X - Xf).abs().max() / Xf.abs().max()).item()
        fp64_ref = {"fp64_lu_solves_per_s": 1.0 / tf, "fp64_lu_ms": tf * 1e3, "fp64_backward_error": be64,
                    "ir_vs_fp64_speedup": (a.steps / t) / (1.0 / tf), "ir_vs_fp64_rel_diff": fwd}
        del R

    # e2e through the host-buffer entry point: H2D of A and B, solve, D2H of X
    Xh = torch.empty((n, n) if a.workload == "gemm" else tuple(B_h.shape), dtype=torch.float64).pin_memory()
    dp = lmb200._np_ptr

    def e2e_step():
        if a.workload == "ir":
            it, be, info = ctypes.c_int(0), ctypes.c_double(0.0), ctypes.c_int(0)
            st = lib.lm_lu_solve_ir_host(ctx.h, n, nrhs, dp(A_h.numpy()), dp(B_h.numpy()), dp(Xh.numpy()), 0.0, 50,
                                         ctypes.byref(it), ctypes.byref(be), ctypes.byref(info))
        elif a.workload == "lu":
            st = lib.lm_lu_solve_host(ctx.h, n, nrhs, dp(A_h.numpy()), dp(B_h.numpy()), dp(Xh.numpy()), None)
        elif a.workload == "chol":
            st = lib.lm_chol_solve_host(ctx.h, n, nrhs, dp(A_h.numpy()), dp(B_h.numpy()), dp(Xh.numpy()), None)
        else:
            st = lib.lm_matmul_host(ctx.h, n, n, kk, dp(A_h.numpy()), dp(B_h.numpy()), dp(Xh.numpy()))
        if st < 0:
            raise lmb200.LMError(st, "e2e step")

    e2e_val = None
    if a.e2e_steps > 0:
        e2e_step()
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(a.e2e_steps):
            e2e_step()
        t_e2e = max_over_ranks(time.perf_counter() - t0, world)
        e2e_val = world * a.e2e_steps / t_e2e
    h2d = A_h.numel() * 8 + B_h.numel() * 8
    d2h = Xh.numel() * 8

    if rank != 0:
        return
    ps = max(a.profile_steps, 1)
    gp = phases["gemm"] if phases else {"flops": 0.0, "ms": 0.0, "launches": 0, "bytes": 0.0}
    total_ms = sum(p["ms"] for p in phases.values()) if phases else 0.0
    extra = {}
    if a.workload == "ir":
        # 3xTF32 trailing updates: about 190 MMA flops per byte of C traffic at
        # k = 256, above the TF32 ridge, so the kernel is tensor-bound; the
        # algorithmic rate counts the logical 2 m n k of each product once,
        # the MMA-issue rate all three TF32 products
        roof_kernel = "sgemm_tf32_kernel (tcgen05 kind::tf32, 3xTF32 split: 3 MMAs per logical product)"
        bound, unit = "tensor", "TFLOP/s"
        mma = gp["flops"] / (gp["ms"] * 1e-3) / 1e12 if gp["ms"] > 0 else None
        achieved = mma / 3.0 if mma else None
        peak = tf32_peak
        peak_src = ("cuBLAS TF32 GEMM (FP32 storage, allow_tf32) 8192^3 measured in this run (MEASURED_PEAKS.json "
                    "has no TF32 figure)")
        hbm_peak, hbm_src = measured_hbm_gbs()
        gbs = gp["bytes"] / (gp["ms"] * 1e-3) / 1e9 if gp["ms"] > 0 else None
        extra = {"mma_issue_tflops": mma, "mma_issue_frac": (mma / peak) if (mma and peak) else None,
                 "hbm_gbs": gbs, "hbm_frac": (gbs / hbm_peak) if gbs else None, "hbm_peak_source": hbm_src}
    else:
        roof_kernel = "dgemm_dmma_kernel (FP64 DMMA)"
        bound, unit = "tensor", "TFLOP/s"
        achieved = gp["flops"] / (gp["ms"] * 1e-3) / 1e12 if gp["ms"] > 0 else None
        peak_src = "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64)"
    line = {
        "metric": metric_name(a), "value": value, "unit": metric_name(a), "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * t / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded numpy Philox, uniform[-1,1])",
        "config": {"workload": workload_name(a), "n": n, "nrhs": nrhs, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (8 n^2 bytes per matrix)"},
        "gpu_launches": launches,
        "e2e": {"value": e2e_val, "unit": metric_name(a), "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": a.e2e_steps, "api": {"lu": "lm_lu_solve_host", "chol": "lm_chol_solve_host", "gemm": "lm_matmul_host",
                                             "ir": "lm_lu_solve_ir_host"}[a.workload]},
        "roofline": {"bound": bound, "kernel": roof_kernel,
                     "achieved": achieved, "peak": peak, "unit": unit,
                     "frac": (achieved / peak) if (achieved and peak) else None,
                     "traffic": traffic_per_launch(a, gp, ps),
                     "peak_source": peak_src,
                     "launches_per_step": gp["launches"] / ps,
                     "timing": f"CUDA events around each launch of the kernel over {a.profile_steps} profiled "
                               f"step(s) run after the timed region ({prof_ms and round(prof_ms, 2)} ms per "
                               f"profiled step, eager launches)", **extra},
        "phases_ms_per_step": ({k: v["ms"] / ps for k, v in phases.items()} if phases else None),
        "phase_share": ({k: (v["ms"] / total_ms if total_ms else None) for k, v in phases.items()} if phases else None),
        "tflops_whole_step": (2.0 * n * n * kk if a.workload == "gemm" else FLOPS[a.workload](n, nrhs)) * a.steps / t / 1e12,
        "host_enqueue_ms_per_step": host_enqueue_ms,
        "accuracy": accuracy,
        "ir": ({**ir_stats, **(fp64_ref or {}), "method": {0: "rbt", 1: "gepp"}.get(ir_method, ir_method),
                "berr_history": ir_hist}
               if a.workload == "ir" else None),
        "clocks": clk,
    }
    if world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(a)
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    world, rank, local = dist_init(a)
    try:
        if a.impl == "reference":
            run_reference(a, world, rank)
        elif a.workload == "batch":
            run_batch(a, world, rank, local)
        elif a.workload == "serve":
            run_serve(a, world, rank, local)
        else:
            run_ours(a, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
