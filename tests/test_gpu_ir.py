"""GPU tests of the mixed-precision path: FP32 LU with tcgen05 TF32 updates,
refined in FP64 (lm_dgesv_ir), for both factorisations: FP32 partial
pivoting (LM_IR_GEPP, the default) and the randomised butterfly +
no-pivoting factor (LM_IR_RBT, falling back to partial pivoting when
refinement stalls).  Bars: normwise backward error <= 1e-15 n (the target of the
FP64 path) and forward error against the FP64 oracle within what that
stopping rule allows: 8 kappa * 1e-15 n (plus the 1e-12 floor of the FP64
path)."""
import numpy as np
import pytest
import torch

import lmb200
import oracle as O
from conftest import philox
from helpers import backward_error, gen_randsvd, rel_forward

pytestmark = pytest.mark.gpu
EPS = 2.220446049250313e-16


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


@pytest.fixture(params=[lmb200.IR_RBT, lmb200.IR_GEPP], ids=["rbt", "gepp"])
def ir_method(request, ctx):
    ctx.set_ir_method(request.param)
    yield request.param
    ctx.set_ir_method(lmb200.IR_GEPP)


def sigma_spectrum(g, n, kappa, reflectors=4):
    """A = U diag(sigma) V^T with U, V products of Householder reflectors and
    sigma geometric from 1 to 1/kappa (the mixed-precision benchmark class)."""
    A = np.diag(kappa ** (-np.arange(n) / max(n - 1, 1)))
    for _ in range(reflectors):
        v = g.standard_normal(n)
        v /= np.linalg.norm(v)
        A -= 2.0 * np.outer(v, v @ A)
    for _ in range(reflectors):
        v = g.standard_normal(n)
        v /= np.linalg.norm(v)
        A -= 2.0 * np.outer(A @ v, v)
    return A


@pytest.mark.parametrize("n,kappa", [(1, 1.0), (7, 10.0), (64, 1e2), (130, 1e2), (257, 1e3), (1000, 1e2),
                                     (1000, 1e3), (2048, 1e2)])
def test_ir_converges_to_fp64_accuracy(ctx, ir_method, n, kappa):
    g = philox(9000 + n + int(np.log10(kappa)))
    A = gen_randsvd(g, n, kappa, -1.0, 1.0)
    b = g.uniform(-1, 1, n)
    x, iters, berr, st = lmb200.luSolveIR(dev(A), dev(b), ctx=ctx)
    x = x.cpu().numpy()
    assert st == 0, f"status {st}, {iters} iterations, berr {berr}"
    assert berr <= 1e-15 * n
    assert backward_error(A, x, b) <= 1e-15 * max(n, 1)
    xo, _, _ = O.lu_solve_p(A, b)
    assert rel_forward(x, xo) <= max(1e-12, 8 * kappa * 1e-15 * n)


def test_ir_multi_rhs_and_host_entry(ctx, ir_method):
    g = philox(9100)
    n, nrhs = 300, 5
    A = gen_randsvd(g, n, 1e2, -1.0, 1.0)
    B = g.uniform(-1, 1, (n, nrhs))
    X, iters, berr, st = lmb200.luSolveIR(dev(A), dev(B), ctx=ctx)
    assert st == 0 and berr <= 1e-15 * n
    Xo, _, _ = O.lu_solve_p(A, B)
    fwd_bar = max(1e-12, 8 * 1e2 * 1e-15 * n)  # kappa = 1e2
    assert rel_forward(X.cpu().numpy(), Xo) <= fwd_bar
    # host form
    import ctypes
    Xh = np.empty_like(B)
    it, be, info = ctypes.c_int(0), ctypes.c_double(0), ctypes.c_int(0)
    dp = lmb200._np_ptr
    A_c, B_c = np.ascontiguousarray(A), np.ascontiguousarray(B)
    s = lmb200.lib().lm_lu_solve_ir_host(ctx.h, n, nrhs, dp(A_c), dp(B_c), dp(Xh), 0.0, 30, ctypes.byref(it),
                                         ctypes.byref(be), ctypes.byref(info))
    assert s == 0 and be.value <= 1e-15 * n
    assert rel_forward(Xh, Xo) <= fwd_bar


def test_ir_uniform_matrix(ctx, ir_method):
    """The FP64 workload's matrix class (uniform[-1,1]) through the refinement path."""
    g = philox(9200)
    n = 1024
    A, b = g.uniform(-1, 1, (n, n)), g.uniform(-1, 1, n)
    x, iters, berr, st = lmb200.luSolveIR(dev(A), dev(b), ctx=ctx)
    assert st == 0 and berr <= 1e-15 * n
    assert backward_error(A, x.cpu().numpy(), b) <= 1e-15 * n


@pytest.mark.parametrize("n,nrhs", [(65, 2), (1000, 3), (4097, 4), (4100, 1)])
def test_ir_few_rhs_persistent_substitution(ctx, ir_method, n, nrhs):
    """nrhs <= 4 runs the substitutions as one persistent launch per direction
    (64-row blocks with inverted diagonal blocks); ragged last blocks included."""
    g = philox(9300 + n + nrhs)
    A = gen_randsvd(g, n, 1e2, -1.0, 1.0)
    B = g.uniform(-1, 1, (n, nrhs))
    X, iters, berr, st = lmb200.luSolveIR(dev(A), dev(B), ctx=ctx)
    assert st == 0 and berr <= 1e-15 * n, f"status {st}, {iters} iterations, berr {berr}"
    Xn = X.cpu().numpy()
    assert backward_error(A, Xn, B) <= 1e-15 * n
    Xo, _, _ = O.lu_solve_p(A, B)
    assert rel_forward(Xn, Xo) <= max(1e-12, 8 * 1e2 * 1e-15 * n)


@pytest.mark.parametrize("n,kappa", [(4096, 1e2), (4096, 1e4), (4096, 1e6), (8192, 1e2), (8192, 1e4),
                                     (8192, 1e6)])
def test_ir_dense_randsvd_vs_oracle(ctx, n, kappa):
    """The mixed-precision workload's matrix class: A = U diag(sigma) V^T with
    U, V dense random orthogonal (the reference's randsvd,
    test/Test/Types.hs:196-213), through the default method (FP32 partial
    pivoting), which must answer by itself, against the oracle's luSolveP."""
    O.set_threads(0)
    g = philox(9700 + n + int(np.log10(kappa)))
    A = gen_randsvd(g, n, kappa)
    b = g.uniform(-1, 1, n)
    x, iters, berr, st = lmb200.luSolveIR(dev(A), dev(b), ctx=ctx)
    assert st == 0 and berr <= 1e-15 * n, f"status {st}, {iters} iterations, berr {berr}"
    assert ctx.ir_last_method() == lmb200.IR_GEPP
    assert iters <= 12, f"{iters} refinement steps"
    xn = x.cpu().numpy()
    assert backward_error(A, xn, b) <= 1e-15 * n
    xo, _, _ = O.lu_solve_p(A, b)
    assert rel_forward(xn, xo) <= max(1e-12, 8 * kappa * 1e-15 * n)


@pytest.mark.parametrize("n,kappa", [(1024, 1e6), (2051, 1e4), (4096, 1e6)])
def test_ir_sigma_spectrum_rbt_path(ctx, n, kappa):
    """The nearly diagonal class (4 reflectors per side) through the randomised
    method: it must converge by itself (no fallback) to the FP64 bar."""
    g = philox(9400 + n)
    A = sigma_spectrum(g, n, kappa)
    b = g.uniform(-1, 1, n)
    ctx.set_ir_method(lmb200.IR_RBT)
    try:
        x, iters, berr, st = lmb200.luSolveIR(dev(A), dev(b), ctx=ctx)
        assert st == 0 and berr <= 1e-15 * n, f"status {st}, {iters} iterations, berr {berr}"
        assert ctx.ir_last_method() == lmb200.IR_RBT
    finally:
        ctx.set_ir_method(lmb200.IR_GEPP)
    xn = x.cpu().numpy()
    assert backward_error(A, xn, b) <= 1e-15 * n
    xo = np.linalg.solve(A, b)
    assert rel_forward(xn, xo) <= max(1e-12, 8 * kappa * 1e-15 * n)


def test_ir_fallback_to_partial_pivoting(ctx):
    """A condition number beyond FP32 preconditioning: the randomised factor
    stalls, the solve is redone with partial pivoting, and the status of that
    method (not converged) is what the caller sees."""
    g = philox(9500)
    n = 256
    A = gen_randsvd(g, n, 1e13, -1.0, 1.0)
    b = g.uniform(-1, 1, n)
    ctx.set_ir_method(lmb200.IR_RBT)
    try:
        x, iters, berr, st = lmb200.luSolveIR(dev(A), dev(b), ctx=ctx, max_iter=6)
    finally:
        ctx.set_ir_method(lmb200.IR_GEPP)
    assert st == lmb200.LM_ERR_NOT_CONVERGED
    assert ctx.ir_last_method() == lmb200.IR_GEPP
    ctx.check()


def test_ir_rbt_bitwise_repeatable(ctx):
    """The butterflies are seeded deterministically: two solves of the same
    system give the same bits (graph replay included)."""
    g = philox(9600)
    n = 700
    A = dev(sigma_spectrum(g, n, 1e3))
    b = dev(g.uniform(-1, 1, n))
    ctx.set_ir_method(lmb200.IR_RBT)
    try:
        xs = [lmb200.luSolveIR(A, b, ctx=ctx)[0].cpu().numpy() for _ in range(3)]
        assert ctx.ir_last_method() == lmb200.IR_RBT
    finally:
        ctx.set_ir_method(lmb200.IR_GEPP)
    assert np.array_equal(xs[0], xs[1]) and np.array_equal(xs[1], xs[2])


def test_ir_gepp_bitwise_repeatable(ctx):
    """Partial pivoting with look-ahead: the same system gives the same bits
    on every solve (eager first call, captured graph, replays)."""
    g = philox(9601)
    n = 2500
    A = dev(gen_randsvd(g, n, 1e5))
    b = dev(g.uniform(-1, 1, n))
    xs = [lmb200.luSolveIR(A, b, ctx=ctx)[0].cpu().numpy() for _ in range(3)]
    assert ctx.ir_last_method() == lmb200.IR_GEPP
    assert np.array_equal(xs[0], xs[1]) and np.array_equal(xs[1], xs[2])


@pytest.mark.parametrize("where", ["matrix", "rhs"])
def test_ir_never_reports_nan_as_converged(ctx, ir_method, where):
    """A NaN in the data makes every iterate NaN; the stopping test must see
    that as not converged (the max-abs reductions return NaN, and a NaN
    denominator once read as a zero backward error)."""
    g = philox(9700)
    n = 300
    A = gen_randsvd(g, n, 1e2, -1.0, 1.0)
    b = g.uniform(-1, 1, n)
    if where == "matrix":
        A[17, 5] = np.nan
    else:
        b[3] = np.nan
    x, iters, berr, st = lmb200.luSolveIR(dev(A), dev(b), ctx=ctx, max_iter=5)
    assert st != 0
    assert not (berr <= 1e-15 * n)
    for prec in (lmb200.IR_PREC_TF32, lmb200.IR_PREC_BF16):
        x, iters, berr, st = lmb200.luSolveIRPrec(dev(A), dev(b), prec=prec, ctx=ctx, max_iter=2)
        assert st != 0
    ctx.check()
