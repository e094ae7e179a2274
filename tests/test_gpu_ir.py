"""GPU tests of the mixed-precision path: FP32 LU with tcgen05 TF32 updates,
refined in FP64 (lm_dgesv_ir).  Bars: normwise backward error <= 1e-15 n
(the target of the FP64 path) and forward error against the FP64 oracle
within what that stopping rule allows: 8 kappa * 1e-15 n (plus the 1e-12
floor of the FP64 path)."""
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


@pytest.mark.parametrize("n,kappa", [(1, 1.0), (7, 10.0), (64, 1e2), (130, 1e2), (257, 1e3), (1000, 1e2),
                                     (1000, 1e3), (2048, 1e2)])
def test_ir_converges_to_fp64_accuracy(ctx, n, kappa):
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


def test_ir_multi_rhs_and_host_entry(ctx):
    g = philox(9100)
    n, nrhs = 300, 5
    A = gen_randsvd(g, n, 1e2, -1.0, 1.0)
    B = g.uniform(-1, 1, (n, nrhs))
    X, iters, berr, st = lmb200.luSolveIR(dev(A), dev(B), ctx=ctx)
    assert st == 0 and berr <= 1e-15 * n
    Xo, _, _ = O.lu_solve_p(A, B)
    assert rel_forward(X.cpu().numpy(), Xo) <= 1e-11
    # host form
    import ctypes
    Xh = np.empty_like(B)
    it, be, info = ctypes.c_int(0), ctypes.c_double(0), ctypes.c_int(0)
    dp = lmb200._np_ptr
    A_c, B_c = np.ascontiguousarray(A), np.ascontiguousarray(B)
    s = lmb200.lib().lm_lu_solve_ir_host(ctx.h, n, nrhs, dp(A_c), dp(B_c), dp(Xh), 0.0, 30, ctypes.byref(it),
                                         ctypes.byref(be), ctypes.byref(info))
    assert s == 0 and be.value <= 1e-15 * n
    assert rel_forward(Xh, Xo) <= 1e-11


def test_ir_uniform_matrix(ctx):
    """The FP64 workload's matrix class (uniform[-1,1]) through the refinement path."""
    g = philox(9200)
    n = 1024
    A, b = g.uniform(-1, 1, (n, n)), g.uniform(-1, 1, n)
    x, iters, berr, st = lmb200.luSolveIR(dev(A), dev(b), ctx=ctx)
    assert st == 0 and berr <= 1e-15 * n
    assert backward_error(A, x.cpu().numpy(), b) <= 1e-15 * n


@pytest.mark.parametrize("n,nrhs", [(65, 2), (1000, 3), (4097, 4), (4100, 1)])
def test_ir_few_rhs_persistent_substitution(ctx, n, nrhs):
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
