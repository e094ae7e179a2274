"""Low-precision factors with GMRES-IR (lm_dgesv_ir_prec): partial-pivoting LU
whose trailing updates run as one TF32 or one BF16 tensor-core product,
refined by GMRES-IR to FP64 accuracy.  Same bars as the other refinement
tests: normwise backward error <= 1e-15 n, forward error against the oracle's
luSolveP within 8 kappa 1e-15 n (with the FP64 path's 1e-12 floor).  The
3xTF32 mode through this entry point gives the same bits as lm_dgesv_ir's
partial-pivoting method."""
import numpy as np
import pytest
import torch

import lmb200
import oracle as O
from conftest import philox
from helpers import backward_error, gen_randsvd, rel_forward

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


@pytest.mark.parametrize("prec,n,kappa", [
    (lmb200.IR_PREC_TF32, 300, 1e2), (lmb200.IR_PREC_TF32, 1000, 1e3), (lmb200.IR_PREC_TF32, 2048, 1e4),
    (lmb200.IR_PREC_TF32, 4096, 1e3),
    (lmb200.IR_PREC_BF16, 64, 1e1), (lmb200.IR_PREC_BF16, 300, 1e2), (lmb200.IR_PREC_BF16, 1000, 1e2),
    (lmb200.IR_PREC_BF16, 2048, 1e3), (lmb200.IR_PREC_BF16, 4096, 1e2)])
def test_low_precision_gmres_ir_vs_oracle(ctx, prec, n, kappa):
    g = philox(40000 + n + int(np.log10(kappa)) + 10 * prec)
    A = gen_randsvd(g, n, kappa)
    b = g.uniform(-1, 1, n)
    x, outer, berr, st = lmb200.luSolveIRPrec(dev(A), dev(b), prec, ctx=ctx)
    assert st == 0 and berr <= 1e-15 * n, f"status {st}, {outer} corrections, berr {berr}"
    xn = x.cpu().numpy()
    assert backward_error(A, xn, b) <= 1e-15 * n
    xo, _, _ = O.lu_solve_p(A, b)
    assert rel_forward(xn, xo) <= max(1e-12, 8 * kappa * 1e-15 * n)


def test_low_precision_multi_rhs(ctx):
    g = philox(40100)
    n, nrhs = 777, 5
    A = gen_randsvd(g, n, 1e2)
    B = g.uniform(-1, 1, (n, nrhs))
    for prec in (lmb200.IR_PREC_TF32, lmb200.IR_PREC_BF16):
        X, outer, berr, st = lmb200.luSolveIRPrec(dev(A), dev(B), prec, ctx=ctx)
        assert st == 0 and berr <= 1e-15 * n
        Xn = X.cpu().numpy()
        Xo, _, _ = O.lu_solve_p(A, B)
        for c in range(nrhs):
            assert backward_error(A, Xn[:, c], B[:, c]) <= 1e-15 * n
            assert rel_forward(Xn[:, c], Xo[:, c]) <= max(1e-12, 8 * 1e2 * 1e-15 * n)


def test_tf32x3_mode_matches_default_entry(ctx):
    g = philox(40200)
    n = 1500
    A = dev(gen_randsvd(g, n, 1e4))
    b = dev(g.uniform(-1, 1, n))
    ctx.set_ir_method(lmb200.IR_GEPP)
    x1 = lmb200.luSolveIR(A, b, ctx=ctx)[0].cpu().numpy()
    x2, _, _, st = lmb200.luSolveIRPrec(A, b, lmb200.IR_PREC_TF32X3, ctx=ctx)
    assert st == 0 and np.array_equal(x1, x2.cpu().numpy())


def test_prec_argument_checked(ctx):
    g = philox(40300)
    A = dev(gen_randsvd(g, 50, 1e1))
    b = dev(g.uniform(-1, 1, 50))
    with pytest.raises(lmb200.LMError):
        lmb200.luSolveIRPrec(A, b, 7, ctx=ctx)
