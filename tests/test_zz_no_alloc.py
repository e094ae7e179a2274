"""lm_dpotrf_noalloc: the Cholesky factorisation for callers that cannot
allocate device memory at call time (a memory-pool-owned runtime, a real-time
loop that forbids allocation, a plugin host with pre-registered buffers only).
Its scratch is a static device array inside the library, shared by every
call.  Checked against the allocating entry point lm_dpotrf on two calls in a
row, against the oracle over a sequence that leaves a failed factorisation's
contents in the shared array, and for its size and alignment limits.
Collected last on purpose: a run that stops at the first failure has run every
other test by then."""
import ctypes

import numpy as np
import pytest
import torch

import lmb200
import oracle as O
from conftest import philox
from helpers import gen_spd

pytestmark = pytest.mark.gpu


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _noalloc(A):
    info = ctypes.c_int(-1)
    n = A.shape[0] if A is not None else 0
    ptr = lmb200._ptr(A) if A is not None else None
    ld = A.stride(0) if A is not None else 0
    st = lmb200.lib().lm_dpotrf_noalloc(_stream(), n, ptr, ld, ctypes.byref(info))
    return st, info.value


def _even_ld(A):
    """A device copy of A with an even leading dimension."""
    n = A.shape[0]
    ld = n + (n & 1)
    d = torch.zeros((n, ld), dtype=torch.float64, device="cuda")[:, :n]
    d.copy_(torch.from_numpy(A))
    torch.cuda.synchronize()
    return d


def test_noalloc_warm_up_call():
    # n = 0 only looks up the static array's address on this device
    assert _noalloc(None) == (0, 0)


@pytest.mark.parametrize("n", [100, 777])
def test_noalloc_matches_allocating_entry_two_calls(n):
    ctx = lmb200.default_context(0)
    for call in range(2):
        A = gen_spd(philox(31000 + 10 * n + call), n)
        ref = torch.from_numpy(A).cuda()
        assert lmb200.dpotrf(ref, ctx) == 0
        got = _even_ld(A)
        st, info = _noalloc(got)
        assert st == 0 and info == 0
        G, Gref = got.cpu().numpy(), ref.cpu().numpy()
        assert np.all(np.triu(G, 1) == 0.0)
        assert np.abs(G - Gref).max() <= 1e-13 * np.abs(Gref).max()


def test_noalloc_sequence_vs_oracle():
    """n = 777, then a factorisation that fails (info > 0) and leaves its
    partial state in the shared array, then n = 100: each result against the
    oracle's choleskySolveP factor."""
    A1 = gen_spd(philox(31500), 777)
    d1 = _even_ld(A1)
    assert _noalloc(d1) == (0, 0)
    G1 = d1.cpu().numpy()
    assert np.abs(G1 - np.tril(O.chol_factor_p(A1))).max() <= 1e-13 * np.abs(G1).max()
    bad = gen_spd(philox(31501), 300)
    bad[200, 200] = -1e6  # not positive definite: the leading 201 x 201 block is indefinite
    st, info = _noalloc(_even_ld(bad))
    assert st == info and 0 < info <= 201
    A3 = gen_spd(philox(31502), 100)
    d3 = _even_ld(A3)
    assert _noalloc(d3) == (0, 0)
    G3 = d3.cpu().numpy()
    assert np.all(np.triu(G3, 1) == 0.0)
    assert np.abs(G3 - np.tril(O.chol_factor_p(A3))).max() <= 1e-13 * np.abs(G3).max()


def test_noalloc_reports_info_and_limits():
    A = np.eye(6)
    A[4, 4] = -1.0
    d = torch.from_numpy(A).cuda()
    st, info = _noalloc(d)
    assert st == 5 and info == 5            # first non-positive diagonal, 1-based
    big = torch.zeros((4100, 4100), dtype=torch.float64, device="cuda")
    st, _ = _noalloc(big)
    assert st == lmb200.LM_ERR_ARG           # beyond the static scratch
    odd = torch.zeros((10, 11), dtype=torch.float64, device="cuda")[:, :9]
    odd9 = odd[:9]
    st, _ = _noalloc(odd9)
    assert st == lmb200.LM_ERR_UNSUPPORTED   # odd leading dimension
