"""lm_dpotrf_noalloc: the Cholesky factorisation for callers that cannot
allocate device memory at call time (a memory-pool-owned runtime, a real-time
loop that forbids allocation, a plugin host with pre-registered buffers only).
Its scratch is a static device array inside the library.  Checked against the
allocating entry point lm_dpotrf on two calls in a row (the array is shared
between calls, so the second call must not see the first one's leftovers),
plus its size and alignment limits.  Collected last on purpose."""
import ctypes

import numpy as np
import pytest
import torch

import lmb200
from conftest import philox
from helpers import gen_spd

pytestmark = pytest.mark.gpu


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _noalloc(A):
    info = ctypes.c_int(-1)
    st = lmb200.lib().lm_dpotrf_noalloc(_stream(), A.shape[0], lmb200._ptr(A), A.stride(0), ctypes.byref(info))
    return st, info.value


@pytest.mark.parametrize("n", [100, 777])
def test_noalloc_matches_allocating_entry_two_calls(n):
    ctx = lmb200.default_context(0)
    ld = n + (n & 1)  # the no-allocation entry needs an even leading dimension
    for call in range(2):
        A = gen_spd(philox(31000 + 10 * n + call), n)
        ref = torch.from_numpy(A).cuda()
        assert lmb200.dpotrf(ref, ctx) == 0
        got = torch.zeros((n, ld), dtype=torch.float64, device="cuda")[:, :n]
        got.copy_(torch.from_numpy(A))
        torch.cuda.synchronize()
        st, info = _noalloc(got)
        assert st == 0 and info == 0
        G, Gref = got.cpu().numpy(), ref.cpu().numpy()
        assert np.all(np.triu(G, 1) == 0.0)
        assert np.abs(G - Gref).max() <= 1e-13 * np.abs(Gref).max()


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
