"""CPU checks of the C ABI: the library builds, loads and exports every symbol
include/lm_b200.h declares; host-only helpers behave; without a GPU the
context constructor fails with a status instead of crashing."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import lmb200
import oracle as O
from conftest import ROOT, philox

HEADER = os.path.join(ROOT, "include", "lm_b200.h")


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(lmb200.LIB_PATH):
        lmb200.build()
    return lmb200.lib()


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lm_[a-z0-9_]+)\s*\(", text)))


def test_header_matches_binding_list():
    assert declared_symbols() == sorted(lmb200.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lmb200.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (lm_[a-z0-9_]+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    for s in declared_symbols():
        assert hasattr(lib, s)


def test_status_strings(lib):
    assert lib.lm_status_string(0) == b"ok"
    assert lib.lm_status_string(-4) == b"device-side wait timed out"
    assert b"info" in lib.lm_status_string(3)


@pytest.mark.parametrize("seed", range(5))
def test_ipiv_to_perm_matches_oracle(lib, seed):
    g = philox(seed)
    n = 50
    ipiv = np.array([g.integers(k, n) for k in range(n)], dtype=np.int32)
    perm = np.zeros(n, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    assert lib.lm_ipiv_to_perm(n, ipiv.ctypes.data_as(ip), perm.ctypes.data_as(ip)) == 0
    assert np.array_equal(perm, O.ipiv_to_perm(ipiv))
    bad = ipiv.copy()
    bad[3] = n + 5
    assert lib.lm_ipiv_to_perm(n, bad.ctypes.data_as(ip), perm.ctypes.data_as(ip)) == lmb200.LM_ERR_ARG


def test_null_context_is_an_argument_error(lib):
    assert lib.lm_dgemm(None, 1, 1, 1, 1.0, None, 1, None, 1, 0.0, None, 1) == lmb200.LM_ERR_ARG
    assert lib.lm_dgetrf(None, 4, None, 4, None, None) == lmb200.LM_ERR_ARG


def test_ctx_create_without_gpu_fails_cleanly(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    h = ctypes.c_void_p()
    st = lib.lm_ctx_create(ctypes.byref(h), 0)
    assert st < 0 and not h.value


def test_host_mirror_header_compiles():
    """The C++ mirror of the Haskell API compiles against the C ABI."""
    src = os.path.join(ROOT, "linear-massiv_b200", "host", "example.cpp")
    out = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I" + os.path.join(ROOT, "include"),
                          "-I" + os.path.join(ROOT, "linear-massiv_b200", "host"), src],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stderr


def test_server_default_config_layout(lib):
    """The ctypes mirror of lm_server_config reads the defaults the library
    writes (a field out of order or missing would show up as garbage here)."""
    c = lmb200.ServerConfig()
    assert lib.lm_server_default_config(ctypes.byref(c)) == 0
    assert (c.hbm_budget, c.large_workers, c.batch_lanes, c.small_max_n) == (0, 8, 2, 256)
    assert (c.max_batch, c.max_n, c.max_nrhs, list(c.nb)) == (4096, 4096, 64, [16, 16, 16, 16])
    assert (c.ir_method, c.device_loop, c.loop_ctas) == (lmb200.IR_GEPP, 1, 16)
    assert (c.lu_fp64_max_n, c.chol_fp64_max_n) == (2048, 4096)
