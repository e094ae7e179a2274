"""Python binding of liblm_b200.so (the C ABI in include/lm_b200.h).

Function names mirror linear-massiv's public API for the dense-solve path
(gemm, matMul, lu, luSolve, cholesky, choleskySolve, det): each takes
device-resident torch float64 tensors, leaves its inputs untouched and returns
fresh results, the way the reference's pure functions return fresh massiv
arrays.  The raw in-place routines (dgetrf, dgetrs, dpotrf, dpotrs, dgemm)
are exposed too.

There is no fallback: if the CUDA library is missing or no GPU is visible,
every call raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PKG_DIR, "liblm_b200.so")

LM_OK = 0
LM_ERR_ARG = -1
LM_ERR_CUDA = -2
LM_ERR_UNSUPPORTED = -3
LM_ERR_TIMEOUT = -4
LM_ERR_NOMEM = -5
LM_ERR_NOT_CONVERGED = -6

# Every symbol include/lm_b200.h declares (checked by the CPU test suite).
EXPORTS = [
    "lm_ctx_create", "lm_ctx_destroy", "lm_ctx_set_stream", "lm_ctx_get_stream",
    "lm_ctx_synchronize", "lm_ctx_check", "lm_ctx_profile", "lm_ctx_profile_read",
    "lm_status_string", "lm_last_error",
    "lm_launch_count", "lm_dmalloc", "lm_dfree", "lm_h2d", "lm_d2h", "lm_dgemm",
    "lm_dgetrf", "lm_dgetrs", "lm_dgesv", "lm_dpotrf", "lm_dpotrs", "lm_dposv",
    "lm_lu_solve_host", "lm_chol_solve_host", "lm_matmul_host", "lm_gemm_host",
    "lm_lu_host", "lm_cholesky_host", "lm_det_host", "lm_ipiv_to_perm", "lm_dresidual",
    "lm_dgesv_ir", "lm_lu_solve_ir_host", "lm_ctx_set_ir_method", "lm_ctx_ir_last_method", "lm_ctx_ir_history", "lm_dpotrf_noalloc",
    "lm_batch_create", "lm_batch_destroy", "lm_batch_offsets", "lm_batch_solve", "lm_batch_results",
    "lm_batch_factors", "lm_batch_solve_host", "lm_batch_tune", "lm_batch_tune_get", "lm_batch_tune_set",
    "lm_server_default_config", "lm_server_create", "lm_server_submit", "lm_server_test", "lm_server_wait",
    "lm_server_cancel", "lm_server_drain", "lm_server_stats", "lm_server_reset_stats", "lm_server_destroy",
    "lm_dgemv", "lm_matvec_host", "lm_dnorm_inf", "lm_norm_inf_host", "lm_dgetrf_nopiv", "lm_lu_nopivot_host",
    "lm_cholesky_gaxpy_host", "lm_dtridiag_solve", "lm_tridiag_solve_host", "lm_dgesv_ir_prec",
]

IR_RBT = 0
IR_GEPP = 1
IR_PREC_TF32X3 = 0
IR_PREC_TF32 = 1
IR_PREC_BF16 = 2
BATCH_GENERAL = 0
BATCH_SPD = 1
PREC_FP64 = 0
PREC_FP32_IR = 1


class LMError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        msg = _lib().lm_status_string(status).decode()
        last = _lib().lm_last_error().decode()
        super().__init__(f"{what}: {msg} ({status}){': ' + last if last else ''}")


def build(verbose: bool = False) -> str:
    """Compile liblm_b200.so in-tree with the package Makefile (sm_100a)."""
    out = None if verbose else subprocess.DEVNULL
    subprocess.run(["make", "-s", "-j8", "-C", PKG_DIR], check=True, stdout=out)
    return LIB_PATH


_L = None
_LOCK = threading.Lock()


def _lib():
    global _L
    with _LOCK:
        if _L is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"liblm_b200.so is not built ({LIB_PATH}); run __graft_entry__.build()")
            L = ctypes.CDLL(LIB_PATH)
            vp, i, d, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
            ip = ctypes.POINTER(ctypes.c_int)
            dp = ctypes.POINTER(ctypes.c_double)
            sigs = {
                "lm_ctx_create": ([ctypes.POINTER(vp), i], i),
                "lm_ctx_destroy": ([vp], i),
                "lm_ctx_set_stream": ([vp, vp], i),
                "lm_ctx_get_stream": ([vp], vp),
                "lm_ctx_synchronize": ([vp], i),
                "lm_ctx_check": ([vp], i),
                "lm_ctx_profile": ([vp, i], i),
                "lm_ctx_set_ir_method": ([vp, i], i),
                "lm_ctx_ir_last_method": ([vp, ip], i),
                "lm_ctx_ir_history": ([vp, dp, i, ip], i),
                "lm_ctx_profile_read": ([vp, ctypes.POINTER(ctypes.c_longlong), dp, dp, dp], i),
                "lm_status_string": ([i], ctypes.c_char_p),
                "lm_last_error": ([], ctypes.c_char_p),
                "lm_launch_count": ([], ctypes.c_longlong),
                "lm_dmalloc": ([vp, ctypes.POINTER(vp), sz], i),
                "lm_dfree": ([vp, vp], i),
                "lm_h2d": ([vp, vp, vp, sz], i),
                "lm_d2h": ([vp, vp, vp, sz], i),
                "lm_dgemm": ([vp, i, i, i, d, vp, i, vp, i, d, vp, i], i),
                "lm_dgetrf": ([vp, i, vp, i, vp, ip], i),
                "lm_dgetrs": ([vp, i, i, vp, i, vp, vp, i], i),
                "lm_dgesv": ([vp, i, i, vp, i, vp, vp, i, ip], i),
                "lm_dpotrf": ([vp, i, vp, i, ip], i),
                "lm_dpotrs": ([vp, i, i, vp, i, vp, i], i),
                "lm_dposv": ([vp, i, i, vp, i, vp, i, ip], i),
                "lm_lu_solve_host": ([vp, i, i, dp, dp, dp, ip], i),
                "lm_chol_solve_host": ([vp, i, i, dp, dp, dp, ip], i),
                "lm_matmul_host": ([vp, i, i, i, dp, dp, dp], i),
                "lm_gemm_host": ([vp, i, i, i, d, dp, dp, d, dp, dp], i),
                "lm_lu_host": ([vp, i, dp, dp, ip, ip], i),
                "lm_cholesky_host": ([vp, i, dp, dp, ip], i),
                "lm_det_host": ([vp, i, dp, dp], i),
                "lm_ipiv_to_perm": ([i, ip, ip], i),
                "lm_dresidual": ([vp, i, i, vp, i, vp, i, vp, i, vp, i], i),
                "lm_dgesv_ir": ([vp, i, i, vp, i, vp, i, vp, i, d, i, ip, dp, ip], i),
                "lm_lu_solve_ir_host": ([vp, i, i, dp, dp, dp, d, i, ip, dp, ip], i),
                "lm_dpotrf_noalloc": ([vp, i, vp, i, ip], i),
                "lm_batch_create": ([vp, ctypes.POINTER(vp), i, ip, ip, ip, i], i),
                "lm_batch_destroy": ([vp], i),
                "lm_batch_offsets": ([vp, vp, vp], i),
                "lm_batch_solve": ([vp, vp, vp, vp, d, i], i),
                "lm_batch_results": ([vp, ip, ip, dp], i),
                "lm_batch_factors": ([vp, ctypes.POINTER(vp), ctypes.POINTER(vp)], i),
                "lm_batch_solve_host": ([vp, dp, dp, dp, d, i], i),
                "lm_batch_tune": ([vp, i, ctypes.c_char_p], i),
                "lm_batch_tune_get": ([vp, ip], i),
                "lm_batch_tune_set": ([vp, ip], i),
                "lm_server_default_config": ([vp], i),
                "lm_server_create": ([ctypes.POINTER(vp), i, vp], i),
                "lm_server_submit": ([vp, i, i, i, vp, vp, vp, ctypes.POINTER(ctypes.c_longlong)], i),
                "lm_server_test": ([vp, ctypes.c_longlong, ip, ip, dp], i),
                "lm_server_wait": ([vp, ctypes.c_longlong, ip, dp, d], i),
                "lm_server_cancel": ([vp, ctypes.c_longlong], i),
                "lm_server_drain": ([vp, d], i),
                "lm_server_stats": ([vp, vp], i),
                "lm_server_reset_stats": ([vp], i),
                "lm_server_destroy": ([vp], i),
                "lm_dgemv": ([vp, i, i, vp, i, vp, vp], i),
                "lm_matvec_host": ([vp, i, i, dp, dp, dp], i),
                "lm_dnorm_inf": ([vp, i, i, vp, i, dp], i),
                "lm_norm_inf_host": ([vp, i, i, dp, dp], i),
                "lm_dgetrf_nopiv": ([vp, i, vp, i, ip], i),
                "lm_lu_nopivot_host": ([vp, i, dp, dp, ip], i),
                "lm_cholesky_gaxpy_host": ([vp, i, dp, dp, ip], i),
                "lm_dtridiag_solve": ([vp, i, vp, vp, vp, vp], i),
                "lm_tridiag_solve_host": ([vp, i, dp, dp, dp, dp], i),
                "lm_dgesv_ir_prec": ([vp, i, i, vp, i, vp, i, vp, i, i, d, i, ip, dp, ip], i),
            }
            for name, (args, res) in sigs.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = res
            _L = L
    return _L


def lib():
    return _lib()


def launch_count() -> int:
    return int(_lib().lm_launch_count())


def _check(status: int, what: str) -> int:
    if status < 0:
        raise LMError(status, what)
    return status


class Context:
    """An lm_ctx bound to one device.  By default its kernels run on torch's
    current stream so torch events and synchronisation see them."""

    def __init__(self, device: int = 0, use_torch_stream: bool = True):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("lmb200 needs a CUDA device; none is visible")
        self.device = device
        h = ctypes.c_void_p()
        _check(_lib().lm_ctx_create(ctypes.byref(h), device), "lm_ctx_create")
        self.h = h
        if use_torch_stream:
            with torch.cuda.device(device):
                s = torch.cuda.current_stream(device).cuda_stream
            _check(_lib().lm_ctx_set_stream(self.h, ctypes.c_void_p(s)), "lm_ctx_set_stream")

    def close(self):
        if getattr(self, "h", None):
            _lib().lm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        _check(_lib().lm_ctx_synchronize(self.h), "lm_ctx_synchronize")

    def check(self):
        _check(_lib().lm_ctx_check(self.h), "device status")

    PHASES = ("gemm", "panel", "swap", "trsm", "other")

    def set_ir_method(self, method: int):
        """IR_GEPP (FP32 partial pivoting; default) or IR_RBT (randomised, no pivoting) for the mixed-precision solves."""
        _check(_lib().lm_ctx_set_ir_method(self.h, int(method)), "lm_ctx_set_ir_method")

    def ir_history(self) -> list:
        """Worst backward error after each refinement step of the last mixed-precision solve."""
        buf = (ctypes.c_double * 256)()
        k = ctypes.c_int(0)
        _check(_lib().lm_ctx_ir_history(self.h, buf, 256, ctypes.byref(k)), "lm_ctx_ir_history")
        return [buf[i] for i in range(min(k.value, 256))]

    def ir_last_method(self) -> int:
        m = ctypes.c_int(-1)
        _check(_lib().lm_ctx_ir_last_method(self.h, ctypes.byref(m)), "lm_ctx_ir_last_method")
        return m.value

    def profile(self, enable: bool = True):
        _check(_lib().lm_ctx_profile(self.h, 1 if enable else 0), "lm_ctx_profile")

    def profile_read(self) -> dict:
        """Per-phase {launches, ms, flops, bytes} since the last read (synchronises)."""
        n = len(self.PHASES)
        L = (ctypes.c_longlong * n)()
        M, F, B = (ctypes.c_double * n)(), (ctypes.c_double * n)(), (ctypes.c_double * n)()
        _check(_lib().lm_ctx_profile_read(self.h, L, M, F, B), "lm_ctx_profile_read")
        return {p: {"launches": int(L[i]), "ms": M[i], "flops": F[i], "bytes": B[i]} for i, p in enumerate(self.PHASES)}


_DEFAULT = {}


def default_context(device: int = 0) -> Context:
    c = _DEFAULT.get(device)
    if c is None:
        c = Context(device)
        _DEFAULT[device] = c
    return c


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _mat(t, name):
    import torch

    if not (t.is_cuda and t.dtype == torch.float64 and t.dim() == 2 and t.stride(1) == 1):
        raise ValueError(f"{name} must be a row-major (stride(1) == 1) float64 CUDA matrix")
    return t


# ---- raw in-place routines ---------------------------------------------------

def dgemm(alpha, A, B, beta, C, ctx: Context | None = None):
    """C <- alpha*A*B + beta*C in place."""
    ctx = ctx or default_context(C.device.index or 0)
    _mat(A, "A"), _mat(B, "B"), _mat(C, "C")
    m, k = A.shape
    n = B.shape[1]
    if B.shape[0] != k or C.shape != (m, n):
        raise ValueError("dimension mismatch")
    _check(_lib().lm_dgemm(ctx.h, m, n, k, float(alpha), _ptr(A), A.stride(0), _ptr(B), B.stride(0),
                           float(beta), _ptr(C), C.stride(0)), "lm_dgemm")
    return C


def dgetrf(A, ipiv, ctx: Context | None = None, sync_info: bool = True) -> int:
    """In-place LU of A; ipiv is an int32 CUDA tensor of length n.  Returns info."""
    ctx = ctx or default_context(A.device.index or 0)
    _mat(A, "A")
    n = A.shape[0]
    info = ctypes.c_int(0)
    st = _lib().lm_dgetrf(ctx.h, n, _ptr(A), A.stride(0), _ptr(ipiv), ctypes.byref(info) if sync_info else None)
    _check(st, "lm_dgetrf")
    return info.value


def dgetrs(LU, ipiv, B, ctx: Context | None = None):
    ctx = ctx or default_context(LU.device.index or 0)
    _mat(LU, "LU"), _mat(B, "B")
    n, nrhs = B.shape
    _check(_lib().lm_dgetrs(ctx.h, n, nrhs, _ptr(LU), LU.stride(0), _ptr(ipiv), _ptr(B), B.stride(0)), "lm_dgetrs")
    return B


def dpotrf(A, ctx: Context | None = None, sync_info: bool = True) -> int:
    ctx = ctx or default_context(A.device.index or 0)
    _mat(A, "A")
    info = ctypes.c_int(0)
    st = _lib().lm_dpotrf(ctx.h, A.shape[0], _ptr(A), A.stride(0), ctypes.byref(info) if sync_info else None)
    _check(st, "lm_dpotrf")
    return info.value


def dpotrs(G, B, ctx: Context | None = None):
    ctx = ctx or default_context(G.device.index or 0)
    _mat(G, "G"), _mat(B, "B")
    n, nrhs = B.shape
    _check(_lib().lm_dpotrs(ctx.h, n, nrhs, _ptr(G), G.stride(0), _ptr(B), B.stride(0)), "lm_dpotrs")
    return B


def dresidual(A, X, B, R, ctx: Context | None = None):
    ctx = ctx or default_context(A.device.index or 0)
    n, nrhs = B.shape
    _check(_lib().lm_dresidual(ctx.h, n, nrhs, _ptr(A), A.stride(0), _ptr(X), X.stride(0), _ptr(B), B.stride(0),
                               _ptr(R), R.stride(0)), "lm_dresidual")
    return R


# ---- the reference's pure API (fresh outputs, inputs untouched) ---------------

def _as_cols(b):
    return (b.unsqueeze(1), True) if b.dim() == 1 else (b, False)


def gemm(alpha, A, B, beta, C, ctx: Context | None = None):
    """gemm alpha A B beta C (Level3.hs:102-131)."""
    out = C.clone()
    return dgemm(alpha, A, B, beta, out, ctx)


def matMul(A, B, ctx: Context | None = None):
    """matMul / matMulP (Level3.hs:144-147, 183-207)."""
    import torch

    C = torch.empty((A.shape[0], B.shape[1]), dtype=torch.float64, device=A.device)
    return dgemm(1.0, A, B, 0.0, C, ctx)


def lu_factor(A, ctx: Context | None = None):
    """Device LU: (packed LU, swap list ipiv, info)."""
    import torch

    LU = A.clone()
    ipiv = torch.empty(A.shape[0], dtype=torch.int32, device=A.device)
    info = dgetrf(LU, ipiv, ctx)
    return LU, ipiv, info


def lu(A, ctx: Context | None = None):
    """lu (LU.hs:121-122): (packed LU, permutation vector perm)."""
    LU, ipiv, _ = lu_factor(A, ctx)
    return LU, ipiv_to_perm(ipiv.cpu().tolist())


def luSolve(A, b, ctx: Context | None = None):
    """luSolve / luSolveP (LU.hs:240-304) for a vector or an n x nrhs matrix."""
    B, vec = _as_cols(b)
    LU, ipiv, _ = lu_factor(A, ctx)
    X = B.clone().contiguous()
    dgetrs(LU, ipiv, X, ctx)
    return X[:, 0] if vec else X


def cholesky(A, ctx: Context | None = None):
    """cholesky (Chol.hs:114-147): G, zeros above the diagonal."""
    G = A.clone()
    dpotrf(G, ctx)
    return G


def choleskySolve(A, b, ctx: Context | None = None):
    """choleskySolve / choleskySolveP (Chol.hs:229-273)."""
    B, vec = _as_cols(b)
    G = cholesky(A, ctx)
    X = B.clone().contiguous()
    dpotrs(G, X, ctx)
    return X[:, 0] if vec else X


def det(A, ctx: Context | None = None) -> float:
    """det (LU.hs:534-545)."""
    import numpy as np

    ctx = ctx or default_context(A.device.index or 0)
    a = np.ascontiguousarray(A.detach().cpu().numpy(), dtype=np.float64)
    out = ctypes.c_double(0.0)
    _check(_lib().lm_det_host(ctx.h, a.shape[0], a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                              ctypes.byref(out)), "lm_det_host")
    return out.value


def matvec(A, x, ctx: Context | None = None):
    """matvec / matvecP (Level2.hs:123-139): y = A x, bitwise the reference's
    rawGemv order."""
    import torch

    ctx = ctx or default_context(A.device.index or 0)
    _mat(A, "A")
    m, n = A.shape
    x = x.contiguous()
    if x.dim() != 1 or x.shape[0] != n or x.dtype != torch.float64 or not x.is_cuda:
        raise ValueError("x must be a float64 CUDA vector of length A.shape[1]")
    y = torch.empty(m, dtype=torch.float64, device=A.device)
    _check(_lib().lm_dgemv(ctx.h, m, n, _ptr(A), A.stride(0), _ptr(x), _ptr(y)), "lm_dgemv")
    return y


def normInf(A, ctx: Context | None = None) -> float:
    """normInf (Norms.hs:135-141); a 1-D tensor gives vnormInf (Norms.hs:94-96)."""
    ctx = ctx or default_context(A.device.index or 0)
    M = A.unsqueeze(1).contiguous() if A.dim() == 1 else A
    _mat(M, "A")
    out = ctypes.c_double(0.0)
    _check(_lib().lm_dnorm_inf(ctx.h, M.shape[0], M.shape[1], _ptr(M), M.stride(0), ctypes.byref(out)),
           "lm_dnorm_inf")
    return out.value


def luNoPivot(A, ctx: Context | None = None):
    """luNoPivot (LU.hs:196-214): packed unit-L / U without interchanges; returns (LU, info)."""
    ctx = ctx or default_context(A.device.index or 0)
    LU = A.clone()
    _mat(LU, "A")
    info = ctypes.c_int(0)
    _check(_lib().lm_dgetrf_nopiv(ctx.h, LU.shape[0], _ptr(LU), LU.stride(0), ctypes.byref(info)),
           "lm_dgetrf_nopiv")
    return LU, info.value


def choleskyGaxpy(A, ctx: Context | None = None):
    """choleskyGaxpy (Chol.hs:173-204): the same G as cholesky."""
    return cholesky(A, ctx)


def tridiagSolve(diag, supdiag, b, ctx: Context | None = None):
    """tridiagSolve (Solve/Banded.hs:292-342): SPD tridiagonal solve from the
    diagonal and the superdiagonal (length n, entries 0..n-2 used)."""
    import torch

    ctx = ctx or default_context(b.device.index or 0)
    diag, supdiag, b = diag.contiguous(), supdiag.contiguous(), b.contiguous()
    x = torch.empty_like(b)
    _check(_lib().lm_dtridiag_solve(ctx.h, b.shape[0], _ptr(diag), _ptr(supdiag), _ptr(b), _ptr(x)),
           "lm_dtridiag_solve")
    return x


def ipiv_to_perm(ipiv):
    n = len(ipiv)
    perm = list(range(n))
    for k, p in enumerate(ipiv):
        perm[k], perm[p] = perm[p], perm[k]
    return perm


def luSolveIR(A, b, tol: float = 0.0, max_iter: int = 30, ctx: Context | None = None):
    """Mixed-precision luSolve: FP32/TF32 LU refined in FP64.

    Returns (x, iterations, backward_error, status); status is 0, info > 0
    for a zero FP32 pivot, or LM_ERR_NOT_CONVERGED (x is the last iterate).
    """
    import torch

    ctx = ctx or default_context(A.device.index or 0)
    B, vec = _as_cols(b)
    B = B.contiguous()
    X = torch.empty_like(B)
    it, be, info = ctypes.c_int(0), ctypes.c_double(0.0), ctypes.c_int(0)
    st = _lib().lm_dgesv_ir(ctx.h, A.shape[0], B.shape[1], _ptr(A), A.stride(0), _ptr(B), B.stride(0), _ptr(X),
                            X.stride(0), float(tol), int(max_iter), ctypes.byref(it), ctypes.byref(be),
                            ctypes.byref(info))
    if st < 0 and st != LM_ERR_NOT_CONVERGED:
        raise LMError(st, "lm_dgesv_ir")
    return (X[:, 0] if vec else X), it.value, be.value, st


# ---- host-buffer entry points (what a pure FFI binding calls) -----------------

def luSolveIRPrec(A, b, prec: int = IR_PREC_TF32X3, tol: float = 0.0, max_iter: int = 30,
                  ctx: Context | None = None):
    """Mixed-precision luSolve with the factor precision prec (IR_PREC_*):
    (x, outer steps, backward error, status)."""
    import torch

    ctx = ctx or default_context(A.device.index or 0)
    B, vec = _as_cols(b)
    B = B.contiguous()
    X = torch.empty_like(B)
    it, be, info = ctypes.c_int(0), ctypes.c_double(0.0), ctypes.c_int(0)
    st = _lib().lm_dgesv_ir_prec(ctx.h, A.shape[0], B.shape[1], _ptr(A), A.stride(0), _ptr(B), B.stride(0), _ptr(X),
                                 X.stride(0), int(prec), float(tol), int(max_iter), ctypes.byref(it), ctypes.byref(be),
                                 ctypes.byref(info))
    if st < 0 and st != LM_ERR_NOT_CONVERGED:
        _check(st, "lm_dgesv_ir_prec")
    return (X[:, 0] if vec else X), it.value, be.value, st


def _np_ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def lu_solve_host(A, B, ctx: Context | None = None):
    """lm_lu_solve_host on host numpy arrays: returns (X, info)."""
    import numpy as np

    ctx = ctx or default_context(0)
    A = np.ascontiguousarray(A, dtype=np.float64)
    vec = B.ndim == 1
    B2 = np.ascontiguousarray(B.reshape(A.shape[0], -1), dtype=np.float64)
    X = np.empty_like(B2)
    info = ctypes.c_int(0)
    _check(_lib().lm_lu_solve_host(ctx.h, A.shape[0], B2.shape[1], _np_ptr(A), _np_ptr(B2), _np_ptr(X),
                                   ctypes.byref(info)), "lm_lu_solve_host")
    return (X[:, 0] if vec else X), info.value


def chol_solve_host(A, B, ctx: Context | None = None):
    import numpy as np

    ctx = ctx or default_context(0)
    A = np.ascontiguousarray(A, dtype=np.float64)
    vec = B.ndim == 1
    B2 = np.ascontiguousarray(B.reshape(A.shape[0], -1), dtype=np.float64)
    X = np.empty_like(B2)
    info = ctypes.c_int(0)
    _check(_lib().lm_chol_solve_host(ctx.h, A.shape[0], B2.shape[1], _np_ptr(A), _np_ptr(B2), _np_ptr(X),
                                     ctypes.byref(info)), "lm_chol_solve_host")
    return (X[:, 0] if vec else X), info.value


def gemm_host(alpha, A, B, beta, C0, ctx: Context | None = None):
    import numpy as np

    ctx = ctx or default_context(0)
    A = np.ascontiguousarray(A, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    C0 = np.ascontiguousarray(C0, dtype=np.float64)
    C = np.empty((A.shape[0], B.shape[1]))
    _check(_lib().lm_gemm_host(ctx.h, A.shape[0], B.shape[1], A.shape[1], float(alpha), _np_ptr(A), _np_ptr(B),
                               float(beta), _np_ptr(C0), _np_ptr(C)), "lm_gemm_host")
    return C


def lu_host(A, ctx: Context | None = None):
    import numpy as np

    ctx = ctx or default_context(0)
    A = np.ascontiguousarray(A, dtype=np.float64)
    n = A.shape[0]
    LU = np.empty_like(A)
    perm = np.zeros(n, dtype=np.int32)
    info = ctypes.c_int(0)
    _check(_lib().lm_lu_host(ctx.h, n, _np_ptr(A), _np_ptr(LU), perm.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                             ctypes.byref(info)), "lm_lu_host")
    return LU, perm, info.value


def cholesky_host(A, ctx: Context | None = None):
    import numpy as np

    ctx = ctx or default_context(0)
    A = np.ascontiguousarray(A, dtype=np.float64)
    G = np.empty_like(A)
    info = ctypes.c_int(0)
    _check(_lib().lm_cholesky_host(ctx.h, A.shape[0], _np_ptr(A), _np_ptr(G), ctypes.byref(info)),
           "lm_cholesky_host")
    return G, info.value


# ---- batched uneven-size solves (one persistent launch) -------------------------

class Batch:
    """A plan for `count` independent solves A_i X_i = B_i of uneven sizes
    (n_i <= 256, nrhs_i <= 16), general (LU) or SPD (Cholesky) per instance,
    run as one persistent kernel.  Inputs are packed back to back
    (offsets()); solve() takes device float64 tensors."""

    def __init__(self, n, nrhs, kind, precision: int = PREC_FP64, ctx: Context | None = None):
        import numpy as np

        self.ctx = ctx or default_context(0)
        self.n = np.ascontiguousarray(n, dtype=np.int32)
        self.nrhs = np.ascontiguousarray(nrhs, dtype=np.int32)
        self.kind = np.ascontiguousarray(kind, dtype=np.int32)
        self.count = len(self.n)
        self.precision = precision
        h = ctypes.c_void_p()
        ip = ctypes.POINTER(ctypes.c_int)
        _check(_lib().lm_batch_create(self.ctx.h, ctypes.byref(h), self.count, self.n.ctypes.data_as(ip),
                                      self.nrhs.ctypes.data_as(ip), self.kind.ctypes.data_as(ip), precision),
               "lm_batch_create")
        self.h = h
        a = np.zeros(self.count + 1, dtype=np.int64)
        b = np.zeros(self.count + 1, dtype=np.int64)
        _check(_lib().lm_batch_offsets(self.h, ctypes.c_void_p(a.ctypes.data), ctypes.c_void_p(b.ctypes.data)),
               "lm_batch_offsets")
        self.a_off, self.b_off = a, b
        self.p_off = np.concatenate([[0], np.cumsum(self.n.astype(np.int64))])

    def offsets(self):
        return self.a_off, self.b_off

    def solve(self, A, B, X, tol: float = 0.0, max_iter: int = 10):
        _check(_lib().lm_batch_solve(self.h, _ptr(A), _ptr(B), _ptr(X), float(tol), int(max_iter)),
               "lm_batch_solve")
        return X

    def solve_host(self, A, B, tol: float = 0.0, max_iter: int = 10):
        import numpy as np

        A = np.ascontiguousarray(A, dtype=np.float64)
        B = np.ascontiguousarray(B, dtype=np.float64)
        X = np.empty_like(B)
        _check(_lib().lm_batch_solve_host(self.h, _np_ptr(A), _np_ptr(B), _np_ptr(X), float(tol), int(max_iter)),
               "lm_batch_solve_host")
        return X

    def results(self):
        """(info, iters, berr) per instance, as numpy arrays (synchronises)."""
        import numpy as np

        info = np.zeros(max(self.count, 1), dtype=np.int32)
        iters = np.zeros(max(self.count, 1), dtype=np.int32)
        berr = np.zeros(max(self.count, 1), dtype=np.float64)
        ip = ctypes.POINTER(ctypes.c_int)
        _check(_lib().lm_batch_results(self.h, info.ctypes.data_as(ip), iters.ctypes.data_as(ip), _np_ptr(berr)),
               "lm_batch_results")
        return info[:self.count], iters[:self.count], berr[:self.count]

    def factors(self):
        """Device pointers (ints) of the factor workspace and the swap lists."""
        f, p = ctypes.c_void_p(), ctypes.c_void_p()
        _check(_lib().lm_batch_factors(self.h, ctypes.byref(f), ctypes.byref(p)), "lm_batch_factors")
        return f.value, p.value

    def close(self):
        if getattr(self, "h", None):
            _lib().lm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_tune(precision: int = PREC_FP64, path: str | None = None, ctx: Context | None = None):
    """Autotune the batch kernel's panel width per size bucket; returns the table nb[2][4]."""
    ctx = ctx or default_context(0)
    _check(_lib().lm_batch_tune(ctx.h, precision, path.encode() if path else None), "lm_batch_tune")
    return batch_tune_get(ctx)


def batch_tune_get(ctx: Context | None = None):
    ctx = ctx or default_context(0)
    t = (ctypes.c_int * 8)()
    _check(_lib().lm_batch_tune_get(ctx.h, t), "lm_batch_tune_get")
    return [list(t[0:4]), list(t[4:8])]


def batch_tune_set(table, ctx: Context | None = None):
    ctx = ctx or default_context(0)
    t = (ctypes.c_int * 8)(*(list(table[0]) + list(table[1])))
    _check(_lib().lm_batch_tune_set(ctx.h, t), "lm_batch_tune_set")


# ---- serving loop ----------------------------------------------------------------

class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_size_t), ("large_workers", ctypes.c_int), ("batch_lanes", ctypes.c_int),
                ("small_max_n", ctypes.c_int), ("small_precision", ctypes.c_int), ("large_precision", ctypes.c_int),
                ("max_batch", ctypes.c_int), ("max_n", ctypes.c_int), ("max_nrhs", ctypes.c_int),
                ("nb", ctypes.c_int * 4), ("ir_method", ctypes.c_int), ("device_loop", ctypes.c_int),
                ("loop_ctas", ctypes.c_int), ("lu_fp64_max_n", ctypes.c_int), ("chol_fp64_max_n", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_longlong), ("rejected", ctypes.c_longlong), ("cancelled", ctypes.c_longlong),
                ("failed", ctypes.c_longlong), ("fp64_fallbacks", ctypes.c_longlong),
                ("queue_peak", ctypes.c_longlong), ("pending", ctypes.c_longlong),
                ("micro_batches", ctypes.c_longlong), ("small_solved", ctypes.c_longlong),
                ("inflight", ctypes.c_int), ("inflight_peak", ctypes.c_int),
                ("arena_bytes", ctypes.c_size_t), ("arena_peak_bytes", ctypes.c_size_t),
                ("fixed_bytes", ctypes.c_size_t),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("span_s", ctypes.c_double), ("solves_per_s", ctypes.c_double),
                ("tflops", ctypes.c_double), ("ir_solves", ctypes.c_longlong), ("ir_gepp", ctypes.c_longlong),
                ("ir_iterations", ctypes.c_longlong)]


class Server:
    """Continuous-batching solve server (lm_server_*).  submit() takes host
    numpy arrays (A n x n, B n x nrhs, float64, C order); the arrays are kept
    referenced until the request completes."""

    def __init__(self, device: int = 0, **cfg):
        c = ServerConfig()
        _check(_lib().lm_server_default_config(ctypes.byref(c)), "lm_server_default_config")
        for k, v in cfg.items():
            if k == "nb":
                c.nb = (ctypes.c_int * 4)(*v)
            else:
                setattr(c, k, v)
        self.config = c
        h = ctypes.c_void_p()
        _check(_lib().lm_server_create(ctypes.byref(h), device, ctypes.byref(c)), "lm_server_create")
        self.h = h
        self._keep = {}

    def submit(self, A, B, kind: int = BATCH_GENERAL):
        """Queue A X = B; returns (id, X) with X the output array (filled on completion)."""
        import numpy as np

        A = np.ascontiguousarray(A, dtype=np.float64)
        B2 = np.ascontiguousarray(B.reshape(A.shape[0], -1), dtype=np.float64)
        X = np.empty_like(B2)
        rid = ctypes.c_longlong(0)
        _check(_lib().lm_server_submit(self.h, A.shape[0], B2.shape[1], kind, ctypes.c_void_p(A.ctypes.data),
                                       ctypes.c_void_p(B2.ctypes.data), ctypes.c_void_p(X.ctypes.data),
                                       ctypes.byref(rid)), "lm_server_submit")
        self._keep[rid.value] = (A, B2, X)
        return rid.value, X

    def submit_raw(self, n, nrhs, kind, A_ptr, B_ptr, X_ptr):
        """Queue with caller-managed buffers (addresses as ints); returns the id."""
        rid = ctypes.c_longlong(0)
        _check(_lib().lm_server_submit(self.h, n, nrhs, kind, ctypes.c_void_p(A_ptr), ctypes.c_void_p(B_ptr),
                                       ctypes.c_void_p(X_ptr), ctypes.byref(rid)), "lm_server_submit")
        return rid.value

    def wait(self, rid: int, timeout_s: float = 0.0):
        """Block until done: (status, latency_ms)."""
        st, lat = ctypes.c_int(0), ctypes.c_double(0.0)
        _check(_lib().lm_server_wait(self.h, rid, ctypes.byref(st), ctypes.byref(lat), float(timeout_s)),
               "lm_server_wait")
        self._keep.pop(rid, None)
        return st.value, lat.value

    def test(self, rid: int):
        """Non-blocking: (done, status, latency_ms)."""
        dn, st, lat = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0.0)
        _check(_lib().lm_server_test(self.h, rid, ctypes.byref(dn), ctypes.byref(st), ctypes.byref(lat)),
               "lm_server_test")
        if dn.value:
            self._keep.pop(rid, None)
        return bool(dn.value), st.value, lat.value

    def cancel(self, rid: int) -> int:
        return _lib().lm_server_cancel(self.h, rid)

    def drain(self, timeout_s: float = 0.0):
        _check(_lib().lm_server_drain(self.h, float(timeout_s)), "lm_server_drain")

    def stats(self) -> dict:
        st = ServerStats()
        _check(_lib().lm_server_stats(self.h, ctypes.byref(st)), "lm_server_stats")
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def reset_stats(self):
        _check(_lib().lm_server_reset_stats(self.h), "lm_server_reset_stats")

    def close(self):
        if getattr(self, "h", None):
            _lib().lm_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
