"""ctypes binding of libbpf.so (the C ABI declared in include/bpf.h).

There is no CPU fallback: importing the solvers without the built library, or calling them
without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_ROOT, "lib", "libbpf.so")

BPF_SUCCESS = 0
BPF_ERR_INVALID_VALUE = 1
BPF_ERR_DIMENSION = 2
BPF_ERR_CUDA = 3
BPF_ERR_ALLOC = 4
BPF_ERR_SINGULAR = 5
BPF_ERR_NOT_SUPPORTED = 6
BPF_ERR_TIMEOUT = 7
BPF_ERR_NUMERIC = 8

BPF_F64 = 0
BPF_F32 = 1

ORDERINGS = {"AMD": 0, "MDQ": 1, "METIS": 2, "RCM": 3, "NATURAL": 4}


class BPFError(RuntimeError):
    """Error raised for a non-success status of the library (Julia's ErrorException)."""

    def __init__(self, status: int, msg: str):
        super().__init__(msg)
        self.status = status


class DimensionMismatch(BPFError, ValueError):
    pass


class SingularException(BPFError):
    pass


class CsrDesc(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_int), ("rowptr", C.c_void_p), ("colind", C.c_void_p),
                ("vals", C.c_void_p), ("index_base", C.c_int), ("dtype", C.c_int)]


class GmresOpts(C.Structure):
    _fields_ = [("memory", C.c_int), ("restart", C.c_int), ("reorthogonalization", C.c_int),
                ("ldiv", C.c_int), ("atol", C.c_double), ("rtol", C.c_double), ("itmax", C.c_int),
                ("timemax", C.c_double), ("verbose", C.c_int), ("history", C.c_int)]


class BicgstabOpts(C.Structure):
    _fields_ = [("atol", C.c_double), ("rtol", C.c_double), ("itmax", C.c_int),
                ("timemax", C.c_double), ("verbose", C.c_int), ("history", C.c_int)]


class BatchOpts(C.Structure):
    _fields_ = [("atol", C.c_double), ("rtol", C.c_double), ("itmax", C.c_int), ("memory", C.c_int),
                ("factor_dtype", C.c_int), ("ordering", C.c_int), ("slice", C.c_int),
                ("ctas_per_sm", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("niter", C.c_int), ("solved", C.c_int), ("status", C.c_int), ("timer", C.c_double),
                ("n_residuals", C.c_int), ("residuals_capacity", C.c_int),
                ("residuals", C.POINTER(C.c_double)), ("npass", C.c_int)]


# (name, restype, argtypes) of every exported entry point of include/bpf.h.
_P = C.c_void_p
_I = C.c_int
_D = C.c_double
SIGNATURES = {
    "bpf_ctx_create": (_I, [C.POINTER(_P), _P]),
    "bpf_ctx_set_stream": (_I, [_P, _P]),
    "bpf_ctx_destroy": (_I, [_P]),
    "bpf_last_error": (C.c_char_p, [_P]),
    "bpf_solve_status_string": (C.c_char_p, [_I]),
    "bpf_ctx_kernel_launches": (C.c_longlong, [_P]),
    "bpf_ctx_set_timing": (_I, [_P, _I]),
    "bpf_ctx_set_wait_limit": (_I, [_P, C.c_longlong]),
    "bpf_selftest_grid_barrier": (_I, [_P, _I, _I, C.POINTER(_I)]),
    "bpf_ctx_kernel_time": (_I, [_P, _I, C.POINTER(_D), C.POINTER(C.c_longlong),
                                 C.POINTER(_D), C.POINTER(_D)]),
    "bpf_spmm": (_I, [_P, C.POINTER(CsrDesc), _I, _D, _P, _I, _D, _P, _I]),
    "bpf_householder": (_I, [_P, _I, _I, _P, _I, _P, _I]),
    "bpf_householder_lapack": (_I, [_P, _I, _I, _P, _I, _P, _I, _P, _I]),
    "bpf_ilu0_create": (_I, [_P, C.POINTER(CsrDesc), _I, _I, C.POINTER(_P)]),
    "bpf_ic0_create": (_I, [_P, C.POINTER(CsrDesc), _I, _I, C.POINTER(_P)]),
    "bpf_ilu0_create_ordered": (_I, [_P, C.POINTER(CsrDesc), _I, _I, _I, C.POINTER(_P)]),
    "bpf_ic0_create_ordered": (_I, [_P, C.POINTER(CsrDesc), _I, _I, _I, C.POINTER(_P)]),
    "bpf_prec_permutation": (_I, [_P, _P]),
    "bpf_block_jacobi_create": (_I, [_P, C.POINTER(CsrDesc), _I, _I, C.POINTER(_P)]),
    "bpf_tc_gemm_bf16": (_I, [_P, _I, _I, _I, _P, _I, _P, _I, _P, _I, _I, _I]),
    "bpf_mlp_create": (_I, [_P, _I, _I, C.c_ulonglong, C.POINTER(_P)]),
    "bpf_mlp_destroy": (_I, [_P]),
    "bpf_mlp_set_scale": (_I, [_P, _D]),
    "bpf_mlp_forward": (_I, [_P, _I, _P, _I, _P, _I]),
    "bpf_mlp_gradients": (_I, [_P, _I, _P, _I, _P, _I, C.POINTER(_D)]),
    "bpf_mlp_train_step": (_I, [_P, _I, _P, _I, _P, _I, _D, C.POINTER(_D)]),
    "bpf_mlp_params": (_I, [_P, _I, C.POINTER(_P), C.POINTER(_P), C.POINTER(C.c_longlong),
                            C.POINTER(C.c_longlong)]),
    "bpf_mlp_refresh": (_I, [_P]),
    "bpf_mlp_param_copy": (_I, [_P, _I, _I, _P, _I]),
    "bpf_mlp_basis": (_I, [_P, _I, C.c_ulonglong, _P, _I]),
    "bpf_prec_refactor": (_I, [_P, _P]),
    "bpf_prec_apply": (_I, [_P, _I, _P, _I, _P, _I]),
    "bpf_prec_apply_noalloc": (_I, [_P, _I, _P, _I, _P, _I]),
    "bpf_prec_factor_values": (_I, [_P, _P]),
    "bpf_prec_levels": (_I, [_P, C.POINTER(_I), C.POINTER(_I)]),
    "bpf_prec_destroy": (_I, [_P]),
    "bpf_block_gmres": (_I, [_P, C.POINTER(CsrDesc), _I, _P, _I, _P, _I, _P, _I, _P, _P,
                             C.POINTER(GmresOpts), C.POINTER(Stats)]),
    "bpf_block_gmres_deflated": (_I, [_P, C.POINTER(CsrDesc), _I, _P, _I, _P, _I, _P, _I, _P, _P,
                             C.POINTER(GmresOpts), _P, _I, _I, C.POINTER(Stats)]),
    "bpf_block_bicgstab": (_I, [_P, C.POINTER(CsrDesc), _I, _P, _I, _P, _I, _P, _I, _P,
                                C.POINTER(BicgstabOpts), C.POINTER(Stats)]),
    "bpf_rf_analyze": (_I, [_P, C.POINTER(CsrDesc), _I, _D, _I, _I, C.POINTER(_P)]),
    "bpf_rf_refactor": (_I, [_P, _P]),
    "bpf_rf_refactor_batch": (_I, [_P, _P, _I]),
    "bpf_rf_solve": (_I, [_P, _I, _P, _I]),
    "bpf_rf_solve_refined": (_I, [_P, C.POINTER(CsrDesc), _I, _P, _I, _P, _I, _I]),
    "bpf_rf_info": (_I, [_P, C.POINTER(_I), C.POINTER(_I), _P, _P]),
    "bpf_rf_destroy": (_I, [_P]),
    "bpf_batch_opts_default": (None, [C.POINTER(BatchOpts)]),
    "bpf_batch_plan": (_I, [_P, _I, _P, _P, C.POINTER(BatchOpts), C.POINTER(_P)]),
    "bpf_batch_plan_sliced": (_I, [_P, _I, _P, _P, _P, C.POINTER(BatchOpts), C.POINTER(_P)]),
    "bpf_batch_solve": (_I, [_P, _P, _P, _P, _P, _P]),
    "bpf_batch_unit_stats": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "bpf_batch_unit_cycles": (_I, [_P, _P]),
    "bpf_batch_info": (_I, [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(C.c_longlong)]),
    "bpf_batch_destroy": (_I, [_P]),
    "bpf_pf_create": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _P, C.POINTER(CsrDesc), C.POINTER(_P)]),
    "bpf_pf_info": (_I, [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)]),
    "bpf_pf_mismatch": (_I, [_P, _P, _P, _D, _P, _P, C.POINTER(_D)]),
    "bpf_pf_jacobian": (_I, [_P, _P, _P, _P, _I]),
    "bpf_pf_destroy": (_I, [_P]),
}

_lib = None
_lock = threading.Lock()


def load():
    """Load libbpf.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"libbpf.so not found at {LIB_PATH}; build it with `make -C "
                    f"blockpowerflow.jl_b200/csrc` (or __graft_entry__.build())")
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name, None)
                if fn is None:
                    continue
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def exported_symbols():
    lib = load()
    return [n for n in SIGNATURES if hasattr(lib, n)]


_ctxs: dict = {}


def context(device=None):
    """Per-device library context, bound to torch's current stream at each call."""
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("blockpowerflow_b200 needs a CUDA device (no CPU fallback)")
    dev = torch.cuda.current_device() if device is None else int(device)
    lib = load()
    ctx = _ctxs.get(dev)
    if ctx is None:
        with torch.cuda.device(dev):
            h = C.c_void_p()
            check(lib.bpf_ctx_create(C.byref(h), C.c_void_p(torch.cuda.current_stream().cuda_stream)), None)
            ctx = h
            _ctxs[dev] = ctx
    stream = torch.cuda.current_stream(dev).cuda_stream
    lib.bpf_ctx_set_stream(ctx, C.c_void_p(stream))
    return ctx


def last_error(ctx) -> str:
    if ctx is None:
        return ""
    msg = load().bpf_last_error(ctx)
    return msg.decode() if msg else ""


def check(status: int, ctx) -> None:
    if status == BPF_SUCCESS:
        return
    msg = last_error(ctx) or f"libbpf status {status}"
    if status == BPF_ERR_DIMENSION:
        raise DimensionMismatch(status, msg)
    if status == BPF_ERR_SINGULAR:
        raise SingularException(status, msg)
    raise BPFError(status, msg)


def kernel_launches(device=None) -> int:
    return int(load().bpf_ctx_kernel_launches(context(device)))


KERNEL_CLASSES = {"spmm": 0, "trsv": 1, "factor": 2, "gram": 3, "tsmm": 4, "small": 5,
                  "chol": 6, "hess": 7, "backsub": 8, "mlp": 9, "batch": 10,
                  "pf": 11}


def set_timing(on: bool, device=None) -> None:
    ctx = context(device)
    check(load().bpf_ctx_set_timing(ctx, int(bool(on))), ctx)


def kernel_time(kernel_class: str, device=None):
    """(total ms, launches, algorithmic bytes, flops) of a kernel class since set_timing(True)."""
    ctx = context(device)
    t, c, b, f = C.c_double(), C.c_longlong(), C.c_double(), C.c_double()
    check(load().bpf_ctx_kernel_time(ctx, KERNEL_CLASSES[kernel_class], C.byref(t), C.byref(c),
                                     C.byref(b), C.byref(f)), ctx)
    return t.value, c.value, b.value, f.value
