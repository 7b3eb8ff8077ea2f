"""block_gmres / block_bicgstab with the reference's keyword arguments and stats types.

Mirrors src/block_gmres.jl:127-154 and src/block_bicgstab.jl:182-185: same argument
meaning, same defaults, same status strings, same error cases; the work runs in libbpf.so.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math

import numpy as np

from . import _lib
from .sparse import CuSparseMatrixCSR, colmajor, empty_colmajor, ld

_SQRT_EPS = math.sqrt(np.finfo(np.float64).eps)


@dataclasses.dataclass
class BlockGMRESStats:
    """BlockGMRESStats (src/block_utils.jl:62-68)."""
    niter: int
    solved: bool
    residuals: list
    timer: float
    status: str
    npass: int = 0


@dataclasses.dataclass
class SimpleStats:
    """SimpleStats (src/block_bicgstab.jl:15-21)."""
    niter: int
    solved: bool
    residuals: list
    timer: float
    status: str


def _status_string(code: int) -> str:
    return _lib.load().bpf_solve_status_string(code).decode()


def _prec_handle(P):
    if P is None:
        return None
    return P.handle


def block_gmres(A: CuSparseMatrixCSR, B, X0=None, *, memory: int = 20, M=None, N=None,
                ldiv: bool = False, restart: bool = False, reorthogonalization: bool = False,
                atol: float = _SQRT_EPS, rtol: float = _SQRT_EPS, itmax: int = 0,
                timemax: float = math.inf, verbose: int = 0, history: bool = False,
                deflation=None):
    """(X, stats) = block_gmres(A, B[, X0]; kwargs...)  (src/block_gmres.jl:127-154).

    M / N: left / right preconditioner (None = identity), applied with ldiv! when ldiv=True.
    deflation: an n x r basis (r <= p) to augment the Krylov space with (GCRO form); an
    addition of this build, typically the learned basis of learned.WarmStartMLP.basis.
    """
    Bc = colmajor(B)
    n, p = Bc.shape
    if A.n != n:
        raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "Inconsistent problem size")
    X = empty_colmajor(n, p, Bc.device)
    x0p, ldx0 = None, n
    if X0 is not None:
        X0c = colmajor(X0)
        if tuple(X0c.shape) != (n, p):
            raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, f"X0 should have size ({n}, {p})")
        x0p, ldx0 = X0c.data_ptr(), ld(X0c)
    lib = _lib.load()
    ctx = _lib.context(Bc.device.index)
    opts = _lib.GmresOpts(int(memory), int(bool(restart)), int(bool(reorthogonalization)),
                          int(bool(ldiv)), float(atol), float(rtol), int(itmax),
                          float(timemax) if math.isfinite(timemax) else 0.0, int(verbose),
                          int(bool(history)))
    cap = (int(itmax) if itmax else 2 * (n // max(p, 1))) + 2
    res = np.zeros(max(cap, 1))
    st = _lib.Stats(0, 0, 0, 0.0, 0, len(res), res.ctypes.data_as(C.POINTER(C.c_double)), 0)
    d = A.desc()
    if deflation is None:
        _lib.check(lib.bpf_block_gmres(ctx, C.byref(d), p, Bc.data_ptr(), ld(Bc), X.data_ptr(), ld(X),
                                       x0p, ldx0, _prec_handle(M), _prec_handle(N), C.byref(opts),
                                       C.byref(st)), ctx)
    else:
        Zc = colmajor(deflation)
        if Zc.shape[0] != n:
            raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "deflation basis must have n rows")
        _lib.check(lib.bpf_block_gmres_deflated(ctx, C.byref(d), p, Bc.data_ptr(), ld(Bc), X.data_ptr(),
                                                ld(X), x0p, ldx0, _prec_handle(M), _prec_handle(N),
                                                C.byref(opts), Zc.data_ptr(), ld(Zc), Zc.shape[1],
                                                C.byref(st)), ctx)
    stats = BlockGMRESStats(st.niter, bool(st.solved),
                            res[: min(st.n_residuals, len(res))].tolist() if history else [],
                            st.timer, _status_string(st.status), st.npass)
    return X, stats


def block_bicgstab(A: CuSparseMatrixCSR, B, *, C=None, N=None, atol: float = _SQRT_EPS,
                   rtol: float = _SQRT_EPS, itmax: int = 0, timemax: float = math.inf,
                   verbose: int = 0, history: bool = False):
    """(X, stats) = block_bicgstab(A, B; C=B, N, kwargs...)  (src/block_bicgstab.jl:182-299).

    N (None = identity) is applied as Y = N \\ P, the operation the reference's comment at
    src/block_bicgstab.jl:247 describes.
    """
    import ctypes

    Bc = colmajor(B)
    n, p = Bc.shape
    if A.n != n:
        raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "Inconsistent problem size")
    X = empty_colmajor(n, p, Bc.device)
    cp, ldc = None, n
    if C is not None:
        Cc = colmajor(C)
        if tuple(Cc.shape) != (n, p):
            raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "C should have the size of B")
        cp, ldc = Cc.data_ptr(), ld(Cc)
    lib = _lib.load()
    ctx = _lib.context(Bc.device.index)
    opts = _lib.BicgstabOpts(float(atol), float(rtol), int(itmax),
                             float(timemax) if math.isfinite(timemax) else 0.0, int(verbose),
                             int(bool(history)))
    cap = (int(itmax) if itmax else 2 * n) + 2
    res = np.zeros(max(cap, 1))
    st = _lib.Stats(0, 0, 0, 0.0, 0, len(res), res.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0)
    d = A.desc()
    _lib.check(lib.bpf_block_bicgstab(ctx, ctypes.byref(d), p, Bc.data_ptr(), ld(Bc), X.data_ptr(),
                                      ld(X), cp, ldc, _prec_handle(N), ctypes.byref(opts),
                                      ctypes.byref(st)), ctx)
    stats = SimpleStats(st.niter, bool(st.solved),
                        res[: min(st.n_residuals, len(res))].tolist() if history else [],
                        st.timer, _status_string(st.status))
    return X, stats


# ---- in-place forms: solver objects, block_gmres! / block_bicgstab!, warm_start! ----------------


def _device_of(B):
    """The solution block follows B (the reference allocates it with B's type); host arrays -> cuda."""
    import torch

    return B.device if isinstance(B, torch.Tensor) else torch.device("cuda")


class BlockGMRESSolver:
    """BlockGMRESSolver (src/block_gmres.jl:21-68): the block a solve writes its solution into
    (X, n x p, column-major), the statistics of the last solve, the basis size `memory` (clamped
    to div(n, p) as the reference does) and a pending warm start.  The Krylov basis and the small
    blocks live in the library's per-device context and are reused from solve to solve, so they
    are not fields here.  BlockGMRESSolver(A, B; memory=5), or from_sizes(m, n, p, memory)."""

    def __init__(self, A, B, *, memory: int = 5):
        m, n = A.shape
        s, p = B.shape
        self._init(m, n, p, memory, _device_of(B))

    @classmethod
    def from_sizes(cls, m: int, n: int, p: int, memory: int, device=None):
        """BlockGMRESSolver(m, n, p, memory, SV, SM)."""
        import torch

        self = cls.__new__(cls)
        self._init(m, n, p, memory, torch.device("cuda") if device is None else torch.device(device))
        return self

    def _init(self, m, n, p, memory, device):
        self.m, self.n, self.p = int(m), int(n), int(p)
        self.memory = min(n // max(p, 1), int(memory))
        self.device = device
        self.X = empty_colmajor(self.n, self.p, device)
        self.dX = None
        self.warm_start = False
        self.stats = BlockGMRESStats(0, False, [], 0.0, "unknown")


def warm_start_(solver: BlockGMRESSolver, X0) -> BlockGMRESSolver:
    """warm_start!(solver, X0) (src/block_gmres.jl:70-79): the next block_gmres_ starts from X0."""
    n, p = solver.n, solver.p
    if tuple(X0.shape) != (n, p):
        raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, f"X0 should have size ({n}, {p})")
    solver.dX = colmajor(X0, device=solver.device).clone()
    solver.warm_start = True
    return solver


def block_gmres_(solver: BlockGMRESSolver, A: CuSparseMatrixCSR, B, X0=None, *, M=None, N=None,
                 ldiv: bool = False, restart: bool = False, reorthogonalization: bool = False,
                 atol: float = _SQRT_EPS, rtol: float = _SQRT_EPS, itmax: int = 0,
                 timemax: float = math.inf, verbose: int = 0, history: bool = False) -> BlockGMRESSolver:
    """block_gmres!(solver, A, B[, X0]; kwargs...) (src/block_gmres.jl:97-411): the solve with
    the solver's basis size; the solution goes into solver.X, the statistics into solver.stats,
    and a warm start (X0 here or an earlier warm_start_) is consumed.  Returns the solver."""
    if X0 is not None:
        warm_start_(solver, X0)
    s, p = B.shape
    if (s, p) != (solver.n, solver.p):
        raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION,
                                     f"B is {s} x {p}, the solver was built for {solver.n} x {solver.p}")
    X, st = block_gmres(A, B, solver.dX if solver.warm_start else None, memory=solver.memory, M=M, N=N,
                        ldiv=ldiv, restart=restart, reorthogonalization=reorthogonalization, atol=atol,
                        rtol=rtol, itmax=itmax, timemax=timemax, verbose=verbose, history=history)
    solver.X.copy_(X)
    solver.stats = st
    solver.warm_start = False
    solver.dX = None
    return solver


class BlockBicgstabSolver:
    """BlockBicgstabSolver (src/block_bicgstab.jl:23-55): the solution block X (n x p,
    column-major) and the statistics of the last solve; the iteration's blocks live in the
    library's per-device context."""

    def __init__(self, A, B):
        n, m = A.shape
        s, p = B.shape
        self.n, self.p = int(n), int(p)
        self.device = _device_of(B)
        self.X = empty_colmajor(self.n, self.p, self.device)
        self.stats = SimpleStats(0, False, [], 0.0, "unknown")


def block_bicgstab_(solver: BlockBicgstabSolver, A: CuSparseMatrixCSR, B, *, C=None, N=None,
                    atol: float = _SQRT_EPS, rtol: float = _SQRT_EPS, itmax: int = 0,
                    timemax: float = math.inf, verbose: int = 0, history: bool = False):
    """block_bicgstab!(solver, A, B; C=B, N, kwargs...) (src/block_bicgstab.jl:187-299): the
    solution into solver.X, the statistics into solver.stats; returns (X, stats) as there."""
    s, p = B.shape
    if (s, p) != (solver.n, solver.p):
        raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION,
                                     f"B is {s} x {p}, the solver was built for {solver.n} x {solver.p}")
    X, st = block_bicgstab(A, B, C=C, N=N, atol=atol, rtol=rtol, itmax=itmax, timemax=timemax,
                           verbose=verbose, history=history)
    solver.X.copy_(X)
    solver.stats = st
    return solver.X, solver.stats
