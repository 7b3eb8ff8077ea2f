"""CUSOLVERRF: sparse LU analyse once, refactor on a fixed pattern, multi-RHS solve.

Mirrors the reference's submodule CUSOLVERRF (src/cusolverRF.jl): CusolverRfLU,
CusolverRfLUBatch, update!, ldiv!, solve!, lu / lu!, rf_batch_refactor!, cudestroy!.
Julia's bang functions are spelled with a trailing underscore (update_, ldiv_, ...).

Differences from the reference, by design:
  * nrhs > 1 is accepted by CusolverRfLU (the reference errors at :228-230): every column is
    solved with the one factorization;
  * a zero pivot in the analysis raises SingularException (the reference builds the exception
    at :164-166 but never throws it);
  * ordering :METIS raises (no METIS library in this build); :AMD and :MDQ use the same
    minimum-degree ordering.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .sparse import CuSparseMatrixCSR, colmajor, empty_colmajor, ld


class _RfBase:
    def __init__(self, A: CuSparseMatrixCSR, batch: int, ordering: str, tol: float,
                 fast_mode: bool):
        if A.shape[0] != A.shape[1]:
            raise AssertionError("only square matrices are supported")
        key = ordering.lstrip(":").upper() if isinstance(ordering, str) else ordering
        if key not in _lib.ORDERINGS:
            raise ValueError(f"unknown ordering {ordering!r}")
        self.n = A.n
        self.m = A.n
        self.nnzA = A.nnz
        self.batchsize = int(batch)
        self._ctx = _lib.context(A.nzVal.device.index)
        h = C.c_void_p()
        d = A.desc()
        _lib.check(_lib.load().bpf_rf_analyze(self._ctx, C.byref(d), _lib.ORDERINGS[key],
                                              float(tol), int(bool(fast_mode)), int(batch),
                                              C.byref(h)), self._ctx)
        self._h = h

    @property
    def handle(self):
        return self._h

    def info(self):
        nl, nu = C.c_int(), C.c_int()
        P = np.zeros(self.n, dtype=np.int32)
        Q = np.zeros(self.n, dtype=np.int32)
        _lib.check(_lib.load().bpf_rf_info(self._h, C.byref(nl), C.byref(nu),
                                           P.ctypes.data_as(C.c_void_p),
                                           Q.ctypes.data_as(C.c_void_p)), self._ctx)
        return dict(nnzL=nl.value, nnzU=nu.value, P=P, Q=Q)

    def _solve_inplace(self, X):
        if X.stride(0) != 1:
            raise ValueError("X must be a column-major block")
        n, p = X.shape
        _lib.check(_lib.load().bpf_rf_solve(self._h, p, X.data_ptr(), ld(X)), self._ctx)

    def solve_refined(self, A: CuSparseMatrixCSR, B, steps: int = 1):
        """X = A \\ B with `steps` rounds of iterative refinement on the refactored LU (A: the
        matrix of the last update!, with its current values).  An addition: the reference's
        ldiv! applies the LU once."""
        Bc = colmajor(B)
        n, p = Bc.shape
        X = empty_colmajor(n, p, Bc.device)
        d = A.desc()
        _lib.check(_lib.load().bpf_rf_solve_refined(self._h, C.byref(d), p, Bc.data_ptr(), ld(Bc), X.data_ptr(),
                                                    ld(X), int(steps)), self._ctx)
        return X

    def destroy(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.load().bpf_rf_destroy(h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class CusolverRfLU(_RfBase):
    """CusolverRfLU(A; nrhs=1, ordering=:AMD, tol=1e-8, fast_mode=true) (:222-301)."""

    def __init__(self, A: CuSparseMatrixCSR, nrhs: int = 1, ordering: str = "AMD",
                 tol: float = 1e-8, fast_mode: bool = True):
        super().__init__(A, 1, ordering, tol, fast_mode)
        self.nrhs = int(nrhs)


class CusolverRfLUBatch(_RfBase):
    """CusolverRfLUBatch(A, batchsize; ordering=:AMD, tol=1e-8, fast_mode=false) (:336-419)."""

    def __init__(self, A: CuSparseMatrixCSR, batchsize: int, ordering: str = "AMD",
                 tol: float = 1e-8, fast_mode: bool = False):
        if batchsize == 1:
            raise ValueError("Please specify a number of batch greater than 1 for `CuSolverRfLUBatch`")
        super().__init__(A, batchsize, ordering, tol, fast_mode)


def update_(rflu: _RfBase, A: CuSparseMatrixCSR) -> None:
    """update!(rflu, A): new values on the same pattern, then refactor (:304-314, :422-434)."""
    _lib.check(_lib.load().bpf_rf_refactor(rflu.handle, A.nzVal.data_ptr()), rflu._ctx)


def rf_batch_refactor_(rflu: CusolverRfLUBatch, Anzval) -> None:
    """rf_batch_refactor!(rflu, Anzval::CuMatrix): replica r takes column r (:472-481)."""
    V = colmajor(Anzval)
    if tuple(V.shape) != (rflu.nnzA, rflu.batchsize):
        raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "Anzval must be nnz x batchsize")
    _lib.check(_lib.load().bpf_rf_refactor_batch(rflu.handle, V.data_ptr(), ld(V)), rflu._ctx)


def ldiv_(*args):
    """ldiv!(x, rflu, b) or ldiv!(rflu, x) (:317-331, :451-470)."""
    import torch

    if len(args) == 3:
        x, rflu, b = args
        vec = b.dim() == 1
        bc = colmajor(b)
        xv = x.reshape(-1, 1) if vec else x
        if xv.stride(0) != 1:
            raise ValueError("x must be column-major")
        if tuple(xv.shape) != tuple(bc.shape):
            raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "size(x) != size(b)")
        if isinstance(rflu, CusolverRfLUBatch) and bc.shape[1] != rflu.batchsize:
            raise AssertionError("size(x, 2) == size(b, 2) == rflu.batchsize")
        if xv.data_ptr() != bc.data_ptr():
            xv.copy_(bc)
        rflu._solve_inplace(xv)
        return x
    rflu, x = args
    xv = x.reshape(-1, 1) if x.dim() == 1 else x
    if isinstance(rflu, CusolverRfLUBatch) and xv.shape[1] != rflu.batchsize:
        raise AssertionError("size(X, 2) == rflu.batchsize")
    rflu._solve_inplace(xv)
    return x


def solve_(X: list, rflu: CusolverRfLUBatch, B: list) -> None:
    """solve!(X::Vector{CuVector}, rflu, B::Vector{CuVector}) (:439-449)."""
    import torch

    if len(X) != rflu.batchsize or len(B) != rflu.batchsize:
        raise AssertionError("one vector per batch replica")
    M = torch.stack([b.to(torch.float64) for b in B], dim=1)
    Mc = M.t().contiguous().t()
    rflu._solve_inplace(Mc)
    for i, x in enumerate(X):
        x.copy_(Mc[:, i])


def lu(A: CuSparseMatrixCSR, **options) -> CusolverRfLU:
    """lu(A::AbstractCuSparseMatrix; options...) (:333)."""
    return CusolverRfLU(A, **options)


def lu_(rflu: _RfBase, A: CuSparseMatrixCSR) -> None:
    """lu!(rflu, A) (:334, :436)."""
    update_(rflu, A)


def cudestroy_(rflu: _RfBase) -> None:
    """cudestroy!(rflu) (:54)."""
    rflu.destroy()
