"""Device CSR matrices and column-major dense blocks (CuSparseMatrixCSR / CuMatrix).

The reference receives ``A::CuSparseMatrixCSR{Float64,Cint}`` (1-based ``rowPtr``/``colVal``)
and ``B::CuMatrix{Float64}`` (column-major n x p).  Here a CSR matrix lives in three torch
CUDA tensors and dense blocks are torch tensors; column-major views are made at the boundary.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


class CuSparseMatrixCSR:
    """n x n CSR matrix in device memory (int32 indices, float64 values)."""

    def __init__(self, rowptr, colind, vals, n: int, index_base: int = 0):
        import torch

        self.rowPtr = rowptr
        self.colVal = colind
        self.nzVal = vals
        self.n = int(n)
        self.index_base = int(index_base)
        assert rowptr.dtype == torch.int32 and colind.dtype == torch.int32
        assert vals.dtype == torch.float64
        assert rowptr.is_cuda and colind.is_cuda and vals.is_cuda

    @classmethod
    def from_scipy(cls, A, device="cuda", index_base: int = 0):
        import scipy.sparse as sp
        import torch

        A = sp.csr_matrix(A)
        A.sort_indices()
        if A.shape[0] != A.shape[1]:
            raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "System must be square")
        rp = torch.as_tensor(np.asarray(A.indptr, dtype=np.int32) + index_base, device=device)
        ci = torch.as_tensor(np.asarray(A.indices, dtype=np.int32) + index_base, device=device)
        v = torch.as_tensor(np.asarray(A.data, dtype=np.float64), device=device)
        return cls(rp, ci, v, A.shape[0], index_base)

    @property
    def shape(self):
        return (self.n, self.n)

    @property
    def nnz(self) -> int:
        return int(self.nzVal.numel())

    def desc(self) -> _lib.CsrDesc:
        return _lib.CsrDesc(self.n, self.nnz, self.rowPtr.data_ptr(), self.colVal.data_ptr(),
                            self.nzVal.data_ptr(), self.index_base, _lib.BPF_F64)

    def to_scipy(self):
        import scipy.sparse as sp

        rp = self.rowPtr.cpu().numpy() - self.index_base
        ci = self.colVal.cpu().numpy() - self.index_base
        return sp.csr_matrix((self.nzVal.cpu().numpy(), ci, rp), shape=self.shape)

    def __matmul__(self, X):
        return mul(self, X)


def colmajor(X, device=None):
    """Return a column-major (Fortran-order) float64 CUDA view/copy of a 2-D block."""
    import torch

    if not isinstance(X, torch.Tensor):
        X = torch.as_tensor(np.asarray(X, dtype=np.float64))
    if X.dim() == 1:
        X = X.reshape(-1, 1)
    if device is None:
        device = "cuda"
    X = X.to(device=device, dtype=torch.float64)
    n, p = X.shape
    if X.stride(0) == 1 and (X.stride(1) >= max(1, n) or p == 1):
        return X
    return X.t().contiguous().t()


def empty_colmajor(n: int, p: int, device="cuda"):
    import torch

    return torch.empty((p, n), dtype=torch.float64, device=device).t()


def ld(X) -> int:
    n, p = X.shape
    return max(1, X.stride(1) if p > 1 else n)


def mul(A: CuSparseMatrixCSR, X, alpha: float = 1.0, beta: float = 0.0, Y=None):
    """mul!(Y, A, X, alpha, beta) on the device (CSR SpMM)."""
    Xc = colmajor(X)
    n, p = Xc.shape
    if n != A.n:
        raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "Inconsistent problem size")
    if Y is None:
        Y = empty_colmajor(n, p, Xc.device)
        beta = 0.0
    lib = _lib.load()
    ctx = _lib.context(Xc.device.index)
    d = A.desc()
    _lib.check(lib.bpf_spmm(ctx, C.byref(d), p, alpha, Xc.data_ptr(), ld(Xc), beta,
                            Y.data_ptr(), ld(Y)), ctx)
    return Y


def householder(A, compact: bool = False, lapack: bool = True):
    """householder(A; compact) on an n x p device block (src/block_utils.jl:38-53): returns
    (Q, R) with LAPACK's conventions -- Q^T Q = I and Q R = A (orgqr's Q), or with compact=True
    geqrf's compact form in Q (R above, the reflector vectors below the diagonal); the
    reflectors' tau are kept as the attribute `householder.tau` of the last call.  lapack=False
    returns the Cholesky-QR2 factors themselves (R with a positive diagonal).  A is not
    modified."""
    import torch

    Qc = colmajor(A)
    if Qc.data_ptr() == getattr(A, "data_ptr", lambda: None)():
        Qc = Qc.t().contiguous().t()
    n, p = Qc.shape
    R = torch.zeros((p, p), dtype=torch.float64, device=Qc.device).t()
    lib = _lib.load()
    ctx = _lib.context(Qc.device.index)
    if not lapack:
        if compact:
            raise ValueError("compact=True needs the LAPACK form (lapack=True)")
        _lib.check(lib.bpf_householder(ctx, n, p, Qc.data_ptr(), ld(Qc), R.data_ptr(), p), ctx)
        return Qc, R
    tau = torch.zeros(p, dtype=torch.float64, device=Qc.device)
    _lib.check(lib.bpf_householder_lapack(ctx, n, p, Qc.data_ptr(), ld(Qc), R.data_ptr(), p, tau.data_ptr(),
                                          int(bool(compact))), ctx)
    householder.tau = tau
    return Qc, R
