"""ILU(0) / IC(0) preconditioners: ilu0, ic0, ldiv! (src/preconditioners_nvidia.jl); and the
block-Jacobi preconditioner the reference's tests use (ExaPF's BlockJacobiPreconditioner)."""
from __future__ import annotations

import ctypes as C

from . import _lib
from .sparse import CuSparseMatrixCSR, colmajor, empty_colmajor, ld


class _DevicePrec:
    kind = ""

    def __init__(self, A: CuSparseMatrixCSR, nrhs: int, factor_dtype: str, creator: str,
                 ordering: str = "natural"):
        self.A = A
        self.n = A.n
        self.nrhs = int(nrhs)
        self.factor_dtype = factor_dtype
        fd = _lib.BPF_F32 if factor_dtype in ("float32", "f32", "Float32") else _lib.BPF_F64
        key = ordering.lstrip(":").upper() if isinstance(ordering, str) else ordering
        if key not in _lib.ORDERINGS:
            raise ValueError(f"unknown ordering {ordering!r}")
        self.ordering = key
        lib = _lib.load()
        self._ctx = _lib.context(A.nzVal.device.index)
        h = C.c_void_p()
        d = A.desc()
        if key == "NATURAL":
            rc = getattr(lib, creator)(self._ctx, C.byref(d), self.nrhs, fd, C.byref(h))
        else:
            rc = getattr(lib, creator + "_ordered")(self._ctx, C.byref(d), self.nrhs, fd,
                                                    _lib.ORDERINGS[key], C.byref(h))
        _lib.check(rc, self._ctx)
        self._h = h

    @property
    def perm(self):
        """perm[i] = the row of A that is row i of the factors (identity when natural)."""
        import numpy as np

        p = np.zeros(self.n, dtype=np.int32)
        _lib.check(_lib.load().bpf_prec_permutation(self._h, p.ctypes.data_as(C.c_void_p)), self._ctx)
        return p

    @property
    def handle(self):
        return self._h

    def levels(self):
        lo, up = C.c_int(), C.c_int()
        _lib.check(_lib.load().bpf_prec_levels(self._h, C.byref(lo), C.byref(up)), self._ctx)
        return lo.value, up.value

    @property
    def P(self):
        """The factor values on A's pattern (NVIDIA_ILU0.P / NVIDIA_IC0.P); for a reordered
        preconditioner, on the pattern of A(perm, perm) (0-based)."""
        import numpy as np
        import torch

        v = torch.empty(self.A.nnz, dtype=torch.float64, device=self.A.nzVal.device)
        _lib.check(_lib.load().bpf_prec_factor_values(self._h, v.data_ptr()), self._ctx)
        if self.ordering == "NATURAL":
            return CuSparseMatrixCSR(self.A.rowPtr, self.A.colVal, v, self.n, self.A.index_base)
        import scipy.sparse as sp

        S = self.A.to_scipy()
        perm = self.perm
        Sh = S[perm][:, perm].tocsr()
        Sh.sort_indices()
        dev = self.A.nzVal.device
        return CuSparseMatrixCSR(torch.as_tensor(Sh.indptr.astype(np.int32), device=dev),
                                 torch.as_tensor(Sh.indices.astype(np.int32), device=dev), v,
                                 self.n, 0)

    def refactor(self, vals) -> None:
        """New values on the same pattern, then the numeric factorization again."""
        _lib.check(_lib.load().bpf_prec_refactor(self._h, vals.data_ptr()), self._ctx)

    def ldiv(self, x):
        y = empty_colmajor(x.shape[0], 1 if x.dim() == 1 else x.shape[1], x.device)
        ldiv_(y, self, x)
        return y if x.dim() == 2 else y[:, 0]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().bpf_prec_destroy(h)
            except Exception:
                pass
            self._h = None


class NVIDIA_ILU0(_DevicePrec):
    kind = "ilu0"


class NVIDIA_IC0(_DevicePrec):
    kind = "ic0"


def ilu0(A: CuSparseMatrixCSR, nrhs: int = 1, factor_dtype: str = "float64",
         ordering: str = "natural") -> NVIDIA_ILU0:
    """ilu0(A, nrhs) (src/preconditioners_nvidia.jl:42-47).  ordering="RCM" / "AMD" factors
    A(perm, perm) instead (an addition: the reference factors A in its natural order)."""
    return NVIDIA_ILU0(A, nrhs, factor_dtype, "bpf_ilu0_create", ordering)


def ic0(A: CuSparseMatrixCSR, nrhs: int = 1, factor_dtype: str = "float64",
        ordering: str = "natural") -> NVIDIA_IC0:
    """ic0(A, nrhs) (src/preconditioners_nvidia.jl:6-11); ordering as for ilu0."""
    return NVIDIA_IC0(A, nrhs, factor_dtype, "bpf_ic0_create", ordering)


def ldiv_(y, P: _DevicePrec, x):
    """ldiv!(y, P, x): y = P \\ x (vector or matrix x).  y must be a column-major block."""
    vec = x.dim() == 1
    xc = colmajor(x)
    yc = y.reshape(-1, 1) if vec else y
    n, p = xc.shape
    if n != P.n or tuple(yc.shape) != (n, p):
        raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "Inconsistent problem size")
    if not (yc.stride(0) == 1):
        raise ValueError("y must be column-major (Fortran order)")
    _lib.check(_lib.load().bpf_prec_apply(P.handle, p, xc.data_ptr(), ld(xc), yc.data_ptr(),
                                          ld(yc)), P._ctx)
    return y


class BlockJacobiPreconditioner:
    """ExaPF's LinearSolvers.BlockJacobiPreconditioner(A, nblocks, device) as the reference's
    tests and benchmark use it (test/block_gmres.jl:5,17,22; benchmarks_nvidia.jl:47-51): the
    dense inverses of the diagonal blocks, applied by mul! (y = P x), so block_gmres takes it with
    ldiv=False.  Blocks are consecutive runs of block_size rows (default: ceil(n / nblocks), at
    most 32) in `ordering` (ExaPF partitions with METIS, which is not available here).
    update(A) recomputes the inverses from A's current values (ExaPF's LS.update)."""

    kind = "block_jacobi"

    def __init__(self, A: CuSparseMatrixCSR, nblocks: int | None = None, *, block_size: int | None = None,
                 ordering: str = "natural"):
        n = A.n
        if block_size is None:
            nb = max(1, int(nblocks)) if nblocks else max(1, n // 32)
            block_size = min(32, -(-n // nb))
        key = ordering.lstrip(":").upper() if isinstance(ordering, str) else ordering
        if key not in _lib.ORDERINGS:
            raise ValueError(f"unknown ordering {ordering!r}")
        self.A, self.n, self.block_size, self.ordering = A, n, int(block_size), key
        lib = _lib.load()
        self._ctx = _lib.context(A.nzVal.device.index)
        h = C.c_void_p()
        d = A.desc()
        _lib.check(lib.bpf_block_jacobi_create(self._ctx, C.byref(d), self.block_size, _lib.ORDERINGS[key],
                                               C.byref(h)), self._ctx)
        self._h = h

    @property
    def handle(self):
        return self._h

    @property
    def order(self):
        """The row order the blocks are cut from."""
        import numpy as np

        p = np.zeros(self.n, dtype=np.int32)
        _lib.check(_lib.load().bpf_prec_permutation(self._h, p.ctypes.data_as(C.c_void_p)), self._ctx)
        return p

    def update(self, A: CuSparseMatrixCSR | None = None) -> None:
        A = self.A if A is None else A
        _lib.check(_lib.load().bpf_prec_refactor(self._h, C.c_void_p(A.nzVal.data_ptr())), self._ctx)

    def mul(self, x):
        """y = P x (a new column-major block)."""
        xc = colmajor(x)
        y = empty_colmajor(xc.shape[0], xc.shape[1], xc.device)
        return mul_(y, self, xc)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _lib.load().bpf_prec_destroy(h)
            except Exception:
                pass
            self._h = None


def mul_(y, P: BlockJacobiPreconditioner, x):
    """mul!(y, P, x): y = P x for the block-Jacobi preconditioner."""
    xc = colmajor(x)
    n, p = xc.shape
    if n != P.n or tuple(y.shape) != (n, p) or y.stride(0) != 1:
        raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "Inconsistent problem size")
    _lib.check(_lib.load().bpf_prec_apply(P.handle, p, xc.data_ptr(), ld(xc), y.data_ptr(), ld(y)), P._ctx)
    return y
