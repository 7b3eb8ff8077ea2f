"""MatrixMarket ingest of the reference's on-disk cases.

The reference's data are MatrixMarket files: the Jacobian of `data/case300.txt` (real general,
530 x 530) and the benchmark dumps `benchmarks/dump/Gx_<case>.mtx` (the n x n Jacobian Gx) with
`Gu_<case>.mtx` (the n x p right-hand sides Gu), which benchmarks/benchmarks_nvidia.jl:29-39 reads
with `mmread`, densifies B = Matrix(Gu) and moves both to the GPU.  This module does the same on
the host (SciPy's reader), hands the Jacobian to the library as a CuSparseMatrixCSR and Gu as a
column-major device block, and runs the benchmark script's solve with its parameters.
"""
from __future__ import annotations

import os

import numpy as np
import scipy.sparse as sp


def read_mtx(path: str, square: bool = True) -> sp.csr_matrix:
    """A real MatrixMarket matrix as sorted CSR (FP64); raises ValueError for a complex,
    pattern-only or (with square=True) non-square file."""
    from scipy.io import mmread, mminfo

    rows, cols, _, fmt, field, _ = mminfo(path)
    if field not in ("real", "integer"):
        raise ValueError(f"{path}: MatrixMarket field {field!r} (real or integer expected)")
    if square and rows != cols:
        raise ValueError(f"{path}: {rows} x {cols} is not square")
    M = mmread(path)
    A = sp.csr_matrix(M, dtype=np.float64)
    A.sort_indices()
    return A


def read_dense_mtx(path: str) -> np.ndarray:
    """A MatrixMarket matrix (coordinate or array) densified, as B = Matrix(mmread(path))."""
    from scipy.io import mmread

    M = mmread(path)
    return np.asarray(M.todense() if sp.issparse(M) else M, dtype=np.float64)


def dump_paths(dump_dir: str, case: str) -> tuple[str, str]:
    """The benchmark dump pair of a case (benchmarks/benchmarks_nvidia.jl:30-31)."""
    return (os.path.join(dump_dir, f"Gx_{case}.mtx"), os.path.join(dump_dir, f"Gu_{case}.mtx"))


def load_dump(dump_dir: str, case: str) -> tuple[sp.csr_matrix, np.ndarray]:
    """(Gx, Gu) of a benchmark case on the host: Gx n x n CSR, Gu dense n x p."""
    pa, pb = dump_paths(dump_dir, case)
    A = read_mtx(pa)
    B = read_dense_mtx(pb)
    if B.ndim == 1:
        B = B[:, None]
    if B.shape[0] != A.shape[0]:
        raise ValueError(f"{case}: Gu has {B.shape[0]} rows, Gx is {A.shape[0]} x {A.shape[1]}")
    return A, B


def to_device(A: sp.csr_matrix, B: np.ndarray | None = None, device: str = "cuda"):
    """(CuSparseMatrixCSR, column-major device block or None), as CuSparseMatrixCSR(A) and
    CuMatrix(B) in the reference's script."""
    import torch

    from .sparse import CuSparseMatrixCSR, colmajor

    Ad = CuSparseMatrixCSR.from_scipy(A, device=device)
    Bd = colmajor(torch.as_tensor(B, device=device)) if B is not None else None
    return Ad, Bd


def solve_dump(A: sp.csr_matrix, B: np.ndarray, *, atol: float = 1e-10, rtol: float = 0.0,
               memory: int = 1, restart: bool = False, itmax: int = 50, ordering: str = "natural"):
    """The benchmark script's solve with a right ILU(0) (benchmarks_nvidia.jl:44,54-65):
    block_gmres(A, B; N=ilu0(A, p), ldiv=true, atol, rtol, memory, restart, itmax).  Returns
    (X on the host, stats, ||B - A X||_F)."""
    from . import krylov, precond

    Ad, Bd = to_device(A, B)
    N = precond.ilu0(Ad, B.shape[1], ordering=ordering)
    X, st = krylov.block_gmres(Ad, Bd, N=N, ldiv=True, atol=atol, rtol=rtol, memory=memory,
                               restart=restart, itmax=itmax)
    Xh = X.cpu().numpy()
    return Xh, st, float(np.linalg.norm(B - A @ Xh))
