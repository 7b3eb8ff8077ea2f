"""bpf_prec_apply_noalloc, the preconditioner apply for callers that cannot allocate device
memory after set-up (stream capture, externally owned memory pools, allocation-free loops).

It must give what bpf_prec_apply gives (same kernels, so the same bits; checked to the 1e-12
relative tolerance of the other triangular-solve tests) on two calls in a row, since the calls
share one static scratch array, and reject blocks larger than that array.  Called through the
C ABI with ctypes.  Kept in a file of its own that pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bpf():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import blockpowerflow_b200 as bpf

    return bpf


def _apply(bpf, fn, P, X):
    Y = bpf.empty_colmajor(X.shape[0], X.shape[1])
    lib = bpf._lib.load()
    st = getattr(lib, fn)(P.handle, X.shape[1], X.data_ptr(), X.stride(1), Y.data_ptr(), Y.stride(1))
    return st, Y


@pytest.mark.parametrize("grid,p", [("case300", 16), ("case9k", 48), ("case300", 300)])
def test_noalloc_apply_matches_prec_apply(bpf, grid, p):
    import torch

    A = bpf.grid.preset_jacobian(grid, 0)
    Ad = bpf.CuSparseMatrixCSR.from_scipy(A)
    P = bpf.ilu0(Ad, p)
    X = bpf.colmajor(torch.as_tensor(np.random.default_rng(p).standard_normal((A.shape[0], p)),
                                     device="cuda"))
    st, ref = _apply(bpf, "bpf_prec_apply", P, X)
    assert st == 0
    ref = ref.cpu().numpy()
    scale = np.abs(ref).max()
    for _ in range(2):
        st, Y = _apply(bpf, "bpf_prec_apply_noalloc", P, X)
        assert st == 0, bpf._lib.last_error(P._ctx)
        np.testing.assert_allclose(Y.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * scale)


def test_noalloc_apply_ic0_two_calls(bpf):
    import scipy.sparse as sp
    import torch

    A = bpf.grid.preset_jacobian("case300", 0)
    S = abs(A) + abs(A).T
    S = sp.csr_matrix(S)
    S.setdiag(0)
    S.eliminate_zeros()
    S = sp.csr_matrix(-S + sp.diags(np.asarray(abs(S).sum(axis=1)).ravel() + 1.0))
    S.sort_indices()
    P = bpf.ic0(bpf.CuSparseMatrixCSR.from_scipy(S), 8)
    X = bpf.colmajor(torch.as_tensor(np.random.default_rng(3).standard_normal((S.shape[0], 8)),
                                     device="cuda"))
    _, ref = _apply(bpf, "bpf_prec_apply", P, X)
    ref = ref.cpu().numpy()
    for _ in range(2):
        st, Y = _apply(bpf, "bpf_prec_apply_noalloc", P, X)
        assert st == 0
        np.testing.assert_allclose(Y.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_noalloc_apply_rejects_oversized_block(bpf):
    import torch

    A = bpf.grid.preset_jacobian("case9k", 0)   # 16,998 unknowns: 64 columns need 1.09M doubles
    P = bpf.ilu0(bpf.CuSparseMatrixCSR.from_scipy(A), 64)
    X = bpf.colmajor(torch.zeros((A.shape[0], 64), dtype=torch.float64, device="cuda"))
    st, _ = _apply(bpf, "bpf_prec_apply_noalloc", P, X)
    assert st == bpf._lib.BPF_ERR_NOT_SUPPORTED
    assert "static scratch" in bpf._lib.last_error(P._ctx)
