"""bpf_prec_apply_noalloc, the preconditioner apply for callers that cannot allocate device
memory after set-up (hosts whose device memory belongs to an external pool or a fixed arena,
real-time loops that forbid allocation).

It must give what bpf_prec_apply gives (same kernels, so the same bits; checked to the 1e-12
relative tolerance of the other triangular-solve tests) on two calls in a row, since the calls
share one static scratch array; it must leave the device's free memory unchanged once its first
call has run; and it must reject blocks larger than that array, and blocks wider than a reordered
preconditioner's own scratch, without allocating.  Called through the C ABI with ctypes.  Kept in
a file of its own that pytest collects last.
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


def _free_bytes():
    import torch

    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _check_two_calls(bpf, P, X):
    """bpf_prec_apply's result, then two noalloc calls in a row that must match it; the second
    call must not change the device's free memory (the first may load the library's module)."""
    st, ref = _apply(bpf, "bpf_prec_apply", P, X)
    assert st == 0, bpf._lib.last_error(P._ctx)
    ref = ref.cpu().numpy()
    scale = np.abs(ref).max()
    Ys = [bpf.empty_colmajor(X.shape[0], X.shape[1]) for _ in range(2)]
    lib = bpf._lib.load()
    for k, Y in enumerate(Ys):
        free0 = _free_bytes()
        st = lib.bpf_prec_apply_noalloc(P.handle, X.shape[1], X.data_ptr(), X.stride(1), Y.data_ptr(),
                                        Y.stride(1))
        free1 = _free_bytes()
        assert st == 0, bpf._lib.last_error(P._ctx)
        if k == 1:
            assert free1 == free0, (free0, free1)
        np.testing.assert_allclose(Y.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * scale)


@pytest.mark.parametrize("grid,p", [("case300", 16), ("case9k", 48), ("case300", 300)])
def test_noalloc_apply_matches_prec_apply(bpf, grid, p):
    import torch

    A = bpf.grid.preset_jacobian(grid, 0)
    Ad = bpf.CuSparseMatrixCSR.from_scipy(A)
    P = bpf.ilu0(Ad, p)
    X = bpf.colmajor(torch.as_tensor(np.random.default_rng(p).standard_normal((A.shape[0], p)),
                                     device="cuda"))
    _check_two_calls(bpf, P, X)


@pytest.mark.parametrize("factor_dtype", ["float64", "float32"])
def test_noalloc_apply_reordered_preconditioner(bpf, factor_dtype):
    """Minimum-degree ILU(0) created for nrhs = 24 columns: 24 columns match bpf_prec_apply; 25
    columns exceed its factor-ordered scratch, which this entry point never grows, and are
    rejected without an allocation."""
    import torch

    A = bpf.grid.preset_jacobian("case300", 0)
    P = bpf.ilu0(bpf.CuSparseMatrixCSR.from_scipy(A), 24, factor_dtype=factor_dtype, ordering="AMD")
    rng = np.random.default_rng(11)
    X = bpf.colmajor(torch.as_tensor(rng.standard_normal((A.shape[0], 24)), device="cuda"))
    _check_two_calls(bpf, P, X)
    X25 = bpf.colmajor(torch.as_tensor(rng.standard_normal((A.shape[0], 25)), device="cuda"))
    Y = bpf.empty_colmajor(A.shape[0], 25)
    free0 = _free_bytes()
    st = bpf._lib.load().bpf_prec_apply_noalloc(P.handle, 25, X25.data_ptr(), X25.stride(1), Y.data_ptr(),
                                                Y.stride(1))
    assert _free_bytes() == free0
    assert st == bpf._lib.BPF_ERR_NOT_SUPPORTED
    assert "bpf_prec_apply_noalloc" in bpf._lib.last_error(P._ctx)


def test_noalloc_apply_block_jacobi(bpf):
    """The block-Jacobi preconditioner (mul! semantics), applied in place on the static array."""
    import torch

    A = bpf.grid.preset_jacobian("case300", 0)
    P = bpf.BlockJacobiPreconditioner(bpf.CuSparseMatrixCSR.from_scipy(A), 32)
    X = bpf.colmajor(torch.as_tensor(np.random.default_rng(4).standard_normal((A.shape[0], 40)),
                                     device="cuda"))
    _check_two_calls(bpf, P, X)


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
    _check_two_calls(bpf, P, X)


def test_noalloc_apply_rejects_oversized_block(bpf):
    import torch

    A = bpf.grid.preset_jacobian("case9k", 0)   # 16,998 unknowns: 64 columns need 1.09M doubles
    P = bpf.ilu0(bpf.CuSparseMatrixCSR.from_scipy(A), 64)
    X = bpf.colmajor(torch.zeros((A.shape[0], 64), dtype=torch.float64, device="cuda"))
    free0 = _free_bytes()
    st, _ = _apply(bpf, "bpf_prec_apply_noalloc", P, X)
    assert _free_bytes() == free0
    assert st == bpf._lib.BPF_ERR_NOT_SUPPORTED
    assert "static scratch" in bpf._lib.last_error(P._ctx)
