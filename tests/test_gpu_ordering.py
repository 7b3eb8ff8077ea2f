"""Reordered ILU(0) / IC(0) (bpf_ilu0_create_ordered): the factors of A(perm, perm), applied
with ldiv! semantics in A's own ordering, y = P' (L U)^{-1} P x.

Parity: the oracle's ILU(0) / IC(0) of A(perm, perm) (csrilu02 / csric02 semantics,
src/preconditioners_nvidia.jl:6-11,42-71) with the permutation the library reports, to the
1e-12 relative tolerance of the other triangular-solve tests.  The reference factors A in its
natural order only; the orderings are the RF analysis's (src/cusolverRF.jl:70-95).
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from conftest import spd_from

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bpf():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import blockpowerflow_b200 as bpf

    return bpf


def _oracle_apply(kind, A, perm, X):
    Ah = A[perm][:, perm].tocsr()
    Ah.sort_indices()
    F = O.ilu0(Ah) if kind == 1 else O.ic0(Ah)
    Yh = O.prec_apply(kind, F, X[perm])
    Y = np.empty_like(Yh)
    Y[perm] = Yh
    return Y


@pytest.mark.parametrize("grid,ordering,p", [("case300", "RCM", 16), ("case300", "AMD", 5),
                                             ("case9k", "RCM", 64), ("case9k", "AMD", 33)])
def test_ordered_ilu0_apply_matches_oracle(bpf, grid, ordering, p):
    import torch

    A = bpf.grid.preset_jacobian(grid, 0)
    N = bpf.ilu0(bpf.CuSparseMatrixCSR.from_scipy(A), p, ordering=ordering)
    perm = N.perm
    assert sorted(perm.tolist()) == list(range(A.shape[0]))
    assert not np.array_equal(perm, np.arange(A.shape[0]))
    X = np.random.default_rng(p).standard_normal((A.shape[0], p))
    Y = N.ldiv(torch.as_tensor(X, device="cuda")).cpu().numpy()
    Yo = _oracle_apply(1, A, perm, X)
    np.testing.assert_allclose(Y, Yo, rtol=1e-12, atol=1e-12 * np.abs(Yo).max())


def test_ordered_ic0_apply_matches_oracle(case300, bpf):
    import torch

    A = spd_from(case300[0])
    N = bpf.ic0(bpf.CuSparseMatrixCSR.from_scipy(A), 8, ordering="RCM")
    X = np.random.default_rng(3).standard_normal((A.shape[0], 8))
    Y = N.ldiv(torch.as_tensor(X, device="cuda")).cpu().numpy()
    Yo = _oracle_apply(2, A, N.perm, X)
    np.testing.assert_allclose(Y, Yo, rtol=1e-12, atol=1e-12 * np.abs(Yo).max())


def test_ordered_refactor_and_factor_values(bpf):
    """New values on the same pattern go through the entry map; .P holds the factors of
    A(perm, perm) on its own pattern."""
    import torch

    gr = bpf.grid.make_grid(300, 68, seed=0)
    A = bpf.grid.jacobian(gr)
    Ad = bpf.CuSparseMatrixCSR.from_scipy(A)
    N = bpf.ilu0(Ad, 4, ordering="RCM")
    v2 = bpf.grid.perturbed_values(gr, A, 3, sigma=0.01, seed=1)
    Ad.nzVal.copy_(torch.as_tensor(v2))
    N.refactor(Ad.nzVal)
    A2 = A.copy()
    A2.data = v2
    perm = N.perm
    X = np.random.default_rng(5).standard_normal((A.shape[0], 4))
    Y = N.ldiv(torch.as_tensor(X, device="cuda")).cpu().numpy()
    Yo = _oracle_apply(1, A2, perm, X)
    np.testing.assert_allclose(Y, Yo, rtol=1e-12, atol=1e-12 * np.abs(Yo).max())
    Ah = A2[perm][:, perm].tocsr()
    Ah.sort_indices()
    Fo = O.ilu0(Ah)
    Fd = N.P.to_scipy()
    np.testing.assert_allclose(Fd.data, Fo.data, rtol=1e-11, atol=1e-11 * np.abs(Fo.data).max())


def test_ordered_scratch_grows_past_nrhs(case300, bpf):
    import torch

    A = case300[0]
    N = bpf.ilu0(bpf.CuSparseMatrixCSR.from_scipy(A), 2, ordering="RCM")
    X = np.random.default_rng(11).standard_normal((A.shape[0], 40))
    Y = N.ldiv(torch.as_tensor(X, device="cuda")).cpu().numpy()
    np.testing.assert_allclose(Y, _oracle_apply(1, A, N.perm, X), rtol=1e-12, atol=1e-10)


def test_ordered_noalloc_uses_the_reserved_scratch(case300, bpf):
    """The allocation-free apply works within the columns reserved at creation (nrhs) and
    refuses wider blocks instead of allocating."""
    import torch

    A = case300[0]
    N = bpf.ilu0(bpf.CuSparseMatrixCSR.from_scipy(A), 8, ordering="RCM")
    lib = bpf._lib.load()
    X = bpf.colmajor(torch.as_tensor(np.random.default_rng(2).standard_normal((A.shape[0], 8)),
                                     device="cuda"))
    Y = bpf.empty_colmajor(A.shape[0], 8)
    st = lib.bpf_prec_apply_noalloc(N.handle, 8, X.data_ptr(), X.stride(1), Y.data_ptr(), Y.stride(1))
    assert st == 0
    np.testing.assert_allclose(Y.cpu().numpy(), _oracle_apply(1, A, N.perm, X.cpu().numpy()),
                               rtol=1e-12, atol=1e-10)
    X2 = bpf.colmajor(torch.zeros((A.shape[0], 9), dtype=torch.float64, device="cuda"))
    Y2 = bpf.empty_colmajor(A.shape[0], 9)
    st = lib.bpf_prec_apply_noalloc(N.handle, 9, X2.data_ptr(), X2.stride(1), Y2.data_ptr(), Y2.stride(1))
    assert st == bpf._lib.BPF_ERR_NOT_SUPPORTED


def test_gmres_with_rcm_ilu0_converges_in_fewer_iterations(bpf):
    """9,000-bus grid, 64 RHS, rtol 1e-8: the RCM-ordered ILU(0) cuts the iterations of
    right-preconditioned block-GMRES at the same true relative residual."""
    import torch

    A = bpf.grid.jacobian(bpf.grid.make_grid(9000, 1000, seed=0))
    B = bpf.grid.gaussian_rhs(A.shape[0], 64, 1000)
    Ad = bpf.CuSparseMatrixCSR.from_scipy(A)
    Bd = torch.as_tensor(B, device="cuda")
    its = {}
    for ordering in ("natural", "RCM"):
        N = bpf.ilu0(Ad, 64, ordering=ordering)
        X, st = bpf.block_gmres(Ad, Bd, N=N, ldiv=True, restart=False, memory=300, atol=0.0,
                                rtol=1e-8, itmax=300)
        Xh = X.cpu().numpy()
        assert st.solved
        assert np.linalg.norm(B - A @ Xh) / np.linalg.norm(B) <= 1e-8
        its[ordering] = st.niter
    assert its["RCM"] < its["natural"], its
