"""CUSOLVERRF replacement on the GPU: the reference's own known-answer tests
(test/cusolverRF.jl) plus multi-RHS, orderings and batch refactor.

Tolerance: isapprox's default rtol = sqrt(eps) as in the reference test, and 1e-10 norm-wise
relative agreement with the FP64 direct solve.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spl

import oracle as O

pytestmark = pytest.mark.gpu
RTOL = np.sqrt(np.finfo(np.float64).eps)


@pytest.fixture(scope="module")
def bpf():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import blockpowerflow_b200 as bpf

    return bpf


def _t(x):
    import torch

    return torch.as_tensor(np.asarray(x), device="cuda")


def test_rf_reference_known_answers(case300, bpf):
    """test/cusolverRF.jl:9-31: J \\ b, then nzVal *= 2 -> solution / 2."""
    RF = bpf.CUSOLVERRF
    A, z = case300
    b, x = z["b"], z["x"]
    gJ = bpf.CuSparseMatrixCSR.from_scipy(A, index_base=1)
    rflu = RF.CusolverRfLU(gJ, ordering="AMD")
    gx = _t(np.zeros_like(b))
    RF.ldiv_(gx, rflu, _t(b))
    np.testing.assert_allclose(gx.cpu().numpy(), x, rtol=RTOL)
    gJ.nzVal.mul_(2.0)
    RF.update_(rflu, gJ)
    RF.ldiv_(gx, rflu, _t(b))
    np.testing.assert_allclose(gx.cpu().numpy(), 0.5 * x, rtol=RTOL)
    RF.cudestroy_(rflu)


def test_rf_reference_batch_known_answers(case300, bpf):
    """test/cusolverRF.jl:34-70: batch 32, vector form and matrix form, i*b -> i*x."""
    import torch

    RF = bpf.CUSOLVERRF
    A, z = case300
    b, x = z["b"], z["x"]
    gJ = bpf.CuSparseMatrixCSR.from_scipy(A, index_base=1)
    nbatch = 32
    rflu = RF.CusolverRfLUBatch(gJ, nbatch)
    gB = [(i + 1) * _t(b) for i in range(nbatch)]
    gX = [torch.zeros_like(gB[0]) for _ in range(nbatch)]
    RF.solve_(gX, rflu, gB)
    for i in range(nbatch):
        np.testing.assert_allclose(gX[i].cpu().numpy(), (i + 1) * x, rtol=RTOL)
    RF.update_(rflu, gJ)
    gBm = bpf.colmajor(torch.stack(gB, dim=1))
    gXm = bpf.empty_colmajor(A.shape[0], nbatch)
    RF.ldiv_(gXm, rflu, gBm)
    for i in range(nbatch):
        np.testing.assert_allclose(gXm[:, i].cpu().numpy(), (i + 1) * x, rtol=RTOL)
    RF.cudestroy_(rflu)


@pytest.mark.parametrize("ordering", ["AMD", "MDQ", "RCM", "NATURAL"])
def test_rf_orderings_multi_rhs(case300, bpf, ordering):
    RF = bpf.CUSOLVERRF
    A, z = case300
    gJ = bpf.CuSparseMatrixCSR.from_scipy(A)
    rflu = RF.CusolverRfLU(gJ, ordering=ordering)
    B = np.random.default_rng(0).standard_normal((A.shape[0], 300))
    X = bpf.colmajor(_t(B)).clone()
    X = X.t().contiguous().t()
    RF.ldiv_(rflu, X)
    Xd = spl.splu(A.tocsc()).solve(B)
    assert np.linalg.norm(X.cpu().numpy() - Xd) <= 1e-10 * np.linalg.norm(Xd)
    info = rflu.info()
    assert sorted(info["P"]) == list(range(A.shape[0]))
    assert sorted(info["Q"]) == list(range(A.shape[0]))


def test_rf_metis_not_supported(case300, bpf):
    A, _ = case300
    with pytest.raises(bpf.BPFError):
        bpf.CUSOLVERRF.CusolverRfLU(bpf.CuSparseMatrixCSR.from_scipy(A), ordering="METIS")


def test_rf_singular_raises(bpf):
    import scipy.sparse as sp

    A = sp.csr_matrix(np.array([[1.0, 2.0, 0.0], [2.0, 4.0, 0.0], [0.0, 0.0, 1.0]]))
    with pytest.raises(bpf.SingularException):
        bpf.CUSOLVERRF.CusolverRfLU(bpf.CuSparseMatrixCSR.from_scipy(A))


def test_rf_refactor_sequence_synthetic(bpf):
    """Fixed pattern, perturbed operating points (third config at small size): refactor + solve."""
    import torch

    RF = bpf.CUSOLVERRF
    g = bpf.grid.make_grid(1000, 110, seed=3)
    A0 = bpf.grid.jacobian(g)
    gA = bpf.CuSparseMatrixCSR.from_scipy(A0)
    rflu = RF.CusolverRfLU(gA)
    B = np.random.default_rng(1).standard_normal((A0.shape[0], 64))
    for t in range(3):
        vals = bpf.grid.perturbed_values(g, A0, t)
        gA.nzVal.copy_(torch.as_tensor(vals, device="cuda"))
        RF.update_(rflu, gA)
        X = bpf.colmajor(_t(B)).t().contiguous().t()
        RF.ldiv_(rflu, X)
        At = A0.copy()
        At.data = vals
        Xd = spl.splu(At.tocsc()).solve(B)
        assert np.linalg.norm(X.cpu().numpy() - Xd) <= 1e-10 * np.linalg.norm(Xd)


def test_rf_batch_distinct_replicas(case300, bpf):
    """rf_batch_refactor!: replica r holds (r+1) * A, so column r of the solve is b / (r+1)."""
    import torch

    RF = bpf.CUSOLVERRF
    A, z = case300
    gJ = bpf.CuSparseMatrixCSR.from_scipy(A)
    nb = 4
    rflu = RF.CusolverRfLUBatch(gJ, nb)
    V = torch.stack([(r + 1) * gJ.nzVal for r in range(nb)], dim=1)
    RF.rf_batch_refactor_(rflu, V)
    b = z["b"]
    Bm = bpf.colmajor(torch.stack([_t(b)] * nb, dim=1))
    Xm = bpf.empty_colmajor(A.shape[0], nb)
    RF.ldiv_(Xm, rflu, Bm)
    for r in range(nb):
        np.testing.assert_allclose(Xm[:, r].cpu().numpy(), z["x"] / (r + 1), rtol=RTOL)


def test_rf_oracle_restatement_agrees(case300, bpf):
    """The device refactor and the oracle's dense pivoted LU give the same solution."""
    RF = bpf.CUSOLVERRF
    A, z = case300
    lu = O.DenseLU(A)
    B = np.random.default_rng(5).standard_normal((A.shape[0], 8))
    Xo = lu.solve(B)
    rflu = RF.CusolverRfLU(bpf.CuSparseMatrixCSR.from_scipy(A))
    X = bpf.colmajor(_t(B)).t().contiguous().t()
    RF.ldiv_(rflu, X)
    assert np.linalg.norm(X.cpu().numpy() - Xo) <= 1e-10 * np.linalg.norm(Xo)


def test_rf_refactor_without_stored_pairs_matches(bpf, monkeypatch):
    """The LU refactorization that finds each L entry's updates by a search in its row (used when
    the update pairs would exceed 2^31 - 1, forced here with BPF_LU_PAIRLESS=1) gives the same
    factor as the stored-pair kernel (to rounding: both add the updates atomically) and the same
    solves, on the 9,000-bus grid's perturbed operating points."""
    import torch

    RF = bpf.CUSOLVERRF
    g = bpf.grid.make_grid(9000, 1000, seed=0)
    A0 = bpf.grid.jacobian(g)
    B = np.random.default_rng(2).standard_normal((A0.shape[0], 8))
    gA = bpf.CuSparseMatrixCSR.from_scipy(A0)
    ref = RF.CusolverRfLU(gA)
    monkeypatch.setenv("BPF_LU_PAIRLESS", "1")
    gB = bpf.CuSparseMatrixCSR.from_scipy(A0)
    pl = RF.CusolverRfLU(gB)
    monkeypatch.delenv("BPF_LU_PAIRLESS")
    for t in range(2):
        vals = torch.as_tensor(bpf.grid.perturbed_values(g, A0, t), device="cuda")
        gA.nzVal.copy_(vals)
        gB.nzVal.copy_(vals)
        RF.update_(ref, gA)
        RF.update_(pl, gB)
        X1 = bpf.colmajor(_t(B)).t().contiguous().t()
        X2 = X1.clone()
        RF.ldiv_(ref, X1)
        RF.ldiv_(pl, X2)
        X1, X2 = X1.cpu().numpy(), X2.cpu().numpy()
        assert np.linalg.norm(X2 - X1) <= 1e-11 * np.linalg.norm(X1), t
        At = A0.copy()
        At.data = vals.cpu().numpy()
        Xd = spl.splu(At.tocsc()).solve(B)
        assert np.linalg.norm(X2 - Xd) <= 1e-10 * np.linalg.norm(Xd)
