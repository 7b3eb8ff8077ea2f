"""The CPU oracle pinned against the reference's own test cases and data (no GPU).

The reference's only assertions are the cusolverRF known-answer tests
(test/cusolverRF.jl:21,28,49-53,63-68) against the direct solve J \\ b; its block-solver
scripts run block_gmres / block_bicgstab on data/case300.txt with B = I[:, 1:32], atol 1e-8,
rtol 0, itmax 500 (test/block_gmres.jl:8-25) and print the status and ||B - J X||.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from conftest import spd_from


def test_oracle_spmm_matches_scipy(case300, oracle_lib):
    A, _ = case300
    X = np.random.default_rng(0).standard_normal((A.shape[0], 7))
    np.testing.assert_allclose(O.spmm(A, X), A @ X, rtol=1e-13, atol=1e-12)
    Y0 = np.random.default_rng(1).standard_normal((A.shape[0], 7))
    np.testing.assert_allclose(O.spmm(A, X, alpha=-2.0, beta=0.5, Y=Y0), -2.0 * (A @ X) + 0.5 * Y0,
                               rtol=1e-13, atol=1e-12)


def test_oracle_ilu0_exact_on_pattern(case300, oracle_lib):
    """ILU(0): (L U)_{ij} = A_{ij} on A's pattern (the defining property of csrilu02)."""
    A, _ = case300
    n = A.shape[0]
    F = O.ilu0(A)
    L = sp.tril(F, -1) + sp.eye(n)
    U = sp.triu(F)
    E = sp.csr_matrix(L @ U - A)
    mask = sp.csr_matrix((np.ones(A.nnz), A.indices, A.indptr), shape=A.shape)
    on = E.multiply(mask)
    assert abs(on).max() <= 1e-10 * abs(A).max()


def test_oracle_ilu0_is_lu_without_fill():
    """Tridiagonal matrix: no fill, so ILU(0) is the exact LU and ldiv! is the exact solve."""
    n = 50
    rng = np.random.default_rng(3)
    A = sp.diags([rng.uniform(-1, 1, n - 1), rng.uniform(4, 5, n), rng.uniform(-1, 1, n - 1)],
                 [-1, 0, 1], format="csr")
    F = O.ilu0(A)
    b = rng.standard_normal((n, 3))
    x = O.prec_apply(1, F, b)
    np.testing.assert_allclose(A @ x, b, rtol=0, atol=1e-12)


def test_oracle_ic0_exact_on_pattern(case300, oracle_lib):
    A, _ = case300
    S = spd_from(A)
    F = O.ic0(S)
    L = sp.tril(F)
    E = sp.csr_matrix(L @ L.T - S)
    lower = sp.csr_matrix(sp.tril(S))
    mask = sp.csr_matrix((np.ones(lower.nnz), lower.indices, lower.indptr), shape=S.shape)
    assert abs(E.multiply(mask)).max() <= 1e-10 * abs(S).max()


def test_oracle_householder_conventions(oracle_lib):
    rng = np.random.default_rng(0)
    A = rng.standard_normal((40, 6))
    Q, R, tau = O.householder(A)
    np.testing.assert_allclose(Q.T @ Q, np.eye(6), atol=1e-13)
    np.testing.assert_allclose(Q @ R, A, atol=1e-12)
    assert np.allclose(R, np.triu(R))
    # LAPACK convention: R_jj = -sign(A_jj after previous reflections) * norm -> compare |R| with
    # numpy's QR (also LAPACK)
    Rn = np.linalg.qr(A, mode="r")
    np.testing.assert_allclose(np.abs(np.diag(R)), np.abs(np.diag(Rn)), rtol=1e-12)
    np.testing.assert_allclose(R, Rn, rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("restart", [False, True])
def test_oracle_block_gmres_reference_test_settings(case300, oracle_lib, restart):
    """test/block_gmres.jl: case300, B = I[:,1:32], atol=1e-8, rtol=0, itmax=500 -> solved."""
    A, z = case300
    B = z["B32"]
    F = O.ilu0(A)
    X, st = O.block_gmres(A, B, N=(1, F), itmax=500, atol=1e-8, rtol=0.0, history=True,
                          restart=restart, memory=20)
    assert st.solved and st.status == "solution good enough given atol and rtol"
    assert np.linalg.norm(B - A @ X) <= 1e-8 * 10
    assert len(st.residuals) == st.niter + 1
    np.testing.assert_allclose(X, z["X32"], rtol=0, atol=1e-6 * np.abs(z["X32"]).max())


def test_oracle_block_gmres_tight_matches_direct(case300, oracle_lib):
    A, z = case300
    b = z["b"].reshape(-1, 1)
    F = O.ilu0(A)
    B = np.hstack([b, 2 * b, np.random.default_rng(5).standard_normal((A.shape[0], 2))])
    X, st = O.block_gmres(A, B, N=(1, F), memory=40, restart=True, atol=0.0, rtol=1e-14,
                          itmax=2000)
    Xd = np.linalg.solve(A.toarray(), B)
    assert np.abs(X - Xd).max() <= 1e-10 * np.abs(Xd).max()
    np.testing.assert_allclose(X[:, 0], z["x"], rtol=1e-9, atol=1e-10)


def test_oracle_block_gmres_warm_start_and_left_prec(case300, oracle_lib):
    A, z = case300
    F = O.ilu0(A)
    B = z["B32"][:, :8]
    Xd = z["X32"][:, :8]
    X0 = Xd + 1e-3 * np.random.default_rng(1).standard_normal(Xd.shape)
    for restart in (False, True):
        X, st = O.block_gmres(A, B, X0, M=(1, F), restart=restart, memory=30, atol=0.0,
                              rtol=1e-12, itmax=300)
        assert st.solved
        assert np.linalg.norm(B - A @ X) <= 1e-6 * np.linalg.norm(B)


def test_oracle_block_gmres_status_itmax(case300, oracle_lib):
    A, z = case300
    X, st = O.block_gmres(A, z["B32"][:, :4], itmax=3, atol=0.0, rtol=1e-14)
    assert not st.solved and st.niter == 3
    assert st.status == "maximum number of iterations exceeded"


def test_oracle_block_bicgstab_spd(oracle_lib, case300):
    A, _ = case300
    S = spd_from(A)
    B = np.random.default_rng(2).standard_normal((S.shape[0], 4))
    X, st = O.block_bicgstab(S, B, N=(2, O.ic0(S)), atol=0.0, rtol=1e-10, itmax=500, history=True)
    assert st.solved
    assert np.linalg.norm(B - S @ X) <= 1e-9 * np.linalg.norm(B)


def test_oracle_rf_known_answers(case300, oracle_lib):
    """test/cusolverRF.jl:21 (J\\b), :24-28 (values*2 -> x/2), :49-53/:63-68 (batch i*b -> i*x)."""
    A, z = case300
    b, x = z["b"], z["x"]
    lu = O.DenseLU(A)
    np.testing.assert_allclose(lu.solve(b)[:, 0], x, rtol=np.sqrt(np.finfo(float).eps))
    lu.refactor(2.0 * A)
    np.testing.assert_allclose(lu.solve(b)[:, 0], 0.5 * x, rtol=np.sqrt(np.finfo(float).eps))
    lu.refactor(A)
    Bm = np.stack([(i + 1) * b for i in range(32)], axis=1)
    Xm = lu.solve(Bm)
    for i in range(32):
        np.testing.assert_allclose(Xm[:, i], (i + 1) * x, rtol=np.sqrt(np.finfo(float).eps))


def test_oracle_on_benchmark_dump(dump300, oracle_lib):
    """benchmarks_nvidia.jl: Gx X = Gu with ILU0 right preconditioning (dense Gu block)."""
    Gx, z = dump300
    Gu = z["Gu"][:, :32]
    F = O.ilu0(Gx)
    X, st = O.block_gmres(Gx, Gu, N=(1, F), memory=30, restart=True, atol=0.0, rtol=1e-12,
                          itmax=600)
    assert st.solved
    np.testing.assert_allclose(X, z["X"][:, :32], rtol=0, atol=1e-8 * np.abs(z["X"]).max())


def test_real_case9241pegase_fixture():
    """The committed Gx_case9241pegase fixture (tests/golden/make_golden.py) is the reference's
    benchmark Jacobian: 17,036 x 17,036 with 129,412 nonzeros, square, every diagonal present."""
    from conftest import load_csr

    J, _ = load_csr("gx_case9241pegase.npz")
    assert J.shape == (17036, 17036) and J.nnz == 129412
    assert np.all(J.diagonal() != 0)
