"""GPU parity of the building blocks, through the C ABI, against the CPU oracle.

Tolerances (FP64): SpMM and triangular solves 1e-12 relative to the operand scale (the sums
are the same terms in another order); factor values 1e-11 relative.
"""
import numpy as np
import pytest
import scipy.sparse as sp

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


def _dev(A, bpf, base=0):
    return bpf.CuSparseMatrixCSR.from_scipy(A, index_base=base)


@pytest.mark.parametrize("p", [1, 3, 8, 16, 31, 64, 100, 128, 256, 300])
def test_spmm_matches_oracle(case300, bpf, p):
    import torch

    A, _ = case300
    X = np.random.default_rng(p).standard_normal((A.shape[0], p))
    Y = bpf.mul(_dev(A, bpf), torch.as_tensor(X, device="cuda"))
    np.testing.assert_allclose(Y.cpu().numpy(), O.spmm(A, X), rtol=1e-12, atol=1e-11)


def test_spmm_one_based_and_alpha_beta(case300, bpf):
    import torch

    A, _ = case300
    n = A.shape[0]
    rng = np.random.default_rng(7)
    X, Y0 = rng.standard_normal((n, 16)), rng.standard_normal((n, 16))
    Yd = bpf.colmajor(torch.as_tensor(Y0, device="cuda")).clone()
    Yd = Yd.t().contiguous().t()
    bpf.mul(_dev(A, bpf, base=1), torch.as_tensor(X, device="cuda"), alpha=-1.5, beta=0.25, Y=Yd)
    np.testing.assert_allclose(Yd.cpu().numpy(), O.spmm(A, X, alpha=-1.5, beta=0.25, Y=Y0),
                               rtol=1e-12, atol=1e-11)


def test_spmm_synthetic_9k(bpf):
    import torch

    A = bpf.grid.preset_jacobian("case9k", 0)
    X = np.random.default_rng(0).standard_normal((A.shape[0], 64))
    Y = bpf.mul(_dev(A, bpf), torch.as_tensor(X, device="cuda")).cpu().numpy()
    np.testing.assert_allclose(Y, A @ X, rtol=1e-12, atol=1e-10)


@pytest.mark.parametrize("name", ["case300", "dump118"])
def test_ilu0_factor_and_apply(request, bpf, name):
    import torch

    A, _ = request.getfixturevalue(name if name != "case300" else "case300")
    P = bpf.ilu0(_dev(A, bpf), 8)
    F = O.ilu0(A)
    got = P.P.nzVal.cpu().numpy()
    np.testing.assert_allclose(got, F.data, rtol=1e-11, atol=1e-11 * np.abs(F.data).max())
    for p in (1, 5, 16, 64, 130):
        X = np.random.default_rng(p).standard_normal((A.shape[0], p))
        Y = bpf.empty_colmajor(A.shape[0], p)
        bpf.ldiv_(Y, P, torch.as_tensor(X, device="cuda"))
        ref = O.prec_apply(1, F, X)
        np.testing.assert_allclose(Y.cpu().numpy(), ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())


def test_ilu0_synthetic_levels_and_apply(bpf):
    import torch

    A = bpf.grid.preset_jacobian("case9k", 1)
    P = bpf.ilu0(_dev(A, bpf), 64)
    lo, up = P.levels()
    assert lo > 1 and up > 1
    F = O.ilu0(A)
    np.testing.assert_allclose(P.P.nzVal.cpu().numpy(), F.data, rtol=1e-10,
                               atol=1e-10 * np.abs(F.data).max())
    X = np.random.default_rng(0).standard_normal((A.shape[0], 64))
    Y = bpf.empty_colmajor(A.shape[0], 64)
    bpf.ldiv_(Y, P, torch.as_tensor(X, device="cuda"))
    ref = O.prec_apply(1, F, X)
    np.testing.assert_allclose(Y.cpu().numpy(), ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())


def test_ilu0_refactor_scaled_values(case300, bpf):
    import torch

    A, _ = case300
    Ad = _dev(A, bpf)
    P = bpf.ilu0(Ad, 4)
    P.refactor(Ad.nzVal * 2.0)
    F = O.ilu0(2.0 * A)
    np.testing.assert_allclose(P.P.nzVal.cpu().numpy(), F.data, rtol=1e-11,
                               atol=1e-11 * np.abs(F.data).max())


def test_ilu0_fp32_factors(case300, bpf):
    import torch

    A, _ = case300
    P = bpf.ilu0(_dev(A, bpf), 16, factor_dtype="float32")
    X = np.random.default_rng(0).standard_normal((A.shape[0], 16))
    Y = bpf.empty_colmajor(A.shape[0], 16)
    bpf.ldiv_(Y, P, torch.as_tensor(X, device="cuda"))
    ref = O.prec_apply(1, O.ilu0(A), X)
    err = np.abs(Y.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err < 1e-4


def test_ic0_factor_and_apply(case300, bpf):
    import torch

    A, _ = case300
    S = spd_from(A)
    P = bpf.ic0(_dev(S, bpf), 8)
    F = O.ic0(S)
    lower = sp.csr_matrix(sp.tril(S))
    got = P.P.to_scipy()
    np.testing.assert_allclose(sp.tril(got).toarray(), sp.tril(F).toarray(), rtol=1e-11,
                               atol=1e-12)
    X = np.random.default_rng(3).standard_normal((S.shape[0], 24))
    Y = bpf.empty_colmajor(S.shape[0], 24)
    bpf.ldiv_(Y, P, torch.as_tensor(X, device="cuda"))
    ref = O.prec_apply(2, F, X)
    np.testing.assert_allclose(Y.cpu().numpy(), ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())


def test_ilu0_missing_diagonal_is_singular(bpf):
    A = sp.csr_matrix(np.array([[0.0, 1.0], [1.0, 2.0]]))
    with pytest.raises(bpf.SingularException):
        bpf.ilu0(_dev(A, bpf), 1)


def test_ilu0_zero_pivot_is_singular(bpf):
    A = sp.csr_matrix(np.array([[1.0, 1.0], [1.0, 1.0]]))
    with pytest.raises(bpf.SingularException):
        bpf.ilu0(_dev(A, bpf), 1)


@pytest.mark.parametrize("p", [1, 4, 16, 33, 64, 128])
def test_householder_qr(bpf, p):
    import torch

    rng = np.random.default_rng(p)
    W = rng.standard_normal((3000, p))
    Q, R = bpf.householder(torch.as_tensor(W, device="cuda"))
    Q, R = Q.cpu().numpy(), R.cpu().numpy()
    np.testing.assert_allclose(Q.T @ Q, np.eye(p), atol=1e-13)
    np.testing.assert_allclose(Q @ R, W, atol=1e-12 * np.abs(W).max())
    assert np.allclose(R, np.triu(R))
    # same R as LAPACK up to the sign of each row
    Rn = np.linalg.qr(W, mode="r")
    np.testing.assert_allclose(np.abs(R), np.abs(Rn), rtol=1e-9, atol=1e-11)


@pytest.mark.parametrize("p", [1, 8, 33, 64, 128])
@pytest.mark.parametrize("compact", [False, True])
def test_householder_lapack_conventions_match_oracle(bpf, p, compact):
    """householder(A; compact) with LAPACK's signs (src/block_utils.jl:38-53): R, tau and Q
    (orgqr's, or geqrf's compact form with the reflector vectors) equal the oracle's geqrf /
    orgqr restatement to rounding."""
    import torch

    rng = np.random.default_rng(100 + p)
    W = rng.standard_normal((3000, p)) * np.logspace(0, 2, p)   # columns of different scales
    Q, R = bpf.householder(torch.as_tensor(W, device="cuda"), compact=compact)
    tau = bpf.householder.tau.cpu().numpy()
    Qo, Ro, to = O.householder(W, compact=compact)
    np.testing.assert_allclose(R.cpu().numpy(), Ro, rtol=1e-10, atol=1e-11 * np.abs(Ro).max())
    np.testing.assert_allclose(tau, to, rtol=1e-9, atol=1e-12)
    Qh = Q.cpu().numpy()
    if compact:
        np.testing.assert_allclose(np.triu(Qh[:p]), np.triu(Ro), rtol=1e-10, atol=1e-11 * np.abs(Ro).max())
        lo, loo = np.tril(Qh, -1), np.tril(Qo, -1)
        np.testing.assert_allclose(lo, loo, rtol=1e-8, atol=1e-10 * np.abs(loo).max())
    else:
        np.testing.assert_allclose(Qh, Qo, rtol=1e-9, atol=1e-12)


def test_householder_rank_deficient_block(bpf):
    """Shifted Cholesky-QR keeps Q orthonormal when the block has dependent columns."""
    import torch

    rng = np.random.default_rng(0)
    W = rng.standard_normal((2000, 8))
    W[:, 5] = W[:, 1] + 1e-14 * rng.standard_normal(2000)
    Q, R = bpf.householder(torch.as_tensor(W, device="cuda"))
    Q, R = Q.cpu().numpy(), R.cpu().numpy()
    np.testing.assert_allclose(Q.T @ Q, np.eye(8), atol=1e-10)
    np.testing.assert_allclose(Q @ R, W, atol=1e-10 * np.abs(W).max())


@pytest.mark.parametrize("ordering,factor_dtype,p", [("natural", "float64", 128), ("AMD", "float64", 64),
                                                     ("AMD", "float32", 100), ("natural", "float64", 17)])
def test_sync_free_triangular_solves_repeat_and_match_oracle(bpf, ordering, factor_dtype, p):
    """Blocks of more than 16 columns on multi-CTA factors take the sync-free solve (ready words
    per row, one launch epoch per apply): ten applies in a row give identical results, equal to
    the oracle's (1e-12 relative for FP64 factors, 1e-4 for FP32)."""
    import torch

    A = bpf.grid.preset_jacobian("case9k", 0)
    N = bpf.ilu0(_dev(A, bpf), p, factor_dtype=factor_dtype, ordering=ordering)
    perm = N.perm if ordering != "natural" else np.arange(A.shape[0])
    X = np.random.default_rng(p).standard_normal((A.shape[0], p))
    Xd = torch.as_tensor(X, device="cuda")
    outs = []
    for _ in range(10):
        Y = bpf.empty_colmajor(A.shape[0], p)
        bpf.ldiv_(Y, N, Xd)
        outs.append(Y.cpu().numpy())
    for Yk in outs[1:]:
        assert np.array_equal(Yk, outs[0])
    Ap = A[perm][:, perm]
    ref = np.empty_like(X)
    ref[perm] = O.prec_apply(1, O.ilu0(Ap), X[perm])
    tol = 1e-12 if factor_dtype == "float64" else 1e-4
    np.testing.assert_allclose(outs[0], ref, rtol=tol, atol=tol * np.abs(ref).max())


def test_sync_free_ic0_solve_matches_oracle(bpf):
    import torch

    S = spd_from(bpf.grid.preset_jacobian("case9k", 0))
    P = bpf.ic0(_dev(S, bpf), 64)
    X = np.random.default_rng(9).standard_normal((S.shape[0], 64))
    Y = bpf.empty_colmajor(S.shape[0], 64)
    bpf.ldiv_(Y, P, torch.as_tensor(X, device="cuda"))
    ref = O.prec_apply(2, O.ic0(S), X)
    np.testing.assert_allclose(Y.cpu().numpy(), ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())
