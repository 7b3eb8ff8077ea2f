"""Block-Jacobi preconditioner (bpf_block_jacobi_create): ExaPF's BlockJacobiPreconditioner as
the reference's tests and benchmark use it, applied by mul! (y = P x).

Parity: the oracle's dense-inverse restatement over the same row order (the library reports it),
to 1e-12 relative; block-GMRES with it (ldiv=false, test/block_gmres.jl:17,22's setting on
data/case300.txt: B = I[:, 1:32]) reaching the tolerance and the direct solve."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bpf():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import blockpowerflow_b200 as bpf

    return bpf


@pytest.mark.parametrize("ordering,bs,p", [("natural", 32, 5), ("RCM", 32, 40), ("AMD", 7, 3), ("natural", 1, 2)])
def test_block_jacobi_apply_matches_oracle(case300, bpf, ordering, bs, p):
    import torch

    A = case300[0]
    Ad = bpf.CuSparseMatrixCSR.from_scipy(A)
    P = bpf.BlockJacobiPreconditioner(Ad, block_size=bs, ordering=ordering)
    order = P.order
    assert sorted(order.tolist()) == list(range(A.shape[0]))
    X = np.random.default_rng(p).standard_normal((A.shape[0], p))
    Y = P.mul(torch.as_tensor(X, device="cuda")).cpu().numpy()
    Yo = O.block_jacobi_apply(A, order, bs, X)
    np.testing.assert_allclose(Y, Yo, rtol=1e-12, atol=1e-12 * np.abs(Yo).max())


def test_block_jacobi_update_reads_new_values(bpf):
    import torch

    gr = bpf.grid.make_grid(300, 68, seed=0)
    A = bpf.grid.jacobian(gr)
    Ad = bpf.CuSparseMatrixCSR.from_scipy(A)
    P = bpf.BlockJacobiPreconditioner(Ad, A.shape[0] // 32)     # ExaPF's nblocks = div(n, 32)
    v2 = bpf.grid.perturbed_values(gr, A, 3, sigma=0.01, seed=1)
    Ad.nzVal.copy_(torch.as_tensor(v2, device="cuda"))
    P.update(Ad)
    A2 = A.copy()
    A2.data = v2
    X = np.random.default_rng(9).standard_normal((A.shape[0], 4))
    Y = P.mul(torch.as_tensor(X, device="cuda")).cpu().numpy()
    np.testing.assert_allclose(Y, O.block_jacobi_apply(A2, P.order, P.block_size, X), rtol=1e-12,
                               atol=1e-12 * np.abs(Y).max())


def test_block_gmres_with_block_jacobi(case300, bpf):
    """test/block_gmres.jl:17,22: block_gmres(A, B; N=BJ) (mul!, ldiv=false) on data/case300.txt
    with B = I[:, 1:32]; here to rtol 1e-10 and against the direct solve."""
    import torch

    A, z = case300
    B = z["B32"]
    Ad = bpf.CuSparseMatrixCSR.from_scipy(A)
    P = bpf.BlockJacobiPreconditioner(Ad, A.shape[0] // 32)
    X, st = bpf.block_gmres(Ad, torch.as_tensor(B, device="cuda"), N=P, ldiv=False, restart=False,
                            memory=200, atol=0.0, rtol=1e-10, itmax=300)
    assert st.solved
    Xh = X.cpu().numpy()
    assert np.linalg.norm(B - A @ Xh) <= 1e-10 * np.linalg.norm(B) * 1.01
    Xd = z["X32"] if "X32" in z else np.linalg.solve(A.toarray(), B)
    assert np.linalg.norm(Xh - Xd) <= 1e-6 * np.linalg.norm(Xd)
    with pytest.raises(bpf.BPFError, match="mul!"):
        bpf.block_gmres(Ad, torch.as_tensor(B, device="cuda"), N=P, ldiv=True)


def test_block_jacobi_rejects_singular_blocks_and_bad_sizes(bpf):
    import torch

    A = sp.csr_matrix((np.array([0.0, 1.0, 1.0, 0.0, 2.0]), np.array([0, 1, 0, 1, 2]), np.array([0, 2, 4, 5])),
                      shape=(3, 3))
    Ad = bpf.CuSparseMatrixCSR.from_scipy(A)
    with pytest.raises(bpf.SingularException):
        bpf.BlockJacobiPreconditioner(Ad, block_size=1)     # the 1 x 1 block A[0, 0] = 0
    P = bpf.BlockJacobiPreconditioner(Ad, block_size=2)     # [[0, 1], [1, 0]] is invertible
    Y = P.mul(torch.eye(3, dtype=torch.float64, device="cuda")).cpu().numpy()
    np.testing.assert_allclose(Y, np.array([[0, 1, 0], [1, 0, 0], [0, 0, 0.5]]), atol=1e-15)
    with pytest.raises(bpf.BPFError):
        bpf.BlockJacobiPreconditioner(Ad, block_size=33)
