"""The oracle's block-Jacobi restatement (no GPU): P = diag(A_b^{-1}) over consecutive runs of
the given order, checked by its defining property P A_blockdiag = I on every block, and against
an explicit dense block inverse."""
import numpy as np
import scipy.sparse as sp

import oracle as O
from blockpowerflow_b200 import grid as G


def test_block_jacobi_oracle_inverts_the_diagonal_blocks():
    A = G.synthetic_jacobian(100, 10, 0).tocsr()
    n = A.shape[0]
    rng = np.random.default_rng(0)
    order = rng.permutation(n)
    bs = 7
    # block-diagonal part of A in that partition
    blk = np.empty(n, dtype=int)
    blk[order] = np.arange(n) // bs
    Ac = A.tocoo()
    keep = blk[Ac.row] == blk[Ac.col]
    D = sp.csr_matrix((Ac.data[keep], (Ac.row[keep], Ac.col[keep])), shape=A.shape)
    X = rng.standard_normal((n, 3))
    Y = O.block_jacobi_apply(A, order, bs, D @ X)
    np.testing.assert_allclose(Y, X, rtol=1e-10, atol=1e-10)
    rows = order[:bs]
    Ab = A[rows][:, rows].toarray()
    np.testing.assert_allclose(O.block_jacobi_apply(A, order, bs, X)[rows], np.linalg.inv(Ab) @ X[rows],
                               rtol=1e-10, atol=1e-12)
