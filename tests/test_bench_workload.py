"""The batched configuration's inputs as bench.py generates them (no GPU): grids of 100 - 3,000
buses, 8 - 64 Gaussian right-hand sides each, square Jacobians with a full diagonal, the same
systems for the same seed."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_batch_workload_matches_the_configuration():
    import bench

    buses, nrhs, mats, Bs = bench.batch_workload(16, seed=0)
    assert len(mats) == len(Bs) == len(nrhs) == 16
    assert all(100 <= b < 3000 for b in buses)
    assert all(8 <= p <= 64 for p in nrhs)
    for A, B, p in zip(mats, Bs, nrhs):
        assert A.shape[0] == A.shape[1] == B.shape[0] and B.shape[1] == p
        assert (A.diagonal() != 0).all()
    b2, p2, m2, B2 = bench.batch_workload(16, seed=0)
    assert list(b2) == list(buses) and p2 == nrhs
    assert all((x != y).nnz == 0 for x, y in zip(mats, m2)) and all(np.array_equal(x, y) for x, y in zip(Bs, B2))
