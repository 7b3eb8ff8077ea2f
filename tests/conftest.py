import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "blockpowerflow.jl_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libbpf.so")


def load_csr(name):
    import scipy.sparse as sp

    z = np.load(os.path.join(GOLDEN, name))
    A = sp.csr_matrix((z["data"], z["indices"], z["indptr"]), shape=tuple(z["shape"]))
    return A, z


@pytest.fixture(scope="session")
def case300():
    return load_csr("case300.npz")


@pytest.fixture(scope="session")
def dump300():
    return load_csr("dump_case300.npz")


@pytest.fixture(scope="session")
def dump118():
    return load_csr("dump_case118.npz")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    oracle.build()
    return oracle


def spd_from(A):
    """An SPD matrix on A's symmetrised pattern (for IC0 tests): |A|+|A|^T made diagonally dominant."""
    import scipy.sparse as sp

    S = abs(A) + abs(A).T
    S = sp.csr_matrix(S)
    S.setdiag(0)
    S.eliminate_zeros()
    S = -S
    d = np.asarray(abs(S).sum(axis=1)).ravel() + 1.0
    S = S + sp.diags(d)
    S = sp.csr_matrix(S)
    S.sort_indices()
    return S
