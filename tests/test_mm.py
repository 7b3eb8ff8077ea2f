"""MatrixMarket ingest of the reference's on-disk cases (no GPU): the benchmark dump pair
Gx_<case>.mtx / Gu_<case>.mtx round-trips through the reader exactly (written here from the
committed fixtures of the reference's own dumps), and malformed files are rejected."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.io import mmwrite

from blockpowerflow_b200 import mm

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _fixture(case):
    d = np.load(os.path.join(GOLDEN, f"dump_{case}.npz"))
    A = sp.csr_matrix((d["data"], d["indices"], d["indptr"]), shape=tuple(d["shape"]))
    return A, d["Gu"], d["X"]


@pytest.mark.parametrize("case", ["case118", "case300"])
def test_dump_pair_round_trip(tmp_path, case):
    A, Gu, X = _fixture(case)
    pa, pb = mm.dump_paths(str(tmp_path), case)
    mmwrite(pa, A)
    mmwrite(pb, sp.coo_matrix(Gu))          # the dumps store Gu in coordinate form
    A2, B2 = mm.load_dump(str(tmp_path), case)
    assert A2.shape == A.shape and A2.has_sorted_indices
    np.testing.assert_array_equal(A2.indptr, A.indptr)
    np.testing.assert_array_equal(A2.indices, A.indices)
    np.testing.assert_allclose(A2.data, A.data, rtol=1e-15, atol=0)
    np.testing.assert_allclose(B2, Gu, rtol=1e-15, atol=0)
    # the fixture's direct solution still solves the re-read system
    assert np.linalg.norm(Gu - A2 @ X) <= 1e-8 * np.linalg.norm(Gu)


def test_array_form_and_vector_rhs(tmp_path):
    A = sp.random(20, 20, density=0.2, random_state=1, format="csr") + sp.eye(20)
    b = np.arange(20.0)
    mmwrite(os.path.join(tmp_path, "Gx_t.mtx"), A)
    mmwrite(os.path.join(tmp_path, "Gu_t.mtx"), b[:, None])   # array (dense) MatrixMarket form
    A2, B2 = mm.load_dump(str(tmp_path), "t")
    assert B2.shape == (20, 1) and np.array_equal(B2[:, 0], b)
    assert abs(A2 - A).max() == 0


def test_rejects_non_square_complex_and_mismatched(tmp_path):
    p = os.path.join(tmp_path, "r.mtx")
    mmwrite(p, sp.random(5, 4, density=0.5, random_state=0))
    with pytest.raises(ValueError, match="not square"):
        mm.read_mtx(p)
    pc = os.path.join(tmp_path, "c.mtx")
    mmwrite(pc, sp.eye(3, dtype=complex) * (1 + 1j))
    with pytest.raises(ValueError, match="field"):
        mm.read_mtx(pc)
    mmwrite(os.path.join(tmp_path, "Gx_m.mtx"), sp.eye(6))
    mmwrite(os.path.join(tmp_path, "Gu_m.mtx"), np.ones((5, 2)))
    with pytest.raises(ValueError, match="rows"):
        mm.load_dump(str(tmp_path), "m")
