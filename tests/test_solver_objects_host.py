"""In-place solver API, host logic (no GPU): BlockGMRESSolver / block_gmres_ / warm_start_ and
BlockBicgstabSolver / block_bicgstab_ mirror src/block_gmres.jl:21-168,397-411 and
src/block_bicgstab.jl:23-55,182-299: memory clamped to div(n, p), the solution written into the
solver's block (on B's device), a warm start consumed by the next solve, size errors.  The device
solves are replaced by a stand-in that records its arguments (their parity is the GPU tests')."""
import types

import numpy as np
import pytest
import torch

from blockpowerflow_b200 import _lib
from blockpowerflow_b200 import krylov as K


@pytest.fixture
def calls(monkeypatch):
    rec = []

    def fake_gmres(A, B, X0=None, **kw):
        rec.append(("gmres", None if X0 is None else X0.clone(), kw))
        return B * 2.0, K.BlockGMRESStats(7, True, [1.0, 0.5], 0.1, "solution good enough given atol and rtol")

    def fake_bicgstab(A, B, **kw):
        rec.append(("bicgstab", None, kw))
        return B * 3.0, K.SimpleStats(4, True, [], 0.2, "solution good enough given atol and rtol")

    monkeypatch.setattr(K, "block_gmres", fake_gmres)
    monkeypatch.setattr(K, "block_bicgstab", fake_bicgstab)
    return rec


A100 = types.SimpleNamespace(shape=(100, 100))


def _B(p, seed=0):
    return torch.as_tensor(np.random.default_rng(seed).standard_normal((100, p)))


def test_memory_is_clamped_to_div_n_p():
    assert K.BlockGMRESSolver(A100, _B(8), memory=50).memory == 12
    assert K.BlockGMRESSolver(A100, _B(8)).memory == 5
    s = K.BlockGMRESSolver.from_sizes(100, 100, 16, 20, device="cpu")
    assert (s.m, s.n, s.p, s.memory) == (100, 100, 16, 6)
    assert s.stats.status == "unknown" and not s.warm_start


def test_block_gmres_writes_into_the_solver(calls):
    B = _B(8)
    s = K.BlockGMRESSolver(A100, B, memory=30)
    X_id = s.X.data_ptr()
    out = K.block_gmres_(s, A100, B, rtol=1e-9, ldiv=True)
    assert out is s
    assert s.X.data_ptr() == X_id and s.X.stride(0) == 1            # in place, column-major
    assert torch.equal(s.X, B * 2.0)
    assert s.stats.niter == 7 and s.stats.solved
    kind, X0, kw = calls[-1]
    assert X0 is None and kw["memory"] == 12 and kw["rtol"] == 1e-9 and kw["ldiv"]


def test_warm_start_is_passed_once(calls):
    B, X0 = _B(4, 1), _B(4, 2)
    s = K.BlockGMRESSolver(A100, B)
    K.warm_start_(s, X0)
    assert s.warm_start
    K.block_gmres_(s, A100, B)
    assert torch.equal(calls[-1][1], X0)
    assert not s.warm_start and s.dX is None
    K.block_gmres_(s, A100, B)                                      # consumed: a cold start
    assert calls[-1][1] is None
    K.block_gmres_(s, A100, B, X0)                                  # the 4-argument form
    assert torch.equal(calls[-1][1], X0)


def test_size_errors():
    s = K.BlockGMRESSolver(A100, _B(4))
    with pytest.raises(_lib.DimensionMismatch, match=r"X0 should have size \(100, 4\)"):
        K.warm_start_(s, _B(5))
    with pytest.raises(_lib.DimensionMismatch):
        K.block_gmres_(s, A100, _B(5))
    b = K.BlockBicgstabSolver(A100, _B(4))
    with pytest.raises(_lib.DimensionMismatch):
        K.block_bicgstab_(b, A100, _B(6))


def test_block_bicgstab_returns_the_solvers_block_and_stats(calls):
    B = _B(6)
    s = K.BlockBicgstabSolver(A100, B)
    X, st = K.block_bicgstab_(s, A100, B, atol=1e-10, itmax=50)
    assert X is s.X and st is s.stats
    assert torch.equal(X, B * 3.0) and st.niter == 4
    assert calls[-1][2]["atol"] == 1e-10 and calls[-1][2]["itmax"] == 50
