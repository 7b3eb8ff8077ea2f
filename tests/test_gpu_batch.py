"""Batched block-GMRES (bpf_batch_*): many independent systems in one graph launch.

Parity: every system against the direct solve (SciPy SuperLU) and, for single-slice units,
the iteration count of the oracle's block-GMRES with the same right ILU(0) (unrestarted, the
reference's block_gmres! with N = ilu0(A), ldiv = true).  Tolerances: the true relative
residual ||B - A X||_F / ||B||_F <= rtol (1e-8) with FP32 factors; with FP64 factors solved to
rtol 1e-12, X within 1e-10 (relative, Frobenius) of the direct solve.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bpf():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import blockpowerflow_b200 as bpf

    return bpf


def _systems(bpf, buses, seed0=0):
    mats = []
    for k, nb in enumerate(buses):
        gr = bpf.grid.make_grid(nb, seed=seed0 + k)
        mats.append(bpf.grid.jacobian(gr).tocsr())
    return mats


def _rhs(bpf, mats, nrhs, seed=7):
    return [bpf.grid.gaussian_rhs(A.shape[0], p, seed + s) for s, (A, p) in enumerate(zip(mats, nrhs))]


def _solve(bpf, mats, Bs, nrhs, **kw):
    import torch

    dm = [bpf.CuSparseMatrixCSR.from_scipy(A) for A in mats]
    plan = bpf.BatchPlan(dm, nrhs, **kw)
    Xs, st = plan.solve([torch.as_tensor(B, device="cuda") for B in Bs])
    return plan, [X.cpu().numpy() for X in Xs], st, dm


BUSES = [100, 150, 220, 300, 450, 600, 800, 1000, 1500, 2000]
NRHS = [3, 8, 13, 16, 20, 31, 32, 40, 64, 7]


def test_batch_fp32_factors_reach_the_tolerance(bpf):
    mats = _systems(bpf, BUSES)
    Bs = _rhs(bpf, mats, NRHS)
    plan, Xs, st, _ = _solve(bpf, mats, Bs, NRHS)
    assert plan.nunits >= len(mats)
    for s, (A, B, X) in enumerate(zip(mats, Bs, Xs)):
        assert st[s].solved, (s, st[s])
        assert st[s].status == "solution good enough given atol and rtol"
        rel = np.linalg.norm(B - A @ X) / np.linalg.norm(B)
        assert rel <= 1e-8 * 1.01, (s, rel)
    u = plan.unit_stats()
    assert (u["q"] <= 16).all() and (u["status"] == 1).all()
    # the slices of each system cover its columns exactly once
    for s, p in enumerate(NRHS):
        cols = sorted((c0, q) for c0, q, ss in zip(u["col0"], u["q"], u["sys"]) if ss == s)
        assert cols[0][0] == 0 and sum(q for _, q in cols) == p
        assert all(a[0] + a[1] == b[0] for a, b in zip(cols, cols[1:]))
    cyc = plan.unit_cycles()
    assert (cyc["total"] > 0).all() and (cyc["gram"] <= cyc["total"]).all()


@pytest.mark.parametrize("ordering", ["AMD", "natural", "RCM"])
def test_batch_fp64_factors_match_the_direct_solve(bpf, ordering):
    mats = _systems(bpf, [120, 400, 900], seed0=20)
    nrhs = [5, 24, 33]
    Bs = _rhs(bpf, mats, nrhs, seed=3)
    plan, Xs, st, _ = _solve(bpf, mats, Bs, nrhs, rtol=1e-12, factor_dtype="float64", ordering=ordering,
                             slice=32)
    for s, (A, B, X) in enumerate(zip(mats, Bs, Xs)):
        assert st[s].solved
        Xd = spla.splu(A.tocsc()).solve(B)
        err = np.linalg.norm(X - Xd) / np.linalg.norm(Xd)
        assert err <= 1e-10, (s, err)


def test_batch_iterations_match_the_oracle(bpf):
    """One unit per system (p <= slice), natural order, FP64 factors: the iteration count of
    the oracle's block_gmres with the same right ILU(0), unrestarted, within one."""
    mats = _systems(bpf, [150, 300, 700], seed0=40)
    nrhs = [4, 16, 32]
    Bs = _rhs(bpf, mats, nrhs, seed=11)
    plan, Xs, st, _ = _solve(bpf, mats, Bs, nrhs, rtol=1e-8, factor_dtype="float64", ordering="natural",
                             slice=32, memory=200)
    for s, (A, B) in enumerate(zip(mats, Bs)):
        F = O.ilu0(A)
        Xo, so = O.block_gmres(A, B, N=(1, F), memory=200, restart=False, atol=0.0, rtol=1e-8,
                               itmax=400)
        assert so.solved and st[s].solved
        assert abs(st[s].niter - so.niter) <= 1, (s, st[s].niter, so.niter)
        np.testing.assert_allclose(Xs[s], Xo, rtol=0, atol=1e-6 * np.abs(Xo).max())


def test_batch_restarts_when_the_basis_is_full(bpf):
    """Basis of 16 blocks: the units restart from the true residual (the reference's
    restart=true) and converge; iteration counts near the oracle's restarted block_gmres.
    (With 12 blocks or fewer, restarted block-GMRES stagnates on these Jacobians, in the oracle
    as well.)"""
    mats = _systems(bpf, [300, 500], seed0=60)
    nrhs = [16, 24]
    Bs = _rhs(bpf, mats, nrhs)
    plan, Xs, st, _ = _solve(bpf, mats, Bs, nrhs, memory=16, itmax=600, factor_dtype="float64",
                             ordering="natural", slice=32)
    for s, (A, B, X) in enumerate(zip(mats, Bs, Xs)):
        assert st[s].solved and st[s].npass > 1, st[s]
        assert np.linalg.norm(B - A @ X) <= 1e-8 * np.linalg.norm(B) * 1.01
        Xo, so = O.block_gmres(A, B, N=(1, O.ilu0(A)), memory=16, restart=True, atol=0.0, rtol=1e-8,
                               itmax=600)
        assert so.solved and abs(st[s].niter - so.niter) <= max(2, so.niter // 10), (st[s].niter, so.niter)


def test_batch_zero_rhs_columns_and_zero_blocks(bpf):
    mats = _systems(bpf, [200, 250], seed0=80)
    nrhs = [6, 4]
    Bs = _rhs(bpf, mats, nrhs)
    Bs[0][:, 2] = 0.0
    Bs[1][:] = 0.0
    plan, Xs, st, _ = _solve(bpf, mats, Bs, nrhs)
    assert st[0].solved and st[1].solved and st[1].niter == 0
    assert np.all(Xs[0][:, 2] == 0.0) and np.all(Xs[1] == 0.0)
    A, B, X = mats[0], Bs[0], Xs[0]
    assert np.linalg.norm(B - A @ X) <= 1e-8 * np.linalg.norm(B) * 1.01


def test_batch_new_values_are_read_by_every_solve(bpf):
    import torch

    gr = bpf.grid.make_grid(400, seed=5)
    A = bpf.grid.jacobian(gr).tocsr()
    dm = bpf.CuSparseMatrixCSR.from_scipy(A)
    plan = bpf.BatchPlan([dm], [8])
    B = bpf.grid.gaussian_rhs(A.shape[0], 8, 1)
    Bd = torch.as_tensor(B, device="cuda")
    X1 = plan.solve([Bd])[0][0].cpu().numpy()
    v2 = bpf.grid.perturbed_values(gr, A, 1, sigma=0.01, seed=2)
    dm.nzVal.copy_(torch.as_tensor(v2, device="cuda"))
    X2, st = plan.solve([Bd])
    A2 = A.copy()
    A2.data = v2
    X2 = X2[0].cpu().numpy()
    assert st[0].solved
    assert np.linalg.norm(B - A2 @ X2) <= 1e-8 * np.linalg.norm(B) * 1.01
    assert np.linalg.norm(X2 - X1) > 1e-6 * np.linalg.norm(X1)


def test_batch_zero_pivot_names_the_system(bpf):
    import torch

    good = _systems(bpf, [150], seed0=90)[0]
    bad = sp.csr_matrix((np.array([0.0, 1.0, 1.0, 0.0]), np.array([0, 1, 0, 1]), np.array([0, 2, 4])),
                        shape=(2, 2))
    dm = [bpf.CuSparseMatrixCSR.from_scipy(good), bpf.CuSparseMatrixCSR.from_scipy(bad)]
    plan = bpf.BatchPlan(dm, [4, 1], ordering="natural")
    Bs = [torch.ones((good.shape[0], 4), dtype=torch.float64, device="cuda"),
          torch.ones((2, 1), dtype=torch.float64, device="cuda")]
    with pytest.raises(bpf.SingularException, match="system 1"):
        plan.solve(Bs)


def test_batch_rejects_bad_arguments(bpf):
    import torch

    A = _systems(bpf, [100], seed0=95)[0]
    dm = [bpf.CuSparseMatrixCSR.from_scipy(A)]
    with pytest.raises(bpf.BPFError):
        bpf.BatchPlan(dm, [4], slice=33)
    with pytest.raises(bpf.BPFError):
        bpf.BatchPlan(dm, [0])
    with pytest.raises(bpf.BPFError):
        bpf.BatchPlan(dm, [4], ordering="METIS")
    plan = bpf.BatchPlan(dm, [4])
    with pytest.raises(bpf.DimensionMismatch):
        plan.solve([torch.zeros((A.shape[0], 5), dtype=torch.float64, device="cuda")])


def test_autotune_times_candidates_and_caches(bpf, tmp_path):
    import torch

    mats = _systems(bpf, [200, 600, 1200], seed0=100)
    nrhs = [8, 24, 40]
    Bs = _rhs(bpf, mats, nrhs)
    dm = [bpf.CuSparseMatrixCSR.from_scipy(A) for A in mats]
    Bd = [torch.as_tensor(B, device="cuda") for B in Bs]
    path = str(tmp_path / "tune.json")
    r = bpf.autotune(dm, nrhs, Bd, cache_path=path, candidates=[(8, 2), (16, 2), (32, 1)], repeats=1)
    assert not r["cached"] and (r["slice"], r["ctas_per_sm"]) in [(8, 2), (16, 2), (32, 1)]
    assert r["ordering"] == "AMD"
    assert all(ok for _, ok in r["timings"].values())
    r2 = bpf.autotune(dm, nrhs, Bd, cache_path=path, candidates=[(8, 2), (16, 2), (32, 1)])
    assert r2["cached"] and r2["slice"] == r["slice"]
    # the default candidates time both fill-reducing orders; the choice builds a plan that solves
    r3 = bpf.autotune(dm, nrhs, Bd, repeats=1)
    assert set(r3["timings"]) == {f"{s}x{c}x{o}" for s, c, o in bpf.batch.CANDIDATES}
    plan = bpf.BatchPlan(dm, nrhs, slice=r3["slice"], ctas_per_sm=r3["ctas_per_sm"], ordering=r3["ordering"])
    Xs, st = plan.solve(Bd)
    assert all(s.solved for s in st)
    for A, B, X in zip(mats, Bs, Xs):
        assert np.linalg.norm(B - A @ X.cpu().numpy()) <= 1.01e-8 * np.linalg.norm(B)
    plan.close()


def test_batch_per_system_slices(bpf):
    """bpf_batch_plan_sliced: a widest slice per system (0 keeps the plan's), each system's
    columns still covered exactly once, every system at the tolerance."""
    mats = _systems(bpf, [300, 800, 1500], seed0=120)
    nrhs = [20, 9, 40]
    Bs = _rhs(bpf, mats, nrhs, seed=21)
    plan, Xs, st, dm = _solve(bpf, mats, Bs, nrhs, slice=32, slices=[0, 3, 8])
    u = plan.unit_stats()
    widest = {s: max(q for q, ss in zip(u["q"], u["sys"]) if ss == s) for s in range(3)}
    assert widest == {0: 20, 1: 3, 2: 8}
    for s, (A, B, X) in enumerate(zip(mats, Bs, Xs)):
        assert st[s].solved, (s, st[s])
        assert np.linalg.norm(B - A @ X) / np.linalg.norm(B) <= 1e-8 * 1.01, s
        assert sum(q for q, ss in zip(u["q"], u["sys"]) if ss == s) == nrhs[s]
    plan.close()
    with pytest.raises(bpf.BPFError):
        bpf.BatchPlan(dm, nrhs, slices=[0, 33, 0])
    with pytest.raises(bpf.DimensionMismatch):
        bpf.BatchPlan(dm, nrhs, slices=[0, 3])


def test_batch_wide_blocks_on_small_systems_converge(bpf):
    """Small grids with wide right-hand-side blocks and FP64 factors, the case where block-GMRES
    exhausts the Krylov space or meets a partial breakdown: the plan narrows the slices of small
    systems and caps their basis inside R^n, and a converged estimate is checked against the true
    residual, so every system reaches the tolerance."""
    mats = _systems(bpf, [100, 120, 180, 250, 350], seed0=110)
    nrhs = [58, 53, 63, 42, 30]
    Bs = _rhs(bpf, mats, nrhs, seed=13)
    plan, Xs, st, _ = _solve(bpf, mats, Bs, nrhs, factor_dtype="float64", slice=32)
    u = plan.unit_stats()
    for s, (A, B, X) in enumerate(zip(mats, Bs, Xs)):
        assert st[s].solved, (s, st[s])
        assert np.linalg.norm(B - A @ X) <= 1e-8 * np.linalg.norm(B) * 1.01
        assert (u["q"][u["sys"] == s] <= max(1, A.shape[0] // 24)).all()
