"""The callers around the solve path, on the device: the Newton power-flow driver (refactor +
solve per step, then the multi-RHS sensitivities Gx^{-1} Gu) and the MatrixMarket dump ingest
with the reference benchmark's solve.

Parity: the Newton iterates of the device solvers against the same loop with SciPy's direct
solve (iteration counts within one, solutions to 1e-8), the sensitivities to 1e-9 relative (RF) /
1e-8 (block-GMRES at rtol 1e-12); the dump solve against the fixture's direct solution of the
reference's own Gx X = Gu (1e-8 relative)."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.io import mmwrite

from blockpowerflow_b200 import grid as G
from blockpowerflow_b200 import newton as NT
from test_newton_host import _SciPyStandIn

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def bpf():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import blockpowerflow_b200 as bpf

    return bpf


@pytest.mark.parametrize("n_bus,solver", [(300, "rf"), (2000, "rf"), (300, "gmres"), (2000, "gmres")])
def test_newton_on_the_device_matches_the_direct_loop(bpf, n_bus, solver):
    prob = NT.make_problem(G.make_grid(n_bus, seed=7))
    x0 = NT.perturbed_start(prob, 0.01, seed=2)
    r = NT.newton(prob, solver=solver, x0=x0, tol=1e-10, sensitivities=True)
    ref = NT.newton(prob, solver=_SciPyStandIn(prob.pattern), x0=x0, tol=1e-10, sensitivities=True)
    assert r.converged and ref.converged, (r.residuals, ref.residuals)
    assert abs(r.iterations - ref.iterations) <= 1, (r.residuals, ref.residuals)
    np.testing.assert_allclose(r.x, ref.x, rtol=0, atol=1e-8)
    tol = 1e-9 if solver == "rf" else 1e-8
    err = np.linalg.norm(r.sensitivities - ref.sensitivities) / np.linalg.norm(ref.sensitivities)
    assert err <= tol, err


@pytest.mark.parametrize("n_bus,seed", [(300, 3), (2000, 7)])
def test_device_assembly_matches_the_numpy_assembly(bpf, n_bus, seed):
    """bpf_pf_mismatch / bpf_pf_jacobian against mismatch(), jacobian_values(), control_jacobian()
    (1e-12 relative: the same formulas, FMA-contracted complex products) and against the oracle's
    entry-by-entry restatement over the same host arguments (1e-11); the trial point x + alpha dx
    bit for bit; max |F| equal to the largest |F| entry."""
    import torch

    import oracle as O

    prob = NT.make_problem(G.make_grid(n_bus, seed=seed))
    A = bpf.CuSparseMatrixCSR.from_scipy(prob.pattern)
    asm = NT.DeviceAssembly(prob, A)
    assert (asm.n, asm.n_ctrl) == (prob.pattern.shape[0], len(prob.ctrl))
    x = NT.perturbed_start(prob, 0.05, seed=seed)
    dx = np.random.default_rng(seed).standard_normal(len(x))
    xd, dxd = (torch.tensor(v, device="cuda") for v in (x, dx))
    F, xt = torch.empty_like(xd), torch.empty_like(xd)
    nrm = asm.mismatch(xd, F)
    F0 = NT.mismatch(prob, x)
    assert np.abs(F.cpu().numpy() - F0).max() <= 1e-12 * np.abs(F0).max()
    Fo, gxo, Guo = O.pf_assemble(*NT.bus_arrays(prob), x, prob.pattern)
    assert np.abs(F.cpu().numpy() - Fo).max() <= 1e-11 * np.abs(Fo).max()
    assert nrm == float(F.abs().max())
    nrm2 = asm.mismatch(xd, F, dx=dxd, alpha=-0.25, x_out=xt)
    x2 = x + (-0.25) * dx
    assert np.array_equal(xt.cpu().numpy(), x2)
    F2 = NT.mismatch(prob, x2)
    assert np.abs(F.cpu().numpy() - F2).max() <= 1e-12 * np.abs(F2).max()
    assert nrm2 == float(F.abs().max())
    Gu = torch.full((asm.n_ctrl, asm.n), 7.0, dtype=torch.float64, device="cuda").t()
    A.nzVal.fill_(7.0)
    asm.jacobian(xd, Gu)
    J0 = NT.jacobian_values(prob, x)
    assert np.abs(A.nzVal.cpu().numpy() - J0).max() <= 1e-12 * np.abs(J0).max()
    Gu0 = NT.control_jacobian(prob, x)
    assert np.abs(Gu.cpu().numpy() - Gu0).max() <= 1e-12 * np.abs(Gu0).max()
    assert np.abs(A.nzVal.cpu().numpy() - gxo).max() <= 1e-11 * np.abs(gxo).max()
    assert np.abs(Gu.cpu().numpy() - Guo).max() <= 1e-11 * np.abs(Guo).max()
    xd[3] = float("nan")
    assert np.isnan(asm.mismatch(xd, F))


def test_device_assembly_rejects_a_pattern_it_cannot_fill(bpf):
    from blockpowerflow_b200 import _lib

    prob = NT.make_problem(G.make_grid(300, seed=3))
    P = prob.pattern.tolil()
    r = 5
    c = [j for j in P.rows[r] if j != r][0]
    P[r, c] = 0
    P = P.tocsr()
    P.eliminate_zeros()
    with pytest.raises(_lib.BPFError, match="lacks entry"):
        NT.DeviceAssembly(prob, bpf.CuSparseMatrixCSR.from_scipy(P))
    small = sp.csr_matrix(prob.pattern[:-1, :-1])
    with pytest.raises(_lib.DimensionMismatch):
        NT.DeviceAssembly(prob, bpf.CuSparseMatrixCSR.from_scipy(small))


def test_a_reused_solver_serves_a_second_power_flow(bpf):
    """One RFSolver (one analysis) for two power flows on the same pattern: the second solve
    repeats the first (the refactorization starts from fresh values every step)."""
    prob = NT.make_problem(G.make_grid(300, seed=7))
    x0 = NT.perturbed_start(prob, 0.01, seed=2)
    lin = NT.RFSolver(prob, len(prob.ctrl))
    r1 = NT.newton(prob, solver=lin, x0=x0, tol=1e-10, sensitivities=True)
    r2 = NT.newton(prob, solver=lin, x0=x0, tol=1e-10, sensitivities=True)
    assert r1.converged and r2.converged and r1.iterations == r2.iterations
    np.testing.assert_allclose(r2.x, r1.x, rtol=0, atol=1e-12)
    err = np.linalg.norm(r2.sensitivities - r1.sensitivities) / np.linalg.norm(r1.sensitivities)
    assert err <= 1e-12, err


def test_dump_ingest_and_the_benchmark_solve(bpf, tmp_path):
    from blockpowerflow_b200 import mm

    d = np.load(os.path.join(GOLDEN, "dump_case300.npz"))
    A = sp.csr_matrix((d["data"], d["indices"], d["indptr"]), shape=tuple(d["shape"]))
    pa, pb = mm.dump_paths(str(tmp_path), "case300")
    mmwrite(pa, A)
    mmwrite(pb, sp.coo_matrix(d["Gu"]))
    Ah, Bh = mm.load_dump(str(tmp_path), "case300")
    X, st, rn = mm.solve_dump(Ah, Bh, atol=0.0, rtol=1e-12, memory=100, itmax=200)
    assert st.solved
    assert np.linalg.norm(X - d["X"]) / np.linalg.norm(d["X"]) <= 1e-8
    assert abs(rn - np.linalg.norm(Bh - Ah @ X)) <= 1e-12 * max(rn, 1.0)
    # the script's own parameters (atol 1e-10, rtol 0, memory 1, restart false, itmax 50)
    X2, st2, rn2 = mm.solve_dump(Ah, Bh)
    assert st2.niter <= 50 and np.isfinite(rn2)
    if st2.solved:
        assert rn2 <= 1e-9, rn2
