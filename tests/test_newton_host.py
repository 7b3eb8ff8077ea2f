"""Host logic of the Newton power-flow driver (no GPU): the mismatch vanishes at the grid's
operating point, the Jacobian on the fixed pattern and the control Jacobian Gu match finite
differences of the mismatch, and Newton's loop (with a SciPy stand-in for the device solves,
passed explicitly; the library has no CPU solver) converges quadratically from an operating point
perturbed by N(0, 0.01)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from blockpowerflow_b200 import grid as G
from blockpowerflow_b200 import newton as NT


@pytest.fixture(scope="module")
def prob():
    return NT.make_problem(G.make_grid(300, 68, seed=3))


def test_mismatch_vanishes_at_the_operating_point(prob):
    g = prob.grid
    x = np.concatenate([g.va[1:], g.vm[g.pq]])
    assert np.abs(NT.mismatch(prob, x)).max() <= 1e-12
    vm, va = NT.state_to_voltages(prob, x)
    np.testing.assert_allclose(vm, g.vm, rtol=0, atol=0)
    np.testing.assert_allclose(va, g.va, rtol=0, atol=0)


def test_jacobians_match_finite_differences(prob):
    rng = np.random.default_rng(0)
    x = NT.flat_start(prob) + 0.05 * rng.standard_normal(prob.pattern.shape[0])
    J = sp.csr_matrix((NT.jacobian_values(prob, x), prob.pattern.indices, prob.pattern.indptr),
                      shape=prob.pattern.shape)
    d = rng.standard_normal(len(x))
    h = 1e-6
    fd = (NT.mismatch(prob, x + h * d) - NT.mismatch(prob, x - h * d)) / (2 * h)
    assert np.linalg.norm(J @ d - fd) <= 1e-6 * np.linalg.norm(fd)
    Gu = NT.control_jacobian(prob, x)
    du = rng.standard_normal(len(prob.ctrl))
    p2 = NT.PowerFlowProblem(prob.grid, prob.s_spec, prob.vm_ctrl + h * du, prob.ctrl, prob.pattern)
    p3 = NT.PowerFlowProblem(prob.grid, prob.s_spec, prob.vm_ctrl - h * du, prob.ctrl, prob.pattern)
    fdu = (NT.mismatch(p2, x) - NT.mismatch(p3, x)) / (2 * h)
    assert np.linalg.norm(Gu @ du - fdu) <= 1e-6 * np.linalg.norm(fdu)


class _SciPyStandIn:
    def __init__(self, pattern):
        self.pattern = pattern
        self.lu = None

    def refactor(self, vals):
        J = sp.csc_matrix(sp.csr_matrix((vals, self.pattern.indices, self.pattern.indptr),
                                        shape=self.pattern.shape))
        self.lu = spla.splu(J)

    def solve(self, B):
        return self.lu.solve(np.asarray(B))


def test_newton_converges_quadratically_with_a_stand_in_solver(prob):
    r = NT.newton(prob, solver=_SciPyStandIn(prob.pattern), tol=1e-10, sensitivities=True,
                  x0=NT.perturbed_start(prob, 0.01, seed=1))
    assert r.converged and r.iterations <= 12, r.residuals
    np.testing.assert_allclose(r.vm, prob.grid.vm, atol=1e-9)
    np.testing.assert_allclose(r.va, prob.grid.va, atol=1e-9)
    # quadratic convergence: each of the last two steps squares the residual (up to a constant)
    rs = r.residuals
    assert rs[-1] <= 100 * rs[-2] ** 2 + 1e-13 and rs[-2] <= 100 * rs[-3] ** 2 + 1e-13, rs
    # the sensitivity of the state to the control voltages, against finite differences of the solve
    h = 1e-6
    du = np.zeros(len(prob.ctrl))
    du[1] = 1.0
    p2 = NT.PowerFlowProblem(prob.grid, prob.s_spec, prob.vm_ctrl + h * du, prob.ctrl, prob.pattern)
    r2 = NT.newton(p2, solver=_SciPyStandIn(prob.pattern), tol=1e-12, x0=r.x)
    fd = (r2.x - r.x) / h
    assert np.linalg.norm(r.sensitivities[:, 1] - fd) <= 1e-4 * np.linalg.norm(fd)


def test_jacobian_values_match_the_sparse_product_jacobian(prob):
    """The position-map assembly of jacobian_values equals grid.jacobian_on_pattern (the sparse
    matrix-product form) on the fixed pattern, and its map is built once per problem."""
    x = NT.perturbed_start(prob, 0.05, seed=4)
    vm, va = NT.state_to_voltages(prob, x)
    ref = G.jacobian_on_pattern(prob.grid, prob.pattern, vm, va)
    got = NT.jacobian_values(prob, x)
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    cached = prob.__dict__["_coupling_cache"]
    NT.jacobian_values(prob, NT.perturbed_start(prob, 0.05, seed=5))
    assert prob.__dict__["_coupling_cache"] is cached
