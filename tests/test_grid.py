"""Synthetic Newton power-flow Jacobians: shapes, determinism and derivative checks (no GPU)."""
import numpy as np

from blockpowerflow_b200 import grid as g


def test_presets_shapes():
    J = g.preset_jacobian("case300", 0)
    assert J.shape == (530, 530)
    assert 3000 < J.nnz < 5000
    J9 = g.preset_jacobian("case9k", 0)
    assert J9.shape[0] == 16998 and 100_000 < J9.nnz < 140_000


def test_seeded_determinism():
    a = g.synthetic_jacobian(500, 50, seed=7)
    b = g.synthetic_jacobian(500, 50, seed=7)
    c = g.synthetic_jacobian(500, 50, seed=8)
    assert (a != b).nnz == 0
    assert a.shape != c.shape or (a != c).nnz > 0


def test_jacobian_matches_finite_differences():
    grid = g.make_grid(40, 6, seed=2)
    J = g.jacobian(grid).toarray()
    Y = grid.ybus()
    nonslack = np.arange(1, grid.n_bus)

    def mismatch(va, vm):
        V = vm * np.exp(1j * va)
        S = V * np.conj(Y @ V)
        return np.concatenate([S.real[nonslack], S.imag[grid.pq]])

    x0 = np.concatenate([grid.va[nonslack], grid.vm[grid.pq]])
    h = 1e-7
    Jfd = np.zeros_like(J)
    for k in range(len(x0)):
        for sgn in (1, -1):
            x = x0.copy()
            x[k] += sgn * h
            va, vm = grid.va.copy(), grid.vm.copy()
            va[nonslack] = x[: len(nonslack)]
            vm[grid.pq] = x[len(nonslack):]
            Jfd[:, k] += sgn * mismatch(va, vm) / (2 * h)
    np.testing.assert_allclose(J, Jfd, rtol=1e-5, atol=1e-5)


def test_perturbed_values_keep_pattern():
    grid = g.make_grid(200, 20, seed=1)
    J = g.jacobian(grid)
    v = g.perturbed_values(grid, J, 3)
    assert v.shape == (J.nnz,)
    assert np.abs(v - J.data).max() > 0
