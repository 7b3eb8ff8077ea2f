"""Device power-flow assembly, host side (no GPU): the arguments bus_arrays() gives bpf_pf_create
describe the same problem as the numpy assembly.  The oracle's entry-by-entry restatement over
those arrays (oracle.pf_assemble: theta / P index of every non-slack bus in bus order, |V| / Q
index of every PQ bus after them, control columns the slack bus then the PV buses in bus order;
per Ybus entry (i, k) the four Gx entries (P_i | Q_i, theta_k | |V|_k) that exist, the index
convention of csrc/pf.cu) must reproduce mismatch(), jacobian_values() and control_jacobian()."""
import numpy as np
import pytest

import oracle as O
from blockpowerflow_b200 import grid as G
from blockpowerflow_b200 import newton as NT


@pytest.mark.parametrize("n_bus,n_pv,seed", [(300, 68, 3), (1200, None, 5)])
def test_oracle_assembly_over_bus_arrays_matches_the_numpy_assembly(n_bus, n_pv, seed):
    prob = NT.make_problem(G.make_grid(n_bus, n_pv, seed=seed))
    x = NT.perturbed_start(prob, 0.05, seed=seed)
    F, gx, Gu = O.pf_assemble(*NT.bus_arrays(prob), x, prob.pattern)
    F0 = NT.mismatch(prob, x)
    assert np.abs(F - F0).max() <= 1e-12 * max(1.0, np.abs(F0).max())
    J0 = NT.jacobian_values(prob, x)
    assert np.abs(gx - J0).max() <= 1e-12 * np.abs(J0).max()
    Gu0 = NT.control_jacobian(prob, x)
    assert Gu.shape == Gu0.shape
    assert np.abs(Gu - Gu0).max() <= 1e-12 * np.abs(Gu0).max()


def test_oracle_assembly_rejects_a_pattern_without_a_coupling_entry():
    prob = NT.make_problem(G.make_grid(300, 68, seed=3))
    P = prob.pattern.tolil()
    r = 5
    c = [j for j in P.rows[r] if j != r][0]
    P[r, c] = 0
    P = P.tocsr()
    P.eliminate_zeros()
    x = NT.perturbed_start(prob, 0.05, seed=3)
    with pytest.raises(ValueError, match="lacks entry"):
        O.pf_assemble(*NT.bus_arrays(prob), x, P)


def test_bus_arrays_reject_a_layout_the_kernels_do_not_index():
    prob = NT.make_problem(G.make_grid(300, 68, seed=3))
    bad = NT.PowerFlowProblem(prob.grid, prob.s_spec, prob.vm_ctrl[::-1].copy(), prob.ctrl[::-1].copy(),
                              prob.pattern)
    with pytest.raises(ValueError):
        NT.bus_arrays(bad)
