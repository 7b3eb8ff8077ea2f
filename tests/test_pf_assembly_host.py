"""Device power-flow assembly, host side (no GPU): the arguments bus_arrays() gives bpf_pf_create
describe the same problem as the numpy assembly.  The index convention of csrc/pf.cu (theta / P
index of every non-slack bus in bus order, |V| / Q index of every PQ bus after them, control
columns: the slack bus then the PV buses in bus order; per Ybus entry (i, k) the four Gx entries
(P_i | Q_i, theta_k | |V|_k) that exist) is restated here in numpy over those arrays and must
reproduce mismatch(), jacobian_values() and control_jacobian()."""
import numpy as np
import pytest
import scipy.sparse as sp

from blockpowerflow_b200 import grid as G
from blockpowerflow_b200 import newton as NT


def _convention(bt):
    nb = len(bt)
    slack = int(np.flatnonzero(bt == 3)[0])
    ia = np.full(nb, -1)
    ia[np.arange(nb) != slack] = np.arange(nb - 1)
    pq = np.flatnonzero(bt == 1)
    im = np.full(nb, -1)
    im[pq] = nb - 1 + np.arange(len(pq))
    ctrl_buses = np.concatenate([[slack], np.flatnonzero(bt == 2)])
    ctrl = np.full(nb, -1)
    ctrl[ctrl_buses] = np.arange(len(ctrl_buses))
    return ia, im, ctrl


def _restated(prob, x):
    rp, ci, yv, bt, vmf, vaf, ss = NT.bus_arrays(prob)
    nb = len(bt)
    ia, im, ctrl = _convention(bt)
    n = int((ia >= 0).sum() + (im >= 0).sum())
    y = yv[0::2] + 1j * yv[1::2]
    rows = np.repeat(np.arange(nb), np.diff(rp))
    assert all(i in ci[rp[i]:rp[i + 1]] for i in range(nb))   # every row holds its diagonal
    va = np.where(ia >= 0, x[np.maximum(ia, 0)], vaf)
    vm = np.where(im >= 0, x[np.maximum(im, 0)], vmf)
    V = vm * np.exp(1j * va)
    t = y * V[ci]
    I = np.bincount(rows, t.real, nb) + 1j * np.bincount(rows, t.imag, nb)
    S = V * np.conj(I) - (ss[0::2] + 1j * ss[1::2])
    F = np.zeros(n)
    F[ia[ia >= 0]] = S.real[ia >= 0]
    F[im[im >= 0]] = S.imag[im >= 0]
    i, k = rows, ci
    diag = i == k
    dth = 1j * V[i] * (np.where(diag, np.conj(I[i]), 0) - np.conj(y * V[k]))
    dm = V[i] * np.conj(y * V[k] / np.abs(V[k])) + np.where(diag, np.conj(I[i]) * V[i] / np.abs(V[i]), 0)
    r, c, v = [], [], []
    for rr, cc, vv in ((ia[i], ia[k], dth.real), (ia[i], im[k], dm.real),
                       (im[i], ia[k], dth.imag), (im[i], im[k], dm.imag)):
        keep = (rr >= 0) & (cc >= 0)
        r.append(rr[keep]), c.append(cc[keep]), v.append(vv[keep])
    Gx = sp.csr_matrix((np.concatenate(v), (np.concatenate(r), np.concatenate(c))), shape=(n, n))
    nctrl = int((ctrl >= 0).sum())
    Gu = np.zeros((n, nctrl))
    sel = ctrl[k] >= 0
    for rr, vv in ((ia[i], dm.real), (im[i], dm.imag)):
        s2 = sel & (rr >= 0)
        Gu[rr[s2], ctrl[k][s2]] = vv[s2]
    return F, Gx, Gu


@pytest.mark.parametrize("n_bus,n_pv,seed", [(300, 68, 3), (1200, None, 5)])
def test_bus_arrays_restate_the_numpy_assembly(n_bus, n_pv, seed):
    prob = NT.make_problem(G.make_grid(n_bus, n_pv, seed=seed))
    x = NT.perturbed_start(prob, 0.05, seed=seed)
    F, Gx, Gu = _restated(prob, x)
    F0 = NT.mismatch(prob, x)
    assert np.abs(F - F0).max() <= 1e-12 * max(1.0, np.abs(F0).max())
    pat = prob.pattern
    J0 = sp.csr_matrix((NT.jacobian_values(prob, x), pat.indices, pat.indptr), shape=pat.shape)
    # every restated entry lies on the fixed pattern (the device map's requirement), same values
    on = sp.csr_matrix((np.ones(pat.nnz), pat.indices, pat.indptr), shape=pat.shape)
    assert (abs(Gx).astype(bool) > on.astype(bool)).nnz == 0
    assert abs(Gx - J0).max() <= 1e-12 * abs(J0).max()
    Gu0 = NT.control_jacobian(prob, x)
    assert Gu.shape == Gu0.shape
    assert np.abs(Gu - Gu0).max() <= 1e-12 * np.abs(Gu0).max()


def test_bus_arrays_reject_a_layout_the_kernels_do_not_index():
    prob = NT.make_problem(G.make_grid(300, 68, seed=3))
    bad = NT.PowerFlowProblem(prob.grid, prob.s_spec, prob.vm_ctrl[::-1].copy(), prob.ctrl[::-1].copy(),
                              prob.pattern)
    with pytest.raises(ValueError):
        NT.bus_arrays(bad)
