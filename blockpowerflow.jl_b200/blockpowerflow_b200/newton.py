"""Newton power-flow driver: the caller of the multi-RHS solve path.

The reference's solvers serve a Newton power-flow loop (ExaPF produced the benchmark dumps
Gx / Gu, benchmarks/benchmarks_nvidia.jl:29-39, and the refactorization is its per-step hot call,
src/cusolverRF.jl:304-314): at every Newton step the Jacobian Gx gets new values on a fixed
sparsity pattern, is refactored, and the correction is solved; at the solution the sensitivities
Gx^{-1} Gu of the state to the controls are a multi-RHS solve.  This module is that loop, with
every linear solve in libbpf.so and, with the device solvers, the mismatch, Gx and Gu assembled
there too (bpf_pf_*), so that only max |F| crosses to the host per evaluation.

Problem: a grid (grid.Grid) with its operating point taken as the solution: the injections
S_spec = V conj(Ybus V) at that point fix P at every non-slack bus and Q at every PQ bus; the
voltage magnitudes of the slack and PV buses and the slack angle are controls.  Unknowns x =
[theta(non-slack); |V|(PQ)], equations F(x) = [P(non-slack); Q(PQ)] of S(V(x)) - S_spec, Jacobian
dF/dx = grid.jacobian (the layout of ExaPF's Gx).  Controls u = |V| at the slack and PV buses;
Gu = dF/du (dense, n x (1 + n_pv)).
"""
from __future__ import annotations

import dataclasses

import numpy as np
import scipy.sparse as sp

from . import grid as G


@dataclasses.dataclass
class PowerFlowProblem:
    grid: G.Grid
    s_spec: np.ndarray        # complex injections at the solution
    vm_ctrl: np.ndarray       # |V| of the control buses (slack and PV), in ctrl order
    ctrl: np.ndarray          # control buses: slack (0) then the PV buses
    pattern: sp.csr_matrix    # fixed sparsity of Gx over every Newton step


def _injections(grid: G.Grid, vm, va) -> np.ndarray:
    V = vm * np.exp(1j * va)
    return V * np.conj(grid.ybus() @ V)


def make_problem(grid: G.Grid) -> PowerFlowProblem:
    """The power flow whose solution is the grid's operating point."""
    s = _injections(grid, grid.vm, grid.va)
    ctrl = np.concatenate([[0], np.setdiff1d(grid.pv, [0])]).astype(np.int64)
    # Structural pattern of Gx: the Jacobian at a generic point (no cancellations), so that
    # every Newton step's values fit it (grid.jacobian_on_pattern checks this).
    rng = np.random.default_rng(12345)
    vm_g = grid.vm * (1.0 + 0.01 * rng.standard_normal(grid.n_bus))
    va_g = grid.va + 0.01 * rng.standard_normal(grid.n_bus)
    va_g[0] = 0.0
    pattern = G.jacobian(grid, vm_g, va_g)
    return PowerFlowProblem(grid, s, grid.vm[ctrl].copy(), ctrl, pattern)


def state_to_voltages(prob: PowerFlowProblem, x: np.ndarray):
    """(vm, va) of every bus from the unknowns x = [theta(non-slack); |V|(PQ)]."""
    g = prob.grid
    nb = g.n_bus
    va = np.zeros(nb)
    va[1:] = x[:nb - 1]
    vm = np.empty(nb)
    vm[prob.ctrl] = prob.vm_ctrl
    vm[g.pq] = x[nb - 1:]
    return vm, va


def flat_start(prob: PowerFlowProblem) -> np.ndarray:
    """theta = 0, |V| = 1 at the PQ buses.  (The synthetic grids' operating points are random, with
    large flows; from the flat start Newton may reach another solution of these lossless networks
    or stall, so the loop is normally started near the previous operating point.)"""
    g = prob.grid
    return np.concatenate([np.zeros(g.n_bus - 1), np.ones(len(g.pq))])


def perturbed_start(prob: PowerFlowProblem, sigma: float = 0.01, seed: int = 0) -> np.ndarray:
    """The solution's state with N(0, sigma) added to every angle and PQ magnitude: the start of
    a Newton step sequence whose operating point moved by N(0, sigma) (the perturbation of the
    refactorization benchmark's Jacobian sequence)."""
    g = prob.grid
    rng = np.random.default_rng(seed)
    x = np.concatenate([g.va[1:], g.vm[g.pq]])
    return x + rng.normal(0.0, sigma, len(x))


def mismatch(prob: PowerFlowProblem, x: np.ndarray) -> np.ndarray:
    """F(x) = [P(non-slack); Q(PQ)] of S(V(x)) - S_spec."""
    vm, va = state_to_voltages(prob, x)
    d = _injections(prob.grid, vm, va) - prob.s_spec
    return np.concatenate([d.real[1:], d.imag[prob.grid.pq]])


def _coupling(prob: PowerFlowProblem):
    """Ybus (CSR, duplicates summed) and, per Ybus entry (i, k), the positions in prob.pattern of
    (P_i | Q_i) x (theta_k | |V|_k) (-1 where the row or column is not an unknown); built once per
    pattern and kept on the problem.  None if a nonempty Ybus row lacks its diagonal (the I_i terms
    attach there)."""
    key = (id(prob.pattern), prob.pattern.nnz)
    cached = prob.__dict__.get("_coupling_cache")
    if cached is not None and cached[0] == key:
        return cached[1]
    g = prob.grid
    nb = g.n_bus
    Y = g.ybus().tocsr()
    Y.sum_duplicates()
    Y.sort_indices()
    rows = np.repeat(np.arange(nb), np.diff(Y.indptr))
    cols = Y.indices
    has_diag = np.zeros(nb, dtype=bool)
    has_diag[rows[rows == cols]] = True
    if np.any(~has_diag & (np.diff(Y.indptr) > 0)):
        prob.__dict__["_coupling_cache"] = (key, None)
        return None
    prow = np.arange(nb) - 1                      # P row / theta column of bus i (-1: slack)
    qrow = np.full(nb, -1)
    qrow[g.pq] = nb - 1 + np.arange(len(g.pq))    # Q row / |V| column of a PQ bus
    P = prob.pattern
    n = P.shape[0]
    keys = np.repeat(np.arange(n, dtype=np.int64), np.diff(P.indptr)) * n + P.indices
    maps = []
    for r, c in ((prow[rows], prow[cols]), (prow[rows], qrow[cols]), (qrow[rows], prow[cols]), (qrow[rows], qrow[cols])):
        ok = (r >= 0) & (c >= 0)
        k = r.astype(np.int64) * n + c
        pos = np.searchsorted(keys, k)
        pos = np.minimum(pos, len(keys) - 1)
        found = ok & (keys[pos] == k)
        if np.any(ok & ~found & (Y.data != 0)):
            raise ValueError("the Jacobian left the fixed sparsity pattern")
        maps.append(np.where(found, pos, -1))
    out = (Y, rows, cols, maps)
    prob.__dict__["_coupling_cache"] = (key, out)
    return out


def jacobian_values(prob: PowerFlowProblem, x: np.ndarray) -> np.ndarray:
    """Gx's values on the fixed pattern (CSR order): per Ybus entry (i, k),
    dS_i/dtheta_k = j V_i ([i == k] conj(I_i) - conj(Y_ik V_k)) and
    dS_i/d|V_k| = V_i conj(Y_ik V_k / |V_k|) + [i == k] conj(I_i) V_i / |V_i|, scattered through
    the position map of _coupling (the assembly the device runs)."""
    vm, va = state_to_voltages(prob, x)
    cpl = _coupling(prob)
    if cpl is None:
        return G.jacobian_on_pattern(prob.grid, prob.pattern, vm, va)
    Y, rows, cols, maps = cpl
    V = vm * np.exp(1j * va)
    I = Y @ V
    y = Y.data
    diag = rows == cols
    dth = 1j * V[rows] * (np.where(diag, np.conj(I[rows]), 0) - np.conj(y * V[cols]))
    dm = V[rows] * np.conj(y * V[cols] / np.abs(V[cols])) + np.where(diag, np.conj(I[rows]) * V[rows] / np.abs(V[rows]), 0)
    out = np.zeros(prob.pattern.nnz)
    for m, v in zip(maps, (dth.real, dm.real, dth.imag, dm.imag)):
        ok = m >= 0
        out[m[ok]] = v[ok]
    return out


def control_jacobian(prob: PowerFlowProblem, x: np.ndarray) -> np.ndarray:
    """Gu = dF/du, u = |V| of the control buses (dense, n_unknowns x n_ctrl):
    dS/d|V| = diag(V) conj(Ybus diag(V / |V|)) + conj(diag(Ybus V)) diag(V / |V|)."""
    g = prob.grid
    vm, va = state_to_voltages(prob, x)
    Y = g.ybus().tocsc()
    V = vm * np.exp(1j * va)
    I = Y @ V
    Vn = V / np.abs(V)
    # only the control columns: the entries of Y(:, ctrl), then the diagonal terms
    sub = Y[:, prob.ctrl]
    rows = sub.indices
    j = np.repeat(np.arange(len(prob.ctrl)), np.diff(sub.indptr))
    k = prob.ctrl[j]
    vals = V[rows] * np.conj(sub.data * Vn[k])
    nb, nc = g.n_bus, len(prob.ctrl)
    # written straight into [P rows (buses 1..nb-1); Q rows (PQ buses)]
    qrow = np.full(nb, -1)
    qrow[g.pq] = nb - 1 + np.arange(len(g.pq))
    out = np.zeros((nb - 1 + len(g.pq), nc))
    for r, c, v in ((rows, j, vals), (prob.ctrl, np.arange(nc), np.conj(I[prob.ctrl]) * Vn[prob.ctrl])):
        p_ok = r >= 1
        np.add.at(out, (r[p_ok] - 1, c[p_ok]), v.real[p_ok])
        q_ok = qrow[r] >= 0
        np.add.at(out, (qrow[r[q_ok]], c[q_ok]), v.imag[q_ok])
    return out


def bus_arrays(prob: PowerFlowProblem):
    """The host arguments of bpf_pf_create for this problem, in its order: Ybus row pointers,
    columns and interleaved (re, im) values (sorted, duplicates summed), bus types (1 PQ, 2 PV,
    3 slack), |V| and angle where they are fixed, interleaved specified injections."""
    g = prob.grid
    nb = g.n_bus
    bus_type = np.ones(nb, dtype=np.int32)
    bus_type[prob.ctrl] = 2
    bus_type[0] = 3
    # the problem's layout: slack bus 0, PV controls and PQ unknowns in bus order
    if (prob.ctrl[0] != 0 or np.any(np.diff(prob.ctrl[1:]) <= 0) or np.any(np.diff(g.pq) <= 0)
            or not np.array_equal(np.flatnonzero(bus_type == 1), g.pq)):
        raise ValueError("power flow: buses must be slack 0, then PV / PQ sets in bus order")
    Y = g.ybus().tocsr()
    Y.sum_duplicates()
    Y.sort_indices()
    vm_fixed = np.ones(nb)
    vm_fixed[prob.ctrl] = prob.vm_ctrl
    return [np.ascontiguousarray(Y.indptr, dtype=np.int32),
            np.ascontiguousarray(Y.indices, dtype=np.int32),
            np.ascontiguousarray(np.column_stack([Y.data.real, Y.data.imag]).ravel()),
            bus_type, vm_fixed, np.zeros(nb),
            np.ascontiguousarray(np.column_stack([prob.s_spec.real, prob.s_spec.imag]).ravel())]


class DeviceAssembly:
    """F, Gx and Gu of a problem assembled on the device (bpf_pf_create / _mismatch / _jacobian):
    the same quantities as mismatch(), jacobian_values() and control_jacobian(), with Gx written
    straight into the values of the solver's matrix A (its pattern is prob.pattern)."""

    def __init__(self, prob: PowerFlowProblem, A):
        import ctypes as C

        from . import _lib

        nb = prob.grid.n_bus
        self._keep = bus_arrays(prob)
        self.A = A
        self._device = A.nzVal.device
        self._dev = A.nzVal.device.index
        self._ctx = _lib.context(self._dev)
        self._lib = _lib
        h = C.c_void_p()
        d = A.desc()
        ptr = [a.ctypes.data for a in self._keep]
        _lib.check(_lib.load().bpf_pf_create(self._ctx, nb, *ptr, C.byref(d), C.byref(h)), self._ctx)
        self._h = h
        n, nc = C.c_int(), C.c_int()
        _lib.check(_lib.load().bpf_pf_info(h, C.byref(n), C.byref(nc), None), self._ctx)
        self.n, self.n_ctrl = n.value, nc.value

    def mismatch(self, x, F, dx=None, alpha=0.0, x_out=None) -> float:
        """F = F(x + alpha dx) (device tensors; x_out, if given, receives that point);
        returns max |F|."""
        import ctypes as C

        for v in (x, F, dx, x_out):
            if v is not None:
                self._check_vector(v)
        self._ctx = self._lib.context(self._dev)    # bound to torch's current stream
        nrm = C.c_double()
        self._lib.check(self._lib.load().bpf_pf_mismatch(
            self._h, x.data_ptr(), None if dx is None else dx.data_ptr(), float(alpha),
            None if x_out is None else x_out.data_ptr(), F.data_ptr(), C.byref(nrm)), self._ctx)
        return nrm.value

    def _check_vector(self, v):
        import torch

        if v.dtype != torch.float64 or v.device != self._device or v.numel() != self.n or not v.is_contiguous():
            raise ValueError(f"power flow: expected a contiguous float64 vector of {self.n} entries on "
                             f"{self._device}")

    def jacobian(self, x, Gu=None) -> None:
        """Gx at x into A.nzVal; Gu (column-major n x n_ctrl device block), if given, = dF/du."""
        import torch

        self._check_vector(x)
        ld = 0 if Gu is None else (Gu.stride(1) if Gu.shape[1] > 1 else Gu.shape[0])
        if Gu is not None and (Gu.dtype != torch.float64 or Gu.device != self._device or Gu.dim() != 2
                               or Gu.stride(0) != 1 or tuple(Gu.shape) != (self.n, self.n_ctrl)
                               or ld < self.n):
            raise ValueError("Gu must be a column-major float64 n x n_ctrl block on the matrix's device")
        if self.A.nzVal.numel() != self.A.nnz:
            raise ValueError("power flow: the matrix's values changed size")
        self._ctx = self._lib.context(self._dev)
        self._lib.check(self._lib.load().bpf_pf_jacobian(
            self._h, x.data_ptr(), self.A.nzVal.data_ptr(), None if Gu is None else Gu.data_ptr(), ld),
            self._ctx)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                self._lib.load().bpf_pf_destroy(h)
            except Exception:
                pass


@dataclasses.dataclass
class NewtonResult:
    x: np.ndarray
    vm: np.ndarray
    va: np.ndarray
    iterations: int
    converged: bool
    residuals: list            # ||F||_inf before each step and at the end
    sensitivities: np.ndarray | None = None   # dx/du = -Gx^{-1} Gu at the solution


class RFSolver:
    """Linear solves of the loop on the cusolverRF-style refactorization: analysis once, then
    refactor + solve per Newton step; the sensitivities reuse the last factorization.  One
    instance serves every power flow on the same pattern (pass it as newton(solver=...)): the
    analysis is then paid once, as the reference's CusolverRfLU object is built once and
    refactored per step (src/cusolverRF.jl:222,304-314)."""

    def __init__(self, prob, nrhs=1, ordering="AMD"):
        import torch

        from . import cusolverrf as RF
        from .sparse import CuSparseMatrixCSR

        self.RF, self.torch = RF, torch
        self.A = CuSparseMatrixCSR.from_scipy(prob.pattern)
        self.rf = RF.CusolverRfLU(self.A, nrhs=max(1, nrhs), ordering=ordering)

    def refactor(self, vals):
        self.A.nzVal.copy_(self.torch.as_tensor(vals, device=self.A.nzVal.device))
        self.RF.update_(self.rf, self.A)

    def solve(self, B):
        from .sparse import colmajor

        X = colmajor(self.torch.as_tensor(np.asarray(B, dtype=np.float64).reshape(B.shape[0], -1),
                                          device=self.A.nzVal.device))
        X = X.clone()
        self.RF.ldiv_(self.rf, X)
        return X.cpu().numpy()

    def refactor_device(self):
        """Refactor from the values already in A.nzVal."""
        self.RF.update_(self.rf, self.A)

    def solve_device(self, B, X=None):
        """X = Gx^{-1} B for a column-major device block B (X: a like-shaped block, or in place)."""
        X = B if X is None else X
        if X.data_ptr() != B.data_ptr():
            X.copy_(B)
        self.RF.ldiv_(self.rf, X)
        return X


class GmresSolver:
    """Linear solves of the loop by ILU(0)-preconditioned block-GMRES (refactor per step); reusable
    across power flows on the same pattern like RFSolver."""

    def __init__(self, prob, nrhs=1, ordering="AMD", rtol=1e-12):
        import torch

        from . import precond
        from .sparse import CuSparseMatrixCSR

        self.torch = torch
        self.A = CuSparseMatrixCSR.from_scipy(prob.pattern)
        self.N = precond.ilu0(self.A, max(1, nrhs), ordering=ordering)
        self.rtol = rtol

    def refactor(self, vals):
        self.A.nzVal.copy_(self.torch.as_tensor(vals, device=self.A.nzVal.device))
        self.N.refactor(self.A.nzVal)

    def solve(self, B):
        """block_gmres on slices of at most 128 columns (the widest block it takes)."""
        from . import krylov

        B2 = np.asarray(B, dtype=np.float64).reshape(B.shape[0], -1)
        out = np.empty_like(B2)
        for c0 in range(0, B2.shape[1], 128):
            Bc = self.torch.as_tensor(np.ascontiguousarray(B2[:, c0:c0 + 128]), device=self.A.nzVal.device)
            X, st = krylov.block_gmres(self.A, Bc, N=self.N, ldiv=True, restart=False, memory=200, atol=0.0,
                                       rtol=self.rtol, itmax=400)
            out[:, c0:c0 + 128] = X.cpu().numpy()
        return out

    def refactor_device(self):
        self.N.refactor(self.A.nzVal)

    def solve_device(self, B, X=None):
        """X = Gx^{-1} B for a column-major device block B, by slices of at most 128 columns."""
        from . import krylov

        X = self.torch.empty_like(B) if X is None or X.data_ptr() == B.data_ptr() else X
        Bm, Xm = B.reshape(B.shape[0], -1), X.reshape(X.shape[0], -1)
        for c0 in range(0, Bm.shape[1], 128):
            Xc, st = krylov.block_gmres(self.A, Bm[:, c0:c0 + 128], N=self.N, ldiv=True, restart=False,
                                        memory=200, atol=0.0, rtol=self.rtol, itmax=400)
            Xm[:, c0:c0 + 128].copy_(Xc)
        return X


def newton(prob: PowerFlowProblem, *, solver="rf", tol: float = 1e-10, maxiter: int = 20,
           x0: np.ndarray | None = None, sensitivities: bool = False, ordering: str = "AMD",
           line_search: bool = True) -> NewtonResult:
    """Newton's method F(x) = 0 from x0 (default: the flat start), stopping at ||F||_inf <= tol;
    with line_search, a step is halved (down to 2^-12) until ||F||_inf decreases.

    solver: "rf" (refactor + direct solve per step on the device, the reference's per-Newton-
    step use of CusolverRfLU), "gmres" (ILU(0) refactor + block-GMRES), an RFSolver /
    GmresSolver built earlier for this pattern (its analysis reused), or an object with
    refactor(values) and solve(B) methods (a host stand-in: then F, Gx and Gu are assembled by
    numpy).  With "rf" / "gmres" the mismatch, Gx and Gu are assembled on the device
    (DeviceAssembly) and x, F and the steps stay there.  With sensitivities=True, dx/du =
    -Gx^{-1} Gu at the solution (one multi-RHS solve)."""
    n_ctrl = len(prob.ctrl)
    nrhs = n_ctrl if sensitivities else 1
    if solver == "rf":
        lin = RFSolver(prob, nrhs, ordering)
    elif solver == "gmres":
        lin = GmresSolver(prob, nrhs, ordering)
    else:
        lin = solver
    if hasattr(lin, "solve_device"):
        return _newton_device(prob, lin, tol, maxiter, x0, sensitivities, line_search)
    x = flat_start(prob) if x0 is None else np.array(x0, dtype=np.float64)
    res = []
    converged = False
    it = 0
    for it in range(maxiter + 1):
        F = mismatch(prob, x)
        res.append(float(np.abs(F).max()))
        if res[-1] <= tol:
            converged = True
            break
        if it == maxiter:
            break
        lin.refactor(jacobian_values(prob, x))
        dx = -lin.solve(F[:, None])[:, 0]
        a = 1.0
        if line_search:
            while a > 2.0 ** -12 and np.abs(mismatch(prob, x + a * dx)).max() >= res[-1]:
                a *= 0.5
        x = x + a * dx
    vm, va = state_to_voltages(prob, x)
    out = NewtonResult(x, vm, va, it, converged, res)
    if sensitivities and converged:
        lin.refactor(jacobian_values(prob, x))
        out.sensitivities = -lin.solve(control_jacobian(prob, x))
    return out


def _newton_device(prob, lin, tol, maxiter, x0, sensitivities, line_search) -> NewtonResult:
    """The loop of newton() with x, F, Gx, Gu and the step on the device (DeviceAssembly), the
    same steps and line search: only max |F| comes to the host per evaluation."""
    import torch

    asm = DeviceAssembly(prob, lin.A)
    dev = lin.A.nzVal.device
    x = torch.tensor(flat_start(prob) if x0 is None else np.asarray(x0, dtype=np.float64),
                     dtype=torch.float64, device=dev)
    if x.shape != (asm.n,):
        raise ValueError(f"x0 has {x.shape[0]} entries, the problem {asm.n} unknowns")
    xt, F, Ft, d = (torch.empty_like(x) for _ in range(4))
    nrm = asm.mismatch(x, F)
    res = []
    converged = False
    it = 0
    for it in range(maxiter + 1):
        res.append(nrm)
        if nrm <= tol:
            converged = True
            break
        if it == maxiter:
            break
        asm.jacobian(x)
        lin.refactor_device()
        d = lin.solve_device(F, d)            # Gx^{-1} F; the Newton step is -d
        a = 1.0
        while True:
            nt = asm.mismatch(x, Ft, dx=d, alpha=-a, x_out=xt)
            if not (line_search and a > 2.0 ** -12 and nt >= nrm):
                break
            a *= 0.5
        x, xt = xt, x
        F, Ft = Ft, F
        nrm = nt
    xh = x.cpu().numpy()
    vm, va = state_to_voltages(prob, xh)
    out = NewtonResult(xh, vm, va, it, converged, res)
    if sensitivities and converged:
        Gu = torch.empty((asm.n_ctrl, asm.n), dtype=torch.float64, device=dev).t()   # column-major
        asm.jacobian(x, Gu)
        lin.refactor_device()
        S = lin.solve_device(Gu).cpu().numpy()
        np.negative(S, out=S)                 # in place: one n x n_ctrl host block, not two
        out.sensitivities = S
    return out
