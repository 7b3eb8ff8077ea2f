"""Seeded synthetic Newton power-flow Jacobians (the inputs of the multi-RHS solve path).

The reference solves ``Gx * X = Gu``, where ``Gx`` is the Newton power-flow Jacobian that
ExaPF builds for a transmission grid (``benchmarks/benchmarks_nvidia.jl:29-39``,
``data/case300.txt``).  ExaPF and the large grid dumps are not available here, so this module
builds grids of the same shape and value distributions:

* topology: buses placed uniformly in the unit square, a Euclidean minimum spanning tree over
  the 8-nearest-neighbour graph, plus nearest-neighbour chords until the number of branches is
  ``branch_ratio * N`` (1.37 matches the 410 branches of a 300-bus case);
* branch values: series impedance ``r ~ U[0.005, 0.05]``, ``x ~ U[0.02, 0.2]``;
* operating point: ``|V| ~ U[0.95, 1.05]``, ``theta ~ N(0, 0.1)``, slack angle 0;
* Jacobian in polar form, rows ``[P(non-slack); Q(PQ)]`` and columns
  ``[theta(non-slack); |V|(PQ)]`` -- the same layout as ExaPF's ``Gx``.

Everything is seeded: the same ``(n_bus, seed)`` always gives the same CSR matrix.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import minimum_spanning_tree
from scipy.spatial import cKDTree

# (n_bus, n_pv) pairs that reproduce the unknown counts of the benchmark grids.
GRID_PRESETS = {
    "case300": (300, 68),        # 530 unknowns
    "case9k": (9000, 1000),      # 16,998 unknowns
    "case25k": (25000, 2000),    # ~48k unknowns
    "case70k": (70000, 5000),    # ~135k unknowns
}


@dataclasses.dataclass
class Grid:
    """A bus-branch network with one operating point."""
    n_bus: int
    f: np.ndarray          # branch from-bus
    t: np.ndarray          # branch to-bus
    r: np.ndarray
    x: np.ndarray
    pv: np.ndarray         # PV bus indices (sorted)
    pq: np.ndarray         # PQ bus indices (sorted)
    vm: np.ndarray         # |V|
    va: np.ndarray         # angle

    @property
    def n_unknowns(self) -> int:
        return (self.n_bus - 1) + len(self.pq)

    def ybus(self) -> sp.csr_matrix:
        y = 1.0 / (self.r + 1j * self.x)
        n = self.n_bus
        rows = np.concatenate([self.f, self.t, self.f, self.t])
        cols = np.concatenate([self.t, self.f, self.f, self.t])
        vals = np.concatenate([-y, -y, y, y])
        return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def make_grid(n_bus: int, n_pv: int | None = None, seed: int = 0,
              branch_ratio: float = 1.37) -> Grid:
    """Random meshed grid with ``n_bus`` buses (bus 0 is the slack)."""
    rng = np.random.default_rng(seed)
    if n_pv is None:
        n_pv = max(1, int(round(0.1 * n_bus)))
    pts = rng.random((n_bus, 2))
    k = min(9, n_bus)
    tree = cKDTree(pts)
    dist, nbr = tree.query(pts, k=k)
    rows = np.repeat(np.arange(n_bus), k - 1)
    cols = nbr[:, 1:].ravel()
    w = dist[:, 1:].ravel() + 1e-12
    knn = sp.coo_matrix((w, (rows, cols)), shape=(n_bus, n_bus)).tocsr()
    knn = knn.maximum(knn.T)
    mst = minimum_spanning_tree(knn).tocoo()
    edges = set()
    for a, b in zip(mst.row.tolist(), mst.col.tolist()):
        edges.add((min(a, b), max(a, b)))
    # Connect any leftover components (kNN graph is almost always connected).
    from scipy.sparse.csgraph import connected_components
    adj = sp.coo_matrix((np.ones(len(edges)), tuple(np.array(list(edges)).T)),
                        shape=(n_bus, n_bus))
    ncomp, lab = connected_components(adj, directed=False)
    if ncomp > 1:
        reps = [np.flatnonzero(lab == c)[0] for c in range(ncomp)]
        for a, b in zip(reps[:-1], reps[1:]):
            edges.add((min(a, b), max(a, b)))
    # Chords: nearest-neighbour pairs not yet used, in random order.
    target = int(round(branch_ratio * n_bus))
    cand = np.stack([np.minimum(rows, cols), np.maximum(rows, cols)], axis=1)
    cand = np.unique(cand, axis=0)
    cand = cand[rng.permutation(len(cand))]
    for a, b in cand.tolist():
        if len(edges) >= target:
            break
        if a != b and (a, b) not in edges:
            edges.add((a, b))
    e = np.array(sorted(edges), dtype=np.int64)
    f, t = e[:, 0], e[:, 1]
    nbr_ = len(e)
    r = rng.uniform(0.005, 0.05, nbr_)
    x = rng.uniform(0.02, 0.2, nbr_)
    pv = np.sort(rng.choice(np.arange(1, n_bus), size=n_pv, replace=False))
    is_pv = np.zeros(n_bus, dtype=bool)
    is_pv[pv] = True
    is_pv[0] = True
    pq = np.flatnonzero(~is_pv)
    vm = rng.uniform(0.95, 1.05, n_bus)
    va = rng.normal(0.0, 0.1, n_bus)
    va[0] = 0.0
    return Grid(n_bus, f, t, r, x, pv, pq, vm, va)


def jacobian(grid: Grid, vm: np.ndarray | None = None, va: np.ndarray | None = None) -> sp.csr_matrix:
    """Polar-form Newton Jacobian ``[dP/dth dP/dV; dQ/dth dQ/dV]`` (sorted CSR, float64).

    Uses the standard complex derivatives of S = V conj(Ybus V):
    dS/dth = j diag(V) conj(diag(I) - Ybus diag(V)),
    dS/dVm = diag(V) conj(Ybus diag(V/|V|)) + conj(diag(I)) diag(V/|V|).
    """
    vm = grid.vm if vm is None else vm
    va = grid.va if va is None else va
    Y = grid.ybus()
    V = vm * np.exp(1j * va)
    I = Y @ V
    dV = sp.diags(V)
    dI = sp.diags(I)
    dVn = sp.diags(V / np.abs(V))
    dS_dth = 1j * dV @ (dI - Y @ dV).conj()
    dS_dvm = dV @ (Y @ dVn).conj() + dI.conj() @ dVn
    dS_dth = dS_dth.tocsr()
    dS_dvm = dS_dvm.tocsr()
    nonslack = np.arange(1, grid.n_bus)
    pq = grid.pq
    j11 = dS_dth[nonslack][:, nonslack].real
    j12 = dS_dvm[nonslack][:, pq].real
    j21 = dS_dth[pq][:, nonslack].imag
    j22 = dS_dvm[pq][:, pq].imag
    J = sp.bmat([[j11, j12], [j21, j22]], format="csr")
    J.sum_duplicates()
    J.sort_indices()
    J.eliminate_zeros()
    return J.astype(np.float64)


def synthetic_jacobian(n_bus: int, n_pv: int | None = None, seed: int = 0) -> sp.csr_matrix:
    return jacobian(make_grid(n_bus, n_pv, seed))


def preset_jacobian(name: str, seed: int = 0) -> sp.csr_matrix:
    n_bus, n_pv = GRID_PRESETS[name]
    return synthetic_jacobian(n_bus, n_pv, seed)


def gaussian_rhs(n: int, p: int, seed: int) -> np.ndarray:
    """i.i.d. N(0,1) right-hand sides, column-major ``(n, p)`` float64."""
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((n, p)))


def perturbed_values(grid: Grid, pattern: sp.csr_matrix, step: int, sigma: float = 0.01,
                     seed: int = 0) -> np.ndarray:
    """CSR values of the Jacobian at a perturbed operating point on the fixed ``pattern``.

    Step ``t`` perturbs ``|V|`` and ``theta`` by ``N(0, sigma)``; the sparsity never changes
    (entries that happen to cancel keep an explicit zero).
    """
    rng = np.random.default_rng(seed * 100003 + step)
    vm = grid.vm + rng.normal(0.0, sigma, grid.n_bus)
    va = grid.va + rng.normal(0.0, sigma, grid.n_bus)
    va[0] = 0.0
    J = jacobian_on_pattern(grid, pattern, vm, va)
    return J


def jacobian_on_pattern(grid: Grid, pattern: sp.csr_matrix, vm, va) -> np.ndarray:
    vm = np.asarray(vm)
    va = np.asarray(va)
    Jt = grid_copy = jacobian(grid, vm, va)
    del grid_copy
    # Scatter Jt's values onto pattern's index set (Jt's pattern is a subset of pattern's,
    # up to exact cancellations that eliminate_zeros dropped).
    out = np.zeros(pattern.nnz)
    n = pattern.shape[0]
    pr, pc = pattern.indptr, pattern.indices
    key_p = np.repeat(np.arange(n, dtype=np.int64), np.diff(pr)) * n + pc
    key_t = np.repeat(np.arange(n, dtype=np.int64), np.diff(Jt.indptr)) * n + Jt.indices
    pos = np.searchsorted(key_p, key_t)
    if np.any(pos >= len(key_p)) or np.any(key_p[np.minimum(pos, len(key_p) - 1)] != key_t):
        raise ValueError("perturbed Jacobian left the fixed sparsity pattern")
    out[pos] = Jt.data
    return out


# ---- the batched benchmark configuration: many independent grids of uneven size ----------
def batch_sizes(nsys: int = 512, seed: int = 0):
    """Bus counts (log-uniform in [100, 3000]) and right-hand-side counts (uniform in 8..64)
    of a batch of ``nsys`` independent grids."""
    rng = np.random.default_rng(seed)
    buses = np.exp(rng.uniform(np.log(100), np.log(3000), nsys)).astype(int)
    nrhs = rng.integers(8, 65, nsys)
    return [int(b) for b in buses], [int(p) for p in nrhs]


def batch_system(k: int, buses, nrhs):
    """System ``k`` of a batch: its Jacobian (sorted CSR) and Gaussian right-hand sides."""
    A = jacobian(make_grid(buses[k], seed=1000 + k)).tocsr()
    B = gaussian_rhs(A.shape[0], nrhs[k], 5000 + k)
    return A, B


def batch_workload(nsys: int = 512, seed: int = 0, systems=None):
    """(buses, nrhs, matrices, right-hand sides) of a batch, for all systems or the listed ones
    (``buses`` and ``nrhs`` always cover the whole batch)."""
    buses, nrhs = batch_sizes(nsys, seed)
    idx = range(nsys) if systems is None else systems
    mats, Bs = [], []
    for k in idx:
        A, B = batch_system(k, buses, nrhs)
        mats.append(A)
        Bs.append(B)
    return buses, nrhs, mats, Bs
