"""ctypes bindings of the CPU oracle (``oracle/bpf_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py``, always as the checker or the timed CPU reference, never
as a fallback of the product path.  Every function follows a reference location that is cited
in ``bpf_oracle.c``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import scipy.sparse as sp

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

STATUS_STRINGS = {
    0: "unknown",
    1: "solution good enough given atol and rtol",
    2: "maximum number of iterations exceeded",
    3: "time limit exceeded",
}


class _Opts(C.Structure):
    _fields_ = [("memory", C.c_int), ("restart", C.c_int), ("reorthogonalization", C.c_int),
                ("atol", C.c_double), ("rtol", C.c_double), ("itmax", C.c_int),
                ("timemax", C.c_double), ("history", C.c_int)]


class _Stats(C.Structure):
    _fields_ = [("niter", C.c_int), ("solved", C.c_int), ("status", C.c_int),
                ("timer", C.c_double), ("n_residuals", C.c_int), ("residuals_cap", C.c_int),
                ("residuals", C.POINTER(C.c_double)), ("npass", C.c_int)]


def build() -> str:
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "bpf_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return path


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(build())
    return _LIB


def set_threads(t: int) -> None:
    lib().orc_set_threads(int(t))


def set_fast_dense(on: bool) -> None:
    """Cache-blocked dense products (the same sums in another order), for timing the oracle as
    the CPU baseline; the checker's default is the plain loops."""
    lib().orc_set_fast_dense(int(bool(on)))


def _ptr(a, ctype=C.c_double):
    return a.ctypes.data_as(C.POINTER(ctype))


def _csr(A: sp.csr_matrix):
    A = sp.csr_matrix(A)
    A.sort_indices()
    rp = np.ascontiguousarray(A.indptr, dtype=np.int32)
    ci = np.ascontiguousarray(A.indices, dtype=np.int32)
    v = np.ascontiguousarray(A.data, dtype=np.float64)
    return A.shape[0], rp, ci, v


def spmm(A, X, alpha=1.0, beta=0.0, Y=None):
    n, rp, ci, v = _csr(A)
    X = np.asfortranarray(X, dtype=np.float64)
    p = X.shape[1]
    Y = np.zeros((n, p), order="F") if Y is None else np.asfortranarray(Y, dtype=np.float64).copy(order="F")
    lib().orc_spmm(n, _ptr(rp, C.c_int), _ptr(ci, C.c_int), _ptr(v), p, C.c_double(alpha),
                   _ptr(X), n, C.c_double(beta), _ptr(Y), n)
    return Y


def ilu0(A) -> sp.csr_matrix:
    """Combined unit-L / U factors on A's pattern (csrilu02 semantics)."""
    n, rp, ci, v = _csr(A)
    v = v.copy()
    st = lib().orc_ilu0(n, _ptr(rp, C.c_int), _ptr(ci, C.c_int), _ptr(v))
    if st != 0:
        raise ZeroDivisionError(f"ILU0 zero pivot at row {-st - 1}")
    return sp.csr_matrix((v, ci, rp), shape=(n, n))


def ic0(A) -> sp.csr_matrix:
    n, rp, ci, v = _csr(A)
    v = v.copy()
    st = lib().orc_ic0(n, _ptr(rp, C.c_int), _ptr(ci, C.c_int), _ptr(v))
    if st != 0:
        raise ZeroDivisionError(f"IC0 non-positive pivot at row {-st - 1}")
    return sp.csr_matrix((v, ci, rp), shape=(n, n))


def trsm(kind: int, F, X):
    n, rp, ci, v = _csr(F)
    X = np.asfortranarray(X, dtype=np.float64)
    p = X.shape[1]
    Y = np.zeros((n, p), order="F")
    lib().orc_trsm(kind, n, _ptr(rp, C.c_int), _ptr(ci, C.c_int), _ptr(v), p, _ptr(X), n,
                   _ptr(Y), n)
    return Y


def prec_apply(kind: int, F, X):
    """kind 1: ILU0 ldiv!, kind 2: IC0 ldiv!, 0: identity."""
    n, rp, ci, v = _csr(F)
    X = np.asfortranarray(X, dtype=np.float64)
    p = X.shape[1]
    Y = np.zeros((n, p), order="F")
    lib().orc_prec_apply(kind, n, _ptr(rp, C.c_int), _ptr(ci, C.c_int), _ptr(v), p, _ptr(X),
                         n, _ptr(Y), n)
    return Y


def householder(Q, compact=False):
    Q = np.asfortranarray(Q, dtype=np.float64).copy(order="F")
    m, k = Q.shape
    R = np.zeros((k, k), order="F")
    tau = np.zeros(k)
    lib().orc_householder(m, k, _ptr(Q), m, _ptr(R), k, _ptr(tau), int(compact))
    return Q, R, tau


class OracleStats:
    def __init__(self, st: _Stats, res: np.ndarray):
        self.niter = st.niter
        self.solved = bool(st.solved)
        self.status = STATUS_STRINGS[st.status]
        self.status_code = st.status
        self.timer = st.timer
        self.npass = st.npass
        self.residuals = res[: min(st.n_residuals, len(res))].copy()

    def __repr__(self):
        return (f"OracleStats(niter={self.niter}, solved={self.solved}, status={self.status!r}, "
                f"timer={self.timer:.3g})")


def _prec_args(P):
    """P is None (identity) or a tuple (kind, factor_csr)."""
    if P is None:
        z = np.zeros(1, dtype=np.int32)
        return (0, _ptr(z, C.c_int), _ptr(z, C.c_int), _ptr(np.zeros(1))), (z,)
    kind, F = P
    n, rp, ci, v = _csr(F)
    return (kind, _ptr(rp, C.c_int), _ptr(ci, C.c_int), _ptr(v)), (rp, ci, v)


def block_gmres(A, B, X0=None, *, memory=20, M=None, N=None, restart=False,
                reorthogonalization=False, atol=None, rtol=None, itmax=0,
                timemax=float("inf"), history=False):
    """Oracle block-GMRES; M/N are ``None`` or ``(kind, factors)`` with ldiv semantics."""
    eps = np.finfo(np.float64).eps
    atol = np.sqrt(eps) if atol is None else atol
    rtol = np.sqrt(eps) if rtol is None else rtol
    n, rp, ci, v = _csr(A)
    B = np.asfortranarray(B, dtype=np.float64)
    p = B.shape[1]
    X = np.zeros((n, p), order="F")
    margs, mkeep = _prec_args(M)
    nargs, nkeep = _prec_args(N)
    x0p = None
    if X0 is not None:
        X0 = np.asfortranarray(X0, dtype=np.float64)
        x0p = _ptr(X0)
    o = _Opts(memory, int(restart), int(reorthogonalization), atol, rtol, itmax, timemax,
              int(history))
    cap = (itmax if itmax else 2 * (n // p)) + 2
    res = np.zeros(cap)
    st = _Stats(0, 0, 0, 0.0, 0, cap, _ptr(res), 0)
    rc = lib().orc_block_gmres(n, _ptr(rp, C.c_int), _ptr(ci, C.c_int), _ptr(v), p, _ptr(B), n,
                               _ptr(X), n, x0p, n, *margs, *nargs, C.byref(o), C.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle block_gmres failed: {rc}")
    return X, OracleStats(st, res)


def block_bicgstab(A, B, *, C_shadow=None, N=None, atol=None, rtol=None, itmax=0,
                   timemax=float("inf"), history=False):
    eps = np.finfo(np.float64).eps
    atol = np.sqrt(eps) if atol is None else atol
    rtol = np.sqrt(eps) if rtol is None else rtol
    n, rp, ci, v = _csr(A)
    B = np.asfortranarray(B, dtype=np.float64)
    p = B.shape[1]
    X = np.zeros((n, p), order="F")
    nargs, nkeep = _prec_args(N)
    cp = None
    if C_shadow is not None:
        C_shadow = np.asfortranarray(C_shadow, dtype=np.float64)
        cp = _ptr(C_shadow)
    o = _Opts(0, 0, 0, atol, rtol, itmax, timemax, int(history))
    cap = (itmax if itmax else 2 * n) + 2
    res = np.zeros(cap)
    st = _Stats(0, 0, 0, 0.0, 0, cap, _ptr(res), 0)
    rc = lib().orc_block_bicgstab(n, _ptr(rp, C.c_int), _ptr(ci, C.c_int), _ptr(v), p, _ptr(B),
                                  n, _ptr(X), n, cp, n, *nargs, C.byref(o), C.byref(st))
    if rc == 5:
        raise np.linalg.LinAlgError("block_bicgstab: singular K")
    if rc != 0:
        raise RuntimeError(f"oracle block_bicgstab failed: {rc}")
    return X, OracleStats(st, res)


class DenseLU:
    """RF oracle: pivoted LU once, refactor on the same pivots, multi-RHS solve."""

    def __init__(self, A, tol=1e-8):
        self.n = A.shape[0]
        self.perm = np.zeros(self.n, dtype=np.int32)
        Ad = np.asfortranarray(sp.csr_matrix(A).toarray())
        st = lib().orc_lu_factor(self.n, _ptr(Ad), _ptr(self.perm, C.c_int), C.c_double(tol))
        if st != 0:
            raise np.linalg.LinAlgError(f"singular at column {-st - 1}")
        self.LU = Ad

    def refactor(self, A):
        Ad = np.asfortranarray(sp.csr_matrix(A).toarray()[self.perm, :])
        st = lib().orc_lu_refactor(self.n, _ptr(Ad), _ptr(self.perm, C.c_int))
        if st != 0:
            raise np.linalg.LinAlgError(f"zero pivot at column {-st - 1}")
        self.LU = Ad

    def solve(self, B):
        X = np.asfortranarray(B, dtype=np.float64).copy(order="F")
        if X.ndim == 1:
            X = X.reshape(-1, 1, order="F")
        lib().orc_lu_solve(self.n, _ptr(self.LU), _ptr(self.perm, C.c_int), X.shape[1], _ptr(X),
                           self.n)
        return X


def block_jacobi_apply(A, order, block_size, X):
    """Block-Jacobi y = P x with P = diag(A_b^{-1}), the blocks A_b = A(rows_b, rows_b) over
    consecutive runs of block_size rows of `order`: the algorithm of ExaPF 0.9.3's
    LinearSolvers.BlockJacobiPreconditioner (dense inverse of every diagonal block, applied by
    mul!), which the reference's tests and benchmark build (test/block_gmres.jl:5,17,22,
    benchmarks/benchmarks_nvidia.jl:47-51).  ExaPF's METIS partition is replaced by the given
    order, as in the library.  Dense LAPACK solves of the small blocks (numpy)."""
    A = sp.csr_matrix(A)
    X = np.asarray(X, dtype=np.float64)
    Y = np.zeros_like(X)
    order = np.asarray(order)
    for b0 in range(0, len(order), block_size):
        rows = order[b0:b0 + block_size]
        Ab = A[rows][:, rows].toarray()
        Y[rows] = np.linalg.solve(Ab, X[rows])
    return Y


def pf_assemble(ybus_rowptr, ybus_colind, ybus_vals, bus_type, vm_fixed, va_fixed, s_spec, x, pattern):
    """Power-flow mismatch F, Jacobian Gx on `pattern` and control Jacobian Gu at the state x,
    restated entry by entry from the host arguments of bpf_pf_create (the Newton loop around the
    reference's solve path; ExaPF, which assembled the reference benchmark's Gx / Gu dumps
    (benchmarks/benchmarks_nvidia.jl:29-39), is not part of the reference).

    Polar form with S = V conj(I), I = Ybus V:
      dS_i/dtheta_k = j V_i ([i == k] conj(I_i) - conj(Y_ik V_k)),
      dS_i/d|V_k|   = V_i conj(Y_ik V_k / |V_k|) + [i == k] conj(I_i) V_i / |V_i|.
    Unknowns: theta at every non-slack bus (bus order), then |V| at the PQ buses (bus order);
    equations P, Q in the same order; controls: |V| of the slack bus, then of the PV buses.
    Returns (F, Gx values in pattern's CSR order, Gu dense n x n_ctrl); raises ValueError if an
    entry the coupling produces is missing from the pattern."""
    rp = np.asarray(ybus_rowptr)
    ci = np.asarray(ybus_colind)
    yv = np.asarray(ybus_vals, dtype=np.float64)
    bt = np.asarray(bus_type)
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
    n = (nb - 1) + len(pq)
    x = np.asarray(x, dtype=np.float64)
    va = np.where(ia >= 0, x[np.maximum(ia, 0)], va_fixed)
    vm = np.where(im >= 0, x[np.maximum(im, 0)], vm_fixed)
    V = vm * np.exp(1j * va)
    y = yv[0::2] + 1j * yv[1::2]
    rows = np.repeat(np.arange(nb), np.diff(rp))
    # the I_i terms attach at the diagonal entry: every nonempty row must hold it (the library
    # inserts a missing one; this restatement does not)
    has_diag = np.zeros(nb, dtype=bool)
    has_diag[rows[rows == ci]] = True
    if np.any(~has_diag & (np.diff(rp) > 0)):
        raise ValueError("a nonempty Ybus row lacks its diagonal entry")
    t = y * V[ci]
    I = np.bincount(rows, t.real, nb) + 1j * np.bincount(rows, t.imag, nb)
    S = V * np.conj(I) - (np.asarray(s_spec)[0::2] + 1j * np.asarray(s_spec)[1::2])
    F = np.zeros(n)
    F[ia[ia >= 0]] = S.real[ia >= 0]
    F[im[im >= 0]] = S.imag[im >= 0]
    i, k = rows, ci
    diag = i == k
    dth = 1j * V[i] * (np.where(diag, np.conj(I[i]), 0) - np.conj(y * V[k]))
    dm = V[i] * np.conj(y * V[k] / np.abs(V[k])) + np.where(diag, np.conj(I[i]) * V[i] / np.abs(V[i]), 0)
    P = sp.csr_matrix(pattern)
    if not P.has_sorted_indices:   # CSR order of the values, as the library requires it
        raise ValueError("pattern columns must be sorted within each row")
    gx = np.zeros(P.nnz)
    for rr, cc, vv in ((ia[i], ia[k], dth.real), (ia[i], im[k], dm.real),
                       (im[i], ia[k], dth.imag), (im[i], im[k], dm.imag)):
        for r_, c_, v_ in zip(rr, cc, vv):
            if r_ < 0 or c_ < 0:
                continue
            lo, hi = P.indptr[r_], P.indptr[r_ + 1]
            pos = lo + np.searchsorted(P.indices[lo:hi], c_)
            if pos >= hi or P.indices[pos] != c_:
                if v_ == 0.0:
                    continue
                raise ValueError(f"pattern lacks entry ({r_}, {c_})")
            gx[pos] = v_
    Gu = np.zeros((n, len(ctrl_buses)))
    sel = ctrl[k] >= 0
    for rr, vv in ((ia[i], dm.real), (im[i], dm.imag)):
        s2 = sel & (rr >= 0)
        Gu[rr[s2], ctrl[k][s2]] = vv[s2]
    return F, gx, Gu
