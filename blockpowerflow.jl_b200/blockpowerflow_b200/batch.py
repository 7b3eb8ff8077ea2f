"""Batched block-GMRES: many independent systems in one CUDA-graph launch (bpf_batch_*).

No counterpart in the reference, whose solvers take one system per call; each system is solved
as block_gmres(A, B; N=ilu0(A), ldiv=true) would (src/block_gmres.jl:127-168), column slices of
at most 32 right-hand sides per work unit, all units of all systems in one persistent kernel.

The autotuner (``autotune``) times the plan's launch shapes (widest column slice, resident CTAs
per SM) and fill-reducing orders (minimum degree, reverse Cuthill-McKee) on the caller's own
systems and keeps the fastest in a JSON cache keyed by the batch's shape and the device name.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import hashlib
import json
import os
import time

import numpy as np

from . import _lib
from .sparse import CuSparseMatrixCSR, colmajor, empty_colmajor, ld

_DTYPES = {"float64": _lib.BPF_F64, "float32": _lib.BPF_F32}


@dataclasses.dataclass
class BatchStats:
    """Per-system outcome of a batched solve (the fields of BlockGMRESStats that apply)."""
    niter: int
    solved: bool
    status: str
    npass: int


def _ordering_code(ordering) -> int:
    key = ordering.lstrip(":").upper() if isinstance(ordering, str) else ordering
    if key not in _lib.ORDERINGS:
        raise ValueError(f"unknown ordering {ordering!r}")
    return _lib.ORDERINGS[key]


class BatchPlan:
    """Analysis of a batch of systems and its captured solve graph.

    mats: CuSparseMatrixCSR per system (their value arrays are re-read by every solve, so new
    values on the same patterns go in place); nrhs: right-hand-side columns per system; slices:
    optional widest column slice per system (0: `slice`), see ``split_longest``.
    """

    PHASES = ("prec", "spmm", "gram", "update", "cholqr", "hess", "backsub", "total")

    def __init__(self, mats: list[CuSparseMatrixCSR], nrhs, *, atol: float = 0.0,
                 rtol: float = 1e-8, itmax: int = 0, memory: int = 0,
                 factor_dtype: str = "float32", ordering="AMD", slice: int = 0,
                 ctas_per_sm: int = 0, slices=None):
        if len(mats) == 0:
            raise ValueError("empty batch")
        nrhs = [int(v) for v in nrhs]
        if len(nrhs) != len(mats):
            raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "one nrhs per system expected")
        if factor_dtype not in _DTYPES:
            raise ValueError(f"factor_dtype must be one of {sorted(_DTYPES)}")
        self.handle = None
        self.mats = list(mats)
        self.nrhs = nrhs
        self.n = [A.n for A in mats]
        self.nsys = len(mats)
        self.device = mats[0].rowPtr.device
        self.opts = _lib.BatchOpts(float(atol), float(rtol), int(itmax), int(memory),
                                   _DTYPES[factor_dtype], _ordering_code(ordering), int(slice),
                                   int(ctas_per_sm))
        lib = _lib.load()
        self._ctx = _lib.context(self.device.index)
        descs = (_lib.CsrDesc * self.nsys)(*[A.desc() for A in mats])
        p_arr = (C.c_int * self.nsys)(*nrhs)
        h = C.c_void_p()
        if slices is None:
            self.slices = None
            _lib.check(lib.bpf_batch_plan(self._ctx, self.nsys, descs, p_arr, C.byref(self.opts),
                                          C.byref(h)), self._ctx)
        else:
            self.slices = [int(v) for v in slices]
            if len(self.slices) != self.nsys:
                raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "one slice width per system expected")
            q_arr = (C.c_int * self.nsys)(*self.slices)
            _lib.check(lib.bpf_batch_plan_sliced(self._ctx, self.nsys, descs, p_arr, q_arr,
                                                 C.byref(self.opts), C.byref(h)), self._ctx)
        self.handle = h
        nu, grid, nbytes = C.c_int(), C.c_int(), C.c_longlong()
        lib.bpf_batch_info(h, C.byref(nu), C.byref(grid), C.byref(nbytes))
        self.nunits, self.grid, self.device_bytes = nu.value, grid.value, nbytes.value

    def solve(self, Bs, Xs=None):
        """Xs[s] = A[s] \\ Bs[s] for every system; returns (Xs, [BatchStats])."""
        if len(Bs) != self.nsys:
            raise _lib.DimensionMismatch(_lib.BPF_ERR_DIMENSION, "one right-hand side per system expected")
        Bc = []
        for s, B in enumerate(Bs):
            b = colmajor(B, self.device)
            if tuple(b.shape) != (self.n[s], self.nrhs[s]):
                raise _lib.DimensionMismatch(
                    _lib.BPF_ERR_DIMENSION,
                    f"B[{s}] should have size ({self.n[s]}, {self.nrhs[s]})")
            Bc.append(b)
        if Xs is None:
            Xs = [empty_colmajor(self.n[s], self.nrhs[s], self.device) for s in range(self.nsys)]
        else:
            for s, X in enumerate(Xs):
                if tuple(X.shape) != (self.n[s], self.nrhs[s]) or X.stride(0) != 1:
                    raise _lib.DimensionMismatch(
                        _lib.BPF_ERR_DIMENSION, f"X[{s}] must be a column-major ({self.n[s]}, {self.nrhs[s]}) block")
        lib = _lib.load()
        self._ctx = _lib.context(self.device.index)
        PtrArr = C.c_void_p * self.nsys
        IntArr = C.c_int * self.nsys
        bp = PtrArr(*[b.data_ptr() for b in Bc])
        xp = PtrArr(*[x.data_ptr() for x in Xs])
        lb = IntArr(*[ld(b) for b in Bc])
        lx = IntArr(*[ld(x) for x in Xs])
        st = (_lib.Stats * self.nsys)()
        _lib.check(lib.bpf_batch_solve(self.handle, bp, lb, xp, lx, st), self._ctx)
        stats = [BatchStats(int(v.niter), bool(v.solved),
                            lib.bpf_solve_status_string(v.status).decode(), int(v.npass)) for v in st]
        return Xs, stats

    def unit_stats(self) -> dict:
        """Per work unit of the last solve: system, first column, width, basis blocks,
        iterations, status code and the initial / final least-squares residual norms."""
        lib = _lib.load()
        nu = self.nunits
        out = {k: np.zeros(nu, dtype=np.int32) for k in ("sys", "col0", "q", "memory", "niter", "status")}
        out["rnorm0"] = np.zeros(nu)
        out["rnorm"] = np.zeros(nu)

        def ptr(a):
            return a.ctypes.data_as(C.c_void_p)

        _lib.check(lib.bpf_batch_unit_stats(self.handle, ptr(out["sys"]), ptr(out["col0"]), ptr(out["q"]),
                                            ptr(out["memory"]), ptr(out["niter"]), ptr(out["status"]),
                                            ptr(out["rnorm0"]), ptr(out["rnorm"])), self._ctx)
        return out

    def unit_cycles(self) -> dict:
        """SM cycles of each unit of the last solve by phase (PHASES), from the kernel's own
        clock64 counters."""
        cyc = np.zeros((self.nunits, len(self.PHASES)), dtype=np.int64)
        _lib.check(_lib.load().bpf_batch_unit_cycles(self.handle, cyc.ctypes.data_as(C.c_void_p)), self._ctx)
        return {k: cyc[:, i] for i, k in enumerate(self.PHASES)}

    def close(self) -> None:
        if getattr(self, "handle", None):
            _lib.load().bpf_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- autotuner ------------------------------------------------------------------------------
# One resident solve CTA per SM: the persistent kernel is compiled for one CTA per SM (all 255
# registers a thread may hold, no spills), so ctas_per_sm = 2 runs as 1 and is not a candidate.
# The order of the ILU(0) factors changes the iteration counts as well as the triangular solves'
# level counts, in either direction depending on the grids, so both fill-reducing orders are
# timed.  A candidate is (slice, ctas_per_sm, ordering); a pair (slice, ctas_per_sm) takes the
# plan's own ordering.
CANDIDATES = [(slice_, 1, order) for order in ("AMD", "RCM") for slice_ in (8, 16, 32)]


def _candidate(c, default_ordering) -> tuple:
    order = c[2] if len(c) > 2 else default_ordering
    if not isinstance(order, str):
        order = {v: k for k, v in _lib.ORDERINGS.items()}[order]
    return int(c[0]), int(c[1]), order.lstrip(":").upper()


def batch_key(n, nrhs, device_name: str, extra: str = "") -> str:
    """Cache key of a batch: its systems' sizes and widths, the device and the options."""
    h = hashlib.sha1()
    h.update(np.asarray(n, dtype=np.int64).tobytes())
    h.update(np.asarray(nrhs, dtype=np.int64).tobytes())
    h.update(device_name.encode())
    h.update(extra.encode())
    return h.hexdigest()[:20]


def load_cache(path: str) -> dict:
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def store_cache(path: str, cache: dict) -> None:
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def pick_best(timings: dict) -> tuple:
    """The candidate with the smallest time among those whose solves all converged;
    timings maps a candidate (slice, ctas_per_sm[, ordering]) -> (seconds, all_solved)."""
    ok = [(t, c) for c, (t, solved) in timings.items() if solved]
    if not ok:
        ok = [(t, c) for c, (t, _) in timings.items()]
    return min(ok)[1]


def cache_extra(candidates, ordering="AMD", refine_rounds: int = 2, min_gain: float = 0.01, **plan_kw) -> str:
    """The part of an autotuner cache key that is not the batch's shape: the plan options, the
    candidates and the refinement settings (autotune's own arguments, defaults included)."""
    cands = [_candidate(c, ordering) for c in candidates]
    extra = json.dumps({k: plan_kw[k] for k in sorted(plan_kw)}, default=str)
    return extra + json.dumps([cands, int(refine_rounds), float(min_gain)])


def split_longest(unit_sys, unit_q, unit_cycles, grid: int, slices, factor: float = 0.9):
    """Per-system widest slices for a refinement round of the plan: every system that has a unit
    longer than `factor` x the balanced bound (the units' total cycles over the resident CTAs)
    gets half its widest slice, rounded up.  The persistent solve cannot end before its longest
    unit, so narrower units of those systems shorten the critical path.  slices: the current
    per-system widths (0: the plan's slice).  Returns the new list, or None when no system
    qualifies."""
    cyc = np.asarray(unit_cycles, dtype=np.float64)
    bal = cyc.sum() / max(int(grid), 1)
    widest = {}
    for sy, q in zip(unit_sys, unit_q):
        widest[int(sy)] = max(widest.get(int(sy), 0), int(q))
    new = [int(v) for v in slices]
    changed = False
    for u in np.argsort(-cyc, kind="stable"):
        if cyc[u] < factor * bal:
            break
        sy = int(unit_sys[u])
        w = (widest[sy] + 1) // 2
        if widest[sy] > 1 and (new[sy] == 0 or new[sy] > w):
            new[sy] = w
            changed = True
    return new if changed else None


def autotune(mats, nrhs, Bs, *, cache_path: str | None = None, candidates=CANDIDATES,
             repeats: int = 2, runner=None, device_name: str | None = None, refine_rounds: int = 2,
             min_gain: float = 0.01, split_factor: float = 0.9, **plan_kw) -> dict:
    """Pick (slice, ctas_per_sm, ordering) for this batch: time each candidate plan's solve of Bs
    (best of `repeats`, after one warm-up) and keep the fastest whose systems all converged.
    Then up to `refine_rounds` rounds of ``split_longest`` on the chosen plan's measured unit
    cycles, each kept only if its solve is at least `min_gain` faster and still converges.
    With cache_path, a cached choice for the same key is returned without timing, and a new one
    is written.  runner(slice, ctas_per_sm, ordering, slices=None) -> (seconds, all_solved[,
    units]) replaces the GPU timing (tests of the selection and cache logic); units = {"sys",
    "q", "cycles", "grid"} of the timed plan, without which no refinement runs.  The result's
    keys are the BatchPlan arguments slice, ctas_per_sm, ordering and slices (None: the plan's
    slice everywhere), plus cached, timings and refinement."""
    if device_name is None:
        import torch
        device_name = torch.cuda.get_device_name(mats[0].rowPtr.device)
    default_ordering = plan_kw.pop("ordering", "AMD")
    cands = [_candidate(c, default_ordering) for c in candidates]
    extra = cache_extra(candidates, default_ordering, refine_rounds, min_gain, **plan_kw)
    if split_factor != 0.9:
        extra += json.dumps(float(split_factor))
    key = batch_key([A.n for A in mats], nrhs, device_name, extra)
    cache = load_cache(cache_path) if cache_path else {}
    if key in cache:
        c = cache[key]
        return {"slice": int(c["slice"]), "ctas_per_sm": int(c["ctas_per_sm"]),
                "ordering": str(c.get("ordering", default_ordering)), "slices": c.get("slices"),
                "cached": True, "timings": c.get("timings", {}), "refinement": c.get("refinement", [])}

    def gpu_runner(slice_, cps, ordering, slices=None):
        import torch
        plan = BatchPlan(mats, nrhs, slice=slice_, ctas_per_sm=cps, ordering=ordering, slices=slices,
                         **plan_kw)
        try:
            plan.solve(Bs)
            best = float("inf")
            solved = True
            for _ in range(max(1, repeats)):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                _, st = plan.solve(Bs)
                torch.cuda.synchronize()
                best = min(best, time.perf_counter() - t0)
                solved = solved and all(s.solved for s in st)
            u = plan.unit_stats()
            units = {"sys": u["sys"], "q": u["q"], "cycles": plan.unit_cycles()["total"], "grid": plan.grid}
            return best, solved, units
        finally:
            plan.close()

    run = runner or gpu_runner
    timings, units = {}, {}
    for c in cands:
        r = run(*c)
        timings[c] = (r[0], r[1])
        units[c] = r[2] if len(r) > 2 else None
    best = pick_best(timings)
    slices, t_best, info = None, timings[best][0], units[best]
    refinement = []
    cur = [0] * len(mats)
    for _ in range(max(0, int(refine_rounds))):
        if info is None:
            break
        new = split_longest(info["sys"], info["q"], info["cycles"], info["grid"], cur, split_factor)
        if new is None:
            break
        r = run(*best, new)
        ok = bool(r[1]) and r[0] < t_best * (1.0 - min_gain)
        refinement.append({"split_systems": int(sum(a != b for a, b in zip(new, cur))), "seconds": float(r[0]),
                           "solved": bool(r[1]), "kept": ok})
        if not ok:
            break
        cur, slices, t_best = new, new, r[0]
        info = r[2] if len(r) > 2 else None
    result = {"slice": best[0], "ctas_per_sm": best[1], "ordering": best[2], "slices": slices, "cached": False,
              "timings": {f"{c[0]}x{c[1]}x{c[2]}": [float(t), bool(ok)] for c, (t, ok) in timings.items()},
              "refinement": refinement}
    if cache_path:
        cache[key] = {k: result[k] for k in ("slice", "ctas_per_sm", "ordering", "slices", "timings", "refinement")}
        store_cache(cache_path, cache)
    return result
