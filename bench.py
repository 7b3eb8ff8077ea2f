#!/usr/bin/env python
"""RHS solves/s at a 1e-8 relative residual on one B200 (one JSON line on stdout).

Workload (the 9,000-bus grid of the second benchmark configuration): a seeded synthetic
Newton power-flow Jacobian with 9,000 buses (16,998 unknowns, ~121k nonzeros) and 64 Gaussian
right-hand sides, solved by block-GMRES with a right ILU(0) preconditioner, no restart (as in
benchmarks_nvidia.jl), atol 0, rtol 1e-8.  One step = ILU(0) numeric refactorization of the
Jacobian's values + the block-GMRES solve; the sparsity analysis is done once at set-up, as a
Newton loop would.  RHS solves/s = converged right-hand sides / time.

  value : device-resident inputs, CUDA-event time of K steps (max over ranks), L2 flushed
          between steps (256 MB write).
  e2e   : the same step through the public Python API with pinned host buffers: Jacobian
          values and B copied host->device and X device->host inside the timed region.
  roofline : the kernel class with the largest share of device time, measured live with
          CUDA events around each of its launches inside the timed region.
  cpu_baseline : the C restatement of the reference's block-GMRES (oracle/) on the host's
          cores, first iterations of the same solve, scaled to the whole solve by operation
          count.

`--impl reference` times that CPU restatement alone (the reference is Julia, and neither Julia
nor its CUDA.jl stack is installed) on the same workload and prints the same metric with
"impl":"reference".
Multi-GPU (torchrun): every rank solves its own grid (seed offset by rank), no collective on
the data path; value = all ranks' converged RHS / max-over-ranks time ("scaling": "weak").
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "blockpowerflow.jl_b200"))

METRIC = "RHS solves/s at 1e-8 residual: mixed+learned vs plain FP64 block-GMRES, 1 B200"
UNIT = "RHS solves/s"
N_BUS, N_PV, P_RHS = 9000, 1000, 64
RTOL = 1e-8
ITMAX = 300
CPU_SAMPLE_ITERS = (4, 10)
CPU_FULL_MAX_S = 15.0   # the whole CPU solve is timed when predicted to take at most this long
# DRAM bytes (read + write) per working launch of the FP64 product classes in the benchmark's
# solve (minimum-degree ILU(0), 57 iterations), from one ncu capture of every launch
# (profiles/launches_grid9k_p64_amd_ilu0_gmres.md): the kernels' total DRAM bytes over the
# launches that always do their work, the ones bench.py's per-class timing counts.
TRAFFIC_PER_LAUNCH = {"gram": 135.58e6, "tsmm": 126.28e6}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def fp64_peak_tflops(device):
    """FP64 tensor-pipe reference: cuBLAS DGEMM (torch.matmul, float64, 8192^3), best of 5
    after 2 warm-up products, CUDA events.  The peaks file has no FP64 figure."""
    import torch

    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return

        def reader():
            for line in self.proc.stdout:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    self.samples.append(parts)

        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if s[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def make_workload(rank):
    from blockpowerflow_b200 import grid as g

    grid = g.make_grid(N_BUS, N_PV, seed=rank)
    J = g.jacobian(grid)
    B = g.gaussian_rhs(J.shape[0], P_RHS, seed=1000 + rank)
    return J, B


def cpu_baseline(J, B, gpu_iters, threads):
    """Oracle block-GMRES (C, OpenMP) on the host.  Two short runs give the cost per iteration
    (constant part + part growing with the basis); when the whole solve is predicted to take at
    most CPU_FULL_MAX_S it is run and timed to the tolerance, else the short runs are
    extrapolated to `gpu_iters` iterations."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    O.set_threads(threads)
    O.set_fast_dense(True)   # cache-blocked dense products while timing (the checker keeps the plain loops)
    try:
        return _cpu_baseline_timed(O, J, B, gpu_iters, threads)
    finally:
        O.set_fast_dense(False)


def _cpu_baseline_timed(O, J, B, gpu_iters, threads):
    import numpy as np

    t0 = time.time()
    F = O.ilu0(J)
    t_factor = time.time() - t0
    times = []
    for it in CPU_SAMPLE_ITERS:
        t0 = time.time()
        O.block_gmres(J, B, N=(1, F), memory=it, restart=False, atol=0.0, rtol=RTOL, itmax=it)
        times.append(time.time() - t0)
    (k1, k2), (t1, t2) = CPU_SAMPLE_ITERS, times
    # T(k) = a k + b k (k + 1) / 2  (SpMM / ILU0 / QR per iteration + Gram-Schmidt over k blocks)
    A_ = np.array([[k1, k1 * (k1 + 1) / 2], [k2, k2 * (k2 + 1) / 2]])
    a, b = np.linalg.solve(A_, np.array([t1, t2]))
    a, b = max(a, 0.0), max(b, 0.0)
    K = gpu_iters
    t_full = t_factor + a * K + b * K * (K + 1) / 2
    if t_full <= CPU_FULL_MAX_S:
        t0 = time.time()
        X, st = O.block_gmres(J, B, N=(1, F), memory=ITMAX, restart=False, atol=0.0, rtol=RTOL, itmax=ITMAX)
        t_run = time.time() - t0
        if st.solved:
            t_full = t_factor + t_run
            return {"value": B.shape[1] / t_full, "unit": UNIT, "cores": threads, "kind": "port",
                    "sample": (f"oracle block-GMRES + ILU0 on the same {J.shape[0]}-unknown system, "
                               f"{B.shape[1]} RHS, cache-blocked dense products: the whole solve to rtol {RTOL:g} ({st.niter} "
                               f"iterations, {t_run:.2f} s) plus the ILU0 factorization ({t_factor:.2f} s)"),
                    "seconds_per_solve": t_full, "iterations": st.niter}
    return {"value": B.shape[1] / t_full, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"oracle block-GMRES + ILU0 on the same {J.shape[0]}-unknown system, "
                       f"{B.shape[1]} RHS, cache-blocked dense products: runs of {k1} and {k2} iterations "
                       f"({t1:.2f} s, {t2:.2f} s) fit T(k)=a k + b k(k+1)/2, extrapolated to the "
                       f"{K} iterations the solve needs, plus the ILU0 factorization ({t_factor:.2f} s)"),
            "seconds_per_solve": t_full}


def run_reference(args, rank, world):
    if rank != 0:
        return
    J, B = make_workload(0)
    threads = os.cpu_count() or 1
    vals = []
    cb = None
    iters = args.ref_iters
    for s in range(args.warmup + args.steps):
        cb = cpu_baseline(J, B, iters, threads)
        if s >= args.warmup:
            vals.append(cb["value"])
    v = statistics.mean(vals)
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * P_RHS / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(world),
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(world):
    return {"workload": "grid9k_p64_block_gmres_ilu0", "n_bus": N_BUS, "n_pv": N_PV,
            "unknowns": 16998, "rhs": P_RHS, "solver": "block_gmres(restart=false, itmax=300)",
            "preconditioner": "ILU0 (right, ldiv); variant below", "rtol": RTOL,
            "step": "ILU0 numeric refactor + block-GMRES solve", "l2": "flushed between steps",
            "parallelism": f"replicas x{world} (independent grids)"}


def kernel_only(name, reps, iters=24, ordering="natural"):
    """A few launches of one kernel on a case whose blocks exceed L2, for ncu captures:
    70,000-bus grid (134,998 unknowns, ~980k nonzeros), 128 right-hand sides."""
    import numpy as np
    import torch

    import blockpowerflow_b200 as bpf

    if name == "gmres":
        # `iters` iterations of the benchmark's solve (9,000-bus grid, 64 RHS; 69 = the whole
        # solve): every kernel of the block-GMRES iteration, for a launch list
        J, B = make_workload(0)
        A = bpf.CuSparseMatrixCSR.from_scipy(J)
        Bd = bpf.colmajor(torch.as_tensor(B, device="cuda"))
        N = bpf.ilu0(A, P_RHS, ordering=ordering)
        for _ in range(reps):
            X, st = bpf.block_gmres(A, Bd, N=N, ldiv=True, restart=False, memory=ITMAX, atol=0.0,
                                    rtol=RTOL, itmax=iters)
        torch.cuda.synchronize()
        print(json.dumps({"kernel_only": name, "n": J.shape[0], "p": P_RHS, "reps": reps,
                          "iterations": st.niter}))
        return
    if name == "mlp":
        # training steps of the learned warm start on the benchmark's grid (16,998 unknowns,
        # hidden 512, batches of 64 solver-style pairs): the tcgen05 GEMMs of forward + backward
        from blockpowerflow_b200 import learned

        J, B = make_workload(0)
        n = J.shape[0]
        mlp = learned.WarmStartMLP(n, 512, seed=0)
        Bd = bpf.colmajor(torch.as_tensor(B, device="cuda"))
        Xd = bpf.colmajor(torch.randn(n, P_RHS, dtype=torch.float64, device="cuda"))
        for _ in range(reps):
            loss = mlp.train_step(Bd, Xd, 1e-4)
        torch.cuda.synchronize()
        print(json.dumps({"kernel_only": name, "n": n, "p": P_RHS, "reps": reps, "loss": loss}))
        return
    J = bpf.grid.preset_jacobian("case70k", 0)
    n = J.shape[0]
    p = 128
    A = bpf.CuSparseMatrixCSR.from_scipy(J)
    X = bpf.colmajor(torch.randn(n, p, dtype=torch.float64, device="cuda"))
    Y = bpf.empty_colmajor(n, p)
    if name in ("trsv", "factor"):
        P = bpf.ilu0(A, p)
    for _ in range(reps):
        if name == "trsv":
            bpf.ldiv_(Y, P, X)
        elif name == "spmm":
            bpf.mul(A, X, Y=Y)
        elif name == "factor":
            P.refactor(A.nzVal)
        elif name == "gram":
            bpf.householder(X[:, :64])
    torch.cuda.synchronize()
    print(json.dumps({"kernel_only": name, "n": n, "p": p, "reps": reps}))


def _class_rates(bpf, classes):
    out = {}
    for kc in classes:
        ms, cnt, by, fl = bpf._lib.kernel_time(kc)
        if cnt:
            out[kc] = {"ms": ms, "launches": cnt, "avg_us": 1e3 * ms / cnt,
                       "GBps": by / (ms / 1e3) / 1e9 if by and ms > 0 else None,
                       "TFLOPs": fl / (ms / 1e3) / 1e12 if fl and ms > 0 else None}
    return out


def config_rf25k(args):
    """Third configuration: cusolverRF-style analyse once, then per step refactor + solve of
    256 RHS on the fixed pattern of a 25,000-bus grid (~48k unknowns), over a sequence of
    Jacobians whose operating point is perturbed by N(0, 0.01) per step.  Ten distinct
    perturbed value sets (seeded) are cycled through the steps; each step copies its values
    host -> device, refactors and solves (RHS solves/s = 256 / step time)."""
    import numpy as np
    import scipy.sparse.linalg as sla
    import torch

    import blockpowerflow_b200 as bpf
    from blockpowerflow_b200 import grid as g

    RF = bpf.CUSOLVERRF
    nrhs, nsets = 256, 10
    gr = g.make_grid(25000, 2000, seed=0)
    J = g.jacobian(gr)
    n = J.shape[0]
    vals = [g.perturbed_values(gr, J, t, sigma=0.01, seed=0) for t in range(nsets)]
    A = bpf.CuSparseMatrixCSR.from_scipy(J)
    vals_h = [torch.as_tensor(v).pin_memory() for v in vals]
    B = g.gaussian_rhs(n, nrhs, 1)
    Bd = bpf.colmajor(torch.as_tensor(B, device="cuda"))
    X = bpf.empty_colmajor(n, nrhs)
    t0 = time.time()
    rf = RF.CusolverRfLU(A, nrhs=nrhs, ordering="AMD")
    torch.cuda.synchronize()
    t_analyze = time.time() - t0
    info = rf.info()

    def step(t):
        A.nzVal.copy_(vals_h[t % nsets], non_blocking=True)
        RF.update_(rf, A)
        X.copy_(Bd)
        RF.ldiv_(rf, X)

    for t in range(max(3, args.warmup)):
        step(t)
    torch.cuda.synchronize()
    # residual of every value set (outside the timed region)
    worst = 0.0
    for t in range(nsets):
        step(t)
        R = bpf.mul(A, X, alpha=-1.0, beta=1.0, Y=Bd.clone())
        worst = max(worst, float(torch.linalg.norm(R) / torch.linalg.norm(Bd)))
    steps = args.steps if args.steps > 5 else 100
    bpf._lib.set_timing(True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for t in range(steps):
        step(t)
    e1.record()
    torch.cuda.synchronize()
    t_ms = e0.elapsed_time(e1)
    kern = _class_rates(bpf, ("factor", "trsv"))
    bpf._lib.set_timing(False)
    # CPU comparison: SuperLU (scipy) factor + 256-RHS solve of the same matrices, 1 thread
    Js = [J.copy() for _ in range(2)]
    for i, Jc in enumerate(Js):
        Jc.data = vals[i].copy()
    tc = time.time()
    for Jc in Js:
        lu = sla.splu(Jc.tocsc(), permc_spec="COLAMD")
        lu.solve(B)
    t_cpu = (time.time() - tc) / len(Js)
    hbm, hbm_src = peaks()
    line = {"config": {"workload": "grid25k_p256_rf_sequence", "n_bus": 25000, "n_pv": 2000,
                       "unknowns": n, "nnz": int(J.nnz), "rhs": nrhs, "steps": steps,
                       "value_sets": nsets, "ordering": "AMD (minimum degree)",
                       "nnzL": info["nnzL"], "nnzU": info["nnzU"]},
            "metric": "RHS solves/s (refactor + solve per step)", "unit": "RHS solves/s",
            "value": nrhs * steps / (t_ms / 1e3), "ms_per_step": t_ms / steps,
            "analyze_s": t_analyze, "max_relres": worst, "dtype": "f64",
            "kernels": kern,
            "roofline_sparse": {k: {"achieved_GBps": v["GBps"], "frac_of_hbm": v["GBps"] / hbm,
                                    "peak_source": hbm_src} for k, v in kern.items() if v["GBps"]},
            "cpu_baseline": {"value": nrhs / t_cpu, "unit": "RHS solves/s", "cores": 1,
                             "kind": "scipy SuperLU (COLAMD) factor + solve per step",
                             "sample": "2 of the value sets"}}
    print(json.dumps(line), flush=True)


def config_gmres300(args):
    """First configuration: the 300-bus grid (530 unknowns), 16 Gaussian RHS, block-GMRES
    (memory 30, restart) + ILU(0), atol 0, rtol 1e-8; the oracle (C restatement) beside it."""
    import numpy as np
    import torch

    import blockpowerflow_b200 as bpf
    from blockpowerflow_b200 import grid as g
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    J = g.preset_jacobian("case300", 0)
    n, p = J.shape[0], 16
    B = g.gaussian_rhs(n, p, 1)
    A = bpf.CuSparseMatrixCSR.from_scipy(J)
    Bd = torch.as_tensor(B, device="cuda")
    N = bpf.ilu0(A, p)

    def solve():
        N.refactor(A.nzVal)
        return bpf.block_gmres(A, Bd, N=N, ldiv=True, memory=30, restart=True, atol=0.0, rtol=1e-8)

    for _ in range(max(3, args.warmup)):
        X, st = solve()
    torch.cuda.synchronize()
    steps = max(args.steps, 20)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        X, st = solve()
    e1.record()
    torch.cuda.synchronize()
    t_ms = e0.elapsed_time(e1)
    Xh = X.cpu().numpy()
    rel = float(np.linalg.norm(B - J @ Xh) / np.linalg.norm(B))
    O.set_threads(1)
    tc = time.time()
    reps = 5
    for _ in range(reps):
        Xo, so = O.block_gmres(J, B, N=(1, O.ilu0(J)), memory=30, restart=True, atol=0.0, rtol=1e-8)
    t_cpu = (time.time() - tc) / reps
    line = {"config": {"workload": "grid300_p16_gmres30_ilu0", "unknowns": n, "nnz": int(J.nnz),
                       "rhs": p, "solver": "block_gmres(memory=30, restart=true)"},
            "metric": "RHS solves/s at 1e-8 residual", "unit": "RHS solves/s",
            "value": p * steps / (t_ms / 1e3), "ms_per_step": t_ms / steps, "iterations": st.niter,
            "oracle_iterations": so.niter, "relres": rel,
            "rel_diff_vs_oracle": float(np.linalg.norm(Xh - Xo) / np.linalg.norm(Xo)),
            "dtype": "f64",
            "cpu_baseline": {"value": p / t_cpu, "unit": "RHS solves/s", "cores": 1, "kind": "port",
                             "sample": f"{reps} full solves"}}
    print(json.dumps(line), flush=True)


def config_bicgstab9k(args):
    """Second configuration: block-BiCGSTAB + ILU(0) on the 9,000-bus grid, 64 RHS, FP64
    factors and FP32 factors; reports iterations, convergence and time."""
    import numpy as np
    import torch

    import blockpowerflow_b200 as bpf

    J, B = make_workload(0)
    n = J.shape[0]
    A = bpf.CuSparseMatrixCSR.from_scipy(J)
    Bd = torch.as_tensor(B, device="cuda")
    out = {}
    for name, fd in (("fp64", "float64"), ("fp32_factors", "float32")):
        N = bpf.ilu0(A, P_RHS, factor_dtype=fd)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        N.refactor(A.nzVal)
        X, st = bpf.block_bicgstab(A, Bd, N=N, atol=0.0, rtol=RTOL, itmax=400)
        e1.record()
        torch.cuda.synchronize()
        Xh = X.cpu().numpy()
        rel = float(np.linalg.norm(B - J @ Xh) / np.linalg.norm(B)) if np.all(np.isfinite(Xh)) else None
        out[name] = {"iterations": st.niter, "solved": bool(st.solved), "status": st.status,
                     "relres": rel, "ms": e0.elapsed_time(e1)}
    line = {"config": {"workload": "grid9k_p64_block_bicgstab_ilu0", "unknowns": n, "rhs": P_RHS,
                       "itmax": 400, "rtol": RTOL},
            "metric": "RHS solves/s at 1e-8 residual", "unit": "RHS solves/s",
            "value": {k: (P_RHS / (v["ms"] / 1e3) if v["solved"] else 0.0) for k, v in out.items()},
            "variants": out, "dtype": "f64"}
    print(json.dumps(line), flush=True)


def config_newton9k(args):
    """The caller of the solve path: Newton power flow on the 9,000-bus grid (16,998 unknowns)
    from an operating point perturbed by N(0, 0.001) (from N(0, 0.01) Newton stalls on this random
    operating point), every step the mismatch and Jacobian assembled on the device, then a
    refactorization + solve on the device (cusolverRF-style path), then the sensitivities dx/du =
    -Gx^{-1} Gu to the 1,001 control voltages (slack and PV) as one multi-RHS solve.  Beside it:
    the same loop with numpy assembly and SciPy's SuperLU (1 core)."""
    import numpy as np
    import torch

    import blockpowerflow_b200 as bpf
    from blockpowerflow_b200 import grid as g
    from blockpowerflow_b200 import newton as NT
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    prob = NT.make_problem(g.make_grid(N_BUS, N_PV, seed=0))
    x0 = NT.perturbed_start(prob, 0.001, seed=1)
    NT.newton(prob, solver="rf", x0=x0, tol=1e-10, sensitivities=True)   # warm-up (analysis, JIT)
    torch.cuda.synchronize()
    # three cold solves (each with its own RF analysis); the median is reported, since their host
    # part (analysis, the 136 MB sensitivity block's copy to the host) meets the shared host's
    # load; kernel times are taken from the first
    cold = []
    for rep in range(3):
        bpf._lib.set_timing(rep == 0)
        t0 = time.time()
        r = NT.newton(prob, solver="rf", x0=x0, tol=1e-10, sensitivities=True)
        torch.cuda.synchronize()
        cold.append(time.time() - t0)
        if rep == 0:
            kern = _class_rates(bpf, ("factor", "trsv", "pf"))
    bpf._lib.set_timing(False)
    t_gpu = float(np.median(cold))
    # the same power flow with the solver (its RF analysis) built once for the pattern and reused,
    # as a sequence of power flows on one network would run
    torch.cuda.synchronize()
    t0 = time.time()
    lin = NT.RFSolver(prob, len(prob.ctrl), "AMD")
    torch.cuda.synchronize()
    t_analysis = time.time() - t0
    NT.newton(prob, solver=lin, x0=x0, tol=1e-10, sensitivities=True)
    torch.cuda.synchronize()
    t0 = time.time()
    rw = NT.newton(prob, solver=lin, x0=x0, tol=1e-10, sensitivities=True)
    torch.cuda.synchronize()
    t_reuse = time.time() - t0

    class _LU:
        def refactor(self, vals):
            J = sp.csc_matrix(sp.csr_matrix((vals, prob.pattern.indices, prob.pattern.indptr),
                                            shape=prob.pattern.shape))
            self.lu = spla.splu(J, permc_spec="COLAMD")

        def solve(self, B):
            return self.lu.solve(np.asarray(B))

    t0 = time.time()
    rc = NT.newton(prob, solver=_LU(), x0=x0, tol=1e-10, sensitivities=True)
    t_cpu = time.time() - t0
    dev_ms = sum(v["ms"] for k, v in kern.items() if k != "pf")
    asm_ms = kern.get("pf", {}).get("ms", 0.0)
    line = {"config": {"workload": "grid9k_newton_powerflow_rf", "unknowns": int(prob.pattern.shape[0]),
                       "controls": int(len(prob.ctrl)), "start": "operating point + N(0, 0.001)",
                       "tol": 1e-10},
            "metric": "Newton power flow + sensitivities, seconds", "unit": "s", "higher_is_better": False,
            "value": t_gpu, "iterations": r.iterations, "converged": bool(r.converged),
            "cold_samples_s": cold, "rf_analysis_s": t_analysis,
            "analysis_reused": {"value": t_reuse, "unit": "s", "iterations": rw.iterations,
                                "converged": bool(rw.converged)},
            "residuals": r.residuals, "device_linear_ms": dev_ms, "device_assembly_ms": asm_ms, "kernels": kern,
            "host_ms": 1e3 * cold[0] - dev_ms - asm_ms,
            "sensitivity_rel_diff_vs_superlu": float(np.linalg.norm(r.sensitivities - rc.sensitivities)
                                                     / np.linalg.norm(rc.sensitivities)),
            "cpu_baseline": {"value": t_cpu, "unit": "s", "cores": 1,
                             "kind": "numpy assembly + scipy SuperLU in the same loop",
                             "iterations": rc.iterations},
            "dtype": "f64", "data": "synthetic"}
    print(json.dumps(line), flush=True)


def batch_workload(nsys=512, seed=0):
    """Fourth configuration's inputs: nsys synthetic grids with log-uniform 100 - 3,000 buses
    and U{8..64} Gaussian right-hand sides each (seeded)."""
    import numpy as np

    from blockpowerflow_b200 import grid as g

    rng = np.random.default_rng(seed)
    buses = np.exp(rng.uniform(np.log(100), np.log(3000), nsys)).astype(int)
    nrhs = rng.integers(8, 65, nsys)
    mats = [g.jacobian(g.make_grid(int(b), seed=1000 + k)).tocsr() for k, b in enumerate(buses)]
    Bs = [g.gaussian_rhs(A.shape[0], int(p), 5000 + k) for k, (A, p) in enumerate(zip(mats, nrhs))]
    return buses, [int(p) for p in nrhs], mats, Bs


def config_batch512(args):
    """Fourth configuration: 512 independent grids (100 - 3,000 buses, log-uniform), 8 - 64
    RHS each, ILU(0) block-GMRES in one persistent CUDA-graph launch (FP32 factors, FP64
    residual and orthogonalization), launch shape chosen by the autotuner.  One step = the
    ILU(0) of every system + the solve of every right-hand side (one graph launch).  Beside it:
    the plain FP64 drop-in (bpf.ilu0 + bpf.block_gmres per system, natural order, one system
    after another) on the same inputs, and the oracle on a sample of the systems."""
    import numpy as np
    import torch

    import blockpowerflow_b200 as bpf
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    nsys = int(os.environ.get("BPF_BATCH_NSYS", "512"))
    buses, nrhs, mats, Bs = batch_workload(nsys)
    total_rhs = int(sum(nrhs))
    dm = [bpf.CuSparseMatrixCSR.from_scipy(A) for A in mats]
    Bd = [torch.as_tensor(B, device="cuda") for B in Bs]
    t0 = time.time()
    tune = bpf.autotune(dm, nrhs, Bd, cache_path=os.environ.get("BPF_TUNE_CACHE"), repeats=1)
    t_tune = time.time() - t0
    t0 = time.time()
    plan = bpf.BatchPlan(dm, nrhs, slice=tune["slice"], ctas_per_sm=tune["ctas_per_sm"])
    torch.cuda.synchronize()
    t_plan = time.time() - t0
    for _ in range(max(3, args.warmup)):
        Xs, st = plan.solve(Bd)
    torch.cuda.synchronize()
    worst = 0.0
    for A, B, X in zip(mats, Bs, Xs):
        worst = max(worst, float(np.linalg.norm(B - A @ X.cpu().numpy()) / np.linalg.norm(B)))
    solved = all(x.solved for x in st)
    units = plan.unit_stats()
    cyc = plan.unit_cycles()
    steps = max(args.steps, 5)
    launches0 = bpf.kernel_launches()
    bpf._lib.set_timing(True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        Xs, st = plan.solve(Bd)
    e1.record()
    torch.cuda.synchronize()
    t_ms = e0.elapsed_time(e1)
    launches = bpf.kernel_launches() - launches0
    ms_b, cnt_b, by_b, fl_b = bpf._lib.kernel_time("batch")
    bpf._lib.set_timing(False)
    # end to end: host (pinned) B in, X out, through the public API
    Bh = [torch.as_tensor(B).pin_memory() for B in Bs]
    h2d = sum(B.numel() * 8 for B in Bh)
    torch.cuda.synchronize()
    te = time.time()
    e_steps = max(2, steps // 2)
    for _ in range(e_steps):
        Xs_e, _ = plan.solve([B.to("cuda", non_blocking=True) for B in Bh])
        Xh = [X.cpu() for X in Xs_e]
    torch.cuda.synchronize()
    t_e2e = (time.time() - te) / e_steps
    # the plain FP64 drop-in, one system after another (natural-order ILU(0), unrestarted)
    torch.cuda.synchronize()
    tp = time.time()
    plain_ok = True
    for A, B, p in zip(dm, Bd, nrhs):
        N = bpf.ilu0(A, p)
        X, s = bpf.block_gmres(A, B, N=N, ldiv=True, restart=False, memory=400, atol=0.0, rtol=RTOL,
                               itmax=400)
        plain_ok = plain_ok and s.solved
    torch.cuda.synchronize()
    t_plain = time.time() - tp
    # CPU: the oracle's block-GMRES on a sample of the systems (1 thread), scaled by RHS
    O.set_threads(1)
    O.set_fast_dense(True)   # cache-blocked dense products while timing
    idx = list(range(0, nsys, max(1, nsys // 8)))[:8]
    tc = time.time()
    for k in idx:
        O.block_gmres(mats[k], Bs[k], N=(1, O.ilu0(mats[k])), memory=400, restart=False, atol=0.0,
                      rtol=RTOL, itmax=400)
    t_cpu = time.time() - tc
    O.set_fast_dense(False)
    cpu_rhs = sum(nrhs[k] for k in idx)
    hbm, hbm_src = peaks()
    achieved = by_b / (ms_b / 1e3) / 1e9 if ms_b > 0 else None
    tot = {k: int(v.sum()) for k, v in cyc.items()}
    value = total_rhs * steps / (t_ms / 1e3)
    line = {"config": {"workload": f"batch{nsys}_grids100-3000_p8-64", "systems": nsys,
                       "unknowns_total": int(sum(A.shape[0] for A in mats)), "rhs_total": total_rhs,
                       "nnz_total": int(sum(A.nnz for A in mats)), "units": plan.nunits,
                       "grid": plan.grid, "slice": tune["slice"], "ctas_per_sm": tune["ctas_per_sm"],
                       "ordering": "AMD (minimum degree)", "factors": "FP32", "rtol": RTOL,
                       "l2": "inputs larger than L2 (all systems' bases)"},
            "metric": "RHS solves/s at 1e-8 residual (batched)", "unit": "RHS solves/s",
            "value": value, "ms_per_step": t_ms / steps, "steps": steps,
            "all_solved": solved, "max_relres": worst,
            "iterations": {"max": int(units["niter"].max()), "mean": float(units["niter"].mean())},
            "phase_share": {k: round(v / max(tot["total"], 1), 4) for k, v in tot.items() if k != "total"},
            "unit_cycles": {"max": int(cyc["total"].max()), "mean": float(cyc["total"].mean()),
                            "sum": int(cyc["total"].sum()),
                            "balanced_bound_ms": float(cyc["total"].sum()) / plan.grid / 1.965e6,
                            "critical_path_ms": float(cyc["total"].max()) / 1.965e6},
            "gpu_launches": launches,
            "e2e": {"value": total_rhs / t_e2e, "unit": "RHS solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": h2d},
            "plain_fp64_dropin": {"value": total_rhs / t_plain, "seconds": t_plain, "all_solved": plain_ok,
                                  "how": "bpf.ilu0 + bpf.block_gmres per system, natural order"},
            "batched_over_plain": value / (total_rhs / t_plain),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm if achieved else None, "peak_source": hbm_src,
                         "kernel": "batch graph (factor + persistent solve)",
                         "bytes_per_step": by_b / max(cnt_b, 1)},
            "autotune": {"seconds": t_tune, **{k: v for k, v in tune.items() if k != "cached"}},
            "plan_seconds": t_plan,
            "cpu_baseline": {"value": cpu_rhs / t_cpu, "unit": "RHS solves/s", "cores": 1, "kind": "port",
                             "sample": f"{len(idx)} of the {nsys} systems, full solves"},
            "dtype": "f64 (FP32 factors)", "data": "synthetic"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel-only", choices=["trsv", "spmm", "factor", "gram", "gmres", "mlp"], default=None,
                    help="launch one kernel a few times on a 135k-unknown case (for ncu)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--iters", type=int, default=24, help="block-GMRES iterations (--kernel-only gmres)")
    ap.add_argument("--ordering", default="natural", help="ILU(0) ordering (--kernel-only gmres)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-iters", type=int, default=69,
                    help="iterations the reference arm extrapolates to (the GPU solve's count)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config", default="headline",
                    choices=["headline", "gmres300", "bicgstab9k", "rf25k", "batch512", "newton9k"],
                    help="the other benchmark configurations (one JSON line each, one GPU)")
    args = ap.parse_args()
    if args.config != "headline":
        {"gmres300": config_gmres300, "bicgstab9k": config_bicgstab9k,
         "rf25k": config_rf25k, "batch512": config_batch512, "newton9k": config_newton9k}[args.config](args)
        return
    if args.kernel_only:
        kernel_only(args.kernel_only, args.reps, args.iters, args.ordering)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_

        dist = dist_
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            import torch

            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import numpy as np
    import torch

    import blockpowerflow_b200 as bpf
    from blockpowerflow_b200 import replicas

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    J, B = make_workload(rank)
    n = J.shape[0]
    A = bpf.CuSparseMatrixCSR.from_scipy(J, device=dev)
    Bd = bpf.colmajor(torch.as_tensor(B, device=dev))
    # plain FP64 ILU(0) drop-in (natural order, as the reference), FP32 factors, and the
    # minimum-degree-ordered ILU(0) with FP64 / FP32 factors (26 dependency levels per sweep
    # instead of 14, 57 iterations instead of 69; reverse Cuthill-McKee needs 46 iterations but
    # 456 levels, which the level-scheduled solves pay for)
    precs = {"fp64": bpf.ilu0(A, P_RHS), "mixed": bpf.ilu0(A, P_RHS, factor_dtype="float32"),
             "amd": bpf.ilu0(A, P_RHS, ordering="AMD"),
             "amd_mixed": bpf.ilu0(A, P_RHS, factor_dtype="float32", ordering="AMD")}
    # learned warm start + rank-16 deflation on the minimum-degree ILU(0), trained before the
    # timed region on the solver's own solves at 16 perturbed operating points of the grid
    from blockpowerflow_b200 import grid as gmod
    from blockpowerflow_b200 import learned

    t_setup = time.time()
    grid_obj = gmod.make_grid(N_BUS, N_PV, seed=rank)
    pairs, l_scale = learned.solver_pairs(grid_obj, J, precs["amd"], blocks=16, p=P_RHS, seed=1 + rank)
    mlp = learned.WarmStartMLP(n, 512, seed=rank)
    mlp.set_scale(l_scale)
    l_hist = learned.train(mlp, pairs, epochs=6, lr=2e-4, batch=64)
    Zl = mlp.basis(16)
    n_pairs = sum(int(b.shape[1]) for b, _ in pairs)
    del pairs
    torch.cuda.synchronize()
    l_setup_s = time.time() - t_setup
    nB = float(np.linalg.norm(B))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    # pinned host buffers for the end-to-end measurement
    vals_h = torch.as_tensor(J.data.astype(np.float64)).pin_memory()
    B_h = torch.as_tensor(np.ascontiguousarray(B.T)).pin_memory()   # column-major n x p
    X_h = torch.empty((P_RHS, n), dtype=torch.float64).pin_memory()

    def solve_on(N, Bm, use_learned):
        N.refactor(A.nzVal)
        if use_learned:   # judged warm start, learned deflation basis, tolerance RTOL ||B||
            X0 = learned.judged_warm_start(mlp, A, Bm)
            return bpf.block_gmres(A, Bm, X0, N=N, ldiv=True, restart=False, memory=ITMAX,
                                   atol=RTOL * nB, rtol=0.0, itmax=ITMAX, deflation=Zl)
        return bpf.block_gmres(A, Bm, N=N, ldiv=True, restart=False, memory=ITMAX, atol=0.0,
                               rtol=RTOL, itmax=ITMAX)

    variants = {"fp64": (precs["fp64"], False), "mixed": (precs["mixed"], False),
                "amd": (precs["amd"], False), "amd_mixed": (precs["amd_mixed"], False),
                "amd_learned": (precs["amd"], True)}

    def step_e2e(name):
        N, use_learned = variants[name]
        A.nzVal.copy_(vals_h, non_blocking=True)
        Bh_dev = torch.empty((P_RHS, n), dtype=torch.float64, device=dev)
        Bh_dev.copy_(B_h, non_blocking=True)  # row-major p x n == column-major n x p
        X, st = solve_on(N, Bh_dev.t(), use_learned)
        X_h.copy_(X.t(), non_blocking=False)
        return st

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(name, sample_clocks):
        """K device-resident steps: time, converged RHS, per-class kernel times, residuals."""
        N, use_learned = variants[name]

        def solve(_N):
            return solve_on(_N, Bd, use_learned)

        for _ in range(max(3, args.warmup)):
            X, st = solve(N)
        torch.cuda.synchronize()
        sampler = ClockSampler(torch.cuda.current_device()) if (rank == 0 and sample_clocks) else None
        l0 = bpf.kernel_launches()
        bpf._lib.set_timing(True)
        barrier()
        if sampler:
            sampler.start()
        ev, solved_rhs = [], 0
        for k in range(args.steps):
            flush.fill_(float(k))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            X, st = solve(N)
            e1.record()
            ev.append((e0, e1))
            solved_rhs += P_RHS if st.solved else 0
        barrier()
        clocks = sampler.stop() if sampler else None
        launches = bpf.kernel_launches() - l0
        t_ms = sum(a.elapsed_time(b) for a, b in ev)
        kern = {}
        for kc in ("spmm", "trsv", "factor", "gram", "tsmm", "small", "chol", "hess", "backsub", "mlp"):
            ms, cnt, by, fl = bpf._lib.kernel_time(kc)
            kern[kc] = {"ms": ms, "launches": cnt, "bytes": by, "flops": fl}
        bpf._lib.set_timing(False)
        tot_rhs, t_max = replicas.aggregate(solved_rhs, t_ms, device=dev)
        value = tot_rhs / (t_max / 1e3)
        R = B - J @ X.cpu().numpy()
        col_rel = np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)
        return {"value": value, "t_ms": t_ms, "t_max": t_max, "iterations": st.niter,
                "solved_fraction": solved_rhs / (P_RHS * args.steps),
                "relres": float(np.linalg.norm(R) / np.linalg.norm(B)),
                "max_column_relres": float(col_rel.max()), "launches": int(launches),
                "kern": kern, "clocks": clocks}

    results = {name: timed(name, name == "fp64") for name in variants}
    ok = {k: r for k, r in results.items() if r["solved_fraction"] == 1.0 and r["relres"] <= RTOL}
    head = max(ok, key=lambda k: ok[k]["value"]) if ok else "fp64"
    r = results[head]
    clocks = results["fp64"]["clocks"]
    iters = r["iterations"]

    # ---- end-to-end timed region (the headline variant) ----------------------------------
    for _ in range(3):
        step_e2e(head)
    barrier()
    e2e_t = 0.0
    e2e_rhs = 0
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st2 = step_e2e(head)
        e1.record()
        torch.cuda.synchronize()
        e2e_t += e0.elapsed_time(e1)
        e2e_rhs += P_RHS if st2.solved else 0
    e2e_tot, e2e_t = replicas.aggregate(e2e_rhs, e2e_t, device=dev)
    e2e_val = e2e_tot / (e2e_t / 1e3)

    # ---- roofline of the dominant kernel class -------------------------------------------
    hbm, hbm_src = peaks()
    kern, t_ms = r["kern"], r["t_ms"]
    breakdown = {}
    for k, v in kern.items():
        if v["launches"] == 0:
            continue
        s = v["ms"] / 1e3
        breakdown[k] = {"share": v["ms"] / max(t_ms, 1e-9), "launches": v["launches"],
                        "avg_us": 1e3 * v["ms"] / v["launches"],
                        "GBps": v["bytes"] / s / 1e9 if v["bytes"] else None,
                        "TFLOPs": v["flops"] / s / 1e12 if v["flops"] else None}
    # The Hessenberg class runs on the second stream, overlapped with the Arnoldi step, so
    # the dominant class is taken among the main-stream classes.
    main = [k for k in kern if k != "hess"]
    dom = max(main, key=lambda k: kern[k]["ms"])
    fp64_peak = fp64_peak_tflops(dev)
    v = kern[dom]
    secs = v["ms"] / 1e3 if v["ms"] > 0 else float("inf")
    if dom in ("gram", "tsmm"):
        ach = v["flops"] / secs / 1e12
        roofline = {"bound": "tensor", "kernel": dom, "achieved": ach, "peak": fp64_peak,
                    "unit": "TFLOP/s", "frac": ach / fp64_peak,
                    "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 (FP64 tensor pipe)",
                    "flops_per_launch": v["flops"] / max(v["launches"], 1),
                    "bytes_per_launch": v["bytes"] / max(v["launches"], 1)}
    else:
        ach = v["bytes"] / secs / 1e9
        roofline = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": hbm, "unit": "GB/s",
                    "frac": ach / hbm, "peak_source": hbm_src,
                    "bytes_per_launch": v["bytes"] / max(v["launches"], 1)}
    roofline.update({"avg_launch_us": 1e3 * v["ms"] / max(v["launches"], 1),
                     "traffic": TRAFFIC_PER_LAUNCH.get(dom),
                     "dominant_share_of_device_time": v["ms"] / max(t_ms, 1e-9)})
    # the HBM-bound sparse kernels beside it (triangular solves, SpMM)
    sparse = {}
    for k in ("trsv", "spmm"):
        w = kern[k]
        if w["ms"] > 0:
            a = w["bytes"] / (w["ms"] / 1e3) / 1e9
            sparse[k] = {"achieved_GBps": a, "frac_of_hbm": a / hbm, "peak_source": hbm_src}
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(J, B, results["fp64"]["iterations"], os.cpu_count() or 1)
    cfg = workload_config(world)
    cfg["variant"] = {"fp64": "plain FP64 ILU0 (natural order)",
                      "mixed": "FP32 ILU0 factors, flexible GMRES",
                      "amd": "minimum-degree-ordered FP64 ILU0",
                      "amd_mixed": "minimum-degree-ordered FP32 ILU0 factors, flexible GMRES",
                      "amd_learned": "minimum-degree ILU0 + learned warm start and rank-16 deflation"}[head]
    line = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": r["t_max"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": cfg,
        "iterations": iters, "relres": r["relres"], "max_column_relres": r["max_column_relres"],
        "solved_fraction": r["solved_fraction"],
        "variants": {k: {"value": x["value"], "iterations": x["iterations"], "relres": x["relres"],
                         "solved_fraction": x["solved_fraction"], "ms_per_step": x["t_max"] / args.steps}
                     for k, x in results.items()},
        "mixed_over_plain_fp64": results["mixed"]["value"] / max(results["fp64"]["value"], 1e-30),
        "headline_over_plain_fp64": r["value"] / max(results["fp64"]["value"], 1e-30),
        "learned": {"train_solves": n_pairs, "epochs": len(l_hist), "final_loss": l_hist[-1],
                    "first_loss": l_hist[0], "setup_s": l_setup_s, "deflation_rank": 16,
                    "iterations": results["amd_learned"]["iterations"],
                    "iterations_without": results["amd"]["iterations"]},
        "e2e": {"value": e2e_val, "unit": UNIT,
                "h2d_bytes_per_step": int(8 * (J.nnz + n * P_RHS)),
                "d2h_bytes_per_step": int(8 * n * P_RHS)},
        "gpu_launches": r["launches"], "roofline": roofline, "roofline_sparse": sparse,
        "kernels": breakdown,
        "cpu_baseline": cb, "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
