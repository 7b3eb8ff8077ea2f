#!/usr/bin/env python
"""RHS solves/s at a 1e-8 relative residual on B200 (one JSON line on stdout).

Default workload (the batched benchmark configuration): 512 independent synthetic power-flow
grids of 100 - 3,000 buses (log-uniform, seeded; 909,646 unknowns in all) with 8 - 64 Gaussian
right-hand sides each (18,919 in all), every system solved by ILU(0)-preconditioned block-GMRES
(right preconditioner, ldiv, unrestarted) to ||B - A X||_F <= 1e-8 ||B||_F.  One step = the ILU(0)
numeric factorization of every system + the solve of every right-hand side; the pattern analysis
is set-up (a Newton loop pays it once per pattern).

  value : the batched path (FP32 ILU(0) factors, FP64 residual and orthogonalization, launch
          shape and fill-reducing order from the autotuner): one CUDA-graph launch per step,
          device-resident blocks, CUDA events around each step (max over ranks), per-kernel
          instrumentation off, L2 flushed between steps.
  plain_fp64_dropin : the reference's call per system, block_gmres(A, B; N=ilu0(A, p), ldiv=true)
          (FP64 natural-order ILU(0)), through this library on the same inputs in the same run.
  e2e   : the batched path through the public API with pinned host blocks: every B copied
          host -> device and every X device -> host inside the timed region.
  err_vs_direct : ||X - X_direct||_F / ||X_direct||_F per system against SciPy's sparse LU
          (FP64), computed outside the timed regions.
  roofline : the persistent solve kernel, from a separate pass with per-kernel CUDA events.
  cpu_baseline : the C restatement of the reference's block-GMRES + ILU(0) (oracle/) on the
          host's cores, one system per thread, on every 8th system of the batch.

`--impl reference` times that CPU restatement alone (the reference is Julia, and neither Julia
nor its CUDA.jl stack is installed) on the same 512 systems, every step a different 1/8 of them.
Multi-GPU (torchrun): the 512 systems are shared out over the ranks by longest-processing-time
assignment, no collective on the data path; value = all systems' converged RHS / max-over-ranks
time ("scaling": "strong": the total work is fixed).

`--config` names the other benchmark configurations (one line each, one GPU).
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
NSYS = 512              # systems of the batched configuration
REF_STRIDE = 8          # the CPU arms solve every REF_STRIDE-th system per step
PLAIN_ITMAX = 400


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
    iters = 69   # the solve's iteration count on this system (natural-order ILU(0))
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


def traffic_record(name):
    """DRAM bytes (read + write) per launch of a kernel on a workload, from the ncu capture
    summarised in profiles/traffic.json (written with the command that produced it); None
    when there is no capture of that kernel on that workload."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            rec = json.load(f).get(name)
        return rec
    except (OSError, ValueError):
        return None


def direct_error(A, B, X):
    """||X - A \\ B||_F / ||A \\ B||_F with SciPy's sparse LU (FP64) as the direct solve."""
    import numpy as np
    import scipy.sparse.linalg as sla

    Xd = sla.splu(A.tocsc(), permc_spec="COLAMD").solve(np.asarray(B, dtype=np.float64))
    return float(np.linalg.norm(X - Xd) / np.linalg.norm(Xd))


def rel_residual(A, B, X):
    import numpy as np

    return float(np.linalg.norm(B - A @ X) / np.linalg.norm(B))


# ---- the batched configuration -----------------------------------------------------------
def batch_sizes(nsys=NSYS, seed=0):
    from blockpowerflow_b200 import grid as g

    return g.batch_sizes(nsys, seed)


def batch_workload(nsys=NSYS, seed=0, systems=None):
    """The batched configuration's inputs (all systems, or the listed ones): grid.batch_workload."""
    from blockpowerflow_b200 import grid as g

    return g.batch_workload(nsys, seed, systems)


def batch_config(nsys=NSYS):
    """The workload, identical in both arms' lines."""
    buses, nrhs = batch_sizes(nsys)
    return {"workload": f"batch{nsys}_grids100-3000_p8-64", "systems": nsys,
            "buses": "log-uniform 100-3000 per system (seeded)", "rhs_per_system": "U{8..64}",
            "rhs_total": int(sum(nrhs)), "rhs": "Gaussian", "rtol": RTOL, "atol": 0.0,
            "solver": "ILU0 block-GMRES (right preconditioner, ldiv), unrestarted",
            "step": "ILU0 numeric factorization of every system + the solve of every right-hand side",
            "l2": "inputs larger than L2 (blocks and bases of all systems), L2 flushed between steps",
            "parallelism": "systems shared out over the ranks (LPT), no data-path collective"}


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    return O


def cpu_batch_sample(mats, Bs, threads):
    """The oracle's block-GMRES + natural-order FP64 ILU(0) (the reference's per-system call) on
    the given systems, one system per host thread (longest first), cache-blocked dense products.
    Returns (seconds, converged RHS, all solved)."""
    from concurrent.futures import ThreadPoolExecutor

    O = _oracle()
    O.set_threads(1)
    O.set_fast_dense(True)

    def one(k):
        A, B = mats[k], Bs[k]
        X, st = O.block_gmres(A, B, N=(1, O.ilu0(A)), memory=PLAIN_ITMAX, restart=False, atol=0.0,
                              rtol=RTOL, itmax=PLAIN_ITMAX)
        return B.shape[1] if st.solved else 0, bool(st.solved)

    order = sorted(range(len(mats)), key=lambda k: -mats[k].shape[0] * Bs[k].shape[1])
    try:
        t0 = time.time()
        with ThreadPoolExecutor(max_workers=threads) as ex:
            res = list(ex.map(one, order))
        dt = time.time() - t0
    finally:
        O.set_fast_dense(False)
    return dt, sum(r for r, _ in res), all(ok for _, ok in res)


def run_reference_batch(args, rank, world):
    """Reference arm: the C restatement of the reference CPU path on all host cores, each step
    every REF_STRIDE-th system of the batch (offset by the step), same metric and config."""
    if rank != 0:
        return
    buses, nrhs, mats, Bs = batch_workload()
    threads = os.cpu_count() or 1
    t_tot, rhs_tot, ok_all = 0.0, 0, True
    for s in range(args.warmup + args.steps):
        idx = list(range(s % REF_STRIDE, NSYS, REF_STRIDE))
        dt, rhs, ok = cpu_batch_sample([mats[k] for k in idx], [Bs[k] for k in idx], threads)
        if s >= args.warmup:
            t_tot += dt
            rhs_tot += rhs
            ok_all = ok_all and ok
    v = rhs_tot / t_tot
    cb = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
          "sample": (f"every {REF_STRIDE}th system of the {NSYS} (offset = step), each step's "
                     f"{NSYS // REF_STRIDE} systems one per host thread, oracle block-GMRES + FP64 "
                     "natural-order ILU0 (the reference's per-system call), cache-blocked dense products"),
          "all_solved": ok_all, "seconds": t_tot}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_tot / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": batch_config(),
            "method": "oracle (C restatement of block_gmres! + csrilu02-semantics ILU0), FP64, natural order",
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def headline_batch(args, rank, world, dist):
    import numpy as np
    import torch

    import blockpowerflow_b200 as bpf
    from blockpowerflow_b200 import replicas

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    buses, nrhs_all = batch_sizes()
    # LPT share of the systems (all of them on one GPU); unknowns ~ 1.89 x buses
    costs = [replicas.batch_system_cost(1.89 * b, p) for b, p in zip(buses, nrhs_all)]
    mine = replicas.assign_systems(costs, world)[rank]
    _, _, mats, Bs = batch_workload(systems=mine)
    nrhs = [nrhs_all[k] for k in mine]
    my_rhs = int(sum(nrhs))
    dm = [bpf.CuSparseMatrixCSR.from_scipy(A, device=dev) for A in mats]
    Bd = [bpf.colmajor(torch.as_tensor(B, device=dev)) for B in Bs]

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- set-up: autotuned launch shape, pattern analysis and graph capture ----
    t0 = time.time()
    tune = bpf.autotune(dm, nrhs, Bd, cache_path=os.environ.get("BPF_TUNE_CACHE"), repeats=1)
    t_tune = time.time() - t0
    t0 = time.time()
    plan = bpf.BatchPlan(dm, nrhs, slice=tune["slice"], ctas_per_sm=tune["ctas_per_sm"],
                         ordering=tune["ordering"], slices=tune["slices"])
    torch.cuda.synchronize()
    t_plan = time.time() - t0
    Xd = [bpf.empty_colmajor(A.shape[0], p, dev) for A, p in zip(mats, nrhs)]
    for _ in range(max(3, args.warmup)):
        _, st = plan.solve(Bd, Xd)
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    # ---- timed region: K graph launches, instrumentation off ----
    bpf._lib.set_timing(False)
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    l0 = bpf.kernel_launches()
    barrier()
    if sampler:
        sampler.start()
    ev, solved_rhs = [], 0
    for k in range(args.steps):
        flush.fill_(float(k))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _, st = plan.solve(Bd, Xd)
        e1.record()
        ev.append((e0, e1))
        solved_rhs += sum(p for p, s in zip(nrhs, st) if s.solved)
    barrier()
    clocks = sampler.stop() if sampler else None
    launches = bpf.kernel_launches() - l0
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    tot_rhs, t_max = replicas.aggregate(solved_rhs, t_ms, device=dev)
    value = tot_rhs / (t_max / 1e3)

    # ---- checks outside the timed regions: true residuals and the direct-solve error ----
    Xh = [X.cpu().numpy() for X in Xd]
    rel = [rel_residual(A, B, X) for A, B, X in zip(mats, Bs, Xh)]
    err = [direct_error(A, B, X) for A, B, X in zip(mats, Bs, Xh)]

    # ---- instrumented pass (per-kernel CUDA events; not part of `value`) ----
    units = plan.unit_stats()
    cyc = plan.unit_cycles()
    bpf._lib.set_timing(True)
    for _ in range(2):
        flush.fill_(1.0)
        plan.solve(Bd, Xd)
    torch.cuda.synchronize()
    kern = _class_rates(bpf, ("factor", "batch"))
    bpf._lib.set_timing(False)

    # ---- end to end: pinned host B in, X out, through the public API ----
    # host blocks p x n row-major = the column-major n x p blocks of the API
    Bh = [torch.from_numpy(np.ascontiguousarray(B.T)).pin_memory() for B in Bs]
    Xh_pin = [torch.empty((p, A.shape[0]), dtype=torch.float64).pin_memory() for A, p in zip(mats, nrhs)]
    Bdev = [torch.empty((p, A.shape[0]), dtype=torch.float64, device=dev) for A, p in zip(mats, nrhs)]
    h2d = int(sum(8 * B.size for B in Bs))

    def step_e2e():
        for bd, bh in zip(Bdev, Bh):
            bd.copy_(bh, non_blocking=True)
        _, s_ = plan.solve([bd.t() for bd in Bdev], Xd)
        for xh, xd in zip(Xh_pin, Xd):
            xh.copy_(xd.t(), non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return s_

    for _ in range(2):
        step_e2e()
    barrier()
    e_ms, e_rhs = 0.0, 0
    for k in range(args.steps):
        flush.fill_(float(k))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        s_ = step_e2e()
        e1.record()
        torch.cuda.synchronize()
        e_ms += e0.elapsed_time(e1)
        e_rhs += sum(p for p, s in zip(nrhs, s_) if s.solved)
    e_tot, e_max = replicas.aggregate(e_rhs, e_ms, device=dev)
    Xe = [x.numpy().T for x in Xh_pin]
    e2e_err = max(float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(Xe, Xh))

    # ---- the plain FP64 drop-in on the same inputs: ilu0(A, p) + block_gmres per system ----
    precs = [bpf.ilu0(A, p) for A, p in zip(dm, nrhs)]

    def plain_pass():
        out, ok = [], 0
        for A, B, N, p in zip(dm, Bd, precs, nrhs):
            N.refactor(A.nzVal)
            X, s = bpf.block_gmres(A, B, N=N, ldiv=True, restart=False, memory=PLAIN_ITMAX, atol=0.0,
                                   rtol=RTOL, itmax=PLAIN_ITMAX)
            out.append((X, s))
            ok += p if s.solved else 0
        return out, ok

    plain_pass()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    pres, p_rhs = plain_pass()
    e1.record()
    torch.cuda.synchronize()
    p_ms = e0.elapsed_time(e1)
    p_tot, p_max = replicas.aggregate(p_rhs, p_ms, device=dev)
    plain_value = p_tot / (p_max / 1e3)
    pX = [X.cpu().numpy() for X, _ in pres]
    # per-system records of both paths, gathered once on rank 0 (the sharded batch's one gather)
    recs = {k: {"niter": int(s_.niter), "solved": bool(s_.solved), "relres": r_, "err": e_,
                "plain_niter": int(ps.niter), "plain_solved": bool(ps.solved),
                "plain_relres": rel_residual(A, B, X), "plain_err": direct_error(A, B, X)}
            for k, s_, r_, e_, (_, ps), A, B, X in zip(mine, st, rel, err, pres, mats, Bs, pX)}
    del precs, pres
    allrec = replicas.gather_to_root(recs)

    # ---- CPU baseline (rank 0 at N = 1): every REF_STRIDE-th system on all host cores ----
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        idx = list(range(0, len(mats), REF_STRIDE))
        dt, c_rhs, c_ok = cpu_batch_sample([mats[k] for k in idx], [Bs[k] for k in idx], threads)
        cb = {"value": c_rhs / dt, "unit": UNIT, "cores": threads, "kind": "port",
              "sample": (f"every {REF_STRIDE}th system of the {NSYS} ({len(idx)} systems, "
                         f"{sum(nrhs[k] for k in idx)} RHS), one system per host thread, oracle block-GMRES "
                         "+ FP64 natural-order ILU0, cache-blocked dense products"),
              "seconds": dt, "all_solved": c_ok}

    # ---- roofline of the persistent solve kernel ----
    hbm, hbm_src = peaks()
    kb = kern.get("batch", {})
    k_launch_us = kb.get("avg_us")
    k_bytes = kb.get("bytes_per_launch")
    ach = (k_bytes / (k_launch_us / 1e6) / 1e9) if k_bytes and k_launch_us else None
    cfg_all = batch_config()
    traffic = traffic_record(f"batch_solve_kernel/{cfg_all['workload']}") if world == 1 else None
    roofline = {"bound": "hbm", "kernel": "batch_solve_kernel (persistent block-GMRES of every unit)",
                "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm if ach else None,
                "peak_source": hbm_src, "avg_launch_us": k_launch_us, "bytes_per_launch": k_bytes,
                "traffic": traffic["dram_bytes_per_launch"] if traffic else None,
                "traffic_source": traffic["source"] if traffic else None,
                "algorithmic_bytes": ("per unit iteration: ILU0 factors (4 + 4)(nnz_L + nnz_U) + 16(n+1) + 4n, "
                                      "SpMM 12 nnz + 4(n+1), the new block 8 n q x 14 passes, plus "
                                      "32 n q per basis block read (four CGS2 passes)")}
    tot = {k: int(v.sum()) for k, v in cyc.items()}
    # the longest units (the makespan is at least the longest one)
    top = np.argsort(cyc["total"])[::-1][:3]
    longest = [{"system": int(mine[units["sys"][u]]), "n": int(mats[units["sys"][u]].shape[0]),
                "q": int(units["q"][u]), "iterations": int(units["niter"][u]), "memory": int(units["memory"][u]),
                "ms": float(cyc["total"][u]) / 1.965e6,
                "phase_share": {k: round(float(cyc[k][u]) / max(float(cyc["total"][u]), 1.0), 3)
                                for k in cyc if k != "total"}} for u in top]
    plan.close()
    if rank != 0:
        return
    assert sorted(allrec) == list(range(NSYS)), "every system solved exactly once"
    R = [allrec[k] for k in range(NSYS)]
    iters = [r["niter"] for r in R]
    p_iters = [r["plain_niter"] for r in R]
    all_ok = all(r["solved"] and r["relres"] <= RTOL * (1 + 1e-7) for r in R)
    max_rel = max(r["relres"] for r in R)
    max_err = max(r["err"] for r in R)
    p_rel = max(r["plain_relres"] for r in R)
    p_err = max(r["plain_err"] for r in R)
    p_ok = all(r["plain_solved"] and r["plain_relres"] <= RTOL * (1 + 1e-7) for r in R)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": t_max / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64 (FP32 ILU0 factors)", "data": "synthetic", "config": cfg_all,
        "method": {"value": "batched: one CUDA-graph launch per step (ILU0 kernel + persistent block-GMRES "
                            "kernel), FP32 ILU0 factors in the autotuned fill-reducing order, FP64 SpMM / "
                            "orthogonalization / Hessenberg least squares / X, flexible GMRES, autotuned "
                            "launch shape",
                   "slice": tune["slice"], "ctas_per_sm": tune["ctas_per_sm"],
                   "ordering": {"AMD": "minimum degree", "RCM": "reverse Cuthill-McKee"}.get(
                       tune["ordering"], tune["ordering"]),
                   "narrowed_systems": int(sum(1 for v in (tune["slices"] or []) if v)), "units": plan.nunits,
                   "grid": plan.grid},
        "all_solved": all_ok, "max_relres": max_rel,
        "err_vs_direct": {"max": max_err, "median": float(np.median([r["err"] for r in R])),
                          "how": "||X - splu(A) \\ B||_F / ||splu(A) \\ B||_F per system"},
        "iterations": {"max": int(max(iters)), "mean": float(np.mean(iters))},
        "plain_fp64_dropin": {"value": plain_value, "ms_per_step": p_max, "all_solved": p_ok,
                              "max_relres": p_rel,
                              "err_vs_direct": {"max": p_err,
                                                "median": float(np.median([r["plain_err"] for r in R]))},
                              "iterations": {"max": int(max(p_iters)), "mean": float(np.mean(p_iters))},
                              "how": "ilu0(A, p) (FP64, natural order) at set-up; per step refactor + "
                                     "block_gmres(A, B; N, ldiv=true, restart=false) per system, one after another"},
        "batched_over_plain": value / plain_value,
        "e2e": {"value": e_tot / (e_max / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(h2d), "max_rel_diff_vs_device_X": e2e_err},
        "gpu_launches": int(launches), "roofline": roofline, "kernels": kern,
        "phase_share": {k: round(v / max(tot["total"], 1), 4) for k, v in tot.items() if k != "total"},
        "unit_cycles": {"max": int(cyc["total"].max()), "mean": float(cyc["total"].mean()),
                        "balanced_bound_ms": float(cyc["total"].sum()) / plan.grid / 1.965e6,
                        "critical_path_ms": float(cyc["total"].max()) / 1.965e6,
                        "longest_units": longest},
        "autotune": {"seconds": t_tune, **{k: v for k, v in tune.items() if k != "cached"}},
        "plan_seconds": t_plan, "systems_this_rank": len(mine), "rhs_this_rank": my_rhs,
        "cpu_baseline": cb, "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def kernel_only(name, reps, iters=24, ordering=None, nsys=64, kgrid="case70k", kp=128, timed=False):
    """A few launches of one kernel on a case whose blocks exceed L2, for ncu captures:
    70,000-bus grid (134,998 unknowns, ~980k nonzeros), 128 right-hand sides."""
    import numpy as np
    import torch

    import blockpowerflow_b200 as bpf

    if name != "batch":
        ordering = ordering or "natural"
    if name == "batch":
        # `reps` solves of the first `nsys` systems of the batched configuration; nsys = 512 is
        # the whole batch.  The plan is the one the default run's autotuner chose when its cache
        # (BPF_TUNE_CACHE, written by that run) holds this batch, so that no tuning launch
        # precedes the captured ones; else the shape it picks for the full batch (slice 32, one
        # CTA per SM, reverse Cuthill-McKee)
        _, nrhs, mats, Bs = batch_workload(systems=range(nsys))
        nrhs = nrhs[:nsys]
        dm = [bpf.CuSparseMatrixCSR.from_scipy(A) for A in mats]
        Bd = [bpf.colmajor(torch.as_tensor(B, device="cuda")) for B in Bs]
        tune = {"slice": 32, "ctas_per_sm": 1, "ordering": ordering or "RCM", "slices": None, "cached": False}
        cache = os.environ.get("BPF_TUNE_CACHE")
        if cache and ordering is None:
            key = bpf.batch.batch_key([A.n for A in dm], nrhs, torch.cuda.get_device_name(),
                                      bpf.batch.cache_extra(bpf.batch.CANDIDATES, "AMD"))
            hit = bpf.batch.load_cache(cache).get(key)
            if hit:
                tune = {**hit, "cached": True}
        plan = bpf.BatchPlan(dm, nrhs, slice=tune["slice"], ctas_per_sm=tune["ctas_per_sm"],
                             ordering=tune["ordering"], slices=tune["slices"])
        for _ in range(reps):
            Xs, st = plan.solve(Bd)
        torch.cuda.synchronize()
        print(json.dumps({"kernel_only": name, "systems": nsys, "rhs": int(sum(nrhs)), "reps": reps,
                          "solved": all(s.solved for s in st), "units": plan.nunits,
                          "plan": {k: tune[k] for k in ("slice", "ordering", "cached")},
                          "narrowed_systems": int(sum(1 for v in (tune["slices"] or []) if v)),
                          "device_bytes": plan.device_bytes}))
        plan.close()
        return
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
    J = bpf.grid.preset_jacobian(kgrid, 0)
    if name == "spmm" and ordering.upper() == "RCM":
        # the same matrix renumbered by reverse Cuthill-McKee (symmetric permutation), as a grid
        # numbered with spatial locality would be: the rows that gather one row of X sit close
        from scipy.sparse.csgraph import reverse_cuthill_mckee

        perm = reverse_cuthill_mckee(J.tocsr(), symmetric_mode=False)
        J = J.tocsr()[perm][:, perm].tocsr()
        J.sort_indices()
    n = J.shape[0]
    p = kp
    A = bpf.CuSparseMatrixCSR.from_scipy(J)
    X = bpf.colmajor(torch.randn(n, p, dtype=torch.float64, device="cuda"))
    Y = bpf.empty_colmajor(n, p)
    if name in ("trsv", "factor"):
        P = bpf.ilu0(A, p, ordering=ordering)

    def run():
        if name == "trsv":
            bpf.ldiv_(Y, P, X)
        elif name == "spmm":
            bpf.mul(A, X, Y=Y)
        elif name == "factor":
            P.refactor(A.nzVal)
        elif name == "gram":
            bpf.householder(X[:, :64], lapack=False)

    out = {"kernel_only": name, "grid": kgrid, "n": n, "p": p, "ordering": ordering, "reps": reps}
    if timed:
        # 3 warm-up launches, then `reps` launches timed by the library's per-class CUDA events
        for _ in range(3):
            run()
        bpf._lib.set_timing(True)
        for _ in range(reps):
            run()
        torch.cuda.synchronize()
        out["timing"] = _class_rates(bpf, (name,))
        bpf._lib.set_timing(False)
        hbm, src = peaks()
        for v in out["timing"].values():
            if v.get("GBps"):
                v["frac_of_hbm"] = v["GBps"] / hbm
                v["peak_source"] = src
    else:
        for _ in range(reps):
            run()
    torch.cuda.synchronize()
    print(json.dumps(out))


def _class_rates(bpf, classes):
    out = {}
    for kc in classes:
        ms, cnt, by, fl = bpf._lib.kernel_time(kc)
        if cnt:
            out[kc] = {"ms": ms, "launches": cnt, "avg_us": 1e3 * ms / cnt,
                       "bytes_per_launch": by / cnt, "flops_per_launch": fl / cnt,
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
    # residual of every value set, and the error against SciPy's sparse LU on two of them
    # (outside the timed region)
    worst, err = 0.0, 0.0
    for t in range(nsets):
        step(t)
        R = bpf.mul(A, X, alpha=-1.0, beta=1.0, Y=Bd.clone())
        worst = max(worst, float(torch.linalg.norm(R) / torch.linalg.norm(Bd)))
        if t < 2:
            Jt = J.copy()
            Jt.data = vals[t].copy()
            err = max(err, direct_error(Jt, B, X.cpu().numpy()))
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
            "err_vs_direct": {"max": err, "how": "||X - splu(A_t) \\ B||_F / ||splu(A_t) \\ B||_F, value sets 0 and 1"},
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
            "err_vs_direct": direct_error(J, B, Xh),
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
                     "relres": rel, "ms": e0.elapsed_time(e1),
                     "err_vs_direct": direct_error(J, B, Xh) if rel is not None else None}
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
            "err_vs_direct": {"max": float(np.linalg.norm(r.sensitivities - rc.sensitivities)
                                           / np.linalg.norm(rc.sensitivities)),
                              "how": "sensitivities dx/du against the SciPy SuperLU loop's"},
            "cpu_baseline": {"value": t_cpu, "unit": "s", "cores": 1,
                             "kind": "numpy assembly + scipy SuperLU in the same loop",
                             "iterations": rc.iterations},
            "dtype": "f64", "data": "synthetic"}
    print(json.dumps(line), flush=True)


def config_learned70k(args):
    """Fifth configuration: the learned warm start and rank-32 deflation basis on the 70,000-bus
    grid (134,998 unknowns), 128 right-hand sides per block.  The right-hand sides are the Newton
    caller's sensitivity solves (Gx X = Gu, benchmarks_nvidia.jl:29-39): at each operating point
    of a sequence (states perturbed by N(0, 0.001)), 128 columns of Gu for controls drawn from a
    fixed set of 512.  The network (3 layers, width 512, BF16 weights, FP32 accumulation) is trained
    by the library's own tcgen05 kernels on the solver's solutions at `--train-points` points (160:
    20,480 solves); at held-out points the learned solve (warm start + deflation, judged by plain
    ILU(0) block-GMRES's stopping test) is timed against the plain solve, both to rtol 1e-8."""
    import numpy as np
    import torch

    import blockpowerflow_b200 as bpf
    from blockpowerflow_b200 import learned
    from blockpowerflow_b200 import newton as NT

    p, T = 128, args.train_points
    nbus, npv = args.learned_buses, max(1, args.learned_buses // 14)
    t0 = time.time()
    prob = NT.make_problem(bpf.grid.make_grid(nbus, npv, seed=0))
    A = bpf.CuSparseMatrixCSR.from_scipy(prob.pattern)
    n = A.n
    N = bpf.ilu0(A, p)
    fam = learned.SensitivityFamily(prob, A, p, sigma=0.001, seed=0)
    t_setup = time.time() - t0
    t0 = time.time()
    pairs, scale = learned.family_pairs(fam, N, range(T), rtol=1e-8, itmax=400)
    torch.cuda.synchronize()
    t_data = time.time() - t0
    t0 = time.time()
    mlp = learned.WarmStartMLP(n, 512, seed=0)
    mlp.set_scale(scale)
    hist = learned.train(mlp, pairs, epochs=args.train_epochs, lr=3e-4, batch=128)
    Z = mlp.basis(32)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    n_solves = sum(int(b.shape[1]) for b, _ in pairs)
    del pairs
    torch.cuda.empty_cache()

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        X, st = fn()
        e1.record()
        torch.cuda.synchronize()
        return X, st, e0.elapsed_time(e1)

    rows, errs = [], {}
    held = list(range(10_000, 10_000 + max(3, args.steps)))
    for k, t in enumerate(held):
        B = fam.point(t)
        nb = float(torch.linalg.norm(B))

        def plain():
            N.refactor(A.nzVal)
            return bpf.block_gmres(A, B, N=N, ldiv=True, restart=False, memory=400, atol=1e-8 * nb, rtol=0.0,
                                   itmax=400)

        def learned_solve():
            N.refactor(A.nzVal)
            return learned.solve(A, B, N, mlp, Z, rtol=1e-8, itmax=400)

        plain()           # warm-up of both paths at this point's shapes
        learned_solve()
        Xp, sp_, ms_p = timed(plain)
        Xl, sl, ms_l = timed(learned_solve)
        rows.append({"point": t, "plain_iterations": sp_.niter, "learned_iterations": sl.niter,
                     "plain_ms": ms_p, "learned_ms": ms_l, "plain_solved": bool(sp_.solved),
                     "learned_solved": bool(sl.solved)})
        if k == 0:   # the direct solve of one held-out point (SciPy sparse LU, FP64)
            J = prob.pattern.copy()
            J.data = A.nzVal.cpu().numpy()
            Bh = B.cpu().numpy()
            errs = {"plain": direct_error(J, Bh, Xp.cpu().numpy()), "learned": direct_error(J, Bh, Xl.cpu().numpy()),
                    "relres_learned": rel_residual(J, Bh, Xl.cpu().numpy())}
    ms_p = float(np.mean([r["plain_ms"] for r in rows]))
    ms_l = float(np.mean([r["learned_ms"] for r in rows]))
    line = {"config": {"workload": f"grid{nbus // 1000}k_p128_learned_warm_start_rank32_deflation", "n_bus": nbus,
                       "n_pv": npv,
                       "unknowns": n, "nnz": int(A.nnz), "rhs": p, "rtol": 1e-8,
                       "rhs_family": "columns of Gu for 128 of a fixed set of 512 controls, at operating points "
                                     "perturbed by N(0, 0.001)",
                       "train_points": T, "held_out_points": len(held)},
            "metric": "RHS solves/s at 1e-8 residual (learned vs plain ILU0 block-GMRES)", "unit": "RHS solves/s",
            "value": p / (ms_l / 1e3), "plain_value": p / (ms_p / 1e3), "learned_over_plain": ms_p / ms_l,
            "iterations": {"plain": [r["plain_iterations"] for r in rows],
                           "learned": [r["learned_iterations"] for r in rows]},
            "held_out": rows, "err_vs_direct": errs,
            "training": {"solves": n_solves, "data_seconds": t_data, "train_seconds": t_train, "epochs": len(hist),
                         "loss_first": hist[0], "loss_last": hist[-1], "setup_seconds": t_setup,
                         "network": "3-layer MLP, width 512, BF16 weights with FP32 masters, tcgen05 GEMMs, Adam"},
            "dtype": "f64 (network BF16)", "data": "synthetic"}
    print(json.dumps(line), flush=True)


def config_gmres9k(args, rank, world, dist):
    """The 9,000-bus grid of the second benchmark configuration (16,998 unknowns, ~121k nonzeros),
    64 Gaussian right-hand sides, block-GMRES with a right ILU(0), no restart (as in
    benchmarks_nvidia.jl), atol 0, rtol 1e-8.  One step = ILU(0) numeric refactorization + the
    solve.  Variants: plain FP64 natural-order ILU(0) (the drop-in), FP32 factors,
    minimum-degree order (FP64 / FP32 factors) and the learned warm start + rank-16 deflation.
    Every rank solves its own grid (seed offset by rank)."""
    local = int(os.environ.get("LOCAL_RANK", "0"))
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
        bpf._lib.set_timing(False)
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
        # instrumented pass (per-kernel CUDA events), separate from the timed steps
        bpf._lib.set_timing(True)
        for _ in range(2):
            flush.fill_(1.0)
            solve(N)
        torch.cuda.synchronize()
        kern = {}
        for kc in ("spmm", "trsv", "factor", "gram", "tsmm", "small", "chol", "hess", "backsub", "mlp"):
            ms, cnt, by, fl = bpf._lib.kernel_time(kc)
            kern[kc] = {"ms": ms, "launches": cnt, "bytes": by, "flops": fl}
        bpf._lib.set_timing(False)
        tot_rhs, t_max = replicas.aggregate(solved_rhs, t_ms, device=dev)
        value = tot_rhs / (t_max / 1e3)
        Xn = X.cpu().numpy()
        R = B - J @ Xn
        col_rel = np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)
        return {"value": value, "t_ms": t_ms, "t_max": t_max, "iterations": st.niter,
                "err_vs_direct": float(np.linalg.norm(Xn - X_direct) / np.linalg.norm(X_direct)),
                "instrumented_steps": 2,
                "solved_fraction": solved_rhs / (P_RHS * args.steps),
                "relres": float(np.linalg.norm(R) / np.linalg.norm(B)),
                "max_column_relres": float(col_rel.max()), "launches": int(launches),
                "kern": kern, "clocks": clocks}

    import scipy.sparse.linalg as sla

    X_direct = sla.splu(J.tocsc(), permc_spec="COLAMD").solve(B)
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
    kern = r["kern"]
    t_ms = sum(v["ms"] for k, v in kern.items() if k != "hess")   # main-stream device time of the instrumented steps
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
                     "traffic": (traffic_record(f"{dom}/grid9k_p64_{head}") or {}).get("dram_bytes_per_launch"),
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
    method = {"fp64": "plain FP64 ILU0 (natural order)",
                      "mixed": "FP32 ILU0 factors, flexible GMRES",
                      "amd": "minimum-degree-ordered FP64 ILU0",
                      "amd_mixed": "minimum-degree-ordered FP32 ILU0 factors, flexible GMRES",
                      "amd_learned": "minimum-degree ILU0 + learned warm start and rank-16 deflation"}[head]
    line = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": r["t_max"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": cfg, "method": method,
        "iterations": iters, "relres": r["relres"], "max_column_relres": r["max_column_relres"],
        "err_vs_direct": r["err_vs_direct"],
        "solved_fraction": r["solved_fraction"],
        "variants": {k: {"value": x["value"], "iterations": x["iterations"], "relres": x["relres"],
                         "err_vs_direct": x["err_vs_direct"],
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



def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel-only", choices=["trsv", "spmm", "factor", "gram", "gmres", "mlp", "batch"],
                    default=None, help="launch one kernel a few times on a small case (for ncu)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--iters", type=int, default=24, help="block-GMRES iterations (--kernel-only gmres)")
    ap.add_argument("--ordering", default=None,
                    help="ILU(0) ordering of --kernel-only (default: natural; RCM for batch)")
    ap.add_argument("--nsys", type=int, default=64, help="systems of the batch (--kernel-only batch)")
    ap.add_argument("--grid", default="case70k", help="preset grid of --kernel-only trsv/spmm/factor/gram")
    ap.add_argument("--p", type=int, default=128, help="right-hand sides of --kernel-only trsv/spmm")
    ap.add_argument("--time", action="store_true", help="--kernel-only: time the launches (CUDA events)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--train-points", type=int, default=160, help="learned70k: training operating points")
    ap.add_argument("--train-epochs", type=int, default=20, help="learned70k: training epochs")
    ap.add_argument("--learned-buses", type=int, default=70000, help="learned70k: grid size (70,000 buses)")
    ap.add_argument("--config", default="batch512",
                    choices=["batch512", "gmres9k", "gmres300", "bicgstab9k", "rf25k", "newton9k", "learned70k"],
                    help="batch512 (default): the batched configuration; the others print one line "
                         "each for the other benchmark configurations")
    args = ap.parse_args()
    if args.kernel_only:
        kernel_only(args.kernel_only, args.reps, args.iters, args.ordering, args.nsys, args.grid, args.p,
                    args.time)
        return
    if args.config in ("gmres300", "bicgstab9k", "rf25k", "newton9k", "learned70k"):
        {"gmres300": config_gmres300, "bicgstab9k": config_bicgstab9k, "rf25k": config_rf25k,
         "newton9k": config_newton9k, "learned70k": config_learned70k}[args.config](args)
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
        # the reference arm's rank 0 runs minutes of CPU work while the other ranks wait at the
        # final barrier; the GPU arm's ranks meet within seconds of each other
        wait_s = 3600 if args.impl == "reference" else 600
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=wait_s))
    try:
        if args.impl == "reference":
            (run_reference_batch if args.config == "batch512" else run_reference)(args, rank, world)
        elif args.config == "batch512":
            headline_batch(args, rank, world, dist)
        else:
            config_gmres9k(args, rank, world, dist)
    finally:
        if dist:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
