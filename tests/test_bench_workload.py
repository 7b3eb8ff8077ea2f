"""The batched configuration's inputs as bench.py generates them (no GPU): grids of 100 - 3,000
buses, 8 - 64 Gaussian right-hand sides each, square Jacobians with a full diagonal, the same
systems for the same seed."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_batch_workload_matches_the_configuration():
    import bench

    buses, nrhs, mats, Bs = bench.batch_workload(16, seed=0)
    assert len(mats) == len(Bs) == len(nrhs) == 16
    assert all(100 <= b < 3000 for b in buses)
    assert all(8 <= p <= 64 for p in nrhs)
    for A, B, p in zip(mats, Bs, nrhs):
        assert A.shape[0] == A.shape[1] == B.shape[0] and B.shape[1] == p
        assert (A.diagonal() != 0).all()
    b2, p2, m2, B2 = bench.batch_workload(16, seed=0)
    assert list(b2) == list(buses) and p2 == nrhs
    assert all((x != y).nnz == 0 for x, y in zip(mats, m2)) and all(np.array_equal(x, y) for x, y in zip(Bs, B2))


def test_cpu_baseline_times_the_whole_solve_when_it_is_short():
    """The oracle's solve of a small system is predicted well under the bound, so the baseline
    runs it to the tolerance and reports its real iteration count; the extrapolation is the
    fallback for long solves."""
    import bench
    from blockpowerflow_b200 import grid as g

    J = g.preset_jacobian("case300", 0)
    B = g.gaussian_rhs(J.shape[0], 8, 3)
    cb = bench.cpu_baseline(J, B, 25, 2)
    assert cb["kind"] == "port" and cb["cores"] == 2 and cb["value"] > 0
    assert "the whole solve" in cb["sample"] and cb["iterations"] > 0
    assert abs(cb["value"] - B.shape[1] / cb["seconds_per_solve"]) <= 1e-9 * cb["value"]


def test_reference_arm_prints_one_contract_line():
    """bench.py --impl reference: the oracle on the host cores, one JSON line with the keys the
    benchmark contract names (no GPU needed)."""
    import json
    import subprocess

    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
