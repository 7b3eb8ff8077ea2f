"""bench.py's host-side contract (no GPU): the reference arm prints one JSON line with the keys the
driver reads, on the same workload description as the GPU arm, and the CPU sample solves its
systems to the tolerance."""
import io
import json
import os
import sys
from contextlib import redirect_stdout

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_reference_arm_line_on_a_small_batch(monkeypatch):
    import bench

    monkeypatch.setattr(bench, "NSYS", 16)
    monkeypatch.setattr(bench, "REF_STRIDE", 8)

    class Args:
        steps, warmup = 2, 1

    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference_batch(Args(), 0, 1)
    line = json.loads(buf.getvalue().strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["value"] > 0 and line["cpu_baseline"]["all_solved"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    # the GPU arm describes its workload with the same function
    assert line["config"] == bench.batch_config()


def test_rank_other_than_zero_prints_nothing():
    import bench

    class Args:
        steps, warmup = 1, 0

    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference_batch(Args(), 1, 2)
    assert buf.getvalue() == ""
