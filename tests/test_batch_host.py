"""Host logic of the batched solve's autotuner (no GPU): candidate selection and the JSON
cache, with a stand-in runner in place of the GPU timing."""
import json

from blockpowerflow_b200 import batch


class _Mat:
    def __init__(self, n):
        self.n = n


def test_pick_best_prefers_converged_candidates():
    t = {(8, 2): (0.5, True), (16, 2): (0.3, False), (32, 1): (0.4, True)}
    assert batch.pick_best(t) == (32, 1)
    assert batch.pick_best({(8, 1): (0.2, False), (16, 1): (0.1, False)}) == (16, 1)


def test_autotune_runs_every_candidate_then_uses_the_cache(tmp_path):
    calls = []

    def runner(slice_, cps):
        calls.append((slice_, cps))
        return {8: 0.30, 16: 0.20, 32: 0.25}[slice_] + (0.01 if cps == 1 else 0.0), True

    mats = [_Mat(500), _Mat(1200)]
    path = str(tmp_path / "tune.json")
    r = batch.autotune(mats, [8, 40], None, cache_path=path, runner=runner, device_name="dev")
    assert (r["slice"], r["ctas_per_sm"]) == (16, 1) and not r["cached"]
    assert sorted(calls) == sorted(batch.CANDIDATES)
    data = json.load(open(path))
    assert len(data) == 1 and list(data.values())[0]["slice"] == 16
    calls.clear()
    r2 = batch.autotune(mats, [8, 40], None, cache_path=path, runner=runner, device_name="dev")
    assert r2["cached"] and r2["slice"] == 16 and calls == []
    # another batch shape or device is a different key
    r3 = batch.autotune(mats, [8, 41], None, cache_path=path, runner=runner, device_name="dev")
    assert not r3["cached"]
    r4 = batch.autotune(mats, [8, 40], None, cache_path=path, runner=runner, device_name="other")
    assert not r4["cached"]
    assert len(json.load(open(path))) == 3


def test_batch_key_depends_on_sizes_widths_device_and_options():
    k = batch.batch_key([10, 20], [3, 4], "d", "x")
    assert k == batch.batch_key([10, 20], [3, 4], "d", "x")
    assert k != batch.batch_key([10, 21], [3, 4], "d", "x")
    assert k != batch.batch_key([10, 20], [3, 5], "d", "x")
    assert k != batch.batch_key([10, 20], [3, 4], "e", "x")
    assert k != batch.batch_key([10, 20], [3, 4], "d", "y")


def test_corrupt_cache_is_ignored(tmp_path):
    path = tmp_path / "tune.json"
    path.write_text("{not json")
    assert batch.load_cache(str(path)) == {}
    r = batch.autotune([_Mat(100)], [4], None, cache_path=str(path), runner=lambda s, c: (1.0 / s, True),
                       device_name="dev", candidates=[(8, 1), (32, 2)])
    assert (r["slice"], r["ctas_per_sm"]) == (32, 2)
