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
    t3 = {(32, 1, "AMD"): (0.7, True), (32, 1, "RCM"): (0.5, True), (16, 1, "RCM"): (0.4, False)}
    assert batch.pick_best(t3) == (32, 1, "RCM")


def test_candidates_cover_slices_and_both_fill_reducing_orders():
    assert sorted({c[0] for c in batch.CANDIDATES}) == [8, 16, 32]
    assert {c[2] for c in batch.CANDIDATES} == {"AMD", "RCM"}
    assert len(set(batch.CANDIDATES)) == 6


def test_autotune_runs_every_candidate_then_uses_the_cache(tmp_path):
    calls = []

    def runner(slice_, cps, ordering):
        calls.append((slice_, cps, ordering))
        t = {8: 0.30, 16: 0.20, 32: 0.25}[slice_] + (0.01 if cps == 1 else 0.0)
        return t * (0.9 if (ordering == "RCM" and slice_ == 32) else 1.0), True

    mats = [_Mat(500), _Mat(1200)]
    path = str(tmp_path / "tune.json")
    r = batch.autotune(mats, [8, 40], None, cache_path=path, runner=runner, device_name="dev")
    assert (r["slice"], r["ctas_per_sm"], r["ordering"]) == (16, 1, "AMD") and not r["cached"]
    assert sorted(calls) == sorted(batch.CANDIDATES)
    assert set(r["timings"]) == {f"{s}x{c}x{o}" for s, c, o in batch.CANDIDATES}
    data = json.load(open(path))
    assert len(data) == 1 and list(data.values())[0]["slice"] == 16
    calls.clear()
    r2 = batch.autotune(mats, [8, 40], None, cache_path=path, runner=runner, device_name="dev")
    assert r2["cached"] and r2["slice"] == 16 and r2["ordering"] == "AMD" and calls == []
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
    r = batch.autotune([_Mat(100)], [4], None, cache_path=str(path), runner=lambda s, c, o: (1.0 / s, True),
                       device_name="dev", candidates=[(8, 1), (32, 2)])
    assert (r["slice"], r["ctas_per_sm"]) == (32, 2)


def test_ordering_is_tuned_when_it_is_faster(tmp_path):
    """A faster order wins, the plan's own ordering fills pairs, and the choice is cached."""
    def runner(slice_, cps, ordering):
        return {"AMD": 0.7, "RCM": 0.5, "NATURAL": 1.0}[ordering] * (32 / slice_) ** 0.1, True

    path = str(tmp_path / "tune.json")
    r = batch.autotune([_Mat(300), _Mat(900)], [9, 33], None, cache_path=path, runner=runner, device_name="dev")
    assert (r["slice"], r["ordering"]) == (32, "RCM")
    assert batch.autotune([_Mat(300), _Mat(900)], [9, 33], None, cache_path=path, runner=runner,
                          device_name="dev")["ordering"] == "RCM"
    seen = []
    r2 = batch.autotune([_Mat(300)], [9], None, runner=lambda s, c, o: (seen.append(o) or 1.0, True),
                        device_name="dev", candidates=[(16, 1), (32, 1)], ordering=":NATURAL")
    assert seen == ["NATURAL", "NATURAL"] and r2["ordering"] == "NATURAL"


def test_split_longest_halves_the_systems_on_the_critical_path():
    sys_, q, cyc = [0, 0, 1, 2], [16, 16, 9, 32], [100, 90, 400, 50]
    # balanced bound 640 / 2 = 320: only system 1's unit (400) is above 0.9 x 320
    assert batch.split_longest(sys_, q, cyc, 2, [0, 0, 0]) == [0, 5, 0]
    # a lower bound (more CTAs) takes more systems; widths only ever shrink
    assert batch.split_longest(sys_, q, cyc, 8, [0, 0, 0]) == [8, 5, 0]
    assert batch.split_longest(sys_, q, cyc, 8, [4, 0, 0]) == [4, 5, 0]
    # nothing above the bound, or only single-column units: no new plan
    assert batch.split_longest([0, 1], [8, 8], [10, 10], 1, [0, 0]) is None
    assert batch.split_longest([0, 1], [1, 8], [100, 1], 2, [0, 0]) is None


def test_autotune_keeps_a_refinement_only_while_it_pays(tmp_path):
    calls = []

    def runner(slice_, cps, ordering, slices=None):
        calls.append((slice_, ordering, None if slices is None else tuple(slices)))
        units = {"sys": [0, 1, 2], "q": [slice_, 9, slice_], "cycles": [10, 100, 10], "grid": 2}
        if slices is None:
            return (1.0 if slice_ == 32 else 2.0), True, units
        if slices[1] == 5:     # first round: system 1 split, faster; still the longest
            return 0.8, True, {"sys": [0, 1, 1, 2], "q": [32, 5, 4, 32], "cycles": [10, 70, 65, 10], "grid": 2}
        return 0.8, True, units   # second round (system 1 at width 3): no gain

    path = str(tmp_path / "tune.json")
    r = batch.autotune([_Mat(300), _Mat(5000), _Mat(900)], [32, 9, 32], None, cache_path=path, runner=runner,
                       device_name="dev", candidates=[(16, 1, "RCM"), (32, 1, "RCM")])
    assert (r["slice"], r["ordering"]) == (32, "RCM")
    assert r["slices"] == [0, 5, 0]
    assert [x["kept"] for x in r["refinement"]] == [True, False]
    assert calls[-1] == (32, "RCM", (0, 3, 0))
    r2 = batch.autotune([_Mat(300), _Mat(5000), _Mat(900)], [32, 9, 32], None, cache_path=path, runner=runner,
                        device_name="dev", candidates=[(16, 1, "RCM"), (32, 1, "RCM")])
    assert r2["cached"] and r2["slices"] == [0, 5, 0]
    # a refinement whose solve does not converge is not kept
    r3 = batch.autotune([_Mat(300), _Mat(5000), _Mat(900)], [32, 9, 32], None, device_name="dev",
                        candidates=[(32, 1, "RCM")],
                        runner=lambda s, c, o, slices=None: (1.0 if slices is None else 0.5, slices is None,
                                                             {"sys": [0, 1, 2], "q": [32, 9, 32],
                                                              "cycles": [1, 100, 1], "grid": 2}))
    assert r3["slices"] is None and r3["refinement"][0]["kept"] is False


def test_cache_key_can_be_rebuilt_by_a_reader(tmp_path):
    """A process that only reads the cache (no timing launches) finds the default run's entry."""
    path = str(tmp_path / "tune.json")
    mats = [_Mat(700), _Mat(1900)]
    batch.autotune(mats, [12, 50], None, cache_path=path, device_name="dev",
                   runner=lambda s, c, o, slices=None: (1.0 / s, True))
    key = batch.batch_key([700, 1900], [12, 50], "dev", batch.cache_extra(batch.CANDIDATES, "AMD"))
    assert list(json.load(open(path))) == [key]
    assert batch.load_cache(path)[key]["slice"] == 32 and batch.load_cache(path)[key]["slices"] is None
