"""The launch-shape autotuner's search and cache on CPU, with a stand-in
batch whose device time is a known function of the three choices: the
coordinate search from the heuristic must reach the fastest choice along the
axes, never report worse than the heuristic, record it under the batch's size
class and device, and set it again on another batch of that class (but not
of another class)."""
import importlib
import json

import pytest


@pytest.fixture(scope="module")
def A():
    return importlib.import_module("lcurve-rs_b200.autotune")


class FakeBatch:
    """Device time = a bowl with its minimum at (chunks 4, split 8, blocks 3)."""

    HEURISTIC = dict(flux_chunks=2, roche_split=2, flux_blocks_per_sm=5)

    def __init__(self, models=1024, evals=4.2e11, roche=1.5e7):
        self._stats = dict(models=models, element_evals=int(evals), roche_elements=int(roche))
        self.t = dict(self.HEURISTIC)
        self.runs = 0

    def set_tuning(self, flux_chunks=0, roche_split=0, flux_blocks_per_sm=0):
        self.t = dict(flux_chunks=flux_chunks or self.HEURISTIC["flux_chunks"],
                      roche_split=roche_split or self.HEURISTIC["roche_split"],
                      flux_blocks_per_sm=flux_blocks_per_sm or self.HEURISTIC["flux_blocks_per_sm"])

    def tuning(self):
        return dict(self.t)

    def stats(self):
        return dict(self._stats)

    def run(self, scale=False):
        self.runs += 1

    def profile(self, scale=False):
        c, s, b = self.t["flux_chunks"], self.t["roche_split"], self.t["flux_blocks_per_sm"]
        flux = 100.0 + 3.0 * abs(c - 4) + 2.0 * abs(b - 3)
        roche = 300.0 + 5.0 * abs(s - 8)
        return dict(phase=0.1, elements=20.0, roche=roche, aux=5.0, flux=flux, epilogue=0.2)


def test_search_reaches_the_fastest_choice_and_caches_it(A, tmp_path):
    cache = tmp_path / "tune.json"
    b = FakeBatch()
    r = A.autotune(b, cache=cache, device_name="B200")
    assert (r["flux_chunks"], r["roche_split"], r["flux_blocks_per_sm"]) == (4, 8, 3)
    assert b.tuning() == dict(flux_chunks=4, roche_split=8, flux_blocks_per_sm=3)
    assert r["ms"] <= r["heuristic_ms"] and r["ms"] == pytest.approx(425.3)
    table = json.loads(cache.read_text())
    assert table["B200"][r["class"]] == dict(flux_chunks=4, roche_split=8, flux_blocks_per_sm=3)
    # another batch of the same class takes the recorded choice; another class does not
    same = FakeBatch(models=1000, evals=4.0e11, roche=1.6e7)
    assert A.apply_cached(same, cache, device_name="B200") and same.tuning()["roche_split"] == 8
    other = FakeBatch(models=16)
    assert not A.apply_cached(other, cache, device_name="B200") and other.tuning() == FakeBatch.HEURISTIC
    assert not A.apply_cached(FakeBatch(), cache, device_name="other-gpu")


def test_batches_without_roche_elements_skip_that_axis(A):
    b = FakeBatch(roche=0)
    seen = []
    orig = b.set_tuning

    def spy(*args):
        seen.append(args)
        orig(*args)
    b.set_tuning = spy
    A.autotune(b)
    assert all(args[1] in (0, FakeBatch.HEURISTIC["roche_split"]) for args in seen)


def test_unsearched_axis_is_cached_as_the_heuristic(A, tmp_path):
    # a batch without Roche-eclipsed elements never times the scan split: the cache keeps 0
    # (the planner's heuristic) for it, so the choice cannot pin a later batch that has them
    cache = tmp_path / "tune.json"
    A.autotune(FakeBatch(roche=0), cache=cache, device_name="B200")
    (choice,) = json.loads(cache.read_text())["B200"].values()
    assert choice["roche_split"] == 0
    later = FakeBatch(roche=0)
    later.t["roche_split"] = 16
    assert A.apply_cached(later, cache, device_name="B200")
    assert later.tuning()["roche_split"] == FakeBatch.HEURISTIC["roche_split"]
