"""The autotuner's host logic (CPU): candidate lists, keys, choice of the fastest setting,
the JSON cache, and the library's validation of tuning settings. A fake timer stands in
for the CUDA-event timing of a step."""

import json

import pytest

from srf_b200 import _lib, tuning


def test_candidates():
    assert tuning.candidates(16) == [(1, 0, 0), (1, 0, 1), (1, 0, 2), (1, 8, 0), (1, 8, 1),
                                     (1, 8, 2), (3, 0, 1), (2, 0, 1)]
    assert tuning.candidates(1) == [(1, 0, 0), (1, 0, 1), (1, 0, 2), (3, 0, 1), (2, 0, 1)]


def test_automatic_multiplier_competes_and_wins_ties(recorder):
    # the automatic grid multiplier (0) is timed like any fixed one and, being first,
    # is kept when a fixed multiplier only ties it
    cands = tuning.candidates(6)
    ms = {c: 5.0 for c in cands}
    ms[(1, 0, 1)] = ms[(1, 0, 0)] = 4.0

    def tune(key):
        timer = FakeTimer(ms)

        def step():
            timer.current = recorder[-1]
        return tuning.Autotuner(timer=timer).tune(key, step, cands)

    best, timings = tune("k")
    assert (1, 0, 0) in timings and best == (1, 0, 0)
    ms[(1, 3, 0)] = 3.0  # the automatic multiplier at half-depth slabs, strictly faster
    best, _ = tune("k2")
    assert best == (1, 3, 0) and recorder[-1] == best


def test_key_buckets():
    k = tuning.key_for([96, 48, 96], 6, 4_500_000, 64)
    assert k == "g96x48x96_p6_n2^22_f64"
    assert tuning.key_for([8, 8, 8], 3, 0) == "g8x8x8_p3_n2^0_f1"
    assert tuning.key_for([8, 8, 8], 3, 1023) != tuning.key_for([8, 8, 8], 3, 1024)


class FakeTimer:
    """Returns a fixed time per setting: the setting applied last by tune()."""

    def __init__(self, ms):
        self.ms, self.calls, self.current = ms, 0, None

    def __call__(self, step, warmup, reps):
        self.calls += 1
        step()
        return self.ms[self.current]


@pytest.fixture
def recorder(monkeypatch):
    applied = []
    real = tuning.set_tuning

    def rec(*c):
        applied.append(tuple(c))
        return real(*c)
    monkeypatch.setattr(tuning, "set_tuning", rec)
    yield applied
    real()


def test_tune_picks_fastest_and_caches(tmp_path, recorder):
    cands = [(1, 0, 1), (1, 0, 2), (2, 0, 1)]
    timer = FakeTimer({(1, 0, 1): 3.0, (1, 0, 2): 2.0, (2, 0, 1): 9.0})
    steps = []

    def step():
        timer.current = recorder[-1]
        steps.append(timer.current)

    cache = tmp_path / "tune.json"
    t = tuning.Autotuner(str(cache), timer=timer)
    best, timings = t.tune("k", step, cands)
    assert best == (1, 0, 2)
    assert timings == {(1, 0, 1): 3.0, (1, 0, 2): 2.0, (2, 0, 1): 9.0}
    assert steps == cands and recorder[-1] == best  # every candidate ran, best applied
    assert json.loads(cache.read_text()) == {"k": [1, 0, 2]}

    # a second tuner reads the cache: the best is applied without timing anything
    t2 = tuning.Autotuner(str(cache), timer=FakeTimer({}))
    best2, timings2 = t2.tune("k", step, cands)
    assert best2 == (1, 0, 2) and timings2 is None and t2.timer.calls == 0
    assert recorder[-1] == (1, 0, 2)


def test_invalid_settings_rejected():
    for bad in [(4, 0, 1), (-1, 0, 1), (1, -1, 1), (1, 0, -1), (1, 0, 9)]:
        with pytest.raises(_lib.SRFError):
            tuning.set_tuning(*bad)
    tuning.set_tuning(1, 0, 0)  # grid multiplier 0: automatic
    tuning.set_tuning()
