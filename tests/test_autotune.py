"""The launch-shape autotuner's selection rule (binder_b200/autotune.py), on CPU: a stand-in batch
whose EM timing depends on the configuration applied to its registrations, so the rule itself --
the fastest of two timings per candidate, the default kept unless another candidate is at least
3% faster, one choice per size class, the JSON cache -- is checked without a GPU."""
import json

import pytest

from binder_b200 import autotune


class _Reg:
    def __init__(self):
        self.cfg = (0, 3)

    def set_estep_grid(self, ctas):
        self.cfg = (ctas, self.cfg[1])

    def set_precision(self, p):
        self.cfg = (self.cfg[0], p)

    def reset(self):
        pass


def _core(ms_per_iteration, jitter=None):
    calls = []

    class Batch:
        def __init__(self, regs):
            self.regs = regs
            self.last_ms = None

        def EM(self, iterations, th, update):
            calls.append(self.regs[0].cfg)
            extra = jitter(len(calls)) if jitter else 0.0
            self.last_ms = (ms_per_iteration[self.regs[0].cfg] + extra) * iterations

    class Core:
        RegistrationBatch = Batch

    return Core, calls


def _times(default, others):
    t = {(c["estep_ctas"], c["precision"]): others for c in autotune.CANDIDATES}
    t[(0, 3)] = default
    return t


def test_clear_winner_is_chosen_and_cached(tmp_path):
    t = _times(1.0, 1.2)
    t[(74, 1)] = 0.8
    core, _ = _core(t)
    regs = [_Reg() for _ in range(4)]
    cache = str(tmp_path / "tune.json")
    table = autotune.tune(core, regs, [(64, 64, 64)] * 2 + [(128, 128, 128)] * 2, cache=cache,
                          retune=True)
    assert set(table) == {"small", "large"}
    for cls in table.values():
        assert (cls["estep_ctas"], cls["precision"]) == (74, 1)
        assert cls["ms_per_iteration"] == pytest.approx(0.8)
    assert all(r.cfg == (74, 1) for r in regs)
    assert json.load(open(cache)) == table
    # a second call reads the cache and times nothing
    core2, calls = _core(_times(1.0, 0.5))
    assert autotune.tune(core2, regs, [(64, 64, 64)] * 4, cache=cache) == table
    assert calls == []


def test_default_kept_within_the_margin():
    t = _times(1.0, 1.1)
    t[(148, 3)] = 1.0 - autotune.MARGIN / 2  # faster, but by less than the margin
    core, _ = _core(t)
    regs = [_Reg() for _ in range(3)]
    table = autotune.tune(core, regs, [(48, 48, 48)] * 3)
    assert (table["small"]["estep_ctas"], table["small"]["precision"]) == (0, 3)
    assert all(r.cfg == (0, 3) for r in regs)


def test_the_faster_of_two_timings_counts():
    """one slow outlier timing of the default does not hand the choice to another candidate"""
    t = _times(1.0, 0.99)
    # the first timed run of the default (the second EM call: the first is the warm-up) is slow
    core, _ = _core(t, jitter=lambda n: 5.0 if n == 2 else 0.0)
    regs = [_Reg() for _ in range(2)]
    table = autotune.tune(core, regs, [(40, 40, 40)] * 2)
    assert (table["small"]["estep_ctas"], table["small"]["precision"]) == (0, 3)
    assert table["small"]["ms_per_iteration"] == pytest.approx(1.0)
