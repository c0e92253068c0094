"""The skin autotuner's bookkeeping (cellsim3d_b200/autotune.py), on a stand-in
for the simulation: population ranges, the fastest skin per range, the
schedule, failures and the same-trajectory check.  No GPU."""
import json

import pytest

from cellsim3d_b200 import OPT_SKIN
from cellsim3d_b200 import autotune as A


class FakeSim:
    """Cells double every 10 steps from 1; a step costs ms_of(skin, n) ms.
    A skin in fail_at stops with a status once the population reaches the
    given count."""

    def __init__(self, ms_of, fail_at=None, drift=None):
        self.ms_of, self.fail_at, self.drift = ms_of, fail_at or {}, drift
        self.skin, self.k, self.last = None, 0, 0.0

    def set_option(self, opt, value):
        assert opt == OPT_SKIN
        self.skin = value * 1e-6

    def n_cells(self):
        n = 2 ** (self.k // 10)
        if self.drift is not None and self.skin is not None and abs(self.skin - self.drift) < 1e-9 and self.k >= 30:
            n += 1
        return n

    def step(self, m, raise_on_error=True):
        n = self.n_cells()
        lim = self.fail_at.get(round(self.skin, 6))
        if lim is not None and n >= lim:
            return 5
        self.last = m * self.ms_of(self.skin, n)
        self.k += m
        return 0

    def last_step_ms(self):
        return self.last

    def close(self):
        pass


def _ms(skin, n):
    # small populations prefer the small skin, large ones the large skin
    return (1.0 + skin) if n < 100 else (2.0 - skin)


def test_range_of():
    b = (1, 10, 100, 1000)
    assert [A.range_of(n, b) for n in (0, 1, 9, 10, 99, 100, 5000)] == [0, 0, 0, 1, 1, 2, 3]


def test_fastest_skin_per_range_and_schedule():
    res = A.tune(lambda: FakeSim(_ms), steps=120, skins=(0.05, 0.1, 0.13), bounds=(1, 10, 100, 1000), chunk=10)
    assert res.best() == {0: 0.05, 1: 0.05, 2: 0.13, 3: 0.13}
    assert res.schedule() == ([1, 100], [0.05, 0.13])
    # the same steps of each range for every skin
    for r in range(4):
        assert len({res.steps[(r, s)] for s in res.skins}) == 1
    d = json.loads(res.to_json())
    assert d["min_cells"] == [1, 100] and d["skins"] == [0.05, 0.13]
    assert d["table"]["100"]["0.13"]["steps"] == res.steps[(2, 0.13)]


def test_a_failing_skin_is_dropped_from_its_range_on():
    res = A.tune(lambda: FakeSim(_ms, fail_at={0.13: 200}), steps=120, skins=(0.05, 0.1, 0.13),
                 bounds=(1, 10, 100, 1000), chunk=10)
    assert res.failed[0.13]["range"] == 2
    assert all(s != 0.13 for (r, s) in res.ms if r >= 2)
    assert res.best()[2] == 0.1 and res.best()[3] == 0.1


def test_runs_that_leave_the_trajectory_are_an_error():
    with pytest.raises(RuntimeError, match="cells at step"):
        A.tune(lambda: FakeSim(_ms, drift=0.1), steps=60, skins=(0.05, 0.1), bounds=(1, 10), chunk=10)


def test_schedule_file_round_trip(tmp_path):
    res = A.tune(lambda: FakeSim(_ms), steps=120, skins=(0.05, 0.13), bounds=(1, 10, 100), chunk=10)
    p = tmp_path / "s.json"
    p.write_text(res.to_json())
    assert A.load_schedule(str(p)) == res.schedule()
