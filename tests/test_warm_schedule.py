"""The warm start that continues the 1/t schedule, on the oracle's restatement (CPU).

After a warm start at ln f = f0 the reference's rule (src/wang_landau.cpp:389-409) switches to
the 1/t stage at the first covered check with f = active / attempted, which early in a run is
far above f0: the small factor of the warm start is thrown away.  Continuing the schedule, the
check halves f0 and enters the 1/t stage at once, counting round(active / f) - attempted
attempts as already made, so f = active / (attempted + offset) starts at f0 / 2 and then falls
as 1/t, rising only when a new bin raises the active count.
No reference counterpart; the restatement defines it.
"""
from __future__ import annotations

import numpy as np

from replica_exchange_wang_landau_b200.engine import Geometry, RunConfig, System, WlParameters


def _walker(oracle, continue_schedule):
    s = System(Geometry.simple_cubic(2, 2, 2, periodic=False))
    p = WlParameters(0.8, 100, 1e-8, 800, 0, True)
    w = oracle.walker(s, 0, -20.0, 20.0, 0.25, (0, 160), p, 1234)
    w.warm_start(np.zeros(160), 1e-3, continue_schedule)
    return w


def test_reference_rule_discards_the_warm_start(oracle):
    w = _walker(oracle, False)
    w.run_attempts(800)
    assert w.flags()[2]  # covered: ready for the next iteration
    w.begin_next_iteration()
    snap = w.snapshot()
    assert snap.stage == 1 and snap.factor > 1e-2  # active / attempted = 22 / 800


def test_continued_schedule_keeps_the_small_factor(oracle):
    w = _walker(oracle, True)
    w.run_attempts(800)
    w.begin_next_iteration()
    snap = w.snapshot()
    assert snap.stage == 1 and snap.factor == 5e-4  # the halved warm-start factor, now 1/t
    offset = round(22 / 5e-4) - 800  # active / f - attempted
    w.run_attempts(5000)
    snap = w.snapshot()
    assert snap.factor == 22 / (5800 + offset) and snap.factor < 5e-4
