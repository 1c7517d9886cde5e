"""The bounded device waits run out cleanly.

Every wait inside the sweep kernels is bounded: a walker that waits for draws longer than its
poll limit records WLG_ERR_TIMEOUT, leaves its state unwritten and returns, and the host reads
the status after the launch.  These tests make the wait run out without any fault: the
engine's failure-injection hook stops the draw-producer warps from publishing anything, so
the walkers' waits for their first draws can only end at their limits.  The run call must
then fail with WLG_ERR_TIMEOUT within seconds, and a fresh engine on the same device must
still run bit for bit like the oracle.
"""
from __future__ import annotations

import time

import pytest

from helpers import random_axes, results_equal, snapshots_equal
from replica_exchange_wang_landau_b200.engine import DeviceError, Engine, Geometry, RunConfig, System, run_rewl

pytestmark = pytest.mark.gpu


def _c1():
    s = System(Geometry.simple_cubic(2, 2, 2, periodic=False))
    c = RunConfig(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=2, seed=1234)
    c.wl.final_factor = 1e-3
    c.resolve_mcs(8)
    return s, c


def _fresh_engine_is_bit_exact(oracle):
    s, c = _c1()
    got, want = run_rewl(s, c), oracle.run_rewl(s, c)
    assert got.converged and results_equal(got, want) == []


def test_split_sweep_wait_runs_out(oracle):
    g = Geometry.simple_cubic(3, 3, 3, periodic=True)
    g.axes = random_axes(27, 11)
    s = System(g)
    c = RunConfig(emin=-60, emax=60, bin_width=0.5, windows=2, walkers=2, seed=21, exchange_interval_mcs=1)
    c.resolve_mcs(27)
    with Engine(s, c) as e:
        e.run_epochs(2)  # ordinary epochs first
        before = [e.snapshot(w) for w in range(e.walkers)]
        e.inject_wait_timeout()
        t0 = time.perf_counter()
        with pytest.raises(DeviceError) as err:
            e.run_epochs(4)
        elapsed = time.perf_counter() - t0
    assert err.value.status == "WLG_ERR_TIMEOUT", str(err.value)
    assert "bounded device wait" in str(err.value)
    assert elapsed < 120.0
    assert all(b.attempted == 2 * c.exchange_interval_attempts for b in before)
    _fresh_engine_is_bit_exact(oracle)


def test_single_window_sweep_wait_runs_out(oracle):
    s, c = _c1()
    with Engine(s, c) as e:
        assert e.window_sweep
        before = [e.snapshot(w) for w in range(e.walkers)]
        e.inject_wait_timeout()
        t0 = time.perf_counter()
        with pytest.raises(DeviceError) as err:
            e.run()
        elapsed = time.perf_counter() - t0
        after = [e.snapshot(w) for w in range(e.walkers)]
    assert err.value.status == "WLG_ERR_TIMEOUT", str(err.value)
    assert elapsed < 120.0
    assert all(snapshots_equal(a, b) == [] for a, b in zip(after, before))  # nothing was written back
    _fresh_engine_is_bit_exact(oracle)
