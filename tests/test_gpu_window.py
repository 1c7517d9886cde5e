"""GPU parity of the single-window sweep (csrc/sweep_window.cu): run_rewl (src/parallel.cpp:276-747)
with one energy window on small dense systems, many epochs per launch, bit for bit against the
oracle and against the engine's per-epoch kernels: 1/t convergence, the attempt limit, the
traditional freeze, forced acceptance, power-of-two and other bin widths, 1 to 4 walkers, 1 to 32
sites; runs split across launches and across the two kernels; which engines are eligible."""
from __future__ import annotations

import pytest

from helpers import random_axes, results_equal, snapshots_equal
from replica_exchange_wang_landau_b200.engine import Engine, Geometry, RunConfig, System, run_rewl

pytestmark = pytest.mark.gpu


def _system(dims, seed=None, periodic=False, box=None):
    g = Geometry.simple_cubic(*dims, 1.0, (0.0, 0.0, 1.0), periodic)
    if seed is not None:
        g.axes = random_axes(g.size(), seed)
    if box:
        g.box = box
    return System(g, 1.0, 0.0)


RUNS = {
    # the N = 8 reference configuration (2x2x2 open, +z axes, [-20, 20] in bins of 0.25, 2
    # walkers, exchange interval and check interval at their defaults), 1/t to ln f <= 1e-5
    "n8_converge": (lambda: _system((2, 2, 2)),
                    dict(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=2, seed=1234),
                    dict(final_factor=1e-5)),
    # 27 spins, periodic, random axes, bins of 0.75 (not a power of two), 3 walkers, attempt limit
    "n27_width075_limit": (lambda: _system((3, 3, 3), 5, True),
                           dict(emin=-60, emax=60, bin_width=0.75, windows=1, walkers=3, seed=7, max_mcs=3000,
                                exchange_interval_mcs=1, check_interval_mcs=7), dict(final_factor=1e-6)),
    # 32 sites (ld 32), slab box, 4 walkers, exchange every MCS, check every 3 MCS, to 1e-3
    "n32_four_walkers": (lambda: _system((4, 4, 2), 9, True, box=(4.0, 4.0, 0.0)),
                         dict(emin=-80, emax=80, bin_width=0.5, windows=1, walkers=4, seed=11, max_mcs=20000,
                              exchange_interval_mcs=1, check_interval_mcs=3), dict(final_factor=1e-3)),
    # 12 sites (ld 16), traditional Wang-Landau: flatness 0.6, halving to 1e-3
    "n12_traditional": (lambda: _system((3, 2, 2), 3),
                        dict(emin=-30, emax=30, bin_width=0.5, windows=1, walkers=2, seed=5, max_mcs=40000,
                             exchange_interval_mcs=2, check_interval_mcs=4),
                        dict(inverse_time_enabled=False, flatness=0.6, minimum_visits=20, final_factor=1e-3)),
    # forced acceptance after half an MCS without a flip, one walker, attempt limit
    "n12_forced": (lambda: _system((3, 2, 2), 4),
                   dict(emin=-30, emax=30, bin_width=0.25, windows=1, walkers=1, seed=3, max_mcs=4000,
                        exchange_interval_mcs=1, force_accept_after_mcs=0.5), dict(final_factor=1e-6)),
    # 17 sites in a 32-wide padded row, a narrow window that cuts the energy range
    "n17_narrow": (lambda: _system((17, 1, 1), 6, False),
                   dict(emin=-10, emax=6, bin_width=0.25, windows=1, walkers=2, seed=13, max_mcs=5000,
                        exchange_interval_mcs=3, check_interval_mcs=6), dict(final_factor=1e-5)),
    # one spin
    "n1": (lambda: _system((1, 1, 1)),
           dict(emin=-1, emax=1, bin_width=0.5, windows=1, walkers=2, seed=2, max_mcs=500, exchange_interval_mcs=1),
           dict()),
}


def _config(kw, wl):
    c = RunConfig(**kw)
    for k, val in wl.items():
        setattr(c.wl, k, val)
    return c


@pytest.mark.parametrize("name", list(RUNS))
def test_window_run_rewl_bitwise(oracle, name):
    make_system, kw, wl = RUNS[name]
    s = make_system()
    c = _config(kw, wl)
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        assert e.window_sweep
        e.run()
        got = e.result()
    assert got.attempted > 0
    assert results_equal(got, oracle.run_rewl(s, c)) == []
    with Engine(s, c) as e:  # the per-epoch kernels give the same run
        e.window_sweep = False
        assert not e.window_sweep
        e.run()
        assert results_equal(got, e.result()) == []


def test_window_run_split_across_launches_and_kernels():
    """A run advanced in uneven pieces, alternating between the single-window kernel and the
    per-epoch kernels, equals the run made in one go: the walker state, the generator (stepped
    back over unconsumed draws) and the epoch counter are handed over exactly."""
    s = _system((3, 3, 3), 21, True)
    c = _config(dict(emin=-60, emax=60, bin_width=0.5, windows=1, walkers=3, seed=17, exchange_interval_mcs=1,
                     check_interval_mcs=5, max_mcs=800), dict(final_factor=1e-4))
    c.resolve_mcs(s.size())
    whole = run_rewl(s, c)
    with Engine(s, c) as e:
        done, k = False, 0
        while not done:
            e.window_sweep = k % 2 == 0
            ran, done = e.run_epochs(1 + (37 * k) % 101)
            k += 1
        pieces = e.result()
    assert k > 4
    assert results_equal(whole, pieces) == []


def test_window_trajectory_matches_single_walker_steps(oracle):
    """After epochs of the single-window kernel every walker's snapshot (spins, fields, energy,
    log g, H, counters, generator) equals the oracle walker's after the same attempts."""
    s = _system((2, 2, 2), 8)
    c = _config(dict(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=2, seed=99, exchange_interval_mcs=4,
                     check_interval_mcs=1000), dict())
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        walkers = [oracle.walker(s, w, c.emin, c.emax, c.bin_width, e.window(0), c.wl, c.seed) for w in range(2)]
        ran, done = e.run_epochs(25)
        assert ran == 25 and not done
        for w, ow in enumerate(walkers):
            ow.run_attempts(25 * c.exchange_interval_attempts)
            assert snapshots_equal(e.snapshot(w), ow.snapshot()) == [], f"walker {w}"


@pytest.mark.parametrize("change", ["two_windows", "33_sites", "five_walkers", "pilot", "nalivaiko", "fp32", "csr"])
def test_window_sweep_eligibility(change):
    dims, kw, wl, precision, cutoff = (2, 2, 2), dict(windows=1, walkers=2), {}, "fp64", 0.0
    if change == "two_windows":
        kw["windows"] = 2
    elif change == "33_sites":
        dims = (11, 3, 1)
    elif change == "five_walkers":
        kw["walkers"] = 5
    elif change == "pilot":
        wl["collect_window_statistics"] = True
    elif change == "nalivaiko":
        wl.update(nalivaiko_mod=True, inverse_time_enabled=False)
    elif change == "fp32":
        precision = "fp32"
    elif change == "csr":
        cutoff = 1.5
    g = Geometry.simple_cubic(*dims, 1.0, (0.0, 0.0, 1.0), False)
    s = System(g, 1.0, cutoff)
    c = _config(dict(emin=-40, emax=40, bin_width=0.25, seed=1, **kw), wl)
    c.coupling_precision = precision
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        assert not e.window_sweep
        e.window_sweep = True  # no effect on an engine that does not qualify
        assert not e.window_sweep
    base = _config(dict(emin=-40, emax=40, bin_width=0.25, seed=1, windows=1, walkers=2), {})
    base.resolve_mcs(8)
    with Engine(System(Geometry.simple_cubic(2, 2, 2, 1.0, (0.0, 0.0, 1.0), False)), base) as e:
        assert e.window_sweep
