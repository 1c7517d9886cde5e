"""GPU parity: the walker kernels and run_rewl (src/wang_landau.cpp, src/parallel.cpp) through
the C-ABI, bit for bit against the CPU oracle, plus the reference's own scenario tests
(tests/test_main.cpp) run on the engine."""
from __future__ import annotations

import math

import numpy as np
import pytest

from helpers import config_from, random_axes, results_equal, snapshots_equal, system_from, unhex, same_double
from replica_exchange_wang_landau_b200.engine import (Engine, EscapedError, Geometry, InitializationError,
                                                      InvalidArgument, LogicError, RunConfig, System, WlgError,
                                                      WlParameters, run_rewl, write_workers_stat_csv)

pytestmark = pytest.mark.gpu


def _random_system(dims, seed, periodic=True, cutoff=0.0, box=None):
    g = Geometry.simple_cubic(*dims, periodic=periodic)
    g.axes = random_axes(g.size(), seed)
    if box:
        g.box = box
    return System(g, 1.0, cutoff)


def _oracle_walkers(oracle, system, engine, config):
    walkers = []
    for w in range(engine.walkers):
        window = engine.window(w // config.walkers)
        init = None
        if config.initial_spins_by_walker is not None and config.initial_spins_by_walker[w] is not None:
            init = np.asarray(config.initial_spins_by_walker[w], dtype=np.int8)
        walkers.append(oracle.walker(system, w, config.emin, config.emax, config.bin_width, window, config.wl,
                                     config.seed, init))
    return walkers


CASES = {
    # name: (system, config kwargs)
    "open8": (lambda: System(Geometry.simple_cubic(2, 2, 2, periodic=False)),
              dict(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=2, seed=1234)),
    "periodic27_3win": (lambda: _random_system((3, 3, 3), 11),
                        dict(emin=-60, emax=60, bin_width=0.5, windows=3, walkers=2, seed=21)),
    "slab40": (lambda: _random_system((5, 4, 2), 12, box=(5.0, 4.0, 0.0)),
               dict(emin=-80, emax=80, bin_width=0.5, windows=4, walkers=2, seed=5, overlap=0.6)),
    "csr64": (lambda: _random_system((4, 4, 4), 13, cutoff=1.8),
              dict(emin=-150, emax=150, bin_width=0.5, windows=2, walkers=3, seed=9)),
    "dense100": (lambda: _random_system((5, 5, 4), 14),
                 dict(emin=-150, emax=150, bin_width=1.0, windows=2, walkers=2, seed=17)),
    # the headline system size (512 sites: eight 64-field chunks per lane) and 216 sites (four)
    "dense512": (lambda: _random_system((8, 8, 8), 18),
                 dict(emin=-228.5, emax=228.0, bin_width=0.5, windows=3, walkers=2, seed=19)),
    "dense216": (lambda: _random_system((6, 6, 6), 20),
                 dict(emin=-150, emax=150, bin_width=0.75, windows=2, walkers=2, seed=23)),
    "collect": (lambda: _random_system((3, 3, 2), 15),
                dict(emin=-40, emax=40, bin_width=0.5, windows=3, walkers=2, seed=2,
                     wl=WlParameters(collect_window_statistics=True))),
    "nalivaiko": (lambda: _random_system((3, 3, 2), 16),
                  dict(emin=-40, emax=40, bin_width=0.5, windows=2, walkers=2, seed=3,
                       wl=WlParameters(nalivaiko_mod=True, inverse_time_enabled=False, flatness=0.5,
                                       minimum_visits=5))),
}


@pytest.mark.parametrize("name", list(CASES))
def test_walker_trajectories_bitwise(oracle, name):
    make_system, kw = CASES[name]
    s = make_system()
    c = RunConfig(**kw)
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        ow = _oracle_walkers(oracle, s, e, c)
        for w in range(e.walkers):
            assert snapshots_equal(e.snapshot(w), ow[w].snapshot()) == [], f"init of walker {w}"
        for rounds in range(3):
            for w in range(e.walkers):
                e.run_attempts(w, 1537 + 311 * rounds)
                ow[w].run_attempts(1537 + 311 * rounds)
                assert snapshots_equal(e.snapshot(w), ow[w].snapshot()) == [], f"walker {w} round {rounds}"


RUNS = {
    "open8_converge": (lambda: System(Geometry.simple_cubic(2, 2, 2, periodic=False)),
                       dict(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=2, seed=1234),
                       dict(final_factor=1e-3)),
    "periodic27_exchange": (lambda: _random_system((3, 3, 3), 11),
                            dict(emin=-60, emax=60, bin_width=0.5, windows=3, walkers=2, seed=21, max_mcs=200,
                                 exchange_interval_mcs=1, check_interval_mcs=10), dict(final_factor=1e-2)),
    "slab_uneven": (lambda: _random_system((5, 4, 2), 12, box=(5.0, 4.0, 0.0)),
                    dict(emin=-80, emax=80, bin_width=0.5, windows=3, walkers=3, seed=5, max_mcs=100,
                         explicit_windows=[(0, 140), (100, 220), (180, 320)], exchange_interval_mcs=2,
                         check_interval_mcs=4), dict(final_factor=1e-2)),
    "csr_exchange": (lambda: _random_system((4, 4, 4), 13, cutoff=1.8),
                     dict(emin=-150, emax=150, bin_width=0.5, windows=2, walkers=3, seed=9, max_mcs=60,
                          exchange_interval_mcs=1, check_interval_mcs=5), dict(final_factor=1e-2)),
    "collect_pilot": (lambda: _random_system((3, 3, 2), 15),
                      dict(emin=-40, emax=40, bin_width=0.5, windows=3, walkers=2, seed=2, max_mcs=120,
                           exchange_interval_mcs=1, check_interval_mcs=4),
                      dict(collect_window_statistics=True, final_factor=1e-2)),
    "traditional_nalivaiko": (lambda: _random_system((3, 3, 2), 16),
                              dict(emin=-40, emax=40, bin_width=0.5, windows=2, walkers=2, seed=3, max_mcs=300,
                                   exchange_interval_mcs=1, check_interval_mcs=3),
                              dict(nalivaiko_mod=True, inverse_time_enabled=False, flatness=0.5, minimum_visits=5,
                                   final_factor=1e-3)),
    "dense512_exchange": (lambda: _random_system((8, 8, 8), 18),
                          dict(emin=-228.5, emax=228.0, bin_width=0.5, windows=4, walkers=2, seed=29, max_mcs=40,
                               exchange_interval_mcs=1, check_interval_mcs=4), dict(final_factor=1e-2)),
    "dense216_frozen": (lambda: _random_system((6, 6, 6), 20),
                        dict(emin=-150, emax=150, bin_width=0.75, windows=2, walkers=2, seed=31, max_mcs=400,
                             exchange_interval_mcs=1, check_interval_mcs=2),
                        dict(flatness=0.2, minimum_visits=2, final_factor=5e-2, inverse_time_enabled=False)),
    "forced": (lambda: _random_system((3, 2, 2), 17),
               dict(emin=-30, emax=30, bin_width=0.25, windows=2, walkers=2, seed=8, max_mcs=80,
                    exchange_interval_mcs=1, force_accept_after_mcs=0.5), dict(final_factor=1e-2)),
}


@pytest.mark.parametrize("name", list(RUNS))
def test_run_rewl_bitwise(oracle, name):
    make_system, kw, wl = RUNS[name]
    s = make_system()
    c = RunConfig(**kw)
    for k, v in wl.items():
        setattr(c.wl, k, v)
    c.resolve_mcs(s.size())
    got = run_rewl(s, c)
    want = oracle.run_rewl(s, c)
    assert got.attempted > 0
    assert results_equal(got, want) == []


@pytest.mark.parametrize("k", [0, 1])
def test_run_rewl_golden(golden, k):
    case = golden["rewl"][k]
    s = system_from(golden["systems"][case["system"]])
    r = run_rewl(s, config_from(case["config"]))
    g = case["result"]
    for key in ("attempted", "accepted", "forced_accepted", "exchange_attempted", "exchange_accepted", "converged"):
        assert getattr(r, key) == g[key], key
    for f, gf in zip(r.fragments, g["fragments"]):
        assert same_double(f.log_g, unhex(gf["log_g"]))
        assert f.histogram.tolist() == gf["histogram"]
        assert same_double(f.standard_error, unhex(gf["standard_error"]))


def test_rewl_vs_exact_2x2x1(oracle):
    """tests/test_main.cpp:364-397: REWL on 2x2x1, 4 walkers, ln f_final = 1e-3 converges,
    keeps every exact occupied bin, RMSE <= 0.05, and repeats bit for bit."""
    s = System(Geometry.simple_cubic(2, 2, 1, 1.0, (0, 0, 1), False))
    c = RunConfig(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=4, seed=1)
    c.exchange_interval_attempts, c.max_attempts = 1000, 0
    c.exchange_interval_uses_mcs = c.max_limit_uses_mcs = False
    c.wl = WlParameters(0.8, 100, 0.001, 1000, 0, True)
    c.check_interval_uses_mcs = c.force_accept_after_uses_mcs = False
    r = run_rewl(s, c)
    assert r.converged
    counts = oracle.exact_counts(s, -20, 20, 0.25)
    occ = counts > 0
    est = r.fragments[0]
    assert np.all(est.valid[occ] == 1)
    exact = np.log(counts[occ].astype(float))
    offset = np.mean(est.log_g[occ] - exact)
    assert math.sqrt(np.mean((est.log_g[occ] - exact - offset) ** 2)) <= 0.05
    again = run_rewl(s, c)
    assert results_equal(r, again) == []


def test_unlimited_and_blocked_runs(tmp_path):
    """tests/test_main.cpp:282-362 (serial part), the blocked walker's workers-stat CSV row included."""
    one = System(Geometry.simple_cubic(1, 1, 1, 1.0, (0, 0, 1), False))
    c = RunConfig(emin=-1, emax=1, bin_width=0.5, windows=1, walkers=1)
    c.exchange_interval_attempts, c.max_attempts = 1, 0
    c.exchange_interval_uses_mcs = c.max_limit_uses_mcs = False
    c.wl = WlParameters(0.1, 1, 0.5, 1)
    c.check_interval_uses_mcs = c.force_accept_after_uses_mcs = False
    r = run_rewl(one, c)
    assert r.converged and r.attempted > 0 and len(r.walker_statistics) == 1

    scaled = RunConfig(emin=-1, emax=1, bin_width=0.5, windows=1, walkers=2)
    scaled.exchange_interval_attempts, scaled.max_attempts = 1, 1
    scaled.exchange_interval_uses_mcs = scaled.max_limit_uses_mcs = False
    scaled.wl = WlParameters(0.1, 3, 0.5, 1)
    scaled.check_interval_uses_mcs = scaled.force_accept_after_uses_mcs = False
    r = run_rewl(one, scaled)
    assert not r.converged and r.attempted == 2

    two = System(Geometry.simple_cubic(2, 1, 1, 1.0, (0, 0, 1), False))
    b = RunConfig(emin=0.5, emax=1.5, bin_width=0.25, windows=1, walkers=1)
    b.exchange_interval_attempts, b.max_attempts = 1, 5
    b.exchange_interval_uses_mcs = b.max_limit_uses_mcs = False
    b.wl = WlParameters(0.8, 100, 1e-8, 1, inverse_time_enabled=False)
    b.check_interval_uses_mcs = b.force_accept_after_uses_mcs = False
    r = run_rewl(two, b)
    assert not r.converged
    st = r.walker_statistics[0]
    assert (st["attempted"], st["accepted"], st["attempts_since_last_accepted"]) == (5, 0, 5)
    assert st["factor"] == 1.0 and st["active_bins"] == 1 and st["minimum_histogram"] == 6
    assert st["mean_histogram"] == 6.0 and st["min_over_mean"] == 1.0 and st["energy"] == 1.0
    write_workers_stat_csv(tmp_path / "ws.csv", r.walker_statistics, two.size())
    assert (tmp_path / "ws.csv").read_text().split("\n")[1] == "0,0,0,5,2.5,0,0,0,5,2.5,1,1,1,6,6,1,0"


def test_forced_acceptance():
    """tests/test_main.cpp:235-258 on the engine."""
    s = System(Geometry.simple_cubic(2, 1, 1, 1.0, (0, 0, 1), False))
    c = RunConfig(emin=-2, emax=2, bin_width=0.5, windows=1, walkers=5, seed=123)
    c.wl = WlParameters(0.8, 1, 1e-8, 100, 3)
    c.check_interval_uses_mcs = c.force_accept_after_uses_mcs = False
    with Engine(s, c) as e:
        w = 4
        snap = e.snapshot(w)
        from replica_exchange_wang_landau_b200.engine import grid_index
        old = grid_index(-2, 2, 0.5, snap.energy)
        new = grid_index(-2, 2, 0.5, snap.energy + -2.0 * snap.spins[0] * snap.fields[0])
        assert old is not None and new is not None and old != new
        snap.log_g[old], snap.log_g[new] = 0.0, 1000.0
        e.restore(w, snap)
        e.run_attempts(w, 3)
        s3 = e.snapshot(w)
        assert (s3.accepted, s3.forced_accepted, s3.last_accepted_attempt) == (0, 0, 0)
        e.run_attempts(w, 1)
        s4 = e.snapshot(w)
        assert (s4.accepted, s4.forced_accepted, s4.last_accepted_attempt) == (1, 1, 4)


def test_histogram_statistics_and_transitions():
    """tests/test_main.cpp:534-625."""
    one = System(Geometry.simple_cubic(1, 1, 1, 1.0, (0, 0, 1), False))
    c = RunConfig(emin=-1, emax=1, bin_width=0.5, windows=1, walkers=4, seed=11)
    c.wl = WlParameters(0.8, 1, 1e-8, 1)
    c.check_interval_uses_mcs = c.force_accept_after_uses_mcs = False
    with Engine(one, c) as e:
        w = 3
        snap = e.snapshot(w)
        snap.active[:] = 0
        snap.histogram[:] = 0
        snap.active[0] = snap.active[1] = 1
        snap.histogram[0], snap.histogram[1] = 80, 120
        e.restore(w, snap)
        st = e.histogram_statistics(w)
        assert (st["active_bins"], st["covered_bins"], st["minimum"]) == (2, 2, 80)
        assert st["mean"] == 100.0 and abs(st["min_over_mean"] - 0.8) < 1e-14 and st["coverage"] == 1.0
        assert e.flat(w) and e.covered(w)
        snap = e.snapshot(w)
        snap.active[2], snap.histogram[2] = 1, 0
        e.restore(w, snap)
        st = e.histogram_statistics(w)
        assert st["active_bins"] == 3 and st["minimum"] == 0 and st["covered_bins"] == 2
        assert abs(st["mean"] - 200.0 / 3.0) < 1e-14 and abs(st["coverage"] - 2.0 / 3.0) < 1e-14
        assert not e.flat(w) and not e.covered(w)
        snap = e.snapshot(w)
        snap.attempted, snap.active[2] = 1000, 0
        e.restore(w, snap)
        assert e.ready_for_iteration(w)
        e.begin_next_iteration(w)
        assert e.histogram_statistics(w)["active_bins"] == 2
        assert e.snapshot(w).factor == 0.5
        snap = e.snapshot(w)
        snap.stage, snap.factor = 0, 1.0
        snap.active[0] = snap.active[1] = 1
        snap.histogram[0], snap.histogram[1] = 1, 1000
        e.restore(w, snap)
        assert not e.flat(w) and e.covered(w) and e.ready_for_iteration(w)
        snap = e.snapshot(w)
        snap.stage, snap.factor = 1, 0.002
        e.restore(w, snap)
        e.run_attempts(w, 1)
        assert abs(e.snapshot(w).factor - 2.0 / 1001.0) < 1e-14
        e.run_attempts(w, 1)
        assert abs(e.snapshot(w).factor - 3.0 / 1002.0) < 1e-14
        with pytest.raises(LogicError, match="WL iteration is not complete"):
            e.begin_next_iteration(w)


def test_refinement_transition():
    """tests/test_main.cpp:260-280."""
    one = System(Geometry.simple_cubic(1, 1, 1), 1.0)
    for inverse in (True, False):
        c = RunConfig(emin=-1, emax=1, bin_width=0.5, windows=1, walkers=3, seed=9)
        c.wl = WlParameters(0.1, 1, 0.01, 1, inverse_time_enabled=inverse)
        c.check_interval_uses_mcs = c.force_accept_after_uses_mcs = False
        with Engine(one, c) as e:
            w = 1 if inverse else 2
            for _ in range(10):
                if e.snapshot(w).stage != 0:
                    break
                e.run_attempts(w, 10)
                assert e.ready_for_iteration(w)
                e.begin_next_iteration(w)
                if not inverse:
                    assert e.snapshot(w).stage != 1
            assert e.snapshot(w).stage == (1 if inverse else 2) or (inverse and e.snapshot(w).stage == 2)


def test_summary_and_exchange():
    """tests/test_main.cpp:690-774: aligned log-mean, SEM, intersection mask, exchange."""
    one = System(Geometry.simple_cubic(1, 1, 1, 1.0, (0, 0, 1), False))
    c = RunConfig(emin=-1, emax=1, bin_width=0.5, windows=1, walkers=2, seed=17)
    c.wl = WlParameters(0.8, 1, 0.01, 1, 0, False)
    c.check_interval_uses_mcs = c.force_accept_after_uses_mcs = False
    with Engine(one, c) as e:
        a, b = e.snapshot(0), e.snapshot(1)
        for s in (a, b):
            s.active[:] = 0
            s.histogram[:] = 0
        a.active[[0, 1, 2]] = 1
        b.active[[1, 2, 3]] = 1
        a.log_g[1], a.log_g[2] = 10.0, 14.0
        b.log_g[1], b.log_g[2] = -3.0, 3.0
        a.histogram[2], b.histogram[2] = 7, 9
        e.restore(0, a)
        e.restore(1, b)
        f = e.fragment(0)
        assert f.valid.tolist() == [0, 1, 1, 0]
        assert f.log_g[1] == 0.0 and f.log_g[2] == 5.0 and f.standard_error[2] == 1.0 and f.histogram[2] == 16
        assert math.isnan(f.log_g[0]) and math.isnan(f.standard_error[0])
        a, b = e.snapshot(0), e.snapshot(1)
        a.stage, a.factor = 2, 0.005
        b.stage, b.factor = 0, 0.5
        e.restore(0, a)
        e.restore(1, b)
        assert math.isfinite(e.exchange_log_probability(0, 1))
        e.swap_configuration(0, 1)
        a2, b2 = e.snapshot(0), e.snapshot(1)
        assert same_double(a2.log_g, a.log_g) and a2.factor == a.factor and a2.stage == a.stage
        assert same_double(b2.log_g, b.log_g) and b2.factor == b.factor and b2.stage == b.stage
        b = e.snapshot(1)
        b.active[:] = 0
        b.active[3] = 1
        e.restore(1, b)
        with pytest.raises(RuntimeError, match="no common active bin"):
            e.fragment(0)


def test_initialization_failure_message(oracle):
    """tests/test_main.cpp:195-216: the message names the window, bounds and search activity."""
    s = System(Geometry.simple_cubic(2, 1, 1, 1.0, (1, 0, 0), False))
    c = RunConfig(emin=-2.0, emax=2.0, bin_width=0.1, windows=3, walkers=1, seed=123,
                  explicit_windows=[(0, 25), (20, 30), (25, 40)])
    c.wl = WlParameters(0.8, 1, 1e-8, 10)
    c.wl.initialization_max_attempts = 10
    c.wl.initialization_stall_attempts_per_spin = 1
    c.check_interval_uses_mcs = c.force_accept_after_uses_mcs = False
    with pytest.raises(InitializationError) as got:
        Engine(s, c)
    from oracle.oracle import CheckerError
    with pytest.raises(CheckerError) as want:
        oracle.run_rewl(s, c)
    assert str(got.value) == str(want.value)
    assert "target band" in str(got.value) and "adaptive search used" in str(got.value)


def test_escaped_walker_is_reported():
    s = System(Geometry.simple_cubic(2, 1, 1, 1.0, (0, 0, 1), False))
    c = RunConfig(emin=-2, emax=2, bin_width=0.5, windows=2, walkers=1, seed=4, explicit_windows=[(0, 5), (3, 8)])
    with Engine(s, c) as e:
        up = e.snapshot(1)
        assert up.energy == 1.0
        up.walker_id = 0
        e.restore(0, up)
        with pytest.raises(EscapedError, match="escaped its energy window"):
            e.run_attempts(0, 1)


def test_invalid_configurations():
    s = System(Geometry.simple_cubic(2, 2, 1, periodic=False))
    with pytest.raises(InvalidArgument, match="Invalid run configuration"):
        Engine(s, RunConfig(emin=-20, emax=20, bin_width=0.25, overlap=1.0))
    with pytest.raises(InvalidArgument, match="integer multiple"):
        Engine(s, RunConfig(emin=-20, emax=20, bin_width=0.3))
    with pytest.raises(InvalidArgument, match="More windows than energy bins"):
        Engine(s, RunConfig(emin=-1, emax=1, bin_width=1.0, windows=3))
    bad = RunConfig(emin=-20, emax=20, bin_width=0.25)
    bad.wl.flatness = 1.5
    with pytest.raises(InitializationError, match="Invalid WL parameters"):
        Engine(s, bad)


def test_checkpoint_single_walker(tmp_path, oracle):
    """Single-walker checkpoint (src/parallel.cpp:354-360, 522-526; src/io.cpp:539-572)."""
    s = System(Geometry.simple_cubic(2, 2, 1, periodic=False))
    path = tmp_path / "walker.chk"
    c = RunConfig(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=1, seed=7, checkpoint_path=str(path),
                  max_mcs=400, checkpoint_interval_mcs=100)
    c.wl.final_factor = 1e-6
    c.resolve_mcs(4)
    first = run_rewl(s, c)
    assert path.exists()
    from replica_exchange_wang_landau_b200.engine import load_checkpoint
    snap = load_checkpoint(str(path))
    assert snap.attempted == 1600
    oc = RunConfig(**{k: getattr(c, k) for k in ("emin", "emax", "bin_width", "windows", "walkers", "seed",
                                                  "max_mcs")})
    oc.wl.final_factor = 1e-6
    oc.checkpoint_path = str(tmp_path / "oracle.chk")
    oc.checkpoint_interval_mcs = 100
    oc.resolve_mcs(4)
    want = oracle.run_rewl(s, oc)
    assert results_equal(first, want) == []
    assert (tmp_path / "oracle.chk").read_bytes() == path.read_bytes()
    # resume: a second run restores the checkpoint and continues to the larger limit
    c2 = RunConfig(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=1, seed=7, checkpoint_path=str(path),
                   max_mcs=800, checkpoint_interval_mcs=100)
    c2.wl.final_factor = 1e-6
    c2.resolve_mcs(4)
    oc2 = RunConfig(**{k: getattr(c2, k) for k in ("emin", "emax", "bin_width", "windows", "walkers", "seed",
                                                    "max_mcs")})
    oc2.wl.final_factor = 1e-6
    oc2.checkpoint_path = str(tmp_path / "oracle.chk")
    oc2.checkpoint_interval_mcs = 100
    oc2.resolve_mcs(4)
    assert results_equal(run_rewl(s, c2), oracle.run_rewl(s, oc2)) == []


def test_converged_run_matches_reference(reference):
    """A run to convergence on a larger system: 3x3x3 periodic (27 spins, random axes), two
    windows of two walkers with exchanges every MCS, no attempt limit, 1/t Wang-Landau to
    ln f <= 1e-5 (about 16 million attempts per walker).  The DOS fragments, counters and
    walker statistics equal those of the compiled reference's own run_rewl bit for bit."""
    g = Geometry.simple_cubic(3, 3, 3, periodic=True)
    g.axes = random_axes(g.size(), 41)
    s = System(g, 1.0, 0.0)
    c = RunConfig(emin=-60, emax=60, bin_width=0.5, windows=2, walkers=2, seed=77, exchange_interval_mcs=1,
                  check_interval_mcs=10)
    c.max_mcs = 0
    c.wl.final_factor = 1e-5
    c.resolve_mcs(s.size())
    got = run_rewl(s, c)
    want = reference.run_rewl(s, c)
    assert got.converged and want.converged
    assert results_equal(got, want) == []


def test_fragments_all_windows_equal_per_window():
    """wlg_engine_fragments (one launch for every window) gives each window's fragment exactly
    as wlg_engine_fragment does, and fails like it on a window without a common active bin."""
    s = _random_system((3, 3, 3), 11)
    c = RunConfig(emin=-60, emax=60, bin_width=0.5, windows=3, walkers=2, seed=21, max_mcs=60,
                  exchange_interval_mcs=1, check_interval_mcs=10)
    c.wl.final_factor = 1e-2
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        e.run()
        together = e.fragments()
        for w in range(c.windows):
            alone = e.fragment(w)
            assert together[w].window == alone.window
            for a, b in ((together[w].log_g, alone.log_g), (together[w].standard_error, alone.standard_error)):
                assert np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))
            assert np.array_equal(together[w].histogram, alone.histogram)
            assert np.array_equal(together[w].valid, alone.valid)
    fresh = RunConfig(emin=-60, emax=60, bin_width=0.5, windows=3, walkers=2, seed=21)
    fresh.resolve_mcs(s.size())
    with Engine(s, fresh) as e:  # no attempt yet: the walkers' visited bins differ
        e.run_attempts(0, 5)
        with pytest.raises(WlgError, match="no common active bin"):
            e.fragments()
        empty = e.fragments(allow_empty=True)
        assert len(empty) == 3
