"""GPU parity of the CSR sweep (csrc/sweep_csr.cu): WangLandauWalker trajectories and run_rewl
(src/wang_landau.cpp:244-315, src/parallel.cpp:276-747) with CsrCouplings (src/physics.cpp:197-236)
bit for bit against the oracle, for couplings rows of 32, 64, 128 and 256 ELLPACK entries, FP64
and FP32 couplings, power-of-two and other bin widths; and, at the 32^3 size, the fields the
sweep maintains against a full recompute."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import random_axes, results_equal, snapshots_equal
from replica_exchange_wang_landau_b200.engine import Engine, Geometry, RunConfig, System, WlParameters, run_rewl

pytestmark = pytest.mark.gpu


def _lattice(dims, seed, cutoff, random=True):
    g = Geometry.simple_cubic(*dims, periodic=True)
    if random:
        g.axes = random_axes(g.size(), seed)
    return System(g, 1.0, cutoff)


CASES = {
    # name: (system, config kwargs, couplings precision)
    # 5^3, cutoff 2.2: 32 neighbours, rows of exactly one 32-entry chunk; N = 125 (site draws by
    # Barrett reduction, not a mask)
    "z32_pow2": (lambda: _lattice((5, 5, 5), 23, 2.2),
                 dict(emin=-120, emax=60, bin_width=0.5, windows=2, walkers=2, seed=31), "fp64"),
    # 6^3, cutoff 2.5: 80 neighbours in 128-entry rows; bin width 0.75
    "z80_width075": (lambda: _lattice((6, 6, 6), 21, 2.5),
                     dict(emin=-200, emax=100, bin_width=0.75, windows=2, walkers=2, seed=32), "fp64"),
    "z80_fp32": (lambda: _lattice((6, 6, 6), 21, 2.5),
                 dict(emin=-200, emax=100, bin_width=0.5, windows=2, walkers=2, seed=33), "fp32"),
    # 8^3, cutoff 3.5: 178 neighbours in 256-entry rows
    "z178": (lambda: _lattice((8, 8, 8), 22, 3.5),
             dict(emin=-300, emax=100, bin_width=1.0, windows=2, walkers=2, seed=34), "fp64"),
    # 4^3, cutoff 1.8: 18 neighbours, +z axes, forced acceptance after 0.3 MCS without a flip
    "z18_forced": (lambda: _lattice((4, 4, 4), 24, 1.8, random=False),
                   dict(emin=-60, emax=40, bin_width=0.25, windows=2, walkers=2, seed=35, force_accept_after_mcs=0.3),
                   "fp64"),
}


def _config(kw, precision):
    c = RunConfig(**kw)
    c.coupling_precision = precision
    return c


@pytest.mark.parametrize("name", list(CASES))
def test_csr_trajectories_bitwise(oracle, name):
    make_system, kw, precision = CASES[name]
    s = make_system()
    c = _config(kw, precision)
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        walkers = []
        for w in range(e.walkers):
            ow = oracle.walker(s, w, c.emin, c.emax, c.bin_width, e.window(w // c.walkers), c.wl, c.seed)
            assert snapshots_equal(e.snapshot(w), ow.snapshot()) == [], f"init of walker {w}"
            if precision == "fp32":
                ow.set_update_fp32(True)  # the engine's walkers are initialised with FP64 couplings
            walkers.append(ow)
        for rounds in range(3):
            for w, ow in enumerate(walkers):
                e.run_attempts(w, 1537 + 311 * rounds)
                ow.run_attempts(1537 + 311 * rounds)
                assert snapshots_equal(e.snapshot(w), ow.snapshot()) == [], f"walker {w} round {rounds}"


RUNS = {
    "z80_exchange": (lambda: _lattice((6, 6, 6), 21, 2.5),
                     dict(emin=-200, emax=100, bin_width=0.75, windows=3, walkers=2, seed=41, max_mcs=40,
                          exchange_interval_mcs=0.5, check_interval_mcs=2), dict(final_factor=1e-2)),
    "z178_exchange": (lambda: _lattice((8, 8, 8), 22, 3.5),
                      dict(emin=-300, emax=100, bin_width=1.0, windows=2, walkers=3, seed=42, max_mcs=20,
                           exchange_interval_mcs=1, check_interval_mcs=2), dict(final_factor=1e-2)),
    "z32_inverse_time": (lambda: _lattice((5, 5, 5), 23, 2.2),
                         dict(emin=-120, emax=60, bin_width=0.5, windows=2, walkers=2, seed=43, max_mcs=400,
                              exchange_interval_mcs=1, check_interval_mcs=5),
                         dict(flatness=0.3, minimum_visits=3, final_factor=1e-4)),
    # pilot statistics: squared displacements, samples, round trips and representatives
    "z80_pilot": (lambda: _lattice((6, 6, 6), 21, 2.5),
                  dict(emin=-200, emax=100, bin_width=0.75, windows=3, walkers=2, seed=44, max_mcs=60,
                       exchange_interval_mcs=0.5, check_interval_mcs=2),
                  dict(collect_window_statistics=True, final_factor=1e-2)),
    "z178_pilot": (lambda: _lattice((8, 8, 8), 22, 3.5),
                   dict(emin=-300, emax=100, bin_width=1.0, windows=2, walkers=3, seed=45, max_mcs=30,
                        exchange_interval_mcs=1, check_interval_mcs=2),
                   dict(collect_window_statistics=True, final_factor=1e-2)),
}


@pytest.mark.parametrize("name", list(RUNS))
def test_csr_run_rewl_bitwise(oracle, name):
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


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_csr_32cubed_fields_consistent(precision):
    """32^3 periodic lattice, cutoff 3.0 (122 neighbours), +z axes: after epochs of the CSR
    sweep every walker's fields equal a full FP64 recompute from its spins to 1e-9, and its
    energy the recomputed total energy; the FP64 run draws no field drift report."""
    g = Geometry.simple_cubic(32, 32, 32, 1.0, (0.0, 0.0, 1.0), True)
    s = System(g, 1.0, 3.0)
    c = RunConfig(emin=-2144.0, emax=1932.0, bin_width=4.0, windows=4, walkers=2, seed=5, overlap=0.75)
    c.wl = WlParameters(0.8, 100, 1e-8, 1000, 0, True)
    c.coupling_precision = precision
    c.exchange_interval_mcs = 0.05
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        e.run_epochs(6)
        t = e.totals()
        assert t["attempted"] == 6 * 8 * c.exchange_interval_attempts
        assert 0 < t["accepted"] < t["attempted"]
        for w in range(e.walkers):
            snap = e.snapshot(w)
            fields, energy = s.local_fields(snap.spins)
            tol = 1e-9 if precision == "fp64" else 1e-4
            assert np.max(np.abs(snap.fields - fields)) <= tol
            assert abs(snap.energy - energy) <= 1e3 * tol
            lo, hi = e.window(w // c.walkers)
            b = int(np.floor((snap.energy - c.emin) / c.bin_width))
            assert lo <= b < hi


@pytest.mark.parametrize("collect", [False, True])
def test_csr_large_system_spins_in_hbm(collect):
    """60^3 lattice (N = 216000), cutoff 1.5: the walkers' spins no longer fit in shared memory
    next to their window, so the initialisation and the generic sweep (pilot statistics) read
    them from HBM; the fields the sweep maintains still equal a full recompute."""
    g = Geometry.simple_cubic(60, 60, 60, 1.0, (0.0, 0.0, 1.0), True)
    s = System(g, 1.0, 1.5)
    c = RunConfig(emin=-20000.0, emax=20000.0, bin_width=100.0, windows=1, walkers=2, seed=7)
    c.wl = WlParameters(0.8, 100, 1e-8, 1000, 0, True, collect_window_statistics=collect)
    c.exchange_interval_mcs = 0.01
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        e.run_epochs(3)
        t = e.totals()
        assert t["attempted"] == 3 * 2 * c.exchange_interval_attempts
        assert 0 < t["accepted"]
        for w in range(e.walkers):
            snap = e.snapshot(w)
            fields, energy = s.local_fields(snap.spins)
            assert np.max(np.abs(snap.fields - fields)) <= 1e-9
            assert abs(snap.energy - energy) <= 1e-6


def test_csr_converged_run_matches_reference(reference):
    """A CSR run to convergence: 5x5x5 periodic (125 spins, random axes, cutoff 2.2), two
    windows of two walkers with exchanges every MCS, 1/t Wang-Landau to ln f <= 1e-5 (about 14
    million attempts per walker), equal to the compiled reference's own run_rewl bit for bit."""
    s = _lattice((5, 5, 5), 43, 2.2)
    c = RunConfig(emin=-120, emax=60, bin_width=1.0, windows=2, walkers=2, seed=78, exchange_interval_mcs=1,
                  check_interval_mcs=10)
    c.max_mcs = 0
    c.wl.final_factor = 1e-5
    c.resolve_mcs(s.size())
    got = run_rewl(s, c)
    want = reference.run_rewl(s, c)
    assert got.converged and want.converged
    assert results_equal(got, want) == []
