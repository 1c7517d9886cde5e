"""Mixed-precision runs: FP32 or BF16 (+ per-row FP32 scale) couplings with FP64 fields and a
periodic FP64 recompute.  The plain FP64 engine and exact enumeration are the references; the
reference has no low-precision path."""
from __future__ import annotations

import math

import numpy as np
import pytest

from replica_exchange_wang_landau_b200.engine import Engine, Geometry, RunConfig, System, WlParameters, run_rewl
from replica_exchange_wang_landau_b200.geometry import simple_cubic_random

pytestmark = pytest.mark.gpu


def _c1_config(precision: str, recompute_mcs: float, final_factor: float = 1e-4) -> RunConfig:
    c = RunConfig(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=2, seed=1234)
    c.wl = WlParameters(0.8, 100, final_factor, 1000, 0, True)
    c.coupling_precision = precision
    c.recompute_interval_mcs = recompute_mcs
    return c


def _rmse_vs_exact(oracle, s, frag) -> float:
    counts = oracle.exact_counts(s, -20, 20, 0.25)
    occ = counts > 0
    assert np.all(frag.valid[occ] == 1)
    exact = np.log(counts[occ].astype(float))
    d = frag.log_g[occ] - exact
    return math.sqrt(np.mean((d - d.mean()) ** 2))


def _c1_system() -> System:
    # 2x2x2 open lattice; easy axes from a seed so that J has irrational entries
    return System(simple_cubic_random(2, 2, 2, seed=7, periodic=False), 1.0, 0.0)


def test_fp32_against_exact(oracle):
    """FP32 J: converges like FP64 and matches the exact DOS as closely (RMSE <= 0.05)."""
    s = _c1_system()
    ref = run_rewl(s, _c1_config("fp64", 0.0).resolve_mcs(s.size()))
    assert ref.converged
    assert ref.precision_report["recomputes"] == 0 and ref.precision_report["max_field_drift"] == 0.0
    r = run_rewl(s, _c1_config("fp32", 5.0).resolve_mcs(s.size()))
    assert r.converged
    rep = r.precision_report
    assert rep["coupling_precision"] == "fp32"
    assert rep["recomputes"] > 0
    assert rep["resynced"] + rep["deferred"] == rep["recomputes"] * 2
    assert 0.0 < rep["max_field_drift"] <= 1e-6
    assert rep["max_energy_drift"] <= 1e-5
    e_ref = _rmse_vs_exact(oracle, s, ref.fragments[0])
    e_low = _rmse_vs_exact(oracle, s, r.fragments[0])
    assert e_ref <= 0.05 and e_low <= 0.05, (e_ref, e_low)


def test_bf16_drift_is_reported(oracle):
    """BF16 J (8 significant bits): with a resync every MCS the drift stays below a tenth of a
    bin and the DOS of the occupied bins stays within 0.3 of the exact one after a bounded run."""
    s = _c1_system()
    c = _c1_config("bf16", 1.0, final_factor=1e-3)
    c.exchange_interval_mcs = 1.0
    c.max_mcs = 20_000.0
    r = run_rewl(s, c.resolve_mcs(s.size()))
    rep = r.precision_report
    assert rep["coupling_precision"] == "bf16" and rep["recomputes"] > 0
    assert 0.0 < rep["max_field_drift"] <= 0.1 and rep["max_energy_drift"] <= 0.1
    counts = oracle.exact_counts(s, -20, 20, 0.25)
    frag = r.fragments[0]
    occ = (counts > 0) & (frag.valid == 1)
    assert occ.sum() >= 0.9 * (counts > 0).sum()
    d = frag.log_g[occ] - np.log(counts[occ].astype(float))
    assert math.sqrt(np.mean((d - d.mean()) ** 2)) <= 0.3


def test_recompute_resyncs_fields_to_fp64(oracle):
    """Right after a recompute every walker's fields and energy are the FP64 values of its spins."""
    geom = simple_cubic_random(4, 4, 4, seed=3, periodic=True)
    s = System(geom, 1.0, 0.0)
    j64 = s.couplings("fp64")
    c = RunConfig(emin=-60, emax=60, bin_width=0.5, windows=2, walkers=2, overlap=0.5, seed=5)
    c.wl = WlParameters(0.8, 100, 1e-6, 1000, 0, True)
    c.coupling_precision = "fp32"
    c.exchange_interval_mcs = 1.0
    c.recompute_interval_mcs = 1.0  # every epoch
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        e.run_epochs(6)
        rep = e.precision_report()
        assert rep["recomputes"] == 6 and rep["deferred"] == 0
        for w in range(4):
            snap = e.snapshot(w)
            f64 = j64 @ snap.spins.astype(np.float64)
            assert np.max(np.abs(snap.fields - f64)) < 1e-12
            assert abs(snap.energy - 0.5 * float(snap.spins.astype(np.float64) @ f64)) < 1e-9
        assert 0.0 < rep["max_field_drift"] < 1e-4


def test_fp64_runs_have_no_recompute():
    s = _c1_system()
    c = _c1_config("fp64", 5.0, final_factor=1e-2).resolve_mcs(s.size())
    with Engine(s, c) as e:
        e.run_epochs(3)
        rep = e.precision_report()
    assert rep["recompute_interval_attempts"] == 0 and rep["recomputes"] == 0


@pytest.mark.parametrize("precision", ["fp64", "fp32", "bf16"])
def test_split_sweep_matches_ring_sweep(precision):
    """Pilot statistics change no trajectory but route the dense sweep to the ring kernel
    (sweep_dense_kernel) instead of the split kernel: the two must agree bit for bit."""
    from helpers import snapshots_equal
    s = System(simple_cubic_random(4, 4, 4, seed=3, periodic=True), 1.0, 0.0)

    def run(collect: bool):
        c = RunConfig(emin=-60, emax=60, bin_width=0.5, windows=2, walkers=2, overlap=0.5, seed=11)
        c.wl = WlParameters(0.8, 100, 1e-6, 1000, 0, True)
        c.wl.collect_window_statistics = collect
        c.coupling_precision = precision
        c.exchange_interval_mcs = 1.0
        c.recompute_interval_mcs = 5.0
        c.resolve_mcs(s.size())
        with Engine(s, c) as e:
            e.run_epochs(25)
            return [e.snapshot(w) for w in range(4)], e.precision_report()

    split, rep_a = run(False)
    ring, rep_b = run(True)
    for a, b in zip(split, ring):
        assert snapshots_equal(a, b) == []
    assert rep_a["max_field_drift"] == rep_b["max_field_drift"]


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
@pytest.mark.parametrize("recompute_mcs", [1.0, 6.0])
def test_low_precision_run_with_recompute_bitwise(oracle, precision, recompute_mcs):
    """FP32 couplings, or BF16 couplings with their FP32 row scales, with the FP64 recompute
    every epoch (inside the epoch graph) and every third epoch (between graph replays), on the
    split sweep, bit for bit against the oracle's restatement of the update, the recompute and
    the resync."""
    from helpers import random_axes, results_equal
    g = Geometry.simple_cubic(5, 4, 4, periodic=True)
    g.axes = random_axes(g.size(), 31)
    s = System(g, 1.0, 0.0)
    c = RunConfig(emin=-200, emax=200, bin_width=0.5, windows=3, walkers=2, seed=12, exchange_interval_mcs=2,
                  check_interval_mcs=6, max_mcs=120)
    c.coupling_precision = precision
    c.recompute_interval_mcs = recompute_mcs
    c.resolve_mcs(s.size())
    got = run_rewl(s, c)
    want = oracle.run_rewl(s, c)
    assert got.precision_report["recomputes"] >= (50 if recompute_mcs == 1.0 else 15)
    assert results_equal(got, want) == []
