"""Batches: several engines advanced by one CUDA-graph launch give the same results as the
engines run one after another."""
from __future__ import annotations

import pytest

from helpers import snapshots_equal
from replica_exchange_wang_landau_b200.engine import Batch, Engine, RunConfig, System, WlParameters
from replica_exchange_wang_landau_b200.geometry import random_sequential, simple_cubic_random

pytestmark = pytest.mark.gpu


def _engines():
    specs = [
        (System(simple_cubic_random(2, 2, 2, seed=7, periodic=False)), -20.0, 20.0, 0.25, 1, "fp64", 1),
        (System(random_sequential(10, 0.5, 0.8, seed=4)), -16.0, 16.0, 0.25, 2, "fp64", 1),
        (System(simple_cubic_random(4, 4, 4, seed=3, periodic=True)), -60.0, 60.0, 0.5, 3, "fp32", 2),
    ]
    out = []
    for s, lo, hi, w, seed, prec, windows in specs:
        c = RunConfig(emin=lo, emax=hi, bin_width=w, windows=windows, walkers=2, overlap=0.5, seed=seed)
        c.wl = WlParameters(0.8, 100, 1e-3, 1000, 0, True)
        c.coupling_precision = prec
        c.recompute_interval_mcs = 0.0  # the batch recomputes at launch boundaries only
        c.exchange_interval_mcs = 5.0
        c.max_mcs = 3000.0
        c.resolve_mcs(s.size())
        out.append((s, c))
    return out


def test_batch_matches_separate_runs():
    specs = _engines()
    separate = []
    for s, c in specs:
        with Engine(s, c) as e:
            e.run()
            separate.append(([e.snapshot(w) for w in range(e.walkers)], e.totals()))
    engines = [Engine(s, c) for s, c in specs]
    try:
        with Batch(engines) as b:
            b.run()
        for e, (snaps, totals) in zip(engines, separate):
            t = e.totals()
            assert t["attempted"] == totals["attempted"] and t["converged"] == totals["converged"]
            for w in range(e.walkers):
                assert snapshots_equal(e.snapshot(w), snaps[w]) == []
    finally:
        for e in engines:
            e.close()


def test_batch_rejects_duplicates():
    s, c = _engines()[0]
    with Engine(s, c) as e:
        with pytest.raises(Exception):
            Batch([e, e])


@pytest.mark.parametrize("cutoff", [0.0, 1.8])
def test_autotune_keeps_results(cutoff):
    """The launch-shape autotuner changes speed only: the run's results are bit-identical."""
    s = System(simple_cubic_random(4, 4, 4, seed=3, periodic=True), 1.0, cutoff)
    c = RunConfig(emin=-60, emax=60, bin_width=0.5, windows=2, walkers=2, overlap=0.5, seed=9)
    c.wl = WlParameters(0.8, 100, 1e-3, 1000, 0, True)
    c.exchange_interval_mcs = 2.0
    c.max_mcs = 4000.0
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        e.run()
        plain = [e.snapshot(w) for w in range(4)]
    with Engine(s, c) as e:
        r = e.autotune(4)
        assert r["epochs_per_graph"] in (4, 8, 16, 32, 64) and 1 <= r["walkers_per_block"] <= 8
        assert r["trials"] >= 5 and r["ms_per_epoch"] > 0
        if cutoff > 0:
            assert r["staging_ring"] == 0  # the CSR sweep has no staging ring
        else:  # the dense engine runs the split sweep: both staging depths are candidates
            assert r["staging_ring"] in (16, 32) and r["trials"] >= 10
        e.run()
        for w in range(4):
            assert snapshots_equal(e.snapshot(w), plain[w]) == []


def test_staging_ring_keeps_results(oracle):
    """The split sweep with a 32-draw staging ring, switched between epochs, runs bit for bit
    like the oracle (512 sites, 3 windows, 1/t stage reached)."""
    from helpers import results_equal
    s = System(simple_cubic_random(8, 8, 8, seed=18, periodic=True), 1.0, 0.0)
    c = RunConfig(emin=-228.5, emax=228.0, bin_width=0.5, windows=3, walkers=2, seed=19, exchange_interval_mcs=1)
    c.wl.final_factor = 1e-2
    c.check_interval_mcs = 5
    c.max_mcs = 300
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        e.set_staging_ring(32)
        e.run_epochs(100)
        e.set_staging_ring(16)
        e.run_epochs(50)
        e.set_staging_ring(32)
        e.run()
        got = e.result()
        with pytest.raises(Exception):
            e.set_staging_ring(24)
    assert results_equal(got, oracle.run_rewl(s, c)) == []
    cs = System(simple_cubic_random(4, 4, 4, seed=3, periodic=True), 1.0, 1.8)
    cc = RunConfig(emin=-60, emax=60, bin_width=0.5, windows=1, walkers=1, seed=9).resolve_mcs(64)
    with Engine(cs, cc) as e:
        with pytest.raises(Exception):
            e.set_staging_ring(32)  # the CSR sweep has no staging ring
