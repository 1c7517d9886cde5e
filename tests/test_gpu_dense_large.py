"""GPU parity of the dense sweep for systems beyond the split sweep's register form (ld > 1024,
the single-warp ring sweep `sweep_dense_kernel`): walker trajectories and run_rewl
(src/wang_landau.cpp:244-315, src/parallel.cpp:276-747) bit for bit against the oracle, FP64 and
FP32 couplings; BF16 through the drift report."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import random_axes, results_equal, snapshots_equal
from replica_exchange_wang_landau_b200.engine import Engine, Geometry, RunConfig, System, run_rewl

pytestmark = pytest.mark.gpu


def _lattice(dims, seed):
    g = Geometry.simple_cubic(*dims, periodic=True)
    g.axes = random_axes(g.size(), seed)
    return System(g, 1.0, 0.0)


CASES = {
    # N = 1089 (ld 1104) and N = 1728: FP64 rows of 8.6 and 13.5 KB
    "n1089_fp64": ((11, 11, 9), 51, dict(emin=-200, emax=200, bin_width=0.5, windows=2, walkers=2, seed=61), "fp64"),
    "n1728_fp64": ((12, 12, 12), 52, dict(emin=-240, emax=240, bin_width=0.75, windows=2, walkers=2,
                                                      seed=62), "fp64"),
    "n1728_fp32": ((12, 12, 12), 53, dict(emin=-240, emax=240, bin_width=0.5, windows=2, walkers=2, seed=63), "fp32"),
}


@pytest.mark.parametrize("name", list(CASES))
def test_large_dense_trajectories_bitwise(oracle, name):
    dims, axes_seed, kw, precision = CASES[name]
    s = _lattice(dims, axes_seed)
    c = RunConfig(**kw)
    c.coupling_precision = precision
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
                e.run_attempts(w, 2311 + 577 * rounds)
                ow.run_attempts(2311 + 577 * rounds)
                assert snapshots_equal(e.snapshot(w), ow.snapshot()) == [], f"walker {w} round {rounds}"


@pytest.mark.parametrize("dims,axes_seed", [((11, 11, 9), 51), ((12, 12, 12), 52)])
def test_large_dense_run_rewl_bitwise(oracle, dims, axes_seed):
    s = _lattice(dims, axes_seed)
    c = RunConfig(emin=-240, emax=240, bin_width=0.75, windows=3, walkers=2, seed=64, max_mcs=12,
                  exchange_interval_mcs=1, check_interval_mcs=2)
    c.wl.final_factor = 1e-2
    c.resolve_mcs(s.size())
    got = run_rewl(s, c)
    want = oracle.run_rewl(s, c)
    assert got.attempted > 0
    assert results_equal(got, want) == []


def test_large_dense_bf16_drift():
    """BF16 rows with a row scale: the FP64 recompute every MCS measures a drift well below a bin
    and the walkers stay consistent with a full recompute after resync."""
    s = _lattice((12, 12, 12), 55)
    c = RunConfig(emin=-240, emax=240, bin_width=0.75, windows=2, walkers=2, seed=65)
    c.coupling_precision = "bf16"
    c.recompute_interval_mcs = 1.0
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        e.run_epochs(4)
        rep = e.precision_report()
        assert rep["recomputes"] >= 3
        assert 0.0 < rep["max_field_drift"] < 0.2
        for w in range(e.walkers):
            snap = e.snapshot(w)
            fields, energy = s.local_fields(snap.spins)
            assert np.max(np.abs(snap.fields - fields)) < 0.2
