"""The adaptive-window pilot on the engine reproduces wl_run's rounds (apps/wl_run.cpp:104-169)
run with the reference: the same windows and seeds after every round, then a production run
on them."""
from __future__ import annotations

import copy

import numpy as np
import pytest

from replica_exchange_wang_landau_b200.adaptive import GOLDEN_GAMMA, AdaptiveParameters, adaptive_pilot
from replica_exchange_wang_landau_b200.engine import RunConfig, System, WlParameters, partition_windows, run_rewl
from replica_exchange_wang_landau_b200.geometry import simple_cubic_random

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cutoff", [0.0, 2.0])  # dense couplings; CSR (the CSR sweep with pilot statistics)
def test_adaptive_pilot_matches_reference(reference, cutoff):
    s = System(simple_cubic_random(4, 4, 4, seed=3, periodic=True), 1.0, cutoff)
    c = RunConfig(emin=-60, emax=60, bin_width=0.5, windows=3, walkers=2, overlap=0.5, seed=17)
    c.wl = WlParameters(0.8, 100, 1e-3, 1000, 0, True)
    c.exchange_interval_mcs = 1.0
    params = AdaptiveParameters(iterations=2, pilot_mcs=300.0)
    lines = []
    windows, seeds = adaptive_pilot(s, c, params, log=lines.append)
    assert len(lines) == 4 and lines[1].startswith("adaptive_window_round_trips=")

    # the same rounds with the reference's run_rewl and host steps
    ref_windows = partition_windows(c.bins(), c.windows, c.overlap)
    ref_seeds = None
    for it in range(params.iterations):
        p = copy.deepcopy(c)
        p.explicit_windows = ref_windows
        p.initial_spins_by_walker = ref_seeds
        p.wl.collect_window_statistics = True
        p.max_mcs = params.pilot_mcs
        p.resolved_spin_count = 0
        p.seed = (c.seed ^ ((it + 1) * GOLDEN_GAMMA)) & 0xFFFFFFFFFFFFFFFF
        p.resolve_mcs(s.size())
        _, ref_windows, ref_seeds, _, _ = reference.pilot_round(s, p)
    assert windows == ref_windows
    for a, b in zip(seeds, ref_seeds):
        assert (a is None) == (b is None) and (a is None or np.array_equal(a, b))

    # production on the adapted windows from the seeds
    prod = copy.deepcopy(c)
    prod.explicit_windows = windows
    prod.initial_spins_by_walker = seeds
    prod.max_mcs = 2000.0
    prod.resolve_mcs(s.size())
    r = run_rewl(s, prod)
    assert [f.window for f in r.fragments] == [tuple(w) for w in windows]
