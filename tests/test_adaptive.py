"""The adaptive-window host steps against the compiled reference, on identical pilot results
(CPU: the pilot run is the reference's own run_rewl)."""
from __future__ import annotations

import numpy as np
import pytest

from replica_exchange_wang_landau_b200.adaptive import (AdaptiveParameters, adapt_energy_windows,
                                                        select_initial_configurations)
from replica_exchange_wang_landau_b200.engine import RunConfig, System, WlParameters, partition_windows
from replica_exchange_wang_landau_b200.geometry import simple_cubic_random


def _pilot_config(seed: int, windows: int = 3) -> tuple:
    s = System(simple_cubic_random(4, 4, 4, seed=3, periodic=True), 1.0, 0.0)
    c = RunConfig(emin=-60, emax=60, bin_width=0.5, windows=windows, walkers=2, overlap=0.5, seed=seed)
    c.wl = WlParameters(0.8, 100, 1e-6, 1000, 0, True)
    c.wl.collect_window_statistics = True
    c.exchange_interval_mcs = 1.0
    c.max_mcs = 300.0
    c.resolve_mcs(s.size())
    return s, c


@pytest.mark.parametrize("seed", [5, 6])
def test_adapted_windows_and_seeds_match_reference(reference, seed):
    s, c = _pilot_config(seed)
    result, ref_windows, ref_seeds, ref_missing, ref_external = reference.pilot_round(s, c)
    windows = partition_windows(c.bins(), c.windows, c.overlap)
    for f, st, w in zip(result.fragments, result.sampling_statistics, windows):
        f.window = w
        st.window = w
    got = adapt_energy_windows(result, c.emin, c.emax, c.bin_width, c.windows, c.overlap, AdaptiveParameters())
    assert got == ref_windows
    seeds, missing, external = select_initial_configurations(c.emin, c.emax, c.bin_width, got,
                                                             result.representatives, s.size(), c.walkers)
    assert (missing, external) == (ref_missing, ref_external)
    for a, b in zip(seeds, ref_seeds):
        assert (a is None) == (b is None)
        if a is not None:
            assert np.array_equal(a, b)


def test_invalid_adaptive_parameters(reference):
    s, c = _pilot_config(5)
    result = reference.pilot_round(s, c)[0]
    for f, st, w in zip(result.fragments, result.sampling_statistics, partition_windows(c.bins(), 3, 0.5)):
        f.window = st.window = w
    with pytest.raises(Exception):
        adapt_energy_windows(result, c.emin, c.emax, c.bin_width, 3, 0.5, AdaptiveParameters(curvature_weight=-1.0))
