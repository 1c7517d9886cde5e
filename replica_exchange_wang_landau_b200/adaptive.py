"""The adaptive-window pilot of wl_run (apps/wl_run.cpp:104-169) on the engine.

Each round runs the engine with pilot statistics on (run_rewl with
collect_window_statistics) over the current windows for pilot_mcs MCS, then chooses the next
windows from the pilot's fragments and sampling statistics (adapt_energy_windows) and seeds
every walker of those windows from the pilot's representative configurations
(select_adaptive_initial_configurations).  The host steps run in the library
(csrc/adaptive.cpp) in the reference's arithmetic order, and the pilot runs are the
engine's bit-identical run_rewl, so the windows and seeds equal the reference's; the
production run then uses them as explicit windows and initial spins.
"""
from __future__ import annotations

import copy
import ctypes as C
from dataclasses import dataclass
from typing import Callable, Optional, Sequence

import numpy as np

from . import _abi
from .engine import (RewlResult, RunConfig, System, _check, _dptr, _fragment_view, _i8ptr, _u8ptr, _u64ptr,
                     load_library, partition_windows, run_rewl)

GOLDEN_GAMMA = 0x9E3779B97F4A7C15


@dataclass
class AdaptiveParameters:
    """wl::AdaptiveWindowParameters (include/wl/analysis.hpp:28-38)."""
    iterations: int = 2
    pilot_mcs: float = 10_000.0
    smoothing_width: float = 0.0
    minimum_width: float = 0.0
    diffusivity_floor_fraction: float = 0.05
    curvature_weight: float = 0.25
    round_trip_target: float = 2.0
    maximum_round_trip_penalty: float = 3.0

    def _struct(self) -> _abi.wlg_adaptive_parameters:
        return _abi.wlg_adaptive_parameters(int(self.iterations), float(self.pilot_mcs), float(self.smoothing_width),
                                            float(self.minimum_width), float(self.diffusivity_floor_fraction),
                                            float(self.curvature_weight), float(self.round_trip_target),
                                            float(self.maximum_round_trip_penalty))


def adapt_energy_windows(result: RewlResult, emin: float, emax: float, width: float, count: int, overlap: float,
                         params: AdaptiveParameters) -> list:
    """Next windows from a pilot result (src/analysis.cpp:183-339)."""
    if len(result.fragments) != count or len(result.sampling_statistics) != count:
        raise ValueError("Adaptive-window pilot fragments are incompatible")
    views, samp, keep = [], [], []
    for f, s in zip(result.fragments, result.sampling_statistics):
        v, arrays = _fragment_view(f)
        sq = np.ascontiguousarray(s.squared_energy_displacement, np.float64)
        ds = np.ascontiguousarray(s.displacement_samples, np.uint64)
        views.append(v)
        samp.append(_abi.wlg_sampling_view(int(s.window[0]), int(s.window[1]), _dptr(sq), _u64ptr(ds),
                                           int(s.round_trips), int(s.walkers)))
        keep += [arrays, sq, ds]
    out = np.zeros(2 * count, np.uint64)
    p = params._struct()
    _check(load_library().wlg_adapt_energy_windows(emin, emax, width, (_abi.wlg_fragment_view * count)(*views),
                                                   (_abi.wlg_sampling_view * count)(*samp), count, overlap,
                                                   C.byref(p), _u64ptr(out)))
    return [(int(out[2 * k]), int(out[2 * k + 1])) for k in range(count)]


def select_initial_configurations(emin: float, emax: float, width: float, windows: Sequence[tuple],
                                  representatives: Sequence[tuple], n: int, walkers_per_window: int):
    """Seeds for every walker (src/analysis.cpp:341-420, one process): a list with one spin
    array or None per walker, and the missing / external counts."""
    reps = len(representatives)
    energy = np.array([e for e, _ in representatives] or [0.0], np.float64)
    spins = np.zeros((max(1, reps), n), np.int8)
    present = np.zeros(max(1, reps), np.uint8)
    for k, (_, s) in enumerate(representatives):
        if s is not None and len(s):
            spins[k] = s
            present[k] = 1
    w = np.array([v for pair in windows for v in pair], np.uint64)
    total = len(windows) * walkers_per_window
    out = np.zeros((total, n), np.int8)
    out_present = np.zeros(total, np.uint8)
    missing, external = C.c_uint64(0), C.c_uint64(0)
    _check(load_library().wlg_select_initial_configurations(
        emin, emax, width, _u64ptr(w), len(windows), _dptr(energy), _i8ptr(spins), _u8ptr(present), reps, n,
        walkers_per_window, _i8ptr(out), _u8ptr(out_present), C.byref(missing), C.byref(external)))
    seeds = [out[k].copy() if out_present[k] else None for k in range(total)]
    return seeds, int(missing.value), int(external.value)


def adaptive_pilot(system: System, config: RunConfig, params: AdaptiveParameters,
                   log: Optional[Callable[[str], None]] = print):
    """wl_run's adaptive-window rounds; returns (windows, initial spins per walker) for the
    production run (config.explicit_windows, config.initial_spins_by_walker)."""
    n = system.size()
    bins = config.bins()
    windows = partition_windows(bins, int(config.windows), float(config.overlap))
    initial = None
    for iteration in range(int(params.iterations)):
        if log:
            log(f"adaptive_window_pilot={iteration + 1}/{params.iterations} pilot_mcs={params.pilot_mcs:g}")
        pilot = copy.deepcopy(config)
        pilot.explicit_windows = windows
        pilot.initial_spins_by_walker = initial
        pilot.wl.collect_window_statistics = True
        pilot.max_mcs = float(params.pilot_mcs)
        pilot.max_limit_uses_mcs = True
        pilot.checkpoint_path = ""
        pilot.resolved_spin_count = 0
        pilot.seed = (int(config.seed) ^ ((iteration + 1) * GOLDEN_GAMMA)) & 0xFFFFFFFFFFFFFFFF
        pilot.resolve_mcs(n)
        result = run_rewl(system, pilot)
        windows = adapt_energy_windows(result, config.emin, config.emax, config.bin_width, int(config.windows),
                                       float(config.overlap), params)
        initial, missing, external = select_initial_configurations(
            config.emin, config.emax, config.bin_width, windows, result.representatives, n, int(config.walkers))
        if log:  # the line wl_run prints (apps/wl_run.cpp:133-160), default stream formatting
            trips = sum(s.round_trips for s in result.sampling_statistics)
            seeded = [e for e, s in result.representatives if s is not None and len(s)]
            lowest = f" minimum_seed_energy={min(seeded):g}" if seeded else ""
            ranges = ";".join(f"[{config.emin + b * config.bin_width:g},{config.emin + e * config.bin_width:g})"
                              for b, e in windows)
            log(f"adaptive_window_round_trips={trips} seeded_walkers={len(initial) - missing}/{len(initial)} "
                f"external_warm_starts={external}{lowest} energy_ranges={ranges}")
    return windows, initial
