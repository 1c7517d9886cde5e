"""Helpers shared by the test modules: fixture decoding and bitwise comparisons."""
from __future__ import annotations

import numpy as np

from replica_exchange_wang_landau_b200.engine import Geometry, RunConfig, System, WlParameters


def unhex(values) -> np.ndarray:
    return np.array([float.fromhex(v) for v in values], dtype=np.float64)


def system_from(golden_system: dict) -> System:
    g = golden_system["geometry"]
    geom = Geometry(unhex(g["positions"]).reshape(-1, 3), unhex(g["axes"]).reshape(-1, 3), tuple(unhex(g["box"])),
                    bool(g["periodic"]))
    return System(geom, golden_system["scale"], golden_system["cutoff"])


def config_from(c: dict) -> RunConfig:
    wl = WlParameters(**c["wl"])
    cfg = RunConfig(emin=c["emin"], emax=c["emax"], bin_width=c["bin_width"], windows=c["windows"],
                    walkers=c["walkers"], overlap=c["overlap"], seed=c["seed"], wl=wl)
    cfg.exchange_interval_attempts = c["exchange_interval_attempts"]
    cfg.max_attempts = c["max_attempts"]
    cfg.checkpoint_interval_attempts = c["checkpoint_interval_attempts"]
    cfg.exchange_interval_uses_mcs = cfg.check_interval_uses_mcs = False
    cfg.force_accept_after_uses_mcs = cfg.max_limit_uses_mcs = cfg.checkpoint_interval_uses_mcs = False
    return cfg


def same_double(a, b) -> bool:
    """Bitwise equality of float64 arrays (NaN == NaN with the same payload class)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def snapshot_matches_json(s, j: dict) -> list:
    """Differences between a Snapshot and a golden snapshot dict (empty when identical)."""
    bad = []
    if s.spins.astype(int).tolist() != j["spins"]:
        bad.append("spins")
    if not same_double(s.fields, unhex(j["fields"])):
        bad.append("fields")
    if float(s.energy).hex() != j["energy"]:
        bad.append("energy")
    lg = {str(i): float(s.log_g[i]).hex() for i in np.nonzero(s.log_g)[0]}
    if lg != j["log_g"]:
        bad.append("log_g")
    h = {str(i): int(s.histogram[i]) for i in np.nonzero(s.histogram)[0]}
    if h != j["histogram"]:
        bad.append("histogram")
    if np.nonzero(s.active)[0].tolist() != j["active"]:
        bad.append("active")
    if float(s.factor).hex() != j["factor"]:
        bad.append("factor")
    for k in ("attempted", "accepted", "forced_accepted", "last_accepted_attempt", "stage"):
        if getattr(s, k) != j[k]:
            bad.append(k)
    if [str(x) for x in s.rng_state] != j["rng_state"]:
        bad.append("rng_state")
    return bad


def snapshots_equal(a, b) -> list:
    bad = []
    for k in ("spins", "histogram", "active"):
        if not np.array_equal(getattr(a, k), getattr(b, k)):
            bad.append(k)
    for k in ("fields", "log_g"):
        if not same_double(getattr(a, k), getattr(b, k)):
            bad.append(k)
    for k in ("energy", "factor"):
        if float(getattr(a, k)).hex() != float(getattr(b, k)).hex():
            bad.append(k)
    for k in ("attempted", "accepted", "forced_accepted", "last_accepted_attempt", "stage", "rng_state"):
        if getattr(a, k) != getattr(b, k):
            bad.append(k)
    return bad


def results_equal(a, b) -> list:
    """Differences between two RewlResult objects, bit for bit."""
    bad = []
    for k in ("attempted", "accepted", "forced_accepted", "exchange_attempted", "exchange_accepted", "converged"):
        if getattr(a, k) != getattr(b, k):
            bad.append(f"{k}: {getattr(a, k)} != {getattr(b, k)}")
    for w, (fa, fb) in enumerate(zip(a.fragments, b.fragments)):
        if not same_double(fa.log_g, fb.log_g):
            bad.append(f"fragment {w} log_g")
        if not np.array_equal(fa.histogram, fb.histogram):
            bad.append(f"fragment {w} histogram")
        if not same_double(fa.standard_error, fb.standard_error):
            bad.append(f"fragment {w} standard_error")
        if not np.array_equal(fa.valid, fb.valid):
            bad.append(f"fragment {w} valid")
    for sa, sb in zip(a.walker_statistics, b.walker_statistics):
        for k, v in sa.items():
            w = sb[k]
            if isinstance(v, float):
                if float(v).hex() != float(w).hex():
                    bad.append(f"walker {sa['walker_id']} {k}: {v} != {w}")
            elif v != w:
                bad.append(f"walker {sa['walker_id']} {k}: {v} != {w}")
    if len(a.sampling_statistics) != len(b.sampling_statistics):
        bad.append("sampling statistics count")
    for w, (sa, sb) in enumerate(zip(a.sampling_statistics, b.sampling_statistics)):
        if not same_double(sa.squared_energy_displacement, sb.squared_energy_displacement) or \
                not np.array_equal(sa.displacement_samples, sb.displacement_samples) or \
                sa.round_trips != sb.round_trips or sa.walkers != sb.walkers:
            bad.append(f"sampling {w}")
    if len(a.representatives) != len(b.representatives):
        bad.append(f"representatives {len(a.representatives)} != {len(b.representatives)}")
    else:
        for k, ((ea, sa), (eb, sb)) in enumerate(zip(a.representatives, b.representatives)):
            if float(ea).hex() != float(eb).hex() or not np.array_equal(sa, sb):
                bad.append(f"representative {k}")
    return bad


def random_axes(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, 3))
    return a / np.linalg.norm(a, axis=1)[:, None]
