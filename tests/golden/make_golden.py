"""Generates tests/golden/*.json from the reference implementation itself.

Run in a container that has the reference sources (it builds oracle/_ref/libwlref.so from
them with oracle/Makefile):

    python tests/golden/make_golden.py

Every double is stored as float.hex() so the fixtures pin results bit for bit.  The
geometries are stored with the fixtures, so the tests never regenerate them.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as ora  # noqa: E402
from replica_exchange_wang_landau_b200.engine import Geometry, RunConfig, System, WlParameters  # noqa: E402

OUT = Path(__file__).resolve().parent


def hx(a) -> list:
    return [float(x).hex() for x in np.asarray(a, dtype=np.float64).ravel()]


def geometry_json(g: Geometry) -> dict:
    return {"positions": hx(g.positions), "axes": hx(g.axes), "box": hx(g.box), "periodic": g.periodic}


def random_axes(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, 3))
    return a / np.linalg.norm(a, axis=1)[:, None]


def snapshot_json(s) -> dict:
    nz = np.nonzero(s.histogram)[0].tolist()
    return {"spins": s.spins.astype(int).tolist(), "fields": hx(s.fields), "energy": float(s.energy).hex(),
            "log_g": {str(i): float(s.log_g[i]).hex() for i in np.nonzero(s.log_g)[0]},
            "histogram": {str(i): int(s.histogram[i]) for i in nz},
            "active": np.nonzero(s.active)[0].tolist(), "factor": float(s.factor).hex(),
            "attempted": s.attempted, "accepted": s.accepted, "forced_accepted": s.forced_accepted,
            "last_accepted_attempt": s.last_accepted_attempt, "stage": s.stage,
            "rng_state": [str(x) for x in s.rng_state]}


def result_json(r) -> dict:
    frags = []
    for f in r.fragments:
        frags.append({"log_g": hx(f.log_g), "histogram": [int(x) for x in f.histogram],
                      "standard_error": hx(f.standard_error), "valid": f.valid.astype(int).tolist()})
    stats = []
    for s in r.walker_statistics:
        stats.append({k: (float(v).hex() if isinstance(v, float) else int(v)) for k, v in s.items()})
    return {"attempted": r.attempted, "accepted": r.accepted, "forced_accepted": r.forced_accepted,
            "exchange_attempted": r.exchange_attempted, "exchange_accepted": r.exchange_accepted,
            "converged": r.converged, "fragments": frags, "walker_statistics": stats}


def config_json(c: RunConfig) -> dict:
    wl = {k: getattr(c.wl, k) for k in WlParameters.__dataclass_fields__}
    return {"emin": c.emin, "emax": c.emax, "bin_width": c.bin_width, "windows": c.windows, "walkers": c.walkers,
            "overlap": c.overlap, "seed": c.seed, "wl": wl, "exchange_interval_attempts": c.exchange_interval_attempts,
            "max_attempts": c.max_attempts, "checkpoint_interval_attempts": c.checkpoint_interval_attempts}


def main() -> None:
    ora.build()
    ref = ora.Reference()
    golden = {"generator": "tests/golden/make_golden.py", "source": "oracle/_ref/libwlref.so (reference sources)"}

    # 1. pair formula and minimum image (tests/test_main.cpp:24-38)
    golden["pair"] = [
        {"d": d, "ai": ai, "aj": aj, "value": ref.dipolar_pair(d, ai, aj, 1.0).hex()}
        for d, ai, aj in [((1, 0, 0), (1, 0, 0), (1, 0, 0)), ((1, 0, 0), (0, 0, 1), (0, 0, 1)),
                          ((2, 0, 0), (0, 0, 1), (0, 0, 1)), ((0.3, -1.2, 0.7), (0.6, 0.0, 0.8), (0.0, 0.6, -0.8))]]
    golden["minimum_image"] = [
        {"d": d, "box": box, "periodic": True, "out": [x.hex() for x in ref.minimum_image(d, box, True)]}
        for d, box in [((6, -5, 3.1), (10, 8, 6)), ((6, -5, 31), (10, 8, 0)), ((0.5, 2.5, -3.5), (1, 5, 7))]]

    # 2. exact enumeration: the 2x2x2 open lattice of the CPU-runnable configuration and 2x2x1
    for name, dims in (("exact_2x2x2", (2, 2, 2)), ("exact_2x2x1", (2, 2, 1))):
        s = System(Geometry.simple_cubic(*dims, periodic=False))
        counts = ref.exact_counts(s, -20.0, 20.0, 0.25)
        golden[name] = {"dims": dims, "emin": -20.0, "emax": 20.0, "width": 0.25,
                        "counts": {str(i): int(c) for i, c in enumerate(counts) if c}}

    # 3. couplings and fields for periodic / slab / open / CSR systems with random axes
    systems = {}
    g = Geometry.simple_cubic(3, 3, 3, periodic=True)
    g.axes = random_axes(27, 11)
    systems["cubic27_periodic"] = System(g, 1.0, 0.0)
    gs = Geometry.simple_cubic(4, 3, 2, periodic=True)
    gs.axes = random_axes(24, 12)
    gs.box = (4.0, 3.0, 0.0)
    systems["slab24"] = System(gs, 0.7, 0.0)
    gc = Geometry.simple_cubic(4, 4, 4, periodic=True)
    gc.axes = random_axes(64, 13)
    systems["csr64_r1.8"] = System(gc, 1.0, 1.8)
    golden["systems"] = {}
    rng = np.random.default_rng(5)
    for name, s in systems.items():
        spins = rng.choice(np.array([-1, 1], dtype=np.int8), size=(3, s.size()))
        fields, energies = ref.local_fields(s, spins)
        golden["systems"][name] = {"geometry": geometry_json(s.geometry), "scale": s.coupling_scale,
                                   "cutoff": s.cutoff, "couplings": hx(ref.couplings(s)),
                                   "spins": spins.astype(int).tolist(), "fields": hx(fields),
                                   "energies": hx(energies)}

    # 4. walker trajectories: constructor (target Metropolis) and 3000 attempts
    golden["walkers"] = []
    for name, grid, window, wid, seed in (("cubic27_periodic", (-60.0, 60.0, 0.5), (40, 200), 5, 77),
                                          ("csr64_r1.8", (-150.0, 150.0, 0.5), (100, 400), 2, 9),
                                          ("slab24", (-40.0, 40.0, 0.25), (0, 320), 0, 3)):
        p = WlParameters(check_interval_attempts=100)
        w = ref.walker(systems[name], wid, *grid, window, p, seed)
        init = snapshot_json(w.snapshot())
        w.run_attempts(3000)
        golden["walkers"].append({"system": name, "grid": grid, "window": window, "walker_id": wid, "seed": seed,
                                  "params": {"check_interval_attempts": 100}, "init": init,
                                  "after_3000": snapshot_json(w.snapshot())})

    # 5. run_rewl: windows x walkers with exchange, and the 2x2x2 system to ln f = 1e-3
    golden["rewl"] = []
    c = RunConfig(emin=-60.0, emax=60.0, bin_width=0.5, windows=3, walkers=2, seed=21, overlap=0.75)
    c.wl.final_factor = 1e-2
    c.max_mcs = 200
    c.exchange_interval_mcs = 1
    c.check_interval_mcs = 10
    c.resolve_mcs(27)
    golden["rewl"].append({"system": "cubic27_periodic", "config": config_json(c),
                           "result": result_json(ref.run_rewl(systems["cubic27_periodic"], c))})
    c1 = RunConfig(emin=-20.0, emax=20.0, bin_width=0.25, windows=1, walkers=2, seed=1234)
    c1.wl.final_factor = 1e-3
    c1.resolve_mcs(8)
    s8 = System(Geometry.simple_cubic(2, 2, 2, periodic=False))
    systems["cubic8_open"] = s8
    golden["systems"]["cubic8_open"] = {"geometry": geometry_json(s8.geometry), "scale": 1.0, "cutoff": 0.0}
    golden["rewl"].append({"system": "cubic8_open", "config": config_json(c1),
                           "result": result_json(ref.run_rewl(s8, c1))})

    (OUT / "reference_golden.json").write_text(json.dumps(golden, indent=1))
    print("wrote", OUT / "reference_golden.json")


if __name__ == "__main__":
    main()
