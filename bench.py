"""Benchmark: spin-flip attempts/s of the dense REWL workload on B200.

Workload (the configuration the reference's headline metric is quoted on): an 8x8x8 simple
cubic lattice (N = 512), periodic box 8, D = 1, easy axes uniform on the unit sphere
(random_sphere_axes, seed 1), dense FP64 minimum-image couplings; 16 energy windows at 75%
overlap x 8 walkers = 128 walkers; replica exchange every 1 MCS (512 attempts); bins of 0.5
over the pilot range +5% ([-228.5, 228.0], 913 bins; pilot: the reference's `wl_run --pilot`
infinite-temperature walk of 1e5 MCS on this system, seed 1).  Synthetic data: the system
is generated from its seed; no dataset is involved.

A step is `--epochs-per-step` epochs; an epoch is one exchange interval of attempts for
every walker, the walker-local check and one even/odd exchange (run_rewl's loop body).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs an independent replica of the workload (the north
star fixes one GPU per run; windows are not sharded), timed on the device, max over ranks.
"""
from __future__ import annotations

import argparse
import copy
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "spin-flip attempts/s"
UNIT = "attempts/s"
WORKLOAD = ("dense REWL: 8x8x8 simple cubic N=512, periodic box 8, random-sphere axes (seed 1), dense FP64 J; "
            "16 windows x 8 walkers at 75% overlap; exchange every 1 MCS; bin 0.5 on [-228.5, 228.0]")
EMIN, EMAX, WIDTH = -228.5, 228.0, 0.5


def make_workload(seed: int):
    from replica_exchange_wang_landau_b200.engine import RunConfig, System
    from replica_exchange_wang_landau_b200.geometry import simple_cubic_random
    geometry = simple_cubic_random(8, 8, 8, seed=1, periodic=True)
    system = System(geometry, 1.0, 0.0)
    config = RunConfig(emin=EMIN, emax=EMAX, bin_width=WIDTH, windows=16, walkers=8, overlap=0.75, seed=seed,
                       exchange_interval_mcs=1.0)
    config.resolve_mcs(geometry.size())
    return system, config


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def ncu_traffic_per_launch():
    """dram bytes per sweep-kernel launch from the committed ncu summary, if present."""
    p = ROOT / "profiles" / "sweep_dense_split_kernel_rewl_n512.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.file = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.file.flush()
        rows = []
        try:
            for line in Path(self.file.name).read_text().splitlines():
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def flush_l2(torch, buf):
    buf.add_(1.0)  # 256 MiB written: larger than the 126 MB L2


def reduce_over_ranks(dist, device, maxima, sums):
    """The whole job's figures from every rank's: the maximum over ranks of each time, the sum
    over ranks of each count (identity with one process).  Every rank calls it at the same point."""
    if dist is None:
        return [float(x) for x in maxima], [float(x) for x in sums]
    import torch
    t = torch.tensor([float(x) for x in maxima], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(x) for x in sums], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return t.tolist(), c.tolist()


def apply_launch(eng, launch: dict) -> None:
    """Gives an engine the launch shape an autotune report chose."""
    eng.set_launch(launch["walkers_per_block"], launch["epochs_per_graph"])
    if launch["staging_ring"]:
        eng.set_staging_ring(launch["staging_ring"])


def run_ours(args, rank: int, world: int, dist, torch) -> None:
    from replica_exchange_wang_landau_b200 import engine as E
    from replica_exchange_wang_landau_b200._abi import wlg_run_config
    local = int(os.environ.get("LOCAL_RANK", "0"))
    E.set_device(local)
    torch.cuda.set_device(local)
    system, config = make_workload(seed=1 + rank)
    n = system.size()
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    # the launch shape (staging ring, epochs per graph replay) from the engine's autotuner, run on
    # a separate engine of the same system and configuration, so that the timed engine's epochs
    # are the epochs it would run without the tuning
    with E.Engine(system, config) as tuner:
        launch = tuner.autotune(16)
    eng = E.Engine(system, config)
    apply_launch(eng, launch)
    epochs = args.epochs_per_step
    for _ in range(args.warmup):
        eng.time_run(epochs)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    total_ms = 0.0
    attempted = accepted = 0
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush_l2(torch, flush)
            torch.cuda.synchronize()
            # the product path: run_epochs (CUDA-graph replays of [sweep, exchange]) with one
            # CUDA event before and one after on the engine's stream
            t = eng.time_run(epochs)
            total_ms += t["total_ms"]
            attempted += t["attempted"]
            accepted += t["accepted"]
        torch.cuda.synchronize()
    # per-kernel device times for the roofline, on the timed epochs themselves: a second
    # engine with the same system and seed replays the warm-up and then exactly the timed
    # steps' epochs, launched one kernel at a time with CUDA events around every launch.  The
    # trajectories are deterministic, so these are the same attempts (checked below).
    twin = E.Engine(system, config)
    apply_launch(twin, launch)
    for _ in range(args.warmup):
        twin.time_epochs(epochs)
    walk_ms = exch_ms = 0.0
    kt = {"epochs": 0, "attempted": 0, "accepted": 0}
    for _ in range(args.steps):
        flush_l2(torch, flush)
        torch.cuda.synchronize()
        t = twin.time_epochs(epochs)
        walk_ms += t["walk_ms"]
        exch_ms += t["exchange_ms"]
        for key in kt:
            kt[key] += t[key]
    twin.close()
    if (kt["attempted"], kt["accepted"]) != (attempted, accepted):
        raise RuntimeError("the kernel-timing replay did not repeat the timed epochs")
    if dist:
        dist.barrier()
    clock = clocks.summary()
    # max over ranks of the device time; total attempts over ranks
    (total_max, walk_max), (att_all, acc_all) = reduce_over_ranks(dist, "cuda", [total_ms, walk_ms],
                                                                  [attempted, accepted])
    att_all, acc_all = int(att_all), int(acc_all)
    value = att_all / (total_max / 1e3)

    # host wall-clock throughput of the same path (run_epochs), for context
    torch.cuda.synchronize()
    g0 = time.perf_counter()
    before = eng.totals()["attempted"]
    eng.run_epochs(epochs * min(args.steps, 5))
    torch.cuda.synchronize()
    graph_rate = (eng.totals()["attempted"] - before) / (time.perf_counter() - g0)
    active_bins = float(np.mean([st["active_bins"] for st in eng.walker_statistics()]))
    window_bins = float(np.mean([e - b for b, e in (eng.window(k) for k in range(config.windows))]))
    eng.close()

    # e2e through the C-ABI with pinned host buffers: create (H2D geometry) -> run -> fragments (D2H)
    lib = E.load_library()
    pos = torch.from_numpy(system.geometry.positions.copy()).pin_memory()
    axes = torch.from_numpy(system.geometry.axes.copy()).pin_memory()
    from replica_exchange_wang_landau_b200.engine import Geometry, System
    pinned_system = System(Geometry(pos.numpy(), axes.numpy(), system.geometry.box, True), 1.0, 0.0)
    bins = config.bins()
    out_lg = torch.empty(config.windows * bins, dtype=torch.float64).pin_memory()
    out_h = torch.empty(config.windows * bins, dtype=torch.int64).pin_memory()
    out_se = torch.empty(config.windows * bins, dtype=torch.float64).pin_memory()
    out_v = torch.empty(config.windows * bins, dtype=torch.uint8).pin_memory()
    p_lg = C.cast(out_lg.data_ptr(), C.POINTER(C.c_double))
    p_h = C.cast(out_h.data_ptr(), C.POINTER(C.c_uint64))
    p_se = C.cast(out_se.data_ptr(), C.POINTER(C.c_double))
    p_v = C.cast(out_v.data_ptr(), C.POINTER(C.c_uint8))
    e2e_steps = max(1, min(args.steps, 5))
    e2e_time = 0.0
    e2e_attempts = e2e_accepted = 0
    h2d = 2 * n * 3 * 8
    d2h = config.windows * bins * (8 + 8 + 8 + 1)
    for k in range(e2e_steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sys_s = pinned_system._struct()
        cfg_s, keep = config._struct(n)
        handle = C.c_void_p()
        E._check(lib.wlg_engine_create(C.byref(sys_s), C.byref(cfg_s), C.byref(handle)))
        # the tuned staging ring; the graph length stays the default 32 epochs, whose capture costs a
        # fresh engine less than the tuned 64-epoch graphs of the long-running engine
        if launch["staging_ring"]:
            E._check(lib.wlg_engine_set_staging_ring(handle, launch["staging_ring"]))
        ran, done = C.c_uint64(0), C.c_int32(0)
        E._check(lib.wlg_engine_run_epochs(handle, epochs, C.byref(ran), C.byref(done)))
        E._check(lib.wlg_engine_fragments(handle, 0, p_lg, p_h, p_se, p_v))  # every window's fragment
        totals = E._abi.wlg_run_totals()
        E._check(lib.wlg_engine_totals(handle, C.byref(totals)))
        lib.wlg_engine_destroy(handle)
        dt = time.perf_counter() - t0
        if k > 0:  # the first call is a warm-up (module load, kernel attributes)
            e2e_time += dt
            e2e_attempts += totals.attempted
            e2e_accepted += totals.accepted
    (e2e_time_max,), (e2e_attempts_all,) = reduce_over_ranks(dist, "cuda", [e2e_time], [e2e_attempts])
    e2e_value = e2e_attempts_all / e2e_time_max

    # roofline of the sweep kernel: algorithmic bytes = one FP64 J row (N x 8 bytes) per
    # accepted flip (fields, spins and the window's log_g/H live in shared memory)
    peaks = load_peaks()
    launches = args.steps * epochs
    k_launches = max(1, kt["epochs"])
    bytes_per_launch = kt["accepted"] * n * 8 / k_launches
    launch_s = (walk_ms / k_launches) / 1e3
    achieved = bytes_per_launch / launch_s / 1e9
    traffic = ncu_traffic_per_launch()

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu_baseline:
        cpu = cpu_baseline(args.cpu_sample_mcs)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOAD, "walkers": 128, "spins": n, "epochs_per_step": epochs,
                       "attempts_per_step_per_gpu": attempted // args.steps,
                       "l2": "flushed between timed steps (256 MiB write); J (2 MB) is L2-resident within a step",
                       "launch": {k: launch[k] for k in ("walkers_per_block", "epochs_per_graph", "staging_ring")},
                       "launch_chosen_by": "wlg_engine_autotune (16 trial epochs per candidate, two passes) on a "
                                           "separate engine of the same system and configuration",
                       "parallelism": f"{world} independent replica(s), one per GPU"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps, "path": "wlg_engine_create -> wlg_engine_set_staging_ring (the tuned ring) "
                                                "-> wlg_engine_run_epochs -> wlg_engine_fragments "
                                                "(all 16 windows) -> wlg_engine_destroy, pinned host buffers",
                    "acceptance": e2e_accepted / max(1, e2e_attempts),
                    "note": "each step is a fresh engine's first epochs; acceptance, and with it the cost of an "
                            "attempt, differs from the long-running engine of value"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                         "kernel": f"sweep_dense_split_kernel<8, pow2 width> (FP64 dense J, "
                                   f"{launch['staging_ring']}-draw staging ring)", "peak_source": peaks["source"],
                         "bytes_per_launch": bytes_per_launch, "launch_ms": launch_s * 1e3,
                         "acceptance": kt["accepted"] / max(1, kt["attempted"]),
                         "kernel_timing": f"the {k_launches} timed epochs (warm-up excluded), replayed after the "
                                          f"timed region by a second engine with the same seed, one kernel at a time "
                                          f"with CUDA events around each launch; same attempts and accepted flips "
                                          f"as the timed region (checked)"},
            "gpu_launches": 2 * launches,
            "wall_clock_attempts_per_s": graph_rate,
            "clocks": clock,
            "exchange_ms_per_epoch": exch_ms / k_launches,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if world == 1 and not args.skip_extras:
            try:
                line["mixed_precision"] = mixed_precision_lines()
            except Exception as exc:  # reported, never fatal to the headline line
                line["mixed_precision"] = {"error": str(exc)}
            try:
                line["batched_instances"] = batched_instances_line()
            except Exception as exc:
                line["batched_instances"] = {"error": str(exc)}
            try:
                line["csr_batched"] = csr_batched_line()
            except Exception as exc:
                line["csr_batched"] = {"error": str(exc)}
            if cpu:
                try:
                    line["time_to_converge"] = time_to_converge(value, cpu["value"], active_bins, window_bins)
                except Exception as exc:
                    line["time_to_converge"] = {"error": str(exc)}
            try:
                line["time_to_accuracy"] = learned_configuration_line()
            except Exception as exc:
                line["time_to_accuracy"] = {"error": str(exc)}
        print(json.dumps(line))


def _pilot_range(J: np.ndarray, mcs: int, seed: int) -> tuple:
    """wl_run --pilot (apps/wl_run.cpp:84-100) restated: an infinite-temperature walk (every
    single-spin flip accepted) from all spins up, then the visited range padded by 5% each side."""
    n = J.shape[0]
    rng = np.random.default_rng(seed)
    s = np.ones(n)
    h = J @ s
    e = 0.5 * float(s @ h)
    lo = hi = e
    for i in rng.integers(0, n, size=mcs * n):
        e += -2.0 * s[i] * h[i]
        h -= 2.0 * s[i] * J[i]
        s[i] = -s[i]
        lo, hi = min(lo, e), max(hi, e)
    pad = max(1e-12, 0.05 * (hi - lo))
    return lo - pad, hi + pad


def mixed_precision_workload(precisions=("fp64", "fp32", "bf16")):
    """The mixed-precision configuration: a 16x16x16 simple cubic lattice with 40% of the sites
    removed (seeded; N = 2458), slab geometry periodic in x and y (box 16, 16, 0), random-sphere
    axes, dense couplings; 32 windows x 8 walkers at 75% overlap, exchange and FP64 recompute
    every MCS.  The grid is the pilot range of a 100-MCS infinite-temperature walk (the
    reference's pilot, seeded here; its runs use longer walks), in bins of 0.5."""
    from replica_exchange_wang_landau_b200.engine import RunConfig, System
    from replica_exchange_wang_landau_b200.geometry import diluted_cubic
    g = diluted_cubic(16, 16, 16, 0.4, seed=1, periodic=True, box=(16.0, 16.0, 0.0))
    system = System(g, 1.0, 0.0)
    lo, hi = _pilot_range(system.couplings("fp64"), 100, seed=1)
    width = 0.5
    emin, emax = width * np.floor(lo / width), width * np.ceil(hi / width)
    configs = {}
    for precision in precisions:
        config = RunConfig(emin=float(emin), emax=float(emax), bin_width=width, windows=32, walkers=8,
                           overlap=0.75, seed=1, exchange_interval_mcs=1.0)
        config.coupling_precision = precision
        config.recompute_interval_mcs = 1.0
        config.resolve_mcs(system.size())
        configs[precision] = config
    return system, configs


def mixed_precision_lines(epochs: int = 10) -> dict:
    """The mixed-precision configuration with FP64, FP32 and BF16 (+ FP32 row scale) couplings:
    device attempts/s of the product path (sweeps, exchanges and, for FP32 / BF16, the FP64
    recompute and resync after every epoch) and the drift the recompute measured."""
    from replica_exchange_wang_landau_b200.engine import Engine
    out = {}
    system, configs = mixed_precision_workload()
    frags = {}
    for precision, config in [*configs.items(), ("fp64_seed2", None)]:
        if config is None:  # the FP64 run with another seed: the sampling noise of log g
            config = copy.deepcopy(configs["fp64"])
            config.seed = 2
        t0 = time.perf_counter()
        with Engine(system, config) as eng:
            create_s = time.perf_counter() - t0
            eng.time_run(2)
            t = eng.time_run(epochs)
            rep = eng.precision_report()
            keys = ("accepted", "active_bins", "minimum_histogram", "mean_histogram")
            frags[precision] = (eng.fragments(allow_empty=True),
                                [tuple(st[k] for k in keys) for st in eng.walker_statistics()])
            split = eng.time_epochs(4)  # the same path one kernel at a time: sweep / exchange / recompute
        if precision == "fp64_seed2":
            continue
        out[precision] = {"value": t["attempted"] / (t["total_ms"] / 1e3), "unit": UNIT, "epochs_timed": t["epochs"],
                          "ms_per_epoch": t["total_ms"] / max(1, t["epochs"]),
                          "recompute_interval_mcs": 1.0 if precision != "fp64" else None,
                          "recomputes": rep["recomputes"], "max_field_drift": rep["max_field_drift"],
                          "max_energy_drift": rep["max_energy_drift"], "deferred": rep["deferred"],
                          "bin_changes": rep["bin_changes"], "engine_create_s": create_s,
                          "acceptance": t["accepted"] / max(1, t["attempted"]),
                          "ms_per_epoch_split": {
                              "sweep": split["walk_ms"] / max(1, split["epochs"]),
                              "exchange": split["exchange_ms"] / max(1, split["epochs"]),
                              "recompute": (split["total_ms"] - split["walk_ms"] - split["exchange_ms"]) /
                              max(1, split["epochs"])}}
    # log g of each form against the FP64 run with the same seed after the same epochs: per window,
    # max |d - mean(d)| over the bins valid in both; the FP64 run with another seed gives the
    # sampling noise at this point of the run.  With the same seed a narrow-J walker takes the
    # FP64 walker's decisions, draw for draw, until an accumulated field error first moves an
    # energy across a bin edge; "same_decisions_walkers" counts the walkers whose accepted count,
    # active bins and histogram minimum and mean are still the FP64 walker's (their energies
    # differ in the last bits from the first accepted flip on).
    base, base_e = frags["fp64"]
    for name in ("fp32", "bf16", "fp64_seed2"):
        if name not in frags:
            continue
        worst = 0.0
        for fa, fb in zip(frags[name][0], base):
            ok = (fa.valid == 1) & (fb.valid == 1)
            if ok.sum() >= 2:
                d = fa.log_g[ok] - fb.log_g[ok]
                worst = max(worst, float(np.max(np.abs(d - d.mean()))))
        same = sum(1 for a, b in zip(frags[name][1], base_e) if a == b)
        key = name if name in out else "fp64_other_seed"
        out.setdefault(key, {}).update({"max_abs_dlog_g_vs_fp64": worst, "same_decisions_walkers": same,
                                        "walkers": len(base_e), "after_epochs": epochs + 2})
    out["workload"] = ("16x16x16 simple cubic, 40% of sites removed (seed 1, N = 2458), slab box (16, 16, 0), "
                       "random-sphere axes, dense J; 32 windows x 8 walkers, exchange and FP64 recompute every MCS; "
                       f"grid [{config.emin:g}, {config.emax:g}] in bins of {config.bin_width:g}")
    return out


def batched_instances_line(count: int = 256, epochs: int = 32) -> dict:
    """The batched configuration's scale: `count` dilute random systems (N uniform in 64..1024,
    random sequential addition in a periodic cube at density 0.3-0.8, minimum separation 0.8,
    random-sphere axes; seeded), each one window x 2 walkers over about +-4 sigma of its
    random-configuration energy distribution in 200 power-of-two bins, in epochs of 8192 attempts
    per walker, advanced together by single graph launches (Batch) and, for comparison, one engine
    after the other; wall-clock attempts/s of both, host synchronisation included."""
    import math
    from replica_exchange_wang_landau_b200.engine import Batch, Engine, RunConfig, System
    from replica_exchange_wang_landau_b200.geometry import random_sequential
    from replica_exchange_wang_landau_b200.warmstart import EPOCH_ATTEMPTS
    t0 = time.perf_counter()
    engines, sizes = [], []
    try:
        for k in range(count):
            rng = np.random.default_rng(50_000 + k)
            n = int(rng.integers(64, 1025))
            s = System(random_sequential(n, float(rng.uniform(0.3, 0.8)), 0.8, seed=50_000 + k), 1.0, 0.0)
            sigma = math.sqrt(0.5 * float(np.sum(s.couplings("fp64") ** 2)))
            w = 2.0 ** round(math.log2(8.0 * sigma / 200.0))
            c = RunConfig(emin=-100.0 * w, emax=100.0 * w, bin_width=w, windows=1, walkers=2, seed=k + 1)
            # epochs of a fixed number of attempts (with one window an epoch only sets when the
            # check runs and how much a launch advances), so that systems of every size keep pace
            c.exchange_interval_uses_mcs = False
            c.exchange_interval_attempts = EPOCH_ATTEMPTS
            c.resolve_mcs(n)
            engines.append(Engine(s, c))
            sizes.append(n)
        setup_s = time.perf_counter() - t0

        def attempted() -> int:
            return sum(e.totals()["attempted"] for e in engines)

        with Batch(engines) as batch:
            batch.run_epochs(16)  # warm
            a0, t1 = attempted(), time.perf_counter()
            batch.run_epochs(epochs)
            batched = (attempted() - a0) / (time.perf_counter() - t1)
        a0, t1 = attempted(), time.perf_counter()
        for e in engines:
            e.run_epochs(epochs)
        sequential = (attempted() - a0) / (time.perf_counter() - t1)
    finally:
        for e in engines:
            e.close()
    return {"value": batched, "unit": UNIT, "systems": count, "walkers": 2 * count,
            "spins": {"min": min(sizes), "mean": float(np.mean(sizes)), "max": max(sizes)},
            "sequential_attempts_per_s": sequential, "batched_over_sequential": batched / sequential,
            "epochs": epochs, "setup_s": setup_s, "timing": "wall clock, host synchronisation included"}


def csr_cpu_baseline(system, config, attempts: int = 2_000_000) -> dict:
    """The reference on the CSR configuration, in steady state: one reference walker
    (WangLandauWalker, compiled from the reference's sources) on the same system, grid and a
    window in the middle of the range.  Its construction (CsrCouplings built from the
    geometry, then local_fields and total_energy, which read J through Couplings::at and so
    cost O(N^2 z), OpenMP over rows) is timed and reported apart; then `attempts` attempts are
    timed on one core.  The full configuration (1024 walkers) cannot run on the host in a
    bounded sample: construction alone is this cost once per walker."""
    from oracle.oracle import Reference
    ref = Reference()
    threads = ref.set_threads(os.cpu_count() or 1)
    bins = int(round((config.emax - config.emin) / config.bin_width))
    middle = int(np.floor((0.0 - config.emin) / config.bin_width))
    window = (max(0, middle - 30), min(bins, middle + 30))
    t0 = time.perf_counter()
    walker = ref.walker(system, 0, config.emin, config.emax, config.bin_width, window, config.wl, config.seed)
    construct_s = time.perf_counter() - t0
    try:
        walker.run_attempts(attempts // 10)  # warm
        a0 = walker.counters()[0]
        t0 = time.perf_counter()
        walker.run_attempts(attempts)
        dt = time.perf_counter() - t0
        acc = walker.counters()
        rate = (acc[0] - a0) / dt
    finally:
        walker.close()
    return {"value": rate, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"one reference walker on the same system and grid, window bins {window[0]}-{window[1]}, "
                      f"{attempts} attempts timed on one core after construction",
            "construction_s": construct_s, "construction_threads": threads,
            "acceptance": acc[1] / max(1, acc[0])}


def csr_batched_line(epochs: int = 40, pilot_mcs: float = 20.0, with_cpu_baseline: bool = True) -> dict:
    """The CSR configuration: 32x32x32 periodic simple cubic (N = 32768), cutoff 3.0 (122
    neighbours), easy axes +z, FP32 CSR values with FP64 fields, 64 adaptive windows x 16
    walkers = 1024 walkers.  The windows and the walkers' seeds come from two adaptive-window
    pilot rounds of pilot_mcs MCS each on the engine (pilot statistics on); the production run
    then starts from them and is timed on the device over graph-replayed epochs of 0.05 MCS
    (1638 attempts per walker)."""
    from replica_exchange_wang_landau_b200.adaptive import AdaptiveParameters, adaptive_pilot
    from replica_exchange_wang_landau_b200.engine import Engine, Geometry, RunConfig, System, WlParameters
    g = Geometry.simple_cubic(32, 32, 32, 1.0, (0.0, 0.0, 1.0), True)
    g.box = (32.0, 32.0, 32.0)
    system = System(g, 1.0, 3.0)
    c = RunConfig(emin=-2144.0, emax=1932.0, bin_width=4.0, windows=64, walkers=16, overlap=0.75, seed=3)
    c.wl = WlParameters(0.8, 100, 1e-8, 1000, 0, True)
    c.coupling_precision = "fp32"
    c.recompute_interval_mcs = 10.0
    c.exchange_interval_mcs = 0.05
    c.resolve_mcs(system.size())
    t0 = time.perf_counter()
    windows, seeds = adaptive_pilot(system, c, AdaptiveParameters(iterations=2, pilot_mcs=pilot_mcs), log=None)
    pilot_s = time.perf_counter() - t0
    c.explicit_windows = windows
    c.initial_spins_by_walker = seeds
    widths = [e - b for b, e in windows]
    t0 = time.perf_counter()
    with Engine(system, c) as e:
        create_s = time.perf_counter() - t0
        e.time_run(8)
        t = e.time_run(epochs)
        rep = e.precision_report()
    cpu = None
    if with_cpu_baseline:
        try:
            cpu = csr_cpu_baseline(system, c)
        except Exception as exc:  # reported, never fatal to the line
            cpu = {"error": str(exc)}
    return {"value": t["attempted"] / (t["total_ms"] / 1e3), "unit": UNIT, "walkers": 1024, "spins": system.size(),
            "cpu_baseline": cpu, "neighbours": 122, "couplings": "fp32 CSR, fp64 fields",
            "windows": {"count": len(windows), "adaptive_rounds": 2, "pilot_mcs_per_round": pilot_mcs,
                        "pilot_s": pilot_s, "min_bins": min(widths), "max_bins": max(widths),
                        "seeded_walkers": sum(1 for x in seeds if x is not None)},
            "epochs_timed": t["epochs"], "ms_per_epoch": t["total_ms"] / max(1, t["epochs"]),
            "engine_create_s": create_s, "acceptance": t["accepted"] / max(1, t["attempted"]),
            "max_field_drift": rep["max_field_drift"]}


def learned_configuration_line(tolerance: float = 0.02, start_factor: float = 1e-3, long_run_factor: float = 3e-6,
                               sequential_sample: int = 8, cpu_sample: int = 8) -> dict:
    """The learned configuration, time to accuracy: 256 generated dilute systems (N uniform in
    64..1024, random sequential addition at density 0.3-0.8, random-sphere axes; one window of 2
    walkers over about +-4 sigma in 200 bins).  The warm-start network is trained on the GPU on
    plain-run DOS curves (ln f = 1e-4) of the first 200; the other 56 are held out.  Each held-out
    system's reference is a long plain FP64 run of its own (flat start, other seeds, ln f =
    long_run_factor).  Time until max |d log g| <= tolerance against that run, for:
      plain_sequential -- the plain FP64 GPU form: flat start, one engine at a time (measured on
                          `sequential_sample` systems, the total for 56 scaled from their mean);
      plain_batched    -- the same engines advanced together in one batch;
      learned_batched  -- batched, FP64, learned warm start at ln f = start_factor continuing
                          the 1/t schedule;
      combined         -- batched, FP32 couplings with an FP64 recompute every epoch, learned
                          warm start (the batched + mixed-precision + learned form).
    Times are run seconds: the wall time of the run calls, which return when their epochs are
    done; the accuracy checks between them (every 8 epochs, a copy of each system's log g and a
    comparison with its reference on the host) are the measurement's, not the method's, and are
    left out of every arm alike (each arm's wall time with them is reported beside).
    Time to ln f <= 1e-8 of each arm is extrapolated from its measured attempts per walker per
    second (1/t: active bins / 1e-8 attempts per walker, less the continued schedule's offset).
    The reference's run_rewl (compiled from its sources, 2 walkers on 2 host threads) is timed
    on the systems the sequential arm timed; its time to the tolerance is each plain run's
    attempts per walker over the reference's rate on that system, 56 systems on all host cores."""
    from replica_exchange_wang_landau_b200.engine import Engine
    from replica_exchange_wang_landau_b200.warmstart import (EPOCH_ATTEMPTS, WarmStartModel, batch_to_accuracy,
                                                             dilute_instance, engine_to_accuracy, plain_dos_many,
                                                             single_window_config)
    t0 = time.perf_counter()
    systems = [dilute_instance(k) for k in range(256)]
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    train = plain_dos_many([(s, lo, hi, w, k + 1) for k, (s, lo, hi, w) in enumerate(systems[:200])], final_factor=1e-4,
                           epoch_attempts=EPOCH_ATTEMPTS)
    curves_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    model = WarmStartModel(hidden=(32, 32), seed=3)
    loss = model.fit(train, steps=4000, learning_rate=3e-3)
    fit_s = time.perf_counter() - t0
    held = systems[200:]
    t0 = time.perf_counter()
    long_runs = plain_dos_many([(s, lo, hi, w, 10_000 + k) for k, (s, lo, hi, w) in enumerate(held)],
                            final_factor=long_run_factor, epoch_attempts=EPOCH_ATTEMPTS)
    long_run_s = time.perf_counter() - t0
    references = [np.where(d.valid, d.log_g, np.nan) for d in long_runs]
    # the learned prior's own error, before any sampling
    prior_err = []
    for (s, lo, hi, w), ref in zip(held, references):
        lg = model.predict_log_g(s, lo, hi, w)
        prior_err.append(float(np.max(np.abs((lg - ref)[np.isfinite(ref)] -
                                             np.nanmean(lg[np.isfinite(ref)] - ref[np.isfinite(ref)])))))

    def engines(precision: str, learned: bool) -> list:
        out = []
        for k, (s, lo, hi, w) in enumerate(held):
            e = Engine(s, single_window_config(lo, hi, w, s.size(), 20_000 + k, 1e-8, precision=precision))
            if learned:
                lg = model.predict_log_g(s, lo, hi, w)
                e.warm_start(lg - lg.max(), start_factor, continue_schedule=True)
            out.append(e)
        return out

    def to_ln_f_1e8(engs, rates) -> float:
        # the batch runs every system at once: the slowest one sets the time (the continued
        # schedule's offset, window bins / 1e-3, is 1e-5 of active / 1e-8 and is left out)
        need = [float(np.mean([x["active_bins"] for x in e.walker_statistics()])) / 1e-8 for e in engs]
        return max(n / r for n, r in zip(need, rates))

    arms = {}
    for name, precision, learned in (("plain_batched", "fp64", False), ("learned_batched", "fp64", True),
                                     ("combined", "fp32", True)):
        engs = engines(precision, learned)
        try:
            r = batch_to_accuracy(engs, references, tolerance, max_seconds=150.0)
            r["ln_f_1e-8_s_extrapolated"] = to_ln_f_1e8(engs, r["attempts_per_walker_per_s"])
            if precision != "fp64":
                reps = [e.precision_report() for e in engs]
                r["max_field_drift"] = max(x["max_field_drift"] for x in reps)
                r["bin_changes"] = sum(x["bin_changes"] for x in reps)
        finally:
            for e in engs:
                e.close()
        hits = [h for h in r["hit_attempts_per_walker"] if h is not None]
        times = sorted(h for h in r["hit_seconds"] if h is not None)
        p90 = times[int(np.ceil(0.9 * len(held))) - 1] if len(times) >= np.ceil(0.9 * len(held)) else None
        arms[name] = {"seconds_all": r["all_seconds"], "seconds_90pct": p90, "reached": r["reached"],
                      "median_attempts_per_walker": float(np.median(hits)) if hits else None,
                      "median_hit_seconds": float(np.median([h for h in r["hit_seconds"] if h is not None]))
                      if hits else None,
                      "max_final_error": max(r["final_errors"]),
                      "ln_f_1e-8_s_extrapolated": r["ln_f_1e-8_s_extrapolated"],
                      "wall_s_with_checks": r["wall_s"],
                      **({k: r[k] for k in ("max_field_drift", "bin_changes") if k in r})}
    seq = []
    for k in range(sequential_sample):
        s, lo, hi, w = held[k]
        with Engine(s, single_window_config(lo, hi, w, s.size(), 20_000 + k, 1e-8)) as e:
            r = engine_to_accuracy(e, references[k], tolerance, max_seconds=40.0)
            active = float(np.mean([x["active_bins"] for x in e.walker_statistics()]))
        r["ln_f_1e-8_s"] = active / 1e-8 / r["attempts_per_walker_per_s"]
        r["active_bins"] = active
        seq.append(r)
    ok = [r for r in seq if r["seconds"] is not None]
    per_system = float(np.mean([r["seconds"] for r in ok])) if ok else None
    arms["plain_sequential"] = {
        "systems_timed": len(seq), "reached": len(ok), "mean_seconds_per_system": per_system,
        "mean_wall_s_with_checks_per_system": float(np.mean([r["wall_s"] for r in seq])),
        "seconds_all_56_scaled": per_system * len(held) if per_system else None,
        "seconds_90pct_scaled": per_system * np.ceil(0.9 * len(held)) if per_system else None,
        "median_attempts_per_walker": float(np.median([r["attempts_per_walker"] for r in ok])) if ok else None,
        "ln_f_1e-8_s_extrapolated_all_56": float(np.mean([r["ln_f_1e-8_s"] for r in seq])) * len(held)}
    # the reference on the host: its rate on each system the sequential arm timed, applied to the
    # attempts that system's plain run needed; 56 systems over the host cores, two threads each
    cpu = None
    try:
        from oracle.oracle import Reference
        ref = Reference()
        threads = ref.set_threads(2)
        seconds, rates, ln_f = [], [], []
        for k in range(min(cpu_sample, len(seq))):
            s, lo, hi, w = held[k]
            c = single_window_config(lo, hi, w, s.size(), 20_000 + k, 1e-8)
            c.max_mcs = 2000.0
            c.resolved_spin_count = 0
            c.resolve_mcs(s.size())
            t1 = time.perf_counter()
            rr = ref.run_rewl(s, c)
            rate = rr.attempted / 2 / (time.perf_counter() - t1)
            rates.append(rate)
            if seq[k]["attempts_per_walker"]:
                seconds.append(seq[k]["attempts_per_walker"] / rate)
            ln_f.append(seq[k]["active_bins"] / 1e-8 / rate)
        parallel = max(1, (os.cpu_count() or 2) // 2)
        cpu = {"attempts_per_walker_per_s": {"min": min(rates), "mean": float(np.mean(rates)), "max": max(rates)},
               "threads_per_system": threads, "systems_in_parallel": parallel,
               "seconds_all_56_extrapolated": float(np.mean(seconds)) * len(held) / parallel if seconds else None,
               "seconds_90pct_extrapolated": float(np.mean(seconds)) * np.ceil(0.9 * len(held)) / parallel
               if seconds else None,
               "ln_f_1e-8_s_all_56_extrapolated": float(np.mean(ln_f)) * len(held) / parallel,
               "sample": f"reference run_rewl (oracle/_ref), 2 walkers on {threads} threads, 2000 MCS, on the "
                         f"{len(rates)} systems the sequential arm timed; each system's time = the plain run's "
                         f"attempts per walker / the reference's rate on it"}
    except Exception as exc:
        cpu = {"error": str(exc)}
    # ratios on the time until 90% of the held-out systems met the tolerance (robust to a system
    # that a capped arm did not finish); the all-systems times are reported beside them
    comb = arms["combined"]["seconds_90pct"]
    seq_all = arms["plain_sequential"]["seconds_90pct_scaled"]
    out = {"tolerance": tolerance, "criterion": "max |d log g - mean| against the system's own long plain FP64 run",
           "systems": 256, "trained_on": 200, "held_out": len(held), "start_factor": start_factor,
           "long_run_final_factor": long_run_factor,
           "training": {"curves": len(train), "final_loss": loss, "curve_seconds": curves_s, "fit_seconds": fit_s},
           "setup_s": setup_s, "long_run_s": long_run_s,
           "prior_error": {"median": float(np.median(prior_err)), "max": float(np.max(prior_err))},
           "arms": arms, "reference_cpu": cpu,
           "combined_over_plain_sequential": seq_all / comb if (seq_all and comb) else None,
           "combined_over_plain_batched": (arms["plain_batched"]["seconds_90pct"] / comb)
           if (comb and arms["plain_batched"]["seconds_90pct"]) else None,
           "ratio_basis": "time until 90% of the 56 held-out systems met the tolerance",
           "epoch_attempts": EPOCH_ATTEMPTS}
    out["target_10x_met"] = bool(out["combined_over_plain_sequential"] and out["combined_over_plain_sequential"] >= 10)
    return out


def c1_config():
    """The plain CPU-runnable configuration: 2x2x2 open simple cubic (N = 8), +z axes, dense FP64
    J, grid [-20, 20] in bins of 0.25, 1 window x 2 walkers, flatness 0.8 then 1/t to ln f = 1e-8,
    seed 1234 (the reference's other defaults)."""
    from replica_exchange_wang_landau_b200.engine import Geometry, RunConfig, System
    g = Geometry.simple_cubic(2, 2, 2, 1.0, (0.0, 0.0, 1.0), False)
    c = RunConfig(emin=-20.0, emax=20.0, bin_width=0.25, windows=1, walkers=2, seed=1234)
    c.wl.final_factor = 1e-8
    c.resolve_mcs(g.size())
    return System(g, 1.0, 0.0), c


def c1_converged_line() -> dict:
    """The plain configuration run to ln f <= 1e-8 and timed, not extrapolated: the engine on the
    GPU (the single-window kernel) and, started at the same moment, the reference's own wl_run
    on two host threads (one per walker) with the same command-line configuration.  Each run's
    merged log g is compared with the exact density of states (enumeration of the 256
    configurations) as max |d - mean(d)| over the exactly occupied bins."""
    from oracle.oracle import Oracle
    from replica_exchange_wang_landau_b200.engine import Engine
    system, config = c1_config()
    config.max_mcs = 0.0
    config.resolved_spin_count = 0
    config.resolve_mcs(system.size())
    counts = Oracle().exact_counts(system, config.emin, config.emax, config.bin_width)
    occ = counts > 0
    exact = np.log(counts[occ].astype(float))

    def error(log_g) -> float:
        d = np.asarray(log_g, dtype=np.float64)[occ] - exact
        return float(np.max(np.abs(d - d.mean())))

    tmp = tempfile.TemporaryDirectory()
    ref = None
    if REFERENCE_WL_RUN.exists():
        cmd = [str(REFERENCE_WL_RUN), "--nx", "2", "--ny", "2", "--nz", "2", "--periodic", "false", "--emin", "-20",
               "--emax", "20", "--bin-width", "0.25", "--windows", "1", "--walkers", "2", "--final-factor", "1e-8",
               "--seed", "1234", "--max-mcs", "0", "--output", str(Path(tmp.name) / "c1")]
        ref = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                               env=dict(os.environ, OMP_NUM_THREADS="2"))
    t0 = time.perf_counter()
    with Engine(system, config) as e:
        timing = e.time_run(1 << 40)
        gpu_wall = time.perf_counter() - t0
        totals = e.totals()
        frag = e.fragments()[0]
    out = {"workload": "2x2x2 open simple cubic, +z axes, dense FP64 J, [-20, 20] in bins of 0.25, 1 window x 2 "
                       "walkers, 1/t to ln f = 1e-8, seed 1234",
           "gpu": {"wall_s": gpu_wall, "device_s": timing["total_ms"] / 1e3, "converged": bool(totals["converged"]),
                   "attempts_per_walker": totals["attempted"] // 2,
                   "max_abs_dlog_g_vs_exact": error(frag.log_g)}}
    if ref is not None:
        stdout, _ = ref.communicate(timeout=7200)
        summary = parse_wl_run_summary(stdout)
        dos = np.genfromtxt(Path(tmp.name) / "c1_window_0.csv", delimiter=",", names=True)
        lg = np.full(config.bins(), np.nan)
        lg[dos["bin"].astype(int)] = dos["log_g"]
        out["reference_cpu"] = {"elapsed_s": float(summary["elapsed_seconds"]), "threads": 2,
                                "converged": summary["converged"] == "yes",
                                "attempts_per_walker": int(summary["attempted_flips"]) // 2,
                                "max_abs_dlog_g_vs_exact": error(lg),
                                "program": "the reference's wl_run (oracle/_ref), OpenMP over the two walkers"}
    tmp.cleanup()
    return out


def time_to_converge(value: float, cpu_value: float, active_bins: float, window_bins: float) -> dict:
    """Time to ln f <= 1e-8 as an extrapolation: in the 1/t stage ln f = active bins / attempts
    per walker, so a walker converges after active_bins / 1e-8 attempts; divided by the measured
    attempts/s per walker.  Walkers run side by side (on the GPU all at once; on the host over
    its cores), so the time is that of one walker at the per-walker rate.  The dense REWL
    workload uses this run's rates (active bins now: a lower bound; window bins: an upper one);
    the N = 8 configuration measures its own rates (2 walkers) on the GPU and on the host."""
    from replica_exchange_wang_landau_b200.engine import Engine
    from oracle.oracle import Reference
    out = {"method": "extrapolation: (active bins / 1e-8) attempts per walker / measured attempts per walker per s"}
    per_walker_gpu, per_walker_cpu = value / 128, cpu_value / 128
    out["dense_rewl_512"] = {"attempts_per_walker": [active_bins / 1e-8, window_bins / 1e-8],
                             "gpu_s": [active_bins / 1e-8 / per_walker_gpu, window_bins / 1e-8 / per_walker_gpu],
                             "reference_cpu_s": [active_bins / 1e-8 / per_walker_cpu,
                                                 window_bins / 1e-8 / per_walker_cpu]}
    system, config = c1_config()
    with Engine(system, config) as eng:
        eng.time_run(20)
        t = eng.time_run(400)
        gpu_rate = t["attempted"] / config.walkers / (t["total_ms"] / 1e3)
        active = float(np.mean([st["active_bins"] for st in eng.walker_statistics()]))
    ref = Reference()
    used = ref.set_threads(config.walkers)
    cfg = copy.deepcopy(config)
    cfg.max_mcs = 2_000_000.0
    cfg.resolved_spin_count = 0
    cfg.resolve_mcs(system.size())
    t0 = time.perf_counter()
    r = ref.run_rewl(system, cfg)
    cpu_rate = r.attempted / config.walkers / (time.perf_counter() - t0)
    need = active / 1e-8
    out["c1_n8"] = {"active_bins": active, "attempts_per_walker": need, "gpu_attempts_per_walker_per_s": gpu_rate,
                    "reference_cpu_attempts_per_walker_per_s": cpu_rate, "reference_threads": used,
                    "gpu_s": need / gpu_rate, "reference_cpu_s": need / cpu_rate}
    return out


# The reference's own program, compiled unmodified from its sources by oracle/Makefile, and
# the workload's geometry in the reference's CSV format (written from
# simple_cubic_random(8, 8, 8, seed=1); tests/test_bench_workload.py checks that the file
# holds exactly the doubles the generator gives).
REFERENCE_WL_RUN = ROOT / "oracle" / "_ref" / "wl_run"
WORKLOAD_CSV = ROOT / "oracle" / "workloads" / "dense_rewl_8x8x8_seed1.csv"


def reference_wl_run_command(mcs: float, seed: int, output_prefix: str) -> list:
    """wl_run's command line for the dense REWL workload (the options of src/io.cpp:300-361)."""
    return [str(REFERENCE_WL_RUN), "--geometry", str(WORKLOAD_CSV), "--box-x", "8", "--box-y", "8", "--box-z", "8",
            "--periodic", "true", "--coupling", "1", "--emin", repr(EMIN), "--emax", repr(EMAX),
            "--bin-width", repr(WIDTH), "--windows", "16", "--walkers", "8", "--overlap", "0.75",
            "--exchange-interval-mcs", "1", "--max-mcs", f"{mcs:g}", "--seed", str(seed), "--output", output_prefix]


def parse_wl_run_summary(stdout: str) -> dict:
    """The key=value summary line wl_run prints after run_rewl (apps/wl_run.cpp:190-197)."""
    for line in stdout.splitlines():
        if line.startswith("attempted_flips="):
            return dict(item.split("=", 1) for item in line.split())
    raise RuntimeError("wl_run printed no summary line")


def reference_rate(mcs: float, threads: int, seed: int = 1):
    """One run of the reference's unmodified wl_run on the workload: (attempts, seconds of
    run_rewl as wl_run measures it -- walker construction included, J build and output
    excluded, threads)."""
    with tempfile.TemporaryDirectory() as d:
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        res = subprocess.run(reference_wl_run_command(mcs, seed, str(Path(d) / "ref")), capture_output=True,
                             text=True, env=env, timeout=1800)
    if res.returncode not in (0, 2):  # 2 = max-mcs reached before the final factor
        raise RuntimeError(f"wl_run failed ({res.returncode}): {res.stderr.strip()[-500:]}")
    summary = parse_wl_run_summary(res.stdout)
    return int(summary["attempted_flips"]), float(summary["elapsed_seconds"]), threads


def cpu_baseline(sample_mcs: float) -> dict:
    threads = os.cpu_count() or 1
    attempted, dt, used = reference_rate(sample_mcs, threads)
    return {"value": attempted / dt, "unit": UNIT, "cores": used, "kind": "reference",
            "sample": f"the reference's wl_run (oracle/_ref, compiled unmodified from its sources, OpenMP over walkers) "
                      f"on the same system (CSV) and 16x8 walkers, {sample_mcs:g} MCS per walker; run_rewl time as "
                      f"wl_run reports it, walker construction included: {dt:.2f} s"}


def run_reference(args, rank: int) -> None:
    """The reference arm: the reference's own wl_run program (its public command line and
    stock code path, nothing of this repository's engine) on the workload, every host core."""
    if rank != 0:
        return
    if not REFERENCE_WL_RUN.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/wl_run was not built"}))
        return
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        reference_rate(args.reference_step_mcs, threads)
    total_t = 0.0
    total_a = 0
    used = threads
    for _ in range(args.steps):
        a, dt, used = reference_rate(args.reference_step_mcs, threads)
        total_t += dt
        total_a += a
    value = total_a / total_t
    sample = (f"the reference's wl_run per step (oracle/_ref, compiled unmodified from its sources, OpenMP over "
              f"walkers) on the same system (CSV) and 16x8 walkers, {args.reference_step_mcs:g} MCS per walker per "
              f"step; run_rewl time as wl_run reports it, walker construction included")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": WORKLOAD, "walkers": 128, "spins": 512},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--epochs-per-step", type=int, default=100)
    ap.add_argument("--cpu-sample-mcs", type=float, default=400.0)
    ap.add_argument("--reference-step-mcs", type=float, default=50.0)
    ap.add_argument("--skip-cpu-baseline", action="store_true")
    ap.add_argument("--skip-extras", action="store_true",
                    help="skip the mixed-precision lines and the learned-vs-plain time to accuracy")
    ap.add_argument("--batched-only", action="store_true",
                    help="print only the batched-instances line (256 dilute systems, N 64..1024)")
    ap.add_argument("--mixed-only", action="store_true",
                    help="print only the mixed-precision configuration's lines (N = 2458, FP64 / FP32 / BF16)")
    ap.add_argument("--csr-only", action="store_true",
                    help="print only the CSR configuration's line (the 32^3 lattice, 1024 walkers)")
    ap.add_argument("--c1-converge", action="store_true",
                    help="run the plain 8-spin configuration to ln f <= 1e-8 on the GPU and the reference's wl_run "
                         "on the host at the same time, and print both (takes minutes)")
    ap.add_argument("--learned-only", action="store_true",
                    help="print only the learned configuration's time to accuracy (256 dilute systems)")
    args = ap.parse_args()
    if args.csr_only:
        print(json.dumps({"csr_batched": csr_batched_line()}))
        return
    if args.c1_converge:
        print(json.dumps({"c1_converged": c1_converged_line()}))
        return
    if args.learned_only:
        print(json.dumps({"time_to_accuracy": learned_configuration_line()}))
        return
    if args.batched_only:
        print(json.dumps({"batched_instances": batched_instances_line()}))
        return
    if args.mixed_only:
        print(json.dumps({"mixed_precision": mixed_precision_lines()}))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as td
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = td
    try:
        run_ours(args, rank, world, dist, torch)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
