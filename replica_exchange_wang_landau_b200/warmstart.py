"""The learned warm start (no counterpart in the reference).

A small MLP, trained on the GPU by the library's own CUDA kernels (csrc/mlp.cu, reached
through the wlg_mlp_* C-ABI), corrects a physics prior for log g(E) of a dipole system.  It
is trained on DOS curves that the plain engine produces on generated systems; for a new
system it predicts log g over the run's grid, and the engine starts its walkers from that
estimate at a small ln f (Engine.warm_start).  Plain Wang-Landau from a flat start stays the
fallback: warm_start_or_flat returns the flat start whenever the prediction is unusable, and
the plain method is the measure of the learned one's error.

Prior: over uniformly random configurations the energy E = sum_{i<j} J_ij s_i s_j has mean 0,
variance sigma^2 = sum_{i<j} J_ij^2 and third cumulant tr(J^3), so
    log g(E) ~ N ln 2 + ln(width) - ln(2 pi sigma^2) / 2 - E^2 / (2 sigma^2)
per bin of the grid.  The network learns the residual log g - prior from
    z = E / sigma, emin / sigma, emax / sigma, skewness tr(J^3) / sigma^3, log(N) / log(1024),
    (E - emin) / (emax - emin), density, nematic order of the easy axes.
Training curves are normalised so that sum_E g(E) = 2^N over the bins the plain run visited.
"""
import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi
from .engine import Engine, RunConfig, System, WlParameters, _check

FEATURES = 8


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Mlp:
    """wlg_mlp: tanh MLP with one output; forward, gradients and Adam on the GPU."""

    def __init__(self, dims: Sequence[int], seed: int = 1):
        self.dims = [int(d) for d in dims]
        self._lib = _abi.load_library()
        d = (C.c_int32 * len(self.dims))(*self.dims)
        h = C.c_void_p()
        _check(self._lib.wlg_mlp_create(len(self.dims) - 1, d, int(seed), C.byref(h)))
        self._h = h

    def close(self) -> None:
        if self._h:
            self._lib.wlg_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def parameter_count(self) -> int:
        return int(self._lib.wlg_mlp_parameter_count(self._h))

    def parameters(self) -> np.ndarray:
        out = np.empty(self.parameter_count, np.float32)
        _check(self._lib.wlg_mlp_get_parameters(self._h, _fptr(out)))
        return out

    def set_parameters(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.parameter_count:
            raise ValueError("parameter count mismatch")
        _check(self._lib.wlg_mlp_set_parameters(self._h, _fptr(p)))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty(x.shape[0], np.float32)
        _check(self._lib.wlg_mlp_forward(self._h, _fptr(x), x.shape[0], _fptr(y)))
        return y

    def gradients(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.empty(self.parameter_count, np.float32)
        loss = C.c_double()
        _check(self._lib.wlg_mlp_gradients(self._h, _fptr(x), _fptr(t), x.shape[0], _fptr(g), C.byref(loss)))
        return loss.value, g

    def train(self, x: np.ndarray, t: np.ndarray, steps: int, learning_rate: float) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_double()
        _check(self._lib.wlg_mlp_train(self._h, _fptr(x), _fptr(t), x.shape[0], int(steps), float(learning_rate),
                                       C.byref(loss)))
        return loss.value


# ---- features and targets ---------------------------------------------------------------


def system_descriptor(system: System) -> dict:
    """Moments of the coupling matrix and geometry descriptors of a dense system."""
    if system.cutoff > 0.0:
        raise ValueError("the warm start supports dense systems")
    g = system.geometry
    n = g.size()
    j = np.asarray(system.couplings("fp64"), dtype=np.float64)[:n, :n]
    sigma = math.sqrt(float(np.sum(np.triu(j, 1) ** 2)))
    kappa3 = float(np.trace(j @ j @ j))
    pos = np.asarray(g.positions, dtype=np.float64)
    box = np.asarray(g.box, dtype=np.float64)
    extent = np.where(box > 0.0, box, np.ptp(pos, axis=0) + 1.0) if g.periodic else np.ptp(pos, axis=0) + 1.0
    density = n / float(np.prod(extent))
    a = np.asarray(g.axes, dtype=np.float64)
    q = 1.5 * (a.T @ a) / n - 0.5 * np.eye(3)
    order = float(np.linalg.eigvalsh(q)[-1])
    return {"n": n, "sigma": sigma, "skew": kappa3 / sigma ** 3 if sigma > 0 else 0.0, "density": density,
            "order": order}


def prior_log_g(desc: dict, emin: float, emax: float, width: float) -> np.ndarray:
    """The Gaussian prior for log g per bin."""
    bins = int(round((emax - emin) / width))
    centre = emin + (np.arange(bins) + 0.5) * width
    s2 = max(desc["sigma"], 1e-12) ** 2
    return desc["n"] * math.log(2.0) + math.log(width) - 0.5 * math.log(2 * math.pi * s2) - centre ** 2 / (2 * s2)


def bin_features(desc: dict, emin: float, emax: float, width: float) -> np.ndarray:
    """Feature rows (bins x FEATURES) of one system on one grid."""
    n = desc["n"]
    sg = max(desc["sigma"], 1e-12)
    bins = int(round((emax - emin) / width))
    centre = emin + (np.arange(bins) + 0.5) * width
    x = np.empty((bins, FEATURES), np.float64)
    x[:, 0] = centre / sg
    x[:, 1] = emin / sg
    x[:, 2] = emax / sg
    x[:, 3] = desc["skew"]
    x[:, 4] = math.log(n) / math.log(1024.0)
    x[:, 5] = (centre - emin) / (emax - emin)
    x[:, 6] = desc["density"]
    x[:, 7] = desc["order"]
    return x


def normalised_log_g(log_g: np.ndarray, valid: np.ndarray, n: int) -> np.ndarray:
    """log g over the valid bins, shifted so that sum g = 2^N (NaN elsewhere)."""
    lg = np.asarray(log_g, dtype=np.float64)
    ok = np.asarray(valid, dtype=bool) & np.isfinite(lg)
    m = lg[ok].max()
    lse = m + math.log(np.exp(lg[ok] - m).sum())
    out = np.full(lg.shape, np.nan)
    out[ok] = lg[ok] - lse + n * math.log(2.0)
    return out


@dataclass
class DosSample:
    """One training curve: a system, its grid and the plain run's log g (with valid bins)."""
    system: System
    emin: float
    emax: float
    width: float
    log_g: np.ndarray
    valid: np.ndarray


def plain_dos(system: System, emin: float, emax: float, width: float, seed: int = 1,
              final_factor: float = 1e-4, walkers: int = 2) -> DosSample:
    """A DOS curve from the plain engine: one window, flat start, 1/t to final_factor."""
    c = RunConfig(emin=emin, emax=emax, bin_width=width, windows=1, walkers=walkers, seed=seed)
    c.wl = WlParameters(0.8, 100, final_factor, 1000, 0, True)
    c.exchange_interval_mcs = 10.0
    c.max_mcs = 1e7
    c.resolve_mcs(system.size())
    with Engine(system, c) as e:
        e.run()
        frag = e.fragment(0, allow_empty=True)
    return DosSample(system, emin, emax, width, np.asarray(frag.log_g, np.float64), np.asarray(frag.valid, bool))


def plain_dos_many(specs: Sequence[tuple], final_factor: float = 1e-4, walkers: int = 2,
                   epoch_attempts: Optional[int] = None) -> list:
    """plain_dos for many (system, emin, emax, width, seed) at once: the engines run side by
    side in one batch (one CUDA-graph launch advances all of them).  epoch_attempts: attempts
    per walker per epoch (default 10 MCS; a fixed count keeps engines of different sizes at the
    same pace in the batch)."""
    from .engine import Batch
    engines = []
    try:
        for system, emin, emax, width, seed in specs:
            c = RunConfig(emin=emin, emax=emax, bin_width=width, windows=1, walkers=walkers, seed=seed)
            c.wl = WlParameters(0.8, 100, final_factor, 1000, 0, True)
            c.exchange_interval_mcs = 10.0
            if epoch_attempts:
                c.exchange_interval_uses_mcs = False
                c.exchange_interval_attempts = int(epoch_attempts)
            c.max_mcs = 1e7
            c.resolve_mcs(system.size())
            engines.append(Engine(system, c))
        with Batch(engines) as batch:
            batch.run()
        out = []
        for (system, emin, emax, width, _), e in zip(specs, engines):
            frag = e.fragment(0, allow_empty=True)
            out.append(DosSample(system, emin, emax, width, np.asarray(frag.log_g, np.float64),
                                 np.asarray(frag.valid, bool)))
        return out
    finally:
        for e in engines:
            e.close()


@dataclass
class WarmStartModel:
    """Feature and target scalings plus the trained network."""
    hidden: tuple = (32, 32)
    seed: int = 1
    x_mean: Optional[np.ndarray] = None
    x_std: Optional[np.ndarray] = None
    t_mean: float = 0.0
    t_std: float = 1.0
    net: Optional[Mlp] = field(default=None, repr=False)
    final_loss: float = math.nan

    def dataset(self, samples: Sequence[DosSample]):
        xs, ts = [], []
        for s in samples:
            desc = system_descriptor(s.system)
            x = bin_features(desc, s.emin, s.emax, s.width)
            t = normalised_log_g(s.log_g, s.valid, desc["n"]) - prior_log_g(desc, s.emin, s.emax, s.width)
            ok = np.isfinite(t)
            xs.append(x[ok])
            ts.append(t[ok])
        return np.concatenate(xs), np.concatenate(ts)

    def fit(self, samples: Sequence[DosSample], steps: int = 4000, learning_rate: float = 3e-3) -> float:
        x, t = self.dataset(samples)
        self.x_mean = x.mean(axis=0)
        self.x_std = np.maximum(x.std(axis=0), 1e-6)
        self.t_mean = float(t.mean())
        self.t_std = max(float(t.std()), 1e-6)
        xn = (x - self.x_mean) / self.x_std
        tn = (t - self.t_mean) / self.t_std
        self.net = Mlp([FEATURES, *self.hidden, 1], seed=self.seed)
        self.final_loss = self.net.train(xn, tn, steps, learning_rate)
        return self.final_loss

    def predict_log_g(self, system: System, emin: float, emax: float, width: float) -> np.ndarray:
        """Predicted log g over every bin of the grid (normalised so that sum g = 2^N)."""
        if self.net is None:
            raise RuntimeError("the warm-start model is not trained")
        desc = system_descriptor(system)
        x = (bin_features(desc, emin, emax, width) - self.x_mean) / self.x_std
        residual = self.net.forward(x).astype(np.float64) * self.t_std + self.t_mean
        return prior_log_g(desc, emin, emax, width) + residual


def warm_start_or_flat(engine: Engine, model: Optional[WarmStartModel], system: System, emin: float, emax: float,
                       width: float, factor: float) -> bool:
    """Starts the engine's walkers from the model's log g at ln f = factor; falls back to the
    plain flat start (and returns False) when there is no model or the prediction is not
    finite."""
    if model is None or model.net is None:
        return False
    lg = model.predict_log_g(system, emin, emax, width)
    if not np.all(np.isfinite(lg)):
        return False
    engine.warm_start(lg - lg.max(), factor)
    return True


def run_to_accuracy(system: System, emin: float, emax: float, width: float, reference_log_g: np.ndarray,
                    tolerance: float, seed: int, model: Optional[WarmStartModel] = None, factor: float = 1e-2,
                    final_factor: float = 1e-6, walkers: int = 2, chunk_epochs: int = 20,
                    max_attempts: int = 200_000_000) -> dict:
    """Time to a given accuracy: one window, 1/t Wang-Landau, flat start (model None) or the
    model's warm start at ln f = factor; every chunk_epochs epochs the merged log g is compared
    with reference_log_g (finite on the reference's occupied bins) as max |d - mean(d)| over
    those bins once all of them are valid.  Returns the attempts per walker and the seconds of
    the run loop until the tolerance was met (None if it never was), and the final error."""
    import time

    c = RunConfig(emin=emin, emax=emax, bin_width=width, windows=1, walkers=walkers, seed=seed)
    c.wl = WlParameters(0.8, 100, final_factor, 1000, 0, True)
    c.exchange_interval_mcs = 10.0
    c.max_mcs = 1e12
    c.resolve_mcs(system.size())
    ref = np.asarray(reference_log_g, dtype=np.float64)
    occ = np.isfinite(ref)

    def error(e: Engine) -> float:
        frag = e.fragment(0, allow_empty=True)
        if not np.all(frag.valid[occ] == 1):
            return math.inf
        d = frag.log_g[occ] - ref[occ]
        return float(np.max(np.abs(d - d.mean())))

    with Engine(system, c) as e:
        warm = warm_start_or_flat(e, model, system, emin, emax, width, factor)
        t0 = time.perf_counter()
        hit_attempts = hit_seconds = None
        err = math.inf
        while True:
            e.run_epochs(chunk_epochs)
            t = e.totals()
            err = error(e)
            per_walker = t["attempted"] // walkers
            if err <= tolerance:
                hit_attempts, hit_seconds = per_walker, time.perf_counter() - t0
                break
            if t["converged"] or per_walker >= max_attempts:
                break
    return {"warm": warm, "attempts": hit_attempts, "seconds": hit_seconds, "final_error": err}


# ---- the learned configuration: generated dilute systems and time to accuracy -----------


def dilute_instance(k: int, seed0: int = 50_000):
    """The k-th generated system of the learned configuration: N uniform in 64..1024, random
    sequential addition in a periodic cube at density 0.3-0.8 (minimum separation 0.8),
    random-sphere axes; one grid over about +-4 sigma of the random-configuration energy
    distribution (sigma^2 = sum_{i<j} J_ij^2) in 200 power-of-two bins.
    Returns (system, emin, emax, width)."""
    from .geometry import random_sequential
    rng = np.random.default_rng(seed0 + k)
    n = int(rng.integers(64, 1025))
    s = System(random_sequential(n, float(rng.uniform(0.3, 0.8)), 0.8, seed=seed0 + k), 1.0, 0.0)
    sigma = math.sqrt(0.5 * float(np.sum(s.couplings("fp64") ** 2)))
    w = 2.0 ** round(math.log2(8.0 * sigma / 200.0))
    return s, -100.0 * w, 100.0 * w, w


def accuracy_error(log_g: np.ndarray, valid: np.ndarray, reference_log_g: np.ndarray) -> float:
    """max |d - mean(d)| with d = log g - reference over the bins the reference found (inf until all of
    them are valid in the run)."""
    ref = np.asarray(reference_log_g, dtype=np.float64)
    occ = np.isfinite(ref)
    if not np.all(np.asarray(valid)[occ] == 1):
        return math.inf
    d = np.asarray(log_g, dtype=np.float64)[occ] - ref[occ]
    return float(np.max(np.abs(d - d.mean())))


EPOCH_ATTEMPTS = 8192  # attempts per walker per epoch of the learned configuration's runs


def single_window_config(emin: float, emax: float, width: float, n: int, seed: int, final_factor: float,
                         walkers: int = 2, precision: str = "fp64") -> RunConfig:
    """One window of `walkers` walkers, 1/t Wang-Landau to final_factor.  The epoch (with one
    window only the interval between checks and launches) is EPOCH_ATTEMPTS attempts whatever
    N is, so that engines of different sizes advanced together in one batch make the same
    number of attempts per launch: the attempts a run needs do not grow with N (the 1/t stage
    takes about bins / ln f of them), so epochs of a fixed number of MCS would hold the small
    systems back to the pace of the largest.  FP64 recompute every 10 MCS for FP32 / BF16."""
    c = RunConfig(emin=emin, emax=emax, bin_width=width, windows=1, walkers=walkers, seed=seed)
    c.wl = WlParameters(0.8, 100, final_factor, 1000, 0, True)
    c.exchange_interval_uses_mcs = False
    c.exchange_interval_attempts = EPOCH_ATTEMPTS
    c.max_mcs = 0.0
    c.coupling_precision = precision
    c.recompute_interval_mcs = 10.0
    c.resolve_mcs(n)
    return c


def batch_to_accuracy(engines: Sequence[Engine], references: Sequence[np.ndarray], tolerance: float,
                      chunk_epochs: int = 8, max_seconds: float = 600.0) -> dict:
    """Advances the engines together (one Batch: one CUDA-graph launch per step for all of them)
    and, every chunk_epochs epochs, measures each engine's error against its reference run.  Returns the
    run seconds and attempts per walker at which each engine first met the tolerance (None if
    not within max_seconds of wall time), the run seconds until all had, and each engine's attempts
    per run second.  Run seconds are the wall time of the run calls (each returns when its epochs
    are done); the accuracy checks between them (a copy of each engine's log g and a comparison on
    the host) measure the run and are not part of it, so they are left out (wall_s includes them)."""
    import time

    from .engine import Batch
    hit_s = [None] * len(engines)
    hit_att = [None] * len(engines)
    errors = [math.inf] * len(engines)
    with Batch(engines) as batch:
        t0 = time.perf_counter()
        run_s = 0.0
        while True:
            t1 = time.perf_counter()
            batch.run_epochs(chunk_epochs)
            run_s += time.perf_counter() - t1
            now = run_s
            for k, (e, ref) in enumerate(zip(engines, references)):
                if hit_s[k] is not None:
                    continue
                frag = e.fragment(0, allow_empty=True)
                errors[k] = accuracy_error(frag.log_g, frag.valid, ref)
                if errors[k] <= tolerance:
                    hit_s[k] = now
                    hit_att[k] = e.totals()["attempted"] // e.walkers
            if all(h is not None for h in hit_s) or time.perf_counter() - t0 > max_seconds:
                break
        wall = time.perf_counter() - t0
    rates = [e.totals()["attempted"] / e.walkers / run_s for e in engines]
    done = [h for h in hit_s if h is not None]
    return {"hit_seconds": hit_s, "hit_attempts_per_walker": hit_att, "final_errors": errors,
            "all_seconds": max(done) if len(done) == len(engines) else None, "reached": len(done),
            "attempts_per_walker_per_s": rates, "elapsed_s": run_s, "wall_s": wall}


def engine_to_accuracy(engine: Engine, reference: np.ndarray, tolerance: float, chunk_epochs: int = 8,
                       max_seconds: float = 120.0) -> dict:
    """One engine alone, chunk_epochs epochs at a time, until its error meets the tolerance; run
    seconds as in batch_to_accuracy (the accuracy checks left out)."""
    import time
    t0 = time.perf_counter()
    run_s = 0.0
    err = math.inf
    while True:
        t1 = time.perf_counter()
        engine.run_epochs(chunk_epochs)
        run_s += time.perf_counter() - t1
        frag = engine.fragment(0, allow_empty=True)
        err = accuracy_error(frag.log_g, frag.valid, reference)
        if err <= tolerance or time.perf_counter() - t0 > max_seconds:
            break
    att = engine.totals()["attempted"] // engine.walkers
    return {"seconds": run_s if err <= tolerance else None, "attempts_per_walker": att if err <= tolerance else None,
            "attempts_per_walker_per_s": att / run_s, "final_error": err, "wall_s": time.perf_counter() - t0}
