"""The learned warm start: the CUDA network against its FP64 checker, training, the engine's
warm-start entry point, and what the trained network gains over plain Wang-Landau."""
from __future__ import annotations

import itertools
import math

import numpy as np
import pytest

from helpers import results_equal
from oracle import mlp_oracle
from replica_exchange_wang_landau_b200.engine import Engine, Geometry, InvalidArgument, LogicError, RunConfig, System
from replica_exchange_wang_landau_b200.geometry import random_sequential
from replica_exchange_wang_landau_b200.warmstart import Mlp, WarmStartModel, plain_dos_many, run_to_accuracy

pytestmark = pytest.mark.gpu


def test_gradients_match_fp64_checker():
    rng = np.random.default_rng(1)
    dims = [8, 32, 32, 1]
    net = Mlp(dims, seed=7)
    x = rng.normal(size=(300, 8)).astype(np.float32)
    t = rng.normal(size=300).astype(np.float32)
    p = net.parameters()
    loss, g = net.gradients(x, t)
    loss64, g64 = mlp_oracle.loss_and_gradients(p.astype(np.float64), dims, x.astype(np.float64),
                                                t.astype(np.float64))
    assert abs(loss - loss64) <= 1e-5 * loss64
    assert np.max(np.abs(g - g64)) <= 1e-4 * np.max(np.abs(g64))
    y = net.forward(x)
    y64 = mlp_oracle.forward(p.astype(np.float64), dims, x.astype(np.float64))[-1][:, 0]
    assert np.max(np.abs(y - y64)) <= 1e-5 * max(1.0, np.max(np.abs(y64)))
    again = net.gradients(x, t)[1]
    assert np.array_equal(again, g)  # deterministic reductions


def test_training_fits_a_smooth_curve():
    x = np.linspace(-1, 1, 400, dtype=np.float32)[:, None].repeat(8, axis=1)
    t = (np.sin(3 * x[:, 0]) * 0.5).astype(np.float32)
    net = Mlp([8, 32, 32, 1], seed=2)
    before = net.gradients(x, t)[0]
    after = net.train(x, t, steps=2000, learning_rate=3e-3)
    assert after < 1e-3 and after < 0.01 * before


def test_warm_start_entry_point():
    s = System(Geometry.simple_cubic(2, 2, 2, 1.0, (0, 0, 1), False))
    c = RunConfig(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=2, seed=3).resolve_mcs(8)
    with Engine(s, c) as e:
        with pytest.raises(InvalidArgument):
            e.warm_start(np.zeros(e.bins - 1), 1e-2)
        with pytest.raises(InvalidArgument):
            e.warm_start(np.zeros(e.bins), 0.0)
        lg = np.linspace(0.0, 3.0, e.bins)
        e.warm_start(lg, 1e-2)
        snap = e.snapshot(0)
        assert np.array_equal(snap.log_g, lg) and snap.factor == 1e-2 and snap.attempted == 0
        e.run_epochs(1)
        with pytest.raises(LogicError):
            e.warm_start(lg, 1e-2)


def _cluster(k: int) -> System:
    rng = np.random.default_rng(k)
    n = int(rng.integers(8, 13))
    return System(random_sequential(n, float(rng.uniform(0.3, 0.8)), 0.8, seed=k), 1.0, 0.0)


def _grid(s: System):
    """Exact energy range by enumeration, padded by one bin; about 64 power-of-two bins."""
    n = s.size()
    j = s.couplings("fp64")[:n, :n]
    states = np.array(list(itertools.product([-1.0, 1.0], repeat=n)))
    e = 0.5 * np.einsum("ki,ij,kj->k", states, j, states)
    w = 2.0 ** round(math.log2((e.max() - e.min()) / 64))
    return math.floor(e.min() / w) * w - w, math.ceil(e.max() / w) * w + w, w


def test_learned_warm_start_ablation(oracle):
    """Ablation of the learned warm start: the network trained on 48 plain-run DOS curves of
    random dipole clusters (8-12 spins) starts 8 held-out clusters at ln f = 1e-2, and every run,
    learned or flat, reaches max |d log g| <= 0.05 against exact enumeration.  At this size the
    learned start gains nothing measurable: over 24 held-out clusters it took 0.99-1.11 times the
    attempts of the flat start depending on the start factor (1e-3 to 1e-1), so the test bounds
    the ratio on both sides instead of asserting a gain."""
    specs = []
    for k in range(1, 49):
        s = _cluster(k)
        specs.append((s, *_grid(s), k))
    train = plain_dos_many(specs, final_factor=1e-4)  # 48 engines in one batch
    model = WarmStartModel(hidden=(32, 32), seed=3)
    assert model.fit(train, steps=4000, learning_rate=3e-3) < 0.5
    flat = learned = 0
    for k in range(1001, 1009):
        s = _cluster(k)
        emin, emax, w = _grid(s)
        counts = oracle.exact_counts(s, emin, emax, w)
        ref = np.where(counts > 0, np.log(np.maximum(counts, 1).astype(float)), np.nan)
        a = run_to_accuracy(s, emin, emax, w, ref, 0.05, k)
        b = run_to_accuracy(s, emin, emax, w, ref, 0.05, k, model=model, factor=1e-2)
        assert not a["warm"] and b["warm"]
        assert a["attempts"] is not None and b["attempts"] is not None
        flat += a["attempts"]
        learned += b["attempts"]
    assert 0.5 * flat <= learned <= 1.5 * flat, (learned, flat)


def _warm_grid(c: RunConfig, scale: float) -> np.ndarray:
    """A smooth, finite warm-start estimate over the whole grid."""
    bins = c.bins()
    x = np.linspace(-1.0, 1.0, bins)
    return -scale * x * x


WARM_RUNS = {
    # dense split sweep with exchanges, three windows of two walkers
    "dense27": (lambda: System(Geometry.simple_cubic(3, 3, 3, periodic=True)),
                dict(emin=-60, emax=60, bin_width=0.5, windows=3, walkers=2, seed=21, max_mcs=600,
                     exchange_interval_mcs=1, check_interval_mcs=10)),
    # the single-window kernel (8 sites, one window of two walkers)
    "window8": (lambda: System(Geometry.simple_cubic(2, 2, 2, periodic=False)),
                dict(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=2, seed=1234, max_mcs=20000,
                     check_interval_mcs=50)),
    # the CSR sweep
    "csr64": (lambda: System(Geometry.simple_cubic(4, 4, 4, periodic=True), 1.0, 1.8),
              dict(emin=-150, emax=150, bin_width=0.5, windows=2, walkers=3, seed=9, max_mcs=300,
                   exchange_interval_mcs=1, check_interval_mcs=5)),
}


@pytest.mark.parametrize("continue_schedule", [False, True])
@pytest.mark.parametrize("name", list(WARM_RUNS))
def test_warm_started_run_bitwise(oracle, name, continue_schedule):
    """run_rewl after a warm start at ln f = 1e-3, with the reference's 1/t rule and with the
    schedule continued (the first covered check enters 1/t from ln f = 5e-4 with f = active /
    (attempted + offset)), bit for bit against the oracle's restatement.  With the schedule
    continued the factor stays near the start's: it rises above 5e-4 only as far as new bins
    raise the active count."""
    make_system, kw = WARM_RUNS[name]
    s = make_system()
    c = RunConfig(**kw)
    c.wl.final_factor = 1e-6
    c.resolve_mcs(s.size())
    lg = _warm_grid(c, 3.0)
    with Engine(s, c) as e:
        e.warm_start(lg, 1e-3, continue_schedule=continue_schedule)
        e.run()
        got = e.result()
        stages = [e.snapshot(w).stage for w in range(e.walkers)]
    want = oracle.run_rewl(s, c, warm_start=(lg, 1e-3, continue_schedule))
    assert results_equal(got, want) == []
    assert stages.count(1) + stages.count(2) > 0  # the 1/t stage was reached
    factors = [st["factor"] for st in got.walker_statistics]
    if continue_schedule:
        assert max(factors) <= 2e-3
