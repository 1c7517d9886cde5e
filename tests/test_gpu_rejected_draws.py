"""Rejected site draws and the zero uniform in every sweep.  bounded() discards a draw below
(2^64 - N) mod N and takes the next one (include/wl/rng.hpp:29-36), and the acceptance test clamps
the uniform at 2^-53 (src/wang_landau.cpp:261); with random generator states neither happens in a
test's lifetime.  Here a walker is restored with a generator state whose k-th draw is exactly 0 (a
state with s1 = 0, stepped back k times), so that draw is rejected when it is a site draw and is
u = 0 when it is an acceptance uniform; trajectories equal the oracle's bit for bit, and the
single-window kernel equals the per-epoch kernels from the same states."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from helpers import random_axes, results_equal, snapshots_equal
from replica_exchange_wang_landau_b200.engine import Engine, Geometry, RunConfig, System

MASK = (1 << 64) - 1


def _rotl(x: int, k: int) -> int:
    return ((x << k) | (x >> (64 - k))) & MASK


def _next(s):
    """Xoshiro256StarStar::operator() (include/wl/rng.hpp:16-23): (draw, next state)."""
    s0, s1, s2, s3 = s
    out = (_rotl((s1 * 5) & MASK, 7) * 9) & MASK
    t = (s1 << 17) & MASK
    s2 ^= s0
    s3 ^= s1
    s1 ^= s2
    s0 ^= s3
    s2 ^= t
    s3 = _rotl(s3, 45)
    return out, (s0, s1, s2, s3)


def _back(s):
    """The inverse of the state transition of _next (a linear map over GF(2))."""
    s0, s1, s2, s3 = s
    a3 = _rotl(s3, 64 - 45)
    p0 = s0 ^ a3
    y = s1 ^ s2  # = p1 ^ (p1 << 17)
    p1 = (y ^ (y << 17) ^ (y << 34) ^ (y << 51)) & MASK
    a2 = s2 ^ ((p1 << 17) & MASK)
    return p0, p1, a2 ^ p0, a3 ^ p1


def zero_draw_state(k: int, seed: int):
    """A generator state whose draw number k (0-based) is 0."""
    rng = np.random.default_rng(seed)
    s = (int(rng.integers(1, 1 << 63)), 0, int(rng.integers(1, 1 << 63)), int(rng.integers(1, 1 << 63)))
    for _ in range(k):
        s = _back(s)
    return s


def test_zero_draw_state_generator():
    for k in (0, 1, 5, 40):
        s = zero_draw_state(k, 7 + k)
        for _ in range(k):
            d, s = _next(s)
            assert d != 0
        assert _next(s)[0] == 0
    s = (123, 456, 789, 1011)
    assert _back(_next(s)[1]) == s


def _lattice(dims, seed, cutoff=0.0):
    g = Geometry.simple_cubic(*dims, periodic=True)
    g.axes = random_axes(g.size(), seed)
    return System(g, 1.0, cutoff)


PATHS = {
    # dense FP64, 27 sites: the split sweep ((2^64 - 27) mod 27 = 25, so a 0 draw is rejected)
    "split": (lambda: _lattice((3, 3, 3), 31), dict(emin=-60, emax=60, bin_width=0.5), {}),
    # the same system with pilot statistics: the ring sweep
    "ring": (lambda: _lattice((3, 3, 3), 31), dict(emin=-60, emax=60, bin_width=0.5),
             dict(collect_window_statistics=True)),
    # 125 sites, cutoff 2.2: the CSR sweep ((2^64 - 125) mod 125 = 116)
    "csr": (lambda: _lattice((5, 5, 5), 32, 2.2), dict(emin=-120, emax=60, bin_width=0.5), {}),
    # the same with the Nalivaiko mask: the generic walk kernel
    "csr_nalivaiko": (lambda: _lattice((5, 5, 5), 32, 2.2), dict(emin=-120, emax=60, bin_width=0.5),
                      dict(nalivaiko_mod=True, inverse_time_enabled=False)),
}


@pytest.mark.gpu
@pytest.mark.parametrize("path", list(PATHS))
def test_rejected_draw_trajectories(oracle, path):
    make_system, kw, wl = PATHS[path]
    s = make_system()
    c = RunConfig(windows=2, walkers=2, seed=51, **kw)
    for key, val in wl.items():
        setattr(c.wl, key, val)
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        for w in range(e.walkers):
            ow = oracle.walker(s, w, c.emin, c.emax, c.bin_width, e.window(w // c.walkers), c.wl, c.seed)
            for rounds, k in enumerate((0, 1, 2, 3, 6, 13)):
                snap = e.snapshot(w)
                snap = dataclasses.replace(snap, rng_state=zero_draw_state(k, 100 * w + k))
                e.restore(w, snap)
                ow.restore(snap)
                e.run_attempts(w, 150 + 37 * rounds)
                ow.run_attempts(150 + 37 * rounds)
                assert snapshots_equal(e.snapshot(w), ow.snapshot()) == [], f"walker {w}, zero draw {k}"


@pytest.mark.gpu
def test_rejected_draws_single_window_kernel():
    """The single-window kernel against the per-epoch kernels, every walker restored with a zero
    draw a few draws ahead, over epochs with checks."""
    s = _lattice((3, 3, 3), 33)
    c = RunConfig(emin=-60, emax=60, bin_width=0.5, windows=1, walkers=3, seed=52, exchange_interval_mcs=1,
                  check_interval_mcs=2, max_mcs=300)
    c.resolve_mcs(s.size())
    results = []
    for window_sweep in (True, False):
        with Engine(s, c) as e:
            e.window_sweep = window_sweep
            for piece in range(4):
                for w in range(e.walkers):
                    snap = e.snapshot(w)
                    e.restore(w, dataclasses.replace(snap, rng_state=zero_draw_state(3 * piece + w, 7 * w + piece)))
                e.run_epochs(9)
            e.run()
            results.append(e.result())
    assert results_equal(results[0], results[1]) == []
