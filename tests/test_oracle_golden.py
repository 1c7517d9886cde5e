"""Pins the CPU oracle (oracle/wl_oracle.c) to the reference: golden vectors generated from
the compiled reference (tests/golden/make_golden.py) and the reference's own known-answer
tests (tests/test_main.cpp).  CPU only."""
from __future__ import annotations

import math

import numpy as np
import pytest

from helpers import config_from, random_axes, same_double, snapshot_matches_json, system_from, unhex
from replica_exchange_wang_landau_b200.engine import Geometry, RunConfig, System, WlParameters


def test_pair_formula(oracle, golden):
    # tests/test_main.cpp:24-28
    assert oracle.dipolar_pair((1, 0, 0), (1, 0, 0), (1, 0, 0)) == pytest.approx(-2, abs=1e-14)
    assert oracle.dipolar_pair((1, 0, 0), (0, 0, 1), (0, 0, 1)) == pytest.approx(1, abs=1e-14)
    assert oracle.dipolar_pair((2, 0, 0), (0, 0, 1), (0, 0, 1)) == pytest.approx(0.125, abs=1e-14)
    for case in golden["pair"]:
        assert oracle.dipolar_pair(case["d"], case["ai"], case["aj"]).hex() == case["value"]


def test_minimum_image(oracle, golden):
    # tests/test_main.cpp:30-38
    d = oracle.minimum_image((6, -5, 3.1), (10, 8, 6))
    assert d == pytest.approx((-4, 3, -2.9), abs=1e-14)
    d = oracle.minimum_image((6, -5, 31), (10, 8, 0))
    assert d == pytest.approx((-4, 3, 31), abs=1e-14)
    for case in golden["minimum_image"]:
        assert [x.hex() for x in oracle.minimum_image(case["d"], case["box"], True)] == case["out"]


@pytest.mark.parametrize("name", ["exact_2x2x2", "exact_2x2x1"])
def test_exact_enumeration(oracle, golden, name):
    g = golden[name]
    s = System(Geometry.simple_cubic(*g["dims"], periodic=False))
    counts = oracle.exact_counts(s, g["emin"], g["emax"], g["width"])
    assert {str(i): int(c) for i, c in enumerate(counts) if c} == g["counts"]
    assert int(counts.sum()) == 2 ** s.size()


def test_exact_2x2x2_known_answer(oracle):
    # the 17 occupied bins of the 2x2x2 open lattice on [-20, 20] / 0.25 (256 states)
    s = System(Geometry.simple_cubic(2, 2, 2, periodic=False))
    counts = oracle.exact_counts(s, -20.0, 20.0, 0.25)
    expected = {27: 2, 42: 4, 48: 8, 53: 16, 61: 32, 64: 16, 74: 8, 77: 16, 80: 52, 82: 16, 85: 8, 93: 32,
                96: 16, 106: 4, 112: 8, 117: 16, 155: 2}
    assert {i: int(c) for i, c in enumerate(counts) if c} == expected


@pytest.mark.parametrize("name", ["cubic27_periodic", "slab24", "csr64_r1.8"])
def test_couplings_and_fields(oracle, golden, name):
    g = golden["systems"][name]
    s = system_from(g)
    assert same_double(oracle.couplings(s).ravel(), unhex(g["couplings"]))
    fields, energies = oracle.local_fields(s, np.array(g["spins"], dtype=np.int8))
    assert same_double(fields.ravel(), unhex(g["fields"]))
    assert same_double(energies, unhex(g["energies"]))


def test_dense_equals_csr_at_large_cutoff(oracle):
    # tests/test_main.cpp:139-154
    g = Geometry.simple_cubic(3, 2, 1, 1.0, (0, 0, 1), False)
    dense, csr = System(g, 0.7), System(g, 0.7, 100.0)
    assert np.allclose(oracle.couplings(dense), oracle.couplings(csr), atol=1e-14, rtol=0)
    spins = np.array([1, -1, 1, 1, -1, -1], dtype=np.int8)
    fields, (energy,) = oracle.local_fields(dense, spins[None])
    fields = fields[0]
    for i in range(6):
        delta = -2.0 * spins[i] * fields[i]
        flipped = spins.copy()
        flipped[i] = -flipped[i]
        exact_fields, (e2,) = oracle.local_fields(dense, flipped[None])
        assert energy + delta == pytest.approx(e2, rel=1e-12, abs=1e-12)


@pytest.mark.parametrize("k", [0, 1, 2])
def test_walker_trajectories(oracle, golden, k):
    w = golden["walkers"][k]
    s = system_from(golden["systems"][w["system"]])
    p = WlParameters(**w["params"])
    walker = oracle.walker(s, w["walker_id"], *w["grid"], w["window"], p, w["seed"])
    assert snapshot_matches_json(walker.snapshot(), w["init"]) == []
    walker.run_attempts(3000)
    assert snapshot_matches_json(walker.snapshot(), w["after_3000"]) == []


@pytest.mark.parametrize("k", [0, 1])
def test_run_rewl(oracle, golden, k):
    case = golden["rewl"][k]
    s = system_from(golden["systems"][case["system"]])
    r = oracle.run_rewl(s, config_from(case["config"]))
    g = case["result"]
    for key in ("attempted", "accepted", "forced_accepted", "exchange_attempted", "exchange_accepted", "converged"):
        assert getattr(r, key) == g[key], key
    for f, gf in zip(r.fragments, g["fragments"]):
        assert same_double(f.log_g, unhex(gf["log_g"]))
        assert f.histogram.tolist() == gf["histogram"]
        assert same_double(f.standard_error, unhex(gf["standard_error"]))
        assert f.valid.tolist() == gf["valid"]
    for st, gs in zip(r.walker_statistics, g["walker_statistics"]):
        for key, v in gs.items():
            got = st[key]
            assert (float(got).hex() if isinstance(v, str) else got) == v, key


def test_grid_and_windows(oracle):
    # tests/test_main.cpp:156-162
    assert oracle.grid_index(-2, 2, 0.5, -2) == 0
    assert oracle.grid_index(-2, 2, 0.5, 2) == 7
    assert oracle.grid_index(-2, 2, 0.5, 2.1) is None
    w = oracle.partition_windows(100, 4, 0.75)
    assert len(w) == 4 and w[0][0] == 0 and w[-1][1] == 100
    assert all(w[i][0] < w[i - 1][1] for i in range(1, 4))


def test_forced_acceptance(oracle):
    # tests/test_main.cpp:235-258
    s = System(Geometry.simple_cubic(2, 1, 1, 1.0, (0, 0, 1), False))
    p = WlParameters(0.8, 1, 1e-8, 100, 3)
    w = oracle.walker(s, 4, -2, 2, 0.5, (0, 8), p, 123)
    snap = w.snapshot()
    old = oracle.grid_index(-2, 2, 0.5, snap.energy)
    proposed = snap.energy + -2.0 * snap.spins[0] * snap.fields[0]
    new = oracle.grid_index(-2, 2, 0.5, proposed)
    assert old is not None and new is not None and old != new
    snap.log_g[old] = 0.0
    snap.log_g[new] = 1000.0
    w.restore(snap)
    w.run_attempts(3)
    assert w.counters()[1:] == (0, 0, 0)
    assert w.attempt_flip()
    assert w.counters() == (4, 1, 1, 4)


def test_histogram_statistics_and_inverse_time(oracle):
    # tests/test_main.cpp:534-596
    s = System(Geometry.simple_cubic(1, 1, 1, 1.0, (0, 0, 1), False))
    w = oracle.walker(s, 3, -1, 1, 0.5, (0, 4), WlParameters(0.8, 1, 1e-8, 1), 11)
    snap = w.snapshot()
    snap.active[:] = 0
    snap.histogram[:] = 0
    snap.active[0] = snap.active[1] = 1
    snap.histogram[0], snap.histogram[1] = 80, 120
    w.restore(snap)
    st = w.histogram_statistics()
    assert (st["active_bins"], st["covered_bins"], st["minimum"]) == (2, 2, 80)
    assert st["mean"] == 100.0 and st["min_over_mean"] == pytest.approx(0.8, abs=1e-14)
    snap = w.snapshot()
    snap.stage = 1
    snap.factor = 0.002
    snap.attempted = 1000
    w.restore(snap)
    w.attempt_flip()
    f1 = w.snapshot().factor
    w.attempt_flip()
    f2 = w.snapshot().factor
    assert f1 == pytest.approx(2.0 / 1001.0, abs=1e-14)
    assert f2 == pytest.approx(3.0 / 1002.0, abs=1e-14)


def test_summary_known_answer(oracle):
    # tests/test_main.cpp:730-748, through run_rewl's summary on two restored walkers is not
    # reachable from the C API, so the aligned-mean arithmetic is checked on a run instead.
    s = System(Geometry.simple_cubic(2, 2, 1, periodic=False))
    c = RunConfig(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=2, seed=3)
    c.wl.final_factor = 0.1
    c.resolve_mcs(4)
    r = oracle.run_rewl(s, c)
    f = r.fragments[0]
    valid = np.nonzero(f.valid)[0]
    assert f.log_g[valid[0]] == 0.0
    assert all(math.isnan(x) for x in f.log_g[f.valid == 0])


@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_matches_compiled_reference(oracle, reference, seed):
    """Live cross-check: restatement vs the reference library on random systems."""
    g = Geometry.simple_cubic(3, 3, 2, periodic=True)
    g.axes = random_axes(18, seed)
    for s in (System(g, 1.0, 0.0), System(g, 1.0, 1.5)):
        assert same_double(oracle.couplings(s), reference.couplings(s))
        c = RunConfig(emin=-40, emax=40, bin_width=0.5, windows=3, walkers=2, seed=seed, overlap=0.6)
        c.wl.final_factor = 0.05
        c.max_mcs = 150
        c.exchange_interval_mcs = 2
        c.check_interval_mcs = 5
        c.wl.collect_window_statistics = seed == 2
        c.resolve_mcs(18)
        from helpers import results_equal
        assert results_equal(oracle.run_rewl(s, c), reference.run_rewl(s, c)) == []


def test_oracle_refuses_what_the_engine_refuses(oracle):
    """BF16 couplings exist for the dense backend only, in the restatement as in the engine."""
    from oracle.oracle import CheckerError
    s = System(Geometry.simple_cubic(3, 3, 3, periodic=True), 1.0, 1.8)
    c = RunConfig(emin=-20, emax=20, bin_width=0.25, windows=1, walkers=1, seed=1, max_mcs=10)
    c.coupling_precision = "bf16"
    c.resolve_mcs(27)
    with pytest.raises(CheckerError, match="dense backend only"):
        oracle.run_rewl(s, c)


def _bf16_exact(x: float) -> float:
    """Round-to-nearest-even to 8 significant bits (exponent floor 2^-133), in exact rationals."""
    from fractions import Fraction
    import math
    if x == 0.0:
        return x
    q = max(math.frexp(x)[1] - 8, -133)
    v = Fraction(x) / Fraction(2) ** q
    n = math.floor(v)
    r = v - n
    if r > Fraction(1, 2) or (r == Fraction(1, 2) and n % 2 == 1):
        n += 1
    return math.ldexp(float(n), q)


def test_bf16_rounding_is_round_to_nearest_even(oracle):
    """The restated BF16 rounding: ties go to the even neighbour, a double just off a tie
    rounds once (not through float first), and subnormal bfloat16 values keep 2^-133 steps."""
    import ctypes as C
    f = oracle.lib.orc_bf16_round
    f.restype, f.argtypes = C.c_double, [C.c_double]
    ties = [1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -(1.0 + 2.0 ** -8), 1.0 + 2.0 ** -8 + 2.0 ** -40,
            1.0 + 2.0 ** -8 - 2.0 ** -40, 2.0 ** -130 * 1.5, 2.0 ** -133 * 0.5, 2.0 ** -133 * 0.75]
    assert [f(x) for x in ties[:5]] == [1.0, 1.0 + 2.0 ** -6, -1.0, 1.0 + 2.0 ** -7, 1.0]
    rng = np.random.default_rng(8)
    xs = ties + list(rng.normal(size=2000)) + list(rng.uniform(-1, 1, 2000) * 2.0 ** rng.integers(-140, 5, 2000))
    assert [f(float(x)) for x in xs] == [_bf16_exact(float(x)) for x in xs]


def test_oracle_fp32_recompute_replaces_drifted_energies(oracle):
    """The restated FP64 recompute of an FP32 run acts: with it every fourth MCS the walkers end
    with other energies (exact FP64 totals) than the same FP32 run without it (drifted sums),
    over the same attempts.  The GPU tests pin the restatement to the engine bit for bit."""
    g = Geometry.simple_cubic(3, 3, 2, periodic=True)
    g.axes = random_axes(18, 4)
    s = System(g, 1.0, 0.0)

    def run(recompute_mcs):
        c = RunConfig(emin=-40, emax=40, bin_width=0.5, windows=2, walkers=2, seed=6)
        c.coupling_precision = "fp32"
        c.exchange_interval_mcs = 2
        c.recompute_interval_mcs = recompute_mcs
        c.max_mcs = 40
        c.check_interval_mcs = 10
        c.resolve_mcs(18)
        return oracle.run_rewl(s, c)

    with_recompute, without = run(4.0), run(0.0)
    assert with_recompute.attempted == without.attempted > 0
    assert [x["energy"] for x in with_recompute.walker_statistics] != [x["energy"] for x in without.walker_statistics]
