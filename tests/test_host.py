"""CPU tests of the host-side logic: configuration defaults and MCS resolution, energy grid,
window partition, checkpoint files, geometry loaders and generators -- against the oracle
and the reference's own known answers (tests/test_main.cpp)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from replica_exchange_wang_landau_b200 import engine as E
from replica_exchange_wang_landau_b200.geometry import (Xoshiro, diluted_cubic, random_sequential,
                                                        random_sphere_axes, simple_cubic_random)


def test_defaults_match_reference():
    c = E.RunConfig()
    assert (c.emin, c.emax, c.bin_width, c.windows, c.walkers, c.overlap, c.seed) == (-20.0, 20.0, 0.1, 1, 1, 0.75, 1)
    w = c.wl
    assert (w.flatness, w.minimum_visits, w.final_factor, w.inverse_time_enabled) == (0.8, 100, 1e-8, True)
    assert (w.initialization_max_attempts, w.initialization_stall_attempts_per_spin) == (1_000_000, 1_000)
    c.resolve_mcs(8)
    assert (c.exchange_interval_attempts, c.wl.check_interval_attempts, c.max_attempts,
            c.checkpoint_interval_attempts, c.wl.force_accept_after_attempts) == (80, 800, 8_000_000, 80_000, 0)
    lib = E.load_library()
    native = E._abi.wlg_run_config()
    assert lib.wlg_default_run_config(8, native) == 0
    assert (native.exchange_interval_attempts, native.wl.check_interval_attempts, native.max_attempts) == (80, 800,
                                                                                                          8_000_000)


def test_mcs_resolution_known_answers():
    # tests/test_main.cpp:69-72, 110-113 (N = 2)
    c = E.RunConfig(exchange_interval_mcs=1.5, check_interval_mcs=2.5, force_accept_after_mcs=3.5, max_mcs=4.5,
                    checkpoint_interval_mcs=5.5)
    c.resolve_mcs(2)
    assert (c.exchange_interval_attempts, c.wl.check_interval_attempts) == (3, 5)
    assert (c.wl.force_accept_after_attempts, c.max_attempts, c.checkpoint_interval_attempts) == (7, 9, 11)
    assert not c.uses_legacy_attempt_units()
    legacy = E.RunConfig(max_attempts=9, max_limit_uses_mcs=False)
    legacy.resolve_mcs(2)
    assert legacy.max_attempts == 9 and legacy.max_mcs == 4.5 and legacy.uses_legacy_attempt_units()
    assert E.attempts_from_mcs(0.1, 3, False) == 1  # never rounds to zero
    with pytest.raises(E.InvalidArgument):
        E.attempts_from_mcs(0.0, 3, False)


def test_grid_index_matches_oracle(oracle):
    rng = np.random.default_rng(3)
    for emin, emax, w in [(-2.0, 2.0, 0.5), (-20.0, 20.0, 0.25), (-228.5, 228.0, 0.5), (-1.0, 1.0, 0.1)]:
        edges = [emin + k * w for k in range(int(round((emax - emin) / w)) + 1)]
        probes = edges + [math.nextafter(x, -math.inf) for x in edges] + [math.nextafter(x, math.inf) for x in edges]
        probes += list(rng.uniform(emin - 1, emax + 1, 2000)) + [math.nan, math.inf, -math.inf]
        for e in probes:
            assert E.grid_index(emin, emax, w, e) == oracle.grid_index(emin, emax, w, e), (emin, emax, w, e)
    assert E.grid_index(-2, 2, 0.5, -2) == 0 and E.grid_index(-2, 2, 0.5, 2) == 7
    assert E.grid_index(-2, 2, 0.5, 2.1) is None
    with pytest.raises(E.InvalidArgument, match="integer multiple"):
        E.grid_bins(-1, 1, 0.3)


def test_partition_windows_matches_oracle(oracle):
    for bins in (2, 7, 100, 797, 913, 4069):
        for count in (1, 2, 3, 8, 16, 64):
            for overlap in (0.0, 0.5, 0.75, 0.9):
                if count > bins:
                    continue
                try:
                    want = oracle.partition_windows(bins, count, overlap)
                except Exception:
                    with pytest.raises(E.InvalidArgument):
                        E.partition_windows(bins, count, overlap)
                    continue
                assert E.partition_windows(bins, count, overlap) == want


def test_checkpoint_roundtrip(tmp_path):
    rng = np.random.default_rng(1)
    n, bins = 10, 40
    s = E.Snapshot(3, rng.choice(np.array([-1, 1], np.int8), n), rng.normal(size=n), -3.25, rng.normal(size=bins),
                   rng.integers(0, 100, bins).astype(np.uint64), (rng.random(bins) > 0.5).astype(np.uint8), 0.125,
                   1000, 400, 3, 990, 1, (1, 2, 3, 2**64 - 1))
    path = tmp_path / "c.chk"
    E.save_checkpoint(str(path), s)
    data = path.read_bytes()
    assert data[:8] == b"WLCHKP3\0"
    assert len(data) == 8 + 8 + (8 + n) + (8 + 8 * n) + 8 + 3 * 8 + 8 * bins * 2 + bins + 8 * 5 + 1 + 32
    r = E.load_checkpoint(str(path))
    for k in ("walker_id", "energy", "factor", "attempted", "accepted", "forced_accepted", "last_accepted_attempt",
              "stage", "rng_state"):
        assert getattr(r, k) == getattr(s, k), k
    for k in ("spins", "fields", "log_g", "histogram", "active"):
        assert np.array_equal(getattr(r, k), getattr(s, k)), k
    (tmp_path / "bad.chk").write_bytes(b"NOTACHKP" + data[8:])
    with pytest.raises(E.WlgError, match="Invalid checkpoint format"):
        E.load_checkpoint(str(tmp_path / "bad.chk"))
    (tmp_path / "short.chk").write_bytes(data[:40])
    with pytest.raises(E.WlgError, match="Truncated"):
        E.load_checkpoint(str(tmp_path / "short.chk"))
    with pytest.raises(E.CheckpointIOError):
        E.load_checkpoint(str(tmp_path / "missing.chk"))


def test_reference_reads_our_checkpoint(tmp_path, reference):
    """A checkpoint written by the engine's writer restores into the reference walker."""
    s = E.System(E.Geometry.simple_cubic(2, 2, 1, periodic=False))
    p = E.WlParameters(0.1, 1, 0.1, 10)
    w = reference.walker(s, 0, -20, 20, 0.25, (0, 160), p, 42)
    w.run_attempts(100)
    snap = w.snapshot()
    E.save_checkpoint(str(tmp_path / "x.chk"), snap)
    back = E.load_checkpoint(str(tmp_path / "x.chk"))
    w2 = reference.walker(s, 0, -20, 20, 0.25, (0, 160), p, 42)
    w2.restore(back)
    assert w2.snapshot().attempted == 100 and w2.snapshot().energy == snap.energy


def test_csv_geometry_roundtrip_and_errors(tmp_path):
    # tests/test_main.cpp:40-58
    csv = tmp_path / "system.csv"
    csv.write_text("x,y,z,mx,my,mz\n0,0,0,0,0,1\n1,0,0,0,0,1\n")
    g = E.Geometry.load_csv(str(csv), (2, 2, 2), False)
    assert g.size() == 2 and g.axes[1, 2] == 1.0
    g2 = simple_cubic_random(3, 2, 2, seed=4)
    g2.to_csv(str(tmp_path / "r.csv"))
    back = E.Geometry.load_csv(str(tmp_path / "r.csv"), g2.box, True)
    assert np.array_equal(back.positions, g2.positions) and np.array_equal(back.axes, g2.axes)
    (tmp_path / "bad.csv").write_text("x,y,z,mx,my\n")
    with pytest.raises(RuntimeError, match="header"):
        E.Geometry.load_csv(str(tmp_path / "bad.csv"))
    (tmp_path / "nonunit.csv").write_text("x,y,z,mx,my,mz\n0,0,0,0,0,2\n")
    with pytest.raises(E.InvalidArgument, match="normalized"):
        E.Geometry.load_csv(str(tmp_path / "nonunit.csv"), (0, 0, 0), False)


def test_geometry_validation_messages():
    bad = E.Geometry(np.zeros((1, 3)), np.array([[0, 0, 1.0]]), (0, 0, 0), True)
    with pytest.raises(E.InvalidArgument, match="At least one periodic box length must be positive"):
        bad.validate()
    bad = E.Geometry(np.array([[math.inf, 0, 0]]), np.array([[0, 0, 1.0]]), (1, 1, 1), True)
    with pytest.raises(E.InvalidArgument, match="finite"):
        bad.validate()


def test_generators_are_seeded_and_valid(oracle):
    r = Xoshiro(1234, 3)
    # the same stream as the engine's / reference's Xoshiro256StarStar(1234, 3)
    assert [r.next() for _ in range(2)] == [16657228507453487946, 6377765824822115752]
    a = random_sphere_axes(200, 9)
    assert np.allclose(np.linalg.norm(a, axis=1), 1.0, atol=1e-14)
    assert np.array_equal(a, random_sphere_axes(200, 9))
    assert abs(a.mean(axis=0)).max() < 0.2
    d = diluted_cubic(6, 6, 6, 0.4, seed=3, periodic=True, box=(6.0, 6.0, 0.0))
    assert d.size() == 216 - round(0.4 * 216)
    rsa = random_sequential(64, 0.5, 0.8, seed=5)
    diff = rsa.positions[:, None, :] - rsa.positions[None, :, :]
    diff -= rsa.box[0] * np.rint(diff / rsa.box[0])
    dist = np.sqrt((diff ** 2).sum(-1)) + np.eye(64) * 10
    assert dist.min() >= 0.8
    oracle.couplings(E.System(rsa))  # no coincident sites
