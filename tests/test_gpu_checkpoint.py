"""Multi-walker run checkpoints: a run saved, restored into a new engine and continued is
bit-identical to the run that never stopped."""
from __future__ import annotations

import pytest

from helpers import snapshots_equal
from replica_exchange_wang_landau_b200.engine import (Engine, InvalidArgument, RunConfig, System, WlParameters,
                                                      WlgError)
from replica_exchange_wang_landau_b200.geometry import simple_cubic_random

pytestmark = pytest.mark.gpu


def _setup(precision="fp64", collect=False, seed=3):
    s = System(simple_cubic_random(4, 4, 4, seed=seed, periodic=True), 1.0, 0.0)
    c = RunConfig(emin=-60, emax=60, bin_width=0.5, windows=3, walkers=2, overlap=0.6, seed=21)
    c.wl = WlParameters(0.8, 100, 1e-4, 1000, 0, True)
    c.wl.collect_window_statistics = collect
    c.coupling_precision = precision
    c.exchange_interval_mcs = 1.0
    c.recompute_interval_mcs = 3.0
    c.resolve_mcs(s.size())
    return s, c


@pytest.mark.parametrize("precision,collect", [("fp64", False), ("fp64", True), ("fp32", False)])
def test_resume_is_bit_identical(tmp_path, precision, collect):
    s, c = _setup(precision, collect)
    with Engine(s, c) as e:
        e.run_epochs(30)
        e.run_epochs(30)
        ref = [e.snapshot(w) for w in range(6)], e.totals(), e.precision_report()
    path = tmp_path / "run.ckpt"
    with Engine(s, c) as e:
        e.run_epochs(30)
        e.save_run(path)
    with Engine(s, c) as e:
        e.load_run(path)
        e.run_epochs(30)
        got = [e.snapshot(w) for w in range(6)], e.totals(), e.precision_report()
    for a, b in zip(ref[0], got[0]):
        assert snapshots_equal(a, b) == []
    for k in ("attempted", "accepted", "exchange_attempted", "exchange_accepted", "epochs"):
        assert ref[1][k] == got[1][k], k
    assert ref[2] == got[2]


def test_checkpoint_path_restores_at_creation(tmp_path):
    s, c = _setup()
    c.checkpoint_path = str(tmp_path / "auto.ckpt")
    c.checkpoint_interval_attempts = 10 * s.size()
    with Engine(s, c) as e:
        e.run_epochs(20)
        t = e.totals()
    assert (tmp_path / "auto.ckpt").exists()
    with Engine(s, c) as e:  # restored from the last checkpoint, at most 10 epochs behind
        assert 0 < e.totals()["epochs"] <= t["epochs"]


def test_incompatible_checkpoint_is_refused(tmp_path):
    s, c = _setup()
    with Engine(s, c) as e:
        e.run_epochs(5)
        e.save_run(tmp_path / "a.ckpt")
    other, c2 = _setup(seed=4)
    with Engine(other, c2) as e:
        with pytest.raises(InvalidArgument):
            e.load_run(tmp_path / "a.ckpt")
    (tmp_path / "bad.ckpt").write_bytes(b"not a checkpoint")
    with Engine(s, c) as e:
        with pytest.raises(WlgError):
            e.load_run(tmp_path / "bad.ckpt")
