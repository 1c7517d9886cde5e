"""stitch_dos and the CSV writers against the compiled reference (CPU; the stitcher and the
writers are host code of the library)."""
from __future__ import annotations

import numpy as np
import pytest

from replica_exchange_wang_landau_b200 import _abi
from replica_exchange_wang_landau_b200.engine import (DosFragment, InvalidArgument, WlgError, stitch_dos,
                                                      write_dos_csv, write_fragment_csv, write_workers_stat_csv,
                                                      _fragment_view)


def _fragments(seed: int, bins: int = 120, windows: int = 4, holes: bool = True):
    """Noisy log g curves of overlapping windows on one grid, each shifted by a constant."""
    rng = np.random.default_rng(seed)
    truth = -0.002 * (np.arange(bins) - 50.0) ** 2 + 0.3 * np.sin(np.arange(bins) / 7.0)
    size = int(np.ceil(bins / (1 + (windows - 1) * 0.4)))
    out = []
    for w in range(windows):
        b = int(round(w * (bins - size) / (windows - 1)))
        e = bins if w == windows - 1 else b + size
        lg = np.full(bins, np.nan)
        valid = np.zeros(bins, np.uint8)
        lg[b:e] = truth[b:e] + rng.normal(scale=0.01, size=e - b) + rng.uniform(-5, 5)
        valid[b:e] = 1
        if holes:
            valid[b + rng.integers(0, e - b, 2)] = 0
        lg[valid == 0] = np.nan
        h = np.where(valid == 1, rng.integers(1, 1000, bins), 0).astype(np.uint64)
        se = np.where(valid == 1, rng.uniform(0, 0.1, bins), np.nan)
        out.append(DosFragment((b, e), lg, h, se, valid))
    return out


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_stitch_matches_reference_bitwise(reference, tmp_path, seed):
    frags = _fragments(seed)
    emin, emax, width = -30.0, 30.0, 0.5
    dos = stitch_dos(frags[::-1], emin, emax, width)  # any order
    views = [_fragment_view(f) for f in frags]
    lg, h, se, v, joins = reference.stitch_dos([x[0] for x in views], emin, emax, width, False, 0,
                                               dos_csv=tmp_path / "ref_dos.csv")
    assert np.array_equal(lg.view(np.uint64), dos.log_g.view(np.uint64))
    assert np.array_equal(se.view(np.uint64), dos.standard_error.view(np.uint64))
    assert np.array_equal(h, dos.histogram) and np.array_equal(v, dos.valid)
    assert [int(j) for j in joins] == dos.join_bins
    assert all(q["common_bins"] > 0 and q["rmse"] < 0.1 for q in dos.joins)
    write_dos_csv(tmp_path / "dos.csv", dos)
    assert (tmp_path / "dos.csv").read_bytes() == (tmp_path / "ref_dos.csv").read_bytes()
    write_fragment_csv(tmp_path / "w1.csv", frags[1], emin, width, 1)
    reference.write_fragment_csv(tmp_path / "ref_w1.csv", views[1][0], emin, emax, width, 1)
    assert (tmp_path / "w1.csv").read_bytes() == (tmp_path / "ref_w1.csv").read_bytes()


def test_complete_range_normalisation(reference):
    frags = _fragments(4, holes=False)
    dos = stitch_dos(frags, -30.0, 30.0, 0.5, complete_range=True, spin_count=10)
    views = [_fragment_view(f) for f in frags]
    lg = reference.stitch_dos([x[0] for x in views], -30.0, 30.0, 0.5, True, 10)[0]
    assert dos.fully_normalized and np.array_equal(lg.view(np.uint64), dos.log_g.view(np.uint64))
    with pytest.raises(WlgError):
        stitch_dos(_fragments(5), -30.0, 30.0, 0.5, complete_range=True, spin_count=10)


def test_stitch_errors():
    frags = _fragments(6)
    with pytest.raises(InvalidArgument):
        stitch_dos([], -30.0, 30.0, 0.5)
    far = DosFragment((100, 120), frags[-1].log_g, frags[-1].histogram, frags[-1].standard_error, frags[-1].valid)
    with pytest.raises(InvalidArgument):
        stitch_dos([frags[0], far], -30.0, 30.0, 0.5)


WORKERS_STAT_HEADER = ("mpi_rank,window,walker_id,attempted_flips,attempted_mcs,accepted,forced_accepted,"
                       "accepted_percent,attempts_since_last_accepted,mcs_since_last_accepted,energy,factor,"
                       "active_bins,min_h,mean_h,min_over_mean,round_trips")


def _stat(**kw) -> dict:
    s = {name: 0 for name, _ in _abi.wlg_walker_statistics._fields_}
    s.update(kw)
    return s


def test_workers_stat_known_answer(tmp_path):
    """The reference's own expected header and row (tests/test_main.cpp:340-360): a blocked
    walker of a 2-spin system after 5 attempts, none accepted."""
    blocked = _stat(attempted=5, attempts_since_last_accepted=5, energy=1.0, factor=1.0, active_bins=1,
                    minimum_histogram=6, mean_histogram=6.0, min_over_mean=1.0)
    write_workers_stat_csv(tmp_path / "ws.csv", [blocked], 2)
    lines = (tmp_path / "ws.csv").read_text().split("\n")
    assert lines[0] == WORKERS_STAT_HEADER
    assert lines[1] == "0,0,0,5,2.5,0,0,0,5,2.5,1,1,1,6,6,1,0"
    assert lines[2:] == [""]


def _random_stats(seed: int, count: int) -> list:
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        attempted = int(rng.integers(0, 1 << 40)) if k else 0  # the first walker made no attempt
        accepted = int(rng.integers(0, attempted + 1))
        out.append(_stat(walker_id=k, window_id=k // 4, mpi_rank=int(rng.integers(0, 3)), attempted=attempted,
                         accepted=accepted, forced_accepted=int(rng.integers(0, accepted + 1)),
                         attempts_since_last_accepted=int(rng.integers(0, 1 << 20)),
                         energy=float(rng.normal(scale=300.0)), factor=float(rng.uniform(0, 1) ** 20),
                         active_bins=int(rng.integers(0, 900)), minimum_histogram=int(rng.integers(0, 1 << 50)),
                         mean_histogram=float(rng.uniform(0, 1e12)), min_over_mean=float(rng.uniform()),
                         round_trips=int(rng.integers(0, 1000))))
    return out


@pytest.mark.parametrize("spins", [1, 7, 512, 32768])
def test_workers_stat_matches_reference_bytes(reference, tmp_path, spins):
    stats = _random_stats(spins, 24)
    write_workers_stat_csv(tmp_path / "ws.csv", stats, spins)
    rows = (_abi.wlg_walker_statistics * len(stats))()
    for k, s in enumerate(stats):
        for name, _ in _abi.wlg_walker_statistics._fields_:
            setattr(rows[k], name, s[name])
    reference.write_workers_stat_csv(tmp_path / "ref_ws.csv", rows, spins)
    assert (tmp_path / "ws.csv").read_bytes() == (tmp_path / "ref_ws.csv").read_bytes()


def test_workers_stat_errors(tmp_path):
    with pytest.raises(InvalidArgument, match="Cannot write MCS statistics for zero spins"):
        write_workers_stat_csv(tmp_path / "ws.csv", [_stat()], 0)
    with pytest.raises(WlgError, match="Cannot write"):
        write_workers_stat_csv(tmp_path / "missing" / "ws.csv", [_stat()], 2)
    write_workers_stat_csv(tmp_path / "empty.csv", [], 2)  # no walkers: the header alone
    assert (tmp_path / "empty.csv").read_text() == WORKERS_STAT_HEADER + "\n"
