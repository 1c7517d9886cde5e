"""stitch_dos and the CSV writers against the compiled reference (CPU; the stitcher is host
code of the library)."""
from __future__ import annotations

import numpy as np
import pytest

from replica_exchange_wang_landau_b200.engine import (DosFragment, InvalidArgument, WlgError, stitch_dos,
                                                      write_dos_csv, write_fragment_csv, _fragment_view)


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
