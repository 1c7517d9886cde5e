"""The stitch on the device (wlg_engine_stitch) against the host stitch (wlg_stitch_dos, itself
byte-identical to the reference's stitch_dos, tests/test_stitch.py): same curve, histogram,
errors, valid mask and joins, bit for bit, on the fragments of real runs; and the reference's
error for a complete-range normalisation with invalid bins."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

from helpers import random_axes, same_double
from replica_exchange_wang_landau_b200.engine import Engine, Geometry, RunConfig, System, WlgError, stitch_dos

pytestmark = pytest.mark.gpu


def _random_system(dims, seed, periodic=True, box=None, cutoff=0.0):
    g = Geometry.simple_cubic(*dims, periodic=periodic)
    g.axes = random_axes(g.size(), seed)
    if box:
        g.box = box
    return System(g, 1.0, cutoff)


def _assert_same(dev, host):
    assert same_double(dev.log_g, host.log_g)
    assert np.array_equal(dev.histogram, host.histogram)
    assert same_double(dev.standard_error, host.standard_error)
    assert np.array_equal(dev.valid, host.valid)
    assert dev.join_bins == host.join_bins
    for a, b in zip(dev.joins, host.joins):
        for k in a:
            assert float(a[k]).hex() == float(b[k]).hex() if isinstance(a[k], float) else a[k] == b[k], k
    assert dev.fully_normalized == host.fully_normalized


CASES = {
    "dense27_3win": (lambda: _random_system((3, 3, 3), 11),
                     dict(emin=-60, emax=60, bin_width=0.5, windows=3, walkers=2, seed=21, max_mcs=300,
                          exchange_interval_mcs=1, check_interval_mcs=10)),
    "slab_uneven": (lambda: _random_system((5, 4, 2), 12, box=(5.0, 4.0, 0.0)),
                    dict(emin=-80, emax=80, bin_width=0.5, windows=3, walkers=3, seed=5, max_mcs=200,
                         explicit_windows=[(0, 140), (100, 220), (180, 320)], exchange_interval_mcs=2,
                         check_interval_mcs=4)),
    "dense512_16win": (lambda: _random_system((8, 8, 8), 1),
                       dict(emin=-228.5, emax=228.0, bin_width=0.5, windows=16, walkers=8, overlap=0.75, seed=1,
                            max_mcs=200, exchange_interval_mcs=1)),
    "csr125": (lambda: _random_system((5, 5, 5), 23, cutoff=2.2),
               dict(emin=-120, emax=60, bin_width=0.5, windows=4, walkers=2, seed=31, max_mcs=150,
                    exchange_interval_mcs=1, check_interval_mcs=5)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_device_stitch_matches_host(name):
    make_system, kw = CASES[name]
    s = make_system()
    c = RunConfig(**kw)
    c.resolve_mcs(s.size())
    with Engine(s, c) as e:
        e.run()
        dev = e.stitch()
        frags = e.fragments()
        complete = None
        if np.all(dev.valid == 1):  # every bin was reached: the complete-range form must agree too
            complete = e.stitch(complete_range=True)
        else:
            with pytest.raises(WlgError) as dev_err:
                e.stitch(complete_range=True)
    _assert_same(dev, stitch_dos(frags, c.emin, c.emax, c.bin_width))
    if complete is not None:
        _assert_same(complete, stitch_dos(frags, c.emin, c.emax, c.bin_width, True, s.size()))
        return
    with pytest.raises(WlgError) as host_err:
        stitch_dos(frags, c.emin, c.emax, c.bin_width, True, s.size())
    assert str(dev_err.value) == str(host_err.value) == \
        "Complete-range normalization requires every DOS bin to be valid"


def _fully_occupied_grid(s: System):
    """A grid over the exact energy range of a small system on which every bin is occupied."""
    n = s.size()
    j = s.couplings("fp64")[:n, :n]
    states = np.array(list(itertools.product([-1.0, 1.0], repeat=n)))
    e = 0.5 * np.einsum("ki,ij,kj->k", states, j, states)
    for bins in (12, 10, 8, 6, 5, 4):
        w = 2.0 ** np.floor(np.log2((e.max() - e.min()) / bins))
        lo, hi = np.floor(e.min() / w) * w, np.floor(e.max() / w) * w + w
        counts = np.bincount(np.minimum(((e - lo) / w).astype(int), int(round((hi - lo) / w)) - 1),
                             minlength=int(round((hi - lo) / w)))
        if np.all(counts > 0):
            return float(lo), float(hi), float(w)
    raise AssertionError("no fully occupied grid")


def test_device_stitch_complete_range():
    s = _random_system((2, 2, 2), 7, periodic=False)
    lo, hi, w = _fully_occupied_grid(s)
    for windows in (1, 2):
        c = RunConfig(emin=lo, emax=hi, bin_width=w, windows=windows, walkers=2, seed=3, overlap=0.5,
                      exchange_interval_mcs=1)
        c.wl.final_factor = 1e-3
        c.max_mcs = 0
        c.resolve_mcs(s.size())
        with Engine(s, c) as e:
            e.run()
            dev = e.stitch(complete_range=True)
            host = stitch_dos(e.fragments(), c.emin, c.emax, c.bin_width, True, s.size())
        assert dev.fully_normalized and np.all(dev.valid == 1)
        _assert_same(dev, host)
