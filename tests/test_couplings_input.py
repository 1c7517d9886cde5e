"""The prebuilt-couplings input (wlg_engine_create_from_couplings), the C-ABI side of
run_rewl's std::shared_ptr<const Couplings> argument (include/wl/parallel.hpp:35-36).

GPU: an engine created from the couplings a system's backend stores (dense matrix or CSR rows)
runs bit for bit like the engine created from the geometry, for dense and CSR systems with FP64
and FP32 couplings.  CPU: the input is validated before any device is touched, with the same
conditions both reference backends satisfy (symmetric, zero diagonal, finite; CSR rows sorted).
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import random_axes, results_equal
from replica_exchange_wang_landau_b200.engine import (Couplings, Engine, Geometry, InvalidArgument, RunConfig,
                                                      System, run_rewl)


def _system(dims, seed, cutoff=0.0):
    g = Geometry.simple_cubic(*dims, periodic=True)
    g.axes = random_axes(g.size(), seed)
    return System(g, 1.0, cutoff)


def _config(n, precision="fp64"):
    c = RunConfig(emin=-150, emax=150, bin_width=0.5, windows=2, walkers=2, seed=9, max_mcs=80,
                  exchange_interval_mcs=1, check_interval_mcs=5)
    c.coupling_precision = precision
    c.recompute_interval_mcs = 0.0
    return c.resolve_mcs(n)


@pytest.mark.gpu
@pytest.mark.parametrize("cutoff,precision", [(0.0, "fp64"), (0.0, "fp32"), (1.8, "fp64"), (1.8, "fp32")])
def test_engine_from_couplings_equals_engine_from_geometry(cutoff, precision):
    s = _system((4, 4, 4), 13, cutoff)
    c = _config(s.size(), precision)
    j = Couplings.of(s)
    assert j.backend == s.backend
    got = run_rewl(j, c)
    want = run_rewl(s, c)
    assert got.attempted > 0 and results_equal(got, want) == []


def _create_error(couplings: Couplings) -> str:
    with pytest.raises(InvalidArgument) as err:
        Engine(couplings, _config(couplings.size()))
    return str(err.value)


def test_couplings_input_is_validated():
    rng = np.random.default_rng(3)
    a = rng.normal(size=(6, 6))
    j = a + a.T
    np.fill_diagonal(j, 0.0)
    bad = j.copy()
    bad[1, 2] += 1e-12
    assert "symmetric" in _create_error(Couplings(dense=bad))
    bad = j.copy()
    bad[3, 3] = 0.5
    assert "zero diagonal" in _create_error(Couplings(dense=bad))
    bad = j.copy()
    bad[0, 4] = bad[4, 0] = np.inf
    assert "finite" in _create_error(Couplings(dense=bad))
    # CSR: rows 0-1-2 coupled in a chain
    ptr = np.array([0, 1, 3, 4], np.uint64)
    assert "ascend" in _create_error(Couplings(row_offsets=ptr, columns=np.array([1, 2, 0, 1], np.uint64),
                                               values=np.array([0.5, 0.3, 0.5, 0.3])))
    assert "symmetric" in _create_error(Couplings(row_offsets=ptr, columns=np.array([1, 0, 2, 1], np.uint64),
                                                  values=np.array([0.5, 0.5, 0.3, 0.4])))
    assert "zero diagonal" in _create_error(Couplings(row_offsets=np.array([0, 1, 1, 1], np.uint64),
                                                      columns=np.array([0], np.uint64), values=np.array([1.0])))
    with pytest.raises(InvalidArgument):
        Couplings(dense=np.zeros((3, 4)))
