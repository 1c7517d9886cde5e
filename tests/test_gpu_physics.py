"""GPU parity: coupling construction and local fields (src/physics.cpp:151-266) through the
C-ABI, bit for bit against the oracle and the golden fixtures."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import random_axes, same_double, system_from, unhex
from replica_exchange_wang_landau_b200.engine import Geometry, InvalidArgument, System

pytestmark = pytest.mark.gpu


def _systems():
    out = []
    for dims, periodic, box, cutoff, seed in [((2, 2, 2), False, None, 0.0, 1), ((3, 3, 3), True, None, 0.0, 2),
                                              ((5, 4, 3), True, (5.0, 4.0, 0.0), 0.0, 3),
                                              ((7, 5, 3), True, None, 0.0, 4), ((4, 4, 4), True, None, 1.8, 5),
                                              ((6, 6, 6), True, None, 3.0, 6), ((5, 3, 2), False, None, 2.5, 7),
                                              ((17, 1, 1), False, None, 0.0, 8)]:
        g = Geometry.simple_cubic(*dims, periodic=periodic)
        g.axes = random_axes(g.size(), seed)
        if box:
            g.box = box
        out.append(System(g, 0.9, cutoff))
    return out


@pytest.mark.parametrize("k", range(8))
def test_couplings_bitwise(oracle, k):
    s = _systems()[k]
    assert same_double(s.couplings(), oracle.couplings(s))


@pytest.mark.parametrize("name", ["cubic27_periodic", "slab24", "csr64_r1.8"])
def test_couplings_golden(golden, name):
    g = golden["systems"][name]
    s = system_from(g)
    assert same_double(s.couplings().ravel(), unhex(g["couplings"]))
    fields, energies = s.local_fields(np.array(g["spins"], dtype=np.int8))
    assert same_double(fields.ravel(), unhex(g["fields"]))
    assert same_double(energies, unhex(g["energies"]))


@pytest.mark.parametrize("k", range(8))
def test_local_fields_bitwise(oracle, k):
    s = _systems()[k]
    rng = np.random.default_rng(k)
    spins = rng.choice(np.array([-1, 1], dtype=np.int8), size=(4, s.size()))
    f, e = s.local_fields(spins)
    fo, eo = oracle.local_fields(s, spins)
    assert same_double(f, fo)
    assert same_double(e, eo)


def test_csr_structure(oracle):
    s = _systems()[5]
    ptr, cols, vals = s.csr()
    dense = oracle.couplings(s)
    n = s.size()
    # in a 6^3 periodic box the images at +3 and -3 along an axis are the same site, so the
    # count is below the 122 neighbours of an infinite lattice; the oracle has the exact count
    assert ptr[-1] == len(cols) == oracle.csr_nnz(s)
    for i in range(n):
        row = cols[ptr[i]:ptr[i + 1]]
        assert np.all(np.diff(row.astype(np.int64)) > 0)  # sorted by column
        assert same_double(vals[ptr[i]:ptr[i + 1]], dense[i, row.astype(np.int64)])


def _cell_systems():
    """Cutoff systems whose cell grid has several cells per axis, or overflows the row sort."""
    from replica_exchange_wang_landau_b200.geometry import random_sequential, simple_cubic_random
    out = {}
    out["periodic12_r2.5"] = System(simple_cubic_random(12, 12, 12, seed=31), 1.0, 2.5)  # 4 cells per axis
    out["periodic12_r3.0"] = System(simple_cubic_random(12, 12, 12, seed=32), 1.0, 3.0)  # 3 cells, pairs at exactly r
    shifted = simple_cubic_random(10, 9, 8, seed=33)
    shifted.positions = shifted.positions + np.array([-7.3, 23.9, -100.25])  # wrapped into the box by the grid
    out["shifted_r2.0"] = System(shifted, 1.0, 2.0)
    out["slab12x12x10_r2.0"] = System(simple_cubic_random(12, 12, 10, seed=34, box=(12.0, 12.0, 0.0)), 1.0, 2.0)
    out["open10_r2.2"] = System(simple_cubic_random(10, 10, 10, seed=35, periodic=False), 1.0, 2.2)
    out["dilute1000_r3.0"] = System(random_sequential(1000, 0.5, 0.8, seed=36), 1.0, 3.0)
    out["long_rows_r6.5"] = System(simple_cubic_random(14, 14, 14, seed=37), 1.0, 6.5)  # > 1024 per row
    return out


@pytest.mark.parametrize("name", list(_cell_systems()))
def test_cell_list_csr_bitwise(oracle, name):
    """The cell-list CSR build (O(N z)) gives the reference's O(N^2) scan exactly: the same
    row lengths, columns in the same order and bit-identical values."""
    s = _cell_systems()[name]
    ptr, cols, vals = s.csr()
    optr, ocols, ovals = oracle.csr(s)
    assert np.array_equal(ptr.astype(np.uint64), optr)
    assert np.array_equal(cols.astype(np.uint64), ocols)
    assert same_double(vals, ovals)


@pytest.mark.parametrize("precision,rtol", [("fp32", 2.0 ** -24), ("bf16", 2.0 ** -8)])
def test_low_precision_couplings(precision, rtol):
    s = _systems()[3]
    j64 = s.couplings("fp64")
    jl = s.couplings(precision)
    scale = np.abs(j64).max(axis=1, keepdims=True) if precision == "bf16" else np.abs(j64)
    assert np.all(np.abs(jl - j64) <= rtol * scale + 1e-300)


def test_coincident_sites_rejected():
    g = Geometry(np.zeros((2, 3)), np.tile([0.0, 0.0, 1.0], (2, 1)), (0, 0, 0), False)
    with pytest.raises(InvalidArgument, match="Coincident dipole sites"):
        System(g).couplings()


def test_local_fields_many_configurations_bitwise(oracle):
    """70 configurations of an 1100-site system in the grouped field kernel (groups of 8 and a
    last group of 6); every field and energy equals the oracle's sequential sum."""
    g = Geometry.simple_cubic(11, 10, 10, periodic=True)
    g.axes = random_axes(g.size(), 77)
    s = System(g, 1.0, 0.0)
    rng = np.random.default_rng(5)
    spins = rng.choice(np.array([-1, 1], dtype=np.int8), size=(70, s.size()))
    f, e = s.local_fields(spins)
    fo, eo = oracle.local_fields(s, spins)
    assert same_double(f, fo)
    assert same_double(e, eo)
