"""The allocation-free local-fields entry point.

wlg_local_fields_noalloc serves callers that cannot allocate device memory -- for example
a host whose memory pool already owns almost all of the GPU, or code that must not add the
device synchronisation that cudaMalloc/cudaFree can cause.  It keeps every intermediate in
one static device array.  These tests call it through the C-ABI and compare it with the
allocating entry point, wlg_local_fields, bit for bit (the tolerance every FP64 parity test
here uses), on two calls in a row, so that the second call shows that what the first call
left in the shared array does not leak into its results.  This file is collected last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from replica_exchange_wang_landau_b200._abi import load_library
from replica_exchange_wang_landau_b200.engine import Geometry, System
from replica_exchange_wang_landau_b200.geometry import random_sphere_axes

pytestmark = pytest.mark.gpu


def _system(dims, seed, box=None, periodic=True):
    g = Geometry.simple_cubic(*dims, periodic=periodic)
    g.axes = random_sphere_axes(g.size(), seed)
    if box is not None:
        g.box = box
    return System(g, 0.8, 0.0)


def _call(fn, system, spins, with_energies=True):
    fields = np.full(spins.shape, np.nan)
    energies = np.full(spins.shape[0], np.nan)
    s = system._struct()
    energy_ptr = energies.ctypes.data_as(C.POINTER(C.c_double)) if with_energies else None
    status = fn(C.byref(s), spins.ctypes.data_as(C.POINTER(C.c_int8)), spins.shape[0],
                fields.ctypes.data_as(C.POINTER(C.c_double)), energy_ptr)
    return status, fields, energies


def test_no_alloc_matches_allocating_entry_point_on_two_calls():
    lib = load_library()
    rng = np.random.default_rng(7)
    # a large call first, then a smaller one: the second must not see the first's leftovers
    cases = [(_system((8, 8, 8), 1), 6), (_system((5, 4, 3), 2, box=(5.0, 4.0, 0.0)), 3)]
    for system, count in cases:
        spins = np.ascontiguousarray(rng.choice(np.array([-1, 1], np.int8), size=(count, system.size())))
        st_a, fa, ea = _call(lib.wlg_local_fields, system, spins)
        st_b, fb, eb = _call(lib.wlg_local_fields_noalloc, system, spins)
        assert st_a == 0 and st_b == 0, lib.wlg_last_error()
        assert np.array_equal(fa.view(np.uint64), fb.view(np.uint64))
        assert np.array_equal(ea.view(np.uint64), eb.view(np.uint64))


def test_no_alloc_single_configuration_and_no_energies():
    # count == 1 takes the one-configuration field kernel; energies may be NULL
    lib = load_library()
    rng = np.random.default_rng(11)
    for system, with_energies in [(_system((6, 6, 6), 8), True), (_system((4, 4, 2), 9, box=(4.0, 4.0, 0.0)), False)]:
        spins = np.ascontiguousarray(rng.choice(np.array([-1, 1], np.int8), size=(1, system.size())))
        st_a, fa, ea = _call(lib.wlg_local_fields, system, spins, with_energies)
        st_b, fb, eb = _call(lib.wlg_local_fields_noalloc, system, spins, with_energies)
        assert st_a == 0 and st_b == 0, lib.wlg_last_error()
        assert np.array_equal(fa.view(np.uint64), fb.view(np.uint64))
        if with_energies:
            assert np.array_equal(ea.view(np.uint64), eb.view(np.uint64))
        else:
            assert np.isnan(eb).all()


def test_no_alloc_rejects_inputs_beyond_its_limits():
    lib = load_library()
    big = _system((11, 10, 10), 3)  # 1100 sites > 1024
    spins = np.ones((1, big.size()), np.int8)
    status, _, _ = _call(lib.wlg_local_fields_noalloc, big, spins)
    assert status == 1 and b"at most 1024 sites" in lib.wlg_last_error()
    csr = System(_system((3, 3, 3), 4).geometry, 1.0, 2.0)
    status, _, _ = _call(lib.wlg_local_fields_noalloc, csr, np.ones((1, 27), np.int8))
    assert status == 1 and b"dense couplings only" in lib.wlg_last_error()
    many = _system((4, 4, 4), 5)
    status, _, _ = _call(lib.wlg_local_fields_noalloc, many, np.ones((20000, 64), np.int8))
    assert status == 1 and b"configurations" in lib.wlg_last_error()
