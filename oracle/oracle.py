"""TEST INFRASTRUCTURE ONLY: Python access to the two CPU checkers.

* ``Oracle``  -- the plain-C restatement of the reference's hot path (wl_oracle.c),
  loaded from oracle/_build/libwl_oracle.so.
* ``Reference`` -- the unmodified reference library compiled from its own sources
  (oracle/_ref/libwlref.so via ref_shim.cpp).

Both expose the same small API (couplings, fields, exact enumeration, single walkers,
run_rewl) over the engine's C-ABI structs, so a test can run one scenario on the GPU
engine and on either checker and compare.  Only tests/, __graft_entry__.smoke() and the
CPU legs of bench.py import this module.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass
from pathlib import Path
from typing import Optional

import numpy as np

from replica_exchange_wang_landau_b200 import _abi
from replica_exchange_wang_landau_b200.engine import (DosFragment, RewlResult, RunConfig, Snapshot, System,
                                                      WindowSamplingStatistics)

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "_build" / "libwl_oracle.so"
REF_LIB = HERE / "_ref" / "libwlref.so"
REF_BIN = HERE / "_ref"

P = C.POINTER
_u64, _i64, _i32, _dbl, _vp, _cp, _sz = C.c_uint64, C.c_int64, C.c_int32, C.c_double, C.c_void_p, C.c_char_p, C.c_size_t


# Where the reference's source tree is read from when it is present (the build container);
# WL_REFERENCE_DIR overrides it.  Machines without it use the prebuilt oracle/_ref files.
REFERENCE_SOURCES = Path(os.environ.get("WL_REFERENCE_DIR", "/root/reference"))


def build() -> None:
    """Runs oracle/Makefile (compiles the restatement; the reference too when its sources
    are present)."""
    cmd = ["make", "-s", "-C", str(HERE)]
    if (REFERENCE_SOURCES / "src" / "physics.cpp").exists():
        cmd.append(f"REF={REFERENCE_SOURCES}")
    subprocess.run(cmd, check=True)


def reference_available() -> bool:
    return REF_LIB.exists()


class CheckerError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = _abi.STATUS_NAMES.get(status, str(status))


def _err():
    return C.create_string_buffer(4096)


def _raise(status: int, buf) -> None:
    if status:
        raise CheckerError(status, buf.value.decode(errors="replace"))


def _dptr(a):
    return a.ctypes.data_as(P(C.c_double))


def _u64ptr(a):
    return a.ctypes.data_as(P(C.c_uint64))


def _i8ptr(a):
    return a.ctypes.data_as(P(C.c_int8))


def _u8ptr(a):
    return a.ctypes.data_as(P(C.c_uint8))


class _Checker:
    """Common wrapper; `prefix` is "orc" (restatement) or "ref" (compiled reference)."""

    prefix = ""
    path: Path = Path()

    def __init__(self):
        if not self.path.exists():
            build()
        self.lib = C.CDLL(str(self.path))
        self._declare()

    def _declare(self):
        raise NotImplementedError

    # physics -------------------------------------------------------------------
    def dipolar_pair(self, d, ai, aj, scale=1.0) -> float:
        f = getattr(self.lib, f"{self.prefix}_dipolar_pair")
        return f((C.c_double * 3)(*d), (C.c_double * 3)(*ai), (C.c_double * 3)(*aj), scale)

    def minimum_image(self, d, box, periodic=True):
        out = (C.c_double * 3)()
        getattr(self.lib, f"{self.prefix}_minimum_image")((C.c_double * 3)(*d), (C.c_double * 3)(*box),
                                                         1 if periodic else 0, out)
        return tuple(out)


class Oracle(_Checker):
    prefix = "orc"
    path = ORACLE_LIB

    def _declare(self):
        L = self.lib
        sig = {
            "orc_dipolar_pair": (_dbl, [P(_dbl), P(_dbl), P(_dbl), _dbl]),
            "orc_minimum_image": (None, [P(_dbl), P(_dbl), C.c_int, P(_dbl)]),
            "orc_couplings_create": (_vp, [P(_abi.wlg_system), _cp, _sz]),
            "orc_couplings_destroy": (None, [_vp]),
            "orc_couplings_size": (_u64, [_vp]),
            "orc_couplings_nnz": (_u64, [_vp]),
            "orc_couplings_set_update_fp32": (None, [_vp, C.c_int]),
            "orc_couplings_csr": (None, [_vp, P(_u64), P(_u64), P(_dbl)]),
            "orc_couplings_dense": (None, [_vp, P(_dbl)]),
            "orc_local_fields": (None, [_vp, P(C.c_int8), P(_dbl)]),
            "orc_total_energy": (_dbl, [_vp, P(C.c_int8)]),
            "orc_grid_bins": (C.c_int, [_dbl, _dbl, _dbl, P(_u64)]),
            "orc_grid_index": (_i64, [_dbl, _dbl, _dbl, _dbl]),
            "orc_partition_windows": (C.c_int, [_u64, _u64, _dbl, P(_u64)]),
            "orc_walker_create": (_vp, [_vp, _u64, _dbl, _dbl, _dbl, _u64, _u64, P(_abi.wlg_wl_parameters), _u64,
                                        P(C.c_int8), _cp, _sz]),
            "orc_walker_destroy": (None, [_vp]),
            "orc_walker_attempt": (C.c_int, [_vp, P(C.c_int), _cp, _sz]),
            "orc_walker_run": (C.c_int, [_vp, _u64, _cp, _sz]),
            "orc_walker_snapshot": (None, [_vp, P(_abi.wlg_snapshot)]),
            "orc_walker_restore": (C.c_int, [_vp, P(_abi.wlg_snapshot), _cp, _sz]),
            "orc_walker_histogram_statistics": (None, [_vp, P(_abi.wlg_histogram_statistics)]),
            "orc_walker_flags": (None, [_vp, P(C.c_int), P(C.c_int), P(C.c_int)]),
            "orc_walker_begin_next_iteration": (C.c_int, [_vp, _cp, _sz]),
            "orc_walker_exchange_log_probability": (_dbl, [_vp, _vp]),
            "orc_walker_swap": (C.c_int, [_vp, _vp, _cp, _sz]),
            "orc_walker_counters": (None, [_vp, P(_u64)]),
            "orc_walker_pilot": (None, [_vp, P(_dbl), P(_u64), P(_u64), P(_dbl), P(C.c_int8), P(C.c_uint8)]),
            "orc_run_rewl": (_vp, [_vp, P(_abi.wlg_run_config), _cp, _sz]),
            "orc_run_rewl_warm": (_vp, [_vp, P(_abi.wlg_run_config), P(_dbl), _dbl, C.c_int, _cp, _sz]),
            "orc_walker_warm_start": (None, [_vp, P(_dbl), _dbl, C.c_int]),
            "orc_result_destroy": (None, [_vp]),
            "orc_result_totals": (None, [_vp, P(_abi.wlg_run_totals)]),
            "orc_result_fragment": (C.c_int, [_vp, _u64, P(_dbl), P(_u64), P(_dbl), P(C.c_uint8)]),
            "orc_result_walker_statistics": (_u64, [_vp, P(_abi.wlg_walker_statistics), _u64]),
            "orc_result_sampling": (C.c_int, [_vp, _u64, P(_dbl), P(_u64), P(_u64), P(_u64)]),
            "orc_result_representatives": (_u64, [_vp, P(_dbl), P(C.c_int8), _u64]),
            "orc_exact_enumeration": (C.c_int, [_vp, _dbl, _dbl, _dbl, P(_u64)]),
        }
        for name, (res, args) in sig.items():
            getattr(L, name).restype = res
            getattr(L, name).argtypes = args

    def _couplings(self, system: System):
        err = _err()
        s = system._struct()
        h = self.lib.orc_couplings_create(C.byref(s), err, len(err))
        if not h:
            raise CheckerError(1, err.value.decode())
        return h

    def couplings(self, system: System) -> np.ndarray:
        h = self._couplings(system)
        n = system.size()
        out = np.zeros((n, n))
        self.lib.orc_couplings_dense(h, _dptr(out))
        self.lib.orc_couplings_destroy(h)
        return out

    def csr_nnz(self, system: System) -> int:
        """Number of stored couplings (CSR) of the restated CsrCouplings."""
        h = self._couplings(system)
        nnz = int(self.lib.orc_couplings_nnz(h))
        self.lib.orc_couplings_destroy(h)
        return nnz

    def csr(self, system: System):
        """(offsets, columns, values) of the restated CsrCouplings."""
        h = self._couplings(system)
        try:
            n = system.size()
            nnz = int(self.lib.orc_couplings_nnz(h))
            ptr = np.zeros(n + 1, np.uint64)
            cols = np.zeros(max(1, nnz), np.uint64)
            vals = np.zeros(max(1, nnz), np.float64)
            self.lib.orc_couplings_csr(h, _u64ptr(ptr), _u64ptr(cols), _dptr(vals))
            return ptr, cols[:nnz], vals[:nnz]
        finally:
            self.lib.orc_couplings_destroy(h)

    def local_fields(self, system: System, spins: np.ndarray):
        h = self._couplings(system)
        s = np.ascontiguousarray(spins, dtype=np.int8).reshape(-1, system.size())
        fields = np.zeros(s.shape)
        energies = np.zeros(s.shape[0])
        for k in range(s.shape[0]):
            row = np.ascontiguousarray(s[k])
            f = np.zeros(system.size())
            self.lib.orc_local_fields(h, _i8ptr(row), _dptr(f))
            fields[k] = f
            energies[k] = self.lib.orc_total_energy(h, _i8ptr(row))
        self.lib.orc_couplings_destroy(h)
        return fields, energies

    def grid_index(self, emin, emax, width, energy) -> Optional[int]:
        b = self.lib.orc_grid_index(emin, emax, width, energy)
        return None if b < 0 else int(b)

    def partition_windows(self, bins, count, overlap):
        out = np.zeros(2 * count, np.uint64)
        st = self.lib.orc_partition_windows(bins, count, overlap, _u64ptr(out))
        if st:
            raise CheckerError(st, "Invalid energy-window partition")
        return [(int(out[2 * i]), int(out[2 * i + 1])) for i in range(count)]

    def exact_counts(self, system: System, emin, emax, width) -> np.ndarray:
        h = self._couplings(system)
        bins = C.c_uint64(0)
        self.lib.orc_grid_bins(emin, emax, width, C.byref(bins))
        counts = np.zeros(bins.value, np.uint64)
        st = self.lib.orc_exact_enumeration(h, emin, emax, width, _u64ptr(counts))
        self.lib.orc_couplings_destroy(h)
        if st:
            raise CheckerError(st, "System too large for exact enumeration")
        return counts

    def walker(self, system: System, walker_id: int, emin, emax, width, window, params, seed,
               spins: Optional[np.ndarray] = None) -> "CheckerWalker":
        return CheckerWalker(self, system, walker_id, emin, emax, width, window, params, seed, spins)

    def run_rewl(self, system: System, config: RunConfig, warm_start=None) -> RewlResult:
        """run_rewl; warm_start = (log_g over the grid, factor, continue_schedule) applies the
        engine's warm start to every walker after construction."""
        h = self._couplings(system)
        try:
            c, keep = config._struct(system.size())
            err = _err()
            if warm_start is None:
                r = self.lib.orc_run_rewl(h, C.byref(c), err, len(err))
            else:
                lg = np.ascontiguousarray(warm_start[0], dtype=np.float64)
                r = self.lib.orc_run_rewl_warm(h, C.byref(c), _dptr(lg), float(warm_start[1]),
                                               1 if warm_start[2] else 0, err, len(err))
            if not r:
                raise CheckerError(6, err.value.decode())
            try:
                return _collect_result(self.lib, "orc", r, system.size(), config)
            finally:
                self.lib.orc_result_destroy(r)
        finally:
            self.lib.orc_couplings_destroy(h)


class Reference(_Checker):
    prefix = "ref"
    path = REF_LIB

    def _declare(self):
        L = self.lib
        sysp, cfgp = P(_abi.wlg_system), P(_abi.wlg_run_config)
        sig = {
            "ref_set_threads": (C.c_int, [C.c_int]),
            "ref_dipolar_pair": (_dbl, [P(_dbl), P(_dbl), P(_dbl), _dbl]),
            "ref_minimum_image": (None, [P(_dbl), P(_dbl), C.c_int, P(_dbl)]),
            "ref_grid_index": (C.c_int, [_dbl, _dbl, _dbl, _dbl, P(_i64)]),
            "ref_partition_windows": (C.c_int, [_u64, _u64, _dbl, P(_u64), _cp, _sz]),
            "ref_couplings_dense": (C.c_int, [sysp, P(_dbl), _cp, _sz]),
            "ref_fields": (C.c_int, [sysp, P(C.c_int8), _u64, P(_dbl), P(_dbl), _cp, _sz]),
            "ref_exact_enumeration": (C.c_int, [sysp, _dbl, _dbl, _dbl, P(_u64), _cp, _sz]),
            "ref_walker_create": (_vp, [sysp, _u64, _dbl, _dbl, _dbl, _u64, _u64, P(_abi.wlg_wl_parameters), _u64,
                                        P(C.c_int8), _cp, _sz]),
            "ref_walker_destroy": (None, [_vp]),
            "ref_walker_run": (C.c_int, [_vp, _u64, _cp, _sz]),
            "ref_walker_attempt": (C.c_int, [_vp, P(C.c_int), _cp, _sz]),
            "ref_walker_snapshot": (C.c_int, [_vp, P(_abi.wlg_snapshot)]),
            "ref_walker_restore": (C.c_int, [_vp, P(_abi.wlg_snapshot), _cp, _sz]),
            "ref_walker_histogram_statistics": (None, [_vp, P(_abi.wlg_histogram_statistics)]),
            "ref_walker_flags": (None, [_vp, P(C.c_int), P(C.c_int), P(C.c_int)]),
            "ref_walker_begin_next_iteration": (C.c_int, [_vp, _cp, _sz]),
            "ref_walker_exchange_log_probability": (_dbl, [_vp, _vp]),
            "ref_walker_swap": (C.c_int, [_vp, _vp, _cp, _sz]),
            "ref_walker_counters": (None, [_vp, P(_u64)]),
            "ref_walker_pilot": (None, [_vp, P(_dbl), P(_u64), P(_u64), P(_dbl), P(C.c_int8), P(C.c_uint8)]),
            "ref_run_rewl": (_vp, [sysp, cfgp, _cp, _sz]),
            "ref_result_destroy": (None, [_vp]),
            "ref_result_totals": (None, [_vp, P(_abi.wlg_run_totals)]),
            "ref_result_fragment": (C.c_int, [_vp, _u64, P(_dbl), P(_u64), P(_dbl), P(C.c_uint8)]),
            "ref_result_walker_statistics": (_u64, [_vp, P(_abi.wlg_walker_statistics), _u64]),
            "ref_result_sampling": (C.c_int, [_vp, _u64, P(_dbl), P(_u64), P(_u64), P(_u64)]),
            "ref_result_representatives": (_u64, [_vp, P(_dbl), P(C.c_int8), _u64]),
            "ref_adapt_windows": (C.c_int, [_vp, _dbl, _dbl, _dbl, _u64, _dbl, P(_u64), _cp, _sz]),
            "ref_stitch_dos": (C.c_int, [_dbl, _dbl, _dbl, P(_abi.wlg_fragment_view), _u64, C.c_int, _u64, P(_dbl),
                                         P(_u64), P(_dbl), P(C.c_uint8), P(_u64), C.c_char_p, _cp, _sz]),
            "ref_write_fragment_csv": (C.c_int, [C.c_char_p, _dbl, _dbl, _dbl, P(_abi.wlg_fragment_view), _u64, _cp,
                                                 _sz]),
            "ref_write_workers_stat_csv": (C.c_int, [C.c_char_p, P(_abi.wlg_walker_statistics), _u64, _u64, _cp,
                                                     _sz]),
            "ref_select_initial": (C.c_int, [_vp, _dbl, _dbl, _dbl, P(_u64), _u64, _u64, _u64, P(C.c_int8),
                                             P(C.c_uint8), P(_u64), P(_u64), _cp, _sz]),
        }
        for name, (res, args) in sig.items():
            getattr(L, name).restype = res
            getattr(L, name).argtypes = args

    def set_threads(self, threads: int) -> int:
        return int(self.lib.ref_set_threads(int(threads)))

    def pilot_round(self, system: System, config: RunConfig):
        """(result, adapted windows, seeds per walker, missing, external) of one reference round."""
        return _pilot_round(self, system, config)

    def stitch_dos(self, views, emin, emax, width, complete_range: bool, spins: int, dos_csv: str = ""):
        """wl::stitch_dos on wlg_fragment_view inputs; also writes <dos_csv> when given."""
        bins = int(round((emax - emin) / width))
        lg, se = np.zeros(bins), np.zeros(bins)
        h, v = np.zeros(bins, np.uint64), np.zeros(bins, np.uint8)
        joins = np.zeros(max(1, len(views) - 1), np.uint64)
        arr = (_abi.wlg_fragment_view * len(views))(*views)
        err = _err()
        _raise(self.lib.ref_stitch_dos(emin, emax, width, arr, len(views), int(complete_range), spins, _dptr(lg),
                                       _u64ptr(h), _dptr(se), _u8ptr(v), _u64ptr(joins), str(dos_csv).encode(), err,
                                       len(err)), err)
        return lg, h, se, v, joins[:len(views) - 1]

    def write_fragment_csv(self, path, view, emin, emax, width, window_id: int) -> None:
        err = _err()
        _raise(self.lib.ref_write_fragment_csv(str(path).encode(), emin, emax, width, C.byref(view), window_id, err,
                                               len(err)), err)

    def write_workers_stat_csv(self, path, rows, spins: int) -> None:
        """wl::write_workers_stat_csv on a ctypes array of wlg_walker_statistics."""
        err = _err()
        _raise(self.lib.ref_write_workers_stat_csv(str(path).encode(), rows, len(rows), spins, err, len(err)), err)

    def couplings(self, system: System) -> np.ndarray:
        n = system.size()
        out = np.zeros((n, n))
        err = _err()
        _raise(self.lib.ref_couplings_dense(C.byref(system._struct()), _dptr(out), err, len(err)), err)
        return out

    def local_fields(self, system: System, spins: np.ndarray):
        s = np.ascontiguousarray(spins, dtype=np.int8).reshape(-1, system.size())
        fields = np.zeros(s.shape)
        energies = np.zeros(s.shape[0])
        err = _err()
        _raise(self.lib.ref_fields(C.byref(system._struct()), _i8ptr(s), s.shape[0], _dptr(fields), _dptr(energies),
                                   err, len(err)), err)
        return fields, energies

    def grid_index(self, emin, emax, width, energy) -> Optional[int]:
        b = C.c_int64(0)
        self.lib.ref_grid_index(emin, emax, width, energy, C.byref(b))
        return None if b.value < 0 else int(b.value)

    def partition_windows(self, bins, count, overlap):
        out = np.zeros(2 * count, np.uint64)
        err = _err()
        _raise(self.lib.ref_partition_windows(bins, count, overlap, _u64ptr(out), err, len(err)), err)
        return [(int(out[2 * i]), int(out[2 * i + 1])) for i in range(count)]

    def exact_counts(self, system: System, emin, emax, width) -> np.ndarray:
        bins = int(round((emax - emin) / width))
        counts = np.zeros(bins, np.uint64)
        err = _err()
        _raise(self.lib.ref_exact_enumeration(C.byref(system._struct()), emin, emax, width, _u64ptr(counts), err,
                                              len(err)), err)
        return counts

    def walker(self, system: System, walker_id: int, emin, emax, width, window, params, seed,
               spins: Optional[np.ndarray] = None) -> "CheckerWalker":
        return CheckerWalker(self, system, walker_id, emin, emax, width, window, params, seed, spins)

    def run_rewl(self, system: System, config: RunConfig) -> RewlResult:
        c, keep = config._struct(system.size())
        err = _err()
        r = self.lib.ref_run_rewl(C.byref(system._struct()), C.byref(c), err, len(err))
        if not r:
            raise CheckerError(6, err.value.decode())
        try:
            return _collect_result(self.lib, "ref", r, system.size(), config)
        finally:
            self.lib.ref_result_destroy(r)


def _pilot_round(ref: "Reference", system: System, config: RunConfig):
    """One adaptive-window round of the reference: run_rewl with pilot statistics, then its
    adapt_energy_windows and select_adaptive_initial_configurations on that result."""
    c, keep = config._struct(system.size())
    err = _err()
    lib = ref.lib
    r = lib.ref_run_rewl(C.byref(system._struct()), C.byref(c), err, len(err))
    if not r:
        raise CheckerError(6, err.value.decode())
    try:
        result = _collect_result(lib, "ref", r, system.size(), config)
        count = int(config.windows)
        w = np.zeros(2 * count, np.uint64)
        _raise(lib.ref_adapt_windows(r, config.emin, config.emax, config.bin_width, count, config.overlap,
                                     _u64ptr(w), err, len(err)), err)
        n = system.size()
        total = count * int(config.walkers)
        spins = np.zeros((total, n), np.int8)
        present = np.zeros(total, np.uint8)
        missing, external = C.c_uint64(0), C.c_uint64(0)
        _raise(lib.ref_select_initial(r, config.emin, config.emax, config.bin_width, _u64ptr(w), count,
                                      int(config.walkers), n, _i8ptr(spins), _u8ptr(present), C.byref(missing),
                                      C.byref(external), err, len(err)), err)
        windows = [(int(w[2 * k]), int(w[2 * k + 1])) for k in range(count)]
        seeds = [spins[k].copy() if present[k] else None for k in range(total)]
        return result, windows, seeds, int(missing.value), int(external.value)
    finally:
        lib.ref_result_destroy(r)


def _collect_result(lib, prefix, r, n, config: RunConfig) -> RewlResult:
    f = lambda name: getattr(lib, f"{prefix}_{name}")  # noqa: E731
    t = _abi.wlg_run_totals()
    f("result_totals")(r, C.byref(t))
    bins = config.bins()
    frags = []
    windows = config.explicit_windows or None
    for w in range(int(config.windows)):
        lg, h, se, v = np.zeros(bins), np.zeros(bins, np.uint64), np.zeros(bins), np.zeros(bins, np.uint8)
        f("result_fragment")(r, w, _dptr(lg), _u64ptr(h), _dptr(se), _u8ptr(v))
        frags.append(DosFragment(tuple(windows[w]) if windows else None, lg, h, se, v))
    count = int(config.windows) * int(config.walkers)
    stats = (_abi.wlg_walker_statistics * count)()
    f("result_walker_statistics")(r, stats, count)
    stat_list = [{name: getattr(s, name) for name, _ in _abi.wlg_walker_statistics._fields_} for s in stats]
    sampling, reps = [], []
    if config.wl.collect_window_statistics:
        for w in range(int(config.windows)):
            sq, ds = np.zeros(bins), np.zeros(bins, np.uint64)
            trips, walkers = C.c_uint64(0), C.c_uint64(0)
            f("result_sampling")(r, w, _dptr(sq), _u64ptr(ds), C.byref(trips), C.byref(walkers))
            sampling.append(WindowSamplingStatistics(None, sq, ds, int(trips.value), int(walkers.value)))
        k = int(f("result_representatives")(r, None, None, 0))
        e = np.zeros(max(1, k))
        s = np.zeros((max(1, k), n), np.int8)
        f("result_representatives")(r, _dptr(e), _i8ptr(s), k)
        reps = [(float(e[i]), s[i].copy()) for i in range(k)]
    return RewlResult(frags, stat_list, sampling, reps, t.attempted, t.accepted, t.forced_accepted,
                      t.exchange_attempted, t.exchange_accepted, bool(t.converged), t.epochs)


class CheckerWalker:
    """A WangLandauWalker held by a checker (restatement or reference)."""

    def __init__(self, checker: _Checker, system: System, walker_id, emin, emax, width, window, params, seed,
                 spins=None):
        self.c = checker
        self.L = checker.lib
        self.p = checker.prefix
        self.n = system.size()
        self.bins = int(round((emax - emin) / width))
        self._system = system
        err = _err()
        sp = None
        if spins is not None:
            self._spins = np.ascontiguousarray(spins, dtype=np.int8)
            sp = _i8ptr(self._spins)
        self._params = params._struct()
        if self.p == "orc":
            self._coup = checker._couplings(system)
            self.h = self.L.orc_walker_create(self._coup, walker_id, emin, emax, width, window[0], window[1],
                                              C.byref(self._params), seed, sp, err, len(err))
        else:
            self._coup = None
            self.h = self.L.ref_walker_create(C.byref(system._struct()), walker_id, emin, emax, width, window[0],
                                              window[1], C.byref(self._params), seed, sp, err, len(err))
        if not self.h:
            raise CheckerError(2, err.value.decode())

    def close(self):
        if self.h:
            getattr(self.L, f"{self.p}_walker_destroy")(self.h)
            self.h = None
        if self._coup:
            self.L.orc_couplings_destroy(self._coup)
            self._coup = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _fn(self, name):
        return getattr(self.L, f"{self.p}_{name}")

    def set_update_fp32(self, on: bool = True):
        """Follow an FP32 engine walker from here on: flips add m * float(J) (restatement only)."""
        if self.p != "orc":
            raise CheckerError(1, "only the restatement has the FP32 update")
        self.L.orc_couplings_set_update_fp32(self._coup, 1 if on else 0)

    def warm_start(self, log_g: np.ndarray, factor: float, continue_schedule: bool = False):
        """The engine's warm start (restatement only; the reference has none)."""
        if self.p != "orc":
            raise CheckerError(7, "the reference has no warm start")
        self._warm = np.ascontiguousarray(log_g, dtype=np.float64)
        self.L.orc_walker_warm_start(self.h, _dptr(self._warm), float(factor), 1 if continue_schedule else 0)

    def run_attempts(self, count: int):
        err = _err()
        _raise(self._fn("walker_run")(self.h, count, err, len(err)), err)

    def attempt_flip(self) -> bool:
        acc = C.c_int(0)
        err = _err()
        _raise(self._fn("walker_attempt")(self.h, C.byref(acc), err, len(err)), err)
        return bool(acc.value)

    def snapshot(self) -> Snapshot:
        s, arrays = Snapshot._empty(self.n, self.bins)
        self._fn("walker_snapshot")(self.h, C.byref(s))
        return Snapshot._from(s, arrays)

    def restore(self, snapshot: Snapshot):
        s, keep = snapshot._struct()
        err = _err()
        _raise(self._fn("walker_restore")(self.h, C.byref(s), err, len(err)), err)

    def histogram_statistics(self) -> dict:
        s = _abi.wlg_histogram_statistics()
        self._fn("walker_histogram_statistics")(self.h, C.byref(s))
        return {name: getattr(s, name) for name, _ in _abi.wlg_histogram_statistics._fields_}

    def flags(self):
        a, b, c = C.c_int(0), C.c_int(0), C.c_int(0)
        self._fn("walker_flags")(self.h, C.byref(a), C.byref(b), C.byref(c))
        return bool(a.value), bool(b.value), bool(c.value)

    def begin_next_iteration(self):
        err = _err()
        _raise(self._fn("walker_begin_next_iteration")(self.h, err, len(err)), err)

    def exchange_log_probability(self, other: "CheckerWalker") -> float:
        return float(self._fn("walker_exchange_log_probability")(self.h, other.h))

    def swap_configuration(self, other: "CheckerWalker"):
        err = _err()
        _raise(self._fn("walker_swap")(self.h, other.h, err, len(err)), err)

    def counters(self):
        out = (C.c_uint64 * 4)()
        self._fn("walker_counters")(self.h, out)
        return tuple(int(x) for x in out)

    def pilot(self):
        sq, ds = np.zeros(self.bins), np.zeros(self.bins, np.uint64)
        trips = C.c_uint64(0)
        e = np.zeros(9)
        s = np.zeros((9, self.n), np.int8)
        present = np.zeros(9, np.uint8)
        self._fn("walker_pilot")(self.h, _dptr(sq), _u64ptr(ds), C.byref(trips), _dptr(e), _i8ptr(s), _u8ptr(present))
        return sq, ds, int(trips.value), e, s, present


def exact_log_g(counts: np.ndarray) -> np.ndarray:
    out = np.full(counts.shape, -math.inf)
    nz = counts > 0
    out[nz] = np.log(counts[nz].astype(np.float64))
    return out
