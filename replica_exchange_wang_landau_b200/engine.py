"""Python face of the engine, shaped like the reference's C++ API.

The reference's seam is ``run_rewl(context, couplings, RunConfig) -> RewlResult``
(include/wl/parallel.hpp:23-36) over ``Geometry`` / ``Couplings`` (include/wl/physics.hpp)
and ``RunConfig`` / ``WlParameters`` (include/wl/io.hpp:12-58,
include/wl/wang_landau.hpp:40-56).  This module offers the same names with the same
defaults and error behaviour, and calls the sm_100a engine through the C-ABI in
include/wlg.h.  There is no CPU path: every call below runs on the GPU (the host-side
helpers -- grid, windows, checkpoint files -- excepted).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._abi import load_library

# ---- errors (the reference's exception types) --------------------------------------------


class WlgError(RuntimeError):
    """An error returned by the engine; `status` is the wlg_status name."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = _abi.STATUS_NAMES.get(status, str(status))


class InvalidArgument(WlgError, ValueError):
    """std::invalid_argument in the reference."""


class InitializationError(WlgError):
    """run_rewl's 'Walker initialization failed: ...' (std::runtime_error)."""


class EscapedError(WlgError):
    """'Walker escaped its energy window' (std::runtime_error)."""


class DeviceError(WlgError):
    """CUDA failure or no sm_100 device."""


class LogicError(WlgError):
    """std::logic_error in the reference."""


class OutOfRange(WlgError, IndexError):
    """std::out_of_range in the reference."""


class CheckpointIOError(WlgError, OSError):
    """A checkpoint file could not be read or written."""


_ERRORS = {1: InvalidArgument, 2: InitializationError, 3: EscapedError, 4: DeviceError, 5: DeviceError,
           6: WlgError, 7: LogicError, 8: OutOfRange, 9: CheckpointIOError}


def _check(status: int) -> None:
    if status:
        message = load_library().wlg_last_error().decode(errors="replace")
        raise _ERRORS.get(status, WlgError)(status, message)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _u64ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _i8ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int8))


def _u8ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


# ---- geometry ---------------------------------------------------------------------------


@dataclass
class Geometry:
    """wl::Geometry (include/wl/physics.hpp:23-35): positions, unit easy axes and a box."""

    positions: np.ndarray
    axes: np.ndarray
    box: tuple = (0.0, 0.0, 0.0)
    periodic: bool = True

    def __post_init__(self):
        self.positions = np.ascontiguousarray(self.positions, dtype=np.float64).reshape(-1, 3)
        self.axes = np.ascontiguousarray(self.axes, dtype=np.float64).reshape(-1, 3)
        self.box = tuple(float(x) for x in self.box)

    def size(self) -> int:
        return int(self.positions.shape[0])

    @staticmethod
    def simple_cubic(nx: int, ny: int, nz: int, spacing: float = 1.0, axis=(0.0, 0.0, 1.0),
                     periodic: bool = True) -> "Geometry":
        """Geometry::simple_cubic (src/physics.cpp:58-75)."""
        if nx == 0 or ny == 0 or nz == 0 or not spacing > 0.0:
            raise InvalidArgument(1, "Invalid simple-cubic dimensions or spacing")
        a = np.array(axis, dtype=np.float64)
        length = math.sqrt(float(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]))
        if not (length > 0.0) or not math.isfinite(length):
            raise InvalidArgument(1, "Ising axes must be finite non-zero vectors")
        a = np.array([a[0] / length, a[1] / length, a[2] / length])
        zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        pos = np.stack([xx.ravel() * spacing, yy.ravel() * spacing, zz.ravel() * spacing], axis=1).astype(np.float64)
        g = Geometry(pos, np.tile(a, (pos.shape[0], 1)), (nx * spacing, ny * spacing, nz * spacing), periodic)
        g.validate()
        return g

    @staticmethod
    def load_csv(path: str, box=(0.0, 0.0, 0.0), periodic: bool = True) -> "Geometry":
        """Geometry::load_csv (src/physics.cpp:99-149): header x,y,z,mx,my,mz, axes must be unit."""
        rows = []
        header = False
        with open(path, "r", encoding="utf-8-sig") as f:
            for number, line in enumerate(f, 1):
                clean = line.strip(" \t\r\n")
                if not clean or clean.startswith("#"):
                    continue
                cols = [c.strip(" \t\r\n") for c in clean.split(",")]
                if not header:
                    if [c.lower() for c in cols] != ["x", "y", "z", "mx", "my", "mz"]:
                        raise RuntimeError("CSV geometry header must be x,y,z,mx,my,mz")
                    header = True
                    continue
                if len(cols) != 6:
                    raise RuntimeError(f"CSV geometry line {number} must have 6 columns")
                try:
                    values = [float(c) for c in cols]
                except ValueError:
                    raise RuntimeError(f"Invalid number at CSV geometry line {number}") from None
                if not all(math.isfinite(v) for v in values):
                    raise RuntimeError(f"Invalid number at CSV geometry line {number}")
                rows.append(values)
        if not header:
            raise RuntimeError("CSV geometry file has no header")
        data = np.array(rows, dtype=np.float64).reshape(-1, 6)
        g = Geometry(data[:, :3], data[:, 3:], box, periodic)
        g.validate()
        return g

    def to_csv(self, path: str) -> None:
        """Writes the reference's CSV geometry format with round-trip-exact numbers."""
        with open(path, "w") as f:
            f.write("x,y,z,mx,my,mz\n")
            for p, a in zip(self.positions, self.axes):
                f.write(",".join(repr(float(x)) for x in (*p, *a)) + "\n")

    def validate(self) -> None:
        """Geometry::validate (src/physics.cpp:34-56)."""
        _check(load_library().wlg_validate_system(C.byref(System(self)._struct())))


@dataclass
class System:
    """A geometry plus coupling scale D and cutoff; cutoff > 0 selects the CSR backend
    (apps/wl_run.cpp:81-83)."""

    geometry: Geometry
    coupling_scale: float = 1.0
    cutoff: float = 0.0

    def size(self) -> int:
        return self.geometry.size()

    @property
    def backend(self) -> str:
        return "csr" if self.cutoff > 0.0 else "dense"

    def _struct(self) -> _abi.wlg_system:
        g = self.geometry
        s = _abi.wlg_system()
        s.n = g.size()
        s.positions = _dptr(g.positions)
        s.axes = _dptr(g.axes)
        s.box = (C.c_double * 3)(*g.box)
        s.periodic = 1 if g.periodic else 0
        s.coupling_scale = float(self.coupling_scale)
        s.cutoff = float(self.cutoff)
        s._keep = (g.positions, g.axes)
        return s

    # physics helpers on the device (src/physics.cpp:172-266)
    def couplings(self, precision: str = "fp64") -> np.ndarray:
        """The n x n matrix Couplings::at(i, j) reads (CSR: zeros off the pattern)."""
        n = self.size()
        out = np.zeros((n, n), dtype=np.float64)
        _check(load_library().wlg_couplings_dense(C.byref(self._struct()), _abi.PRECISION[precision], _dptr(out)))
        return out

    def csr(self):
        """CsrCouplings (row_offsets, columns, values)."""
        lib = load_library()
        s = self._struct()
        nnz = C.c_uint64(0)
        _check(lib.wlg_couplings_csr(C.byref(s), C.byref(nnz), None, None, None))
        ptr = np.zeros(self.size() + 1, dtype=np.uint64)
        cols = np.zeros(max(1, nnz.value), dtype=np.uint64)
        vals = np.zeros(max(1, nnz.value), dtype=np.float64)
        _check(lib.wlg_couplings_csr(C.byref(s), C.byref(nnz), _u64ptr(ptr), _u64ptr(cols), _dptr(vals)))
        return ptr, cols[: nnz.value], vals[: nnz.value]

    def local_fields(self, spins: np.ndarray):
        """local_fields + total_energy for one (n,) or many (k, n) configurations."""
        s = np.ascontiguousarray(spins, dtype=np.int8)
        single = s.ndim == 1
        s = s.reshape(-1, self.size())
        fields = np.zeros(s.shape, dtype=np.float64)
        energies = np.zeros(s.shape[0], dtype=np.float64)
        _check(load_library().wlg_local_fields(C.byref(self._struct()), _i8ptr(s), s.shape[0], _dptr(fields),
                                               _dptr(energies)))
        return (fields[0], energies[0]) if single else (fields, energies)


class Couplings:
    """Prebuilt couplings as wl::Couplings::at(i, j) exports them (include/wl/physics.hpp:41-49):
    a dense (n, n) matrix, or CSR rows (row_offsets, columns, values) sorted by column.  An
    Engine built from them runs exactly as one built from the geometry they came from."""

    def __init__(self, dense: Optional[np.ndarray] = None, row_offsets=None, columns=None, values=None):
        if (dense is None) == (row_offsets is None):
            raise InvalidArgument(1, "give either a dense matrix or CSR rows")
        if dense is not None:
            self.dense = np.ascontiguousarray(dense, dtype=np.float64)
            if self.dense.ndim != 2 or self.dense.shape[0] != self.dense.shape[1]:
                raise InvalidArgument(1, "dense couplings must be a square matrix")
            self.n = int(self.dense.shape[0])
        else:
            self.dense = None
            self.row_offsets = np.ascontiguousarray(row_offsets, dtype=np.uint64)
            self.columns = np.ascontiguousarray(columns, dtype=np.uint64)
            self.values = np.ascontiguousarray(values, dtype=np.float64)
            self.n = int(self.row_offsets.shape[0]) - 1
            if self.columns.shape != self.values.shape:
                raise InvalidArgument(1, "CSR columns and values differ in length")

    @staticmethod
    def of(system: "System") -> "Couplings":
        """The couplings the reference's backend for `system` stores (dense or CSR)."""
        if system.backend == "csr":
            ptr, cols, vals = system.csr()
            return Couplings(row_offsets=ptr, columns=cols, values=vals)
        return Couplings(dense=system.couplings("fp64"))

    @property
    def backend(self) -> str:
        return "dense" if self.dense is not None else "csr"

    def size(self) -> int:
        return self.n

    def _struct(self) -> _abi.wlg_couplings:
        c = _abi.wlg_couplings()
        c.n = self.n
        if self.dense is not None:
            c.dense = _dptr(self.dense)
            c._keep = (self.dense,)
        else:
            c.nnz = int(self.columns.shape[0])
            c.row_offsets = _u64ptr(self.row_offsets)
            c.columns = _u64ptr(self.columns)
            c.values = _dptr(self.values)
            c._keep = (self.row_offsets, self.columns, self.values)
        return c


# ---- configuration -------------------------------------------------------------------


@dataclass
class WlParameters:
    """wl::WlParameters (include/wl/wang_landau.hpp:40-56) with the same defaults."""

    flatness: float = 0.8
    minimum_visits: int = 100
    final_factor: float = 1e-8
    check_interval_attempts: int = 10_000
    force_accept_after_attempts: int = 0
    inverse_time_enabled: bool = True
    initialization_max_attempts: int = 1_000_000
    initialization_target_fraction: float = 0.5
    initialization_temperature_fraction: float = 0.05
    initialization_stall_attempts_per_spin: int = 1_000
    initialization_temperature_multiplier: float = 2.0
    initialization_max_temperature_fraction: float = 0.5
    collect_window_statistics: bool = False
    round_trip_margin_fraction: float = 0.1
    nalivaiko_mod: bool = False

    def _struct(self) -> _abi.wlg_wl_parameters:
        p = _abi.wlg_wl_parameters()
        for name, _ in _abi.wlg_wl_parameters._fields_:
            v = getattr(self, name)
            setattr(p, name, int(v) if isinstance(v, bool) else v)
        return p


def attempts_from_mcs(mcs: float, spin_count: int, allow_zero: bool, name: str = "mcs") -> int:
    """attempts_from_mcs (src/io.cpp:75-87), rounded in x87 long double like the reference."""
    if spin_count == 0:
        raise InvalidArgument(1, "Cannot resolve MCS for an empty system")
    if not math.isfinite(mcs) or mcs < 0.0 or (not allow_zero and mcs == 0.0):
        raise InvalidArgument(1, f"Invalid MCS value for {name}")
    if mcs == 0.0:
        return 0
    raw = np.longdouble(mcs) * np.longdouble(spin_count)
    if raw > np.longdouble(2.0**64) - np.longdouble(0.5):
        raise OverflowError(f"MCS value is too large for {name}")
    return max(1, int(np.floor(raw + np.longdouble(0.5))))


@dataclass
class RunConfig:
    """The part of wl::RunConfig (include/wl/io.hpp:12-58) that run_rewl reads, with the
    reference's defaults and its MCS-or-attempts interval switches."""

    emin: float = -20.0
    emax: float = 20.0
    bin_width: float = 0.1
    windows: int = 1
    walkers: int = 1  # walkers_per_rank
    overlap: float = 0.75
    explicit_windows: Optional[Sequence[tuple]] = None
    initial_spins_by_walker: Optional[Sequence[Optional[np.ndarray]]] = None
    seed: int = 1
    wl: WlParameters = field(default_factory=WlParameters)
    exchange_interval_attempts: int = 1000
    max_attempts: int = 10_000_000
    checkpoint_interval_attempts: int = 1_000_000
    exchange_interval_mcs: float = 10.0
    check_interval_mcs: float = 100.0
    force_accept_after_mcs: float = 0.0
    max_mcs: float = 1_000_000.0
    checkpoint_interval_mcs: float = 10_000.0
    exchange_interval_uses_mcs: bool = True
    check_interval_uses_mcs: bool = True
    force_accept_after_uses_mcs: bool = True
    max_limit_uses_mcs: bool = True
    checkpoint_interval_uses_mcs: bool = True
    resolved_spin_count: int = 0
    checkpoint_path: str = ""
    progress_interval_seconds: float = 0.0
    coupling_precision: str = "fp64"
    # FP32/BF16 couplings: FP64 recompute of fields and energies every this many MCS (0 = never).
    # No counterpart in the reference.
    recompute_interval_mcs: float = 1.0

    def resolve_mcs(self, spin_count: int) -> "RunConfig":
        """RunConfig::resolve_mcs (src/io.cpp:210-236)."""
        if spin_count == 0:
            raise InvalidArgument(1, "MCS requires at least one spin")
        if self.resolved_spin_count not in (0, spin_count):
            raise RuntimeError("MCS intervals were resolved for a different spin count")
        n = spin_count
        if self.exchange_interval_uses_mcs:
            self.exchange_interval_attempts = attempts_from_mcs(self.exchange_interval_mcs, n, False, "exchange_interval_mcs")
        else:
            self.exchange_interval_mcs = self.exchange_interval_attempts / n
        if self.check_interval_uses_mcs:
            self.wl.check_interval_attempts = attempts_from_mcs(self.check_interval_mcs, n, False, "check_interval_mcs")
        else:
            self.check_interval_mcs = self.wl.check_interval_attempts / n
        if self.force_accept_after_uses_mcs:
            self.wl.force_accept_after_attempts = attempts_from_mcs(self.force_accept_after_mcs, n, True, "force_accept_after_mcs")
        else:
            self.force_accept_after_mcs = self.wl.force_accept_after_attempts / n
        if self.max_limit_uses_mcs:
            self.max_attempts = attempts_from_mcs(self.max_mcs, n, True, "max_mcs")
        else:
            self.max_mcs = self.max_attempts / n
        if self.checkpoint_interval_uses_mcs:
            self.checkpoint_interval_attempts = attempts_from_mcs(self.checkpoint_interval_mcs, n, False, "checkpoint_interval_mcs")
        else:
            self.checkpoint_interval_mcs = self.checkpoint_interval_attempts / n
        self.resolved_spin_count = n
        return self

    def uses_legacy_attempt_units(self) -> bool:
        return not (self.exchange_interval_uses_mcs and self.check_interval_uses_mcs and
                    self.force_accept_after_uses_mcs and self.max_limit_uses_mcs and
                    self.checkpoint_interval_uses_mcs)

    def bins(self) -> int:
        return grid_bins(self.emin, self.emax, self.bin_width)

    def _struct(self, n: int):
        """Builds wlg_run_config; returns (struct, keep-alive objects)."""
        c = _abi.wlg_run_config()
        c.emin, c.emax, c.bin_width = float(self.emin), float(self.emax), float(self.bin_width)
        c.windows = int(self.windows)
        c.walkers_per_window = int(self.walkers)
        c.overlap = float(self.overlap)
        keep = []
        if self.explicit_windows is not None:
            w = np.array([v for pair in self.explicit_windows for v in pair], dtype=np.uint64)
            keep.append(w)
            c.explicit_windows = _u64ptr(w)
        c.seed = int(self.seed) & 0xFFFFFFFFFFFFFFFF
        c.wl = self.wl._struct()
        c.exchange_interval_attempts = int(self.exchange_interval_attempts)
        c.max_attempts = int(self.max_attempts)
        c.checkpoint_interval_attempts = int(self.checkpoint_interval_attempts)
        if self.checkpoint_path:
            b = str(self.checkpoint_path).encode()
            keep.append(b)
            c.checkpoint_path = b
        if self.initial_spins_by_walker:
            total = int(self.windows) * int(self.walkers)
            if len(self.initial_spins_by_walker) != total:
                raise InvalidArgument(1, "Adaptive initial-configuration count mismatch")
            spins = np.zeros((total, n), dtype=np.int8)
            present = np.zeros(total, dtype=np.uint8)
            for k, s in enumerate(self.initial_spins_by_walker):
                if s is None or len(s) == 0:
                    continue
                if len(s) != n:
                    raise InvalidArgument(1, "Adaptive initial spin count mismatch")
                spins[k] = np.asarray(s, dtype=np.int8)
                present[k] = 1
            keep += [spins, present]
            c.initial_spins = _i8ptr(spins)
            c.initial_spins_present = _u8ptr(present)
        c.progress_interval_seconds = float(self.progress_interval_seconds)
        c.coupling_precision = _abi.PRECISION[self.coupling_precision]
        c.recompute_interval_attempts = attempts_from_mcs(self.recompute_interval_mcs, n, True,
                                                          "recompute_interval_mcs")
        return c, keep


# ---- results ----------------------------------------------------------------------------


@dataclass
class DosFragment:
    """wl::DosFragment (include/wl/analysis.hpp:13-19), arrays over the whole grid."""

    window: tuple
    log_g: np.ndarray
    histogram: np.ndarray
    standard_error: np.ndarray
    valid: np.ndarray


@dataclass
class WindowSamplingStatistics:
    window: tuple
    squared_energy_displacement: np.ndarray
    displacement_samples: np.ndarray
    round_trips: int
    walkers: int


@dataclass
class RewlResult:
    """wl::RewlResult (include/wl/parallel.hpp:23-31)."""

    fragments: list
    walker_statistics: list
    sampling_statistics: list
    representatives: list
    attempted: int = 0
    accepted: int = 0
    forced_accepted: int = 0
    exchange_attempted: int = 0
    exchange_accepted: int = 0
    converged: bool = False
    epochs: int = 0
    precision_report: Optional[dict] = None  # mixed-precision drift (no reference counterpart)


@dataclass
class Snapshot:
    """wl::WalkerSnapshot (include/wl/wang_landau.hpp:74-89)."""

    walker_id: int
    spins: np.ndarray
    fields: np.ndarray
    energy: float
    log_g: np.ndarray
    histogram: np.ndarray
    active: np.ndarray
    factor: float
    attempted: int
    accepted: int
    forced_accepted: int
    last_accepted_attempt: int
    stage: int
    rng_state: tuple

    def _struct(self):
        s = _abi.wlg_snapshot()
        keep = [np.ascontiguousarray(self.spins, dtype=np.int8), np.ascontiguousarray(self.fields, dtype=np.float64),
                np.ascontiguousarray(self.log_g, dtype=np.float64),
                np.ascontiguousarray(self.histogram, dtype=np.uint64), np.ascontiguousarray(self.active, dtype=np.uint8)]
        s.walker_id = int(self.walker_id)
        s.spins, s.fields = _i8ptr(keep[0]), _dptr(keep[1])
        s.energy = float(self.energy)
        s.log_g, s.histogram, s.active = _dptr(keep[2]), _u64ptr(keep[3]), _u8ptr(keep[4])
        s.factor = float(self.factor)
        s.attempted, s.accepted = int(self.attempted), int(self.accepted)
        s.forced_accepted, s.last_accepted_attempt = int(self.forced_accepted), int(self.last_accepted_attempt)
        s.stage = int(self.stage)
        s.rng_state = (C.c_uint64 * 4)(*[int(x) for x in self.rng_state])
        return s, keep

    @staticmethod
    def _empty(n: int, bins: int):
        arrays = [np.zeros(n, np.int8), np.zeros(n, np.float64), np.zeros(bins, np.float64), np.zeros(bins, np.uint64),
                  np.zeros(bins, np.uint8)]
        s = _abi.wlg_snapshot()
        s.spins, s.fields = _i8ptr(arrays[0]), _dptr(arrays[1])
        s.log_g, s.histogram, s.active = _dptr(arrays[2]), _u64ptr(arrays[3]), _u8ptr(arrays[4])
        return s, arrays

    @staticmethod
    def _from(s, arrays) -> "Snapshot":
        return Snapshot(int(s.walker_id), arrays[0], arrays[1], float(s.energy), arrays[2], arrays[3], arrays[4],
                        float(s.factor), int(s.attempted), int(s.accepted), int(s.forced_accepted),
                        int(s.last_accepted_attempt), int(s.stage), tuple(int(x) for x in s.rng_state))


def _stat_dict(s: _abi.wlg_walker_statistics) -> dict:
    return {name: getattr(s, name) for name, _ in _abi.wlg_walker_statistics._fields_}


# ---- the engine ---------------------------------------------------------------------------


class Engine:
    """One REWL run resident on the current CUDA device (run_rewl's state, src/parallel.cpp:276-534)."""

    def __init__(self, system: "System | Couplings", config: RunConfig, walkers_per_block: int | None = None):
        """`system` is a System (geometry: J is built on the device) or prebuilt Couplings."""
        self._lib = load_library()
        self.system = system
        self.config = config
        n = system.size()
        self._sys = system._struct()
        self._cfg, self._keep = config._struct(n)
        handle = C.c_void_p()
        create = self._lib.wlg_engine_create_from_couplings if isinstance(system, Couplings) else \
            self._lib.wlg_engine_create
        _check(create(C.byref(self._sys), C.byref(self._cfg), C.byref(handle)))
        self._h = handle
        self.n = n
        self.bins = int(self._lib.wlg_engine_bins(self._h))
        if walkers_per_block:
            self.set_launch(walkers_per_block, 0)
        self.walkers = int(self._lib.wlg_engine_walkers(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.wlg_engine_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # run control
    def run(self) -> dict:
        t = _abi.wlg_run_totals()
        _check(self._lib.wlg_engine_run(self._h, C.byref(t)))
        return {name: getattr(t, name) for name, _ in _abi.wlg_run_totals._fields_}

    def run_epochs(self, epochs: int):
        ran, done = C.c_uint64(0), C.c_int32(0)
        _check(self._lib.wlg_engine_run_epochs(self._h, int(epochs), C.byref(ran), C.byref(done)))
        return int(ran.value), bool(done.value)

    def time_epochs(self, epochs: int) -> dict:
        """Runs `epochs` epochs with CUDA events around every kernel (device time, ms)."""
        t = _abi.wlg_epoch_timing()
        _check(self._lib.wlg_engine_time_epochs(self._h, int(epochs), C.byref(t)))
        return {name: getattr(t, name) for name, _ in _abi.wlg_epoch_timing._fields_}

    def time_run(self, epochs: int) -> dict:
        """Runs `epochs` epochs through the product path (graph replays) with CUDA events
        around the whole run (device time, ms)."""
        t = _abi.wlg_epoch_timing()
        _check(self._lib.wlg_engine_time_run(self._h, int(epochs), C.byref(t)))
        return {name: getattr(t, name) for name, _ in _abi.wlg_epoch_timing._fields_}

    def save_run(self, path: str) -> None:
        """Checkpoint of every walker and the run counters (no reference counterpart)."""
        _check(self._lib.wlg_engine_save_run(self._h, str(path).encode()))

    def load_run(self, path: str) -> None:
        """Restores a save_run checkpoint into this compatible engine."""
        _check(self._lib.wlg_engine_load_run(self._h, str(path).encode()))

    def autotune(self, trial_epochs: int = 16) -> dict:
        """Times candidate launch shapes on real epochs and keeps the fastest (results are
        unchanged by the launch shape)."""
        r = _abi.wlg_autotune_report()
        _check(self._lib.wlg_engine_autotune(self._h, int(trial_epochs), C.byref(r)))
        return {name: getattr(r, name) for name, _ in _abi.wlg_autotune_report._fields_}

    def precision_report(self) -> dict:
        """Drift of a mixed-precision run over its periodic FP64 recomputes (zeros for FP64)."""
        r = _abi.wlg_precision_report()
        _check(self._lib.wlg_engine_precision_report(self._h, C.byref(r)))
        out = {name: getattr(r, name) for name, _ in _abi.wlg_precision_report._fields_ if name != "pad"}
        out["coupling_precision"] = {v: k for k, v in _abi.PRECISION.items()}[r.coupling_precision]
        return out

    def warm_start(self, log_g: np.ndarray, factor: float, continue_schedule: bool = False) -> None:
        """Seeds every walker's window slice of log g (whole-grid array) and its ln f before
        the first attempt (no counterpart in the reference).  continue_schedule: the 1/t
        stage continues from ln f = factor (f = active / (attempted + window bins / factor))
        instead of restarting at active / attempted."""
        lg = np.ascontiguousarray(log_g, dtype=np.float64)
        if lg.shape != (self.bins,):
            raise InvalidArgument(1, "The log g estimate must have one entry per grid bin")
        fn = self._lib.wlg_engine_warm_start_continue if continue_schedule else self._lib.wlg_engine_warm_start
        _check(fn(self._h, _dptr(lg), float(factor)))

    def set_staging_ring(self, entries: int) -> None:
        """The split sweep's staging ring: 16 or 32 draws with their J rows (0 = 16)."""
        _check(self._lib.wlg_engine_set_staging_ring(self._h, int(entries)))

    def inject_wait_timeout(self) -> None:
        """Failure injection for tests: the draw producers of the split and single-window sweeps
        publish nothing from the next epoch on, so the walkers' bounded waits run out and the
        next run call raises a DeviceError with status WLG_ERR_TIMEOUT."""
        _check(self._lib.wlg_engine_inject_wait_timeout(self._h))

    def set_launch(self, walkers_per_block: int = 0, epochs_per_graph: int = 0) -> None:
        _check(self._lib.wlg_engine_set_launch(self._h, int(walkers_per_block), int(epochs_per_graph)))

    @property
    def window_sweep(self) -> bool:
        """Whether epochs run in the single-window kernel (one window, small dense FP64 system;
        many epochs per launch).  Setting False selects the per-epoch kernels (same results)."""
        return bool(self._lib.wlg_engine_window_sweep(self._h))

    @window_sweep.setter
    def window_sweep(self, enabled: bool) -> None:
        _check(self._lib.wlg_engine_set_window_sweep(self._h, int(bool(enabled))))

    def totals(self) -> dict:
        t = _abi.wlg_run_totals()
        _check(self._lib.wlg_engine_totals(self._h, C.byref(t)))
        return {name: getattr(t, name) for name, _ in _abi.wlg_run_totals._fields_}

    def window(self, w: int) -> tuple:
        b, e = C.c_uint64(0), C.c_uint64(0)
        _check(self._lib.wlg_engine_window(self._h, w, C.byref(b), C.byref(e)))
        return int(b.value), int(e.value)

    def fragment(self, w: int, allow_empty: bool = False) -> DosFragment:
        B = self.bins
        lg, h, se, v = np.zeros(B), np.zeros(B, np.uint64), np.zeros(B), np.zeros(B, np.uint8)
        _check(self._lib.wlg_engine_fragment(self._h, w, int(allow_empty), _dptr(lg), _u64ptr(h), _dptr(se), _u8ptr(v)))
        return DosFragment(self.window(w), lg, h, se, v)

    def fragments(self, allow_empty: bool = False) -> list:
        """Every window's DosFragment from one launch (wlg_engine_fragments)."""
        W, B = int(self.config.windows), self.bins
        lg, h, se, v = np.zeros(W * B), np.zeros(W * B, np.uint64), np.zeros(W * B), np.zeros(W * B, np.uint8)
        _check(self._lib.wlg_engine_fragments(self._h, int(allow_empty), _dptr(lg), _u64ptr(h), _dptr(se), _u8ptr(v)))
        return [DosFragment(self.window(w), lg[w * B:(w + 1) * B].copy(), h[w * B:(w + 1) * B].copy(),
                            se[w * B:(w + 1) * B].copy(), v[w * B:(w + 1) * B].copy()) for w in range(W)]

    def stitch(self, complete_range: bool = False) -> "DensityOfStates":
        """stitch_dos (src/analysis.cpp:45-130) of every window's fragment, on the device."""
        c = self.config
        lg, se = np.empty(self.bins), np.empty(self.bins)
        h, ok = np.empty(self.bins, np.uint64), np.empty(self.bins, np.uint8)
        count = int(c.windows)
        joins = (_abi.wlg_join_quality * max(1, count - 1))()
        full = C.c_int32(0)
        _check(self._lib.wlg_engine_stitch(self._h, int(complete_range), _dptr(lg), _u64ptr(h), _dptr(se), _u8ptr(ok),
                                           joins, C.byref(full)))
        q = [{name: getattr(joins[k], name) for name, _ in _abi.wlg_join_quality._fields_} for k in range(count - 1)]
        return DensityOfStates(c.emin, c.emax, c.bin_width, lg, h, se, ok, [j["join_bin"] for j in q], q,
                               bool(full.value))

    def sampling_statistics(self, w: int) -> WindowSamplingStatistics:
        B = self.bins
        sq, ds = np.zeros(B), np.zeros(B, np.uint64)
        trips, walkers = C.c_uint64(0), C.c_uint64(0)
        _check(self._lib.wlg_engine_sampling_statistics(self._h, w, _dptr(sq), _u64ptr(ds), C.byref(trips),
                                                        C.byref(walkers)))
        return WindowSamplingStatistics(self.window(w), sq, ds, int(trips.value), int(walkers.value))

    def walker_statistics(self) -> list:
        out = (_abi.wlg_walker_statistics * self.walkers)()
        _check(self._lib.wlg_engine_walker_statistics(self._h, out, self.walkers))
        return [_stat_dict(s) for s in out]

    def representatives(self) -> list:
        count = C.c_uint64(0)
        _check(self._lib.wlg_engine_representatives(self._h, None, None, 0, C.byref(count)))
        k = int(count.value)
        e = np.zeros(max(1, k))
        s = np.zeros((max(1, k), self.n), np.int8)
        _check(self._lib.wlg_engine_representatives(self._h, _dptr(e), _i8ptr(s), k, C.byref(count)))
        return [(float(e[i]), s[i].copy()) for i in range(k)]

    def result(self) -> RewlResult:
        """RewlResult as run_rewl assembles it after the loop (src/parallel.cpp:536-580)."""
        t = self.totals()
        collect = self.config.wl.collect_window_statistics
        fragments = self.fragments(allow_empty=collect)
        sampling = [self.sampling_statistics(w) for w in range(int(self.config.windows))] if collect else []
        reps = self.representatives() if collect else []
        return RewlResult(fragments, self.walker_statistics(), sampling, reps, t["attempted"], t["accepted"],
                          t["forced_accepted"], t["exchange_attempted"], t["exchange_accepted"], bool(t["converged"]),
                          t["epochs"], self.precision_report())

    # single-walker operations (include/wl/wang_landau.hpp:98-138)
    def run_attempts(self, walker: int, count: int) -> None:
        _check(self._lib.wlg_walker_run_attempts(self._h, walker, int(count)))

    def snapshot(self, walker: int) -> Snapshot:
        s, arrays = Snapshot._empty(self.n, self.bins)
        _check(self._lib.wlg_walker_snapshot(self._h, walker, C.byref(s)))
        return Snapshot._from(s, arrays)

    def restore(self, walker: int, snapshot: Snapshot) -> None:
        if len(snapshot.spins) != self.n or len(snapshot.fields) != self.n or len(snapshot.log_g) != self.bins or \
                len(snapshot.histogram) != self.bins or len(snapshot.active) != self.bins:
            raise InvalidArgument(1, "Checkpoint is incompatible with walker")
        s, keep = snapshot._struct()
        _check(self._lib.wlg_walker_restore(self._h, walker, C.byref(s)))

    def histogram_statistics(self, walker: int) -> dict:
        s = _abi.wlg_histogram_statistics()
        _check(self._lib.wlg_walker_histogram_statistics(self._h, walker, C.byref(s)))
        return {name: getattr(s, name) for name, _ in _abi.wlg_histogram_statistics._fields_}

    def flags(self, walker: int) -> tuple:
        f, c, r = C.c_int32(0), C.c_int32(0), C.c_int32(0)
        _check(self._lib.wlg_walker_flags(self._h, walker, C.byref(f), C.byref(c), C.byref(r)))
        return bool(f.value), bool(c.value), bool(r.value)

    def flat(self, walker: int) -> bool:
        return self.flags(walker)[0]

    def covered(self, walker: int) -> bool:
        return self.flags(walker)[1]

    def ready_for_iteration(self, walker: int) -> bool:
        return self.flags(walker)[2]

    def begin_next_iteration(self, walker: int) -> None:
        _check(self._lib.wlg_walker_begin_next_iteration(self._h, walker))

    def exchange_log_probability(self, left: int, right: int) -> float:
        lp = C.c_double(0.0)
        _check(self._lib.wlg_walker_exchange_log_probability(self._h, left, right, C.byref(lp)))
        return float(lp.value)

    def swap_configuration(self, left: int, right: int) -> None:
        _check(self._lib.wlg_walker_swap(self._h, left, right))


class Batch:
    """Engines on one device advanced together by single CUDA-graph launches (no counterpart
    in the reference).  The engines must stay open while the batch is used."""

    def __init__(self, engines: Sequence["Engine"]):
        self.engines = list(engines)
        self._lib = load_library()
        arr = (C.c_void_p * len(self.engines))(*[e._h.value if isinstance(e._h, C.c_void_p) else e._h
                                                 for e in self.engines])
        h = C.c_void_p()
        _check(self._lib.wlg_batch_create(arr, len(self.engines), C.byref(h)))
        self._h = h

    def run_epochs(self, max_epochs: int) -> bool:
        """Runs until every engine has terminated or about max_epochs epochs; True if all did."""
        launches, done = C.c_uint64(0), C.c_int32(0)
        _check(self._lib.wlg_batch_run_epochs(self._h, int(max_epochs), C.byref(launches), C.byref(done)))
        return bool(done.value)

    def run(self) -> None:
        while not self.run_epochs(1 << 62):
            pass

    def close(self) -> None:
        if self._h:
            self._lib.wlg_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_rewl(system: System, config: RunConfig, walkers_per_block: int | None = None) -> RewlResult:
    """run_rewl (src/parallel.cpp:276-747) on one GPU."""
    with Engine(system, config, walkers_per_block) as e:
        e.run()
        return e.result()


# ---- host helpers ---------------------------------------------------------------------


def set_device(device: int) -> None:
    """Selects the CUDA device for engines created afterwards on this thread."""
    _check(load_library().wlg_set_device(int(device)))


def grid_bins(emin: float, emax: float, width: float) -> int:
    b = C.c_uint64(0)
    _check(load_library().wlg_grid_bins(emin, emax, width, C.byref(b)))
    return int(b.value)


def grid_index(emin: float, emax: float, width: float, energy: float) -> Optional[int]:
    b = C.c_int64(0)
    _check(load_library().wlg_grid_index(emin, emax, width, energy, C.byref(b)))
    return None if b.value < 0 else int(b.value)


def partition_windows(bins: int, count: int, overlap: float) -> list:
    out = np.zeros(2 * count, dtype=np.uint64)
    _check(load_library().wlg_partition_windows(bins, count, overlap, _u64ptr(out)))
    return [(int(out[2 * i]), int(out[2 * i + 1])) for i in range(count)]


def save_checkpoint(path: str, snapshot: Snapshot) -> None:
    s, keep = snapshot._struct()
    _check(load_library().wlg_checkpoint_save(str(path).encode(), C.byref(s), len(snapshot.spins),
                                              len(snapshot.log_g)))


def load_checkpoint(path: str) -> Snapshot:
    lib = load_library()
    s = _abi.wlg_snapshot()
    n, b = C.c_uint64(0), C.c_uint64(0)
    _check(lib.wlg_checkpoint_load(str(path).encode(), C.byref(s), C.byref(n), C.byref(b)))
    s, arrays = Snapshot._empty(int(n.value), int(b.value))
    _check(lib.wlg_checkpoint_load(str(path).encode(), C.byref(s), C.byref(n), C.byref(b)))
    return Snapshot._from(s, arrays)


# ---- stitching and output (wl::stitch_dos, src/analysis.cpp:45-130; src/io.cpp:398-421) ---


@dataclass
class DensityOfStates:
    """wl::DensityOfStates (include/wl/analysis.hpp:40-48) plus the per-join overlap quality."""

    emin: float
    emax: float
    width: float
    log_g: np.ndarray
    histogram: np.ndarray
    standard_error: np.ndarray
    valid: np.ndarray
    join_bins: list
    joins: list
    fully_normalized: bool


def _fragment_view(frag: DosFragment):
    arrays = (np.ascontiguousarray(frag.log_g, dtype=np.float64), np.ascontiguousarray(frag.histogram, dtype=np.uint64),
              np.ascontiguousarray(frag.standard_error, dtype=np.float64),
              np.ascontiguousarray(frag.valid, dtype=np.uint8))
    v = _abi.wlg_fragment_view(int(frag.window[0]), int(frag.window[1]), _dptr(arrays[0]), _u64ptr(arrays[1]),
                               _dptr(arrays[2]), _u8ptr(arrays[3]))
    return v, arrays


def stitch_dos(fragments: Sequence[DosFragment], emin: float, emax: float, width: float,
               complete_range: bool = False, spin_count: int = 0) -> DensityOfStates:
    """stitch_dos (src/analysis.cpp:45-130), bit-identical, with the overlap quality of each join."""
    bins = grid_bins(emin, emax, width)
    views, keep = [], []
    for f in fragments:
        v, arrays = _fragment_view(f)
        views.append(v)
        keep.append(arrays)
    lg, se = np.empty(bins), np.empty(bins)
    h, ok = np.empty(bins, np.uint64), np.empty(bins, np.uint8)
    joins = (_abi.wlg_join_quality * max(1, len(views) - 1))()
    full = C.c_int32(0)
    arr = (_abi.wlg_fragment_view * max(1, len(views)))(*views)
    _check(load_library().wlg_stitch_dos(emin, emax, width, arr, len(views), int(complete_range), int(spin_count),
                                         _dptr(lg), _u64ptr(h), _dptr(se), _u8ptr(ok), joins, C.byref(full)))
    q = [{name: getattr(joins[k], name) for name, _ in _abi.wlg_join_quality._fields_} for k in range(len(views) - 1)]
    return DensityOfStates(emin, emax, width, lg, h, se, ok, [j["join_bin"] for j in q], q, bool(full.value))


def write_dos_csv(path: str, dos: DensityOfStates) -> None:
    """<prefix>_dos.csv in the reference's format (src/io.cpp:398-408), byte for byte."""
    _check(load_library().wlg_write_dos_csv(str(path).encode(), dos.emin, dos.width, len(dos.log_g),
                                            _dptr(np.ascontiguousarray(dos.log_g, np.float64)),
                                            _u64ptr(np.ascontiguousarray(dos.histogram, np.uint64)),
                                            _dptr(np.ascontiguousarray(dos.standard_error, np.float64)),
                                            _u8ptr(np.ascontiguousarray(dos.valid, np.uint8))))


def write_workers_stat_csv(path: str, statistics: Sequence[dict], spin_count: int) -> None:
    """<prefix>_workers_stat.csv in the reference's format (src/io.cpp:430-451), byte for byte, from
    walker statistics as RewlResult.walker_statistics and Engine.walker_statistics() hold them;
    spin_count 0 raises InvalidArgument, as the reference's invalid_argument."""
    rows = (_abi.wlg_walker_statistics * max(1, len(statistics)))()
    for k, s in enumerate(statistics):
        for name, _ in _abi.wlg_walker_statistics._fields_:
            setattr(rows[k], name, s[name])
    _check(load_library().wlg_write_workers_stat_csv(str(path).encode(), rows, len(statistics), int(spin_count)))


def write_fragment_csv(path: str, fragment: DosFragment, emin: float, width: float, window_id: int) -> None:
    """<prefix>_window_<w>.csv in the reference's format (src/io.cpp:410-421), byte for byte."""
    v, arrays = _fragment_view(fragment)
    _check(load_library().wlg_write_fragment_csv(str(path).encode(), emin, width, int(window_id), v.window_begin,
                                                 v.window_end, v.log_g, v.histogram, v.standard_error, v.valid))
