"""ctypes mirror of include/wlg.h (the engine's C-ABI) and the loader of libwlg.so.

The struct layouts below follow the header field for field; tests/test_abi.py compiles a
small C program against the header and checks every size and offset.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
LIBRARY_PATH = PACKAGE / "libwlg.so"

WLG_ABI_VERSION = 1

STATUS_NAMES = {
    0: "WLG_OK",
    1: "WLG_ERR_INVALID_ARGUMENT",
    2: "WLG_ERR_INIT_FAILED",
    3: "WLG_ERR_ESCAPED",
    4: "WLG_ERR_DEVICE",
    5: "WLG_ERR_TIMEOUT",
    6: "WLG_ERR_RUNTIME",
    7: "WLG_ERR_LOGIC",
    8: "WLG_ERR_OUT_OF_RANGE",
    9: "WLG_ERR_IO",
}

PRECISION = {"fp64": 0, "fp32": 1, "bf16": 2}


class wlg_system(C.Structure):
    _fields_ = [
        ("n", C.c_uint64),
        ("positions", C.POINTER(C.c_double)),
        ("axes", C.POINTER(C.c_double)),
        ("box", C.c_double * 3),
        ("periodic", C.c_int32),
        ("coupling_scale", C.c_double),
        ("cutoff", C.c_double),
    ]


class wlg_couplings(C.Structure):
    _fields_ = [
        ("n", C.c_uint64),
        ("dense", C.POINTER(C.c_double)),
        ("nnz", C.c_uint64),
        ("row_offsets", C.POINTER(C.c_uint64)),
        ("columns", C.POINTER(C.c_uint64)),
        ("values", C.POINTER(C.c_double)),
    ]


class wlg_wl_parameters(C.Structure):
    _fields_ = [
        ("flatness", C.c_double),
        ("minimum_visits", C.c_uint64),
        ("final_factor", C.c_double),
        ("check_interval_attempts", C.c_uint64),
        ("force_accept_after_attempts", C.c_uint64),
        ("inverse_time_enabled", C.c_int32),
        ("initialization_max_attempts", C.c_uint64),
        ("initialization_target_fraction", C.c_double),
        ("initialization_temperature_fraction", C.c_double),
        ("initialization_stall_attempts_per_spin", C.c_uint64),
        ("initialization_temperature_multiplier", C.c_double),
        ("initialization_max_temperature_fraction", C.c_double),
        ("collect_window_statistics", C.c_int32),
        ("round_trip_margin_fraction", C.c_double),
        ("nalivaiko_mod", C.c_int32),
    ]


class wlg_run_config(C.Structure):
    _fields_ = [
        ("emin", C.c_double),
        ("emax", C.c_double),
        ("bin_width", C.c_double),
        ("windows", C.c_uint64),
        ("walkers_per_window", C.c_uint64),
        ("overlap", C.c_double),
        ("explicit_windows", C.POINTER(C.c_uint64)),
        ("seed", C.c_uint64),
        ("wl", wlg_wl_parameters),
        ("exchange_interval_attempts", C.c_uint64),
        ("max_attempts", C.c_uint64),
        ("checkpoint_interval_attempts", C.c_uint64),
        ("checkpoint_path", C.c_char_p),
        ("initial_spins", C.POINTER(C.c_int8)),
        ("initial_spins_present", C.POINTER(C.c_uint8)),
        ("progress_interval_seconds", C.c_double),
        ("coupling_precision", C.c_int32),
        ("recompute_interval_attempts", C.c_uint64),
    ]


class wlg_histogram_statistics(C.Structure):
    _fields_ = [
        ("active_bins", C.c_uint64),
        ("covered_bins", C.c_uint64),
        ("minimum", C.c_uint64),
        ("mean", C.c_double),
        ("min_over_mean", C.c_double),
        ("coverage", C.c_double),
    ]


class wlg_walker_statistics(C.Structure):
    _fields_ = [
        ("walker_id", C.c_uint64),
        ("window_id", C.c_uint64),
        ("mpi_rank", C.c_int32),
        ("attempted", C.c_uint64),
        ("accepted", C.c_uint64),
        ("forced_accepted", C.c_uint64),
        ("attempts_since_last_accepted", C.c_uint64),
        ("energy", C.c_double),
        ("factor", C.c_double),
        ("active_bins", C.c_uint64),
        ("minimum_histogram", C.c_uint64),
        ("mean_histogram", C.c_double),
        ("min_over_mean", C.c_double),
        ("round_trips", C.c_uint64),
    ]


class wlg_run_totals(C.Structure):
    _fields_ = [
        ("attempted", C.c_uint64),
        ("accepted", C.c_uint64),
        ("forced_accepted", C.c_uint64),
        ("exchange_attempted", C.c_uint64),
        ("exchange_accepted", C.c_uint64),
        ("converged", C.c_int32),
        ("epochs", C.c_uint64),
    ]


class wlg_epoch_timing(C.Structure):
    _fields_ = [
        ("epochs", C.c_uint64),
        ("walk_ms", C.c_double),
        ("exchange_ms", C.c_double),
        ("total_ms", C.c_double),
        ("attempted", C.c_uint64),
        ("accepted", C.c_uint64),
    ]


class wlg_precision_report(C.Structure):
    _fields_ = [
        ("coupling_precision", C.c_int32),
        ("pad", C.c_int32),
        ("recompute_interval_attempts", C.c_uint64),
        ("recomputes", C.c_uint64),
        ("resynced", C.c_uint64),
        ("deferred", C.c_uint64),
        ("bin_changes", C.c_uint64),
        ("max_field_drift", C.c_double),
        ("max_energy_drift", C.c_double),
    ]


class wlg_autotune_report(C.Structure):
    _fields_ = [
        ("walkers_per_block", C.c_int32),
        ("epochs_per_graph", C.c_int32),
        ("ms_per_epoch", C.c_double),
        ("trials", C.c_uint64),
        ("staging_ring", C.c_int32),
        ("pad", C.c_int32),
    ]


class wlg_fragment_view(C.Structure):
    _fields_ = [
        ("window_begin", C.c_uint64),
        ("window_end", C.c_uint64),
        ("log_g", C.POINTER(C.c_double)),
        ("histogram", C.POINTER(C.c_uint64)),
        ("standard_error", C.POINTER(C.c_double)),
        ("valid", C.POINTER(C.c_uint8)),
    ]


class wlg_join_quality(C.Structure):
    _fields_ = [
        ("join_bin", C.c_uint64),
        ("common_bins", C.c_uint64),
        ("rmse", C.c_double),
        ("max_abs_difference", C.c_double),
        ("slope_difference", C.c_double),
    ]


class wlg_adaptive_parameters(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint64),
        ("pilot_mcs", C.c_double),
        ("smoothing_width", C.c_double),
        ("minimum_width", C.c_double),
        ("diffusivity_floor_fraction", C.c_double),
        ("curvature_weight", C.c_double),
        ("round_trip_target", C.c_double),
        ("maximum_round_trip_penalty", C.c_double),
    ]


class wlg_sampling_view(C.Structure):
    _fields_ = [
        ("window_begin", C.c_uint64),
        ("window_end", C.c_uint64),
        ("squared_energy_displacement", C.POINTER(C.c_double)),
        ("displacement_samples", C.POINTER(C.c_uint64)),
        ("round_trips", C.c_uint64),
        ("walkers", C.c_uint64),
    ]


class wlg_snapshot(C.Structure):
    _fields_ = [
        ("walker_id", C.c_uint64),
        ("spins", C.POINTER(C.c_int8)),
        ("fields", C.POINTER(C.c_double)),
        ("energy", C.c_double),
        ("log_g", C.POINTER(C.c_double)),
        ("histogram", C.POINTER(C.c_uint64)),
        ("active", C.POINTER(C.c_uint8)),
        ("factor", C.c_double),
        ("attempted", C.c_uint64),
        ("accepted", C.c_uint64),
        ("forced_accepted", C.c_uint64),
        ("last_accepted_attempt", C.c_uint64),
        ("stage", C.c_uint8),
        ("rng_state", C.c_uint64 * 4),
    ]


STRUCTS = {
    "wlg_system": wlg_system,
    "wlg_couplings": wlg_couplings,
    "wlg_wl_parameters": wlg_wl_parameters,
    "wlg_run_config": wlg_run_config,
    "wlg_histogram_statistics": wlg_histogram_statistics,
    "wlg_walker_statistics": wlg_walker_statistics,
    "wlg_run_totals": wlg_run_totals,
    "wlg_snapshot": wlg_snapshot,
    "wlg_epoch_timing": wlg_epoch_timing,
    "wlg_precision_report": wlg_precision_report,
    "wlg_autotune_report": wlg_autotune_report,
    "wlg_fragment_view": wlg_fragment_view,
    "wlg_join_quality": wlg_join_quality,
    "wlg_adaptive_parameters": wlg_adaptive_parameters,
    "wlg_sampling_view": wlg_sampling_view,
}

P = C.POINTER
_u64, _i64, _i32, _dbl = C.c_uint64, C.c_int64, C.c_int32, C.c_double
_vp = C.c_void_p

# name -> (restype, argtypes); the full list of entry points declared in include/wlg.h
SIGNATURES = {
    "wlg_abi_version": (_i32, []),
    "wlg_last_error": (C.c_char_p, []),
    "wlg_set_device": (_i32, [_i32]),
    "wlg_default_run_config": (_i32, [_u64, P(wlg_run_config)]),
    "wlg_grid_bins": (_i32, [_dbl, _dbl, _dbl, P(_u64)]),
    "wlg_grid_index": (_i32, [_dbl, _dbl, _dbl, _dbl, P(_i64)]),
    "wlg_partition_windows": (_i32, [_u64, _u64, _dbl, P(_u64)]),
    "wlg_validate_system": (_i32, [P(wlg_system)]),
    "wlg_checkpoint_save": (_i32, [C.c_char_p, P(wlg_snapshot), _u64, _u64]),
    "wlg_checkpoint_load": (_i32, [C.c_char_p, P(wlg_snapshot), P(_u64), P(_u64)]),
    "wlg_couplings_dense": (_i32, [P(wlg_system), _i32, P(_dbl)]),
    "wlg_couplings_csr": (_i32, [P(wlg_system), P(_u64), P(_u64), P(_u64), P(_dbl)]),
    "wlg_local_fields": (_i32, [P(wlg_system), P(C.c_int8), _u64, P(_dbl), P(_dbl)]),
    "wlg_local_fields_noalloc": (_i32, [P(wlg_system), P(C.c_int8), _u64, P(_dbl), P(_dbl)]),
    "wlg_engine_create": (_i32, [P(wlg_system), P(wlg_run_config), P(_vp)]),
    "wlg_engine_create_from_couplings": (_i32, [P(wlg_couplings), P(wlg_run_config), P(_vp)]),
    "wlg_engine_destroy": (None, [_vp]),
    "wlg_engine_inject_wait_timeout": (_i32, [_vp]),
    "wlg_engine_set_staging_ring": (_i32, [_vp, _i32]),
    "wlg_engine_run": (_i32, [_vp, P(wlg_run_totals)]),
    "wlg_engine_run_epochs": (_i32, [_vp, _u64, P(_u64), P(_i32)]),
    "wlg_engine_totals": (_i32, [_vp, P(wlg_run_totals)]),
    "wlg_engine_time_epochs": (_i32, [_vp, _u64, P(wlg_epoch_timing)]),
    "wlg_engine_time_run": (_i32, [_vp, _u64, P(wlg_epoch_timing)]),
    "wlg_engine_autotune": (_i32, [_vp, _u64, P(wlg_autotune_report)]),
    "wlg_engine_save_run": (_i32, [_vp, C.c_char_p]),
    "wlg_engine_load_run": (_i32, [_vp, C.c_char_p]),
    "wlg_engine_precision_report": (_i32, [_vp, P(wlg_precision_report)]),
    "wlg_engine_warm_start": (_i32, [_vp, P(_dbl), _dbl]),
    "wlg_engine_warm_start_continue": (_i32, [_vp, P(_dbl), _dbl]),
    "wlg_stitch_dos": (_i32, [_dbl, _dbl, _dbl, P(wlg_fragment_view), _u64, _i32, _u64, P(_dbl), P(_u64), P(_dbl),
                               P(C.c_uint8), P(wlg_join_quality), P(_i32)]),
    "wlg_engine_stitch": (_i32, [_vp, _i32, P(_dbl), P(_u64), P(_dbl), P(C.c_uint8), P(wlg_join_quality), P(_i32)]),
    "wlg_write_dos_csv": (_i32, [C.c_char_p, _dbl, _dbl, _u64, P(_dbl), P(_u64), P(_dbl), P(C.c_uint8)]),
    "wlg_write_fragment_csv": (_i32, [C.c_char_p, _dbl, _dbl, _u64, _u64, _u64, P(_dbl), P(_u64), P(_dbl),
                                      P(C.c_uint8)]),
    "wlg_write_workers_stat_csv": (_i32, [C.c_char_p, P(wlg_walker_statistics), _u64, _u64]),
    "wlg_adapt_energy_windows": (_i32, [_dbl, _dbl, _dbl, P(wlg_fragment_view), P(wlg_sampling_view), _u64, _dbl,
                                        P(wlg_adaptive_parameters), P(_u64)]),
    "wlg_select_initial_configurations": (_i32, [_dbl, _dbl, _dbl, P(_u64), _u64, P(_dbl), P(C.c_int8),
                                                 P(C.c_uint8), _u64, _u64, _u64, P(C.c_int8), P(C.c_uint8), P(_u64),
                                                 P(_u64)]),
    "wlg_batch_create": (_i32, [P(_vp), _u64, P(_vp)]),
    "wlg_batch_run_epochs": (_i32, [_vp, _u64, P(_u64), P(_i32)]),
    "wlg_batch_destroy": (None, [_vp]),
    "wlg_mlp_create": (_i32, [_i32, P(_i32), _u64, P(_vp)]),
    "wlg_mlp_destroy": (None, [_vp]),
    "wlg_mlp_parameter_count": (_u64, [_vp]),
    "wlg_mlp_get_parameters": (_i32, [_vp, P(C.c_float)]),
    "wlg_mlp_set_parameters": (_i32, [_vp, P(C.c_float)]),
    "wlg_mlp_forward": (_i32, [_vp, P(C.c_float), _u64, P(C.c_float)]),
    "wlg_mlp_gradients": (_i32, [_vp, P(C.c_float), P(C.c_float), _u64, P(C.c_float), P(_dbl)]),
    "wlg_mlp_train": (_i32, [_vp, P(C.c_float), P(C.c_float), _u64, _u64, _dbl, P(_dbl)]),
    "wlg_engine_set_launch": (_i32, [_vp, _i32, _i32]),
    "wlg_engine_set_window_sweep": (_i32, [_vp, _i32]),
    "wlg_engine_window_sweep": (_i32, [_vp]),
    "wlg_engine_walkers": (_u64, [_vp]),
    "wlg_engine_bins": (_u64, [_vp]),
    "wlg_engine_spins": (_u64, [_vp]),
    "wlg_engine_window": (_i32, [_vp, _u64, P(_u64), P(_u64)]),
    "wlg_engine_fragment": (_i32, [_vp, _u64, _i32, P(_dbl), P(_u64), P(_dbl), P(C.c_uint8)]),
    "wlg_engine_fragments": (_i32, [_vp, _i32, P(_dbl), P(_u64), P(_dbl), P(C.c_uint8)]),
    "wlg_engine_sampling_statistics": (_i32, [_vp, _u64, P(_dbl), P(_u64), P(_u64), P(_u64)]),
    "wlg_engine_walker_statistics": (_i32, [_vp, P(wlg_walker_statistics), _u64]),
    "wlg_engine_representatives": (_i32, [_vp, P(_dbl), P(C.c_int8), _u64, P(_u64)]),
    "wlg_walker_run_attempts": (_i32, [_vp, _u64, _u64]),
    "wlg_walker_snapshot": (_i32, [_vp, _u64, P(wlg_snapshot)]),
    "wlg_walker_restore": (_i32, [_vp, _u64, P(wlg_snapshot)]),
    "wlg_walker_histogram_statistics": (_i32, [_vp, _u64, P(wlg_histogram_statistics)]),
    "wlg_walker_flags": (_i32, [_vp, _u64, P(_i32), P(_i32), P(_i32)]),
    "wlg_walker_begin_next_iteration": (_i32, [_vp, _u64]),
    "wlg_walker_exchange_log_probability": (_i32, [_vp, _u64, _u64, P(_dbl)]),
    "wlg_walker_swap": (_i32, [_vp, _u64, _u64]),
}

_LIB = None


def load_library(path: Path | None = None) -> C.CDLL:
    """Loads libwlg.so (built in-tree by replica_exchange_wang_landau_b200.build).

    There is no fallback: a missing library is an error.
    """
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    target = Path(path) if path else LIBRARY_PATH
    if not target.exists():
        raise ImportError(
            f"{target} is missing; build it with `python -m replica_exchange_wang_landau_b200.build` "
            "(the engine has no CPU fallback)")
    lib = C.CDLL(str(target))
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    if lib.wlg_abi_version() != WLG_ABI_VERSION:
        raise ImportError("libwlg.so ABI version mismatch")
    if path is None:
        _LIB = lib
    return lib
