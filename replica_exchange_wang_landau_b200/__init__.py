"""B200-native replica-exchange Wang-Landau walker engine.

The sampling path of the reference sampler (Faikert/replica_exchange_wang_landau) --
run_rewl and everything under it -- implemented as sm_100a CUDA kernels behind the C-ABI
in include/wlg.h.  Importing the package loads libwlg.so; there is no CPU fallback.
"""
from ._abi import LIBRARY_PATH, load_library
from .engine import (Couplings, DosFragment, Engine, Geometry, InitializationError, InvalidArgument, RewlResult, RunConfig,
                     Snapshot, System, WlgError, WlParameters, attempts_from_mcs, grid_bins, grid_index,
                     load_checkpoint, partition_windows, run_rewl, save_checkpoint)

__all__ = [
    "LIBRARY_PATH", "load_library", "Couplings", "DosFragment", "Engine", "Geometry", "InitializationError", "InvalidArgument",
    "RewlResult", "RunConfig", "Snapshot", "System", "WlgError", "WlParameters", "attempts_from_mcs", "grid_bins",
    "grid_index", "load_checkpoint", "partition_windows", "run_rewl", "save_checkpoint",
]
