"""CPU checks of the C-ABI boundary: libwlg.so loads and exports every entry point that
include/wlg.h declares, the ctypes structs match the C layouts, and the exact integer
helpers of the kernels are right.  No GPU needed."""
from __future__ import annotations

import ctypes as C
import json
import re
import shutil
import subprocess
from pathlib import Path

import pytest

from replica_exchange_wang_landau_b200 import _abi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "wlg.h"


def declared_functions() -> set:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(wlg_[a-z_0-9]+)\s*\(", text))


def test_library_exports_every_declared_symbol():
    lib = _abi.load_library()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert missing == []
    assert set(_abi.SIGNATURES) == names, "ctypes signature table out of sync with include/wlg.h"
    nm = subprocess.run(["nm", "-D", "--defined-only", str(_abi.LIBRARY_PATH)], capture_output=True, text=True)
    exported = set(re.findall(r"\bT (wlg_\w+)", nm.stdout))
    assert names <= exported


def test_abi_version_and_error_channel():
    lib = _abi.load_library()
    assert lib.wlg_abi_version() == _abi.WLG_ABI_VERSION
    bins = C.c_uint64(0)
    assert lib.wlg_grid_bins(-1.0, 1.0, 0.3, C.byref(bins)) == 1
    assert b"integer multiple" in lib.wlg_last_error()


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_struct_layouts_match_header(tmp_path):
    exe = tmp_path / "abi_layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(ROOT / "tests" / "native" / "abi_layout.c"), "-o",
                    str(exe)], check=True)
    layout = json.loads(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout)
    for name, cls in _abi.STRUCTS.items():
        assert C.sizeof(cls) == layout[name], name
        for field, _ in cls._fields_:
            assert getattr(cls, field).offset == layout[f"{name}.{field}"], f"{name}.{field}"


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_kernel_integer_helpers_exact(tmp_path):
    """x87_mean reproduces the reference's long-double histogram mean; fast_mod, the generator's
    step back and the add-based bin floor are exact."""
    exe = tmp_path / "host_math_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-frounding-math", "-I/usr/local/cuda/include",
                    str(ROOT / "tests" / "native" / "host_math_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout


def test_engine_fails_loudly_without_a_device():
    import os
    if os.path.exists("/dev/nvidia0"):
        pytest.skip("a GPU is present")
    from replica_exchange_wang_landau_b200.engine import DeviceError, Engine, Geometry, RunConfig, System
    with pytest.raises(DeviceError):
        Engine(System(Geometry.simple_cubic(2, 2, 1, periodic=False)), RunConfig(emin=-20, emax=20, bin_width=0.25))
