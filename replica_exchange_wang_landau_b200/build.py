"""Builds the engine's shared library, libwlg.so, in-tree with nvcc for sm_100a.

Usage:  python -m replica_exchange_wang_landau_b200.build [--verbose-ptxas]

Every translation unit is compiled with ``--fmad=false`` so that no multiply-add is
contracted: the engine evaluates the reference's floating-point expressions in the same
order and with the same roundings, which is what makes its trajectories bit-identical.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
CSRC = PACKAGE / "csrc"
BUILD = PACKAGE / "_build"
LIBRARY = PACKAGE / "libwlg.so"
SOURCES = ["physics.cu", "walker.cu", "sweep.cu", "sweep_csr.cu", "sweep_window.cu", "rewl.cu", "stitch.cu", "precision.cu", "mlp.cu", "noalloc.cu", "engine.cpp", "host.cpp", "stitch.cpp", "adaptive.cpp", "api.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found; the engine needs the CUDA toolkit to build")


def _flags(source: str, ptxas_verbose: bool) -> list[str]:
    flags = ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]
    if source.endswith(".cu"):
        flags = ARCH + flags + ["--expt-relaxed-constexpr"]
        if ptxas_verbose:
            flags += ["-Xptxas", "-v"]
    else:
        flags = flags + ["-x", "cu"] + ARCH  # host files use CUDA runtime types
    return flags


def _compile(source: str, ptxas_verbose: bool) -> tuple[str, str]:
    src = CSRC / source
    obj = BUILD / (source + ".o")
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + [PACKAGE.parent / "include" / "wlg.h"]
    newest = max(p.stat().st_mtime for p in [src, *headers])
    if obj.exists() and obj.stat().st_mtime >= newest and not ptxas_verbose:
        return source, ""
    cmd = [nvcc(), *_flags(source, ptxas_verbose), "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {source}:\n{res.stdout}\n{res.stderr}")
    return source, res.stderr


def build(ptxas_verbose: bool = False, quiet: bool = True) -> Path:
    BUILD.mkdir(exist_ok=True)
    logs = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as pool:
        for source, log in pool.map(lambda s: _compile(s, ptxas_verbose), SOURCES):
            if log:
                logs.append(f"== {source}\n{log}")
    objects = [str(BUILD / (s + ".o")) for s in SOURCES]
    newest_obj = max(Path(o).stat().st_mtime for o in objects)
    if not LIBRARY.exists() or LIBRARY.stat().st_mtime < newest_obj:
        tmp = LIBRARY.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objects]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIBRARY)
    if logs and not quiet:
        print("\n".join(logs), file=sys.stderr)
    return LIBRARY


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--verbose-ptxas", action="store_true", help="print registers/spills per kernel")
    args = parser.parse_args()
    path = build(ptxas_verbose=args.verbose_ptxas, quiet=False)
    print(path)


if __name__ == "__main__":
    main()
