"""The drop-in, end to end: the reference's own wl_run program with its sampling on the GPU.

oracle/Makefile compiles the reference's unmodified apps/wl_run.cpp twice: as wl_run (CPU,
the reference as shipped) and as wl_run_b200, with the adapter
(replica_exchange_wang_landau_b200/adapter) force-included so that both run_rewl call sites
(apps/wl_run.cpp:126 and :176) call run_rewl_b200, which hands the run to the engine through
the C-ABI.  Both programs get the same command line; every file they write (DOS, window
fragments, thermodynamics, metadata, worker statistics) and their summary line must be
byte-identical, except the elapsed time.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

import pytest

from helpers import random_axes
from replica_exchange_wang_landau_b200.engine import Geometry

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parents[1] / "oracle" / "_ref"
WL_RUN, WL_RUN_B200 = REF / "wl_run", REF / "wl_run_b200"


def _run(binary: Path, args: list, out: Path):
    out.mkdir(parents=True, exist_ok=True)
    env = dict(os.environ, OMP_NUM_THREADS="4")
    res = subprocess.run([str(binary), *args, "--output", str(out / "run")], capture_output=True, text=True,
                         env=env, timeout=900)
    summary = [line for line in res.stdout.splitlines() if not line.startswith("adaptive_window_elapsed")]
    summary = [" ".join(x for x in line.split() if not x.startswith("elapsed_seconds=")) for line in summary]
    files = {p.name: p.read_bytes() for p in sorted(out.iterdir())}
    return res.returncode, summary, files, res.stderr


def _compare(tmp_path, args):
    if not (WL_RUN.exists() and WL_RUN_B200.exists()):
        pytest.skip("oracle/_ref/wl_run and wl_run_b200 were not built")
    rc_a, out_a, files_a, err_a = _run(WL_RUN, args, tmp_path / "cpu")
    rc_b, out_b, files_b, err_b = _run(WL_RUN_B200, args, tmp_path / "gpu")
    assert rc_a in (0, 2), err_a
    assert rc_b == rc_a, err_b
    assert out_b == out_a
    assert sorted(files_b) == sorted(files_a)
    for name in files_a:
        assert files_b[name] == files_a[name], name
    return rc_a, files_a


def test_drop_in_plain_lattice_converges(tmp_path):
    # the plain configuration: 2x2x2 open lattice, +z axes, [-20, 20] in bins of 0.25, one
    # window of two walkers, 1/t to ln f = 1e-4, seed 1234
    rc, files = _compare(tmp_path, ["--nx", "2", "--ny", "2", "--nz", "2", "--periodic", "false", "--emin", "-20",
                                    "--emax", "20", "--bin-width", "0.25", "--windows", "1", "--walkers", "2",
                                    "--final-factor", "1e-4", "--seed", "1234"])
    assert rc == 0 and "run_dos.csv" in files and "run_workers_stat.csv" not in files


def test_drop_in_csv_geometry_with_exchange(tmp_path):
    # a CSV geometry (random axes), three windows of two walkers with exchanges every MCS,
    # stopped by max-mcs before convergence: the worker statistics file is written too
    g = Geometry.simple_cubic(3, 3, 3, periodic=True)
    g.axes = random_axes(g.size(), 5)
    tmp_path.mkdir(exist_ok=True)
    csv = tmp_path / "system.csv"
    g.to_csv(str(csv))
    rc, files = _compare(tmp_path, ["--geometry", str(csv), "--box-x", "3", "--box-y", "3", "--box-z", "3",
                                    "--periodic", "true", "--emin", "-60", "--emax", "60", "--bin-width", "0.5",
                                    "--windows", "3", "--walkers", "2", "--exchange-interval-mcs", "1",
                                    "--check-interval-mcs", "10", "--max-mcs", "300", "--seed", "21"])
    assert rc == 2 and "run_workers_stat.csv" in files and "run_window_2.csv" in files


def test_drop_in_csr_adaptive_windows(tmp_path):
    # the CSR backend (cutoff 1.8) and the adaptive-window pilot: both call sites of run_rewl
    rc, files = _compare(tmp_path, ["--nx", "4", "--ny", "4", "--nz", "4", "--periodic", "true", "--box-x", "4",
                                    "--box-y", "4", "--box-z", "4", "--cutoff", "1.8", "--emin", "-60", "--emax",
                                    "40", "--bin-width", "0.5", "--windows", "3", "--walkers", "2",
                                    "--adaptive-windows", "true", "--adaptive-iterations", "2",
                                    "--adaptive-pilot-mcs", "30", "--exchange-interval-mcs", "1", "--max-mcs", "100",
                                    "--seed", "9"])
    assert rc == 2 and "run_window_0.csv" in files


def test_drop_in_single_walker_checkpoint_and_resume(tmp_path):
    # one window of one walker writes the reference's WLCHKP3 checkpoint (src/parallel.cpp:522-525);
    # a second run with a higher max-mcs restores it (src/parallel.cpp:354-360) and continues
    if not (WL_RUN.exists() and WL_RUN_B200.exists()):
        pytest.skip("oracle/_ref/wl_run and wl_run_b200 were not built")
    base = ["--nx", "3", "--ny", "2", "--nz", "2", "--periodic", "false", "--emin", "-30", "--emax", "30",
            "--bin-width", "0.25", "--windows", "1", "--walkers", "1", "--seed", "8", "--checkpoint-interval-mcs", "50"]
    outputs = {}
    for name, binary in (("cpu", WL_RUN), ("gpu", WL_RUN_B200)):
        out = tmp_path / name
        chk = out / "run.chk"
        first = _run(binary, base + ["--checkpoint", str(chk), "--max-mcs", "200"], out)
        second = _run(binary, base + ["--checkpoint", str(chk), "--max-mcs", "400"], out)
        outputs[name] = (first, second)
    for k in (0, 1):
        rc_a, out_a, files_a, err_a = outputs["cpu"][k]
        rc_b, out_b, files_b, err_b = outputs["gpu"][k]
        assert rc_a == rc_b == 2, (err_a, err_b)
        assert out_b == out_a
        assert sorted(files_b) == sorted(files_a) and "run.chk" in files_a
        for name in files_a:
            assert files_b[name] == files_a[name], name
