"""The bench's two arms run the same system, and the reference arm runs the reference alone.

bench.py's reference arm runs the reference's own wl_run program on the dense REWL workload
read from oracle/workloads/dense_rewl_8x8x8_seed1.csv (the reference's CSV geometry format),
while the engine's arm generates the system with simple_cubic_random(8, 8, 8, seed=1).  These
tests check that the file holds exactly the generator's doubles, that the wl_run command line
sets the configuration the engine's arm uses, and that the reference arm loads nothing of this
repository's engine.
"""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_workload_csv_is_the_generated_system():
    from replica_exchange_wang_landau_b200.engine import Geometry
    from replica_exchange_wang_landau_b200.geometry import simple_cubic_random
    want = simple_cubic_random(8, 8, 8, seed=1, periodic=True)
    got = Geometry.load_csv(str(bench.WORKLOAD_CSV), box=(8.0, 8.0, 8.0), periodic=True)
    assert np.array_equal(got.positions.view(np.uint64), want.positions.view(np.uint64))
    assert np.array_equal(got.axes.view(np.uint64), want.axes.view(np.uint64))
    assert tuple(want.box) == (8.0, 8.0, 8.0) and want.periodic


def test_wl_run_command_matches_the_engine_configuration():
    system, config = bench.make_workload(seed=1)
    cmd = bench.reference_wl_run_command(50, 1, "/tmp/x")
    opts = dict(zip(cmd[1::2], cmd[2::2]))
    assert float(opts["--emin"]) == config.emin and float(opts["--emax"]) == config.emax
    assert float(opts["--bin-width"]) == config.bin_width
    assert int(opts["--windows"]) == config.windows and int(opts["--walkers"]) == config.walkers
    assert float(opts["--overlap"]) == config.overlap
    assert float(opts["--exchange-interval-mcs"]) == config.exchange_interval_mcs
    assert int(opts["--seed"]) == config.seed
    assert [float(opts[k]) for k in ("--box-x", "--box-y", "--box-z")] == list(system.geometry.box)
    assert opts["--periodic"] == "true" and float(opts["--coupling"]) == system.coupling_scale


def test_parse_wl_run_summary():
    out = ("seed=1 source=configured\nspins=512 exchange_interval_mcs=1\n"
           "attempted_flips=3276800 aggregate_mcs=6400 accepted=2276659 forced=0 exchanges=1151/3000 "
           "converged=no elapsed_seconds=1.3641\n")
    s = bench.parse_wl_run_summary(out)
    assert s["attempted_flips"] == "3276800" and float(s["elapsed_seconds"]) == 1.3641


@pytest.mark.skipif(not bench.REFERENCE_WL_RUN.exists(), reason="oracle/_ref/wl_run is not built")
def test_reference_arm_loads_no_engine_code():
    probe = (
        "import json, runpy, sys\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', '--reference-step-mcs', '1']\n"
        "runpy.run_path('bench.py', run_name='__main__')\n"
        "bad = sorted(m for m in sys.modules if m.split('.')[0] in ('replica_exchange_wang_landau_b200', 'oracle', 'torch'))\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'modules': bad, 'libwlg': 'libwlg.so' in maps, 'libwlref': 'libwlref.so' in maps}))\n")
    res = subprocess.run([sys.executable, "-c", probe], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr
    lines = [json.loads(x) for x in res.stdout.splitlines() if x.startswith("{")]
    line, probe_out = lines[0], lines[-1]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["value"] == line["value"]
    assert probe_out == {"modules": [], "libwlg": False, "libwlref": False}
