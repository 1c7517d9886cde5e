"""GPU parity at the shapes bench.py measures, bit for bit against the oracle.

The bench's figures come from three configurations; each is run here through the same
product path (CUDA-graph replays of [sweep, exchange]) and compared with the oracle's
run_rewl (src/parallel.cpp:276-534) on the identical system and configuration:

* the dense REWL workload (8x8x8 periodic, random axes, 16 windows x 8 walkers, 913 bins of
  0.5, exchange every MCS): 1300 MCS, past the switch to the 1/t stage, through the split
  sweep (sweep_dense_split_kernel);
* the mixed-precision configuration with FP64, FP32 and row-scaled BF16 couplings (16x16x16
  lattice with 40% of the sites removed, N = 2458, slab box (16, 16, 0), 32 windows x 8
  walkers; FP64 recompute after every MCS for the FP32 and BF16 forms): 3 MCS through the ring
  sweep for systems beyond 1024 sites;
* the CSR configuration (32^3 periodic, cutoff 3.0, 122 neighbours in 128-wide ELLPACK rows,
  64 windows x 16 walkers = 1024 walkers, exchange every 0.05 MCS), FP64 and FP32 couplings:
  0.2 MCS through sweep_csr_kernel.  The bench seeds its windows from an adaptive pilot
  (tested on its own in test_gpu_adaptive.py); here the windows are the uniform partition of
  the same grid.

The oracle takes about a minute of host time for each.
"""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

from helpers import results_equal
from replica_exchange_wang_landau_b200.engine import Engine, Geometry, RunConfig, System, WlParameters

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
import bench  # noqa: E402

pytestmark = pytest.mark.gpu


def _run(system, config):
    with Engine(system, config) as e:
        e.run()
        stages = [e.snapshot(w).stage for w in range(e.walkers)]
        return e.result(), stages


def test_dense_rewl_workload_bitwise(oracle):
    system, config = bench.make_workload(seed=1)
    config.max_mcs = 1300.0
    config.resolved_spin_count = 0
    config.resolve_mcs(system.size())
    assert config.bins() == 913 and config.windows * config.walkers == 128
    got, stages = _run(system, config)
    want = oracle.run_rewl(system, config)
    assert got.attempted == 128 * 1300 * 512
    assert results_equal(got, want) == []
    assert stages.count(1) > 0, "no walker reached the 1/t stage"


def test_mixed_precision_workload_fp64_bitwise(oracle):
    system, configs = bench.mixed_precision_workload(precisions=("fp64",))
    config = configs["fp64"]
    assert system.size() == 2458 and config.windows * config.walkers == 256
    config.max_mcs = 3.0
    config.resolved_spin_count = 0
    config.resolve_mcs(system.size())
    got, _ = _run(system, config)
    want = oracle.run_rewl(system, config)
    assert got.attempted == 256 * 3 * 2458
    assert results_equal(got, want) == []


def _csr_workload(precision):
    g = Geometry.simple_cubic(32, 32, 32, 1.0, (0.0, 0.0, 1.0), True)
    g.box = (32.0, 32.0, 32.0)
    system = System(g, 1.0, 3.0)
    c = RunConfig(emin=-2144.0, emax=1932.0, bin_width=4.0, windows=64, walkers=16, overlap=0.75, seed=3)
    c.wl = WlParameters(0.8, 100, 1e-8, 1000, 0, True)
    c.coupling_precision = precision
    c.recompute_interval_mcs = 10.0
    c.exchange_interval_mcs = 0.05
    c.max_mcs = 0.2
    c.resolve_mcs(system.size())
    return system, c


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_csr_workload_bitwise(oracle, precision):
    system, config = _csr_workload(precision)
    got, _ = _run(system, config)
    want = oracle.run_rewl(system, config)
    assert got.attempted == 1024 * config.max_attempts  # 0.2 MCS: four epochs of 1638 attempts and one of 2
    assert got.exchange_attempted > 0
    assert results_equal(got, want) == []



@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_mixed_precision_workload_low_precision_bitwise(oracle, precision):
    """The mixed-precision configuration with FP32 (or row-scaled BF16) couplings and the FP64
    recompute after every MCS (the bench's FP32 and BF16 lines): rounded couplings in every
    accepted flip, the recompute and resync after every epoch, bit for bit against the oracle's
    restatement."""
    system, configs = bench.mixed_precision_workload(precisions=(precision,))
    config = configs[precision]
    config.max_mcs = 3.0
    config.resolved_spin_count = 0
    config.resolve_mcs(system.size())
    got, _ = _run(system, config)
    want = oracle.run_rewl(system, config)
    assert got.precision_report["recomputes"] >= 2
    assert results_equal(got, want) == []
