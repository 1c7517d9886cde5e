"""The N > 1 path of bench.py on the CPU: two ranks over gloo (one process per rank, as the
launcher starts them per GPU) reduce their figures to the whole job's — the maximum of each time,
the sum of each count — and run independent replicas with different seeds."""
from __future__ import annotations

import json
import os
import socket
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        maxima, sums = bench.reduce_over_ranks(dist, "cpu", [1.5 + rank, 10.0 * rank], [100 + rank, 7])
        _, config = bench.make_workload(seed=1 + rank)
        dist.barrier()
    finally:
        dist.destroy_process_group()
    Path(out_dir, f"rank{rank}.json").write_text(json.dumps({"maxima": maxima, "sums": sums, "seed": config.seed}))


def test_two_ranks_over_gloo(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    got = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for g in got:
        assert g["maxima"] == [2.5, 10.0]
        assert g["sums"] == [201.0, 14.0]
    assert got[0]["seed"] != got[1]["seed"]  # independent replicas


def test_one_process_is_the_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.reduce_over_ranks(None, "cpu", [3.0, 4.0], [5, 6]) == ([3.0, 4.0], [5.0, 6.0])
