"""bench.py's multi-rank path on CPU: two gloo ranks take the max of their
times, run independent seeded problems (weak scaling, no data-path
collective) and agree on the batch workload."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(dist)
        t = bench.allreduce_max(dist, 10.0 + rank)  # rank 1 is the slower one
        w = bench.make_workload("weno_fq_32", rank)
        out[rank] = (t, w["case"].seed, bench.parse_batch("batch12_s7"))
        bench.barrier(dist)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_as_max_and_run_independent_seeds():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 11.0          # max over ranks
    assert {res[0][1], res[1][1]} == {1000, 1001}  # one seeded problem per rank
    assert res[0][2] == res[1][2] == (12, 7)


def test_single_process_path_needs_no_process_group():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    assert bench.allreduce_max(None, 3.5) == 3.5
    assert bench.parse_batch("batch256") == (256, 500)
