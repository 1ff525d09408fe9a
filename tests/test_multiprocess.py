"""World-size-2 gloo run of the multi-rank plumbing used by bench.py: each
rank takes its own share of independent days, and timings reduce as the max
over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from solweig_cuda_b200 import shard
    days = list(range(172, 202))
    mine = shard.split(days, rank, world)
    t = shard.max_over_ranks([float(len(mine)) + rank * 0.5, float(rank)])
    out[rank] = (mine, t)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_day_sharding_and_max_reduction():
    port = _free_port()
    manager = mp.Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    (d0, t0), (d1, t1) = out[0], out[1]
    assert d0 + d1 == list(range(172, 202)) and not set(d0) & set(d1)
    assert t0 == t1 == [15.5, 1.0]


def _series_worker(rank, world, port, folder, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from test_series_host import run_stub
    files = run_stub(folder, days=5, save_tmrt=True)  # rank and world from the process group
    out[rank] = files
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_run_timeseries_union_equals_single_rank(tmp_path):
    """Two gloo ranks drive the series driver (day assignment, output writer)
    over a shared output folder; the union of their days and files equals a
    single-rank run."""
    import numpy as np
    from test_series_host import run_stub
    port = _free_port()
    manager = mp.Manager()
    out = manager.dict()
    mp.start_processes(_series_worker, args=(2, port, str(tmp_path / "two"), out), nprocs=2, join=True,
                       start_method="spawn")
    whole = run_stub(tmp_path / "one", days=5, save_tmrt=True, rank=0, world_size=1)
    d0, d1 = out[0]["days"], out[1]["days"]
    assert len(d0) == 3 and len(d1) == 2 and not set(d0) & set(d1)
    merged = {**d0, **d1}
    assert sorted(merged) == sorted(whole["days"])
    for date, rec in whole["days"].items():
        for var, paths in rec.items():
            assert np.array_equal(np.load(paths[0]), np.load(merged[date][var][0]))
