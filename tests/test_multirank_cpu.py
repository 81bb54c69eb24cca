"""The multi-GPU path of bench.py on CPU: world_size 2 over gloo.

`bench.py --gpus N` runs one replica of the H-matrix per rank (independent
H-matrices, no exchange in the data path); the only collective is the max over
ranks of the per-rank time, and the whole-job value counts every rank's bytes.
"""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms_local = [12.5, 20.0][rank]                 # rank 1 is the slower replica
    ms = bench.job_time(ms_local, dist, "cpu")
    value = bench.job_value(1e9, world, ms)
    out.put((rank, ms, value))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value in res:
        assert ms == 20.0                         # the max over ranks on every rank
        assert value == pytest.approx(2 * 1e9 / 20e-3 / 1e9)


def test_single_rank_passthrough():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.job_time(7.0, None, "cpu") == 7.0
    assert bench.job_value(2e9, 1, 10.0) == pytest.approx(200.0)
