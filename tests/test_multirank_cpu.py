"""The multi-GPU paths on CPU: world_size 2 over gloo.

`bench.py --gpus N` row-shards one H-matrix over the ranks (strong scaling):
each rank multiplies its own rows and one all-gather of the row shards leaves
H*x on every rank; the job time is the max over ranks.  `--replicas` runs N
independent copies instead (weak scaling), and `--batch` splits independent
problems over the ranks with no exchange.  These tests cover the timing
reductions, the shard boundaries (never inside a leaf, balanced by bytes),
the all-gather assembly and the problem split.
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


def test_row_splits_keep_leaves_whole():
    # the shard boundaries of the multi-GPU matvec never cut a leaf of the
    # partition (aca2 route, identity adjacency), checked on the C oracle's
    # partition of a 1-D and a 2-D tree
    import sys
    import numpy as np
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "hmatrix.jl_b200"))
    from hmatrix.cluster import construct_cluster
    from hmatrix.shard import row_splits
    from oracle import hm_oracle_c as O
    import ctypes as C
    for G, mb, minb in ((np.linspace(0, 10, 5000), 512, 64),
                        (np.random.default_rng(5).uniform(0, 1, (3000, 2)), 256, 32)):
        c = construct_cluster(G, minb, "bisect")
        s, e, l, r = (np.ascontiguousarray(a, np.int64) for a in (c.s, c.e, c.left, c.right))
        L = O.lib()
        n = int(c.e[0])
        cnt = L.orc_partition(O._p(s), O._p(e), O._p(l), O._p(r), minb, mb, 0, n, 0, C.c_void_p(0))
        lv = np.zeros((cnt, 5), np.int64)
        L.orc_partition(O._p(s), O._p(e), O._p(l), O._p(r), minb, mb, 0, n, cnt, O._p(lv))
        for world in (2, 3, 4, 8):
            b = row_splits(c, mb, world)
            assert b[0] == 0 and b[-1] == n and all(b[i] <= b[i + 1] for i in range(world))
            for t in b[1:-1]:
                cut = (lv[:, 1] < t) & (lv[:, 1] + lv[:, 3] > t)
                assert not cut.any()
            sizes = np.diff(b)
            assert sizes.max() - sizes.min() <= 2 * mb


def _shard_worker(rank, world, port, out):
    # the all-gather that assembles H*x from the shards, over gloo: each rank
    # holds its rows of a dense product (garbage elsewhere), shards of unequal
    # length, one vector and one block of 3 columns
    import datetime
    import sys
    import numpy as np
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "hmatrix.jl_b200"))
    from hmatrix.shard import gather_rows
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    rng = np.random.default_rng(0)
    A = rng.standard_normal((40, 40))
    x = rng.standard_normal((40, 3))
    b = [0, 17, 40]
    err = 0.0
    for X in (x[:, 0], x):
        y = torch.full((40,) + X.shape[1:], float(rank + 7), dtype=torch.float64)
        y[b[rank]:b[rank + 1]] = torch.tensor(A[b[rank]:b[rank + 1]] @ X)
        gather_rows(y, b, rank, dist)
        err = max(err, float(np.abs(y.numpy() - A @ X).max()))
    out.put((rank, err))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_reduction_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, err in res:
        assert err <= 1e-12


def test_host_partition_matches_oracle():
    # hm_partition (the library's host-side partition, no device) lists the
    # same leaves in the same order as the oracle's partition of __c1
    import sys
    import numpy as np
    import ctypes as C
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "hmatrix.jl_b200"))
    import hmatrix as hm
    from hmatrix.cluster import construct_cluster
    from hmatrix.shard import partition_leaves
    from oracle import hm_oracle_c as O
    for G, mb, minb, tree in ((np.linspace(0, 10, 5000), 512, 64, "bisect"),
                              (np.linspace(0, 10, 3000), 512, 64, "kmeans"),
                              (np.random.default_rng(5).uniform(0, 1, (3000, 2)), 256, 32, "bisect")):
        c = construct_cluster(G, minb, tree)
        prm = hm.Params(Geom=G, Kernel=hm.Cauchy(1.0), MaxBlock=mb, MinBlock=minb, ConsMethod="aca2")
        got = partition_leaves(prm, c)
        s, e, l, r = (np.ascontiguousarray(a, np.int64) for a in (c.s, c.e, c.left, c.right))
        L = O.lib()
        n = int(c.e[0])
        cnt = L.orc_partition(O._p(s), O._p(e), O._p(l), O._p(r), minb, mb, 0, n, 0, C.c_void_p(0))
        lv = np.zeros((cnt, 5), np.int64)
        L.orc_partition(O._p(s), O._p(e), O._p(l), O._p(r), minb, mb, 0, n, cnt, O._p(lv))
        assert np.array_equal(got, lv)


def test_byte_balanced_splits():
    # on a 2-D tree the byte-balanced cut points give shards whose streamed
    # bytes are closer to equal than the row-balanced ones, and never cut a leaf
    import sys
    import numpy as np
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "hmatrix.jl_b200"))
    import hmatrix as hm
    from hmatrix.cluster import construct_cluster
    from hmatrix.shard import partition_leaves, row_bytes, row_splits
    G = np.random.default_rng(7).uniform(0, 1, (20000, 2))
    G[:6000] *= 0.2                                   # a dense corner: uneven rows
    c = construct_cluster(G, 32, "bisect")
    prm = hm.Params(Geom=G, Kernel=hm.Cauchy(1.0), MaxBlock=256, MinBlock=32, ConsMethod="aca2")
    lv = partition_leaves(prm, c)
    w = row_bytes(lv, 20000)
    cw = np.concatenate([[0.0], np.cumsum(w)])
    for world in (2, 4, 8):
        br = row_splits(c, 256, world)
        bb = row_splits(c, 256, world, w)
        spread = lambda b: max(cw[b[i + 1]] - cw[b[i]] for i in range(world)) / (cw[-1] / world)
        assert spread(bb) <= spread(br) + 1e-12
        for t in bb[1:-1]:
            assert not ((lv[:, 1] < t) & (lv[:, 1] + lv[:, 3] > t)).any()


def test_split_problems_cover_and_balance():
    # the batched uneven problems over 1..8 ranks: every problem on exactly one
    # rank, the most loaded rank within the LPT bound (mean + largest cost)
    import sys
    import numpy as np
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "hmatrix.jl_b200"))
    import bench
    from hmatrix.shard import problem_cost, split_problems
    probs = bench.batched_problems(256)
    costs = np.array([problem_cost(len(p[0]), 256) for p in probs])
    assert problem_cost(256, 256) < problem_cost(257, 256) < problem_cost(65536, 256)
    for world in (1, 2, 3, 4, 8):
        parts = split_problems(costs, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(probs)))
        loads = np.array([costs[p].sum() for p in parts])
        assert loads.max() <= costs.sum() / world + costs.max() + 1e-9
        if world > 1:
            assert loads.max() <= 1.05 * costs.sum() / world
    # fewer problems than ranks: the extra ranks get none
    parts = split_problems([5.0, 1.0], 4)
    assert parts == [[0], [1], [], []]


def _batch_worker(rank, world, port, out):
    # each rank takes its share of the batch with no exchange; only the
    # counts, the job time (max) and the worst residual (max) are reduced
    import datetime
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "hmatrix.jl_b200"))
    import bench
    from hmatrix.shard import problem_cost, split_problems
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    probs = bench.batched_problems(32)
    mine = split_problems([problem_cost(len(p[0]), 256) for p in probs], world)[rank]
    cnt = torch.tensor([float(len(mine)), float(sum(len(probs[i][0]) for i in mine))], dtype=torch.float64)
    dist.all_reduce(cnt)
    ms = bench.job_time([3.0, 5.0][rank], dist, "cpu")
    worst = bench.job_time([1e-12, 4e-11][rank], dist, "cpu")
    out.put((rank, int(cnt[0]), int(cnt[1]), ms, worst, sum(len(p[0]) for p in probs)))
    dist.barrier()
    dist.destroy_process_group()


def test_batch_split_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, count, sum_n, ms, worst, total_n in res:
        assert count == 32 and sum_n == total_n
        assert ms == 5.0 and worst == 4e-11
