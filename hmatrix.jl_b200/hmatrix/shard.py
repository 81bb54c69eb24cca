"""Multi-GPU work split (one process per GPU): row-sharded H-matvec, and
independent problems of a batch spread over the ranks.

Every rank builds the same cluster tree (deterministic), owns a contiguous
range of rows and builds only the leaves of those rows (``Params.RowRange``):
its construction and its factor memory are 1/N of the whole.  H*x on a rank
gives its rows and zeros elsewhere; one all-reduce over the ranks (NCCL on
GPUs) then leaves the full H*x on every rank.  The row ranges are cut at the
starts of the maximal clusters of at most MaxBlock points: every leaf's rows
lie inside one of them (a block is subdivided while it has more rows than
MaxBlock, and dense leaves are at most MinBlock rows), so no leaf is cut.
"""
from __future__ import annotations

import dataclasses

import numpy as np


def block_starts(c, max_block):
    """Sorted starts of the maximal clusters with at most ``max_block`` points."""
    out = []
    stack = [0]
    while stack:
        i = stack.pop()
        if c.e[i] - c.s[i] <= max_block or c.left[i] < 0:
            out.append(int(c.s[i]))
        else:
            stack.append(int(c.right[i]))
            stack.append(int(c.left[i]))
    return sorted(out)


def row_splits(c, max_block, world):
    """Boundaries 0 = b_0 <= ... <= b_world = n (rank r owns [b_r, b_r+1)),
    each at a cluster start of :func:`block_starts`, nearest to r n / world."""
    n = int(c.e[0])
    starts = np.array(block_starts(c, max_block) + [n])
    b = [0]
    for r in range(1, world):
        t = r * n / world
        j = int(np.argmin(np.abs(starts - t)))
        b.append(max(b[-1], int(starts[j])))
    b.append(n)
    return b


def reduce_rows(y, dist, group=None):
    """The full H*x from every rank's rows (zeros elsewhere), in place."""
    if dist is not None and dist.get_world_size(group) > 1:
        dist.all_reduce(y, group=group)
    return y


class ShardedHmat:
    """This rank's shard of H (prm on the cluster tree of prm.Geom)."""

    def __init__(self, prm, rank, world, cluster=None):
        from . import construct_cluster, new_on_cluster
        X = np.asarray(prm.Geom, dtype=np.float64)
        if X.ndim == 1:
            X = X.reshape(-1, 1)
        if prm.MaxBlock == -1:
            prm.MaxBlock = X.shape[0] // 4
        self.c = cluster if cluster is not None else construct_cluster(X, prm.MinBlock, prm.Tree)
        self.splits = row_splits(self.c, prm.MaxBlock, world)
        self.lo, self.hi = self.splits[rank], self.splits[rank + 1]
        self.rank, self.world = rank, world
        sprm = dataclasses.replace(prm, RowRange=(self.lo, self.hi) if world > 1 else (0, 0))
        self.H = new_on_cluster(sprm, self.c)
        self.n = self.H.n

    def matvec(self, x, dist=None, group=None):
        """H*x on every rank (x: the full vector, a CUDA float64 tensor)."""
        return reduce_rows(self.H.matvec(x), dist, group)


def problem_cost(n, max_block):
    """Predicted relative cost of ``lu!`` + refined solve of one problem of n
    points whose tile level has T = ceil(n / max_block) tiles: the right-looking
    tile elimination recompresses about T^3 / 3 off-diagonal tiles, and each of
    its T steps carries a fixed launch latency worth about 64 tile updates."""
    T = max(1, -(-int(n) // int(max_block)))
    return 64.0 * T + T ** 3 / 3.0


def split_problems(costs, world):
    """Independent problems over ``world`` ranks, no exchange between them:
    longest predicted cost first, each to the rank with the least work so far
    (ties to the lowest rank).  Returns one sorted index list per rank; every
    index appears exactly once, and the most loaded rank carries at most the
    mean load plus the largest single cost."""
    costs = np.asarray(costs, dtype=np.float64)
    load = np.zeros(world)
    out = [[] for _ in range(world)]
    for i in np.argsort(-costs, kind="stable"):
        r = int(np.argmin(load))
        out[r].append(int(i))
        load[r] += costs[i]
    return [sorted(o) for o in out]
