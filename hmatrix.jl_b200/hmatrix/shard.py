"""Multi-GPU work split (one process per GPU): row-sharded H-matvec, and
independent problems of a batch spread over the ranks.

Every rank builds the same cluster tree (deterministic), owns a contiguous
range of rows and builds only the leaves of those rows (``Params.RowRange``):
its construction and its factor memory are its share of the whole.  The row
ranges are cut at the starts of the maximal clusters of at most MaxBlock
points: every leaf's rows lie inside one of them (a block is subdivided while
it has more rows than MaxBlock, and dense leaves are at most MinBlock rows),
so no leaf is cut.  Among those cut points the split balances the bytes the
shards will stream per matvec, read off the block partition
(``hm_partition``, computed on the host): dense leaves m*n entries, low-rank
leaves (m+n)*k with k estimated, since ranks are known only after the
compression.

H*x on a rank gives its own rows (zeros elsewhere); one all-gather of the row
shards over the ranks (NCCL on GPUs) then leaves the full H*x on every rank:
each rank receives the n - (its rows) values it lacks, half the traffic of an
all-reduce of the full vector.
"""
from __future__ import annotations

import ctypes as C
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


def partition_leaves(prm, c):
    """The leaves of the block partition of ``prm`` on the tree ``c``, from the
    library's host-side partition (no device): rows (type 0 dense / 1
    low-rank, row0, col0, m, n)."""
    from . import _lib, _params_struct
    from ._lib import check, lib
    X = np.asarray(c.X, dtype=np.float64)
    d = 1 if X.ndim == 1 else X.shape[1]
    if prm.MaxBlock == -1:
        prm.MaxBlock = int(c.e[0]) // 4
    p = _params_struct(prm, d)
    arrs = [np.ascontiguousarray(a, np.int64) for a in (c.s, c.e, c.left, c.right)]
    ptr = [C.c_void_p(a.ctypes.data) for a in arrs]
    from .cluster import neighbor_pairs
    nb = neighbor_pairs(c, prm.Adj)
    nbp = None if nb is None else np.ascontiguousarray(nb)
    nbv = None if nbp is None else C.c_void_p(nbp.ctypes.data)
    cnt = C.c_int64(0)
    n = int(c.e[0])
    check(lib().hm_partition(C.byref(p), n, len(arrs[0]), *ptr, 0 if nb is None else len(nb), nbv, 0, None,
                             C.byref(cnt)))
    out = np.zeros((cnt.value, 5), np.int64)
    check(lib().hm_partition(C.byref(p), n, len(arrs[0]), *ptr, 0 if nb is None else len(nb), nbv, cnt.value,
                             C.c_void_p(out.ctypes.data), C.byref(cnt)))
    return out


def row_bytes(leaves, n, rank_est=3, eb=8, deb=8):
    """Bytes a matvec streams for each row: every leaf's stored entries spread
    evenly over its rows (dense m*n, low-rank (m+n)*rank_est)."""
    L = np.asarray(leaves, dtype=np.int64).reshape(-1, 5)
    t, r0, m, nn = L[:, 0], L[:, 1], L[:, 3].astype(np.float64), L[:, 4].astype(np.float64)
    per_row = np.where(t == 0, deb * m * nn, eb * (m + nn) * rank_est) / m
    w = np.zeros(n + 1)
    np.add.at(w, r0, per_row)
    np.add.at(w, r0 + L[:, 3], -per_row)
    return np.cumsum(w)[:n]


def row_splits(c, max_block, world, weights=None):
    """Boundaries 0 = b_0 <= ... <= b_world = n (rank r owns [b_r, b_r+1)),
    each at a cluster start of :func:`block_starts`.  Without ``weights`` the
    cut nearest to r n / world; with per-row ``weights`` (bytes), the cut whose
    cumulative weight is nearest to r / world of the total."""
    n = int(c.e[0])
    starts = np.array(block_starts(c, max_block) + [n])
    if weights is None:
        cum = starts.astype(np.float64)
        total = float(n)
    else:
        cw = np.concatenate([[0.0], np.cumsum(np.asarray(weights, dtype=np.float64))])
        cum = cw[starts]
        total = float(cw[-1])
    b = [0]
    for r in range(1, world):
        t = r * total / world
        j = int(np.argmin(np.abs(cum - t)))
        b.append(max(b[-1], int(starts[j])))
    b.append(n)
    return b


def gather_rows(y, splits, rank, dist, group=None):
    """The full H*x on every rank from every rank's own rows [splits[r],
    splits[r+1]) of ``y`` (a torch vector or n x c block, rows first), in
    place: one all-gather of the row shards, padded to the longest."""
    world = len(splits) - 1
    if dist is None or world <= 1:
        return y
    import torch
    lens = [splits[r + 1] - splits[r] for r in range(world)]
    L = max(lens)
    tail = tuple(y.shape[1:])
    send = torch.zeros((L,) + tail, dtype=y.dtype, device=y.device)
    send[:lens[rank]] = y[splits[rank]:splits[rank + 1]]
    recv = [torch.empty_like(send) for _ in range(world)]
    dist.all_gather(recv, send, group=group)
    for r in range(world):
        if r != rank:
            y[splits[r]:splits[r + 1]] = recv[r][:lens[r]]
    return y


class ShardedHmat:
    """This rank's shard of H (prm on the cluster tree of prm.Geom)."""

    def __init__(self, prm, rank, world, cluster=None, balance="bytes", rank_est=3):
        from . import construct_cluster, new_on_cluster
        X = np.asarray(prm.Geom, dtype=np.float64)
        if X.ndim == 1:
            X = X.reshape(-1, 1)
        if prm.MaxBlock == -1:
            prm.MaxBlock = X.shape[0] // 4
        self.c = cluster if cluster is not None else construct_cluster(X, prm.MinBlock, prm.Tree)
        w = None
        if world > 1 and balance == "bytes" and prm.ConsMethod != "svd":
            eb = {0: 8, 1: 4, 2: 2}[prm.Storage]
            w = row_bytes(partition_leaves(prm, self.c), X.shape[0], rank_est, eb, 8 if eb == 8 else 4)
        self.splits = row_splits(self.c, prm.MaxBlock, world, w)
        self.lo, self.hi = self.splits[rank], self.splits[rank + 1]
        self.rank, self.world = rank, world
        sprm = dataclasses.replace(prm, RowRange=(self.lo, self.hi) if world > 1 else (0, 0))
        self.H = new_on_cluster(sprm, self.c)
        self.n = self.H.n

    def matvec(self, x, dist=None, group=None):
        """H*x on every rank (x: the full vector, a CUDA float64 tensor)."""
        return gather_rows(self.H.matvec(x), self.splits, self.rank, dist, group)


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
