"""Host-side cluster tree (src/cluster.jl:196-256).

The reference bisects each cluster with sklearn ``KMeans(n_clusters=2,
random_state=0)`` (label 0 becomes the left child, both children keep the
increasing index order of ``findall``), assigns ids in the pre-order of the
downward pass and a cluster is a leaf once ``N <= MinBlock``.  ``method=
"bisect"`` replaces KMeans by a median split of the widest coordinate, which
is deterministic and fast at n = 2^20.  The KMeans tree of a large n spends
minutes in thousands of KMeans calls; below its top levels the subtrees are
independent and go to a pool of host processes.
"""
from __future__ import annotations

import numpy as np


class Cluster:
    """Mirror of the reference ``Cluster`` (src/cluster.jl:7-19) for the root.

    ``X`` is the permuted geometry (n x d), ``P`` the 0-based permutation
    (``X == Geom[P]``); the flattened tree is in ``s, e, left, right``
    (0-based start, exclusive end, child index or -1) in pre-order.
    """

    def __init__(self, X, P, s, e, left, right):
        self.X, self.P = X, P
        self.s, self.e, self.left, self.right = s, e, left, right
        self.N = X.shape[0]

    @property
    def ncluster(self):
        return len(self.s)


def _split_kmeans(X):
    from sklearn.cluster import KMeans
    from threadpoolctl import threadpool_limits
    # single-threaded: multi-threaded Lloyd reductions pick between mirror
    # image splits of near-equal inertia non-deterministically
    with threadpool_limits(limits=1):
        L = KMeans(n_clusters=2, random_state=0, n_init=10).fit(X).labels_
    return np.flatnonzero(L == 0), np.flatnonzero(L == 1)


def _split_bisect(X):
    N = X.shape[0]
    ext = X.max(axis=0) - X.min(axis=0)
    q = int(np.argmax(ext))
    order = np.argsort(X[:, q], kind="stable")
    h = (N + 1) // 2
    return np.sort(order[:h]), np.sort(order[h:])


def construct_cluster(Geom, Nleaf, method="kmeans", workers=None):
    """Build the cluster tree; returns a :class:`Cluster` root.

    ``workers``: host processes for the KMeans tree (None: up to 16 when n is
    above 32768, else 1).  Every split is the same single-threaded KMeans call
    whichever process makes it, so the tree does not depend on ``workers``."""
    X = np.asarray(Geom, dtype=np.float64)
    if X.ndim == 1:
        X = X.reshape(-1, 1)
    n = X.shape[0]
    if method == "bisect" and X.shape[1] == 1 and n > 1 and np.all(np.diff(X[:, 0]) >= 0):
        return _bisect_sorted_1d(X, Nleaf)
    if method == "kmeans":
        if workers is None:
            import os
            workers = min(16, os.cpu_count() or 1) if n > 32768 else 1
        if workers > 1:
            return _kmeans_parallel(X, Nleaf, workers)
    s, e, left, right, perm = _build_tree(X, Nleaf, method)
    return Cluster(X[perm], perm, s, e, left, right)


def _build_tree(X, Nleaf, method):
    """The downward pass of src/cluster.jl:223-240 on X: flattened arrays in
    pre-order (ids 0..) and the permutation."""
    n = X.shape[0]
    split = _split_kmeans if method == "kmeans" else _split_bisect
    s, e, left, right = [], [], [], []
    leaves_P = []
    # explicit stack: (indices into the original geometry, start, parent slot)
    stack = [(np.arange(n), 0, None, 0)]
    while stack:
        P, start, parent, side = stack.pop()
        cid = len(s)
        s.append(start)
        e.append(start + len(P))
        left.append(-1)
        right.append(-1)
        if parent is not None:
            (left if side == 0 else right)[parent] = cid
        if len(P) <= Nleaf:
            leaves_P.append((start, P))
            continue
        P1, P2 = split(X[P])
        stack.append((P[P2], start + len(P1), cid, 1))
        stack.append((P[P1], start, cid, 0))
    perm = np.empty(n, np.int64)
    for start, P in leaves_P:
        perm[start:start + len(P)] = P
    return (np.asarray(s, np.int64), np.asarray(e, np.int64), np.asarray(left, np.int64),
            np.asarray(right, np.int64), perm)


def _subtree_job(args):
    X, Nleaf = args
    return _build_tree(X, Nleaf, "kmeans")


def _kmeans_parallel(X, Nleaf, workers):
    """The KMeans tree with the subtrees below the top levels built in a pool
    of host processes (spawned: safe after CUDA is initialised), then spliced
    into the pre-order of the whole tree."""
    import concurrent.futures as cf
    import multiprocessing as mp
    n = X.shape[0]
    # top levels on this process: split the largest pending cluster until there
    # are enough subtrees to keep the pool busy
    # node: [P (indices into X), children or None, subtree slot or None]
    root = [np.arange(n), None, None]
    pending = [root]
    target = 4 * workers
    while len(pending) < target:
        pending.sort(key=lambda nd: -len(nd[0]))
        nd = pending[0]
        if len(nd[0]) <= Nleaf or len(nd[0]) < 4096:
            break
        P1, P2 = _split_kmeans(X[nd[0]])
        a, b = [nd[0][P1], None, None], [nd[0][P2], None, None]
        nd[1] = (a, b)
        pending = pending[1:] + [a, b]
    jobs = [nd for nd in pending if len(nd[0]) > Nleaf]
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        futs = [ex.submit(_subtree_job, (X[nd[0]], Nleaf)) for nd in jobs]
        for nd, f in zip(jobs, futs):
            nd[2] = f.result()
    s, e, left, right = [], [], [], []
    perm = np.empty(n, np.int64)

    def emit(nd, start, parent, side):
        cid = len(s)
        if nd[1] is None and nd[2] is not None:          # a subtree built by a worker
            ss, ee, ll, rr, pp = nd[2]
            s.extend((ss + start).tolist())
            e.extend((ee + start).tolist())
            left.extend(np.where(ll >= 0, ll + cid, -1).tolist())
            right.extend(np.where(rr >= 0, rr + cid, -1).tolist())
            perm[start:start + len(pp)] = nd[0][pp]
        else:
            s.append(start)
            e.append(start + len(nd[0]))
            left.append(-1)
            right.append(-1)
            if nd[1] is None:                             # a leaf cluster
                perm[start:start + len(nd[0])] = nd[0]
        if parent >= 0:
            (left if side == 0 else right)[parent] = cid
        if nd[1] is not None:
            a, b = nd[1]
            emit(a, start, cid, 0)
            emit(b, start + len(a[0]), cid, 1)

    emit(root, 0, -1, 0)
    return Cluster(X[perm], perm, np.asarray(s, np.int64), np.asarray(e, np.int64),
                   np.asarray(left, np.int64), np.asarray(right, np.int64))


def _bisect_sorted_1d(X, Nleaf):
    """Median bisection of already sorted 1-D points: pure index arithmetic."""
    n = X.shape[0]
    s, e, left, right = [], [], [], []
    stack = [(0, n, -1, 0)]
    while stack:
        a, b, parent, side = stack.pop()
        cid = len(s)
        s.append(a)
        e.append(b)
        left.append(-1)
        right.append(-1)
        if parent >= 0:
            (left if side == 0 else right)[parent] = cid
        if b - a <= Nleaf:
            continue
        h = a + (b - a + 1) // 2
        stack.append((h, b, cid, 1))
        stack.append((a, h, cid, 0))
    perm = np.arange(n, dtype=np.int64)
    return Cluster(X.copy(), perm, np.asarray(s, np.int64), np.asarray(e, np.int64),
                   np.asarray(left, np.int64), np.asarray(right, np.int64))


def neighbor_pairs(c, adj):
    """Neighbour cluster pairs of src/cluster.jl:140-169 for a sparse ``adj``
    in the original ordering (None: identity adjacency, handled on the device
    side by the range-intersection rule)."""
    if adj is None:
        return None
    import scipy.sparse as sp
    A = sp.csr_matrix(adj)[c.P, :][:, c.P].tocoo()
    n = c.N
    # clusters containing each point: walk the pre-order tree
    p2c = [[] for _ in range(n)]
    for cid in range(c.ncluster):
        for i in range(c.s[cid], c.e[cid]):
            p2c[i].append(cid)
    pairs = set()
    for i, j in zip(A.row, A.col):
        for k1 in p2c[i]:
            for k2 in p2c[j]:
                pairs.add((k1, k2))
    return np.asarray(sorted(pairs), np.int64).reshape(-1, 2)
