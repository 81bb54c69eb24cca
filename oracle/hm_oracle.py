"""CPU FP64 oracle for the Hmatrix.jl hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` may import it.
The product path (``hmatrix.jl_b200``) never calls it, and nothing here is
ever the thing that is measured as the GPU result.

It restates, in plain numpy/scipy/sklearn FP64, the reference algorithms of
Hmatrix.jl for the hot path, following the reference files line by line
(paths relative to the Hmatrix.jl project root):

* cluster tree ..................... src/cluster.jl:196-256
* geometric neighbours .............. src/cluster.jl:140-169
* block partition ``__c1`` ......... src/cluster.jl:36-133
* dense kernel blocks ``FullMat`` ... src/cluster.jl:45,258-275
* ``compress`` / ``rank_truncate`` .. src/hlu.jl:144-190
* ``aca2`` (d-D form) ............... src/hlu.jl:59-111
* ``bbfmm`` Chebyshev interpolation . src/hlu.jl:20-29,113-132, deps/src/lowrank.cpp:24-222
* fully pivoted ACA ................. deps/src/ACA_FullyPivoted.cpp:9-236
* H-matvec .......................... src/harithm.jl:317-371
* H-add / recompression ............. src/harithm.jl:4-159,374-420
* ``coarsening`` .................... src/utils.jl:29-59
* H x H product ``hmul`` ............ src/harithm.jl:162-315
* shifts / scaling .................. src/harithm.jl:456-502
* copy / densify / ``info`` ......... src/utils.jl:83-192
* H-LU, triangular solves, ``\\`` ... src/hlu.jl:193-562

Choices the reference leaves open (they are fixed here and stated):

* ``Hparams.Adj`` defaults to ``nothing`` in the reference, which makes
  ``compute_geom_info`` throw (src/cluster.jl:141).  ``adj=None`` here means
  the identity adjacency ``sparse(I,n,n)``: two clusters are neighbours iff
  their index ranges intersect.
* ``aca2`` (d-D) replaces its row pivot by ``rand(findall(Ia))`` from an
  unseeded RNG inside its "patience" loop (src/hlu.jl:72-85).  The oracle
  keeps the deterministic first choice (row 1, then the arg-max of the last
  column), so the same inputs always give the same factors.
* ``compress`` uses LowRankApprox ``psvd`` for square blocks (src/hlu.jl:171);
  numpy's LAPACK SVD stands in for it (same truncation rule).
* The cluster tree uses sklearn ``KMeans(n_clusters=2, random_state=0)``
  (src/cluster.jl:197).  ``n_init=10`` pins the default of the scikit-learn
  releases of the reference's era, and KMeans runs on one thread: with
  several threads its reductions make the pick between mirror-image splits
  of near-equal inertia vary from run to run, so the reference's own tree is
  not reproducible.  A second, deterministic tree
  ("bisect": split at the median of the widest coordinate) is offered for
  large n, where thousands of KMeans calls take minutes.

Parity status: the reference (Julia) cannot run in this environment, so this
restatement is pinned against the reference's own known-answer tests
(test/cluster.jl:9, test/harithm.jl:11,26, test/lu.jl:14,31,49) and the
driver example of ACA_FullyPivoted.cpp:240-255 (see tests/test_oracle.py).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

# ----------------------------------------------------------------------------
# configuration (src/utils.jl:8-26)
# ----------------------------------------------------------------------------


@dataclass
class Params:
    """Mirror of the reference ``Params`` struct (src/utils.jl:8-24)."""
    Geom: Optional[np.ndarray] = None
    Adj: Optional[object] = None          # None == identity adjacency
    εComp: float = 1e-10
    MaxRank: int = 16
    MaxBlock: int = -1
    MinBlock: int = 64
    Kernel: Optional[Callable] = None     # vectorised f(Xrows, Ycols) -> (m, n)
    CompMethod: str = "svd"
    ConsMethod: str = "bbfmm"
    εTrunc: float = 1e-10
    verbose: bool = False
    aca_force: bool = False
    Tree: str = "kmeans"                  # "kmeans" (reference) | "bisect"


# ----------------------------------------------------------------------------
# kernels.  Vectorised numpy forms of the kernels used by the reference tests
# and the benchmark configurations.  Each takes (X (m,d), Y (n,d)) -> (m,n).
# Arithmetic order is the one a device kernel uses, so rational kernels agree
# bit for bit with the GPU.
# ----------------------------------------------------------------------------


def _sqdist(X, Y, scale=None):
    X = np.asarray(X, dtype=np.float64).reshape(len(X), -1)
    Y = np.asarray(Y, dtype=np.float64).reshape(len(Y), -1)
    s = None
    for q in range(X.shape[1]):
        d = X[:, q][:, None] - Y[:, q][None, :]
        if scale is not None:
            d = d / scale
        t = d * d
        s = t if s is None else s + t
    return s


def kernel_cauchy(ell=1.0):
    """k(x,y) = 1/(1 + |x-y|^2/ell^2), as ``(x,y)->1/(1+(x-y)^2)`` (README.md:27)."""
    def f(X, Y):
        s = _sqdist(X, Y, None if ell == 1.0 else ell)
        return 1.0 / (1.0 + s)
    f.hm_kind = ("cauchy", float(ell))
    return f


def kernel_invquad(c):
    """k(x,y) = 1/(c + |x-y|^2), as ``(x,y)->1/(100+sum((x-y).^2))`` (test/cluster.jl:17)."""
    def f(X, Y):
        return 1.0 / (c + _sqdist(X, Y))
    f.hm_kind = ("invquad", float(c))
    return f


def kernel_gauss(ell):
    """k(x,y) = exp(-|x-y|^2 / (2 ell^2))."""
    def f(X, Y):
        return np.exp(-_sqdist(X, Y) / (2.0 * ell * ell))
    f.hm_kind = ("gauss", float(ell))
    return f


def FullMat(f, X, Y):
    """``FullMat``/``kernel_full`` (src/cluster.jl:45,258-275)."""
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    return np.ascontiguousarray(f(X.reshape(len(X), -1), Y.reshape(len(Y), -1)))


# ----------------------------------------------------------------------------
# cluster tree (src/cluster.jl:7-19, 196-256)
# ----------------------------------------------------------------------------


class Cluster:
    __slots__ = ("X", "P", "left", "right", "m", "n", "N", "isleaf", "s", "e", "id")

    def __init__(self, X, P, N, s, e):
        self.X, self.P, self.N, self.s, self.e = X, P, N, s, e
        self.left = self.right = None
        self.m = self.n = 0
        self.isleaf = False
        self.id = 0

    # Base.:(==) (src/cluster.jl:135-137)
    def same(self, other):
        return self.s == other.s and self.e == other.e


def bisect_cluster_kmeans(X):
    """src/cluster.jl:196-205: label 0 -> first child, indices in increasing order."""
    from sklearn.cluster import KMeans
    from threadpoolctl import threadpool_limits
    # one thread: sklearn's multi-threaded Lloyd reductions make the choice
    # between mirror-image splits of near-equal inertia non-deterministic
    with threadpool_limits(limits=1):
        L = KMeans(n_clusters=2, random_state=0, n_init=10).fit(X).labels_
    P1 = np.flatnonzero(L == 0)
    P2 = np.flatnonzero(L == 1)
    return P1, P2


def bisect_cluster_coord(X):
    """Deterministic median split along the widest coordinate.

    The first child receives the ceil(N/2) points of smallest coordinate
    (stable order on ties); both children keep increasing original order, as
    ``findall`` does in src/cluster.jl:200-201.
    """
    N = X.shape[0]
    ext = X.max(axis=0) - X.min(axis=0)
    q = int(np.argmax(ext))
    order = np.argsort(X[:, q], kind="stable")
    h = (N + 1) // 2
    P1 = np.sort(order[:h])
    P2 = np.sort(order[h:])
    return P1, P2


def construct_cluster(X, Nleaf, method="kmeans"):
    """src/cluster.jl:216-256.  Returns (ncluster, root).

    ``s``/``e`` are kept 1-based and inclusive as in the reference; ``P`` is
    0-based (numpy indices).  Ids are assigned in the pre-order of the
    downward pass, as ``__id`` is (src/cluster.jl:223-226).
    """
    X = np.asarray(X, dtype=np.float64)
    if X.ndim == 1:
        X = X.reshape(-1, 1)
    split = bisect_cluster_kmeans if method == "kmeans" else bisect_cluster_coord
    counter = [0]

    root = Cluster(X, np.arange(X.shape[0]), X.shape[0], 1, X.shape[0])
    stack = [root]
    # iterative pre-order (left before right) == the reference recursion
    while stack:
        c = stack.pop()
        counter[0] += 1
        c.id = counter[0]
        if c.N <= Nleaf:
            c.isleaf = True
            continue
        P1, P2 = split(c.X)
        X1, X2 = c.X[P1, :], c.X[P2, :]
        P1, P2 = c.P[P1], c.P[P2]
        c.left = Cluster(X1, P1, len(P1), c.s, c.s + len(P1) - 1)
        c.right = Cluster(X2, P2, len(P2), c.s + len(P1), c.e)
        c.m, c.n = c.left.N, c.right.N
        stack.append(c.right)
        stack.append(c.left)

    # upward pass (src/cluster.jl:242-250)
    _iter_upward(root)
    return counter[0], root


def _iter_upward(root):
    order = []
    stack = [root]
    while stack:
        c = stack.pop()
        order.append(c)
        if not c.isleaf:
            stack.append(c.left)
            stack.append(c.right)
    for c in reversed(order):
        if not c.isleaf:
            c.P = np.concatenate([c.left.P, c.right.P])
            c.X = np.concatenate([c.left.X, c.right.X], axis=0)


def clusters_preorder(root):
    out = []
    stack = [root]
    while stack:
        c = stack.pop()
        out.append(c)
        if not c.isleaf:
            stack.append(c.right)
            stack.append(c.left)
    return out


def cluster_arrays(root):
    """Flatten the tree to 0-based arrays indexed by ``id-1`` (pre-order).

    Returns dict(perm, s, e, left, right) where ``s`` is the 0-based start,
    ``e`` the exclusive end and ``left``/``right`` are child ids-1 or -1.
    """
    cl = clusters_preorder(root)
    nc = len(cl)
    s = np.zeros(nc, np.int64)
    e = np.zeros(nc, np.int64)
    left = -np.ones(nc, np.int64)
    right = -np.ones(nc, np.int64)
    for c in cl:
        i = c.id - 1
        s[i] = c.s - 1
        e[i] = c.e
        if not c.isleaf:
            left[i] = c.left.id - 1
            right[i] = c.right.id - 1
    return dict(perm=root.P.astype(np.int64), s=s, e=e, left=left, right=right)


# ----------------------------------------------------------------------------
# neighbours (src/cluster.jl:140-169)
# ----------------------------------------------------------------------------


def make_neighbors(root, ncluster, adj=None):
    """Return a predicate ``nb(s, t) -> bool`` equal to ``Neighbors[s.id,t.id] != 0``.

    ``adj`` is None (identity adjacency) or a scipy sparse matrix in the
    ORIGINAL ordering; it is permuted by ``c.P`` as src/cluster.jl:141 does.
    """
    if adj is None:
        return lambda s, t: not (s.e < t.s or t.e < s.s)
    import scipy.sparse as sp
    A = sp.csr_matrix(adj)[root.P, :][:, root.P].tocoo()
    n = root.N
    p2c = [[] for _ in range(n)]
    for c in clusters_preorder(root):
        for i in range(c.s - 1, c.e):
            p2c[i].append(c.id)
    pairs = set()
    for i, j in zip(A.row, A.col):
        if A.data is not None:
            pass
        for k1 in p2c[i]:
            for k2 in p2c[j]:
                pairs.add((k1, k2))
    return lambda s, t: (s.id, t.id) in pairs


# ----------------------------------------------------------------------------
# H-matrix type (src/cluster.jl:21-34)
# ----------------------------------------------------------------------------


class Hmat:
    __slots__ = ("A", "B", "C", "P", "is_rk", "is_full", "is_h", "m", "n",
                 "children", "s", "t")

    def __init__(self, m=0, n=0, s=None, t=None):
        self.A = np.zeros((0, 0))
        self.B = np.zeros((0, 0))
        self.C = np.zeros((0, 0))
        self.P = np.zeros(0, np.int64)
        self.is_rk = self.is_full = self.is_h = False
        self.m, self.n = m, n
        self.children = None
        self.s, self.t = s, t

    @property
    def shape(self):
        return (self.m, self.n)


def rkmat(A, B, s, t):
    """src/utils.jl:112-114."""
    H = Hmat(A.shape[0], B.shape[0], s, t)
    H.is_rk = True
    H.A, H.B = A, B
    return H


def fullmat(C, s=None, t=None):
    H = Hmat(C.shape[0], C.shape[1], s, t)
    H.is_full = True
    H.C = C
    return H


# ----------------------------------------------------------------------------
# compression (src/hlu.jl:144-190, 31-111) and fully pivoted ACA
# ----------------------------------------------------------------------------


def rank_truncate(S, εTrunc):
    """src/hlu.jl:144-154."""
    if len(S) == 0:
        return 0
    k = np.flatnonzero(S / S[0] > εTrunc)
    return 0 if len(k) == 0 else int(k[-1]) + 1


def compress(C, prm: Params):
    """src/hlu.jl:159-190 ("svd" method)."""
    C = np.asarray(C, dtype=np.float64)
    if np.sum(np.abs(C)) < 1e-5:
        return np.zeros((C.shape[0], 1)), np.zeros((C.shape[1], 1))
    if prm.CompMethod != "svd":
        raise NotImplementedError(
            "CompMethod %r: the reference's 'aca' and 'rrqr' branches are "
            "broken as shipped (src/hlu.jl:136,181)" % prm.CompMethod)
    U, S, Vt = np.linalg.svd(C, full_matrices=False)
    k = rank_truncate(S, prm.εTrunc)
    assert k > 0
    A = U[:, :k].copy()
    B = (Vt[:k, :].T * S[:k]).copy()
    return A, B


def aca2(f, X, Y, Rrank, εComp):
    """Partially pivoted ACA, d-D form of src/hlu.jl:59-111.

    Up to ``Rrank+1`` terms; stops after the first term r with
    ``|a_r||b_r| / (|a_1||b_1|) <= εComp`` (that term is kept) or on an
    exactly zero pivot (that term is dropped).  Row pivots are deterministic
    (first row, then arg-max of |a_r| over unused rows) where the reference
    draws ``rand(findall(Ia))``.
    """
    X = np.asarray(X, dtype=np.float64).reshape(len(X), -1)
    Y = np.asarray(Y, dtype=np.float64).reshape(len(Y), -1)
    m, n = X.shape[0], Y.shape[0]
    A = np.zeros((m, Rrank + 1))
    B = np.zeros((n, Rrank + 1))
    Ia = np.ones(m, dtype=bool)
    tau = 0
    for r in range(Rrank + 1):
        row = f(X[tau:tau + 1], Y)[0]
        if r > 0:
            row = row - B[:, :r] @ A[tau, :r]
        sigma = int(np.argmax(np.abs(row)))
        delta = row[sigma]
        if delta == 0:
            return A[:, :r].copy(), B[:, :r].copy()
        Ia[tau] = False
        col = f(X, Y[sigma:sigma + 1])[:, 0]
        if r > 0:
            col = col - A[:, :r] @ B[sigma, :r]
        A[:, r] = col / delta
        B[:, r] = row
        free = np.flatnonzero(Ia)
        if len(free) == 0:
            return A[:, :r + 1].copy(), B[:, :r + 1].copy()
        tau = int(free[np.argmax(np.abs(A[free, r]))])
        eps = (np.linalg.norm(A[:, r]) * np.linalg.norm(B[:, r])
               / np.linalg.norm(A[:, 0]) / np.linalg.norm(B[:, 0]))
        if eps <= εComp:
            return A[:, :r + 1].copy(), B[:, :r + 1].copy()
    return A, B


def chebyshev_points(r, a, b):
    """``Chebyshev_points(n, a, b)`` / ``Interpolation`` (deps/src/lowrank.cpp:26-44):
    cos(pi (2i+1) / (2r)) on [-1, 1], mapped as u (b - a) / 2 + (a + b) / 2,
    with libm's cos and the same operation order."""
    u = np.array([math.cos(math.pi * (2.0 * i + 1.0) / (2.0 * r)) for i in range(r)])
    return u * (b - a) / 2.0 + (a + b) / 2.0


def lagrange_matrix(X, cheb):
    """``Interpolation::ComputeMatrix`` (deps/src/lowrank.cpp:48-61):
    P(i, j) = prod_{k != j} (X_i - c_k) / (c_j - c_k), multiplied in k order."""
    X = np.asarray(X, dtype=np.float64)
    r = len(cheb)
    P = np.ones((len(X), r))
    for j in range(r):
        for k in range(r):
            if k != j:
                P[:, j] *= (X - cheb[k]) / (cheb[j] - cheb[k])
    return P


def bbfmm1d(f, X, Y, r):
    """``bbfmm1D`` (deps/src/lowrank.cpp:186-200, src/hlu.jl:113-121):
    U = P_X S (m x r), V = P_Y (n x r), S_ij = f(cX_i, cY_j), nodes on
    [min X, max X] and [min Y, max Y]."""
    X = np.asarray(X, dtype=np.float64).reshape(-1)
    Y = np.asarray(Y, dtype=np.float64).reshape(-1)
    cx = chebyshev_points(r, X.min(), X.max())
    cy = chebyshev_points(r, Y.min(), Y.max())
    S = f(cx.reshape(-1, 1), cy.reshape(-1, 1))
    return lagrange_matrix(X, cx) @ S, lagrange_matrix(Y, cy)


def _interp_2d(X, r):
    """``Interpolation_2d`` (deps/src/lowrank.cpp:100-136): nodes (cx_i, cy_j)
    at row i r + j, and the matrix with column i r + j = Lx_i * Ly_j."""
    cx = chebyshev_points(r, X[:, 0].min(), X[:, 0].max())
    cy = chebyshev_points(r, X[:, 1].min(), X[:, 1].max())
    nodes = np.stack([np.repeat(cx, r), np.tile(cy, r)], axis=1)
    Lx, Ly = lagrange_matrix(X[:, 0], cx), lagrange_matrix(X[:, 1], cy)
    P = (Lx[:, :, None] * Ly[:, None, :]).reshape(len(X), r * r)
    return nodes, P


def bbfmm2d(f, X, Y, r):
    """``bbfmm2D`` / ``Compute_lowrank`` (deps/src/lowrank.cpp:139-222,
    src/hlu.jl:123-132): U = P_X S (m x r^2), V = P_Y (n x r^2),
    S(a, b) = f(node a of X, node b of Y)."""
    X = np.asarray(X, dtype=np.float64).reshape(len(X), 2)
    Y = np.asarray(Y, dtype=np.float64).reshape(len(Y), 2)
    nx, PX = _interp_2d(X, r)
    ny, PY = _interp_2d(Y, r)
    return PX @ f(nx, ny), PY


def bbfmm(f, X, Y, Rrank):
    """``bbfmm`` (src/hlu.jl:20-29).  1-D geometry takes the ``bbfmm1d``
    branch (the reference's n x 1 cluster points reach ``bbfmm2d`` and read
    past the end of X, deps/src/lowrank.cpp:207-208); 2-D lowers Rrank to
    floor(sqrt(max(m, n))) when Rrank^2 exceeds max(m, n)."""
    X = np.asarray(X, dtype=np.float64).reshape(len(X), -1)
    Y = np.asarray(Y, dtype=np.float64).reshape(len(Y), -1)
    if X.shape[1] == 1:
        return bbfmm1d(f, X, Y, Rrank)
    if X.shape[1] != 2:
        raise NotImplementedError("bbfmm2D reads two coordinates (deps/src/lowrank.cpp:203-211)")
    if Rrank ** 2 > max(len(X), len(Y)):
        Rrank = int(math.floor(math.sqrt(max(len(X), len(Y)))))
    return bbfmm2d(f, X, Y, Rrank)


def aca_fully_pivoted(A, epsilon, min_rank=1):
    """deps/src/ACA_FullyPivoted.cpp:9-151 (the ``rank==0`` branch).

    Returns (U, V, rank).  Stops when the Frobenius norm of the residual is
    <= ``epsilon`` (an absolute threshold, line 60) or <= machine epsilon,
    or the rank reaches min(m, n), but never before ``min_rank`` terms.  The
    pivot is the first maximum of each column's |R| (Eigen ``maxCoeff``) and
    then the first column attaining the overall maximum.
    """
    A = np.asarray(A, dtype=np.float64)
    m, n = A.shape
    max_rank = min(m, n)
    R = A.copy()
    Us, Vs = [], []
    rank = 0
    meps = np.finfo(np.float64).eps
    Rnorm = np.linalg.norm(R)
    while (rank < max_rank and Rnorm > epsilon and Rnorm > meps) or rank < min_rank:
        absR = np.abs(R)
        col_idx = np.argmax(absR, axis=0)             # first max per column
        col_max = absR[col_idx, np.arange(n)]
        sel_col = int(np.argmax(col_max))             # first column with the max
        sel_row = int(col_idx[sel_col])
        Max = R[sel_row, sel_col]
        if abs(Max) > meps and not math.isnan(Max):
            u = R[:, sel_col] * (1.0 / Max)
            v = R[sel_row, :].copy()
        else:
            u = np.zeros(m)
            u[rank] = 1.0
            v = np.zeros(n)
        Us.append(u)
        Vs.append(v)
        R = R - np.outer(u, v)
        rank += 1
        Rnorm = np.linalg.norm(R)
        if math.isnan(Rnorm):
            if m < n:
                return np.eye(m), A.T.copy(), m
            return A.copy(), np.eye(n), n
    U = np.array(Us).T.reshape(m, rank)
    V = np.array(Vs).T.reshape(n, rank)
    return U, V, rank


def aca_wrapper(A, epsilon, rank):
    """deps/src/ACA_FullyPivoted.cpp:218-236 and src/hlu.jl:9-18.

    Returns (U, V, R): at most ``rank+1`` columns are copied out and the
    untruncated rank ``R`` is returned, as the C entry point does.
    """
    U, V, r = aca_fully_pivoted(A, epsilon, 1)
    M = min(r, rank + 1)
    return U[:, :M].copy(), V[:, :M].copy(), r


# ----------------------------------------------------------------------------
# construction (src/cluster.jl:36-133)
# ----------------------------------------------------------------------------


def NewHmat(prm: Params):
    """src/cluster.jl:36-43 + ``__c1`` (48-133).  Returns (c, H)."""
    X = np.asarray(prm.Geom, dtype=np.float64)
    if X.ndim == 1:
        X = X.reshape(-1, 1)
    if prm.MaxBlock == -1:
        prm.MaxBlock = X.shape[0] // 4
    ncluster, c = construct_cluster(X, prm.MinBlock, prm.Tree)
    nb = make_neighbors(c, ncluster, prm.Adj)
    return c, build_hmat(c, prm, nb)


def build_hmat(c, prm: Params, nb):
    f = prm.Kernel
    MaxBlock = prm.MaxBlock
    root = Hmat()
    stack = [(root, c, c)]
    while stack:
        H, s, t = stack.pop()
        H.m, H.n, H.s, H.t = s.N, t.N, s, t
        U = V = None
        if (H.m <= prm.MinBlock or H.n <= prm.MinBlock) or s.isleaf or t.isleaf:
            H.is_full = True
        elif H.m > MaxBlock or H.n > MaxBlock:
            H.is_h = True
        elif s.same(t):
            H.is_h = True
        elif prm.ConsMethod == "aca2":
            if not nb(s, t):
                H.is_rk = True
                U, V = aca2(f, s.X, t.X, prm.MaxRank - 1, prm.εComp)
                if prm.aca_force and U.shape[1] > prm.MaxRank:
                    H.is_rk, H.is_h = False, True
            else:
                H.is_h = True
        elif prm.ConsMethod == "bbfmm":
            if not nb(s, t):
                H.is_rk = True
                U, V = bbfmm(f, s.X, t.X, prm.MaxRank)
            else:
                H.is_h = True
        elif prm.ConsMethod == "svd":
            A = FullMat(f, s.X, t.X)
            U, V = compress(A, prm)
            if U.shape[1] <= prm.MaxRank:
                H.is_rk = True
            else:
                H.is_h = True
        else:
            raise NotImplementedError(
                "ConsMethod %r is outside the hot path (separate needs user closures)" % prm.ConsMethod)

        if H.is_full:
            H.C = FullMat(f, s.X, t.X)
        elif H.is_rk:
            H.A, H.B = U, V
        else:
            H.children = [[Hmat(), Hmat()], [Hmat(), Hmat()]]
            stack.append((H.children[1][1], s.right, t.right))
            stack.append((H.children[1][0], s.right, t.left))
            stack.append((H.children[0][1], s.left, t.right))
            stack.append((H.children[0][0], s.left, t.left))
    return root


def leaves(H, r0=0, c0=0):
    """Yield (H_leaf, row0, col0) in the order of the reference recursion."""
    stack = [(H, r0, c0)]
    while stack:
        h, r, c = stack.pop()
        if h.is_h:
            m = h.children[0][0].m
            n = h.children[0][0].n
            stack.append((h.children[1][1], r + m, c + n))
            stack.append((h.children[1][0], r + m, c))
            stack.append((h.children[0][1], r, c + n))
            stack.append((h.children[0][0], r, c))
        else:
            yield h, r, c


def block_list(H):
    """Flattened leaf list: (type, row0, col0, m, n, rank) with type 0 dense, 1 Rk."""
    out = []
    for h, r, c in leaves(H):
        if h.is_full:
            out.append((0, r, c, h.m, h.n, 0))
        else:
            out.append((1, r, c, h.m, h.n, h.A.shape[1]))
    return out


def info(H):
    """src/utils.jl:83-110: (dense count, Rk count, depth, compression ratio)."""
    dmat = rk = 0
    level = 0
    ratio = 0.0
    stack = [(H, 1)]
    while stack:
        h, l = stack.pop()
        if h.is_full:
            dmat += 1
            level = max(level, l)
            ratio += h.m * h.n
        elif h.is_rk:
            rk += 1
            level = max(level, l)
            ratio += h.A.size + h.B.size
        else:
            for row in h.children:
                for ch in row:
                    stack.append((ch, l + 1))
    return dmat, rk, level, ratio / H.m / H.n


# ----------------------------------------------------------------------------
# matvec (src/harithm.jl:317-371, 243-260)
# ----------------------------------------------------------------------------


def hmat_matvec(r, a, v, s):
    """``r += s * a * v`` (src/harithm.jl:340-354); r, v are 1-D or 2-D views."""
    if a.is_full:
        r += s * (a.C @ v)
    elif a.is_rk:
        r += s * (a.A @ (a.B.T @ v))
    else:
        m, n = a.children[0][0].m, a.children[0][0].n
        hmat_matvec(r[:m], a.children[0][0], v[:n], s)
        hmat_matvec(r[:m], a.children[0][1], v[n:], s)
        hmat_matvec(r[m:], a.children[1][0], v[:n], s)
        hmat_matvec(r[m:], a.children[1][1], v[n:], s)


def matvec(a, v):
    """``Base.:*(a::Hmat, v)`` (src/harithm.jl:317-329)."""
    v = np.asarray(v, dtype=np.float64)
    r = np.zeros((a.m,) + v.shape[1:])
    hmat_matvec(r, a, v, 1.0)
    return r


def transpose_hmat_mat_mul(H, V):
    """Hᵀ V (src/harithm.jl:243-260)."""
    if H.is_full:
        return H.C.T @ V
    if H.is_rk:
        return H.B @ (H.A.T @ V)
    h11, h12 = H.children[0]
    h21, h22 = H.children[1]
    V1 = transpose_hmat_mat_mul(h11, V[:h11.m]) + transpose_hmat_mat_mul(h21, V[h11.m:])
    V2 = transpose_hmat_mat_mul(h12, V[:h11.m]) + transpose_hmat_mat_mul(h22, V[h11.m:])
    return np.concatenate([V1, V2], axis=0)


def vec_mat(v, a):
    """``Base.:*(v::Matrix, a::Hmat)`` via ``hmat_matvec2`` (src/harithm.jl:331-371)."""
    v = np.atleast_2d(np.asarray(v, dtype=np.float64))
    return transpose_hmat_mat_mul(a, v.T).T


# ----------------------------------------------------------------------------
# copy / densify (src/utils.jl:130-192)
# ----------------------------------------------------------------------------


def hmat_copy(A):
    H = Hmat(A.m, A.n, A.s, A.t)
    H.P = A.P.copy()
    if A.is_full:
        H.C = A.C.copy()
        H.is_full = True
    elif A.is_rk:
        H.A, H.B = A.A.copy(), A.B.copy()
        H.is_rk = True
    else:
        H.is_h = True
        H.children = [[hmat_copy(A.children[i][j]) for j in range(2)] for i in range(2)]
    return H


def to_fmat(A):
    """Dense copy; for a factorised H the packed L\\U (src/utils.jl:162-192)."""
    M = np.zeros((A.m, A.n))
    for h, r, c in leaves(A):
        if h.is_full:
            M[r:r + h.m, c:c + h.n] = h.C
        else:
            M[r:r + h.m, c:c + h.n] = h.A @ h.B.T
    return M


def getl(A, unitdiag=True):
    """src/hlu.jl:193-199."""
    L = np.tril(A)
    if unitdiag:
        np.fill_diagonal(L, 1.0)
    return L


def getu(A, unitdiag=False):
    """src/hlu.jl:201-207."""
    U = np.triu(A)
    if unitdiag:
        np.fill_diagonal(U, 1.0)
    return U


# ----------------------------------------------------------------------------
# shifts / scaling (src/harithm.jl:456-502)
# ----------------------------------------------------------------------------


def add_identity(A, lam):
    """``λI + H`` (src/harithm.jl:457-473): λ on the diagonal of diagonal leaves."""
    if len(A.P) > 0:
        raise RuntimeError("Hmatrix is frozen after factorization")
    H = hmat_copy(A)

    def helper(h):
        if h.children is None:
            h.C = h.C + lam * np.eye(h.C.shape[0], h.C.shape[1])
        else:
            helper(h.children[0][0])
            helper(h.children[1][1])
    helper(H)
    return H


def scale(u, A):
    """``u * H`` (src/harithm.jl:478-498)."""
    if len(A.P) > 0:
        raise RuntimeError("Hmatrix is frozen after factorization")
    H = hmat_copy(A)
    for h, _, _ in leaves(H):
        if h.is_full:
            h.C = h.C * u
        else:
            h.A = h.A * u
    return H


# ----------------------------------------------------------------------------
# H-add and recompression (src/harithm.jl:4-159, 374-420)
# ----------------------------------------------------------------------------


def _qr(M):
    Q, R = np.linalg.qr(M, mode="reduced")
    return Q, R


def hmat_full_add(a, b, scalar, prm):
    """``a += scalar*b`` with b dense (src/harithm.jl:4-32)."""
    if a.is_full:
        a.C = a.C + scalar * b
    elif a.is_rk:
        C = a.A @ a.B.T + scalar * b
        a.A, a.B = compress(C, prm)
    elif a.is_h:
        m, n = a.children[0][0].m, a.children[0][0].n
        hmat_full_add(a.children[0][0], b[:m, :n], scalar, prm)
        hmat_full_add(a.children[0][1], b[:m, n:], scalar, prm)
        hmat_full_add(a.children[1][0], b[m:, :n], scalar, prm)
        hmat_full_add(a.children[1][1], b[m:, n:], scalar, prm)
    else:
        raise RuntimeError("Should not be here")


def full_hmat_add(A, H):
    """src/harithm.jl:34-47: A + dense(H)."""
    return A + to_fmat(H)


def compress_low_rank(A, B, prm):
    """src/harithm.jl:49-56."""
    QA, RA = _qr(A)
    QB, RB = _qr(B)
    W = RA @ RB.T
    A1, A2 = compress(W, prm)
    return QA @ A1, QB @ A2


def rkmat_hmat_add(A, B, scalar, H, prm):
    """A Bᵀ + scalar*H as a low-rank pair (src/harithm.jl:58-91)."""
    if H.is_full:
        return compress(A @ B.T + scalar * H.C, prm)
    if H.is_rk:
        return _rkmat_add(A, B, scalar * H.A, H.B, prm)
    if H.is_h:
        m, n = H.children[0][0].m, H.children[0][0].n
        A11, B11 = rkmat_hmat_add(A[:m], B[:n], scalar, H.children[0][0], prm)
        A12, B12 = rkmat_hmat_add(A[:m], B[n:], scalar, H.children[0][1], prm)
        A21, B21 = rkmat_hmat_add(A[m:], B[:n], scalar, H.children[1][0], prm)
        A22, B22 = rkmat_hmat_add(A[m:], B[n:], scalar, H.children[1][1], prm)
        z = np.zeros
        A0 = np.block([[A11, A12, z((A11.shape[0], A21.shape[1])), z((A11.shape[0], A22.shape[1]))],
                       [z((A21.shape[0], A11.shape[1])), z((A21.shape[0], A12.shape[1])), A21, A22]])
        B0 = np.block([[B11, z((B11.shape[0], B12.shape[1])), B21, z((B11.shape[0], B22.shape[1]))],
                       [z((B12.shape[0], B11.shape[1])), B12, z((B12.shape[0], B21.shape[1])), B22]])
        return compress_low_rank(A0, B0, prm)
    raise RuntimeError("Invalid")


def _rkmat_add(A1, B1, A2, B2, prm):
    """src/harithm.jl:374-396."""
    if A2.shape[1] == 0:
        return A1, B1
    if A1.shape[1] == 0:
        return A2, B2
    QA, RA = _qr(np.hstack([A1, A2]))
    QB, RB = _qr(np.hstack([B1, B2]))
    W = RA @ RB.T
    U, V = compress(W, prm)
    return QA @ U, QB @ V


def rkmat_add(a, b, scalar, prm):
    """src/harithm.jl:398-420 (a rank-0 ``a`` stays unchanged, as there)."""
    A1, B1, A2, B2 = a.A, a.B, scalar * b.A, b.B
    if A2.shape[1] == 0:
        return
    if A1.shape[1] == 0:
        return
    a.A, a.B = _rkmat_add(A1, B1, A2, B2, prm)


def hmat_add(a, b, scalar, prm):
    """``a += scalar*b``, format of ``a`` preserved (src/harithm.jl:95-151)."""
    if b.is_full:
        hmat_full_add(a, b.C, scalar, prm)
    elif a.is_full and b.is_rk:
        if b.A.size == 0:
            return
        a.C = a.C + scalar * (b.A @ b.B.T)
    elif a.is_full and b.is_h:
        # src/harithm.jl:112 as written: a.C += scalar*(a.C + dense(b)).
        # Unreachable from lu! (a dense target has a leaf row or column
        # cluster, so the product b is never an H-matrix there).
        a.C = a.C + scalar * full_hmat_add(a.C, b)
    elif a.is_rk and b.is_rk:
        rkmat_add(a, b, scalar, prm)
    elif a.is_rk and b.is_h:
        a.A, a.B = rkmat_hmat_add(a.A, a.B, scalar, b, prm)
    elif a.is_h and b.is_rk:
        m, n = a.children[0][0].m, a.children[0][0].n
        C11 = rkmat(b.A[:m], b.B[:n], None, None)
        C21 = rkmat(b.A[m:], b.B[:n], None, None)
        C12 = rkmat(b.A[:m], b.B[n:], None, None)
        C22 = rkmat(b.A[m:], b.B[n:], None, None)
        hmat_add(a.children[0][0], C11, scalar, prm)
        hmat_add(a.children[1][0], C21, scalar, prm)
        hmat_add(a.children[0][1], C12, scalar, prm)
        hmat_add(a.children[1][1], C22, scalar, prm)
    elif a.is_h and b.is_h:
        for i in range(2):
            for j in range(2):
                hmat_add(a.children[i][j], b.children[i][j], scalar, prm)


def hadd(a, b, prm, scalar=1.0):
    """``hadd`` (src/harithm.jl:153-157), and ``a - b`` with scalar = -1."""
    c = hmat_copy(a)
    hmat_add(c, b, scalar, prm)
    return c


def coarsening(H, prm):
    """``coarsening`` (src/utils.jl:29-59): every dense leaf whose row and
    column clusters differ becomes U_k, V_k S_k when its truncated SVD rank
    k = findlast(S/S[1] > εTrunc) is at most MaxRank.  A block with S[1] = 0
    stays dense (the reference divides by it and fails there)."""
    G = hmat_copy(H)

    def helper(h):
        if h.is_full and not h.s.same(h.t):
            U, S, Vt = np.linalg.svd(h.C, full_matrices=False)
            if S[0] == 0:
                return
            k = rank_truncate(S, prm.εTrunc)
            if k <= prm.MaxRank:
                h.A = U[:, :k].copy()
                h.B = (S[:k, None] * Vt[:k, :]).T.copy()
                h.C = None
                h.is_rk, h.is_full = True, False
        elif h.is_h:
            for i in range(2):
                for j in range(2):
                    helper(h.children[i][j])
    helper(G)
    return G


# ----------------------------------------------------------------------------
# H x H product (src/harithm.jl:162-315)
# ----------------------------------------------------------------------------


def full_mat_mul(a, b):
    """dense a times b (src/harithm.jl:164-202)."""
    H = Hmat()
    if b.is_h and not a.s.isleaf and not a.t.isleaf:
        # src/harithm.jl:167-188 passes raw sub-matrices to full_mat_mul,
        # which has no such method; a dense block always has a leaf cluster,
        # so this branch is never taken.
        raise NotImplementedError("unreachable branch of full_mat_mul")
    elif b.is_h:
        H.is_full = True
        H.C = a.C @ to_fmat(b)
    elif b.is_full:
        H.is_full = True
        H.C = a.C @ b.C
    else:
        H.is_rk = True
        H.A = a.C @ b.A
        H.B = b.B
    return H


def mat_full_mul(a, b):
    """a times dense b (src/harithm.jl:204-241)."""
    B = b.C
    H = Hmat()
    if a.is_h and not b.s.isleaf and not b.t.isleaf:
        raise NotImplementedError("unreachable branch of mat_full_mul")
    elif a.is_h:
        H.is_full = True
        H.C = matvec(a, B)
    elif a.is_full:
        H.is_full = True
        H.C = a.C @ B
    else:
        H.is_rk = True
        H.A = a.A
        H.B = B.T @ a.B
    return H


def hmul(a, b, prm):
    """src/harithm.jl:262-314."""
    if a.is_full:
        H = full_mat_mul(a, b)
    elif b.is_full:
        H = mat_full_mul(a, b)
    elif a.is_rk and b.is_rk:
        H = Hmat()
        H.is_rk = True
        H.A = a.A
        H.B = b.B @ (b.A.T @ a.B)
    elif a.is_rk and b.is_h:
        H = Hmat()
        H.is_rk = True
        H.A = a.A
        H.B = transpose_hmat_mat_mul(b, a.B)
    elif a.is_h and b.is_rk:
        H = Hmat()
        H.is_rk = True
        H.A = matvec(a, b.A)
        H.B = b.B
    elif a.is_h and b.is_h:
        H = Hmat()
        H.is_h = True
        m = a.children[0][0].m
        n = b.children[0][0].n
        m1, n1 = a.m - m, b.n - n
        H.children = [[Hmat(m, n), Hmat(m, n1)], [Hmat(m1, n), Hmat(m1, n1)]]
        for i in range(2):
            for j in range(2):
                H1 = hmul(a.children[i][0], b.children[0][j], prm)
                H2 = hmul(a.children[i][1], b.children[1][j], prm)
                H.children[i][j] = hadd(H1, H2, prm)
    else:
        raise RuntimeError("Undefined")
    H.s, H.t, H.m, H.n = a.s, b.t, a.m, b.n
    return H


def hmat_sub_mul(c, a, b, prm):
    """``c -= a*b`` (src/hlu.jl:230-233)."""
    M = hmul(a, b, prm)
    hmat_add(c, M, -1.0, prm)


# ----------------------------------------------------------------------------
# triangular solves, LU, solve (src/hlu.jl:235-562)
# ----------------------------------------------------------------------------


def _trsm_lower(L, B, unit):
    """LAPACK trtrs('L','N',unit) in place: B <- L^{-1} B."""
    import scipy.linalg as sla
    B[...] = sla.solve_triangular(L, B, lower=True, unit_diagonal=unit, check_finite=False)


def _trsm_upper_t(U, B, unit):
    """LAPACK trtrs('U','T',unit) in place: B <- U^{-T} B."""
    import scipy.linalg as sla
    B[...] = sla.solve_triangular(U, B, lower=False, trans="T", unit_diagonal=unit,
                                  check_finite=False)


def _trsv_upper(U, y, unit):
    import scipy.linalg as sla
    y[...] = sla.solve_triangular(U, y, lower=False, unit_diagonal=unit, check_finite=False)


def mat_full_solve(a, b, unitdiag, ul="L"):
    """src/hlu.jl:236-295.  ``b`` is a 2-D array modified in place."""
    if a.is_rk:
        raise RuntimeError("A should not be a low-rank matrix")
    if ul == "L":
        if a.is_full:
            _trsm_lower(a.C, b, unitdiag)
        else:
            a11, a21, a22 = a.children[0][0], a.children[1][0], a.children[1][1]
            n = a11.m
            b1 = b[:n].copy()
            b2 = b[n:].copy()
            mat_full_solve(a11, b1, unitdiag, ul)
            b2 = b2 - matvec(a21, b1)
            mat_full_solve(a22, b2, unitdiag, ul)
            b[:n] = b1
            b[n:] = b2
    else:
        if a.is_full:
            c = np.array(b.T)
            _trsm_upper_t(a.C, c, unitdiag)
            b[...] = c.T
        elif a.is_h:
            a11, a12, a22 = a.children[0][0], a.children[0][1], a.children[1][1]
            n = a11.m
            b1 = b[:, :n].copy()
            b2 = b[:, n:].copy()
            mat_full_solve(a11, b1, unitdiag, ul)
            b2 = b2 - vec_mat(b1, a12)
            mat_full_solve(a22, b2, unitdiag, ul)
            b[:, :n] = b1
            b[:, n:] = b2


def hmat_trisolve(a, b, islower, unitdiag, prm):
    """src/hlu.jl:299-442."""
    if a.is_rk:
        raise RuntimeError("A should not be a low-rank matrix")
    if islower:
        if a.is_full and b.is_full:
            _trsm_lower(a.C, b.C, unitdiag)
        elif a.is_full and b.is_rk:
            if b.A.shape[0] == 0:
                return
            _trsm_lower(a.C, b.A, unitdiag)
        elif a.is_full and b.is_h:
            raise RuntimeError("This is never used")
        elif a.is_h and b.is_h:
            a11, a12 = a.children[0]
            a21, a22 = a.children[1]
            b11, b12 = b.children[0]
            b21, b22 = b.children[1]
            hmat_trisolve(a11, b11, islower, unitdiag, prm)
            hmat_trisolve(a11, b12, islower, unitdiag, prm)
            hmat_sub_mul(b21, a21, b11, prm)
            hmat_sub_mul(b22, a21, b12, prm)
            hmat_trisolve(a22, b21, islower, unitdiag, prm)
            hmat_trisolve(a22, b22, islower, unitdiag, prm)
        elif a.is_h and b.is_full:
            mat_full_solve(a, b.C, unitdiag)
        elif a.is_h and b.is_rk:
            mat_full_solve(a, b.A, unitdiag)
    else:
        if a.is_full and b.is_full:
            c = np.array(b.C.T)
            _trsm_upper_t(a.C, c, unitdiag)
            b.C = c.T.copy()
        elif a.is_full and b.is_rk:
            if b.A.shape[0] == 0:
                return
            _trsm_upper_t(a.C, b.B, unitdiag)
        elif a.is_h and b.is_full:
            mat_full_solve(a, b.C, unitdiag, "U")
        elif a.is_h and b.is_rk:
            bt = np.array(b.B.T)
            mat_full_solve(a, bt, unitdiag, "U")
            b.B = bt.T.copy()
        elif a.is_h and b.is_h:
            a11, a12 = a.children[0]
            a21, a22 = a.children[1]
            b11, b12 = b.children[0]
            b21, b22 = b.children[1]
            hmat_trisolve(a11, b11, islower, unitdiag, prm)
            hmat_trisolve(a11, b21, islower, unitdiag, prm)
            hmat_sub_mul(b12, b11, a12, prm)
            hmat_sub_mul(b22, b21, a12, prm)
            hmat_trisolve(a22, b12, islower, unitdiag, prm)
            hmat_trisolve(a22, b22, islower, unitdiag, prm)
        else:
            raise RuntimeError("Invalid")


def permute_hmat(H, P):
    """src/hlu.jl:446-463."""
    if H.is_full:
        H.C = H.C[P, :]
    elif H.is_rk:
        H.A = H.A[P, :]
    else:
        m = H.children[0][0].m
        P1 = P[:m]
        P2 = P[m:] - m
        permute_hmat(H.children[0][0], P1)
        permute_hmat(H.children[0][1], P1)
        permute_hmat(H.children[1][0], P2)
        permute_hmat(H.children[1][1], P2)


def _getrf(C):
    """LAPACK getrf with partial pivoting: returns (packed L\\U, p) with
    ``C[p] == L @ U`` and ``p`` 0-based (Julia's ``F.p`` minus one)."""
    import scipy.linalg as sla
    lu, piv = sla.lu_factor(C, check_finite=False)
    p = np.arange(C.shape[0])
    for i, j in enumerate(piv):
        p[i], p[j] = p[j], p[i]
    return lu, p


def lu_inplace(H, prm):
    """``lu!`` (src/hlu.jl:465-515).  ``H.P`` is 0-based."""
    if len(H.P) > 0:
        return None
    if H.is_rk:
        raise RuntimeError("H should not be a low-rank matrix")
    if H.is_full:
        H.C, H.P = _getrf(H.C)
    else:
        c = H.children
        lu_inplace(c[0][0], prm)
        permute_hmat(c[0][1], c[0][0].P)
        hmat_trisolve(c[0][0], c[0][1], True, True, prm)
        hmat_trisolve(c[0][0], c[1][0], False, False, prm)
        hmat_sub_mul(c[1][1], c[1][0], c[0][1], prm)
        lu_inplace(c[1][1], prm)
        permute_hmat(c[1][0], c[1][1].P)
        H.P = np.concatenate([c[0][0].P, c[1][1].P + c[0][0].m])
    return H


def lu(H, prm):
    """``lu(H)`` (src/hlu.jl:517-521)."""
    A = hmat_copy(H)
    return lu_inplace(A, prm)


def hmat_solve(a, y, lower):
    """src/hlu.jl:524-549; ``y`` is modified in place."""
    if a.is_rk:
        raise RuntimeError("a cannot be a low-rank matrix")
    if lower:
        if a.is_full:
            _trsm_lower(a.C, y, True)
        elif a.is_h:
            m = a.children[0][0].m
            hmat_solve(a.children[0][0], y[:m], True)
            hmat_matvec(y[m:], a.children[1][0], y[:m], -1.0)
            hmat_solve(a.children[1][1], y[m:], True)
    else:
        if a.is_full:
            _trsv_upper(a.C, y, False)
        elif a.is_h:
            m = a.children[0][0].m
            hmat_solve(a.children[1][1], y[m:], False)
            hmat_matvec(y[:m], a.children[0][1], y[m:], -1.0)
            hmat_solve(a.children[0][0], y[:m], False)


def solve(a, y):
    """``a \\ y`` for a factorised H (src/hlu.jl:553-562)."""
    if len(a.P) == 0:
        raise RuntimeError("a has not been factorized")
    w = np.array(y, dtype=np.float64)[a.P].copy()
    hmat_solve(a, w, True)
    hmat_solve(a, w, False)
    return w
