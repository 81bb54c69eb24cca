"""hmatrix -- host-side mirror of Hmatrix.jl's hot path over libhmatb200.

Same names and meaning as the reference API (README.md:22-44,
src/utils.jl:8-26, src/cluster.jl:36-45, src/harithm.jl:317-329,
src/hlu.jl:465-562)::

    Hparams.Geom = np.linspace(0, 10, 2000)
    Hparams.Kernel = Cauchy(1.0)            # (x,y)->1/(1+(x-y)^2)
    Hparams.MaxBlock, Hparams.MinBlock, Hparams.MaxRank = 500, 64, 5
    c, H = NewHmat()
    A = FullMat(Hparams.Kernel, c.X, c.X)
    H * y ; lu(H) ; H.solve(y)               # H\\y

Vectors live in the cluster-permuted order ``c.X`` exactly as in the
reference.  All arithmetic runs in the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from ._lib import HmError, check, lib
from .cluster import Cluster, construct_cluster, neighbor_pairs
from .kernels import Cauchy, CauchyDP, Gauss, GaussDP, InvQuad, InvQuadDP, Kernel

__all__ = [
    "Hparams", "Params", "NewHmat", "FullMat", "Hmat", "lu", "lu_", "getl", "getu", "info",
    "Cauchy", "InvQuad", "Gauss", "Kernel", "Cluster", "construct_cluster", "HmError",
    "aca_wrapper", "F64", "F32", "BF16", "new_on_cluster", "load", "coarsening", "CauchyDP", "InvQuadDP", "GaussDP",
    "lu_batch", "lu_batch_", "solve_batch", "solve_refined_batch", "matvec_batch", "gmres", "bicgstab", "gmres_ir", "new_like",
]

F64, F32, BF16 = _lib.HM_F64, _lib.HM_F32, _lib.HM_BF16


@dataclass
class Params:
    """``Params`` of src/utils.jl:8-24 (plus the device-side choices)."""
    Geom: Optional[np.ndarray] = None
    Adj: Optional[object] = None          # None: identity adjacency sparse(I,n,n)
    εComp: float = 1e-10
    MaxRank: int = 16
    MaxBlock: int = -1
    MinBlock: int = 64
    Kernel: Optional[Kernel] = None
    CompMethod: str = "svd"
    ConsMethod: str = "aca2"
    εTrunc: float = 1e-10
    verbose: bool = False
    aca_force: bool = False
    Tree: str = "kmeans"                  # "kmeans" (reference) | "bisect"
    Storage: int = F64                    # precision of the stored factors
    Shift: float = 0.0                    # lambda of H + lambda*I applied at construction
    Device: int = 0
    RankCap: int = 0                      # rank capacity during H-LU (0: automatic)
    LuMode: str = "auto"                  # "auto" | "recursive" (lu! as written) | "tiles"
    εTruncLU: float = 0.0                 # truncation inside H-LU (0: εTrunc, as in the reference)
    RowRange: tuple = (0, 0)              # build only rows [lo, hi) (a multi-GPU shard); (0, 0): all
    KeepPivots: bool = False              # aca2: keep the pivots, for new_like


Hparams = Params()


def FullMat(f, X, Y):
    """``FullMat``/``kernel_full`` (src/cluster.jl:45,258-275), evaluated on the host."""
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    return np.ascontiguousarray(f(X.reshape(len(X), -1), Y.reshape(len(Y), -1)))


def _params_struct(prm: Params, dim: int):
    p = _lib.hm_params()
    check(lib().hm_default_params(C.byref(p)))
    if not isinstance(prm.Kernel, Kernel):
        raise HmError(_lib.HM_ERR_ARG, "Hparams.Kernel must be a device kernel (Cauchy/InvQuad/Gauss); "
                      "an arbitrary closure cannot run on the GPU")
    p.dim = dim
    p.kernel = prm.Kernel.kind
    p.kparam = prm.Kernel.p
    p.shift = prm.Shift
    p.eps_comp = prm.εComp
    p.eps_trunc = prm.εTrunc
    p.max_rank = prm.MaxRank
    p.max_block = prm.MaxBlock
    p.min_block = prm.MinBlock
    if prm.ConsMethod == "aca2":
        p.cons_method = _lib.HM_CONS_ACA2
    elif prm.ConsMethod == "svd":
        p.cons_method = _lib.HM_CONS_SVD
    elif prm.ConsMethod == "bbfmm":
        p.cons_method = _lib.HM_CONS_BBFMM
    else:
        raise HmError(_lib.HM_ERR_ARG, "ConsMethod %r is not on the device path (use 'aca2', 'svd' or 'bbfmm')"
                      % prm.ConsMethod)
    if prm.CompMethod != "svd":
        raise HmError(_lib.HM_ERR_ARG, "CompMethod %r: only 'svd' works in the reference" % prm.CompMethod)
    p.aca_force = int(prm.aca_force)
    p.storage = prm.Storage
    p.device = prm.Device
    p.rank_cap = prm.RankCap
    p.lu_mode = {"auto": 0, "recursive": 1, "tiles": 2}[prm.LuMode]
    p.eps_trunc_lu = prm.εTruncLU
    p.row_lo, p.row_hi = int(prm.RowRange[0]), int(prm.RowRange[1])
    p.build_flags = _lib.HM_BUILD_KEEP_PIVOTS if prm.KeepPivots else 0
    return p


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


def _torch_stream():
    """cudaStream_t of torch's current stream; the legacy default stream is
    handle 0 in torch, passed as cudaStreamLegacy (0x1) so that the library
    does not fall back to its own stream."""
    import torch
    s = torch.cuda.current_stream().cuda_stream
    return C.c_void_p(s if s else 1)


class Hmat:
    """Opaque H-matrix living on the GPU (mirror of ``Hmat``, src/cluster.jl:21-34)."""

    __array_ufunc__ = None        # ndarray * H defers to H.__rmul__

    def __init__(self, handle, n, cluster=None):
        self._h = C.c_void_p(handle)
        self.m = self.n = n
        self.c = cluster

    def __del__(self):
        try:
            if self._h and self._h.value:
                lib().hm_destroy(self._h)
                self._h = C.c_void_p(0)
        except Exception:
            pass

    @property
    def shape(self):
        return (self.m, self.n)

    # -- structure -----------------------------------------------------------
    def info(self):
        o = _lib.hm_info_t()
        check(lib().hm_info(self._h, C.byref(o)))
        return o

    def leaves(self):
        cnt = C.c_int64(0)
        check(lib().hm_leaves(self._h, 0, None, C.byref(cnt)))
        out = np.zeros((cnt.value, 6), np.int64)
        check(lib().hm_leaves(self._h, cnt.value, _ptr(out), C.byref(cnt)))
        return out

    def leaf_factors(self, i):
        L = self.leaves()[i]
        A = np.zeros((L[3], L[5]), order="F")
        B = np.zeros((L[4], L[5]), order="F")
        check(lib().hm_leaf_factors(self._h, int(i), _ptr(A), _ptr(B)))
        return A, B

    def to_dense(self):
        """``Array(H)`` (src/utils.jl:192); for a factorised H the packed L\\U."""
        out = np.zeros((self.n, self.n), order="F")
        check(lib().hm_to_dense(self._h, _ptr(out), 0))
        return out

    # -- arithmetic ------------------------------------------------------------
    def matvec(self, x, trans=False):
        """``H*x`` / ``H'*x`` for a vector or an n x k matrix (src/harithm.jl:317-329)."""
        try:
            import torch
            if isinstance(x, torch.Tensor):
                return self._matvec_torch(x, trans)
        except ImportError:
            pass
        x = np.asarray(x, dtype=np.float64)
        X = np.asfortranarray(x.reshape(self.n, -1))
        Y = np.zeros_like(X, order="F")
        check(lib().hm_matvec(self._h, _ptr(X), _ptr(Y), X.shape[1], int(bool(trans)), 0, None))
        return Y.reshape(x.shape)

    def _matvec_torch(self, x, trans):
        import torch
        if not x.is_cuda or x.dtype != torch.float64:
            raise HmError(_lib.HM_ERR_ARG, "torch input must be a CUDA float64 tensor")
        X = x.reshape(self.n, -1).t().contiguous()      # columns contiguous
        Y = torch.empty_like(X)
        check(lib().hm_matvec(self._h, C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()), X.shape[0],
                              int(bool(trans)), _lib.HM_FLAG_DEVICE_PTRS, _torch_stream()))
        return Y.t().reshape(x.shape)

    def __mul__(self, x):
        if isinstance(x, (int, float)):
            return self.scaled(float(x))
        return self.matvec(x)

    __matmul__ = __mul__

    def __rmul__(self, x):
        if isinstance(x, (int, float)):
            return self.scaled(float(x))
        # v*H  (src/harithm.jl:331-337): rows of v times H = (H' v')'
        v = np.atleast_2d(np.asarray(x, dtype=np.float64))
        return self.matvec(v.T, trans=True).T

    def autotune(self, ncols=1, calls=5):
        """Choose the matvec launch shapes on this H-matrix's own data
        (hm_autotune); returns the timing table {name: ms} and the choice."""
        t = np.zeros(15)
        check(lib().hm_autotune(self._h, int(ncols), int(calls), _ptr(t)))
        table = {}
        for a, sp in enumerate((2, 4, 8)):
            for b, wv in enumerate((1, 2, 4)):
                table["split%d_waves%d" % (sp, wv)] = float(t[3 * a + b])
        for b, wv in enumerate((1, 2, 4)):
            if t[12 + b] >= 0:
                table["clusters_waves%d" % wv] = float(t[12 + b])
        for q, nc in enumerate((16, 32, 64)):
            if t[9 + q] >= 0:
                table["tc_nc%d_cols%d" % (nc, ncols)] = float(t[9 + q])
        o = self.info()
        choice = {"p2_split": o.tune_p2_split, "p1_waves": o.tune_p1_waves,
                  "tc_nc": [int(v) for v in o.tune_tc_nc]}
        return table, choice

    def set_tune(self, p2_split, p1_waves=1):
        """Pin the single-column matvec launch shapes (hm_set_tune): p2_split
        2, 4 or 8 CTAs per phase-2 window, or 1 for phase 2 by tree clusters."""
        check(lib().hm_set_tune(self._h, int(p2_split), int(p1_waves)))

    def residual(self, x, b, trans=False):
        """b - H x (b - H' x) summed in twice the FP64 precision (hm_residual):
        the residual of iterative refinement.  numpy arrays or CUDA float64
        tensors (n or n x k)."""
        try:
            import torch
            if isinstance(x, torch.Tensor):
                X = x.reshape(self.n, -1).t().contiguous()
                B = b.reshape(self.n, -1).t().contiguous()
                R = torch.empty_like(X)
                check(lib().hm_residual(self._h, C.c_void_p(X.data_ptr()), C.c_void_p(B.data_ptr()),
                                        C.c_void_p(R.data_ptr()), X.shape[0], int(bool(trans)),
                                        _lib.HM_FLAG_DEVICE_PTRS, _torch_stream()))
                return R.t().reshape(x.shape)
        except ImportError:
            pass
        x = np.asarray(x, dtype=np.float64)
        X = np.asfortranarray(x.reshape(self.n, -1))
        B = np.asfortranarray(np.asarray(b, dtype=np.float64).reshape(self.n, -1))
        R = np.zeros_like(X, order="F")
        check(lib().hm_residual(self._h, _ptr(X), _ptr(B), _ptr(R), X.shape[1], int(bool(trans)), 0, None))
        return R.reshape(x.shape)

    def exact_rows(self, rows, x):
        """Exact FP64 rows of (K + shift I) x: the dense FullMat oracle for sampled rows."""
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(len(rows))
        check(lib().hm_exact_rows(self._h, _ptr(rows), len(rows), _ptr(x), _ptr(y), 0, None))
        return y

    def copy(self):
        out = C.c_void_p()
        check(lib().hm_copy(self._h, C.byref(out)))
        return Hmat(out.value, self.n, self.c)

    def save(self, path):
        """Write the (unfactorised) H-matrix to ``path``; the cluster tree and
        permutation of ``self.c`` go into the file's user block."""
        import io
        blob = b""
        if self.c is not None:
            buf = io.BytesIO()
            np.savez(buf, X=self.c.X, P=self.c.P, s=self.c.s, e=self.c.e, left=self.c.left, right=self.c.right)
            blob = buf.getvalue()
        cb = C.create_string_buffer(blob, len(blob)) if blob else None
        check(lib().hm_save(self._h, os.fsencode(path), C.cast(cb, C.c_void_p) if cb else None, len(blob)))

    def add_identity(self, lam):
        """``lam*I + H`` (src/harithm.jl:457-473), returning a new H."""
        H = self.copy()
        check(lib().hm_add_identity(H._h, float(lam)))
        return H

    def scaled(self, u):
        """``u*H`` (src/harithm.jl:478-498), returning a new H."""
        H = self.copy()
        check(lib().hm_scale(H._h, float(u)))
        return H

    def hadd(self, other, scalar=1.0):
        """``self + scalar*other`` for two H-matrices on the same block
        partition (``hadd``/``hmat_add!``, src/harithm.jl:4-159, 374-420):
        a new H-matrix in the formats of ``self``."""
        out = C.c_void_p()
        check(lib().hm_add(self._h, other._h, float(scalar), C.byref(out)))
        return Hmat(out.value, self.n, self.c)

    def __add__(self, other):
        if isinstance(other, _Identity):
            return self.add_identity(other.lam)
        if isinstance(other, Hmat):
            return self.hadd(other, 1.0)                 # src/harithm.jl:158
        raise TypeError("H + %r is outside the hot path" % type(other))

    __radd__ = __add__

    def __sub__(self, other):
        if isinstance(other, Hmat):
            return self.hadd(other, -1.0)                # src/harithm.jl:159
        if isinstance(other, _Identity):
            return self.add_identity(-other.lam)
        raise TypeError("H - %r is outside the hot path" % type(other))

    def __neg__(self):
        return self.scaled(-1.0)

    # -- LU / solve ------------------------------------------------------------
    def lu_(self):
        """``lu!(H)`` (src/hlu.jl:465-515), in place."""
        check(lib().hm_lu(self._h))
        return self

    @property
    def P(self):
        """Row permutation (0-based) of a factorised H: H[P,:] = L*U."""
        if not self.info().factorized:
            return np.zeros(0, np.int64)
        P = np.zeros(self.n, np.int64)
        check(lib().hm_lu_perm(self._h, _ptr(P)))
        return P

    def solve(self, y, trans=False):
        """``a\\y`` (src/hlu.jl:553-562) for a factorised H; ``trans`` solves with H'."""
        tf = _lib.HM_FLAG_TRANS if trans else 0
        try:
            import torch
            if isinstance(y, torch.Tensor):
                Y = y.reshape(self.n, -1).t().contiguous()
                X = torch.empty_like(Y)
                check(lib().hm_solve(self._h, C.c_void_p(Y.data_ptr()), C.c_void_p(X.data_ptr()), Y.shape[0],
                                     _lib.HM_FLAG_DEVICE_PTRS | tf, _torch_stream()))
                return X.t().reshape(y.shape)
        except ImportError:
            pass
        y = np.asarray(y, dtype=np.float64)
        B = np.asfortranarray(y.reshape(self.n, -1))
        X = np.zeros_like(B, order="F")
        check(lib().hm_solve(self._h, _ptr(B), _ptr(X), B.shape[1], tf, None))
        return X.reshape(y.shape)

    def solve_refined(self, y, tol=1e-10, max_iter=10, trans=False):
        """H\\y with FP64 iterative refinement on the unfactorised H's matvec.
        Returns (x, refinement steps, final max relative residual)."""
        y = np.asarray(y, dtype=np.float64)
        B = np.asfortranarray(y.reshape(self.n, -1))
        X = np.zeros_like(B, order="F")
        it = C.c_int32(0)
        rr = C.c_double(0.0)
        check(lib().hm_solve_refined(self._h, _ptr(B), _ptr(X), B.shape[1], float(tol), int(max_iter),
                                     _lib.HM_FLAG_TRANS if trans else 0, None, C.byref(it), C.byref(rr)))
        return X.reshape(y.shape), it.value, rr.value


class _Identity:
    def __init__(self, lam=1.0):
        self.lam = lam

    def __mul__(self, s):
        return _Identity(self.lam * s)

    __rmul__ = __mul__


I = _Identity(1.0)


def NewHmat(prm: Params = None):
    """``c, H = NewHmat()`` (src/cluster.jl:36-43)."""
    prm = Hparams if prm is None else prm
    if prm.Geom is None:
        raise HmError(_lib.HM_ERR_ARG, "Hparams.Geom is not set")
    X = np.asarray(prm.Geom, dtype=np.float64)
    if X.ndim == 1:
        X = X.reshape(-1, 1)
    n, d = X.shape
    if not np.all(np.isfinite(X)):
        # the library refuses such geometry too; KMeans would fail first here
        raise HmError(_lib.HM_ERR_NONFINITE, "Hparams.Geom holds a non-finite coordinate")
    if prm.MaxBlock == -1:
        prm.MaxBlock = n // 4                          # src/cluster.jl:37-39
    c = construct_cluster(X, prm.MinBlock, prm.Tree)
    return c, new_on_cluster(prm, c)


def new_on_cluster(prm: Params, c: Cluster):
    """The H-matrix of ``prm`` on an existing cluster tree ``c`` (as NewHmat
    after construct_cluster): H-matrices of several kernels on one tree share
    the permutation and the block partition."""
    X = np.asarray(c.X, dtype=np.float64)
    if X.ndim == 1:
        X = X.reshape(-1, 1)
    n, d = X.shape
    if prm.MaxBlock == -1:
        prm.MaxBlock = n // 4                          # src/cluster.jl:37-39
    p = _params_struct(prm, d)
    geom = np.asfortranarray(X)
    nb = neighbor_pairs(c, prm.Adj)
    out = C.c_void_p()
    check(lib().hm_new(C.byref(p), n, _ptr(geom), c.ncluster, _ptr(c.s), _ptr(c.e), _ptr(c.left),
                       _ptr(c.right), 0 if nb is None else len(nb),
                       None if nb is None else _ptr(np.ascontiguousarray(nb)), C.byref(out)))
    return Hmat(out.value, n, c)


def new_like(H: "Hmat", prm: Params):
    """The H-matrix of ``prm`` (a different kernel parameter, kernel or shift)
    on the structure of ``H``: same tree, partition and ranks, every low-rank
    block's cross approximation taken at ``H``'s pivots (``H`` built with
    ``KeepPivots=True``), so that its factors vary smoothly with the kernel
    parameter."""
    X = np.asarray(H.c.X, dtype=np.float64)
    d = 1 if X.ndim == 1 else X.shape[1]
    if prm.MaxBlock == -1:
        prm.MaxBlock = H.n // 4
    p = _params_struct(prm, d)
    p.build_flags = _lib.HM_BUILD_KEEP_PIVOTS
    out = C.c_void_p()
    check(lib().hm_new_like(H._h, C.byref(p), C.byref(out)))
    return Hmat(out.value, H.n, H.c)


def load(path, device=0):
    """An H-matrix written by :meth:`Hmat.save`, rebuilt on ``device``;
    returns (c, H) like :func:`NewHmat`."""
    import io
    from .cluster import Cluster
    p = os.fsencode(path)
    ub = C.c_int64(0)
    check(lib().hm_load_user(p, None, 0, C.byref(ub)))
    c = None
    if ub.value > 0:
        buf = C.create_string_buffer(ub.value)
        check(lib().hm_load_user(p, C.cast(buf, C.c_void_p), ub.value, C.byref(ub)))
        z = np.load(io.BytesIO(buf.raw), allow_pickle=False)
        c = Cluster(z["X"], z["P"], z["s"], z["e"], z["left"], z["right"])
    out = C.c_void_p()
    check(lib().hm_load(p, int(device), C.byref(out)))
    info = _lib.hm_info_t()
    check(lib().hm_info(out, C.byref(info)))
    return c, Hmat(out.value, int(info.n), c)


def coarsening(H: Hmat):
    """``coarsening(H)`` (src/utils.jl:29-59): a copy in which every dense leaf
    off the diagonal with truncated SVD rank <= MaxRank becomes low-rank."""
    out = C.c_void_p()
    check(lib().hm_coarsen(H._h, C.byref(out)))
    return Hmat(out.value, H.n, H.c)


def lu(H: Hmat):
    """``lu(H)`` (src/hlu.jl:517-521): a factorised copy."""
    return H.copy().lu_()


def lu_(H: Hmat):
    return H.lu_()


# -- independent problems in one call (no counterpart in the reference) ------
def _handles(Hs):
    return (C.c_void_p * len(Hs))(*[H._h for H in Hs])


def _batch_check(status, st):
    if status != _lib.HM_OK:
        raise HmError(status, _lib.last_error())


def lu_batch_(Hs, nthreads=0):
    """``lu!`` on every H-matrix of ``Hs`` in one library call; the problems
    run concurrently, each on its own stream."""
    Hs = list(Hs)
    st = np.zeros(len(Hs), np.int32)
    _batch_check(lib().hm_batch_lu(_handles(Hs), len(Hs), int(nthreads), _ptr(st)), st)
    return Hs


def lu_batch(Hs, nthreads=0):
    """``lu`` (factorised copies) of every H-matrix of ``Hs``."""
    return lu_batch_([H.copy() for H in Hs], nthreads)


def _rhs_list(Ls, ys):
    Bs = [np.asfortranarray(np.asarray(y, dtype=np.float64).reshape(L.n, -1)) for L, y in zip(Ls, ys)]
    nc = {B.shape[1] for B in Bs}
    if len(nc) > 1:
        raise HmError(_lib.HM_ERR_ARG, "every problem needs the same number of right-hand sides")
    Xs = [np.zeros_like(B, order="F") for B in Bs]
    pb = (C.c_void_p * len(Bs))(*[B.ctypes.data for B in Bs])
    px = (C.c_void_p * len(Xs))(*[X.ctypes.data for X in Xs])
    return Bs, Xs, pb, px, (nc.pop() if nc else 1)


def solve_batch(Ls, ys, trans=False, nthreads=0):
    """``L\\y`` for every factorised ``L`` of ``Ls`` with its right-hand side."""
    Ls, ys = list(Ls), list(ys)
    if len(Ls) != len(ys):
        raise HmError(_lib.HM_ERR_ARG, "one right-hand side per problem")
    Bs, Xs, pb, px, nc = _rhs_list(Ls, ys)
    st = np.zeros(len(Ls), np.int32)
    _batch_check(lib().hm_batch_solve(_handles(Ls), len(Ls), pb, px, nc,
                                      _lib.HM_FLAG_TRANS if trans else 0, int(nthreads), _ptr(st)), st)
    return [X.reshape(np.shape(y)) for X, y in zip(Xs, ys)]


def solve_refined_batch(Ls, ys, tol=1e-10, max_iter=10, trans=False, nthreads=0):
    """Refined solves of every problem; returns (xs, refinement steps, residuals)."""
    Ls, ys = list(Ls), list(ys)
    if len(Ls) != len(ys):
        raise HmError(_lib.HM_ERR_ARG, "one right-hand side per problem")
    Bs, Xs, pb, px, nc = _rhs_list(Ls, ys)
    st = np.zeros(len(Ls), np.int32)
    it = np.zeros(len(Ls), np.int32)
    rr = np.zeros(len(Ls), np.float64)
    _batch_check(lib().hm_batch_solve_refined(_handles(Ls), len(Ls), pb, px, nc, float(tol), int(max_iter),
                                              _lib.HM_FLAG_TRANS if trans else 0, int(nthreads), _ptr(st),
                                              _ptr(it), _ptr(rr)), st)
    return [X.reshape(np.shape(y)) for X, y in zip(Xs, ys)], it, rr


def matvec_batch(Hs, xs, trans=False, nthreads=0):
    """``H*x`` for every H-matrix of ``Hs`` with its vector."""
    Hs, xs = list(Hs), list(xs)
    if len(Hs) != len(xs):
        raise HmError(_lib.HM_ERR_ARG, "one vector per problem")
    Bs, Ys, pb, py, nc = _rhs_list(Hs, xs)
    st = np.zeros(len(Hs), np.int32)
    _batch_check(lib().hm_batch_matvec(_handles(Hs), len(Hs), pb, py, nc, int(bool(trans)), 0, int(nthreads),
                                       _ptr(st)), st)
    return [Y.reshape(np.shape(x)) for Y, x in zip(Ys, xs)]


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


def info(H: Hmat):
    """``info(H)`` (src/utils.jl:83-110): (dense count, Rk count, depth, compression ratio)."""
    o = H.info()
    return o.n_dense, o.n_rk, o.depth, o.compress_ratio


def aca_wrapper(A, eps, rank):
    """The reference's native ``aca_wrapper`` (deps/src/ACA_FullyPivoted.cpp:218-236)
    called as in src/hlu.jl:9-18: returns (U, V) with min(R, rank+1) columns."""
    A = np.asfortranarray(A, dtype=np.float64)
    m, n = A.shape
    U = np.zeros((m, min(m, n, rank + 1)), order="F")
    V = np.zeros((n, min(m, n, rank + 1)), order="F")
    Uf = np.zeros((m, max(1, min(m, n))), order="F")
    Vf = np.zeros((n, max(1, min(m, n))), order="F")
    pd = C.POINTER(C.c_double)
    R = lib().aca_wrapper(A.ctypes.data_as(pd), Uf.ctypes.data_as(pd), Vf.ctypes.data_as(pd), m, n,
                          float(eps), int(rank))
    if R < 0:
        raise HmError(-R, _lib.last_error())
    M = min(R, rank + 1)
    return Uf[:, :M].copy(), Vf[:, :M].copy(), R


from .krylov import bicgstab, gmres, gmres_ir  # noqa: E402  (src/tools.jl:7-65)
