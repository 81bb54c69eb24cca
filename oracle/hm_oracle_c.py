"""ctypes loader of the C oracle (oracle/hm_oracle_c.c).

TEST INFRASTRUCTURE ONLY: used by tests/ and by the CPU legs of bench.py.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "build", "liborc.so")
_lib = None

KIND = {"cauchy": 1, "invquad": 2, "gauss": 3}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            import subprocess
            subprocess.run(["make", "-C", _HERE], check=True)
        L = C.CDLL(LIB)
        vp, i64, dbl, i32 = C.c_void_p, C.c_int64, C.c_double, C.c_int
        L.orc_partition.argtypes = [vp, vp, vp, vp, i64, i64, i64, i64, i64, vp]
        L.orc_partition.restype = i64
        L.orc_aca2.argtypes = [i32, i32, dbl, vp, i64, i64, i64, i32, i32, i32, dbl, vp, vp]
        L.orc_aca2.restype = i32
        L.orc_build.argtypes = [i32, i32, dbl, vp, i64, i64, i64, vp, i32, dbl, vp, vp, vp]
        L.orc_build.restype = None
        L.orc_matvec.argtypes = [i64, i64, vp, vp, vp, vp, vp, vp, i64, i64]
        L.orc_matvec.restype = None
        L.orc_kernel_value.argtypes = [i32, i32, dbl, vp, i64, i64, i64]
        L.orc_kernel_value.restype = dbl
        _lib = L
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _ranges(n, parts):
    parts = max(1, min(parts, n))
    b = np.linspace(0, n, parts + 1).astype(np.int64)
    return [(int(b[i]), int(b[i + 1])) for i in range(parts)]


def _threads(nthreads):
    if nthreads and nthreads > 0:
        return nthreads
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


class Sample:
    """Leaves of an aca2-route H-matrix (identity adjacency) restricted to the
    rows [rlo, rhi), with FP64 factors built by the C restatement of aca2."""

    def __init__(self, kind, p, geom, tree, min_block, max_block, max_rank, eps_comp, rlo, rhi,
                 nthreads=0):
        from concurrent.futures import ThreadPoolExecutor
        L = lib()
        self.geom = np.asfortranarray(np.asarray(geom, dtype=np.float64).reshape(len(geom), -1))
        self.ng, self.dim = self.geom.shape
        s, e, l, r = (np.ascontiguousarray(tree[k], np.int64) for k in ("s", "e", "left", "right"))
        cnt = L.orc_partition(_p(s), _p(e), _p(l), _p(r), min_block, max_block, rlo, rhi, 0,
                              C.c_void_p(0))
        self.lv = np.zeros((cnt, 5), np.int64)
        L.orc_partition(_p(s), _p(e), _p(l), _p(r), min_block, max_block, rlo, rhi, cnt, _p(self.lv))
        self.rlo, self.rhi = rlo, rhi
        self.kind, self.p, self.R, self.eps = kind, p, max_rank, eps_comp
        self.rank = np.zeros(cnt, np.int32)
        self.threads = _threads(nthreads)
        dummy = np.zeros(1, np.int64)
        rg = _ranges(cnt, self.threads * 8)
        with ThreadPoolExecutor(self.threads) as ex:
            list(ex.map(lambda ab: L.orc_build(kind, self.dim, p, _p(self.geom), self.ng, ab[0], ab[1],
                                               _p(self.lv), max_rank, eps_comp, _p(self.rank), _p(dummy),
                                               C.c_void_p(0)), rg))
        sizes = np.where(self.lv[:, 0] == 0, self.lv[:, 3] * self.lv[:, 4],
                         self.rank * (self.lv[:, 3] + self.lv[:, 4]))
        self.off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        self.pool = np.zeros(int(sizes.sum()) + 1)
        with ThreadPoolExecutor(self.threads) as ex:
            list(ex.map(lambda ab: L.orc_build(kind, self.dim, p, _p(self.geom), self.ng, ab[0], ab[1],
                                               _p(self.lv), max_rank, eps_comp, _p(self.rank), _p(self.off),
                                               _p(self.pool)), rg))
        self.stored = int(sizes.sum())
        self.dense_entries = int(sizes[self.lv[:, 0] == 0].sum())
        self.rk_entries = int(sizes[self.lv[:, 0] == 1].sum())
        self._rg = _ranges(cnt, self.threads)
        self._ybufs = [np.zeros(rhi - rlo) for _ in self._rg]
        self._ex = ThreadPoolExecutor(self.threads)

    def matvec(self, x):
        """y[rlo:rhi] of H x, leaves split over the threads, partial sums added."""
        L = lib()
        x = np.ascontiguousarray(x, np.float64)

        def run(t):
            a, b = self._rg[t]
            yb = self._ybufs[t]
            yb[:] = 0.0
            L.orc_matvec(a, b, _p(self.lv), _p(self.rank), _p(self.off), _p(self.pool), _p(x), _p(yb),
                         self.rlo, self.rhi)

        list(self._ex.map(run, range(len(self._rg))))
        y = self._ybufs[0].copy()
        for yb in self._ybufs[1:]:
            y += yb
        return y

    def bytes_per_matvec(self):
        """Algorithmic bytes: every stored FP64 value once, plus x segments and y."""
        return 8 * self.stored + 8 * 2 * (self.rhi - self.rlo)
