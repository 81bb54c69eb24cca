"""Kernel descriptions for ``Hparams.Kernel``.

The reference takes an arbitrary Julia closure ``(x,y)->Float64``
(src/utils.jl:16).  A closure cannot run on the device, so the kernels of the
reference tests and the benchmark configurations are described by an id and a
parameter; each object is also callable on the host (vectorised numpy) so that
``FullMat`` keeps working as in src/cluster.jl:45.
"""
from __future__ import annotations

import numpy as np

from . import _lib


class Kernel:
    kind = 0

    def __init__(self, p=1.0):
        self.p = float(p)

    def _sq(self, X, Y, scale=None):
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

    def __repr__(self):
        return "%s(%g)" % (type(self).__name__, self.p)

    def dp(self):
        """The derivative kernel dk/dp (same parameter p), for hyper-parameter
        gradients; an H-matrix built with it compresses dk/dp itself."""
        raise NotImplementedError("%s has no derivative kernel" % type(self).__name__)


class Cauchy(Kernel):
    """k(x,y) = 1/(1 + |x-y|^2/ell^2); ``(x,y)->1/(1+(x-y)^2)`` of README.md:27 is Cauchy(1)."""
    kind = _lib.HM_KERNEL_CAUCHY

    def __call__(self, X, Y):
        return 1.0 / (1.0 + self._sq(X, Y, None if self.p == 1.0 else self.p))

    def dp(self):
        return CauchyDP(self.p)


class InvQuad(Kernel):
    """k(x,y) = 1/(c + |x-y|^2); ``(x,y)->1/(100+sum((x-y).^2))`` of test/cluster.jl:17 is InvQuad(100)."""
    kind = _lib.HM_KERNEL_INVQUAD

    def __call__(self, X, Y):
        return 1.0 / (self.p + self._sq(X, Y))

    def dp(self):
        return InvQuadDP(self.p)


class Gauss(Kernel):
    """k(x,y) = exp(-|x-y|^2/(2 ell^2))."""
    kind = _lib.HM_KERNEL_GAUSS

    def __call__(self, X, Y):
        return np.exp(-self._sq(X, Y) / (2.0 * self.p * self.p))

    def dp(self):
        return GaussDP(self.p)


class CauchyDP(Kernel):
    """d/d ell of Cauchy(ell): 2 s/ell / (1 + s)^2 with s = |x-y|^2/ell^2."""
    kind = _lib.HM_KERNEL_CAUCHY_DP

    def __call__(self, X, Y):
        s = self._sq(X, Y, self.p)
        return 2.0 * s / self.p / ((1.0 + s) * (1.0 + s))


class InvQuadDP(Kernel):
    """d/dc of InvQuad(c): -1/(c + |x-y|^2)^2."""
    kind = _lib.HM_KERNEL_INVQUAD_DP

    def __call__(self, X, Y):
        t = self.p + self._sq(X, Y)
        return -1.0 / (t * t)


class GaussDP(Kernel):
    """d/d ell of Gauss(ell): exp(-|x-y|^2/(2 ell^2)) |x-y|^2 / ell^3."""
    kind = _lib.HM_KERNEL_GAUSS_DP

    def __call__(self, X, Y):
        s = self._sq(X, Y)
        return np.exp(-s / (2.0 * self.p * self.p)) * s / self.p ** 3
