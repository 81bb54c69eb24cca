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


class Cauchy(Kernel):
    """k(x,y) = 1/(1 + |x-y|^2/ell^2); ``(x,y)->1/(1+(x-y)^2)`` of README.md:27 is Cauchy(1)."""
    kind = _lib.HM_KERNEL_CAUCHY

    def __call__(self, X, Y):
        return 1.0 / (1.0 + self._sq(X, Y, None if self.p == 1.0 else self.p))


class InvQuad(Kernel):
    """k(x,y) = 1/(c + |x-y|^2); ``(x,y)->1/(100+sum((x-y).^2))`` of test/cluster.jl:17 is InvQuad(100)."""
    kind = _lib.HM_KERNEL_INVQUAD

    def __call__(self, X, Y):
        return 1.0 / (self.p + self._sq(X, Y))


class Gauss(Kernel):
    """k(x,y) = exp(-|x-y|^2/(2 ell^2))."""
    kind = _lib.HM_KERNEL_GAUSS

    def __call__(self, X, Y):
        return np.exp(-self._sq(X, Y) / (2.0 * self.p * self.p))
