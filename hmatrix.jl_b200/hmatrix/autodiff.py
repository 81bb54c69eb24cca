"""Reverse-mode derivatives of H*y and H\\y for torch autograd.

The reference has no derivatives.  This module gives the adjoints the H-matrix
path needs for gradient-based use (a Gaussian-process likelihood, a kernel
hyper-parameter fit): for H(theta) = K_p + sigma2*I on a fixed cluster tree,

* d(H y)     : grad_y = H' g,            grad_p = g'(dK/dp) y,     grad_sigma2 = g'y
* d(H \\ y)  : w = H' \\ g, grad_y = w,  grad_p = -w'(dK/dp) x,    grad_sigma2 = -w'x

with the transposed H-matvec, the transposed triangular H-solve on the stored LU,
and an H-matrix of the derivative kernel dK/dp compressed from the kernel itself
(not stored alongside H).  Vectors are CUDA float64 tensors (n or n x c, in the
cluster-permuted order c.X); p and sigma2 are CPU float64 scalars with
requires_grad.  The forward values use the H-matrices built for the current
(p, sigma2): after changing them, build a new KernelOperator.
"""
from __future__ import annotations

import dataclasses

import torch

from . import Params, NewHmat, new_like, new_on_cluster, lu


class KernelOperator:
    """H = K_p + sigma2 I (``prm.Kernel`` = K_p, ``prm.Shift`` = sigma2) with its
    LU and the H-matrix of dK/dp, both built on first use."""

    def __init__(self, prm: Params, cluster=None, refine_tol: float = 0.0, like=None):
        """like: another KernelOperator built with ``prm.KeepPivots``; H is then
        built on its structure and pivots (``new_like``), so that losses at
        nearby kernel parameters differ smoothly (finite-difference checks)."""
        self.prm = prm
        if like is not None:
            self.c, self.H = like.c, new_like(like.H, prm)
        elif cluster is None:
            self.c, self.H = NewHmat(prm)
        else:
            self.c, self.H = cluster, new_on_cluster(prm, cluster)
        self.p = torch.tensor(float(prm.Kernel.p), dtype=torch.float64, requires_grad=True)
        self.sigma2 = torch.tensor(float(prm.Shift), dtype=torch.float64, requires_grad=True)
        self.refine_tol = refine_tol          # > 0: solves refined to this relative residual
        self._dH = None
        self._L = None

    @property
    def dH(self):
        if self._dH is None:
            dprm = dataclasses.replace(self.prm, Kernel=self.prm.Kernel.dp(), Shift=0.0)
            self._dH = new_on_cluster(dprm, self.c)
        return self._dH

    @property
    def L(self):
        if self._L is None:
            self._L = lu(self.H)
        return self._L

    def _solve(self, y, trans=False):
        if self.refine_tol > 0:
            x, _, _ = self.L.solve_refined(y.detach().cpu().numpy(), tol=self.refine_tol, trans=trans)
            return torch.as_tensor(x, device=y.device)
        return self.L.solve(y.contiguous(), trans=trans)

    def matvec(self, y):
        """H y, differentiable in y, p and sigma2."""
        return _MatVec.apply(y, self.p, self.sigma2, self)

    def solve(self, y):
        """H \\ y, differentiable in y, p and sigma2."""
        return _Solve.apply(y, self.p, self.sigma2, self)


def _dot(a, b):
    return torch.sum(a * b).detach().cpu()


class _MatVec(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y, p, sigma2, op):
        ctx.op = op
        ctx.save_for_backward(y)
        return op.H.matvec(y.detach().contiguous())

    @staticmethod
    def backward(ctx, g):
        (y,) = ctx.saved_tensors
        op = ctx.op
        g = g.contiguous()
        gy = op.H.matvec(g, trans=True) if ctx.needs_input_grad[0] else None
        gp = _dot(g, op.dH.matvec(y.detach().contiguous())) if ctx.needs_input_grad[1] else None
        gs = _dot(g, y.detach()) if ctx.needs_input_grad[2] else None
        return gy, gp, gs, None


class _Solve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y, p, sigma2, op):
        ctx.op = op
        x = op._solve(y.detach())
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        op = ctx.op
        w = op._solve(g.contiguous(), trans=True)
        gp = -_dot(w, op.dH.matvec(x.contiguous())) if ctx.needs_input_grad[1] else None
        gs = -_dot(w, x) if ctx.needs_input_grad[2] else None
        return (w if ctx.needs_input_grad[0] else None), gp, gs, None
