"""``gmres`` and ``bicgstab`` (src/tools.jl:7-65) on the GPU.

The reference wraps scipy's solvers: A (a matrix, an Hmat or a function) is the
operator x -> A*x and M (a matrix, a factorised Hmat or a function) the
preconditioner x -> M\\x.  Here the iteration itself runs on the device: the
vectors are CUDA float64 tensors, A*x is the H-matvec and M\\x the H-solve on the
stored LU, so nothing returns to the host inside the iteration.  Both solvers
use right preconditioning and stop on the true relative residual
|b - A x| <= tol |b|; like the reference they warn when the tolerance is not
reached and return the last iterate (a numpy array for numpy input).
"""
from __future__ import annotations

import warnings

import numpy as np
import torch


def _operator(A, n, precond):
    from . import Hmat
    if A is None:
        return None
    if isinstance(A, Hmat):
        if precond:
            return lambda v: A.solve(v)
        return lambda v: A.matvec(v)
    if isinstance(A, np.ndarray):
        T = torch.as_tensor(np.asarray(A, dtype=np.float64), device="cuda")
        if precond:
            LU, piv = torch.linalg.lu_factor(T)
            return lambda v: torch.linalg.lu_solve(LU, piv, v.reshape(n, 1)).reshape(n)
        return lambda v: T @ v
    if callable(A):
        def f(v):
            out = A(v)
            if not isinstance(out, torch.Tensor):
                out = A(v.cpu().numpy())
            return torch.as_tensor(np.asarray(out) if not isinstance(out, torch.Tensor) else out,
                                   dtype=torch.float64, device="cuda").reshape(n)
        return f
    raise TypeError("A and M must be a matrix, an Hmat or a function")


def _setup(A, b, x0, M):
    host = not isinstance(b, torch.Tensor)
    bt = torch.as_tensor(np.asarray(b, dtype=np.float64) if host else b, dtype=torch.float64, device="cuda")
    n = bt.numel()
    bt = bt.reshape(n)
    x = torch.zeros_like(bt) if x0 is None else torch.as_tensor(
        np.asarray(x0, dtype=np.float64) if host else x0, dtype=torch.float64, device="cuda").reshape(n).clone()
    Aop = _operator(A, n, False)
    Mop = _operator(M, n, True) or (lambda v: v)
    return host, bt, x, Aop, Mop, n


def _finish(x, host, converged, what):
    if not converged:
        warnings.warn("%s: convergence to tolerance not achieved" % what)
    return x.cpu().numpy() if host else x


def gmres(A, b, x0=None, *, tol=1e-05, restart=None, maxiter=None, M=None, callback=None):
    """Restarted GMRES (restart = 20 by default, as scipy's) with modified
    Gram-Schmidt; ``callback(residual_norm_ratio)`` after every inner step."""
    host, b, x, Aop, Mop, n = _setup(A, b, x0, M)
    m = min(restart or 20, n)
    maxiter = maxiter or 10 * n
    bnorm = float(torch.linalg.norm(b)) or 1.0
    V = torch.empty((m + 1, n), dtype=torch.float64, device="cuda")
    Z = torch.empty((m, n), dtype=torch.float64, device="cuda")
    it = 0
    r = b - Aop(x)
    beta = float(torch.linalg.norm(r))
    converged = beta <= tol * bnorm
    while not converged and it < maxiter:
        V[0] = r / beta
        Hh = np.zeros((m + 1, m))
        g = np.zeros(m + 1)
        g[0] = beta
        cs, sn = np.zeros(m), np.zeros(m)
        j_end = 0
        for j in range(m):
            Z[j] = Mop(V[j])
            w = Aop(Z[j])
            for i in range(j + 1):
                hij = float(torch.dot(w, V[i]))
                Hh[i, j] = hij
                w = w - hij * V[i]
            Hh[j + 1, j] = float(torch.linalg.norm(w))
            if Hh[j + 1, j] > 0:
                V[j + 1] = w / Hh[j + 1, j]
            for i in range(j):                       # apply the previous rotations
                t = cs[i] * Hh[i, j] + sn[i] * Hh[i + 1, j]
                Hh[i + 1, j] = -sn[i] * Hh[i, j] + cs[i] * Hh[i + 1, j]
                Hh[i, j] = t
            d = np.hypot(Hh[j, j], Hh[j + 1, j])
            cs[j], sn[j] = (Hh[j, j] / d, Hh[j + 1, j] / d) if d > 0 else (1.0, 0.0)
            Hh[j, j] = cs[j] * Hh[j, j] + sn[j] * Hh[j + 1, j]
            Hh[j + 1, j] = 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            it += 1
            j_end = j + 1
            if callback is not None:
                callback(abs(g[j + 1]) / bnorm)
            if abs(g[j + 1]) <= tol * bnorm or it >= maxiter:
                break
        y = np.linalg.solve(np.triu(Hh[:j_end, :j_end]), g[:j_end])
        x = x + torch.as_tensor(y, device="cuda") @ Z[:j_end]
        r = b - Aop(x)
        beta = float(torch.linalg.norm(r))
        converged = beta <= tol * bnorm
        if beta == 0:
            break
    return _finish(x, host, converged, "gmres")


def bicgstab(A, b, x0=None, *, tol=1e-05, maxiter=None, M=None, callback=None):
    """Right-preconditioned BiCGSTAB; ``callback(x)`` after every iteration."""
    host, b, x, Aop, Mop, n = _setup(A, b, x0, M)
    maxiter = maxiter or 10 * n
    bnorm = float(torch.linalg.norm(b)) or 1.0
    r = b - Aop(x)
    rhat = r.clone()
    rho_old = alpha = omega = 1.0
    v = torch.zeros_like(b)
    p = torch.zeros_like(b)
    converged = float(torch.linalg.norm(r)) <= tol * bnorm
    it = 0
    while not converged and it < maxiter:
        rho = float(torch.dot(rhat, r))
        if rho == 0.0:
            warnings.warn("bicgstab: breakdown")
            break
        beta = (rho / rho_old) * (alpha / omega) if it > 0 else 0.0
        p = r + beta * (p - omega * v) if it > 0 else r.clone()
        ph = Mop(p)
        v = Aop(ph)
        alpha = rho / float(torch.dot(rhat, v))
        s = r - alpha * v
        if float(torch.linalg.norm(s)) <= tol * bnorm:
            x = x + alpha * ph
            converged = True
            it += 1
            break
        sh = Mop(s)
        t = Aop(sh)
        tt = float(torch.dot(t, t))
        omega = float(torch.dot(t, s)) / tt if tt > 0 else 0.0
        x = x + alpha * ph + omega * sh
        r = s - omega * t
        rho_old = rho
        it += 1
        if callback is not None:
            callback(x)
        converged = float(torch.linalg.norm(r)) <= tol * bnorm
        if omega == 0.0:
            break
    if converged:
        converged = float(torch.linalg.norm(b - Aop(x))) <= 10 * tol * bnorm
    return _finish(x, host, converged, "bicgstab")


def gmres_ir(H, L, b, *, tol=1e-10, inner_tol=1e-4, restart=30, max_outer=20, trans=False):
    """H \\ b (H' \\ b with ``trans``) to a relative residual ``tol`` by
    GMRES-based iterative refinement (Carson & Higham, "A new analysis of
    iterative refinement and its application to accurate solution of
    ill-conditioned sparse linear systems", 2017): the residual b - H x comes
    from the compensated H-matvec (twice the FP64 precision, ``H.residual``),
    and each correction solves H d = r by GMRES preconditioned with the H-LU
    ``L`` to ``inner_tol``.  Stationary refinement contracts by the LU's error
    times cond(H) a step and stalls when that nears 1; GMRES-IR does not.
    Returns (x, outer steps, relative residual); vectors as in :func:`gmres`."""
    host = not isinstance(b, torch.Tensor)
    bt = torch.as_tensor(np.asarray(b, dtype=np.float64) if host else b, dtype=torch.float64,
                         device="cuda").reshape(-1)
    n = bt.numel()
    Aop = (lambda v: H.matvec(v, trans=True)) if trans else (lambda v: H.matvec(v))
    Mop = (lambda v: L.solve(v, trans=True)) if trans else (lambda v: L.solve(v))
    bnorm = float(torch.linalg.norm(bt)) or 1.0
    x = Mop(bt)
    it, rel = 0, float("inf")
    for it in range(max_outer + 1):
        r = H.residual(x, bt, trans=trans)
        rel = float(torch.linalg.norm(r)) / bnorm
        if rel <= tol or it == max_outer:
            break
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            d = gmres(Aop, r, M=Mop, tol=inner_tol, restart=restart, maxiter=10 * restart)
        x = x + d
    if rel > tol:
        warnings.warn("gmres_ir: convergence to tolerance not achieved")
    return (x.cpu().numpy() if host else x), it, rel
