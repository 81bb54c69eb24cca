"""The 2-D point-cloud configuration at a size the dense FP64 reference handles:
points i.i.d. uniform in [0,1]^2 (seed 5), coordinate bisection, kernel
1/(1+|x-y|^2) + 1e-3 I, MaxBlock 512, MinBlock 64, MaxRank 32, ACA tolerance
1e-9, 8 N(0,1) right-hand sides.  A looser factorisation (truncation 1e-8 inside
the H-LU) refined with the FP64 H-matvec to a relative residual <= 1e-10, and
the transposed (adjoint) solve, against the dense solve.  This smooth kernel on
the unit square makes H + 1e-3 I ill-conditioned (cond ~ 1e6): the refinement
converges only while the factorisation error stays below the smallest
eigenvalue, i.e. for a truncation tolerance well below 1e-3 / |H| ~ 4e-7."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
N = 4096


def test_2d_mixed_lu_refined_and_adjoint_solve():
    import hmatrix as hm
    rng = np.random.default_rng(5)
    G = rng.uniform(0, 1, (N, 2))
    prm = hm.Params(Geom=G, Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64, MaxRank=32, ConsMethod="aca2",
                    εComp=1e-9, Tree="bisect", Shift=1e-3, εTruncLU=1e-8)
    c, H = hm.NewHmat(prm)
    D = hm.FullMat(hm.Cauchy(1.0), c.X, c.X) + 1e-3 * np.eye(N)
    # the H-matrix approximates the dense matrix to the ACA tolerance
    X0 = rng.standard_normal((N, 2))
    assert np.linalg.norm(H * X0 - D @ X0) <= 1e-7 * np.linalg.norm(D @ X0)
    L = hm.lu(H)
    B = rng.standard_normal((N, 8))
    X, it, rr = L.solve_refined(B, tol=1e-10, max_iter=30)
    assert rr <= 1e-10
    # the refined solution solves the H-matrix system; against the dense system
    # it carries the compression error times cond(H)
    Hd = H.to_dense()
    assert np.linalg.norm(Hd @ X - B) <= 1e-9 * np.linalg.norm(B)
    Xt, it2, rr2 = L.solve_refined(B, tol=1e-10, max_iter=30, trans=True)
    assert rr2 <= 1e-10
    assert np.linalg.norm(Hd.T @ Xt - B) <= 1e-9 * np.linalg.norm(B)
    Xd = np.linalg.solve(D, B)
    assert np.linalg.norm(X - Xd) <= 1e-3 * np.linalg.norm(Xd)


def test_2d_gmres_ir_and_adjoint():
    # GMRES-based refinement (compensated residual, GMRES preconditioned by the
    # H-LU for the corrections) to 1e-11, forward and transposed
    import hmatrix as hm
    rng = np.random.default_rng(5)
    G = rng.uniform(0, 1, (N, 2))
    prm = hm.Params(Geom=G, Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64, MaxRank=32, ConsMethod="aca2",
                    εComp=1e-9, Tree="bisect", Shift=1e-3, εTruncLU=1e-6)
    c, H = hm.NewHmat(prm)
    L = hm.lu(H)
    b = rng.standard_normal(N)
    x, it, rr = hm.gmres_ir(H, L, b, tol=1e-11)
    assert rr <= 1e-11
    Hd = H.to_dense()
    assert np.linalg.norm(Hd @ x - b) <= 1e-10 * np.linalg.norm(b)
    xt, it2, rr2 = hm.gmres_ir(H, L, b, tol=1e-11, trans=True)
    assert rr2 <= 1e-11
    assert np.linalg.norm(Hd.T @ xt - b) <= 1e-10 * np.linalg.norm(b)
