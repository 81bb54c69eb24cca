"""GPU checks of gmres / bicgstab (src/tools.jl:7-65) with the H-matvec as the
operator and the H-LU solve as the preconditioner, against the dense solve and
against scipy's solvers, which the reference calls, on the same operators."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
N = 4096


def build(hm, epslu=0.0):
    prm = hm.Params(Geom=np.linspace(0, 10, N), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64, MaxRank=16,
                    ConsMethod="aca2", εComp=1e-10, Tree="bisect", Shift=1.0, εTruncLU=epslu)
    return hm.NewHmat(prm)


@pytest.mark.parametrize("solver", ["gmres", "bicgstab"])
def test_krylov_with_hlu_preconditioner(solver):
    import hmatrix as hm
    c, H = build(hm)
    _, Hp = build(hm, epslu=1e-3)              # a cheap, loose factorisation as preconditioner
    M = hm.lu(Hp)
    D = H.to_dense()
    b = np.random.default_rng(9).standard_normal(N)
    xd = np.linalg.solve(D, b)
    f = getattr(hm, solver)
    its = []
    x = f(H, b, tol=1e-12, M=M, callback=lambda *a: its.append(1))
    assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)
    assert len(its) <= 10                      # the H-LU preconditioner leaves a few iterations
    x2 = f(H, b, tol=1e-10)                    # unpreconditioned (shifted, well conditioned)
    assert np.linalg.norm(x2 - xd) <= 1e-7 * np.linalg.norm(xd)


def test_krylov_operator_forms_and_scipy():
    import scipy.sparse.linalg as ssl
    import hmatrix as hm
    c, H = build(hm)
    D = H.to_dense()
    b = np.random.default_rng(10).standard_normal(N)
    xd = np.linalg.solve(D, b)
    # dense matrix, function, Hmat: the same solution
    for A in (D, lambda v: H * v, H):
        x = hm.gmres(A, b, tol=1e-11, restart=30)
        assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
    # the reference's route: scipy with LinearOperators over H*x and M\x
    M = hm.lu(H)
    lo = ssl.LinearOperator((N, N), matvec=lambda v: H * v)
    mo = ssl.LinearOperator((N, N), matvec=lambda v: M.solve(v))
    xs, info = ssl.gmres(lo, b, rtol=1e-11, M=mo)
    assert info == 0
    xg = hm.gmres(H, b, tol=1e-11, M=M)
    assert np.linalg.norm(xg - xs) <= 1e-8 * np.linalg.norm(xs)


def test_krylov_warns_when_not_converged():
    import hmatrix as hm
    c, H = build(hm)
    b = np.random.default_rng(11).standard_normal(N)
    with pytest.warns(UserWarning, match="convergence"):
        hm.bicgstab(H, b, tol=1e-14, maxiter=1)
