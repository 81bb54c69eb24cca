"""The oracle against the reference's own known-answer tests (CPU only).

The reference ships no golden vectors; its tests pin the path with these
checks (test/cluster.jl:9, test/harithm.jl:11,26, test/lu.jl:14,31,49) and
ACA_FullyPivoted.cpp:240-255 prints A - U V' for a 20x20 Hilbert matrix.
"""
import numpy as np
import pytest

from oracle import hm_oracle as O

SQRT_EPS = np.sqrt(np.finfo(float).eps)


def readme(max_rank, cons="svd"):
    return O.Params(Geom=np.linspace(0, 10, 2000), Kernel=O.kernel_cauchy(), MaxBlock=500,
                    MinBlock=64, MaxRank=max_rank, ConsMethod=cons)


@pytest.fixture(scope="module")
def h25():
    prm = readme(25)
    c, H = O.NewHmat(prm)
    return prm, c, H


def test_newhmat_known_answer(h25):
    # test/cluster.jl:1-10
    prm, c, H = h25
    A = O.FullMat(prm.Kernel, c.X, c.X)
    assert np.abs(A - O.to_fmat(H)).max() < 1e-8


def test_matmul_known_answer():
    # test/harithm.jl:1-12 (isapprox with rtol sqrt(eps))
    prm = readme(5)
    c, H = O.NewHmat(prm)
    A = O.FullMat(prm.Kernel, c.X, c.X)
    y = np.random.default_rng(0).random(2000)
    r = O.matvec(H, y)
    assert np.linalg.norm(A @ y - r) <= SQRT_EPS * max(np.linalg.norm(A @ y), np.linalg.norm(r))


def test_lu_known_answer(h25):
    # test/lu.jl:2-15
    prm, c, H = h25
    L = O.lu(H, prm)
    F = O.to_fmat(L)
    assert sorted(L.P.tolist()) == list(range(2000))
    assert np.abs(O.getl(F) @ O.getu(F) - O.to_fmat(H)[L.P]).max() < 1e-8


def test_solve_known_answer(h25):
    # test/lu.jl:17-32
    prm, c, H = h25
    Hs = O.add_identity(H, 10.0)
    y = np.random.default_rng(1).random(2000)
    x1 = np.linalg.solve(O.to_fmat(Hs), y)
    Ls = O.lu_inplace(O.hmat_copy(Hs), prm)
    x2 = O.solve(Ls, y)
    assert np.linalg.norm(x1 - x2) <= SQRT_EPS * max(np.linalg.norm(x1), np.linalg.norm(x2))


def test_lu2_and_matmul2_known_answer():
    # test/lu.jl:34-50 and test/harithm.jl:14-27 (2-D, 50x50 grid, MaxRank 3)
    x = np.linspace(0, 10, 50)
    XX, YY = np.meshgrid(x, x)
    G = np.stack([XX.ravel(order="F"), YY.ravel(order="F")], 1)
    prm = O.Params(Geom=G, Kernel=O.kernel_invquad(100.0), MaxBlock=500, MinBlock=64, MaxRank=3,
                   ConsMethod="svd")
    c, H = O.NewHmat(prm)
    A = O.FullMat(prm.Kernel, c.X, c.X)
    y = np.random.default_rng(2).random(2500)
    assert np.linalg.norm(A @ y - O.matvec(H, y)) <= SQRT_EPS * np.linalg.norm(A @ y)
    prm.MaxBlock = 256
    c, H = O.NewHmat(prm)
    Hs = O.add_identity(H, 10.0)
    L = O.lu(Hs, prm)
    F = O.to_fmat(L)
    assert np.abs(O.getl(F) @ O.getu(F) - O.to_fmat(Hs)[L.P]).max() < 1e-8


def test_aca_fully_pivoted_driver():
    # ACA_FullyPivoted.cpp:240-255: Hilbert 20x20, eps 1e-3 (absolute Frobenius stop)
    i = np.arange(20)
    A = 1.0 / (i[:, None] + i[None, :] + 1)
    U, V, r = O.aca_fully_pivoted(A, 1e-3, 1)
    assert np.linalg.norm(A - U @ V.T) <= 1e-3
    assert 1 <= r < 20
    U2, V2, r2 = O.aca_wrapper(A, 1e-3, 2)
    assert r2 == r and U2.shape[1] == min(r, 3)


def test_aca2_lu_jl_case():
    # test/lu.jl:79-84 (computed, not asserted there): two separated groups
    X = np.concatenate([np.linspace(0, 1, 100), np.linspace(5, 6, 100)])
    U, V = O.aca2(O.kernel_cauchy(), X, X, 20, 1e-10)
    A = O.FullMat(O.kernel_cauchy(), X, X)
    assert np.abs(A - U @ V.T).max() < 1e-4


def test_aca2_route_accuracy():
    # aca2 construction (ConsMethod="aca2", Adj = I) reaches the aca tolerance
    prm = O.Params(Geom=np.linspace(0, 10, 4096), Kernel=O.kernel_cauchy(), MaxBlock=512,
                   MinBlock=64, MaxRank=16, ConsMethod="aca2", εComp=1e-8, Tree="bisect")
    c, H = O.NewHmat(prm)
    A = O.FullMat(prm.Kernel, c.X, c.X)
    assert np.abs(A - O.to_fmat(H)).max() < 1e-7


def test_golden_fixtures_match_oracle():
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "readme_case.npz")
    g = np.load(path)
    prm = readme(5)
    c, H = O.NewHmat(prm)
    assert np.array_equal(c.P, g["perm"])
    assert np.array_equal(np.asarray(O.block_list(H), np.int64), g["blocks5"])
    y = g["y"]
    assert np.allclose(O.matvec(H, y), g["Hy5"], rtol=1e-13, atol=0)
