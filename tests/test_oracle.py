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


# --- bbfmm (deps/src/lowrank.cpp:24-222, src/hlu.jl:20-29,113-132) ---------
# The reference's C++ needs Eigen (absent), so the restatement is pinned by
# the identities Chebyshev interpolation must satisfy.

def test_bbfmm_nodes_and_lagrange_identity():
    from oracle import hm_oracle as O
    for r in (1, 2, 5, 16):
        c = O.chebyshev_points(r, -1.0, 1.0)
        assert np.allclose(c, np.cos(np.pi * (2 * np.arange(r) + 1) / (2 * r)), rtol=0, atol=1e-15)
        c = O.chebyshev_points(r, 3.0, 7.0)
        assert np.all((c > 3.0) & (c < 7.0))
        # L_j(c_i) = delta_ij exactly: a zero factor off the diagonal, x/x on it
        assert np.array_equal(O.lagrange_matrix(c, c), np.eye(r))


def test_bbfmm_reproduces_polynomials():
    # a kernel of degree < r in each coordinate is interpolated exactly
    from oracle import hm_oracle as O
    rng = np.random.default_rng(0)
    f1 = lambda X, Y: (1.0 + X[:, 0][:, None] * Y[:, 0][None, :]) ** 3
    X, Y = np.sort(rng.uniform(0, 1, 70)), np.sort(rng.uniform(2, 3, 50))
    U, V = O.bbfmm(f1, X, Y, 4)
    assert U.shape == (70, 4) and V.shape == (50, 4)
    A = f1(X.reshape(-1, 1), Y.reshape(-1, 1))
    assert np.abs(U @ V.T - A).max() <= 1e-12 * np.abs(A).max()
    f2 = lambda X, Y: (1.0 + X @ Y.T) ** 2
    X2, Y2 = rng.uniform(0, 1, (90, 2)), rng.uniform(2, 3, (80, 2))
    U, V = O.bbfmm(f2, X2, Y2, 3)
    assert U.shape == (90, 9) and V.shape == (80, 9)
    A = f2(X2, Y2)
    assert np.abs(U @ V.T - A).max() <= 1e-12 * np.abs(A).max()


def test_bbfmm_converges_and_rank_rule():
    from oracle import hm_oracle as O
    rng = np.random.default_rng(1)
    f = O.kernel_cauchy()
    X, Y = np.sort(rng.uniform(0, 1, 64)), np.sort(rng.uniform(3, 4, 64))
    A = f(X.reshape(-1, 1), Y.reshape(-1, 1))
    errs = []
    for r in (2, 4, 8, 12):
        U, V = O.bbfmm(f, X, Y, r)
        errs.append(np.abs(U @ V.T - A).max() / np.abs(A).max())
    assert all(errs[i + 1] < errs[i] for i in range(3)) and errs[-1] < 1e-9
    # 2-D: r lowered to floor(sqrt(max(m, n))) when r^2 > max(m, n) (hlu.jl:24-26)
    X2, Y2 = rng.uniform(0, 1, (40, 2)), rng.uniform(3, 4, (30, 2))
    U, V = O.bbfmm(f, X2, Y2, 16)
    assert U.shape == (40, 36) and V.shape == (30, 36)        # floor(sqrt(40)) = 6
    U, V = O.bbfmm(f, X2, Y2, 5)
    assert U.shape == (40, 25)


def test_bbfmm_newhmat_2d_accuracy():
    # test/cluster.jl:9's bar on the bbfmm route (its default ConsMethod) in 2-D
    from oracle import hm_oracle as O
    G = np.random.default_rng(2).uniform(0, 1, (1200, 2))
    prm = O.Params(Geom=G, Kernel=O.kernel_invquad(100.0), MaxBlock=300, MinBlock=32, MaxRank=6,
                   ConsMethod="bbfmm", Tree="bisect")
    c, H = O.NewHmat(prm)
    A = O.FullMat(prm.Kernel, c.X, c.X)
    lv = np.asarray(O.block_list(H))
    assert (lv[:, 0] == 1).any()
    assert np.abs(O.to_fmat(H) - A).max() < 1e-8


# --- coarsening and H + H (src/utils.jl:29-59, src/harithm.jl:4-159,374-420) --

def _readme(O, max_rank, kernel=None):
    prm = O.Params(Geom=np.linspace(0, 10, 2000), Kernel=kernel or O.kernel_cauchy(), MaxBlock=500,
                   MinBlock=64, MaxRank=max_rank, ConsMethod="svd")
    c, H = O.NewHmat(prm)
    return prm, c, H


def test_coarsening_oracle():
    from oracle import hm_oracle as O
    prm, c, H = _readme(O, 5)
    G = O.coarsening(H, prm)
    b0, b1 = np.asarray(O.block_list(H)), np.asarray(O.block_list(G))
    assert np.array_equal(b0[:, 1:5], b1[:, 1:5])                 # same partition
    conv = (b0[:, 0] == 0) & (b1[:, 0] == 1)
    assert conv.sum() > 0 and (b1[conv, 5] <= 5).all()
    diag = (b0[:, 1] == b0[:, 2]) & (b0[:, 3] == b0[:, 4])
    assert not (conv & diag).any()                                # diagonal leaves stay dense
    A = O.FullMat(O.kernel_cauchy(), c.X, c.X)
    assert np.abs(O.to_fmat(G) - A).max() < 1e-8                  # test/cluster.jl:9's bar
    assert O.info(G)[3] < O.info(H)[3] or O.info(G)[3] <= O.info(H)[3]


def test_hadd_oracle():
    from oracle import hm_oracle as O
    # aca2 route: the partition depends on the geometry only, so two kernels share it
    kw = dict(Geom=np.linspace(0, 10, 1500), MaxBlock=300, MinBlock=32, MaxRank=16, ConsMethod="aca2",
              Tree="bisect")
    _, A1 = O.NewHmat(O.Params(Kernel=O.kernel_cauchy(), **kw))
    _, A2 = O.NewHmat(O.Params(Kernel=O.kernel_invquad(3.0), **kw))
    assert np.array_equal(np.asarray(O.block_list(A1))[:, :5], np.asarray(O.block_list(A2))[:, :5])
    prm, c, H1 = _readme(O, 5)
    S = O.hadd(A1, A2, prm)
    D = O.to_fmat(A1) + O.to_fmat(A2)
    assert np.abs(O.to_fmat(S) - D).max() <= 1e-9 * np.abs(D).max()
    H2 = O.scale(0.7, H1)
    S = O.hadd(H1, H2, prm)
    D = O.to_fmat(H1) + O.to_fmat(H2)
    assert np.abs(O.to_fmat(S) - D).max() <= 1e-9 * np.abs(D).max()
    Z = O.hadd(H1, H1, prm, -1.0)
    assert np.abs(O.to_fmat(Z)).max() <= 1e-13
    # mixed formats: a coarsened copy against the original
    G = O.coarsening(H1, prm)
    for a, b in ((H1, G), (G, H1)):
        M = O.hadd(a, b, prm)
        assert np.abs(O.to_fmat(M) - 2 * O.to_fmat(H1)).max() <= 1e-8


def test_c_restatement_matches_python_oracle():
    # the C restatement of the partition, aca2 and hmat_matvec! (the CPU baseline
    # of bench.py) against the Python oracle: same leaves and ranks, same product
    import sys
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "hmatrix.jl_b200"))
    from oracle import hm_oracle as O
    from oracle.hm_oracle_c import Sample
    from hmatrix.cluster import construct_cluster
    n = 4096
    G = np.linspace(0, 10, n)
    c = construct_cluster(G, 64, "bisect")
    S = Sample(1, 1.0, c.X, {"s": c.s, "e": c.e, "left": c.left, "right": c.right}, 64, 512, 16, 1e-8, 0, n)
    _, OH = O.NewHmat(O.Params(Geom=G, Kernel=O.kernel_cauchy(), MaxBlock=512, MinBlock=64, MaxRank=16,
                               ConsMethod="aca2", εComp=1e-8, Tree="bisect"))
    ref = np.asarray(O.block_list(OH), np.int64)
    assert np.array_equal(S.lv, ref[:, :5])
    assert np.array_equal(np.where(S.lv[:, 0] == 1, S.rank, 0), ref[:, 5])
    x = np.random.default_rng(1).standard_normal(n)
    yo = O.matvec(OH, x)
    assert np.linalg.norm(S.matvec(x) - yo) <= 1e-13 * np.linalg.norm(yo)
