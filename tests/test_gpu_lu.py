"""GPU parity: H-LU (lu / lu!) and the triangular H-solve (H\\y) vs the oracle.

Tolerances are the reference's own (test/lu.jl:14,31,49): max|L U - H[P,:]| <
1e-8 and H\\y against the dense solve with isapprox's sqrt(eps).  Pivots are
index work and must equal the oracle's exactly.
"""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
SQRT_EPS = np.sqrt(np.finfo(float).eps)


def golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "readme_case.npz"))


def readme(hm, mr, mode="recursive"):
    return hm.Params(Geom=np.linspace(0, 10, 2000), Kernel=hm.Cauchy(1.0), MaxBlock=500, MinBlock=64,
                     MaxRank=mr, ConsMethod="svd", LuMode=mode)


def close(a, b, rtol):
    return np.linalg.norm(a - b) <= rtol * max(np.linalg.norm(a), np.linalg.norm(b))


def leaf_local(P, leaves):
    """P maps the rows of every diagonal leaf onto themselves (pivoting stays
    inside diagonal leaves, src/hlu.jl:474-476, 510)."""
    if sorted(P.tolist()) != list(range(len(P))):
        return False
    for t, r0, c0, m, n, k in leaves:
        if r0 == c0 and m == n and t == 0:
            seg = P[r0:r0 + m]
            if seg.min() < r0 or seg.max() >= r0 + m:
                return False
    return True


def test_lu_readme_rank25():
    # test/lu.jl:2-15.  The unshifted Cauchy matrix is numerically singular:
    # after the first leaves the Schur complements are rounding noise, so the
    # pivots there are decided by noise and cannot be compared entry by entry
    # with LAPACK's; the reference's own check is L U == H[P,:] with its P.
    import hmatrix as hm
    g = golden()
    c, H = hm.NewHmat(readme(hm, 25))
    L = hm.lu(H)
    P = L.P
    assert leaf_local(P, H.leaves())
    assert leaf_local(g["P_noshift25"], H.leaves())          # the oracle's P has the same structure
    F = L.to_dense()
    D = H.to_dense()
    assert np.abs(hm.getl(F) @ hm.getu(F) - D[P]).max() < 1e-8
    # H itself is untouched by lu(H) (a copy is factorised)
    assert np.array_equal(H.to_dense(), D)


@pytest.mark.parametrize("mr", [5, 25])
def test_solve_readme_shifted(mr):
    # test/lu.jl:17-32: H += 10I, lu!(H), H\y ≈ dense(H)\y
    import hmatrix as hm
    g = golden()
    c, H = hm.NewHmat(readme(hm, mr))
    Hs = H + 10 * hm.I
    dH = Hs.to_dense()
    y = g["y"]
    x1 = np.linalg.solve(dH, y)
    Hs.lu_()
    assert np.array_equal(Hs.P, g["P_shift%d" % mr])
    x2 = Hs.solve(y)
    assert close(x1, x2, SQRT_EPS)
    assert close(x2, g["x_shift%d" % mr], 1e-10)            # the oracle's own H\y


@pytest.mark.parametrize("mr", [5, 25])
def test_lu_packed_factors_vs_oracle(mr):
    # same recursion, same formats, same truncation points: the packed L\U of
    # the well-conditioned H + 10I agrees with the oracle's, pivots exactly
    import hmatrix as hm
    from oracle import hm_oracle as O
    c, H = hm.NewHmat(readme(hm, mr))
    L = hm.lu(H + 10 * hm.I)
    oprm = O.Params(Geom=np.linspace(0, 10, 2000), Kernel=O.kernel_cauchy(), MaxBlock=500, MinBlock=64,
                    MaxRank=mr, ConsMethod="svd")
    oc, OH = O.NewHmat(oprm)
    OL = O.lu(O.add_identity(OH, 10.0), oprm)
    F, Fo = L.to_dense(), O.to_fmat(OL)
    assert np.array_equal(L.P, OL.P)
    assert np.abs(F - Fo).max() <= 1e-9 * np.abs(Fo).max()


def test_transposed_and_refined_solve():
    import hmatrix as hm
    c, H = hm.NewHmat(readme(hm, 5))
    Hs = H + 10 * hm.I
    D = Hs.to_dense()
    L = hm.lu(Hs)
    y = np.random.default_rng(6).standard_normal((2000, 2))
    # the factors are truncated at εTrunc = 1e-10: the direct solves are accurate to ~1e-10
    assert close(L.solve(y, trans=True), np.linalg.solve(D.T, y), 1e-9)
    assert close(L.solve(y), np.linalg.solve(D, y), 1e-9)
    x, it, rr = L.solve_refined(y, tol=1e-14, max_iter=5)
    assert rr <= 1e-14 and 0 <= it <= 5
    assert close(x, np.linalg.solve(D, y), 1e-13)
    xt, it, rr = L.solve_refined(y, tol=1e-14, max_iter=5, trans=True)
    assert rr <= 1e-14
    assert close(xt, np.linalg.solve(D.T, y), 1e-13)


def test_lu2_2d():
    # test/lu.jl:34-50: 2-D 50x50 grid, 1/(100+|x-y|^2), MaxBlock 256, MaxRank 3, +10I
    import hmatrix as hm
    x = np.linspace(0, 10, 50)
    XX, YY = np.meshgrid(x, x)
    G = np.stack([XX.ravel(order="F"), YY.ravel(order="F")], 1)
    prm = hm.Params(Geom=G, Kernel=hm.InvQuad(100.0), MaxBlock=256, MinBlock=64, MaxRank=3, ConsMethod="svd")
    c, H = hm.NewHmat(prm)
    Hs = H + 10 * hm.I
    L = hm.lu(Hs)
    F = L.to_dense()
    assert np.abs(hm.getl(F) @ hm.getu(F) - Hs.to_dense()[L.P]).max() < 1e-8
    y = np.random.default_rng(3).random(2500)
    assert close(L.solve(y), np.linalg.solve(Hs.to_dense(), y), SQRT_EPS)


@pytest.mark.parametrize("mode", ["recursive", "tiles"])
def test_aca2_route_lu_solve_multi_rhs(mode):
    # aca2 construction (Adj = I) with a diagonal shift, several right-hand sides;
    # this partition has a tile level, so both schedules apply
    import hmatrix as hm
    n = 4096
    prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64, MaxRank=16,
                    ConsMethod="aca2", εComp=1e-10, Tree="bisect", Shift=1.0, LuMode=mode)
    c, H = hm.NewHmat(prm)
    D = H.to_dense()
    L = hm.lu(H)
    F = L.to_dense()
    assert leaf_local(L.P, H.leaves())
    assert np.abs(hm.getl(F) @ hm.getu(F) - D[L.P]).max() < 1e-8
    B = np.random.default_rng(4).standard_normal((n, 3))
    X = L.solve(B)
    assert close(X, np.linalg.solve(D, B), 1e-9)
    assert close(L.solve(B, trans=True), np.linalg.solve(D.T, B), 1e-9)
    Xr, it, rr = L.solve_refined(B, tol=1e-13, max_iter=5)
    assert rr <= 1e-13 and close(Xr, np.linalg.solve(D, B), 1e-12)


def test_tiles_match_recursion_kmeans_tree():
    # the tile schedule on a KMeans tree (uneven tiles) against the recursion
    import hmatrix as hm
    n = 6000
    out = {}
    for mode in ("recursive", "tiles"):
        prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64,
                        MaxRank=16, ConsMethod="aca2", εComp=1e-10, Tree="kmeans", Shift=1.0, LuMode=mode)
        c, H = hm.NewHmat(prm)
        L = hm.lu(H)
        y = np.random.default_rng(8).standard_normal(n)
        out[mode] = (L.P, L.solve(y), H.to_dense(), y)
    P1, x1, D, y = out["recursive"]
    P2, x2, _, _ = out["tiles"]
    assert np.array_equal(P1, P2)                  # well conditioned: same pivots
    assert close(x1, x2, 1e-9)
    assert close(x2, np.linalg.solve(D, y), 1e-9)


def test_lu_state_errors():
    import hmatrix as hm
    c, H = hm.NewHmat(readme(hm, 5))
    with pytest.raises(hm.HmError) as e:
        H.solve(np.ones(2000))                           # src/hlu.jl:554-556
    assert "not been factorized" in str(e.value)
    L = hm.lu(H + 10 * hm.I)
    with pytest.raises(hm.HmError) as e:
        L.lu_()                                          # src/hlu.jl:466-468
    assert "already factorized" in str(e.value)
    with pytest.raises(hm.HmError) as e:
        L + 1.0 * hm.I                                   # src/harithm.jl:458-460
    assert "frozen" in str(e.value)
    with pytest.raises(hm.HmError):
        L * np.ones(2000)


def test_lu_copy_of_factorised():
    import hmatrix as hm
    c, H = hm.NewHmat(readme(hm, 5))
    L = hm.lu(H + 10 * hm.I)
    L2 = L.copy()
    y = np.random.default_rng(5).random(2000)
    assert np.array_equal(L.solve(y), L2.solve(y))
    assert np.array_equal(L.P, L2.P)


@pytest.mark.parametrize("mode", ["recursive", "tiles"])
def test_captured_solve_replays(mode):
    # the first solve of each shape (ncols, transposed) runs directly and is
    # captured into a CUDA graph; later solves of that shape replay the graph
    # on fresh right-hand sides.  More than 64 columns run directly every time.
    import hmatrix as hm
    n = 4096
    prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64, MaxRank=16,
                    ConsMethod="aca2", εComp=1e-10, Tree="bisect", Shift=1.0, LuMode=mode)
    c, H = hm.NewHmat(prm)
    D = H.to_dense()
    L = hm.lu(H)
    rng = np.random.default_rng(11)
    for shape in [(n,), (n, 3), (n, 70)]:
        for trans in (False, True):
            A = D.T if trans else D
            ys = [rng.standard_normal(shape) for _ in range(3)]
            xs = [L.solve(y, trans=trans) for y in ys]
            for y, x in zip(ys, xs):
                assert close(x, np.linalg.solve(A, y), 1e-9)
            assert np.array_equal(L.solve(ys[0], trans=trans), xs[0])   # replay == first run
    Xr, it, rr = L.solve_refined(rng.standard_normal((n, 2)), tol=1e-13, max_iter=5)
    assert rr <= 1e-13


@pytest.mark.parametrize("eps_lu", [1e-6, 1e-3])
def test_mixed_fp32_core_refined(eps_lu):
    # the tile schedule's recompressions run in FP32 from a truncation of 1e-6
    # on; refined with the compensated FP64 residual the solve reaches the
    # FP64 path's accuracy, forward and transposed
    import hmatrix as hm
    n = 8192
    base = dict(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=256, MinBlock=32, MaxRank=12,
                ConsMethod="aca2", εComp=1e-10, Tree="bisect", Shift=1.0)
    _, H = hm.NewHmat(hm.Params(**base))
    L64 = hm.lu(H)
    _, Hm = hm.NewHmat(hm.Params(εTruncLU=eps_lu, **base))
    Lm = hm.lu(Hm)
    assert Lm.info().lu_tiles > 0
    y = np.random.default_rng(51).standard_normal(n)
    x64, _, r64 = L64.solve_refined(y, tol=1e-12, max_iter=10)
    for trans in (False, True):
        x, it, rr = Lm.solve_refined(y, tol=1e-12, max_iter=40, trans=trans)
        assert rr <= 1e-12, (trans, it, rr)
        if not trans:
            assert np.linalg.norm(x - x64) <= 1e-10 * np.linalg.norm(x64)
