"""GPU parity: Chebyshev-interpolation construction ("bbfmm", the reference's
default ConsMethod: src/cluster.jl:68-75, src/hlu.jl:20-29,113-132,
deps/src/lowrank.cpp:24-222) against the oracle, through the C ABI.

Bars: partition and per-leaf ranks equal; the V factors (interpolation
matrices of the column points) bit-exact; the U = P_X S factors within 1e-13
of the oracle's (an FP64 product in another summation order); the H-matvec
within 1e-13; the whole matrix within the interpolation error of the kernel."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _compare(H, c, OH, oc, nleaf=60):
    from oracle import hm_oracle as O
    assert np.array_equal(c.P, oc.P)
    ref = np.asarray(O.block_list(OH), np.int64)
    lv = H.leaves()
    assert np.array_equal(lv[:, :5], ref[:, :5])
    assert np.array_equal(lv[:, 5], ref[:, 5])
    olv = {(rr, cc): h for h, rr, cc in O.leaves(OH)}
    rk = np.flatnonzero(lv[:, 0] == 1)
    assert len(rk) > 0
    for i in rk[:: max(1, len(rk) // nleaf)]:
        A, B = H.leaf_factors(i)
        oh = olv[(lv[i, 1], lv[i, 2])]
        assert np.array_equal(B, oh.B)                                   # V = P_Y
        assert np.abs(A - oh.A).max() <= 1e-13 * np.abs(oh.A).max()      # U = P_X S
    y = np.random.default_rng(3).standard_normal(H.n)
    r = H * y
    ro = O.matvec(OH, y)
    assert np.linalg.norm(r - ro) <= 1e-13 * np.linalg.norm(ro)
    rt = H.matvec(y, trans=True)
    assert np.linalg.norm(rt - O.vec_mat(y, OH)[0]) <= 1e-13 * np.linalg.norm(rt)
    return lv


def test_bbfmm_1d_vs_oracle():
    import hmatrix as hm
    from oracle import hm_oracle as O
    n = 4096
    G = np.linspace(0, 10, n)
    c, H = hm.NewHmat(hm.Params(Geom=G, Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64, MaxRank=10,
                                ConsMethod="bbfmm", Tree="bisect"))
    oc, OH = O.NewHmat(O.Params(Geom=G, Kernel=O.kernel_cauchy(), MaxBlock=512, MinBlock=64, MaxRank=10,
                                ConsMethod="bbfmm", Tree="bisect"))
    lv = _compare(H, c, OH, oc)
    assert set(lv[lv[:, 0] == 1, 5]) == {10}
    A = O.FullMat(O.kernel_cauchy(), oc.X, oc.X)
    assert np.abs(H.to_dense() - A).max() < 1e-5          # 10 Chebyshev nodes


@pytest.mark.parametrize("max_rank,max_block,n", [(6, 300, 1500), (16, 128, 1500), (16, 400, 3000)])
def test_bbfmm_2d_vs_oracle(max_rank, max_block, n):
    import hmatrix as hm
    from oracle import hm_oracle as O
    G = np.random.default_rng(2).uniform(0, 1, (n, 2))
    c, H = hm.NewHmat(hm.Params(Geom=G, Kernel=hm.InvQuad(100.0), MaxBlock=max_block, MinBlock=32,
                                MaxRank=max_rank, ConsMethod="bbfmm", Tree="bisect"))
    oc, OH = O.NewHmat(O.Params(Geom=G, Kernel=O.kernel_invquad(100.0), MaxBlock=max_block, MinBlock=32,
                                MaxRank=max_rank, ConsMethod="bbfmm", Tree="bisect"))
    lv = _compare(H, c, OH, oc)
    ranks = set(lv[lv[:, 0] == 1, 5])
    if max_rank == 6:
        assert ranks == {36}
    elif max_block == 128:                  # r lowered to floor(sqrt(max(m, n))) < 16
        assert max(ranks) < 256 and all(int(round(np.sqrt(k))) ** 2 == k for k in ranks)
    else:                                   # the reference's default MaxRank: rank 256 leaves
        assert 256 in ranks
    A = O.FullMat(O.kernel_invquad(100.0), oc.X, oc.X)
    assert np.abs(H.to_dense() - A).max() < 1e-8


def test_bbfmm_reduced_storage_and_lu():
    import hmatrix as hm
    G = np.random.default_rng(4).uniform(0, 1, (2000, 2))
    kw = dict(Geom=G, Kernel=hm.Cauchy(0.5), MaxBlock=256, MinBlock=32, MaxRank=5, ConsMethod="bbfmm",
              Tree="bisect", Shift=1.0)
    c, H = hm.NewHmat(hm.Params(**kw))
    _, H32 = hm.NewHmat(hm.Params(Storage=hm.F32, **kw))
    y = np.random.default_rng(5).standard_normal(2000)
    r64, r32 = H * y, H32 * y
    assert np.linalg.norm(r32 - r64) <= 1e-6 * np.linalg.norm(r64)
    # lu! and the refined solve on the interpolated factors (rank 25 leaves)
    L = hm.lu(H)
    x, it, rr = L.solve_refined(y, tol=1e-10, max_iter=20)
    assert rr <= 1e-10
    assert np.linalg.norm(H.to_dense() @ x - y) <= 1e-9 * np.linalg.norm(y)


def test_bbfmm_refuses_3d():
    import hmatrix as hm
    G = np.random.default_rng(6).uniform(0, 1, (500, 3))
    with pytest.raises(hm.HmError):
        hm.NewHmat(hm.Params(Geom=G, Kernel=hm.Cauchy(1.0), MaxBlock=128, MinBlock=32, MaxRank=4,
                             ConsMethod="bbfmm", Tree="bisect"))
