"""GPU parity: coarsening (src/utils.jl:29-59) and H + H / H - H (hadd,
hmat_add!, src/harithm.jl:4-159, 374-420) through the C ABI, against the
oracle.  Bars: leaf formats and ranks equal to the oracle's; every block
within 1e-12 (relative to the largest entry) of the oracle's result; the
reference's accuracy bar (test/cluster.jl:9) against the dense kernel."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _readme(hm, O, max_rank):
    G = np.linspace(0, 10, 2000)
    c, H = hm.NewHmat(hm.Params(Geom=G, Kernel=hm.Cauchy(1.0), MaxBlock=500, MinBlock=64, MaxRank=max_rank,
                                ConsMethod="svd"))
    prm = O.Params(Geom=G, Kernel=O.kernel_cauchy(), MaxBlock=500, MinBlock=64, MaxRank=max_rank,
                   ConsMethod="svd")
    oc, OH = O.NewHmat(prm)
    assert np.array_equal(c.P, oc.P)
    return c, H, prm, OH


def _match(H, OH, tol=1e-12):
    from oracle import hm_oracle as O
    lv = H.leaves()
    ref = np.asarray(O.block_list(OH), np.int64)
    assert np.array_equal(lv, ref)                       # formats, extents and ranks
    D, R = H.to_dense(), O.to_fmat(OH)
    assert np.abs(D - R).max() <= tol * max(np.abs(R).max(), 1e-300)
    y = np.random.default_rng(4).standard_normal(H.n)
    r = O.matvec(OH, y)
    assert np.linalg.norm(H * y - r) <= 10 * tol * max(np.linalg.norm(r), 1e-300)
    return lv


def test_coarsening_vs_oracle():
    import hmatrix as hm
    from oracle import hm_oracle as O
    c, H, prm, OH = _readme(hm, O, 5)
    Hc = hm.coarsening(H)
    OG = O.coarsening(OH, prm)
    lv = _match(Hc, OG)
    before = H.leaves()
    assert ((before[:, 0] == 0) & (lv[:, 0] == 1)).sum() > 0
    A = O.FullMat(O.kernel_cauchy(), c.X, c.X)
    assert np.abs(Hc.to_dense() - A).max() < 1e-8                  # test/cluster.jl:9
    assert Hc.info().pool_bytes < H.info().pool_bytes
    # H itself is unchanged
    assert np.array_equal(H.leaves(), before)


def test_hadd_same_partition_vs_oracle():
    import hmatrix as hm
    from oracle import hm_oracle as O
    kw = dict(Geom=np.linspace(0, 10, 1500), MaxBlock=300, MinBlock=32, MaxRank=16, ConsMethod="aca2",
              Tree="bisect")
    _, A1 = hm.NewHmat(hm.Params(Kernel=hm.Cauchy(1.0), **kw))
    _, A2 = hm.NewHmat(hm.Params(Kernel=hm.InvQuad(3.0), **kw))
    prm1 = O.Params(Kernel=O.kernel_cauchy(), **kw)
    _, O1 = O.NewHmat(prm1)
    _, O2 = O.NewHmat(O.Params(Kernel=O.kernel_invquad(3.0), **kw))
    _match(A1 + A2, O.hadd(O1, O2, prm1))
    _match(A1 - A2, O.hadd(O1, O2, prm1, -1.0))
    Z = (A1 - A1).to_dense()
    assert np.abs(Z).max() <= 1e-13
    # the operands are unchanged
    _match(A1, O1)


def test_hadd_mixed_formats_vs_oracle():
    import hmatrix as hm
    from oracle import hm_oracle as O
    c, H, prm, OH = _readme(hm, O, 5)
    G, OG = hm.coarsening(H), O.coarsening(OH, prm)
    _match(H + G, O.hadd(OH, OG, prm))          # dense + low-rank, low-rank + low-rank, dense + dense
    _match(G + H, O.hadd(OG, OH, prm))          # low-rank + dense: compress of the sum
    S = H.hadd(H.scaled(0.5), 2.0)              # a + 2 b
    _match(S, O.hadd(OH, O.scale(0.5, OH), prm, 2.0))


def test_hadd_f32_and_refusals():
    import hmatrix as hm
    kw = dict(Geom=np.linspace(0, 10, 2048), MaxBlock=256, MinBlock=32, MaxRank=12, ConsMethod="aca2",
              Tree="bisect")
    _, A = hm.NewHmat(hm.Params(Kernel=hm.Cauchy(1.0), **kw))
    _, B = hm.NewHmat(hm.Params(Kernel=hm.Gauss(0.7), **kw))
    _, A32 = hm.NewHmat(hm.Params(Kernel=hm.Cauchy(1.0), Storage=hm.F32, **kw))
    _, B32 = hm.NewHmat(hm.Params(Kernel=hm.Gauss(0.7), Storage=hm.F32, **kw))
    D = (A + B).to_dense()
    D32 = (A32 + B32).to_dense()
    assert np.abs(D32 - D).max() <= 1e-6 * np.abs(D).max()
    with pytest.raises(hm.HmError) as e:
        A + A32                                                    # storage differs
    assert e.value.code == 8
    _, C = hm.NewHmat(hm.Params(Geom=np.linspace(0, 10, 2048), Kernel=hm.Cauchy(1.0), MaxBlock=512,
                                MinBlock=64, MaxRank=12, ConsMethod="aca2", Tree="bisect"))
    with pytest.raises(hm.HmError) as e:
        A + C                                                      # partition differs
    assert e.value.code == 8
    L = hm.lu(A)
    with pytest.raises(hm.HmError) as e:
        hm.coarsening(L)
    assert e.value.code == 4
