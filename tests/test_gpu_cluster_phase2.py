"""GPU parity: phase 2 of the single-column H-matvec by tree clusters
(hm_set_tune(h, 1, waves): one warp per 128-row chunk of an output cluster,
tree level by tree level) against the oracle's H*x and x'*H
(src/harithm.jl:310-337) and against the window shapes, on bisection and
KMeans trees whose cluster boundaries fall anywhere in a row window."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def params(mod, n, tree, **kw):
    kern = mod.Cauchy(1.0) if hasattr(mod, "Cauchy") else mod.kernel_cauchy()
    return mod.Params(Geom=np.linspace(0, 10, n), Kernel=kern, MaxBlock=kw.pop("MaxBlock", 512), MinBlock=64,
                      MaxRank=16, ConsMethod="aca2", εComp=1e-8, Tree=tree, **kw)


@pytest.mark.parametrize("n,tree", [(6000, "kmeans"), (5003, "bisect"), (4096, "bisect")])
def test_cluster_phase2_vs_oracle(n, tree):
    import hmatrix as hm
    from oracle import hm_oracle as O
    c, H = hm.NewHmat(params(hm, n, tree))
    oc, OH = O.NewHmat(params(O, n, tree))
    assert np.array_equal(c.P, oc.P)
    y = np.random.default_rng(7).standard_normal(n)
    H.set_tune(1)
    r = H * y
    ro = O.matvec(OH, y)
    assert np.linalg.norm(r - ro) <= 1e-13 * np.linalg.norm(ro)
    rt = H.matvec(y, trans=True)
    rto = O.vec_mat(y, OH)[0]
    assert np.linalg.norm(rt - rto) <= 1e-13 * np.linalg.norm(rto)
    for waves in (2, 4):                                # phase-1 grid does not change phase 2
        H.set_tune(1, waves)
        assert np.array_equal(H * y, r)
    H.set_tune(4)
    assert np.linalg.norm(H * y - r) <= 1e-14 * np.linalg.norm(r)
    assert np.linalg.norm(H.matvec(y, trans=True) - rt) <= 1e-14 * np.linalg.norm(rt)


@pytest.mark.parametrize("n,tree,maxblock", [(1 << 16, "bisect", 512), (50021, "kmeans", 2048)])
def test_cluster_phase2_large_vs_windows(n, tree, maxblock):
    """Clusters of up to 2048 rows (16 units each) and a deep tree: the same
    sums as the window shapes up to FP64 summation order, H*x and H'*x."""
    import hmatrix as hm
    c, H = hm.NewHmat(params(hm, n, tree, MaxBlock=maxblock))
    X = np.random.default_rng(8).standard_normal(n)     # one column: the single-vector kernels
    H.set_tune(4)
    R4 = H * X
    RT4 = H.matvec(X, trans=True)
    H.set_tune(1)
    R1 = H * X
    RT1 = H.matvec(X, trans=True)
    assert np.linalg.norm(R1 - R4) <= 1e-14 * np.linalg.norm(R4)
    assert np.linalg.norm(RT1 - RT4) <= 1e-14 * np.linalg.norm(RT4)


# FP32 factors: FP32 products and partial sums over 8-32 entries before the
# FP64 sum, as in the window shapes (whose groups differ): both within the
# FP32 bound of the FP64 product
def test_cluster_phase2_f32():
    import hmatrix as hm
    n = 20011
    _, H = hm.NewHmat(params(hm, n, "kmeans", Storage=hm.F32))
    _, H64 = hm.NewHmat(params(hm, n, "kmeans"))
    x = np.random.default_rng(9).standard_normal(n)
    y64 = H64 * x
    yt64 = H64.matvec(x, trans=True)
    H.set_tune(1)
    assert np.linalg.norm(H * x - y64) <= 1e-5 * np.linalg.norm(y64)
    assert np.linalg.norm(H.matvec(x, trans=True) - yt64) <= 1e-5 * np.linalg.norm(yt64)


def test_cluster_phase2_device_pointers():
    import torch
    import hmatrix as hm
    n = 9000
    _, H = hm.NewHmat(params(hm, n, "kmeans"))
    x = np.random.default_rng(10).standard_normal(n)
    H.set_tune(1)
    yh = H * x
    yd = H.matvec(torch.tensor(x, device="cuda", dtype=torch.float64))
    assert np.array_equal(yd.cpu().numpy(), yh)


def test_set_tune_rejects():
    import hmatrix as hm
    n = 3000
    _, H = hm.NewHmat(params(hm, n, "bisect", Storage=hm.BF16))
    with pytest.raises(Exception):
        H.set_tune(1)                                   # BF16 factors: own phase 2
    with pytest.raises(Exception):
        H.set_tune(3)
    with pytest.raises(Exception):
        H.set_tune(4, 3)
    H.set_tune(8, 2)
    assert H.info().tune_p2_split == 8 and H.info().tune_p1_waves == 2
