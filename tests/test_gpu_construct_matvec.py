"""GPU parity: construction (partition + compression) and H-matvec vs the oracle."""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SQRT_EPS = np.sqrt(np.finfo(float).eps)


def golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "readme_case.npz"))


def readme_params(hm, max_rank, storage=None, cons="svd"):
    return hm.Params(Geom=np.linspace(0, 10, 2000), Kernel=hm.Cauchy(1.0), MaxBlock=500, MinBlock=64,
                     MaxRank=max_rank, ConsMethod=cons, Storage=hm.F64 if storage is None else storage)


@pytest.mark.parametrize("mr", [5, 25])
def test_readme_svd_structure_and_accuracy(mr):
    import hmatrix as hm
    g = golden()
    c, H = hm.NewHmat(readme_params(hm, mr))
    assert np.array_equal(c.P, g["perm"])
    leaves = H.leaves()
    ref = g["blocks%d" % mr]
    # partition (type, row0, col0, m, n) is index work: bit-exact
    assert np.array_equal(leaves[:, :5], ref[:, :5])
    # SVD ranks: the same truncation rule on the same blocks
    assert np.array_equal(leaves[:, 5], ref[:, 5])
    A = hm.FullMat(hm.Cauchy(1.0), c.X, c.X)
    D = H.to_dense()
    assert np.abs(A - D).max() < 1e-8                       # test/cluster.jl:9


def test_readme_matvec_vs_oracle():
    import hmatrix as hm
    g = golden()
    c, H = hm.NewHmat(readme_params(hm, 5))
    y = g["y"]
    r = H * y
    assert np.linalg.norm(r - g["Hy5"]) <= 1e-13 * np.linalg.norm(g["Hy5"])
    A = hm.FullMat(hm.Cauchy(1.0), c.X, c.X)
    assert np.linalg.norm(A @ y - r) <= SQRT_EPS * np.linalg.norm(A @ y)   # test/harithm.jl:11
    rt = H.matvec(y, trans=True)
    assert np.linalg.norm(rt - g["HTy5"]) <= 1e-13 * np.linalg.norm(g["HTy5"])
    # v*H (src/harithm.jl:331-337)
    vh = y[None, :] * H
    assert np.allclose(vh[0], rt, rtol=1e-14, atol=0)


def test_dense_leaves_bitexact():
    """Rational kernels: dense leaves equal the oracle's kernel_full bit for bit."""
    import hmatrix as hm
    from oracle import hm_oracle as O
    c, H = hm.NewHmat(readme_params(hm, 5))
    D = H.to_dense()
    A = O.FullMat(O.kernel_cauchy(), c.X, c.X)
    for t, r0, c0, m, n, k in H.leaves():
        if t == 0:
            assert np.array_equal(D[r0:r0 + m, c0:c0 + n], A[r0:r0 + m, c0:c0 + n])


@pytest.mark.parametrize("n,tree", [(4096, "bisect"), (6000, "kmeans")])
def test_aca2_vs_oracle(n, tree):
    import hmatrix as hm
    from oracle import hm_oracle as O
    prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64,
                    MaxRank=16, ConsMethod="aca2", εComp=1e-8, Tree=tree)
    c, H = hm.NewHmat(prm)
    oprm = O.Params(Geom=np.linspace(0, 10, n), Kernel=O.kernel_cauchy(), MaxBlock=512, MinBlock=64,
                    MaxRank=16, ConsMethod="aca2", εComp=1e-8, Tree=tree)
    oc, OH = O.NewHmat(oprm)
    assert np.array_equal(c.P, oc.P)
    ref = np.asarray(O.block_list(OH), np.int64)
    lv = H.leaves()
    assert np.array_equal(lv[:, :5], ref[:, :5])
    assert np.array_equal(lv[:, 5], ref[:, 5])               # same ACA ranks
    # factors: A B' equal the oracle's within FP64 round-off of the ACA
    for i in np.flatnonzero(lv[:, 0] == 1)[:40]:
        A, B = H.leaf_factors(i)
        t, r0, c0, m, nn, k = lv[i]
        oh = [h for h, rr, cc in O.leaves(OH) if rr == r0 and cc == c0][0]
        M1, M2 = A @ B.T, oh.A @ oh.B.T
        assert np.abs(M1 - M2).max() <= 1e-12 * np.abs(M2).max()
    y = np.random.default_rng(3).standard_normal(n)
    r = H * y
    ro = O.matvec(OH, y)
    assert np.linalg.norm(r - ro) <= 1e-13 * np.linalg.norm(ro)
    rt = H.matvec(y, trans=True)
    assert np.linalg.norm(rt - O.vec_mat(y, OH)[0]) <= 1e-13 * np.linalg.norm(rt)
    A = O.FullMat(O.kernel_cauchy(), oc.X, oc.X)
    assert np.abs(A - H.to_dense()).max() < 1e-7


# FP32 factors are multiplied and summed in FP32 over a few terms before the
# FP64 sum: with random x the row sums cancel (|H x| is about 20 times below
# |H| |x| here), so the relative error is about 20 x 2^-24 per partial sum
@pytest.mark.parametrize("storage,tol", [("F32", 1e-5), ("BF16", 2e-2)])
def test_reduced_storage_matvec(storage, tol):
    import hmatrix as hm
    n = 8192
    prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64,
                    MaxRank=16, ConsMethod="aca2", εComp=1e-8, Tree="bisect",
                    Storage=getattr(hm, storage))
    c, H = hm.NewHmat(prm)
    prm64 = hm.Params(**{**prm.__dict__, "Storage": hm.F64})
    _, H64 = hm.NewHmat(prm64)
    X = np.random.default_rng(4).standard_normal((n, 3))
    R = H * X
    R64 = H64 * X
    assert np.linalg.norm(R - R64) <= tol * np.linalg.norm(R64)
    rows = np.random.default_rng(5).choice(n, 256, replace=False)
    ex = H64.exact_rows(rows, X[:, 0])
    assert np.linalg.norm(ex - R64[rows, 0]) <= 1e-7 * np.linalg.norm(ex)


def test_exact_rows_vs_numpy():
    import hmatrix as hm
    from oracle import hm_oracle as O
    n = 3000
    prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64,
                    MaxRank=16, ConsMethod="aca2", εComp=1e-8, Tree="bisect", Shift=0.5)
    c, H = hm.NewHmat(prm)
    x = np.random.default_rng(6).standard_normal(n)
    rows = np.arange(0, n, 7)
    A = O.FullMat(O.kernel_cauchy(), c.X, c.X) + 0.5 * np.eye(n)
    assert np.allclose(H.exact_rows(rows, x), A[rows] @ x, rtol=1e-13, atol=1e-12)
    assert np.linalg.norm(H * x - A @ x) <= 1e-7 * np.linalg.norm(A @ x)


def test_shift_scale_copy():
    import hmatrix as hm
    from oracle import hm_oracle as O
    c, H = hm.NewHmat(readme_params(hm, 5))
    D = H.to_dense()
    H2 = H + 10 * hm.I
    assert np.allclose(H2.to_dense(), D + 10 * np.eye(2000), rtol=0, atol=1e-15)
    assert np.array_equal(H.to_dense(), D)                 # H unchanged (copy)
    H3 = 2.5 * H
    assert np.allclose(H3.to_dense(), 2.5 * D, rtol=1e-15, atol=1e-15)
    y = np.random.default_rng(7).random(2000)
    assert np.allclose((-H) * y, -(H * y), rtol=1e-15, atol=0)


def test_torch_device_pointers():
    import torch
    import hmatrix as hm
    c, H = hm.NewHmat(readme_params(hm, 5))
    y = np.random.default_rng(8).random(2000)
    yt = torch.tensor(y, device="cuda", dtype=torch.float64)
    r = H.matvec(yt).cpu().numpy()
    assert np.allclose(r, H * y, rtol=0, atol=0)


def test_aca_wrapper_dropin():
    import hmatrix as hm
    from oracle import hm_oracle as O
    i = np.arange(20)
    A = 1.0 / (i[:, None] + i[None, :] + 1)
    U, V, R = hm.aca_wrapper(A, 1e-3, 5)
    Uo, Vo, Ro = O.aca_wrapper(A, 1e-3, 5)
    assert R == Ro and U.shape == Uo.shape
    assert np.allclose(U, Uo, rtol=1e-12, atol=1e-14) and np.allclose(V, Vo, rtol=1e-12, atol=1e-14)
    # a larger random low-rank block
    rng = np.random.default_rng(9)
    M = rng.standard_normal((120, 7)) @ rng.standard_normal((7, 90))
    U, V, R = hm.aca_wrapper(M, 1e-9, 10)
    Uo, Vo, Ro = O.aca_wrapper(M, 1e-9, 10)
    assert R == Ro == 7
    assert np.abs(U @ V.T - M).max() < 1e-9
