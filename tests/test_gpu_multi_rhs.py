"""GPU parity of the multi-RHS H-matvec (K5): H*X and H'*X for an n x c block
against the single-vector kernels column by column (same stored factors, so
only the summation order differs) and against the oracle's dense matrix.
*(Hmat, Matrix) in the reference loops over columns (src/harithm.jl:323-329)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


# the single-vector kernels round x to FP32 for FP32/BF16 factors; the block
# products of FP32/BF16 factors run on the tensor cores (three TF32 products
# per term for FP32 factors, X split into two BF16 parts for BF16 factors),
# both with FP32 accumulation
TOL = {"F64": 1e-13, "F32": 1e-5, "BF16": 2e-5}


def _cols(H, X, trans):
    return np.stack([H.matvec(X[:, j], trans=trans) for j in range(X.shape[1])], 1)


@pytest.mark.parametrize("storage", ["F64", "F32", "BF16"])
@pytest.mark.parametrize("tree,n", [("bisect", 4096), ("kmeans", 3000)])
def test_multi_rhs_matches_columns(storage, tree, n):
    import hmatrix as hm
    prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64,
                    MaxRank=16, ConsMethod="aca2", εComp=1e-8, Tree=tree, Storage=getattr(hm, storage))
    c, H = hm.NewHmat(prm)
    rng = np.random.default_rng(12)
    for nc in (2, 3, 8, 13, 16, 17, 40):
        X = rng.standard_normal((n, nc))
        for trans in (False, True):
            Y = H.matvec(X, trans=trans)
            R = _cols(H, X, trans)
            assert np.linalg.norm(Y - R) <= TOL[storage] * np.linalg.norm(R), (nc, trans)


def test_multi_rhs_readme_vs_dense():
    # the svd route (MaxBlock 500): leaves start on rows that are not 2- or
    # 4-aligned, dense leaves read transposed in H'*X
    import hmatrix as hm
    prm = hm.Params(Geom=np.linspace(0, 10, 2000), Kernel=hm.Cauchy(1.0), MaxBlock=500, MinBlock=64,
                    MaxRank=5, ConsMethod="svd")
    c, H = hm.NewHmat(prm)
    D = H.to_dense()
    X = np.random.default_rng(13).random((2000, 6))
    assert np.allclose(H * X, D @ X, rtol=1e-13, atol=1e-12)
    assert np.allclose(H.matvec(X, trans=True), D.T @ X, rtol=1e-13, atol=1e-12)


def test_multi_rhs_torch_device_pointers():
    import torch
    import hmatrix as hm
    prm = hm.Params(Geom=np.linspace(0, 10, 4096), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64,
                    MaxRank=16, ConsMethod="aca2", εComp=1e-8, Tree="bisect")
    c, H = hm.NewHmat(prm)
    X = np.random.default_rng(14).standard_normal((4096, 5))
    Xt = torch.tensor(X, device="cuda", dtype=torch.float64)
    assert np.array_equal(H.matvec(Xt).cpu().numpy(), H * X)
