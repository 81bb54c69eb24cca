"""The compensated residual b - H x (hm_residual) of iterative refinement.

Every product is split exactly by an FMA and every sum keeps its rounding
error, so the residual equals the one computed in higher precision from the
same stored factors.  The reference (README case, svd route) is the sum over
the leaves in numpy's 80-bit long double, from the leaf factors and dense
leaves the library returns; the plain FP64 matvec residual is off by about
eps |H| |x|, the compensated one by far less."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _longdouble_residual(H, x, b, trans=False):
    """b - H x (b - H' x) from the stored leaves, summed in long double."""
    D = H.to_dense()                     # dense leaves are copied as stored
    lv = H.leaves()
    xl = x.astype(np.longdouble)
    y = np.zeros(H.n, np.longdouble)
    for i, (t, r0, c0, m, n, k) in enumerate(lv):
        if t == 0:
            C = D[r0:r0 + m, c0:c0 + n].astype(np.longdouble)
            if trans:
                y[c0:c0 + n] += C.T @ xl[r0:r0 + m]
            else:
                y[r0:r0 + m] += C @ xl[c0:c0 + n]
        elif k > 0:
            A, B = (f.astype(np.longdouble) for f in H.leaf_factors(i))
            if trans:
                y[c0:c0 + n] += B @ (A.T @ xl[r0:r0 + m])
            else:
                y[r0:r0 + m] += A @ (B.T @ xl[c0:c0 + n])
    return b.astype(np.longdouble) - y


def test_compensated_residual_vs_long_double():
    import hmatrix as hm
    prm = hm.Params(Geom=np.linspace(0, 10, 2000), Kernel=hm.Cauchy(1.0), MaxBlock=500, MinBlock=64,
                    MaxRank=5, ConsMethod="svd")
    c, H = hm.NewHmat(prm)
    rng = np.random.default_rng(31)
    x = rng.standard_normal(2000) * 1e3
    b = H * x + rng.standard_normal(2000) * 1e-9          # a residual 1e-12 of b
    ref = _longdouble_residual(H, x, b)
    r = H.residual(x, b)
    r64 = b - H * x
    # the size of the summed terms, |H| |x|, sets the rounding of any sum
    scale = float(np.linalg.norm(np.abs(H.to_dense()) @ np.abs(x)))
    err = float(np.linalg.norm((r - ref).astype(np.float64)))
    err64 = float(np.linalg.norm((r64 - ref).astype(np.float64)))
    assert err <= 1e-17 * scale, err / scale
    assert err64 > 10 * err                               # the plain FP64 residual is coarser
    # transposed: b - H' x against the same long-double sum over the leaves
    rt = H.residual(x, b, trans=True)
    reft = _longdouble_residual(H, x, b, trans=True)
    assert float(np.linalg.norm((rt - reft).astype(np.float64))) <= 1e-17 * scale


def test_residual_device_pointers_two_columns():
    import torch
    import hmatrix as hm
    prm = hm.Params(Geom=np.linspace(0, 10, 4096), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64,
                    MaxRank=16, ConsMethod="aca2", εComp=1e-8, Tree="bisect", Shift=0.5)
    c, H = hm.NewHmat(prm)
    X = np.random.default_rng(32).standard_normal((4096, 2))
    B = np.random.default_rng(33).standard_normal((4096, 2))
    R = H.residual(X, B)
    Rt = H.residual(torch.tensor(X, device="cuda"), torch.tensor(B, device="cuda")).cpu().numpy()
    assert np.array_equal(R, Rt)
    assert np.allclose(R, B - H * X, rtol=0, atol=1e-12 * np.abs(H * X).max())
