"""The matvec autotuner (hm_autotune): it times every phase-2 shape and
phase-1 grid on the handle's own data and keeps the fastest.  The window
shapes are the same arithmetic in the same order (they only move rows between
CTAs), so H*x is bit-identical under any of them; the cluster shape sums the
same products in another order.  For FP32 factors it also picks the
tensor-core column block of a block product."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_single_and_block():
    import hmatrix as hm
    n = 1 << 16
    prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64, MaxRank=16,
                    ConsMethod="aca2", εComp=1e-8, Tree="bisect")
    c, H = hm.NewHmat(prm)
    x = np.random.default_rng(41).standard_normal(n)
    y0 = H * x
    table, choice = H.autotune(ncols=1, calls=3)
    assert len(table) == 12 and all(v > 0 for v in table.values())
    assert {"clusters_waves1", "clusters_waves2", "clusters_waves4"} <= set(table)
    assert choice["p2_split"] in (1, 2, 4, 8) and choice["p1_waves"] in (1, 2, 4)
    assert H.info().tuned == 1
    if choice["p2_split"] == 1:
        assert np.linalg.norm(H * x - y0) <= 1e-14 * np.linalg.norm(y0)
    else:
        assert np.array_equal(H * x, y0)
    _, H32 = hm.NewHmat(hm.Params(**{**prm.__dict__, "Storage": hm.F32}))
    X = np.random.default_rng(42).standard_normal((n, 40))
    Y0 = H32 * X
    table, choice = H32.autotune(ncols=40, calls=2)
    assert set(k for k in table if k.startswith("tc_")) == {"tc_nc16_cols40", "tc_nc32_cols40", "tc_nc64_cols40"}
    assert choice["tc_nc"][2] in (16, 32, 64)
    assert np.linalg.norm(H32 * X - Y0) <= 1e-5 * np.linalg.norm(Y0)
