"""Failure paths of the C ABI, each injected on the host: no test here faults,
traps or hangs a GPU.

The reference reports these conditions with Julia errors or lets NaNs through:
ACA_FullyPivoted.cpp:122-147 falls back to a full-rank copy when the ACA
residual turns NaN, and lu! refuses a frozen or non-factorisable matrix
(src/hlu.jl:466-472).  Here every entry point returns a status instead:

* HM_ERR_NONFINITE -- a NaN or infinite coordinate in the host geometry
  (checked before the device is touched, so that part runs without a GPU),
  and a NaN right-hand side of the refined solve;
* HM_ERR_SINGULAR  -- an exactly zero pivot in a diagonal leaf: with every
  point at the same place every kernel entry is 1, and the second pivot of
  each diagonal leaf is 1 - 1*1 = 0 exactly;
* HM_ERR_OOM       -- an allocation the device cannot hold (a single dense
  2^20 x 2^20 leaf, 8 TiB in FP64); the library keeps working afterwards.
"""
import ctypes as C

import numpy as np
import pytest


def _prm(hm, geom, **kw):
    base = dict(Geom=geom, Kernel=hm.Cauchy(1.0), MaxBlock=128, MinBlock=32, MaxRank=8,
                ConsMethod="aca2", Tree="bisect")
    base.update(kw)
    return hm.Params(**base)


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_nonfinite_geometry_refused(bad):
    import hmatrix as hm
    from hmatrix import _lib
    g = np.linspace(0, 10, 300)
    g[123] = bad
    with pytest.raises(hm.HmError) as ei:
        hm.NewHmat(_prm(hm, g))
    assert ei.value.code == _lib.HM_ERR_NONFINITE
    # the C ABI refuses it too, before any device call (this runs without a GPU)
    from hmatrix.cluster import construct_cluster
    c = construct_cluster(np.linspace(0, 10, 300), 32, "bisect")
    geom = np.asfortranarray(c.X.copy())
    geom[123, 0] = bad
    p = hm._params_struct(_prm(hm, g), 1)
    out = C.c_void_p()
    ptr = lambda a: C.c_void_p(a.ctypes.data)
    s = _lib.lib().hm_new(C.byref(p), 300, ptr(geom), c.ncluster, ptr(c.s), ptr(c.e), ptr(c.left),
                          ptr(c.right), 0, None, C.byref(out))
    assert s == _lib.HM_ERR_NONFINITE
    assert "point 123" in _lib.last_error()
    assert not out.value


@pytest.mark.gpu
def test_zero_pivot_is_singular_and_handle_stays_usable():
    import hmatrix as hm
    from hmatrix import _lib
    n = 512
    c, H = hm.NewHmat(_prm(hm, np.zeros(n)))          # K = ones(n, n)
    with pytest.raises(hm.HmError) as ei:
        H.lu_()
    assert ei.value.code == _lib.HM_ERR_SINGULAR
    assert "zero pivot" in str(ei.value)
    # the failed lu! leaves H unfactorised: its matvec still works
    assert H.info().factorized == 0
    y = np.random.default_rng(0).standard_normal(n)
    assert np.allclose(H * y, np.full(n, y.sum()), rtol=1e-12, atol=1e-9)


@pytest.mark.gpu
def test_nan_rhs_of_refined_solve():
    import hmatrix as hm
    from hmatrix import _lib
    n = 1024
    c, H = hm.NewHmat(_prm(hm, np.linspace(0, 10, n), Shift=1.0))
    H.lu_()
    y = np.random.default_rng(1).standard_normal(n)
    x, it, rr = H.solve_refined(y, tol=1e-10, max_iter=5)
    assert rr <= 1e-10
    y[77] = np.nan
    with pytest.raises(hm.HmError) as ei:
        H.solve_refined(y, tol=1e-10, max_iter=5)
    assert ei.value.code == _lib.HM_ERR_NONFINITE
    # the next call on the same handle is unaffected
    y[77] = 0.0
    x, it, rr = H.solve_refined(y, tol=1e-10, max_iter=5)
    assert rr <= 1e-10


@pytest.mark.gpu
def test_allocation_failure_is_oom_and_library_recovers():
    import hmatrix as hm
    from hmatrix import _lib
    n = 1 << 20
    # MinBlock >= n: the root cluster is one leaf and H one dense block of n^2
    # entries, far beyond the device's memory; the pool allocation fails
    with pytest.raises(hm.HmError) as ei:
        hm.NewHmat(_prm(hm, np.linspace(0, 10, n), MaxBlock=512, MinBlock=n))
    assert ei.value.code == _lib.HM_ERR_OOM
    assert "pool" in str(ei.value)
    # a normal construction, matvec and factorisation on the same device next
    m = 2048
    c, H = hm.NewHmat(_prm(hm, np.linspace(0, 10, m), Shift=1.0))
    y = np.random.default_rng(2).standard_normal(m)
    r = H * y
    assert np.all(np.isfinite(r))
    H.lu_()
    x, it, rr = H.solve_refined(y, tol=1e-10, max_iter=5)
    assert rr <= 1e-10
