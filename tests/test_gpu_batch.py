"""GPU parity of the batched entry points (hm_batch_lu / hm_batch_solve /
hm_batch_solve_refined / hm_batch_matvec) on independent uneven 1-D problems:
K = 1/(1+((x-y)/l)^2) + delta_xy, MaxBlock 256, MinBlock 32, MaxRank 12 -- the
batched configuration at sizes the test finishes in seconds.  Every problem of
a batch must give what the single-problem calls give (same kernels, each
problem on its own stream)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def problems(count, seed, nmin=2 ** 10, nmax=2 ** 13):
    import hmatrix as hm
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(2 ** rng.uniform(np.log2(nmin), np.log2(nmax))))
        L = rng.uniform(5, 20)
        ell = rng.uniform(0.5, 2)
        x = np.sort(rng.uniform(0, L, n))
        prm = hm.Params(Geom=x, Kernel=hm.Cauchy(ell), MaxBlock=256, MinBlock=32, MaxRank=12,
                        ConsMethod="aca2", εComp=1e-10, Tree="bisect", Shift=1.0)
        c, H = hm.NewHmat(prm)
        out.append((H, rng.standard_normal(n)))
    return out


def test_batch_lu_solve_matches_single():
    import hmatrix as hm
    P = problems(6, 3)
    Hs = [H for H, _ in P]
    ys = [y for _, y in P]
    Ls = hm.lu_batch(Hs, nthreads=4)
    singles = [hm.lu(H) for H in Hs]
    for L, S in zip(Ls, singles):
        assert np.array_equal(L.P, S.P)
    xs = hm.solve_batch(Ls, ys)
    for x, S, y, H in zip(xs, singles, ys, Hs):
        xsg = S.solve(y)
        assert np.abs(x - xsg).max() <= 1e-13 * np.abs(xsg).max()
        D = H.to_dense()
        assert np.linalg.norm(x - np.linalg.solve(D, y)) <= 1e-9 * np.linalg.norm(x)
    xts = hm.solve_batch(Ls, ys, trans=True)
    for x, H, y in zip(xts, Hs, ys):
        D = H.to_dense()
        assert np.linalg.norm(x - np.linalg.solve(D.T, y)) <= 1e-9 * np.linalg.norm(x)
    xr, it, rr = hm.solve_refined_batch(Ls, ys, tol=1e-12, max_iter=5)
    assert (rr <= 1e-12).all() and (it >= 0).all()
    for x, H, y in zip(xr, Hs, ys):
        assert np.linalg.norm(H * x - y) <= 1e-11 * np.linalg.norm(y)


def test_batch_matvec_matches_single():
    import hmatrix as hm
    P = problems(5, 7)
    Hs = [H for H, _ in P]
    xs = [np.random.default_rng(i).standard_normal((H.n, 2)) for i, H in enumerate(Hs)]
    ys = hm.matvec_batch(Hs, xs, nthreads=3)
    for H, x, y in zip(Hs, xs, ys):
        assert np.array_equal(y, H * x)
    yt = hm.matvec_batch(Hs, xs, trans=True)
    for H, x, y in zip(Hs, xs, yt):
        assert np.array_equal(y, H.matvec(x, trans=True))


def test_batch_errors_per_problem():
    import hmatrix as hm
    from hmatrix import _lib
    P = problems(3, 9, nmax=2 ** 11)
    Hs = [H.copy() for H, _ in P]
    with pytest.raises(hm.HmError) as e:
        hm.lu_batch_([Hs[0], Hs[1], Hs[0]])            # the same handle twice
    assert "repeats a handle" in str(e.value)
    Hs[1].lu_()                                         # already factorised: src/hlu.jl:466-468
    st = np.zeros(3, np.int32)
    import ctypes as C
    s = hm.lib().hm_batch_lu(hm._handles(Hs), 3, 2, C.c_void_p(st.ctypes.data))
    assert s == _lib.HM_ERR_STATE
    assert st.tolist() == [_lib.HM_OK, _lib.HM_ERR_STATE, _lib.HM_OK]
    assert "problem 1" in _lib.last_error() and "already factorized" in _lib.last_error()
    # the other two were factorised
    assert Hs[0].info().factorized and Hs[2].info().factorized
