"""aca_wrapper_noalloc: the allocation-free fully pivoted ACA.

It serves callers that cannot call cudaMalloc (their device memory belongs to
another allocator's pool, or they cannot afford an allocation's
synchronisation): they pass device buffers for A, U and V and the residual
lives in the library's fixed device array.  Its results must equal those of
the allocating entry point aca_wrapper, call after call, since every call
reuses (and keeps) the same array.

This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = dict(rtol=1e-12, atol=1e-14)


def _eps(A):
    return 1e-3 if A.shape == (20, 20) else 1e-9


def _noalloc(A, rank):
    import torch
    from hmatrix import _lib
    m, n = A.shape
    keep = min(m, n, rank + 1)
    dA = torch.tensor(np.asfortranarray(A).ravel(order="F"), device="cuda", dtype=torch.float64)
    dU = torch.full((keep * m,), np.nan, device="cuda", dtype=torch.float64)
    dV = torch.full((keep * n,), np.nan, device="cuda", dtype=torch.float64)
    stream = torch.cuda.current_stream().cuda_stream or 1
    R = _lib.lib().aca_wrapper_noalloc(C.c_void_p(dA.data_ptr()), C.c_void_p(dU.data_ptr()),
                                       C.c_void_p(dV.data_ptr()), m, n, _eps(A), rank, C.c_void_p(stream))
    if R < 0:
        raise RuntimeError(_lib.last_error())
    M = min(R, rank + 1)
    U = dU.cpu().numpy().reshape(keep, m).T[:, :M]
    V = dV.cpu().numpy().reshape(keep, n).T[:, :M]
    return U, V, R


def _reference(A, rank):
    import hmatrix as hm
    return hm.aca_wrapper(A, _eps(A), rank)


def _cases():
    i = np.arange(20)
    hilbert = 1.0 / (i[:, None] + i[None, :] + 1)          # ACA_FullyPivoted.cpp:240-255
    rng = np.random.default_rng(11)
    lowrank = rng.standard_normal((300, 9)) @ rng.standard_normal((9, 200))
    x = np.linspace(0, 1, 256)
    cauchy = 1.0 / (1.0 + (x[:, None] - (x[None, :] + 3.0)) ** 2)
    return [(hilbert, 5), (lowrank, 12), (cauchy, 16)]


def test_noalloc_matches_allocating_entry_point_twice():
    for A, rank in _cases():
        Ur, Vr, Rr = _reference(A, rank)
        for _ in range(2):                                   # two calls in a row
            U, V, R = _noalloc(A, rank)
            assert R == Rr
            assert U.shape == Ur.shape and V.shape == Vr.shape
            assert np.allclose(U, Ur, **TOL) and np.allclose(V, Vr, **TOL)


def _edge_cases():
    rng = np.random.default_rng(12)
    fat_nan = rng.standard_normal((40, 70))
    fat_nan[7, 11] = np.nan
    thin_nan = rng.standard_normal((90, 30))
    thin_nan[50, 3] = np.nan
    lowrank = rng.standard_normal((60, 4)) @ rng.standard_normal((4, 50))
    return [
        ("zero, fat", np.zeros((30, 50)), 4),          # every pivot below machine epsilon
        ("zero, thin", np.zeros((50, 30)), 4),
        ("NaN, fat", fat_nan, 6),                      # full-rank fallback, ACA_FullyPivoted.cpp:122-147
        ("NaN, thin", thin_nan, 6),
        ("rank 0", lowrank, 0),                        # only the first term is kept
    ]


@pytest.mark.parametrize("name,A,rank", _edge_cases(), ids=[c[0] for c in _edge_cases()])
def test_noalloc_edge_cases_match_allocating_entry_point(name, A, rank):
    # the sub-epsilon pivot branch (unit column, zero row), the NaN fallback
    # (written on the device here, on the host by aca_wrapper) and rank = 0
    Ur, Vr, Rr = _reference(A, rank)
    for _ in range(2):
        U, V, R = _noalloc(A, rank)
        assert R == Rr, (name, R, Rr)
        assert U.shape == Ur.shape and V.shape == Vr.shape
        assert np.allclose(U, Ur, equal_nan=True, **TOL) and np.allclose(V, Vr, equal_nan=True, **TOL), name


def test_noalloc_rejects_oversize():
    import torch
    from hmatrix import _lib
    m, n = 1024, 1024                                        # above the fixed scratch
    d = torch.zeros(8, device="cuda", dtype=torch.float64)
    p = C.c_void_p(d.data_ptr())
    R = _lib.lib().aca_wrapper_noalloc(p, p, p, m, n, 1e-9, 4, None)
    assert R == -_lib.HM_ERR_ARG
    assert "exceeds the fixed scratch" in _lib.last_error()
