"""Tensor-core (tcgen05) multi-RHS H-matvec for FP32 and BF16 factors.

*(Hmat, Matrix) (src/harithm.jl:317-329) evaluates one column at a time; here
the stacked factor products run as tensor-core GEMMs.  Checked:

* the operand layouts and descriptors on one tile (hm_tc_selftest) against
  numpy, for both kinds (TF32, BF16), B as the X / Z tiles and A in shared
  memory (K-major) or in tensor memory (as the converters write it);
* H*X and H'*X on the tensor cores against the CUDA-core block kernels on the
  same stored factors (HM_FLAG_MV_SIMT) and against the FP64-factor product:
  FP32 factors use three TF32 products per term and FP32 accumulation; the
  rows of H X cancel (|H X| is about 20 times below |H| |X| for random X), so
  both FP32-accumulated paths sit a few 1e-6 from the FP64 result: 1e-5.  BF16
  factors multiply a two-part BF16 split of X: 2e-5 against the CUDA-core
  path, far inside the BF16 storage error itself (about 3e-3 against FP64
  factors);
* both the median-bisection tree (every leaf on a 16-byte row boundary) and
  the reference's KMeans tree (leaves at arbitrary rows: the unaligned gather
  path).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"F32": 1e-5, "BF16": 2e-5}


def _bf16(x):
    """Round float32 values to the nearest BF16 value (kept as float32)."""
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
    return b.astype(np.uint32).view(np.float32)


def _tf32(x):
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x1000) & 0xFFFFE000
    return b.astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("a_src", [0, 2])
@pytest.mark.parametrize("nc", [16, 64])
def test_tc_layout_selftest(kind, a_src, nc):
    from hmatrix import _lib
    rng = np.random.default_rng(100 + 10 * kind + a_src + nc)
    K = 16 if kind == 0 else 32
    rnd = _tf32 if kind == 0 else _bf16
    A = rnd(rng.standard_normal((128, K)).astype(np.float32))
    B = rnd(rng.standard_normal((2 * nc, K)).astype(np.float32))
    D = np.zeros((128, 2 * nc), np.float32)
    p = lambda a: C.c_void_p(a.ctypes.data)
    _lib.check(_lib.lib().hm_tc_selftest(kind, a_src, nc, p(A), p(B), p(D)))
    R = A.astype(np.float64) @ B.astype(np.float64).T
    assert np.abs(D - R).max() <= 1e-5 * np.abs(R).max(), (kind, a_src, nc)


def _build(storage, tree, n):
    import hmatrix as hm
    prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64,
                    MaxRank=16, ConsMethod="aca2", εComp=1e-8, Tree=tree, Storage=getattr(hm, storage))
    return hm.NewHmat(prm)


def _simt(H, X, trans):
    from hmatrix import _lib
    X = np.asfortranarray(X)
    Y = np.zeros_like(X, order="F")
    p = lambda a: C.c_void_p(a.ctypes.data)
    _lib.check(_lib.lib().hm_matvec(H._h, p(X), p(Y), X.shape[1], int(trans), _lib.HM_FLAG_MV_SIMT, None))
    return Y


@pytest.mark.parametrize("storage", ["F32", "BF16"])
@pytest.mark.parametrize("tree,n", [("bisect", 4096), ("kmeans", 3000), ("bisect", 20000)])
def test_tc_matches_cuda_cores(storage, tree, n):
    c, H = _build(storage, tree, n)
    rng = np.random.default_rng(21)
    for nc in (2, 16, 17, 40, 64, 80):
        X = rng.standard_normal((n, nc))
        for trans in (False, True):
            Y = H.matvec(X, trans=trans)
            R = _simt(H, X, trans)
            err = np.linalg.norm(Y - R) / np.linalg.norm(R)
            assert err <= TOL[storage], (nc, trans, err)


def test_tc_against_fp64_factors():
    # the FP32-factor tensor-core product stays at the FP32 storage error
    # against the FP64-factor product (ACA tolerance 1e-8)
    import hmatrix as hm
    n = 8192
    _, H32 = _build("F32", "bisect", n)
    _, H64 = _build("F64", "bisect", n)
    X = np.random.default_rng(22).standard_normal((n, 16))
    R = H64 * X
    assert np.linalg.norm(H32 * X - R) <= 1e-5 * np.linalg.norm(R)
    assert H32.info().factorized == 0


def test_tc_long_windows():
    # at n = 2^17 a 512-row window holds about 800 Z slots: phase 2 adds its FP32
    # accumulator into the FP64 Y every 512 slots (16 columns), so the product
    # stays near the FP32 storage level against the FP64-factor product
    n = 1 << 17
    _, H32 = _build("F32", "bisect", n)
    _, H64 = _build("F64", "bisect", n)
    X = np.random.default_rng(25).standard_normal((n, 16))
    R = H64 * X
    err = np.linalg.norm(H32 * X - R) / np.linalg.norm(R)
    assert err <= 5e-6, err


def test_tc_range_fallback():
    # factors beyond 2^100 in magnitude take the CUDA-core block kernels (the
    # converters' hi/lo split is exact only below 2^100); the check is redone
    # when hm_scale changes the factors of a handle that already multiplied
    from hmatrix import _lib
    n = 4096
    _, H = _build("F32", "bisect", n)
    X = np.random.default_rng(24).standard_normal((n, 16))
    Y = H * X                                   # tensor cores (plan built, factors in range)
    _lib.check(_lib.lib().hm_scale(H._h, 2.0 ** 110))
    Yb = H * X
    assert np.all(np.isfinite(Yb))
    assert np.array_equal(Yb, _simt(H, X, False))
    assert np.abs(Yb * 2.0 ** -110 - Y).max() <= 1e-5 * np.abs(Y).max()
    _lib.check(_lib.lib().hm_scale(H._h, 2.0 ** -110))
    assert np.abs(H * X - Y).max() <= 1e-12 * np.abs(Y).max()     # back in range: tensor cores again


def test_tc_device_pointers_and_status():
    import torch
    import hmatrix as hm
    from hmatrix import _lib
    n = 4096
    _, H = _build("F32", "bisect", n)
    X = np.random.default_rng(23).standard_normal((n, 16))
    Xt = torch.tensor(X, device="cuda", dtype=torch.float64)
    Yt = H.matvec(Xt)
    _lib.check(_lib.lib().hm_status(H._h, None))
    assert np.allclose(Yt.cpu().numpy(), H * X, rtol=0, atol=1e-12 * np.abs(H * X).max())
