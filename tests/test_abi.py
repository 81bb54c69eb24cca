"""The C-ABI library loads and exports every symbol include/hmatrix_b200.h declares (CPU)."""
import ctypes as C
import os
import re

import numpy as np

from conftest import ROOT


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "hmatrix_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"^\s*int\s+(\w+)\s*\(", hdr, flags=re.M)))


def test_library_exports_header():
    from hmatrix import _lib
    L = _lib.lib()
    names = declared_symbols()
    assert "hm_matvec" in names and "aca_wrapper" in names
    for n in names:
        assert hasattr(L, n), n
    assert sorted(_lib.EXPORTED) == names


def test_struct_layouts():
    from hmatrix import _lib
    assert C.sizeof(_lib.hm_params) == 4 * 2 + 8 * 4 + 4 * 8 + 4 * 6
    assert C.sizeof(_lib.hm_info_t) == 8 * 20


def test_defaults_and_errors_without_gpu():
    """Calls that need no GPU: defaults, error text, argument checks."""
    from hmatrix import _lib
    L = _lib.lib()
    p = _lib.hm_params()
    assert L.hm_default_params(C.byref(p)) == 0
    # src/utils.jl:12-23 defaults
    assert (p.eps_comp, p.max_rank, p.max_block, p.min_block, p.eps_trunc) == (1e-10, 16, -1, 64, 1e-10)
    assert L.hm_version() >= 100
    out = C.c_void_p()
    p.kernel = 99
    s = L.hm_new(C.byref(p), 10, None, 0, None, None, None, None, 0, None, C.byref(out))
    assert s == _lib.HM_ERR_ARG and "kernel" in _lib.last_error()


def test_python_mirror_rejects_closures():
    import hmatrix as hm
    prm = hm.Params(Geom=np.linspace(0, 1, 100), Kernel=lambda x, y: 1.0)
    try:
        hm.NewHmat(prm)
    except hm.HmError as e:
        assert "device kernel" in str(e)
    else:
        raise AssertionError("closure kernel accepted")


def test_host_tree_matches_oracle():
    """The product's host cluster tree equals the oracle's (same sklearn call)."""
    from hmatrix.cluster import construct_cluster
    from oracle import hm_oracle as O
    g = np.load(os.path.join(ROOT, "tests", "golden", "readme_case.npz"))
    c = construct_cluster(np.linspace(0, 10, 2000), 64, "kmeans")
    assert np.array_equal(c.P, g["perm"])
    for k in ("s", "e", "left", "right"):
        assert np.array_equal(getattr(c, k), g["cl_" + k])
    for n in (1000, 4096, 5000):
        X = np.linspace(0, 10, n)
        a = construct_cluster(X, 64, "bisect")
        _, r = O.construct_cluster(X, 64, "bisect")
        ca = O.cluster_arrays(r)
        assert np.array_equal(a.P, ca["perm"])
        assert np.array_equal(a.s, ca["s"]) and np.array_equal(a.left, ca["left"])
    rng = np.random.default_rng(5)
    X2 = rng.random((3000, 2))
    a = construct_cluster(X2, 64, "bisect")
    _, r = O.construct_cluster(X2, 64, "bisect")
    ca = O.cluster_arrays(r)
    assert np.array_equal(a.P, ca["perm"]) and np.array_equal(a.e, ca["e"])
