"""ctypes binding of libhmatb200.so (declared in include/hmatrix_b200.h).

The library is the product: every numerical call below goes to the sm_100a
kernels.  There is no CPU fallback; a missing library or a missing GPU is an
error.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libhmatb200.so")

HM_OK = 0
HM_ERR_ARG, HM_ERR_CUDA, HM_ERR_OOM, HM_ERR_STATE = 1, 2, 3, 4
HM_ERR_SINGULAR, HM_ERR_RANK, HM_ERR_NONFINITE, HM_ERR_UNSUPPORTED, HM_ERR_TIMEOUT = 5, 6, 7, 8, 9
HM_KERNEL_CAUCHY, HM_KERNEL_INVQUAD, HM_KERNEL_GAUSS = 1, 2, 3
HM_KERNEL_CAUCHY_DP, HM_KERNEL_INVQUAD_DP, HM_KERNEL_GAUSS_DP = 4, 5, 6
HM_CONS_ACA2, HM_CONS_SVD, HM_CONS_BBFMM = 1, 2, 3
HM_F64, HM_F32, HM_BF16 = 0, 1, 2
HM_FLAG_DEVICE_PTRS = 1
HM_FLAG_TRANS = 2
HM_FLAG_MV_SIMT = 4
HM_BUILD_KEEP_PIVOTS = 1

STATUS_NAMES = {
    1: "HM_ERR_ARG", 2: "HM_ERR_CUDA", 3: "HM_ERR_OOM", 4: "HM_ERR_STATE", 5: "HM_ERR_SINGULAR",
    6: "HM_ERR_RANK", 7: "HM_ERR_NONFINITE", 8: "HM_ERR_UNSUPPORTED", 9: "HM_ERR_TIMEOUT",
    10: "HM_ERR_IO",
}

# every symbol include/hmatrix_b200.h declares
EXPORTED = [
    "hm_version", "hm_last_error", "hm_default_params", "hm_new", "hm_new_like", "hm_partition", "hm_destroy", "hm_info",
    "hm_leaves", "hm_leaf_factors", "hm_to_dense", "hm_matvec", "hm_autotune", "hm_set_tune", "hm_residual", "hm_status", "hm_tc_selftest", "hm_matvec_profile", "hm_exact_rows",
    "hm_add_identity", "hm_scale", "hm_copy", "hm_coarsen", "hm_add", "hm_save", "hm_load", "hm_load_user", "hm_lu", "hm_lu_perm", "hm_solve", "hm_solve_refined",
    "hm_batch_lu", "hm_batch_solve", "hm_batch_solve_refined", "hm_batch_matvec",
    "aca_wrapper",
    "aca_wrapper_noalloc",
]


class hm_params(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("kernel", C.c_int32), ("kparam", C.c_double), ("shift", C.c_double),
        ("eps_comp", C.c_double), ("eps_trunc", C.c_double), ("max_rank", C.c_int32),
        ("max_block", C.c_int32), ("min_block", C.c_int32), ("cons_method", C.c_int32),
        ("aca_force", C.c_int32), ("storage", C.c_int32), ("device", C.c_int32),
        ("rank_cap", C.c_int32), ("lu_mode", C.c_int32), ("build_flags", C.c_int32),
        ("eps_trunc_lu", C.c_double), ("row_lo", C.c_int32), ("row_hi", C.c_int32),
    ]


class hm_info_t(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("n_dense", C.c_int64), ("n_rk", C.c_int64), ("depth", C.c_int64),
        ("compress_ratio", C.c_double), ("dense_entries", C.c_int64), ("rk_entries", C.c_int64),
        ("max_rank", C.c_int64), ("pool_bytes", C.c_int64), ("matvec_bytes", C.c_int64),
        ("n_row_groups", C.c_int64), ("factorized", C.c_int64), ("lu_tiles", C.c_int64),
        ("lu_rank_cap", C.c_int64), ("tune_p2_split", C.c_int64), ("tune_p1_waves", C.c_int64),
        ("tune_tc_nc", C.c_int64 * 3), ("tuned", C.c_int64),
    ]


class HmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (STATUS_NAMES.get(code, str(code)), msg))
        self.code = code


_lib = None


def lib():
    """Load the shared library once; raise if it is absent (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libhmatb200.so is not built (%s); run __graft_entry__.build()" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    p64 = C.POINTER(C.c_int64)
    pd = C.POINTER(C.c_double)
    vp = C.c_void_p
    L.hm_version.restype = C.c_int
    L.hm_last_error.argtypes = [C.c_char_p, C.c_int64]
    L.hm_default_params.argtypes = [C.POINTER(hm_params)]
    L.hm_new.argtypes = [C.POINTER(hm_params), C.c_int64, vp, C.c_int64, vp, vp, vp, vp, C.c_int64, vp,
                         C.POINTER(vp)]
    L.hm_new_like.argtypes = [vp, C.POINTER(hm_params), C.POINTER(vp)]
    L.hm_partition.argtypes = [C.POINTER(hm_params), C.c_int64, C.c_int64, vp, vp, vp, vp, C.c_int64, vp,
                               C.c_int64, vp, p64]
    L.hm_destroy.argtypes = [vp]
    L.hm_info.argtypes = [vp, C.POINTER(hm_info_t)]
    L.hm_leaves.argtypes = [vp, C.c_int64, vp, p64]
    L.hm_leaf_factors.argtypes = [vp, C.c_int64, vp, vp]
    L.hm_to_dense.argtypes = [vp, vp, C.c_uint32]
    L.hm_matvec.argtypes = [vp, vp, vp, C.c_int64, C.c_int32, C.c_uint32, vp]
    L.hm_status.argtypes = [vp, vp]
    L.hm_autotune.argtypes = [vp, C.c_int64, C.c_int32, vp]
    L.hm_set_tune.argtypes = [vp, C.c_int32, C.c_int32]
    L.hm_residual.argtypes = [vp, vp, vp, vp, C.c_int64, C.c_int32, C.c_uint32, vp]
    L.hm_tc_selftest.argtypes = [C.c_int32, C.c_int32, C.c_int32, vp, vp, vp]
    L.hm_matvec_profile.argtypes = [vp, vp, vp, C.c_int32, vp, C.POINTER(C.c_float)]
    L.hm_exact_rows.argtypes = [vp, vp, C.c_int64, vp, vp, C.c_uint32, vp]
    L.hm_add_identity.argtypes = [vp, C.c_double]
    L.hm_scale.argtypes = [vp, C.c_double]
    L.hm_copy.argtypes = [vp, C.POINTER(vp)]
    L.hm_coarsen.argtypes = [vp, C.POINTER(vp)]
    L.hm_add.argtypes = [vp, vp, C.c_double, C.POINTER(vp)]
    L.hm_save.argtypes = [vp, C.c_char_p, vp, C.c_int64]
    L.hm_load.argtypes = [C.c_char_p, C.c_int32, C.POINTER(vp)]
    L.hm_load_user.argtypes = [C.c_char_p, vp, C.c_int64, p64]
    L.hm_lu.argtypes = [vp]
    L.hm_lu_perm.argtypes = [vp, vp]
    L.hm_solve.argtypes = [vp, vp, vp, C.c_int64, C.c_uint32, vp]
    L.hm_solve_refined.argtypes = [vp, vp, vp, C.c_int64, C.c_double, C.c_int32, C.c_uint32, vp,
                                   C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    L.hm_batch_lu.argtypes = [vp, C.c_int64, C.c_int32, vp]
    L.hm_batch_solve.argtypes = [vp, C.c_int64, vp, vp, C.c_int64, C.c_uint32, C.c_int32, vp]
    L.hm_batch_solve_refined.argtypes = [vp, C.c_int64, vp, vp, C.c_int64, C.c_double, C.c_int32, C.c_uint32,
                                         C.c_int32, vp, vp, vp]
    L.hm_batch_matvec.argtypes = [vp, C.c_int64, vp, vp, C.c_int64, C.c_int32, C.c_uint32, C.c_int32, vp]
    L.aca_wrapper.argtypes = [pd, pd, pd, C.c_int, C.c_int, C.c_double, C.c_int]
    L.aca_wrapper.restype = C.c_int
    L.aca_wrapper_noalloc.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_double, C.c_int, vp]
    L.aca_wrapper_noalloc.restype = C.c_int
    for name in EXPORTED:
        f = getattr(L, name)
        if f.restype is None:
            f.restype = C.c_int
    _lib = L
    return L


def last_error():
    buf = C.create_string_buffer(4096)
    lib().hm_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status):
    if status != HM_OK:
        raise HmError(status, last_error())
    return status
