"""ctypes binding of libbcmgx.so (the C ABI declared in include/bcmgx.h).

The shared library is built in-tree by ``make -C bootcmatchgx_b200/csrc`` (or
``__graft_entry__.build()``). Importing this module fails loudly when it is missing: there is
no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libbcmgx.so")

OK = 0
ERR_INVALID_INPUT = -1
ERR_UNSUPPORTED = -2
ERR_NO_CONVERGENCE = -3
ERR_CUDA = -4
ERR_TIMEOUT = -5
ERR_OOM = -6
ERR_NOT_SPD = -7
ERR_INTERNAL = -8

MAX_LEVELS = 64


class BcmgxError(RuntimeError):
    def __init__(self, code, what, message):
        super().__init__(f"{what} failed ({code}): {message}")
        self.code = code


class Params(C.Structure):
    """struct bcmgx_params; the first fields mirror the reference's struct params."""
    _fields_ = [
        ("solver", C.c_int), ("itnlim", C.c_int), ("rtol", C.c_double), ("dispnorm", C.c_int),
        ("preconditioner", C.c_int), ("bootstrap_type", C.c_int), ("max_hrc", C.c_int),
        ("conv_ratio", C.c_double), ("matchtype", C.c_int), ("aggrsweeps", C.c_int),
        ("aggr_type", C.c_int), ("max_levels", C.c_int), ("cycle_type", C.c_int),
        ("coarse_solver", C.c_int), ("relax_type", C.c_int), ("relaxnumber_coarse", C.c_int),
        ("prerelax_sweeps", C.c_int), ("postrelax_sweeps", C.c_int), ("l1jacsweeps", C.c_int),
        ("sstep", C.c_int), ("stop_criterion", C.c_int), ("ru_res", C.c_int),
        ("rec_res_int", C.c_int), ("error", C.c_int),
        ("vcycle_precision", C.c_int), ("record_sweeps", C.c_int), ("use_graph", C.c_int),
        ("device", C.c_int), ("autotune", C.c_int), ("stream", C.c_void_p),
    ]


class Csr(C.Structure):
    _fields_ = [("n", C.c_int), ("m", C.c_int), ("nnz", C.c_int64), ("row", C.c_void_p),
                ("col", C.c_void_p), ("val", C.c_void_p), ("on_device", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("retv", C.c_int), ("niter", C.c_int), ("delta0", C.c_double),
                ("exit_res", C.c_double), ("solve_ms", C.c_double), ("full_n", C.c_int64)]


class HierarchyInfo(C.Structure):
    _fields_ = [("num_levels", C.c_int), ("n", C.c_int * MAX_LEVELS),
                ("nnz", C.c_int64 * MAX_LEVELS), ("op_cmplx", C.c_double),
                ("op_wcmplx", C.c_double), ("avg_cratio", C.c_double),
                ("maxcoarsesize", C.c_int), ("ftcoarse", C.c_int),
                ("num_sweep_records", C.c_int), ("setup_ms", C.c_double),
                ("tpr", C.c_int * MAX_LEVELS), ("index_bytes", C.c_int * MAX_LEVELS),
                ("value_codes", C.c_int * MAX_LEVELS)]


# name -> (restype, argtypes); every symbol include/bcmgx.h declares
_vp, _ip, _dp, _i64p = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int64)
SIGNATURES = {
    "bcmgx_params_default": (C.c_int, [C.POINTER(Params)]),
    "bcmgx_params_from_properties": (C.c_int, [C.c_char_p, C.POINTER(Params)]),
    "bcmgx_params_from_legacy_file": (C.c_int, [C.c_char_p, C.POINTER(Params)]),
    "bcmgx_params_dump": (C.c_int, [C.POINTER(Params), C.c_char_p]),
    "bcmgx_setup": (C.c_int, [C.POINTER(Csr), C.POINTER(Params), C.POINTER(C.c_void_p)]),
    "bcmgx_solve": (C.c_int, [_vp, _vp, _vp, C.c_int, C.POINTER(SolveInfo)]),
    "bcmgx_solve_multi": (C.c_int, [_vp, C.c_int, _vp, _vp, C.c_int, C.POINTER(SolveInfo)]),
    "bcmgx_solve_adjoint": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int, C.POINTER(SolveInfo)]),
    "bcmgx_free": (C.c_int, [_vp]),
    "bcmgx_setup_batch": (C.c_int, [C.c_int, _vp, C.POINTER(Params), C.c_int, C.POINTER(C.c_void_p)]),
    "bcmgx_batch_from_hierarchies": (C.c_int, [C.c_int, _vp, C.POINTER(C.c_void_p)]),
    "bcmgx_batch_get_hierarchy": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_void_p)]),
    "bcmgx_batch_solve": (C.c_int, [_vp, _vp, _vp, _vp]),
    "bcmgx_batch_set_lockstep": (C.c_int, [_vp, C.c_int]),
    "bcmgx_batch_free": (C.c_int, [_vp]),
    "bcmgx_hierarchy_get_info": (C.c_int, [_vp, C.POINTER(HierarchyInfo)]),
    "bcmgx_hierarchy_get_level": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "bcmgx_hierarchy_get_afsai": (C.c_int, [_vp, _i64p, _vp, _vp, _vp]),
    "bcmgx_hierarchy_get_prolongator": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "bcmgx_hierarchy_get_sweep": (C.c_int, [_vp, C.c_int, _ip, _ip, _ip, _ip, _vp, _vp, _vp, _vp]),
    "bcmgx_prec_apply": (C.c_int, [_vp, _vp, _vp, C.c_int]),
    "bcmgx_time_kernels": (C.c_int, [_vp, C.c_int, C.c_int, _vp]),
    "bcmgx_time_block_kernels": (C.c_int, [_vp, C.c_int, C.c_int, _vp]),
    "bcmgx_spmv": (C.c_int, [C.c_int, C.c_int, C.c_int64, _vp, _vp, _vp, _vp, _vp, C.c_double,
                             C.c_double, C.c_int, _vp]),
    "bcmgx_spmm": (C.c_int, [C.c_int, C.c_int, C.c_int64, _vp, _vp, _vp, C.c_int, _vp, _vp, C.c_double,
                             C.c_double, _vp]),
    "bcmgx_edge_weights": (C.c_int, [C.c_int, C.c_int64, _vp, _vp, _vp, _vp, _vp, _dp, _vp]),
    "bcmgx_edge_weights_noalloc": (C.c_int, [C.c_int, C.c_int64, _vp, _vp, _vp, _vp, _vp, _dp, _vp]),
    "bcmgx_suitor_matching": (C.c_int, [C.c_int, C.c_int64, _vp, _vp, _vp, _vp, _vp]),
    "bcmgx_laplacian_3d_size": (C.c_int, [C.c_int] * 7 + [_i64p, _i64p]),
    "bcmgx_laplacian_3d": (C.c_int, [C.c_int] * 7 + [_vp, _vp, _vp]),
    "bcmgx_read_laplacian_cfg": (C.c_int, [C.c_char_p, _ip]),
    "bcmgx_read_matrix_market": (C.c_int, [C.c_char_p, _ip, _ip, _i64p, C.POINTER(_vp),
                                           C.POINTER(_vp), C.POINTER(_vp)]),
    "bcmgx_host_free": (None, [_vp]),
    "bcmgx_diffusion_7p": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp]),
    "bcmgx_last_error_string": (C.c_char_p, []),
    "bcmgx_version": (C.c_char_p, []),
    "bcmgx_launch_count": (C.c_int64, []),
    "bcmgx_dist_setup_local": (C.c_int, [C.POINTER(Csr), C.c_int, _vp, C.POINTER(Params), C.POINTER(C.c_void_p)]),
    "bcmgx_dist_setup_nccl": (C.c_int, [C.POINTER(Csr), C.c_int64, C.c_int64, _vp, C.POINTER(Params),
                                        C.POINTER(C.c_void_p)]),
    "bcmgx_dist_solve": (C.c_int, [_vp, _vp, _vp, C.c_int, C.POINTER(SolveInfo)]),
    "bcmgx_dist_get_info": (C.c_int, [_vp, C.POINTER(HierarchyInfo)]),
    "bcmgx_dist_get_level": (C.c_int, [_vp, C.c_int, _ip, _i64p, _vp, _vp, _vp, _vp]),
    "bcmgx_dist_get_prolongator": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "bcmgx_dist_free": (C.c_int, [_vp]),
    "bcmgx_nccl_unique_id": (C.c_int, [_vp]),
    "bcmgx_nccl_comm_init": (C.c_int, [C.c_int, C.c_int, _vp, C.POINTER(C.c_void_p)]),
    "bcmgx_nccl_comm_destroy": (C.c_int, [_vp]),
}

_lib = None


def lib():
    """Load libbcmgx.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C bootcmatchgx_b200/csrc` "
                "(or __graft_entry__.build()); there is no fallback implementation")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error():
    s = lib().bcmgx_last_error_string()
    return s.decode() if s else ""


def check(rc, what):
    if rc != OK:
        raise BcmgxError(rc, what, last_error())
    return rc
