"""ctypes binding of the CPU oracle (oracle/bcmgx_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` as the checker
and by ``bench.py`` for the CPU-baseline leg. The product package never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")

SOLVERS = {"CGHS": 0, "FCG": 1, "CGS": 2, "PIPELINED_CGS": 3, "CGS_CUBLAS": 4}
PRECONDITIONERS = {"NONE": 0, "L1_JACOBI": 1, "BCMG": 2, "AFSAI": 3}
CYCLES = {"V_CYCLE": 0, "H_CYCLE": 1, "W_CYCLE": 2, "VARIABLE_V_CYCLE": 3}


class OrcParams(C.Structure):
    _fields_ = [
        ("solver", C.c_int), ("itnlim", C.c_int), ("rtol", C.c_double),
        ("dispnorm", C.c_int), ("preconditioner", C.c_int), ("bootstrap_type", C.c_int),
        ("max_hrc", C.c_int), ("conv_ratio", C.c_double), ("matchtype", C.c_int),
        ("aggrsweeps", C.c_int), ("aggr_type", C.c_int), ("max_levels", C.c_int),
        ("cycle_type", C.c_int), ("coarse_solver", C.c_int), ("relax_type", C.c_int),
        ("relaxnumber_coarse", C.c_int), ("prerelax_sweeps", C.c_int),
        ("postrelax_sweeps", C.c_int), ("l1jacsweeps", C.c_int), ("sstep", C.c_int),
        ("stop_criterion", C.c_int), ("ru_res", C.c_int), ("rec_res_int", C.c_int),
    ]


def build():
    """Compile liboracle.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
        L.orc_matrix_lap3d.restype = vp
        L.orc_matrix_lap3d.argtypes = [C.c_int] * 7
        L.orc_matrix_from_csr.restype = vp
        L.orc_matrix_from_csr.argtypes = [C.c_int, C.c_int, C.c_long, vp, vp, vp]
        L.orc_matrix_info.argtypes = [vp, ip, ip, C.POINTER(C.c_long)]
        L.orc_matrix_export.argtypes = [vp, vp, vp, vp]
        L.orc_matrix_free.argtypes = [vp]
        L.orc_spmv.argtypes = [vp, vp, vp]
        L.orc_edge_weights.restype = C.c_double
        L.orc_edge_weights.argtypes = [vp, vp, vp]
        L.orc_match.argtypes = [vp, vp, C.c_int, vp]
        L.orc_setup.restype = vp
        L.orc_setup.argtypes = [vp, C.POINTER(OrcParams), C.c_int]
        L.orc_setup_parts.restype = vp
        L.orc_setup_parts.argtypes = [vp, C.POINTER(OrcParams), C.c_int, C.c_int, vp]
        L.orc_hier_level_parts.restype = C.c_int
        L.orc_hier_level_parts.argtypes = [vp, C.c_int, vp]
        L.orc_hier_free.argtypes = [vp]
        L.orc_hier_levels.argtypes = [vp]
        L.orc_hier_stats.argtypes = [vp, vp]
        L.orc_hier_level_info.argtypes = [vp, C.c_int, ip, C.POINTER(C.c_long)]
        L.orc_hier_level_matrix.restype = vp
        L.orc_hier_level_matrix.argtypes = [vp, C.c_int]
        L.orc_hier_afsai.restype = vp
        L.orc_hier_afsai.argtypes = [vp]
        L.orc_hier_level_prolongator.argtypes = [vp, C.c_int, vp, vp, vp]
        L.orc_hier_num_records.argtypes = [vp]
        L.orc_hier_record.argtypes = [vp, C.c_int, ip, ip, ip, ip]
        L.orc_hier_record_data.argtypes = [vp, C.c_int, vp, vp, vp, vp]
        L.orc_galerkin.restype = vp
        L.orc_galerkin.argtypes = [vp, vp, vp, vp]
        L.orc_vcycle.argtypes = [vp, vp, vp]
        L.orc_solve.restype = C.c_int
        L.orc_solve.argtypes = [vp, vp, vp, ip, dp, dp]
        L.orc_num_threads.restype = C.c_int
        L.orc_num_threads.argtypes = [C.c_int]
        L.orc_params_default.argtypes = [C.POINTER(OrcParams)]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def num_threads(n=0):
    return lib().orc_num_threads(n)


def params(**kw):
    p = OrcParams()
    lib().orc_params_default(C.byref(p))
    p.solver = SOLVERS["FCG"]
    p.preconditioner = PRECONDITIONERS["BCMG"]
    p.dispnorm = 0
    for k, v in kw.items():
        if k == "solver" and isinstance(v, str):
            v = SOLVERS[v]
        if k == "preconditioner" and isinstance(v, str):
            v = PRECONDITIONERS[v]
        if k == "cycle_type" and isinstance(v, str):
            v = CYCLES[v]
        setattr(p, k, v)
    return p


class Matrix:
    """CSR matrix owned by the oracle (or borrowed from a hierarchy when ``owned`` is False)."""

    def __init__(self, handle, owned=True):
        self.h = handle
        self.owned = owned

    @classmethod
    def lap3d(cls, stencil, nx, ny, nz, P=1, Q=1, R=1):
        return cls(lib().orc_matrix_lap3d(stencil, nx, ny, nz, P, Q, R))

    @classmethod
    def from_csr(cls, row, col, val, m=None):
        row = np.ascontiguousarray(row, dtype=np.int32)
        col = np.ascontiguousarray(col, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        n = row.size - 1
        return cls(lib().orc_matrix_from_csr(n, m or n, col.size, _p(row), _p(col), _p(val)))

    def info(self):
        n, m, nnz = C.c_int(), C.c_int(), C.c_long()
        lib().orc_matrix_info(self.h, C.byref(n), C.byref(m), C.byref(nnz))
        return n.value, m.value, nnz.value

    def csr(self):
        n, _, nnz = self.info()
        row = np.empty(n + 1, np.int32)
        col = np.empty(nnz, np.int32)
        val = np.empty(nnz, np.float64)
        lib().orc_matrix_export(self.h, _p(row), _p(col), _p(val))
        return row, col, val

    def spmv(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.info()[0])
        lib().orc_spmv(self.h, _p(x), _p(y))
        return y

    def edge_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        W = np.empty(self.info()[2])
        mn = lib().orc_edge_weights(self.h, _p(w), _p(W))
        return W, mn

    def match(self, W, method=1):
        W = np.ascontiguousarray(W, dtype=np.float64)
        M = np.empty(self.info()[0], np.int32)
        lib().orc_match(self.h, _p(W), method, _p(M))
        return M

    def galerkin(self, M, w):
        M = np.ascontiguousarray(M, dtype=np.int32)
        w = np.ascontiguousarray(w, dtype=np.float64)
        wc = np.empty(self.info()[0])
        C_ = Matrix(lib().orc_galerkin(self.h, _p(M), _p(w), _p(wc)))
        return C_, wc[: C_.info()[0]].copy()

    def __del__(self):
        if getattr(self, "owned", False) and self.h:
            lib().orc_matrix_free(self.h)
            self.h = None


class Hierarchy:
    """The oracle's set-up. parts: row offsets of the ranks (P + 1 entries, from 0 to n) for the
    reference's np = P set-up (rank-local matching and aggregate numbering), or None for np = 1."""

    def __init__(self, A: Matrix, prm: OrcParams, record=False, parts=None):
        self.A = A
        if parts is None:
            self.h = lib().orc_setup(A.h, C.byref(prm), 1 if record else 0)
        else:
            pt = np.ascontiguousarray(parts, dtype=np.int32)
            self.h = lib().orc_setup_parts(A.h, C.byref(prm), 1 if record else 0, pt.size - 1, _p(pt))

    def level_parts(self, l):
        k = lib().orc_hier_level_parts(self.h, l, None)
        pt = np.empty(k + 1, np.int32)
        lib().orc_hier_level_parts(self.h, l, _p(pt))
        return pt

    def levels(self):
        return lib().orc_hier_levels(self.h)

    def level_sizes(self):
        out = []
        for l in range(self.levels()):
            n, nnz = C.c_int(), C.c_long()
            lib().orc_hier_level_info(self.h, l, C.byref(n), C.byref(nnz))
            out.append((n.value, nnz.value))
        return out

    def stats(self):
        s = np.empty(5)
        lib().orc_hier_stats(self.h, _p(s))
        return {"op_cmplx": s[0], "op_wcmplx": s[1], "avg_cratio": s[2],
                "maxcoarsesize": int(s[3]), "ftcoarse": int(s[4])}

    def level_matrix(self, l):
        return Matrix(lib().orc_hier_level_matrix(self.h, l), owned=False)

    def prolongator(self, l):
        n = self.level_sizes()[l][0]
        agg = np.empty(n, np.int32)
        p = np.empty(n)
        M = np.empty(n)
        lib().orc_hier_level_prolongator(self.h, l, _p(agg), _p(p), _p(M))
        return agg, p, M

    def records(self):
        out = []
        for k in range(lib().orc_hier_num_records(self.h)):
            lv, sw, n, nc = C.c_int(), C.c_int(), C.c_int(), C.c_int()
            lib().orc_hier_record(self.h, k, C.byref(lv), C.byref(sw), C.byref(n), C.byref(nc))
            M = np.empty(n.value, np.int32)
            agg = np.empty(n.value, np.int32)
            p = np.empty(n.value)
            w = np.empty(n.value)
            lib().orc_hier_record_data(self.h, k, _p(M), _p(agg), _p(p), _p(w))
            out.append({"level": lv.value, "sweep": sw.value, "nc": nc.value,
                        "match": M, "agg": agg, "p": p, "w": w})
        return out

    def vcycle(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        v = np.zeros_like(r)
        lib().orc_vcycle(self.h, _p(r), _p(v))
        return v

    def afsai_factor(self):
        """The AFSAI factor G of an AFSAI hierarchy as CSR arrays."""
        return Matrix(lib().orc_hier_afsai(self.h), owned=False).csr()

    def solve(self, b, x0=None):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
        it, d0, er = C.c_int(), C.c_double(), C.c_double()
        rv = lib().orc_solve(self.h, _p(b), _p(x), C.byref(it), C.byref(d0), C.byref(er))
        return x, {"retv": rv, "niter": it.value, "delta0": d0.value, "exit_res": er.value}

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_hier_free(self.h)
            self.h = None
