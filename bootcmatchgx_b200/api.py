"""Host-side interface of the B200 BCMG/FCG path, mirroring the reference's operator API.

Reference entry points and their counterparts here:
  Params::initFromPropertiesFile (BCMGX/src/config/Params.cu:330)  -> init_from_properties_file
  Params::initFromFile (Params.cu:406)                            -> init_from_file
  prec_setup (BCMGX/src/preconditioner/prec_setup.cu:5)           -> prec_setup -> Hierarchy
  solve (BCMGX/src/solver/solve.cu:11)                            -> solve / Hierarchy.solve
  prec_apply (BCMGX/src/preconditioner/prec_apply.cu:6)           -> Hierarchy.prec_apply
  prec_finalize (BCMGX/src/preconditioner/prec_finalize.cu:8)     -> prec_finalize / Hierarchy.free
  generate_lap3d_local_matrix / generate_lap_local_matrix
  (BCMGX/src/utility/input.cu:85-138)                             -> laplacian_3d, laplacian
  read_matrix_from_file (BCMGX/src/datastruct/CSR.cu:1944)        -> read_matrix_market
Host arrays are numpy; device arrays are CUDA torch tensors (pointers are passed through).
All work runs in libbcmgx.so; errors raise BcmgxError with the library's status code.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import BcmgxError, check, lib

SOLVERS = {"CGHS": 0, "FCG": 1, "CGS": 2, "PIPELINED_CGS": 3, "CGS_CUBLAS": 4, "INVALID": 5}
PRECONDITIONERS = {"NONE": 0, "L1_JACOBI": 1, "BCMG": 2, "AFSAI": 3, "INVALID": 4}
BOOTSTRAP = {"MULTIPLICATIVE": 0, "SYMMETRIZED_MULTIPLICATIVE": 1, "ADDITIVE": 2, "INVALID": 3}
CYCLES = {"V_CYCLE": 0, "H_CYCLE": 1, "W_CYCLE": 2, "VARIABLE_V_CYCLE": 3, "INVALID": 4}
VCYCLE = {"FP64": 0, "FP32": 1}
_ENUMS = {"solver": SOLVERS, "preconditioner": PRECONDITIONERS, "bootstrap_type": BOOTSTRAP,
          "cycle_type": CYCLES, "vcycle_precision": VCYCLE}


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def _is_device(a):
    """True for a CUDA tensor. The library orders its own stream after the legacy default stream
    (torch's default); work that torch queued on another current stream is waited for here."""
    if not (hasattr(a, "is_cuda") and a.is_cuda):
        return False
    import torch
    cur = torch.cuda.current_stream(a.device)
    if cur.cuda_stream != 0:
        cur.synchronize()
    return True


def params_default(**overrides) -> L.Params:
    """Defaults of struct params (BCMGX/src/config/Params.h:238-291), then overrides."""
    p = L.Params()
    check(lib().bcmgx_params_default(C.byref(p)), "bcmgx_params_default")
    return set_params(p, **overrides)


def set_params(p: L.Params, **kw) -> L.Params:
    for k, v in kw.items():
        if k in _ENUMS and isinstance(v, str):
            v = _ENUMS[k][v]
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def init_from_properties_file(path, **overrides) -> L.Params:
    p = L.Params()
    check(lib().bcmgx_params_from_properties(str(path).encode(), C.byref(p)), "reading settings")
    return set_params(p, **overrides)


def init_from_file(path, **overrides) -> L.Params:
    p = L.Params()
    check(lib().bcmgx_params_from_legacy_file(str(path).encode(), C.byref(p)), "reading settings")
    return set_params(p, **overrides)


def params_to_dict(p: L.Params) -> dict:
    return {name: getattr(p, name) for name, _ in L.Params._fields_ if name != "stream"}


# ---------------------------------------------------------------------------------------------
# input generation
# ---------------------------------------------------------------------------------------------
def laplacian_3d_size(stencil, nx, ny, nz, P=1, Q=1, R=1):
    n, z = C.c_int64(), C.c_int64()
    check(lib().bcmgx_laplacian_3d_size(stencil, nx, ny, nz, P, Q, R, C.byref(n), C.byref(z)),
          "bcmgx_laplacian_3d_size")
    return n.value, z.value


def laplacian_3d(stencil, nx, ny, nz, P=1, Q=1, R=1):
    """(row, col, val) of the 7p/27p Laplacian in the reference's global row order."""
    n, z = laplacian_3d_size(stencil, nx, ny, nz, P, Q, R)
    row = np.empty(n + 1, np.int32)
    col = np.empty(z, np.int32)
    val = np.empty(z, np.float64)
    check(lib().bcmgx_laplacian_3d(stencil, nx, ny, nz, P, Q, R, _ptr(row), _ptr(col), _ptr(val)),
          "bcmgx_laplacian_3d")
    return row, col, val


def laplacian(n):
    """The -a n matrix (generateLocalLaplacian3D): 7-point on n^3, lexicographic."""
    return laplacian_3d(7, n, n, n)


def read_laplacian_cfg(path):
    out = (C.c_int * 6)()
    check(lib().bcmgx_read_laplacian_cfg(str(path).encode(), out), "reading the laplacian file")
    return dict(zip(("nx", "ny", "nz", "P", "Q", "R"), list(out)))


def read_matrix_market(path):
    n, m, z = C.c_int(), C.c_int(), C.c_int64()
    r, c, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
    check(lib().bcmgx_read_matrix_market(str(path).encode(), C.byref(n), C.byref(m), C.byref(z),
                                         C.byref(r), C.byref(c), C.byref(v)), "reading the matrix")
    try:
        row = np.ctypeslib.as_array((C.c_int * (n.value + 1)).from_address(r.value)).copy()
        col = np.ctypeslib.as_array((C.c_int * max(z.value, 1)).from_address(c.value))[: z.value].copy()
        val = np.ctypeslib.as_array((C.c_double * max(z.value, 1)).from_address(v.value))[: z.value].copy()
    finally:
        for p in (r, c, v):
            lib().bcmgx_host_free(p)
    return row, col, val


def diffusion_7p(nx, ny, nz, kappa):
    kappa = np.ascontiguousarray(kappa, dtype=np.float64).reshape(-1)
    n, z = laplacian_3d_size(7, nx, ny, nz)
    if kappa.size != n:
        raise ValueError("kappa must have nx*ny*nz entries")
    row = np.empty(n + 1, np.int32)
    col = np.empty(z, np.int32)
    val = np.empty(z, np.float64)
    check(lib().bcmgx_diffusion_7p(nx, ny, nz, _ptr(kappa), _ptr(row), _ptr(col), _ptr(val)),
          "bcmgx_diffusion_7p")
    return row, col, val


# ---------------------------------------------------------------------------------------------
# set-up / solve / finalize
# ---------------------------------------------------------------------------------------------
class Hierarchy:
    """The BCMG hierarchy of one matrix (what prec_setup builds into cgsprec)."""

    def __init__(self, row, col, val, params: L.Params):
        dev = _is_device(row)
        if not dev:
            row = np.ascontiguousarray(row, dtype=np.int32)
            col = np.ascontiguousarray(col, dtype=np.int32)
            val = np.ascontiguousarray(val, dtype=np.float64)
        n = int(row.shape[0]) - 1
        self._keep = (row, col, val)
        A = L.Csr(n, n, int(col.shape[0]), _ptr(row), _ptr(col), _ptr(val), 1 if dev else 0)
        h = C.c_void_p()
        check(lib().bcmgx_setup(C.byref(A), C.byref(params), C.byref(h)), "prec_setup")
        self.h = h
        self.n = n
        self.nnz = int(col.shape[0])
        self.params = params
        self._keep = None

    # -- solve ------------------------------------------------------------------------------
    def solve(self, b, x0=None, raise_on_no_convergence=False):
        """FCG solve of A x = b. Host numpy in -> numpy out; CUDA tensors are updated in place."""
        info = L.SolveInfo()
        if _is_device(b):
            import torch
            x = torch.zeros_like(b) if x0 is None else x0
            rc = lib().bcmgx_solve(self.h, _ptr(b), _ptr(x), 1, C.byref(info))
        else:
            b = np.ascontiguousarray(b, dtype=np.float64)
            if x0 is None:
                x = np.zeros(self.n)
            elif isinstance(x0, np.ndarray) and x0.dtype == np.float64 and x0.flags.c_contiguous and x0.flags.writeable:
                x = x0   # updated in place, as the reference writes x0
            else:
                x = np.array(x0, dtype=np.float64)
            rc = lib().bcmgx_solve(self.h, _ptr(b), _ptr(x), 0, C.byref(info))
        if rc != L.OK and (rc != L.ERR_NO_CONVERGENCE or raise_on_no_convergence):
            raise BcmgxError(rc, "solve", L.last_error())
        out = {"retv": info.retv, "niter": info.niter, "delta0": info.delta0,
               "exit_res": info.exit_res, "solve_ms": info.solve_ms, "status": rc}
        return x, out

    def solve_multi(self, B, X0=None, raise_on_no_convergence=False):
        """FCG solve of A X = B for up to 32 right-hand sides at once; B is n x k (row-major).

        Host numpy in -> numpy out; a CUDA X0 is updated in place. Returns X and one info dict
        per column."""
        k = int(B.shape[1])
        infos = (L.SolveInfo * k)()
        if _is_device(B):
            import torch
            B = B.contiguous()
            X = torch.zeros_like(B) if X0 is None else X0
            rc = lib().bcmgx_solve_multi(self.h, k, _ptr(B), _ptr(X), 1, infos)
        else:
            B = np.ascontiguousarray(B, dtype=np.float64)
            X = np.zeros_like(B) if X0 is None else np.array(X0, dtype=np.float64, order="C")
            rc = lib().bcmgx_solve_multi(self.h, k, _ptr(B), _ptr(X), 0, infos)
        if rc != L.OK and (rc != L.ERR_NO_CONVERGENCE or raise_on_no_convergence):
            raise BcmgxError(rc, "solve_multi", L.last_error())
        out = [{"retv": i.retv, "niter": i.niter, "delta0": i.delta0, "exit_res": i.exit_res,
                "solve_ms": i.solve_ms, "status": rc} for i in infos]
        return X, out

    def adjoint(self, g, x=None, want_dA=True):
        """lambda = A^{-1} g and dL/dA on A's pattern (-lambda_i x_j), for g = dL/dx."""
        info = L.SolveInfo()
        if _is_device(g):
            import torch
            lam = torch.empty_like(g)
            dA = torch.empty(self.nnz, dtype=torch.float64, device=g.device) if want_dA else None
            rc = lib().bcmgx_solve_adjoint(self.h, _ptr(g), _ptr(x), _ptr(lam), _ptr(dA), 1, C.byref(info))
        else:
            g = np.ascontiguousarray(g, dtype=np.float64)
            lam = np.empty_like(g)
            xx = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
            dA = np.empty(self.nnz) if want_dA else None
            rc = lib().bcmgx_solve_adjoint(self.h, _ptr(g), _ptr(xx), _ptr(lam), _ptr(dA), 0, C.byref(info))
        if rc != L.OK:
            raise BcmgxError(rc, "adjoint solve", L.last_error())
        return lam, dA, {"niter": info.niter, "solve_ms": info.solve_ms}

    def prec_apply(self, r):
        if _is_device(r):
            import torch
            v = torch.empty_like(r)
            check(lib().bcmgx_prec_apply(self.h, _ptr(r), _ptr(v), 1), "prec_apply")
            return v
        r = np.ascontiguousarray(r, dtype=np.float64)
        v = np.empty_like(r)
        check(lib().bcmgx_prec_apply(self.h, _ptr(r), _ptr(v), 0), "prec_apply")
        return v

    # -- inspection -------------------------------------------------------------------------
    def info(self):
        hi = L.HierarchyInfo()
        check(lib().bcmgx_hierarchy_get_info(self.h, C.byref(hi)), "get_info")
        nl = hi.num_levels
        return {"num_levels": nl, "n": list(hi.n[:nl]), "nnz": list(hi.nnz[:nl]),
                "op_cmplx": hi.op_cmplx, "op_wcmplx": hi.op_wcmplx, "avg_cratio": hi.avg_cratio,
                "maxcoarsesize": hi.maxcoarsesize, "ftcoarse": hi.ftcoarse,
                "num_sweep_records": hi.num_sweep_records, "setup_ms": hi.setup_ms,
                "tpr": list(hi.tpr[:nl]), "index_bytes": list(hi.index_bytes[:nl]),
                "value_codes": list(hi.value_codes[:nl])}

    def afsai_factor(self):
        """The AFSAI factor G (CSR row, col, val) of an AFSAI hierarchy."""
        z = C.c_int64()
        check(lib().bcmgx_hierarchy_get_afsai(self.h, C.byref(z), None, None, None), "get_afsai")
        row = np.empty(self.n + 1, np.int32)
        col = np.empty(z.value, np.int32)
        val = np.empty(z.value, np.float64)
        check(lib().bcmgx_hierarchy_get_afsai(self.h, C.byref(z), _ptr(row), _ptr(col), _ptr(val)), "get_afsai")
        return row, col, val

    def level(self, l):
        inf = self.info()
        n, z = inf["n"][l], inf["nnz"][l]
        row = np.empty(n + 1, np.int32)
        col = np.empty(z, np.int32)
        val = np.empty(z, np.float64)
        check(lib().bcmgx_hierarchy_get_level(self.h, l, _ptr(row), _ptr(col), _ptr(val)), "get_level")
        return row, col, val

    def prolongator(self, l):
        n = self.info()["n"][l]
        agg = np.empty(n, np.int32)
        p = np.empty(n)
        M = np.empty(n)
        check(lib().bcmgx_hierarchy_get_prolongator(self.h, l, _ptr(agg), _ptr(p), _ptr(M)),
              "get_prolongator")
        return agg, p, M

    def sweeps(self):
        out = []
        for k in range(self.info()["num_sweep_records"]):
            lv, sw, n, nc = C.c_int(), C.c_int(), C.c_int(), C.c_int()
            check(lib().bcmgx_hierarchy_get_sweep(self.h, k, C.byref(lv), C.byref(sw), C.byref(n),
                                                  C.byref(nc), None, None, None, None), "get_sweep")
            M = np.empty(n.value, np.int32)
            agg = np.empty(n.value, np.int32)
            p = np.empty(n.value)
            w = np.empty(n.value)
            check(lib().bcmgx_hierarchy_get_sweep(self.h, k, None, None, None, None, _ptr(M),
                                                  _ptr(agg), _ptr(p), _ptr(w)), "get_sweep")
            out.append({"level": lv.value, "sweep": sw.value, "nc": nc.value, "match": M,
                        "agg": agg, "p": p, "w": w})
        return out

    def time_kernels(self, level=0, reps=20):
        """Average ms per launch of the level's Jacobi sweep, residual, FP64 SpMV, and on level 0
        the FCG SpMV+dots, the FP32 cycle's sweep with FP64 output and the FCG update."""
        out = np.zeros(6)
        check(lib().bcmgx_time_kernels(self.h, level, reps, _ptr(out)), "bcmgx_time_kernels")
        return {"jacobi": out[0], "residual": out[1], "spmv": out[2], "fcg_spmv_dots": out[3],
                "jacobi_fp64_out": out[4], "fcg_update": out[5]}

    def time_block_kernels(self, nrhs=32, reps=20):
        """Average ms per launch of the level-0 block Jacobi sweep, block residual, FP64 block SpMM
        and block FCG SpMV+dots for nrhs right-hand sides."""
        out = np.zeros(4)
        check(lib().bcmgx_time_block_kernels(self.h, nrhs, reps, _ptr(out)), "bcmgx_time_block_kernels")
        return {"jacobi": out[0], "residual": out[1], "spmm": out[2], "fcg_spmm_dots": out[3]}

    def free(self):
        if getattr(self, "h", None):
            check(lib().bcmgx_free(self.h), "prec_finalize")
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class _Borrowed(Hierarchy):
    """A hierarchy owned by a Batch (not freed by this wrapper)."""

    def __init__(self, handle, n, nnz, params):
        self.h = handle
        self.n = n
        self.nnz = nnz
        self.params = params

    def free(self):
        self.h = None


class Batch:
    """Independent systems whose set-ups run concurrently and whose solves run as one CUDA graph
    launch (bcmgx_setup_batch / bcmgx_batch_solve). systems: list of host (row, col, val).
    lockstep: True (the library's default) runs every step as one kernel over all systems of a
    level-count group (results equal single solves to rounding); False gives every system its own
    graph branch (results equal single solves bit for bit); None keeps the library's default."""

    def __init__(self, systems, params, nthreads=0, lockstep=None):
        arrs = []
        descs = (L.Csr * len(systems))()
        for k, (row, col, val) in enumerate(systems):
            row = np.ascontiguousarray(row, dtype=np.int32)
            col = np.ascontiguousarray(col, dtype=np.int32)
            val = np.ascontiguousarray(val, dtype=np.float64)
            arrs.append((row, col, val))
            n = row.size - 1
            descs[k] = L.Csr(n, n, col.size, _ptr(row), _ptr(col), _ptr(val), 0)
        h = C.c_void_p()
        check(lib().bcmgx_setup_batch(len(systems), descs, C.byref(params), nthreads, C.byref(h)), "batch set-up")
        self.h = h
        self.params = params
        self.sizes = [(r.size - 1, c.size) for r, c, _ in arrs]
        if lockstep is not None:
            self.set_lockstep(lockstep)

    def set_lockstep(self, on):
        check(lib().bcmgx_batch_set_lockstep(self.h, 1 if on else 0), "batch_set_lockstep")

    def __len__(self):
        return len(self.sizes)

    def hierarchy(self, k):
        hh = C.c_void_p()
        check(lib().bcmgx_batch_get_hierarchy(self.h, k, C.byref(hh)), "batch_get_hierarchy")
        return _Borrowed(hh, self.sizes[k][0], self.sizes[k][1], self.params)

    def solve(self, bs, xs=None):
        """bs, xs: lists of CUDA float64 tensors (xs updated in place; zeros when None)."""
        import torch
        if xs is None:
            # one zeroed block for all systems (one fill instead of one per system), split into views
            flat = torch.zeros(sum(int(b.numel()) for b in bs), dtype=torch.float64, device=bs[0].device)
            xs = list(flat.split([int(b.numel()) for b in bs]))
        m = len(bs)
        pb = (C.c_void_p * m)(*[b.data_ptr() for b in bs])
        px = (C.c_void_p * m)(*[x.data_ptr() for x in xs])
        infos = (L.SolveInfo * m)()
        rc = lib().bcmgx_batch_solve(self.h, pb, px, infos)
        if rc not in (L.OK, L.ERR_NO_CONVERGENCE):
            raise BcmgxError(rc, "batch solve", L.last_error())
        return xs, [{"niter": i.niter, "retv": i.retv, "exit_res": i.exit_res, "delta0": i.delta0,
                     "solve_ms": i.solve_ms, "status": rc} for i in infos]

    def free(self):
        if getattr(self, "h", None):
            check(lib().bcmgx_batch_free(self.h), "batch_free")
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Dist:
    """The row-partitioned (multi-rank) set-up and solve: the reference's prec_setup / solve at
    np > 1, FP64 V-cycle (bcmgx_dist_*).

    Dist.local(row, col, val, offsets, params): all ranks' row blocks in this process on one device
    (offsets: the ranks' first rows, ending with n). Dist.nccl(row, col, val, row_offset, n_global,
    comm, nranks, params): this rank's rows (global column ids) on its own GPU, comm from
    nccl_comm()."""

    def __init__(self, h, params, nrows, nranks):
        self.h = h
        self.params = params
        self.n = nrows
        self.nranks = nranks

    @classmethod
    def local(cls, row, col, val, offsets, params):
        dev = _is_device(row)
        if not dev:
            row = np.ascontiguousarray(row, dtype=np.int32)
            col = np.ascontiguousarray(col, dtype=np.int32)
            val = np.ascontiguousarray(val, dtype=np.float64)
        n = int(row.shape[0]) - 1
        A = L.Csr(n, n, int(col.shape[0]), _ptr(row), _ptr(col), _ptr(val), 1 if dev else 0)
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        h = C.c_void_p()
        check(lib().bcmgx_dist_setup_local(C.byref(A), off.size - 1, _ptr(off), C.byref(params), C.byref(h)),
              "dist_setup_local")
        return cls(h, params, n, off.size - 1)

    @classmethod
    def nccl(cls, row, col, val, row_offset, n_global, comm, nranks, params):
        dev = _is_device(row)
        if not dev:
            row = np.ascontiguousarray(row, dtype=np.int32)
            col = np.ascontiguousarray(col, dtype=np.int32)
            val = np.ascontiguousarray(val, dtype=np.float64)
        n = int(row.shape[0]) - 1
        A = L.Csr(n, int(n_global), int(col.shape[0]), _ptr(row), _ptr(col), _ptr(val), 1 if dev else 0)
        h = C.c_void_p()
        check(lib().bcmgx_dist_setup_nccl(C.byref(A), int(row_offset), int(n_global), comm, C.byref(params),
                                          C.byref(h)), "dist_setup_nccl")
        return cls(h, params, n, nranks)

    def solve(self, b, x0=None, raise_on_no_convergence=False):
        info = L.SolveInfo()
        if _is_device(b):
            import torch
            x = torch.zeros_like(b) if x0 is None else x0
            rc = lib().bcmgx_dist_solve(self.h, _ptr(b), _ptr(x), 1, C.byref(info))
        else:
            b = np.ascontiguousarray(b, dtype=np.float64)
            x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
            rc = lib().bcmgx_dist_solve(self.h, _ptr(b), _ptr(x), 0, C.byref(info))
        if rc != L.OK and (rc != L.ERR_NO_CONVERGENCE or raise_on_no_convergence):
            raise BcmgxError(rc, "dist solve", L.last_error())
        return x, {"retv": info.retv, "niter": info.niter, "delta0": info.delta0, "exit_res": info.exit_res,
                   "solve_ms": info.solve_ms, "status": rc}

    def info(self):
        inf = L.HierarchyInfo()
        check(lib().bcmgx_dist_get_info(self.h, C.byref(inf)), "dist_get_info")
        k = inf.num_levels
        return {"num_levels": k, "n": list(inf.n[:k]), "nnz": list(inf.nnz[:k]), "op_cmplx": inf.op_cmplx,
                "maxcoarsesize": inf.maxcoarsesize, "ftcoarse": inf.ftcoarse, "setup_ms": inf.setup_ms}

    def level(self, l):
        """This process's rows of level l with global column ids, and the level's rank offsets."""
        rows, nnz = C.c_int(), C.c_int64()
        check(lib().bcmgx_dist_get_level(self.h, l, C.byref(rows), C.byref(nnz), None, None, None, None),
              "dist_get_level")
        row = np.empty(rows.value + 1, np.int32)
        col = np.empty(nnz.value, np.int32)
        val = np.empty(nnz.value, np.float64)
        off = np.empty(self.nranks + 1, np.int64)
        check(lib().bcmgx_dist_get_level(self.h, l, C.byref(rows), C.byref(nnz), _ptr(row), _ptr(col), _ptr(val),
                                         _ptr(off)), "dist_get_level")
        return row, col, val, off

    def prolongator(self, l, rows):
        agg = np.empty(rows, np.int32)
        p = np.empty(rows)
        M = np.empty(rows)
        check(lib().bcmgx_dist_get_prolongator(self.h, l, _ptr(agg), _ptr(p), _ptr(M)), "dist_get_prolongator")
        return agg, p, M

    def free(self):
        if getattr(self, "h", None):
            check(lib().bcmgx_dist_free(self.h), "dist_free")
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def nccl_unique_id() -> bytes:
    buf = (C.c_ubyte * 128)()
    check(lib().bcmgx_nccl_unique_id(buf), "nccl_unique_id")
    return bytes(buf)


def nccl_comm(nranks, rank, uid: bytes):
    """An NCCL communicator for bcmgx_dist_setup_nccl on the current device."""
    buf = (C.c_ubyte * 128).from_buffer_copy(uid)
    c = C.c_void_p()
    check(lib().bcmgx_nccl_comm_init(nranks, rank, buf, C.byref(c)), "nccl_comm_init")
    return c


def nccl_comm_destroy(comm):
    check(lib().bcmgx_nccl_comm_destroy(comm), "nccl_comm_destroy")


def prec_setup(row, col, val, params) -> Hierarchy:
    return Hierarchy(row, col, val, params)


def solve(h: Hierarchy, rhs, x0=None):
    return h.solve(rhs, x0)


def prec_finalize(h: Hierarchy):
    h.free()


# ---------------------------------------------------------------------------------------------
# kernels on caller-owned device memory (CUDA torch tensors)
# ---------------------------------------------------------------------------------------------
def _stream_ptr(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def spmv(row, col, val, x, y, alpha=1.0, beta=0.0, threads_per_row=0, stream=None):
    n = int(row.shape[0]) - 1
    check(lib().bcmgx_spmv(n, int(x.shape[0]), int(col.shape[0]), _ptr(row), _ptr(col), _ptr(val),
                           _ptr(x), _ptr(y), alpha, beta, threads_per_row, _stream_ptr(stream)),
          "bcmgx_spmv")
    return y


def spmm(row, col, val, X, Y, alpha=1.0, beta=0.0, stream=None):
    """Y = alpha A X + beta Y for row-major blocks X (m x k) and Y (n x k), k <= 32 (CUDA tensors)."""
    n = int(row.shape[0]) - 1
    check(lib().bcmgx_spmm(n, int(X.shape[0]), int(col.shape[0]), _ptr(row), _ptr(col), _ptr(val),
                           int(X.shape[1]), _ptr(X), _ptr(Y), alpha, beta, _stream_ptr(stream)),
          "bcmgx_spmm")
    return Y


def edge_weights(row, col, val, w, stream=None):
    import torch
    W = torch.empty_like(val)
    mn = C.c_double()
    n = int(row.shape[0]) - 1
    check(lib().bcmgx_edge_weights(n, int(col.shape[0]), _ptr(row), _ptr(col), _ptr(val), _ptr(w),
                                   _ptr(W), C.byref(mn), _stream_ptr(stream)), "bcmgx_edge_weights")
    return W, mn.value


def suitor_matching(row, col, W, stream=None):
    import torch
    n = int(row.shape[0]) - 1
    M = torch.empty(n, dtype=torch.int32, device=row.device)
    check(lib().bcmgx_suitor_matching(n, int(col.shape[0]), _ptr(row), _ptr(col), _ptr(W), _ptr(M),
                                      _stream_ptr(stream)), "bcmgx_suitor_matching")
    return M
