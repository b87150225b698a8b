"""The reference's other Krylov solvers (CGHS, the s-step CG behind CGS / PIPELINED_CGS /
CGS_CUBLAS) and preconditioners (standalone l1-Jacobi, AFSAI), against the oracle's
restatements of cghs/CG_HS.cu, cgs/CGs.cu, l1jacobi/l1jacobi.cu and afsai/afsai.cu."""
import numpy as np
import pytest

from test_gpu_parity import as_csr

pytestmark = pytest.mark.gpu

SOLVERS = [("CGHS", 1), ("CGS", 1), ("CGS", 2), ("CGS", 4), ("PIPELINED_CGS", 2), ("CGS_CUBLAS", 3)]


def _params(bx, **kw):
    kw.setdefault("dispnorm", 0)
    return bx.params_default(**kw)


def _oracle_params(oracle, **kw):
    return oracle.params(**kw)


@pytest.mark.parametrize("case", [("lap7", (20, 20, 20)), ("lap27", (14, 14, 14)), ("diff", (16, 2))])
@pytest.mark.parametrize("pre", ["BCMG", "L1_JACOBI", "AFSAI", "NONE"])
@pytest.mark.parametrize("solver,s", SOLVERS)
def test_solver_matches_oracle(bx, oracle, cuda, case, pre, solver, s):
    """Status, iterations within +-1 (5 % without a preconditioner: hundreds of iterations on the
    ill-conditioned diffusion matrix, where the summation order of the dot products, which for
    the oracle depends on the host's thread count, and the single-precision square root of the
    s-step scalar work move the count) and the solution within 1e-6 of the oracle (1e-5 without
    a preconditioner: cond(A) * rtol is larger there). Both stop at rtol 1e-8. An s-step basis
    whose moment matrix is not positive definite ends the solve in both."""
    A = as_csr(bx, case)
    n = A.shape[0]
    b = A @ np.random.default_rng(3).uniform(-1, 1, n)
    kw = dict(solver=solver, preconditioner=pre, sstep=s, rtol=1e-8)
    h = bx.prec_setup(A.indptr, A.indices, A.data, _params(bx, **kw))
    Ho = oracle.Hierarchy(oracle.Matrix.from_csr(A.indptr, A.indices, A.data), _oracle_params(oracle, **kw))
    xo, io = Ho.solve(b)
    if io["retv"] == 1:   # moment matrix not positive definite
        with pytest.raises(bx.BcmgxError) as e:
            h.solve(b, raise_on_no_convergence=True)
        assert e.value.code == -7
        return
    x, info = h.solve(b)
    assert io["retv"] == 0 and info["status"] == 0, (io, info)
    slack = max(1, round((0.05 if pre == "NONE" else 0.02) * io["niter"]))
    assert abs(info["niter"] - io["niter"]) <= slack, (info["niter"], io["niter"])
    assert np.linalg.norm(b - A @ x) < 1e-8 * np.linalg.norm(b) * 1.0001
    xtol = 1e-5 if pre == "NONE" else 1e-6
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < xtol
    assert abs(info["delta0"] - io["delta0"]) <= 1e-12 * io["delta0"]


@pytest.mark.parametrize("variant", [dict(ru_res=0), dict(rec_res_int=3), dict(stop_criterion=0, rtol=1e-6)])
@pytest.mark.parametrize("pre", ["L1_JACOBI", "NONE"])
def test_sstep_residual_options(bx, oracle, cuda, variant, pre):
    """ru_res = 0 (residual recomputed every iteration), rec_res_int (recomputed every k-th) and
    stop_criterion = 0 (absolute tolerance) against the oracle."""
    A = as_csr(bx, ("lap7", (18, 18, 18)))
    n = A.shape[0]
    b = A @ np.random.default_rng(4).uniform(-1, 1, n)
    kw = dict(solver="CGS", preconditioner=pre, sstep=2, rtol=1e-8)
    kw.update(variant)
    h = bx.prec_setup(A.indptr, A.indices, A.data, _params(bx, **kw))
    Ho = oracle.Hierarchy(oracle.Matrix.from_csr(A.indptr, A.indices, A.data), _oracle_params(oracle, **kw))
    xo, io = Ho.solve(b)
    x, info = h.solve(b)
    assert io["retv"] == 0 and info["status"] == 0
    assert abs(info["niter"] - io["niter"]) <= 1
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-5
    assert info["delta0"] == pytest.approx(io["delta0"], rel=1e-12)


def test_l1jacobi_preconditioner_application(bx, oracle, cuda):
    """One application of the standalone l1-Jacobi preconditioner (l1jacsweeps sweeps from zero
    with D = a_ii + sum |a_ij|, j != i) against the oracle, also on a matrix with a negative
    diagonal entry, where D differs from the absolute row sum."""
    A = as_csr(bx, ("rand", (3000, 0.003, 5))).tolil()
    A[7, 7] = -A[7, 7]
    A = A.tocsr()
    A.sort_indices()
    r = np.random.default_rng(6).uniform(-1, 1, A.shape[0])
    for k in (1, 2, 5):
        kw = dict(solver="FCG", preconditioner="L1_JACOBI", l1jacsweeps=k)
        h = bx.prec_setup(A.indptr, A.indices, A.data, _params(bx, **kw))
        Ho = oracle.Hierarchy(oracle.Matrix.from_csr(A.indptr, A.indices, A.data), _oracle_params(oracle, **kw))
        v = h.prec_apply(r)
        vo = Ho.vcycle(r)
        assert np.linalg.norm(v - vo) / np.linalg.norm(vo) < 1e-13


@pytest.mark.parametrize("solver,s", [("CGHS", 1), ("CGS", 2)])
@pytest.mark.parametrize("pre", ["BCMG", "NONE"])
def test_graph_and_stream_drivers_agree(bx, cuda, solver, s, pre):
    """The captured solve and the stream-driven one run the same kernels: identical iterates; a
    second solve relaunches the captured graph."""
    A = as_csr(bx, ("lap27", (16, 16, 16)))
    b = A @ np.random.default_rng(7).uniform(-1, 1, A.shape[0])
    out = {}
    for g in (0, 1):
        h = bx.prec_setup(A.indptr, A.indices, A.data, _params(bx, solver=solver, sstep=s, preconditioner=pre,
                                                                rtol=1e-9, use_graph=g))
        x1, i1 = h.solve(b)
        x2, i2 = h.solve(3.0 * b)
        out[g] = (x1, i1["niter"], x2, i2["niter"])
    assert out[0][1] == out[1][1] and out[0][3] == out[1][3]
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][2], out[1][2])


@pytest.mark.parametrize("case", [("lap7", (12, 12, 12)), ("lap27", (10, 9, 8)), ("diff", (12, 2)),
                                  ("rand", (2000, 0.004, 8))])
def test_afsai_factor_bit_exact(bx, oracle, cuda, case):
    """The AFSAI factor G (pattern and values) equals the oracle's restatement bit for bit:
    every step is separately rounded on both sides, and ties in the gradient go to the smallest
    column on both. Its application G^T G r agrees to rounding."""
    A = as_csr(bx, case)
    kw = dict(solver="FCG", preconditioner="AFSAI")
    h = bx.prec_setup(A.indptr, A.indices, A.data, _params(bx, **kw))
    Ho = oracle.Hierarchy(oracle.Matrix.from_csr(A.indptr, A.indices, A.data), _oracle_params(oracle, **kw))
    row, col, val = h.afsai_factor()
    ro, co, vo = Ho.afsai_factor()
    assert np.array_equal(row, ro) and np.array_equal(col, co)
    assert np.array_equal(val, vo)
    assert (np.diff(row) <= 31).all() and (np.diff(row) >= 1).all()
    r = np.random.default_rng(9).uniform(-1, 1, A.shape[0])
    v, vo_ = h.prec_apply(r), Ho.vcycle(r)
    assert np.linalg.norm(v - vo_) / np.linalg.norm(vo_) < 1e-13


def test_solver_parameter_errors(bx, cuda):
    A = as_csr(bx, ("lap7", (6, 6, 6)))
    B = A.copy()
    B.data[B.indices == np.repeat(np.arange(B.shape[0]), np.diff(B.indptr))] *= -1.0
    with pytest.raises(bx.BcmgxError) as e:
        bx.prec_setup(B.indptr, B.indices, B.data, _params(bx, preconditioner="AFSAI"))
    assert e.value.code == -1 and "diagonal" in str(e.value)
    for kw, code in ((dict(preconditioner=9), -1), (dict(solver="CGS", sstep=9), -1),
                     (dict(solver="CGS", sstep=0), -1), (dict(preconditioner="L1_JACOBI", l1jacsweeps=0), -1)):
        with pytest.raises(bx.BcmgxError) as e:
            bx.prec_setup(A.indptr, A.indices, A.data, _params(bx, **kw))
        assert e.value.code == code, kw
    p = _params(bx, solver="CGHS")
    with pytest.raises(bx.BcmgxError) as e:
        bx.Batch([(A.indptr, A.indices, A.data)], p)
    assert e.value.code == -2
