"""The persistent coarse cycle (persist.cuh): the cycle's steps on the levels of at most 2^21
entries (BCMGX_PERSIST_NNZ) run in one cooperative kernel with grid barriers between them. Every
step does the arithmetic of the kernel it stands for, so solves equal the multi-launch cycle's
(BCMGX_PERSIST_NNZ=0) bit for bit, for programs of the whole cycle (all levels small) and of its
coarse part, V, W and VARIABLE_V cycles, FP64 and FP32. A barrier wait that runs out (test hook:
block 0 leaves before the first barrier and the others wait 2 ms) ends the solve with
BCMGX_ERR_TIMEOUT, and the next solve succeeds."""
import numpy as np
import pytest

from test_gpu_parity import as_csr, fcg

pytestmark = pytest.mark.gpu


def run(bx, monkeypatch, A, b, persist, **kw):
    monkeypatch.setenv("BCMGX_PERSIST_NNZ", "2097152" if persist else "0")
    try:
        h = bx.prec_setup(A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data, fcg(bx, **kw))
        x, info = h.solve(b.copy())
        x2, info2 = h.solve(2.0 * b)
    finally:
        monkeypatch.delenv("BCMGX_PERSIST_NNZ")
    hi = h.info()
    h.free()
    return x, info, x2, info2, hi


CASES = [("lap7", (50, 50, 50)), ("lap27", (48, 48, 48)), ("diff", (20, 7)), ("rand", (20000, 0.0005, 3))]


@pytest.mark.parametrize("cycle", ["V_CYCLE", "W_CYCLE", "VARIABLE_V_CYCLE"])
@pytest.mark.parametrize("prec", ["FP64", "FP32"])
@pytest.mark.parametrize("case", CASES)
def test_persistent_cycle_bit_identical(bx, cuda, monkeypatch, case, prec, cycle):
    A = as_csr(bx, case)
    b = A @ np.random.default_rng(12).uniform(-1, 1, A.shape[0])
    p = run(bx, monkeypatch, A, b, True, rtol=1e-8, vcycle_precision=prec, cycle_type=cycle)
    m = run(bx, monkeypatch, A, b, False, rtol=1e-8, vcycle_precision=prec, cycle_type=cycle)
    assert p[1]["status"] == 0 and m[1]["status"] == 0
    assert p[1]["niter"] == m[1]["niter"] and p[3]["niter"] == m[3]["niter"]
    assert np.array_equal(p[0], m[0]) and np.array_equal(p[2], m[2])


def test_persistent_barrier_timeout(bx, cuda, monkeypatch):
    A = as_csr(bx, ("lap27", (20, 20, 20)))
    b = A @ np.random.default_rng(13).uniform(-1, 1, A.shape[0])
    monkeypatch.setenv("BCMGX_PERSIST_NNZ", "2097152")
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-8, itnlim=3, use_graph=0))
    monkeypatch.setenv("BCMGX_TEST_PERSIST_FAULT", "2000000")
    with pytest.raises(bx.BcmgxError) as e:
        h.solve(b, raise_on_no_convergence=True)
    assert e.value.code == -5 and "grid barrier" in str(e.value)
    monkeypatch.delenv("BCMGX_TEST_PERSIST_FAULT")
    # the same hierarchy solves again: every solve starts from fresh barrier words
    x, info = h.solve(b)
    assert info["status"] in (0, -3)
    h.free()
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-8))
    x, info = h.solve(b)
    assert info["status"] == 0
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b) * 1.0001
    h.free()
