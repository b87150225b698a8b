"""Failure detection on the GPU path, exercised without a GPU fault.

Every failure is made on the host or by a bounded device wait that runs out on purpose:
* a NaN in the right-hand side ends the solve with BCMGX_ERR_NOT_SPD (both solve drivers), and
  the hierarchy then solves a proper right-hand side;
* an injected allocation failure (BCMGX_TEST_FAIL_ALLOC=k fails the k-th device allocation of a
  set-up) makes bcmgx_setup return BCMGX_ERR_OOM at every point of the set-up, and after 100 such
  set-ups the device memory pool holds no more than before;
* a suitor step budget of 0 (BCMGX_TEST_SUITOR_BUDGET) makes the matching give up and the set-up
  return BCMGX_ERR_TIMEOUT;
* the staged row kernels' stage waits (BCMGX_TEST_STAGE_FAULT=<ns> drops block 0's first tile copy
  and shortens the producer's and consumers' waits; the drain of copies in flight keeps its
  one-second limit) run out: the solve returns BCMGX_ERR_TIMEOUT, and the next solve on the same
  context succeeds.
The reference has no counterpart: it exits on every error (BCMGX/src/utility/mpi.h:25-32).
"""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def multi_launch_cycle(monkeypatch):
    """These tests exercise the cycle's own kernels: the persistent coarse cycle stays off."""
    monkeypatch.setenv("BCMGX_PERSIST_NNZ", "0")

OOM, TIMEOUT, NOT_SPD = -6, -5, -7


def fcg(bx, **kw):
    kw.setdefault("solver", "FCG")
    kw.setdefault("preconditioner", "BCMG")
    kw.setdefault("dispnorm", 0)
    return bx.params_default(**kw)


def lap(bx, st, g):
    row, col, val = bx.laplacian_3d(st, *g)
    n = row.size - 1
    return row, col, val, sp.csr_matrix((val, col, row), shape=(n, n))


def pool_used_bytes():
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(0)
    assert err == rt.cudaError_t.cudaSuccess
    err, v = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    assert err == rt.cudaError_t.cudaSuccess
    return int(v)


@pytest.mark.parametrize("use_graph", [0, 1])
def test_nan_in_rhs(bx, cuda, use_graph):
    row, col, val, A = lap(bx, 27, (12, 12, 12))
    n = A.shape[0]
    h = bx.prec_setup(row, col, val, fcg(bx, rtol=1e-8, use_graph=use_graph))
    b = np.ones(n)
    b[n // 3] = np.nan
    with pytest.raises(bx.BcmgxError) as e:
        h.solve(b)
    assert e.value.code == NOT_SPD
    xs = np.random.default_rng(0).uniform(-1, 1, n)
    x, info = h.solve(A @ xs)
    assert info["status"] == 0
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-6
    h.free()


def test_injected_allocation_failure(bx, cuda, monkeypatch):
    import torch
    row, col, val, A = lap(bx, 7, (14, 13, 12))
    prm = fcg(bx, rtol=1e-8)
    h = bx.prec_setup(row, col, val, prm)    # the first set-up fills the process-wide caches
    h.free()
    torch.cuda.synchronize()
    base = pool_used_bytes()
    failed = 0
    for k in range(1, 101):
        monkeypatch.setenv("BCMGX_TEST_FAIL_ALLOC", str(k))
        try:
            h = bx.prec_setup(row, col, val, prm)
        except bx.BcmgxError as e:
            assert e.code == OOM, (k, e.code, str(e))
            assert "BCMGX_TEST_FAIL_ALLOC" in str(e)
            failed += 1
        else:
            assert failed == k - 1   # once a set-up needs fewer allocations, none fails any more
            h.free()
        torch.cuda.synchronize()
        assert pool_used_bytes() <= base, k
    monkeypatch.delenv("BCMGX_TEST_FAIL_ALLOC")
    assert failed >= 20
    h = bx.prec_setup(row, col, val, prm)
    xs = np.random.default_rng(1).uniform(-1, 1, A.shape[0])
    x, info = h.solve(A @ xs)
    assert info["status"] == 0
    h.free()


def test_suitor_budget_exhausted(bx, cuda, monkeypatch):
    row, col, val, A = lap(bx, 27, (10, 10, 10))
    monkeypatch.setenv("BCMGX_TEST_SUITOR_BUDGET", "0")
    with pytest.raises(bx.BcmgxError) as e:
        bx.prec_setup(row, col, val, fcg(bx))
    assert e.value.code == TIMEOUT
    monkeypatch.delenv("BCMGX_TEST_SUITOR_BUDGET")
    h = bx.prec_setup(row, col, val, fcg(bx))
    x, info = h.solve(np.ones(A.shape[0]))
    assert info["status"] == 0
    h.free()


@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_staged_stage_wait_times_out(bx, cuda, monkeypatch, prec):
    row, col, val, A = lap(bx, 27, (24, 24, 24))
    n = A.shape[0]
    xs = np.random.default_rng(2).uniform(-1, 1, n)
    b = A @ xs
    monkeypatch.setenv("BCMGX_TPR", "-4")          # the staged row kernel on every level
    prm = fcg(bx, rtol=1e-8, itnlim=2, use_graph=0, vcycle_precision=prec)
    h = bx.prec_setup(row, col, val, prm)
    assert all(t == -4 for t in h.info()["tpr"])
    monkeypatch.setenv("BCMGX_TEST_STAGE_FAULT", "2000000")   # 2 ms waits, block 0's first tile dropped
    with pytest.raises(bx.BcmgxError) as e:
        h.solve(b, raise_on_no_convergence=True)
    assert e.value.code == TIMEOUT and "stage" in str(e.value)
    monkeypatch.delenv("BCMGX_TEST_STAGE_FAULT")
    h.free()
    # the same context goes on: a full solve through the staged kernels
    h = bx.prec_setup(row, col, val, fcg(bx, rtol=1e-8, vcycle_precision=prec))
    x, info = h.solve(b)
    assert info["status"] == 0
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-6
    h.free()
