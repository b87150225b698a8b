"""The staged row kernels (matrix entries streamed through shared-memory stages by bulk async
copies, staged.cuh) against the plain row kernels (rowops.cuh). With the same threads per row both
sum every row in the same order, so whole set-ups and solves must agree bit for bit. The
environment variable BCMGX_TPR forces the kernel on every level: S for the plain kernel, -S for the
staged one."""
import numpy as np
import pytest
import scipy.sparse as sp

from test_gpu_parity import as_csr, fcg

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def multi_launch_cycle(monkeypatch):
    """These tests exercise the cycle's own kernels: the persistent coarse cycle stays off."""
    monkeypatch.setenv("BCMGX_PERSIST_NNZ", "0")


def far_columns(n, seed):
    """SPD, each row coupled to its neighbours and to the row n/2 away: column offsets beyond
    int16, so level 0 keeps int32 columns."""
    rng = np.random.default_rng(seed)
    i = np.arange(n)
    rows = np.concatenate([i, i, i])
    cols = np.concatenate([(i + 1) % n, (i - 1) % n, (i + n // 2) % n])
    B = sp.csr_matrix((-rng.uniform(0.5, 1.5, rows.size), (rows, cols)), shape=(n, n))
    B = (B + B.T).tocsr()
    d = np.asarray(abs(B).sum(axis=1)).ravel() + 0.1
    A = (B + sp.diags(d)).tocsr()
    A.sort_indices()
    return A


def matrix(bx, case):
    kind, arg = case
    if kind == "far":
        return far_columns(*arg)
    return as_csr(bx, case)


def setup_solve(bx, monkeypatch, A, b, code, **kw):
    monkeypatch.setenv("BCMGX_TPR", str(code))
    try:
        h = bx.prec_setup(A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data, fcg(bx, **kw))
    finally:
        monkeypatch.delenv("BCMGX_TPR")
    x, info = h.solve(b.copy())
    hi = h.info()
    h.free()
    return x, info, hi


# the arrow matrix's dense rows (3000 entries) hold more entries than a stage: their tiles are read
# from global memory
CASES = [("lap27", (23, 17, 19)), ("lap7", (40, 33, 31)), ("diff", (24, 3)), ("rand", (5000, 0.01, 2, True)),
         ("far", (80000, 4)), ("arrow", (3000, 4, 5))]


@pytest.mark.parametrize("prec", ["FP64", "FP32"])
@pytest.mark.parametrize("S", [1, 2, 4, 8])
@pytest.mark.parametrize("case", CASES)
def test_staged_solve_bit_identical(bx, cuda, monkeypatch, case, S, prec):
    """Every level on the staged kernel with S threads per row gives the plain kernel's
    iterations and solution bit for bit (set-up, V-cycle sweeps and residuals, FCG residual)."""
    A = matrix(bx, case)
    n = A.shape[0]
    b = A @ np.random.default_rng(3).uniform(-1, 1, n)
    x0, i0, h0 = setup_solve(bx, monkeypatch, A, b, S, vcycle_precision=prec, rtol=1e-8)
    x1, i1, h1 = setup_solve(bx, monkeypatch, A, b, -S, vcycle_precision=prec, rtol=1e-8)
    assert h0["tpr"] == [S] * h0["num_levels"] and h1["tpr"] == [-S] * h1["num_levels"]
    if case[0] == "far":
        assert h0["index_bytes"][0] == 4
    assert i0["status"] == 0 and i1["status"] == 0
    assert i0["niter"] == i1["niter"]
    assert np.array_equal(x0, x1)
    assert np.linalg.norm(b - A @ x1) <= 1e-8 * np.linalg.norm(b) * 1.0001


def test_staged_hierarchies_in_batch_graph(bx, cuda, monkeypatch):
    """Hierarchies set up for the staged kernel: the batch graph captures the plain row kernels
    (side by side with other systems), their single solves (also graph-captured) the staged ones;
    both give the same results bit for bit, and the batch leaves the hierarchies staged."""
    import torch
    from test_gpu_batch import _systems
    systems = _systems(bx, 4, 21, lo=20, hi=34)
    p = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=1e-8, dispnorm=0, vcycle_precision="FP32")
    monkeypatch.setenv("BCMGX_TPR", "-4")
    B = bx.Batch(systems, p, nthreads=2, lockstep=False)
    singles = [bx.prec_setup(r, c, v, p) for r, c, v in systems]
    monkeypatch.delenv("BCMGX_TPR")
    rng = np.random.default_rng(8)
    bs = [torch.from_numpy(rng.uniform(-1, 1, r.size - 1)).to(cuda) for r, _, _ in systems]
    xs, infos = B.solve(bs)
    for k, h in enumerate(singles):
        x, info = h.solve(bs[k])
        assert info["niter"] == infos[k]["niter"]
        assert torch.equal(x, xs[k])
        h.free()
    assert B.hierarchy(0).info()["tpr"][0] == -4
    x1, i1 = B.hierarchy(0).solve(bs[0])
    assert i1["niter"] == infos[0]["niter"] and torch.equal(x1, xs[0])
    B.free()


def test_autotuned_codes_are_reported(bx, cuda):
    """With the autotuner on (the default), every level reports a threads-per-row code of the
    plain (1..32), the staged (-1, -2, -4, -8) or the sliced (64) kernel."""
    A = as_csr(bx, ("lap27", (40, 40, 40)))
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, vcycle_precision="FP32"))
    for t in h.info()["tpr"]:
        assert t in (1, 2, 4, 8, 16, 32, -1, -2, -4, -8, 64)
    h.free()


def test_forced_codes_per_level(bx, cuda, monkeypatch):
    """BCMGX_TPR takes one code per level; levels past the list take its last code, so the list
    spelled out to every level gives the same codes and the same solution bit for bit; a malformed
    list is an invalid input."""
    A = as_csr(bx, ("lap27", (40, 40, 40)))
    b = np.random.default_rng(5).uniform(-1, 1, A.shape[0])
    monkeypatch.setenv("BCMGX_TPR", "-2,4")
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, vcycle_precision="FP32"))
    tpr = h.info()["tpr"]
    assert len(tpr) >= 3 and tpr[:2] == [-2, 4] and all(t == 4 for t in tpr[2:])
    x1, i1 = h.solve(b)
    h.free()
    monkeypatch.setenv("BCMGX_TPR", "-2," + ",".join(["4"] * (len(tpr) - 1)))
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, vcycle_precision="FP32"))
    assert h.info()["tpr"] == tpr
    x2, i2 = h.solve(b)
    h.free()
    assert i1["niter"] == i2["niter"] and np.array_equal(x1, x2)
    monkeypatch.setenv("BCMGX_TPR", "-2,x")
    with pytest.raises(bx.BcmgxError) as e:
        bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx))
    assert e.value.code == -1 and "BCMGX_TPR" in str(e.value)


# matrices of at least 2^20 entries with few distinct values: their row kernels stream one-byte
# value codes (value-indexed CSR) on the large levels
CODED = [("lap27", (40, 40, 40)), ("lap7", (110, 100, 100)), ("shift", (100, 100, 100))]


def coded_matrix(bx, case):
    kind, arg = case
    if kind == "shift":   # 7-point Laplacian with a per-row diagonal shift taking 7 values
        A = as_csr(bx, ("lap7", arg)).tocsr()
        d = A.diagonal() + 0.125 * (np.arange(A.shape[0]) % 7)
        A.setdiag(d)
        A.sort_indices()
        return A
    return as_csr(bx, case)


def solve_with_codes(bx, monkeypatch, A, b, codes, tpr, **kw):
    monkeypatch.setenv("BCMGX_VALUE_CODES", "1" if codes else "0")
    if tpr:
        monkeypatch.setenv("BCMGX_TPR", str(tpr))
    try:
        h = bx.prec_setup(A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data, fcg(bx, **kw))
    finally:
        monkeypatch.delenv("BCMGX_VALUE_CODES")
        if tpr:
            monkeypatch.delenv("BCMGX_TPR")
    x, info = h.solve(b.copy())
    hi = h.info()
    h.free()
    return x, info, hi


@pytest.mark.parametrize("prec", ["FP64", "FP32"])
@pytest.mark.parametrize("tpr", [0, -4, 4, -1])
@pytest.mark.parametrize("case", CODED)
def test_value_codes_bit_identical(bx, cuda, monkeypatch, case, tpr, prec):
    """Level matrices with at most 256 distinct values stream one-byte codes into a table of those
    values (value-indexed CSR); the set-up and the solve give the same iterations and solution
    bit for bit as with the stored values, on the staged and the plain row kernels (tpr 0: the
    autotuner's choice)."""
    A = coded_matrix(bx, case)
    b = A @ np.random.default_rng(9).uniform(-1, 1, A.shape[0])
    xc, ic, hc = solve_with_codes(bx, monkeypatch, A, b, True, tpr, rtol=1e-8, vcycle_precision=prec)
    xs, is_, hs = solve_with_codes(bx, monkeypatch, A, b, False, tpr, rtol=1e-8, vcycle_precision=prec)
    assert hc["value_codes"][0] > 0 and all(v == 0 for v in hs["value_codes"])
    assert ic["status"] == 0 and is_["status"] == 0
    if tpr or hc["tpr"] == hs["tpr"]:
        assert ic["niter"] == is_["niter"]
        assert np.array_equal(xc, xs)
    else:   # the autotuner chose other lanes per row on some level: another summation order
        assert abs(ic["niter"] - is_["niter"]) <= 1
        assert np.linalg.norm(xc - xs) / np.linalg.norm(xs) < 1e-9


def test_value_codes_need_few_values(bx, cuda):
    """A level with more than 256 distinct values keeps its stored values."""
    A = coded_matrix(bx, ("lap7", (110, 100, 100))).tocsr()
    A.data = A.data * (1.0 + 1e-3 * np.random.default_rng(1).random(A.nnz))
    A = ((A + A.T) * 0.5).tocsr()
    A.sort_indices()
    h = bx.prec_setup(A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data, fcg(bx))
    assert h.info()["value_codes"][0] == 0
    h.free()
