"""The sliced row kernels (32-row slices, one lane per row, sliced.cuh) against the plain row
kernel with one thread per row (rowops.cuh k_rowop<1>). Both add each row's entries in CSR order
with the same multiply-adds, so whole set-ups and solves must agree bit for bit. BCMGX_TPR=64
forces the sliced kernels on every level, BCMGX_TPR=1 the plain kernel with one thread per row."""
import numpy as np
import pytest

from test_gpu_parity import fcg
from test_gpu_staged import matrix, setup_solve, CASES

pytestmark = pytest.mark.gpu

SLICED = 64


@pytest.fixture(autouse=True)
def multi_launch_cycle(monkeypatch):
    """These tests exercise the cycle's own kernels: the persistent coarse cycle stays off."""
    monkeypatch.setenv("BCMGX_PERSIST_NNZ", "0")


# the 27- and 7-point cases above a million entries keep one-byte value codes on level 0 (the
# sliced copy then streams codes); the others store their values (FP32 and FP64 sliced copies)
SLICED_CASES = CASES + [("lap27", (44, 40, 36)), ("lap7", (120, 110, 100))]


@pytest.mark.parametrize("prec", ["FP64", "FP32"])
@pytest.mark.parametrize("case", SLICED_CASES)
def test_sliced_solve_bit_identical(bx, cuda, monkeypatch, case, prec):
    """Every level on the sliced kernels gives the one-thread-per-row kernel's iterations and
    solution bit for bit (V-cycle sweeps and residuals, the FCG SpMV)."""
    A = matrix(bx, case)
    n = A.shape[0]
    b = A @ np.random.default_rng(3).uniform(-1, 1, n)
    x0, i0, h0 = setup_solve(bx, monkeypatch, A, b, 1, vcycle_precision=prec, rtol=1e-8)
    x1, i1, h1 = setup_solve(bx, monkeypatch, A, b, SLICED, vcycle_precision=prec, rtol=1e-8)
    assert h0["tpr"] == [1] * h0["num_levels"] and h1["tpr"] == [SLICED] * h1["num_levels"]
    if case == ("lap27", (44, 40, 36)):
        # a coded 27-point level: pattern-indexed rows (index_bytes 0: one byte per row)
        assert h1["value_codes"][0] > 0 and h1["index_bytes"][0] == 0
    if case[0] == "far":
        assert h1["index_bytes"][0] == 4
    assert i0["status"] == 0 and i1["status"] == 0
    assert i0["niter"] == i1["niter"]
    assert np.array_equal(x0, x1)
    assert np.linalg.norm(b - A @ x1) <= 1e-8 * np.linalg.norm(b) * 1.0001


@pytest.mark.parametrize("op", ["spmv", "prec"])
def test_sliced_spmv_and_cycle_on_device_vectors(bx, cuda, monkeypatch, op):
    """A level-0 SpMV through the hierarchy's FCG kernel path and one V-cycle application on
    device vectors: sliced and one-thread-per-row hierarchies agree bit for bit, on a coded
    27-point matrix with a ragged last slice (rows not a multiple of 32)."""
    import torch
    A = matrix(bx, ("lap27", (45, 41, 37)))
    n = A.shape[0]
    assert n % 32 != 0
    r = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, n)).to(cuda)
    outs = []
    for code in (1, SLICED):
        monkeypatch.setenv("BCMGX_TPR", str(code))
        h = bx.prec_setup(A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data,
                          fcg(bx, vcycle_precision="FP32", rtol=1e-8))
        monkeypatch.delenv("BCMGX_TPR")
        if op == "prec":
            outs.append(h.prec_apply(r).cpu().numpy())
        else:
            x, _ = h.solve(r.clone())
            outs.append(x.cpu().numpy())
        h.free()
    assert np.array_equal(outs[0], outs[1])


def test_sliced_hierarchies_in_batch_graph(bx, cuda, monkeypatch):
    """Hierarchies set up for the sliced kernels: the batch graph captures the CSR kernel with one
    thread per row, their single solves the sliced kernels; both give the same results bit for
    bit, and the batch leaves the hierarchies sliced."""
    import torch
    from test_gpu_batch import _systems
    systems = _systems(bx, 4, 22, lo=20, hi=34)
    p = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=1e-8, dispnorm=0, vcycle_precision="FP32")
    monkeypatch.setenv("BCMGX_TPR", str(SLICED))
    B = bx.Batch(systems, p, nthreads=2, lockstep=False)
    singles = [bx.prec_setup(r, c, v, p) for r, c, v in systems]
    monkeypatch.delenv("BCMGX_TPR")
    rng = np.random.default_rng(9)
    bs = [torch.from_numpy(rng.uniform(-1, 1, r.size - 1)).to(cuda) for r, _, _ in systems]
    xs, infos = B.solve(bs)
    for k, h in enumerate(singles):
        assert h.info()["tpr"][0] == SLICED
        x, info = h.solve(bs[k].clone())
        assert info["niter"] == infos[k]["niter"]
        assert torch.equal(x, xs[k])
        h.free()
    B.free()


def test_sliced_timing_hooks(bx, cuda, monkeypatch):
    """The kernel timing hook runs the level's sliced kernels (positive times on every level)."""
    A = matrix(bx, ("lap27", (44, 40, 36)))
    monkeypatch.setenv("BCMGX_TPR", str(SLICED))
    h = bx.prec_setup(A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data,
                      fcg(bx, vcycle_precision="FP32", rtol=1e-8))
    monkeypatch.delenv("BCMGX_TPR")
    for l in range(h.info()["num_levels"]):
        t = h.time_kernels(l, reps=2)
        assert t["jacobi"] > 0 and t["residual"] > 0
    h.free()
