"""Many right-hand sides of one system: the CSR SpMM kernel (bcmgx_spmm) and the block FCG
(bcmgx_solve_multi), checked column by column against scipy, the oracle's FCG and the
single-vector solve."""
import numpy as np
import pytest

from test_gpu_parity import as_csr, fcg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", [1, 5, 32])
@pytest.mark.parametrize("case", [("lap27", (14, 13, 12)), ("rand", (3000, 0.004, 3)), ("rand", (1500, 0.04, 4))])
def test_spmm_matches_scipy(bx, cuda, case, k):
    """Y = alpha A X + beta Y against scipy in FP64 (entries summed in row order: 1e-14 relative).
    The last matrix has about 60 entries per row, more than a warp step stages in shared memory,
    so its products read the entries from global memory."""
    import torch
    A = as_csr(bx, case)
    n = A.shape[0]
    rng = np.random.default_rng(k)
    X = rng.uniform(-1, 1, (n, k))
    Y0 = rng.uniform(-1, 1, (n, k))
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    row, col, val = d(A.indptr.astype(np.int32)), d(A.indices.astype(np.int32)), d(A.data)
    Yd = d(Y0)
    bx.spmm(row, col, val, d(X), Yd, alpha=-0.5, beta=2.0)
    torch.cuda.synchronize()
    ref = -0.5 * (A @ X) + 2.0 * Y0
    got = Yd.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-14 * (np.abs(A) @ np.abs(X)).max() * 4 + 1e-14 * np.abs(Y0).max() * 4


@pytest.mark.parametrize("case", [("lap27", (20, 20, 20)), ("lap7", (30, 30, 30)), ("diff", (20, 2))])
@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_multi_solve_matches_single_and_oracle(bx, oracle, cuda, case, prec):
    """Each column of a 9-column block solve: the same iterations as the single-vector solve of
    that column (+-1), its solution within 1e-9 of it, the true residual at the tolerance, and
    (FP64 cycle) the oracle's FCG iterations +-1 and solution within 1e-6."""
    A = as_csr(bx, case)
    n = A.shape[0]
    k = 9
    rng = np.random.default_rng(11)
    B = A @ rng.uniform(-1, 1, (n, k))
    B[:, 3] *= 1e6   # column scaling must not change that column's iterations
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-8, vcycle_precision=prec))
    X, infos = h.solve_multi(B)
    if prec == "FP64":
        Ho = oracle.Hierarchy(oracle.Matrix.from_csr(A.indptr, A.indices, A.data), oracle.params(rtol=1e-8))
    for j in range(k):
        b = B[:, j].copy()
        x, info = h.solve(b)
        assert infos[j]["status"] == 0
        assert abs(infos[j]["niter"] - info["niter"]) <= 1, (j, infos[j]["niter"], info["niter"])
        assert np.linalg.norm(b - A @ X[:, j]) <= 1e-8 * np.linalg.norm(b) * 1.0001
        tol = 1e-9 if infos[j]["niter"] == info["niter"] else 1e-6
        assert np.linalg.norm(X[:, j] - x) / np.linalg.norm(x) < tol
        assert abs(infos[j]["delta0"] - info["delta0"]) <= 1e-12 * info["delta0"]
        if prec == "FP64" and j in (0, 3, 8):
            xo, io = Ho.solve(b)
            assert abs(infos[j]["niter"] - io["niter"]) <= 1
            assert np.linalg.norm(X[:, j] - xo) / np.linalg.norm(xo) < 1e-6


@pytest.mark.parametrize("pre", ["L1_JACOBI", "AFSAI", "NONE"])
@pytest.mark.parametrize("case", [("lap27", (16, 16, 16)), ("diff", (16, 2))])
def test_multi_solve_other_preconditioners(bx, cuda, case, pre):
    """The standalone l1-Jacobi and AFSAI preconditioners (and none) on a 6-column block solve: each
    column reaches the tolerance in the iterations of the single-vector solve with the same
    preconditioner, to within 2 % (at least 1), and its solution is within 1e-7 of the single solve's
    when the counts agree, else no more than 10x further from x* than the single solve's. The block
    kernels sum a row in entry order, the single-vector ones over S lanes; with these weak
    preconditioners the heterogeneous diffusion matrix takes over 300 iterations, over which that
    rounding difference moves the count by a few iterations."""
    A = as_csr(bx, case)
    n = A.shape[0]
    k = 6
    Xt = np.random.default_rng(12).uniform(-1, 1, (n, k))
    B = A @ Xt
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-8, preconditioner=pre, l1jacsweeps=3))
    X, infos = h.solve_multi(B)
    for j in range(k):
        b = B[:, j].copy()
        x, info = h.solve(b)
        assert infos[j]["status"] == 0
        slack = max(1, int(np.ceil(0.02 * info["niter"])))
        assert abs(infos[j]["niter"] - info["niter"]) <= slack, (j, infos[j]["niter"], info["niter"])
        assert np.linalg.norm(b - A @ X[:, j]) <= 1e-8 * np.linalg.norm(b) * 1.0001
        if infos[j]["niter"] == info["niter"]:
            assert np.linalg.norm(X[:, j] - x) / np.linalg.norm(x) < 1e-7
        else:
            xt = Xt[:, j]
            e_single = max(np.linalg.norm(x - xt), 1e-12 * np.linalg.norm(xt))
            assert np.linalg.norm(X[:, j] - xt) <= 10 * e_single


def test_multi_columns_independent_and_deterministic(bx, cuda):
    """Identical columns give bit-identical results; a zero column stops at once with x = x0 = 0;
    host and device entry points agree bit for bit; the block graph is rebuilt when k changes
    (another padded width sums the SpMM entries in another order: equal to rounding only)."""
    import torch
    A = as_csr(bx, ("lap27", (16, 16, 16)))
    n = A.shape[0]
    b = A @ np.random.default_rng(2).uniform(-1, 1, n)
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-8, vcycle_precision="FP32"))
    B = np.stack([b, b, np.zeros(n), b, 3.0 * b], axis=1)
    X, infos = h.solve_multi(B)
    for j in (1, 3):
        assert np.array_equal(X[:, j], X[:, 0])
    assert not X[:, 2].any() and infos[2]["niter"] == 1 and infos[2]["delta0"] == 0.0
    assert abs(infos[4]["niter"] - infos[0]["niter"]) <= 1
    assert all(i["status"] == 0 for i in infos)
    X2, _ = h.solve_multi(B[:, :2])           # another k: new workspace and graph
    X3, _ = h.solve_multi(B)                  # back to 5 columns
    assert np.array_equal(X3, X)
    assert np.linalg.norm(X2[:, 0] - X[:, 0]) <= 1e-9 * np.linalg.norm(X[:, 0])
    Bd = torch.from_numpy(B).to(cuda)
    Xd = torch.zeros_like(Bd)
    h.solve_multi(Bd, Xd)
    assert np.array_equal(Xd.cpu().numpy(), X)


def test_multi_nonzero_x0_and_no_preconditioner(bx, cuda):
    """A nonzero x0 per column and preconditioner NONE (plain CG on the block) against single solves."""
    A = as_csr(bx, ("lap7", (12, 12, 12)))
    n = A.shape[0]
    rng = np.random.default_rng(5)
    B = rng.uniform(-1, 1, (n, 4))
    X0 = rng.uniform(-1, 1, (n, 4))
    for pre in ("BCMG", "NONE"):
        h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-9, preconditioner=pre))
        X, infos = h.solve_multi(B, X0)
        for j in range(4):
            x, info = h.solve(B[:, j].copy(), X0[:, j].copy())
            assert abs(infos[j]["niter"] - info["niter"]) <= 1
            tol = 1e-9 if infos[j]["niter"] == info["niter"] else 1e-6
            assert np.linalg.norm(X[:, j] - x) / np.linalg.norm(x) < tol


def test_multi_bad_arguments(bx, cuda):
    A = as_csr(bx, ("lap7", (6, 6, 6)))
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx))
    for k in (0, 33):
        with pytest.raises(bx.BcmgxError) as e:
            h.solve_multi(np.ones((A.shape[0], k)))
        assert e.value.code == -1


@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_multi_graph_and_stream_drivers_agree(bx, cuda, prec):
    """The captured block solve (WHILE conditional node) and the stream-driven one run the same
    kernels: identical iterations and solutions."""
    A = as_csr(bx, ("lap27", (18, 18, 18)))
    B = A @ np.random.default_rng(8).uniform(-1, 1, (A.shape[0], 6))
    out = {}
    for g in (0, 1):
        h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-9, use_graph=g, vcycle_precision=prec))
        X, infos = h.solve_multi(B)
        out[g] = (X, [i["niter"] for i in infos])
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])


def test_block_kernel_timing_hook(bx, cuda):
    """bcmgx_time_block_kernels times the four level-0 block kernels; a solve afterwards is unchanged."""
    A = as_csr(bx, ("lap27", (20, 20, 20)))
    B = np.random.default_rng(8).uniform(-1, 1, (A.shape[0], 5))
    p = bx.params_default(solver="FCG", rtol=1e-9, dispnorm=0, vcycle_precision="FP32")
    h = bx.prec_setup(A.indptr, A.indices, A.data, p)
    X0, _ = h.solve_multi(B)
    t = h.time_block_kernels(5, reps=3)
    assert all(t[key] > 0 for key in ("jacobi", "residual", "spmm", "fcg_spmm_dots")), t
    X1, _ = h.solve_multi(B)
    assert np.array_equal(X0, X1)
    with pytest.raises(bx.BcmgxError):
        h.time_block_kernels(33)
