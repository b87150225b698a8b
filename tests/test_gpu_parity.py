"""GPU parity of libbcmgx.so against the CPU oracle and the reference's golden solutions.

Tolerances: integer results (matchings, aggregates, hierarchy sizes, patterns) and the set-up
values (weights, prolongators, Galerkin matrices) are compared bit for bit; solve-phase vectors
within 1e-12 relative for one V-cycle (different summation order only), iteration counts within
one, solutions within the reference's 1e-5 compareSolutions threshold against the goldens.
"""
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import ROOT

pytestmark = pytest.mark.gpu

GRIDS = [(1, 1, 1), (2, 1, 1), (2, 2, 1), (2, 2, 2)]


def fcg(bx, **kw):
    kw.setdefault("solver", "FCG")
    kw.setdefault("preconditioner", "BCMG")
    kw.setdefault("dispnorm", 0)
    return bx.params_default(**kw)


def random_spd(n, density, seed, ragged=False):
    rng = np.random.default_rng(seed)
    B = sp.random(n, n, density=density, random_state=rng, format="csr")
    if ragged:   # a few long rows
        for r in rng.choice(n, 5, replace=False):
            B[r, rng.choice(n, min(n - 1, 60), replace=False)] = rng.random(min(n - 1, 60))
    B = (B + B.T).tocsr()
    B.data = -np.abs(B.data)
    d = np.asarray(abs(B).sum(axis=1)).ravel() + 0.5 + rng.random(n)
    A = (B + sp.diags(d)).tocsr()
    A.sort_indices()
    return A


def arrow(n, k, seed):
    """SPD tridiagonal band plus k dense rows and columns (rows of n entries)."""
    rng = np.random.default_rng(seed)
    i = np.arange(n - 1)
    B = sp.csr_matrix((-rng.uniform(0.5, 1.5, n - 1), (i, i + 1)), shape=(n, n)).tolil()
    for r in rng.choice(n, k, replace=False):
        B[r, :] = -rng.uniform(0, 0.01, n)
    B = B.tocsr()
    B.setdiag(0)
    B.eliminate_zeros()
    B = (B + B.T).tocsr()
    d = np.asarray(abs(B).sum(axis=1)).ravel() + 0.5
    A = (B + sp.diags(d)).tocsr()
    A.sort_indices()
    return A


def heterogeneous(bx, n, seed):
    rng = np.random.default_rng(seed)
    kappa = np.exp(1.5 * rng.normal(size=n ** 3))
    row, col, val = bx.diffusion_7p(n, n, n, kappa)
    return sp.csr_matrix((val, col, row), shape=(n ** 3, n ** 3))


def as_csr(bx, case):
    kind, arg = case
    if kind == "lap7":
        r, c, v = bx.laplacian_3d(7, *arg)
    elif kind == "lap27":
        r, c, v = bx.laplacian_3d(27, *arg)
    elif kind == "rand":
        A = random_spd(*arg)
        r, c, v = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data
    elif kind == "arrow":
        A = arrow(*arg)
        r, c, v = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data
    else:
        A = heterogeneous(bx, *arg)
        r, c, v = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data
    n = r.size - 1
    return sp.csr_matrix((v, c, r), shape=(n, n))


def to_dev(torch, A, cuda):
    return (torch.from_numpy(A.indptr.astype(np.int32)).to(cuda), torch.from_numpy(A.indices.astype(np.int32)).to(cuda),
            torch.from_numpy(A.data.astype(np.float64)).to(cuda))


# ----------------------------------------------------------------------------------------------
@pytest.mark.parametrize("st", [7, 27])
@pytest.mark.parametrize("PQR", GRIDS)
def test_golden_solutions(bx, cuda, golden, st, PQR):
    """A x = 1 with FCG_BCMG.properties settings reproduces the reference's solution files
    (BCMGX/src/test/data/cmp/lap3d_*_sol.txt) within compareSolutions' 1e-5."""
    row, col, val = bx.laplacian_3d(st, 10, 10, 10, *PQR)
    h = bx.prec_setup(row, col, val, fcg(bx))
    x, info = h.solve(np.ones(row.size - 1))
    g = golden[f"sol__lap3d_{st}p_10x10x10_{PQR[0]}x{PQR[1]}x{PQR[2]}_sol"]
    assert info["status"] == 0 and info["retv"] == 0
    assert np.linalg.norm(x - g) / np.linalg.norm(g) < 1e-5


def test_bcsstk09_golden(bx, oracle, cuda, golden, tmp_path):
    """bcsstk09 read by the library's MatrixMarket reader and solved on the GPU (A x = 1, FCG+BCMG)
    reproduces BCMGX/src/test/data/cmp/bcsstk09_sol.txt within compareSolutions' 1e-5, in the
    oracle's iterations (+-1)."""
    path = tmp_path / "bcsstk09.mtx"
    path.write_text(str(golden["mtxtext__bcsstk09"]))
    row, col, val = bx.read_matrix_market(path)
    n = row.size - 1
    h = bx.prec_setup(row, col, val, fcg(bx))
    x, info = h.solve(np.ones(n))
    g = golden["sol__bcsstk09_sol"]
    assert info["status"] == 0 and info["retv"] == 0
    assert np.linalg.norm(x - g) / np.linalg.norm(g) < 1e-5
    Ho = oracle.Hierarchy(oracle.Matrix.from_csr(row, col, val), oracle.params())
    _, io = Ho.solve(np.ones(n))
    assert abs(info["niter"] - io["niter"]) <= 1


@pytest.mark.parametrize("tpr", [1, 2, 4, 8, 16, 32])
@pytest.mark.parametrize("case", [("lap27", (12, 11, 10)), ("rand", (3000, 0.004, 1, True)), ("lap7", (1, 1, 1))])
def test_spmv(bx, cuda, tpr, case):
    import torch
    A = as_csr(bx, case)
    r, c, v = to_dev(torch, A, cuda)
    rng = np.random.default_rng(tpr)
    x = rng.uniform(-1, 1, A.shape[1])
    y0 = rng.uniform(-1, 1, A.shape[0])
    for alpha, beta in [(1.0, 0.0), (-1.0, 1.0), (0.5, -2.0)]:
        y = torch.from_numpy(y0.copy()).to(cuda)
        bx.spmv(r, c, v, torch.from_numpy(x).to(cuda), y, alpha, beta, tpr)
        ref = alpha * (A @ x) + beta * y0
        got = y.cpu().numpy()
        assert np.max(np.abs(got - ref)) <= 1e-13 * (np.max(np.abs(ref)) + 1)


def test_spmv_empty_rows(bx, cuda):
    import torch
    A = sp.csr_matrix(np.diag([1.0, 0, 2.0, 0, 0, 3.0]))
    A.eliminate_zeros()
    r, c, v = to_dev(torch, A, cuda)
    y = torch.full((6,), 7.0, dtype=torch.float64, device=cuda)
    bx.spmv(r, c, v, torch.ones(6, dtype=torch.float64, device=cuda), y, 1.0, 0.0, 4)
    assert y.cpu().numpy().tolist() == [1.0, 0.0, 2.0, 0.0, 0.0, 3.0]


CASES = [("lap7", (14, 13, 12)), ("lap27", (11, 12, 10)), ("rand", (2500, 0.003, 3)),
         ("diff", (12, 5))]


@pytest.mark.parametrize("case", CASES)
def test_weights_and_matching(bx, oracle, cuda, case):
    """Edge weights: same minimum and values (log may differ by an ulp between CUDA and libm);
    the suitor matching computed on the GPU's weights equals the oracle's greedy matching on
    the same weights, bit for bit."""
    import torch
    A = as_csr(bx, case)
    n = A.shape[0]
    r, c, v = to_dev(torch, A, cuda)
    w = np.random.default_rng(7).uniform(0.5, 2.0, n)
    Wg, mng = bx.edge_weights(r, c, v, torch.from_numpy(w).to(cuda))
    Wg = Wg.cpu().numpy()
    Mo = oracle.Matrix.from_csr(A.indptr, A.indices, A.data)
    Wo, mno = Mo.edge_weights(w)
    assert mng == mno
    ulps = np.abs(Wg.view(np.int64) - Wo.view(np.int64))
    assert ulps.max() <= 1
    Mg = bx.suitor_matching(r, c, torch.from_numpy(Wg).to(cuda)).cpu().numpy()
    Mgreedy = Mo.match(Wg, 0)
    assert np.array_equal(Mg, Mgreedy)
    m = Mg >= 0
    assert np.all(Mg[Mg[m]] == np.nonzero(m)[0])


@pytest.mark.parametrize("case", [("lap7", (20, 20, 20)), ("lap27", (16, 16, 16)), ("lap7", (9, 30, 7)),
                                  ("rand", (3000, 0.003, 5)), ("diff", (14, 9)), ("rand", (1500, 0.05, 9)),
                                  ("arrow", (3000, 4, 5)), ("arrow", (10000, 3, 7))])
def test_hierarchy_bit_exact(bx, oracle, cuda, case):
    """Every sweep's matching, aggregates, prolongator values and weight vector, every level's
    matrix and the composite prolongators equal the oracle's bit for bit. The sixth matrix has
    about 150 entries per row: its sweeps store the edge weights (rows over 32 entries), run the
    matching kernels on whole warps and the Galerkin product with 64-bit keys (over 128 candidate
    entries per coarse row). The arrow matrices have dense rows of 3000 and 10000 entries: the
    coarse rows holding them exceed a warp's 512 candidates in the first Galerkin launch and go to
    the second (one warp per block), and those over a block's 7314 to the global-memory path
    (candidates sorted per row with CUB's segmented sort)."""
    A = as_csr(bx, case)
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, record_sweeps=1))
    Ao = oracle.Matrix.from_csr(A.indptr, A.indices, A.data)
    Ho = oracle.Hierarchy(Ao, oracle.params(), record=True)
    gi = h.info()
    assert [(n, z) for n, z in zip(gi["n"], gi["nnz"])] == Ho.level_sizes()
    so, sg = Ho.records(), h.sweeps()
    assert len(so) == len(sg)
    for a, b in zip(so, sg):
        assert (a["level"], a["sweep"], a["nc"]) == (b["level"], b["sweep"], b["nc"])
        assert np.array_equal(a["w"], b["w"])
        assert np.array_equal(a["match"], b["match"])
        assert np.array_equal(a["agg"], b["agg"])
        assert np.array_equal(a["p"], b["p"])
    for l in range(gi["num_levels"]):
        rg, cg, vg = h.level(l)
        ro, co, vo = Ho.level_matrix(l).csr()
        assert np.array_equal(rg, ro) and np.array_equal(cg, co) and np.array_equal(vg, vo)
        ag, pg, Mg = h.prolongator(l) if l + 1 < gi["num_levels"] else (None, None, None)
        ao, po, Mo = Ho.prolongator(l)
        if ag is not None:
            assert np.array_equal(ag, ao) and np.array_equal(pg, po) and np.array_equal(Mg, Mo)
    st = Ho.stats()
    assert gi["maxcoarsesize"] == st["maxcoarsesize"] and gi["ftcoarse"] == st["ftcoarse"]
    assert abs(gi["op_cmplx"] - st["op_cmplx"]) < 1e-12


def test_long_row_in_a_large_matrix(bx, oracle, cuda):
    """A 7-point 100^3 Laplacian with one row coupled to 2000 others: the Galerkin scratch is the
    fine matrix's entries (not the coarse rows times the longest row, which here would be 24 GB),
    the levels match the oracle's sizes and the solve reaches the tolerance."""
    r, c, v = bx.laplacian_3d(7, 100, 100, 100)
    n = r.size - 1
    rng = np.random.default_rng(4)
    k = 12345
    cols = rng.choice(np.setdiff1d(np.arange(n), [k]), 2000, replace=False)
    B = sp.csr_matrix((-0.01 * np.ones(2000), (np.full(2000, k), cols)), shape=(n, n))
    B = (B + B.T).tocsr()
    A = (sp.csr_matrix((v, c, r), shape=(n, n)) + B + sp.diags(np.asarray(abs(B).sum(axis=1)).ravel())).tocsr()
    A.sort_indices()
    row, col = A.indptr.astype(np.int32), A.indices.astype(np.int32)
    h = bx.prec_setup(row, col, A.data, fcg(bx, rtol=1e-8))
    Ho = oracle.Hierarchy(oracle.Matrix.from_csr(row, col, A.data), oracle.params())
    gi = h.info()
    assert [(n_, z) for n_, z in zip(gi["n"], gi["nnz"])] == Ho.level_sizes()
    b = A @ rng.uniform(-1, 1, n)
    x, info = h.solve(b)
    assert info["status"] == 0
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b) * 1.0001
    h.free()


@pytest.mark.parametrize("cycle", ["V_CYCLE", "H_CYCLE", "W_CYCLE", "VARIABLE_V_CYCLE"])
def test_vcycle_application(bx, oracle, cuda, cycle):
    A = as_csr(bx, ("lap27", (18, 17, 16)))
    prm = fcg(bx, cycle_type=cycle)
    h = bx.prec_setup(A.indptr, A.indices, A.data, prm)
    Ho = oracle.Hierarchy(oracle.Matrix.from_csr(A.indptr, A.indices, A.data), oracle.params(cycle_type=cycle))
    rv = np.random.default_rng(1).uniform(-1, 1, A.shape[0])
    vg = h.prec_apply(rv)
    vo = Ho.vcycle(rv)
    assert np.linalg.norm(vg - vo) / np.linalg.norm(vo) < 1e-12


@pytest.mark.parametrize("case", [("lap7", (30, 30, 30)), ("lap27", (24, 24, 24)), ("diff", (20, 2)),
                                  ("rand", (5000, 0.002, 9))])
@pytest.mark.parametrize("cycle", ["V_CYCLE", "W_CYCLE"])
def test_solve_matches_oracle(bx, oracle, cuda, case, cycle):
    A = as_csr(bx, case)
    n = A.shape[0]
    xs = np.random.default_rng(0).uniform(-1, 1, n)
    b = A @ xs
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-8, cycle_type=cycle))
    x, info = h.solve(b)
    Ho = oracle.Hierarchy(oracle.Matrix.from_csr(A.indptr, A.indices, A.data), oracle.params(rtol=1e-8, cycle_type=cycle))
    xo, io = Ho.solve(b)
    assert info["status"] == 0
    assert abs(info["niter"] - io["niter"]) <= 1
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b) * 1.0001
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-6
    assert abs(info["delta0"] - io["delta0"]) <= 1e-12 * io["delta0"]


@pytest.mark.parametrize("case", [("lap27", (32, 32, 32)), ("lap7", (40, 40, 40)), ("diff", (24, 4))])
def test_fp32_vcycle(bx, cuda, case):
    """FP32 V-cycle inside FP64 FCG: iterations within 10% (+1) of the FP64 cycle, solution
    error vs x* no worse than 10x the FP64 one, true residual at the tolerance."""
    A = as_csr(bx, case)
    n = A.shape[0]
    xs = np.random.default_rng(1).uniform(-1, 1, n)
    b = A @ xs
    out = {}
    for prec in ("FP64", "FP32"):
        h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-8, vcycle_precision=prec))
        x, info = h.solve(b)
        assert info["status"] == 0
        out[prec] = (x, info)
    i64, i32 = out["FP64"][1]["niter"], out["FP32"][1]["niter"]
    assert i32 <= 1.1 * i64 + 1
    e64 = np.linalg.norm(out["FP64"][0] - xs) / np.linalg.norm(xs)
    e32 = np.linalg.norm(out["FP32"][0] - xs) / np.linalg.norm(xs)
    assert e32 < 10 * e64 + 1e-12
    assert np.linalg.norm(b - A @ out["FP32"][0]) <= 1e-8 * np.linalg.norm(b) * 1.0001


def test_device_pointers_and_prec_none(bx, cuda):
    import torch
    A = as_csr(bx, ("lap7", (16, 16, 16)))
    r, c, v = to_dev(torch, A, cuda)
    xs = np.random.default_rng(3).uniform(-1, 1, A.shape[0])
    b = torch.from_numpy(A @ xs).to(cuda)
    h = bx.prec_setup(r, c, v, fcg(bx, rtol=1e-10))
    x, info = h.solve(b)
    assert x.is_cuda and info["status"] == 0
    assert np.linalg.norm(x.cpu().numpy() - xs) / np.linalg.norm(xs) < 1e-7
    h2 = bx.prec_setup(r, c, v, fcg(bx, rtol=1e-10, preconditioner="NONE"))
    x2, info2 = h2.solve(b)
    assert info2["status"] == 0 and info2["niter"] > info["niter"]
    assert np.linalg.norm(x2.cpu().numpy() - xs) / np.linalg.norm(xs) < 1e-7


def test_error_paths(bx, cuda):
    A = as_csr(bx, ("lap7", (6, 6, 6)))
    n = A.shape[0]
    # no diagonal in row 3
    B = A.tolil()
    B[3, 3] = 0
    B = B.tocsr()
    B.eliminate_zeros()
    with pytest.raises(bx.BcmgxError) as e:
        bx.prec_setup(B.indptr, B.indices, B.data, fcg(bx))
    assert e.value.code == -1 and "diagonal" in str(e.value)
    # unsorted columns
    c = A.indices.copy()
    c[A.indptr[5]], c[A.indptr[5] + 1] = c[A.indptr[5] + 1], c[A.indptr[5]]
    with pytest.raises(bx.BcmgxError) as e:
        bx.prec_setup(A.indptr, c, A.data, fcg(bx))
    assert e.value.code == -1
    # invalid solver / unsupported preconditioner
    with pytest.raises(bx.BcmgxError) as e:
        bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, solver=7))
    assert e.value.code == -1
    with pytest.raises(bx.BcmgxError) as e:
        bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, preconditioner=9))
    assert e.value.code == -1
    # itnlim reached: status NO_CONVERGENCE, retv -1 as SolverOut
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-14, itnlim=2))
    x, info = h.solve(np.ones(n))
    assert info["status"] == -3 and info["retv"] == -1 and info["niter"] == 3
    with pytest.raises(bx.BcmgxError):
        h.solve(np.ones(n), raise_on_no_convergence=True)


def test_cli_matches_golden(golden, cuda, tmp_path):
    cfg = tmp_path / "lap.cfg"
    cfg.write_text("nx = 10\nny = 10\nnz = 10\nP = 2\nQ = 2\nR = 1\n")
    props = tmp_path / "FCG_BCMG.properties"
    props.write_text(str(golden["prop__FCG_BCMG.properties"]))
    sol = tmp_path / "sol.txt"
    info = tmp_path / "info.txt"
    cli = os.path.join(ROOT, "bootcmatchgx_b200", "bin", "bcmgx_driverSolve")
    r = subprocess.run([cli, "-g", "27p", "-l", str(cfg), "-s", str(props), "-o", str(sol), "-i", str(info)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    x = np.loadtxt(sol)
    g = golden["sol__lap3d_27p_10x10x10_2x2x1_sol"]
    assert np.linalg.norm(x - g) / np.linalg.norm(g) < 1e-5
    text = info.read_text()
    assert "Total iterations" in text and "Number of levels" in text and "TOTAL SOLVE TIME" in text


@pytest.mark.parametrize("case", [("lap27", (20, 20, 20)), ("diff", (18, 3)), ("lap7", (3, 3, 3))])
@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_graph_and_stream_drivers_agree(bx, cuda, case, prec):
    """The graph-captured solve (WHILE conditional node) and the stream solve (one-iteration
    lookahead) run the same kernels: identical iterations and identical solutions. A second solve
    on the same hierarchy relaunches the captured graph."""
    A = as_csr(bx, case)
    b = A @ np.random.default_rng(4).uniform(-1, 1, A.shape[0])
    out = {}
    for g in (0, 1):
        h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-9, use_graph=g, vcycle_precision=prec))
        x1, i1 = h.solve(b)
        x2, i2 = h.solve(2.0 * b)
        assert i1["status"] == 0 and i2["status"] == 0
        out[g] = (x1, i1["niter"], x2, i2["niter"])
    assert out[0][1] == out[1][1] and out[0][3] == out[1][3]
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][2], out[1][2])


def test_suitor_with_a_row_of_65536_entries(bx, oracle, cuda):
    """A row of 70,000 entries (an arrowhead pattern over a chain) takes the suitor with 32-bit
    offer words; its matching on given symmetric weights equals the oracle's greedy matching.
    Most weights of the long row are <= 0 (no candidates), so its ranking stays short."""
    import torch
    n = 70000
    rng = np.random.default_rng(21)
    i = np.arange(n - 1)
    chain = sp.coo_matrix((np.ones(n - 1), (i, i + 1)), shape=(n, n))
    arrow = sp.coo_matrix((np.ones(n - 2), (np.zeros(n - 2, int), np.arange(2, n))), shape=(n, n))
    U = (chain + arrow).tocsr()
    U.data = rng.uniform(-2.0, 2.0, U.nnz)
    U[0, 2:] = -np.abs(U[0, 2:].toarray())
    U[0, rng.choice(np.arange(2, n), 100, replace=False)] = rng.uniform(0.5, 2.0, 100)
    W = (U + U.T + sp.identity(n)).tocsr()   # symmetric weights on a symmetric pattern, with a diagonal
    W.sort_indices()
    assert np.diff(W.indptr).max() >= 65536
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    Mg = bx.suitor_matching(d(W.indptr.astype(np.int32)), d(W.indices.astype(np.int32)), d(W.data)).cpu().numpy()
    Mo = oracle.Matrix.from_csr(W.indptr, W.indices, np.ones(W.nnz)).match(W.data, 0)
    assert np.array_equal(Mg, Mo)
    m = Mg >= 0
    assert m.sum() > n // 2 and np.all(Mg[Mg[m]] == np.nonzero(m)[0])
