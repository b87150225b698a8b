"""The CPU oracle against the reference's own fixtures (golden solutions, generator matrices),
and its internal consistency (greedy matching == sequential suitor)."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import golden_mtx

GRIDS = [(1, 1, 1), (2, 1, 1), (2, 2, 1), (2, 2, 2)]


@pytest.mark.parametrize("st", [7, 27])
@pytest.mark.parametrize("PQR", GRIDS)
def test_golden_solutions(oracle, golden, st, PQR):
    """FCG+BCMG on A x = 1 (FCG_BCMG.properties: rtol 1e-6) reproduces
    BCMGX/src/test/data/cmp/lap3d_{st}p_10x10x10_{PxQxR}_sol.txt within compareSolutions' 1e-5."""
    P, Q, R = PQR
    A = oracle.Matrix.lap3d(st, 10, 10, 10, P, Q, R)
    H = oracle.Hierarchy(A, oracle.params())
    x, info = H.solve(np.ones(A.info()[0]))
    g = golden[f"sol__lap3d_{st}p_10x10x10_{P}x{Q}x{R}_sol"]
    assert info["retv"] == 0
    assert np.linalg.norm(x - g) / np.linalg.norm(g) < 1e-5


@pytest.mark.parametrize("name,st,dims", [
    ("lap3d_7p_2x2x5_3x4x2", 7, (2, 2, 5, 3, 4, 2)),
    ("lap3d_7p_4x14x4_2x2x1", 7, (4, 14, 4, 2, 2, 1)),
    ("lap3d_27p_5x5x5_1x2x2", 27, (5, 5, 5, 1, 2, 2)),
    ("lap3d_27p_5x5x5_4x2x1", 27, (5, 5, 5, 4, 2, 1)),
])
def test_generator_fixtures(oracle, golden, name, st, dims):
    """Generator = the Matlab fixtures of BCMGX/testGenerators.mk, bit for bit."""
    M = golden_mtx(golden, name)
    row, col, val = oracle.Matrix.lap3d(st, *dims).csr()
    G = sp.csr_matrix((val, col, row), shape=M.shape)
    assert G.nnz == M.nnz
    assert abs(G - M).max() == 0


def _random_spd(n, density, seed):
    rng = np.random.default_rng(seed)
    B = sp.random(n, n, density=density, random_state=rng, format="csr")
    B = B + B.T
    B.data = -np.abs(B.data)
    d = np.asarray(abs(B).sum(axis=1)).ravel() + 1.0 + rng.random(n)
    A = (B + sp.diags(d)).tocsr()
    A.sort_indices()
    return A


@pytest.mark.parametrize("seed", range(4))
def test_greedy_equals_suitor(oracle, seed):
    A = _random_spd(400, 0.02, seed)
    M_ = oracle.Matrix.from_csr(A.indptr, A.indices, A.data)
    W, mn = M_.edge_weights(np.ones(400) + np.random.default_rng(seed).random(400))
    g = M_.match(W, 0)
    s = M_.match(W, 1)
    assert np.array_equal(g, s)
    m = g >= 0
    assert np.all(g[g[m]] == np.nonzero(m)[0])   # symmetric


def test_ties_prefer_higher_ids(oracle):
    """Equal weights: the suitor tie rule picks the larger id (suitor.cu:108-122), so on a
    path 0-1-2-3 the pairs are (2,3) and (0,1)."""
    row = np.array([0, 2, 5, 8, 10], np.int32)
    col = np.array([0, 1, 0, 1, 2, 1, 2, 3, 2, 3], np.int32)
    val = np.array([2, -1, -1, 2, -1, -1, 2, -1, -1, 2], float)
    A = oracle.Matrix.from_csr(row, col, val)
    W, _ = A.edge_weights(np.ones(4))
    assert list(A.match(W, 0)) == [1, 0, 3, 2]
    assert list(A.match(W, 1)) == [1, 0, 3, 2]


def test_hierarchy_shape_50(oracle):
    """50^3 7-point: maxcoarsesize = (int)(40*50) truncated as AMG.cu:238-241 does."""
    A = oracle.Matrix.lap3d(7, 50, 50, 50)
    H = oracle.Hierarchy(A, oracle.params(rtol=1e-8))
    st = H.stats()
    assert st["maxcoarsesize"] == int(40 * 125000 ** (1 / 3))
    sizes = H.level_sizes()
    assert sizes[0] == (125000, 860000)
    assert sizes[-1][0] <= st["ftcoarse"] * st["maxcoarsesize"]
    x_star = np.random.default_rng(0).uniform(-1, 1, 125000)
    b = A.spmv(x_star)
    x, info = H.solve(b)
    assert info["retv"] == 0
    assert np.linalg.norm(x - x_star) / np.linalg.norm(x_star) < 1e-6


@pytest.mark.parametrize("solver,s", [("CGHS", 1), ("CGS", 1), ("CGS", 3), ("PIPELINED_CGS", 2)])
@pytest.mark.parametrize("pre", ["BCMG", "L1_JACOBI", "NONE"])
def test_oracle_krylov_solvers(oracle, solver, s, pre):
    """The oracle's CGHS and s-step CG reach rtol 1e-8 on a 7-point Poisson system, agree with a
    direct solve, and (s = 1) take the iterations of the oracle's FCG: with a symmetric
    preconditioner the three are the same method."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    M = oracle.Matrix.lap3d(7, 16, 16, 16, 1, 1, 1)
    row, col, val = M.csr()
    A = sp.csr_matrix((val, col, row))
    n = A.shape[0]
    b = A @ np.random.default_rng(1).uniform(-1, 1, n)
    xs = spl.spsolve(A.tocsc(), b)
    H = oracle.Hierarchy(oracle.Matrix.from_csr(row, col, val), oracle.params(rtol=1e-8, solver=solver,
                                                                               preconditioner=pre, sstep=s))
    x, info = H.solve(b)
    assert info["retv"] == 0
    assert np.linalg.norm(b - A @ x) < 1e-8 * np.linalg.norm(b)
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-6
    if s == 1:
        Hf = oracle.Hierarchy(oracle.Matrix.from_csr(row, col, val), oracle.params(rtol=1e-8, solver="FCG",
                                                                                    preconditioner=pre))
        _, fi = Hf.solve(b)
        assert abs(fi["niter"] - info["niter"]) <= 1


def test_bcsstk09_golden(oracle, golden, bx, tmp_path):
    """The --matrix path of driverSolve on bcsstk09 (BCMGX/launchAndCompare.mk:136,207): the
    library's MatrixMarket reader expands the symmetric file exactly as scipy does, and FCG+BCMG
    on A x = 1 reproduces BCMGX/src/test/data/cmp/bcsstk09_sol.txt within compareSolutions' 1e-5."""
    import scipy.io
    path = tmp_path / "bcsstk09.mtx"
    path.write_text(str(golden["mtxtext__bcsstk09"]))
    row, col, val = bx.read_matrix_market(path)
    n = row.size - 1
    ref = scipy.io.mmread(str(path)).tocsr()
    ref.sort_indices()
    assert ref.shape == (n, n)
    assert np.array_equal(row, ref.indptr) and np.array_equal(col, ref.indices) and np.array_equal(val, ref.data)
    H = oracle.Hierarchy(oracle.Matrix.from_csr(row, col, val), oracle.params())
    x, info = H.solve(np.ones(n))
    g = golden["sol__bcsstk09_sol"]
    assert info["retv"] == 0
    assert np.linalg.norm(x - g) / np.linalg.norm(g) < 1e-5


def rank_offsets(nx, ny, nz, P, Q, R):
    """Row offsets of the P*Q*R ranks of the reference's rank-block-major Laplacian."""
    per = nx * ny * nz
    return [k * per for k in range(P * Q * R + 1)]


@pytest.mark.parametrize("st", [7, 27])
@pytest.mark.parametrize("PQR", GRIDS[1:])
def test_partitioned_golden_solutions(oracle, golden, st, PQR):
    """The np = P restatement (rank-local matching and aggregate numbering) on the grids that the
    reference's multi-rank runs produced: each rank holds its 10^3 block, and the solution matches
    BCMGX/src/test/data/cmp/lap3d_{st}p_10x10x10_{PxQxR}_sol.txt within compareSolutions' 1e-5."""
    P, Q, R = PQR
    A = oracle.Matrix.lap3d(st, 10, 10, 10, P, Q, R)
    parts = rank_offsets(10, 10, 10, P, Q, R)
    H = oracle.Hierarchy(A, oracle.params(), parts=parts)
    x, info = H.solve(np.ones(A.info()[0]))
    g = golden[f"sol__lap3d_{st}p_10x10x10_{P}x{Q}x{R}_sol"]
    assert info["retv"] == 0
    assert np.linalg.norm(x - g) / np.linalg.norm(g) < 1e-5
    assert list(H.level_parts(0)) == parts


def test_partitioned_matching_stays_inside_blocks(oracle):
    """Rank-local matching: no aggregate of any sweep crosses a block boundary, each block's
    aggregates are numbered after the previous block's, and one block gives the np = 1 set-up."""
    A = oracle.Matrix.lap3d(27, 9, 8, 7)
    n = A.info()[0]
    one = oracle.Hierarchy(A, oracle.params(), record=True)
    same = oracle.Hierarchy(A, oracle.params(), record=True, parts=[0, n])
    assert one.level_sizes() == same.level_sizes()
    for a, b in zip(one.records(), same.records()):
        assert np.array_equal(a["agg"], b["agg"]) and np.array_equal(a["p"], b["p"])
    parts = [0, 150, 311, n]
    H = oracle.Hierarchy(A, oracle.params(), record=True, parts=parts)
    recs = H.records()
    pt = np.array(parts)
    crossed_somewhere = False
    for r in recs:
        m = r["match"]
        if r["level"] == 0 and r["sweep"] == 0:
            blk = np.searchsorted(pt, np.arange(n), side="right") - 1
            ok = m >= 0
            assert np.all(blk[m[ok]] == blk[ok])
            crossed_somewhere = np.any(one.records()[0]["match"][ok] != m[ok])
            # aggregates of block b are numbered after those of blocks < b
            agg = r["agg"]
            for b in range(3):
                lo, hi = agg[pt[b]:pt[b + 1]].min(), agg[pt[b]:pt[b + 1]].max()
                if b:
                    assert lo == prev_hi + 1
                prev_hi = hi
    assert crossed_somewhere
    lv0 = H.level_parts(1)
    assert lv0[0] == 0 and lv0[-1] == H.level_sizes()[1][0] and len(lv0) == 4
