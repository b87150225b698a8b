"""The row-partitioned multi-rank path (bcmgx_dist_*) against the oracle's np = P set-up.

The reference runs its solver on P MPI ranks, each holding a block of rows; the matching and
the aggregate numbering are rank-local, the rest of the method is the np = 1 arithmetic with halo
exchanges. The local form of the library keeps all ranks' blocks on one GPU with exchanges as
device copies, so the whole partitioned machinery (halo plans, packing, exchanges of vectors and
of prolongator rows, rank-local matching, sums over ranks) runs here:
* every level matrix (global column ids), row partition, composite prolongator and divisor equals
  the oracle's np = P hierarchy bit for bit;
* the FCG solve to 1e-8 takes the oracle's iterations (+-1) and agrees with its solution to 1e-6;
* the reference's multi-rank golden solutions (cmp/lap3d_*_10x10x10_{2x1x1,2x2x1,2x2x2}_sol.txt,
  made at np = 2, 4 and 8) are reproduced on the same rank blocks within 1e-5;
* one rank equals the single-GPU path, and the NCCL transport on a one-rank communicator gives the
  local form's iterates exactly.
"""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def fcg(bx, **kw):
    kw.setdefault("solver", "FCG")
    kw.setdefault("preconditioner", "BCMG")
    kw.setdefault("dispnorm", 0)
    return bx.params_default(**kw)


def matrix(bx, case):
    kind, arg = case
    if kind in ("lap7", "lap27"):
        r, c, v = bx.laplacian_3d(7 if kind == "lap7" else 27, *arg)
        n = r.size - 1
        return sp.csr_matrix((v, c, r), shape=(n, n))
    if kind == "diff":
        g, seed = arg
        rng = np.random.default_rng(seed)
        r, c, v = bx.diffusion_7p(g, g, g, np.exp(1.5 * rng.normal(size=g ** 3)))
        return sp.csr_matrix((v, c, r), shape=(g ** 3, g ** 3))
    n, dens, seed = arg
    rng = np.random.default_rng(seed)
    B = sp.random(n, n, density=dens, random_state=rng, format="csr")
    B = (B + B.T).tocsr()
    B.data = -np.abs(B.data)
    A = (B + sp.diags(np.asarray(abs(B).sum(axis=1)).ravel() + 0.5 + rng.random(n))).tocsr()
    A.sort_indices()
    return A


def offsets(n, cuts):
    return [0] + [int(c * n) for c in cuts] + [n]


CASES = [
    (("lap7", (10, 10, 10, 2, 1, 1)), [0.5]),
    (("lap27", (16, 15, 14)), [0.3, 0.55]),
    (("lap7", (12, 12, 12)), [0.1, 0.4, 0.7]),
    (("rand", (3000, 0.003, 5)), [0.25, 0.5, 0.75]),
    (("diff", (14, 9)), [0.5]),
    (("lap27", (10, 10, 10, 2, 2, 2)), [k / 8 for k in range(1, 8)]),
]


@pytest.mark.parametrize("case,cuts", CASES)
def test_dist_hierarchy_matches_partitioned_oracle(bx, oracle, cuda, case, cuts):
    A = matrix(bx, case)
    n = A.shape[0]
    offs = offsets(n, cuts)
    D = bx.Dist.local(A.indptr, A.indices, A.data, offs, fcg(bx))
    Ho = oracle.Hierarchy(oracle.Matrix.from_csr(A.indptr, A.indices, A.data), oracle.params(), parts=offs)
    gi = D.info()
    assert [(a, b) for a, b in zip(gi["n"], gi["nnz"])] == Ho.level_sizes()
    st = Ho.stats()
    assert gi["maxcoarsesize"] == st["maxcoarsesize"] and gi["ftcoarse"] == st["ftcoarse"]
    for l in range(gi["num_levels"]):
        rg, cg, vg, og = D.level(l)
        ro, co, vo = Ho.level_matrix(l).csr()
        assert np.array_equal(rg, ro) and np.array_equal(cg, co) and np.array_equal(vg, vo), l
        assert np.array_equal(og, Ho.level_parts(l)), l
        if l + 1 < gi["num_levels"]:
            ag, pg, Mg = D.prolongator(l, gi["n"][l])
            ao, po, Mo = Ho.prolongator(l)
            assert np.array_equal(ag, ao) and np.array_equal(pg, po) and np.array_equal(Mg, Mo), l
    D.free()


@pytest.mark.parametrize("case,cuts", CASES)
def test_dist_solve_matches_partitioned_oracle(bx, oracle, cuda, case, cuts):
    A = matrix(bx, case)
    n = A.shape[0]
    offs = offsets(n, cuts)
    xs = np.random.default_rng(3).uniform(-1, 1, n)
    b = A @ xs
    D = bx.Dist.local(A.indptr, A.indices, A.data, offs, fcg(bx, rtol=1e-8))
    x, info = D.solve(b)
    Ho = oracle.Hierarchy(oracle.Matrix.from_csr(A.indptr, A.indices, A.data), oracle.params(rtol=1e-8), parts=offs)
    xo, io = Ho.solve(b)
    assert info["status"] == 0 and io["retv"] == 0
    assert abs(info["niter"] - io["niter"]) <= 1
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b) * 1.0001
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-6
    assert abs(info["delta0"] - io["delta0"]) <= 1e-12 * io["delta0"]
    D.free()


@pytest.mark.parametrize("st", [7, 27])
@pytest.mark.parametrize("PQR", [(2, 1, 1), (2, 2, 1), (2, 2, 2)])
def test_dist_reproduces_multirank_goldens(bx, cuda, golden, st, PQR):
    """A x = 1 with FCG_BCMG settings on the rank blocks of the reference's multi-rank runs."""
    r, c, v = bx.laplacian_3d(st, 10, 10, 10, *PQR)
    P = PQR[0] * PQR[1] * PQR[2]
    offs = [k * 1000 for k in range(P + 1)]
    D = bx.Dist.local(r, c, v, offs, fcg(bx))
    x, info = D.solve(np.ones(r.size - 1))
    g = golden[f"sol__lap3d_{st}p_10x10x10_{PQR[0]}x{PQR[1]}x{PQR[2]}_sol"]
    assert info["status"] == 0
    assert np.linalg.norm(x - g) / np.linalg.norm(g) < 1e-5
    D.free()


def test_dist_one_rank_equals_single_gpu_path(bx, cuda):
    A = matrix(bx, ("lap27", (18, 17, 16)))
    n = A.shape[0]
    b = A @ np.random.default_rng(5).uniform(-1, 1, n)
    D = bx.Dist.local(A.indptr, A.indices, A.data, [0, n], fcg(bx, rtol=1e-9))
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-9, record_sweeps=0))
    gi, hi = D.info(), h.info()
    assert gi["n"] == hi["n"] and gi["nnz"] == hi["nnz"]
    for l in range(gi["num_levels"]):
        rg, cg, vg, _ = D.level(l)
        rh, ch, vh = h.level(l)
        assert np.array_equal(rg, rh) and np.array_equal(cg, ch) and np.array_equal(vg, vh)
    xd, idd = D.solve(b)
    xh, ih = h.solve(b)
    assert idd["niter"] == ih["niter"]
    assert np.linalg.norm(xd - xh) / np.linalg.norm(xh) < 1e-10
    D.free()
    h.free()


def test_dist_nccl_transport_on_one_rank(bx, cuda):
    """The NCCL form (ncclAllGather / ncclAllReduce / grouped send-receive on the hierarchy's
    stream) on a one-rank communicator gives the local form's hierarchy and iterates exactly."""
    import torch
    A = matrix(bx, ("lap7", (16, 14, 12)))
    n = A.shape[0]
    b = A @ np.random.default_rng(6).uniform(-1, 1, n)
    uid = bx.nccl_unique_id()
    comm = bx.nccl_comm(1, 0, uid)
    try:
        Dn = bx.Dist.nccl(A.indptr, A.indices, A.data, 0, n, comm, 1, fcg(bx, rtol=1e-8))
        Dl = bx.Dist.local(A.indptr, A.indices, A.data, [0, n], fcg(bx, rtol=1e-8))
        assert Dn.info()["n"] == Dl.info()["n"] and Dn.info()["nnz"] == Dl.info()["nnz"]
        xn, inn = Dn.solve(b)
        xl, il = Dl.solve(b)
        assert inn["status"] == 0 and inn["niter"] == il["niter"]
        assert np.array_equal(xn, xl)
        bd = torch.from_numpy(b).to(cuda)
        xd, ind = Dn.solve(bd)
        assert np.array_equal(xd.cpu().numpy(), xl)
        Dn.free()
        Dl.free()
    finally:
        bx.nccl_comm_destroy(comm)


def test_dist_rejects_bad_partitions(bx, cuda):
    A = matrix(bx, ("lap7", (6, 6, 6)))
    n = A.shape[0]
    for offs in ([0, n + 1], [1, n], [0, 50, 50, n]):
        with pytest.raises(bx.BcmgxError) as e:
            bx.Dist.local(A.indptr, A.indices, A.data, offs, fcg(bx))
        assert e.value.code == -1
    with pytest.raises(bx.BcmgxError) as e:
        bx.Dist.local(A.indptr, A.indices, A.data, [0, n], fcg(bx, vcycle_precision="FP32"))
    assert e.value.code == -2
