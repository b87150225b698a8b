"""Batched solves: independent uneven systems set up concurrently and solved in one CUDA graph
launch. In the per-system form (one graph branch per system) every system gives exactly the
results of its own solve; in the lockstep form (every step one kernel over all systems of a
level-count group, each system with its own FCG scalars and stopping test) the V-cycle is every
system's own and the per-system sums differ in order only, so iterations agree within one and
solutions to rounding."""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _systems(bx, m, seed, lo=4, hi=14):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(m):
        dims = rng.integers(lo, hi + 1, size=3)
        row, col, val = bx.laplacian_3d(7, *[int(d) for d in dims])
        A = sp.csr_matrix((val, col, row), shape=(row.size - 1,) * 2) + rng.uniform(0, 0.5) * sp.identity(row.size - 1)
        A = A.tocsr()
        A.sort_indices()
        out.append((A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data))
    return out


@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_batch_matches_single_solves(bx, cuda, prec):
    import torch
    systems = _systems(bx, 12, 4)
    p = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=1e-8, dispnorm=0, vcycle_precision=prec)
    B = bx.Batch(systems, p, nthreads=4, lockstep=False)
    rng = np.random.default_rng(5)
    bs = [torch.from_numpy(rng.uniform(-1, 1, r.size - 1)).to(cuda) for r, _, _ in systems]
    xs, infos = B.solve(bs)
    xs2, infos2 = B.solve([2 * b for b in bs])   # relaunch of the same graph
    for k, (row, col, val) in enumerate(systems):
        h = bx.prec_setup(row, col, val, p)
        x, info = h.solve(bs[k])
        assert info["niter"] == infos[k]["niter"]
        assert torch.equal(x, xs[k])
        assert infos2[k]["niter"] == infos[k]["niter"]
        assert torch.allclose(xs2[k], 2 * xs[k], rtol=1e-6, atol=1e-12)
        A = sp.csr_matrix((val, col, row), shape=(row.size - 1,) * 2)
        r = bs[k].cpu().numpy() - A @ xs[k].cpu().numpy()
        assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(bs[k].cpu().numpy()) * 1.0001
    # the batch's own hierarchies also solve one by one
    x1, i1 = B.hierarchy(3).solve(bs[3])
    assert i1["niter"] == infos[3]["niter"] and torch.equal(x1, xs[3])
    B.free()


@pytest.mark.parametrize("pre", ["L1_JACOBI", "AFSAI", "NONE"])
def test_batch_other_preconditioners(bx, cuda, pre):
    """The standalone l1-Jacobi and AFSAI preconditioners (and none) in a batch: every system gives
    bit for bit the iterations and solution of its own single solve."""
    import torch
    systems = _systems(bx, 5, 8)
    p = bx.params_default(solver="FCG", preconditioner=pre, rtol=1e-8, dispnorm=0, l1jacsweeps=2)
    B = bx.Batch(systems, p, nthreads=2)   # lockstep needs BCMG: the per-system form runs
    rng = np.random.default_rng(9)
    bs = [torch.from_numpy(rng.uniform(-1, 1, r.size - 1)).to(cuda) for r, _, _ in systems]
    xs, infos = B.solve(bs)
    for k, (row, col, val) in enumerate(systems):
        x, info = bx.prec_setup(row, col, val, p).solve(bs[k])
        assert infos[k]["status"] == 0
        assert info["niter"] == infos[k]["niter"]
        assert torch.equal(x, xs[k])
    B.free()


def test_batch_setup_error_is_reported(bx, cuda):
    systems = _systems(bx, 3, 6)
    r, c, v = systems[1]
    c = c.copy()
    c[r[2]], c[r[2] + 1] = c[r[2] + 1], c[r[2]]   # unsorted row in system 1
    systems[1] = (r, c, v)
    p = bx.params_default(solver="FCG", preconditioner="BCMG", dispnorm=0)
    with pytest.raises(bx.BcmgxError) as e:
        bx.Batch(systems, p, nthreads=2)
    assert e.value.code == -1


@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_lockstep_matches_single_solves(bx, cuda, prec):
    """Uneven systems (2 and 3 levels: two groups) in lockstep: every system reaches the tolerance,
    within one iteration of its own solve, its solution within rounding of that solve's."""
    import torch
    systems = _systems(bx, 14, 11, lo=6, hi=40)
    p = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=1e-8, dispnorm=0, vcycle_precision=prec)
    B = bx.Batch(systems, p, nthreads=4)   # the default form
    rng = np.random.default_rng(12)
    bs = [torch.from_numpy(rng.uniform(-1, 1, r.size - 1)).to(cuda) for r, _, _ in systems]
    xs, infos = B.solve(bs)
    levels = set()
    for k, (row, col, val) in enumerate(systems):
        h = bx.prec_setup(row, col, val, p)
        levels.add(h.info()["num_levels"])
        x, info = h.solve(bs[k])
        h.free()
        assert infos[k]["status"] == 0
        assert abs(info["niter"] - infos[k]["niter"]) <= 1
        xk = xs[k].cpu().numpy()
        assert np.linalg.norm(xk - x.cpu().numpy()) <= 1e-6 * np.linalg.norm(x.cpu().numpy())
        A = sp.csr_matrix((val, col, row), shape=(row.size - 1,) * 2)
        r = bs[k].cpu().numpy() - A @ xk
        assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(bs[k].cpu().numpy()) * 1.0001
    assert len(levels) >= 2
    # a second launch of the same graph (right-hand sides doubled), and the per-system form
    xs2, infos2 = B.solve([2 * b for b in bs])
    for k in range(len(systems)):
        assert infos2[k]["niter"] == infos[k]["niter"]
        assert torch.allclose(xs2[k], 2 * xs[k], rtol=1e-6, atol=1e-12)
    B.set_lockstep(False)
    xs3, infos3 = B.solve(bs)
    for k in range(len(systems)):
        assert abs(infos3[k]["niter"] - infos[k]["niter"]) <= 1
    B.free()


def test_lockstep_cycle_is_each_systems_own(bx, cuda, monkeypatch):
    """With the same row kernel forced on every level of the members and of the union, the
    lockstep solve of systems that stop together takes the single solves' iterations, and its
    solutions agree with theirs to rounding of the per-system sums only."""
    import torch
    monkeypatch.setenv("BCMGX_TPR", "2")
    systems = _systems(bx, 6, 13, lo=16, hi=18)
    p = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=1e-8, dispnorm=0, vcycle_precision="FP64")
    B = bx.Batch(systems, p, nthreads=2)
    singles = [bx.prec_setup(r, c, v, p) for r, c, v in systems]
    rng = np.random.default_rng(14)
    bs = [torch.from_numpy(rng.uniform(-1, 1, r.size - 1)).to(cuda) for r, _, _ in systems]
    xs, infos = B.solve(bs)   # the first solve sets up the union's levels (the forced kernel too)
    monkeypatch.delenv("BCMGX_TPR")
    for k, h in enumerate(singles):
        x, info = h.solve(bs[k])
        assert info["niter"] == infos[k]["niter"]
        assert torch.allclose(xs[k], x, rtol=1e-9, atol=1e-12)
        h.free()
    B.free()


def test_lockstep_reports_breakdown_and_itnlim(bx, cuda):
    """A right-hand side with a NaN breaks its own system down (BCMGX_ERR_NOT_SPD for the batch)
    while the others converge; itnlim reached is reported as no convergence."""
    import torch
    systems = _systems(bx, 4, 15, lo=8, hi=20)
    p = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=1e-8, dispnorm=0)
    B = bx.Batch(systems, p, nthreads=2)
    rng = np.random.default_rng(16)
    bs = [torch.from_numpy(rng.uniform(-1, 1, r.size - 1)).to(cuda) for r, _, _ in systems]
    bs[2][3] = float("nan")
    with pytest.raises(bx.BcmgxError) as e:
        B.solve(bs)
    assert e.value.code == -7
    bs[2][3] = 0.5
    xs, infos = B.solve(bs)
    assert all(i["status"] == 0 for i in infos)
    B.free()
    p2 = bx.params_default(solver="FCG", preconditioner="BCMG", rtol=1e-14, dispnorm=0, itnlim=3)
    B = bx.Batch(systems, p2, nthreads=2)
    xs, infos = B.solve(bs)
    assert all(i["retv"] == -1 and i["niter"] == 4 for i in infos)
    B.free()
