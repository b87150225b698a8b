"""Batched solves: independent uneven systems set up concurrently and solved in one CUDA graph
launch must give exactly the results of solving each system on its own."""
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
    B = bx.Batch(systems, p, nthreads=4)
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
    B = bx.Batch(systems, p, nthreads=2)
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
