"""GPU parity against the CPU oracle on the benchmark configurations themselves.

* 7-point Poisson 50^3 (125,000 rows; x* ~ U[-1,1] from numpy default_rng(0)) and the 7-point
  finite-volume diffusion 96^3 (884,736 rows; kappa = exp(theta), theta a Gaussian random field
  of length 8 and sigma 2 from seed 5): every sweep's matching, aggregates, prolongator and weight
  vector, every level matrix, every composite prolongator and divisor equal the oracle's bit for
  bit; the FCG solve to 1e-8 takes the oracle's iterations (+-1) and its solution agrees with the
  oracle's within 1e-6.
* 27-point Poisson 160^3 (4,096,000 rows, 109,215,352 non-zeros; x* from default_rng(1)): the
  same bit-for-bit checks on every sweep and every level (the oracle's set-up takes several
  seconds on the host cores), the FP64-cycle solve within one iteration of the oracle's and
  within 1e-6 of its solution, and the FP32-cycle solve within 10 % of the oracle's iterations.
* The driverSolve CLI reproduces all eight reference solution files of the 10^3 grids
  (BCMGX/src/test/data/cmp/lap3d_{7p,27p}_10x10x10_{1x1x1,2x1x1,2x2x1,2x2x2}_sol.txt, the
  multi-rank grids in rank-block-major order) within compareSolutions' 1e-5.
"""
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import ROOT

pytestmark = pytest.mark.gpu


def fcg(bx, **kw):
    kw.setdefault("solver", "FCG")
    kw.setdefault("preconditioner", "BCMG")
    kw.setdefault("dispnorm", 0)
    return bx.params_default(**kw)


def poisson(bx, stencil, g, seed):
    row, col, val = bx.laplacian_3d(stencil, *g)
    n = row.size - 1
    xs = np.random.default_rng(seed).uniform(-1.0, 1.0, n)
    A = sp.csr_matrix((val, col, row), shape=(n, n))
    return A, xs, A @ xs


def diffusion96(bx):
    from bootcmatchgx_b200 import problems
    g = (96, 96, 96)
    theta = problems.gaussian_random_field(g, 8.0, 2.0, 5).reshape(-1, order="F")
    row, col, val = bx.diffusion_7p(*g, np.exp(theta))
    n = row.size - 1
    A = sp.csr_matrix((val, col, row), shape=(n, n))
    xs = np.random.default_rng(5).uniform(-1.0, 1.0, n)
    return A, xs, A @ xs


def check_hierarchy(bx, oracle, A, Ao, prm_kw=None):
    """Set-up on the GPU with sweep records vs the oracle's set-up with records: bit for bit."""
    prm_kw = prm_kw or {}
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, record_sweeps=1, **prm_kw))
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
        assert np.array_equal(rg, ro) and np.array_equal(cg, co) and np.array_equal(vg, vo), l
        if l + 1 < gi["num_levels"]:
            ag, pg, Mg = h.prolongator(l)
            ao, po, Mo = Ho.prolongator(l)
            assert np.array_equal(ag, ao) and np.array_equal(pg, po) and np.array_equal(Mg, Mo), l
    st = Ho.stats()
    assert gi["maxcoarsesize"] == st["maxcoarsesize"] and gi["ftcoarse"] == st["ftcoarse"]
    assert abs(gi["op_cmplx"] - st["op_cmplx"]) < 1e-12
    h.free()
    return Ho


def check_solve(bx, A, xs, b, xo, io, prec="FP64"):
    h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-8, vcycle_precision=prec))
    x, info = h.solve(b)
    h.free()
    assert info["status"] == 0
    if prec == "FP64":
        assert abs(info["niter"] - io["niter"]) <= 1, (info["niter"], io["niter"])
    else:
        assert info["niter"] <= 1.1 * io["niter"] + 1, (info["niter"], io["niter"])
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b) * 1.0001
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-6
    return x, info


@pytest.mark.parametrize("which", ["poisson7_50", "diffusion7_96"])
def test_config_hierarchy_and_solve(bx, oracle, cuda, which):
    A, xs, b = poisson(bx, 7, (50, 50, 50), 0) if which == "poisson7_50" else diffusion96(bx)
    Ao = oracle.Matrix.from_csr(A.indptr, A.indices, A.data)
    check_hierarchy(bx, oracle, A, Ao)
    Ho = oracle.Hierarchy(Ao, oracle.params(rtol=1e-8))
    xo, io = Ho.solve(b)
    assert io["retv"] == 0
    for prec in ("FP64", "FP32"):
        check_solve(bx, A, xs, b, xo, io, prec)


def test_config_poisson27_160(bx, oracle, cuda):
    """The headline workload: hierarchy bit for bit against the oracle, then both solves."""
    A, xs, b = poisson(bx, 27, (160, 160, 160), 1)
    assert A.nnz == 109215352
    oracle.num_threads(os.cpu_count() or 1)
    Ao = oracle.Matrix.from_csr(A.indptr, A.indices, A.data)
    check_hierarchy(bx, oracle, A, Ao)
    Ho = oracle.Hierarchy(Ao, oracle.params(rtol=1e-8))
    xo, io = Ho.solve(b)
    assert io["retv"] == 0
    del Ho
    x64, i64 = check_solve(bx, A, xs, b, xo, io, "FP64")
    x32, i32 = check_solve(bx, A, xs, b, xo, io, "FP32")
    # both forms stop at the same residual tolerance: their errors against x* are the same size
    e64 = np.linalg.norm(x64 - xs) / np.linalg.norm(xs)
    e32 = np.linalg.norm(x32 - xs) / np.linalg.norm(xs)
    assert e32 < 1.5 * e64 + 1e-12


@pytest.mark.parametrize("st", [7, 27])
@pytest.mark.parametrize("PQR", [(1, 1, 1), (2, 1, 1), (2, 2, 1), (2, 2, 2)])
def test_cli_reproduces_every_golden(golden, cuda, tmp_path, st, PQR):
    """driverSolve -g {7p,27p} -l <cfg> -s FCG_BCMG.properties: A x = 1 on the (10P x 10Q x 10R)
    grid in the reference's rank-block-major row order, solution file vs the golden."""
    cfg = tmp_path / "lap.cfg"
    cfg.write_text(f"nx = 10\nny = 10\nnz = 10\nP = {PQR[0]}\nQ = {PQR[1]}\nR = {PQR[2]}\n")
    props = tmp_path / "FCG_BCMG.properties"
    props.write_text(str(golden["prop__FCG_BCMG.properties"]))
    sol = tmp_path / "sol.txt"
    cli = os.path.join(ROOT, "bootcmatchgx_b200", "bin", "bcmgx_driverSolve")
    r = subprocess.run([cli, "-g", f"{st}p", "-l", str(cfg), "-s", str(props), "-o", str(sol)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    x = np.loadtxt(sol)
    g = golden[f"sol__lap3d_{st}p_10x10x10_{PQR[0]}x{PQR[1]}x{PQR[2]}_sol"]
    assert x.size == g.size
    assert np.linalg.norm(x - g) / np.linalg.norm(g) < 1e-5


def test_config_diffusion7_256_hierarchy(bx, oracle, cuda):
    """The heterogeneous-diffusion workload (7-point finite volume 256^3, 16,777,216 rows,
    kappa = exp(theta), theta a Gaussian random field of length 8 and sigma 2 from seed 2): every
    sweep and every level bit for bit against the oracle's set-up, and the GPU's FP64 and FP32
    solves to 1e-8 reach the tolerance (b ~ U[0,1] from seed 3)."""
    from bootcmatchgx_b200 import problems
    g = (256, 256, 256)
    theta = problems.gaussian_random_field(g, 8.0, 2.0, 2).reshape(-1, order="F")
    row, col, val = bx.diffusion_7p(*g, np.exp(theta))
    n = row.size - 1
    A = sp.csr_matrix((val, col, row), shape=(n, n))
    assert A.nnz == 117047296
    oracle.num_threads(os.cpu_count() or 1)
    Ao = oracle.Matrix.from_csr(A.indptr, A.indices, A.data)
    Ho = check_hierarchy(bx, oracle, A, Ao)
    del Ho
    b = np.random.default_rng(3).uniform(0.0, 1.0, n)
    for prec in ("FP64", "FP32"):
        h = bx.prec_setup(A.indptr, A.indices, A.data, fcg(bx, rtol=1e-8, vcycle_precision=prec))
        x, info = h.solve(b)
        h.free()
        assert info["status"] == 0
        assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b) * 1.0001
