"""Launch and pass variants that the library reads from the environment once per process, each run
in a child process and compared bit for bit with the default: the dependent launches turned off
(BCMGX_PDL=0) or given to every solve kernel (BCMGX_PDL=7: row, element-wise and FCG kernels), and the
transposed positions and the a_hat minimum in two passes (BCMGX_TPOS_FUSE=0), and the sliced levels without
their pattern-indexed rows (BCMGX_SLPAT=0). None of them changes a
value: they only change when kernels start or how the set-up's passes are grouped. The children use the
default threads per row (no autotuning), so that all of them sum each row in the same order."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import bootcmatchgx_b200 as bx
out = {}
for name, st, g, prec, graph in (("p27", 27, 40, "FP32", 1), ("p7", 7, 48, "FP64", 0), ("p27s", 27, 32, "FP64", 1)):
    row, col, val = bx.laplacian_3d(st, g, g, g)
    n = row.size - 1
    b = np.random.default_rng(3).uniform(-1, 1, n)
    # the kernel choices fixed (no timing-based autotuning, whose choice sets a row's summation order)
    p = bx.params_default(solver="FCG", preconditioner="BCMG", dispnorm=0, rtol=1e-8, vcycle_precision=prec,
                          use_graph=graph, autotune=0)
    h = bx.prec_setup(row, col, val, p)
    x, info = h.solve(b)
    inf = h.info()
    out[name] = {"x": x.tobytes().hex(), "niter": info["niter"], "status": info["status"],
                 "levels": inf["n"], "level_nnz": inf["nnz"]}
    h.free()
print(json.dumps(out))
"""


def child(env_extra):
    env = dict(os.environ)
    for k in ("BCMGX_PDL", "BCMGX_TPOS_FUSE", "BCMGX_SLPAT", "BCMGX_TPR"):
        env.pop(k, None)
    env.update(env_extra)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.fixture(scope="module")
def default_run(cuda):
    return child({})


@pytest.fixture(scope="module")
def sliced_run(cuda):
    return child({"BCMGX_TPR": "64"})


@pytest.mark.parametrize("env", [{"BCMGX_PDL": "0"}, {"BCMGX_PDL": "7"}, {"BCMGX_TPOS_FUSE": "0"}])
def test_launch_mode_bit_identical(default_run, env):
    other = child(env)
    for name, ref in default_run.items():
        got = other[name]
        assert ref["status"] == 0 and got["status"] == 0
        assert got["levels"] == ref["levels"] and got["level_nnz"] == ref["level_nnz"]
        assert got["niter"] == ref["niter"]
        assert got["x"] == ref["x"], f"{name}: solution differs with {env}"


def test_pattern_rows_bit_identical(sliced_run):
    """Every level on the sliced kernels (BCMGX_TPR=64): the pattern-indexed form of the stencil
    levels against the plain sliced form (BCMGX_SLPAT=0)."""
    other = child({"BCMGX_TPR": "64", "BCMGX_SLPAT": "0"})
    for name, ref in sliced_run.items():
        got = other[name]
        assert ref["status"] == 0 and got["status"] == 0
        assert got["levels"] == ref["levels"] and got["niter"] == ref["niter"]
        assert got["x"] == ref["x"], f"{name}: solution differs without the pattern form"
