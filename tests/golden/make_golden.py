"""Regenerate tests/golden/reference_fixtures.npz from the reference's own test data.

Run where the BootCMatchGX sources are available, with their root as the argument; the GPU box
never runs this. It packs, without modification:
  * BCMGX/src/test/data/cmp/lap3d_{7p,27p}_10x10x10_{1x1x1,2x1x1,2x2x1,2x2x2}_sol.txt
    (FCG+BCMG solutions of A x = 1, rtol 1e-6, checked by compareSolutions at 1e-5,
    BCMGX/launchAndCompare.mk:320-330), in the reference's rank-block-major row order;
  * BCMGX/src/test/data/mtx/lap3d_*.mtx (Matlab-generated Laplacians used by
    BCMGX/testGenerators.mk) as COO triplets;
  * BCMGX/src/test/data/settings/{FCG_BCMG,FCG_BCMG.prova,sample}.properties as text;
  * BCMGX/src/test/data/mtx/bcsstk09.mtx as text (the --matrix input of driverSolve, read by the
    library's own MatrixMarket reader in the tests) and cmp/bcsstk09_sol.txt (its FCG+BCMG solution
    of A x = 1, BCMGX/launchAndCompare.mk:136,207). The bcsstk13 / bcsstk24 solution files are all
    zeros (their _aux.txt: FLAG = 1, ITER = 0) and pin nothing, so they are not packed.

Usage: python tests/golden/make_golden.py REFERENCE_ROOT
"""
import os
import sys

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_fixtures.npz")
DATA = None


def read_mtx(path):
    with open(path) as f:
        lines = [l for l in f if not l.startswith("%")]
    n, m, nnz = (int(t) for t in lines[0].split())
    trip = np.array([[float(t) for t in l.split()] for l in lines[1:1 + nnz]])
    return n, m, trip[:, 0].astype(np.int32) - 1, trip[:, 1].astype(np.int32) - 1, trip[:, 2]


def main():
    global DATA
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT (the BootCMatchGX source tree)")
    DATA = os.path.join(sys.argv[1], "BCMGX", "src", "test", "data")
    out = {}
    for st in ("7p", "27p"):
        for grid in ("1x1x1", "2x1x1", "2x2x1", "2x2x2"):
            name = f"lap3d_{st}_10x10x10_{grid}_sol"
            out["sol__" + name] = np.loadtxt(os.path.join(DATA, "cmp", name + ".txt"))
    for f in sorted(os.listdir(os.path.join(DATA, "mtx"))):
        if f.startswith("lap3d_") and f.endswith(".mtx"):
            n, m, r, c, v = read_mtx(os.path.join(DATA, "mtx", f))
            key = "mtx__" + f[:-4]
            out[key + "__shape"] = np.array([n, m], np.int64)
            out[key + "__row"] = r
            out[key + "__col"] = c
            out[key + "__val"] = v
    for f in ("FCG_BCMG.properties", "FCG_BCMG.prova.properties", "sample.properties"):
        with open(os.path.join(DATA, "settings", f)) as fh:
            out["prop__" + f] = np.array(fh.read())
    with open(os.path.join(DATA, "mtx", "bcsstk09.mtx")) as fh:
        out["mtxtext__bcsstk09"] = np.array(fh.read())
    out["sol__bcsstk09_sol"] = np.loadtxt(os.path.join(DATA, "cmp", "bcsstk09_sol.txt"))
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, len(out), "arrays")


if __name__ == "__main__":
    main()
