"""Host-side parts of libbcmgx.so that need no GPU: the exported C ABI, the settings readers,
the generators and readers of the driver's input plumbing, and the CLI's argument checks."""
import os
import re
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import ROOT, golden_mtx

HEADER = os.path.join(ROOT, "include", "bcmgx.h")
CLI = os.path.join(ROOT, "bootcmatchgx_b200", "bin", "bcmgx_driverSolve")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?(?:int64_t|int|void|const char\*)\s*\*?\s*(bcmgx_\w+)\s*\(", text, re.M)))


def test_abi_exports_every_declared_symbol(bx):
    import ctypes
    from bootcmatchgx_b200 import _lib
    names = declared_functions()
    assert len(names) >= 20
    L = ctypes.CDLL(_lib.LIB_PATH)
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)
    assert bx.lib().bcmgx_version().startswith(b"bcmgx")


def test_params_defaults(bx):
    p = bx.params_to_dict(bx.params_default())
    assert p["solver"] == 0 and p["itnlim"] == 2000 and p["rtol"] == 1e-6 and p["dispnorm"] == 1
    assert p["preconditioner"] == 0 and p["aggrsweeps"] == 2 and p["max_levels"] == 39
    assert p["relaxnumber_coarse"] == 20 and p["prerelax_sweeps"] == 4 and p["postrelax_sweeps"] == 4
    assert p["conv_ratio"] == 0.8 and p["max_hrc"] == 1 and p["l1jacsweeps"] == 4


def _write(tmp_path, name, text):
    f = tmp_path / name
    f.write_text(text)
    return str(f)


def test_properties_fixtures(bx, golden, tmp_path):
    f = _write(tmp_path, "FCG_BCMG.properties", str(golden["prop__FCG_BCMG.properties"]))
    p = bx.params_to_dict(bx.init_from_properties_file(f))
    assert p["solver"] == 1 and p["preconditioner"] == 2 and p["rtol"] == 1e-6
    f = _write(tmp_path, "prova.properties", str(golden["prop__FCG_BCMG.prova.properties"]))
    p = bx.params_to_dict(bx.init_from_properties_file(f))
    assert p["itnlim"] == 1000 and p["prerelax_sweeps"] == 4
    f = _write(tmp_path, "sample.properties", str(golden["prop__sample.properties"]))
    p = bx.params_to_dict(bx.init_from_properties_file(f))
    assert p["solver"] == 0 and p["preconditioner"] == 3 and p["rtol"] == 1e-6
    assert p["relaxnumber_coarse"] == 20 and p["cycle_type"] == 0 and p["aggrsweeps"] == 2


def test_properties_rules(bx, tmp_path):
    # '#' starts a comment; unknown keys are ignored; the last '=' splits; spaces trimmed
    f = _write(tmp_path, "a.properties",
               "# comment = ignored\n\n   \nsolver=FCG\n rtol = 1e-8 # trailing comment\nfoo = bar\n"
               "preconditioner = BCMG\ncycle_type = W_CYCLE\nitnlim = 7\n")
    p = bx.params_to_dict(bx.init_from_properties_file(f))
    assert p["solver"] == 1 and p["rtol"] == 1e-8 and p["preconditioner"] == 2
    assert p["cycle_type"] == 2 and p["itnlim"] == 7
    # an enum value followed by a comment is not recognised (Params.cu:311 keeps it in the value)
    f = _write(tmp_path, "b.properties", "solver = FCG # comment\n")
    assert bx.params_to_dict(bx.init_from_properties_file(f))["solver"] == 5
    # a non-blank line without '=' is an error
    f = _write(tmp_path, "c.properties", "solver FCG\n")
    with pytest.raises(bx.BcmgxError) as e:
        bx.init_from_properties_file(f)
    assert e.value.code == -1 and "could not find '='" in str(e.value)
    with pytest.raises(bx.BcmgxError):
        bx.init_from_properties_file(str(tmp_path / "missing.properties"))
    f = _write(tmp_path, "d.properties", "itnlim = many\n")
    with pytest.raises(bx.BcmgxError):
        bx.init_from_properties_file(f)


def test_legacy_settings(bx, tmp_path):
    lines = ["NONE", "NONE", "FCG", "MULTIPLICATIVE", "1", "0.8", "SUITOR", "2", "0", "39", "V_CYCLE",
             "L1_JACOBI", "L1_JACOBI", "20", "0", "4", "4", "2000", "1.e-8", "1", "1", "1", "BCMG", "4", "0",
             "0", "0"]
    f = _write(tmp_path, "s.txt", "\n".join(l + " % note" for l in lines) + "\n")
    p = bx.params_to_dict(bx.init_from_file(f))
    assert p["solver"] == 1 and p["preconditioner"] == 2 and p["rtol"] == 1e-8 and p["error"] == 0
    lines[4] = "3"   # max_hrc != 1 -> error flag (Params.cu:463-466)
    f = _write(tmp_path, "s2.txt", "\n".join(lines) + "\n")
    assert bx.params_to_dict(bx.init_from_file(f))["error"] == 1
    f = _write(tmp_path, "s3.txt", "\n".join(lines[:5]) + "\n")
    with pytest.raises(bx.BcmgxError):
        bx.init_from_file(f)


@pytest.mark.parametrize("st,dims", [(7, (10, 10, 10, 1, 1, 1)), (27, (10, 10, 10, 2, 2, 2)),
                                     (7, (2, 2, 5, 3, 4, 2)), (27, (5, 5, 5, 4, 2, 1)),
                                     (7, (1, 1, 1, 1, 1, 1)), (27, (1, 7, 2, 1, 1, 3))])
def test_generator_matches_oracle(bx, oracle, st, dims):
    n, z = bx.laplacian_3d_size(st, *dims)
    row, col, val = bx.laplacian_3d(st, *dims)
    r2, c2, v2 = oracle.Matrix.lap3d(st, *dims).csr()
    assert n == row.size - 1 and z == col.size
    assert np.array_equal(row, r2) and np.array_equal(col, c2) and np.array_equal(val, v2)


def test_generator_fixture_and_size_160(bx, golden):
    M = golden_mtx(golden, "lap3d_27p_5x5x5_1x2x2")
    row, col, val = bx.laplacian_3d(27, 5, 5, 5, 1, 2, 2)
    assert abs(sp.csr_matrix((val, col, row), shape=M.shape) - M).max() == 0
    assert bx.laplacian_3d_size(27, 160, 160, 160) == (4096000, 109215352)
    assert bx.laplacian_3d_size(7, 50, 50, 50) == (125000, 860000)
    assert bx.laplacian_3d_size(7, 256, 256, 256) == (16777216, 117047296)


def test_laplacian_cfg(bx, tmp_path):
    f = _write(tmp_path, "g.cfg", "# grid\nnx = 10\nny = 12\nnz = 14\nP = 2\nQ = 1\nR = 3\n")
    assert bx.read_laplacian_cfg(f) == {"nx": 10, "ny": 12, "nz": 14, "P": 2, "Q": 1, "R": 3}
    with pytest.raises(bx.BcmgxError):
        bx.read_laplacian_cfg(_write(tmp_path, "h.cfg", "nx 10\n"))


def test_matrix_market_reader(bx, golden, tmp_path):
    M = golden_mtx(golden, "lap3d_7p_4x14x4_2x2x1").tocoo()
    f = tmp_path / "m.mtx"
    with open(f, "w") as fh:
        fh.write("%%MatrixMarket matrix coordinate real general\n% c\n")
        fh.write(f"{M.shape[0]} {M.shape[1]} {M.nnz}\n")
        order = np.random.default_rng(0).permutation(M.nnz)
        for k in order:
            fh.write(f"{M.row[k] + 1} {M.col[k] + 1} {M.data[k]:.17g}\n")
    row, col, val = bx.read_matrix_market(f)
    A = sp.csr_matrix((val, col, row), shape=M.shape)
    assert abs(A - M.tocsr()).max() == 0 and np.all(np.diff(row) >= 0)
    # symmetric storage is mirrored
    U = sp.triu(M.tocsr()).tocoo()
    g = tmp_path / "s.mtx"
    with open(g, "w") as fh:
        fh.write("%%MatrixMarket matrix coordinate real symmetric\n")
        fh.write(f"{U.shape[0]} {U.shape[1]} {U.nnz}\n")
        for r, c, v in zip(U.col, U.row, U.data):   # lower triangle, as symmetric files store it
            fh.write(f"{r + 1} {c + 1} {v:.17g}\n")
    row, col, val = bx.read_matrix_market(g)
    assert abs(sp.csr_matrix((val, col, row), shape=M.shape) - M.tocsr()).max() == 0
    h = tmp_path / "p.mtx"
    h.write_text("%%MatrixMarket matrix coordinate pattern general\n2 2 1\n1 1\n")
    with pytest.raises(bx.BcmgxError):
        bx.read_matrix_market(h)


def test_diffusion_spd(bx):
    rng = np.random.default_rng(2)
    kappa = np.exp(rng.normal(size=6 * 5 * 4))
    row, col, val = bx.diffusion_7p(6, 5, 4, kappa)
    A = sp.csr_matrix((val, col, row), shape=(120, 120))
    assert abs(A - A.T).max() < 1e-14
    assert np.linalg.eigvalsh(A.toarray()).min() > 0
    assert np.all(np.diff(col[row[0]:row[1]]) > 0)
    with pytest.raises(bx.BcmgxError):
        bx.diffusion_7p(2, 2, 2, -np.ones(8))


def test_cli_usage_and_errors(tmp_path):
    r = subprocess.run([CLI], capture_output=True, text=True)
    assert r.returncode != 0 and "Usage" in r.stdout
    r = subprocess.run([CLI, "-a", "4", "-s", str(tmp_path / "nope.properties")], capture_output=True, text=True)
    assert r.returncode != 0 and "Error opening setting file" in r.stderr
    r = subprocess.run([CLI, "-l", "x.cfg", "-g", "9p", "-s", "a.properties"], capture_output=True, text=True)
    assert r.returncode != 0 and "Usage" in r.stdout


def test_diffusion_assembler_matches_generator(bx):
    import torch
    from bootcmatchgx_b200 import problems
    theta = problems.gaussian_random_field((7, 6, 5), length=2.0, sigma=1.5, seed=3)
    kappa = np.exp(theta)
    row, col, val = bx.diffusion_7p(7, 6, 5, kappa)
    asm = problems.DiffusionAssembler(7, 6, 5, torch.device("cpu"))
    v = asm.values(torch.from_numpy(kappa.reshape(-1))).numpy()
    assert np.array_equal(asm.row.numpy(), row) and np.array_equal(asm.col.numpy(), col)
    assert np.max(np.abs(v - val)) <= 1e-14 * np.max(np.abs(val))


def test_gaussian_random_field_statistics():
    from bootcmatchgx_b200 import problems
    f = problems.gaussian_random_field((48, 48, 48), length=4.0, sigma=2.0, seed=2)
    assert abs(f.std() - 2.0) < 0.3 and abs(f.mean()) < 0.5
    # correlation at lag 4 along x ~ exp(-16/32) for the squared-exponential kernel
    c = np.mean(f * np.roll(f, 4, axis=0)) / np.mean(f * f)
    assert abs(c - np.exp(-0.5)) < 0.1


def _replica_rank(rank, world, port, out):
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        # every rank times its own replica; the job reports the slowest one
        mine = 10.0 + 5.0 * rank
        got = bench.max_over_ranks(mine, world)
        dist.barrier()
        # the reference arm runs on rank 0 only; the other ranks return without work
        import argparse
        line = bench.reference_arm(argparse.Namespace(gpus=world, steps=1, warmup=0, workload="poisson7_50"),
                                   bench.WORKLOADS["poisson7_50"], rank, world) if rank != 0 else "rank0"
        out.put((rank, got, line))
    finally:
        dist.destroy_process_group()


def test_replica_timing_over_gloo_ranks():
    """bench.py at N > 1 (replicas): two gloo ranks on CPU agree on the slowest rank's time, and
    the reference arm does no work on ranks other than 0."""
    import multiprocessing as mp
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_replica_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == (0, 15.0, "rank0") and res[1] == (1, 15.0, None)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5


def _shard_rank(rank, world, port, out):
    """One gloo rank of test_replica_sharding_over_gloo_ranks: solves its share of independent
    systems and of right-hand-side columns with a stand-in solver (a dense solve on the CPU)."""
    import datetime
    import torch.distributed as dist
    from bootcmatchgx_b200 import replicas
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(11)
        mats = []
        for k in range(9):   # uneven systems, the same on every rank
            m = 3 + k
            B = rng.uniform(-1, 1, (m, m))
            mats.append((B @ B.T + m * np.eye(m), rng.uniform(-1, 1, m)))
        mine = replicas.systems_of_rank(len(mats), rank, world)
        xs = [np.linalg.solve(*mats[k]) for k in mine]
        allx = replicas.gather_in_order(xs, mine, len(mats), world)
        A, _ = mats[-1]
        Bk = rng.uniform(-1, 1, (A.shape[0], 32))
        cols = replicas.columns_of_rank(32, rank, world)
        Xk = np.linalg.solve(A, Bk[:, cols.start:cols.stop])
        allc = replicas.gather_in_order([Xk[:, j] for j in range(Xk.shape[1])], list(cols), 32, world)
        out.put((rank, mine, list(cols), [x.tolist() for x in allx], np.stack(allc, axis=1).tolist()))
    finally:
        dist.destroy_process_group()


def test_replica_sharding_over_gloo_ranks():
    """The batched forms at N > 1: systems go round robin and right-hand-side columns in
    contiguous slices; every system and column is solved on exactly one rank, and the gathered
    results equal the single-rank results in the single-rank order (two gloo ranks on CPU)."""
    import multiprocessing as mp
    import socket
    from bootcmatchgx_b200 import replicas
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_shard_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(res[0][1] + res[1][1]) == list(range(9)) and not set(res[0][1]) & set(res[1][1])
    assert res[0][2] + res[1][2] == list(range(32))
    rng = np.random.default_rng(11)
    mats = []
    for k in range(9):
        m = 3 + k
        B = rng.uniform(-1, 1, (m, m))
        mats.append((B @ B.T + m * np.eye(m), rng.uniform(-1, 1, m)))
    single = [np.linalg.solve(*mk) for mk in mats]
    Bk = rng.uniform(-1, 1, (mats[-1][0].shape[0], 32))
    Xs = np.linalg.solve(mats[-1][0], Bk)
    for r in res:
        assert all(np.allclose(a, b, rtol=0, atol=1e-12) for a, b in zip(r[3], single))
        assert np.allclose(np.array(r[4]), Xs, rtol=0, atol=1e-12)
    # the split functions on their own: 33 columns over 4 ranks, 10 systems over 3 ranks
    assert [len(replicas.columns_of_rank(33, r, 4)) for r in range(4)] == [9, 8, 8, 8]
    assert replicas.systems_of_rank(10, 1, 3) == [1, 4, 7]


def test_reference_arm_builds_the_same_problems(bx):
    """bench.py's reference arm builds its matrices without the product library: the diffusion
    matrix assembled in numpy equals bcmgx_diffusion_7p bit for bit, and the oracle's Laplacian
    generator equals the library's."""
    import bench
    from oracle import pyoracle as O
    rng = np.random.default_rng(3)
    for g in [(5, 4, 3), (7, 7, 7), (1, 2, 9)]:
        kappa = np.exp(rng.normal(size=int(np.prod(g))))
        r1, c1, v1 = bx.diffusion_7p(*g, kappa)
        r2, c2, v2 = bench.diffusion_csr_numpy(*g, kappa)
        assert np.array_equal(r1, r2) and np.array_equal(c1, c2) and np.array_equal(v1, v2)
    for st in (7, 27):
        r1, c1, v1 = bx.laplacian_3d(st, 6, 5, 4)
        r2, c2, v2 = O.Matrix.lap3d(st, 6, 5, 4).csr()
        assert np.array_equal(r1, r2) and np.array_equal(c1, c2) and np.array_equal(v1, v2)
